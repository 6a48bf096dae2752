"""The C ABI library loads and exports every symbol include/edgpu.h declares; host-only
entry points (no GPU compute) behave like the reference's helpers. Runs without a GPU."""
import ctypes as C
import math
import os
import re
import subprocess

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "edgpu.h")


def header_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(edg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "edg_hxv_z" in syms and "edg_tridiag_d" in syms and "edg_ground_state" in syms
    assert len(syms) >= 30


def test_library_exports_every_header_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    # nothing but the C ABI leaks out of the library
    assert all(s.startswith("edg_") for s in exported if not s.startswith("_")), sorted(exported)[:20]


def test_binding_covers_header():
    assert sorted(L.SIGNATURES) == header_symbols()
    lib = L.lib()
    for s in header_symbols():
        assert getattr(lib, s) is not None


def test_host_helpers_match_reference():
    lib = L.lib()
    for n in range(0, 31):
        for k in range(0, n + 1):
            assert lib.edg_binomial(n, k) == math.comb(n, k)
    for ns in (6, 16):
        for nup in range(ns + 1):
            for ndw in range(ns + 1):
                isec = lib.edg_get_sector(ns, nup, ndw)
                assert isec == O.lib().orc_get_sector(ns, nup, ndw)
                assert lib.edg_get_nup(ns, isec) == nup and lib.edg_get_ndw(ns, isec) == ndw


def test_random_vector_formula():
    x = E.random_vector(2024, 1000)
    assert np.array_equal(x, O.random_vector(2024, 1000))
    assert x.min() >= -1.0 and x.max() < 1.0


def test_tridiag_eigh_and_poles_vs_oracle():
    rng = np.random.default_rng(1)
    a = rng.normal(size=60)
    b = np.concatenate([[0.0], rng.uniform(0.2, 1.5, 59)])
    w, z = E.tridiag_eigh(a, b)
    wo, Zo = O.tridiag_eigh(a, b)
    assert np.allclose(w, wo, atol=1e-12)
    assert np.allclose(z ** 2, Zo[0] ** 2, atol=1e-12)
    p, wt = E.poles_weights(a, b, 0.7, -3.0, -1)
    po, wto = O.poles_weights(a, b, 0.7, -3.0, -1)
    assert np.allclose(p, po, atol=1e-12) and np.allclose(wt, wto, atol=1e-12)
    assert abs(wt.sum() - 0.7) < 1e-12


def test_tridiag_eigh_degenerate_and_tiny():
    w, z = E.tridiag_eigh(np.array([2.0]), np.array([0.0]))
    assert w[0] == 2.0 and z[0] == 1.0
    w, z = E.tridiag_eigh(np.array([1.0, 1.0, 1.0]), np.array([0.0, 0.0, 0.0]))
    assert np.allclose(w, 1.0)


def test_model_errors_match_reference_stops():
    lib = L.lib()
    h = C.c_void_p()
    bad = np.array([[0.0, 1.0], [2.0, 0.0]])  # not Hermitian -> Hij_build stop
    st = lib.edg_model_create(2, 1, bad.ctypes.data_as(L._pd), None, None, None, 1.0, 0.0, 1, 0, C.byref(h))
    assert st == L.EDG_ERR_ARG and b"Hermitian" in lib.edg_last_error()
    ok = np.zeros((3, 3))
    assert lib.edg_model_create(0, 1, ok.ctypes.data_as(L._pd), None, None, None, 1.0, 0.0, 1, 0,
                                C.byref(h)) == L.EDG_ERR_ARG
    assert lib.edg_model_create(31, 1, ok.ctypes.data_as(L._pd), None, None, None, 1.0, 0.0, 1, 0,
                                C.byref(h)) == L.EDG_ERR_ARG
    nan = np.array([[0.0, np.nan], [np.nan, 0.0]])
    assert lib.edg_model_create(2, 1, nan.ctypes.data_as(L._pd), None, None, None, 1.0, 0.0, 1, 0,
                                C.byref(h)) == L.EDG_ERR_ARG
    with pytest.raises(L.EdgError):
        E.Model(bad)


def test_model_create_and_complex_flag():
    h = np.array([[0.0, -1.0 + 0.5j], [-1.0 - 0.5j, 0.0]])
    m = E.Model(h, uloc=2.0)
    assert m.ns == 2
    m.close()


def test_null_handles_are_errors_not_crashes():
    lib = L.lib()
    d = C.c_int64()
    assert lib.edg_sector_dims(None, C.byref(d), None, None) == L.EDG_ERR_ARG
    assert lib.edg_hxv_d(None, 1, None, None) == L.EDG_ERR_ARG
    assert lib.edg_sector_destroy(None) == L.EDG_OK
    assert lib.edg_model_destroy(None) == L.EDG_OK


def _lanczos_tridiag(h, m, seed):
    """a, b (b[0] = 0) of m steps of fully reorthogonalised Lanczos on the dense h."""
    rng = np.random.default_rng(seed)
    q = rng.standard_normal(h.shape[0])
    Q = [q / np.linalg.norm(q)]
    a, b = [], [0.0]
    for j in range(m):
        w = h @ Q[j]
        a.append(Q[j] @ w)
        for _ in range(2):
            w -= np.array(Q).T @ (np.array(Q) @ w)
        bj = np.linalg.norm(w)
        if j + 1 < m:
            b.append(bj)
            Q.append(w / bj)
    return np.array(a), np.array(b)


@pytest.mark.parametrize("n,k,seed", [(1, 4, 0), (2, 1, 1), (7, 3, 2), (60, 4, 3), (230, 8, 4)])
def test_tridiag_lowest_vs_numpy(n, k, seed):
    """edg_tridiag_lowest: the k lowest eigenvalues and |last eigenvector components| of a
    random tridiagonal against numpy's dense eigh."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=n) * 3 - 20
    e = np.abs(rng.normal(size=n)) + 0.3
    e[0] = 0.0
    T = np.diag(d) + np.diag(e[1:], 1) + np.diag(e[1:], -1)
    wr, V = np.linalg.eigh(T)
    w, zn = E.tridiag_lowest(d, e, k)
    kk = min(k, n)
    span = np.abs(wr).max()
    assert w.shape == (kk,)
    assert np.abs(w - wr[:kk]).max() <= 4e-15 * span
    assert np.abs(zn - np.abs(V[-1, :kk])).max() <= 1e-12


def test_tridiag_lowest_on_converged_lanczos():
    """A Lanczos tridiagonal whose lowest Ritz values have converged: their last components
    are tiny, and the twisted factorisation keeps them to high relative accuracy; QL's last
    row holds them to absolute accuracy, so both agree to ~1e-15 absolute."""
    rng = np.random.default_rng(9)
    n = 400
    A = rng.standard_normal((n, n))
    h = (A + A.T) / 2 + np.diag(np.linspace(-40, 0, n))
    a, b = _lanczos_tridiag(h, 150, 1)
    w, zn = E.tridiag_lowest(a, b, 4)
    wq, Zq = O.tridiag_eigh(a, b)
    wr = np.linalg.eigvalsh(h)
    assert np.abs(w - wq[:4]).max() <= 1e-12 * np.abs(wq).max()
    assert np.abs(w - wr[:4]).max() < 1e-8  # converged
    Tm = np.diag(a) + np.diag(b[1:], 1) + np.diag(b[1:], -1)
    V = np.linalg.eigh(Tm)[1]
    assert np.abs(zn - np.abs(V[-1, :4])).max() <= 1e-14
    assert zn.max() < 1e-6


def test_tridiag_lowest_close_pair():
    """Two nearly decoupled blocks with equal spectra give eigenvalue pairs 1e-14 apart:
    the eigenvalues stay exact to rounding and the last components stay finite in [0, 1]."""
    rng = np.random.default_rng(5)
    m = 20
    d1 = rng.normal(size=m)
    e1 = np.abs(rng.normal(size=m)) + 0.5
    d = np.concatenate([d1, d1])
    e = np.concatenate([e1, e1])
    e[0] = 0.0
    e[m] = 1e-14
    T = np.diag(d) + np.diag(e[1:], 1) + np.diag(e[1:], -1)
    wr = np.linalg.eigvalsh(T)
    w, zn = E.tridiag_lowest(d, e, 4)
    assert np.abs(w - wr[:4]).max() <= 1e-14 * np.abs(wr).max()
    assert np.all(np.isfinite(zn)) and np.all((zn >= 0) & (zn <= 1 + 1e-12))
