"""GPU parity of the lowest-k sector solver and the finite-temperature driver on the 3x4
disordered Hubbard lattice (t=1, U=4, XMU=2, eps_i quantised to 2^-16, all 169 sectors):
the dense sector matrix against the oracle's, the lowest four levels of every sector against
the committed fixture (dense LAPACK for D <= 4000, ARPACK over the oracle's H x v above), and
the thermal state list, Z and site observables at beta=20 against the same fixture."""
import math
import os

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200.diag import DiagParams, diagonalize_lattice, lanc_observables, partition_function
from ed_lattice_b200.edlat import square_lattice
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(GOLDEN, "thermal3x4.npz"))


def _hij(eps):
    H = square_lattice(3, 4)
    H[np.diag_indices(12)] = eps
    return H


def _sectors(fx, pred):
    out = []
    for isector in range(1, 170):
        nup, ndw = (isector - 1) // 13, (isector - 1) % 13
        if pred(int(fx["dims"][isector - 1])):
            out.append((isector, nup, ndw))
    return out


def test_dense_matrix_and_lowest_k_small_sectors(fx):
    """Every sector with D <= 4000: edg_sector_dense equals the oracle's dense matrix, and the
    lowest four Lanczos eigenpairs match dense diagonalisation (E to 1e-10, residual of the
    vector under the oracle's H x v to 1e-8)."""
    H = _hij(fx["eps"])
    gm, om = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False), O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    small = _sectors(fx, lambda d: d <= 4000)
    assert len(small) == 68
    for isector, nup, ndw in small:
        s = E.Sector(gm, nup, ndw)
        hd = O.dense_h(om, nup, ndw)
        assert np.allclose(s.dense(), hd, rtol=0, atol=1e-13), (nup, ndw)
        ev, vecs, resid, m = s.lowest_k(4, seed=17, tol=1e-11)
        kk = min(4, s.dim)
        ref = fx["energies"][isector - 1, :kk]
        assert np.allclose(ev, ref, rtol=0, atol=1e-10), (nup, ndw, ev, ref)
        for r in range(kk):
            x = vecs[r]
            assert abs(np.dot(x, x) - 1.0) < 1e-10
            assert np.linalg.norm(hd @ x - ev[r] * x) < 1e-8, (nup, ndw, r)
        s.delete()


@pytest.mark.parametrize("mode", [E.EDG_LK_F64, E.EDG_LK_F32_REFINE], ids=["f64", "f32refine"])
@pytest.mark.parametrize("nup,ndw", [(6, 6), (5, 6), (3, 2), (7, 4)])
def test_lowest_k_large_sectors(fx, nup, ndw, mode):
    """Sectors beyond the dense range (D up to 853,776) against ARPACK's levels, FP64 and FP32
    bulk + FP64 refinement (the same tolerances: the refinement is FP64)."""
    H = _hij(fx["eps"])
    gm, om = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False), O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, nup, ndw)
    ev, vecs, resid, m = s.lowest_k(4, seed=3, tol=1e-10, mode=mode)
    ref = fx["energies"][gm.get_sector(nup, ndw) - 1]
    assert np.allclose(ev, ref, rtol=0, atol=1e-9), (ev, ref)
    assert np.all(resid <= 1e-10 * np.maximum(1.0, np.abs(ev)))
    st = O.Stored(om, nup, ndw)
    for r in range(4):
        x = vecs[r]
        assert np.linalg.norm(st.matvec_d(x) - ev[r] * x) < 1e-8
        for q in range(r):
            assert abs(np.dot(x, vecs[q])) < 1e-9
    s.delete()


def test_lowest_k_start_vector_and_argument_checks(fx):
    H = _hij(fx["eps"])
    gm = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, 3, 3)
    v0 = E.random_vector(17, s.dim)
    a = s.lowest_k(2, v0=v0, tol=1e-10)
    b = s.lowest_k(2, seed=17, tol=1e-10)
    assert np.array_equal(a[0], b[0])  # the seeded start vector is edg_random_vector's
    with pytest.raises(E.EdgError):
        s.lowest_k(17)
    with pytest.raises(E.EdgError):
        s.lowest_k(2, tol=0.0)
    one = E.Sector(gm, 0, 0)
    ev, vecs, _, _ = one.lowest_k(4)
    assert ev.shape == (1,) and abs(abs(vecs[0, 0]) - 1.0) < 1e-15
    s.delete()
    one.delete()


@pytest.mark.parametrize("dim_threshold,fp32,twin", [(4000, False, False), (0, False, False), (1024, True, False),
                                                    (1024, True, True)])
def test_thermal_beta20_all_sectors(fx, dim_threshold, fp32, twin):
    """diagonalize_lattice + partition_function + lanc_observables at T=0.05 over the 169
    sectors (lowest 4 each), with the dense branch up to D=4000, with Lanczos everywhere, with
    FP32 bulk + FP64 refinement in the Lanczos sectors, and with twin sectors (the 91 sectors
    with Nup >= Ndw solved, the others taken as spin-flipped copies)."""
    H = _hij(fx["eps"])
    gm = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    p = DiagParams(finite_temp=True, temp=0.05, cutoff=1e-9, lanc_nstates_sector=4,
                   lanc_dim_threshold=dim_threshold, lanc_tolerance=1e-10, lanc_fp32_bulk=fp32, ed_twin=twin)
    sl, eigs = diagonalize_lattice(gm, p, seed=1234)
    assert len(eigs) == (91 if twin else 169)
    for isector, ev, _ in eigs:
        ref = fx["energies"][isector - 1]
        assert np.allclose(ev, ref[: ev.size], rtol=0, atol=1e-9), (isector, ev, ref)
    zeta = partition_function(sl, p)
    assert sl.emin == pytest.approx(float(fx["egs"]), abs=1e-10)
    if twin:  # the twins' levels are copies: the kept list is the same set of states
        assert all(s.vec is not None for s in sl.states[: sl.trimd_size])
    assert sl.trimd_size == int(fx["nkept"])
    assert sorted(s.sector for s in sl.states[: sl.trimd_size]) == sorted(fx["kept_sectors"].tolist())
    assert zeta == pytest.approx(float(fx["zeta"]), rel=1e-8)
    obs = lanc_observables(gm, sl, zeta, p)
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.allclose(obs[k], fx[k], rtol=0, atol=1e-8), (k, obs[k], fx[k])
    assert math.isclose(obs["dens"].sum(), float(fx["dens"].sum()), abs_tol=1e-8)
