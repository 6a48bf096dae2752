"""Block chains (edg_tridiag_block_dev, edg_gf_chain_block, edg_chi_chain_block) against the
single-chain entry points and the oracle.

Every column of a block runs the single chain's arithmetic (same kernels, same reduction
order), so its Lanczos coefficients equal the single chain's bit for bit; the device QL of
the block's eigenproblems agrees with the host QL to rounding. Chains that stop early
(b < threshold) leave the others running, as the reference's per-chain loop does
(src/GF/GF_ELECTRONS.f90:202-290)."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _block_tridiag(s, X, nlanc, prec):
    k = X.shape[0]
    a, b = np.zeros(k * nlanc), np.zeros(k * nlanc)
    n2 = np.zeros(k)
    ns = np.zeros(k, dtype=np.int32)
    L.check(L.lib().edg_tridiag_block_dev(s.handle, k, C.c_void_p(X.data_ptr()), nlanc, 1e-9, prec,
                                          a.ctypes.data_as(L._pd), b.ctypes.data_as(L._pd), n2.ctypes.data_as(L._pd),
                                          ns.ctypes.data_as(L._pi)), "block")
    return a.reshape(k, nlanc), b.reshape(k, nlanc), n2, ns


def _single_tridiag(s, x, nlanc, prec):
    a, b = np.zeros(nlanc), np.zeros(nlanc)
    n2, ns = C.c_double(), C.c_int()
    L.check(L.lib().edg_tridiag_dev_f64(s.handle, C.c_void_p(x.data_ptr()), nlanc, 1e-9, prec,
                                        a.ctypes.data_as(L._pd), b.ctypes.data_as(L._pd), C.byref(n2), C.byref(ns)),
            "single")
    return a, b, n2.value, ns.value


def _start_block(s, k, seed):
    import torch
    return torch.tensor(np.stack([O.random_vector(seed + c, s.vlen) for c in range(k)]), dtype=torch.float64,
                        device="cuda")


@pytest.mark.parametrize("prec", [E.EDG_PREC_F64, E.EDG_PREC_F32], ids=["f64", "f32"])
def test_block_equals_single_chains(prec):
    """3x4 lattice, sector (7,6) (D = 731,808), 5 chains of 60 steps: bit-identical a, b."""
    model = E.Model(E.square_lattice(3, 4), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(model, 7, 6)
    X = _start_block(s, 5, 40)
    X[2] *= 1e-3  # a column of a different norm
    a, b, n2, ns = _block_tridiag(s, X, 60, prec)
    for c in range(5):
        a1, b1, n21, ns1 = _single_tridiag(s, X[c], 60, prec)
        assert ns[c] == ns1 == 60
        assert n2[c] == n21
        assert np.array_equal(a[c], a1) and np.array_equal(b[c], b1), c
    s.delete()


def test_block_early_stops_and_zero_columns():
    """One electron on the 2x3 lattice, sector (1,0) (D = 6): the uniform vector is an exact
    eigenvector of the translation-invariant hopping (b_1 = 0, one step), a single basis state
    and a random vector close their Krylov spaces within 6 steps, and a zero start vector
    gives norm2 = 0 and no steps; the other columns keep running when one stops, and every
    column equals the single chain."""
    import torch
    model = E.Model(E.square_lattice(2, 3), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(model, 1, 0)
    assert s.dim == 6
    X = torch.zeros(4, 6, dtype=torch.float64, device="cuda")
    X[0] = torch.tensor(O.random_vector(7, 6), dtype=torch.float64)
    X[2] = 1.0
    X[3, 0] = 1.0
    a, b, n2, ns = _block_tridiag(s, X, 40, E.EDG_PREC_F64)
    assert ns[1] == 0 and n2[1] == 0.0
    assert ns[2] == 1 and ns[0] <= 6 and ns[3] <= 6
    for c in range(4):
        a1, b1, n21, ns1 = _single_tridiag(s, X[c], 40, E.EDG_PREC_F64)
        assert ns[c] == ns1
        assert np.array_equal(a[c], a1) and np.array_equal(b[c], b1), c
    s.delete()


def test_gf_chain_block_vs_single_and_oracle():
    """Green's-function chains c^+_{i,up} of the ring-8 ground state into (5,4), all sites,
    one block, against edg_gf_chain (host QL) and the oracle chain of site 1."""
    h = E.ring(8)
    model = E.Model(h, uloc=4.0, xmu=2.0, hfmode=False)
    gs = E.Sector(model, 4, 4)
    e0, vec, _ = E.sp_lanc_eigh(gs, seed=3, tol=1e-14)
    to = E.Sector(model, 5, 4)
    sites = np.arange(1, 9)
    blk = E.gf_chain_block(gs, to, +1, sites, 1, 80, e0)
    for c, site in enumerate(sites):
        one = E.gf_chain(gs, to, +1, site, 1, 80, e0)
        assert blk[c].poles.size == one.poles.size
        assert blk[c].norm2 == one.norm2
        np.testing.assert_allclose(blk[c].poles, one.poles, rtol=0, atol=1e-11)
        np.testing.assert_allclose(blk[c].weight, one.weight, rtol=0, atol=1e-12)
    om = O.Model(h, uloc=4.0, xmu=2.0, hfmode=False)
    x = O.apply_cop(8, 4, 4, +1, 1, 1, vec)
    a, b, n2, n = O.Stored(om, 5, 4).tridiag(x, 80)
    p, w = O.poles_weights(a[:n], b[:n], n2, e0, +1)
    wm = np.pi / 50.0 * (2 * np.arange(1, 257) - 1)
    g = lambda pp, ww: (ww[None, :] / (1j * wm[:, None] - pp[None, :])).sum(1)
    assert np.abs(g(blk[0].poles, blk[0].weight) - g(p, w)).max() <= 1e-10 * np.abs(g(p, w)).max()
    # mixed (c_1 + c_j) chains in the same block form
    mix = E.gf_chain_block(gs, to, +1, [1, 1, 1], 1, 40, e0, sites2=[2, 3, 4])
    for c, j in enumerate((2, 3, 4)):
        one = E.gf_chain(gs, to, +1, 1, 1, 40, e0, site2=j)
        np.testing.assert_allclose(mix[c].weight, one.weight, rtol=0, atol=1e-12)
    for sct in (gs, to):
        sct.delete()


@pytest.mark.parametrize("prec", [E.EDG_PREC_F64, E.EDG_PREC_F32], ids=["f64", "f32"])
def test_chi_chain_block_momentum(prec):
    """Spin and charge momentum chains of the 3x4 ground state (sector (6,6)) for all 12
    momenta in one block each, against edg_chi_chain per momentum; the weights add up to
    <psi|O_q^+ O_q|psi> = norm2 of each chain."""
    lx, ly = 3, 4
    model = E.Model(E.square_lattice(lx, ly), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(model, 6, 6)
    e0, _, _ = E.sp_lanc_eigh(s, seed=5, tol=1e-13, want_vector=False)
    E.sp_lanc_eigh(s, seed=5, tol=1e-13)  # keeps the state
    xs, ys = np.meshgrid(np.arange(lx), np.arange(ly), indexing="xy")
    r = np.stack([xs.ravel(), ys.ravel()], 1)  # site i = x + lx*y
    qs = [(2 * np.pi * m / lx, 2 * np.pi * n / ly) for n in range(ly) for m in range(lx)]
    qcos = np.array([np.cos(q[0] * r[:, 0] + q[1] * r[:, 1]) for q in qs])
    # the chains have the same coefficients; the poles and weights come from the device QL
    # (block) and the host QL (single). The q = 0 charge operator is the conserved total N, so
    # its start vector is an eigenvector: with FP32 vectors the chain continues on rounding
    # noise, and the weights of those nearly decoupled poles agree only to FP32 level
    wtol = 1e-12 if prec == E.EDG_PREC_F64 else 1e-8
    for kind in (0, 1):
        blk = E.chi_chain_block(s, 60, e0, kind=kind, qcos=qcos, precision=prec)
        for c in range(len(qs)):
            one = E.chi_chain(s, 1, 60, e0, kind=kind, qcos=qcos[c], precision=prec)
            assert blk[c].norm2 == one.norm2
            np.testing.assert_allclose(blk[c].weight, one.weight, rtol=0, atol=wtol * max(1.0, one.norm2))
            mb = [(blk[c].weight * blk[c].poles ** n).sum() for n in range(5)]
            mo = [(one.weight * one.poles ** n).sum() for n in range(5)]
            assert np.allclose(mb, mo, rtol=1e-10, atol=1e-12), (kind, c)
            assert abs(blk[c].weight.sum() - blk[c].norm2) <= 1e-9 * max(1.0, blk[c].norm2)
    s.delete()


def test_poles_weights_block_vs_host():
    rng = np.random.default_rng(3)
    k, nl = 7, 90
    a = rng.normal(size=(k, nl))
    b = np.abs(rng.normal(size=(k, nl)))
    b[:, 0] = 0.0
    ns = np.array([90, 1, 45, 90, 0, 17, 89], dtype=np.int32)
    n2 = rng.uniform(0.1, 2.0, k)
    p = np.zeros(k * nl)
    w = np.zeros(k * nl)
    L.check(L.lib().edg_poles_weights_block(k, nl, a.ctypes.data_as(L._pd), b.ctypes.data_as(L._pd),
                                            n2.ctypes.data_as(L._pd), ns.ctypes.data_as(L._pi), 0.25, -1,
                                            p.ctypes.data_as(L._pd), w.ctypes.data_as(L._pd)), "poles_block")
    p, w = p.reshape(k, nl), w.reshape(k, nl)
    for c in range(k):
        m = ns[c]
        if m == 0:
            continue
        ph, wh = E.poles_weights(a[c, :m], b[c, :m], n2[c], 0.25, -1)
        np.testing.assert_allclose(p[c, :m], ph, rtol=0, atol=1e-12 * np.abs(ph).max())
        np.testing.assert_allclose(w[c, :m], wh, rtol=0, atol=1e-12)
