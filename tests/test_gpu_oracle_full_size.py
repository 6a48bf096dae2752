"""The benchmarked sector against the oracle at full size, and the north-star tolerances.

Workload: 4x4 periodic square lattice, t=1, U=8, XMU=4 (mu = U/2), sector (8,8),
D = 12870^2 = 165,636,900 -- the sector of the H x v and E0 benchmarks.

* FP64 H x v, stored form (spMatVec, src/DIAG/HAMILTONIAN_STORED_HxV.f90:159-220) and
  direct form (directMatVec, src/DIAG/HAMILTONIAN_DIRECT_HxV.f90:19-59): every matrix
  element is an integer and both sides sum each output element in the reference's order,
  so the device result equals the oracle's bit for bit.
* E0: the oracle's FP64 Lanczos (the sp_lanc_eigh contract) to |dE0| <= 1e-13 |E0| per step,
  against the device's plain FP64 path (1e-10 relative) and FP32 + FP64 refinement
  (1e-8 relative); the first 40 Lanczos coefficients of the same start vector to 1e-9.
* GF spectral weights with FP32 vectors: the 3x4 disordered lattice of the thermal
  workload, c^+_{1,up} from the (6,6) ground state into (7,6) (D = 792 x 924 = 731,808), 150
  steps, against the oracle's FP64 chain: the Matsubara function, the low spectral moments
  and the converged poles' weights to 1e-6 (FP64 vectors: 1e-10).
"""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LX, LY, U = 4, 4, 8.0


def _on_torch_stream(s):
    import torch
    L.check(L.lib().edg_sector_set_stream(s.handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    return s


def _hxv_dev(s, v_host):
    import torch
    x = torch.from_numpy(v_host).cuda()
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    L.check(L.lib().edg_hxv_dev_f64(s.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "hxv")
    torch.cuda.synchronize()
    out = y.cpu().numpy()
    del x, y
    return out


@pytest.fixture(scope="module")
def models():
    h = E.square_lattice(LX, LY)
    return E.Model(h, uloc=U, xmu=U / 2, hfmode=False), O.Model(h, uloc=U, xmu=U / 2, hfmode=False)


@pytest.fixture(scope="module")
def oracle_stored(models):
    return O.Stored(models[1], 8, 8)


def test_stored_hxv_bit_exact_full_size(models, oracle_stored):
    em, _ = models
    s = _on_torch_stream(E.Sector(em, 8, 8, E.EDG_FORM_STORED))
    assert s.dim == 165636900 == oracle_stored.dim
    v = O.random_vector(31, s.dim)
    ref = oracle_stored.matvec_d(v)
    got = _hxv_dev(s, v)
    s.delete()
    assert np.array_equal(got, ref), f"max |diff| {np.abs(got - ref).max()}"


def test_f32_hxv_every_up_pass_full_size(models, oracle_stored):
    """FP32 H x v of the benchmarked sector on each FP32 up pass (SELL, packed 16-bit with
    negated copies or sign bits, Kronecker) after the default down pass, against the oracle's
    FP64 spMatVec: 2e-6 of max|Hv|. The Kronecker pass sums each element's terms in another
    order than the SELL pass, so its result differs from it in rounding only."""
    import torch
    em, _ = models
    s = _on_torch_stream(E.Sector(em, 8, 8, E.EDG_FORM_STORED))
    v = O.random_vector(33, s.dim)
    ref = oracle_stored.matvec_d(v)
    scale = np.abs(ref).max()
    x = torch.from_numpy(v).cuda().float()
    got = {}
    for up in range(4):
        s.set_kernels(up, E.EDG_PREC_F32)  # candidate 4*down + up, down pass 0
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        L.check(L.lib().edg_hxv_dev_f32(s.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "hxv")
        torch.cuda.synchronize()
        got[up] = y.double().cpu().numpy()
        assert np.abs(got[up] - ref).max() <= 2e-6 * scale, (up, np.abs(got[up] - ref).max() / scale)
    assert not np.array_equal(got[3], got[0])  # the Kronecker schedule is the one that ran
    del x, y
    s.delete()
    torch.cuda.empty_cache()


def test_direct_hxv_bit_exact_full_size(models):
    em, om = models
    s = _on_torch_stream(E.Sector(em, 8, 8, E.EDG_FORM_DIRECT))
    v = O.random_vector(32, s.dim)
    ref = O.direct_matvec_d(om, 8, 8, v)
    got = _hxv_dev(s, v)
    s.delete()
    assert np.array_equal(got, ref), f"max |diff| {np.abs(got - ref).max()}"


def test_e0_and_coefficients_vs_oracle_lanczos(models, oracle_stored):
    import torch
    em, _ = models
    s = _on_torch_stream(E.Sector(em, 8, 8))
    v0 = O.random_vector(2024, s.dim)
    e_o, _, a_o, b_o = oracle_stored.ground_state(v0, maxit=400, tol=1e-13, want_vector=False)
    # the first 40 coefficients of the same start vector (FP64 device recurrence)
    a, b, n2, ns = E.tridiag_Hv_sector(s, v0, 40)
    assert ns == 40
    assert np.abs(a - a_o[:40]).max() <= 1e-9
    assert np.abs(b[1:] - b_o[1:40]).max() <= 1e-9
    e64, _, _ = E.sp_lanc_eigh(s, v0=v0, maxit=600, tol=1e-12, mode=E.EDG_GS_F64, want_vector=False)
    assert abs(e64 - e_o) <= 1e-10 * abs(e_o), (e64, e_o)
    e32, x, it = E.sp_lanc_eigh(s, v0=v0, maxit=600, tol=1e-8, mode=E.EDG_GS_F32_REFINE, want_vector=True)
    assert abs(e32 - e_o) <= 1e-8 * abs(e_o), (e32, e_o)
    # the returned vector is normalised and its Rayleigh quotient is E0 to the same bar;
    # the residual |H x - E0 x| is the square root of the E0 error times the gap, so only
    # its size is bounded here
    hx = _hxv_dev(s, x)
    nx = float(np.dot(x, x))
    rq = float(np.dot(x, hx)) / nx
    res = float(np.linalg.norm(hx - e32 * x))
    assert abs(nx - 1.0) <= 1e-12
    assert abs(rq - e_o) <= 1e-8 * abs(e_o), (rq, e_o)
    assert res <= 1e-2 * abs(e_o), res
    s.delete()
    torch.cuda.empty_cache()


def _thermal_model():
    rng = np.random.default_rng(7)
    h = E.square_lattice(3, 4)
    h[np.diag_indices(12)] = np.round(rng.uniform(-1, 1, 12) * 65536) / 65536
    return h


def test_fp32_gf_weights_vs_oracle_chain():
    """Spectral weights of the c^+ chain, FP32 and FP64 vectors, against the oracle's FP64
    chain from the same ground state: G(iw_n) on 4096 Matsubara frequencies at beta=50, the
    moments sum_k w_k p_k^n (n <= 8, which the first steps of any Lanczos chain fix), and the
    weight and position of every CONVERGED pole (Ritz residual b_151 |z_150,k| below 1e-8).
    After 150 steps the remaining poles are unconverged Ritz values of the 731,808-state
    sector: they depend on the rounding of each recurrence and are not compared one by one."""
    h = _thermal_model()
    em, om = E.Model(h, uloc=4.0, xmu=2.0, hfmode=False), O.Model(h, uloc=4.0, xmu=2.0, hfmode=False)
    st66 = O.Stored(om, 6, 6)
    e0, psi, _, _ = st66.ground_state(O.random_vector(5, st66.dim), maxit=400, tol=1e-15)
    vec = O.apply_cop(12, 6, 6, +1, 1, 1, psi)
    a_o, b_o, n2_o, n_o = O.Stored(om, 7, 6).tridiag(vec, 151)
    assert n_o == 151
    p_o, w_o = O.poles_weights(a_o[:150], b_o[:150], n2_o, e0, +1)
    _, Z = O.tridiag_eigh(a_o[:150], b_o[:150])
    res = np.abs(b_o[150] * Z[-1, :])  # same (ascending) order as p_o
    conv = (res < 1e-8) & (w_o > 1e-6)
    assert conv.any()
    gs = E.Sector(em, 6, 6)
    gs.set_state(psi)
    part = E.Sector(em, 7, 6)
    ch = {prec: E.gf_chain(gs, part, +1, 1, 1, 150, e0, precision=prec) for prec in (E.EDG_PREC_F64, E.EDG_PREC_F32)}
    gs.delete()
    part.delete()
    wm = np.pi / 50.0 * (2 * np.arange(1, 4097) - 1)

    def gmats(p, w):
        return (w[None, :] / (1j * wm[:, None] - p[None, :])).sum(1)

    def moments(p, w):
        return np.array([(w * p ** k).sum() for k in range(9)])

    g_o = gmats(p_o, w_o)
    m_o = moments(p_o, w_o)
    for prec, tol in ((E.EDG_PREC_F64, 1e-10), (E.EDG_PREC_F32, 1e-6)):
        c = ch[prec]
        assert c.poles.size == 150
        assert abs(c.norm2 - n2_o) <= tol * n2_o
        g = gmats(c.poles, c.weight)
        assert np.abs(g - g_o).max() <= tol * np.abs(g_o).max(), (prec, np.abs(g - g_o).max())
        assert np.all(np.abs(moments(c.poles, c.weight) - m_o) <= tol * np.abs(m_o)), prec
        for pk, wk in zip(p_o[conv], w_o[conv]):
            near = np.abs(c.poles - pk) <= 1e-4
            # a recurrence that loses orthogonality may repeat a converged pole: the copies sit
            # at its position and share its weight; an unconverged Ritz value that happens to
            # lie within 1e-4 of it carries no weight of its own
            copies = np.abs(c.poles - pk) <= tol * max(1.0, abs(pk))
            assert copies.any(), (prec, pk, c.poles[near])
            assert abs(c.weight[near].sum() - wk) <= tol, (prec, pk, wk, c.weight[near].sum())
            assert c.weight[near & ~copies].sum() <= tol, (prec, pk, c.poles[near], c.weight[near])
