"""Every H x v kernel pair of the autotuner's list against the oracle: the FP64 stored-form
H x v is bit-exact for every pair (the passes keep the reference's summation order), the
FP32 one agrees with FP64 to 2e-6 relative, and the fused Lanczos step and block chains run
on the pinned pair. Sectors: the 3x4 disordered lattice's (6,6) (D = 853,776) and the
4x4 U=8 (5,5) sector (D = 19,079,424, DimUp 4368 < 2^15: the packed schedules apply).
FP32 candidates are 4*down + up with up 3 the Kronecker schedule and down 3 the single-pass
H x v (no up pass); the last FP32 candidate (the single pass) also runs the fused FP32
Lanczos steps."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _models(case):
    if case == "sq3x4_66":
        rng = np.random.default_rng(7)
        h = E.square_lattice(3, 4)
        h[np.diag_indices(12)] = np.round(rng.uniform(-1, 1, 12) * 65536) / 65536
        return h, 4.0, (6, 6)
    return E.square_lattice(4, 4), 8.0, (5, 5)


def _hxv(s, x, fn):
    import torch
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    L.check(fn(s.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "hxv")
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("case", ["sq3x4_66", "sq4x4_55"])
def test_all_kernel_pairs(case):
    import torch
    h, u, (nup, ndw) = _models(case)
    em, om = E.Model(h, uloc=u, xmu=u / 2, hfmode=False), O.Model(h, uloc=u, xmu=u / 2, hfmode=False)
    s = E.Sector(em, nup, ndw)
    L.check(L.lib().edg_sector_set_stream(s.handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "st")
    v = O.random_vector(9, s.dim)
    ref = O.Stored(om, nup, ndw).matvec_d(v)
    x64 = torch.from_numpy(v).cuda()
    x32 = x64.float()
    scale = np.abs(ref).max()
    for cand in range(4):
        s.set_kernels(cand, E.EDG_PREC_F64)
        y = _hxv(s, x64, L.lib().edg_hxv_dev_f64).cpu().numpy()
        assert np.array_equal(y, ref), (case, "f64", cand, np.abs(y - ref).max())
    for cand in range(16):
        s.set_kernels(cand, E.EDG_PREC_F32)
        y = _hxv(s, x32, L.lib().edg_hxv_dev_f32).double().cpu().numpy()
        assert np.abs(y - ref).max() <= 2e-6 * scale, (case, "f32", cand, np.abs(y - ref).max() / scale)
    # the fused FP32 Lanczos step on the last pair: E0 against the FP64 path
    e32, _, _ = E.sp_lanc_eigh(s, seed=4, tol=1e-10, mode=E.EDG_GS_F32_REFINE, want_vector=False)
    e64, _, _ = E.sp_lanc_eigh(s, seed=4, tol=1e-12, mode=E.EDG_GS_F64, want_vector=False)
    assert abs(e32 - e64) <= 1e-10 * abs(e64)
    # autotune leaves a valid choice that reproduces the FP64 result bit for bit
    t = s.autotune(E.EDG_PREC_F64, reps=1)
    assert len(t["ms"]) == 4 and 0 <= t["best"] < 4
    y = _hxv(s, x64, L.lib().edg_hxv_dev_f64).cpu().numpy()
    assert np.array_equal(y, ref)
    with pytest.raises(E.EdgError):
        s.set_kernels(16, E.EDG_PREC_F32)
    s.delete()
