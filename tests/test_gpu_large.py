"""Full-size checks on the 4x4 half-filled sector (D = 165,636,900, U=8),
where the CPU oracle is too slow to run: size-independent properties of the operator and
agreement between the FP32 and FP64 device paths (the FP64 path is bit-exact against the
oracle on the smaller sectors of test_gpu_parity.py)."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L

pytestmark = pytest.mark.gpu


def on_torch_stream(s):
    """The _dev entry points are ordered on the sector's stream; put it on torch's stream
    so the kernels see tensors torch has just written."""
    import torch
    L.check(L.lib().edg_sector_set_stream(s.handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    return s


@pytest.fixture(scope="module")
def sector():
    model = E.Model(E.square_lattice(4, 4), uloc=8.0, xmu=4.0, hfmode=False)
    s = on_torch_stream(E.Sector(model, 8, 8))
    yield s
    s.delete()


def hxv(s, x):
    import torch
    torch.cuda.synchronize()
    y = torch.empty_like(x)
    fn = L.lib().edg_hxv_dev_f64 if x.dtype == torch.float64 else L.lib().edg_hxv_dev_f32
    L.check(fn(s.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "hxv")
    torch.cuda.synchronize()
    return y


def test_large_f32_matches_f64(sector):
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(sector.dim, device="cuda", dtype=torch.float64, generator=g) * 2 - 1
    y64 = hxv(sector, x)
    y32 = hxv(sector, x.float())
    err = (y32.double() - y64).abs().max().item()
    scale = y64.abs().max().item()
    assert err <= 2e-6 * scale
    del y32
    # linearity and symmetry (<x|H z> = <H x|z>) at full size, FP64
    z = torch.rand(sector.dim, device="cuda", dtype=torch.float64, generator=g) * 2 - 1
    hz = hxv(sector, z)
    lhs = hxv(sector, 0.5 * x - 2.0 * z)
    assert (lhs - (0.5 * y64 - 2.0 * hz)).abs().max().item() <= 1e-12 * scale
    a = torch.dot(x, hz).item()
    b = torch.dot(y64, z).item()
    assert abs(a - b) <= 1e-10 * abs(a)


def test_large_stored_vs_direct(sector):
    import torch
    model = E.Model(E.square_lattice(4, 4), uloc=8.0, xmu=4.0, hfmode=False)
    sd = on_torch_stream(E.Sector(model, 8, 8, E.EDG_FORM_DIRECT))
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.rand(sector.dim, device="cuda", dtype=torch.float64, generator=g) * 2 - 1
    ys = hxv(sector, x)
    yd = hxv(sd, x)
    # integer matrix elements, sources ascending in both: only the order of the two spin
    # parts differs (stored: diag, DW, UP; direct: diag, UP, DW)
    assert (ys - yd).abs().max().item() <= 1e-12 * ys.abs().max().item()
    sd.delete()


def test_gf_chains_4x4_U4_full_size():
    """4x4 lattice at U=4: ground state of (8,8), then c^+_{1,up} into (9,8) and c_{1,up} into
    (7,8) (D = 147,232,800 each). The particle and hole norms add up to 1 (the anticommutator
    {c, c^+} = 1 on a normalised state), their difference is 1 - 2 n_{1,up} from the state's
    observables, and the FP32 chains reproduce the FP64 G(iw_n) at beta=50."""
    model = E.Model(E.square_lattice(4, 4), uloc=4.0, xmu=2.0, hfmode=False)
    gs = E.Sector(model, 8, 8)
    part, hole = E.Sector(model, 9, 8), E.Sector(model, 7, 8)
    e0, it = C.c_double(), C.c_int()
    L.check(L.lib().edg_ground_state_keep(gs.handle, None, C.c_uint64(2024), 600, 1e-10, E.EDG_GS_F32_REFINE,
                                          C.byref(e0), C.byref(it)), "gs")
    n_up = gs.observables()["dens_up"][0]
    en = gs.energy()  # E0 = Ekin + Epot + Eknot - xmu N at full size (16 electrons, XMU=2)
    assert abs(en["ekin"] + en["epot"] + en["eknot"] - 2.0 * 16 - e0.value) <= 1e-9 * abs(e0.value)
    sp = {}
    for prec in (E.EDG_PREC_F64, E.EDG_PREC_F32):
        sp[prec] = (E.gf_chain(gs, part, +1, 1, 1, 150, e0.value, precision=prec),
                    E.gf_chain(gs, hole, -1, 1, 1, 150, e0.value, precision=prec))
    p64, h64 = sp[E.EDG_PREC_F64]
    assert abs(p64.norm2 + h64.norm2 - 1.0) < 1e-12
    assert abs((p64.norm2 - h64.norm2) - (1.0 - 2.0 * n_up)) < 1e-12
    wm = np.pi / 50.0 * (2 * np.arange(1, 65) - 1)
    g = {}
    for prec, (pa, ho) in sp.items():
        g[prec] = sum((ch.weight[None, :] / (1j * wm[:, None] - ch.poles[None, :])).sum(1) for ch in (pa, ho))
    assert np.abs(g[E.EDG_PREC_F32] - g[E.EDG_PREC_F64]).max() <= 1e-5 * np.abs(g[E.EDG_PREC_F64]).max()
    for s in (gs, part, hole):
        s.delete()
