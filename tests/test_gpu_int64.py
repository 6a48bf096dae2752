"""The 6x3 periodic lattice at half filling, sector (9,9): D = 48,620^2 = 2,363,904,400 > 2^31,
beyond the reference's int32 Dim. Checks of the 64-bit indexing at full size: exact columns
H e_i for indices past 2^31 (integer matrix elements, so FP32 is exact), FP32 against FP64,
and the symmetry <x|H z> = <H x|z>."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NS, N, U, XMU = 18, 9, 4.0, 2.0


@pytest.fixture(scope="module")
def big():
    import torch
    model = E.Model(E.square_lattice(6, 3), uloc=U, xmu=XMU, hfmode=False)
    s = E.Sector(model, N, N)
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    assert s.dim == 2_363_904_400 and s.dim > 2**31
    yield s
    s.delete()
    torch.cuda.empty_cache()


def hxv(s, x, y):
    import torch
    fn = L.lib().edg_hxv_dev_f64 if x.dtype == torch.float64 else L.lib().edg_hxv_dev_f32
    L.check(fn(s.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "hxv")
    torch.cuda.synchronize()


def chunked_dot(a, b, chunk=1 << 28):
    tot = 0.0
    for i in range(0, a.numel(), chunk):
        tot += float((a[i:i + chunk].double() * b[i:i + chunk].double()).sum().item())
    return tot


def expected_column(i, maps, tabs, dimup):
    """H e_i from the oracle's hop tables: diagonal -XMU*(2N) + U*popcount(up & dw) (eps = 0,
    HFMODE=F), up hops along the row of idw, down hops along the column of iup."""
    iup, idw = i % dimup, i // dimup
    mu, md = int(maps[iup]), int(maps[idw])
    cols = {i: -XMU * 2 * N + U * bin(mu & md).count("1")}
    rp, c, v = tabs
    for k in range(rp[iup], rp[iup + 1]):
        cols[int(c[k]) + idw * dimup] = float(v[k])
    for k in range(rp[idw], rp[idw + 1]):
        cols[iup + int(c[k]) * dimup] = float(v[k])
    return cols


def test_diag_formula_small_sector():
    """The diagonal used below, checked against the oracle's stored H x v on sector (2,2)."""
    om = O.Model(E.square_lattice(6, 3), uloc=U, xmu=XMU, hfmode=False)
    st = O.Stored(om, 2, 2)
    maps = O.build_map(NS, 2)
    for i in (0, 77, st.dim - 1):
        e = np.zeros(st.dim)
        e[i] = 1.0
        iup, idw = i % maps.size, i // maps.size
        assert st.matvec_d(e)[i] == -XMU * 4 + U * bin(int(maps[iup]) & int(maps[idw])).count("1")


def test_columns_past_int32(big):
    import torch
    om = O.Model(E.square_lattice(6, 3), uloc=U, xmu=XMU, hfmode=False)
    maps = O.build_map(NS, N)
    tabs = O.hop_csr(om, 1, N)  # same table for both spins (same N, spin-independent Hij)
    x = torch.zeros(big.dim, dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    for i in (0, 2**31 - 5, 2**31 + 12_345, big.dim - big.dimup + 17, big.dim - 1):
        x[i] = 1.0
        hxv(big, x, y)
        x[i] = 0.0
        exp = expected_column(i, maps, tabs, big.dimup)
        idx = torch.tensor(sorted(exp), dtype=torch.int64, device="cuda")
        got = y[idx].double().cpu().numpy()
        want = np.array([exp[j] for j in sorted(exp)])
        assert np.array_equal(got, want), i
        assert int((y != 0).sum().item()) == sum(1 for val in exp.values() if val != 0), i
    del x, y
    torch.cuda.empty_cache()


def test_f32_f64_and_symmetry(big):
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    x64 = torch.rand(big.dim, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    y64 = torch.empty_like(x64)
    hxv(big, x64, y64)
    x32 = x64.float()
    y32 = torch.empty_like(x32)
    hxv(big, x32, y32)
    err = 0.0
    chunk = 1 << 28
    for i in range(0, big.dim, chunk):
        err = max(err, (y32[i:i + chunk].double() - y64[i:i + chunk]).abs().max().item())
    scale = y64[: 1 << 26].abs().max().item()
    assert err <= 2e-6 * scale
    del y64, x64
    torch.cuda.empty_cache()
    z32 = torch.rand(big.dim, dtype=torch.float32, device="cuda", generator=g) * 2 - 1
    hz = torch.empty_like(z32)
    hxv(big, z32, hz)
    a = chunked_dot(x32, hz)
    b = chunked_dot(y32, z32)
    assert abs(a - b) <= 1e-5 * max(abs(a), 1.0)
    del x32, y32, z32, hz
    torch.cuda.empty_cache()


def test_ground_state_and_momentum_chi_full_size(big):
    """The full 2.36e9-state sector: FP32+refine ground state to 1e-8 (its energy terms add up
    to E0: one FP64 H x v of the state), then spin and charge susceptibility chains at
    q = (pi, 0) (site weights (-1)^x) with FP32 and FP64 vectors agreeing on chi(i nu_n)."""
    e0, it = C.c_double(), C.c_int()
    L.check(L.lib().edg_ground_state_keep(big.handle, None, C.c_uint64(2024), 400, 1e-8, E.EDG_GS_F32_REFINE,
                                          C.byref(e0), C.byref(it)), "gs")
    en = big.energy()
    assert abs(en["ekin"] + en["epot"] + en["eknot"] - XMU * 2 * N - e0.value) <= 1e-8 * abs(e0.value)
    qcos = np.array([(-1.0) ** (i % 6) for i in range(NS)])
    beta = 10.0
    vm = 2 * np.pi / beta * np.arange(0, 12)
    for kind in (0, 1):
        chi = {}
        for prec in (E.EDG_PREC_F64, E.EDG_PREC_F32):
            sp = E.chi_chain(big, 1, 60, e0.value, kind=kind, qcos=qcos, precision=prec)
            assert sp.norm2 > 0 and np.all(sp.weight >= 0)
            w, p_ = sp.weight, sp.poles
            chi[prec] = np.array([(w * 2 * p_ / (v * v + p_ * p_)).sum() if v > 0 else (2 * w / np.maximum(p_, 1e-12)).sum()
                                  for v in vm])
            chi[(prec, "n2")] = sp.norm2
        assert abs(chi[(E.EDG_PREC_F32, "n2")] - chi[(E.EDG_PREC_F64, "n2")]) <= 1e-12 * chi[(E.EDG_PREC_F64, "n2")]
        assert np.abs(chi[E.EDG_PREC_F32][1:] - chi[E.EDG_PREC_F64][1:]).max() <= 1e-5 * np.abs(chi[E.EDG_PREC_F64]).max()


@pytest.mark.parametrize("nup,ndw,hop", [(7, 1, "uniform"), (7, 2, "random"), (2, 7, "uniform")])
def test_split_up_pass_vs_oracle(nup, ndw, hop):
    """DimUp = C(18,7) = 31,824: an FP64 row (255 KB) exceeds shared memory, so the FP64 up
    pass stages it in two column parts. FP64 against the oracle: bit-exact for integer matrix
    elements (same summation order), 1e-13 with random hoppings (non-uniform tables); FP32
    within 2e-6. (2,7) puts the long dimension on the down spin instead."""
    import torch
    H = E.square_lattice(6, 3)
    if hop == "random":
        rng = np.random.default_rng(11)
        f = np.round(rng.uniform(0.5, 1.5, H.shape) * 4096) / 4096
        H = H * (f + f.T) / 2
    gm = E.Model(H, uloc=U, xmu=XMU, hfmode=False)
    om = O.Model(H, uloc=U, xmu=XMU, hfmode=False)
    s = E.Sector(gm, nup, ndw)
    v = O.random_vector(23, s.dim)
    ref = O.Stored(om, nup, ndw).matvec_d(v)
    hv = s.hxv_real(v)
    if hop == "uniform":
        assert np.array_equal(hv, ref)
    else:
        assert np.abs(hv - ref).max() <= 1e-13 * np.abs(ref).max()
    dv = torch.tensor(v, dtype=torch.float32, device="cuda")
    dh = torch.empty_like(dv)
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    L.check(L.lib().edg_hxv_dev_f32(s.handle, C.c_void_p(dv.data_ptr()), C.c_void_p(dh.data_ptr())), "f32")
    torch.cuda.synchronize()
    assert np.abs(dh.double().cpu().numpy() - ref).max() <= 2e-6 * np.abs(ref).max()
    s.delete()
