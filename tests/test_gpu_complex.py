"""Complex Hij on the device (Peierls phases, complex random hoppings): the complex H x v
of both reference forms against the oracle's complex restatements (orc_stored_matvec_z,
orc_direct_matvec_z), including the reference's conjugation quirk between the forms; the
Lanczos chain and the ground state against a numpy restatement of the same recurrence and
dense diagonalisation built from the oracle's H x v. FP64 within 1e-13 relative per H x v
(the complex products are fused differently from std::complex), coefficients within 1e-9,
E0 within 1e-10; FP32 within FP32 round-off."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from ed_lattice_b200.edlat import ring
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def flux_ring(ns, phi, t=1.0, seed=None):
    """Ring threaded by flux phi: Hij(i, i+1) = -t e^{i phi/ns}, Hermitian; optional site
    energies quantised to 2^-16."""
    H = np.zeros((ns, ns), complex)
    for i in range(ns):
        j = (i + 1) % ns
        H[i, j] = -t * np.exp(1j * phi / ns)
        H[j, i] = np.conj(H[i, j])
    if seed is not None:
        rng = np.random.default_rng(seed)
        H[np.diag_indices(ns)] = np.round(rng.uniform(-1, 1, ns) * 65536) / 65536
    return H


def random_hermitian(ns, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(ns, ns)) + 1j * rng.normal(size=(ns, ns))
    return (A + A.conj().T) / 2


def models(h, **kw):
    return E.Model(h, **kw), O.Model(h, **kw)


def cvec(seed, n):
    rng = np.random.default_rng(seed)
    return rng.normal(size=n) + 1j * rng.normal(size=n)


def np_lanczos(matvec, v0, nlanc):
    """sp_lanc_tridiag's recurrence on complex vectors (real a, b): the reference's
    convention b[0] = 0, b[j] = b_{j+1}."""
    v = v0 / np.linalg.norm(v0)
    vp = np.zeros_like(v)
    a, b = np.zeros(nlanc), np.zeros(nlanc)
    bj = 0.0
    for j in range(nlanc):
        w = matvec(v) - bj * vp
        a[j] = np.vdot(v, w).real
        w = w - a[j] * v
        bj = np.linalg.norm(w)
        if j + 1 < nlanc:
            b[j + 1] = bj
        vp, v = v, w / bj
    return a, b


def dense_from_matvec(matvec, dim):
    H = np.zeros((dim, dim), complex)
    for i in range(dim):
        e = np.zeros(dim, complex)
        e[i] = 1.0
        H[:, i] = matvec(e)
    return H


@pytest.mark.parametrize("form", [E.EDG_FORM_STORED, E.EDG_FORM_DIRECT])
@pytest.mark.parametrize("case", ["flux", "random", "nspin2"])
def test_complex_hxv_vs_oracle(form, case):
    if case == "flux":
        H, nup, ndw = flux_ring(8, 0.7, seed=3), 4, 3
    elif case == "random":
        H, nup, ndw = random_hermitian(6, 5), 3, 2
    else:
        H, nup, ndw = np.stack([flux_ring(6, 0.4), flux_ring(6, -1.1, t=0.5, seed=2)]), 3, 2
    gm, om = models(H, uloc=2.0, xmu=0.3, hfmode=True)
    s = E.Sector(gm, nup, ndw, form)
    assert s.cplx and s.vlen == 2 * s.dim
    v = cvec(7, s.dim)
    ref = O.Stored(om, nup, ndw).matvec_z(v) if form == E.EDG_FORM_STORED else O.direct_matvec_z(om, nup, ndw, v)
    hv = s.HxV(v)
    assert np.abs(hv - ref).max() <= 1e-13 * np.abs(ref).max()
    s.delete()


def test_complex_forms_differ_by_conjugation():
    """The reference's stored form keeps conjg(Hij) where the direct form uses Hij: on the
    device as in the oracle, stored(H) = direct(conj H) and stored(H) != direct(H)."""
    H = flux_ring(8, 1.3, seed=1)
    gm = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    gc = E.Model(H.conj(), uloc=4.0, xmu=2.0, hfmode=False)
    st = E.Sector(gm, 4, 4, E.EDG_FORM_STORED)
    dr = E.Sector(gm, 4, 4, E.EDG_FORM_DIRECT)
    dc = E.Sector(gc, 4, 4, E.EDG_FORM_DIRECT)
    v = cvec(2, st.dim)
    a, b, c = st.HxV(v), dr.HxV(v), dc.HxV(v)
    assert np.abs(a - c).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(a - b).max() > 1e-3 * np.abs(a).max()
    for s in (st, dr, dc):
        s.delete()


def test_complex_hermitian_and_device_f32():
    """<x|H y> = <H x|y> on the device, and the FP32 device H x v on interleaved vectors
    against FP64 within FP32 round-off."""
    import torch
    gm, _ = models(flux_ring(10, 0.9, seed=4), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, 5, 5)
    x, y = cvec(1, s.dim), cvec(2, s.dim)
    hx, hy = s.HxV(x), s.HxV(y)
    assert abs(np.vdot(x, hy) - np.vdot(hx, y)) <= 1e-12 * np.abs(np.vdot(x, hy))
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    dx = torch.tensor(x.view(np.float64), dtype=torch.float32, device="cuda")
    dh = torch.empty_like(dx)
    L.check(L.lib().edg_hxv_dev_f32(s.handle, C.c_void_p(dx.data_ptr()), C.c_void_p(dh.data_ptr())), "f32")
    torch.cuda.synchronize()
    h32 = dh.double().cpu().numpy().view(np.complex128)
    assert np.abs(h32 - hx).max() <= 2e-6 * np.abs(hx).max()
    s.delete()


@pytest.mark.parametrize("precision,tol", [(E.EDG_PREC_F64, 1e-9), (E.EDG_PREC_F32, 2e-4)])
def test_complex_tridiag_vs_numpy(precision, tol):
    """tridiag_Hv_sector on a complex start vector: norm2, a(1:40), b(2:40) against the same
    recurrence in numpy over the oracle's complex stored H x v."""
    gm, om = models(flux_ring(8, 0.7, seed=3), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, 4, 4)
    st = O.Stored(om, 4, 4)
    v0 = cvec(11, s.dim)
    a, b, n2, k = E.tridiag_Hv_sector(s, v0, nlanc=40, precision=precision)
    ar, br = np_lanczos(st.matvec_z, v0, 40)
    assert k == 40
    assert abs(n2 - np.vdot(v0, v0).real) <= 1e-12 * n2
    assert np.abs(a - ar).max() <= tol * np.abs(ar).max()
    assert np.abs(b[1:] - br[1:]).max() <= tol * np.abs(br).max()
    assert b[0] == 0.0
    s.delete()


@pytest.mark.parametrize("mode", [E.EDG_GS_F64, E.EDG_GS_F32_REFINE])
def test_complex_ground_state_vs_dense(mode):
    """sp_lanc_eigh on a complex sector: E0 against dense diagonalisation of the oracle's
    complex H (1e-10 relative), the eigenvector's residual under the oracle's H x v."""
    gm, om = models(flux_ring(8, 1.1, seed=6), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, 4, 4)
    st = O.Stored(om, 4, 4)
    Hd = dense_from_matvec(st.matvec_z, s.dim)
    assert np.abs(Hd - Hd.conj().T).max() < 1e-12
    e_ref = np.linalg.eigvalsh(Hd)[0]
    e0, vec, _ = E.sp_lanc_eigh(s, tol=1e-12, mode=mode)
    assert abs(e0 - e_ref) <= 1e-10 * abs(e_ref)
    assert vec.dtype == np.complex128 and abs(np.linalg.norm(vec) - 1.0) < 1e-10
    assert np.linalg.norm(st.matvec_z(vec) - e0 * vec) < 1e-6
    s.delete()


def test_complex_errors():
    """Real host vectors are refused by edg_hxv_d on a complex sector; state sizes are checked;
    c/c+ between a complex and a real sector is refused."""
    gm = E.Model(flux_ring(6, 0.5), uloc=1.0)
    s = E.Sector(gm, 3, 3)
    with pytest.raises(E.EdgError) as ei:
        s.hxv_real(np.zeros(s.dim))
    assert ei.value.status == L.EDG_ERR_ARG
    E.sp_lanc_eigh(s, tol=1e-10)
    r4 = E.Sector(E.Model(ring(6), uloc=1.0), 4, 3)
    with pytest.raises(E.EdgError) as ei:
        E.gf_chain(s, r4, +1, 1, 1, 10, 0.0)
    assert ei.value.status == L.EDG_ERR_ARG
    r4.delete()
    with pytest.raises(ValueError):
        s.set_state(np.zeros(s.dim + 1))
    s.delete()
    # a real model keeps real vectors
    r = E.Sector(E.Model(ring(6), uloc=1.0), 3, 3)
    assert not r.cplx and r.vlen == r.dim
    r.delete()


# ----------------------------------------------------------------------------- excitations
def _dev(x):
    import torch
    return torch.tensor(np.ascontiguousarray(x).view(np.float64), dtype=torch.float64, device="cuda")


def _host(t, cplx):
    import torch
    torch.cuda.synchronize()
    a = t.cpu().numpy()
    return a.view(np.complex128) if cplx else a


@pytest.mark.parametrize("op,spin", [(+1, 1), (-1, 1), (+1, 2), (-1, 2)])
def test_complex_cop_and_diagop_match_real_parts(op, spin):
    """c^+/c and S^z, N (with momentum weights) are real-linear: on a complex vector they equal
    the real-Hij path applied to its real and imaginary parts, bit for bit."""
    import torch
    gc = E.Model(flux_ring(6, 0.8), uloc=2.0)
    gr = E.Model(ring(6), uloc=2.0)
    nupJ, ndwJ = 3 + (op if spin == 1 else 0), 2 + (op if spin == 2 else 0)
    sc, scJ = E.Sector(gc, 3, 2), E.Sector(gc, nupJ, ndwJ)
    sr, srJ = E.Sector(gr, 3, 2), E.Sector(gr, nupJ, ndwJ)
    x = cvec(4, sc.dim)
    dx, dxr, dxi = _dev(x), _dev(x.real.copy()), _dev(x.imag.copy())
    out = torch.empty(2 * scJ.dim, dtype=torch.float64, device="cuda")
    outr = torch.empty(scJ.dim, dtype=torch.float64, device="cuda")
    outi = torch.empty_like(outr)
    for site in (1, 4):
        L.check(L.lib().edg_apply_cop_dev_f64(sc.handle, scJ.handle, op, site, spin, 1.0, 0, C.c_void_p(dx.data_ptr()),
                                              C.c_void_p(out.data_ptr())), "cop")
        for src, dst in ((dxr, outr), (dxi, outi)):
            L.check(L.lib().edg_apply_cop_dev_f64(sr.handle, srJ.handle, op, site, spin, 1.0, 0,
                                                  C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr())), "cop")
        z = _host(out, True)
        assert np.array_equal(z.real, _host(outr, False)) and np.array_equal(z.imag, _host(outi, False))
    q = np.cos(np.pi / 3 * np.arange(6))
    out = torch.empty(2 * sc.dim, dtype=torch.float64, device="cuda")
    outr = torch.empty(sc.dim, dtype=torch.float64, device="cuda")
    outi = torch.empty_like(outr)
    for kind in (0, 1):
        L.check(L.lib().edg_apply_diagop_dev_f64(sc.handle, kind, 0, 0, q.ctypes.data_as(L._pd),
                                                 C.c_void_p(dx.data_ptr()), C.c_void_p(out.data_ptr())), "diagop")
        for src, dst in ((dxr, outr), (dxi, outi)):
            L.check(L.lib().edg_apply_diagop_dev_f64(sr.handle, kind, 0, 0, q.ctypes.data_as(L._pd),
                                                     C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr())), "diagop")
        z = _host(out, True)
        assert np.array_equal(z.real, _host(outr, False)) and np.array_equal(z.imag, _host(outi, False))
    for s_ in (sc, scJ, sr, srJ):
        s_.delete()


def _current_restated(H, ns, nup, ndw, psi):
    """lanc_ed_build_oc's J|psi> / i (src/OC/OC_ELECTRONS.f90:139-198) in plain Python: bond
    (i, i+1) periodic, + Hij(i,j) c^+_i c_j - conjg(Hij(j,i)) c^+_j c_i per spin."""
    mu, md = O.build_map(ns, nup), O.build_map(ns, ndw)
    du = mu.size
    out = np.zeros(psi.size, complex)
    for i in range(psi.size):
        iup, idw = i % du, i // du
        for isite in range(ns):
            jsite = (isite + 1) % ns
            for io, jo, coef in ((isite, jsite, H[isite, jsite]), (jsite, isite, -np.conj(H[jsite, isite]))):
                if H[io, jo] == 0:
                    continue
                for spin, m in ((1, int(mu[iup])), (2, int(md[idw]))):
                    if not ((m >> jo) & 1) or ((m >> io) & 1):
                        continue
                    k1, sg1 = O.c_op(jo + 1, m)
                    k2, sg2 = O.cdg_op(io + 1, k1)
                    if spin == 1:
                        j = int(np.searchsorted(mu, k2)) + idw * du
                    else:
                        j = iup + int(np.searchsorted(md, k2)) * du
                    out[j] += coef * sg1 * sg2 * psi[i]
    return out


def test_complex_current_vs_restatement():
    import torch
    H = flux_ring(6, 0.9, seed=8)
    gm = E.Model(H, uloc=2.0)
    s = E.Sector(gm, 3, 2)
    x = cvec(6, s.dim)
    dx = _dev(x)
    out = torch.empty_like(dx)
    L.check(L.lib().edg_apply_current_dev_f64(s.handle, C.c_void_p(dx.data_ptr()), C.c_void_p(out.data_ptr())), "J")
    ref = _current_restated(H, 6, 3, 2, x)
    assert np.abs(_host(out, True) - ref).max() <= 1e-14 * np.abs(ref).max()
    s.delete()


def test_complex_observables_and_energy_identity():
    """Site densities and double occupancies of a complex ground state against the oracle on
    |psi| (they depend on |psi|^2 only); ekin + epot + eknot - xmu N = E0."""
    U, XMU = 4.0, 2.0
    gm, om = models(flux_ring(8, 1.1, seed=6), uloc=U, xmu=XMU, hfmode=False)
    s = E.Sector(gm, 4, 3)
    e0, vec, _ = E.sp_lanc_eigh(s, tol=1e-13)
    obs = s.observables()
    ref = O.observables(8, 4, 3, np.abs(vec), 1.0)
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.abs(obs[k] - ref[k]).max() < 1e-12, k
    en = s.energy()
    assert abs(en["ekin"] + en["epot"] + en["eknot"] - XMU * 7 - e0) <= 1e-10 * abs(e0)
    s.delete()


def test_complex_gf_chain_vs_lehmann():
    """Particle and hole chains from a complex ground state against the Lehmann sums of dense
    diagonalisation of the oracle's complex H in the target sectors (c^+ psi formed in numpy
    from the oracle's c/cdg), compared on the Matsubara axis."""
    ns = 6
    H = flux_ring(ns, 0.7, seed=9)
    gm, om = models(H, uloc=3.0, xmu=1.5, hfmode=False)
    s = E.Sector(gm, 3, 3)
    e0, psi, _ = E.sp_lanc_eigh(s, tol=1e-14)
    mu = O.build_map(ns, 3)
    wm = np.pi * 0.05 * (2 * np.arange(32) + 1)
    for op in (+1, -1):
        nupJ = 3 + op
        sJ = E.Sector(gm, nupJ, 3)
        muJ = O.build_map(ns, nupJ)
        x = np.zeros(sJ.dim, complex)
        for i in range(psi.size):
            iup, idw = i % mu.size, i // mu.size
            m = int(mu[iup])
            pos = 1  # site 1, spin up
            if op > 0 and not (m & 1):
                k, sg = O.cdg_op(pos, m)
            elif op < 0 and (m & 1):
                k, sg = O.c_op(pos, m)
            else:
                continue
            x[int(np.searchsorted(muJ, k)) + idw * muJ.size] += sg * psi[i]
        Hd = dense_from_matvec(O.Stored(om, nupJ, 3).matvec_z, sJ.dim)
        w, V = np.linalg.eigh(Hd)
        amp = np.abs(V.conj().T @ x) ** 2
        g_ref = (amp[None, :] / (1j * wm[:, None] - op * (w[None, :] - e0))).sum(1)
        sp = E.gf_chain(s, sJ, op, 1, 1, sJ.dim, e0)
        g = (sp.weight[None, :] / (1j * wm[:, None] - sp.poles[None, :])).sum(1)
        assert abs(sp.norm2 - np.vdot(x, x).real) <= 1e-12
        assert np.abs(g - g_ref).max() <= 1e-8 * np.abs(g_ref).max()
        sJ.delete()
    s.delete()


# ----------------------------------------------------------------------------- lowest k, dense, driver
def test_complex_dense_matrix_vs_oracle():
    gm, om = models(flux_ring(6, 0.6, seed=12), uloc=2.0, xmu=1.0, hfmode=True)
    s = E.Sector(gm, 3, 2)
    Hd = dense_from_matvec(O.Stored(om, 3, 2).matvec_z, s.dim)
    assert np.abs(s.dense() - Hd).max() < 1e-14
    s.delete()


@pytest.mark.parametrize("seed", [17, 3])
def test_complex_lowest_k_vs_dense(seed):
    """Lowest four levels of a complex sector (D = 1568) with their vectors: levels to 1e-10
    against dense diagonalisation (so no level appears twice: complex Gram-Schmidt keeps the
    i-rotated copies of the basis out), residuals under the oracle's H x v, orthonormality."""
    gm, om = models(flux_ring(8, 1.3, seed=5), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(gm, 2, 3)
    st = O.Stored(om, 2, 3)
    ref = np.linalg.eigvalsh(dense_from_matvec(st.matvec_z, s.dim))[:4]
    ev, vecs, resid, m = s.lowest_k(4, seed=seed, tol=1e-11)
    assert np.abs(ev - ref).max() <= 1e-10 * np.abs(ref).max(), (ev, ref)
    assert vecs.dtype == np.complex128
    for r in range(4):
        x = vecs[r]
        assert abs(np.vdot(x, x).real - 1.0) < 1e-10
        assert np.linalg.norm(st.matvec_z(x) - ev[r] * x) < 1e-8
        for q in range(r):
            assert abs(np.vdot(vecs[q], x)) < 1e-9
    s.delete()


def test_complex_thermal_driver_vs_brute_force():
    """diagonalize_lattice + partition_function + lanc_observables on a complex model (6-site
    ring with flux, all 49 sectors, Lanczos everywhere) against every eigenstate of every
    sector from dense diagonalisation of the oracle's complex H."""
    import math

    from ed_lattice_b200.diag import DiagParams, diagonalize_lattice, lanc_observables, partition_function

    ns, temp = 6, 0.3
    H = flux_ring(ns, 0.9, seed=21)
    gm, om = models(H, uloc=3.0, xmu=1.5, hfmode=False)
    p = DiagParams(finite_temp=True, temp=temp, lanc_nstates_sector=4, lanc_dim_threshold=0, lanc_tolerance=1e-11)
    sl, eigs = diagonalize_lattice(gm, p, seed=7)
    zeta = partition_function(sl, p)
    obs = lanc_observables(gm, sl, zeta, p)
    states = []
    for nup in range(ns + 1):
        for ndw in range(ns + 1):
            D = math.comb(ns, nup) * math.comb(ns, ndw)
            w, V = np.linalg.eigh(dense_from_matvec(O.Stored(om, nup, ndw).matvec_z, D))
            states += [(w[i], nup, ndw, V[:, i]) for i in range(min(4, D))]
    egs = min(st[0] for st in states)
    kept = sorted((st for st in states if math.exp(-(st[0] - egs) / temp) > p.cutoff), key=lambda st: st[0])
    zref = sum(math.exp(-(st[0] - egs) / temp) for st in kept)
    assert sl.emin == pytest.approx(egs, abs=1e-10)
    assert zeta == pytest.approx(zref, rel=1e-9)
    ref = {k: np.zeros(ns) for k in ("dens", "dens_up", "dens_dw", "docc")}
    for e, nup, ndw, v in kept:
        o = O.observables(ns, nup, ndw, np.abs(v), math.exp(-(e - egs) / temp) / zref)
        for k in ref:
            ref[k] += o[k]
    for k in ref:
        assert np.allclose(obs[k], ref[k], atol=1e-9), k
