"""Pins for the CPU oracle (no GPU): known answers from the mathematics, dense
diagonalisation, the reference's own stored-vs-direct and Lanczos-vs-full-ED cross checks,
and the committed golden fixtures. The reference itself cannot be run here (Fortran +
SciFortran are absent), so these are what make the oracle trustworthy."""
import math
import os

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import oracle as O
from ed_lattice_b200.edlat import ring, square_lattice

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_binomial_and_sector_numbering():
    for n in range(0, 31):
        for k in range(-1, n + 2):
            assert O.binomial(n, k) == (math.comb(n, k) if 0 <= k <= n else 0)
    for ns in (4, 8, 16):
        for nup in range(ns + 1):
            for ndw in range(ns + 1):
                isec = O.lib().orc_get_sector(ns, nup, ndw)
                assert O.lib().orc_get_nup(ns, isec) == nup
                assert O.lib().orc_get_ndw(ns, isec) == ndw
    assert O.lib().orc_get_sector(16, 0, 0) == 1
    assert O.lib().orc_get_sector(16, 16, 16) == 17 * 17


def test_build_map_ascending_popcount():
    for ns in (1, 5, 8, 12):
        for n in range(ns + 1):
            m = O.build_map(ns, n)
            assert m.size == math.comb(ns, n)
            assert np.all(np.diff(m) > 0)
            assert all(bin(int(x)).count("1") == n for x in m)


def test_binary_search_positions_and_missing():
    m = O.build_map(10, 4)
    for pos in (0, 1, 7, m.size // 2, m.size - 1):
        assert O.binary_search(m, int(m[pos])) == pos + 1
    assert O.binary_search(m, 0b1111111) == 0  # popcount 7: absent
    assert O.binary_search(m[:0], 5) == 0


def test_c_cdg_sign_convention():
    # src/AUX_FUNX.f90:76-102: sign = (-1)^(set bits below pos)
    s = 0b101101
    out, sg = O.c_op(3, s)  # pos 3 (1-based) -> bit 2 set; bits below: bit0 -> 1 -> sign -1
    assert out == 0b101001 and sg == -1.0
    out, sg = O.cdg_op(2, s)  # bit 1 empty; below: bit0 -> sign -1
    assert out == 0b101111 and sg == -1.0
    out, sg = O.cdg_op(7, s)  # below: bits 0,2,3,5 -> 4 -> +1
    assert out == s | (1 << 6) and sg == 1.0


@pytest.mark.parametrize("U", [0.0, 2.0, 8.0])
def test_hubbard_dimer_closed_form(U):
    m = O.Model(np.array([[0.0, -1.0], [-1.0, 0.0]]), uloc=U, xmu=0.0, hfmode=False)
    w = np.linalg.eigvalsh(O.dense_h(m, 1, 1))
    assert abs(w[0] - (U - math.sqrt(U * U + 16.0)) / 2) < 1e-12
    # all four (1,1) levels: E = 0, U, (U +- sqrt(U^2+16))/2
    ref = sorted([0.0, U, (U - math.sqrt(U * U + 16)) / 2, (U + math.sqrt(U * U + 16)) / 2])
    assert np.allclose(w, ref, atol=1e-12)


@pytest.mark.parametrize("lat,nup,ndw", [("ring8", 4, 4), ("ring8", 3, 5), ("sq3x4", 6, 5)])
def test_free_fermion_limit(lat, nup, ndw):
    h = ring(8) if lat == "ring8" else square_lattice(3, 4)
    rng = np.random.default_rng(3)
    h = h + np.diag(np.round(rng.uniform(-1, 1, h.shape[0]) * 2 ** 16) / 2 ** 16)
    m = O.Model(h, uloc=0.0, xmu=0.0, hfmode=False)
    ev = np.linalg.eigvalsh(h)
    exact = ev[:nup].sum() + ev[:ndw].sum()
    st = O.Stored(m, nup, ndw)
    e0, _, _, _ = st.ground_state(O.random_vector(5, st.dim), maxit=400, tol=1e-15)
    assert abs(e0 - exact) < 1e-9 * max(1.0, abs(exact))


def test_atomic_limit():
    # t = 0: diagonal H; E0 = min over configurations of sum eps n + U n_up n_dw - xmu N
    eps = np.array([0.3, -0.7, 0.1, -0.2, 0.5, -0.4])
    m = O.Model(np.diag(eps), uloc=3.0, xmu=0.25, hfmode=False)
    H = O.dense_h(m, 3, 2)
    assert np.allclose(H, np.diag(np.diag(H)))
    mu, md = O.build_map(6, 3), O.build_map(6, 2)
    best = min(sum(eps[i] * (((u >> i) & 1) + ((d >> i) & 1)) + 3.0 * ((u >> i) & (d >> i) & 1) - 0.25 * (
        ((u >> i) & 1) + ((d >> i) & 1)) for i in range(6)) for d in md for u in mu)
    assert abs(np.diag(H).min() - best) < 1e-12


def test_stored_vs_direct_real_and_conjugation_quirk():
    rng = np.random.default_rng(0)
    ns = 6
    A = rng.normal(size=(ns, ns)) + 1j * rng.normal(size=(ns, ns))
    A = (A + A.conj().T) / 2
    v = rng.normal(size=20 * 15) + 1j * rng.normal(size=20 * 15)
    # real Hij: the two reference forms agree
    mr = O.Model(A.real.copy(), uloc=2.0, xmu=0.3, hfmode=True)
    st = O.Stored(mr, 3, 2)
    assert np.abs(st.matvec_z(v) - O.direct_matvec_z(mr, 3, 2, v)).max() < 1e-13
    # complex Hij: stored stores conjg(Hij) (stored/H_up.f90:20) -> equals direct with Hij^*
    mc = O.Model(A, uloc=2.0, xmu=0.3, hfmode=True)
    mcc = O.Model(A.conj(), uloc=2.0, xmu=0.3, hfmode=True)
    assert np.abs(O.Stored(mc, 3, 2).matvec_z(v) - O.direct_matvec_z(mcc, 3, 2, v)).max() < 1e-12


def test_direct_filling_shift_rule():
    # direct form applies xmu only when ed_filling == 0 (direct/HxV_local.f90:63); stored always
    h = ring(6)
    v = O.random_vector(11, 20 * 15)
    m0 = O.Model(h, uloc=4.0, xmu=1.5, hfmode=True, ed_filling=0)
    m5 = O.Model(h, uloc=4.0, xmu=1.5, hfmode=True, ed_filling=5)
    d0 = O.direct_matvec_d(m0, 3, 2, v)
    d5 = O.direct_matvec_d(m5, 3, 2, v)
    shift = (1.5 + 2.0) * 5  # (xmu + U/2) * N
    assert np.allclose(d0 - d5, -shift * v, atol=1e-12)
    assert np.allclose(O.Stored(m5, 3, 2).matvec_d(v), d0, atol=1e-12)


def test_hermitian_dense_and_lanczos_vs_dense():
    m = O.Model(ring(8), uloc=4.0, xmu=2.0, hfmode=False)
    H = O.dense_h(m, 4, 4)
    assert np.abs(H - H.T).max() == 0.0
    st = O.Stored(m, 4, 4)
    v = O.random_vector(1, st.dim)
    assert np.allclose(st.matvec_d(v), H @ v, atol=1e-12)
    w = np.linalg.eigvalsh(H)
    e0, vec, _, _ = st.ground_state(v, maxit=300, tol=1e-15)
    assert abs(e0 - w[0]) < 1e-10 * abs(w[0])
    assert np.linalg.norm(H @ vec - e0 * vec) < 1e-5


def test_lanczos_coefficients_vs_reorthogonalised_numpy():
    # independent implementation: Lanczos with full reorthogonalisation in numpy; the first
    # steps (before orthogonality is lost) must agree with the oracle's plain recurrence
    m = O.Model(ring(8), uloc=4.0, xmu=2.0, hfmode=False)
    H = O.dense_h(m, 4, 4)
    st = O.Stored(m, 4, 4)
    v0 = O.random_vector(2024, st.dim)
    a, b, n2, n = st.tridiag(v0, 25)
    assert abs(n2 - v0 @ v0) < 1e-12 * n2
    Q = [v0 / np.sqrt(v0 @ v0)]
    aa, bb = [], [0.0]
    for j in range(25):
        w = H @ Q[-1]
        aa.append(Q[-1] @ w)
        for q in Q:
            w -= (q @ w) * q
        for q in Q:
            w -= (q @ w) * q
        bb.append(np.linalg.norm(w))
        Q.append(w / bb[-1])
    assert np.allclose(a, aa, rtol=1e-9, atol=1e-9)
    assert np.allclose(b[1:], bb[1:25], rtol=1e-9, atol=1e-9)
    assert b[0] == 0.0


def test_tridiag_eigh_vs_scipy():
    rng = np.random.default_rng(4)
    d = rng.normal(size=40)
    e = np.concatenate([[0.0], rng.uniform(0.1, 2, 39)])
    w, Z = O.tridiag_eigh(d, e)
    ws, Zs = sla.eigh_tridiagonal(d, e[1:])
    assert np.allclose(w, ws, atol=1e-12)
    assert np.allclose(Z[0, :] ** 2, Zs[0, :] ** 2, atol=1e-12)


def test_gf_lanczos_vs_full_lehmann():
    # the reference's full-ED Lehmann sum (full_eval_gf_electrons_diag) as the check on the
    # Lanczos poles/weights (add_to_lanczos_gf_normal): ring of 6, (3,3), site 2, spin up
    m = O.Model(ring(6), uloc=3.0, xmu=1.5, hfmode=False)
    HI = O.dense_h(m, 3, 3)
    w, V = np.linalg.eigh(HI)
    e0, psi = w[0], V[:, 0]
    wm = np.pi * 0.05 * (2 * np.arange(1, 33) - 1)
    g_lanc = np.zeros(wm.size, complex)
    g_full = np.zeros(wm.size, complex)
    for op, isign, (nu, nd) in ((+1, +1, (4, 3)), (-1, -1, (2, 3))):
        x = O.apply_cop(6, 3, 3, op, 2, 1, psi)
        HJ = O.dense_h(m, nu, nd)
        stJ = O.Stored(m, nu, nd)
        n = min(stJ.dim, 200)
        a, b, n2, k = stJ.tridiag(x, n)
        p, wt = O.poles_weights(a[:k], b[:k], n2, e0, isign)
        assert abs(wt.sum() - n2) < 1e-12
        g_lanc += (wt[None, :] / (1j * wm[:, None] - p[None, :])).sum(1)
        wj, Vj = np.linalg.eigh(HJ)
        amp = (Vj.T @ x) ** 2
        g_full += (amp[None, :] / (1j * wm[:, None] - isign * (wj[None, :] - e0))).sum(1)
    assert np.abs(g_lanc - g_full).max() < 1e-9


def test_observables_vs_numpy():
    rng = np.random.default_rng(8)
    psi = rng.normal(size=56 * 28)
    psi /= np.linalg.norm(psi)
    obs = O.observables(8, 3, 2, psi)
    mu, md = O.build_map(8, 3), O.build_map(8, 2)
    P = (psi.reshape(md.size, mu.size)) ** 2
    nu = ((mu[None, :] >> np.arange(8)[:, None]) & 1).astype(float)  # [site, iup]
    nd = ((md[None, :] >> np.arange(8)[:, None]) & 1).astype(float)
    assert np.allclose(obs["dens_up"], nu @ P.sum(0))
    assert np.allclose(obs["dens_dw"], nd @ P.sum(1))
    assert np.allclose(obs["docc"], np.einsum("si,sj,ji->s", nu, nd, P))


def test_golden_fixtures_reproduce():
    g = np.load(os.path.join(GOLDEN, "ring8_U4_sector44.npz"))
    m = O.Model(ring(8), uloc=4.0, xmu=2.0, hfmode=False)
    st = O.Stored(m, 4, 4)
    v0 = O.random_vector(2024, st.dim)
    assert np.array_equal(v0, g["v0"])
    assert np.array_equal(st.matvec_d(v0), g["hv_stored"])
    assert np.array_equal(O.direct_matvec_d(m, 4, 4, v0), g["hv_direct"])
    a, b, n2, _ = st.tridiag(v0, 100)
    assert np.array_equal(a, g["alanc"]) and np.array_equal(b, g["blanc"])
    assert np.array_equal(O.build_map(8, 4), g["map_up"])
    g2 = np.load(os.path.join(GOLDEN, "disorder3x4.npz"))
    H = square_lattice(3, 4)
    H[np.diag_indices(12)] = g2["eps"]
    m2 = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    rp, c, v = O.hop_csr(m2, 1, 3)
    assert np.array_equal(rp, g2["rp_up"]) and np.array_equal(c, g2["c_up"]) and np.array_equal(v, g2["v_up"])
    assert np.array_equal(O.Stored(m2, 3, 2).matvec_d(g2["v0"]), g2["hv"])


@pytest.mark.parametrize("hfmode", [False, True])
def test_energy_terms_add_up_to_e0(hfmode):
    """lanc_energy's terms of an eigenstate rebuild its energy: E = Ekin + Epot + Eknot - xmu N
    (Epot includes the Hartree term), on a disordered 6-ring; U=0 gives Epot = Ehartree."""
    rng = np.random.default_rng(1)
    H = ring(6).astype(float)
    H[np.diag_indices(6)] = rng.uniform(-1, 1, 6)
    for u in (3.0, 0.0):
        m = O.Model(H, uloc=u, xmu=1.2, hfmode=hfmode)
        w, z = np.linalg.eigh(O.dense_h(m, 3, 2))
        for k in (0, 3):
            ekin, epot, eknot, eh = O.energy(m, 3, 2, z[:, k])
            assert abs(ekin + epot + eknot - 1.2 * 5 - w[k]) < 1e-12
            assert abs(eh - (-0.5 * u * 5 if hfmode else 0.0)) < 1e-12
            if u == 0.0:
                assert epot == eh


@pytest.mark.parametrize("phi,nup,ndw", [(0.7, 3, 3), (1.9, 2, 4), (np.pi, 3, 2)])
def test_complex_flux_ring_free_fermions(phi, nup, ndw):
    """The oracle's complex H x v (both forms) at U=0 on a 6-site ring threaded by flux phi,
    Hij(i, i+1) = -e^{i phi/L}: the lowest level of the dense matrix it defines equals the
    sum of the lowest single-particle energies -2 cos(2 pi m/L + phi/L) (stored form, which
    keeps conjg(Hij)) and -2 cos(2 pi m/L - phi/L) (direct form, Hij itself): the same set
    of energies, since the two are the spectra of H and of its complex conjugate."""
    L = 6
    H = np.zeros((L, L), complex)
    for i in range(L):
        H[i, (i + 1) % L] = -np.exp(1j * phi / L)
        H[(i + 1) % L, i] = -np.exp(-1j * phi / L)
    eps = np.sort(np.linalg.eigvalsh(H))
    ks = 2 * np.pi * np.arange(L) / L
    assert np.allclose(eps, np.sort(-2 * np.cos(ks + phi / L)), atol=1e-12)
    exact = eps[:nup].sum() + eps[:ndw].sum()
    m = O.Model(H, uloc=0.0, xmu=0.0, hfmode=False)
    D = math.comb(L, nup) * math.comb(L, ndw)
    st = O.Stored(m, nup, ndw)
    for matvec in (st.matvec_z, lambda v: O.direct_matvec_z(m, nup, ndw, v)):
        Hd = np.zeros((D, D), complex)
        for i in range(D):
            e = np.zeros(D, complex)
            e[i] = 1.0
            Hd[:, i] = matvec(e)
        assert np.abs(Hd - Hd.conj().T).max() < 1e-13
        assert abs(np.linalg.eigvalsh(Hd)[0] - exact) < 1e-10
