"""Host logic of the sector-diagonalisation driver (no GPU): the state list (es_*), the
finite-T bookkeeping of ed_diag_d, partition_function_lattice and lanc_observables. The
per-sector eigensolver and the observables of one state are injected from the CPU oracle
(dense diagonalisation), and the thermal averages are checked against a brute-force sum over
every eigenstate of every sector."""
import math

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200.diag import DiagParams, StateList, diagonalize_lattice, lanc_observables, partition_function
from oracle import oracle as O


def test_state_list_order_cap_and_pop():
    sl = StateList()
    for e, sec in ((0.5, 1), (-1.0, 2), (0.5, 3), (2.0, 4)):
        sl.add_state(e, None, sec)
    # equal energies: the newcomer goes before the older entry (es_insert_state)
    assert [s.sector for s in sl.states] == [2, 3, 1, 4]
    assert sl.emin == -1.0 and sl.emax == 2.0
    sl.pop_state()
    assert sl.energy() == 0.5 and sl.emax == 2.0  # pop keeps the running maximum
    # capped insert: a full list only takes states below its last entry
    sl.add_state(1.0, None, 5, size=3)
    assert sl.size == 3 and 5 not in [s.sector for s in sl.states]
    sl.add_state(0.0, None, 6, size=3)
    assert [s.e for s in sl.states] == [-1.0, 0.0, 0.5]
    sl.pop_state(1)
    assert sl.energy(1) == 0.0
    sl.free()
    assert sl.size == 0 and sl.emin == math.inf
    with pytest.raises(E.EdgError):
        sl.pop_state()


def test_state_list_trim_and_degeneracy():
    sl = StateList()
    for e in (0.0, 1e-10, 0.3, 0.6, 5.0):
        sl.add_state(e, None, 1)
    assert sl.gs_degeneracy(1e-9) == 2
    # T=0.1, cutoff 1e-9: exp(-E/T) > 1e-9 for E < 2.07
    assert sl.trim_size(0.1, 1e-9, True) == 4
    assert sl.trim_size(0.1, 1e-9, False) == 5


def test_setup_state_counts():
    p = DiagParams(finite_temp=True, lanc_nstates_sector=3).setup(169)
    assert p.lanc_nstates_sector == 4 and p.lanc_nstates_total == 4 * 169 + 10
    p = DiagParams(finite_temp=True, lanc_nstates_sector=2).setup(25)
    assert p.lanc_nstates_total == 60
    with pytest.raises(E.EdgError):
        DiagParams(lanc_method="nope").setup(4)


def _chain4(seed=3):
    rng = np.random.default_rng(seed)
    H = E.ring(4).astype(float)
    H[np.diag_indices(4)] = np.round(rng.uniform(-1, 1, 4) * 2**16) / 2**16
    return H


def _oracle_solver(om):
    def solve(model, nup, ndw, neigen, lanc_solve, params, seed):
        w, z = np.linalg.eigh(O.dense_h(om, nup, ndw))
        return w[:neigen], z[:, :neigen].T.copy()
    return solve


def _oracle_observer(model, isector, vec, bw):
    return O.observables(model.ns, model.get_nup(isector), model.get_ndw(isector), vec, bw)


def _brute_force(om, ns, temp, cutoff):
    """Every eigenstate of every sector: Z and weighted observables with the reference cutoff."""
    states = []
    for nup in range(ns + 1):
        for ndw in range(ns + 1):
            w, z = np.linalg.eigh(O.dense_h(om, nup, ndw))
            states += [(w[i], nup, ndw, z[:, i]) for i in range(w.size)]
    egs = min(s[0] for s in states)
    kept = [s for s in states if math.exp(-(s[0] - egs) / temp) > cutoff]
    zeta = sum(math.exp(-(s[0] - egs) / temp) for s in kept)
    acc = {k: np.zeros(ns) for k in ("dens", "dens_up", "dens_dw", "docc", "magz")}
    for e, nup, ndw, v in kept:
        o = O.observables(ns, nup, ndw, v, math.exp(-(e - egs) / temp) / zeta)
        for k in acc:
            acc[k] += o[k]
    return egs, zeta, acc


@pytest.mark.parametrize("temp", [0.05, 0.5])
def test_finite_temperature_against_brute_force(temp):
    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    # 36 states per sector = every state of the 4-site sectors: the list is exact up to the cutoff
    p = DiagParams(finite_temp=True, temp=temp, lanc_nstates_sector=36)
    sl, eigs = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    assert len(eigs) == 25
    zeta = partition_function(sl, p)
    obs = lanc_observables(m, sl, zeta, p, observer=_oracle_observer)
    egs, zref, ref = _brute_force(om, 4, temp, p.cutoff)
    assert sl.emin == pytest.approx(egs, abs=1e-13)
    assert zeta == pytest.approx(zref, rel=1e-12)
    for k in ref:
        assert np.allclose(obs[k], ref[k], atol=1e-12), k
    assert np.allclose(obs["mag"], obs["dens_up"] - obs["dens_dw"])


def test_cutoff_condition_not_met_raises():
    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    p = DiagParams(finite_temp=True, temp=5.0, lanc_nstates_sector=2)
    with pytest.raises(E.EdgError, match="Cutoff"):
        diagonalize_lattice(m, p, solver=_oracle_solver(om))


def test_zero_temperature_ground_manifold():
    H = _chain4(seed=11)
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    p = DiagParams(finite_temp=False, lanc_nstates_sector=2)
    sl, _ = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    # brute force: lowest level over all sectors and its multiplet (spin degeneracy across Sz)
    lev = sorted((np.linalg.eigvalsh(O.dense_h(om, a, b))[0], a, b) for a in range(5) for b in range(5))
    e0 = lev[0][0]
    manifold = [(a, b) for (e, a, b) in lev if abs(e - e0) <= 1e-9]
    assert sl.size == len(manifold) == sl.gs_degeneracy()
    assert sorted((m.get_nup(s.sector), m.get_ndw(s.sector)) for s in sl.states) == sorted(manifold)
    zeta = partition_function(sl, p)
    assert zeta == float(len(manifold))
    obs = lanc_observables(m, sl, zeta, p, observer=_oracle_observer)
    assert obs["dens"].sum() == pytest.approx(sum(a + b for a, b in manifold) / len(manifold), abs=1e-10)


def test_filling_restricts_sectors():
    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False, ed_filling=4)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False, ed_filling=4)
    p = DiagParams(finite_temp=True, temp=0.2, lanc_nstates_sector=36)
    sl, eigs = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    assert len(eigs) == 5  # (0,4) (1,3) (2,2) (3,1) (4,0)
    assert all(m.get_nup(s.sector) + m.get_ndw(s.sector) == 4 for s in sl.states)


def test_thermal_energy_identity():
    """lanc_energy over the state list with the oracle's per-state energies: the thermal
    <H> = Ekin + Epot + Eknot - xmu <N> equals sum_i p_i E_i."""
    from ed_lattice_b200.diag import lanc_energy
    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=True)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=True)
    p = DiagParams(finite_temp=True, temp=0.5, lanc_nstates_sector=36)
    sl, _ = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    zeta = partition_function(sl, p)

    def energy_fn(model, isector, vec, bw):
        ek, ep, ekn, eh = O.energy(om, model.get_nup(isector), model.get_ndw(isector), vec, bw)
        return {"ekin": ek, "epot": ep, "eknot": ekn, "ehartree": eh}

    en = lanc_energy(m, sl, zeta, p, energy_fn=energy_fn)
    obs = lanc_observables(m, sl, zeta, p, observer=_oracle_observer)
    egs = sl.emin
    n = sl.trimd_size
    h_avg = sum(math.exp(-(sl.energy(i) - egs) / p.temp) * sl.energy(i) for i in range(1, n + 1)) / zeta
    assert en["ekin"] + en["epot"] + en["eknot"] - 2.0 * obs["dens"].sum() == pytest.approx(h_avg, abs=1e-12)
    assert en["ehartree"] == pytest.approx(-0.5 * 4.0 * obs["dens"].sum(), abs=1e-12)


@pytest.mark.parametrize("temp,finite_temp", [(0.4, True), (0.001, False)])
def test_gf_driver_against_lehmann(temp, finite_temp):
    """build_gf_electrons + eval_gf_electrons over the state list (oracle chains injected)
    against the brute-force Lehmann sum, diagonal and off-diagonal (via the (c_i + c_j)
    chains and G_ij = (G~_ij - G_ii - G_jj)/2), at finite T and at T=0."""
    from ed_lattice_b200.gf import build_gf_electrons, eval_gf_electrons
    from gf_reference import lehmann_g, oracle_chain_fn
    H = _chain4(seed=5)
    m = E.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    om = O.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    p = DiagParams(finite_temp=finite_temp, temp=temp, lanc_nstates_sector=36 if finite_temp else 2)
    sl, _ = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    zeta = partition_function(sl, p)
    gm = build_gf_electrons(m, sl, offdiag=True, chain_fn=oracle_chain_fn(m, om))
    assert len(gm) == 16 and all(len(v) == sl.size for v in gm.values())
    wm = np.pi * temp * (2 * np.arange(1, 33) - 1)
    wr = np.linspace(-4, 4, 41)
    gmats, greal = eval_gf_electrons(gm, sl, zeta, p.temp, p.finite_temp, p.cutoff, wm, wr, 0.1, 1, 4, backend="host")
    pairs = [(1, 1), (2, 2), (1, 2), (1, 3), (4, 2)]
    ref_m = lehmann_g(om, 4, temp, p.cutoff, finite_temp, pairs, 1j * wm)
    ref_r = lehmann_g(om, 4, temp, p.cutoff, finite_temp, pairs, wr + 0.1j)
    for (i, j) in pairs:
        assert np.abs(gmats[0, i - 1, j - 1] - ref_m[(i, j)]).max() < 1e-9, (i, j)
        assert np.abs(greal[0, i - 1, j - 1] - ref_r[(i, j)]).max() < 1e-7, (i, j)  # eta=0.1: pole errors x 1/eta^2


@pytest.mark.parametrize("kind", [0, 1])
def test_chi_driver_against_exact_spectra(kind):
    """build_chi + eval_chi_electrons (oracle chains injected) against the same evaluation of
    exact Lehmann spectra per state, at finite T: S^z (kind 0) and charge (kind 1)."""
    from ed_lattice_b200.edlat import grids
    from ed_lattice_b200.gf import build_chi, eval_chi_electrons
    from gf_reference import exact_channels, spectra_all_sectors
    H = _chain4(seed=7)
    m = E.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    om = O.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    p = DiagParams(finite_temp=True, temp=0.5, lanc_nstates_sector=36)
    sl, _ = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    zeta = partition_function(sl, p)

    def chain(isector, vec, io, nlanc, ei):
        nup, ndw = m.get_nup(isector), m.get_ndw(isector)
        x = O.apply_diagop(4, nup, ndw, kind, io, vec)
        st = O.Stored(om, nup, ndw)
        a, b, n2, n = st.tridiag(x, min(nlanc, st.dim), 1e-9)
        if n == 0 or n2 == 0.0:
            return E.Spectrum(np.zeros(0), np.zeros(0), n2)
        pp, ww = O.poles_weights(a[:n], b[:n], n2, ei, +1)
        return E.Spectrum(pp, ww, n2)

    cm = build_chi(m, sl, kind=kind, chain_fn=chain)
    _, vm, _, vr, tau = grids(p.temp, lmats=16, lreal=64, ltau=64)
    ct, cw, civ = eval_chi_electrons(cm, sl, zeta, p.temp, True, p.cutoff, tau, vr, 0.05, 4, vm=vm)
    spec = spectra_all_sectors(om, 4)
    exact = {io: [] for io in range(1, 5)}
    for st in sl.states:
        nup, ndw = m.get_nup(st.sector), m.get_ndw(st.sector)
        for io in range(1, 5):
            op = lambda v, io=io: O.apply_diagop(4, nup, ndw, kind, io, v)
            exact[io].append(exact_channels(om, 4, nup, ndw, st.vec, st.e, op, spec))
    et, ew, eiv = eval_chi_electrons(exact, sl, zeta, p.temp, True, p.cutoff, tau, vr, 0.05, 4, vm=vm)
    assert np.abs(ct - et).max() < 1e-9 and np.abs(cw - ew).max() < 1e-8 and np.abs(civ - eiv).max() < 1e-8
    assert np.all(ct[np.arange(4), np.arange(4), 0] > 0)


def test_oc_driver_and_drude_weight():
    """build_oc + eval_oc_electrons (oracle J chains injected) against exact spectra; the Drude
    weight takes Ekin from lanc_energy."""
    from ed_lattice_b200.diag import lanc_energy
    from ed_lattice_b200.gf import build_oc, eval_oc_electrons
    from gf_reference import exact_channels, spectra_all_sectors
    H = _chain4(seed=9)  # disorder: no degenerate levels, so no zero-energy J poles
    m = E.Model(H, uloc=2.0, xmu=1.0, hfmode=False)
    om = O.Model(H, uloc=2.0, xmu=1.0, hfmode=False)
    p = DiagParams(finite_temp=True, temp=0.25, lanc_nstates_sector=36)
    sl, _ = diagonalize_lattice(m, p, solver=_oracle_solver(om))
    zeta = partition_function(sl, p)

    def chain(isector, vec, nlanc, ei):
        nup, ndw = m.get_nup(isector), m.get_ndw(isector)
        x = O.apply_current(om, nup, ndw, vec)
        st = O.Stored(om, nup, ndw)
        a, b, n2, n = st.tridiag(x, min(nlanc, st.dim), 1e-9)
        if n == 0 or n2 == 0.0:
            return E.Spectrum(np.zeros(0), np.zeros(0), n2)
        pp, ww = O.poles_weights(a[:n], b[:n], n2, ei, +1)
        return E.Spectrum(pp, ww, n2)

    ocm = build_oc(m, sl, chain_fn=chain)
    spec = spectra_all_sectors(om, 4)
    exact = []
    for st in sl.states:
        nup, ndw = m.get_nup(st.sector), m.get_ndw(st.sector)
        exact.append(exact_channels(om, 4, nup, ndw, st.vec, st.e, lambda v: O.apply_current(om, nup, ndw, v), spec))

    def energy_fn(model, isector, vec, bw):
        ek, ep, ekn, eh = O.energy(om, model.get_nup(isector), model.get_ndw(isector), vec, bw)
        return {"ekin": ek, "epot": ep, "eknot": ekn, "ehartree": eh}

    ekin = lanc_energy(m, sl, zeta, p, energy_fn=energy_fn)["ekin"]
    vr = np.linspace(0.0, 5.0, 51)
    dw, oc = eval_oc_electrons(ocm, sl, zeta, p.temp, True, 1e-6, vr, 0.1, ekin, 4)
    dw_ex, oc_ex = eval_oc_electrons(exact, sl, zeta, p.temp, True, 1e-6, vr, 0.1, ekin, 4)
    # plain Lanczos chains (no reorthogonalisation) split weight over ghost copies of a pole:
    # sums like D = sum w/dE agree with the exact spectra to ~1e-7 relative
    assert abs(dw - dw_ex) < 1e-6 * abs(dw_ex) and np.abs(oc - oc_ex).max() < 1e-6 * np.abs(oc_ex).max()
    assert ekin < 0.0


def test_sector_scheduler_admission():
    """SectorScheduler: a solve waits until its bytes fit, and one larger than the whole
    capacity is clamped so it runs alone instead of waiting for ever."""
    import threading

    from ed_lattice_b200.diag import SectorScheduler

    sch = SectorScheduler(100)
    a = sch.acquire(60)
    assert a == 60 and sch.free == 40
    got = []
    t = threading.Thread(target=lambda: got.append(sch.acquire(50)))
    t.start()
    t.join(0.2)
    assert t.is_alive() and not got  # 50 > 40 free: waits
    sch.release(a)
    t.join(5)
    assert got == [50] and sch.free == 50
    sch.release(50)
    assert sch.acquire(10**6) == 100 and sch.free == 0


def test_threaded_sector_solves_match_sequential_and_respect_capacity():
    """solve_sectors with 4 threads and the oracle's dense solver: the same eigenpairs as the
    sequential run, keyed by sector; solves start largest first; the byte estimates held at
    once never exceed the capacity; a failing sector raises after the others end."""
    import threading
    import time

    from ed_lattice_b200.diag import sector_device_bytes, solve_sectors

    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    p = DiagParams(finite_temp=True, temp=0.1, lanc_nstates_sector=4, lanc_dim_threshold=0)
    jobs = []
    for isector in range(1, 26):
        nup, ndw = m.get_nup(isector), m.get_ndw(isector)
        dim = math.comb(4, nup) * math.comb(4, ndw)
        jobs.append((isector, nup, ndw, min(4, dim), dim > 4))
    base = _oracle_solver(om)
    lock = threading.Lock()
    state = {"held": 0, "peak": 0, "starts": []}
    cap = 2 * max(sector_device_bytes(math.comb(4, j[1]) * math.comb(4, j[2]), j[3], j[4], p) for j in jobs)

    def solver(model, nup, ndw, neigen, lanc_solve, params, seed):
        b = sector_device_bytes(math.comb(4, nup) * math.comb(4, ndw), neigen, lanc_solve, params)
        with lock:
            state["held"] += b
            state["peak"] = max(state["peak"], state["held"])
            state["starts"].append(math.comb(4, nup) * math.comb(4, ndw))
        time.sleep(0.05)  # long enough that the four workers start their first jobs first
        try:
            return base(model, nup, ndw, neigen, lanc_solve, params, seed)
        finally:
            with lock:
                state["held"] -= b

    seq = solve_sectors(m, jobs, p, 1, solver=base)
    par = solve_sectors(m, jobs, p, 1, solver=solver, threads=4, capacity=cap)
    assert sorted(par) == sorted(seq) == [j[0] for j in jobs]
    for k in seq:
        assert np.array_equal(par[k][0], seq[k][0]) and np.array_equal(par[k][1], seq[k][1])
    assert state["peak"] <= cap
    state["starts"].clear()
    solve_sectors(m, jobs, p, 1, solver=solver, threads=4, capacity=1 << 40)
    assert sorted(state["starts"][:4]) == sorted(state["starts"])[-4:]  # largest dispatched first

    def failing(model, nup, ndw, neigen, lanc_solve, params, seed):
        if (nup, ndw) == (2, 2):
            raise RuntimeError("sector (2,2) failed")
        return base(model, nup, ndw, neigen, lanc_solve, params, seed)

    with pytest.raises(RuntimeError, match=r"\(2,2\)"):
        solve_sectors(m, jobs, p, 1, solver=failing, threads=4, capacity=cap)


def test_threaded_state_map_contexts_and_errors():
    """gf._map_states with 4 threads: every owned state once, one context per worker thread
    (never shared between threads at once), all contexts closed, and a failing state raised
    after the others end."""
    import threading
    import time

    from ed_lattice_b200.gf import _map_states

    sl = StateList()
    for i in range(20):
        sl.add_state(-1.0 - 0.01 * i, np.zeros(3), 1 + i % 5, size=100)
    made = []

    class Ctx:
        def __init__(self):
            self.thread = threading.get_ident()
            self.closed = False
            made.append(self)

        def close(self):
            self.closed = True

    def fn(istate, st, ctx):
        assert ctx.thread == threading.get_ident()
        time.sleep(0.002)
        return (istate, st.sector)

    out = _map_states(sl, None, "test", fn, 4, Ctx)
    assert out == {i: (i, sl.states[i - 1].sector) for i in range(1, 21)}
    assert 1 <= len(made) <= 4 and all(c.closed for c in made)

    def bad(istate, st, ctx):
        if istate == 7:
            raise ValueError("state 7")
        return istate

    made.clear()
    with pytest.raises(ValueError, match="state 7"):
        _map_states(sl, None, "test", bad, 4, Ctx)
    assert all(c.closed for c in made)
    assert _map_states(sl, None, "test", lambda i, st, c: i, 1) == {i: i for i in range(1, 21)}


def test_device_chain_cache_eviction(monkeypatch):
    """gf._DeviceChains keeps the `keep` most recently used sectors, deletes the others, and
    reloads a state whose source sector was evicted (fake sectors: no device needed)."""
    from ed_lattice_b200 import gf

    made, deleted, loads = [], [], []

    class FakeSector:
        def __init__(self, isector):
            self.isector = isector
            made.append(isector)

        @classmethod
        def from_index(cls, model, isector):
            return cls(isector)

        def delete(self):
            deleted.append(self.isector)

        def set_state(self, vec):
            loads.append(self.isector)

    monkeypatch.setattr(gf, "Sector", FakeSector)
    dc = gf._DeviceChains(model=None, precision=0, keep=3)
    for i in (1, 2, 3, 4):
        dc.sector(i)
    assert list(dc.sectors) == [2, 3, 4] and deleted == [1]
    v = np.zeros(2)
    dc.load(2, v)
    dc.load(2, v)  # same state: no reload
    assert loads == [2] and list(dc.sectors) == [3, 4, 2]
    dc.sector(5)
    dc.sector(6)
    assert deleted == [1, 3, 4] and list(dc.sectors) == [2, 5, 6]
    dc.sector(7)  # evicts 2, which held the loaded state
    assert deleted == [1, 3, 4, 2] and dc.loaded is None
    dc.load(2, v)
    assert loads == [2, 2] and made.count(2) == 2
    dc.close()
    assert sorted(deleted) == [1, 2, 2, 3, 4, 5, 6, 7] and not dc.sectors


def test_device_plan_shrinks_with_sector_size(monkeypatch):
    """gf._device_plan: small sectors keep 4 threads and 8 cached sectors; sectors whose work
    vectors would overrun half the free memory get fewer threads and a smaller cache."""
    import types

    from ed_lattice_b200 import gf

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(is_available=lambda: True,
                                                                  mem_get_info=lambda: (100 << 30, 180 << 30)))
    monkeypatch.setitem(__import__("sys").modules, "torch", fake_torch)
    small = E.Model(E.square_lattice(3, 4), uloc=4.0)
    sl = StateList()
    sl.add_state(-1.0, np.zeros(1), small.get_sector(6, 6), size=10)
    assert gf._device_plan(small, sl, 4) == (4, 8)
    big = E.Model(E.square_lattice(4, 4), uloc=4.0)  # neighbours of (8,8): D up to 165,636,900
    sl2 = StateList()
    sl2.add_state(-1.0, np.zeros(1), big.get_sector(8, 8), size=10)
    assert gf._device_plan(big, sl2, 4) == (1, 3)  # 3 sectors of 13.25 GB fit in 50 GB, 6 do not


def test_state_list_twin_pairs():
    """es_insert_state with twin=.true. puts a vectorless twin of the same energy right after
    the state; es_pop_state removes a twin pair together whichever of the two is hit, and a
    capped list drops the pair at its end (src/EIGENSPACE.f90:198-332)."""
    sl = StateList()
    v = np.arange(6.0)  # a (DimUp=3) x (DimDw=2) sector vector, element iup + idw*3
    sl.add_state(0.2, v, 7, twin=(9, (3, 2)))
    sl.add_state(-0.1, None, 1)
    sl.add_state(0.2, None, 4)
    assert [(s.sector, s.twin) for s in sl.states] == [(1, False), (4, False), (7, False), (9, True)]
    tw = sl.states[3]
    assert tw.e == 0.2 and tw.partner is sl.states[2]
    # twin vector: the transpose of the partner's matrix, element idw + iup*2
    assert np.array_equal(tw.vec, v.reshape(2, 3).T.ravel())
    assert np.array_equal(sl.vector(4), [0.0, 3.0, 1.0, 4.0, 2.0, 5.0])
    sl.pop_state()                      # the last entry is a twin: its partner goes too
    assert [s.sector for s in sl.states] == [1, 4]
    sl.add_state(0.5, v, 7, twin=(9, (3, 2)))
    sl.pop_state(3)                     # a state followed by its twin: both go
    assert [s.sector for s in sl.states] == [1, 4]
    sl.add_state(0.3, v, 7, twin=(9, (3, 2)), size=3)  # size 2 < 3: the pair goes in (size 4)
    assert sl.size == 4
    sl.add_state(0.0, None, 5, size=4)  # full: the pair at the end is dropped for the newcomer
    assert [s.sector for s in sl.states] == [1, 5, 4]


def test_twin_sectors_thermal_and_vectors():
    """ED_TWIN: only Nup >= Ndw is solved; Z and the observables equal the run that visits
    every sector, and each twin vector is an eigenvector of its own sector (spin flip)."""
    H = _chain4()
    m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    res = {}
    for twin in (False, True):
        p = DiagParams(finite_temp=True, temp=0.5, lanc_nstates_sector=36, ed_twin=twin)
        sl, eigs = diagonalize_lattice(m, p, solver=_oracle_solver(om))
        zeta = partition_function(sl, p)
        res[twin] = (sl, eigs, zeta, lanc_observables(m, sl, zeta, p, observer=_oracle_observer))
    sl, eigs, zeta, obs = res[True]
    assert len(eigs) == 15  # Nup >= Ndw of the 25 sectors
    assert all(m.get_nup(isec) >= m.get_ndw(isec) for isec, _, _ in eigs)
    assert zeta == pytest.approx(res[False][2], rel=1e-12)
    for k in obs:
        assert np.allclose(obs[k], res[False][3][k], atol=1e-12), k
    ntwin = 0
    for st in sl.states:
        if not st.twin:
            continue
        ntwin += 1
        nup, ndw = m.get_nup(st.sector), m.get_ndw(st.sector)
        hb = O.dense_h(om, nup, ndw)
        assert np.abs(hb @ st.vec - st.e * st.vec).max() <= 1e-10
    assert ntwin > 0
