"""The state-list drivers on the device: diagonalize_lattice, then the GF, CHI and OC builders
and lanc_energy with their default device chains, against brute-force Lehmann sums and exact
spectra from the oracle's dense matrices (disordered 4-site chain, all 25 sectors, finite T)."""
import math

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200.diag import DiagParams, diagonalize_lattice, lanc_energy, lanc_observables, partition_function
from ed_lattice_b200.edlat import grids
from ed_lattice_b200.gf import (build_chi, build_gf_electrons, build_oc, eval_chi_electrons, eval_gf_electrons,
                                eval_oc_electrons)
from gf_reference import exact_channels, lehmann_g, spectra_all_sectors
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    rng = np.random.default_rng(5)
    H = E.ring(4).astype(float)
    H[np.diag_indices(4)] = np.round(rng.uniform(-1, 1, 4) * 2**16) / 2**16
    m = E.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    om = O.Model(H, uloc=3.0, xmu=1.5, hfmode=False)
    p = DiagParams(finite_temp=True, temp=0.3, lanc_nstates_sector=36, lanc_dim_threshold=8)
    sl, eigs = diagonalize_lattice(m, p, seed=11)
    zeta = partition_function(sl, p)
    return m, om, p, sl, zeta, spectra_all_sectors(om, 4)


def test_state_list_levels(setup):
    m, om, p, sl, zeta, spec = setup
    for st in sl.states[: sl.trimd_size]:
        w, _ = spec[(m.get_nup(st.sector), m.get_ndw(st.sector))]
        assert np.min(np.abs(w - st.e)) < 1e-10


def test_gf_driver_device(setup):
    m, om, p, sl, zeta, spec = setup
    gm = build_gf_electrons(m, sl, offdiag=True)
    wm = np.pi * p.temp * (2 * np.arange(1, 33) - 1)
    wr = np.linspace(-4, 4, 41)
    gmats, greal = eval_gf_electrons(gm, sl, zeta, p.temp, True, p.cutoff, wm, wr, 0.1, 1, 4)
    hm, hr = eval_gf_electrons(gm, sl, zeta, p.temp, True, p.cutoff, wm, wr, 0.1, 1, 4, backend="host")
    assert np.abs(gmats - hm).max() < 1e-12 and np.abs(greal - hr).max() < 1e-10  # device pole sums
    pairs = [(1, 1), (3, 3), (1, 2), (2, 4)]
    ref = lehmann_g(om, 4, p.temp, p.cutoff, True, pairs, 1j * wm, spec=spec)
    for (i, j) in pairs:
        assert np.abs(gmats[0, i - 1, j - 1] - ref[(i, j)]).max() < 1e-8, (i, j)


def test_chi_oc_energy_device(setup):
    m, om, p, sl, zeta, spec = setup
    _, vm, _, vr, tau = grids(p.temp, lmats=16, lreal=64, ltau=64)
    cm = build_chi(m, sl, kind=0)
    exact = {io: [] for io in range(1, 5)}
    ocx = []
    for st in sl.states:
        nup, ndw = m.get_nup(st.sector), m.get_ndw(st.sector)
        for io in range(1, 5):
            exact[io].append(exact_channels(om, 4, nup, ndw, st.vec, st.e,
                                            lambda v, io=io: O.apply_diagop(4, nup, ndw, 0, io, v), spec))
        ocx.append(exact_channels(om, 4, nup, ndw, st.vec, st.e, lambda v: O.apply_current(om, nup, ndw, v), spec))
    ct, cw, _ = eval_chi_electrons(cm, sl, zeta, p.temp, True, p.cutoff, tau, vr, 0.05, 4)
    et, ew, _ = eval_chi_electrons(exact, sl, zeta, p.temp, True, p.cutoff, tau, vr, 0.05, 4)
    assert np.abs(ct - et).max() < 1e-8 and np.abs(cw - ew).max() < 1e-7
    en = lanc_energy(m, sl, zeta, p)

    def energy_fn(model, isector, vec, bw):
        ek, ep, ekn, eh = O.energy(om, model.get_nup(isector), model.get_ndw(isector), vec, bw)
        return {"ekin": ek, "epot": ep, "eknot": ekn, "ehartree": eh}

    en_ref = lanc_energy(m, sl, zeta, p, energy_fn=energy_fn)
    for k in en:
        assert abs(en[k] - en_ref[k]) < 1e-11 * max(1.0, abs(en_ref[k])), k
    obs = lanc_observables(m, sl, zeta, p)
    h_avg = sum(math.exp(-(sl.energy(i) - sl.emin) / p.temp) * sl.energy(i) for i in range(1, sl.trimd_size + 1)) / zeta
    assert abs(en["ekin"] + en["epot"] + en["eknot"] - 1.5 * obs["dens"].sum() - h_avg) < 1e-10
    ocm = build_oc(m, sl)
    vr2 = np.linspace(0.0, 5.0, 51)
    dw, oc = eval_oc_electrons(ocm, sl, zeta, p.temp, True, 1e-6, vr2, 0.1, en["ekin"], 4)
    dw_ex, oc_ex = eval_oc_electrons(ocx, sl, zeta, p.temp, True, 1e-6, vr2, 0.1, en["ekin"], 4)
    assert abs(dw - dw_ex) < 1e-6 * abs(dw_ex) and np.abs(oc - oc_ex).max() < 1e-6 * np.abs(oc_ex).max()
