"""Host-side logic of the package (no GPU): lattice input, grids, evaluation of poles on
frequency grids, GFmatrix restart I/O."""
import io
import math

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200.edlat import Spectrum


def test_square_lattice_bond_counts():
    # NN periodic bond counts quoted for the configs: 8 / 32 / 24 / 36
    for (lx, ly), nb in (((8, 1), 8), ((4, 4), 32), ((3, 4), 24), ((6, 3), 36)):
        H = E.square_lattice(lx, ly)
        assert np.count_nonzero(np.triu(H)) == nb
        assert np.allclose(H, H.T)


def test_hij_builder_and_read(tmp_path):
    b = E.Hij(4)
    for i in range(1, 5):
        j = i % 4 + 1
        b.add_link(i, j, 1, 1, 1, -1.0)
        b.add_link(j, i, 1, 1, 1, -1.0)
    H = b.build()
    assert np.allclose(H[0].real, E.ring(4))
    p = tmp_path / "hij.in"
    p.write_text("\n".join(f"{i} {j} 1 1 1 {v} 0.0" for (i, j, _, _, _, v) in
                           [(a, c, 1, 1, 1, -1.0) for a in range(1, 5) for c in (a % 4 + 1,)] +
                           [(c, a, 1, 1, 1, -1.0) for a in range(1, 5) for c in (a % 4 + 1,)]) + "\n")
    b2 = E.Hij(4)
    b2.read(str(p))
    assert np.allclose(b2.build(), H)
    with pytest.raises(ValueError):
        b.add_link(5, 1, 1, 1, 1, 1.0)
    bad = E.Hij(2)
    bad.add_link(1, 2, 1, 1, 1, 1.0)
    with pytest.raises(E.EdgError):
        bad.build()


def test_grids_match_allocate_grids():
    wm, vm, wr, vr, tau = E.grids(0.02, lmats=16, lreal=11, ltau=8, wini=-5, wfin=5)
    assert np.allclose(wm, math.pi * 0.02 * (2 * np.arange(1, 17) - 1))
    assert vm[0] == 0.0 and np.isclose(vm[3], 2 * math.pi * 0.02 * 3)
    assert np.allclose(wr, np.linspace(-5, 5, 11)) and np.allclose(vr, np.linspace(0, 5, 11))
    assert tau.size == 51  # Ltau = max(int(1/T), Ltau) = 50


def test_eval_gf_chi_oc_against_loops():
    rng = np.random.default_rng(0)
    ch = Spectrum(rng.normal(size=7), rng.uniform(0, 1, 7))
    wm = np.pi * 0.1 * (2 * np.arange(1, 9) - 1)
    wr = np.linspace(-3, 3, 13)
    gm, gr = E.eval_gf([ch], wm, wr, 0.05, pesoBZ=0.5)
    for i in range(wm.size):
        assert np.isclose(gm[i], sum(0.5 * w / (1j * wm[i] - p) for p, w in zip(ch.poles, ch.weight)))
    beta = 10.0
    tau = np.linspace(0, beta, 11)
    vr = np.linspace(0, 3, 7)
    pos = Spectrum(np.abs(ch.poles) + 0.1, ch.weight)
    ct, cw, civ = E.eval_chi([pos], beta, tau, vr, 0.05, vm=np.pi * 0.2 * np.arange(5))
    # symmetric about beta/2 by construction
    assert np.allclose(ct, ct[::-1])
    D, oc = E.eval_oc([pos], vr, 0.05)
    assert np.isclose(D, np.sum(pos.weight / pos.poles))
    assert np.isclose(E.drude_weight(D, -4.0, 16), -math.pi / 16 * (-4.0 + 2 * D))


def test_gfmatrix_restart_roundtrip():
    states = [[Spectrum(np.array([0.5, -1.25]), np.array([0.1, 0.2])), Spectrum(np.zeros(0), np.zeros(0))],
              [Spectrum(np.array([3.0]), np.array([1e-17]))]]
    f = io.StringIO()
    E.write_gfmatrix(f, states)
    E.write_gfmatrix(f, None)
    f.seek(0)
    back = E.read_gfmatrix(f)
    assert len(back) == 2 and len(back[0]) == 2
    assert np.array_equal(back[0][0].poles, states[0][0].poles)
    assert np.array_equal(back[1][0].weight, states[1][0].weight)
    assert back[0][1].poles.size == 0
    assert E.read_gfmatrix(f) is None


def test_read_input_file(tmp_path):
    """ed_read_input's key file: case-insensitive keys, comments, Fortran reals and logicals,
    per-orbital lists, defaults for absent keys, and the objects built from it."""
    from ed_lattice_b200.inputvars import DEFAULTS, diag_params, model_from_input, read_input, sector_form
    p = tmp_path / "inputED.conf"
    p.write_text("ULOC=4.d0          ! local interaction\n"
                 "xmu=2D0\n"
                 "HFMODE=F\n"
                 "ED_FINITE_TEMP=.true.\n"
                 "TEMP=0.05\n"
                 "LANC_NSTATES_SECTOR=4\n"
                 "LANC_TOLERANCE=1.d-18\n"
                 "ED_SPARSE_H=F\n"
                 "GF_FLAG=T\n"
                 "   \n"
                 "! a comment line\n"
                 "MY_KEY=something\n")
    cfg = read_input(str(p))
    assert cfg["ULOC"] == [4.0] and cfg["XMU"] == 2.0 and cfg["HFMODE"] is False
    assert cfg["ED_FINITE_TEMP"] is True and cfg["TEMP"] == 0.05 and cfg["GF_FLAG"] == [True]
    assert cfg["LMATS"] == DEFAULTS["LMATS"] and cfg["MY_KEY"] == "something"
    dp = diag_params(cfg)
    assert dp.finite_temp and dp.temp == 0.05 and dp.lanc_nstates_sector == 4 and dp.lanc_tolerance == 1e-12
    assert sector_form(cfg) == E.EDG_FORM_DIRECT
    m = model_from_input(cfg, E.ring(4))
    assert m.uloc == 4.0 and m.xmu == 2.0 and not m.hfmode
    bad = tmp_path / "bad.conf"
    bad.write_text("HFMODE=maybe\n")
    with pytest.raises(E.EdgError):
        read_input(str(bad))
