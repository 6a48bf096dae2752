"""Response functions over the state list: the build and evaluation loops of the GF, CHI
and OC modules.

    build_gf_electrons  build_gf_electrons + lanc_build_gf_electrons_diag/_mix
                        (src/GF/GF_ELECTRONS.f90:33-98,202-405)
    eval_gf_electrons   eval_gf_electrons + lanc_eval_gf_electrons
                        (src/GF/GF_ELECTRONS.f90:100-185,472-512)
    build_chi           build_chi_spin_electrons + lanc_build_spinChi_diag
                        (src/CHI/CHI_SPIN_ELECTRONS.f90:33-95,189-240); kind 1 = charge
    eval_chi_electrons  eval_chi_spin_electrons + lanc_eval_spinChi_electrons (:97-188,380-468)
    build_oc            build_oc_electrons + lanc_ed_build_oc (src/OC/OC_ELECTRONS.f90:36-214)
    eval_oc_electrons   lanc_ed_eval_oc + eval_oc_lattice's Drude weight
                        (src/OC/OC_ELECTRONS.f90:270-319, src/OC/OC_FUNCTIONS.f90:50-70)

GF: for every state of the list, site (pair) and spin, one particle chain (c^+ into the
sector with one more electron of that spin) and one hole chain (c into the sector with one
less) run on the device through edg_gf_chain; a sector without such a neighbour gives an
empty channel (Nexc=0). CHI and OC: one same-sector chain per state (and site) on
O|state>. Weights and poles are those of the add_to_lanczos_* routines. Chains of a state
run on the rank that holds its vector; the spectra are all-gathered.

On the device, the states of a rank are shared out among host threads (`threads`, default
4): each thread keeps its own sectors (a bounded cache) and runs all the chains of one state
at a time on them, so chains of different states overlap on the GPU. Results are keyed by
state, so they do not depend on which thread ran what.
"""
from __future__ import annotations

import threading
from collections import OrderedDict
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _edgpu_lib as L
from .diag import StateList, _allgather, _rank_world
from .edlat import (Model, Sector, Spectrum, chi_chain, chi_chain_block, drude_weight, eval_chi, eval_oc, eval_poles,
                    gf_chain, gf_chain_block, oc_chain)

LANC_NGFITER = 200  # LANC_NGFITER default (src/INPUT_VARS.f90:161)
STATE_THREADS = 4   # host threads that run the chains of different states at once
BLOCK_WIDTH = 16    # chains of one state and target sector run as blocks of at most this many


def get_cdg_sector(model: Model, ispin: int, isector: int) -> int:
    """getCDGsector(1,ispin,isector): the sector with one more electron of spin ispin, 0 if none."""
    nup, ndw = model.get_nup(isector), model.get_ndw(isector)
    nup, ndw = (nup + 1, ndw) if ispin == 1 else (nup, ndw + 1)
    return model.get_sector(nup, ndw) if nup <= model.ns and ndw <= model.ns else 0


def get_c_sector(model: Model, ispin: int, isector: int) -> int:
    """getCsector(1,ispin,isector): the sector with one less electron of spin ispin, 0 if none."""
    nup, ndw = model.get_nup(isector), model.get_ndw(isector)
    nup, ndw = (nup - 1, ndw) if ispin == 1 else (nup, ndw - 1)
    return model.get_sector(nup, ndw) if nup >= 0 and ndw >= 0 else 0


class _DeviceChains:
    """Default chain runner of one thread: the sectors it has used, built once and kept (the
    `keep` most recently used), and the state loaded into its source sector."""

    def __init__(self, model: Model, precision: int, keep: int = 8):
        self.model, self.precision, self.keep = model, precision, max(keep, 2)
        self.sectors: OrderedDict[int, Sector] = OrderedDict()
        self.loaded = None  # (isector, vec) whose vector the source sector holds

    def sector(self, isector: int) -> Sector:
        s = self.sectors.get(isector)
        if s is None:
            s = self.sectors[isector] = Sector.from_index(self.model, isector)
            while len(self.sectors) > self.keep:
                old, sec = self.sectors.popitem(last=False)
                sec.delete()
                if self.loaded is not None and self.loaded[0] == old:
                    self.loaded = None
        else:
            self.sectors.move_to_end(isector)
        return s

    def load(self, isector: int, vec) -> Sector:
        src = self.sector(isector)
        if self.loaded is None or self.loaded[0] != isector or self.loaded[1] is not vec:
            src.set_state(vec)
            self.loaded = (isector, vec)
        return src

    def __call__(self, isector, vec, jsector, op, io, jo, ispin, nlanc, ei) -> Spectrum:
        src = self.load(isector, vec)
        dst = self.sector(jsector)
        return gf_chain(src, dst, op, io, ispin, min(nlanc, dst.dim), ei, site2=jo, precision=self.precision)

    def gf_block(self, isector, vec, jsector, op, ios, jos, ispin, nlanc, ei) -> list:
        """The chains (ios[c], jos[c]) of one state into jsector as blocks of BLOCK_WIDTH
        (block H x V); the same spectra as one __call__ per chain."""
        src = self.load(isector, vec)
        dst = self.sector(jsector)
        out = []
        for c0 in range(0, len(ios), BLOCK_WIDTH):
            out += gf_chain_block(src, dst, op, ios[c0:c0 + BLOCK_WIDTH], ispin, min(nlanc, dst.dim), ei,
                                  sites2=jos[c0:c0 + BLOCK_WIDTH], precision=self.precision)
        return out

    def chi_block(self, isector, vec, sites, kind, nlanc, ei) -> list:
        sec = self.load(isector, vec)
        out = []
        for c0 in range(0, len(sites), BLOCK_WIDTH):
            out += chi_chain_block(sec, min(nlanc, sec.dim), ei, kind=kind, sites=sites[c0:c0 + BLOCK_WIDTH],
                                   precision=self.precision)
        return out

    def close(self):
        for s in self.sectors.values():
            s.delete()
        self.sectors.clear()


def _device_plan(model: Model, state_list: StateList, threads: int) -> tuple[int, int]:
    """(threads, sectors cached per thread) for the device builders: each thread keeps at most
    `keep` sectors of about ten work vectors each, sized by the largest sector a state of the
    list or a neighbour of it (one electron more or less) can have; thread count and cache
    shrink until that fits in half of the free HBM."""
    import math

    ns = model.ns
    dmax = 1
    for st in state_list.states:
        nup, ndw = model.get_nup(st.sector), model.get_ndw(st.sector)
        for du, dd in ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)):
            a, b = nup + du, ndw + dd
            if 0 <= a <= ns and 0 <= b <= ns:
                dmax = max(dmax, math.comb(ns, a) * math.comb(ns, b))
    cplx = bool(np.iscomplexobj(model.hij) and np.any(np.imag(model.hij) != 0))
    per_sector = 10 * dmax * (16 if cplx else 8)
    try:
        import torch

        free = torch.cuda.mem_get_info()[0] if torch.cuda.is_available() else 1 << 62
    except Exception:
        free = 1 << 62
    keep = 8
    while keep > 3 and threads * keep * per_sector > free // 2:
        keep -= 1
    while threads > 1 and threads * keep * per_sector > free // 2:
        threads -= 1
    return threads, keep


def _map_states(state_list: StateList, comm, what: str, fn, threads: int, make_ctx=None) -> dict:
    """{istate: fn(istate, state, ctx)} over the states this rank owns. With threads > 1 the
    states are shared out among that many host threads, each with its own ctx = make_ctx()
    (closed at the end); the first failure in state order is raised once all have ended."""
    rank, _ = _rank_world(comm)
    todo = []
    for istate in range(1, state_list.size + 1):
        st = state_list.states[istate - 1]
        if st.owner != rank:
            continue
        if st.vec is None:
            raise L.EdgError(L.EDG_ERR_STATE, what, "state list holds no vectors")
        todo.append((istate, st))
    ctxs = []
    lock = threading.Lock()
    local = threading.local()

    def context():
        c = getattr(local, "ctx", None)
        if c is None and make_ctx is not None:
            c = local.ctx = make_ctx()
            with lock:
                ctxs.append(c)
        return c

    try:
        if threads <= 1 or len(todo) <= 1:
            return {istate: fn(istate, st, context()) for istate, st in todo}
        import torch

        dev = torch.cuda.current_device() if torch.cuda.is_available() else None

        def work(item):
            if dev is not None:
                torch.cuda.set_device(dev)
            return fn(item[0], item[1], context())

        with ThreadPoolExecutor(max_workers=threads) as ex:
            futs = [ex.submit(work, item) for item in todo]
        return {item[0]: f.result() for item, f in zip(todo, futs)}
    finally:
        for c in ctxs:
            c.close()


def build_gf_electrons(model: Model, state_list: StateList, nlanc: int = LANC_NGFITER, offdiag: bool = False,
                       precision: int = L.EDG_PREC_F64, chain_fn=None, comm=None, threads: int | None = None) -> dict:
    """impGmatrix: {(ispin, io, jo): [[particle, hole] per state]} with 1-based sites, for
    io == jo (the diagonal) and, with `offdiag`, every ordered pair io != jo built from
    (c_io + c_jo) chains. `chain_fn(isector, vec, jsector, op, io, jo, ispin, nlanc, ei)`
    returns one channel (jo = 0 for a single site); the default runs on the device, on
    `threads` host threads (default STATE_THREADS; 1 for a caller-supplied chain_fn)."""
    if threads is None:
        threads = 1 if chain_fn else STATE_THREADS
    ns = model.ns
    pairs = [(io, io) for io in range(1, ns + 1)]
    if offdiag:
        pairs += [(io, jo) for io in range(1, ns + 1) for jo in range(1, ns + 1) if io != jo]

    def run(istate, st, dev):
        runner = chain_fn or dev
        out = {}
        for ispin in range(1, model.nspin + 1):
            jp, jh = get_cdg_sector(model, ispin, st.sector), get_c_sector(model, ispin, st.sector)
            if not chain_fn:  # the device runs the chains of each target sector as blocks
                ios = [io for io, _ in pairs]
                jos = [0 if io == jo else jo for io, jo in pairs]
                per_op = []
                for jsec, op in ((jp, +1), (jh, -1)):
                    if jsec == 0:
                        per_op.append([Spectrum(np.zeros(0), np.zeros(0), 0.0)] * len(pairs))
                    else:
                        per_op.append(dev.gf_block(st.sector, st.vec, jsec, op, ios, jos, ispin, nlanc, st.e))
                for c, (io, jo) in enumerate(pairs):
                    out[(ispin, io, jo)] = [per_op[0][c], per_op[1][c]]
                continue
            for io, jo in pairs:
                chans = []
                for jsec, op in ((jp, +1), (jh, -1)):
                    if jsec == 0:
                        chans.append(Spectrum(np.zeros(0), np.zeros(0), 0.0))
                    else:
                        chans.append(runner(st.sector, st.vec, jsec, op, io, 0 if io == jo else jo, ispin,
                                            nlanc, st.e))
                out[(ispin, io, jo)] = chans
        return out

    keep = 8
    if not chain_fn:
        threads, keep = _device_plan(model, state_list, threads)
    per = _map_states(state_list, comm, "build_gf_electrons", run, threads,
                      None if chain_fn else (lambda: _DeviceChains(model, precision, keep)))
    mine = {(ispin, io, jo, istate): chans for istate, res in per.items() for (ispin, io, jo), chans in res.items()}
    gm: dict = {}
    for part in _allgather(mine, comm):
        for (ispin, io, jo, istate), chans in part.items():
            gm.setdefault((ispin, io, jo), [None] * state_list.size)[istate - 1] = chans
    return gm


def eval_gf_electrons(gmatrix: dict, state_list: StateList, zeta: float, temp: float, finite_temp: bool,
                      cutoff: float, wm: np.ndarray, wr: np.ndarray, eps: float, nspin: int, ns: int,
                      backend: str = "device"):
    """impGmats[nspin, ns, ns, Lmats] and impGreal[nspin, ns, ns, Lreal] (0-based site axes):
    lanc_eval_gf_electrons' sum over the trimmed list with pesoBZ = exp(-(Ei-Egs)/T)/Z (1/Z
    at T=0), then G_ij = (G~_ij - G_ii - G_jj)/2 for the off-diagonal pairs (:168-176).
    backend "device": every pole of an entry in one edg_eval_poles call per axis; "host": numpy."""
    if backend not in ("device", "host"):
        raise L.EdgError(L.EDG_ERR_ARG, "eval_gf_electrons", f"backend={backend!r}")
    gmats = np.zeros((nspin, ns, ns, wm.size), dtype=np.complex128)
    greal = np.zeros((nspin, ns, ns, wr.size), dtype=np.complex128)
    egs = state_list.emin
    n = state_list.trim_size(temp, cutoff, finite_temp)
    zm, zr = 1j * wm, wr + 1j * eps
    for (ispin, io, jo), states in gmatrix.items():
        ps, ws = [], []
        for istate in range(1, n + 1):
            chans = states[istate - 1]
            if chans is None:
                continue
            ei = state_list.energy(istate)
            peso_bz = (np.exp(-(ei - egs) / temp) if finite_temp else 1.0) / zeta
            for ch in chans:
                if ch.poles.size:
                    ps.append(ch.poles)
                    ws.append(peso_bz * ch.weight)
        if not ps:
            continue
        p, w = np.concatenate(ps), np.concatenate(ws)
        if backend == "device":
            gmats[ispin - 1, io - 1, jo - 1] = eval_poles(p, w, zm)
            greal[ispin - 1, io - 1, jo - 1] = eval_poles(p, w, zr)
        else:
            for lo in range(0, p.size, 512):
                pp, ww = p[lo:lo + 512], w[lo:lo + 512]
                gmats[ispin - 1, io - 1, jo - 1] += (ww[None, :] / (zm[:, None] - pp[None, :])).sum(1)
                greal[ispin - 1, io - 1, jo - 1] += (ww[None, :] / (zr[:, None] - pp[None, :])).sum(1)
    for (ispin, io, jo) in gmatrix:
        if io == jo:
            continue
        s, i, j = ispin - 1, io - 1, jo - 1
        gmats[s, i, j] = 0.5 * (gmats[s, i, j] - gmats[s, i, i] - gmats[s, j, j])
        greal[s, i, j] = 0.5 * (greal[s, i, j] - greal[s, i, i] - greal[s, j, j])
    return gmats, greal


def _per_state(state_list: StateList, comm, what: str, fn, threads: int = 1, make_ctx=None) -> list:
    """fn(istate, state, ctx) on the rank that owns each state (see _map_states); results
    gathered in list order."""
    mine = _map_states(state_list, comm, what, fn, threads, make_ctx)
    out = [None] * state_list.size
    for part in _allgather(mine, comm):
        for istate, res in part.items():
            out[istate - 1] = res
    return out


def build_chi(model: Model, state_list: StateList, kind: int = 0, nlanc: int = LANC_NGFITER,
              precision: int = L.EDG_PREC_F64, chain_fn=None, comm=None, threads: int | None = None) -> dict:
    """SpinChiMatrix (kind 0: S^z_i) or the charge analogue (kind 1: n_i): {io: [[chain] per
    state]} for every site (1-based), a same-sector chain on O_io|state> per state. Norb=1
    has no mixed spin-chi (the reference builds those only for Norb > 1).
    `chain_fn(isector, vec, io, nlanc, ei)` returns one channel; the default runs on the device
    on `threads` host threads (default STATE_THREADS)."""
    if threads is None:
        threads = 1 if chain_fn else STATE_THREADS

    def run(istate, st, dev):
        if not chain_fn:  # one block of chains over the sites
            sites = list(range(1, model.ns + 1))
            return {io: [ch] for io, ch in zip(sites, dev.chi_block(st.sector, st.vec, sites, kind, nlanc, st.e))}
        return {io: [chain_fn(st.sector, st.vec, io, nlanc, st.e)] for io in range(1, model.ns + 1)}

    keep = 8
    if not chain_fn:
        threads, keep = _device_plan(model, state_list, threads)
    per = _per_state(state_list, comm, "build_chi", run, threads,
                     None if chain_fn else (lambda: _DeviceChains(model, precision, keep)))
    return {io: [per[k][io] for k in range(state_list.size)] for io in range(1, model.ns + 1)}


def _peso_bz(state_list: StateList, istate: int, zeta: float, temp: float, finite_temp: bool) -> float:
    ei, egs = state_list.energy(istate), state_list.emin
    return (np.exp(-(ei - egs) / temp) if finite_temp else 1.0) / zeta


def eval_chi_electrons(chimatrix: dict, state_list: StateList, zeta: float, temp: float, finite_temp: bool,
                       cutoff: float, tau: np.ndarray, vr: np.ndarray, eps: float, ns: int, vm=None):
    """spinChi_tau[ns, ns, Ltau+1], spinChi_w[ns, ns, Lreal] (and spinChi_iv when vm is given,
    the formula the reference keeps commented out) summed over the trimmed list with pesoBZ
    as in lanc_eval_spinChi_electrons; beta = 1/temp (temp is the IR cut-off at T=0)."""
    beta = 1.0 / temp
    ct = np.zeros((ns, ns, tau.size))
    cw = np.zeros((ns, ns, vr.size), dtype=np.complex128)
    civ = np.zeros((ns, ns, vm.size), dtype=np.complex128) if vm is not None else None
    n = state_list.trim_size(temp, cutoff, finite_temp)
    for io, states in chimatrix.items():
        for istate in range(1, n + 1):
            chans = states[istate - 1]
            if not chans:
                continue
            t, w, v = eval_chi(chans, beta, tau, vr, eps, vm=vm,
                               pesoBZ=_peso_bz(state_list, istate, zeta, temp, finite_temp))
            ct[io - 1, io - 1] += t
            cw[io - 1, io - 1] += w
            if civ is not None:
                civ[io - 1, io - 1] += v
    return ct, cw, civ


def build_oc(model: Model, state_list: StateList, nlanc: int = LANC_NGFITER, precision: int = L.EDG_PREC_F64,
             chain_fn=None, comm=None, threads: int | None = None) -> list:
    """OcMatrix: [[chain] per state], the chain of the current J (hop i+1 -> i minus h.c.
    along the ring of sites) on each state, in its own sector. `chain_fn(isector, vec, nlanc,
    ei)` returns one channel; the default runs on the device on `threads` host threads
    (default STATE_THREADS)."""
    if threads is None:
        threads = 1 if chain_fn else STATE_THREADS

    def run(istate, st, dev):
        if chain_fn:
            return [chain_fn(st.sector, st.vec, nlanc, st.e)]
        sec = dev.load(st.sector, st.vec)
        return [oc_chain(sec, min(nlanc, sec.dim), st.e, precision=precision)]

    keep = 8
    if not chain_fn:
        threads, keep = _device_plan(model, state_list, threads)
    return _per_state(state_list, comm, "build_oc", run, threads,
                      None if chain_fn else (lambda: _DeviceChains(model, precision, keep)))


def eval_oc_electrons(ocmatrix: list, state_list: StateList, zeta: float, temp: float, finite_temp: bool,
                      cutoff: float, vr: np.ndarray, eps: float, ekin: float, nsites: int):
    """(Drude weight, OptCond_w[Lreal]): lanc_ed_eval_oc's sums over the trimmed list with
    pesoBZ, then Drude_weight = -pi/Nsites (Ekin + 2 D) (src/OC/OC_FUNCTIONS.f90:65) with
    Ekin from lanc_energy."""
    d_tot = 0.0
    oc = np.zeros(vr.size)
    n = state_list.trim_size(temp, cutoff, finite_temp)
    for istate in range(1, n + 1):
        chans = ocmatrix[istate - 1]
        if not chans:
            continue
        d, o = eval_oc(chans, vr, eps, cutoff=cutoff, pesoBZ=_peso_bz(state_list, istate, zeta, temp, finite_temp))
        d_tot += d
        oc += o
    return drude_weight(d_tot, ekin, nsites), oc

