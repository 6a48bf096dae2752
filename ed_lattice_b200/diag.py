"""Sector diagonalisation and the finite-temperature state list.

    StateList            sparse_espace and its es_* routines (src/EIGENSPACE.f90:94-512)
    DiagParams           the keys that steer ed_diag_d (src/INPUT_VARS.f90:120-163) and the
                         state-count setup (src/SETUP.f90:89-117,248-251)
    diagonalize_lattice  ed_diag_d (src/DIAG/DIAG.f90:103-332)
    partition_function   partition_function_lattice (src/DIAG/DIAG.f90:52-92)
    lanc_observables     lanc_observables (src/OBSERVABLES.f90:78-192)
    lanc_energy          lanc_energy (src/ENERGY.f90:76-356), Norb=1 terms

The eigenpairs of each sector come from the device: edg_lowest_k for the sp_eigh (ARPACK)
branch, edg_ground_state for lanc_method="lanczos", and for dim <= lanc_dim_threshold the dense
sector matrix of edg_sector_dense_dev handed to the device dense eigensolver (the LAPACK
branch). With ed_twin (DiagParams.ed_twin) only the sectors with Nup >= Ndw are solved; each
state of a sector with Nup != Ndw enters the list with a vectorless twin in (Ndw, Nup),
whose vector is the transpose of its partner's DimDw x DimUp matrix (twin_sector_order,
src/SECTOR.f90:507-554).

Sectors are independent, so the device solves several at once: a pool of host threads takes
them largest first, each on its own library stream, and a sector starts only when the HBM
it needs is free (SectorScheduler). Small sectors are bound by launch and synchronisation
latency, which overlaps across threads. The state list is assembled in sector order
afterwards, so the result does not depend on the order in which sectors finish.
"""
from __future__ import annotations

import bisect
import math
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _edgpu_lib as L
from .edlat import Model, Sector, sp_lanc_eigh


# ----------------------------------------------------------------------------- state list
class EState:
    """One entry of the state list (sparse_estate, src/EIGENSPACE.f90:16-25). A twin entry
    (itwin) carries no vector of its own: its vector is the spin-flipped copy of its partner's,
    the transpose of the partner's DimDw x DimUp matrix without any sign (es_return_cvector,
    src/EIGENSPACE.f90:490-510, with twin_sector_order / flip_state, src/SECTOR.f90:507-554),
    built on first use and kept."""

    __slots__ = ("e", "_vec", "sector", "owner", "twin", "partner", "shape")

    def __init__(self, e: float, vec, sector: int, owner: int = 0, twin: bool = False, partner=None,
                 shape: tuple[int, int] | None = None):
        self.e, self._vec, self.sector, self.owner = e, vec, sector, owner
        self.twin, self.partner, self.shape = twin, partner, shape  # shape: the partner's (DimUp, DimDw)

    @property
    def vec(self):
        if self.twin and self._vec is None and self.partner is not None:
            pv = self.partner.vec
            if pv is None:
                return None
            dup, ddw = self.shape
            self._vec = np.ascontiguousarray(np.asarray(pv).reshape(ddw, dup).T).ravel()
        return self._vec

    @vec.setter
    def vec(self, v):
        self._vec = v


class StateList:
    """Energy-ordered list of (E, vector, sector) (sparse_espace, src/EIGENSPACE.f90:94-104).

    emin/emax are running extremes of every inserted energy: es_insert_state updates them and
    es_pop_state does not (src/EIGENSPACE.f90:216-217,260-332), which ed_diag_d's cutoff check
    relies on. Positions are 1-based like es_return_energy(space, n)."""

    def __init__(self):
        self.states: list[EState] = []
        self._energies: list[float] = []
        self.emin = math.inf
        self.emax = -math.inf
        self.trimd_size = 0

    @property
    def size(self) -> int:
        return len(self.states)

    def insert_state(self, e: float, vec, sector: int, owner: int = 0, twin=None) -> None:
        """es_insert_state (src/EIGENSPACE.f90:198-247): before the first entry with e <= E.
        twin = (twin sector, (DimUp, DimDw) of `sector`) also inserts, right after it, the
        vectorless twin entry of the same energy."""
        pos = bisect.bisect_left(self._energies, e)
        st = EState(float(e), vec, sector, owner)
        self.states.insert(pos, st)
        self._energies.insert(pos, float(e))
        if twin is not None:
            self.states.insert(pos + 1, EState(float(e), None, twin[0], owner, True, st, twin[1]))
            self._energies.insert(pos + 1, float(e))
        self.emax = max(self.emax, e)
        self.emin = min(self.emin, e)

    def add_state(self, e: float, vec, sector: int, size: int | None = None, owner: int = 0, twin=None) -> None:
        """es_add_state (src/EIGENSPACE.f90:167-190): with `size`, a full list takes a new state
        only if it lies below the last one, which is dropped (with its twin)."""
        if size is None or self.size < size:
            self.insert_state(e, vec, sector, owner, twin)
        elif e < self.energy():
            self.pop_state()
            self.insert_state(e, vec, sector, owner, twin)

    def pop_state(self, n: int | None = None) -> None:
        """es_pop_state: remove the n-th (default last) state (src/EIGENSPACE.f90:260-332); a
        twin pair goes together: a twin entry takes its partner (the entry before it) along,
        and an entry followed by its twin takes the twin along."""
        if self.size == 0:
            raise L.EdgError(L.EDG_ERR_STATE, "es_pop_state", "empty list")
        pos = self.size if n is None else n
        if pos > self.size:
            raise L.EdgError(L.EDG_ERR_ARG, "es_pop_state", "pos > espace.size")
        i = pos - 1
        if self.states[i].twin:
            lo, hi = i - 1, i + 1
        elif i + 1 < self.size and self.states[i + 1].twin:
            lo, hi = i, i + 2
        else:
            lo, hi = i, i + 1
        del self.states[lo:hi]
        del self._energies[lo:hi]

    def free(self) -> None:
        """es_free_espace (src/EIGENSPACE.f90:136-153)."""
        self.states.clear()
        self._energies.clear()
        self.emin = math.inf
        self.emax = -math.inf

    def energy(self, n: int | None = None) -> float:
        """es_return_energy (src/EIGENSPACE.f90:407-430): emax for an empty list."""
        pos = self.size if n is None else n
        if pos > self.size:
            raise L.EdgError(L.EDG_ERR_ARG, "es_return_energy", "n > espace.size")
        if self.size == 0:
            return self.emax
        return self.states[pos - 1].e

    def sector(self, n: int) -> int:
        return self.states[n - 1].sector

    def vector(self, n: int):
        return self.states[n - 1].vec

    def trim_size(self, temp: float, cutoff: float, finite_temp: bool) -> int:
        """es_trim_size (src/EIGENSPACE.f90:440-471): the leading states with Boltzmann factor
        exp(-(E-Emin)/T) above the cutoff."""
        self.trimd_size = self.size
        if not finite_temp:
            return self.trimd_size
        egs = self.emin
        pos = 0
        for st in self.states:
            if math.exp(-(st.e - egs) / temp) <= cutoff:
                break
            pos += 1
        self.trimd_size = pos
        if pos == 0:
            raise L.EdgError(L.EDG_ERR_STATE, "es_trim_size", "list does not contain any node")
        return pos

    def gs_degeneracy(self, gs_threshold: float = 1e-9) -> int:
        """es_return_gs_degeneracy (src/EIGENSPACE.f90:342-369)."""
        oldzero = 1000.0
        numzero = 0
        for st in self.states:
            if st.e < oldzero - 10.0 * gs_threshold:
                numzero = 1
                oldzero = st.e
            elif abs(st.e - oldzero) <= gs_threshold:
                numzero += 1
                oldzero = min(oldzero, st.e)
        return numzero


# ----------------------------------------------------------------------------- parameters
@dataclass
class DiagParams:
    """Input keys of the diagonalisation step (src/INPUT_VARS.f90:120-163), with the reference's
    defaults except LANC_TOLERANCE: the reference passes 1e-18 to ARPACK, i.e. "to machine
    precision"; here it is the residual bound b|z| <= tol*max(1,|E|) of edg_lowest_k (and the
    relative E0 error bound of edg_ground_state), so 1e-10 gives eigenvalues to ~1e-20 and
    vectors to ~1e-10 relative to the gap."""
    finite_temp: bool = False        # ED_FINITE_TEMP
    temp: float = 0.001              # TEMP
    cutoff: float = 1e-9             # CUTOFF
    gs_threshold: float = 1e-9       # GS_THRESHOLD
    lanc_method: str = "arpack"      # LANC_METHOD: "arpack" (lowest k) or "lanczos" (one state)
    lanc_nstates_sector: int = 2     # LANC_NSTATES_SECTOR
    lanc_niter: int = 512            # LANC_NITER: Lanczos basis size here
    lanc_tolerance: float = 1e-10    # LANC_TOLERANCE
    lanc_dim_threshold: int = 1024   # LANC_DIM_THRESHOLD
    lanc_nstates_total: int = 1      # set by setup()
    ed_twin: bool = False            # ED_TWIN: solve Nup >= Ndw only, twins by spin flip
    lanc_fp32_bulk: bool = False     # lowest-k sectors: FP32 bulk + FP64 refinement (no reference key)
    sector_threads: int = 8          # sectors solved at once on one device (no reference key)

    def setup(self, nsectors: int) -> "DiagParams":
        """State counts of the Lanczos method (src/SETUP.f90:89-104): at finite T an even
        lanc_nstates_sector and lanc_nstates_total = lanc_nstates_sector*Nsectors+10 (even);
        at T=0 the list holds the ground-state manifold only."""
        if self.lanc_method not in ("arpack", "lanczos"):
            raise L.EdgError(L.EDG_ERR_ARG, "DiagParams", f"lanc_method={self.lanc_method!r}")
        if self.finite_temp:
            if self.lanc_nstates_sector % 2:
                self.lanc_nstates_sector += 1
            self.lanc_nstates_total = self.lanc_nstates_sector * nsectors + 10
            if self.lanc_nstates_total % 2:
                self.lanc_nstates_total += 1
        return self


# ----------------------------------------------------------------------------- sector solvers
def _dense_lowest(sec: Sector, neigen: int):
    """LAPACK branch of ed_diag_d (src/DIAG/DIAG.f90:229-254): dense matrix built on the
    device, device dense eigensolver, lowest neigen pairs kept."""
    import torch

    if not torch.cuda.is_available():
        raise L.EdgError(L.EDG_ERR_NODEVICE, "ed_diag_d", "dense branch needs a CUDA device")
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    h = torch.empty((sec.dim, sec.dim), dtype=torch.complex128 if sec.cplx else torch.float64, device=dev)
    sec.set_stream(stream.cuda_stream)
    sec.dense_dev(h.data_ptr())
    # the buffer is column-major: read row-major it is H^T (= H for real, conj(H) for complex)
    w, z = torch.linalg.eigh(h.mT if sec.cplx else h)
    return w[:neigen].cpu().numpy(), z[:, :neigen].T.contiguous().cpu().numpy()


def device_solver(model: Model, nup: int, ndw: int, neigen: int, lanc_solve: bool, params: DiagParams, seed: int):
    """Eigenpairs of one sector on the device: (evals[neigen], evecs[neigen, dim])."""
    sec = Sector(model, nup, ndw)
    try:
        if not lanc_solve:
            return _dense_lowest(sec, neigen)
        maxit = min(sec.dim, params.lanc_niter)
        if params.lanc_method == "lanczos":
            e0, vec, _ = sp_lanc_eigh(sec, seed=seed, maxit=maxit, tol=params.lanc_tolerance)
            return np.array([e0]), vec[None, :]
        ev, vecs, resid, _ = sec.lowest_k(neigen, seed=seed, maxit=maxit, tol=params.lanc_tolerance,
                                          mode=L.EDG_LK_F32_REFINE if params.lanc_fp32_bulk else L.EDG_LK_F64)
        bad = resid > params.lanc_tolerance * np.maximum(1.0, np.abs(ev))
        if np.any(bad):
            raise L.EdgError(L.EDG_ERR_NOCONV, "sp_eigh",
                             f"sector ({nup},{ndw}): residuals {resid[bad]} above tolerance after {maxit} vectors")
        return ev, vecs
    finally:
        sec.delete()


def sector_device_bytes(dim: int, neigen: int, lanc_solve: bool, params: DiagParams, cplx: bool = False) -> int:
    """Device memory one sector solve holds at its peak, in bytes: the Lanczos basis of
    edg_lowest_k plus its Ritz, start, work and (real sectors) restart vectors, the
    ground-state vectors of edg_ground_state, or the dense matrix with the eigensolver's
    copy and workspace; twice that for the complex vectors of a complex-Hij model. A real
    sector's basis holds Ncv = max(10 k, 2k + 16) vectors (all of a sector of at most 4 Ncv
    states), a complex sector's min(lanc_niter, dim). The hop tables are small beside these."""
    w = 16 if cplx else 8
    if not lanc_solve:
        return 3 * dim * dim * w + (1 << 20)
    if params.lanc_method == "lanczos":
        return 8 * dim * w + (1 << 20)
    if cplx:
        return (min(params.lanc_niter, dim) + neigen + 4) * dim * w + (1 << 20)
    ncv = min(dim, max(10 * neigen, 2 * neigen + 16))
    if dim <= 4 * ncv:
        ncv = dim
    kept = neigen + (ncv - neigen) // 4 if ncv < dim else 0
    return (ncv + kept + neigen + 4) * dim * w + (1 << 20)


class SectorScheduler:
    """Admits sector solves by device memory: a solve starts when its byte estimate fits in
    what is left of `capacity`, and a solve larger than the whole capacity runs alone."""

    def __init__(self, capacity: int):
        self.capacity = max(int(capacity), 1)
        self.free = self.capacity
        self.cv = threading.Condition()

    def acquire(self, nbytes: int) -> int:
        need = min(int(nbytes), self.capacity)
        with self.cv:
            while self.free < need:
                self.cv.wait()
            self.free -= need
        return need

    def release(self, held: int) -> None:
        with self.cv:
            self.free += held
            self.cv.notify_all()


def _device_capacity() -> int:
    """Free HBM of the current device less a 2 GB reserve (the library's own admission
    checks keep a further margin)."""
    import torch

    free, _ = torch.cuda.mem_get_info()
    return max(free - (2 << 30), 1)


def solve_sectors(model: Model, jobs, params: DiagParams, seed: int, solver=None, threads: int | None = None,
                  capacity: int | None = None) -> dict:
    """Runs solver(model, nup, ndw, neigen, lanc_solve, params, seed) over `jobs`, a list of
    (key, nup, ndw, neigen, lanc_solve); returns {key: (evals, evecs)}.

    `threads` solves run at once (default: params.sector_threads for the device solver, 1
    for a caller-supplied one), largest sector first, each admitted by SectorScheduler
    against `capacity` bytes (default: the device's free HBM). With one thread the jobs run
    in the given order. The first failure in job order is raised once every started solve
    has ended."""
    fn = solver or device_solver
    if threads is None:
        threads = params.sector_threads if solver is None else 1
    if threads <= 1 or len(jobs) <= 1:
        return {key: fn(model, nup, ndw, ne, lz, params, seed) for key, nup, ndw, ne, lz in jobs}
    import torch

    on_gpu = torch.cuda.is_available()
    dev = torch.cuda.current_device() if on_gpu else None
    if on_gpu and solver is None and any(not job[4] for job in jobs):
        # torch loads its dense eigensolver on first use, and that first use must not
        # happen on several threads at once
        torch.linalg.eigh(torch.ones((1, 1), dtype=torch.float64, device=torch.device("cuda", dev)))
    sched = SectorScheduler(capacity if capacity is not None else _device_capacity())
    ns = model.ns
    cplx = bool(np.iscomplexobj(model.hij) and np.any(np.imag(model.hij) != 0))

    def run(job):
        key, nup, ndw, ne, lz = job
        if on_gpu:
            torch.cuda.set_device(dev)
        held = sched.acquire(sector_device_bytes(math.comb(ns, nup) * math.comb(ns, ndw), ne, lz, params, cplx))
        try:
            return fn(model, nup, ndw, ne, lz, params, seed)
        finally:
            sched.release(held)

    order = sorted(range(len(jobs)), key=lambda i: -math.comb(ns, jobs[i][1]) * math.comb(ns, jobs[i][2]))
    with ThreadPoolExecutor(max_workers=threads) as ex:
        futs = {i: ex.submit(run, jobs[i]) for i in order}
    return {job[0]: futs[i].result() for i, job in enumerate(jobs)}


# ----------------------------------------------------------------------------- ranks
def _rank_world(comm):
    """(rank, world size) of a torch.distributed process group, (0, 1) without one."""
    if comm is None:
        return 0, 1
    import torch.distributed as dist

    return dist.get_rank(comm), dist.get_world_size(comm)


def _allgather(obj, comm):
    if comm is None:
        return [obj]
    import torch.distributed as dist

    out = [None] * dist.get_world_size(comm)
    dist.all_gather_object(out, obj, group=comm)
    return out


def _allreduce_sum(arrays: dict, comm) -> dict:
    if comm is None:
        return arrays
    import torch
    import torch.distributed as dist

    keys = sorted(arrays)
    flat = torch.from_numpy(np.concatenate([arrays[k] for k in keys]))
    if dist.get_backend(comm) == "nccl":
        flat = flat.cuda()
    dist.all_reduce(flat, group=comm)
    flat = flat.cpu().numpy()
    out, o = {}, 0
    for k in keys:
        out[k] = flat[o:o + arrays[k].size].copy()
        o += arrays[k].size
    return out


# ----------------------------------------------------------------------------- drivers
def diagonalize_lattice(model: Model, params: DiagParams, seed: int = 1234, solver=None,
                        keep_vectors: bool = True, comm=None):
    """ed_diag_d (src/DIAG/DIAG.f90:103-332) over all sectors (isector = 1 + Nup*(Ns+1) + Ndw,
    skipping those of the wrong filling when ED_FILLING != 0). Returns (state_list, eig_list)
    where eig_list holds (isector, evals, lanc_solve) per visited sector, the content of
    eigenvalues_list.ed. `solver(model, nup, ndw, neigen, lanc_solve, params, seed)` returns
    (evals, evecs); the default runs on the device, params.sector_threads sectors at once.

    With a torch.distributed group `comm`, the visited sectors are dealt round-robin to the
    ranks (independent units, one GPU each). Each rank solves its own sectors and keeps their
    vectors; the eigenvalues are all-gathered so that every rank builds the same state list,
    in the same sector order as one process would. A state's vector lives on its owner rank
    only (EState.vec is None elsewhere); lanc_observables sums over ranks."""
    rank, world = _rank_world(comm)
    ns = model.ns
    nsectors = (ns + 1) ** 2
    params.setup(nsectors)
    finite_t = params.finite_temp
    visit = []
    if params.ed_twin and model.nspin > 1:
        import warnings

        warnings.warn("using twin_sector with Nspin>1")  # the reference's warning (src/SETUP.f90:197-199)
    for isector in range(1, nsectors + 1):
        nup, ndw = model.get_nup(isector), model.get_ndw(isector)
        if model.ed_filling != 0 and nup + ndw != model.ed_filling:
            continue
        if params.ed_twin and nup < ndw:  # twin_mask (src/SETUP.f90:254-260)
            continue
        dim = math.comb(ns, nup) * math.comb(ns, ndw)
        neigen = 1 if params.lanc_method == "lanczos" else min(dim, params.lanc_nstates_sector)
        lanc_solve = not (neigen == dim or dim <= params.lanc_dim_threshold)
        visit.append((isector, nup, ndw, neigen, lanc_solve))
    mine, vectors = [], {}
    jobs = [v for pos, v in enumerate(visit) if pos % world == rank]
    results = solve_sectors(model, jobs, params, seed, solver)
    for isector, nup, ndw, neigen, lanc_solve in jobs:
        evals, evecs = results[isector]
        evals = np.asarray(evals, dtype=np.float64)[:neigen]
        mine.append((isector, evals))
        if keep_vectors and evecs is not None:
            vectors[isector] = evecs
    solved = {}
    for owner, part in enumerate(_allgather(mine, comm)):
        for isector, evals in part:
            solved[isector] = (evals, owner)
    state_list = StateList()
    eig_list = []
    oldzero = 1000.0
    for isector, nup, ndw, neigen, lanc_solve in visit:
        evals, owner = solved[isector]
        eig_list.append((isector, evals.copy(), lanc_solve))
        vecs = vectors.get(isector) if owner == rank else None
        # Tflag (src/DIAG/DIAG.f90:136-137): the twin of a sector with Nup != Ndw
        twin = (model.get_sector(ndw, nup), (math.comb(ns, nup), math.comb(ns, ndw))) \
            if params.ed_twin and nup != ndw else None
        for i in range(neigen):
            vec = vecs[i] if vecs is not None else None
            e = float(evals[i])
            if finite_t:
                state_list.add_state(e, vec, isector, size=params.lanc_nstates_total, owner=owner, twin=twin)
            elif e < oldzero - 10.0 * params.gs_threshold:
                oldzero = e
                state_list.free()
                state_list.add_state(e, vec, isector, owner=owner, twin=twin)
            elif abs(e - oldzero) <= params.gs_threshold:
                oldzero = min(oldzero, e)
                state_list.add_state(e, vec, isector, owner=owner, twin=twin)
    if finite_t:
        egs, ec = state_list.emin, state_list.emax
        if math.exp(-(ec - egs) / params.temp) > params.cutoff:
            raise L.EdgError(L.EDG_ERR_STATE, "ED_DIAG",
                             "exp(-(Ei-Egs)/T)>Cutoff condition not met, try increasing lanc_nstates_sector")
        ei = state_list.energy()
        while math.exp(-(ei - egs) / params.temp) <= params.cutoff:
            state_list.pop_state()
            ei = state_list.energy()
    return state_list, eig_list


def partition_function(state_list: StateList, params: DiagParams) -> float:
    """partition_function_lattice, Lanczos branch (src/DIAG/DIAG.f90:65-75)."""
    egs = state_list.emin
    if not params.finite_temp:
        return float(state_list.size)
    n = state_list.trim_size(params.temp, params.cutoff, True)
    return float(sum(math.exp(-(state_list.energy(i) - egs) / params.temp) for i in range(1, n + 1)))


def lanc_observables(model: Model, state_list: StateList, zeta: float, params: DiagParams, observer=None,
                     comm=None) -> dict:
    """Thermal averages of n_i, n_i,up, n_i,dw, d_i and m_i = n_i,up - n_i,dw over the trimmed
    list with weights exp(-(E-Egs)/T)/Z (1/Z at T=0) (src/OBSERVABLES.f90:78-192).
    `observer(model, isector, vec, weight)` returns the weighted per-site arrays of one state;
    the default loads the state into the device sector and runs edg_observables. With `comm`,
    each rank adds the states it owns and the sums are all-reduced."""
    rank, _ = _rank_world(comm)
    ns = model.ns
    egs = state_list.emin
    n = state_list.trim_size(params.temp, params.cutoff, params.finite_temp)
    out = {k: np.zeros(ns) for k in ("dens", "dens_up", "dens_dw", "docc", "magz")}
    sectors: dict[int, Sector] = {}
    try:
        for istate in range(1, n + 1):
            st = state_list.states[istate - 1]
            if st.owner != rank:
                continue
            bw = math.exp(-(st.e - egs) / params.temp) if params.finite_temp else 1.0
            bw /= zeta
            if st.vec is None:
                raise L.EdgError(L.EDG_ERR_STATE, "lanc_observables", "state list holds no vectors")
            if observer is not None:
                obs = observer(model, st.sector, st.vec, bw)
            else:
                sec = sectors.get(st.sector)
                if sec is None:
                    sec = sectors[st.sector] = Sector.from_index(model, st.sector)
                sec.set_state(st.vec)
                obs = sec.observables(bw)
            for k in out:
                out[k] += obs[k]
    finally:
        for sec in sectors.values():
            sec.delete()
    out = _allreduce_sum(out, comm)
    out["mag"] = out["dens_up"] - out["dens_dw"]
    return out


def lanc_energy(model: Model, state_list: StateList, zeta: float, params: DiagParams, energy_fn=None,
                comm=None) -> dict:
    """Thermal ed_Ekin, ed_Epot (Hartree term included, as src/ENERGY.f90:343), ed_Eknot and
    ed_Ehartree over the trimmed list with weights exp(-(E-Egs)/T)/Z (1/Z at T=0)
    (src/ENERGY.f90:76-356, Norb=1 terms). `energy_fn(model, isector, vec, weight)` returns the
    weighted dict of one state; the default loads the state into the device sector and runs
    edg_energy. With `comm`, each rank adds the states it owns and the sums are all-reduced."""
    rank, _ = _rank_world(comm)
    egs = state_list.emin
    n = state_list.trim_size(params.temp, params.cutoff, params.finite_temp)
    out = {k: np.zeros(1) for k in ("ekin", "epot", "eknot", "ehartree")}
    sectors: dict[int, Sector] = {}
    try:
        for istate in range(1, n + 1):
            st = state_list.states[istate - 1]
            if st.owner != rank:
                continue
            bw = math.exp(-(st.e - egs) / params.temp) if params.finite_temp else 1.0
            bw /= zeta
            if st.vec is None:
                raise L.EdgError(L.EDG_ERR_STATE, "lanc_energy", "state list holds no vectors")
            if energy_fn is not None:
                en = energy_fn(model, st.sector, st.vec, bw)
            else:
                sec = sectors.get(st.sector)
                if sec is None:
                    sec = sectors[st.sector] = Sector.from_index(model, st.sector)
                sec.set_state(st.vec)
                en = sec.energy(bw)
            for k in out:
                out[k] += en[k]
    finally:
        for sec in sectors.values():
            sec.delete()
    out = _allreduce_sum(out, comm)
    return {k: float(v[0]) for k, v in out.items()}

