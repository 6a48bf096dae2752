"""Host-side mirror of the EDlattice interfaces on the sector-Lanczos path.

Names, argument meanings and error behaviour follow the reference (file:line cited per
object, paths relative to the EDlattice project root); the work happens in libedgpu.so.
Errors that the reference reports with `stop` raise EdgError here.

    Hij            Hij_init / Hij_add_link / Hij_read / Hij_build / Hij_get  (src/GRAPH_MATRIX.f90)
    Model          Hij plus the hot-path input keys ULOC, XMU, HFMODE, ED_FILLING
    Sector         build_Hv_sector / delete_Hv_sector / vecDim_Hv_sector    (src/DIAG/HAMILTONIAN.f90:53-239)
    Sector.HxV     the dd_sparse_HxV callback (src/VARS_GLOBAL.f90:102-108)
    tridiag_Hv_sector, sp_lanc_eigh, the GF/CHI/OC chain builders and evaluators.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _edgpu_lib as L


def _pd(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(L._pd)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------------------- lattice input
class Hij:
    """Hopping matrix builder: Hij_init(Nsites,Nspin) / Hij_add_link / Hij_read / Hij_build
    (src/GRAPH_MATRIX.f90:79-329). One orbital: siteI/siteJ index the Ns sites, 1-based."""

    def __init__(self, nsites: int, nspin: int = 1):
        if nspin not in (1, 2):
            raise ValueError("Hij_init: Nspin must be 1 or 2")
        self.ns = int(nsites)
        self.nspin = nspin
        self.links: list[tuple[int, int, int, int, int, complex]] = []

    def add_link(self, siteI: int, siteJ: int, orbI: int, orbJ: int, spin: int, hval: complex) -> None:
        # checks of Hij_add_link (src/GRAPH_MATRIX.f90:171-179)
        if spin > self.nspin or spin <= 0:
            raise ValueError("Hij_add_link ERROR: spinI or spinJ either > Nspin OR < 0")
        if orbI != 1 or orbJ != 1:
            raise ValueError("Hij_add_link ERROR: orbI or orbJ either > Norb OR < 0")
        if siteI > self.ns or siteJ > self.ns or siteI <= 0 or siteJ <= 0:
            raise ValueError("Hij_add_link ERROR: siteI or siteJ either > Nlat OR < 0")
        self.links.append((siteI, siteJ, orbI, orbJ, spin, complex(hval)))

    def read(self, path: str) -> None:
        """Hij_read: one link per line, `i j a b spin re im` (src/GRAPH_MATRIX.f90:280-301)."""
        with open(path) as f:
            for line in f:
                tok = line.split()
                if not tok:
                    continue
                i, j, a, b, spin = (int(x) for x in tok[:5])
                re_, im_ = float(tok[5]), float(tok[6])
                self.add_link(i, j, a, b, spin, complex(re_, im_))

    def build(self) -> np.ndarray:
        """Hij_build: later links overwrite earlier ones; Hermiticity asserted at 1e-6
        (src/GRAPH_MATRIX.f90:306-329). Returns H[nspin, Ns, Ns] (complex)."""
        H = np.zeros((self.nspin, self.ns, self.ns), dtype=np.complex128)
        for (i, j, _a, _b, spin, val) in self.links:
            H[spin - 1, i - 1, j - 1] = val
        for s in range(self.nspin):
            if not np.all(np.abs(H[s] - H[s].conj().T) < 1e-6):
                raise L.EdgError(L.EDG_ERR_ARG, "Hij_build", "Hij_build ERROR: Hij is not Hermitian")
        return H


def square_lattice(lx: int, ly: int, t: float = 1.0, periodic: bool = True) -> np.ndarray:
    """Nearest-neighbour Hij = -t on an lx x ly lattice, site index x + lx*y (0-based)."""
    ns = lx * ly
    H = np.zeros((ns, ns))
    for y in range(ly):
        for x in range(lx):
            i = x + lx * y
            for dx, dy in ((1, 0), (0, 1)):
                xx, yy = x + dx, y + dy
                if periodic:
                    xx %= lx
                    yy %= ly
                elif xx >= lx or yy >= ly:
                    continue
                j = xx + lx * yy
                if i == j:
                    continue
                H[i, j] = -t
                H[j, i] = -t
    return H


def ring(L_: int, t: float = 1.0) -> np.ndarray:
    """Periodic 1-D ring of L_ sites, Hij = -t."""
    return square_lattice(L_, 1, t, periodic=True)


# ----------------------------------------------------------------------------- model / sector
class Model:
    """Hij (Ns x Ns, or [2,Ns,Ns] for Nspin=2; real or complex) with Uloc, xmu, HFMODE,
    ED_FILLING. With complex Hij the sectors' vectors are complex."""

    def __init__(self, hij, uloc: float = 0.0, xmu: float = 0.0, hfmode: bool = True, ed_filling: int = 0):
        H = np.asarray(hij)
        if H.ndim == 2:
            H = H[None]
        self.nspin = H.shape[0]
        self.ns = H.shape[1]
        self.hij = H
        self.uloc, self.xmu, self.hfmode, self.ed_filling = float(uloc), float(xmu), bool(hfmode), int(ed_filling)
        re0 = _f64(H[0].real)
        im0 = _f64(H[0].imag) if np.iscomplexobj(H) else None
        re1 = _f64(H[1].real) if self.nspin == 2 else None
        im1 = _f64(H[1].imag) if (self.nspin == 2 and np.iscomplexobj(H)) else None
        self._keep = (re0, im0, re1, im1)
        h = C.c_void_p()
        L.check(L.lib().edg_model_create(self.ns, self.nspin, _pd(re0), _pd(im0), _pd(re1), _pd(im1), self.uloc,
                                         self.xmu, int(self.hfmode), self.ed_filling, C.byref(h)), "edg_model_create")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            L.lib().edg_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # sector numbering (src/SECTOR.f90:370-424)
    def get_sector(self, nup: int, ndw: int) -> int:
        return L.lib().edg_get_sector(self.ns, nup, ndw)

    def get_nup(self, isector: int) -> int:
        return L.lib().edg_get_nup(self.ns, isector)

    def get_ndw(self, isector: int) -> int:
        return L.lib().edg_get_ndw(self.ns, isector)


class Sector:
    """build_Hv_sector(isector) on the device (src/DIAG/HAMILTONIAN.f90:53-162)."""

    def __init__(self, model: Model, nup: int, ndw: int, form: int = L.EDG_FORM_STORED):
        self.model = model
        self.nup, self.ndw, self.form = nup, ndw, form
        h = C.c_void_p()
        L.check(L.lib().edg_sector_create(model.handle, nup, ndw, form, C.byref(h)), "build_Hv_sector")
        self.handle = h
        d, du, dd = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(L.lib().edg_sector_dims(h, C.byref(d), C.byref(du), C.byref(dd)), "edg_sector_dims")
        self.dim, self.dimup, self.dimdw = d.value, du.value, dd.value
        vl = C.c_int64()
        L.check(L.lib().edg_sector_vlen(h, C.byref(vl)), "edg_sector_vlen")
        self.vlen = vl.value            # reals per vector
        self.cplx = self.vlen != self.dim  # complex Hij: complex vectors, stored interleaved

    @classmethod
    def from_index(cls, model: Model, isector: int, form: int = L.EDG_FORM_STORED) -> "Sector":
        return cls(model, model.get_nup(isector), model.get_ndw(isector), form)

    def delete(self):
        """delete_Hv_sector (src/DIAG/HAMILTONIAN.f90:166-212)."""
        if getattr(self, "handle", None):
            L.lib().edg_sector_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass

    def vecDim(self) -> int:
        """vecDim_Hv_sector: DimUp*DimDw on one GPU (src/DIAG/HAMILTONIAN.f90:215-239)."""
        return self.dim

    def maps(self) -> tuple[np.ndarray, np.ndarray]:
        mu = np.zeros(self.dimup, dtype=np.int32)
        md = np.zeros(self.dimdw, dtype=np.int32)
        L.check(L.lib().edg_sector_get_maps(self.handle, mu.ctypes.data_as(L._pi32), md.ctypes.data_as(L._pi32)),
                "edg_sector_get_maps")
        return mu, md

    def hops(self, spin: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        nnz = C.c_int64()
        L.check(L.lib().edg_sector_get_hops(self.handle, spin, None, None, None, C.byref(nnz)), "edg_sector_get_hops")
        dim = self.dimup if spin == 1 else self.dimdw
        rp = np.zeros(dim + 1, dtype=np.int64)
        cols = np.zeros(max(nnz.value, 1), dtype=np.int32)
        vals = np.zeros(max(nnz.value, 1), dtype=np.float64)
        L.check(L.lib().edg_sector_get_hops(self.handle, spin, rp.ctypes.data_as(L._pi64), cols.ctypes.data_as(L._pi32),
                                            _pd(vals), C.byref(nnz)), "edg_sector_get_hops")
        return rp, cols[: nnz.value], vals[: nnz.value]

    def HxV(self, v: np.ndarray) -> np.ndarray:
        """dd_sparse_HxV(Nloc,v,Hv): complex(8) in, complex(8) out (Hv overwritten)."""
        v = np.ascontiguousarray(v, dtype=np.complex128)
        hv = np.empty_like(v)
        L.check(L.lib().edg_hxv_z(self.handle, v.size, v.view(np.float64).ctypes.data_as(L._pd),
                                  hv.view(np.float64).ctypes.data_as(L._pd)), "spHtimesV")
        return hv

    def hxv_real(self, v: np.ndarray) -> np.ndarray:
        """H x v on a real host vector (real Hij only)."""
        v = _f64(v)
        hv = np.empty_like(v)
        L.check(L.lib().edg_hxv_d(self.handle, v.size, _pd(v), _pd(hv)), "spHtimesV")
        return hv

    def autotune(self, precision: int = L.EDG_PREC_F32, reps: int = 5) -> dict:
        """Time the H x v kernel variants on this sector and keep the fastest for `precision`
        (edg_sector_autotune): {"ms": per-candidate ms per H x v, "best": index kept}."""
        ms = np.zeros(64)  # room for every candidate of either precision
        nc, best = C.c_int(), C.c_int()
        L.check(L.lib().edg_sector_autotune(self.handle, precision, reps, _pd(ms), C.byref(nc), C.byref(best)),
                "edg_sector_autotune")
        return {"ms": ms[: nc.value].tolist(), "best": best.value}

    def set_kernels(self, candidate: int, precision: int = L.EDG_PREC_F32) -> None:
        """Pin the H x v kernel pair (an index of autotune()'s candidate list)."""
        L.check(L.lib().edg_sector_set_kernels(self.handle, precision, candidate), "edg_sector_set_kernels")

    def release_work(self) -> None:
        """Hand the sector's work buffers (Lanczos vectors, FP32 basis, block vectors) back to
        the library's pool; tables and the state buffer stay."""
        L.check(L.lib().edg_sector_release_work(self.handle), "edg_sector_release_work")

    def set_stream(self, stream: int | None) -> None:
        """Run the sector's device work on `stream` (a cudaStream_t as an int; None = the legacy default stream)."""
        L.check(L.lib().edg_sector_set_stream(self.handle, C.c_void_p(stream)), "edg_sector_set_stream")

    def lowest_k(self, k: int, v0: np.ndarray | None = None, seed: int = 1234, maxit: int = 512,
                 tol: float = 1e-10, want_vectors: bool = True, mode: int = L.EDG_LK_F64):
        """Lowest k eigenpairs (the sp_eigh branch of ed_diag_d, src/DIAG/DIAG.f90:191-202),
        FP64 (mode EDG_LK_F64) or FP32 bulk + FP64 refinement (EDG_LK_F32_REFINE).
        Real sectors run thick-restarted with the reference's Ncv = 10 k basis vectors.
        Returns (evals[k'], evecs[k', dim] or None, resid[k'], H x v applications), k' = min(k, dim)."""
        kk = min(k, self.dim)
        ev = np.zeros(k)
        rs = np.zeros(k)
        vecs = np.empty((kk, self.vlen)) if want_vectors else None
        it = C.c_int()
        v0a = self._vec(v0, "v0") if v0 is not None else None
        L.check(L.lib().edg_lowest_k_mode(self.handle, k, _pd(v0a), C.c_uint64(seed), maxit, tol, mode, _pd(ev),
                                          _pd(vecs), _pd(rs), C.byref(it)), "sp_eigh")
        if vecs is not None and self.cplx:
            vecs = vecs.view(np.complex128)
        return ev[:kk], vecs, rs[:kk], it.value

    def dense(self) -> np.ndarray:
        """Dense sector matrix of ed_buildh(Hmat) (src/DIAG/HAMILTONIAN_STORED_HxV.f90:81-117),
        complex for a complex-Hij sector."""
        if self.cplx:
            h = np.empty((self.dim, self.dim), dtype=np.complex128, order="F")  # the library writes column-major
            L.check(L.lib().edg_sector_dense(self.handle, h.ctypes.data_as(L._pd)), "ed_buildh")
            return h
        h = np.empty((self.dim, self.dim))
        L.check(L.lib().edg_sector_dense(self.handle, _pd(h)), "ed_buildh")
        return h  # symmetric: row- and column-major read the same

    def dense_dev(self, dh_ptr: int) -> None:
        """Dense sector matrix into device memory (dim*dim doubles, or dim*dim interleaved
        complex for a complex-Hij sector; column-major) on the sector's stream."""
        L.check(L.lib().edg_sector_dense_dev(self.handle, C.c_void_p(dh_ptr)), "ed_buildh")

    # ---- state buffer (the eigenvector kept on the device)
    def get_state(self) -> np.ndarray:
        """The state kept on the device: real, or complex for a complex-Hij sector."""
        x = np.empty(self.vlen)
        L.check(L.lib().edg_state_get(self.handle, _pd(x)), "edg_state_get")
        return x.view(np.complex128) if self.cplx else x

    def set_state(self, x: np.ndarray) -> None:
        x = self._vec(x, "state")
        L.check(L.lib().edg_state_set(self.handle, _pd(x)), "edg_state_set")

    def _vec(self, x, what: str) -> np.ndarray:
        """x as the library's FP64 layout for this sector: real [dim], or complex [dim]
        interleaved as [2*dim] reals (a real x is taken as a complex vector with zero
        imaginary part)."""
        if self.cplx:
            x = np.ascontiguousarray(x, dtype=np.complex128)
            if x.size != self.dim:
                raise ValueError(f"{what} size != sector dimension")
            return x.view(np.float64)
        x = _f64(np.real(x))
        if x.size != self.dim:
            raise ValueError(f"{what} size != sector dimension")
        return x

    def observables(self, weight: float = 1.0) -> dict:
        """lanc_observables for the stored state (src/OBSERVABLES.f90:127-152)."""
        ns = self.model.ns
        out = {k: np.zeros(ns) for k in ("dens", "dens_up", "dens_dw", "docc", "magz")}
        L.check(L.lib().edg_observables(self.handle, weight, _pd(out["dens"]), _pd(out["dens_up"]), _pd(out["dens_dw"]),
                                        _pd(out["docc"]), _pd(out["magz"])), "edg_observables")
        return out


    def energy(self, weight: float = 1.0) -> dict:
        """lanc_energy's Norb=1 terms for the stored state (src/ENERGY.f90:118-226):
        ekin, epot (Hartree term included), eknot, ehartree, each times weight."""
        out = [C.c_double(0.0) for _ in range(4)]
        L.check(L.lib().edg_energy(self.handle, weight, *[C.byref(x) for x in out]), "lanc_energy")
        return dict(zip(("ekin", "epot", "eknot", "ehartree"), (x.value for x in out)))


def release_cached_memory() -> None:
    """Hand the device memory the library keeps for reuse between sectors (up to a quarter of
    the current device's memory) back to the driver, e.g. before a large torch workload in the
    same process."""
    L.check(L.lib().edg_release_cached_memory(), "edg_release_cached_memory")


# ----------------------------------------------------------------------------- Lanczos
def random_vector(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    L.check(L.lib().edg_random_vector(C.c_uint64(seed), n, _pd(out)), "edg_random_vector")
    return out


def tridiag_Hv_sector(sector: Sector, vvinit: np.ndarray, nlanc: int | None = None, threshold: float = 1e-9,
                      precision: int = L.EDG_PREC_F64):
    """tridiag_Hv_sector(isector,vvinit,alanc,blanc,norm2) (src/DIAG/HAMILTONIAN.f90:242-275).
    nlanc defaults to Nlanc = min(Dim, lanc_nGFiter=200) (src/SECTOR.f90:112).
    Returns (alanc, blanc, norm2, nsteps) with blanc[0] = 0."""
    if nlanc is None:
        nlanc = min(sector.dim, 200)
    try:
        v = sector._vec(vvinit, "vvinit")
    except ValueError as e:
        raise L.EdgError(L.EDG_ERR_ARG, "tridiag_Hv_sector", str(e)) from None
    a = np.zeros(max(nlanc, 1))
    b = np.zeros(max(nlanc, 1))
    n2 = C.c_double()
    ns = C.c_int()
    L.check(L.lib().edg_tridiag_d(sector.handle, _pd(v), nlanc, threshold, precision, _pd(a), _pd(b), C.byref(n2),
                                  C.byref(ns)), "tridiag_Hv_sector")
    return a[:nlanc], b[:nlanc], n2.value, ns.value


def sp_lanc_eigh(sector: Sector, v0: np.ndarray | None = None, seed: int = 1234, maxit: int = 512,
                 tol: float = 1e-12, mode: int = L.EDG_GS_F64, want_vector: bool = True):
    """Lowest eigenpair of the sector (contract of sp_lanc_eigh, src/DIAG/DIAG.f90:212-217).
    The eigenvector also stays on the device as the sector's state.
    Returns (E0, evec or None, number of H x v applications)."""
    e0 = C.c_double()
    it = C.c_int()
    v0a = sector._vec(v0, "v0") if v0 is not None else None
    if not want_vector:
        mode |= L.EDG_GS_E0_ONLY
    L.check(L.lib().edg_ground_state_keep(sector.handle, _pd(v0a), C.c_uint64(seed), maxit, tol, mode, C.byref(e0),
                                          C.byref(it)), "sp_lanc_eigh")
    vec = sector.get_state() if want_vector else None
    return e0.value, vec, it.value


def tridiag_eigh(d: np.ndarray, e: np.ndarray):
    """eigh(diag,subdiag) with first components (e[0] ignored)."""
    d, e = _f64(d), _f64(e)
    n = d.size
    w, z = np.zeros(n), np.zeros(n)
    L.check(L.lib().edg_tridiag_eigh(n, _pd(d), _pd(e), _pd(w), _pd(z)), "eigh")
    return w, z


def tridiag_lowest(d: np.ndarray, e: np.ndarray, k: int):
    """k lowest eigenvalues of the tridiagonal (e[0] ignored) and |last component| of each
    unit eigenvector."""
    d, e = _f64(d), _f64(e)
    n = d.size
    kk = min(k, n)
    w, zn = np.zeros(kk), np.zeros(kk)
    L.check(L.lib().edg_tridiag_lowest(n, _pd(d), _pd(e), kk, _pd(w), _pd(zn)), "tridiag_lowest")
    return w, zn


def poles_weights(alanc, blanc, norm2: float, ei: float, isign: int):
    """add_to_lanczos_gf_normal's loop (src/GF/GF_ELECTRONS.f90:445-456)."""
    a, b = _f64(alanc), _f64(blanc)
    n = a.size
    p, w = np.zeros(n), np.zeros(n)
    L.check(L.lib().edg_poles_weights(n, _pd(a), _pd(b), norm2, ei, isign, _pd(p), _pd(w)), "poles_weights")
    return p, w


# ----------------------------------------------------------------------------- response chains
@dataclass
class Spectrum:
    """One GFspectrum channel (src/VARS_GLOBAL.f90:47-51): poles and weights."""
    poles: np.ndarray
    weight: np.ndarray
    norm2: float = 0.0


def _chain_out(nlanc):
    return np.zeros(max(nlanc, 1)), np.zeros(max(nlanc, 1)), C.c_double(), C.c_int()


def gf_chain(from_sector: Sector, to_sector: Sector, op: int, site: int, spin: int, nlanc: int, ei: float,
             site2: int = 0, precision: int = L.EDG_PREC_F64) -> Spectrum:
    """c^+ (op=+1) or c (op=-1) chain of lanc_build_gf_electrons_diag/_mix
    (src/GF/GF_ELECTRONS.f90:202-405) + add_to_lanczos_gf_normal (:417-457)."""
    p, w, n2, n = _chain_out(nlanc)
    L.check(L.lib().edg_gf_chain(from_sector.handle, to_sector.handle, op, site, site2, spin, nlanc, precision, ei,
                                 _pd(p), _pd(w), C.byref(n2), C.byref(n)), "gf_chain")
    return Spectrum(p[: n.value].copy(), w[: n.value].copy(), n2.value)


def _block_out(k, nlanc):
    return (np.zeros(k * nlanc), np.zeros(k * nlanc), np.zeros(k), np.zeros(k, dtype=np.int32))


def _spectra(k, nlanc, p, w, n2, n):
    return [Spectrum(p[c * nlanc: c * nlanc + n[c]].copy(), w[c * nlanc: c * nlanc + n[c]].copy(), float(n2[c]))
            for c in range(k)]


def gf_chain_block(from_sector: Sector, to_sector: Sector, op: int, sites, spin: int, nlanc: int, ei: float,
                   sites2=None, precision: int = L.EDG_PREC_F64) -> list:
    """The chains c^+_{sites[c]} (op=+1) or c_{sites[c]} (op=-1) of one state into one target
    sector as one block (block H x V; edg_gf_chain_block): the inner loop of
    lanc_build_gf_electrons_diag/_mix over sites (src/GF/GF_ELECTRONS.f90:202-405) with
    add_to_lanczos_gf_normal per chain (:417-457). Returns one Spectrum per site."""
    si = np.ascontiguousarray(sites, dtype=np.int32)
    k = si.size
    s2 = np.ascontiguousarray(sites2, dtype=np.int32) if sites2 is not None else None
    p, w, n2, n = _block_out(k, nlanc)
    L.check(L.lib().edg_gf_chain_block(from_sector.handle, to_sector.handle, op, k, si.ctypes.data_as(L._pi),
                                       s2.ctypes.data_as(L._pi) if s2 is not None else None, spin, nlanc, precision,
                                       ei, _pd(p), _pd(w), _pd(n2), n.ctypes.data_as(L._pi)), "gf_chain_block")
    return _spectra(k, nlanc, p, w, n2, n)


def chi_chain_block(sector: Sector, nlanc: int, ei: float, kind: int = 0, sites=None, sites2=None, qcos=None,
                    precision: int = L.EDG_PREC_F64) -> list:
    """Susceptibility chains of one state as one block (edg_chi_chain_block): kind 0 = S^z,
    1 = N, one chain per site of `sites` (+ sites2), or per row of qcos [k, Ns] (momentum
    combinations). add_to_lanczos_spinChi per chain (src/CHI/CHI_SPIN_ELECTRONS.f90:305-366)."""
    q = np.ascontiguousarray(qcos, dtype=np.float64) if qcos is not None else None
    si = np.ascontiguousarray(sites, dtype=np.int32) if sites is not None else None
    s2 = np.ascontiguousarray(sites2, dtype=np.int32) if sites2 is not None else None
    k = q.shape[0] if q is not None else si.size
    p, w, n2, n = _block_out(k, nlanc)
    L.check(L.lib().edg_chi_chain_block(sector.handle, kind, k, si.ctypes.data_as(L._pi) if si is not None else None,
                                        s2.ctypes.data_as(L._pi) if s2 is not None else None,
                                        _pd(q.ravel()) if q is not None else None, nlanc, precision, ei, _pd(p), _pd(w),
                                        _pd(n2), n.ctypes.data_as(L._pi)), "chi_chain_block")
    return _spectra(k, nlanc, p, w, n2, n)


def chi_chain(sector: Sector, site: int, nlanc: int, ei: float, kind: int = 0, site2: int = 0, qcos=None,
              precision: int = L.EDG_PREC_F64) -> Spectrum:
    """S^z (kind 0) or N (kind 1) chain of lanc_build_spinChi_diag/_mix
    (src/CHI/CHI_SPIN_ELECTRONS.f90:189-293) + add_to_lanczos_spinChi (:305-366).
    qcos (site weights, e.g. cos(q.r_i)) gives the momentum combination."""
    p, w, n2, n = _chain_out(nlanc)
    q = _f64(qcos) if qcos is not None else None
    L.check(L.lib().edg_chi_chain(sector.handle, kind, site, site2, _pd(q), nlanc, precision, ei, _pd(p), _pd(w),
                                  C.byref(n2), C.byref(n)), "chi_chain")
    return Spectrum(p[: n.value].copy(), w[: n.value].copy(), n2.value)


def oc_chain(sector: Sector, nlanc: int, ei: float, precision: int = L.EDG_PREC_F64) -> Spectrum:
    """J chain of lanc_ed_build_oc (src/OC/OC_ELECTRONS.f90:103-214) + add_to_lanczos_oc."""
    p, w, n2, n = _chain_out(nlanc)
    L.check(L.lib().edg_oc_chain(sector.handle, nlanc, precision, ei, _pd(p), _pd(w), C.byref(n2), C.byref(n)),
            "oc_chain")
    return Spectrum(p[: n.value].copy(), w[: n.value].copy(), n2.value)


# ----------------------------------------------------------------------------- evaluation on grids
def grids(temp: float, lmats: int = 4096, lreal: int = 5000, ltau: int = 1024, wini: float = -5.0, wfin: float = 5.0):
    """allocate_grids (src/AUX_FUNX.f90:357-372): wm, vm, wr, vr, tau."""
    ltau = max(int(1.0 / temp), ltau)
    wm = math.pi * temp * (2 * np.arange(1, lmats + 1) - 1)
    vm = math.pi * temp * 2 * np.arange(0, lmats + 1)
    wr = np.linspace(wini, wfin, lreal)
    vr = np.linspace(0.0, wfin, lreal)
    tau = np.linspace(0.0, 1.0 / temp, ltau + 1)
    return wm, vm, wr, vr, tau


def eval_poles(poles: np.ndarray, weights: np.ndarray, z: np.ndarray) -> np.ndarray:
    """sum_k weights[k] / (z - poles[k]) for every z, on the device (edg_eval_poles)."""
    p, w = _f64(poles), _f64(weights)
    z = np.ascontiguousarray(z, dtype=np.complex128)
    zr, zi = _f64(z.real), _f64(z.imag)
    ore, oim = np.zeros(z.size), np.zeros(z.size)
    L.check(L.lib().edg_eval_poles(p.size, _pd(p), _pd(w), z.size, _pd(zr), _pd(zi), _pd(ore), _pd(oim)),
            "edg_eval_poles")
    return ore + 1j * oim


def eval_gf(channels: list[Spectrum], wm: np.ndarray, wr: np.ndarray, eps: float, pesoBZ: float = 1.0):
    """lanc_eval_gf_electrons' sum (src/GF/GF_ELECTRONS.f90:503-508)."""
    gm = np.zeros(wm.size, dtype=np.complex128)
    gr = np.zeros(wr.size, dtype=np.complex128)
    zm = 1j * wm
    zr = wr + 1j * eps
    for ch in channels:
        for peso, de in zip(ch.weight, ch.poles):
            gm += pesoBZ * peso / (zm - de)
            gr += pesoBZ * peso / (zr - de)
    return gm, gr


def eval_chi(channels: list[Spectrum], beta: float, tau: np.ndarray, vr: np.ndarray, eps: float, vm=None,
             pesoBZ: float = 1.0):
    """lanc_eval_spinChi_electrons' sums (src/CHI/CHI_SPIN_ELECTRONS.f90:420-446): chi(tau)
    symmetrised about beta/2 and chi(w); chi(iv) from the formula the reference keeps
    commented out (:430-433), evaluated when vm is given."""
    ltau = tau.size - 1
    ct = np.zeros(ltau + 1)
    cw = np.zeros(vr.size, dtype=np.complex128)
    civ = np.zeros(vm.size, dtype=np.complex128) if vm is not None else None
    h = ltau // 2
    for ch in channels:
        for w_, dE in zip(ch.weight, ch.poles):
            peso = w_ * pesoBZ
            ct[:h] += peso * np.exp(-tau[:h] * dE)
            ct[h] += peso * 0.5 * (np.exp(-tau[h] * dE) + np.exp(-(beta - tau[h]) * dE))
            ct[h + 1:] += peso * np.exp(-(beta - tau[h + 1:]) * dE)
            z = vr + 1j * eps
            cw += -peso * (1.0 - np.exp(-beta * dE)) * (1.0 / (z - dE) - 1.0 / (z + dE))
            if civ is not None:
                if beta * dE > 1e-3:
                    civ[0] += 2 * peso * (1.0 - np.exp(-beta * dE)) / dE
                civ[1:] += peso * (1.0 - np.exp(-beta * dE)) * 2.0 * dE / (vm[1:] ** 2 + dE ** 2)
    return ct, cw, civ


def eval_oc(channels: list[Spectrum], vr: np.ndarray, eps: float, cutoff: float = 1e-9, pesoBZ: float = 1.0):
    """lanc_ed_eval_oc's sums (src/OC/OC_ELECTRONS.f90:301-316): (jj-correlator D, sigma(w))."""
    D = 0.0
    oc = np.zeros(vr.size)
    for ch in channels:
        for w_, dE in zip(ch.weight, ch.poles):
            peso = w_ * pesoBZ
            with np.errstate(divide="ignore", invalid="ignore"):
                r = peso / dE
            if not np.isfinite(r) or abs(dE) < cutoff or abs(r) < cutoff:
                continue
            D += r
            oc += r * eps / ((vr - dE) ** 2 + eps ** 2)
    return D, oc


def drude_weight(jj: float, ekin: float, nsites: int) -> float:
    """Drude_weight = -pi/Nsites*(Ekin + 2 D) (src/OC/OC_FUNCTIONS.f90:65)."""
    return -math.pi / nsites * (ekin + 2.0 * jj)


# ----------------------------------------------------------------------------- GFmatrix I/O
def write_gfmatrix(f, states: list[list[Spectrum]] | None) -> None:
    """write_formatted_gfmatrix (src/VARS_GLOBAL.f90:587-607): status, Nstates, per state
    Nchan, per channel Nexc, poles, weights (list-directed, one record per line)."""
    if states is None:
        f.write(" F\n")
        return
    f.write(" T\n")
    f.write(f" {len(states)}\n")
    for chans in states:
        f.write(f" {len(chans)}\n")
        for ch in chans:
            f.write(f" {len(ch.poles)}\n")
            f.write(" " + " ".join(f"{x: .17E}" for x in ch.poles) + "\n")
            f.write(" " + " ".join(f"{x: .17E}" for x in ch.weight) + "\n")
    f.write("\n")


def read_gfmatrix(f) -> list[list[Spectrum]] | None:
    """read_formatted_gfmatrix (src/VARS_GLOBAL.f90:612-632)."""
    def nxt():
        while True:
            line = f.readline()
            if line == "":
                raise EOFError
            if line.strip():
                return line.split()
    status = nxt()[0].upper().startswith("T")
    if not status:
        return None
    nstates = int(nxt()[0])
    out = []
    for _ in range(nstates):
        nch = int(nxt()[0])
        chans = []
        for _ in range(nch):
            nexc = int(nxt()[0])
            poles = np.array([float(x) for x in nxt()]) if nexc else np.zeros(0)
            weights = np.array([float(x) for x in nxt()]) if nexc else np.zeros(0)
            chans.append(Spectrum(poles, weights))
        out.append(chans)
    return out
