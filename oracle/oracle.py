"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU restatement (edlat_oracle.cpp).

Imported by tests/, by __graft_entry__.smoke() as the checker and by bench.py for the CPU
baseline. The product package never imports this module.

Parity status: unpinned against reference outputs (see the header of edlat_oracle.cpp);
pinned against known answers from the mathematics in tests/test_oracle_known_answers.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libedlat_oracle.so")


def build() -> str:
    src = os.path.join(HERE, "edlat_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


class OrcModel(C.Structure):
    _fields_ = [("ns", C.c_int), ("nspin", C.c_int), ("hij_re", C.c_void_p), ("hij_im", C.c_void_p),
                ("hijdw_re", C.c_void_p), ("hijdw_im", C.c_void_p), ("uloc", C.c_double), ("xmu", C.c_double),
                ("hfmode", C.c_int), ("ed_filling", C.c_int)]


_d, _i, _i64, _p = C.c_double, C.c_int, C.c_int64, C.c_void_p
_SIG = {
    "orc_binomial": (_i, [_i, _i]),
    "orc_get_sector": (_i, [_i, _i, _i]),
    "orc_get_nup": (_i, [_i, _i]),
    "orc_get_ndw": (_i, [_i, _i]),
    "orc_build_map": (_i64, [_i, _i, _p]),
    "orc_binary_search": (_i64, [_p, _i64, _i64]),
    "orc_c": (None, [_i, _i64, _p, _p]),
    "orc_cdg": (None, [_i, _i64, _p, _p]),
    "orc_hop_csr": (_i64, [_p, _i, _i, _p, _p, _p]),
    "orc_direct_matvec_z": (None, [_p, _i, _i, _p, _p]),
    "orc_direct_matvec_d": (None, [_p, _i, _i, _p, _p, _i64, _i64]),
    "orc_stored_create": (_p, [_p, _i, _i]),
    "orc_stored_destroy": (None, [_p]),
    "orc_stored_dim": (_i64, [_p]),
    "orc_stored_matvec_z": (None, [_p, _p, _p]),
    "orc_stored_matvec_d": (None, [_p, _p, _p]),
    "orc_stored_matvec_rows_d": (None, [_p, _p, _p, _i64, _i64]),
    "orc_stored_matvec_sweeps_d": (None, [_p, _p, _p, _i64, _i64]),
    "orc_stored_dimdw": (_i64, [_p]),
    "orc_dense_h": (None, [_p, _i, _i, _p]),
    "orc_tridiag_eigh": (None, [_i, _p, _p, _p, _p]),
    "orc_tridiag_d": (_i, [_p, _p, _i, _d, _p, _p, _p]),
    "orc_lanczos_gs_d": (_i, [_p, _p, _i, _d, _p, _p, _p, _p]),
    "orc_apply_cop_d": (None, [_i, _i, _i, _i, _i, _i, _p, _p, _i]),
    "orc_apply_diagop_d": (None, [_i, _i, _i, _i, _i, _i, _p, _p]),
    "orc_apply_current_d": (None, [_p, _i, _i, _p, _p]),
    "orc_poles_weights": (None, [_i, _p, _p, _d, _d, _i, _p, _p]),
    "orc_observables_d": (None, [_i, _i, _i, _p, _d, _p, _p, _p, _p, _p]),
    "orc_energy_d": (None, [_p, _i, _i, _p, _d, _p, _p, _p, _p]),
    "orc_num_threads": (_i, []),
}

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        for k, (r, a) in _SIG.items():
            f = getattr(_LIB, k)
            f.restype = r
            f.argtypes = a
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Model:
    """Hubbard model as the oracle reads it: Hij [Ns,Ns] or [2,Ns,Ns] (complex allowed)."""

    def __init__(self, hij, uloc=0.0, xmu=0.0, hfmode=True, ed_filling=0):
        H = np.asarray(hij)
        if H.ndim == 2:
            H = H[None]
        self.ns = H.shape[1]
        self.nspin = H.shape[0]
        self._re = [np.ascontiguousarray(H[s].real, dtype=np.float64) for s in range(self.nspin)]
        self._im = [np.ascontiguousarray(H[s].imag, dtype=np.float64) for s in range(self.nspin)] \
            if np.iscomplexobj(H) else [None] * self.nspin
        self.s = OrcModel(self.ns, self.nspin, _ptr(self._re[0]), _ptr(self._im[0]),
                          _ptr(self._re[1]) if self.nspin == 2 else None,
                          _ptr(self._im[1]) if self.nspin == 2 else None, float(uloc), float(xmu), int(bool(hfmode)),
                          int(ed_filling))
        self.uloc, self.xmu = float(uloc), float(xmu)

    @property
    def ref(self):
        return C.byref(self.s)


def build_map(ns: int, n: int) -> np.ndarray:
    dim = lib().orc_build_map(ns, n, None)
    out = np.zeros(dim, dtype=np.int32)
    lib().orc_build_map(ns, n, _ptr(out))
    return out


def binomial(n, k):
    return lib().orc_binomial(n, k)


def binary_search(a: np.ndarray, value: int) -> int:
    a = np.ascontiguousarray(a, dtype=np.int32)
    return lib().orc_binary_search(_ptr(a), a.size, value)


def c_op(pos1: int, state: int):
    out, s = C.c_int64(), C.c_double()
    lib().orc_c(pos1, state, C.byref(out), C.byref(s))
    return out.value, s.value


def cdg_op(pos1: int, state: int):
    out, s = C.c_int64(), C.c_double()
    lib().orc_cdg(pos1, state, C.byref(out), C.byref(s))
    return out.value, s.value


def hop_csr(m: Model, spin: int, n: int):
    nnz = lib().orc_hop_csr(m.ref, spin, n, None, None, None)
    dim = binomial(m.ns, n)
    rp = np.zeros(dim + 1, dtype=np.int64)
    cols = np.zeros(max(nnz, 1), dtype=np.int32)
    vals = np.zeros(max(nnz, 1))
    lib().orc_hop_csr(m.ref, spin, n, _ptr(rp), _ptr(cols), _ptr(vals))
    return rp, cols[:nnz], vals[:nnz]


def direct_matvec_z(m: Model, nup, ndw, v):
    v = np.ascontiguousarray(v, dtype=np.complex128)
    hv = np.zeros_like(v)
    lib().orc_direct_matvec_z(m.ref, nup, ndw, _ptr(v), _ptr(hv))
    return hv


def direct_matvec_d(m: Model, nup, ndw, v, row_lo=0, row_hi=-1, out=None):
    v = np.ascontiguousarray(v, dtype=np.float64)
    hv = np.zeros_like(v) if out is None else out
    lib().orc_direct_matvec_d(m.ref, nup, ndw, _ptr(v), _ptr(hv), row_lo, row_hi)
    return hv


class Stored:
    """ed_buildh + spMatVec restatement, kept alive across calls."""

    def __init__(self, m: Model, nup: int, ndw: int):
        self.m = m
        self.h = lib().orc_stored_create(m.ref, nup, ndw)
        self.dim = lib().orc_stored_dim(self.h)

    def matvec_d(self, v, out=None):
        v = np.ascontiguousarray(v, dtype=np.float64)
        hv = np.empty_like(v) if out is None else out
        lib().orc_stored_matvec_d(self.h, _ptr(v), _ptr(hv))
        return hv

    def matvec_rows_d(self, v, hv, row_lo, row_hi):
        """Output rows idw in [row_lo,row_hi) of spMatVec (bounded CPU-baseline sample)."""
        lib().orc_stored_matvec_rows_d(self.h, _ptr(v), _ptr(hv), row_lo, row_hi)

    def matvec_sweeps_d(self, v, hv, row_lo, row_hi):
        """Output rows idw in [row_lo,row_hi) of spMatVec in the reference's loop order:
        diagonal, then the DW sweep (iup outer, stride DimUp), then the UP sweep."""
        lib().orc_stored_matvec_sweeps_d(self.h, _ptr(v), _ptr(hv), row_lo, row_hi)

    @property
    def dimdw(self):
        return lib().orc_stored_dimdw(self.h)

    def matvec_z(self, v):
        v = np.ascontiguousarray(v, dtype=np.complex128)
        hv = np.empty_like(v)
        lib().orc_stored_matvec_z(self.h, _ptr(v), _ptr(hv))
        return hv

    def tridiag(self, vvinit, nlanc, threshold=1e-9):
        a, b, n2 = np.zeros(nlanc), np.zeros(nlanc), C.c_double()
        v = np.ascontiguousarray(vvinit, dtype=np.float64)
        n = lib().orc_tridiag_d(self.h, _ptr(v), nlanc, threshold, _ptr(a), _ptr(b), C.byref(n2))
        return a, b, n2.value, n

    def ground_state(self, v0, maxit=300, tol=1e-14, want_vector=True):
        """Returns (E0, eigenvector or None, a[:m], b[:m]); without the vector the
        recurrence keeps three vectors only."""
        e0 = C.c_double()
        evec = np.zeros(self.dim) if want_vector else None
        a, b = np.zeros(maxit + 1), np.zeros(maxit + 1)
        v = np.ascontiguousarray(v0, dtype=np.float64)
        m = lib().orc_lanczos_gs_d(self.h, _ptr(v), maxit, tol, C.byref(e0), _ptr(evec), _ptr(a), _ptr(b))
        return e0.value, evec, a[:m], b[:m]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_stored_destroy(self.h)
            self.h = None


def dense_h(m: Model, nup, ndw) -> np.ndarray:
    D = binomial(m.ns, nup) * binomial(m.ns, ndw)
    H = np.zeros((D, D), order="F")
    lib().orc_dense_h(m.ref, nup, ndw, H.ctypes.data_as(C.c_void_p))
    return H


def tridiag_eigh(d, e):
    d = np.ascontiguousarray(d, dtype=np.float64)
    e = np.ascontiguousarray(e, dtype=np.float64)
    n = d.size
    w = np.zeros(n)
    Z = np.zeros((n, n), order="F")
    lib().orc_tridiag_eigh(n, _ptr(d), _ptr(e), _ptr(w), Z.ctypes.data_as(C.c_void_p))
    return w, Z


def apply_cop(ns, nupI, ndwI, op, site, spin, psi, out=None):
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    nupJ = nupI + (op if spin == 1 else 0)
    ndwJ = ndwI + (op if spin == 2 else 0)
    dimJ = binomial(ns, nupJ) * binomial(ns, ndwJ)
    acc = out is not None
    if out is None:
        out = np.zeros(dimJ)
    lib().orc_apply_cop_d(ns, nupI, ndwI, op, site, spin, _ptr(psi), _ptr(out), int(acc))
    return out


def apply_diagop(ns, nup, ndw, kind, site, psi, site2=0):
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = np.zeros_like(psi)
    lib().orc_apply_diagop_d(ns, nup, ndw, kind, site, site2, _ptr(psi), _ptr(out))
    return out


def apply_current(m: Model, nup, ndw, psi):
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = np.zeros_like(psi)
    lib().orc_apply_current_d(m.ref, nup, ndw, _ptr(psi), _ptr(out))
    return out


def poles_weights(a, b, norm2, ei, isign):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = a.size
    p, w = np.zeros(n), np.zeros(n)
    lib().orc_poles_weights(n, _ptr(a), _ptr(b), norm2, ei, isign, _ptr(p), _ptr(w))
    return p, w


def observables(ns, nup, ndw, psi, bw=1.0):
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = {k: np.zeros(ns) for k in ("dens", "dens_up", "dens_dw", "docc", "magz")}
    lib().orc_observables_d(ns, nup, ndw, _ptr(psi), bw, _ptr(out["dens"]), _ptr(out["dens_up"]),
                            _ptr(out["dens_dw"]), _ptr(out["docc"]), _ptr(out["magz"]))
    return out


def energy(m: Model, nup, ndw, psi, bw=1.0):
    """lanc_energy's Norb=1 terms for one real state: (ekin, epot incl. ehartree, eknot, ehartree)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = [C.c_double(0.0) for _ in range(4)]
    lib().orc_energy_d(m.ref, nup, ndw, _ptr(psi), bw, *[C.byref(x) for x in out])
    ekin, epot, eknot, ehartree = (x.value for x in out)
    return ekin, epot + ehartree, eknot, ehartree


def square_lattice(lx: int, ly: int, t: float = 1.0) -> np.ndarray:
    """Hij of the periodic lx x ly square lattice with nearest-neighbour hopping -t, sites
    numbered x + lx*y (the model mapping of the hot-path workloads)."""
    ns = lx * ly
    h = np.zeros((ns, ns))
    for y in range(ly):
        for x in range(lx):
            i = x + lx * y
            for j in ((x + 1) % lx + lx * y, x + lx * ((y + 1) % ly)):
                if j != i:
                    h[i, j] = h[j, i] = -t
    return h


def num_threads() -> int:
    return lib().orc_num_threads()


def random_vector(seed: int, n: int) -> np.ndarray:
    """The engine's documented start vector (splitmix64 counter stream), restated in numpy."""
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + i + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0
