"""The allocation-free tridiagonalisation (edg_tridiag_dev_f64_noalloc) against the regular
entry point (edg_tridiag_dev_f64).

It serves callers that cannot call cudaMalloc themselves (device memory owned by another
runtime's pool, or loops that must not wait on the allocator): all its scratch lives in a
fixed file-scope device array. Two calls in a row with different start vectors check that
the contents the array keeps from the previous call never leak into the next result.
This file sorts last so a first-failure run has already run every other test; it needs no
state from them and passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-9  # the FP64 Lanczos-coefficient tolerance of the parity tests


def _run(fn, sector, dv, nlanc):
    a = np.zeros(nlanc)
    b = np.zeros(nlanc)
    n2 = C.c_double()
    ns = C.c_int()
    if fn == "noalloc":
        st = L.lib().edg_tridiag_dev_f64_noalloc(sector.handle, C.c_void_p(dv.data_ptr()), nlanc, 1e-9,
                                                 a.ctypes.data_as(L._pd), b.ctypes.data_as(L._pd), C.byref(n2),
                                                 C.byref(ns))
    else:
        st = L.lib().edg_tridiag_dev_f64(sector.handle, C.c_void_p(dv.data_ptr()), nlanc, 1e-9, E.EDG_PREC_F64,
                                         a.ctypes.data_as(L._pd), b.ctypes.data_as(L._pd), C.byref(n2),
                                         C.byref(ns))
    L.check(st, fn)
    return a, b, n2.value, ns.value


@pytest.mark.parametrize("lat,nup,ndw,nlanc", [("ring8", 4, 4, 60), ("sq3x4", 6, 6, 40)])
def test_noalloc_matches_regular_entry_two_calls(lat, nup, ndw, nlanc):
    import torch
    h = E.ring(8) if lat == "ring8" else E.square_lattice(3, 4)
    model = E.Model(h, uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(model, nup, ndw)
    for seed in (11, 12):  # two calls in a row
        v = E.random_vector(seed, s.dim)
        dv = torch.tensor(v, dtype=torch.float64, device="cuda")
        a0, b0, n20, k0 = _run("regular", s, dv, nlanc)
        a1, b1, n21, k1 = _run("noalloc", s, dv, nlanc)
        assert k1 == k0
        assert abs(n21 - n20) <= TOL * n20
        assert np.abs(a1 - a0).max() <= TOL
        assert np.abs(b1 - b0).max() <= TOL
        assert b1[0] == 0.0


def test_noalloc_rejects_oversized_sector():
    import torch
    model = E.Model(E.square_lattice(4, 4), uloc=8.0, xmu=4.0, hfmode=False)
    s = E.Sector(model, 7, 6)  # 11440 * 8008 states > 2^20
    dv = torch.zeros(8, dtype=torch.float64, device="cuda")
    a = np.zeros(4)
    b = np.zeros(4)
    n2, ns = C.c_double(), C.c_int()
    st = L.lib().edg_tridiag_dev_f64_noalloc(s.handle, C.c_void_p(dv.data_ptr()), 4, 1e-9, a.ctypes.data_as(L._pd),
                                             b.ctypes.data_as(L._pd), C.byref(n2), C.byref(ns))
    assert st == L.EDG_ERR_ARG
