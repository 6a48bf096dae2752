"""The allocation-free tridiagonalisation (edg_tridiag_dev_f64_noalloc) against the regular
entry point (edg_tridiag_dev_f64).

It serves callers that cannot call cudaMalloc themselves (device memory owned by another
runtime's pool, or loops that must not wait on the allocator): all its scratch lives in a
fixed file-scope device array that every call shares and that keeps the last call's
contents. Each case makes two calls in a row, the second on a SMALLER sector than the
first, so that values a larger earlier call left in the array beyond the second sector's
length could only stay out of its result if the call never reads them; both H x v forms
(stored and direct) and a complex-Hij sector (vectors of (re, im) pairs, twice the
dimension in reals) are covered.
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


def flux_ring(ns, phi, t=1.0):
    """Ring threaded by flux phi: Hij(i, i+1) = -t e^{i phi/ns} (Hermitian, complex)."""
    H = np.zeros((ns, ns), complex)
    for i in range(ns):
        j = (i + 1) % ns
        H[i, j] = -t * np.exp(1j * phi / ns)
        H[j, i] = np.conj(H[i, j])
    return H


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


def _start(sector, seed):
    import torch
    v = E.random_vector(seed, sector.vlen)  # complex sectors: vlen reals = dim (re, im) pairs
    return torch.tensor(v, dtype=torch.float64, device="cuda")


def _compare(sector, seed, nlanc):
    dv = _start(sector, seed)
    a0, b0, n20, k0 = _run("regular", sector, dv, nlanc)
    a1, b1, n21, k1 = _run("noalloc", sector, dv, nlanc)
    assert k1 == k0
    assert abs(n21 - n20) <= TOL * n20
    assert np.abs(a1 - a0).max() <= TOL
    assert np.abs(b1 - b0).max() <= TOL
    assert b1[0] == 0.0


@pytest.mark.parametrize("form", [E.EDG_FORM_STORED, E.EDG_FORM_DIRECT], ids=["stored", "direct"])
def test_noalloc_matches_regular_entry_two_calls(form):
    """sq3x4 (6,6) (853,776 states), then ring8 (4,4) (4,900 states) in the same array."""
    big = E.Sector(E.Model(E.square_lattice(3, 4), uloc=4.0, xmu=2.0, hfmode=False), 6, 6, form)
    small = E.Sector(E.Model(E.ring(8), uloc=4.0, xmu=2.0, hfmode=False), 4, 4, form)
    _compare(big, 11, 40)
    _compare(small, 12, 60)
    big.delete()
    small.delete()


def test_noalloc_complex_sector():
    """A flux-threaded 10-site ring (complex Hij), sector (5,4): 252 x 210 = 52,920 complex
    states, 105,840 reals per vector; then the 8-site ring (4,3) in the same array."""
    s1 = E.Sector(E.Model(flux_ring(10, 0.9), uloc=4.0, xmu=2.0, hfmode=False), 5, 4)
    s2 = E.Sector(E.Model(flux_ring(8, 0.7), uloc=4.0, xmu=2.0, hfmode=False), 4, 3)
    assert s1.cplx and s2.cplx
    _compare(s1, 21, 50)
    _compare(s2, 22, 50)
    s1.delete()
    s2.delete()


def test_noalloc_rejects_oversized_vector():
    """Complex 3x4 sector (6,6): 853,776 states, but 1,707,552 reals per vector > 2^20."""
    import torch
    H = E.square_lattice(3, 4).astype(complex)
    H[0, 1] *= np.exp(0.3j)
    H[1, 0] = np.conj(H[0, 1])
    s = E.Sector(E.Model(H, uloc=4.0, xmu=2.0, hfmode=False), 6, 6)
    assert s.cplx and s.vlen == 2 * 853776
    dv = torch.zeros(8, dtype=torch.float64, device="cuda")
    a = np.zeros(4)
    b = np.zeros(4)
    n2, ns = C.c_double(), C.c_int()
    st = L.lib().edg_tridiag_dev_f64_noalloc(s.handle, C.c_void_p(dv.data_ptr()), 4, 1e-9, a.ctypes.data_as(L._pd),
                                             b.ctypes.data_as(L._pd), C.byref(n2), C.byref(ns))
    assert st == L.EDG_ERR_ARG
    s.delete()
