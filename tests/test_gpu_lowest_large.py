"""edg_lowest_k on a larger sector than the 3x4 thermal workload: the 4x4 lattice at U=8,
sector (5,5) (D = 4368^2 = 19,079,424), lowest 4 levels to 1e-10.

The solver's second Gram-Schmidt pass comes from the Gram matrix of the basis rather than
from a second read of it. Here that is checked where the basis is long (hundreds of vectors)
and the vectors large: two solves from different start vectors give the same levels, the
returned vectors are orthonormal and are eigenvectors to the requested tolerance (their
residuals are recomputed with independent FP64 H x v), and the lowest level equals the
plain Lanczos ground state."""
import ctypes as C

import numpy as np
import pytest

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L

pytestmark = pytest.mark.gpu


def test_lowest_k_4x4_sector55():
    import torch
    model = E.Model(E.square_lattice(4, 4), uloc=8.0, xmu=4.0, hfmode=False)
    s = E.Sector(model, 5, 5)
    L.check(L.lib().edg_sector_set_stream(s.handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "st")
    assert s.dim == 19079424
    runs = []
    for seed in (11, 12):
        ev, vecs, resid, m = s.lowest_k(4, seed=seed, maxit=600, tol=1e-10)
        assert np.all(resid <= 1e-10 * np.maximum(1.0, np.abs(ev))), resid
        runs.append((ev, vecs, m))
    (ev, vecs, m), (ev2, _, _) = runs
    assert np.all(np.abs(ev - ev2) <= 1e-10 * np.abs(ev)), (ev, ev2)
    V = torch.tensor(vecs, device="cuda")
    gram = (V @ V.T).cpu().numpy()
    assert np.abs(gram - np.eye(4)).max() <= 1e-10
    HV = torch.empty_like(V)
    for r in range(4):
        torch.cuda.synchronize()
        L.check(L.lib().edg_hxv_dev_f64(s.handle, C.c_void_p(V[r].data_ptr()), C.c_void_p(HV[r].data_ptr())), "hxv")
    torch.cuda.synchronize()
    res = torch.linalg.vector_norm(HV - torch.tensor(ev, device="cuda")[:, None] * V, dim=1).cpu().numpy()
    assert np.all(res <= 1e-9 * np.maximum(1.0, np.abs(ev))), res
    e0, _, _ = E.sp_lanc_eigh(s, seed=3, maxit=600, tol=1e-13, want_vector=False)
    assert abs(e0 - ev[0]) <= 1e-10 * abs(e0)
    del V, HV
    s.delete()
    torch.cuda.empty_cache()
