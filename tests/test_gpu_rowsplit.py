"""Row-split H x v (edg_hxv_cols_dev_* + edg_hxv_rows_dev_*, ed_lattice_b200.rowsplit) on one
GPU: the ranks are threads of this process on one CUDA stream, and the collectives are copies
between their buffers at a barrier (no kernel waits on another rank). The split H x v must
equal the one-GPU H x v bit for bit, and the split ground state the one-GPU E0."""
import threading

import numpy as np
import pytest
import torch

import ed_lattice_b200 as E
from ed_lattice_b200 import _edgpu_lib as L
from ed_lattice_b200.rowsplit import RowSplitHxv, ground_state

pytestmark = pytest.mark.gpu


class _Emulated:
    """`size` ranks in one process (one thread each); all CUDA work on one stream, so the
    barriers order the copies of the collectives after every rank's producing work."""

    def __init__(self, size):
        self.size = size
        self.barrier = threading.Barrier(size, timeout=120)
        self.slots = [None] * size

    def rank(self, r):
        return _Rank(self, r)


class _Rank:
    def __init__(self, em, r):
        self.em, self.rank, self.size = em, r, em.size

    def all_to_all_single(self, out, inp, out_splits, in_splits):
        em = self.em
        em.slots[self.rank] = (inp, list(in_splits))
        em.barrier.wait()
        o = 0
        for s in range(self.size):
            sinp, ss = em.slots[s]
            off, n = sum(ss[:self.rank]), ss[self.rank]
            assert n == out_splits[s]
            if n:
                out[o:o + n].copy_(sinp[off:off + n])
            o += n
        em.barrier.wait()

    def all_reduce_sum(self, t):
        em = self.em
        em.slots[self.rank] = t.clone()
        em.barrier.wait()
        total = sum(em.slots[s] for s in range(self.size))
        em.barrier.wait()
        t.copy_(total)


def _run_ranks(size, fn):
    """fn(rank_comm) in `size` threads on one shared stream; returns the results by rank."""
    em = _Emulated(size)
    stream = torch.cuda.Stream()
    out, err = [None] * size, []

    def body(r):
        try:
            with torch.cuda.stream(stream):
                out[r] = fn(em.rank(r))
        except BaseException as e:  # noqa: BLE001 -- reported below
            err.append(e)
            em.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if err:
        raise err[0]
    torch.cuda.synchronize()
    return out


CASES = [("ring8_44", lambda: (E.ring(8), 4.0, 4, 4)), ("sq3x4_66", lambda: (E.square_lattice(3, 4), 4.0, 6, 6))]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("ranks", [1, 3, 4])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_split_hxv_bit_exact(case, ranks, dtype):
    h, u, nup, ndw = case[1]()
    model = E.Model(h, uloc=u, xmu=u / 2, hfmode=False)
    s = E.Sector(model, nup, ndw)
    prec = L.EDG_PREC_F64 if dtype == torch.float64 else L.EDG_PREC_F32
    s.set_kernels(0, prec)  # the two-pass pair, which the split form uses
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    v = (torch.rand(s.dim, device="cuda", generator=g, dtype=torch.float64) - 0.5).to(dtype)
    ref = torch.empty_like(v)
    f = L.lib().edg_hxv_dev_f64 if dtype == torch.float64 else L.lib().edg_hxv_dev_f32
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    L.check(f(s.handle, v.data_ptr(), ref.data_ptr()), "hxv")
    torch.cuda.synchronize()

    def rank_fn(comm):
        hx = RowSplitHxv(s, comm=comm, dtype=dtype)
        lo, n = hx.row0 * s.dimup, hx.local_size()
        hv = torch.empty(n, dtype=dtype, device="cuda")
        hx.apply(v[lo:lo + n].contiguous(), hv)
        return hv

    parts = _run_ranks(ranks, rank_fn)
    assert torch.equal(torch.cat(parts), ref)
    s.delete()


def test_split_ground_state_matches_one_gpu():
    """E0 and the vector of the 3x4 (6,6) sector over 3 emulated ranks against edg_ground_state."""
    model = E.Model(E.square_lattice(3, 4), uloc=4.0, xmu=2.0, hfmode=False)
    s = E.Sector(model, 6, 6)
    e_ref, _, _ = E.sp_lanc_eigh(s, seed=5, tol=1e-14, want_vector=False)
    v0 = torch.from_numpy(E.random_vector(9, s.dim)).cuda()

    def rank_fn(comm):
        hx = RowSplitHxv(s, comm=comm)
        lo, n = hx.row0 * s.dimup, hx.local_size()
        e0, steps, x = ground_state(hx, v0[lo:lo + n].contiguous(), maxit=400, tol=1e-12)
        hv = torch.empty_like(x)
        hx.apply(x, hv)
        r2 = hx.dot(hv - e0 * x, hv - e0 * x)
        return e0, steps, r2

    out = _run_ranks(3, rank_fn)
    e0, steps, r2 = out[0]
    assert all(o[0] == e0 for o in out)
    assert abs(e0 - e_ref) <= 1e-10 * abs(e_ref), (e0, e_ref, steps)
    assert r2 ** 0.5 < 1e-5
    s.delete()


def test_slab_entry_checks():
    model = E.Model(E.ring(6), uloc=2.0, xmu=1.0, hfmode=False)
    s = E.Sector(model, 3, 3)
    x = torch.zeros(s.dim, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(L.EdgError):
        L.check(L.lib().edg_hxv_rows_dev_f64(s.handle, s.dimdw - 1, 2, x.data_ptr(), y.data_ptr()), "rows")
    with pytest.raises(L.EdgError):
        L.check(L.lib().edg_hxv_cols_dev_f64(s.handle, -1, 1, x.data_ptr(), y.data_ptr()), "cols")
    L.check(L.lib().edg_hxv_cols_dev_f64(s.handle, 0, 0, x.data_ptr(), y.data_ptr()), "empty slab")
    s.delete()
