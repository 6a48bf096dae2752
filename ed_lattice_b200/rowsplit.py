"""Row-split stored H x v and Lanczos ground state, for sectors beyond one GPU's memory.

A vector of the sector (element iup + idw*DimUp) is split over the ranks of a process group by
rows idw, as the reference's MPI "DW split" does (src/DIAG/HAMILTONIAN.f90:107-121: the first
mod(DimDw, P) ranks take one row more). The sector object on each rank holds only the
O(DimUp + DimDw) tables. One H x v, after spMatVec_mpi (src/DIAG/HAMILTONIAN_STORED_HxV.f90:
227-313):

1. transpose: every rank sends to rank q the columns of q (DimUp split by the same rule) of its
   own rows, in one all_to_all_single; rank q then holds all DimDw rows of its columns,
   row-major (the reference: MPI_AllToAllV and a local transpose,
   src/DIAG/HAMILTONIAN_COMMON.f90:53-118);
2. edg_hxv_cols_dev_*: the diagonal and H_dw on those columns;
3. the transpose back, one all_to_all_single;
4. edg_hxv_rows_dev_*: += H_up on the rank's own rows.

Every element is computed in the order of edg_hxv_dev_*, so the split H x v equals the
one-GPU H x v bit for bit. The packing around the transposes is strided tensor copies; the
library's kernels run on the caller's current CUDA stream (the sector's stream is set to
it), so the copies, the collectives and the kernels need no other synchronisation.

`comm` is a torch.distributed process group (NCCL between GPUs), None for one rank, or any
object with `rank`, `size`, `all_to_all_single(out, inp, out_splits, in_splits)` and
`all_reduce_sum(tensor)`. The H x v itself can be replaced (`cols_fn`, `rows_fn`) to drive
the exchange with host tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _edgpu_lib as L
from .edlat import tridiag_lowest


def split_sizes(n: int, p: int) -> list[int]:
    """The reference's split of n items over p ranks: the first n mod p ranks take one more."""
    return [n // p + (1 if r < n % p else 0) for r in range(p)]


def _starts(sizes: list[int]) -> list[int]:
    out, o = [], 0
    for x in sizes:
        out.append(o)
        o += x
    return out


class _TorchGroup:
    """torch.distributed process group (or a single rank) behind the small interface above."""

    def __init__(self, group):
        import torch.distributed as dist

        self.group = group
        self.rank = dist.get_rank(group) if group is not None else 0
        self.size = dist.get_world_size(group) if group is not None else 1

    def all_to_all_single(self, out, inp, out_splits, in_splits):
        if self.group is None:
            out.copy_(inp)
            return
        import torch.distributed as dist

        dist.all_to_all_single(out, inp, output_split_sizes=out_splits, input_split_sizes=in_splits,
                               group=self.group)

    def all_reduce_sum(self, t):
        if self.group is None:
            return
        import torch.distributed as dist

        dist.all_reduce(t, group=self.group)


def _group(comm):
    if comm is None or not all(hasattr(comm, a) for a in ("rank", "size", "all_to_all_single", "all_reduce_sum")):
        return _TorchGroup(comm)
    return comm


class RowSplitHxv:
    """H x v of `sector` on row-split vectors: this rank holds rows [row0, row0 + nrows), a
    contiguous (nrows * DimUp) tensor of `dtype` (float64 or float32)."""

    def __init__(self, sector, comm=None, dtype=torch.float64, device=None, cols_fn=None, rows_fn=None):
        self.sector = sector
        self.g = _group(comm)
        self.rank, self.size = self.g.rank, self.g.size
        self.dtype = dtype
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.dimup, self.dimdw = sector.dimup, sector.dimdw
        self.rows = split_sizes(self.dimdw, self.size)
        self.cols = split_sizes(self.dimup, self.size)
        self.row0s, self.col0s = _starts(self.rows), _starts(self.cols)
        self.nrows, self.row0 = self.rows[self.rank], self.row0s[self.rank]
        self.ncols, self.col0 = self.cols[self.rank], self.col0s[self.rank]
        # transpose splits (elements): to rank q my rows x q's columns; from rank s its rows x my columns
        self.to_cols = [self.nrows * c for c in self.cols]
        self.from_rows = [r * self.ncols for r in self.rows]
        z = dict(dtype=dtype, device=self.device)
        self.send = torch.empty(self.nrows * self.dimup, **z)
        self.colv = torch.empty(self.dimdw * self.ncols, **z)   # all rows of my columns
        self.colh = torch.empty(self.dimdw * self.ncols, **z)
        self.recv = torch.empty(self.nrows * self.dimup, **z)
        if cols_fn is None or rows_fn is None:
            if getattr(sector, "cplx", False) or sector.form != L.EDG_FORM_STORED:
                raise L.EdgError(L.EDG_ERR_UNSUPPORTED, "RowSplitHxv", "real stored-form sectors only")
            sector.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
            f64 = dtype == torch.float64
            lib = L.lib()
            fc = lib.edg_hxv_cols_dev_f64 if f64 else lib.edg_hxv_cols_dev_f32
            fr = lib.edg_hxv_rows_dev_f64 if f64 else lib.edg_hxv_rows_dev_f32
            h = sector.handle
            cols_fn = cols_fn or (lambda c0, nc, v, hv: L.check(fc(h, c0, nc, C.c_void_p(v.data_ptr()),
                                                                   C.c_void_p(hv.data_ptr())), "edg_hxv_cols_dev"))
            rows_fn = rows_fn or (lambda r0, nr, v, hv: L.check(fr(h, r0, nr, C.c_void_p(v.data_ptr()),
                                                                  C.c_void_p(hv.data_ptr())), "edg_hxv_rows_dev"))
        self.cols_fn, self.rows_fn = cols_fn, rows_fn

    def local_size(self) -> int:
        return self.nrows * self.dimup

    # The three stages of one H x v; apply() runs them with the two transposes between.
    def stage(self, v: torch.Tensor) -> None:
        """Pack my rows by destination column block: block q is (nrows x cols[q]) row-major."""
        vr = v.view(self.nrows, self.dimup)
        o = 0
        for q in range(self.size):
            n = self.to_cols[q]
            if n:
                self.send[o:o + n].view(self.nrows, self.cols[q]).copy_(vr[:, self.col0s[q]:self.col0s[q] + self.cols[q]])
            o += n

    def apply_cols(self) -> None:
        """diag + H_dw on all rows of my columns (colv, row-major, row length ncols)."""
        if self.ncols:
            self.cols_fn(self.col0, self.ncols, self.colv, self.colh)

    def finish(self, v: torch.Tensor, hv: torch.Tensor) -> None:
        """Unpack the transposed-back result into my rows, then += H_up on them."""
        hr = hv.view(self.nrows, self.dimup)
        o = 0
        for q in range(self.size):
            n = self.to_cols[q]
            if n:
                hr[:, self.col0s[q]:self.col0s[q] + self.cols[q]].copy_(self.recv[o:o + n].view(self.nrows, self.cols[q]))
            o += n
        if self.nrows:
            self.rows_fn(self.row0, self.nrows, v, hv)

    def apply(self, v: torch.Tensor, hv: torch.Tensor) -> None:
        """hv = H v on this rank's rows (v, hv: contiguous nrows*DimUp tensors)."""
        self.stage(v)
        self.g.all_to_all_single(self.colv, self.send, self.from_rows, self.to_cols)
        self.apply_cols()
        self.g.all_to_all_single(self.recv, self.colh, self.to_cols, self.from_rows)
        self.finish(v, hv)

    def dot(self, x: torch.Tensor, y: torch.Tensor) -> float:
        """<x, y> over all ranks (FP64 accumulation; one all_reduce of a scalar)."""
        t = torch.dot(x.double(), y.double()).reshape(1)
        self.g.all_reduce_sum(t)
        return float(t.item())


def ground_state(hx: RowSplitHxv, v0: torch.Tensor, maxit: int = 512, tol: float = 1e-12,
                 want_vector: bool = True):
    """Lowest eigenpair of the sector with the row-split H x v: the three-term Lanczos
    recurrence of sp_lanc_eigh (src/DIAG/DIAG.f90:185-217; a_j = <v_j|H|v_j>, b_{j+1} = |w|,
    no reorthogonalisation) on this rank's rows, with every dot summed over the ranks. The
    lowest Ritz value of the tridiagonal (edg_tridiag_lowest) is tested every step; the run
    stops when its residual b_{m+1} |z_m| falls below tol * max(1, |E0|). With want_vector, a
    second pass of the same recurrence forms x = sum_j z_j v_j (the reference's
    eigenvector pass). Returns (E0, steps, x or None): x holds this rank's rows."""
    dt = hx.dtype
    u = v0.to(dt).clone()
    nrm = hx.dot(u, u) ** 0.5
    if nrm == 0.0:
        raise ValueError("ground_state: zero start vector")
    u /= nrm
    start = u.clone()
    up = torch.zeros_like(u)
    w = torch.empty_like(u)
    a, b = [], [0.0]
    e0, m = 0.0, 0
    for j in range(maxit):
        hx.apply(u, w)
        if j > 0:
            w.add_(up, alpha=-b[j])
        aj = hx.dot(u, w)
        w.add_(u, alpha=-aj)
        bj = hx.dot(w, w) ** 0.5
        a.append(aj)
        b.append(bj)
        m = j + 1
        th, zl = tridiag_lowest(np.array(a), np.array(b[:m]), 1)
        e0 = float(th[0])
        if bj * abs(float(zl[0])) <= tol * max(1.0, abs(e0)) or bj == 0.0:
            break
        up, u = u, w / bj
    if not want_vector:
        return e0, m, None
    # lowest eigenvector of the m x m tridiagonal (host LAPACK through numpy), then the second pass
    t = np.diag(np.array(a[:m])) + np.diag(np.array(b[1:m]), 1) + np.diag(np.array(b[1:m]), -1)
    z0 = np.linalg.eigh(t)[1][:, 0]
    u = start.clone()
    up = torch.zeros_like(u)
    x = torch.zeros(u.shape, dtype=torch.float64, device=u.device)
    for j in range(m):
        x.add_(u.double(), alpha=float(z0[j]))
        if j == m - 1:
            break
        hx.apply(u, w)
        if j > 0:
            w.add_(up, alpha=-b[j])
        w.add_(u, alpha=-a[j])
        up, u = u, w / b[j + 1]
    xn = hx.dot(x, x) ** 0.5
    return e0, m, (x / xn).to(dt)
