"""Row-split H x v and ground state over gloo ranks on the host (no GPU): the transposes,
splits and reductions of ed_lattice_b200.rowsplit, with the two slab H x v stages replaced by
host operators of the same form (diag + H_dw x I on column slabs, I x H_up on row slabs),
against the dense operator diag + kron(H_dw, I) + kron(I, H_up) on one process."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _Shape:
    form = 0

    def __init__(self, dimup, dimdw):
        self.dimup, self.dimdw = dimup, dimdw


def _operators(dimup, dimdw):
    rng = np.random.default_rng(11)
    hu = rng.normal(size=(dimup, dimup))
    hd = rng.normal(size=(dimdw, dimdw))
    hu, hd = hu + hu.T, hd + hd.T
    diag = rng.normal(size=(dimdw, dimup)) * 3.0
    h = np.diag(diag.ravel()) + np.kron(hd, np.eye(dimup)) + np.kron(np.eye(dimdw), hu)
    return hu, hd, diag, h


def _worker(rank, world, port, dimup, dimdw):
    import datetime

    import torch
    import torch.distributed as dist

    from ed_lattice_b200.rowsplit import RowSplitHxv, ground_state, split_sizes

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        hu, hd, diag, h = _operators(dimup, dimdw)

        def cols_fn(c0, nc, v, hv):
            x = v.view(dimdw, nc).numpy()
            hv.view(dimdw, nc).copy_(torch.from_numpy(diag[:, c0:c0 + nc] * x + hd @ x))

        def rows_fn(r0, nr, v, hv):
            hv.view(nr, dimup).add_(torch.from_numpy(v.view(nr, dimup).numpy() @ hu.T))

        hx = RowSplitHxv(_Shape(dimup, dimdw), comm=dist.group.WORLD, device="cpu", cols_fn=cols_fn,
                         rows_fn=rows_fn)
        assert hx.rows == split_sizes(dimdw, world) and hx.nrows == hx.rows[rank]
        lo, hi = hx.row0 * dimup, (hx.row0 + hx.nrows) * dimup
        v = np.random.default_rng(4).normal(size=dimup * dimdw)
        hv = torch.empty(hx.local_size(), dtype=torch.float64)
        hx.apply(torch.from_numpy(v[lo:hi].copy()), hv)
        assert np.allclose(hv.numpy(), (h @ v)[lo:hi], rtol=0, atol=1e-12)
        # ground state through the split recurrence
        w, z = np.linalg.eigh(h)
        e0, steps, x = ground_state(hx, torch.from_numpy(v[lo:hi].copy()), maxit=200, tol=1e-12)
        assert abs(e0 - w[0]) <= 1e-10 * abs(w[0]), (e0, w[0], steps)
        xs = [None] * world
        dist.all_gather_object(xs, x.numpy())
        xf = np.concatenate(xs)
        assert abs(abs(xf @ z[:, 0]) - 1.0) < 1e-9
        assert np.linalg.norm(h @ xf - e0 * xf) < 1e-7
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dimup,dimdw", [(2, 7, 5), (3, 8, 7), (3, 4, 2)])
def test_row_split_matches_dense(world, dimup, dimdw):
    """Uneven splits; (3, 4, 2) leaves one rank without rows (the reference shrinks its
    communicator there, src/DIAG/HAMILTONIAN.f90:79-99; here that rank holds an empty slab)."""
    mp.spawn(_worker, args=(world, _free_port(), dimup, dimdw), nprocs=world, join=True)
