"""Sector sharding of the diagonalisation driver over ranks (no GPU): two gloo ranks on the
host, each solving half of the sectors with the oracle injected as the eigensolver, must
build the same state list, partition function and observables as one process."""
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


def _worker(rank, world, port, temp, finite_temp):
    import datetime

    import torch.distributed as dist

    import ed_lattice_b200 as E
    from ed_lattice_b200.diag import DiagParams, diagonalize_lattice, lanc_observables, partition_function
    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(3)
        H = E.ring(4).astype(float)
        H[np.diag_indices(4)] = np.round(rng.uniform(-1, 1, 4) * 2**16) / 2**16
        m = E.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
        om = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
        calls = []

        def solver(model, nup, ndw, neigen, lanc_solve, params, seed):
            calls.append((nup, ndw))
            w, z = np.linalg.eigh(O.dense_h(om, nup, ndw))
            return w[:neigen], z[:, :neigen].T.copy()

        def observer(model, isector, vec, bw):
            return O.observables(model.ns, model.get_nup(isector), model.get_ndw(isector), vec, bw)

        def params():
            return DiagParams(finite_temp=finite_temp, temp=temp, lanc_nstates_sector=36 if finite_temp else 2)

        p1 = params()
        sl1, eig1 = diagonalize_lattice(m, p1, solver=solver)
        z1 = partition_function(sl1, p1)
        o1 = lanc_observables(m, sl1, z1, p1, observer=observer)
        calls.clear()
        p2 = params()
        sl2, eig2 = diagonalize_lattice(m, p2, solver=solver, comm=dist.group.WORLD)
        # each rank solved only its share of the 25 sectors
        assert len(calls) == (13 if rank == 0 else 12)
        z2 = partition_function(sl2, p2)
        o2 = lanc_observables(m, sl2, z2, p2, observer=observer, comm=dist.group.WORLD)
        assert [(s.e, s.sector) for s in sl1.states] == [(s.e, s.sector) for s in sl2.states]
        assert all((s.vec is not None) == (s.owner == rank) for s in sl2.states)
        assert [(i, list(e)) for i, e, _ in eig1] == [(i, list(e)) for i, e, _ in eig2]
        assert z1 == z2
        for k in o1:
            assert np.allclose(o1[k], o2[k], rtol=0, atol=1e-14), k
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("temp,finite_temp", [(0.3, True), (0.001, False)])
def test_two_ranks_match_one_process(temp, finite_temp):
    mp.spawn(_worker, args=(2, _free_port(), temp, finite_temp), nprocs=2, join=True)
