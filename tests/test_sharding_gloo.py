"""Trajectory sharding over ranks (one process per GPU in production), exercised with two
gloo ranks on CPU: rank r owns global trajectories r*m .. r*m+m-1 (tr_base = r*m), so the
sharded ensemble draws exactly the numbers of one run of all trajectories, and the ensemble
observable is the all-reduced sum of the shards (the one exchange of the path)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle_py as O
from tests.helpers import dimer_problem

N_TR, WORLD, PERIODS = 12, 2, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ensemble(P, n, tr_base):
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, seed=7, record=1, tr_base=tr_base)
    ens.init(0, 0)
    assert ens.run_periods(PERIODS) == 0
    return ens


def _rank(rank, port, out):
    import torch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        P = dimer_problem(8, deep=12)
        m = N_TR // WORLD
        ens = _ensemble(P, m, tr_base=rank * m)
        ob = ens.observables()
        local = torch.tensor([float(np.sum(8 - 2.0 * ob["mean"])), float(m)], dtype=torch.float64)
        dist.all_reduce(local)
        parts = [torch.zeros(m, P["d"], 2, dtype=torch.float64) for _ in range(WORLD)]
        dist.all_gather(parts, torch.from_numpy(np.stack([ens.phi.real, ens.phi.imag], -1)))
        if rank == 0:
            out.put((local.numpy(), np.concatenate([p.numpy() for p in parts])))
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_equals_single_run():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    reduced, psi = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    P = dimer_problem(8, deep=12)
    full = _ensemble(P, N_TR, tr_base=0)
    assert np.array_equal(psi[..., 0] + 1j * psi[..., 1], full.phi)  # shards are bit-identical
    ob = full.observables()
    assert reduced[1] == N_TR
    assert np.isclose(reduced[0] / reduced[1], np.mean(8 - 2.0 * ob["mean"]), rtol=1e-12)
