"""Multi-process layout on CPU (gloo, world size 2): column sharding is
exact and the time step is the global minimum (calc_timestep.f90:144-145)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gitm_b200 import abi, synthetic
from gitm_b200.parallel import global_dt, shard_member, shard_range


def test_shard_range_covers():
    for n in (0, 1, 5, 64800, 101):
        for w in (1, 2, 3, 8):
            spans = [shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p = abi.default_params()
    m = synthetic.make_member(10, 20, seed=51)
    part = shard_member(m, rank, world)
    local = oracle.cfl_dt(part, p, 0.75)
    dt = global_dt(local)
    oracle.advance(part, p, 2.0, 1, nthreads=1)
    import torch
    t = torch.from_numpy(np.ascontiguousarray(part.ndensity_s))
    gathered = [None] * world
    dist.all_gather_object(gathered, (shard_range(m.n_cols, rank, world), t.numpy()))
    if rank == 0:
        out.put((dt, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_match_single_process(oracle_lib):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    dt, gathered = q.get(timeout=120)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p = abi.default_params()
    m = synthetic.make_member(10, 20, seed=51)
    assert dt == oracle_lib.cfl_dt(m, p, 0.75)
    oracle_lib.advance(m, p, 2.0, 1, nthreads=1)
    for (c0, c1), ns in gathered:
        np.testing.assert_array_equal(ns, m.ndensity_s[..., c0:c1])
