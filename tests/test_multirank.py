"""Multi-rank logic of bench.py on CPU: world size 2, gloo backend.

Each rank simulates its own realisation (seed + rank) with no collective on
the data path; the job's time is the maximum over ranks and its work the sum.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import importlib
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ks = importlib.import_module("kessler-syndrom-simulation_b200")
    st, _, _ = ks.generate_population(bench.realisation_seed(100, rank), 500, 800, 2, 3600.0)
    device_ms = [12.5, 20.0][rank]
    work = [1000.0, 3000.0][rank]
    out[rank] = (float(st[:, 0].sum()), bench.max_over_ranks(dist, device_ms), bench.sum_over_ranks(dist, work))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (s0, m0, w0), (s1, m1, w1) = out[0], out[1]
    assert s0 != s1, "ranks must simulate different realisations"
    assert m0 == m1 == 20.0, "job time = slowest rank"
    assert w0 == w1 == 4000.0, "job work = sum over ranks"
    # weak-scaling throughput the bench reports: total work / slowest time
    assert np.isclose(w0 / (m0 * 1e-3), 2e5)


def test_single_rank_reductions_are_identity():
    import bench
    assert bench.max_over_ranks(None, 3.0) == 3.0
    assert bench.sum_over_ranks(None, 4.0) == 4.0
    assert bench.realisation_seed(7, 0) == 7
