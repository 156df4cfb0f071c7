"""The multi-GPU replica path's host logic (diffsoup_b200/replicas.py, used by
bench.py --gpus N) on two gloo ranks on CPU: rendezvous, max-over-ranks
timing, whole-job throughput, and per-rank benchmark inputs that differ
between ranks while keeping their shapes."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from diffsoup_b200 import replicas

    r = replicas.init(backend="gloo", timeout_s=60)
    ms = 10.0 + 5.0 * r.rank  # rank 1 is the slower one
    replicas.barrier(r)
    ms_max = replicas.max_over_ranks(r, ms)
    thr = replicas.job_throughput(r, 8 * 100, ms_max)
    import bench

    _, _, sets = bench.make_inputs(r.rank, nviews=2)
    out[rank] = (r.world, ms_max, thr, [x.shape for x in sets[0]], float(sets[0][2][:1000].sum()))
    replicas.shutdown(r)


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, out)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    (w0, m0, t0, s0, c0), (w1, m1, t1, s1, c1) = out[0], out[1]
    assert w0 == w1 == 2
    assert m0 == m1 == 15.0  # the job's time is the slowest rank's
    assert t0 == t1 == 8 * 100 * 2 / 0.015
    assert s0 == s1  # same workload shape on every rank ...
    assert not np.isclose(c0, c1)  # ... with the rank's own targets
