"""The multi-rank timing logic of bench.py on CPU: two gloo ranks (the GPU run
uses the same class with NCCL), a barrier, then MAX and SUM reductions of
per-rank timings and unit counts."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    r, w, local = bench.dist_env()
    d = bench.Dist(w, "gloo")
    d.barrier()
    got = (r, w, local, d.max(1.5 + r), d.sum(10.0 * (r + 1)))
    d.close()
    q.put(got)


def test_two_gloo_ranks_reduce_timings():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[:3] for o in out] == [(0, 2, 0), (1, 2, 1)]
    for o in out:
        assert o[3] == pytest.approx(2.5) and o[4] == pytest.approx(30.0)


def test_single_rank_needs_no_process_group():
    import bench

    d = bench.Dist(1, "gloo")
    assert d.max(3.0) == 3.0 and d.sum(4.0) == 4.0
    d.barrier()
    d.close()
