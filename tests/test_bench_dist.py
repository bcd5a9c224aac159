"""The multi-process path of bench.py on CPU: two gloo ranks run the same rendezvous and
reductions as the GPU run (replicas, no data-path collective). The job time is the slowest
rank's, and the whole-job throughput counts every rank's cubes (weak scaling)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, local, dist = bench.dist_setup(world, backend="gloo")
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * r, dist)          # rank 1 is the slow one
        dist.barrier()
        v = bench.job_mvox_per_s(w, 512 ** 3, 10, t)
        q.put((r, w, local, t, v))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
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
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 15.0 for o in out)                       # both ranks see the slowest time
    want = 2 * 512 ** 3 * 10 / (15.0e-3) / 1e6
    assert all(abs(o[4] - want) <= 1e-9 * want for o in out)


def test_single_process_is_identity():
    import bench
    assert bench.dist_setup(1) == (0, 1, 0, None) or os.environ.get("WORLD_SIZE", "1") != "1"
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.job_mvox_per_s(1, 1000000, 2, 1000.0) == 2.0
