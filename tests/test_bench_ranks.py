"""The replica plumbing of bench.py across ranks (gloo, world size 2, CPU): every rank
takes the same barrier/all-reduce steps and the reported time is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r = bench.Ranks(world)
    try:
        r.barrier()
        m = r.max(10.0 * (rank + 1))
        out.put((rank, m))
    finally:
        r.close()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert res == {0: 20.0, 1: 20.0}


def test_roofline_formula_matches_design():
    import bench
    C, N = 3_000_000, 1_000_000
    # full 6-dof rows (the figure roofline.achieved uses), FP64: 1.06 GB per iteration at
    # 1M spheres / 3M contacts, and 0.56 GB in FP32
    assert abs(bench.roofline_bytes_per_iter(C, N, 8) - 1.056e9) < 1e6
    assert abs(bench.roofline_bytes_per_iter(C, N, 4) - 0.564e9) < 1e6
    # 2D: 4 values per contact, 3N particle slots
    assert bench.roofline_bytes_per_iter(C, N, 8, dim=2) == 3 * C * (4 * 8 + 8) + 6 * C * 8 + 4 * (3 * N) * 8
    # torque-free rows (normal only), FP32: what the kernel streams
    assert (bench.roofline_bytes_per_iter(C, N, 4, torque_free=True)
            == 3 * C * (3 * 4 + 8) + 6 * C * 4 + 4 * (3 * N) * 4)
