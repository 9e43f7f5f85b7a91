"""The N>1 host path of bench.py, as world-size-2 gloo ranks on the CPU:
process-group setup from the torchrun environment, the barrier, the
max-over-ranks time that the whole-job value divides by, and the reference
arm, which only rank 0 runs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        gpus = world
        steps = 1
        warmup = 0
        nsys = 2

    ws, r, local, pg = bench.dist_setup(Args)
    try:
        bench.barrier(pg)
        t = bench.max_over_ranks(1.0 + rank, pg)      # rank 1 is the slow one
        called = []
        import oracle
        # records the arm's first step and keeps it to its control flow
        oracle.reference_available = lambda: called.append(Args.nsys) or False
        bench.run_reference_arm(Args, ws, r, pg)     # only rank 0 does any work
        out.put((rank, ws, t, called))
    finally:
        pg.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2, 2]
    assert [r[2] for r in res] == [2.0, 2.0]          # both ranks see the slowest time
    assert res[0][3] == [2] and res[1][3] == []       # the reference arm runs on rank 0 only


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
