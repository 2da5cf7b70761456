"""The multi-GPU path of bench.py, on the CPU with gloo (world size 2).

One process per GPU, no data-path collective: each rank works on its own
seeded batch and only the timings cross ranks (max over ranks).  These tests
run bench.RankContext -- the same code the GPU run uses with nccl -- in two
spawned processes rendezvousing on 127.0.0.1.
"""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        import bench
        from lzx_b200 import CRT_SET_30BIT, synth
        ctx = bench.RankContext("gloo", "cpu", timeout_s=60)
        ctx.barrier()
        slowest = ctx.max_over_ranks(1.5 * (rank + 1))
        first = synth.crt_batch(bench.rank_seed(1234, ctx.rank), CRT_SET_30BIT, 2, 256)[0, 0, :4].tolist()
        ctx.barrier()
        ctx.close()

        class A:
            warmup, steps, gpus = 1, 1, world
        ref_rc = bench.run_reference(A()) if rank == 1 else None  # rank 1 of the reference arm: no work
        q.put((rank, ctx.world, slowest, first, ref_rc))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None, None))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(2):
            r = q.get(timeout=120)
            results[r[0]] = r
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    for r in (0, 1):
        assert results[r][1] == 2, results[r]
        assert results[r][2] == pytest.approx(3.0)  # both ranks see the slowest time
    assert results[0][3] != results[1][3]  # each rank commits/transforms its own inputs
    assert results[1][4] == 0  # the reference arm's non-zero ranks exit at once
