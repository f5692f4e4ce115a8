"""CPU tests (world size 2, gloo) of the host logic `bench.py` runs under
torchrun: rank and world size from the environment, the max-over-ranks
reduction of the timed region (every rank gets the largest time), the
aggregate whole-job value, and the reference arm doing its work on rank 0
only (the other ranks return at once and exit 0). No GPU is touched."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    try:
        os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": "2",
                           "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
        sys.path.insert(0, ROOT)
        import argparse
        import bench
        args = argparse.Namespace(steps=10, warmup=3, gpus=2, config="kh2d")
        ws, r, local, dist = bench.dist_setup(args, backend="gloo")
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, dist, device="cpu")   # rank 1 is slower
        value = ws * args.steps / (ms / 1e3)
        ref = bench.run_reference(args, bench.WORKLOADS["kh2d"], ws, r) if r != 0 else "skipped"
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ws, r, local, ms, value, ref))
    except Exception as e:   # reported to the parent, which fails the test
        q.put((rank, "error", repr(e)))


def test_two_ranks_reduce_the_time_and_only_rank0_runs_the_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        item = q.get(timeout=120)
        out[item[0]] = item
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r][1] != "error", out[r]
        _, ws, rank, local, ms, value, ref = out[r]
        assert (ws, rank, local) == (2, r, r)
        assert ms == 150.0                      # the max over ranks, on every rank
        assert abs(value - 2 * 10 / 0.150) < 1e-9   # whole-job steps/s over the max time
    assert out[1][6] is None                    # rank 1: no reference work
