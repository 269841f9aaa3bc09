"""Multi-process host logic of bench.py on CPU (gloo, world size 2): the
timed duration is the maximum over ranks, the value aggregates all replicas,
and under --impl reference only rank 0 prints (rank 1 exits 0 without work)."""
import io
import json
import os
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
    rate = bench.whole_job_rate(world, 20, ms)
    dist.destroy_process_group()
    # --impl reference: ranks other than 0 return before any work or output.
    buf = io.StringIO()
    rc = None
    if rank != 0:
        sys.argv = ["bench.py", "--impl", "reference", "--gpus", str(world)]
        with redirect_stdout(buf):
            rc = bench.main()
    out.put((rank, ms, rate, rc, buf.getvalue()))


def test_max_over_ranks_and_rank0_output():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate, rc, text in res:
        assert ms == pytest.approx(15.0)
        assert rate == pytest.approx(2 * 20 / 0.015)
    assert res[1][3] == 0 and res[1][4] == ""
