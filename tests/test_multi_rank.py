"""The multi-rank host logic of bench.py on CPU: two gloo ranks on 127.0.0.1
(each rank owns its batch; the timing is the max over ranks; the reference
arm runs on rank 0 only).  No GPU and no collective on the data path."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch.distributed as dist
    import bench

    class A:
        gpus, steps, warmup, batch = world, 1, 0, 2

    w, r, _ = bench.dist_setup(A)
    # every rank reports a different time; all see the max
    t = bench.max_over_ranks(1.0 + r, w)
    bench.barrier(w)
    # each rank's batch comes from its own seed (weak scaling, no exchange)
    digest = float(np.sum(bench.gen_images(1, 1 + r)[0, :4, :4]))
    out = io.StringIO()
    with redirect_stdout(out):
        rc = bench.run_reference(A)
    q.put((r, t, digest, rc, out.getvalue()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, d0, rc0, out0), (r1, t1, d1, rc1, out1) = res
    assert t0 == t1 == 2.0          # max over ranks
    assert d0 != d1                 # distinct per-rank batches
    assert rc0 == rc1 == 0
    assert out1 == ""               # only rank 0 reports
    line = json.loads(out0.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["config"] == bench_config_of(2, 2)


def bench_config_of(batch, world):
    sys.path.insert(0, ROOT)
    import bench
    return bench.bench_config(batch, world)
