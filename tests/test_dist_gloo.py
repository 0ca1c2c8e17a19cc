"""The multi-rank path of bench.py on CPU ranks (gloo, world size 2).

The solve does not shard (world size 1 per system); under torchrun each rank
runs an independent replica, and bench.py only needs a barrier and the max
of the per-rank times.  These tests run that bookkeeping as two gloo ranks
and the reference arm under torchrun, where rank 0 alone measures and prints.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(world, rank, backend="gloo")
    d.barrier()
    out[rank] = d.max(values[rank])
    d.barrier()
    d.close()


def test_dist_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, [1.5, 3.25], out))
                 for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        assert out[0] == 3.25 and out[1] == 3.25


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--size", "12"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["steps"] == 1
