"""Host logic of the N > 1 path on CPU: two gloo ranks, and bench.py's reference arm."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))
    from fmmb200 import replicas

    w, r, lr = replicas.env_ranks()
    replicas.init("gloo", lr, timeout_s=60)
    replicas.barrier(w)
    ms = 10.0 + 5.0 * r  # rank 1 is the slowest
    m = replicas.max_over_ranks(w, ms)
    out.put((r, m, replicas.aggregate_rate(w, 1000, m)))
    import torch.distributed as dist

    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [15.0, 15.0]
    assert res[0][2] == pytest.approx(2 * 1000 / 15e-3)


@pytest.mark.parametrize("rank", ["0", "1"])
def test_reference_arm_prints_on_rank0_only(rank):
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--ref-sample", "4096", "--N", "4096", "--N0", "64"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    if rank == "1":
        assert r.stdout.strip() == ""
    else:
        d = json.loads(r.stdout.strip().splitlines()[-1])
        assert d["impl"] == "reference" and d["unit"] == "particles/s" and d["value"] > 0
        assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
