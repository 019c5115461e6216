"""The sharded forward (fmmb200_set_shard) on the GPU.

* One process: the shards' fields add up to the unsharded forward bit for bit, every
  particle's field comes from exactly one shard, for FP64 and the mixed form, for shard
  counts that do and do not divide the number of leaves, and with more shards than
  leaves.
* Two processes on the one GPU joined by gloo (fmmb200.sharded.sharded_fields): each gets
  the unsharded fields of its own particles bit for bit.  Their kernels never wait on each
  other; the exchange runs on host copies.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("world", [2, 3, 8])
def test_shards_add_up_to_the_unsharded_forward(gpu_ctx, precision, world):
    import fmmb200
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(50000, seed=11)
    alg = fmmb200.FMMB200(n=4, N0=64, eta=0.5, precision=precision)
    E, B = gpu_ctx.forward(pos, mom, alg)
    Es, Bs = np.zeros_like(E), np.zeros_like(B)
    owner = np.zeros(len(E), dtype=int)
    for r in range(world):
        gpu_ctx.set_shard(r, world)
        try:
            Er, Br = gpu_ctx.forward(pos, mom, alg)
        finally:
            gpu_ctx.set_shard(0, 1)
        mine = np.any(Er != 0, axis=1) | np.any(Br != 0, axis=1)
        owner += mine
        Es += Er
        Bs += Br
    assert np.all(owner == 1)
    assert np.array_equal(Es, E) and np.array_equal(Bs, B)


def test_more_shards_than_leaves(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(300, seed=2)  # 8 leaves
    alg = fmmb200.FMMB200(n=3, N0=40, eta=0.5)
    E, B = gpu_ctx.forward(pos, mom, alg)
    tot = np.zeros_like(E)
    empty = 0
    for r in range(11):
        gpu_ctx.set_shard(r, 11)
        Er, _ = gpu_ctx.forward(pos, mom, alg)
        empty += not np.any(Er)
        tot += Er
    gpu_ctx.set_shard(0, 1)
    assert empty == 3 and np.array_equal(tot, E)


def test_shard_arguments_and_adjoint_are_checked(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    for r, w in [(0, 0), (2, 2), (-1, 3)]:
        with pytest.raises(fmmb200.FMMB200Error) as ei:
            gpu_ctx.set_shard(r, w)
        assert ei.value.status == fmmb200.ERR_INVALID_ARGUMENT
    pos, mom = beams.gaussian_bunch(2000, seed=1)
    gpu_ctx.set_shard(1, 2)
    try:
        with pytest.raises(fmmb200.FMMB200Error) as ei:
            gpu_ctx.forward(pos, mom, fmmb200.FMMB200(n=3, N0=64, eta=0.5), save_for_backward=True)
        assert ei.value.status == fmmb200.ERR_INVALID_ARGUMENT
    finally:
        gpu_ctx.set_shard(0, 1)


def _worker(rank, world, initf, counts, out):
    sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))
    import torch
    import torch.distributed as dist

    import fmmb200
    from fmmb200 import beams, sharded

    dist.init_process_group("gloo", init_method=f"file://{initf}", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    pos, mom = beams.gaussian_bunch(sum(counts), seed=5)
    lo = sum(counts[:rank])
    sl = slice(lo, lo + counts[rank])
    alg = fmmb200.FMMB200(n=4, N0=100, eta=0.5, precision="mixed")
    with fmmb200.Context(0) as ctx:
        E, B = sharded.sharded_fields(torch.tensor(pos[sl], device="cuda"), torch.tensor(mom[sl], device="cuda"), alg,
                                      ctx=ctx)
        Eref, Bref = ctx.forward(pos, mom, alg)
    ok = np.array_equal(E.cpu().numpy(), Eref[sl]) and np.array_equal(B.cpu().numpy(), Bref[sl])
    out.put((rank, ok, tuple(E.shape)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_processes_share_one_beam(tmp_path):
    import torch.multiprocessing as mp

    counts = [30000, 12345]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    initf = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, 2, initf, counts, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=600) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [ok for _, ok, _ in res] == [True, True]
    assert [s for _, _, s in res] == [(30000, 3), (12345, 3)]
