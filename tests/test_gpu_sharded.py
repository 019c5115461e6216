"""One beam over several GPUs on the GPU.

* The leaf-range shards of fmmb200_set_shard (every rank holds the whole tree): in one
  process they add up to the unsharded forward bit for bit, every particle's field coming
  from exactly one shard, for FP64 and the mixed form, for shard counts that do and do not
  divide the number of leaves, and with more shards than leaves.
* The memory-sharded forward (fmmb200.sharded: the tree split at level log2(ranks), each
  rank holding its subtree, the whole tree's boxes and the halo it receives): 2, 4 and 8
  ranks in one process (LoopbackComm, the ranks evaluated in turn) give the single-GPU
  forward's fields with the same p_avg bit for bit, FP64 and mixed, Gaussian bunch and
  beamlets, eta below and above 1/2, ranks with different numbers of particles (none, for
  one), on the third of three calls with the same contexts; each rank holds far less device
  memory than the single-GPU forward.  At N = 2^22 with 2 ranks the same holds for the
  benchmark's distribution and parameters.
* Two processes on the one GPU joined by gloo (fmmb200.sharded.sharded_fields): each gets
  the single-GPU fields of its own particles bit for bit.  Their kernels never wait on each
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


def _slots(pos, mom, counts):
    import torch

    import fmmb200

    out, lo = [], 0
    for c in counts:
        out.append(dict(pos=torch.tensor(pos[lo:lo + c], device="cuda"), mom=torch.tensor(mom[lo:lo + c], device="cuda"),
                        ctx=fmmb200.Context(0), ctx_lists=fmmb200.Context(0)))
        lo += c
    return out


@pytest.mark.parametrize("world,counts,kind,n,N0,eta,precision", [
    (2, [40000, 20000], "gauss", 4, 64, 0.5, "fp64"),
    (2, [40000, 20000], "gauss", 4, 64, 0.5, "mixed"),
    (4, [0, 30000, 17000, 13000], "gauss", 3, 50, 0.5, "mixed"),
    (8, [7500] * 8, "beamlets", 5, 64, 0.5, "mixed"),
    (8, [9000, 0, 11000, 7000, 8000, 5000, 9000, 11000], "gauss", 4, 40, 0.6, "fp64"),
    (4, [20000, 20000, 10000, 10000], "uniform", 4, 64, 0.5, "mixed"),
])
def test_memory_sharded_forward_equals_the_single_gpu_forward(gpu_ctx, world, counts, kind, n, N0, eta, precision):
    import fmmb200
    from fmmb200 import beams, sharded

    pos, mom = {"gauss": beams.gaussian_bunch, "beamlets": beams.beamlets, "uniform": beams.uniform}[kind](
        sum(counts), seed=9)
    alg = fmmb200.FMMB200(n=n, N0=N0, eta=eta, precision=precision)
    slots = _slots(pos, mom, counts)
    try:
        # several calls on the same contexts: buffers grown by one call are reused by the next
        for _ in range(3):
            out = sharded.forward_slots(sharded.LoopbackComm(world), slots, alg, charge=-1.0, lambda_=2.0)
        pavg = slots[0]["info"]["pavg"]
        assert all(s["info"]["pavg"] == pavg for s in slots)
        with fmmb200.Context(0) as one:
            E, B = one.forward(pos, mom, alg, charge=-1.0, lambda_=2.0, p_avg=pavg)
            single_bytes = one.stats()["device_bytes"]
        Es = np.concatenate([e.cpu().numpy() for e, _ in out])
        Bs = np.concatenate([b.cpu().numpy() for _, b in out])
        assert np.array_equal(Es, E) and np.array_equal(Bs, B)
        for s in slots:
            assert s["info"]["device_bytes"] + s["info"]["list_device_bytes"] < single_bytes
    finally:
        for s in slots:
            s["ctx"].close()
            s["ctx_lists"].close()


@pytest.mark.parametrize("N", [2**22, 2**24], ids=["2^22", "2^24"])
def test_memory_sharded_forward_two_ranks_at_benchmark_sizes(gpu_ctx, N):
    """The benchmark's bunch and parameters (n = 4, N0 = 125, eta = 0.5, mixed) over two ranks,
    the case with the largest per-rank traversal, on the third call, with torch's work on its
    default stream (the contexts must run after it: handle 0 is passed as cudaStreamLegacy)."""
    import fmmb200
    from fmmb200 import beams, sharded

    pos, mom = beams.gaussian_bunch(N, seed=0)
    alg = fmmb200.FMMB200(n=4, N0=125, eta=0.5, precision="mixed")
    slots = _slots(pos, mom, [N // 2, N - N // 2])
    try:
        for _ in range(3):
            out = sharded.forward_slots(sharded.LoopbackComm(2), slots, alg)
        pavg = slots[0]["info"]["pavg"]
        halo = [s["info"]["halo_particles"] for s in slots]
        E = np.concatenate([e.cpu().numpy() for e, _ in out])
        del out
    finally:
        for s in slots:
            s["ctx"].close()
            s["ctx_lists"].close()
    with fmmb200.Context(0) as one:
        E1, _ = one.forward(pos, mom, alg, p_avg=pavg)
    assert np.array_equal(E, E1)
    assert max(halo) < 1.5 * min(halo)  # the two sides of the split plane need similar halos


def test_memory_sharded_lists_are_checked(gpu_ctx):
    """shard_evaluate refuses lists that point outside the local clusters or records."""
    import ctypes

    import torch

    import fmmb200
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(5000, seed=3)
    with fmmb200.Context(0) as ctx:
        L = ctx._lib
        dp = torch.tensor(pos, device="cuda")
        dm = torch.tensor(mom, device="cuda")
        pa = np.array([0.0, 0.0, 200.0])
        ctx._check(L.fmmb200_shard_subtree(ctx.handle, 5000, ctypes.c_void_p(dp.data_ptr()),
                                           ctypes.c_void_p(dm.data_ptr()), 50, 7, pa.ctypes.data_as(fmmb200._lib.p_f64),
                                           3, fmmb200.PRECISION_FP64))
        nc_sub = 255
        ntop = 3
        mb = ctypes.c_int64()
        L.fmmb200_shard_record_bytes(3, fmmb200.PRECISION_FP64, ctypes.byref(mb), None)
        nc_loc = nc_sub + ntop
        bext = torch.zeros((ntop, 6), dtype=torch.float64, device="cuda")
        bext[:, 3:] = 1.0
        mext = torch.zeros((ntop, mb.value), dtype=torch.uint8, device="cuda")
        lext = torch.tensor([[0, -1]] * ntop, dtype=torch.int32, device="cuda")
        ptr = torch.zeros(nc_loc + 1, dtype=torch.int32, device="cuda")
        ptr[64:] = 1  # one M2L pair on cluster 63, whose source is out of range
        src = torch.tensor([nc_loc + 5], dtype=torch.int32, device="cuda")
        pptr = torch.zeros(nc_loc + 1, dtype=torch.int32, device="cuda")
        E = torch.empty((5000, 3), dtype=torch.float64, device="cuda")
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        st = L.fmmb200_shard_evaluate(ctx.handle, 1, 0, 40, 0.5, ntop, vp(bext), vp(mext), vp(lext), 0, None, vp(ptr),
                                      vp(src), 1, vp(pptr), None, 0, -1.0, 1.0, vp(E), vp(E))
        assert st == fmmb200.ERR_INVALID_ARGUMENT


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
        info = {}
        E, B = sharded.sharded_fields(torch.tensor(pos[sl], device="cuda"), torch.tensor(mom[sl], device="cuda"), alg,
                                      ctx=ctx, info=info)
        Eref, Bref = ctx.forward(pos, mom, alg, p_avg=info["pavg"])
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
