"""Size-independent properties at the benchmark's full sizes (N = 2^24 and N = 25,600,000
Gaussian bunches).  The oracle comparison at these sizes (tree, lists and FP64 fields at
N = 2^20, 2^22 and 2^24, and the direct sum) is in test_gpu_parity_fullsize.py; the checks
here need no oracle run:

* The mixed form stays within 1e-5 (relative L2 over all particles) of FP64 for n = 2..6.
* Both forms agree with an FP64 direct sum at 4096 seeded targets to the FMM's truncation
  error, which falls as n grows (eta = 1/2), and the two forms' errors agree.
* The tree is a permutation of the particles, every leaf at the last level holds
  floor or ceil of N / 2^ml particles, and every box contains its particles.
* The shards of a sharded forward add up bit for bit to the unsharded fields.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev_ctx():
    import torch

    import fmmb200

    ctx = fmmb200.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    yield ctx
    ctx.close()


def _beam(N, seed):
    import torch

    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(N, seed=seed)
    return torch.from_numpy(pos).cuda(), torch.from_numpy(mom).cuda()


def _forward(ctx, pos, mom, alg):
    import torch

    E = torch.empty_like(pos)
    B = torch.empty_like(pos)
    ctx.forward_device(pos.shape[0], pos.data_ptr(), mom.data_ptr(), E.data_ptr(), B.data_ptr(), alg)
    torch.cuda.synchronize()
    return E, B


def _direct(ctx, pos, mom, tg):
    import torch

    Ed = torch.empty((tg.numel(), 3), dtype=torch.float64, device="cuda")
    Bd = torch.empty_like(Ed)
    L = ctx._lib
    ctx._check(L.fmmb200_direct_device(ctx.handle, pos.shape[0], ctypes.c_void_p(pos.data_ptr()),
                                       ctypes.c_void_p(mom.data_ptr()), -1.0, 1.0, tg.numel(),
                                       ctypes.c_void_p(tg.data_ptr()), ctypes.c_void_p(Ed.data_ptr()),
                                       ctypes.c_void_p(Bd.data_ptr())))
    torch.cuda.synchronize()
    return Ed, Bd


def _rel(a, b):
    import torch

    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _targets(N, k=4096, seed=100):
    import torch

    return torch.from_numpy(np.random.default_rng(seed).choice(N, size=k, replace=False).astype(np.int64)).cuda()


def test_degree_sweep_at_2_24(dev_ctx):
    import fmmb200

    N = 2**24
    pos, mom = _beam(N, 0)
    tg = _targets(N)
    Ed, Bd = _direct(dev_ctx, pos, mom, tg)
    errs = []
    for n in (2, 3, 4, 5, 6):
        E, B = _forward(dev_ctx, pos, mom, fmmb200.FMMB200(n=n, N0=125, eta=0.5))
        e64 = _rel(E[tg], Ed)
        Em, Bm = _forward(dev_ctx, pos, mom, fmmb200.FMMB200(n=n, N0=125, eta=0.5, precision="mixed"))
        assert _rel(Em, E) < 1e-5 and _rel(Bm, B) < 1e-5, (n, _rel(Em, E), _rel(Bm, B))
        assert abs(_rel(Em[tg], Ed) - e64) < 1e-5
        assert _rel(B[tg], Bd) < 2 * e64 + 1e-12
        errs.append(e64)
        del E, B, Em, Bm
    assert errs[2] < 1e-2, errs
    assert all(errs[i + 1] < errs[i] for i in range(len(errs) - 1)), errs


def test_tree_invariants_at_2_24(dev_ctx):
    import fmmb200

    N = 2**24
    pos, mom = _beam(N, 3)
    _forward(dev_ctx, pos, mom, fmmb200.FMMB200(n=2, N0=125, eta=0.5, precision="mixed"))
    t = dev_ctx.tree()
    ml = t["max_level"]
    assert ml == 18
    perm = t["parindices"]
    assert np.array_equal(np.sort(perm), np.arange(N))
    lo, hi = t["parlohis"][:, 0], t["parlohis"][:, 1]
    leaves = np.arange(2**ml - 1, 2 ** (ml + 1) - 1)
    cnt = hi[leaves] - lo[leaves] + 1
    assert set(np.unique(cnt)) <= {N >> ml, (N + 2**ml - 1) >> ml}
    assert cnt.sum() == N and np.all(lo[leaves][1:] == hi[leaves][:-1] + 1)
    p = pos.cpu().numpy()[perm]
    bb = t["bboxes"]
    leaf_of = np.repeat(leaves, cnt)
    assert np.all(p >= bb[leaf_of, :3]) and np.all(p <= bb[leaf_of, 3:])
    root = bb[0]
    assert np.array_equal(root[:3], p.min(axis=0)) and np.array_equal(root[3:], p.max(axis=0))


def test_25_6_million(dev_ctx):
    import fmmb200

    N = 25_600_000
    pos, mom = _beam(N, 1)
    E, B = _forward(dev_ctx, pos, mom, fmmb200.FMMB200(n=4, N0=125, eta=0.5))
    info = dev_ctx.tree_info()
    assert info["max_level"] == 18
    Em, Bm = _forward(dev_ctx, pos, mom, fmmb200.FMMB200(n=4, N0=125, eta=0.5, precision="mixed"))
    assert _rel(Em, E) < 1e-5 and _rel(Bm, B) < 1e-5
    tg = _targets(N, seed=101)
    Ed, _ = _direct(dev_ctx, pos, mom, tg)
    assert _rel(E[tg], Ed) < 1e-2


def test_shards_add_up_at_2_24(dev_ctx):
    import torch

    import fmmb200

    N = 2**24
    pos, mom = _beam(N, 2)
    alg = fmmb200.FMMB200(n=4, N0=125, eta=0.5, precision="mixed")
    E, B = _forward(dev_ctx, pos, mom, alg)
    Es = torch.zeros_like(E)
    Bs = torch.zeros_like(B)
    for r in range(4):
        dev_ctx.set_shard(r, 4)
        try:
            Er, Br = _forward(dev_ctx, pos, mom, alg)
        finally:
            dev_ctx.set_shard(0, 1)
        Es += Er
        Bs += Br
    assert torch.equal(Es, E) and torch.equal(Bs, B)
