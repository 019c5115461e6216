"""Host logic of one beam over several ranks (fmmb200.sharded) on CPU: gloo ranks that
hold different numbers of particles (none, for one of them) exchange them, run a
stand-in for the sharded forward and sum the shards.  The stand-in evaluates the
oracle's FMM of the gathered beam and keeps one share of its particles per rank, so
the exchange must return every rank exactly the oracle's fields of its own particles."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT


def _beam(n):
    rng = np.random.default_rng(7)
    pos = rng.normal(0.0, 1.0, (n, 3)) * np.array([1.0, 1.0, 0.1])
    mom = np.c_[rng.normal(0, 0.01, (n, 2)), rng.normal(200.0, 0.2, n)]
    return pos, mom


def _stand_in(gpos, gmom, alg, rank, world, charge, lambda_):
    import torch

    sys.path.insert(0, ROOT)
    import oracle

    E, B, _ = oracle.fmm(gpos.numpy(), gmom.numpy(), charge, lambda_, alg.n, alg.N0, alg.eta,
                         variant=oracle.VARIANT_GPU)
    keep = (np.arange(len(E)) % world) == rank  # a share unrelated to who holds the particle
    E[~keep] = 0.0
    B[~keep] = 0.0
    return torch.from_numpy(E), torch.from_numpy(B)


def _worker(rank, world, initf, counts, out):
    sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))
    import torch.distributed as dist

    import fmmb200
    from fmmb200 import sharded

    dist.init_process_group("gloo", init_method=f"file://{initf}", rank=rank, world_size=world)
    pos, mom = _beam(sum(counts))
    lo = sum(counts[:rank])
    mine = slice(lo, lo + counts[rank])
    alg = fmmb200.FMMB200(n=3, N0=40, eta=0.5)
    E, B = sharded.sharded_fields(pos[mine], mom[mine], alg, charge=-1.0, lambda_=2.0, compute=_stand_in)
    out.put((rank, E, B))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("counts", [[700, 300], [0, 500, 523]])
def test_ranks_get_the_oracle_fields_of_their_own_particles(tmp_path, counts):
    import torch.multiprocessing as mp

    sys.path.insert(0, ROOT)
    import oracle

    world = len(counts)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    initf = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, initf, counts, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pos, mom = _beam(sum(counts))
    E, B, _ = oracle.fmm(pos, mom, -1.0, 2.0, 3, 40, 0.5, variant=oracle.VARIANT_GPU)
    lo = 0
    for r, Er, Br in res:
        assert Er.shape == (counts[r], 3)
        assert np.array_equal(Er, E[lo:lo + counts[r]]) and np.array_equal(Br, B[lo:lo + counts[r]])
        lo += counts[r]
