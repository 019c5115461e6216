"""Host logic of one beam over several ranks (fmmb200.sharded) on CPU.

The tree is split at level L = log2(ranks): the ranks partition its first L levels
together (exact boxes by all-reduce, an exact distributed selection of each node's split)
and move every particle to the rank of its level-L cluster.  Checked against the oracle's
ClusterTree (src/cluster_tree/clusters.jl:21-70) with the same stretch:

* every rank receives exactly the particles of its level-L cluster, in ascending global
  index order, and the top levels' boxes are the oracle's, bit for bit;
* with ranks in one process (LoopbackComm) for 2, 4 and 8 ranks, and with 2 and 4 gloo
  processes (DistComm), ranks holding different numbers of particles (none, for one);
* ties on the split coordinate (a lattice) are broken by the global index, as the
  oracle's id-tie-broken selection does;
* the gloo collectives of DistComm behave as LoopbackComm's.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))


def _beam(n, kind="gauss", seed=7):
    rng = np.random.default_rng(seed)
    if kind == "lattice":
        g = np.arange(16, dtype=float)
        pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:n]
        pos = pos[rng.permutation(len(pos))]
        mom = np.zeros_like(pos)
        mom[:, 2] = 3.0
        return pos, mom
    pos = rng.normal(0.0, 1.0, (n, 3)) * np.array([1.0, 1.0, 0.1])
    mom = np.c_[rng.normal(0, 0.01, (n, 2)), rng.normal(200.0, 0.2, n)]
    return pos, mom


def _split(pos, mom, counts):
    import torch

    out, lo = [], 0
    for c in counts:
        out.append(dict(pos=torch.from_numpy(pos[lo:lo + c].copy()), mom=torch.from_numpy(mom[lo:lo + c].copy())))
        lo += c
    return out


def _partition(comm, slots, N0):
    from fmmb200 import sharded

    beam = sharded.prepare(comm, slots, N0)
    top = sharded._partition_top(comm, slots, beam["N"], beam["L"], beam["stretch"])
    sharded.redistribute(comm, slots, beam)
    return beam, top


def _check_against_oracle(pos, N0, beam, top, got):
    """got: {rank: received global indices in order}."""
    import oracle

    ref = oracle.cluster_tree(pos, N0, beam["stretch"])
    L = beam["L"]
    assert np.array_equal(ref["bboxes"][: (1 << L) - 1], top)
    lo, hi = ref["parlohis"][:, 0], ref["parlohis"][:, 1]
    for r, gids in got.items():
        g = (1 << L) - 1 + r
        want = np.sort(ref["parindices"][lo[g]:hi[g] + 1])
        assert np.array_equal(gids, want), r
        assert np.all(np.diff(gids) > 0)


@pytest.mark.parametrize("world,counts,kind", [(2, [700, 300], "gauss"), (4, [0, 500, 523, 977], "gauss"),
                                               (8, [400] * 8, "gauss"), (4, [1000, 1000, 1000, 1096], "lattice")])
def test_loopback_partition_matches_the_oracle_tree(world, counts, kind):
    from fmmb200 import sharded

    pos, mom = _beam(sum(counts), kind)
    slots = _split(pos, mom, counts)
    N0 = 20
    beam, top = _partition(sharded.LoopbackComm(world), slots, N0)
    _check_against_oracle(pos, N0, beam, top, {s["rank"]: s["sub_gid"].numpy() for s in slots})
    for s in slots:  # the received rows are the particles' own positions and momenta
        assert np.array_equal(s["sub_pos"].numpy(), pos[s["sub_gid"].numpy()])
        assert np.array_equal(s["sub_mom"].numpy(), mom[s["sub_gid"].numpy()])


def test_too_many_ranks_for_the_tree_is_refused():
    from fmmb200 import sharded

    pos, mom = _beam(100)
    with pytest.raises(ValueError):
        sharded.prepare(sharded.LoopbackComm(8), _split(pos, mom, [13] * 7 + [9]), 20)
    with pytest.raises(ValueError):
        sharded.prepare(sharded.LoopbackComm(3), _split(pos, mom, [40, 30, 30]), 20)


def _worker(rank, world, initf, counts, out):
    sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))
    import torch
    import torch.distributed as dist

    from fmmb200 import sharded

    dist.init_process_group("gloo", init_method=f"file://{initf}", rank=rank, world_size=world)
    try:
        comm = sharded.DistComm()
        pos, mom = _beam(sum(counts))
        lo = sum(counts[:rank])
        slot = dict(pos=torch.from_numpy(pos[lo:lo + counts[rank]].copy()),
                    mom=torch.from_numpy(mom[lo:lo + counts[rank]].copy()))
        beam, top = _partition(comm, [slot], 20)
        # the collectives against their loopback meaning
        x = torch.arange(rank + 1, dtype=torch.int64) + 10 * rank
        gathered = [t.tolist() for t in comm.all_gather([x])[0]]
        a2a = [t.tolist() for t in comm.all_to_all([[torch.full((q + 1,), 100 * rank + q) for q in range(world)]])[0]]
        red = comm.all_reduce([torch.tensor([float(rank), -float(rank)])], "max")[0].tolist()
        out.put((rank, slot["sub_gid"].numpy(), top, beam["stretch"], gathered, a2a, red))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("counts", [[700, 300], [0, 500, 523, 977]])
def test_gloo_ranks_partition_like_the_oracle(tmp_path, counts):
    import torch.multiprocessing as mp

    world = len(counts)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    initf = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, initf, counts, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=240) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
    for p in procs:
        assert p.exitcode == 0
    pos, _ = _beam(sum(counts))
    beam = dict(L=world.bit_length() - 1, stretch=res[0][3])
    _check_against_oracle(pos, 20, beam, res[0][2], {r: g for r, g, *_ in res})
    for r, _, top, _, gathered, a2a, red in res:
        assert np.array_equal(top, res[0][2])
        assert gathered == [[10 * k + i for i in range(k + 1)] for k in range(world)]
        assert a2a == [[100 * k + r] * (r + 1) for k in range(world)]
        assert red == [float(world - 1), 0.0]


def _brute_local(g, L, ml, rank, remote):
    """Local cluster number of global heap id g on `rank`, by walking the tree."""
    lev = (g + 1).bit_length() - 1
    nc_sub = (2 << (ml - L)) - 1
    ntop = (2 << L) - 1
    a = g
    while (a + 1).bit_length() - 1 > L:
        a = (a - 1) // 2
    owner = a - ((1 << L) - 1) if lev >= L else -1
    if owner == rank:
        d = lev - L
        return (1 << d) - 1 + (g - ((1 << lev) - 1) - (rank << d))
    if lev <= L:
        return nc_sub + g
    return nc_sub + ntop + remote.index(g)


@pytest.mark.parametrize("L,ml,rank", [(1, 4, 0), (2, 5, 1), (3, 6, 6)])
def test_local_numbering_and_local_csr_match_a_tree_walk(L, ml, rank):
    """_Plan.local: a rank's own subtree first (heap order, its level-L root at 0), then the whole
    tree's top 2^(L+1) - 1 clusters (nc_sub + heap id), then the remote clusters in ascending
    global id.
    _csr_to_local keeps every row's source order and orders rows by local target."""
    import torch

    from fmmb200 import sharded

    rng = np.random.default_rng(L * 100 + rank)
    nc = (2 << ml) - 1
    levels = np.floor(np.log2(np.arange(nc) + 1)).astype(int)
    g_root = (1 << L) - 1 + rank

    def mine_or_ancestor(t):
        a = t
        while a > g_root:
            a = (a - 1) // 2
        b = g_root
        while b > t:
            b = (b - 1) // 2
        return a == g_root or b == t

    targets = [t for t in range(nc) if mine_or_ancestor(t)]
    rows = {t: sorted(rng.choice(nc, size=rng.integers(0, 6), replace=False).tolist()) for t in targets}
    ptr = np.zeros(nc + 1, np.int64)
    for t in range(nc):
        ptr[t + 1] = ptr[t] + len(rows.get(t, []))
    src = np.array([s for t in range(nc) for s in rows.get(t, [])], np.int64)
    below = sorted({int(s) for s in src if levels[s] > L})
    remote = [s for s in below if ((s + 1) >> (levels[s] - L)) - 1 != g_root]  # outside the own subtree
    plan = sharded._Plan(L, ml, rank, torch.tensor(remote, dtype=torch.int64))
    every = [t for t in range(nc) if levels[t] <= L or ((t + 1) >> (levels[t] - L)) - 1 == g_root] + remote
    got = plan.local(torch.tensor(every, dtype=torch.int64)).tolist()
    want = [_brute_local(g, L, ml, rank, remote) for g in every]
    assert got == want
    nc_loc = plan.nc_sub + plan.ntop + len(remote)
    # every local number once, except the top part's slot of the rank's own root: the top levels
    # keep every level-L root's moments there (a contiguous heap for their M2M), while the
    # own root's rows live at local 0
    assert sorted(want) == [x for x in range(nc_loc) if x != plan.nc_sub + g_root]
    lptr, lsrc = sharded._csr_to_local(plan, torch.tensor(ptr, dtype=torch.int32), torch.tensor(src, dtype=torch.int32),
                                       nc_loc)
    lrows = {}
    for t in targets:
        lrows[_brute_local(t, L, ml, rank, remote)] = [_brute_local(s, L, ml, rank, remote) for s in rows[t]]
    wptr = np.zeros(nc_loc + 1, np.int64)
    for lt in range(nc_loc):
        wptr[lt + 1] = wptr[lt] + len(lrows.get(lt, []))
    wsrc = [s for lt in range(nc_loc) for s in lrows.get(lt, [])]
    assert lptr.tolist() == wptr.tolist()
    assert lsrc.tolist() == wsrc
