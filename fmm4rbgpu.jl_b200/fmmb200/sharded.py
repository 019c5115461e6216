"""One beam over the ranks of a process group, each rank holding only its part of the tree.

The reference has no multi-GPU path: ``update_particles_field!(beam, FMMGPU(...))``
(``src/update_particles_field.jl:66-148``) builds the whole tree (``ClusterTree``,
``src/cluster_tree/cluster_tree.jl:12-18``) and evaluates the whole beam on one device.
Here, with 2^L ranks, the tree is split at level L:

1. p_avg from the ranks' momentum sums; the tree's shape from the beam's size.
2. The first L levels are partitioned across the ranks as ``fillclusters!``
   (``src/cluster_tree/clusters.jl:21-70``) would: per node the exact box (an all-reduce of
   minima and maxima), the split axis argmax(stretch .* extent), and an exact distributed
   selection of the ceil(cnt/2)-th particle in (coordinate, global index) order
   (histograms of 8-bit digits, one all-reduce per digit).
3. An all-to-all moves every particle to the rank that owns its level-L cluster; rank r
   holds cluster 2^L - 1 + r, in ascending global index order, and builds its subtree and
   moments on its GPU (``fmmb200_shard_subtree``).
4. The ranks all-gather their subtrees' boxes and roots' moments; each rank runs the dual
   traversal of the whole tree from the boxes, keeping only its own rows
   (``fmmb200_shard_lists``).
5. Each rank asks the owners for the moments of the remote clusters in its M2L rows and the
   particles of the remote leaves in its P2P rows (two all-to-alls), and evaluates its own
   particles' fields (``fmmb200_shard_evaluate``).
6. An all-to-all returns every field to the rank that passed the particle in.

Every kernel runs on the same data in the same order as in the single-GPU forward, so the
fields equal ``Context.forward(..., p_avg=p_avg)`` with the same p_avg bit for bit.  Per-rank
device memory is that of the rank's own particles and subtree plus the halo it receives and
the whole tree's boxes (48 bytes per cluster).

The collectives go through a ``Comm``: ``DistComm`` over a torch.distributed group (NCCL on
GPUs, or gloo, whose collectives run on host copies), or ``LoopbackComm``, which holds every
rank in one process (one GPU evaluating all ranks in turn).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib as L
from .api import Context, FMMB200, FMMB200Error

# ----------------------------------------------------------------------------- collectives


class Comm:
    """Collectives over `slots`: the ranks this process holds (one per process under
    torch.distributed; every rank for the loopback).  Each method takes one input per
    slot and returns one output per slot."""

    world: int
    ranks: list

    def all_gather(self, xs):
        """xs[i]: slot i's tensor (any length along dim 0) -> per slot, the list over all ranks."""
        raise NotImplementedError

    def all_to_all(self, sends):
        """sends[i][q]: what slot i sends rank q -> per slot, the list of what each rank sent it."""
        raise NotImplementedError

    def all_reduce(self, xs, op: str):
        """Elementwise "sum", "min" or "max" over the ranks -> per slot, the result."""
        raise NotImplementedError


class LoopbackComm(Comm):
    """Every rank in this process: the collectives are copies between the slots."""

    def __init__(self, world: int):
        self.world = world
        self.ranks = list(range(world))

    def all_gather(self, xs):
        return [list(xs) for _ in xs]

    def all_to_all(self, sends):
        return [[sends[q][r] for q in range(self.world)] for r in range(self.world)]

    def all_reduce(self, xs, op):
        import torch

        out = xs[0].clone()
        for x in xs[1:]:
            if op == "sum":
                out = out + x
            elif op == "min":
                out = torch.minimum(out, x)
            else:
                out = torch.maximum(out, x)
        return [out.clone() for _ in xs]


class DistComm(Comm):
    """This process's rank of a torch.distributed group.  NCCL works on device tensors;
    other backends (gloo) get host copies."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.ranks = [dist.get_rank(group)]
        self.nccl = dist.get_backend(group) == "nccl"
        self.dev = torch.device("cuda", torch.cuda.current_device()) if self.nccl else torch.device("cpu")

    def _sizes(self, n: int):
        import torch

        mine = torch.tensor([n], dtype=torch.int64, device=self.dev)
        every = [torch.zeros(1, dtype=torch.int64, device=self.dev) for _ in range(self.world)]
        self.dist.all_gather(every, mine, group=self.group)
        return [int(c.item()) for c in every]

    def all_gather(self, xs):
        import torch

        (x,) = xs
        home = x.device
        x = x.to(self.dev).contiguous()
        sizes = self._sizes(x.shape[0])
        m = max(sizes)
        pad = torch.zeros((m,) + tuple(x.shape[1:]), dtype=x.dtype, device=self.dev)
        pad[: x.shape[0]] = x
        blocks = [torch.empty_like(pad) for _ in range(self.world)]
        self.dist.all_gather(blocks, pad, group=self.group)
        return [[b[:s].to(home) for b, s in zip(blocks, sizes)]]

    def all_to_all(self, sends):
        import torch

        (row,) = sends
        home = row[0].device
        tail = tuple(row[0].shape[1:])
        dtype = row[0].dtype
        flat = torch.cat([t.to(self.dev).reshape((t.shape[0],) + tail) for t in row], dim=0).contiguous()
        out_n = torch.tensor([t.shape[0] for t in row], dtype=torch.int64, device=self.dev)
        in_n = torch.empty_like(out_n)
        self.dist.all_to_all_single(in_n, out_n, group=self.group)
        in_sizes = [int(v) for v in in_n.tolist()]
        recv = torch.empty((sum(in_sizes),) + tail, dtype=dtype, device=self.dev)
        self.dist.all_to_all_single(recv, flat, output_split_sizes=in_sizes,
                                    input_split_sizes=[t.shape[0] for t in row], group=self.group)
        return [[p.to(home) for p in torch.split(recv, in_sizes, dim=0)]]

    def all_reduce(self, xs, op):
        (x,) = xs
        home = x.device
        y = x.to(self.dev).clone()
        ops = {"sum": self.dist.ReduceOp.SUM, "min": self.dist.ReduceOp.MIN, "max": self.dist.ReduceOp.MAX}
        self.dist.all_reduce(y, op=ops[op], group=self.group)
        return [y.to(home)]


# ----------------------------------------------------------------------------- tree shape


def max_level(N: int, N0: int) -> int:
    """maxlevel (src/cluster_tree/treeinfo.jl:6-26) with the reference's float formula."""
    return int(math.ceil(math.log(N / N0) / math.log(2.0))) if N > N0 else 0


def node_ranges(N: int, level: int):
    """(lo, hi) tree positions of the 2^level nodes of a level (left child: ceil(cnt/2))."""
    lo = np.zeros(1, np.int64)
    hi = np.full(1, N - 1, np.int64)
    for _ in range(level):
        mid = (lo + hi) >> 1
        lo, hi = np.stack([lo, mid + 1], 1).reshape(-1), np.stack([mid, hi], 1).reshape(-1)
    return lo, hi


def _order_keys(x):
    """Signed 64-bit keys in the order of the float64 values (-0 == +0), the device's
    double_key shifted to signed order."""
    import torch

    b = x.contiguous().view(torch.int64).clone()
    b[b == torch.iinfo(torch.int64).min] = 0
    return torch.where(b < 0, b ^ 0x7FFFFFFFFFFFFFFF, b)


# ----------------------------------------------------------------------------- the partition


def _partition_top(comm, slots, N, L, stretch):
    """The first L levels of the tree across the ranks (``fillclusters!``): returns per slot
    the owner rank of every particle and the boxes of the top clusters (2^L - 1 heap ids)."""
    import torch

    top_boxes = np.zeros(((1 << L) - 1, 6))
    sv = torch.tensor(stretch, dtype=torch.float64)
    for l in range(L):
        K, base = 1 << l, (1 << l) - 1
        lo, hi = node_ranges(N, l)
        mins, maxs = [], []
        for s in slots:
            dev = s["pos"].device
            node = s["node"] - base
            mn = torch.full((K, 3), float("inf"), dtype=torch.float64, device=dev)
            mx = torch.full((K, 3), float("-inf"), dtype=torch.float64, device=dev)
            if node.numel():
                idx = node[:, None].expand(-1, 3)
                mn = mn.scatter_reduce(0, idx, s["pos"], reduce="amin", include_self=True)
                mx = mx.scatter_reduce(0, idx, s["pos"], reduce="amax", include_self=True)
            mins.append(mn)
            maxs.append(mx)
        mins = comm.all_reduce(mins, "min")
        maxs = comm.all_reduce(maxs, "max")
        bmin, bmax = mins[0].cpu(), maxs[0].cpu()
        top_boxes[base:base + K, :3] = bmin.numpy()
        top_boxes[base:base + K, 3:] = bmax.numpy()
        # splitdir = argmax(stretch .* (bmax - bmin)), the first maximal axis
        v = sv[None, :] * (bmax - bmin)
        axis = torch.argmax(v, dim=1)
        rank_k = torch.from_numpy(((lo + hi) >> 1) - lo)  # 0-based rank of the left half's last particle
        # exact selection of that particle in (coordinate, global index) order: 8 digits of
        # the coordinate key, then 4 of the index, each from all-reduced digit histograms
        keys, cand = [], []
        for s in slots:
            ax = axis.to(s["pos"].device)[s["node"] - base]
            coord = torch.gather(s["pos"], 1, ax[:, None])[:, 0]
            keys.append(_order_keys(coord) ^ torch.iinfo(torch.int64).min)  # unsigned order, as int64 bits
            cand.append(torch.ones(s["node"].numel(), dtype=torch.bool, device=s["pos"].device))
        want = rank_k.clone()
        kstar = torch.zeros(K, dtype=torch.int64)
        istar = torch.zeros(K, dtype=torch.int64)
        for stage, shifts in (("key", range(56, -8, -8)), ("id", range(24, -8, -8))):
            for sh in shifts:
                hists = []
                for s, kk, c in zip(slots, keys, cand):
                    val = kk if stage == "key" else s["gid"]
                    dig = (val >> sh) & 255
                    nd = s["node"] - base
                    h = torch.bincount((nd * 256 + dig)[c], minlength=K * 256)
                    hists.append(h.to(torch.int64))
                H = comm.all_reduce(hists, "sum")[0].cpu().reshape(K, 256)
                cum = torch.cumsum(H, dim=1)
                d = torch.searchsorted(cum, want[:, None], right=True)[:, 0]
                before = torch.where(d > 0, torch.gather(cum, 1, (d - 1).clamp(min=0)[:, None])[:, 0],
                                     torch.zeros_like(d))
                want = want - before
                if stage == "key":
                    kstar = kstar | (d << sh)
                else:
                    istar = istar | (d << sh)
                for j, (s, kk) in enumerate(zip(slots, keys)):
                    val = kk if stage == "key" else s["gid"]
                    dd = d.to(val.device)[s["node"] - base]
                    cand[j] = cand[j] & (((val >> sh) & 255) == dd)
        for s, kk in zip(slots, keys):
            dev = kk.device
            nd = s["node"] - base
            ks = (kstar.to(dev) ^ torch.iinfo(torch.int64).min)[nd]
            ids = istar.to(dev)[nd]
            ksig = kk ^ torch.iinfo(torch.int64).min  # back to signed order
            left = (ksig < ks) | ((ksig == ks) & (s["gid"] <= ids))
            s["node"] = 2 * s["node"] + torch.where(left, 1, 2)
    for s in slots:
        s["owner"] = s["node"] - ((1 << L) - 1)
    return top_boxes


# ----------------------------------------------------------------------------- local numbering


def _pow2(e):
    import torch

    return torch.bitwise_left_shift(torch.ones_like(e), e)


class _Plan:
    """Global cluster ids -> this rank's local cluster numbers: its subtree (0 .. nc_sub-1),
    the whole tree's top 2^(L+1) - 1 clusters (nc_sub + heap id), then the remote clusters
    (ascending global id)."""

    def __init__(self, L, ml, rank, remote):
        import torch

        self.L, self.ml, self.rank = L, ml, rank
        self.g_root = (1 << L) - 1 + rank
        self.nc_sub = (2 << (ml - L)) - 1
        self.ntop = (2 << L) - 1
        self.remote = remote  # sorted int64 global ids
        self.bounds = torch.tensor([(1 << l) - 1 for l in range(ml + 2)], dtype=torch.int64)

    def levels(self, g):
        import torch

        return torch.searchsorted(self.bounds.to(g.device), g, right=True) - 1

    def owner(self, g, lev):
        import torch

        below = (lev - self.L).clamp(min=0)
        return torch.where(lev >= self.L, (g - (_pow2(lev) - 1)) >> below, torch.full_like(g, -1))

    def sub_local(self, g, lev):
        """Subtree heap id inside the owner's subtree (levels >= L)."""
        d = (lev - self.L).clamp(min=0)
        return (_pow2(d) - 1) + ((g - (_pow2(lev) - 1)) & (_pow2(d) - 1))

    def local(self, g):
        import torch

        lev = self.levels(g)
        own = self.owner(g, lev)
        out = torch.empty_like(g)
        top = lev <= self.L
        out[top] = self.nc_sub + g[top]
        mine = (own == self.rank) & (lev >= self.L)
        out[mine] = self.sub_local(g[mine], lev[mine])
        rem = (lev > self.L) & (own != self.rank)
        pos = torch.searchsorted(self.remote.to(g.device), g[rem])
        out[rem] = self.nc_sub + self.ntop + pos
        return out


def _csr_to_local(plan, ptr, src, nc_loc):
    """Global-id CSR rows (targets t, sources ascending) -> CSR over local targets with
    local sources, each row's order kept."""
    import torch

    dev = ptr.device
    lens = (ptr[1:] - ptr[:-1]).to(torch.int64)
    tgt = torch.repeat_interleave(torch.arange(lens.numel(), device=dev, dtype=torch.int64), lens)
    lt = plan.local(tgt)
    order = torch.sort(lt, stable=True).indices
    lsrc = plan.local(src.to(torch.int64))[order]
    cnt = torch.bincount(lt, minlength=nc_loc)
    lptr = torch.zeros(nc_loc + 1, dtype=torch.int64, device=dev)
    lptr[1:] = torch.cumsum(cnt, 0)
    return lptr.to(torch.int32), lsrc.to(torch.int32)


# ----------------------------------------------------------------------------- the forward


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def _check(ctx: Context, st: int):
    ctx._check(st)


class _Clock:
    """Host time of a rank's library calls, which return once their GPU work is done:
    the rank's compute, without the collectives."""

    def __init__(self, slot, stage):
        self.slot, self.stage = slot, stage

    def __enter__(self):
        import time

        self.t0 = time.perf_counter()

    def __exit__(self, *exc):
        import time

        ms = self.slot.setdefault("ms", {})
        ms[self.stage] = ms.get(self.stage, 0.0) + 1e3 * (time.perf_counter() - self.t0)


def prepare(comm: Comm, slots, N0: int):
    """Sizes, global indices, p_avg (the ranks' momentum sums added in rank order) and the
    tree's shape.  Returns a dict of the beam-wide quantities; sets slot["rank"], ["gid"]."""
    import torch

    world = comm.world
    if world & (world - 1):
        raise ValueError("the tree is split at level log2(ranks): the number of ranks must be a power of two")
    Lv = world.bit_length() - 1
    n_local = [int(s["pos"].shape[0]) for s in slots]
    counts_all = comm.all_gather([torch.tensor([n], dtype=torch.int64) for n in n_local])[0]
    counts = [int(c[0]) for c in counts_all]
    N = sum(counts)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    if N < 1:
        raise ValueError("the beam has no particles")
    sums = comm.all_gather([s["mom"].sum(dim=0).to(torch.float64).cpu()[None, :] for s in slots])[0]
    tot = sums[0][0].clone()
    for x in sums[1:]:
        tot = tot + x[0]
    pavg = (tot / N).numpy().astype(np.float64)
    p0, p1, p2 = (float(v) for v in pavg)
    stretch = [1.0, 1.0, math.sqrt(1.0 + ((p0 * p0 + p1 * p1) + p2 * p2))]
    ml = max_level(N, N0)
    if Lv < 1 or ml - Lv < 1:
        raise ValueError(f"{world} ranks need a tree of more than {Lv} levels (this beam has {ml})")
    for s, r in zip(slots, comm.ranks):
        dev = s["pos"].device
        s["rank"] = r
        s["gid"] = torch.arange(int(offs[r]), int(offs[r]) + s["pos"].shape[0], dtype=torch.int64, device=dev)
        s["node"] = torch.zeros(s["pos"].shape[0], dtype=torch.int64, device=dev)
    return dict(world=world, L=Lv, N=N, counts=counts, offs=offs, pavg=pavg, stretch=stretch, ml=ml)


def redistribute(comm: Comm, slots, beam):
    """Every particle to the owner of its level-L cluster (after ``_partition_top``):
    sets slot["sub_pos"], ["sub_mom"], ["sub_gid"], the owner's particles in ascending
    global index order."""
    import torch

    world, N, Lv = beam["world"], beam["N"], beam["L"]
    sends = []
    for s in slots:
        rows = torch.cat([s["pos"], s["mom"], s["gid"].to(torch.float64)[:, None]], dim=1)
        sends.append([rows[s["owner"] == q] for q in range(world)])
    recv = comm.all_to_all(sends)
    sub_lo, sub_hi = node_ranges(N, Lv)
    for s, rv in zip(slots, recv):
        rows = torch.cat(rv, dim=0)
        r = s["rank"]
        if rows.shape[0] != sub_hi[r] - sub_lo[r] + 1:
            raise FMMB200Error(L.ERR_DEVICE, "the top-level partition gave a wrong subtree size")
        s["sub_pos"] = rows[:, 0:3].contiguous()
        s["sub_mom"] = rows[:, 3:6].contiguous()
        s["sub_gid"] = rows[:, 6].to(torch.int64)


def forward_slots(comm: Comm, slots, alg: FMMB200, *, charge=-1.0, lambda_=1.0):
    """The sharded forward of every slot held here.  slots[i]: dict with "pos", "mom"
    ((n, 3) float64 device tensors of that rank's particles), "ctx" and "ctx_lists"
    (Contexts on that rank's GPU).  Returns per slot (E, B) of its particles, and sets
    slot["info"] (sizes and device bytes of the rank).

    Both contexts of every slot are set to run on torch's current stream of its device:
    the library's steps read tensors that torch ops have just written, and on the same
    stream they run after those ops (each step returns once its own work is done)."""
    import torch

    for s in slots:
        st = torch.cuda.current_stream(s["pos"].device).cuda_stream
        s["ctx"].set_stream(st)
        s["ctx_lists"].set_stream(st)
    beam = prepare(comm, slots, alg.N0)
    world, Lv, N, ml = beam["world"], beam["L"], beam["N"], beam["ml"]
    counts, offs, pavg = beam["counts"], beam["offs"], beam["pavg"]
    top_boxes = _partition_top(comm, slots, N, Lv, beam["stretch"])
    redistribute(comm, slots, beam)
    prec = alg.precision_code
    mbytes, pbytes = ctypes.c_int64(), ctypes.c_int64()
    lib = slots[0]["ctx"]._lib
    if lib.fmmb200_shard_record_bytes(alg.n, prec, ctypes.byref(mbytes), ctypes.byref(pbytes)) != L.OK:
        raise FMMB200Error(L.ERR_INVALID_ARGUMENT, "bad degree or precision")
    mb, pb = mbytes.value, pbytes.value
    depth = ml - Lv
    nc_sub = (2 << depth) - 1
    pa = np.ascontiguousarray(pavg)
    for s in slots:
        dev = s["sub_pos"].device
        ctx = s["ctx"]
        with _Clock(s, "subtree"):
            _check(ctx, lib.fmmb200_shard_subtree(ctx.handle, s["sub_pos"].shape[0], _vp(s["sub_pos"]),
                                                  _vp(s["sub_mom"]), alg.N0, depth, pa.ctypes.data_as(L.p_f64),
                                                  alg.n, prec))
        s["boxes"] = torch.empty((nc_sub, 6), dtype=torch.float64, device=dev)
        _check(ctx, lib.fmmb200_shard_boxes(ctx.handle, _vp(s["boxes"])))
        root = torch.zeros(1, dtype=torch.int32, device=dev)
        s["root_mom"] = torch.empty(mb, dtype=torch.uint8, device=dev)
        _check(ctx, lib.fmmb200_shard_pack(ctx.handle, 1, _vp(root), _vp(s["root_mom"]), 0, None, None, None))
    all_boxes = comm.all_gather([s["boxes"] for s in slots])
    all_roots = comm.all_gather([s["root_mom"][None, :] for s in slots])
    nc = (2 << ml) - 1
    ntop = (2 << Lv) - 1
    out = []
    for j, s in enumerate(slots):
        dev = s["sub_pos"].device
        r = s["rank"]
        ctx, ctxg = s["ctx"], s["ctx_lists"]
        # the whole tree's boxes in heap order
        gb = torch.empty((nc, 6), dtype=torch.float64, device=dev)
        gb[: (1 << Lv) - 1] = torch.from_numpy(top_boxes).to(dev)
        for l in range(Lv, ml + 1):
            d = l - Lv
            base = (1 << l) - 1
            for q in range(world):
                gb[base + (q << d): base + ((q + 1) << d)] = all_boxes[j][q][(1 << d) - 1: (2 << d) - 1]
        counts2 = (ctypes.c_int64 * 2)()
        with _Clock(s, "lists"):
            _check(ctxg, lib.fmmb200_shard_lists(ctxg.handle, nc, ml, _vp(gb), pa.ctypes.data_as(L.p_f64), alg.eta,
                                                 Lv, r, counts2))
        nm2l, np2p = counts2[0], counts2[1]
        mptr = torch.empty(nc + 1, dtype=torch.int32, device=dev)
        pptr = torch.empty(nc + 1, dtype=torch.int32, device=dev)
        msrc = torch.empty(max(nm2l, 1), dtype=torch.int32, device=dev)
        psrc = torch.empty(max(np2p, 1), dtype=torch.int32, device=dev)
        _check(ctxg, lib.fmmb200_shard_get_lists(ctxg.handle, _vp(mptr), _vp(msrc), _vp(pptr), _vp(psrc)))
        msrc, psrc = msrc[:nm2l].to(torch.int64), psrc[:np2p].to(torch.int64)
        # remote clusters: M2L sources (moments) and P2P source leaves (particles) below level L
        probe = _Plan(Lv, ml, r, torch.zeros(0, dtype=torch.int64, device=dev))
        need_m = msrc[(probe.levels(msrc) > Lv)]
        need_m = torch.unique(need_m[probe.owner(need_m, probe.levels(need_m)) != r])
        need_p = psrc[(probe.levels(psrc) > Lv)]
        need_p = torch.unique(need_p[probe.owner(need_p, probe.levels(need_p)) != r])
        remote = torch.unique(torch.cat([need_m, need_p]))
        plan = _Plan(Lv, ml, r, remote)
        s.update(plan=plan, gb=gb, need_m=need_m, need_p=need_p, mptr=mptr, msrc=msrc, pptr=pptr, psrc=psrc,
                 nm2l=nm2l, np2p=np2p)
    # requests: the owners' subtree ids of the remote clusters (moments) and leaves (particles)
    req_sends = []
    for s in slots:
        plan = s["plan"]
        rows = []
        for q in range(world):
            rm = s["need_m"][plan.owner(s["need_m"], plan.levels(s["need_m"])) == q]
            rp = s["need_p"][plan.owner(s["need_p"], plan.levels(s["need_p"])) == q]
            rows.append(torch.cat([plan.sub_local(rm, plan.levels(rm)), -1 - plan.sub_local(rp, plan.levels(rp))]))
        req_sends.append(rows)
    reqs = comm.all_to_all(req_sends)
    # leaf particle counts from the tree's shape: leaf j of the whole tree holds positions
    # lo..hi, and a subtree's leaves are consecutive
    leaf_lo, leaf_hi = node_ranges(N, ml)
    pay_sends = []
    for s, rq in zip(slots, reqs):
        dev = s["sub_pos"].device
        r = s["rank"]
        ctx = s["ctx"]
        rows = []
        nl_sub = 1 << depth
        own_leaf_cnt = torch.from_numpy(leaf_hi[r * nl_sub:(r + 1) * nl_sub] - leaf_lo[r * nl_sub:(r + 1) * nl_sub]
                                        + 1).to(dev)
        for q in range(world):
            ask = rq[q]
            cm = ask[ask >= 0].to(torch.int32)
            cl = (-1 - ask[ask < 0])
            cnt = own_leaf_cnt[cl - (nl_sub - 1)] if cl.numel() else torch.zeros(0, dtype=torch.int64, device=dev)
            offs_l = torch.zeros(cl.numel(), dtype=torch.int64, device=dev)
            if cl.numel() > 1:
                offs_l[1:] = torch.cumsum(cnt, 0)[:-1]
            moms = torch.empty(cm.numel() * mb, dtype=torch.uint8, device=dev)
            recs = torch.empty(int(cnt.sum().item()) * pb, dtype=torch.uint8, device=dev)
            clid = cl.to(torch.int32)
            with _Clock(s, "pack"):
                _check(ctx, lib.fmmb200_shard_pack(ctx.handle, cm.numel(), _vp(cm), _vp(moms), clid.numel(),
                                                   _vp(clid), _vp(offs_l), _vp(recs)))
            rows.append(torch.cat([moms, recs]))
        pay_sends.append(rows)
    pays = comm.all_to_all(pay_sends)
    for j, (s, pay) in enumerate(zip(slots, pays)):
        dev = s["sub_pos"].device
        r = s["rank"]
        plan = s["plan"]
        ctx = s["ctx"]
        nrem = plan.remote.numel()
        next_ = ntop + nrem
        nc_loc = nc_sub + next_
        # appended clusters: boxes, moments (top level L: every root; remote: received),
        # particle ranges of the remote leaves in the halo records
        gids_ext = torch.cat([torch.arange(ntop, device=dev, dtype=torch.int64), plan.remote])
        bext = s["gb"][gids_ext].contiguous()
        mext = torch.zeros((next_, mb), dtype=torch.uint8, device=dev)
        roots = torch.cat([x.to(dev) for x in all_roots[j]], dim=0)
        mext[(1 << Lv) - 1: ntop] = roots
        lext = torch.zeros((next_, 2), dtype=torch.int32, device=dev)
        lext[:, 1] = -1
        halo = []
        hoff = 0
        for q in range(world):
            rm = s["need_m"][plan.owner(s["need_m"], plan.levels(s["need_m"])) == q]
            rp = s["need_p"][plan.owner(s["need_p"], plan.levels(s["need_p"])) == q]
            buf = pay[q]
            mbuf = buf[: rm.numel() * mb].reshape(-1, mb) if rm.numel() else None
            if rm.numel():
                mext[ntop + torch.searchsorted(plan.remote, rm)] = mbuf
            recs = buf[rm.numel() * mb:]
            if rp.numel():
                li = rp - ((1 << ml) - 1)
                cnt = torch.from_numpy(leaf_hi - leaf_lo + 1).to(dev)[li]
                start = hoff + torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), torch.cumsum(cnt, 0)[:-1]])
                pos_r = ntop + torch.searchsorted(plan.remote, rp)
                lext[pos_r, 0] = start.to(torch.int32)
                lext[pos_r, 1] = (start + cnt - 1).to(torch.int32)
                hoff += int(cnt.sum().item())
                halo.append(recs)
        halo_recs = torch.cat(halo) if halo else torch.zeros(0, dtype=torch.uint8, device=dev)
        nhalo = hoff
        lmptr, lmsrc = _csr_to_local(plan, s["mptr"], s["msrc"], nc_loc)
        lpptr, lpsrc = _csr_to_local(plan, s["pptr"], s["psrc"], nc_loc)
        E = torch.empty_like(s["sub_pos"])
        B = torch.empty_like(s["sub_pos"])
        max_leaf = int((leaf_hi - leaf_lo + 1).max())
        with _Clock(s, "evaluate"):
            _check(ctx, lib.fmmb200_shard_evaluate(
                ctx.handle, Lv, r, max_leaf, float(alg.eta), next_, _vp(bext), _vp(mext), _vp(lext), nhalo,
                _vp(halo_recs), _vp(lmptr), _vp(lmsrc), int(lmsrc.numel()), _vp(lpptr), _vp(lpsrc),
                int(lpsrc.numel()), float(charge), float(lambda_), _vp(E), _vp(B)))
        s["sub_E"], s["sub_B"] = E, B
        s["info"] = dict(rank=r, particles=int(s["sub_pos"].shape[0]), halo_particles=nhalo,
                         halo_bytes=int(halo_recs.numel()), remote_moment_bytes=int(s["need_m"].numel() * mb),
                         remote_clusters=int(nrem), subtree_clusters=nc_sub, nm2l=int(lmsrc.numel()),
                         np2p=int(lpsrc.numel()), device_bytes=int(ctx.stats()["device_bytes"]),
                         list_device_bytes=int(s["ctx_lists"].stats()["device_bytes"]), pavg=pavg.tolist())
    # fields back to the ranks that passed the particles in
    starts = torch.from_numpy(offs[1:-1].astype(np.int64))
    back = []
    for s in slots:
        dev = s["sub_pos"].device
        src = torch.searchsorted(starts.to(dev), s["sub_gid"], right=True)
        rows = torch.cat([s["sub_E"], s["sub_B"], s["sub_gid"].to(torch.float64)[:, None]], dim=1)
        back.append([rows[src == q] for q in range(world)])
    got = comm.all_to_all(back)
    for s, g in zip(slots, got):
        rows = torch.cat(g, dim=0)
        r = s["rank"]
        idx = rows[:, 6].to(torch.int64) - int(offs[r])
        E = torch.empty((counts[r], 3), dtype=torch.float64, device=rows.device)
        B = torch.empty_like(E)
        E[idx] = rows[:, 0:3]
        B[idx] = rows[:, 3:6]
        out.append((E, B))
    return out


def sharded_fields(pos, mom, alg: FMMB200, *, charge: float = -1.0, lambda_: float = 1.0, group=None,
                   ctx: Context | None = None, ctx_lists: Context | None = None, info: dict | None = None):
    """E and B at this rank's particles from the whole beam spread over the group.

    pos, mom: this rank's (n, 3) float64 positions and momenta (torch tensors on this rank's
    GPU, or numpy arrays, copied there).  Every rank of ``group`` must call with the same
    ``alg``, ``charge`` and ``lambda_``; ranks may hold different numbers of particles, zero
    included.  The number of ranks must be a power of two (one process: the plain
    forward).  ``info``, if given, receives this rank's sizes, device bytes and the p_avg
    used.  Returns (E, B) for this rank's particles, of the type of ``pos``.
    """
    import torch
    import torch.distributed as dist

    as_numpy = isinstance(pos, np.ndarray)
    dev = torch.device("cuda", torch.cuda.current_device())
    pos_t = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64)).to(dev) if as_numpy else pos
    mom_t = torch.as_tensor(np.ascontiguousarray(mom, dtype=np.float64)).to(dev) if as_numpy else mom
    if pos_t.ndim != 2 or pos_t.shape[1] != 3 or mom_t.shape != pos_t.shape:
        raise ValueError("pos and mom must be (n, 3) arrays of the same shape")
    ctx = ctx or Context(torch.cuda.current_device())
    single = not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1
    if single:
        E = torch.empty_like(pos_t)
        B = torch.empty_like(pos_t)
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ctx.forward_device(pos_t.shape[0], pos_t.data_ptr(), mom_t.data_ptr(), E.data_ptr(), B.data_ptr(), alg,
                           charge=charge, lambda_=lambda_)
        torch.cuda.synchronize(dev)
    else:
        ctx_lists = ctx_lists or Context(torch.cuda.current_device())
        slot = dict(pos=pos_t.contiguous(), mom=mom_t.contiguous(), ctx=ctx, ctx_lists=ctx_lists)
        ((E, B),) = forward_slots(DistComm(group), [slot], alg, charge=charge, lambda_=lambda_)
        if info is not None:
            info.update(slot["info"])
    if as_numpy:
        return E.cpu().numpy(), B.cpu().numpy()
    return E, B
