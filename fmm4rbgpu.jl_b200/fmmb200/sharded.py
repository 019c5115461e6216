"""One beam over the ranks of a torch.distributed process group, one process per GPU.

The reference has no multi-GPU path: ``update_particles_field!(beam, FMMGPU(...))``
(``src/update_particles_field.jl:66-148``) runs the whole beam on one device.  Here
every rank holds its own particles and one call

1. all-gathers the positions and momenta (48 B per particle): the tree, the pair lists
   and the moments are built from the whole beam on every rank;
2. runs the sharded forward (``Context.set_shard(rank, world)``): M2L, P2P, L2L and L2P
   only for the clusters over this rank's share of the leaves, every other particle's
   field written as 0;
3. sums the ranks' field arrays and keeps this rank's own particles (a reduce-scatter
   under NCCL, an all-reduce with other backends, whose collectives run on host copies).

Each particle's field comes from exactly one rank and the others add exact zeros, so the
result is bit-identical to the single-GPU forward of the whole beam.
"""
from __future__ import annotations

import numpy as np

from .api import Context, FMMB200


def _dist():
    import torch.distributed as dist

    return dist


def _counts(n_local: int, group, dev):
    import torch

    dist = _dist()
    world = dist.get_world_size(group)
    mine = torch.tensor([n_local], dtype=torch.int64, device=dev)
    every = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(every, mine, group=group)
    return [int(c.item()) for c in every]


def _all_gather_rows(x, counts, group, dev):
    """Rows of every rank, concatenated in rank order (x: this rank's (n, 3) rows)."""
    import torch

    dist = _dist()
    m = max(counts)
    pad = torch.zeros((m, 3), dtype=torch.float64, device=dev)
    pad[: x.shape[0]] = x.to(dev)
    blocks = [torch.empty_like(pad) for _ in counts]
    dist.all_gather(blocks, pad, group=group)
    return torch.cat([b[:c] for b, c in zip(blocks, counts)], dim=0)


def _sum_own_rows(full, counts, rank, group, dev, nccl):
    """Sum of every rank's full (N, 3) array, restricted to this rank's rows."""
    import torch

    dist = _dist()
    m, world = max(counts), len(counts)
    padded = torch.zeros((world, m, 3), dtype=torch.float64, device=dev)
    o = 0
    for r, c in enumerate(counts):
        padded[r, :c] = full[o:o + c].to(dev)
        o += c
    if nccl:
        out = torch.empty((m, 3), dtype=torch.float64, device=dev)
        dist.reduce_scatter_tensor(out, padded.reshape(-1), group=group)
    else:
        dist.all_reduce(padded, group=group)
        out = padded[rank]
    return out[: counts[rank]]


def device_compute(ctx: Context):
    """The sharded forward on the context's GPU: full (N, 3) fields, zero outside the shard."""
    import torch

    def compute(gpos, gmom, alg: FMMB200, rank: int, world: int, charge: float, lambda_: float):
        gpos = gpos.contiguous()
        gmom = gmom.contiguous()
        E = torch.empty_like(gpos)
        B = torch.empty_like(gpos)
        ctx.set_stream(torch.cuda.current_stream(gpos.device).cuda_stream)
        ctx.set_shard(rank, world)
        try:
            ctx.forward_device(gpos.shape[0], gpos.data_ptr(), gmom.data_ptr(), E.data_ptr(), B.data_ptr(), alg,
                               charge=charge, lambda_=lambda_)
        finally:
            ctx.set_shard(0, 1)
        return E, B

    return compute


def sharded_fields(pos, mom, alg: FMMB200, *, charge: float = -1.0, lambda_: float = 1.0, group=None,
                   ctx: Context | None = None, compute=None):
    """E and B at this rank's particles from the whole beam spread over the group.

    pos, mom: this rank's (n, 3) float64 positions and momenta, torch tensors on this
    rank's GPU (or numpy arrays, copied there).  Every rank of ``group`` must call with
    the same ``alg``, ``charge`` and ``lambda_``; ranks may hold different numbers of
    particles, zero included.  ``compute`` replaces the GPU forward (signature of
    ``device_compute(ctx)``'s result) for tests of the exchange on hosts without a GPU.
    Returns (E, B) for this rank's particles, of the type of ``pos``.
    """
    import torch

    dist = _dist()
    single = not (dist.is_available() and dist.is_initialized())  # one process: no exchange
    rank, world = (0, 1) if single else (dist.get_rank(group), dist.get_world_size(group))
    as_numpy = isinstance(pos, np.ndarray)
    pos_t = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64)) if as_numpy else pos
    mom_t = torch.as_tensor(np.ascontiguousarray(mom, dtype=np.float64)) if as_numpy else mom
    if pos_t.ndim != 2 or pos_t.shape[1] != 3 or mom_t.shape != pos_t.shape:
        raise ValueError("pos and mom must be (n, 3) arrays of the same shape")
    if compute is None:
        if ctx is None:
            ctx = Context(torch.cuda.current_device())
        compute = device_compute(ctx)
        work = torch.device("cuda", torch.cuda.current_device())
    else:
        work = pos_t.device
    if single:
        counts = [pos_t.shape[0]]
        gpos, gmom = pos_t.to(work, torch.float64), mom_t.to(work, torch.float64)
    else:
        nccl = dist.get_backend(group) == "nccl"
        coll = work if nccl else torch.device("cpu")
        counts = _counts(pos_t.shape[0], group, coll)
        gpos = _all_gather_rows(pos_t.to(torch.float64), counts, group, coll).to(work)
        gmom = _all_gather_rows(mom_t.to(torch.float64), counts, group, coll).to(work)
    if sum(counts) == 0:
        E = torch.zeros((0, 3), dtype=torch.float64, device=pos_t.device)
        return (E.numpy(), E.numpy().copy()) if as_numpy else (E, E.clone())
    Ef, Bf = compute(gpos, gmom, alg, rank, world, charge, lambda_)
    if single:
        E, B = Ef.to(pos_t.device), Bf.to(pos_t.device)
    else:
        E = _sum_own_rows(Ef, counts, rank, group, coll, nccl).to(pos_t.device)
        B = _sum_own_rows(Bf, counts, rank, group, coll, nccl).to(pos_t.device)
    if as_numpy:
        return E.cpu().numpy(), B.cpu().numpy()
    return E, B
