"""Parity with the oracle at the benchmark configurations' own sizes.

The OpenMP build of the oracle (the serial FMM of src/fmm/*.jl restated, bit-identical
to its one-thread run) finishes N = 2^24 in about two minutes on the host cores, so
the benchmarked configurations are checked against it directly rather than only
through size-independent properties:

* config 2: the Gaussian bunch at N = 2^20, n = 4, N0 = 125, eta = 0.5;
* config 5: eight beamlets at N = 2^22, n = 5, N0 = 64, eta = 0.5;
* config 3: the Gaussian bunch at N = 2^24, n = 4, N0 = 125, eta = 0.5.

Each case asserts the device tree (per-leaf particle sets, ranges, levels, parents,
children, boxes) and both pair lists bit-exact against the oracle's ClusterTree /
dualtraversefill! (src/cluster_tree/clusters.jl:21-70,
src/fmm/interaction_lists.jl:23-58), and the FP64 E and B within 1e-12 relative L2 of
the oracle's FMM (src/update_particles_field.jl:40-64).

The GPU direct sum is the large-N accuracy oracle of the benchmark, so it is pinned
here too: fmmb200_direct against the oracle's BruteForce
(src/update_particles_field.jl:21-38) over all 65,536 particles of config 1 within 1e-13
relative L2, and fmmb200_direct_device against the oracle's direct sum on the first 1,024
of the benchmark's 4,096 seeded targets of the N = 2^24 bunch within 1e-12: both sum the
same 16.7 million terms per target in different orders, so their rounding differs by
about sqrt(N) ulps (1.1e-13 measured).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
DIRECT_TOL = 1e-13
DIRECT_TOL_2_24 = 1e-12  # 16.7 million terms per target, summed in another order
# every host core: the oracle's OpenMP loops are the long pole of these tests
BIG_THREADS = max(1, os.cpu_count() or 1)


def rel(a, b):
    from fmmb200.beams import rel_l2

    return rel_l2(a, b)


def make(kind, N, seed):
    from fmmb200 import beams

    return {"uniform": beams.uniform, "gauss": beams.gaussian_bunch, "beamlets": beams.beamlets}[kind](N, seed=seed)


def sorted_pairs(p):
    return p[np.lexsort((p[:, 1], p[:, 0]))]


@pytest.mark.parametrize("N,kind,n,N0", [(2**20, "gauss", 4, 125), (2**22, "beamlets", 5, 64),
                                         (2**24, "gauss", 4, 125)],
                         ids=["config2_2^20", "config5_2^22", "config3_2^24"])
def test_benchmark_configuration_matches_oracle(gpu_ctx, oracle_mod, N, kind, n, N0):
    import fmmb200

    eta = 0.5
    pos, mom = make(kind, N, 0)
    E, B = gpu_ctx.forward(pos, mom, fmmb200.FMMB200(n=n, N0=N0, eta=eta), charge=-1.0, lambda_=1.0)
    got = gpu_ctx.tree()
    m2l, p2p = gpu_ctx.lists()

    stretch = oracle_mod.stretch(oracle_mod.pavg(mom))
    ref = oracle_mod.cluster_tree(pos, N0, stretch)
    assert ref["complete"]
    for key in ("parlohis", "parindices", "levels", "parents", "children"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)
    assert np.array_equal(got["bboxes"], ref["bboxes"])
    del got
    rp2p, rm2l = oracle_mod.interaction_lists(ref["children"], ref["bboxes"], stretch, eta)
    del ref
    np.testing.assert_array_equal(m2l, sorted_pairs(rm2l))
    np.testing.assert_array_equal(p2p, sorted_pairs(rp2p))
    del m2l, p2p, rm2l, rp2p

    Eo, Bo, st = oracle_mod.fmm(pos, mom, -1.0, 1.0, n, N0, eta, nthreads=BIG_THREADS)
    i = gpu_ctx.tree_info()
    assert (i["nm2l"], i["np2p"]) == (st["nm2l"], st["np2p"])
    assert rel(E, Eo) < FP64_TOL, rel(E, Eo)
    assert rel(B, Bo) < FP64_TOL, rel(B, Bo)


def test_gpu_direct_sum_matches_oracle_bruteforce_at_65536(gpu_ctx, oracle_mod):
    import fmmb200

    N = 65536
    for kind in ("uniform", "gauss"):
        pos, mom = make(kind, N, 0)
        E = np.empty((N, 3))
        B = np.empty((N, 3))
        L = gpu_ctx._lib
        gpu_ctx._check(L.fmmb200_direct(gpu_ctx.handle, N, fmmb200.api._pd(pos), fmmb200.api._pd(mom), -1.0, 1.0,
                                        N, None, fmmb200.api._pd(E), fmmb200.api._pd(B)))
        Eo, Bo = oracle_mod.bruteforce(pos, mom, -1.0, 1.0, nthreads=BIG_THREADS)
        assert rel(E, Eo) < DIRECT_TOL, (kind, rel(E, Eo))
        if kind == "uniform":
            assert np.all(B == 0.0) and np.all(Bo == 0.0)
        else:
            assert rel(B, Bo) < DIRECT_TOL, (kind, rel(B, Bo))


def test_gpu_direct_sum_matches_oracle_on_sampled_targets_at_2_24(oracle_mod):
    """The accuracy figures of the benchmark at N = 2^24 come from fmmb200_direct_device on
    4,096 seeded targets (bench.py's direct_targets seed): the same kernel call on the first
    1,024 of them against the oracle's FP64 direct sum over every source (about 90 s of the
    oracle on 16 cores)."""
    import ctypes

    import torch

    import fmmb200

    N = 2**24
    pos, mom = make("gauss", N, 0)
    tg = np.random.default_rng(100).choice(N, size=4096, replace=False).astype(np.int64)[:1024]
    with fmmb200.Context(0) as ctx:
        dpos = torch.from_numpy(pos).cuda()
        dmom = torch.from_numpy(mom).cuda()
        dtg = torch.from_numpy(tg).cuda()
        Ed = torch.empty((tg.size, 3), dtype=torch.float64, device="cuda")
        Bd = torch.empty_like(Ed)
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        vp = ctypes.c_void_p
        ctx._check(ctx._lib.fmmb200_direct_device(ctx.handle, N, vp(dpos.data_ptr()), vp(dmom.data_ptr()), -1.0, 1.0,
                                                  tg.size, vp(dtg.data_ptr()), vp(Ed.data_ptr()), vp(Bd.data_ptr())))
        torch.cuda.synchronize()
        E, B = Ed.cpu().numpy(), Bd.cpu().numpy()
        del dpos, dmom, dtg, Ed, Bd
    Eo, Bo = oracle_mod.direct_targets(pos, mom, -1.0, 1.0, tg, nthreads=BIG_THREADS)
    assert rel(E, Eo) < DIRECT_TOL_2_24, rel(E, Eo)
    assert rel(B, Bo) < DIRECT_TOL_2_24, rel(B, Bo)
