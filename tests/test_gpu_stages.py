"""Kernel-level parity of every device stage against the CPU oracle.

Each stage is called through the C-ABI stage entry points (the counterparts of
the reference's gpu_P2M!/gpu_M2M!/gpu_M2L!/gpu_P2P!/gpu_L2L!/gpu_L2P! kernels,
ClusterTree and InteractionListsGPU) on the same inputs as the oracle.

Tolerances: tree permutation, ranges, bounding boxes and pair lists are
compared bit-exactly; FP64 stage outputs within 1e-13 relative L2 (the device
reassociates sums); the mixed form within 1e-5.
"""
import numpy as np
import pytest

from conftest import NTHREADS

pytestmark = pytest.mark.gpu

FP64_STAGE_TOL = 1e-13
MIXED_STAGE_TOL = 1e-5


def rel(a, b):
    from fmmb200.beams import rel_l2

    return rel_l2(a, b)


def isapprox(x, y, rtol):
    x, y = np.asarray(x, float), np.asarray(y, float)
    return np.linalg.norm(x - y) <= rtol * max(np.linalg.norm(x), np.linalg.norm(y))


def make(kind, N, seed):
    from fmmb200 import beams

    return {"uniform": beams.uniform, "gauss": beams.gaussian_bunch, "beamlets": beams.beamlets}[kind](N, seed=seed)


# ------------------------------------------------------------------------- tree
@pytest.mark.parametrize("N,N0,kind", [(10000, 32, "uniform"), (65536, 125, "gauss"), (100003, 50, "beamlets"),
                                       (1000, 400, "uniform"), (100, 200, "uniform"), (1, 5, "uniform"),
                                       (20000, 5000, "gauss"), (100000, 2, "uniform"), (300000, 100, "gauss")])
def test_cluster_tree_bit_exact(gpu_ctx, oracle_mod, N, N0, kind):
    pos, mom = make(kind, N, 3)
    stretch = oracle_mod.stretch(oracle_mod.pavg(mom))
    ref = oracle_mod.cluster_tree(pos, N0, stretch)
    got = gpu_ctx.cluster_tree(pos, N0, stretch)
    assert ref["complete"]
    for key in ("parlohis", "parindices", "levels", "parents", "children"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)
    assert np.array_equal(got["bboxes"], ref["bboxes"])  # == (IEEE), exact min/max


def test_cluster_tree_leaves_reference_case(gpu_ctx):
    # test/test_cluster_tree/test_clusters.jl:10-28 on the device tree
    N, N0 = 10000, 32
    pos = np.random.default_rng(0).random((N, 3))
    t = gpu_ctx.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    ml = t["max_level"]
    lrg = slice((1 << ml) - 1, (1 << (ml + 1)) - 1)
    assert np.all(t["levels"][lrg] == ml)
    assert np.all(t["children"][lrg] == -1)


def test_tree_with_ties_is_deterministic(gpu_ctx, oracle_mod):
    # lattice positions: every split coordinate has ties; ids break them
    g = np.arange(16, dtype=float)
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = pos[np.random.default_rng(1).permutation(len(pos))]
    ref = oracle_mod.cluster_tree(pos, 20, [1.0, 1.0, 1.0])
    got = gpu_ctx.cluster_tree(pos, 20, [1.0, 1.0, 1.0])
    np.testing.assert_array_equal(got["parindices"], ref["parindices"])
    assert np.array_equal(got["bboxes"], ref["bboxes"])


# ------------------------------------------------------------------------- lists
@pytest.mark.parametrize("N,N0,kind,eta", [(65536, 125, "uniform", 0.5), (65536, 125, "gauss", 0.5),
                                           (30000, 64, "beamlets", 0.5), (20000, 100, "gauss", 0.8),
                                           (5000, 50, "uniform", 0.3)])
def test_interaction_lists_match(gpu_ctx, oracle_mod, N, N0, kind, eta):
    pos, mom = make(kind, N, 4)
    stretch = oracle_mod.stretch(oracle_mod.pavg(mom))
    t = gpu_ctx.cluster_tree(pos, N0, stretch)
    m2l, p2p = gpu_ctx.interaction_lists(stretch, eta)
    rp2p, rm2l = oracle_mod.interaction_lists(t["children"], t["bboxes"], stretch, eta)
    for got, ref in ((m2l, rm2l), (p2p, rp2p)):
        ref = ref[np.lexsort((ref[:, 1], ref[:, 0]))]
        np.testing.assert_array_equal(got, ref)
    # the CSR grouping of InteractionListsGPU: sorted by target
    assert np.all(np.diff(m2l[:, 0]) >= 0) and np.all(np.diff(p2p[:, 0]) >= 0)


def test_interaction_lists_two_extreme_etas(gpu_ctx):
    # test/test_fmm/test_interaction_lists.jl:9-25
    N, N0 = 1000, 400
    pos = np.random.default_rng(5).random((N, 3))
    gpu_ctx.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    m2l, _ = gpu_ctx.interaction_lists([1.0, 1.0, 1.0], 999.0)
    assert len(m2l) == 2
    _, p2p = gpu_ctx.interaction_lists([1.0, 1.0, 1.0], 0.0)
    assert len(p2p) == 16


def test_single_leaf_lists(gpu_ctx):
    pos = np.random.default_rng(6).random((50, 3))
    gpu_ctx.cluster_tree(pos, 64, [1.0, 1.0, 1.0])
    m2l, p2p = gpu_ctx.interaction_lists([1.0, 1.0, 1.0], 0.5)
    assert len(m2l) == 0
    np.testing.assert_array_equal(p2p, [[0, 0]])


# ------------------------------------------------------------------------- stage fixtures
def tree_case(oracle_mod, N=6000, N0=40, kind="gauss", seed=8):
    pos, mom = make(kind, N, seed)
    stretch = oracle_mod.stretch(oracle_mod.pavg(mom))
    t = oracle_mod.cluster_tree(pos, N0, stretch)
    ml = t["max_level"]
    leaves = np.arange((1 << ml) - 1, (1 << (ml + 1)) - 1)
    return pos, mom, stretch, t, leaves


@pytest.mark.parametrize("n", [2, 4, 5])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_p2m_matches_oracle(gpu_ctx, oracle_mod, n, precision):
    pos, mom, _, t, leaves = tree_case(oracle_mod)
    NN = (n + 1) ** 3
    g = np.zeros(NN * t["nc"])
    m = np.zeros(3 * NN * t["nc"])
    rg, rm = g.copy(), m.copy()
    gpu_ctx.p2m(n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, g, m, precision=precision)
    oracle_mod.p2m(oracle_mod.VARIANT_GPU, n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, rg, rm)
    tol = FP64_STAGE_TOL if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(g, rg) < tol and rel(m, rm) < tol


def test_p2m_conservation_reference_case(gpu_ctx):
    # test/test_gpu_fmm/test_gpu_upwardpass.jl:2-37
    N, N0, n = 100, 200, 2
    pos = np.random.default_rng(2).random((N, 3))
    mom = np.zeros((N, 3))
    mom[:, 2] = 2.0
    t = gpu_ctx.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    NN = (n + 1) ** 3
    g = np.zeros(NN)
    m = np.zeros(3 * NN)
    gpu_ctx.p2m(n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], [0], g, m)
    assert isapprox(m.reshape(-1, 3).sum(axis=0), N * mom[0], 0.01)
    np.testing.assert_allclose(m.reshape(-1, 3).sum(axis=0), N * mom[0], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("n", [2, 4])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_upward_pass_matches_oracle(gpu_ctx, oracle_mod, n, precision):
    pos, mom, _, t, leaves = tree_case(oracle_mod, N=5000, N0=40)
    ml = t["max_level"]
    NN = (n + 1) ** 3
    g = np.zeros(NN * t["nc"])
    m = np.zeros(3 * NN * t["nc"])
    rg, rm = g.copy(), m.copy()
    gpu_ctx.p2m(n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, g, m, precision=precision)
    oracle_mod.p2m(oracle_mod.VARIANT_GPU, n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, rg, rm)
    for lev in range(ml - 1, -1, -1):  # gpu_M2M! over parent levels (update_particles_field.jl:105-110)
        gpu_ctx.m2m(n, t["children"], t["bboxes"], lev, g, m, precision=precision)
        oracle_mod.m2m(oracle_mod.VARIANT_GPU, n, lev + 1, t["parents"], t["children"], t["bboxes"], rg, rm)
    tol = 1e-12 if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(g, rg) < tol and rel(m, rm) < tol


def test_upward_conservation_reference_case(gpu_ctx):
    # test/test_gpu_fmm/test_gpu_upwardpass.jl:39-85
    N, N0, n = 1000, 80, 2
    pos = np.random.default_rng(3).random((N, 3))
    mom = np.zeros((N, 3))
    gamma = 30.0
    mom[:, 2] = np.sqrt(gamma**2 - 1.0)
    t = gpu_ctx.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    ml = t["max_level"]
    NN = (n + 1) ** 3
    g = np.zeros(NN * t["nc"])
    m = np.zeros(3 * NN * t["nc"])
    leaves = np.arange((1 << ml) - 1, (1 << (ml + 1)) - 1)
    gpu_ctx.p2m(n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, g, m)
    for lev in range(ml - 1, -1, -1):
        gpu_ctx.m2m(n, t["children"], t["bboxes"], lev, g, m)
    assert isapprox(g[:NN].sum(), N * gamma, 1e-12)
    assert isapprox(m.reshape(-1, 3)[:NN].sum(axis=0), N * mom[0], 1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_m2l_far_field_reference_case(gpu_ctx, precision):
    # test/test_gpu_fmm/test_gpu_interaction.jl:2-48
    distance, n = 10000.0, 3
    NN = (n + 1) ** 3
    bboxes = np.array([[-1, -1, -1, 1, 1, 1], [-1, -1, -1 + distance, 1, 1, 1 + distance]], dtype=float)
    g = np.ones(2 * NN)
    m = np.zeros(3 * 2 * NN)
    e = np.zeros(3 * 2 * NN)
    b = np.zeros(3 * 2 * NN)
    gpu_ctx.m2l(n, bboxes, g, m, [[0, 1], [1, 0]], [0.0, 0.0, 0.0], e, b, precision=precision)
    far = NN * np.array([0, 0, distance]) / distance**3
    assert isapprox(e.reshape(-1, 3)[NN], far, 1e-3)
    assert isapprox(e.reshape(-1, 3)[0], -far, 1e-3)
    assert np.all(b == 0.0)


@pytest.mark.parametrize("n", [1, 3, 4, 6, 8])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_m2l_matches_oracle(gpu_ctx, oracle_mod, n, precision):
    pos, mom, stretch, t, _ = tree_case(oracle_mod, N=4000, N0=30)
    NN = (n + 1) ** 3
    nc = t["nc"]
    rng = np.random.default_rng(n)
    g = rng.random(NN * nc)
    m = rng.normal(0, 1, 3 * NN * nc) + np.tile([0.0, 0.0, 50.0], NN * nc)
    _, m2l = oracle_mod.interaction_lists(t["children"], t["bboxes"], stretch, 0.5)
    m2l = oracle_mod.sort_by_target(m2l)
    pavg = np.array([0.01, -0.02, 50.0])
    e = np.zeros(3 * NN * nc)
    b = np.zeros(3 * NN * nc)
    re, rb = e.copy(), b.copy()
    gpu_ctx.m2l(n, t["bboxes"], g, m, m2l, pavg, e, b, precision=precision)
    oracle_mod.m2l(oracle_mod.VARIANT_GPU, n, t["bboxes"], g, m, m2l, pavg, re, rb)
    if n == 1:  # the reference's GPU weight table for n = 1 is not used: M2L has no weights
        pass
    tol = FP64_STAGE_TOL if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(e, re) < tol and rel(b, rb) < tol


@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("eta", [0.5, 0.7])
def test_m2l_mixed_engines_agree(gpu_ctx, oracle_mod, n, eta):
    """Both mixed M2L engines match the oracle within the mixed tolerance: the
    tensor-core form (tcgen05 TF32 hi/lo MMAs, n <= 4, eta <= 1/2) and the packed
    FP32x2 CUDA-core kernel.  eta = 0.7 admits coincident nodes: both engines then
    run the non-factored CUDA-core accumulation."""
    pos, mom, stretch, t, _ = tree_case(oracle_mod, N=4000, N0=30)
    NN = (n + 1) ** 3
    nc = t["nc"]
    rng = np.random.default_rng(10 + n)
    g = rng.random(NN * nc)
    m = rng.normal(0, 1, 3 * NN * nc) + np.tile([0.0, 0.0, 50.0], NN * nc)
    _, m2l = oracle_mod.interaction_lists(t["children"], t["bboxes"], stretch, eta)
    m2l = oracle_mod.sort_by_target(m2l)
    pavg = np.array([0.01, -0.02, 50.0])
    re, rb = np.zeros(3 * NN * nc), np.zeros(3 * NN * nc)
    oracle_mod.m2l(oracle_mod.VARIANT_GPU, n, t["bboxes"], g, m, m2l, pavg, re, rb)
    got = {}
    try:
        for engine in ("tensor_cores", "cuda_cores"):
            gpu_ctx.set_m2l_engine(engine)
            e, b = np.zeros(3 * NN * nc), np.zeros(3 * NN * nc)
            gpu_ctx.m2l(n, t["bboxes"], g, m, m2l, pavg, e, b, precision="mixed")
            assert np.all(np.isfinite(e)) and np.all(np.isfinite(b))
            assert rel(e, re) < MIXED_STAGE_TOL and rel(b, rb) < MIXED_STAGE_TOL, engine
            got[engine] = (e, b)
    finally:
        gpu_ctx.set_m2l_engine("auto")
    if eta > 0.5:  # same kernel either way
        assert np.array_equal(got["tensor_cores"][0], got["cuda_cores"][0])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_p2p_far_field_reference_case(gpu_ctx, precision):
    # test/test_gpu_fmm/test_gpu_interaction.jl:50-96
    npar, sep = 200, 10000.0
    pos = np.random.default_rng(4).random((npar, 3))
    mom = np.zeros((npar, 3))
    pos[: npar // 2, 2] += sep
    parlohis = np.array([[0, 99], [100, 199]])
    bboxes = np.array([np.r_[pos[:100].min(0), pos[:100].max(0)], np.r_[pos[100:].min(0), pos[100:].max(0)]])
    e = np.zeros((npar, 3))
    b = np.zeros((npar, 3))
    gpu_ctx.p2p(pos, mom, np.arange(npar), parlohis, bboxes, [[0, 1], [1, 0]], e, b, precision=precision)
    far = npar / 2 * np.array([0, 0, sep]) / sep**3
    assert isapprox(e[0], far, 1e-3)
    assert isapprox(e[npar - 1], -far, 1e-3)
    assert np.all(b == 0.0)


@pytest.mark.parametrize("N0,kind", [(40, "gauss"), (125, "uniform"), (20, "beamlets"), (300, "gauss")])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_p2p_matches_oracle(gpu_ctx, oracle_mod, N0, kind, precision):
    pos, mom, stretch, t, _ = tree_case(oracle_mod, N=6000, N0=N0, kind=kind)
    p2p, _ = oracle_mod.interaction_lists(t["children"], t["bboxes"], stretch, 0.5)
    e = np.zeros_like(pos)
    b = np.zeros_like(pos)
    re, rb = e.copy(), b.copy()
    gpu_ctx.p2p(pos, mom, t["parindices"], t["parlohis"], t["bboxes"], p2p, e, b, precision=precision)
    oracle_mod.p2p(oracle_mod.VARIANT_GPU, pos, mom, t["parindices"], t["parlohis"], oracle_mod.sort_by_target(p2p),
                   re, rb)
    tol = FP64_STAGE_TOL if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(e, re) < tol and rel(b, rb) < tol


@pytest.mark.parametrize("n", [2, 4, 7])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_downward_pass_matches_oracle(gpu_ctx, oracle_mod, n, precision):
    pos, mom, _, t, leaves = tree_case(oracle_mod, N=5000, N0=40)
    ml = t["max_level"]
    NN = (n + 1) ** 3
    nc = t["nc"]
    rng = np.random.default_rng(11)
    e = rng.normal(0, 1, 3 * NN * nc)
    b = rng.normal(0, 1, 3 * NN * nc)
    re, rb = e.copy(), b.copy()
    for lev in range(1, ml + 1):
        gpu_ctx.l2l(n, t["parents"], t["bboxes"], lev, e, b, precision=precision)
        oracle_mod.l2l(oracle_mod.VARIANT_GPU, n, lev, t["parents"], t["bboxes"], re, rb)
    tol = 1e-12 if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(e, re) < tol and rel(b, rb) < tol
    pe = np.zeros_like(pos)
    pb = np.zeros_like(pos)
    rpe, rpb = pe.copy(), pb.copy()
    gpu_ctx.l2p(n, pos, t["parindices"], t["parlohis"], t["bboxes"], leaves, re, rb, pe, pb, precision=precision)
    oracle_mod.l2p(oracle_mod.VARIANT_GPU, n, pos, t["parindices"], t["parlohis"], t["bboxes"], leaves, re, rb, rpe,
                   rpb)
    tol = FP64_STAGE_TOL if precision == "fp64" else MIXED_STAGE_TOL
    assert rel(pe, rpe) < tol and rel(pb, rpb) < tol
