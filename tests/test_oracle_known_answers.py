"""The CPU oracle pinned against the reference's own known-answer tests.

Each test restates a testset of FMM4RBGPU.jl's test suite (file:line given) with
fixed seeds (the reference draws rand() unseeded).  These run on CPU only.
"""
import numpy as np
import pytest

from conftest import NTHREADS


def isapprox(x, y, rtol):
    """Julia's isapprox for vectors: norm(x - y) <= rtol * max(norm(x), norm(y))."""
    x, y = np.asarray(x, float), np.asarray(y, float)
    return np.linalg.norm(x - y) <= rtol * max(np.linalg.norm(x), np.linalg.norm(y))


def test_ncluster_known_answers(oracle_mod):
    # test/test_cluster_tree/test_treeinfo.jl:3-10
    O = oracle_mod
    assert O.ncluster(4, 2) == 3
    assert O.ncluster(11, 3) == 7
    assert O.ncluster(18, 3) == 15
    assert O.ncluster(2, 4) == 1


def test_bbox_diameter(oracle_mod):
    # test/test_utils/test_bbox.jl:3-9
    assert oracle_mod.diameter([0.0, 0.0, 0.0, 1.0, 1.0, 1.0]) == 0.8660254037844386


def test_cheb2_nodes(oracle_mod):
    # test/test_utils/test_cheb2.jl:2-6
    n = 5
    ref = np.array([np.cos(np.pi * i / n) for i in range(n + 1)])
    np.testing.assert_array_equal(oracle_mod.cheb2(n), ref)
    np.testing.assert_array_equal(oracle_mod.cheb2(n, 0.0, 1.0), (ref + 1.0) / 2.0)


def test_lomuto_partition(oracle_mod):
    # test/test_utils/test_partition.jl:2-9 (1-based labels 1..n -> 0-based)
    data = np.array([1, 1, 5, 2, 4, 4, 3, 3], dtype=float)
    n = len(data)
    labels, _ = oracle_mod.partition(np.arange(n), 0, n - 1, data, pvtindex=n - 1)
    assert np.all(data[labels[:3]] < 3)
    assert np.all(data[labels[3:]] >= 3)


@pytest.mark.parametrize("k1,kval", [(3, 3), (4, 4)])
@pytest.mark.parametrize("seed", [1, 2, 3, 99])
def test_kpermute(oracle_mod, k1, kval, seed):
    # test/test_utils/test_partition.jl:11-28
    data = np.array([2, 1, 3, 4, 4, 6], dtype=float)
    n = len(data)
    labels, ret = oracle_mod.kpermute(np.arange(n), 0, n - 1, data, k=k1 - 1, seed=seed)
    assert ret == k1 - 1
    assert np.all(data[labels[:k1]] <= kval)
    assert np.all(data[labels[k1:]] >= kval)


def test_admissible(oracle_mod):
    # test/test_fmm/test_interaction_lists.jl:2-7
    b1 = [0.0, 0.0, 0.0, 0.5, 0.5, 0.5]
    b2 = [0.5, 0.5, 0.5, 1.0, 1.0, 1.0]
    assert oracle_mod.admissible(b1, b2, [1.0, 1.0, 1.0], 0.50) is False
    assert oracle_mod.admissible(b1, b2, [1.0, 1.0, 2.0], 0.55) is True


def test_cluster_tree_leaves(oracle_mod):
    # test/test_cluster_tree/test_clusters.jl:10-28
    N, N0 = 10000, 32
    pos = np.random.default_rng(0).random((N, 3))
    t = oracle_mod.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    ml = oracle_mod.maxlevel(N, N0)
    assert t["complete"]
    assert len(t["levels"]) == oracle_mod.ncluster(N, N0)
    lrg = slice((1 << ml) - 1, (1 << (ml + 1)) - 1)
    assert np.all(t["levels"][lrg] == ml)
    assert np.all(t["children"][lrg] == -1)
    # every leaf holds a contiguous, ascending block of the permutation
    assert sorted(t["parindices"].tolist()) == list(range(N))


def test_interaction_list_counts_two_etas(oracle_mod):
    # test/test_fmm/test_interaction_lists.jl:9-25
    N, N0 = 1000, 400
    rng = np.random.default_rng(5)
    pos = rng.random((N, 3))
    t = oracle_mod.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    _, m2l = oracle_mod.interaction_lists(t["children"], t["bboxes"], [1.0, 1.0, 1.0], 999.0)
    assert len(m2l) == 2
    p2p, _ = oracle_mod.interaction_lists(t["children"], t["bboxes"], [1.0, 1.0, 1.0], 0.0)
    assert len(p2p) == 16


def test_p2m_momentum_conservation(oracle_mod):
    # test/test_fmm/test_upwardpass.jl:2-17
    O = oracle_mod
    N, N0, n = 100, 200, 2
    rng = np.random.default_rng(2)
    pos = rng.random((N, 3))
    mom = np.zeros((N, 3))
    mom[:, 2] = 2.0
    t = O.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    NN = (n + 1) ** 3
    g = np.zeros(NN * t["nc"])
    m = np.zeros(3 * NN * t["nc"])
    O.p2m(O.VARIANT_CPU, n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], [0], g, m)
    np.testing.assert_allclose(m.reshape(-1, 3)[:NN].sum(axis=0), N * mom[0], rtol=1e-12)


@pytest.mark.parametrize("variant", [0, 1])
def test_upwardpass_conservation(oracle_mod, variant):
    # test/test_fmm/test_upwardpass.jl:19-37, test_gpu_upwardpass.jl:39-85
    O = oracle_mod
    N, N0, n = 1000, 80, 2
    rng = np.random.default_rng(3)
    pos = rng.random((N, 3))
    mom = np.zeros((N, 3))
    gamma = 30.0
    mom[:, 2] = np.sqrt(gamma**2 - 1.0)
    t = O.cluster_tree(pos, N0, [1.0, 1.0, 1.0])
    ml = t["max_level"]
    NN = (n + 1) ** 3
    g = np.zeros(NN * t["nc"])
    m = np.zeros(3 * NN * t["nc"])
    leaves = np.arange((1 << ml) - 1, (1 << (ml + 1)) - 1)
    O.p2m(variant, n, pos, mom, t["parindices"], t["parlohis"], t["bboxes"], leaves, g, m)
    for lev in range(ml, 0, -1):
        O.m2m(variant, n, lev, t["parents"], t["children"], t["bboxes"], g, m)
    np.testing.assert_allclose(g[:NN].sum(), N * gamma, rtol=1e-12)
    np.testing.assert_allclose(m.reshape(-1, 3)[:NN].sum(axis=0), N * mom[0], rtol=1e-12)


@pytest.mark.parametrize("variant", [0, 1])
def test_m2l_far_field(oracle_mod, variant):
    # test/test_fmm/test_interaction.jl:2-30, test_gpu_interaction.jl:2-48
    O = oracle_mod
    distance, n = 10000.0, 3
    NN = (n + 1) ** 3
    bboxes = np.array([[-1, -1, -1, 1, 1, 1], [-1, -1, -1 + distance, 1, 1, 1 + distance]], dtype=float)
    g = np.ones(2 * NN)
    m = np.zeros(3 * 2 * NN)
    e = np.zeros(3 * 2 * NN)
    b = np.zeros(3 * 2 * NN)
    O.m2l(variant, n, bboxes, g, m, [[0, 1], [1, 0]], [0.0, 0.0, 0.0], e, b)
    far = NN * np.array([0, 0, distance]) / distance**3
    assert isapprox(e.reshape(-1, 3)[NN], far, 1e-3)
    assert isapprox(e.reshape(-1, 3)[0], -far, 1e-3)
    assert np.all(b == 0.0)


@pytest.mark.parametrize("variant", [0, 1])
def test_p2p_far_field(oracle_mod, variant):
    # test/test_fmm/test_interaction.jl:32-60
    O = oracle_mod
    npar, sep = 200, 10000.0
    rng = np.random.default_rng(4)
    pos = rng.random((npar, 3))
    mom = np.zeros((npar, 3))
    pos[100:, 2] += sep
    e = np.zeros((npar, 3))
    b = np.zeros((npar, 3))
    O.p2p(variant, pos, mom, np.arange(npar), np.array([[0, 99], [100, 199]]), [[0, 1], [1, 0]], e, b)
    far = npar / 2 * np.array([0, 0, sep]) / sep**3
    assert isapprox(e[0], -far, 1e-3)
    assert isapprox(e[100], far, 1e-3)
    assert np.all(b == 0.0)


def test_fmm_omp_bit_identical_to_serial(oracle_mod):
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(6000, seed=7)
    for variant in (0, 1):
        E1, B1, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 3, 60, 0.5, variant=variant, nthreads=1)
        E8, B8, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 3, 60, 0.5, variant=variant, nthreads=NTHREADS)
        assert np.array_equal(E1, E8) and np.array_equal(B1, B8)


def test_fmm_converges_to_bruteforce(oracle_mod):
    """Truncation error of the serial FMM against BruteForce decreases with n."""
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(8192, seed=11)
    Eb, Bb = oracle_mod.bruteforce(pos, mom, -1.0, 1.0, NTHREADS)
    errs, errs_b = [], []
    for n in (2, 4, 6):
        E, B, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, n, 125, 0.5, nthreads=NTHREADS)
        errs.append(beams.rel_l2(E, Eb))
        errs_b.append(beams.rel_l2(B, Bb))
    assert errs[0] > errs[1] > errs[2]
    assert errs_b[0] > errs_b[1] > errs_b[2]
    assert errs[1] < 5e-3 and errs_b[1] < 5e-3


def test_cpu_and_gpu_variants_agree(oracle_mod):
    """FMM (cheb2 nodes) and FMMGPU (cheb2coord nodes) differ only by rounding."""
    from fmmb200 import beams

    pos, mom = beams.uniform(4096, seed=0)
    Ec, Bc, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 4, 125, 0.5, variant=0, nthreads=NTHREADS)
    Eg, Bg, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 4, 125, 0.5, variant=1, nthreads=NTHREADS)
    assert beams.rel_l2(Eg, Ec) < 1e-12
    assert np.all(Bc == 0.0) and np.all(Bg == 0.0)


def test_tree_leaf_above_max_level_is_reported(oracle_mod):
    # N = 2*N0 + 1: the right child of the root holds N0 particles (a leaf at level 1 < ml = 2)
    pos = np.random.default_rng(0).random((251, 3))
    t = oracle_mod.cluster_tree(pos, 125, [1.0, 1.0, 1.0])
    assert not t["complete"]


def test_empty_lists_give_empty_csr(oracle_mod):
    assert oracle_mod.ilistptrs(np.zeros((0, 2), np.int64)).tolist() == [0]
    ptrs = oracle_mod.ilistptrs(oracle_mod.sort_by_target([[2, 0], [0, 1], [2, 3], [0, 0]]))
    assert ptrs.tolist() == [0, 2, 4]


def test_coincident_nodes_weights(oracle_mod):
    """A box of zero extent makes all n+1 interpolation nodes coincide.  The serial
    reference's lgweight (src/fmm/upwardpass.jl:6-9) then returns a weight of 1 on every
    node (convert.(Float64, bitarr)), so its weights sum to n+1; the GPU kernels'
    exact-node rule puts the single weight on the last matching node
    (src/gpu_fmm/gpu_upwardpass.jl:52-54).  The oracle keeps both; the device follows
    the second, which is the one that reproduces the direct sum on planar inputs."""
    import numpy as np

    nodes = np.full(5, 0.25)
    w_cpu = oracle_mod.lgweight(0.25, nodes, gpu=False)
    w_gpu = oracle_mod.lgweight(0.25, nodes, gpu=True)
    assert np.array_equal(w_cpu, np.ones(5))
    assert np.array_equal(w_gpu, np.array([0.0, 0.0, 0.0, 0.0, 1.0]))


def test_planar_input_gpu_variant_matches_bruteforce(oracle_mod):
    import numpy as np
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(4000, seed=0)
    pos[:, 2] = 0.0
    Eb, _ = oracle_mod.bruteforce(pos, mom, -1.0, 1.0, 4)
    Eg, _, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 4, 64, 0.5, variant=oracle_mod.VARIANT_GPU, nthreads=4)
    Ec, _, _ = oracle_mod.fmm(pos, mom, -1.0, 1.0, 4, 64, 0.5, variant=oracle_mod.VARIANT_CPU, nthreads=4)
    err = lambda a: float(np.linalg.norm(a - Eb) / np.linalg.norm(Eb))  # noqa: E731
    assert err(Eg) < 1e-3  # the FMM truncation error
    assert err(Ec) > 1.0  # the serial reference's all-ones weights on coincident nodes
