"""The hand-written adjoint of (E, B) = F(positions, momenta).

Loss L = sum_i (w_i . E_i + v_i . B_i) with w, v ~ N(0, 1) (seed 1).  Checks:
  * N <= N0 (one leaf: the FMM is the direct sum): the gradient equals torch
    autograd of an FP64 direct sum (the stand-in for the ForwardDiff gradient of
    the reference's BruteForce) to 1e-10;
  * a multi-level tree: central finite differences (h = 1e-6) of the C-ABI
    forward on 64 seeded coordinates, tree and lists unchanged at x +- h,
    agree within 1e-4 relative L2;
  * against the autograd direct sum at N = 4096 within the FMM's truncation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R_E = 2.8179403699772166e-15


def direct_grad_torch(pos, mom, w, v, charge=-1.0, lam=1.0):
    import torch

    x = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    u = torch.tensor(mom, dtype=torch.float64, requires_grad=True)
    amp = R_E * charge / lam
    R = x[:, None, :] - x[None, :, :]
    uj = u[None, :, :].expand_as(R)
    d = (R * R).sum(-1) + (uj * R).sum(-1) ** 2 + 2.220446049250313e-16
    eye = torch.eye(len(pos), dtype=torch.bool)
    f = torch.where(eye, torch.zeros_like(d), d ** -1.5)
    K = R * f[..., None]
    g = torch.sqrt(1.0 + (u * u).sum(-1))
    E = amp * (g[None, :, None] * K).sum(1)
    B = amp * torch.linalg.cross(uj, K, dim=-1).sum(1)
    L = (torch.tensor(w) * E).sum() + (torch.tensor(v) * B).sum()
    L.backward()
    return float(L), x.grad.numpy(), u.grad.numpy()


def fmm_loss_grad(ctx, pos, mom, alg, w, v):
    E, B = ctx.forward(pos, mom, alg, save_for_backward=True)
    L = float((w * E).sum() + (v * B).sum())
    gx, gu = ctx.backward(w, v)
    return L, gx, gu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("N", [2, 57, 200])
def test_single_leaf_matches_autograd_direct_sum(gpu_ctx, N):
    import fmmb200
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(N, seed=3)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    L, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=4, N0=256, eta=0.5), w, v)
    Lt, gxt, gut = direct_grad_torch(pos, mom, w, v)
    assert abs(L - Lt) <= 1e-12 * abs(Lt)
    assert rel(gx, gxt) < 1e-10
    assert rel(gu, gut) < 1e-10


def _fd_case(gpu_ctx, alg, N, seed=5, ncoord=64, h=1e-6):
    from fmmb200 import beams

    pos, mom = beams.gaussian_bunch(N, seed=seed)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    L, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, alg, w, v)
    t0 = gpu_ctx.tree()
    m0, p0 = gpu_ctx.lists()
    pick = np.random.default_rng(7).choice(6 * N, size=ncoord, replace=False)
    fd, an = [], []
    for k in pick:
        arr, idx = (pos, k) if k < 3 * N else (mom, k - 3 * N)
        i, c = divmod(idx, 3)
        vals = []
        for sgn in (1.0, -1.0):
            a2 = arr.copy()
            a2[i, c] += sgn * h
            P, U = (a2, mom) if arr is pos else (pos, a2)
            E, B = gpu_ctx.forward(P, U, alg)
            t = gpu_ctx.tree()
            m, p = gpu_ctx.lists()
            assert np.array_equal(t["parindices"], t0["parindices"]), "tree changed under the perturbation"
            assert np.array_equal(m, m0) and np.array_equal(p, p0), "lists changed under the perturbation"
            vals.append(float((w * E).sum() + (v * B).sum()))
        fd.append((vals[0] - vals[1]) / (2 * h))
        an.append((gx if arr is pos else gu)[i, c])
    return np.array(fd), np.array(an)


@pytest.mark.parametrize("n,N0", [(4, 64), (3, 40)])
def test_gradient_matches_finite_differences(gpu_ctx, n, N0):
    import fmmb200

    fd, an = _fd_case(gpu_ctx, fmmb200.FMMB200(n=n, N0=N0, eta=0.5), 4096)
    assert rel(an, fd) < 1e-4, (rel(an, fd), np.c_[fd, an][:8])


def test_gradient_matches_finite_differences_at_262144(gpu_ctx):
    """The same check on a 262,144-particle Gaussian bunch, n = 4, N0 = 125, eta = 1/2."""
    import fmmb200

    fd, an = _fd_case(gpu_ctx, fmmb200.FMMB200(n=4, N0=125, eta=0.5), 262144)
    assert rel(an, fd) < 1e-4, rel(an, fd)


def test_mixed_forward_adjoint_matches_fp64(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    N = 20000
    pos, mom = beams.beamlets(N, seed=2)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    _, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=5, N0=64, eta=0.5), w, v)
    _, gxm, gum = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=5, N0=64, eta=0.5, precision="mixed"), w, v)
    assert rel(gxm, gx) < 1e-4 and rel(gum, gu) < 1e-4


@pytest.mark.parametrize("kind,N,n,N0,eta", [("gauss", 30000, 4, 125, 0.5), ("gauss", 30000, 4, 32, 0.5),
                                              ("uniform", 20000, 3, 100, 0.5), ("beamlets", 20000, 2, 200, 0.5),
                                              ("gauss", 20000, 4, 64, 0.7), ("duplicates", 20000, 4, 64, 0.5),
                                              ("gauss", 20000, 1, 32, 0.5), ("gauss", 30000, 6, 400, 0.5),
                                              ("uniform", 30000, 7, 600, 0.5), ("gauss", 30000, 8, 800, 0.5)])
def test_mixed_adjoint_kernels_match_fp64(gpu_ctx, kind, N, n, N0, eta):
    """The mixed form's adjoint runs M2L^T and P2P^T in FP32 (hi/lo coordinates in
    the near field); it stays within 1e-4 of the FP64 adjoint for every lane-group
    width (leaf sizes 32..256), for eta > 1/2 (masked nodes, packed unfactored
    M2L^T), for n = 1..7 (scalar factored M2L^T) and n = 8 (packed unfactored)."""
    import fmmb200
    from fmmb200 import beams

    gen = {"gauss": beams.gaussian_bunch, "uniform": beams.uniform, "beamlets": beams.beamlets,
           "duplicates": beams.gaussian_bunch}[kind]
    pos, mom = gen(N, seed=4)
    if kind == "duplicates":  # twins at one position: the regularised kernel's derivative at R = 0
        pos[1::2] = pos[0::2]
    if kind == "uniform":
        mom = np.random.default_rng(5).normal(0, 0.5, (N, 3))  # nonzero momenta: B and d/du are exercised
    rng = np.random.default_rng(2)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    _, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=n, N0=N0, eta=eta), w, v)
    _, gxm, gum = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=n, N0=N0, eta=eta, precision="mixed"), w, v)
    assert np.all(np.isfinite(gxm)) and np.all(np.isfinite(gum))
    assert rel(gxm, gx) < 1e-4 and rel(gum, gu) < 1e-4, (rel(gxm, gx), rel(gum, gu))


def test_mixed_single_leaf_matches_autograd_direct_sum(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    N = 200
    pos, mom = beams.gaussian_bunch(N, seed=11)
    rng = np.random.default_rng(3)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    _, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=4, N0=256, eta=0.5, precision="mixed"), w, v)
    _, gxt, gut = direct_grad_torch(pos, mom, w, v)
    assert rel(gx, gxt) < 1e-5 and rel(gu, gut) < 1e-5


def test_gradient_matches_finite_differences_eta_above_half(gpu_ctx):
    import fmmb200

    fd, an = _fd_case(gpu_ctx, fmmb200.FMMB200(n=3, N0=40, eta=0.7), 4096)
    assert rel(an, fd) < 1e-4, (rel(an, fd), np.c_[fd, an][:8])


def test_gradient_close_to_autograd_direct_sum(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    N = 4096
    pos, mom = beams.gaussian_bunch(N, seed=9)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    _, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=6, N0=64, eta=0.5), w, v)
    _, gxt, gut = direct_grad_torch(pos, mom, w, v)
    # the FMM's own truncation error bounds the agreement
    assert rel(gx, gxt) < 2e-2 and rel(gu, gut) < 2e-2


def test_backward_without_saved_forward_is_an_error(gpu_ctx):
    import fmmb200
    from fmmb200 import beams

    ctx = fmmb200.Context(0)
    pos, mom = beams.gaussian_bunch(1000, seed=1)
    with pytest.raises(fmmb200.FMMB200Error) as ei:
        ctx.backward(np.zeros_like(pos), np.zeros_like(pos))
    assert ei.value.status == fmmb200.ERR_NO_STATE
    ctx.forward(pos, mom, fmmb200.FMMB200(n=3, N0=64, eta=0.5))  # not saved
    with pytest.raises(fmmb200.FMMB200Error) as ei:
        ctx.backward(np.zeros_like(pos), np.zeros_like(pos))
    assert ei.value.status == fmmb200.ERR_NO_STATE
    ctx.close()


@pytest.mark.parametrize("eta", [0.5, 0.6])
def test_mixed_adjoint_on_a_line_stays_finite(gpu_ctx, eta):
    """Half a million particles on a line: the boxes are flat in y and z, and neighbouring
    boxes' end nodes can lie ~1e-12 apart, where s^5 = d^-5/2 exceeds the FP32 range.  The
    mixed adjoint forms those terms as f (s^2 ...) and stays finite and within 1e-4 of FP64
    (it returned NaN for eta = 0.6 before)."""
    import fmmb200
    from fmmb200 import beams

    N = 500000
    pos, _ = beams.uniform(N, seed=16)
    pos[:, 1] = 0.2
    pos[:, 2] = 0.7
    mom = np.random.default_rng(16).normal(0, 0.5, (N, 3))
    rng = np.random.default_rng(3)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    _, gx, gu = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=1, N0=64, eta=eta), w, v)
    _, gxm, gum = fmm_loss_grad(gpu_ctx, pos, mom, fmmb200.FMMB200(n=1, N0=64, eta=eta, precision="mixed"), w, v)
    assert np.all(np.isfinite(gxm)) and np.all(np.isfinite(gum))
    assert rel(gxm, gx) < 1e-4 and rel(gum, gu) < 1e-4, (rel(gxm, gx), rel(gum, gu))


def _random_case(k):
    rng = np.random.default_rng(1000 + k)
    N = int(rng.choice([20000, 100000, 300000]))
    n = int(rng.integers(1, 9))
    N0 = int(rng.choice([16, 40, 64, 125, 200, 400]))
    eta = float(rng.choice([0.3, 0.5, 0.6, 0.7]))
    dist = str(rng.choice(["gauss", "uniform", "beamlets", "planar", "line"]))
    return N, n, N0, eta, dist


@pytest.mark.parametrize("k", range(12))
def test_random_configurations_mixed_vs_fp64(gpu_ctx, k):
    """Seeded random (N, n, N0, eta, distribution) cases, degenerate planar and collinear
    beams included: the mixed forward within 1e-5 and its adjoint within 1e-4 of FP64,
    every value finite."""
    import fmmb200
    from fmmb200 import beams

    N, n, N0, eta, dist = _random_case(k)
    if dist == "gauss":
        pos, mom = beams.gaussian_bunch(N, seed=k)
    elif dist == "beamlets":
        pos, mom = beams.beamlets(N, seed=k)
    else:
        pos, _ = beams.uniform(N, seed=k)
        mom = np.random.default_rng(k).normal(0, 0.5, (N, 3))
        if dist == "planar":
            pos[:, 2] = 0.3
        elif dist == "line":
            pos[:, 1] = 0.2
            pos[:, 2] = 0.7
    rng = np.random.default_rng(k + 7)
    w = rng.normal(size=(N, 3))
    v = rng.normal(size=(N, 3))
    res = {}
    for prec in ("fp64", "mixed"):
        alg = fmmb200.FMMB200(n=n, N0=N0, eta=eta, precision=prec)
        E, B = gpu_ctx.forward(pos, mom, alg, save_for_backward=True)
        gx, gu = gpu_ctx.backward(w, v)
        res[prec] = (E, B, gx, gu)
    for a in res["mixed"]:
        assert np.all(np.isfinite(a))
    (E, B, gx, gu), (Em, Bm, gxm, gum) = res["fp64"], res["mixed"]
    case = (N, n, N0, eta, dist)
    assert rel(Em, E) < 1e-5 and rel(Bm, B) < 1e-5, (case, rel(Em, E), rel(Bm, B))
    assert rel(gxm, gx) < 1e-4 and rel(gum, gu) < 1e-4, (case, rel(gxm, gx), rel(gum, gu))
