"""Golden vectors (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle reproduces its committed vectors bit for bit.
GPU: the device tree, lists and FP64 fields reproduce them (tree and lists
bit-exact, fields within 1e-12 relative L2).
"""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT

FILES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - b) / nb) if nb else float(np.abs(a).max())


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_oracle_reproduces_golden(oracle_mod, path):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden

    g = np.load(path)
    new = make_golden.make(os.path.basename(path)[:-4])
    for key in g.files:
        assert np.array_equal(np.asarray(new[key]), g[key]), key


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_device_matches_golden(gpu_ctx, path):
    import fmmb200

    g = np.load(path)
    n, N0, eta, q, lam = g["params"]
    alg = fmmb200.FMMB200(n=int(n), N0=int(N0), eta=float(eta))
    E, B = gpu_ctx.forward(g["pos"], g["mom"], alg, charge=float(q), lambda_=float(lam))
    assert rel(E, g["E_fmm"]) < 1e-12 and rel(B, g["B_fmm"]) < 1e-12
    assert rel(E, g["E_fmmgpu"]) < 1e-12
    t = gpu_ctx.tree()
    np.testing.assert_array_equal(t["parindices"], g["parindices"])
    np.testing.assert_array_equal(t["parlohis"], g["parlohis"])
    assert np.array_equal(t["bboxes"], g["bboxes"])
    m2l, p2p = gpu_ctx.lists()
    for got, ref in ((m2l, g["m2l"]), (p2p, g["p2p"])):
        ref = ref[np.lexsort((ref[:, 1], ref[:, 0]))]
        np.testing.assert_array_equal(got, ref)
    st = gpu_ctx.stats()
    assert st["pavg"] == g["pavg"].tolist() and st["stretch"] == g["stretch"].tolist()
