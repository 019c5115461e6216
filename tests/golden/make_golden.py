"""Generates tests/golden/*.npz with the CPU oracle (the restatement of the
reference's serial FMM, BruteForce, ClusterTree and dual traversal).

Run from the repository root:  python tests/golden/make_golden.py
The reference itself (Julia) cannot run in this environment; its own
known-answer tests are ported in tests/test_oracle_known_answers.py.  These
fixtures pin the oracle's current outputs so that later changes to it (and the
device path) are compared against fixed vectors.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))

import oracle  # noqa: E402
from fmmb200 import beams  # noqa: E402

CASES = {
    # name: (generator, N, seed, n, N0, eta, charge, lambda)
    "uniform_n4": (beams.uniform, 2000, 0, 4, 125, 0.5, -1.0, 1.0),
    "bunch_n3": (beams.gaussian_bunch, 3000, 1, 3, 50, 0.5, -1.0, 1.0),
    "beamlets_n5": (beams.beamlets, 2500, 2, 5, 64, 0.5, -1.0, 2.0),
}


def make(name):
    gen, N, seed, n, N0, eta, q, lam = CASES[name]
    pos, mom = gen(N, seed=seed)
    p = oracle.pavg(mom)
    s = oracle.stretch(p)
    tree = oracle.cluster_tree(pos, N0, s)
    p2p, m2l = oracle.interaction_lists(tree["children"], tree["bboxes"], s, eta)
    E, B, st = oracle.fmm(pos, mom, q, lam, n, N0, eta, variant=oracle.VARIANT_CPU, nthreads=4)
    Eg, Bg, _ = oracle.fmm(pos, mom, q, lam, n, N0, eta, variant=oracle.VARIANT_GPU, nthreads=4)
    Eb, Bb = oracle.bruteforce(pos, mom, q, lam, 4)
    return dict(pos=pos, mom=mom, params=np.array([n, N0, eta, q, lam]), pavg=p, stretch=s,
                parindices=tree["parindices"], parlohis=tree["parlohis"], bboxes=tree["bboxes"],
                m2l=m2l, p2p=p2p, E_fmm=E, B_fmm=B, E_fmmgpu=Eg, B_fmmgpu=Bg, E_bf=Eb, B_bf=Bb,
                nm2l=np.int64(st["nm2l"]), np2p=np.int64(st["np2p"]))


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make(name))
        print("wrote", name)
