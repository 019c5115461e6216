"""ctypes access to the CPU oracle (``oracle/build/liboracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is the checker for the CUDA path and the
timed CPU baseline; only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU arms import this module.  The product library never calls it.

Arrays follow the reference's memory layouts (see ``fmm_oracle.h``): particle
vectors are ``(N, 3)`` float64 (AoS, the layout of ``Vector{SVector{3,Float64}}``),
node and particle indices are 0-based int64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")

VARIANT_CPU = 0  # serial `FMM` (src/fmm/*.jl)
VARIANT_GPU = 1  # `FMMGPU` kernels (src/gpu_fmm/*.jl) without the gpu_M2L! race

_lib = None
_lock = threading.Lock()

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int64)
_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_int = ctypes.c_int


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(_HERE, "fmm_oracle.c")
            if not os.path.exists(LIB_PATH) or (
                os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(LIB_PATH)
            ):
                build()
            L = ctypes.CDLL(LIB_PATH)
            sig = {
                "orc_maxlevel": (_i64, [_i64, _i64]),
                "orc_ncluster": (_i64, [_i64, _i64]),
                "orc_pavg": (None, [_i64, _d, _d]),
                "orc_stretch": (None, [_d, _d]),
                "orc_partition": (_i64, [_i, _i64, _i64, _d, _i64, _i64, _i64, _int]),
                "orc_kpermute": (_i64, [_i, _i64, _i64, _d, _i64, _i64, _i64, ctypes.c_uint64, _int]),
                "orc_cluster_tree": (_int, [_i64, _d, _i64, _d, ctypes.c_uint64, _int, _i, _i, _i, _i, _i, _d]),
                "orc_diameter": (_f64, [_d, _d]),
                "orc_admissible": (_int, [_d, _d, _d, _f64]),
                "orc_interaction_lists": (_int, [_i64, _i, _d, _d, _f64, _i, _i64, _i, _i, _i64, _i]),
                "orc_sort_by_target": (None, [_i64, _i]),
                "orc_ilistptrs": (_i64, [_i64, _i, _i]),
                "orc_cheb2": (None, [_int, _f64, _f64, _d]),
                "orc_cheb2coord": (_f64, [_i64, _f64, _f64, _int]),
                "orc_lgweight": (None, [_f64, _d, _int, _d]),
                "orc_lgweight_gpu": (None, [_f64, _d, _int, _d]),
                "orc_p2m": (None, [_int, _int, _d, _d, _i, _i, _d, _i64, _i, _d, _d]),
                "orc_m2m": (None, [_int, _int, _i64, _i, _i, _d, _d, _d]),
                "orc_m2l": (None, [_int, _int, _d, _d, _d, _i64, _i, _d, _d, _d]),
                "orc_p2p": (None, [_int, _d, _d, _i, _i, _i64, _i, _d, _d]),
                "orc_l2l": (None, [_int, _int, _i64, _i, _d, _d, _d]),
                "orc_l2p": (None, [_int, _int, _d, _i, _i, _d, _i64, _i, _d, _d, _d, _d]),
                "orc_fmm": (_int, [_int, _i64, _d, _d, _f64, _f64, _int, _i64, _f64, _d,
                                   ctypes.c_uint64, _int, _d, _d, _d]),
                "orc_bruteforce": (None, [_i64, _d, _d, _f64, _f64, _int, _d, _d]),
                "orc_direct_targets": (None, [_i64, _d, _d, _f64, _f64, _i64, _i, _int, _d, _d]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_d)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def _f(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _n(a):
    return np.ascontiguousarray(a, dtype=np.int64)


# --------------------------------------------------------------------------- tree shape
def maxlevel(N: int, N0: int) -> int:
    return int(lib().orc_maxlevel(N, N0))


def ncluster(N: int, N0: int) -> int:
    return int(lib().orc_ncluster(N, N0))


def pavg(mom) -> np.ndarray:
    mom = _f(mom, (-1, 3))
    out = np.zeros(3)
    lib().orc_pavg(mom.shape[0], _dp(mom), _dp(out))
    return out


def stretch(p) -> np.ndarray:
    p = _f(p, (3,))
    out = np.zeros(3)
    lib().orc_stretch(_dp(p), _dp(out))
    return out


def partition(labels, lo, hi, data, pvtindex, tiebreak=False):
    labels = _n(labels).copy()
    data = _f(data, (-1,))
    j = lib().orc_partition(_ip(labels), lo, hi, _dp(data), 1, 0, pvtindex, int(tiebreak))
    return labels, int(j)


def kpermute(labels, lo, hi, data, k, seed=1, tiebreak=False):
    labels = _n(labels).copy()
    data = _f(data, (-1,))
    j = lib().orc_kpermute(_ip(labels), lo, hi, _dp(data), 1, 0, k, seed, int(tiebreak))
    return labels, int(j)


def cluster_tree(pos, N0: int, stretch_, seed: int = 1, canonical: bool = True) -> dict:
    pos = _f(pos, (-1, 3))
    N = pos.shape[0]
    nc = ncluster(N, N0)
    t = dict(
        parindices=np.zeros(N, np.int64),
        levels=np.zeros(nc, np.int64),
        parlohis=np.zeros((nc, 2), np.int64),
        parents=np.zeros(nc, np.int64),
        children=np.zeros((nc, 2), np.int64),
        bboxes=np.zeros((nc, 6)),
    )
    s = _f(stretch_, (3,))
    rc = lib().orc_cluster_tree(N, _dp(pos), N0, _dp(s), seed, int(canonical),
                                _ip(t["parindices"]), _ip(t["levels"]), _ip(t["parlohis"]),
                                _ip(t["parents"]), _ip(t["children"]), _dp(t["bboxes"]))
    t["complete"] = rc == 0
    t["max_level"] = maxlevel(N, N0)
    t["nc"] = nc
    return t


def diameter(bbox, stretch_=(1.0, 1.0, 1.0)) -> float:
    return float(lib().orc_diameter(_dp(_f(bbox, (6,))), _dp(_f(stretch_, (3,)))))


def admissible(b1, b2, stretch_, eta) -> bool:
    return bool(lib().orc_admissible(_dp(_f(b1, (6,))), _dp(_f(b2, (6,))), _dp(_f(stretch_, (3,))), eta))


def interaction_lists(children, bboxes, stretch_, eta):
    """DFS-ordered (p2p, m2l) pair lists as (n, 2) int64 arrays."""
    children = _n(children).reshape(-1, 2)
    bboxes = _f(bboxes, (-1, 6))
    s = _f(stretch_, (3,))
    np2p = ctypes.c_int64(0)
    nm2l = ctypes.c_int64(0)
    L = lib()
    L.orc_interaction_lists(children.shape[0], _ip(children), _dp(bboxes), _dp(s), eta,
                            None, 0, ctypes.byref(np2p), None, 0, ctypes.byref(nm2l))
    p2p = np.zeros((max(np2p.value, 1), 2), np.int64)
    m2l = np.zeros((max(nm2l.value, 1), 2), np.int64)
    rc = L.orc_interaction_lists(children.shape[0], _ip(children), _dp(bboxes), _dp(s), eta,
                                 _ip(p2p), p2p.shape[0], ctypes.byref(np2p), _ip(m2l), m2l.shape[0],
                                 ctypes.byref(nm2l))
    assert rc == 0
    return p2p[: np2p.value].copy(), m2l[: nm2l.value].copy()


def sort_by_target(pairs):
    pairs = _n(pairs).reshape(-1, 2).copy()
    lib().orc_sort_by_target(pairs.shape[0], _ip(pairs))
    return pairs


def ilistptrs(pairs):
    pairs = _n(pairs).reshape(-1, 2)
    ptrs = np.zeros(pairs.shape[0] + 1, np.int64)
    ng = lib().orc_ilistptrs(pairs.shape[0], _ip(pairs), _ip(ptrs))
    return ptrs[: ng + 1].copy()


# --------------------------------------------------------------------------- interpolation
def cheb2(n, a=-1.0, b=1.0):
    out = np.zeros(n + 1)
    lib().orc_cheb2(n, a, b, _dp(out))
    return out


def cheb2coord(i1, a, b, D):
    return float(lib().orc_cheb2coord(i1, a, b, D))


def lgweight(x, nodes, gpu=False):
    nodes = _f(nodes, (-1,))
    out = np.zeros_like(nodes)
    fn = lib().orc_lgweight_gpu if gpu else lib().orc_lgweight
    fn(x, _dp(nodes), nodes.shape[0] - 1, _dp(out))
    return out


# --------------------------------------------------------------------------- passes (in place)
def p2m(variant, n, pos, mom, parindices, parlohis, bboxes, leaf_ids, gammas, mmom):
    lib().orc_p2m(variant, n, _dp(pos), _dp(mom), _ip(parindices), _ip(parlohis), _dp(bboxes),
                  len(leaf_ids), _ip(_n(leaf_ids)), _dp(gammas), _dp(mmom))


def m2m(variant, n, level, parents, children, bboxes, gammas, mmom):
    lib().orc_m2m(variant, n, level, _ip(parents), _ip(children), _dp(bboxes), _dp(gammas), _dp(mmom))


def m2l(variant, n, bboxes, gammas, mmom, pairs, p_avg, mef, mbf):
    pairs = _n(pairs).reshape(-1, 2)
    lib().orc_m2l(variant, n, _dp(bboxes), _dp(gammas), _dp(mmom), pairs.shape[0], _ip(pairs),
                  _dp(_f(p_avg, (3,))), _dp(mef), _dp(mbf))


def p2p(variant, pos, mom, parindices, parlohis, pairs, ef, bf):
    pairs = _n(pairs).reshape(-1, 2)
    lib().orc_p2p(variant, _dp(pos), _dp(mom), _ip(parindices), _ip(parlohis), pairs.shape[0],
                  _ip(pairs), _dp(ef), _dp(bf))


def l2l(variant, n, level, parents, bboxes, mef, mbf):
    lib().orc_l2l(variant, n, level, _ip(parents), _dp(bboxes), _dp(mef), _dp(mbf))


def l2p(variant, n, pos, parindices, parlohis, bboxes, leaf_ids, mef, mbf, ef, bf):
    lib().orc_l2p(variant, n, _dp(pos), _ip(parindices), _ip(parlohis), _dp(bboxes), len(leaf_ids),
                  _ip(_n(leaf_ids)), _dp(mef), _dp(mbf), _dp(ef), _dp(bf))


# --------------------------------------------------------------------------- drivers
STATS_KEYS = ("max_level", "nc", "nm2l", "np2p", "t_tree", "t_up", "t_lists", "t_m2l", "t_p2p", "t_down")


def fmm(pos, mom, charge, lam, n, N0, eta, variant=VARIANT_CPU, p_avg=None, seed=1, nthreads=1):
    """update_particles_field!(beam, FMM(...) / FMMGPU(...); lambda) -> (E, B, stats)."""
    pos = _f(pos, (-1, 3))
    mom = _f(mom, (-1, 3))
    N = pos.shape[0]
    E = np.zeros((N, 3))
    B = np.zeros((N, 3))
    st = np.zeros(len(STATS_KEYS))
    pa = None if p_avg is None else _f(p_avg, (3,))
    rc = lib().orc_fmm(variant, N, _dp(pos), _dp(mom), charge, lam, n, N0, eta, _dp(pa), seed,
                       nthreads, _dp(E), _dp(B), _dp(st))
    if rc != 0:
        raise RuntimeError(f"oracle fmm failed with status {rc}")
    return E, B, dict(zip(STATS_KEYS, st.tolist()))


def bruteforce(pos, mom, charge, lam, nthreads=1):
    pos = _f(pos, (-1, 3))
    mom = _f(mom, (-1, 3))
    E = np.zeros_like(pos)
    B = np.zeros_like(pos)
    lib().orc_bruteforce(pos.shape[0], _dp(pos), _dp(mom), charge, lam, nthreads, _dp(E), _dp(B))
    return E, B


def direct_targets(pos, mom, charge, lam, targets, nthreads=1):
    pos = _f(pos, (-1, 3))
    mom = _f(mom, (-1, 3))
    targets = _n(targets)
    E = np.zeros((targets.shape[0], 3))
    B = np.zeros((targets.shape[0], 3))
    lib().orc_direct_targets(pos.shape[0], _dp(pos), _dp(mom), charge, lam, targets.shape[0],
                             _ip(targets), nthreads, _dp(E), _dp(B))
    return E, B
