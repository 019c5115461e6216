"""Host-side mirror of the reference's interface for the space-charge field path.

Reference (FMM4RBGPU.jl):
  Particles(; pos, mom, charge=-1.0, mass=1.0)          src/particles.jl:11-22
  const Beam = Particles                                 src/particles.jl:25
  FMMGPU(; n, N0, eta)                                   src/update_particles_field.jl:15-19
  update_particles_field!(particles, alg; lambda)        src/update_particles_field.jl:66-148
  ClusterTree(particles; N0, stretch)                    src/cluster_tree/cluster_tree.jl:12-18
  InteractionListsGPU(clusters; stretch, eta)            src/gpu_fmm/gpu_interaction_lists.jl:27-40
  gpu_P2M!/gpu_M2M!/gpu_M2L!/gpu_P2P!/gpu_L2L!/gpu_L2P!  src/gpu_fmm/*.jl

Here the algorithm is ``FMMB200(eta, N0, n)`` and every stage runs on the GPU
through libfmmb200.so.  Indices are 0-based (the reference is 1-based).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import FMMB200Error

R_E = 2.8179403699772166e-15
# cudaStreamLegacy ((cudaStream_t)0x1): the legacy default stream as an explicit handle
CUDA_STREAM_LEGACY = 1


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _i64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a if shape is None else a.reshape(shape)


def _pd(a):
    return None if a is None else a.ctypes.data_as(L.p_f64)


def _pi(a):
    return None if a is None else a.ctypes.data_as(L.p_i64)


class Particles:
    """Particle container (src/particles.jl:1-22).

    ``pos`` and ``mom`` are 3 x N matrices like the reference's constructor
    arguments (an N x 3 array is accepted too).  Fields are stored as N x 3
    float64 arrays -- the memory layout of Vector{SVector{3,Float64}}.
    Momenta are u = p/(mc) = gamma*beta.
    """

    def __init__(self, *, pos, mom, charge: float = -1.0, mass: float = 1.0):
        pos = np.asarray(pos, dtype=np.float64)
        mom = np.asarray(mom, dtype=np.float64)
        if pos.shape != mom.shape:
            raise ValueError("size(pos) must equal size(mom)")  # particles.jl:12
        if pos.ndim != 2 or 3 not in pos.shape:
            raise ValueError("pos must be 3 x N")  # particles.jl:13
        if pos.shape[0] == 3:  # the reference's 3 x N matrices (a 3 x 3 input is read this way too)
            pos, mom = pos.T, mom.T
        self.npar = pos.shape[0]
        self.charge = float(charge)
        self.mass = float(mass)
        self.positions = np.ascontiguousarray(pos)
        self.momenta = np.ascontiguousarray(mom)
        self.efields = np.zeros((self.npar, 3))
        self.bfields = np.zeros((self.npar, 3))


Beam = Particles


@dataclass(frozen=True)
class FMMB200:
    """The B200 algorithm selector; fields as the reference's FMMGPU (n, N0, eta).

    ``precision`` is "fp64" (the plain FP64 path, the drop-in) or "mixed" (FP32
    arithmetic whose per-source partial sums are folded into FP64 sums, FP64
    geometry and final accumulation).
    """

    n: int
    N0: int
    eta: float
    precision: str = "fp64"

    @staticmethod
    def positional(eta: float, N0: int, n: int, precision: str = "fp64") -> "FMMB200":
        """FMMB200(eta, N0, n) in the argument order of the field evaluation call."""
        return FMMB200(n=n, N0=N0, eta=eta, precision=precision)

    @property
    def precision_code(self) -> int:
        if self.precision == "fp64":
            return L.PRECISION_FP64
        if self.precision == "mixed":
            return L.PRECISION_MIXED
        raise ValueError("precision must be 'fp64' or 'mixed'")


class Context:
    """One libfmmb200 context (device memory, stream, saved forward state)."""

    def __init__(self, device: int = 0):
        self._lib = L.load()
        h = ctypes.c_void_p()
        st = self._lib.fmmb200_create(ctypes.byref(h), int(device))
        if st != L.OK:
            raise FMMB200Error(st, f"fmmb200_create(device={device}) failed (no CUDA device?)")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fmmb200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != L.OK:
            msg = self._lib.fmmb200_last_error(self._h)
            raise FMMB200Error(st, msg.decode() if msg else "")

    # ---------------------------------------------------------------- settings
    def set_stream(self, stream_ptr: int | None):
        """Run on a cudaStream_t handle (``torch.cuda.Stream.cuda_stream``); None: the
        context's own stream.  The handle 0, torch's default stream, is the legacy default
        stream and is passed as cudaStreamLegacy: the library reads a NULL handle as its own
        stream, which is non-blocking and would not be ordered after torch's work."""
        handle = None if stream_ptr is None else (CUDA_STREAM_LEGACY if stream_ptr == 0 else stream_ptr)
        self._check(self._lib.fmmb200_set_stream(self._h, ctypes.c_void_p(handle)))

    def set_timing(self, enable: bool):
        self._check(self._lib.fmmb200_set_timing(self._h, int(bool(enable))))

    def set_m2l_engine(self, engine: str):
        """Mixed-form M2L engine: "auto" / "cuda_cores" (packed FP32x2 kernel) or
        "tensor_cores" (tcgen05 TF32 MMAs for n <= 4 and eta <= 1/2)."""
        codes = {"auto": L.M2L_AUTO, "cuda_cores": L.M2L_CUDA_CORES, "tensor_cores": L.M2L_TENSOR_CORES}
        if engine not in codes:
            raise ValueError(f"engine must be one of {sorted(codes)}")
        self._check(self._lib.fmmb200_set_m2l_engine(self._h, codes[engine]))

    def set_tree_reuse(self, enable: bool):
        """Keep the previous tree when new positions would split every node the same
        way (checked exactly on the device); see fmmb200_set_tree_reuse."""
        self._check(self._lib.fmmb200_set_tree_reuse(self._h, int(bool(enable))))

    def set_shard(self, rank: int, world: int):
        """Later forwards compute only the fields of the particles in this shard's
        leaves (rank of world) and write 0 for every other particle; the sum over the
        shards is the unsharded result bit for bit.  See fmmb200_set_shard."""
        self._check(self._lib.fmmb200_set_shard(self._h, int(rank), int(world)))

    def debug_fail_alloc(self, k: int):
        self._check(self._lib.fmmb200_debug_fail_alloc(self._h, int(k)))

    def stats(self) -> dict:
        s = L.Stats()
        self._check(self._lib.fmmb200_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    # ---------------------------------------------------------------- field evaluation
    def update_particles_field(self, particles: Particles, alg: FMMB200, lambda_: float = 1.0):
        """update_particles_field!(particles, alg; lambda): overwrites efields/bfields."""
        pos = _f64(particles.positions, (-1, 3))
        mom = _f64(particles.momenta, (-1, 3))
        E = np.empty_like(pos)
        B = np.empty_like(pos)
        self._check(self._lib.fmmb200_update_particles_field(
            self._h, particles.npar, particles.charge, _pd(pos), _pd(mom), _pd(E), _pd(B), int(alg.n),
            int(alg.N0), float(alg.eta), float(lambda_), alg.precision_code))
        particles.efields[...] = E
        particles.bfields[...] = B

    def forward(self, pos, mom, alg: FMMB200, *, charge=-1.0, lambda_=1.0, p_avg=None, save_for_backward=False):
        pos = _f64(pos, (-1, 3))
        mom = _f64(mom, (-1, 3))
        E = np.empty_like(pos)
        B = np.empty_like(pos)
        pa = None if p_avg is None else _f64(p_avg, (3,))
        self._check(self._lib.fmmb200_forward(
            self._h, pos.shape[0], _pd(pos), _pd(mom), float(charge), float(lambda_), int(alg.n), int(alg.N0),
            float(alg.eta), alg.precision_code, _pd(pa), int(bool(save_for_backward)), _pd(E), _pd(B)))
        return E, B

    def forward_device(self, npar: int, d_pos: int, d_mom: int, d_e: int, d_b: int, alg: FMMB200, *, charge=-1.0,
                       lambda_=1.0, p_avg=None, save_for_backward=False):
        """Device-pointer forward (asynchronous on the context stream)."""
        pa = None if p_avg is None else _f64(p_avg, (3,))
        self._check(self._lib.fmmb200_forward_device(
            self._h, int(npar), ctypes.c_void_p(d_pos), ctypes.c_void_p(d_mom), float(charge), float(lambda_),
            int(alg.n), int(alg.N0), float(alg.eta), alg.precision_code, _pd(pa), int(bool(save_for_backward)),
            ctypes.c_void_p(d_e), ctypes.c_void_p(d_b)))

    def backward(self, grad_e, grad_b):
        ge = _f64(grad_e, (-1, 3))
        gb = _f64(grad_b, (-1, 3))
        gx = np.empty_like(ge)
        gu = np.empty_like(ge)
        self._check(self._lib.fmmb200_backward(self._h, _pd(ge), _pd(gb), _pd(gx), _pd(gu)))
        return gx, gu

    def backward_device(self, d_grad_e: int, d_grad_b: int, d_grad_pos: int, d_grad_mom: int):
        """Device-pointer adjoint of the saved forward (asynchronous on the context stream)."""
        self._check(self._lib.fmmb200_backward_device(self._h, ctypes.c_void_p(d_grad_e), ctypes.c_void_p(d_grad_b),
                                                      ctypes.c_void_p(d_grad_pos), ctypes.c_void_p(d_grad_mom)))

    # ---------------------------------------------------------------- introspection
    def tree_info(self) -> dict:
        info = np.zeros(8, np.int64)
        self._check(self._lib.fmmb200_get_tree_info(self._h, _pi(info)))
        return dict(npar=int(info[0]), N0=int(info[1]), max_level=int(info[2]), nc=int(info[3]),
                    nm2l=int(info[4]), np2p=int(info[5]), n=int(info[6]))

    def tree(self) -> dict:
        i = self.tree_info()
        N, nc = i["npar"], i["nc"]
        t = dict(parindices=np.zeros(N, np.int64), levels=np.zeros(nc, np.int64),
                 parlohis=np.zeros((nc, 2), np.int64), parents=np.zeros(nc, np.int64),
                 children=np.zeros((nc, 2), np.int64), bboxes=np.zeros((nc, 6)))
        self._check(self._lib.fmmb200_get_tree(self._h, _pi(t["parindices"]), _pi(t["levels"]),
                                               _pi(t["parlohis"]), _pi(t["parents"]), _pi(t["children"]),
                                               _pd(t["bboxes"])))
        t.update(max_level=i["max_level"], nc=nc)
        return t

    def lists(self):
        """(m2l, p2p) pairs as (n, 2) int64 arrays sorted by (target, source)."""
        i = self.tree_info()
        m2l = np.zeros((max(i["nm2l"], 1), 2), np.int64)
        p2p = np.zeros((max(i["np2p"], 1), 2), np.int64)
        self._check(self._lib.fmmb200_get_lists(self._h, _pi(m2l), _pi(p2p)))
        return m2l[: i["nm2l"]].copy(), p2p[: i["np2p"]].copy()

    def expansions(self):
        i = self.tree_info()
        NN = (i["n"] + 1) ** 3
        nc = i["nc"]
        g = np.zeros(NN * nc)
        m = np.zeros(3 * NN * nc)
        e = np.zeros(3 * NN * nc)
        b = np.zeros(3 * NN * nc)
        self._check(self._lib.fmmb200_get_expansions(self._h, _pd(g), _pd(m), _pd(e), _pd(b)))
        return g, m, e, b

    # ---------------------------------------------------------------- stage entry points
    def cluster_tree(self, pos, N0: int, stretch) -> dict:
        """ClusterTree(particles; N0, stretch) built on the device."""
        pos = _f64(pos, (-1, 3))
        N = pos.shape[0]
        s = _f64(stretch, (3,))
        self._check(self._lib.fmmb200_cluster_tree(self._h, N, _pd(pos), int(N0), _pd(s), None, None, None, None,
                                                   None, None))
        return self.tree()

    def interaction_lists(self, stretch, eta: float):
        """InteractionListsGPU(clusters; stretch, eta) on the last cluster_tree; returns (m2l, p2p)."""
        s = _f64(stretch, (3,))
        counts = np.zeros(2, np.int64)
        self._check(self._lib.fmmb200_interaction_lists(self._h, _pd(s), float(eta), _pi(counts)))
        return self.lists()

    def p2m(self, n, pos, mom, parindices, parlohis, bboxes, leaf_ids, gammas, mp_momenta, precision="fp64"):
        pos, mom = _f64(pos, (-1, 3)), _f64(mom, (-1, 3))
        parindices, parlohis, leaf_ids = _i64(parindices), _i64(parlohis, (-1, 2)), _i64(leaf_ids)
        bboxes = _f64(bboxes, (-1, 6))
        self._check(self._lib.fmmb200_p2m(self._h, n, _prec(precision), pos.shape[0], _pd(pos), _pd(mom),
                                          _pi(parindices), bboxes.shape[0], _pi(parlohis), _pd(bboxes),
                                          leaf_ids.shape[0], _pi(leaf_ids), _pd(gammas), _pd(mp_momenta)))

    def m2m(self, n, children, bboxes, level, gammas, mp_momenta, precision="fp64"):
        children, bboxes = _i64(children, (-1, 2)), _f64(bboxes, (-1, 6))
        self._check(self._lib.fmmb200_m2m(self._h, n, _prec(precision), bboxes.shape[0], _pi(children),
                                          _pd(bboxes), int(level), _pd(gammas), _pd(mp_momenta)))

    def m2l(self, n, bboxes, gammas, mp_momenta, pairs, p_avg, mp_efields, mp_bfields, precision="fp64"):
        bboxes, pairs = _f64(bboxes, (-1, 6)), _i64(pairs, (-1, 2))
        pa = _f64(p_avg, (3,))
        self._check(self._lib.fmmb200_m2l(self._h, n, _prec(precision), bboxes.shape[0], _pd(bboxes),
                                          _pd(_f64(gammas)), _pd(_f64(mp_momenta)), pairs.shape[0], _pi(pairs),
                                          _pd(pa), _pd(mp_efields), _pd(mp_bfields)))

    def p2p(self, pos, mom, parindices, parlohis, bboxes, pairs, efields, bfields, precision="fp64"):
        pos, mom = _f64(pos, (-1, 3)), _f64(mom, (-1, 3))
        parindices, parlohis, pairs = _i64(parindices), _i64(parlohis, (-1, 2)), _i64(pairs, (-1, 2))
        bboxes = _f64(bboxes, (-1, 6))
        self._check(self._lib.fmmb200_p2p(self._h, _prec(precision), pos.shape[0], _pd(pos), _pd(mom),
                                          _pi(parindices), bboxes.shape[0], _pi(parlohis), _pd(bboxes),
                                          pairs.shape[0], _pi(pairs), _pd(efields), _pd(bfields)))

    def l2l(self, n, parents, bboxes, level, mp_efields, mp_bfields, precision="fp64"):
        parents, bboxes = _i64(parents), _f64(bboxes, (-1, 6))
        self._check(self._lib.fmmb200_l2l(self._h, n, _prec(precision), bboxes.shape[0], _pi(parents),
                                          _pd(bboxes), int(level), _pd(mp_efields), _pd(mp_bfields)))

    def l2p(self, n, pos, parindices, parlohis, bboxes, leaf_ids, mp_efields, mp_bfields, efields, bfields,
            precision="fp64"):
        pos = _f64(pos, (-1, 3))
        parindices, parlohis, leaf_ids = _i64(parindices), _i64(parlohis, (-1, 2)), _i64(leaf_ids)
        bboxes = _f64(bboxes, (-1, 6))
        self._check(self._lib.fmmb200_l2p(self._h, n, _prec(precision), pos.shape[0], _pd(pos), _pi(parindices),
                                          bboxes.shape[0], _pi(parlohis), _pd(bboxes), leaf_ids.shape[0],
                                          _pi(leaf_ids), _pd(_f64(mp_efields)), _pd(_f64(mp_bfields)),
                                          _pd(efields), _pd(bfields)))


def _prec(p) -> int:
    if p in ("fp64", L.PRECISION_FP64):
        return L.PRECISION_FP64
    if p in ("mixed", L.PRECISION_MIXED):
        return L.PRECISION_MIXED
    raise ValueError("precision must be 'fp64' or 'mixed'")


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def update_particles_field(particles: Particles, alg: FMMB200, *, lambda_: float = 1.0, ctx: Context | None = None):
    """update_particles_field!(particles, FMMB200(eta, N0, n); lambda) -> None (fields overwritten)."""
    (ctx or default_context()).update_particles_field(particles, alg, lambda_)


update_particles_field_ = update_particles_field  # the reference spells it with a bang


def fmm_fields(pos, mom, alg: FMMB200, *, charge=-1.0, lambda_=1.0, ctx: Context | None = None):
    """Non-mutating (E, B) = F(positions, momenta); the forward of the adjoint pair."""
    return (ctx or default_context()).forward(pos, mom, alg, charge=charge, lambda_=lambda_)
