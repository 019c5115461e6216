"""fmmb200 -- B200 (sm_100a) interpolation-based FMM for relativistic space-charge
E/B fields, a drop-in for FMM4RBGPU.jl's FMMGPU field evaluation.

All compute runs in libfmmb200.so (hand-written CUDA for sm_100a); this package
is the host-side mirror of the reference interface (Particles/Beam,
update_particles_field!, the algorithm struct, and the kernel-level stages).
"""
from ._lib import (ERR_CAPACITY, ERR_CUDA, ERR_DEVICE, ERR_INVALID_ARGUMENT, ERR_NO_STATE, ERR_OUT_OF_MEMORY,
                   ERR_TREE_SHAPE, OK, PRECISION_FP64, PRECISION_MIXED, SIGNATURES, FMMB200Error, load)
from ._build import LIB_PATH, build
from .api import (R_E, Beam, Context, FMMB200, Particles, default_context, fmm_fields,
                  update_particles_field, update_particles_field_)

__all__ = [
    "Beam", "Context", "FMMB200", "FMMB200Error", "Particles", "R_E", "build", "default_context", "fmm_fields",
    "load", "update_particles_field", "update_particles_field_", "LIB_PATH", "SIGNATURES", "OK",
    "ERR_INVALID_ARGUMENT", "ERR_OUT_OF_MEMORY", "ERR_CUDA", "ERR_TREE_SHAPE", "ERR_NO_STATE", "ERR_DEVICE",
    "ERR_CAPACITY", "PRECISION_FP64", "PRECISION_MIXED",
]
