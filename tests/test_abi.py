"""The C-ABI library: builds for sm_100a, loads, and exports exactly what
include/fmmb200.h declares.  No compute calls (these run without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fmmb200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmmb200_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared_functions()
    for required in ("fmmb200_create", "fmmb200_destroy", "fmmb200_update_particles_field", "fmmb200_forward",
                     "fmmb200_backward", "fmmb200_cluster_tree", "fmmb200_interaction_lists", "fmmb200_m2l",
                     "fmmb200_p2p"):
        assert required in names


def test_library_loads_and_exports_every_declared_symbol():
    import fmmb200

    lib = fmmb200.load()
    assert os.path.exists(fmmb200.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert sorted(fmmb200.SIGNATURES) == declared_functions()
    assert lib.fmmb200_version() == 1


def test_library_targets_sm100a_only():
    import fmmb200

    fmmb200.load()
    import subprocess

    out = subprocess.run(["cuobjdump", "--list-elf", fmmb200.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    archs = set(re.findall(r"sm_(\d+a?)", out.stdout))
    assert archs == {"100a"}, archs


def test_null_and_bad_arguments_return_status_without_gpu():
    import fmmb200

    lib = fmmb200.load()
    assert lib.fmmb200_create(None, 0) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_destroy(None) == fmmb200.OK
    assert lib.fmmb200_last_error(None) == b"null context"
    assert lib.fmmb200_set_timing(None, 1) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_set_m2l_engine(None, 0) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_set_tree_reuse(None, 1) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_set_shard(None, 0, 1) == fmmb200.ERR_INVALID_ARGUMENT


def test_create_without_a_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import fmmb200

    lib = fmmb200.load()
    h = ctypes.c_void_p()
    assert lib.fmmb200_create(ctypes.byref(h), 0) == fmmb200.ERR_CUDA
    with pytest.raises(fmmb200.FMMB200Error):
        fmmb200.Context(0)


def test_particles_mirror_reference_constructor():
    # test/test_particles.jl:1-29
    import fmmb200

    rng = np.random.default_rng(0)
    pos = rng.random((3, 10))
    mom = rng.random((3, 10))
    p = fmmb200.Particles(pos=pos, mom=mom)
    assert p.npar == 10
    np.testing.assert_array_equal(p.positions, pos.T)
    np.testing.assert_array_equal(p.momenta, mom.T)
    assert np.all(p.efields == 0) and np.all(p.bfields == 0)
    assert p.charge == -1.0 and p.mass == 1.0
    b = fmmb200.Beam(pos=np.zeros((3, 10)), mom=np.zeros((3, 10)))
    assert isinstance(b, fmmb200.Particles)
    with pytest.raises(ValueError):
        fmmb200.Particles(pos=np.zeros((3, 4)), mom=np.zeros((3, 5)))


def test_algorithm_struct():
    import fmmb200

    a = fmmb200.FMMB200.positional(0.5, 125, 4)
    assert (a.n, a.N0, a.eta, a.precision) == (4, 125, 0.5, "fp64")
    assert fmmb200.FMMB200(n=4, N0=125, eta=0.5, precision="mixed").precision_code == fmmb200.PRECISION_MIXED
    with pytest.raises(ValueError):
        fmmb200.FMMB200(n=4, N0=125, eta=0.5, precision="fp16").precision_code


JULIA = os.path.join(ROOT, "fmm4rbgpu.jl_b200", "julia", "FMMB200.jl")


def _header_arities():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(fmmb200_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def _julia_ccalls(src):
    """(symbol, number of argument types) of every ccall((:sym, libfmmb200), Ret, (types...), ...)."""
    calls = []
    for m in re.finditer(r"ccall\(\(:(fmmb200_[a-z0-9_]+),\s*libfmmb200\),\s*[A-Za-z0-9_{}]+,\s*\(", src):
        i, depth, parts, cur = m.end(), 1, [], ""
        while depth:
            c = src[i]
            if c in "({":
                depth += 1
            elif c in ")}":
                depth -= 1
            if depth == 1 and c == ",":
                parts.append(cur)
                cur = ""
            elif depth:
                cur += c
            i += 1
        parts.append(cur)
        calls.append((m.group(1), len([p for p in parts if p.strip()])))
    return calls


def test_julia_binding_module_and_exports():
    """The binding's module does not shadow the constructor it exports: `module FMMB200` would
    bind FMMB200 to the module itself, so `FMMB200(0.5, 125, 4)` must come from a module of
    another name that exports a function of that name."""
    src = open(JULIA).read()
    mod = re.search(r"^module\s+(\w+)", src, flags=re.M).group(1)
    assert mod != "FMMB200"
    assert not re.search(r"^\s*const\s+FMMB200\b", src, flags=re.M)
    exported = set()
    for line in re.findall(r"^export\s+(.+)$", src, flags=re.M):
        exported |= {w.strip() for w in line.split(",")}
    assert {"FMMB200", "FMMB200Alg", "fmm_fields"} <= exported
    # positional (eta, N0, n) and keyword forms, both returning the struct
    assert re.search(r"^FMMB200\(eta::Real,\s*N0::Integer,\s*n::Integer.*\)\s*=\s*\n?\s*FMMB200Alg\(", src, flags=re.M)
    assert re.search(r"^FMMB200\(;\s*n::Integer,\s*N0::Integer,\s*eta::Real", src, flags=re.M)
    assert re.search(r"function update_particles_field!\(p::Particles\{Float64\},\s*alg::FMMB200Alg;\s*lambda\)", src)


def test_julia_ccalls_match_the_header():
    src = open(JULIA).read()
    arity = _header_arities()
    calls = _julia_ccalls(src)
    names = {c[0] for c in calls}
    assert {"fmmb200_create", "fmmb200_destroy", "fmmb200_last_error", "fmmb200_update_particles_field",
            "fmmb200_forward", "fmmb200_backward"} <= names
    for name, nargs in calls:
        assert name in arity, name
        assert nargs == arity[name], (name, nargs, arity[name])


def test_julia_rrule_reuses_pooled_contexts():
    src = open(JULIA).read()
    body = src[src.index("function ChainRulesCore.rrule"):]
    body = body[: body.index("\nend\n")]
    assert "Context(" not in body  # no new device context per differentiated call
    assert "_acquire()" in body and "_release(ctx)" in body
    # the error message is read before the context goes back to the pool
    assert body.index("_error(ctx, st)") < body.index("_release(ctx)\n        err")


def test_direct_entry_points_reject_more_targets_than_particles_without_a_list():
    """With no target list the targets are particles 0..ntarget-1, so ntarget > npar would
    read past the caller's buffers: both device-pointer entry points refuse it before any
    CUDA call (the pointers are never dereferenced)."""
    import fmmb200

    lib = fmmb200.load()
    buf = np.zeros(64)
    p = ctypes.c_void_p(buf.ctypes.data)
    assert lib.fmmb200_direct_noalloc(10, p, p, -1.0, 1.0, 11, None, p, p, None) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_direct_noalloc(10, p, p, -1.0, 0.0, 5, None, p, p, None) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_direct_device(None, 10, p, p, -1.0, 1.0, 11, None, p, p) == fmmb200.ERR_INVALID_ARGUMENT


def test_shard_record_sizes_without_gpu():
    """The exchange buffers of the sharded forward are sized from fmmb200_shard_record_bytes:
    4 (n+1)^3 moment values of the precision's type, and 64 (FP64) or 80 (mixed) bytes per
    particle record.  Bad degrees or precisions are refused."""
    import fmmb200

    lib = fmmb200.load()
    m = ctypes.c_int64()
    p = ctypes.c_int64()
    assert lib.fmmb200_shard_record_bytes(4, fmmb200.PRECISION_FP64, ctypes.byref(m), ctypes.byref(p)) == fmmb200.OK
    assert (m.value, p.value) == (4 * 125 * 8, 64)
    assert lib.fmmb200_shard_record_bytes(5, fmmb200.PRECISION_MIXED, ctypes.byref(m), ctypes.byref(p)) == fmmb200.OK
    assert (m.value, p.value) == (4 * 216 * 4, 80)
    assert lib.fmmb200_shard_record_bytes(0, 0, None, None) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_shard_record_bytes(4, 7, None, None) == fmmb200.ERR_INVALID_ARGUMENT
    assert lib.fmmb200_shard_subtree(None, 10, None, None, 5, 1, None, 4, 0) == fmmb200.ERR_INVALID_ARGUMENT


def test_set_stream_passes_the_legacy_default_stream_explicitly():
    """torch's default stream has the handle 0, and fmmb200_set_stream reads a NULL handle as
    the context's own (non-blocking) stream, which is not ordered after torch's work: the
    Python wrapper passes 0 as cudaStreamLegacy (0x1), other handles as given, and None as
    NULL (the own stream)."""
    import fmmb200
    from fmmb200 import api

    got = []

    class FakeLib:
        def fmmb200_set_stream(self, h, stream):
            got.append(stream.value)
            return fmmb200.OK

    ctx = api.Context.__new__(api.Context)
    ctx._lib, ctx._h = FakeLib(), ctypes.c_void_p(1234)
    for handle in (0, None, 0x7F00DEAD):
        ctx.set_stream(handle)
    ctx._h = None  # nothing to destroy
    assert got == [api.CUDA_STREAM_LEGACY, None, 0x7F00DEAD]
    assert api.CUDA_STREAM_LEGACY == 1
