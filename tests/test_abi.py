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
