"""fmmb200_direct_noalloc: the direct sum without any allocation by the library.

Some callers cannot let a library allocate device memory -- their memory belongs
to their own pool allocator, or a cudaMalloc/cudaFree (which synchronises the
device) is not acceptable in their loop.  This entry point takes the caller's
device inputs and outputs and keeps its scratch in a fixed-size array compiled
into the library.  The tests call it through the C ABI:

* twice in a row, each result against the context-based fmmb200_direct_device on
  the same inputs (the same summation up to the source-slice count: 1e-13 relative);
* against the CPU oracle's FP64 BruteForce, with and without a target list and on a
  stream other than the default one, so that a defect shared by both GPU entry
  points cannot pass.

Collected last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_context_direct_sum_twice():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fmmb200
    from fmmb200 import beams

    lib = fmmb200.load()
    torch.cuda.set_device(0)
    ctx = fmmb200.Context(0)
    vp = ctypes.c_void_p
    for call, (N, nt, seed) in enumerate(((20000, 1000, 3), (50000, 4096, 4))):
        pos_h, mom_h = beams.gaussian_bunch(N, seed=seed)
        pos = torch.from_numpy(pos_h).cuda()
        mom = torch.from_numpy(mom_h).cuda()
        tg = torch.from_numpy(np.random.default_rng(seed).choice(N, nt, replace=False).astype(np.int64)).cuda()
        e_ref = torch.empty((nt, 3), dtype=torch.float64, device="cuda")
        b_ref = torch.empty_like(e_ref)
        e = torch.full_like(e_ref, float("nan"))
        b = torch.full_like(e_ref, float("nan"))
        st = lib.fmmb200_direct_device(ctx.handle, N, vp(pos.data_ptr()), vp(mom.data_ptr()), -1.0, 1.0, nt,
                                       vp(tg.data_ptr()), vp(e_ref.data_ptr()), vp(b_ref.data_ptr()))
        assert st == fmmb200.OK
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream().cuda_stream
        st = lib.fmmb200_direct_noalloc(N, vp(pos.data_ptr()), vp(mom.data_ptr()), -1.0, 1.0, nt,
                                        vp(tg.data_ptr()), vp(e.data_ptr()), vp(b.data_ptr()), vp(stream))
        assert st == fmmb200.OK, call
        torch.cuda.synchronize()
        assert _rel(e.cpu().numpy(), e_ref.cpu().numpy()) < TOL, call
        assert _rel(b.cpu().numpy(), b_ref.cpu().numpy()) < TOL, call
    ctx.close()


def test_noalloc_rejects_more_targets_than_its_scratch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fmmb200

    lib = fmmb200.load()
    x = torch.zeros((70000, 3), dtype=torch.float64, device="cuda")
    vp = ctypes.c_void_p
    st = lib.fmmb200_direct_noalloc(70000, vp(x.data_ptr()), vp(x.data_ptr()), -1.0, 1.0, 70000, None,
                                    vp(x.data_ptr()), vp(x.data_ptr()), None)
    assert st == fmmb200.ERR_CAPACITY


def test_noalloc_matches_oracle_bruteforce_on_a_side_stream():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fmmb200
    import oracle
    from fmmb200 import beams

    lib = fmmb200.load()
    vp = ctypes.c_void_p
    N = 2000
    pos_h, mom_h = beams.gaussian_bunch(N, seed=7)
    Eo, Bo = oracle.bruteforce(pos_h, mom_h, -1.0, 1.0)
    pos = torch.from_numpy(pos_h).cuda()
    mom = torch.from_numpy(mom_h).cuda()
    side = torch.cuda.Stream()
    for targets in (None, np.random.default_rng(8).choice(N, 700, replace=False).astype(np.int64)):
        nt = N if targets is None else targets.size
        tg = None if targets is None else torch.from_numpy(targets).cuda()
        e = torch.full((nt, 3), float("nan"), dtype=torch.float64, device="cuda")
        b = torch.full_like(e, float("nan"))
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            st = lib.fmmb200_direct_noalloc(N, vp(pos.data_ptr()), vp(mom.data_ptr()), -1.0, 1.0, nt,
                                            None if tg is None else vp(tg.data_ptr()), vp(e.data_ptr()),
                                            vp(b.data_ptr()), vp(side.cuda_stream))
        assert st == fmmb200.OK
        side.synchronize()
        sel = slice(None) if targets is None else targets
        assert _rel(e.cpu().numpy(), Eo[sel]) < TOL
        assert _rel(b.cpu().numpy(), Bo[sel]) < TOL
