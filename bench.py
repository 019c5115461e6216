#!/usr/bin/env python
"""Benchmark of the B200 space-charge FMM (FMMB200) on the N = 2^24 Gaussian bunch.

A step is one field evaluation -- update_particles_field!(beam, FMMB200(0.5, 125, 4);
lambda=1) from positions/momenta to E and B -- over the whole synthetic beam:
tree build, traversal, P2M/M2M, M2L, P2P, L2L/L2P.

  value    mixed (FP32 arithmetic, FP64 geometry) form, particles/s with the
           inputs resident in HBM (device-pointer C-ABI call)
  fp64     the plain FP64 path on the same inputs
  e2e      the mixed form through the host-pointer C-ABI (the call the drop-in
           makes): pinned host inputs copied in and fields copied out every step
  fwd_bwd  one forward (saving its state) plus the hand-written adjoint of
           L = sum(w.E + v.B) back to positions and momenta, device-resident
  reuse    a drifting beam (x += 1e-12 u between calls, outside the timed region)
           evaluated with fmmb200_set_tree_reuse: the forward keeps the tree when
           a rebuild would give the same one (checked exactly on the device)
  roofline the dominant kernel (M2L) against the measured CUDA-core FMA peak
  accuracy rel-L2 of mixed vs FP64 over all particles, and of both vs an FP64
           direct sum (GPU) on 4096 seeded targets
  nsweep   the same beam at other (n, eta): mixed and FP64 ms/step and both forms'
           rel-L2 against the FP64 direct sum, and the cheapest setting whose
           error is <= 1e-5 (the accuracy target of the mixed form)
  large    the N = 25,600,000 bunch of the reference's published comparison
           (mixed, FP64, and mixed through the host-pointer call)

--impl reference times the reference's algorithm on the host cores: the
oracle's restatement of the serial FMM (parallel over targets with OpenMP,
bit-identical to serial) on a bounded sample of the same workload.

Multi-GPU (--gpus N under torchrun): the field evaluation is replicated, one
independent beam per rank (weak scaling); the timing is the max over ranks.
With --shard, one beam of --N particles is split over the ranks instead (strong
scaling): each step all-gathers positions and momenta, every rank builds the tree
and lists of the whole beam and evaluates its share of the leaves, and a
reduce-scatter returns each rank the fields of its own particles.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fmm4rbgpu.jl_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from fmmb200 import replicas  # noqa: E402

METRIC = "particles/s at N=2^24: FP32 form vs FP64 plain at stated rel err; fwd+bwd time"
SM_COUNT_NOTE = "B200, 148 SMs"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--N", type=int, default=2**24)
    ap.add_argument("--n", type=int, default=4)
    ap.add_argument("--N0", type=int, default=125)
    ap.add_argument("--eta", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--dist", choices=["gauss", "beamlets", "uniform"], default="gauss",
                    help="gauss: the Gaussian bunch; beamlets: 8 Gaussian beamlets with centres U[-5,5]^3 "
                         "(sigma=(0.3,0.3,0.03), u_z~N(100,0.1)); uniform: U[0,1]^3 at rest")
    ap.add_argument("--ntargets", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=2**17, help="particles in the CPU-baseline sample")
    ap.add_argument("--ref-sample", type=int, default=2**20, help="particles per reference-arm step")
    ap.add_argument("--ref-large-sample", type=int, default=2**22,
                    help="one more reference-arm evaluation at this size, outside the timed steps, so that "
                         "the growth of the CPU cost per particle with N is visible (0: skip)")
    ap.add_argument("--skip-nsweep", action="store_true")
    ap.add_argument("--skip-configs", action="store_true", help="skip the other benchmark configurations")
    ap.add_argument("--nsweep", default="2:0.5,3:0.5,4:0.5,5:0.5,6:0.5,4:0.4,4:0.3,4:0.25,4:0.2",
                    help="n:eta settings of the accuracy/throughput sweep (the FMM's error against the direct sum "
                         "has a floor set by eta, from the mean momentum in its far-field kernel, so the sweep "
                         "lowers eta rather than only raising n)")
    ap.add_argument("--large-N", type=int, default=25_600_000, help="particles of the large line (0: skip)")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-backward", action="store_true")
    ap.add_argument("--skip-reuse", action="store_true")
    ap.add_argument("--m2l-engine", choices=["auto", "cuda_cores", "tensor_cores"], default="auto",
                    help="mixed-form M2L engine (fmmb200_set_m2l_engine)")
    ap.add_argument("--bwd-steps", type=int, default=3, help="timed fwd+bwd steps (after 2 warm-up steps)")
    ap.add_argument("--shard", action="store_true",
                    help="one beam of --N particles split over the ranks (strong scaling, fmmb200.sharded: the "
                         "tree split at level log2(ranks), each rank holding its subtree) instead of one "
                         "independent beam per rank")
    ap.add_argument("--shard-emulate", default="",
                    help="comma-separated rank counts: run the memory-sharded forward of --N particles with that "
                         "many ranks on this one GPU (the ranks in turn, the collectives as local copies) and "
                         "print per-rank compute time and device memory; not a multi-GPU measurement")
    return ap.parse_args()


DISTS = {
    "gauss": "Gaussian bunch (sigma=(1,1,0.1), u_z~N(200,0.2), u_x,u_y~N(0,0.01))",
    "beamlets": "8 Gaussian beamlets, centres U[-5,5]^3 (sigma=(0.3,0.3,0.03), u_z~N(100,0.1), u_x,u_y~N(0,0.005))",
    "uniform": "uniform U[0,1]^3 at rest",
}


def generate(args, N, seed):
    from fmmb200 import beams

    gen = {"gauss": beams.gaussian_bunch, "beamlets": beams.beamlets, "uniform": beams.uniform}[args.dist]
    return gen(N, seed=seed)


def workload(args):
    return {
        "workload": f"{DISTS[args.dist]} N={args.N}, "
                    f"n={args.n}, N0={args.N0}, eta={args.eta}, lambda=1; value = mixed form, fp64 = plain path",
        "npar": args.N, "n": args.n, "N0": args.N0, "eta": args.eta, "lambda": 1.0, "dist": args.dist,
        "l2": "inputs larger than L2 (AoS positions+momenta 48 B/particle resident in HBM; no flush)",
    }


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during a region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            if self.uuid and f[0] != self.uuid:
                continue
            try:
                rows.append(dict(sm=float(f[1]), smax=float(f[2]), power=float(f[3]), hw=f[5], hwt=f[6], swt=f[7],
                                 swp=f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        load = [r for r in rows if r["power"] > 300.0] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("swp", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(load), "power_w_max": max(r["power"] for r in rows)}


# ---------------------------------------------------------------------------- helpers
def model_flops(st: dict, n: int, N: int) -> float:
    """Algorithmic flop count: 41 per kernel evaluation plus the interpolation terms
    (the reference's dense M2M/L2L counts)."""
    M = n + 1
    NN = M ** 3
    nc = st["ncluster"]
    return (41.0 * (st["m2l_kernel_evals"] + st["p2p_kernel_evals"]) + N * (10 * NN + 12 * M + 6)
            + N * (14 * NN + 12 * M) + 10.0 * NN * NN * (nc - 1) + 14.0 * NN * NN * (nc - 1))


def dist_setup(args):
    import torch

    world, rank, local = replicas.env_ranks()
    if world > 1:
        replicas.init("nccl", local)
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    replicas.barrier(world)


def max_over_ranks(world, v: float) -> float:
    return replicas.max_over_ranks(world, v, device="cuda")


# ---------------------------------------------------------------------------- reference arm
def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    from fmmb200 import beams

    nthreads = os.cpu_count() or 1
    N = min(args.ref_sample, args.N)
    pos, mom = generate(args, N, args.seed)
    for _ in range(args.warmup):
        oracle.fmm(pos, mom, -1.0, 1.0, args.n, args.N0, args.eta, nthreads=nthreads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.fmm(pos, mom, -1.0, 1.0, args.n, args.N0, args.eta, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    v = N / t
    # the CPU cost per particle grows with the tree depth: one evaluation at a larger size
    by_sample = {str(N): v}
    NL = min(args.ref_large_sample, args.N)
    if NL > N:
        posl, moml = generate(args, NL, args.seed)
        t0 = time.perf_counter()
        oracle.fmm(posl, moml, -1.0, 1.0, args.n, args.N0, args.eta, nthreads=nthreads)
        by_sample[str(NL)] = NL / (time.perf_counter() - t0)
        del posl, moml
    sample = (f"one FMM field evaluation of a {N}-particle sample of the workload's distribution (same n, N0, eta) "
              f"per step; the oracle's restatement of the reference's serial FMM (src/fmm/*.jl), OpenMP over "
              f"targets; rate_by_sample adds one evaluation at {NL} particles")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian bunch)",
        "config": workload(args),
        "cpu_baseline": {"value": v, "unit": "particles/s", "cores": nthreads, "kind": "port", "sample": sample,
                         "rate_by_sample": by_sample},
        "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cpu_baseline(args):
    import oracle
    from fmmb200 import beams

    N = min(args.cpu_sample, args.N)
    pos, mom = generate(args, N, args.seed + 1)
    t0 = time.perf_counter()
    oracle.fmm(pos, mom, -1.0, 1.0, args.n, args.N0, args.eta, nthreads=1)
    t = time.perf_counter() - t0
    return {"value": N / t, "unit": "particles/s", "cores": 1, "kind": "port",
            "sample": f"one serial FMM field evaluation (the oracle's restatement of src/fmm/*.jl, 1 thread) of a "
                      f"{N}-particle Gaussian bunch with the same distribution, n, N0 and eta; {t:.1f} s"}


# ---------------------------------------------------------------------------- sweeps
def _events_ms(stream, fn, steps, warmup):
    import torch

    for _ in range(warmup):
        fn()
    stream.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        fn()
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1) / steps


def run_nsweep(args, ctx, stream, N, pos, mom, tg, Ed, Bd):
    """Both forms at each (n, eta) of --nsweep on the benchmark beam: ms/step (1 warm-up,
    then 2 timed steps, 1 above a second) and rel-L2 of E and B on the direct sum's targets."""
    import torch

    import fmmb200

    E = torch.empty_like(pos)
    B = torch.empty_like(pos)

    def rel(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    rows = []
    for item in args.nsweep.split(","):
        n_s, eta_s = item.split(":")
        n, eta = int(n_s), float(eta_s)
        row = {"n": n, "eta": eta}
        for prec in ("mixed", "fp64"):
            alg = fmmb200.FMMB200(n=n, N0=args.N0, eta=eta, precision=prec)
            try:
                step = lambda: ctx.forward_device(N, pos.data_ptr(), mom.data_ptr(), E.data_ptr(),  # noqa: E731
                                                  B.data_ptr(), alg)
                ms = _events_ms(stream, step, 1, 1)
                if ms < 1000.0:  # a second timed step where it is cheap
                    ms = _events_ms(stream, step, 2, 0)
            except fmmb200.FMMB200Error as e:  # e.g. out of device memory at the largest n
                row[prec] = {"error": str(e)}
                continue
            st = ctx.stats()
            row[prec] = {"ms_per_step": ms, "value": N / (ms * 1e-3), "err_E": rel(E[tg], Ed), "err_B": rel(B[tg], Bd),
                         "ms_m2l": st["ms_m2l"], "ms_p2p": st["ms_p2p"]}
            row.update(nm2l=st["nm2l"], np2p=st["np2p"], device_bytes=st["device_bytes"])
        if "ms_per_step" in row.get("mixed", {}) and "ms_per_step" in row.get("fp64", {}):
            row["mixed_speedup"] = row["fp64"]["ms_per_step"] / row["mixed"]["ms_per_step"]
        rows.append(row)
        print(json.dumps({"nsweep_row": row}), file=sys.stderr, flush=True)
    target = 1e-5
    ok = [r for r in rows if "err_E" in r.get("mixed", {})
          and max(r["mixed"]["err_E"], r["mixed"]["err_B"]) <= target]
    best = min(ok, key=lambda r: r["mixed"]["ms_per_step"]) if ok else None
    closest = min((r for r in rows if "err_E" in r.get("mixed", {})),
                  key=lambda r: max(r["mixed"]["err_E"], r["mixed"]["err_B"]), default=None)
    return {"N": N, "N0": args.N0, "targets": int(tg.numel()), "target_rel_err": target, "rows": rows,
            "cheapest_meeting_target": None if best is None else
            {"n": best["n"], "eta": best["eta"], "mixed_ms": best["mixed"]["ms_per_step"],
             "mixed_value": best["mixed"]["value"], "mixed_speedup": best.get("mixed_speedup"),
             "err_E": best["mixed"]["err_E"], "err_B": best["mixed"]["err_B"]},
            "most_accurate": None if closest is None else {"n": closest["n"], "eta": closest["eta"],
                                                          "err_E": closest["mixed"]["err_E"],
                                                          "err_B": closest["mixed"]["err_B"]}}


def run_large(args, ctx, stream, dev):
    """The N = --large-N bunch (the reference's published comparison size) at the
    benchmark's n, N0, eta: mixed and FP64 device-resident, mixed through the host call."""
    import torch

    import fmmb200

    N = args.large_N
    pos_h, mom_h = generate(args, N, args.seed + 11)
    pos = torch.from_numpy(pos_h).to(dev)
    mom = torch.from_numpy(mom_h).to(dev)
    E = torch.empty_like(pos)
    B = torch.empty_like(pos)
    out = {"N": N}
    for prec in ("mixed", "fp64"):
        alg = fmmb200.FMMB200(n=args.n, N0=args.N0, eta=args.eta, precision=prec)
        ms = _events_ms(stream, lambda: ctx.forward_device(N, pos.data_ptr(), mom.data_ptr(), E.data_ptr(),
                                                           B.data_ptr(), alg), 3, 1)
        out[prec] = {"ms_per_step": ms, "value": N / (ms * 1e-3)}
    st = ctx.stats()
    out.update(max_level=st["max_level"], nm2l=st["nm2l"], np2p=st["np2p"])
    del pos, mom, E, B
    ph = torch.from_numpy(pos_h).pin_memory()
    mh = torch.from_numpy(mom_h).pin_memory()
    eh = torch.empty((N, 3), dtype=torch.float64).pin_memory()
    bh = torch.empty((N, 3), dtype=torch.float64).pin_memory()
    dp = ctypes.POINTER(ctypes.c_double)
    args_c = [ctypes.cast(t.data_ptr(), dp) for t in (ph, mh, eh, bh)]
    L = ctx._lib

    def host_step():
        ctx._check(L.fmmb200_update_particles_field(ctx.handle, N, -1.0, *args_c, args.n, args.N0, args.eta, 1.0,
                                                    fmmb200.PRECISION_MIXED))

    ms = _events_ms(stream, host_step, 3, 1)
    out["e2e_mixed"] = {"ms_per_step": ms, "value": N / (ms * 1e-3), "h2d_bytes_per_step": 48 * N,
                        "d2h_bytes_per_step": 48 * N}
    return out


def run_configs(args, stream, dev):
    """The other configurations of the benchmark list: per configuration the mixed and FP64
    forwards (device-resident, each on a context of its own, with its device bytes), the
    mixed-vs-FP64 error, and for the two adjoint configurations the mixed forward + adjoint time
    and the mixed context's device bytes with the adjoint's buffers."""
    import torch

    import fmmb200
    from fmmb200 import beams

    def rel(a, b):
        nb = float(torch.linalg.norm(b))
        return float(torch.linalg.norm(a - b) / nb) if nb > 0 else float(torch.linalg.norm(a))

    cases = [("uniform_65536", beams.uniform, 65536, 4, 125, False),
             ("gauss_1048576", beams.gaussian_bunch, 2**20, 4, 125, False),
             ("adjoint_gauss_262144", beams.gaussian_bunch, 262144, 4, 125, True),
             ("beamlets_4194304_n5_N0_64", beams.beamlets, 2**22, 5, 64, True)]
    out = {}
    for name, gen, N, n, N0, adjoint in cases:
        pos_h, mom_h = gen(N, seed=args.seed)
        pos = torch.from_numpy(pos_h).to(dev)
        mom = torch.from_numpy(mom_h).to(dev)
        res = {"N": N, "n": n, "N0": N0, "eta": args.eta}
        fields, ctxs = {}, {}
        for prec in ("mixed", "fp64"):
            # a context per precision, so that its device bytes are this run's alone
            ctxs[prec] = c = fmmb200.Context(dev.index)
            c.set_stream(stream.cuda_stream)
            alg = fmmb200.FMMB200(n=n, N0=N0, eta=args.eta, precision=prec)
            e, b = torch.empty_like(pos), torch.empty_like(pos)
            ms = _events_ms(stream, lambda: c.forward_device(N, pos.data_ptr(), mom.data_ptr(), e.data_ptr(),
                                                             b.data_ptr(), alg), 3, 2)
            res[prec] = {"ms_per_step": ms, "value": N / (ms * 1e-3), "device_bytes": int(c.stats()["device_bytes"])}
            fields[prec] = (e, b)
        ctx = ctxs["mixed"]
        res["mixed_vs_fp64"] = {"E": rel(fields["mixed"][0], fields["fp64"][0]),
                                "B": rel(fields["mixed"][1], fields["fp64"][1])}
        if adjoint:
            alg = fmmb200.FMMB200(n=n, N0=N0, eta=args.eta, precision="mixed")
            e, b = fields["mixed"]
            gen_t = torch.Generator(device=dev).manual_seed(args.seed + 1)
            gE = torch.randn((N, 3), dtype=torch.float64, device=dev, generator=gen_t)
            gB = torch.randn((N, 3), dtype=torch.float64, device=dev, generator=gen_t)
            gx, gu = torch.empty_like(gE), torch.empty_like(gE)

            def fb():
                ctx.forward_device(N, pos.data_ptr(), mom.data_ptr(), e.data_ptr(), b.data_ptr(), alg,
                                   save_for_backward=True)
                ctx.backward_device(gE.data_ptr(), gB.data_ptr(), gx.data_ptr(), gu.data_ptr())

            ms = _events_ms(stream, fb, 2, 2)
            res["fwd_bwd_mixed"] = {"ms_per_step": ms, "ratio_to_forward": ms / res["mixed"]["ms_per_step"],
                                    "grad_finite": bool(torch.isfinite(gx).all() and torch.isfinite(gu).all())}
            res["device_bytes_with_backward"] = int(ctx.stats()["device_bytes"])
        out[name] = res
        for c in ctxs.values():
            c.close()
        del pos, mom, fields
    return out


# ---------------------------------------------------------------------------- our arm
def run_ours(args, world, rank, local):
    import torch

    import fmmb200
    from fmmb200 import beams

    dev = torch.device("cuda", local)
    N = args.N
    pos_h, mom_h = generate(args, N, args.seed + rank)
    pos = torch.from_numpy(pos_h).to(dev)
    mom = torch.from_numpy(mom_h).to(dev)
    E = torch.empty_like(pos)
    B = torch.empty_like(pos)
    E64 = torch.empty_like(pos)
    B64 = torch.empty_like(pos)
    stream = torch.cuda.Stream(device=dev)
    ctx = fmmb200.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_timing(True)
    ctx.set_m2l_engine(args.m2l_engine)
    L = ctx._lib
    alg_mixed = fmmb200.FMMB200(n=args.n, N0=args.N0, eta=args.eta, precision="mixed")
    alg_fp64 = fmmb200.FMMB200(n=args.n, N0=args.N0, eta=args.eta, precision="fp64")

    def step(alg, e, b):
        ctx.forward_device(N, pos.data_ptr(), mom.data_ptr(), e.data_ptr(), b.data_ptr(), alg)

    def timed(alg, e, b, steps, warmup):
        for _ in range(warmup):
            step(alg, e, b)
        stream.synchronize()
        barrier(world)
        torch.cuda.synchronize(dev)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        stage = []
        ev0.record(stream)
        for _ in range(steps):
            step(alg, e, b)
            stage.append(ctx.stats())
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize(dev)
        barrier(world)
        ms = ev0.elapsed_time(ev1) / steps
        return max_over_ranks(world, ms), stage

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    with ClockSampler(uuid) as clk:
        ms_mixed, st_mixed = timed(alg_mixed, E, B, args.steps, args.warmup)
        ms_fp64, st_fp64 = timed(alg_fp64, E64, B64, args.steps, args.warmup)
    clocks = clk.summary()

    st = st_mixed[-1]
    st64 = st_fp64[-1]
    # accuracy: mixed vs fp64 (all particles), both vs an FP64 direct sum on seeded targets
    rel_e = float(torch.linalg.norm(E - E64) / torch.linalg.norm(E64))
    rel_b = float(torch.linalg.norm(B - B64) / torch.linalg.norm(B64))
    tg = torch.from_numpy(np.random.default_rng(args.seed + 100).choice(N, size=min(args.ntargets, N),
                                                                          replace=False).astype(np.int64)).to(dev)
    Ed = torch.empty((tg.numel(), 3), dtype=torch.float64, device=dev)
    Bd = torch.empty_like(Ed)
    st_ = L.fmmb200_direct_device(ctx.handle, N, ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(mom.data_ptr()),
                                  -1.0, 1.0, tg.numel(), ctypes.c_void_p(tg.data_ptr()),
                                  ctypes.c_void_p(Ed.data_ptr()), ctypes.c_void_p(Bd.data_ptr()))
    ctx._check(st_)
    stream.synchronize()

    def rel(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    E_main = E.clone()  # the timed region's fields, for the host-pointer check below
    acc = {"mixed_vs_fp64": {"E": rel_e, "B": rel_b},
           "fp64_vs_direct": {"E": rel(E64[tg], Ed), "B": rel(B64[tg], Bd)},
           "mixed_vs_direct": {"E": rel(E[tg], Ed), "B": rel(B[tg], Bd)},
           "direct_targets": int(tg.numel())}

    # forward + adjoint (the gradient path of the fields), device-resident
    fwd_bwd = None
    bwd_bytes = None
    if not args.skip_backward:
        gen = torch.Generator(device=dev).manual_seed(args.seed + 7)
        gE = torch.randn((N, 3), dtype=torch.float64, device=dev, generator=gen)
        gB = torch.randn((N, 3), dtype=torch.float64, device=dev, generator=gen)
        gx = torch.empty_like(gE)
        gu = torch.empty_like(gE)

        def fb_step(alg, e, b):
            ctx.forward_device(N, pos.data_ptr(), mom.data_ptr(), e.data_ptr(), b.data_ptr(), alg,
                               save_for_backward=True)
            ctx.backward_device(gE.data_ptr(), gB.data_ptr(), gx.data_ptr(), gu.data_ptr())

        fwd_bwd = {}
        for name, alg, e, b, ms_f in (("mixed", alg_mixed, E, B, ms_mixed), ("fp64", alg_fp64, E64, B64, ms_fp64)):
            for _ in range(2):
                fb_step(alg, e, b)
            stream.synchronize()
            barrier(world)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(args.bwd_steps):
                fb_step(alg, e, b)
            ev1.record(stream)
            ev1.synchronize()
            ms_fb = max_over_ranks(world, ev0.elapsed_time(ev1) / args.bwd_steps)
            bwd_bytes = max(bwd_bytes or 0, int(ctx.stats()["device_bytes"]))
            fwd_bwd[name] = {"ms_per_step": ms_fb, "value": replicas.aggregate_rate(world, N, ms_fb),
                             "unit": "particles/s", "ratio_to_forward": ms_fb / ms_f, "steps": args.bwd_steps,
                             "warmup": 2, "grad_finite": bool(torch.isfinite(gx).all() and torch.isfinite(gu).all())}

    # tree reuse on a slowly drifting beam (mixed form)
    reuse = None
    if not args.skip_reuse:
        posd = pos.clone()
        ctx.set_tree_reuse(True)
        step(alg_mixed, E, B)  # builds the tree this loop starts from
        step(alg_mixed, E, B)
        stream.synchronize()
        total, kept = 0.0, 0
        for _ in range(args.steps):
            posd.add_(mom, alpha=1e-12)
            torch.cuda.synchronize(dev)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            ctx.forward_device(N, posd.data_ptr(), mom.data_ptr(), E.data_ptr(), B.data_ptr(), alg_mixed)
            ev1.record(stream)
            ev1.synchronize()
            total += ev0.elapsed_time(ev1)
            kept += int(ctx.stats()["tree_reused"])
        ctx.set_tree_reuse(False)
        ms_r = max_over_ranks(world, total / args.steps)
        reuse = {"ms_per_step": ms_r, "value": replicas.aggregate_rate(world, N, ms_r), "unit": "particles/s",
                 "steps": args.steps, "steps_tree_kept": kept, "ms_tree_last": ctx.stats()["ms_tree"]}

    # roofline of the dominant kernel (M2L) against the measured CUDA-core FMA peak
    p64 = ctypes.c_double()
    p32 = ctypes.c_double()
    p2 = ctypes.c_double()
    ctx._check(L.fmmb200_measure_fma_peak(ctx.handle, ctypes.byref(p64), ctypes.byref(p32), ctypes.byref(p2)))
    m2l_flops = 41.0 * st["m2l_kernel_evals"]
    ach32 = m2l_flops / (st["ms_m2l"] * 1e-3) / 1e12 if st["ms_m2l"] > 0 else 0.0
    ach64 = 41.0 * st64["m2l_kernel_evals"] / (st64["ms_m2l"] * 1e-3) / 1e12 if st64["ms_m2l"] > 0 else 0.0
    kname = "m2l_tc_kernel" if (args.m2l_engine == "tensor_cores" and args.n <= 4) else "m2l_x2_kernel"
    # DRAM bytes of the packed M2L kernel per M2L pair (read + write), from an ncu capture of the
    # same kernel on the N = 2^22 bunch (1.056e9 B for 2,557,114 pairs), scaled by this run's pairs
    traffic = 413.0 * st["nm2l"] if kname == "m2l_x2_kernel" and args.n == 4 else None
    roof = {"kernel": f"{kname}<{args.n}> (mixed)", "bound": "fp32", "achieved": ach32, "peak": p32.value,
            "unit": "TFLOP/s", "frac": ach32 / p32.value if p32.value else None, "traffic": traffic,
            "traffic_unit": "bytes per launch (scaled by M2L pairs from the N=2^22 capture)",
            "peak_source": "measured FP32 FMA throughput of this GPU (fmmb200_measure_fma_peak): the kernel runs "
                           "on the CUDA cores, so neither the HBM nor the bf16 tensor figure bounds it",
            "peak_fp32x2_measured": p2.value,
            "flops_per_launch": m2l_flops, "ms_per_launch": st["ms_m2l"],
            "fp64": {"kernel": f"m2l_kernel<{args.n}> (fp64)", "achieved": ach64, "peak": p64.value,
                     "frac": ach64 / p64.value if p64.value else None, "ms_per_launch": st64["ms_m2l"]}}
    # The FP32 pipe executes one FMA-class operation per lane per cycle, packed or not, so an
    # operation count per evaluation turns the kernel time into the pipe's occupancy:
    # M2L 15 per evaluation (3 denominator, 2 s^3, 10 factored sums), P2P 30 for tiles near
    # the target leaf (9 for R from hi/lo parts, 3 R.R, 3 u.R, 1 d, 2 s^3, 3 K, 3 E, 6 B) and
    # 24 for the far ones (R from the hi parts alone); the peak is the measured FMA rate / 2.
    pipe = p32.value * 1e12 / 2.0
    if st["ms_m2l"] > 0 and pipe > 0:
        roof["fp32_pipe_occupancy"] = 15.0 * st["m2l_kernel_evals"] / (st["ms_m2l"] * 1e-3) / pipe
    if st["ms_p2p"] > 0:
        ach_p = 41.0 * st["p2p_kernel_evals"] / (st["ms_p2p"] * 1e-3) / 1e12
        # the attainable rate of the kernel's own evaluation body (sources in shared memory,
        # no staging or barriers), for far and near tiles: the ceiling of this instruction mix
        bfar = ctypes.c_double()
        bnear = ctypes.c_double()
        ctx._check(L.fmmb200_measure_p2p_body(ctx.handle, ctypes.byref(bfar), ctypes.byref(bnear)))
        rate = st["p2p_kernel_evals"] / (st["ms_p2p"] * 1e-3)
        roof["p2p"] = {"kernel": "p2p_x2_kernel (mixed)", "achieved": ach_p, "peak": p32.value, "unit": "TFLOP/s",
                       "frac": ach_p / p32.value if p32.value else None, "ms_per_launch": st["ms_p2p"],
                       "fp32_pipe_occupancy_if_all_near": 30.0 * rate / pipe if pipe > 0 else None,
                       "fp32_pipe_occupancy_if_all_far": 24.0 * rate / pipe if pipe > 0 else None,
                       "evals_per_s": rate, "body_rate_far": bfar.value, "body_rate_near": bnear.value,
                       "frac_of_body_rate_far": rate / bfar.value if bfar.value else None,
                       "frac_of_body_rate_near": rate / bnear.value if bnear.value else None,
                       "min_ms_at_body_rate_far": st["p2p_kernel_evals"] / bfar.value * 1e3 if bfar.value else None}

    # end to end through the host-pointer C-ABI (pinned host buffers)
    e2e = None
    if not args.skip_e2e:
        ph = torch.from_numpy(pos_h).pin_memory()
        mh = torch.from_numpy(mom_h).pin_memory()
        eh = torch.empty((N, 3), dtype=torch.float64).pin_memory()
        bh = torch.empty((N, 3), dtype=torch.float64).pin_memory()
        pd = ctypes.cast(ph.data_ptr(), ctypes.POINTER(ctypes.c_double))
        md = ctypes.cast(mh.data_ptr(), ctypes.POINTER(ctypes.c_double))
        ed = ctypes.cast(eh.data_ptr(), ctypes.POINTER(ctypes.c_double))
        bd = ctypes.cast(bh.data_ptr(), ctypes.POINTER(ctypes.c_double))

        def host_step():
            ctx._check(L.fmmb200_update_particles_field(ctx.handle, N, -1.0, pd, md, ed, bd, args.n, args.N0,
                                                        args.eta, 1.0, fmmb200.PRECISION_MIXED))

        for _ in range(args.warmup):
            host_step()
        barrier(world)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            host_step()
        ev1.record(stream)
        ev1.synchronize()
        ms_e2e = max_over_ranks(world, ev0.elapsed_time(ev1) / args.steps)
        assert torch.equal(eh, E_main.cpu()), "host-pointer and device-pointer paths must agree"
        e2e = {"value": replicas.aggregate_rate(world, N, ms_e2e), "unit": "particles/s", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": 2 * 24 * N, "d2h_bytes_per_step": 2 * 24 * N}

    nsweep = None
    large = None
    configs = None
    if world == 1 and not args.skip_nsweep:
        nsweep = run_nsweep(args, ctx, stream, N, pos, mom, tg, Ed, Bd)
    if world == 1 and args.large_N > 0:
        large = run_large(args, ctx, stream, dev)
    if world == 1 and not args.skip_configs:
        configs = run_configs(args, stream, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        cpu = cpu_baseline(args)

    if rank == 0:
        stages = {k: st[k] for k in ("ms_tree", "ms_upward", "ms_lists", "ms_m2l", "ms_p2p", "ms_downward")}
        stages64 = {k: st64[k] for k in ("ms_tree", "ms_upward", "ms_lists", "ms_m2l", "ms_p2p", "ms_downward")}
        mf = model_flops(st, args.n, N)
        out = {
            "metric": METRIC, "value": replicas.aggregate_rate(world, N, ms_mixed), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded Gaussian bunch per rank (the reference benchmarks no public dataset)",
            "config": workload(args),
            "fp64": {"value": replicas.aggregate_rate(world, N, ms_fp64), "unit": "particles/s", "ms_per_step": ms_fp64,
                     "stages_ms": stages64, "mixed_speedup": ms_fp64 / ms_mixed},
            "accuracy": acc,
            "stages_ms": stages,
            "work": {"nm2l": st["nm2l"], "np2p": st["np2p"], "m2l_kernel_evals": st["m2l_kernel_evals"],
                     "p2p_kernel_evals": st["p2p_kernel_evals"], "max_level": st["max_level"],
                     "ncluster": st["ncluster"], "model_flops_per_step": mf,
                     "model_tflops_mixed": mf / (ms_mixed * 1e-3) / 1e12,
                     "model_tflops_fp64": mf / (ms_fp64 * 1e-3) / 1e12, "device_bytes": st["device_bytes"],
                     "device_bytes_with_backward": bwd_bytes,
                     "torch_peak_bytes": int(torch.cuda.max_memory_allocated(dev))},
            "fwd_bwd": fwd_bwd,
            "reuse": reuse,
            "nsweep": nsweep,
            "large": large,
            "configs": configs,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(st["kernel_launches"]) * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    ctx.close()


def run_sharded(args, world, rank, local):
    """One beam of args.N particles over the ranks: mixed form, device-resident, the
    exchange (all-gather in, reduce-scatter out) inside the timed region."""
    import torch

    import fmmb200
    from fmmb200 import sharded

    dev = torch.device("cuda", local)
    N = args.N
    pos_h, mom_h = generate(args, N, args.seed)
    lo, hi = N * rank // world, N * (rank + 1) // world
    pos = torch.from_numpy(pos_h[lo:hi]).to(dev)
    mom = torch.from_numpy(mom_h[lo:hi]).to(dev)
    ctx = fmmb200.Context(local)
    ctx_lists = fmmb200.Context(local)
    alg = fmmb200.FMMB200(n=args.n, N0=args.N0, eta=args.eta, precision="mixed")
    info = {}

    def step():
        return sharded.sharded_fields(pos, mom, alg, ctx=ctx, ctx_lists=ctx_lists, info=info)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier(world)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(uuid) as clk:
        ev0.record()
        for _ in range(args.steps):
            E, B = step()
        ev1.record()
        ev1.synchronize()
    torch.cuda.synchronize(dev)
    barrier(world)
    ms = max_over_ranks(world, ev0.elapsed_time(ev1) / args.steps)
    if rank == 0:
        cfg = workload(args)
        cfg["workload"] = cfg["workload"].replace("value = mixed form, fp64 = plain path",
                                                  f"one beam split over {world} rank(s), mixed form")
        cfg["parallelism"] = f"shard{world}"
        print(json.dumps({
            "metric": METRIC, "value": N / (ms * 1e-3), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: one seeded Gaussian bunch split over the ranks", "config": cfg,
            "shard": {k: info.get(k) for k in ("particles", "halo_particles", "remote_clusters", "subtree_clusters",
                                                  "device_bytes", "list_device_bytes", "halo_bytes",
                                                  "remote_moment_bytes")},
            "clocks": clk.summary(),
        }), flush=True)
    ctx.close()
    ctx_lists.close()


def run_shard_emulate(args):
    """The memory-sharded forward with G ranks evaluated in turn on this one GPU: per-rank
    compute time (the rank's library calls, which return when their GPU work is done) and
    device memory, and whether the fields equal the single-GPU forward's bit for bit."""
    import torch

    import fmmb200
    from fmmb200 import sharded

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    N = args.N
    pos_h, mom_h = generate(args, N, args.seed)
    alg = fmmb200.FMMB200(n=args.n, N0=args.N0, eta=args.eta, precision="mixed")
    out = {"workload": workload(args)["workload"], "N": N, "ranks": {}}
    for G in [int(x) for x in args.shard_emulate.split(",") if x]:
        bounds = [N * r // G for r in range(G + 1)]
        slots = [dict(pos=torch.tensor(pos_h[bounds[r]:bounds[r + 1]], device=dev),
                      mom=torch.tensor(mom_h[bounds[r]:bounds[r + 1]], device=dev),
                      ctx=fmmb200.Context(0), ctx_lists=fmmb200.Context(0)) for r in range(G)]
        comm = sharded.LoopbackComm(G)
        res = sharded.forward_slots(comm, slots, alg)  # warm-up: allocates every rank's buffers
        for s in slots:
            s["ms"] = {}
        steps = max(1, min(args.steps, 3))
        for _ in range(steps):
            res = sharded.forward_slots(comm, slots, alg)
        pavg = slots[0]["info"]["pavg"]
        per_rank = []
        for s in slots:
            ms = {k: v / steps for k, v in s["ms"].items()}
            per_rank.append(dict(ms=ms, ms_total=sum(ms.values()), **{k: s["info"][k] for k in (
                "particles", "halo_particles", "remote_clusters", "device_bytes", "list_device_bytes", "halo_bytes",
                "remote_moment_bytes")}))
        E = torch.cat([e for e, _ in res])
        B = torch.cat([b for _, b in res])
        del res
        for s in slots:
            s["ctx"].close()
            s["ctx_lists"].close()
        del slots
        torch.cuda.empty_cache()
        with fmmb200.Context(0) as one:
            pos = torch.tensor(pos_h, device=dev)
            mom = torch.tensor(mom_h, device=dev)
            E1 = torch.empty_like(pos)
            B1 = torch.empty_like(pos)
            one.set_stream(torch.cuda.current_stream(dev).cuda_stream)
            one.set_timing(True)
            for _ in range(2):
                one.forward_device(N, pos.data_ptr(), mom.data_ptr(), E1.data_ptr(), B1.data_ptr(), alg, p_avg=pavg)
            torch.cuda.synchronize(dev)
            single = one.stats()
            same = bool(torch.equal(E, E1) and torch.equal(B, B1))
            del pos, mom, E1, B1
        out["ranks"][str(G)] = {"max_rank_ms": max(r["ms_total"] for r in per_rank),
                                "max_rank_device_bytes": max(r["device_bytes"] + r["list_device_bytes"]
                                                             for r in per_rank),
                                "single_gpu_device_bytes": single["device_bytes"],
                                "single_gpu_ms": single["ms_tree"] + single["ms_upward"] + single["ms_lists"]
                                + single["ms_m2l"] + single["ms_p2p"] + single["ms_downward"],
                                "bit_identical_to_single_gpu": same, "per_rank": per_rank}
        del E, B
        torch.cuda.empty_cache()
        print(json.dumps({"shard_emulate_rows": G, **out["ranks"][str(G)]}), file=sys.stderr, flush=True)
    print(json.dumps({"shard_emulated": out}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        world, rank, _ = replicas.env_ranks()
        run_reference(args, world, rank)
        return
    if args.shard_emulate:
        run_shard_emulate(args)
        return
    world, rank, local = dist_setup(args)
    try:
        (run_sharded if args.shard else run_ours)(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
