#!/usr/bin/env python3
"""bench.py -- RK4 steps/s of the GPE real-time hot path on B200.

Workload (the headline configuration): single-component real-time quench on a
128^3 grid over [-10,10]^3 in oscillator units, V = 0.5(x^2 + y^2 + (2z)^2),
starting from the imaginary-time ground state at g = 1000 computed in the same
run (heavy-ball scheme of the reference), then g -> 1100 at t = 0 and RK4 with
dt = 5e-4.  The measured form is complex64 fields/FFTs with FP64 stage
coefficients and FP64 compensated reductions; the plain complex128 drop-in is
timed beside it, and the accuracy of the complex64 form after 10^4 steps is
reported against complex128 (pinned to the FP64 oracle by the test suite).

One "step" = one full RK4 step (4 stages x 4 fused axis passes, run as one
persistent launch when the tuner picks the persistent step).  L2 is
flushed (256 MiB write) before every timed step; each step is bracketed by
CUDA events on the library's stream.  `--impl reference` times the FP64 host
oracle port of the reference's algorithm (the reference has no CPU path).
Multi-GPU: the path does not shard (replicas only); every rank runs its own
instance and value = total steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 128
L_BOX = 10.0
G0, G1 = 1000.0, 1100.0
DT = 5e-4
PI_REF = 3.141592653589793
F_PER_STEP_KERNELS = {"x_fwd": 2.0, "x_inv": 7.75, "s_fwd": 2.0, "s_inv": 2.0, "s_fki": 2.0, "x_full": 0.0,
                      "flow": 55.0, "s_flow": 6.0}
# Algorithmic field transfers per launch of each pass kind in the 1-component
# complex64 real-time RK4 step (F = one field): x-forward reads the stage
# state and writes the work field (it runs only before the first stage of a
# call); strided passes read and write the work field; the x-inverse
# epilogue of stage 1/2/3/4 moves 5/7/7/8 fields (stage 4 also reads and
# writes the low part of the compensated state) and writes the x-forward
# transform of the state it produced for the next stage (+1 field): mean 7.75.
# The persistent step kernel ("flow") runs all sixteen passes of a step in
# one launch: 12 strided passes x 2 F + the four x passes' 6 + 8 + 8 + 9 F;
# the persistent strided stage ("s_flow") the three strided passes of a stage.


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--accuracy-steps", type=int, default=10000)
    p.add_argument("--quick", action="store_true", help="skip the 10^4-step accuracy run and the CPU baseline")
    p.add_argument("--grid", type=int, default=N_GRID)
    p.add_argument("--ground-steps", type=int, default=3000, help="heavy-ball iterations for the initial state")
    p.add_argument("--cufft", action="store_true",
                   help="print the comparison line: cuFFT (torch.fft) 3D forward + inverse at the same grid")
    p.add_argument("--workload", default="quench3d", choices=["quench3d", "sweep2d", "control2d", "imag3d"],
                   help="sweep2d: 256 batched 2D imaginary-time instances; control2d: adjoint gradient of a "
                        "256^2 optimal-control problem (separate JSON lines)")
    p.add_argument("--fd-components", type=int, default=32, help="control2d: finite-difference checks")
    p.add_argument("--sweep-instances", type=int, default=256)
    p.add_argument("--no-tune", action="store_true", help="keep the default pass variants (no autotuning)")
    p.add_argument("--tune-cache", default=None,
                   help="JSON-lines tuning cache to reuse: grids with a line there are not tuned again")
    p.add_argument("--persistent-step", default="tuned", choices=["tuned", "on", "strided", "off"],
                   help="complex64 persistent launches (gpe_set_flow): the tuner's choice, one launch per step "
                        "(on), one launch per stage's strided passes (strided), or the per-pass chain (off)")
    p.add_argument("--oracle-steps", type=int, default=0,
                   help="also run the FP64 oracle (the checker of the CPU leg) to this many steps and compare "
                        "both GPU forms with it there (10000: about 14 min on 16 host cores)")
    p.add_argument("--sweep-converge", action="store_true",
                   help="sweep2d: also run every instance to |dmu| < 1e-8 and report the iterations")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_config(n, precision, g, imag=False):
    import fgpe_b200 as gp
    prms = np.zeros(32)
    prms[0:3] = g / (4 * PI_REF)
    return gp.make_config((n, n, n), L_BOX, dt=(2e-3 if imag else DT), precision=precision, prms=prms,
                          beta=0.9, npart=(1.0, 1.0), epsilon_e=1e-12)


def trap(cfg):
    import fgpe_b200 as gp
    x, y, z = gp.grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return 0.5 * (X ** 2 + Y ** 2 + (2 * Z) ** 2) + 0j


def initial_psi(cfg, seed=1):
    import fgpe_b200 as gp
    x, y, z = gp.grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rng = np.random.default_rng(seed)
    g = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 2.0)
    psi = g * (1 + 1e-3 * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)))
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    return psi / np.sqrt(np.sum(np.abs(psi) ** 2) * dv)


def cached_or_tune(cfg, workload, cache):
    """The cache's line for cfg's grid (nb = 1), or a fresh tuning stored there."""
    import fgpe_b200 as gp
    if os.path.exists(cache):
        nf = cfg.ncomp + (1 if cfg.hamiltonian in (gp.HAM_DIPOLAR, gp.HAM_SOFT) else 0)
        for line in open(cache):
            try:
                d = json.loads(line)
            except ValueError:
                continue
            if (d.get("nx"), d.get("ny"), d.get("nz"), d.get("prec"), d.get("nf"), d.get("nb")) == \
                    (cfg.nx, cfg.ny, cfg.nz, cfg.precision, nf, 1):
                return {"default_us": d["default_us"], "tuned_us": d["tuned_us"], "from_cache": cache,
                        "variants": [d[k] for k in ("s10", "s11", "s12", "s20", "s21", "s22")],
                        "xrows": d["xrows"], "yz": d.get("yz", 0), "flow": d.get("flow", 0),
                        "xstage": d.get("xstage", 0)}
    return gp.tune(cfg, workload, cache)


def workload_conf(n, world=1):
    """The `config` object both arms print (the same workload)."""
    return {"workload": f"real-time RK4 quench, {n}^3 on [-10,10]^3, V=0.5(x^2+y^2+4z^2), g 1000->1100, dt 5e-4",
            "grid": [n, n, n], "parallelism": "replicas" if world > 1 else "single GPU"}


def ground_state(n, stream_ptr, iters=3000):
    """Heavy-ball imaginary time (the reference's scheme) at g = 1000, complex128."""
    import fgpe_b200 as gp
    cfg = workload_config(n, gp.C128, G0, imag=True)
    s = gp.Solver(cfg)
    s.set_stream(stream_ptr)
    s.set_vext(0, trap(cfg))
    s.set_psi(0, initial_psi(cfg))
    done, conv = s.step_imag(0, iters)
    st = s.imag_state()
    psi = s.get_psi(0)
    s.close()
    return psi, {"iterations": done, "converged": bool(conv), "mu": float(st[1]), "E": float(st[2])}


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"gpe_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        top = sorted(sm)[len(sm) // 2:] if len(sm) > 4 else sm  # samples under load
        return {"sm_mhz": float(np.median(top)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def time_steps(solver, torch, flush, steps, first_it, profile=False):
    """K RK4 steps, L2 flushed before each, CUDA events on the library stream."""
    st = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    solver.profile(profile)
    if profile:
        solver.profile_read()
    l0 = solver.launches
    for k in range(steps):
        flush.zero_()
        evs[k][0].record(st)
        solver.step_real(first_it + k, 1)
        evs[k][1].record(st)
    torch.cuda.synchronize()
    launches = solver.launches - l0
    ms = float(sum(a.elapsed_time(b) for a, b in evs))
    prof = solver.profile_read() if profile else None
    solver.profile(False)
    return ms, launches, prof


def run_ours(args):
    import torch
    import fgpe_b200 as gp

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    stream_ptr = torch.cuda.current_stream().cuda_stream
    n = args.grid
    K, W = args.steps, max(args.warmup, 3)

    psi_gs, prep = ground_state(n, stream_ptr, args.ground_steps)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # autotune the pass variants of both forms for this grid (setup, like a
    # transform planner: outside the timed region), then create the handles
    tune_cache = args.tune_cache or os.path.join("/tmp", f"gpe_tune_{os.getpid()}.jsonl")
    tuning = {}
    if not args.no_tune:
        for name, prec in (("c64", gp.C64), ("c128", gp.C128)):
            tuning[name] = cached_or_tune(workload_config(n, prec, G1), 0, tune_cache)
        gp.set_tune_cache(tune_cache)
    solvers = {}
    for name, prec in (("c64", gp.C64), ("c128", gp.C128)):
        cfg = workload_config(n, prec, G1)
        s = gp.Solver(cfg)
        s.set_stream(stream_ptr)
        s.set_vext(0, trap(cfg))
        s.set_psi(0, psi_gs)
        if name == "c64" and args.persistent_step != "tuned":
            s.set_flow({"on": 1, "strided": 2, "off": 0}[args.persistent_step])
        solvers[name] = s

    results = {}
    with Clocks(dev) as clk:
        for name, s in solvers.items():
            for w in range(W):
                flush.zero_()
                s.step_real(w, 1)
            torch.cuda.synchronize()
            ms, launches, _ = time_steps(s, torch, flush, K, W)
            ms_p, _, prof = time_steps(s, torch, flush, K, W + K, profile=True)
            results[name] = {"ms": ms, "launches": launches, "ms_prof": ms_p, "prof": prof}
        # the per-pass chain beside the persistent step (same handle, same work)
        s = solvers["c64"]
        persistent = {"active": s.flow_active}
        if s.flow_active:
            mode = s.flow_active
            s.set_flow(0)
            for w in range(W):
                flush.zero_()
                s.step_real(W + 2 * K + w, 1)
            ms_chain, l_chain, _ = time_steps(s, torch, flush, K, 2 * W + 2 * K)
            s.set_flow(mode)
            persistent.update({"ms_per_step_persistent": round(results["c64"]["ms"] / K, 5),
                               "ms_per_step_chain": round(ms_chain / K, 5),
                               "launches_per_step_persistent": results["c64"]["launches"] / K,
                               "launches_per_step_chain": l_chain / K,
                               "speedup_persistent_over_chain": round(ms_chain / results["c64"]["ms"], 3)})
    clocks = clk.summary()

    # max over ranks
    ms64, ms128 = results["c64"]["ms"], results["c128"]["ms"]
    if dist is not None:
        t = torch.tensor([ms64, ms128], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms64, ms128 = float(t[0]), float(t[1])
        dist.barrier()
    if rank != 0:
        for s in solvers.values():
            s.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    N = n ** 3
    F64 = 8 * N  # one complex64 field in bytes
    value = world * K / (ms64 / 1e3)
    value128 = world * K / (ms128 / 1e3)

    # roofline of the dominant pass kernel (complex64 form), live event timing
    prof = results["c64"]["prof"]
    dom = max((k for k in prof if prof[k][1] > 0), key=lambda k: prof[k][0])
    dom_ms, dom_cnt = prof[dom]
    dom_bytes = F_PER_STEP_KERNELS[dom] * F64
    achieved = dom_bytes / (dom_ms / dom_cnt / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    insitu = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic_128cubed_c64.txt")
    if os.path.exists(tpath) and n == 128:
        for line in open(tpath):
            f = line.split()
            if len(f) >= 2 and f[0] == dom:
                traffic = float(f[1])
            if len(f) >= 2 and f[0] == "step_insitu":
                insitu = float(f[1])
    step_bytes = sum(F_PER_STEP_KERNELS[k] * F64 * prof[k][1] for k in prof) / K
    step_ms = ms64 / K

    # e2e through the C ABI: H2D of the step's psi (pinned, complex128) + 1 step + D2H of observables
    import torch as _t
    s = solvers["c64"]
    host = _t.empty(2 * N, dtype=_t.float64, pin_memory=True)
    hv = host.numpy().view(np.complex128)
    hv[:] = psi_gs.reshape(-1)
    e2e_t = []
    for k in range(W + K):
        t0 = time.perf_counter()
        s.set_psi(0, hv)
        s.step_real(k, 1, want_obs=True)
        t1 = time.perf_counter()
        if k >= W:
            e2e_t.append(t1 - t0)
    e2e = {"value": world * K / sum(e2e_t), "unit": "steps/s", "h2d_bytes_per_step": 16 * N,
           "d2h_bytes_per_step": 208, "note": "gpe_set_psi(host pinned complex128) + gpe_step_real(1, observables)"}

    line = {
        "metric": "RK4 steps/s at 128^3 (complex64 + FP64 reductions, real-time quench)",
        "value": round(value, 2),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(step_ms, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Gaussian -> heavy-ball ground state at g=1000, quench to g=1100)",
        "config": workload_conf(n, world),
        "form": "complex64 fields/FFT, FP64 stage coefficients and reductions",
        "l2": "flushed before every timed step (256 MiB write)",
        "plain_c128": {"value": round(value128, 2), "unit": "steps/s", "ms_per_step": round(ms128 / K, 5),
                       "speedup_c64_over_c128": round(value / value128, 3)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                     "step_algorithmic_bytes": step_bytes,
                     "step_achieved_gbs": round(step_bytes / (step_ms / 1e3) / 1e9, 1),
                     "step_frac": round(step_bytes / (step_ms / 1e3) / 1e9 / peak, 4),
                     "survey_45F_step_frac": round(45 * F64 / (step_ms / 1e3) / 1e9 / peak, 4),
                     "per_kind_ms_per_launch": {k: round(v[0] / v[1], 5) for k, v in prof.items() if v[1]},
                     "profiled_ms_per_step": round(results["c64"]["ms_prof"] / K, 5),
                     # ncu with caches kept between the 16 launches of a flushed step: the
                     # step's six fields (101 MB) stay in the 126 MB L2, so the passes are
                     # bound by L2 latency and issue, not by HBM bandwidth
                     "insitu_dram_bytes_per_step": insitu,
                     "l2_resident_fields": insitu is not None and insitu < 0.5 * step_bytes},
        "e2e": e2e,
        "persistent_step": persistent,
        "tuning": tuning or "off (--no-tune): default pass variants",
        "gpu_launches": results["c64"]["launches"],
        "clocks": clocks,
        "prep": prep,
    }

    if not args.quick:
        line["accuracy"] = accuracy(solvers, psi_gs, args.accuracy_steps)
        line["cpu_baseline"] = cpu_baseline(n, psi_gs, solvers, long_steps=args.oracle_steps)
        if world == 1:
            # the reference's own CUDA build (complex128, cuFFT) on this GPU,
            # same loop: the GPU-vs-GPU comparison figure
            rb = reference_cuda_build(n)
            if "steps_per_s" in rb:
                rb["c64_over_reference_build"] = round(value / rb["steps_per_s"], 3)
                rb["c128_over_reference_build"] = round(value128 / rb["steps_per_s"], 3)
            line["reference_cuda_build"] = rb
    else:
        line["cpu_baseline"] = None
    for s2 in solvers.values():
        s2.close()
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def accuracy(solvers, psi_gs, nsteps):
    """complex64 vs complex128 after nsteps RK4 steps from the same ground state."""
    out = {"steps": nsteps}
    res = {}
    for name, s in solvers.items():
        s.set_psi(0, psi_gs)
        o0 = s.observables(0.0)
        chunk = 500
        for k in range(0, nsteps, chunk):
            s.step_real(k, min(chunk, nsteps - k))
        o1 = s.observables(nsteps * DT)
        res[name] = (s.get_psi(0), o0, o1)
    p64, a0, a1 = res["c64"]
    p128, b0, b1 = res["c128"]
    out["psi_rel_l2_c64_vs_c128"] = float(np.linalg.norm(p64 - p128) / np.linalg.norm(p128))
    norm = b1[0]
    out["E_rel_err"] = float(abs(a1[2] / a1[0] - b1[2] / b1[0]) / abs(b1[2] / b1[0]))
    out["mu_rel_err"] = float(abs(a1[1] / a1[0] - b1[1] / b1[0]) / abs(b1[1] / b1[0]))
    out["norm_drift_c64"] = float(a1[0] / a0[0] - 1)
    out["norm_drift_c128"] = float(b1[0] / b0[0] - 1)
    out["energy_drift_c64"] = float(a1[2] / a0[2] - 1)
    out["energy_drift_c128"] = float(b1[2] / b0[2] - 1)
    out["E_c128"] = float(b1[2] / norm)
    out["reference_for_error"] = "complex128 path (parity-tested against the FP64 oracle at <= 1e-12)"
    return out


def cpu_baseline(n, psi_gs, solvers=None, budget_s=12.0, long_steps=0):
    """FP64 oracle port of the reference algorithm on the host cores, timed
    over a bounded sample of the workload: k RK4 steps from the same ground
    state.  The oracle's state after the sample is then the checker for both
    GPU forms run over the same k steps (psi, E and mu relative errors).
    long_steps > k: the oracle continues to long_steps steps (untimed, as the
    checker only) and both GPU forms are compared with it there, with the
    norm and energy drift of each against its own start."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    import fgpe_b200 as gp
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    cfg = workload_config(n, gp.C128, G1)
    o = orc.OracleSolver(cfg)
    o.set_vext(0, trap(cfg))
    o.set_psi(0, psi_gs)
    t0 = time.perf_counter()
    o.step_real(0, 1)
    one = time.perf_counter() - t0
    k = max(1, int(budget_s / max(one, 1e-3)))
    t0 = time.perf_counter()
    oo = o.step_real(1, k, want_obs=True)
    dt = time.perf_counter() - t0
    po = o.get_psi(0)
    long_run = None
    if solvers and long_steps > k + 1:
        o0 = orc.OracleSolver(cfg)
        o0.set_vext(0, trap(cfg))
        o0.set_psi(0, psi_gs)
        ostart = o0.observables(0.0)
        o0.close()
        o.step_real(k + 1, long_steps - (k + 1))
        ol = o.observables(long_steps * DT)
        pl = o.get_psi(0)
        long_run = {"steps": long_steps,
                    "oracle_norm_drift": float(ol[0] / ostart[0] - 1),
                    "oracle_energy_drift": float((ol[2] / ol[0]) / (ostart[2] / ostart[0]) - 1)}
        for name, s in solvers.items():
            s.set_psi(0, psi_gs)
            g0 = s.observables(0.0)
            done = 0
            while done < long_steps:
                m = min(500, long_steps - done)
                s.step_real(done, m)
                done += m
            gl = s.observables(long_steps * DT)
            pg = s.get_psi(0)
            long_run[name] = {"psi_rel_l2": float(np.linalg.norm(pg - pl) / np.linalg.norm(pl)),
                              "E_rel_err": float(abs(gl[2] / gl[0] - ol[2] / ol[0]) / abs(ol[2] / ol[0])),
                              "mu_rel_err": float(abs(gl[1] / gl[0] - ol[1] / ol[0]) / abs(ol[1] / ol[0])),
                              "norm_drift": float(gl[0] / g0[0] - 1),
                              "energy_drift": float((gl[2] / gl[0]) / (g0[2] / g0[0]) - 1)}
    o.close()
    out = {"value": round(k / dt, 4), "unit": "steps/s", "cores": threads, "kind": "port",
           "sample": f"{k + 1} RK4 steps of the same {n}^3 workload from the same ground state in FP64 "
                     f"(oracle/gpe_oracle.cpp, OpenMP); {k} of them timed"}
    if solvers:
        par = {"steps": k + 1}
        for name, s in solvers.items():
            s.set_psi(0, psi_gs)
            og = s.step_real(0, k + 1, want_obs=True)
            pg = s.get_psi(0)
            par[name] = {"psi_rel_l2": float(np.linalg.norm(pg - po) / np.linalg.norm(po)),
                         "E_rel_err": float(abs(og[2] / og[0] - oo[2] / oo[0]) / abs(oo[2] / oo[0])),
                         "mu_rel_err": float(abs(og[1] / og[0] - oo[1] / oo[0]) / abs(oo[1] / oo[0])),
                         "norm_rel_err": float(abs(og[0] / oo[0] - 1))}
        if long_run is not None:
            par["long_run"] = long_run
        out["parity_vs_port"] = par
    return out


def reference_cuda_build(n, imag=False):
    """The reference's own CUDA build (complex128, cuFFT; oracle/_ref, built
    from its sources) timed on this GPU for the same real-time RK4 loop (or,
    imag, its heavy-ball imaginary-time loop): a comparison figure."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import tempfile
        import time_ref_build as trb
        if not os.path.exists(trb.BIN):
            return {"unavailable": "oracle/_ref/gpe_ref_trace not built"}
        n1, n2, rep = 200, 1200, 3
        with tempfile.TemporaryDirectory() as work:
            trb.run(n, 10, work, imag)
            diffs = sorted((trb.run(n, n2, work, imag) - trb.run(n, n1, work, imag)) / (n2 - n1)
                           for _ in range(rep))
        per = diffs[len(diffs) // 2]
        loop = "runImagTimeEvol" if imag else "runRealTimeEvol"
        return {"steps_per_s": round(1.0 / per, 2), "ms_per_step": round(1e3 * per, 4), "dtype": "f64",
                "method": f"median over {rep} of loop(niter={n2}) - loop(niter={n1}), device-synchronised wall "
                          f"time of the reference's own {loop} loop"}
    except Exception as e:  # comparison only: never fail the arm
        return {"unavailable": str(e)[:200]}


def run_reference(args):
    """CPU reference arm: the FP64 oracle port of the reference's algorithm on
    the host cores (the reference has no CPU path), same workload, warm-up and
    config as the GPU arm.  Its line also carries the reference's own CUDA
    build timed on this GPU (comparison only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    import fgpe_b200 as gp
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    n = args.grid
    cfg = workload_config(n, gp.C128, G1)
    o = orc.OracleSolver(cfg)
    o.set_vext(0, trap(cfg))
    o.set_psi(0, initial_psi(cfg))
    W, K = max(args.warmup, 3), args.steps
    t0 = time.perf_counter()
    o.step_real(0, 1)
    one = time.perf_counter() - t0
    o.step_real(1, W - 1)
    # bounded sample: at most ~60 s of timed CPU work
    K = max(1, min(K, int(60.0 / max(one, 1e-3))))
    t0 = time.perf_counter()
    o.step_real(W, K)
    dt = time.perf_counter() - t0
    v = K / dt
    line = {"impl": "reference", "metric": "RK4 steps/s at 128^3 (complex64 + FP64 reductions, real-time quench)",
            "value": round(v, 4), "unit": "steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": round(1e3 * dt / K, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian start)",
            "config": workload_conf(n, world),
            "form": "complex128 FP64 (oracle port of the reference's algorithm)",
            "cpu_baseline": {"value": round(v, 4), "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": f"{K} FP64 RK4 steps of the {n}^3 workload after {W} warm-up steps "
                                       f"(oracle port of the reference algorithm; the reference has no CPU path)"},
            "e2e": {"value": round(v, 4), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    o.close()
    line["reference_cuda_build"] = reference_cuda_build(n)
    print(json.dumps(line))


def run_cufft(args):
    """Comparison only: one 3D forward + inverse transform pair with cuFFT
    (through torch.fft) per precision, L2 flushed before each pair."""
    import torch
    n = args.grid
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"impl": "cuFFT (torch.fft.fftn + ifftn), comparison only", "grid": [n, n, n]}
    for name, dt in (("c64", torch.complex64), ("c128", torch.complex128)):
        x = torch.randn(n, n, n, dtype=dt, device="cuda")
        for _ in range(3):
            torch.fft.ifftn(torch.fft.fftn(x))
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        for a, b in evs:
            flush.zero_()
            a.record()
            y = torch.fft.fftn(x)
            x = torch.fft.ifftn(y)
            b.record()
        torch.cuda.synchronize()
        ms = sorted(a.elapsed_time(b) for a, b in evs)[len(evs) // 2]
        out[name + "_fwd_inv_pair_ms"] = round(ms, 5)
    print(json.dumps(out))


SWEEP_SIZES = (64, 96, 128, 192, 256, 384, 512)
SWEEP_DT = 4e-4


def sweep_instances(n_inst, precision, seed=4):
    """Seeded 2D imaginary-time sweep: N from SWEEP_SIZES, box [-L, L]^2 with
    L = 8 sqrt(N/64), g ~ U[10, 2000], omega_y/omega_x ~ U[1, 4], RK4 in
    imaginary time until |dmu| < 1e-8; Gaussian start with seeded 1e-3
    complex noise.  dt = 4e-4: the largest eigenvalue of H on the 512^2 grid
    (kinetic 2 pi^2 (kx^2 + ky^2) ~ 1.3e3 at the corner of k-space, trap
    ~ 4.4e3 at the corner of the box for omega_y/omega_x = 4) times dt must
    stay inside RK4's real stability interval (2.785)."""
    import fgpe_b200 as gp
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_inst):
        n = int(rng.choice(SWEEP_SIZES))
        g = float(rng.uniform(10.0, 2000.0))
        aniso = float(rng.uniform(1.0, 4.0))
        L = 8.0 * np.sqrt(n / 64.0)
        cfg = gp.make_config((n, n, 1), (L, L, 1.0), dt=SWEEP_DT, precision=precision, g=g,
                             imag_scheme=gp.IMAG_RK4, epsilon_e=1e-8)
        x, y, _ = gp.grid_axes(cfg)
        Y, X = np.meshgrid(y, x, indexing="ij")
        V = (0.5 * (X ** 2 + (aniso * Y) ** 2) + 0j).reshape(1, n, n)
        r2 = np.random.default_rng(1000 + i)
        p = np.exp(-(X ** 2 + Y ** 2) / 2.0)
        p = p * (1 + 1e-3 * (r2.standard_normal(p.shape) + 1j * r2.standard_normal(p.shape)))
        dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
        p = (p / np.sqrt(np.sum(np.abs(p) ** 2) * dv)).reshape(1, n, n)
        out.append((cfg, V, p, n, g, aniso))
    return out


def run_sweep(args):
    """Batched 2D sweep (one launch per pass per grid size, one CUDA graph per
    iteration) against the same instances solved one after another as plain
    complex128 handles; both as instance-iterations per second over a bounded
    number of iterations."""
    import torch
    import fgpe_b200 as gp
    from fgpe_b200 import sweep
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    K, W = args.steps, max(args.warmup, 3)
    everything = sweep_instances(args.sweep_instances, gp.C64)
    # shard by estimated cost; no data-path collective (instances are independent)
    mine = sweep.my_instances([(n, n, 1) for (_, _, _, n, _, _) in everything], rank, world)
    inst = [everything[i] for i in mine]
    stream = torch.cuda.Stream()
    b = gp.Batch([c for c, *_ in inst])
    b.set_stream(stream.cuda_stream)
    # autotune every geometry group in place: per group the default and the
    # tuned microseconds per iteration, measured on the same work
    tune_rep = None if args.no_tune else b.tune(os.path.join("/tmp", f"gpe_tune_{os.getpid()}.jsonl"))
    def timed(mode):
        """W warm-up and K timed iterations of every instance from the seeded
        start under one launch mode (per group; one cooperative launch per
        stage; one launch per pass over all groups)."""
        b.set_launch_mode(mode)
        for i, (c, V, p, *_ ) in enumerate(inst):
            b.set_vext(i, V)
            b.set_psi(i, p)
        b.step_imag(W)
        torch.cuda.synchronize()
        l0 = b.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, cv = b.step_imag(K)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), it, cv, b.launches - l0

    # both launch modes on the same work; the faster one is the headline
    mode_ids = {"per_group": gp.BATCH_PER_GROUP, "persistent": gp.BATCH_PERSISTENT, "grouped": gp.BATCH_GROUPED}
    modes = {}
    with Clocks(torch.cuda.current_device()) as clk:
        for name, mid in mode_ids.items():
            try:
                modes[name] = timed(mid)
            except gp.GPEError as e:
                modes[name] = str(e)
    best = min((k for k in modes if not isinstance(modes[k], str)), key=lambda k: modes[k][0])
    b.set_launch_mode(mode_ids[best])
    ms, it, cv, launches = modes[best]
    launch_modes = {k: (v if isinstance(v, str) else
                        {"ms_per_step": round(v[0] / K, 4), "launches_per_iteration": round(v[3] / K, 2),
                         "instance_steps_per_s": round(int(v[1].sum()) / (v[0] / 1e3), 1)})
                    for k, v in modes.items()}
    launch_modes["chosen"] = best
    inst_steps = int(it.sum())
    if dist is not None:
        t = torch.tensor([ms, float(inst_steps)], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        ms, inst_steps = float(tmax[0]), int(t[1])
    value = inst_steps / (ms / 1e3)
    points = sum(n * n for *_, n, _, _ in inst)
    # 45 F per RK4 imaginary step (plus its reductions), F = N*8 bytes
    alg_bytes = 45 * 8 * sum(n * n * int(k) for (_, _, _, n, _, _), k in zip(inst, it))
    peak, peak_kind = peaks()
    conv = None
    if args.sweep_converge:
        total = it.astype(np.int64).copy()
        t0 = time.perf_counter()
        for _ in range(60):  # at most 30000 iterations
            it2, cv = b.step_imag(500)
            total += it2
            if cv.all():
                break
        conv = {"all_converged": bool(cv.all()), "iterations_min": int(total.min()),
                "iterations_max": int(total.max()), "wall_s": round(time.perf_counter() - t0, 2)}
    b.close()
    if rank != 0:
        dist.barrier()
        dist.destroy_process_group()
        return
    # sequential complex128 solves, a bounded number of iterations each
    k_seq = max(3, min(20, K))
    seq_ms, seq_steps = 0.0, 0
    st = torch.cuda.current_stream()
    for (c, V, p, *_ ) in inst:
        c128 = c.copy()
        c128.precision = gp.C128
        s = gp.Solver(c128)
        s.set_stream(st.cuda_stream)
        s.set_vext(0, V)
        s.set_psi(0, p)
        s.step_imag(0, 2)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        done, _ = s.step_imag(2, k_seq)
        a1.record(st)
        torch.cuda.synchronize()
        seq_ms += a0.elapsed_time(a1)
        seq_steps += done
        s.close()
    seq_value = seq_steps / (seq_ms / 1e3)
    counts = {str(n): sum(1 for *_, m, _, _ in inst if m == n) for n in SWEEP_SIZES}
    line = {"metric": "instance-steps/s, 256 batched 2D imaginary-time instances (complex64 + FP64 reductions)",
            "value": round(value, 1), "unit": "instance-steps/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded sizes, couplings, anisotropies; Gaussian start)",
            "config": {"workload": "2D imaginary-time RK4 sweep", "instances": len(inst), "grid_counts": counts,
                       "points_total": points, "dt": SWEEP_DT, "epsilon_mu": 1e-8,
                       "l2": "inputs larger than L2 (%.0f MB of complex64 fields)" % (5 * 8 * points / 1e6)},
            "sequential_c128": {"value": round(seq_value, 1), "unit": "instance-steps/s",
                                "iterations_per_instance": k_seq,
                                "speedup_batched_over_sequential": round(value / seq_value, 2)},
            "roofline": {"bound": "hbm", "achieved": round(alg_bytes / (ms / 1e3) / 1e9, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(alg_bytes / (ms / 1e3) / 1e9 / peak, 4), "traffic": None,
                         "model": "45 F per RK4 imaginary iteration, F = N*8 B"},
            "tuning": tuning_summary(tune_rep, inst), "launch_modes": launch_modes, "clocks": clk.summary(),
            "gpu_launches": launches, "convergence": conv,
            "cpu_baseline": sweep_cpu_leg(everything, stream)}
    if world > 1:
        line["n_gpus"] = world
        line["config"]["parallelism"] = "instances sharded over ranks by estimated cost (no data-path collective)"
    print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def tuning_summary(rep, inst):
    """Per-group autotuner result of the sweep: default and tuned iteration
    times of each geometry group, and the sum over groups (one iteration of
    every group, as the captured graph runs them)."""
    if rep is None:
        return "off (--no-tune): default pass variants"
    sizes = []
    for (c, *_rest) in inst:
        key = (c.nx, c.ny)
        if key not in sizes:
            sizes.append(key)
    groups = {f"{nx}x{ny}": {"default_us": round(d, 2), "tuned_us": round(t, 2)} for (nx, ny), (d, t) in
              zip(sizes, rep)}
    tot_d = sum(d for d, _ in rep)
    tot_t = sum(t for _, t in rep)
    return {"groups": groups, "iteration_default_us": round(tot_d, 2), "iteration_tuned_us": round(tot_t, 2),
            "speedup": round(tot_d / tot_t, 3) if tot_t > 0 else None}


def sweep_cpu_leg(everything, stream, k=20, sizes=(64, 192, 512)):
    """CPU leg of the sweep: the FP64 oracle port timed on one seeded instance
    of each of a few sizes for k RK4 imaginary-time iterations, and, as the
    checker, those instances advanced together as one complex64 batch over
    the same iterations (psi, E, mu relative errors)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    import fgpe_b200 as gp
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    picks = []
    for want in sizes:
        for i, item in enumerate(everything):
            if item[3] == want:
                picks.append(i)
                break
    b = gp.Batch([everything[i][0] for i in picks])
    b.set_stream(stream.cuda_stream)
    for j, i in enumerate(picks):
        b.set_vext(j, everything[i][1])
        b.set_psi(j, everything[i][2])
    b.step_imag(k)
    res, t_cpu, pts = {}, 0.0, 0
    for j, i in enumerate(picks):
        cfg, V, p, n, g, aniso = everything[i]
        c128 = cfg.copy()
        c128.precision = gp.C128
        o = orc.OracleSolver(c128)
        o.set_vext(0, V)
        o.set_psi(0, p)
        t0 = time.perf_counter()
        o.step_imag(0, k)
        t_cpu += time.perf_counter() - t0
        pts += k
        so, po = o.imag_state(), o.get_psi(0)
        o.close()
        sb, pb = b.imag_state(j), b.get_psi(j)
        res[f"instance_{i}_N{n}"] = {"g": round(g, 3), "aniso": round(aniso, 4),
                                     "psi_rel_l2": float(np.linalg.norm(pb - po) / np.linalg.norm(po)),
                                     "E_rel_err": float(abs(sb[2] / so[2] - 1)),
                                     "mu_rel_err": float(abs(sb[1] / so[1] - 1))}
    b.close()
    return {"value": round(pts / t_cpu, 3), "unit": "instance-steps/s", "cores": threads, "kind": "port",
            "sample": f"{k} RK4 imaginary-time iterations of {len(picks)} seeded instances (N = {list(sizes)}) in "
                      f"FP64 (oracle/gpe_oracle.cpp)",
            "parity_vs_port": {"iterations": k, "form": "complex64 batch", "instances": res}}


def control_problem(precision, nsteps=2000, n=256, seed=5):
    """2D real-time control: 256^2 on [-10,10]^2, g = 200, psi0 = ground state of
    V0 = (x^2 + y^2)/2 (heavy ball in the same run), 16 Gaussian controls
    exp(-|x - c_k|^2/2) on a seeded 4x4 lattice of spacing 2, u ~ N(0, 0.1)
    piecewise constant per RK4 step (dt = 1e-3), target the dipole state
    x |psi0| normalised (the first excited state of the trap without
    interaction)."""
    import fgpe_b200 as gp
    rng = np.random.default_rng(seed)
    prms = np.zeros(32)
    prms[0:3] = 200.0 / (4 * PI_REF)
    cfg = gp.make_config((n, n, 1), (10.0, 10.0, 1.0), dt=1e-3, precision=precision, prms=prms,
                         beta=0.9, epsilon_e=1e-12)
    x, y, _ = gp.grid_axes(cfg)
    Y, X = np.meshgrid(y, x, indexing="ij")
    V0 = (0.5 * (X ** 2 + Y ** 2) + 0j).reshape(1, n, n)
    off = rng.uniform(-0.5, 0.5, size=2)
    cs = [(-3.0 + 2.0 * i + off[0], -3.0 + 2.0 * j + off[1]) for i in range(4) for j in range(4)]
    G = np.stack([np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / 2.0) for cx, cy in cs]).reshape(16, 1, n, n)
    u = rng.normal(0.0, 0.1, size=(nsteps, 16))
    return cfg, V0, G, u, X, Y


def run_control(args):
    """Adjoint gradient of the 256^2 control problem: gradient evaluations/s
    (forward + adjoint with checkpoints every 50 steps), complex64; finite
    differences of the complex128 forward on seeded components."""
    import torch
    import fgpe_b200 as gp
    torch.cuda.set_device(0)
    cfg64, V0, G, u, X, Y = control_problem(gp.C64)
    # ground state of V0 (complex128 heavy ball), then the dipole target
    cfgg = cfg64.copy()
    cfgg.precision = gp.C128
    s = gp.Solver(cfgg)
    s.set_vext(0, V0)
    dv = cfgg.dx[0] * cfgg.dx[1] * cfgg.dx[2]
    p0 = np.exp(-(X ** 2 + Y ** 2) / 2.0).reshape(V0.shape) + 0j
    s.set_psi(0, p0 / np.sqrt(np.sum(np.abs(p0) ** 2) * dv))
    gs_iters, _ = s.step_imag(0, 4000)
    psi0 = s.get_psi(0)
    s.close()
    target = X.reshape(psi0.shape) * np.abs(psi0)
    target = target / np.sqrt(np.sum(np.abs(target) ** 2) * dv) + 0j
    tuning = {}
    if not args.no_tune:
        cache = os.path.join("/tmp", f"gpe_tune_{os.getpid()}.jsonl")
        for name, cfg in (("c64", cfg64), ("c128", cfgg)):
            tuning[name] = gp.tune(cfg, 0, cache)
        gp.set_tune_cache(cache)
    solvers = {}
    for name, cfg in (("c64", cfg64), ("c128", cfgg)):
        sv = gp.Solver(cfg)
        sv.set_stream(torch.cuda.current_stream().cuda_stream)
        sv.set_vext(0, V0)
        sv.set_psi(0, psi0)
        sv.control_set_basis(G)
        solvers[name] = sv
    s64 = solvers["c64"]
    W = max(1, min(args.warmup, 2))
    for _ in range(W):
        s64.control_gradient(u, target, 50)
    K = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    l0 = s64.launches
    t0 = time.perf_counter()
    for _ in range(K):
        L, grad = s64.control_gradient(u, target, 50)
    wall = (time.perf_counter() - t0) / K
    launches = (s64.launches - l0) // K
    t0 = time.perf_counter()
    s64.control_gradient(u, target, 50, want_grad=False)
    fwd = time.perf_counter() - t0
    # finite differences of the complex128 forward map: the fourth-order
    # central stencil (-L(u+2h) + 8 L(u+h) - 8 L(u-h) + L(u-2h)) / 12h, whose
    # truncation error (h^4) stays far below the 1e-4 bar; the second-order
    # stencil's h^2 L''' term alone reaches ~5e-5 on this nearly degenerate
    # loss (L ~ 1 - 3e-7).  h = 1e-3: at 1e-4 the loss's own rounding (its
    # FP64 reductions over 65536 points, ~1e-13 of L) divided by h already
    # reaches ~1e-4 of the small gradient components
    rng = np.random.default_rng(7)
    h = 1e-3
    s128 = solvers["c128"]
    L128, g128 = s128.control_gradient(u, target, 50)
    errs = []

    def loss_at(n, k, d):
        uu = u.copy()
        uu[n, k] += d
        return s128.control_gradient(uu, target, 50, want_grad=False)[0]

    for _ in range(args.fd_components):
        n, k = rng.integers(u.shape[0]), rng.integers(u.shape[1])
        fd = (-loss_at(n, k, 2 * h) + 8 * loss_at(n, k, h) - 8 * loss_at(n, k, -h) + loss_at(n, k, -2 * h)) / (12 * h)
        errs.append((abs(grad[n, k] - fd), abs(fd), abs(g128[n, k] - fd)))
    gmax = float(np.abs(g128).max())
    big = [e / f for e, f, _ in errs if f > 1e-2 * gmax]
    big128 = [e / f for _, f, e in errs if f > 1e-2 * gmax]
    line = {"metric": "control-gradient evaluations/s, 256^2 x 2000 RK4 steps x 16 controls "
                      "(complex64 + FP64 reductions)",
            "value": round(1.0 / wall, 4), "unit": "gradients/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": round(1e3 * wall, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded controls and lattice; ground state computed in the run)",
            "config": {"workload": "adjoint optimal control", "grid": [256, 256], "rk4_steps": int(u.shape[0]),
                       "controls": 16, "checkpoint_every": 50, "dt": 1e-3, "g": 200.0},
            "loss_c64": L, "loss_c128": L128, "forward_only_s": round(fwd, 4),
            "gradient_s": round(wall, 4), "rk4_step_equivalents_per_s": round(u.shape[0] / wall, 1),
            "grad_rel_l2_c64_vs_c128": float(np.linalg.norm(grad - g128) / np.linalg.norm(g128)),
            "fd": {"components": len(errs), "h": h, "fd_of": "complex128 forward", "stencil": "4th-order central",
                   "max_rel_err_components_above_1pct_of_max": max(big) if big else None,
                   "max_abs_err_over_max_grad": max(e for e, _, _ in errs) / gmax,
                   "complex128_adjoint_max_rel_err": max(big128) if big128 else None},
            "ground_state_iterations": int(gs_iters), "gpu_launches_per_gradient": int(launches),
            "tuning": tuning or "off (--no-tune): default pass variants"}
    for sv in solvers.values():
        sv.close()
    if not args.quick:
        line["cpu_baseline"] = control_cpu_leg(cfgg, V0, G, psi0, target, u, grad, g128)
    print(json.dumps(line))


def control_cpu_leg(cfg, V0, G, psi0, target, u, grad64, grad128):
    """CPU leg of the control workload: the FP64 numpy restatement of the
    controlled RK4 step and its discrete adjoint (oracle/adjoint_oracle.py),
    timed for one full gradient (2000 steps x 16 controls at 256^2), and, as
    the checker, both GPU gradients against it."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import adjoint_oracle as ad
    o = ad.ControlProblem(cfg, V0, G, psi0, target)
    t0 = time.perf_counter()
    Lo, go = o.gradient(u)
    dt = time.perf_counter() - t0
    nrm = float(np.linalg.norm(go))
    gmax = float(np.abs(go).max())
    big = np.abs(go) > 1e-2 * gmax
    return {"value": round(1.0 / dt, 5), "unit": "gradients/s", "cores": 1, "kind": "port",
            "sample": "one full gradient in FP64 numpy (oracle/adjoint_oracle.py)", "loss": float(Lo),
            "parity_vs_port": {"grad_rel_l2_c128": float(np.linalg.norm(grad128 - go) / nrm),
                               "grad_rel_l2_c64": float(np.linalg.norm(grad64 - go) / nrm),
                               "max_rel_err_c64_components_above_1pct_of_max":
                                   float(np.max(np.abs(grad64 - go)[big] / np.abs(go)[big]))}}


def imag_case(name, precision, scheme):
    """Imaginary-time cases: 'ground64' (64^3 on [-8,8]^3, V = r^2/2, g = 500,
    norm 1, dt = 1e-3, stop at |dmu| < 1e-9 or 2000 steps), 'dipolar'
    (128x128x64 on [-12,12]^2 x [-6,6], omega = (1,1,3), g = 1000, dipoles
    along z with eps_dd = 0.8 and a spherical cut-off R = 6, dt = 5e-4, stop at
    |dmu| < 1e-8) and 'twocomp' (96^3, g11 = 1000, g22 = 950, g12 = 900, norms
    0.5 each, identical traps, dt = 5e-4); Gaussian starts with seeded 1e-3
    complex noise."""
    import fgpe_b200 as gp
    prms = np.zeros(32)
    if name == "ground64":
        shape, xm, w, dt, eps, ncomp, ham = (64, 64, 64), (8.0, 8.0, 8.0), (1.0, 1.0, 1.0), 1e-3, 1e-9, 1, gp.HAM_BEC
        prms[0:3] = 500.0 / (4 * PI_REF)
        npart = (1.0, 1.0)
    elif name == "dipolar":
        shape, xm, w, dt, eps, ncomp, ham = (128, 128, 64), (12.0, 12.0, 6.0), (1.0, 1.0, 3.0), 5e-4, 1e-8, 1, \
            gp.HAM_DIPOLAR
        a = 1000.0 / (4 * PI_REF)
        prms[0:3] = a
        prms[6] = 0.8 * a
        prms[7:10] = [0.0, 0.0, 1.0]
        prms[10] = 6.0
        npart = (1.0, 1.0)
    else:
        shape, xm, w, dt, eps, ncomp, ham = (96, 96, 96), (8.0, 8.0, 8.0), (1.0, 1.0, 1.0), 5e-4, 1e-8, 2, \
            gp.HAM_BEC2
        prms[0:3] = [1000.0 / (4 * PI_REF), 950.0 / (4 * PI_REF), 900.0 / (4 * PI_REF)]
        npart = (0.5, 0.5)
    cfg = gp.make_config(shape, xm, dt=dt, precision=precision, prms=prms, hamiltonian=ham, ncomp=ncomp,
                         imag_scheme=scheme, beta=0.9, npart=npart, epsilon_e=eps)
    x, y, z = gp.grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    V = 0.5 * ((w[0] * X) ** 2 + (w[1] * Y) ** 2 + (w[2] * Z) ** 2) + 0j
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    psis = []
    for c in range(ncomp):
        rng = np.random.default_rng(1 + c)
        g = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 2.0)
        p = g * (1 + 1e-3 * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)))
        psis.append(p * np.sqrt(npart[c] / (np.sum(np.abs(p) ** 2) * dv)))
    return cfg, V, psis


def run_imag(args):
    """Imaginary-time iterations/s of the three imaginary-time cases in each
    form, timed with CUDA events over a bounded number of iterations, and the
    iterations to convergence (capped) with the final mu and E."""
    import torch
    import fgpe_b200 as gp
    torch.cuda.set_device(0)
    st = torch.cuda.current_stream()
    out = {"metric": "imaginary-time iterations/s", "unit": "iterations/s", "n_gpus": 1, "cases": {}}
    forms = [("c128_heavyball", gp.C128, gp.IMAG_HEAVYBALL), ("c128_rk4", gp.C128, gp.IMAG_RK4),
             ("c64_rk4", gp.C64, gp.IMAG_RK4)]
    cache = os.path.join("/tmp", f"gpe_tune_{os.getpid()}.jsonl")
    if not args.no_tune:
        gp.set_tune_cache(cache)
    for name in ("ground64", "dipolar", "twocomp"):
        res = {}
        for form, prec, scheme in forms:
            cfg, V, psis = imag_case(name, prec, scheme)
            tuned = None if args.no_tune else gp.tune(cfg, 1, cache)
            s = gp.Solver(cfg)
            s.set_stream(st.cuda_stream)
            for c in range(cfg.ncomp):
                s.set_vext(c, V)
                s.set_psi(c, psis[c])
            s.step_imag(0, 3)
            K = 200
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            done, _ = s.step_imag(3, K)
            e1.record(st)
            torch.cuda.synchronize()
            ips = done / (e0.elapsed_time(e1) / 1e3)
            total, conv = 3 + done, False
            cap = 2000 if name == "ground64" else 20000
            while total < cap and not conv:
                d, conv = s.step_imag(total, min(2000, cap - total))
                total += d
            st8 = s.imag_state()
            res[form] = {"iterations_per_s": round(ips, 1), "converged": bool(conv), "iterations": int(total),
                         "tuning": tuned,
                         "mu": [float(st8[4 * c + 1]) for c in range(cfg.ncomp)],
                         "E": [float(st8[4 * c + 2]) for c in range(cfg.ncomp)]}
            s.close()
        for form in ("c128_rk4", "c64_rk4"):
            if res[form]["converged"] and res["c128_rk4"]["converged"]:
                res[form]["E_rel_vs_c128_converged"] = float(abs(res[form]["E"][0] / res["c128_rk4"]["E"][0] - 1))
                res[form]["mu_rel_vs_c128_converged"] = float(abs(res[form]["mu"][0] / res["c128_rk4"]["mu"][0] - 1))
        res["cpu_baseline"] = imag_cpu_leg(name, st)
        if name == "ground64":
            # the drop-in comparison: the reference's own build, heavy ball at 64^3
            rb = reference_cuda_build(64, imag=True)
            if "steps_per_s" in rb:
                rb["c128_heavyball_over_reference_build"] = round(
                    res["c128_heavyball"]["iterations_per_s"] / rb["steps_per_s"], 3)
            res["reference_cuda_build"] = rb
        out["cases"][name] = res
    print(json.dumps(out))


def imag_cpu_leg(name, st, budget_s=8.0):
    """CPU leg of an imaginary-time case: the FP64 oracle port timed over a
    bounded number of RK4 imaginary-time iterations from the case's start,
    and, as the checker, both GPU forms over the same iterations (psi, E, mu
    relative errors and the norm after renormalisation)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    import fgpe_b200 as gp
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    cfg, V, psis = imag_case(name, gp.C128, gp.IMAG_RK4)
    o = orc.OracleSolver(cfg)
    for c in range(cfg.ncomp):
        o.set_vext(c, V)
        o.set_psi(c, psis[c])
    t0 = time.perf_counter()
    o.step_imag(0, 1)
    one = time.perf_counter() - t0
    k = max(1, min(50, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    o.step_imag(1, k)
    dt = time.perf_counter() - t0
    so = o.imag_state()
    po = [o.get_psi(c) for c in range(cfg.ncomp)]
    o.close()
    out = {"value": round(k / dt, 4), "unit": "iterations/s", "cores": threads, "kind": "port",
           "sample": f"{k + 1} RK4 imaginary-time iterations of the case in FP64 (oracle/gpe_oracle.cpp); {k} timed"}
    par = {"iterations": k + 1}
    for form, prec in (("c128_rk4", gp.C128), ("c64_rk4", gp.C64)):
        cfg2, V2, psis2 = imag_case(name, prec, gp.IMAG_RK4)
        s = gp.Solver(cfg2)
        s.set_stream(st.cuda_stream)
        for c in range(cfg2.ncomp):
            s.set_vext(c, V2)
            s.set_psi(c, psis2[c])
        s.step_imag(0, k + 1)
        sg = s.imag_state()
        e = {"psi_rel_l2": [float(np.linalg.norm(s.get_psi(c) - po[c]) / np.linalg.norm(po[c]))
                            for c in range(cfg2.ncomp)],
             "E_rel_err": [float(abs(sg[4 * c + 2] / so[4 * c + 2] - 1)) for c in range(cfg2.ncomp)],
             "mu_rel_err": [float(abs(sg[4 * c + 1] / so[4 * c + 1] - 1)) for c in range(cfg2.ncomp)]}
        obs = s.observables(0.0)
        e["norm_rel_err"] = [float(abs(obs[3 * c] / cfg2.npart[c] - 1)) for c in range(cfg2.ncomp)]
        s.close()
        par[form] = e
    out["parity_vs_port"] = par
    return out


def main():
    args = parse()
    if args.workload == "imag3d":
        run_imag(args)
        return
    if args.workload == "control2d":
        run_control(args)
        return
    if args.workload == "sweep2d":
        run_sweep(args)
        return
    if args.cufft:
        run_cufft(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
