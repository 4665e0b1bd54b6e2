#!/usr/bin/env python3
"""Benchmark of the B200 time step (grid-point-steps/s).

Default workload: the mixed-precision single run, Nx=Ny=512, 12 subdomains x 33
GLL points (nz=396), Re=5000, A=0.1, noise 1e-3, dt=2.5e-4 (FP32 fields, FFTs,
products and filters; FP64 band solves, mean mode and projection).  The same
steps are also run with the plain FP64 path on the same input to report the
mixed/FP64 speed ratio and the mixed path's field error against FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config C3|C2|C0] [--precision mixed|fp64]

N>1 (torchrun): independent replicas, one per GPU (the step does not shard),
value = all ranks' grid-point-steps / max-over-ranks time.
--impl reference: the CPU restatement of the reference step (all host
threads) on a bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from iwrepo_b200 import config as cf  # noqa: E402

METRIC = "grid-pt-steps/s, mixed+batched vs plain FP64 on 1 B200 at <=1e-5 rel L2 err"
UNIT = "grid-pt-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="C3")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the C1 and C4 keys of the default line")
    # smaller horizontal grid with the same vertical grid and physics, for
    # profiling the same kernels on a case that fits a profiler's replay
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--ny", type=int, default=None)
    # C3 mixed against C3 FP64 over this many steps: field, kinetic-energy and
    # noise growth-rate errors (a report, not a bench line)
    ap.add_argument("--error-report", type=int, default=0)
    # interface averaging every N steps (the workloads' default is 1; 0 turns it off)
    ap.add_argument("--navg", type=int, default=None)
    return ap.parse_args()


def workload_cfg(name: str, precision: str, nx=None, ny=None, navg=None):
    prec = cf.IW_PREC_MIXED if precision == "mixed" else cf.IW_PREC_FP64
    kw = {k: v for k, v in (("nx", nx), ("ny", ny)) if v}
    if navg is not None:
        kw["navgintrfc"] = navg
    return cf.baseline(name, precision=prec, **kw)


def _base_xy(name):
    b = cf.baseline(name)
    return (b.nx, b.ny)


def describe(cfg, precision):
    amp, noise = cf.BASELINE_IC.get(cfg.name, (0.05, 1e-4))
    return {
        "workload": f"{cfg.name}{'' if (cfg.nx, cfg.ny) == _base_xy(cfg.name) else ' vertical grid and physics'}: "
                    f"{cfg.nx}x{cfg.ny}x({cfg.nsubd}x{cfg.nzloc}={cfg.nz}) Boussinesq step, "
                    f"Re={1 / cfg.xnu:.0f}, A={amp}, noise={noise}, dt={cfg.dt}, "
                    f"{'FP32 fields + FP64 solves' if precision == 'mixed' else 'plain FP64'}",
        "nx": cfg.nx, "ny": cfg.ny, "nz": cfg.nz, "nsubd": cfg.nsubd, "nzloc": cfg.nzloc,
        "grid_points": cfg.grid_points, "bc": "no-slip bottom / free-slip top",
        "filter": "exponential order 8, amp 36, every step",
        "l2": (f"no flush: every launch streams more than the 126 MB L2 (one field is "
               f"{cfg.ntot * (4 if precision == 'mixed' else 8) / 1e6:.0f} MB; the smallest launch moves "
               f"2 fields plus its solver tables)"),
        "parallelism": "replicas (no sharding)",
    }


# ----------------------------------------------------------------------
# clocks sampled during the timed region
class Clocks:
    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------
CPU_SAMPLE_XY = 32
# the CPU legs start with the three start-up steps (Euler, BDF2, BDF3: each
# builds new tables) and then time at least 5 steady steps
CPU_WARMUP, CPU_STEPS = 3, 5


def cpu_sample_cfg(cfg):
    """Bounded sample of the workload for the CPU restatement: the same
    vertical structure, physics and dt on a 32x32 horizontal grid."""
    return cfg.replace(nx=CPU_SAMPLE_XY, ny=CPU_SAMPLE_XY, precision=cf.IW_PREC_FP64)


def host_cpu():
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "logical_cpus": os.cpu_count()}


def cpu_rate(cfg, threads: int, warm: int, steps: int, faithful: bool):
    import oracle
    oracle.set_threads(threads)
    s = cpu_sample_cfg(cfg)
    amp, noise = cf.BASELINE_IC.get(cfg.name, (0.05, 1e-4))
    o = oracle.Oracle(s, cache=not faithful)
    o.init_mode1(amp, noise, 1234)
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return s.grid_points * steps / dt, s, dt


def cpu_sample_note(s, cfg, warm, steps, threads):
    return {"nx": s.nx, "ny": s.ny, "nz": s.nz, "nsubd": s.nsubd, "nzloc": s.nzloc, "grid_points": s.grid_points,
            "of": f"{cfg.name} {cfg.nx}x{cfg.ny}x({cfg.nsubd}x{cfg.nzloc})", "warmup_steps": warm,
            "timed_steps": steps, "threads": threads, "host": host_cpu(),
            "rule": "grid-pt-steps/s of the sample, reported as is: the per-point work of the faithful "
                    "restatement (per-column penalty assembly and band LU, z operators) does not depend on "
                    "nx, ny; only the FFT share grows, by log2(nx ny)/log2(32*32) = 1.8x at 512^2, so the "
                    "full grid would run somewhat slower per point"}


def run_reference(args, rank, world):
    cfg = workload_cfg(args.config, args.precision, args.nx, args.ny)
    if rank != 0:
        return
    import oracle
    threads = oracle.max_threads()
    steps, warm = CPU_STEPS, CPU_WARMUP
    rate, s, dt = cpu_rate(cfg, threads, warm, steps, faithful=True)
    note = cpu_sample_note(s, cfg, warm, steps, threads)
    sample = (f"{s.nx}x{s.ny}x({s.nsubd}x{s.nzloc}) sample of {cfg.name} (same vertical grid/physics), "
              f"{warm} start-up + {steps} timed steps, faithful (refactor every step), FP64, {threads} threads")
    conf = describe(s, "fp64")
    conf["workload"] = f"CPU sample of {describe(cfg, args.precision)['workload']}: {s.nx}x{s.ny} horizontally"
    conf["sample"] = note
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": conf,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "detail": note},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------
PHASE_FIELDS = {  # algorithmic fields moved per launch (reads + writes of ntot-sized arrays)
    "stageA": 12, "y_inverse": 20, "x_row_nl": 23, "y_forward": 19, "stageE": 40,
    "pressure": 6, "solve_uv": 4, "solve_w": 2, "solve_rho": 2,
}
# kernels launched per step: stage A, y-inverse, x rows, 2 y-forward, wall BC,
# stage E, pressure (2 when ill-conditioned systems get a residual sweep),
# u/v, w, rho, interface averaging (2 gathers, 2 y transforms, rows, planes)
LAUNCHES_PER_STEP = 18


def dram_traffic(cfg, precision, phase):
    """DRAM bytes per launch of `phase` from the committed ncu figures
    (profiles/dram_traffic.json), scaled from the captured workload to this one
    by grid points when they differ; None when no figure exists."""
    try:
        tab = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
    except Exception:
        return None
    ent = tab.get(precision, {}).get(phase)
    if not ent:
        return None
    return ent["bytes_per_launch"] * cfg.ntot / ent["ntot"]


def run_ours(args, rank, world):
    import torch
    import iwrepo_b200 as iw

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as tdist
        import datetime
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    cfg = workload_cfg(args.config, args.precision, args.nx, args.ny)
    amp, noise = cf.BASELINE_IC.get(cfg.name, (0.05, 1e-4))
    seed = 1000 + rank
    s = iw.Solver(cfg, device=dev)
    s.init_mode1(amp, noise, seed)
    tuning = s.autotune()  # launch choices for this device and size (state unchanged)
    ext = torch.cuda.ExternalStream(s.stream())

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    s.step(args.warmup)
    barrier()
    clocks = Clocks(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the NVTX range lets a profiler capture only the timed steps
    # (ncu --nvtx --nvtx-include "timed_steps/")
    torch.cuda.nvtx.range_push("timed_steps")
    e0.record(ext)
    s.step(args.steps)
    e1.record(ext)
    torch.cuda.nvtx.range_pop()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    # per-phase CUDA events from a second pass of the same number of steps,
    # after the timed one, so that the timed steps carry no event records and
    # no per-step host waits
    s.profile(True)
    s.step(args.steps)
    barrier()
    ph = s.profile_read()
    s.profile(False)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cfg.grid_points * args.steps / (ms / 1e3)

    # per-phase device time of the timed steps -> dominant kernel
    elem = 4 if args.precision == "mixed" else 8
    fb = cfg.ntot * elem
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    phases = {}
    for k, (t_ms, n) in ph.items():
        if n:
            avg = t_ms / n
            nb = PHASE_FIELDS.get(k)
            phases[k] = {"ms": avg, "gbs": (nb * fb / (avg / 1e3) / 1e9) if nb else None}
    dom = max((k for k in phases if PHASE_FIELDS.get(k)), key=lambda k: phases[k]["ms"])
    dom_gbs = phases[dom]["gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": dom_gbs, "peak": hbm, "unit": "GB/s",
                "frac": dom_gbs / hbm, "traffic": dram_traffic(cfg, args.precision, dom),
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_launch": PHASE_FIELDS[dom] * fb}
    b_alg = 28 * elem * (cfg.nx + 2) / cfg.nx
    step_frac = (value / world) * b_alg / (hbm * 1e9)

    line = {}
    if rank == 0:
        # e2e through the public API, a restart-style run: the 5 time levels
        # the timed steps left are downloaded into pinned host buffers; the
        # timed region uploads them with their step count (steady-state
        # coefficients, so no table rebuild), runs K steps each reading the
        # mean profiles back, and downloads level 0 into a pinned buffer
        d0 = s.diag()
        shape = s.shape
        pin = lambda: torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(shape)
        levels = [s.state(lev, out=pin()) for lev in range(5)]
        out = pin()
        prof_host = torch.empty(4 * cfg.nz, dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_state(*levels, t=d0["t"], istep=d0["istep"])
        t1 = time.perf_counter()
        for k in range(args.steps):
            s.step(1)
            s.mean_profiles(prof_host)  # per-step device -> host result (waits for the step)
        t2 = time.perf_counter()
        s.state(0, out=out)
        t3 = time.perf_counter()
        del levels
        e2e_s = t3 - t0
        e2e_val = cfg.grid_points * args.steps / e2e_s
        state_bytes = 4 * cfg.ntot * 8
        line_e2e = {"value": world * e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(5 * state_bytes / args.steps),
                    "d2h_bytes_per_step": int(state_bytes / args.steps) + 4 * cfg.nz * 8,
                    "breakdown_ms": {"h2d_upload_5_levels": 1e3 * (t1 - t0), "steps_with_profile_reads": 1e3 * (t2 - t1),
                                     "d2h_download": 1e3 * (t3 - t2), "table_build": 0.0},
                    "note": "restart-style run through the C ABI (host wall clock): FP64 state upload of 5 levels "
                            "from pinned host memory with the step count it came from (no table rebuild), K steps "
                            "each reading the mean profiles back, download of level 0 into pinned host memory"}

        fp64 = None
        err = None
        if args.precision == "mixed" and not args.no_fp64_compare:
            s.close()
            del s
            torch.cuda.empty_cache()
            c64 = cfg.replace(precision=cf.IW_PREC_FP64)
            r64 = iw.Solver(c64, device=dev)
            r64.init_mode1(amp, noise, seed)
            r64.step(args.warmup)
            ext64 = torch.cuda.ExternalStream(r64.stream())
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(ext64)
            r64.step(args.steps)
            a1.record(ext64)
            torch.cuda.synchronize()
            ms64 = a0.elapsed_time(a1)
            fp64 = cfg.grid_points * args.steps / (ms64 / 1e3)
            # same initial condition and step count for the error
            xs = out
            r64b = r64
            ref = r64b.state(0)
            # mixed ran warmup + steps (+ profiled) steps; compare fresh runs instead
            r64.close()
            del r64
            sm = iw.Solver(cfg, device=dev)
            sm.init_mode1(amp, noise, seed)
            nerr = args.warmup + args.steps
            sm.step(nerr)
            a = sm.state(0)
            sm.close()
            r2 = iw.Solver(c64, device=dev)
            r2.init_mode1(amp, noise, seed)
            r2.step(nerr)
            b = r2.state(0)
            r2.close()
            err = {f: float(np.linalg.norm(a[q] - b[q]) / max(np.linalg.norm(b[q]), 1e-300))
                   for q, f in enumerate("uvwr")}
            err["steps"] = nerr
            del xs, ref

        cpu = None
        if not args.no_cpu:
            try:
                rate, smp, dt = cpu_rate(cfg, 1, CPU_WARMUP, CPU_STEPS, faithful=True)
                cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                       "sample": f"{smp.nx}x{smp.ny}x({smp.nsubd}x{smp.nzloc}) sample of {cfg.name}, "
                                 f"{CPU_WARMUP} start-up + {CPU_STEPS} timed steps, single thread, faithful FP64 "
                                 f"({dt:.1f} s)",
                       "detail": cpu_sample_note(smp, cfg, CPU_WARMUP, CPU_STEPS, 1)}
            except Exception as e:  # the baseline is reported, never required
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "sample": f"failed: {e}"}

        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fields/FFTs + f64 solves" if args.precision == "mixed" else "f64",
            "data": "synthetic (mode-1 wave + seeded noise)",
            "config": dict(describe(cfg, args.precision), tuning=tuning),
            "e2e": line_e2e, "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "roofline": roofline, "step_roofline_frac": step_frac, "phases": phases,
            "cpu_baseline": cpu, "clocks": clk,
        }
        if fp64 is not None:
            line["fp64_value"] = fp64
            line["mixed_over_fp64"] = value / world / fp64
            line["mixed_rel_l2_vs_fp64"] = err
        if not args.no_extra and world == 1 and args.config == "C3" and not (args.nx or args.ny):
            # the other two batched workloads of the metric, reported beside the headline
            import types
            try:
                c1 = run_c1(types.SimpleNamespace(steps=5, warmup=2), emit=False)
                line["c1_isolated_solves"] = {"solves_per_s": c1["rates_solves_per_s"],
                                              "ms_per_batch": c1["ms_per_batch"],
                                              "fp32_refined_vs_fp64_rel_l2": c1["fp32_refined_vs_fp64_rel_l2"]}
            except Exception as e:  # reported, never required
                line["c1_isolated_solves"] = {"failed": str(e)}
            try:
                c4 = run_c4(types.SimpleNamespace(steps=6, warmup=4), emit=False)
                line["c4_ensemble"] = {k: c4[k] for k in ("value", "ms_per_step", "steps", "warmup",
                                                            "fp64_sequential_value",
                                                            "batched_mixed_over_sequential_fp64")}
                line["c4_ensemble"]["workload"] = c4["config"]["workload"]
            except Exception as e:
                line["c4_ensemble"] = {"failed": str(e)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_c4(args, emit=True):
    """C4: 48 independent runs of uneven sizes, mixed precision, advanced
    together (one CUDA-graph launch per ensemble step once every member is in
    steady state), against the same members run one by one in plain FP64."""
    import torch
    import iwrepo_b200 as iw

    torch.cuda.set_device(0)
    members = cf.ensemble_members(48)
    pts = sum(m.grid_points for m in members)
    ens = []
    for m in members:
        s = iw.Solver(m.replace(precision=cf.IW_PREC_MIXED), device=0)
        s.init_mode1(m.member_amp, 1e-4, m.member_seed)
        ens.append(s)
    iw.ensemble_run(ens, args.warmup)
    torch.cuda.synchronize()
    ext = torch.cuda.ExternalStream(ens[0].stream())
    clocks = Clocks(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    iw.ensemble_run(ens, args.steps)  # ends with every member stream after the graph launches
    e1.record(ext)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    value = pts * args.steps / (ms / 1e3)
    for s in ens:
        s.close()
    del ens
    torch.cuda.empty_cache()
    # baseline: the members one by one, plain FP64, eager
    seq_ms = 0.0
    for m in members:
        s = iw.Solver(m.replace(precision=cf.IW_PREC_FP64), device=0)
        s.init_mode1(m.member_amp, 1e-4, m.member_seed)
        s.step(args.warmup)
        torch.cuda.synchronize()
        x = torch.cuda.ExternalStream(s.stream())
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(x)
        s.step(args.steps)
        a1.record(x)
        torch.cuda.synchronize()
        seq_ms += a0.elapsed_time(a1)
        s.close()
    seq = pts * args.steps / (seq_ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 fields/FFTs + f64 solves", "data": "synthetic (mode-1 waves + seeded noise, 48 members)",
        "config": {"workload": "C4: 48-member ensemble, Nx=Ny in {64,96,128,192}, 3-8 subdomains of 17-25 points, "
                               "Re in [1000,5000], A in [0.01,0.1], one CUDA-graph launch per ensemble step",
                   "members": len(members), "grid_points_total": pts,
                   "l2": "the ensemble state (several GB) exceeds L2; no flush needed"},
        "gpu_launches": args.steps, "clocks": clk,
        "fp64_sequential_value": seq, "batched_mixed_over_sequential_fp64": value / seq,
        "note": "gpu_launches counts graph launches; each replays every member's step kernels",
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_c1(args, emit=True):
    """C1: 256 x 129 isolated penalty-Helmholtz columns over 8 x 25 GLL points,
    lambda = kx^2 + ky^2 + 11/(6 dt), dt = 1e-3, seeded N(0,1) complex RHS.
    FP64 factor + solve (first call), FP64 solve with cached factors, and FP32
    solve + one FP64 residual sweep (iw_helm_solve_batched modes 0 and 1)."""
    import torch
    import iwrepo_b200 as iw

    torch.cuda.set_device(0)
    cfg = cf.Config(nx=256, ny=256, nzloc=25, nsubd=8, dt=1e-3, xnu=1.0, xkappa=1.0,
                    precision=cf.IW_PREC_FP64, name="C1").validate()
    s = iw.Solver(cfg, device=0)
    kx = np.arange(cfg.nx // 2 + 1)
    ky = np.fft.fftfreq(cfg.ny, 1.0 / cfg.ny)
    lam = (kx[None, :] ** 2 + ky[:, None] ** 2).ravel() + 11.0 / (6 * cfg.dt)
    ncol = lam.size
    rng = np.random.default_rng(2024)
    rhs = torch.tensor(rng.standard_normal((ncol, cfg.nz, 2)), dtype=torch.float64, device="cuda")
    dl = torch.tensor(lam, dtype=torch.float64, device="cuda")
    out = {m: torch.zeros_like(rhs) for m in (0, 1)}
    ext = torch.cuda.ExternalStream(s.stream())

    def timed(mode, reps):
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(ext)
        for _ in range(reps):
            iw.helm_solve_batched(s, dl.data_ptr(), ncol, 0, 1, rhs.data_ptr(), out[mode].data_ptr(), mode)
        a1.record(ext)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / reps

    t_fact = timed(0, 1)  # builds and caches the factors of the distinct lambdas
    for _ in range(args.warmup):
        timed(0, 1)
        timed(1, 1)
    t64 = timed(0, max(args.steps, 1))
    t32 = timed(1, max(args.steps, 1))
    x0, x1 = out[0].cpu().numpy(), out[1].cpu().numpy()
    per_col = np.linalg.norm((x1 - x0).reshape(ncol, -1), axis=1) / np.linalg.norm(x0.reshape(ncol, -1), axis=1)
    b_alg = 2 * cfg.nz * 16  # complex RHS in + solution out
    peak = 6553.0
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        pass
    rates = {"fp64_factor_and_solve": ncol / (t_fact / 1e3), "fp64_solve": ncol / (t64 / 1e3),
             "fp32_solve_fp64_refine": ncol / (t32 / 1e3)}
    line = {
        "metric": "solves/s", "value": rates["fp32_solve_fp64_refine"], "unit": "solves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "data": "synthetic (seeded N(0,1) RHS)",
        "config": {"workload": "C1: 33,024 penalty-Helmholtz systems (kx 0..128 x ky 256), nz = 8 x 25, "
                               "lambda = k^2 + 11/(6 dt), dt = 1e-3, u-type BCs (Dirichlet bottom, Neumann top)",
                   "distinct_systems": int(np.unique(lam).size)},
        "rates_solves_per_s": rates,
        "ms_per_batch": {"fp64_factor_and_solve": t_fact, "fp64_solve": t64, "fp32_solve_fp64_refine": t32},
        "fp32_refined_vs_fp64_rel_l2": {"max_over_columns": float(per_col.max()), "median": float(np.median(per_col))},
        "hbm_roofline_frac_rhs_and_solution": {k: v * b_alg / (peak * 1e9) for k, v in rates.items()},
        "note": "relative residuals are checked in tests/test_gpu_parity.py::test_helm_batched_modes "
                "(<1e-11 FP64, <1e-7 FP32 + refinement)",
    }
    if emit:
        print(json.dumps(line), flush=True)
    s.close()
    return line


def run_error_report(args):
    """C3 mixed vs C3 FP64 from the same seeded state for args.error_report
    steps: final relative L2 per field and for the velocity vector, the largest
    relative KE difference over the run, and the growth rate of the rms of w
    in the bottom 20 % of the depth (the seeded noise) in each precision."""
    import iwrepo_b200 as iw

    base = workload_cfg(args.config, "mixed", args.nx, args.ny, args.navg)
    amp, noise = cf.BASELINE_IC.get(base.name, (0.05, 1e-4))
    runs = {"mixed": iw.Solver(base, device=0), "fp64": iw.Solver(base.replace(precision=cf.IW_PREC_FP64), device=0)}
    for r in runs.values():
        r.init_mode1(amp, noise, 1000)
    # the flow's own sensitivity: FP64 from the mixed run's initial state, i.e.
    # the FP64 initial state rounded to FP32 and nothing else changed
    st0 = runs["mixed"].state(0)
    runs["fp64_from_rounded_start"] = iw.Solver(base.replace(precision=cf.IW_PREC_FP64), device=0)
    z = np.zeros_like(st0)
    runs["fp64_from_rounded_start"].set_state(st0, z, z, z, z, t=0.0, istep=0)
    del st0, z
    hist = {k: [] for k in runs}
    every = 10
    for k in range(0, args.error_report, every):
        for name, r in runs.items():
            r.run(min(every, args.error_report - k), graph=True)
            d = r.diag()
            hist[name].append((d["t"], d["ke"], d["wrms_bottom"]))
    a, b = runs["mixed"].state(0), runs["fp64"].state(0)
    c = runs["fp64_from_rounded_start"].state(0)
    err = {f: float(np.linalg.norm(a[q] - b[q]) / np.linalg.norm(b[q])) for q, f in enumerate("uvwr")}
    err["velocity"] = float(np.linalg.norm(a[:3] - b[:3]) / np.linalg.norm(b[:3]))
    sens = {f: float(np.linalg.norm(c[q] - b[q]) / np.linalg.norm(b[q])) for q, f in enumerate("uvwr")}
    sens["velocity"] = float(np.linalg.norm(c[:3] - b[:3]) / np.linalg.norm(b[:3]))
    del c
    hm, hd = np.array(hist["mixed"]), np.array(hist["fp64"])
    ke_err = float(np.max(np.abs(hm[:, 1] - hd[:, 1]) / np.abs(hd[:, 1])))

    def rate(h):  # least-squares slope of log(w rms) over the second half of the run
        n2 = len(h) // 2
        return float(np.polyfit(h[n2:, 0], np.log(h[n2:, 2]), 1)[0])

    gm, gd = rate(hm), rate(hd)
    line = {"report": "mixed vs fp64", "workload": describe(base, "mixed")["workload"], "steps": args.error_report,
            "navgintrfc": base.navgintrfc,
            "field_rel_l2": err, "ke_max_rel_diff": ke_err,
            "fp64_from_fp32_rounded_start_rel_l2": sens,
            "noise_growth_rate": {"mixed": gm, "fp64": gd, "rel_diff": abs(gm - gd) / abs(gd)},
            "samples_every_steps": every}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.error_report > 0:
        run_error_report(args)
        return
    if args.config == "C4" and args.impl == "ours":
        run_c4(args)
        return
    if args.config == "C1" and args.impl == "ours":
        run_c1(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.impl == "ours" else 1)))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world != args.gpus and "RANK" not in os.environ:
        world = 1
    run_ours(args, rank, world)


if __name__ == "__main__":
    main()
