"""Zone-updates/s of the GAMERA step on B200.

Workload: the 3D MHD blast wave on the warped non-orthogonal grid -- 256^3 active cells on
[-0.5,0.5]^3, corners mapped by x' = x + 0.04 sin(2 pi y) sin(2 pi z) (cyclic), rho=1, p=0.1 with
p=10 inside r<0.1, B=(1,1,0)/sqrt(2), gamma=5/3, zero-gradient (outflow) boundaries, CFL 0.3.
Grid metrics and the initial state are built on the device (Corners2Grid + 12^3-point Gauss ICs).

A step is one full stepGamera (predictor, E field/CT, fluxes, update, CalcDT, BCs); one zone-update is
one active cell advanced by one step. The state (~2.5 GB per buffer) is far larger than the 126 MB L2,
so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--prec fp64|fp32flux] [--impl ours|reference]

Under torchrun every rank advances its own replica (weak scaling); value = all ranks' zone-updates /
the slowest rank's device time. `--impl reference` times the CPU oracle (the reference restated in
C++, OpenMP on all host cores; the Fortran reference cannot be compiled on this image) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200: FP32-flux & learned-closure vs plain FP64, matched L1"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
FP64_NOMINAL_TFLOPS = 37.0   # B200 datasheet FP64 (non-tensor); no measured FP64 peak on this pool


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=256, help="active cells per side")
    ap.add_argument("--prec", default="fp64", choices=["fp64", "fp32flux"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--fp32-steps", type=int, default=200,
                    help="steps of the FP32-flux vs FP64 comparison (the configuration's 200)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the FP32-flux and closure side measurements (run on 1 GPU only)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(n, prec, extra=None):
    cfg = {"workload": f"3D MHD blast wave, warped grid, {n}^3, zero-gradient BCs, {prec}",
           "cells": [n, n, n], "ghosts": 4, "grid": "x'=x+0.04 sin(2 pi y) sin(2 pi z) cyclic",
           "ic": "rho=1 p=0.1 (p=10 r<0.1) B=(1,1,0)/sqrt(2)", "CFL": 0.3, "recon": "8CENT+PDM pdmb=0.75",
           "l2": "inputs larger than L2 (state ~2.5 GB/buffer), no flush"}
    if extra:
        cfg.update(extra)
    return cfg


def model_for(n):
    from kaiju_b200 import gamera as gm
    return gm.Model(n, n, n, CFL=0.3, tFin=1.0e30, bc=(gm.GAM_BC_ZEROGRAD,) * 6)


class ClockSampler:
    """nvidia-smi clocks every 50 ms with timestamps; started before the warm-up so that it is sampling when
    the timed region starts, and summarised over the samples inside that region (window())."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"kaiju_b200_clocks_rank{index}_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def window(self, t0, t1):
        """wall-clock bounds (time.time()) of the timed region"""
        self.t0, self.t1 = t0, t1

    def summary(self):
        import datetime
        try:
            rows = [[x.strip() for x in r.split(",")] for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None

        def stamp(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except Exception:
                return None
        t0, t1 = getattr(self, "t0", None), getattr(self, "t1", None)
        inside = [r for r in rows if t0 is not None and stamp(r) is not None and t0 - 0.05 <= stamp(r) <= t1 + 0.05]
        if inside:
            rows = inside
        if not rows:
            return None
        num = lambda x: x.replace(".", "").isdigit()
        sm = [float(r[2]) for r in rows if len(r) > 2 and num(r[2])]
        mx = [float(r[3]) for r in rows if len(r) > 3 and num(r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if len(r) > 6 + q and r[6 + q] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "in_timed_region": bool(inside)}


def traffic_per_unit(kernel, prec):
    """DRAM bytes per interface/edge of a kernel from the committed ncu summary (profiles/), or None."""
    try:
        for line in open(os.path.join(ROOT, "profiles", "roofline_traffic.txt")):
            f = line.split()
            if len(f) >= 3 and not line.startswith("#") and f[0] == kernel and f[1] == prec:
                return float(f[2])
    except OSError:
        pass
    return None


def peaks():
    try:
        return json.load(open(PEAKS_PATH)), "measured"
    except Exception:
        return {"hbm_gbs": FALLBACK_HBM_GBS}, "fallback"


# Algorithmic bytes and flops of the flux kernel (one launch = all interfaces of one direction).
# Per interface it must read once: half-state primitives (5) and B (3), state-n primitives (5) and
# B (3) for the limiter, the volume (1), the face triad (9), the area (1) and the half-state normal
# flux (1) = 28 doubles, and write 5 gas + 3 magnetic fluxes = 8 doubles: 36 doubles = 288 B.
FLUX_BYTES_PER_IFACE = 36 * 8
# FP32-flux path: the same 28 inputs as floats (112 B) and the 8 area-scaled fluxes written as floats
# (32 B) = 144 B.
FLUX_BYTES_PER_IFACE_F32 = 28 * 4 + 8 * 4
FLUX_FLOPS_PER_IFACE = 700.0
# Whole-step compulsory traffic per zone-update on a curvilinear grid, FP64: state n and n-1 in,
# n+1 out (24 doubles) + metrics (volume 1, face 3, edge 3, Tf 27, Te 27, Teb 12, xfc 9, xyzcc 3,
# di/dj/dk 3 = 88 doubles) = 112 doubles = 896 B.
STEP_BYTES_PER_ZONE = 896


def run_ours(args, rank, world, local):
    import torch
    from kaiju_b200 import build as kb, gamera as gm
    kb.build()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    n = args.n
    model = model_for(n)
    xyz = gm.corners_warped(model, (-0.5, 0.5) * 3, 0.04)
    g = gm.GameraGPU.from_corners(model, xyz, "BW")
    if args.prec == "fp32flux":
        g.set_precision(gm.GAM_FP32FLUX)
    zones = n * n * n
    with ClockSampler(local) as clk:
        # warm-up (also builds the two step graphs)
        g.run_steps(max(args.warmup, 3), check=False)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        launches0 = g.status()["kernelLaunches"]
        t0 = time.time()
        ms, rc = g.run_steps_timed(args.steps)
        torch.cuda.synchronize()
        clk.window(t0, time.time())
    # the library's own count of the kernels its step graphs launched in the timed region
    timed_launches = g.status()["kernelLaunches"] - launches0
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    st = g.status()
    value = world * zones * args.steps / (ms / 1e3)

    # per-phase device times (eager launches, CUDA events on the library stream)
    ph = g.profile_phases(2)
    # end to end through the C ABI with host buffers: per step, State and oState in from pinned host
    # memory, one stepGamera, State out
    shapes = gm.array_shapes(model)
    pin = {}
    for nm in ("gas", "magflux", "ogas", "omagflux", "bxyz"):
        tt = torch.empty(int(np.prod(shapes[nm])), dtype=torch.float64, pin_memory=True)
        pin[nm] = tt.numpy().reshape(shapes[nm], order="F")
    g.sync_to_host(gas=pin["gas"], magflux=pin["magflux"], bxyz=pin["bxyz"], ogas=pin["ogas"],
                   omagflux=pin["omagflux"])
    s0 = g.status()
    ke = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        g.sync_to_device(gas=pin["gas"], magflux=pin["magflux"], ogas=pin["ogas"], omagflux=pin["omagflux"],
                         time=s0["time"], otime=s0["otime"])
        g.step()
        g.sync_to_host(gas=pin["gas"], magflux=pin["magflux"], bxyz=pin["bxyz"])
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / ke
    h2d = sum(pin[nm].nbytes for nm in ("gas", "magflux", "ogas", "omagflux"))
    d2h = sum(pin[nm].nbytes for nm in ("gas", "magflux", "bxyz"))
    e2e_val = world * zones / e2e_s
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_val = world * zones / float(t.item())

    # roofline of the dominant phase
    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", FALLBACK_HBM_GBS))
    dom = max(ph, key=ph.get)
    n_if = (n + 1) * n * n   # interfaces per direction launch
    flux_launch_ms = ph["fluxes"] / 3.0
    fbytes = FLUX_BYTES_PER_IFACE if args.prec == "fp64" else FLUX_BYTES_PER_IFACE_F32
    achieved = fbytes * n_if / (flux_launch_ms / 1e3) / 1e9
    tpu = traffic_per_unit("k_flux_tile", args.prec)
    roof = {"kernel": "k_flux_tile<double>" if args.prec == "fp64" else "k_flux_tile<float>",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": (round(tpu * n_if) if tpu else None),
            "algorithmic_bytes": fbytes * n_if, "peak_source": pk_kind,
            "launch_ms": round(flux_launch_ms, 4),
            ("fp64_tflops" if args.prec == "fp64" else "fp32_tflops"):
                round(FLUX_FLOPS_PER_IFACE * n_if / (flux_launch_ms / 1e3) / 1e12, 3),
            "fp64_peak_nominal_tflops": FP64_NOMINAL_TFLOPS,
            "dominant_phase": dom, "phase_ms": {k: round(v, 4) for k, v in ph.items()},
            "step_bytes_per_zone": STEP_BYTES_PER_ZONE,
            "step_hbm_frac": round(STEP_BYTES_PER_ZONE * zones / (ms / args.steps / 1e3) / 1e9 / hbm, 4)}
    spz = traffic_per_unit("step", args.prec)
    if spz:
        # measured DRAM bytes of one whole step (all its kernels) per active zone, times this run's zones
        roof["step_traffic"] = {"bytes_per_zone": spz, "bytes_per_step": round(spz * zones),
                                "over_compulsory": round(spz / STEP_BYTES_PER_ZONE, 2),
                                "achieved_gbs": round(spz * zones / (ms / args.steps / 1e3) / 1e9, 1),
                                "source": "ncu dram bytes of one step at 128^3, per active zone "
                                          "(profiles/step_traffic_128cubed_fp64.md)"}
    clocks = clk.summary()
    g.close()
    out = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.prec == "fp64" else "f32-flux/f64-state",
        "data": "synthetic (problem generated on the device)",
        "config": workload_config(n, args.prec, {"parallelism": f"replicas x{world}"}),
        "e2e": {"value": e2e_val, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": ke},
        "gpu_launches": timed_launches,
        "roofline": roof, "clocks": clocks, "status": st["status"], "t_sim": st["t"], "dt": st["dt"],
    }
    if world == 1 and not args.no_extras:
        out["headline_extras"] = headline_extras(n, args.fp32_steps)
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(n, steps=2)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return out


def headline_extras(n, steps):
    """The rest of the headline metric on the same GPU: the FP32-flux path against the FP64 path on the
    same problem (device ms per step and the L1 difference of the gas state after `steps` steps -- the
    configuration's 200 by default -- relative to the mean |value| per variable), and the cost of a step with the learned closure on the coarse
    turbulence grid next to the plain coarse and the fine step (the closure's accuracy comes from its
    training run, kaiju_b200/closure_train.py)."""
    from kaiju_b200 import gamera as gm, turbulence as tu
    out = {}
    model = model_for(n)
    xyz = gm.corners_warped(model, (-0.5, 0.5) * 3, 0.04)
    g64 = gm.GameraGPU.from_corners(model, xyz, "BW")
    g32 = gm.GameraGPU.from_corners(model, xyz, "BW")
    g32.set_precision(gm.GAM_FP32FLUX)
    ms64, _ = g64.run_steps_timed(steps)
    ms32, _ = g32.run_steps_timed(steps)
    a, b = g64.fetch("gas")[4:-4, 4:-4, 4:-4], g32.fetch("gas")[4:-4, 4:-4, 4:-4]
    l1 = [float(np.mean(np.abs(a[..., v] - b[..., v])) / max(np.mean(np.abs(a[..., v])), 1e-300)) for v in range(5)]
    g64.close()
    g32.close()
    out["fp32flux"] = {"ms_per_step": ms32 / steps, "fp64_ms_per_step": ms64 / steps,
                       "speedup_vs_fp64": ms64 / ms32, "steps": steps,
                       "l1_rel_vs_fp64_per_var": l1, "l1_rel_vs_fp64": max(l1),
                       "value": n ** 3 * steps / (ms32 / 1e3)}
    # closure cost: 128^3 coarse turbulence with the net attached (its weights do not change the cost)
    nc = 128
    fine = tu.turbulence_problem(2 * nc, 64)
    fine.run_steps(3)
    msf, _ = fine.run_steps_timed(10)
    c = tu.coarse_problem(nc)
    c.restrict_from(fine, gm.GAM_SYNC_STATE)
    c.restrict_from(fine, gm.GAM_SYNC_OSTATE)
    fine.close()
    st = c.status()
    c.set_scalars(st["t"], 1.0e-3, 0.0, 1, st["time"], st["time"] - 1.0e-3)
    c.run_steps(3)
    msp, _ = c.run_steps_timed(10)
    cl = gm.Closure(nc, nc, nc, seed=0)
    c.set_closure(cl)
    c.run_steps(3)
    msc, _ = c.run_steps_timed(10)
    c.set_closure(None)
    c.close()
    cl.close()
    out["closure"] = {"coarse_cells": [nc] * 3, "fine_cells": [2 * nc] * 3,
                      "fine_ms_per_step": msf / 10, "coarse_plain_ms_per_step": msp / 10,
                      "coarse_closure_ms_per_step": msc / 10,
                      "fine_over_closure_per_coarse_step": 2 * (msf / 10) / (msc / 10)}
    return out


# The CPU sample: a 256 x 256 x 16 k-slab (|z| <= 8/256, through the blast centre) of the same warped
# blast wave -- the GPU workload's own i-j planes and cell spacing, 1/16 of its cells, with zero-gradient
# boundaries on every face. Its set-up (Corners2Grid and the 12^3-point IC quadrature on the host) is
# excluded from the timing.
SAMPLE_NK = 16


def oracle_sample(n, threads):
    from oracle import pyoracle as po
    po.build()
    h = SAMPLE_NK / (2.0 * n)
    return po.Oracle(n, n, SAMPLE_NK, ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5, -0.5, 0.5, -h, h),
                     CFL=0.3, bc=[1] * 6, threads=threads)


def sample_text(n, steps, warm, threads):
    return (f"{n}x{n}x{SAMPLE_NK} k-slab (|z| <= {SAMPLE_NK}/{2 * n}, through the blast centre) of the same "
            f"warped blast wave, {steps} timed steps after {warm} warm-up steps (set-up excluded), OpenMP "
            f"{threads} threads; the oracle (C++ restatement of the Fortran reference, which cannot be "
            f"compiled on this image)")


def cpu_baseline(n, steps=2):
    """The oracle (C++ restatement of the reference, OpenMP on all host cores) on the CPU sample."""
    threads = os.cpu_count() or 1
    o = oracle_sample(n, threads)
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": n * n * SAMPLE_NK * steps / dt, "unit": "zone-updates/s", "cores": threads, "kind": "port",
            "sample": sample_text(n, steps, 1, threads)}


def run_reference(args, rank, world):
    """The reference arm: the oracle on the CPU sample of this arm's workload, K timed steps after W
    warm-up steps, on rank 0 only (the other ranks exit without work)."""
    if rank != 0:
        return None
    n = args.n
    threads = os.cpu_count() or 1
    o = oracle_sample(n, threads)
    o.step(max(1, args.warmup))
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    v = n * n * SAMPLE_NK * steps / dt
    return {"metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(n, "fp64", {"parallelism": f"replicas x{world}"}),
            "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": threads, "kind": "port",
                             "sample": sample_text(n, steps, max(1, args.warmup), threads)},
            "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    else:
        out = run_ours(args, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
