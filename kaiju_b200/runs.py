"""Long runs on the device. The spherical configuration: `magnetosphere` runs the Earth deck's Gamera part
(ionospheric inner and solar-wind outer boundaries, cut dipole, gravity) on the LFM-type grid; `spherical`
runs the reference's LFM blast-wave deck on the same kind of grid with ring averaging about the axis, the
axis boundaries, Boris and a dipole background. Both run the plain FP64 path and the FP32-flux path side by
side. The learned closure's step cost, the Kelvin-Helmholtz ensemble and k-tiling have their own runs.

    python -m kaiju_b200.runs spherical --n 96 96 128 --steps 2000
    python -m kaiju_b200.runs magnetosphere --n 96 96 128 --steps 2000   # the Earth deck with a solar wind
    python -m kaiju_b200.runs closure-step --n 128 --steps 20
    python -m kaiju_b200.runs ensemble --steps 20          # 96 Kelvin-Helmholtz members, FP32-flux
    python -m kaiju_b200.runs ensemble-run --t-end 2       # the same members run to t = 2
    python -m kaiju_b200.runs tiles --n 256 --steps 10     # the 256^3 blast wave as 1, 2 and 4 k-tiles
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import gamera as gm


def _fp32_to_t_end(g32, t_end, steps, cells, fresh):
    """The FP32-flux path to the FP64 run's end time: g32 (created with tFin = t_end) takes single steps until
    its time reaches t_end, which counts the steps it needs (CalcDT's tFin clamp lands the last one on t_end;
    steps after it would advance by TINY). A second problem from `fresh()` times `steps` graph steps."""
    done, rc = 0, 0
    while g32.status()["t"] < t_end * (1.0 - 1e-14) and done < 4 * steps:
        g32.step()
        done += 1
    g = fresh()
    g.set_precision(gm.GAM_FP32FLUX)
    ms32, rc = g.run_steps_timed(steps)
    g.close()
    st = g32.status()
    return {"ms_per_step": ms32 / steps, "zone_updates_per_s": cells * steps / (ms32 / 1e3),
            "steps_to_t_end": done, "t": st["t"], "status": rc}


def spherical_model(Nip: int, Njp: int, Nkp: int) -> gm.Model:
    """The reference's LFM blast-wave deck (tests/gamera/lfmbw.xml: 7UP, pdmb 1, Boris Ca 10, floors 1e-4 /
    1e-6, fixed-gas shells, predictor fix, dt over the active cells) with a dipole background."""
    return gm.Model(Nip, Njp, Nkp, CFL=0.3, pdmb=1.0, rmeth="7UP", dFloor=1e-4, pFloor=1e-6, doBoris=True,
                    Ca=10.0, tFin=1.0e30, bc=(gm.GAM_BC_LFMBW, gm.GAM_BC_LFMBW, gm.GAM_BC_LFMPOLE,
                                               gm.GAM_BC_LFMPOLE, gm.GAM_BC_PERIODIC, gm.GAM_BC_PERIODIC),
                    ring=dict(recon="PPM"), predFixLFM=True, bwD0=1.0, bwP0=0.1, dtActive=True,
                    doBackground=True)


def spherical(n=(96, 96, 128), steps=2000, dipole=2000.0, grid=(10.0, 100.0, 1.03, 0.05)):
    """The FP64 path for `steps` steps (device-timed), then the FP32-flux path from the same start to the
    same end time (CalcDT's tFin clamp lands it there), and the L1 difference of the two states."""
    import dataclasses
    model = spherical_model(*n)
    xyz = gm.corners_lfm(model, *grid)
    out = {"cells": list(n), "steps": steps, "dipole_moment": dipole, "grid_r_theta0": list(grid)}
    cells = n[0] * n[1] * n[2]
    g64 = gm.GameraGPU.from_corners(model, xyz, "LFMBW", b0=("dipole", dipole))
    ms, rc = g64.run_steps_timed(steps)
    t_end = g64.status()["t"]
    out["fp64"] = {"ms_per_step": ms / steps, "zone_updates_per_s": cells * steps / (ms / 1e3), "status": rc,
                   "t_end": t_end}
    m32 = dataclasses.replace(model, tFin=t_end)
    g32 = gm.GameraGPU.from_corners(m32, xyz, "LFMBW", b0=("dipole", dipole))
    g32.set_precision(gm.GAM_FP32FLUX)
    out["fp32flux"] = _fp32_to_t_end(g32, t_end, steps, cells,
                                     lambda: gm.GameraGPU.from_corners(m32, xyz, "LFMBW", b0=("dipole", dipole)))
    a, b = g64.fetch("gas")[4:-4, 4:-4, 4:-4], g32.fetch("gas")[4:-4, 4:-4, 4:-4]
    l1 = [float(np.mean(np.abs(a[..., v] - b[..., v])) / np.mean(np.abs(a[..., v]))) for v in range(5)]
    out["fp32flux"]["l1_rel_vs_fp64_per_var"] = l1
    out["fp32flux"]["speedup_vs_fp64_per_step"] = out["fp64"]["ms_per_step"] / out["fp32flux"]["ms_per_step"]
    out["divb"] = {"fp64": g64.divb(), "fp32flux": g32.divb()}
    g64.close()
    g32.close()
    return out


def magnetosphere(n=(96, 96, 128), steps: int = 2000):
    """The spherical configuration as specified: the Earth deck's magnetosphere (kaiju_b200/magnetosphere.py)
    on the 96x96x128 LFM-type grid r in [2, 30] with a 3.1e4 nT dipole and a constant solar wind
    (5 amu/cc, -400 km/s, Bz = -5 nT, 1e5 K) entering at the outer shell. The FP64 path for `steps` steps
    (device-timed), then the FP32-flux path from the same start to the same end time, and their difference."""
    import dataclasses
    from . import magnetosphere as ms
    cells = n[0] * n[1] * n[2]
    out = {"cells": list(n), "steps": steps, "grid_r_stretch_theta0": list(ms.GRID),
           "code_params": [float(v) for v in ms.Magnetosphere().code_params()]}
    g64 = ms.magnetosphere_problem(n)
    ms64, rc = g64.run_steps_timed(steps)
    st = g64.status()
    t_end = st["t"]
    out["fp64"] = {"ms_per_step": ms64 / steps, "zone_updates_per_s": cells * steps / (ms64 / 1e3), "status": rc,
                   "t_end_code": t_end, "t_end_s": t_end * ms.Magnetosphere().gT0}
    g32 = ms.magnetosphere_problem(n, tFin=t_end)
    g32.set_precision(gm.GAM_FP32FLUX)
    out["fp32flux"] = _fp32_to_t_end(g32, t_end, steps, cells, lambda: ms.magnetosphere_problem(n, tFin=t_end))
    a, b = g64.fetch("gas")[4:-4, 4:-4, 4:-4], g32.fetch("gas")[4:-4, 4:-4, 4:-4]
    out["fp32flux"]["l1_rel_vs_fp64_per_var"] = [
        float(np.mean(np.abs(a[..., v] - b[..., v])) / np.mean(np.abs(a[..., v]))) for v in range(5)]
    out["fp32flux"]["speedup_vs_fp64_per_step"] = out["fp64"]["ms_per_step"] / out["fp32flux"]["ms_per_step"]
    out["divb"] = {"fp64": g64.divb(), "fp32flux": g32.divb()}
    rho = a[..., 0]
    out["fp64"]["density_min_max"] = [float(rho.min()), float(rho.max())]
    g64.close()
    g32.close()
    return out


def closure_step(n: int = 128, steps: int = 20, seed: int = 64):
    """Device ms per step of the n^3 turbulence problem, plain and with a (freshly initialised) closure
    attached: the closure's cost does not depend on its weights."""
    from . import turbulence as tu
    g = tu.turbulence_problem(n, seed)
    g.run_steps(3)
    ms_plain, _ = g.run_steps_timed(steps)
    c = gm.Closure(n, n, n, seed=0)
    g.set_closure(c)
    g.run_steps(3)
    ms_cl, _ = g.run_steps_timed(steps)
    out = {"n": n, "steps": steps, "plain_ms": ms_plain / steps, "closure_ms": ms_cl / steps,
           "rejects": g.closure_rejects()}
    g.set_closure(None)
    g.close()
    c.close()
    return out


def ensemble(steps: int = 20, members: int = 96, seed: int = 0):
    """Device ms per batch step of the Kelvin-Helmholtz ensemble (FP32-flux members of uneven sizes): one
    graph per batch step with the members as concurrent branches, with the persistent tile-queue flux
    kernel, after the autotuner's choice, and the members stepped one after another."""
    import ctypes as C
    pars = gm.kh_ensemble_params(members, seed)
    mem = [gm.kh_member(p, True) for p in pars]
    cells = sum(p["nx"] * (p["nx"] // 2) * 4 for p in pars)
    out = {"members": members, "cells": cells, "steps": steps}
    zu = lambda ms: cells * steps / (ms / 1e3)
    with gm.Ensemble(mem) as e:
        for name, queue in (("branches", False), ("queue", True)):
            e.set_queue(queue)
            e.run_steps(3)
            rc, ms = e.run_steps_timed(steps)
            out[name] = {"ms_per_batch_step": ms / steps, "zone_updates_per_s": zu(ms), "status": rc}
        e.autotune(4)
        e.run_steps(3)
        rc, ms = e.run_steps_timed(steps)
        out["autotuned"] = {"ms_per_batch_step": ms / steps, "zone_updates_per_s": zu(ms), "status": rc,
                            "queue": bool(e.queue)}
    tot = 0.0
    for g in mem:
        v = C.c_double()
        gm.load_library().gam_gpu_run_steps_timed(g.h, steps, C.byref(v))
        tot += v.value
    out["one_by_one"] = {"ms_per_batch_step": tot / steps, "zone_updates_per_s": zu(tot)}
    for g in mem:
        g.close()
    return out


def ensemble_run(t_end: float = 2.0, members: int = 96, seed: int = 0, chunk: int = 16):
    """The batched-ensemble configuration to its end time: 96 Kelvin-Helmholtz members (FP32-flux, uneven
    sizes) advanced together to t_end, members dropping out as CalcDT's tFin clamp lands them on t_end.
    The tile shapes (and queue or branches) come from the autotuner, whose timing steps are ordinary steps
    of the run. Throughput = the members' zone-updates over the wall time of the whole advance (the host
    checks the members' times every `chunk` batch steps)."""
    import time
    pars = gm.kh_ensemble_params(members, seed)
    mem = [gm.kh_member(p, True, tFin=t_end) for p in pars]
    cells = [p["nx"] * (p["nx"] // 2) * 4 for p in pars]
    out = {"members": members, "cells": sum(cells), "t_end": t_end}
    with gm.Ensemble(mem) as e:
        rows = e.autotune(4)
        ts0 = [g.status()["ts"] for g in mem]
        t0 = time.perf_counter()
        rc, batch_steps = e.advance(t_end, chunk=chunk)
        wall = time.perf_counter() - t0
        st = [g.status() for g in mem]
    zone_updates = sum(c * (s["ts"] - a) for c, s, a in zip(cells, st, ts0))
    out.update({"status": rc, "batch_steps": batch_steps, "wall_s": wall, "zone_updates": zone_updates,
                "zone_updates_per_s": zone_updates / wall, "autotune_rows": sorted(set(rows)),
                "queue": bool(e.queue), "member_steps_min": min(s["ts"] for s in st),
                "member_steps_max": max(s["ts"] for s in st),
                "t_min": min(s["t"] for s in st), "t_max": max(s["t"] for s in st),
                "worst_status": max(s["status"] for s in st)})
    for g in mem:
        g.close()
    return out


def tiles(n: int = 256, steps: int = 10):
    """Device ms per step of the n^3 warped blast wave undivided and as 2 and 4 k-tiles on this GPU (one
    graph per step over all tiles), FP64 and FP32-flux."""
    from . import tiling as tl
    out = {"n": n, "steps": steps}
    for prec in ("fp64", "fp32flux"):
        model = gm.Model(n, n, n, CFL=0.3, tFin=1.0e30, bc=(gm.GAM_BC_ZEROGRAD,) * 6)
        xyz = gm.corners_warped(model, (-0.5, 0.5) * 3, 0.04)
        g = gm.GameraGPU.from_corners(model, xyz, "BW")
        if prec == "fp32flux":
            g.set_precision(gm.GAM_FP32FLUX)
        g.run_steps(3, check=False)
        ms, _ = g.run_steps_timed(steps)
        out[f"{prec}_single_ms"] = ms / steps
        g.close()
        for T in (2, 4):
            ts, _ = tl.make_tiles(model, xyz, T, "BW", fp32=(prec == "fp32flux"))
            grp = gm.TileGroup(ts, periodic_k=False)
            grp.run_steps(3, check=False)
            out[f"{prec}_tiles{T}_ms"] = grp.run_steps_timed(steps) / steps
            grp.close()
            for t in ts:
                t.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("run", choices=["spherical", "magnetosphere", "closure-step", "ensemble", "ensemble-run", "tiles"])
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--n", type=int, nargs="+", default=None)
    ap.add_argument("--steps", type=int, default=None)
    a = ap.parse_args(argv)
    if a.run == "spherical":
        print(json.dumps(spherical(tuple(a.n or [96, 96, 128]), a.steps or 2000), indent=1))
    elif a.run == "magnetosphere":
        print(json.dumps(magnetosphere(tuple(a.n or [96, 96, 128]), a.steps or 2000), indent=1))
    elif a.run == "ensemble":
        print(json.dumps(ensemble(a.steps or 20), indent=1))
    elif a.run == "ensemble-run":
        print(json.dumps(ensemble_run(a.t_end), indent=1))
    elif a.run == "tiles":
        print(json.dumps(tiles((a.n or [256])[0], a.steps or 10), indent=1))
    else:
        print(json.dumps(closure_step((a.n or [128])[0], a.steps or 20)))


if __name__ == "__main__":
    main()
