"""Training and evaluation of the learned flux closure on decaying MHD turbulence.

Data: fine runs (2n)^3 of the turbulence problem (kaiju_b200/turbulence.py) generate training samples on
the n^3 grid. A sample is one coarse step: State and oState are the fine state restricted at two times
two fine steps apart, the step's dt is the next two fine steps, and the target is the restricted fine
state at the end. The closure stores the net input of the coarse State and the residual
restrict(fine) - plain coarse step. Training minimises, by Adam on the device (the net's own tensor-core
forward and backward kernels), the mean over cells of sum_v ((dt/V * div(corrections)_v - residual_v) /
rms_v)^2: the face corrections are fitted to what the plain coarse fluxes miss. With --loss face the
samples also carry face targets -- the fine fluxes of the two fine steps, time-integrated and summed over
the fine sub-faces of each coarse face, over the coarse dt, minus the plain coarse step's flux -- and the
net is fitted to them face by face (the correction that gives the coarse faces the restricted fine fluxes).

Evaluation on held-out seeds: (1) the same loss with the trained net against no correction (the gain of
the net on one step); (2) rollouts to a common end time: the fine run, the plain coarse run and the coarse
run with the closure, L1 errors of the coarse runs against the restricted fine state, and the GPU time of
each run.

    python -m kaiju_b200.closure_train --n 128 --train-seeds 0-7 --eval-seeds 64-67 --out report.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import gamera as gm
from . import turbulence as tu

GAMMA = 5.0 / 3.0


def _seeds(spec: str):
    out = []
    for part in spec.split(","):
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        elif part:
            out.append(int(part))
    return out


def primitive_stats(g: gm.GameraGPU):
    """Mean and spread of rho, v, P, B over the active cells of a problem."""
    gas = g.fetch("gas")
    b = g.fetch("bxyz")
    G = 4
    a = (slice(G, -G),) * 3
    rho = gas[a + (0,)]
    v = [gas[a + (q,)] / rho for q in (1, 2, 3)]
    P = (GAMMA - 1.0) * (gas[a + (4,)] - 0.5 * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    w = [rho] + v + [P] + [b[a + (q,)] for q in range(3)]
    mean = np.array([x.mean() for x in w])
    std = np.array([max(x.std(), 1e-3) for x in w])
    return mean, std


def collect(closure: gm.Closure, n: int, seeds, per_seed: int, warm: int, gap: int, slot0: int = 0,
            set_input_norm: bool = True, faces: bool = False):
    """Samples from fine runs of each seed into consecutive slots from slot0; returns the slots. faces: also
    accumulate the two fine steps' fluxes for each sample's face target."""
    coarse = tu.coarse_problem(n)
    slots = []
    slot = slot0
    for seed in seeds:
        fine = tu.turbulence_problem(2 * n, seed)
        for _ in range(warm):
            fine.step()
        for s in range(per_seed):
            coarse.restrict_from(fine, gm.GAM_SYNC_OSTATE)
            ta = fine.status()["time"]
            fine.step()
            fine.step()
            tb = fine.status()["time"]
            coarse.restrict_from(fine, gm.GAM_SYNC_STATE)
            if set_input_norm and slot == 0:
                closure.in_mean, closure.in_std = primitive_stats(coarse)
                closure.set_norm(closure.in_mean, closure.in_std, np.ones(8), np.ones(5))
            t_prev = tb
            for q in range(2):
                fine.step()
                if faces:
                    t_now = fine.status()["time"]
                    closure.accum_fine(fine, t_now - t_prev, reset=(q == 0))
                    t_prev = t_now
            tc = fine.status()["time"]
            coarse.set_scalars(tb, tc - tb, 0.0, 1, tb, ta)
            closure.capture(slot, coarse, fine)
            slots.append(slot)
            slot += 1
            for _ in range(gap):
                fine.step()
        fine.close()
    coarse.close()
    return slots


def set_output_norm(closure: gm.Closure, n: int, slots, emf: bool = True):
    """Residual rms per gas variable over the samples, and the flux scale that turns an O(1) net output
    into a correction of that size in one step. emf: also the EMF scale from the face magnetic-flux residual
    (an O(1) output changes a face's flux by about that residual in one step) and the loss's B terms."""
    rms = np.zeros(5)
    dts = []
    for s in slots:
        r, dt = closure.residual_rms(s)
        rms += r ** 2
        dts.append(dt)
    rms = np.sqrt(rms / len(slots))
    rms = np.maximum(rms, 1e-12)
    dx = 1.0 / n
    dt = float(np.mean(dts))
    flux = np.concatenate([rms, rms[1:4]]) * dx / dt
    closure.set_norm(closure.in_mean, closure.in_std, flux, rms)
    closure.res_scale = rms
    if emf:
        rb = np.sqrt(np.mean([closure.residual_rms_b(s) ** 2 for s in slots], axis=0))
        rb = np.maximum(rb, 1e-15)
        closure.set_norm_emf(rb / (dt * dx), rb)
    return rms, flux


def set_output_norm_faces(closure: gm.Closure, slots):
    """Flux scale from the face targets: the rms over the samples of target / area per flux, so an O(1) net
    output is a correction of the targets' size."""
    acc = np.zeros(8)
    for s in slots:
        r, _ = closure.face_stats(s)
        acc += r ** 2
    flux = np.maximum(np.sqrt(acc / len(slots)), 1e-12)
    closure.set_norm(closure.in_mean, closure.in_std, flux, closure.res_scale)
    return flux


def train(closure: gm.Closure, slots, epochs: int, lr: float, seed: int = 0, log=None):
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        order = list(rng.permutation(slots))
        lr_e = lr * 0.5 * (1.0 + np.cos(np.pi * ep / max(epochs, 1)))   # cosine decay
        loss = closure.train(order, max(lr_e, lr * 0.02))
        hist.append(loss)
        if log:
            log(f"epoch {ep}: loss {loss:.5f}")
    return hist


def l1_error(a: gm.GameraGPU, b: gm.GameraGPU):
    """Mean over the gas variables of the L1 difference of the active cells, relative to b's mean |value|
    (the momenta relative to the rms momentum); the per-variable list ends with the cell magnetic field's L1
    difference relative to b's rms field (reported, not in the mean)."""
    G = 4
    x, y = a.fetch("gas")[G:-G, G:-G, G:-G], b.fetch("gas")[G:-G, G:-G, G:-G]
    errs = []
    mom = np.sqrt(np.mean(y[..., 1] ** 2 + y[..., 2] ** 2 + y[..., 3] ** 2))
    for v in range(5):
        den = mom if v in (1, 2, 3) else np.mean(np.abs(y[..., v]))
        errs.append(float(np.mean(np.abs(x[..., v] - y[..., v])) / den))
    bx, by = a.fetch("bxyz")[G:-G, G:-G, G:-G], b.fetch("bxyz")[G:-G, G:-G, G:-G]
    brms = np.sqrt(np.mean((by ** 2).sum(-1)))
    b_err = float(np.mean(np.abs(bx - by).sum(-1)) / brms)
    return float(np.mean(errs)), errs + [b_err]


def _timed_advance(g: gm.GameraGPU, t_end: float):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = 0
    t = g.status()["t"]
    while t < t_end * (1.0 - 1e-12):
        _, _, t = g.step()
        steps += 1
    torch.cuda.synchronize()
    return time.perf_counter() - t0, steps


def rollout(closure: gm.Closure, n: int, seed: int, t_end: float):
    """Fine run, plain coarse run and closure coarse run of one seed from t = 0 to t_end."""
    # every run stops at t_end exactly through CalcDT's tFin clamp
    fine = _problem_with_tfin(2 * n, seed, t_end)
    runs = {}
    for name in ("plain", "closure"):
        c = _coarse_from(fine, n, t_end)
        if name == "closure":
            c.set_closure(closure)
        runs[name] = c
    t_fine, s_fine = _timed_advance(fine, t_end)
    out = {"seed": seed, "t_end": t_end, "fine": {"seconds": t_fine, "steps": s_fine}}
    for name, c in runs.items():
        sec, st = _timed_advance(c, t_end)
        ref = _coarse_from(fine, n, t_end)   # the fine state at t_end, restricted
        err, per = l1_error(c, ref)
        out[name] = {"seconds": sec, "steps": st, "l1": err, "l1_per_var": per,
                     "rejects": c.closure_rejects() if name == "closure" else 0}
        if name == "closure":
            c.set_closure(None)
        c.close()
        ref.close()
    fine.close()
    return out


def three_levels(closure: gm.Closure, n: int, seed: int, t_end: float):
    """Errors against a truth run two levels finer: the truth (4n)^3, the fine (2n)^3 run and the coarse n^3
    runs (plain and with the closure) all start from restrictions of the truth's initial state and run to
    t_end; each is compared, restricted to n^3, with the restricted truth. The closure reaches the fine-grid
    error when its L1 is at most the fine run's."""
    truth = _problem_with_tfin(4 * n, seed, t_end)
    fine = _coarse_from(truth, 2 * n, t_end)
    plain = _coarse_from(fine, n, t_end)
    cl = _coarse_from(fine, n, t_end)
    cl.set_closure(closure)
    out = {"seed": seed, "t_end": t_end, "cells": [n, 2 * n, 4 * n]}
    for name, g in (("truth", truth), ("fine", fine), ("plain", plain), ("closure", cl)):
        sec, st = _timed_advance(g, t_end)
        out[name] = {"seconds": sec, "steps": st}
    t2 = _coarse_from(truth, 2 * n, t_end)
    ref = _coarse_from(t2, n, t_end)
    f1 = _coarse_from(fine, n, t_end)
    for name, g in (("fine", f1), ("plain", plain), ("closure", cl)):
        err, per = l1_error(g, ref)
        out[name].update({"l1": err, "l1_per_var": per})
    out["closure"]["rejects"] = cl.closure_rejects()
    cl.set_closure(None)
    for g in (truth, fine, plain, cl, t2, ref, f1):
        g.close()
    return out


def step_costs(closure: gm.Closure, n: int, seed: int, steps: int = 20):
    """Device ms per step (CUDA events over graph-replayed steps) of the fine problem, the plain coarse
    problem and the coarse problem with the closure."""
    fine = tu.turbulence_problem(2 * n, seed)
    out = {}
    fine.run_steps(3)
    ms, _ = fine.run_steps_timed(steps)
    out["fine_ms"] = ms / steps
    for name in ("plain", "closure"):
        c = _coarse_from(fine, n, 1.0e30)
        if name == "closure":
            c.set_closure(closure)
        c.run_steps(3)
        ms, _ = c.run_steps_timed(steps)
        out[name + "_ms"] = ms / steps
        if name == "closure":
            c.set_closure(None)
        c.close()
    fine.close()
    return out


def _problem_with_tfin(n, seed, t_end):
    model = tu.turbulence_model(n)
    model.tFin = t_end
    xyz = gm.corners_uniform(model, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    g = gm.GameraGPU.from_corners(model, xyz, "OT2D")
    gas, magflux, _ = tu.turbulence_fields(n, seed)
    g.sync_to_device(gas=gas, magflux=magflux, ogas=gas, omagflux=magflux, time=0.0, otime=0.0)
    g.init_dt()
    return g


def _coarse_from(fine: gm.GameraGPU, n: int, t_end: float):
    """A coarse problem (CFL dt) whose State and oState are the restriction of the fine State."""
    model = tu.turbulence_model(n)
    model.tFin = t_end
    xyz = gm.corners_uniform(model, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    c = gm.GameraGPU.from_corners(model, xyz, "OT2D")
    c.restrict_from(fine, gm.GAM_SYNC_STATE)
    c.restrict_from(fine, gm.GAM_SYNC_OSTATE)
    st = fine.status()
    c.set_scalars(st["t"], 0.0, 0.0, 0, st["time"], st["time"])
    c.init_dt()
    return c


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--train-seeds", default="0-7")
    ap.add_argument("--eval-seeds", default="64-67")
    ap.add_argument("--per-seed", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--warm", type=int, default=20)
    ap.add_argument("--gap", type=int, default=6)
    ap.add_argument("--t-end", type=float, default=0.1)
    ap.add_argument("--rollouts", type=int, default=2)
    ap.add_argument("--three-levels", type=int, default=0,
                    help="also evaluate this many held-out seeds against a truth run at 4n (needs (4n)^3 to fit)")
    ap.add_argument("--loss", choices=["cell", "face"], default="cell",
                    help="fit the cell residual through the divergence, or the face targets directly")
    ap.add_argument("--no-emf", action="store_true",
                    help="leave the EMF outputs unused (face-flux corrections only)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    report = train_and_evaluate(a.n, _seeds(a.train_seeds), _seeds(a.eval_seeds), a.per_seed, a.epochs, a.lr,
                                a.warm, a.gap, a.t_end, a.rollouts, three=a.three_levels, loss=a.loss,
                                emf=not a.no_emf)
    s = json.dumps(report, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s)
    print(s)


def train_and_evaluate(n, train_seeds, eval_seeds, per_seed, epochs, lr, warm, gap, t_end, rollouts, log=print,
                       three=0, loss="cell", emf=True):
    t0 = time.perf_counter()
    closure = gm.Closure(n, n, n, seed=0)
    closure.reserve(per_seed * (len(train_seeds) + len(eval_seeds)))
    faces = loss == "face"
    # the input normalisation comes from the first sample's restricted state
    tr = collect(closure, n, train_seeds, per_seed, warm, gap, 0, faces=faces)
    ev = collect(closure, n, eval_seeds, per_seed, warm, gap, len(tr), set_input_norm=False, faces=faces)
    t_data = time.perf_counter() - t0
    rms, flux = set_output_norm(closure, n, tr, emf=emf and not faces)
    face_check = None
    if faces:
        flux = set_output_norm_faces(closure, tr)
        closure.set_loss(gm.GAM_CLOSURE_LOSS_FACE)
        face_check = closure.face_stats(tr[0])[1].tolist()
    before = closure.eval(ev)
    t1 = time.perf_counter()
    hist = train(closure, tr, epochs, lr, log=log)
    t_train = time.perf_counter() - t1
    after_tr = closure.eval(tr)
    after = closure.eval(ev)
    rolls = [rollout(closure, n, s, t_end) for s in eval_seeds[:rollouts]]
    levels = [three_levels(closure, n, s, t_end) for s in eval_seeds[:three]]
    costs = step_costs(closure, n, eval_seeds[0])
    closure.close()
    return {
        "n_coarse": n, "n_fine": 2 * n, "train_seeds": list(train_seeds), "eval_seeds": list(eval_seeds),
        "samples": {"train": len(tr), "eval": len(ev)}, "epochs": epochs, "lr": lr, "loss": loss,
        "emf": bool(emf and not faces),
        "face_target_vs_residual": face_check,
        "seconds": {"data": t_data, "train": t_train},
        "residual_rms": rms.tolist(), "flux_scale": flux.tolist(),
        "loss_history": hist,
        "train_loss": {"net": after_tr[0], "none": after_tr[1]},
        "eval_loss": {"untrained": before[0], "net": after[0], "none": after[1],
                      "gain": after[1] / after[0] if after[0] > 0 else None},
        "rollouts": rolls,
        "three_levels": levels,
        "step_ms": costs,
    }


if __name__ == "__main__":
    main()
