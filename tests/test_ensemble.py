"""Kelvin-Helmholtz ensemble: the device IC against the oracle's, and batched (ensemble graph) runs against
the same members stepped one by one."""
import ctypes as C

import numpy as np
import pytest

from helpers import per_var_rel


def test_ensemble_create_rejects_bad_arguments():
    from kaiju_b200 import build as kb, gamera as gm
    kb.build()
    L = gm.load_library()
    e = C.c_void_p()
    assert L.gam_gpu_ensemble_create(C.byref(e), None, 0) == gm.GAM_ERR_ARG
    arr = (C.c_void_p * 1)(None)
    assert L.gam_gpu_ensemble_create(C.byref(e), arr, 1) == gm.GAM_ERR_ARG


def test_kh_params_follow_the_seed():
    from kaiju_b200 import gamera as gm
    p = gm.kh_ensemble_params(96, seed=0)
    assert len(p) == 96 and {x["nx"] for x in p} <= {64, 128, 256, 512}
    assert all(0.01 <= x["a"] <= 0.05 and 0.0 <= x["Bx"] <= 0.2 for x in p)
    assert p == gm.kh_ensemble_params(96, seed=0)


@pytest.mark.gpu
def test_kh_device_ic_matches_oracle(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    par = dict(nx=64, a=0.03, Bx=0.1, amp=0.01, seed=5)
    m = gm.kh_model(64)
    o = oracle_lib.Oracle(64, 32, 4, ic="KH", grid="uniform", bounds=gm.kh_bounds(64), CFL=0.3, bc=[0, 0, 1, 1, 0, 0],
                          kh=(0.03, 0.1, 0.01, 5))
    with gm.GameraGPU.from_corners(m, o.get("xyz"), "KH", ic_par=(0.03, 0.1, 0.01, 5.0)) as g:
        for name in ("gas", "magflux", "bxyz"):
            assert max(per_var_rel(g.fetch(name), o.get(name))) <= 1e-12, name
        o.step(3)
        g.run_steps(3)
        for v, e in enumerate(per_var_rel(g.fetch("gas"), o.get("gas"))):
            assert e <= 1e-10, (v, e)


@pytest.mark.gpu
def test_ensemble_equals_members_stepped_alone(gpu_lib):
    """Three members of different sizes and precisions: five batch steps give bit-identical states to the
    same members stepped on their own, and every member keeps its own dt."""
    from kaiju_b200 import gamera as gm
    pars = [dict(nx=64, a=0.02, Bx=0.05, amp=0.01, seed=1), dict(nx=128, a=0.04, Bx=0.15, amp=0.01, seed=2),
            dict(nx=64, a=0.03, Bx=0.0, amp=0.01, seed=3)]
    fp32 = [True, False, True]
    alone = [gm.kh_member(p, f) for p, f in zip(pars, fp32)]
    batch = [gm.kh_member(p, f) for p, f in zip(pars, fp32)]
    try:
        for g in alone:
            assert g.run_steps(5) == 0
        with gm.Ensemble(batch) as e:
            assert e.run_steps(5) == 0
        dts = set()
        for a, b in zip(alone, batch):
            assert np.array_equal(a.fetch("gas"), b.fetch("gas"))
            assert np.array_equal(a.fetch("magflux"), b.fetch("magflux"))
            sa, sb = a.status(), b.status()
            assert sa["ts"] == sb["ts"] == 5 and sa["dt"] == sb["dt"]
            dts.add(sb["dt"])
        assert len(dts) == 3
    finally:
        for g in alone + batch:
            g.close()


@pytest.mark.gpu
def test_ensemble_advance_to_time(gpu_lib):
    from kaiju_b200 import gamera as gm
    pars = [dict(nx=64, a=0.02, Bx=0.05, amp=0.01, seed=1), dict(nx=128, a=0.04, Bx=0.15, amp=0.01, seed=2)]
    t_end = 0.02
    members = [gm.kh_member(p, True, tFin=t_end) for p in pars]
    try:
        with gm.Ensemble(members) as e:
            rc, steps = e.advance(t_end, chunk=4, max_steps=1000)
            assert rc == 0 and 0 < steps < 1000
        for g in members:
            st = g.status()
            assert st["t"] >= t_end * (1 - 1e-12)
    finally:
        for g in members:
            g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [False, True])
def test_flux_tile_height_does_not_change_results(gpu_lib, fp32):
    """4-row and 8-row flux tiles compute every interface from the same staged values: bit-identical runs."""
    from kaiju_b200 import gamera as gm
    par = dict(nx=128, a=0.03, Bx=0.1, amp=0.01, seed=4)
    a, b = gm.kh_member(par, fp32), gm.kh_member(par, fp32)
    try:
        b.set_tile(gm.GAM_TILE_FLUX_ROWS, 4)
        assert a.run_steps(6) == 0 and b.run_steps(6) == 0
        for name in ("gas", "magflux"):
            assert np.array_equal(a.fetch(name), b.fetch(name)), name
        with pytest.raises(gm.GamError):
            b.set_tile(gm.GAM_TILE_FLUX_ROWS, 5)
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_ensemble_autotune_is_transparent(gpu_lib):
    """The autotuner picks a tile height per member shape by timing batch steps; the run it takes part in
    is bit-identical to the same ensemble stepped without it."""
    from kaiju_b200 import gamera as gm
    pars = [dict(nx=64, a=0.02, Bx=0.05, amp=0.01, seed=1), dict(nx=256, a=0.04, Bx=0.15, amp=0.01, seed=2),
            dict(nx=64, a=0.03, Bx=0.0, amp=0.01, seed=3)]
    tuned = [gm.kh_member(p, True) for p in pars]
    plain = [gm.kh_member(p, True) for p in pars]
    try:
        with gm.Ensemble(tuned) as e:
            rows = e.autotune(steps=2)   # (2 shapes x 2 heights + 2 flux modes) x (1 + 2) batch steps
            assert len(rows) == 3 and set(rows) <= {4, 8} and rows[0] == rows[2]
            assert e.queue in (True, False)
            assert e.run_steps(2) == 0
        with gm.Ensemble(plain) as e:
            assert e.run_steps((2 * 2 + 2) * 3 + 2) == 0
        for a, b in zip(tuned, plain):
            assert a.status()["ts"] == b.status()["ts"]
            assert np.array_equal(a.fetch("gas"), b.fetch("gas"))
    finally:
        for g in tuned + plain:
            g.close()


@pytest.mark.gpu
def test_tile_queue_equals_per_member_launches(gpu_lib):
    """One persistent flux launch over every member's tiles gives bit-identical states to each member
    launching its own flux kernels (members of two sizes, FP32-flux and FP64 mixed)."""
    from kaiju_b200 import gamera as gm
    pars = [dict(nx=64, a=0.02, Bx=0.05, amp=0.01, seed=1), dict(nx=128, a=0.04, Bx=0.15, amp=0.01, seed=2),
            dict(nx=64, a=0.03, Bx=0.0, amp=0.01, seed=3)]
    fp32 = [True, False, True]
    q = [gm.kh_member(p, f) for p, f in zip(pars, fp32)]
    plain = [gm.kh_member(p, f) for p, f in zip(pars, fp32)]
    try:
        with gm.Ensemble(q) as e:
            e.set_queue(True)
            assert e.run_steps(4) == 0
        with gm.Ensemble(plain) as e:
            assert e.run_steps(4) == 0
        for a, b in zip(q, plain):
            for name in ("gas", "magflux"):
                assert np.array_equal(a.fetch(name), b.fetch(name)), name
    finally:
        for g in q + plain:
            g.close()
