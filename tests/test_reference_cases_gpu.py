"""The reference's accuracy cases (tests/cases/testCases.pf) run on the device at their deck sizes.

testAdv1D / testAdv1D_8CENT (:115-180), testAdv2D (:61-86), testLoop2D (:33-58), testAlfven (:89-112) and
testOTSym (:183-225) are the reference's own answers for the flux / reconstruction / CT core of the scheme.
Each case here:
  * builds the deck's problem with the device's own set-up (corners, IC, BCs, dt) and checks the set-up
    against the oracle's at a small size (relative L-infinity <= 1e-12);
  * runs the device to the deck's tFin with the test's loop condition and asserts the test's thresholds;
  * compares the run with the oracle's run of the same deck recorded in tests/golden/reference_cases.json
    (tests/golden/make_case_fixtures.py): the same number of steps, the same end time and the same final
    state to within CASE_FIELD_TOL (block sums of the field each test looks at);
  * re-synchronises the oracle to the device's state half-way through the run and compares one step of
    each at relative L-infinity <= 1e-10 per variable.
"""
import json
import os

import numpy as np
import pytest

from helpers import (CASES, case_device, case_field, case_model, case_properties, case_running, device_to_oracle,
                     per_var_rel)

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10
# final-state fingerprint agreement with the recorded oracle run (relative to the largest block sum). The
# device and the oracle agree to round-off per step (<= 1e-10, test below); over thousands of steps the
# smooth advection cases stay at that level, while Orszag-Tang's shocks let round-off grow.
CASE_FIELD_TOL = {"adv1d": 1e-9, "adv1d_8cent": 1e-9, "adv2d": 1e-9, "loop2d": 1e-9, "alfven": 1e-9, "otsym": 1e-6}


def _fixtures():
    with open(os.path.join(HERE, "golden", "reference_cases.json")) as f:
        return json.load(f)


SMALL = {"adv1d": (32, 1, 1), "adv1d_8cent": (32, 1, 1), "adv2d": (32, 32, 1), "loop2d": (32, 32, 1),
         "alfven": (16, 32, 1), "otsym": (32, 32, 1)}


@pytest.mark.parametrize("name", ["adv1d", "adv2d", "loop2d", "alfven"])
def test_case_setup_matches_oracle(gpu_lib, oracle_lib, name, monkeypatch):
    """Device-built grid and IC of the new accuracy-case ICs against the oracle's (init on the device)."""
    from oracle.pyoracle import Oracle
    import helpers
    n = SMALL[name]
    monkeypatch.setitem(helpers.CASES, name, dict(helpers.CASES[name], n=n))
    okw, model, _ = case_model(name)
    o = Oracle(*n, **okw)
    with case_device(name) as g:
        for arr in ("gas", "magflux", "bxyz"):
            errs = per_var_rel(g.fetch(arr), o.get(arr))
            assert max(errs) <= 1e-12, (arr, errs)
        sc = o.scalars()
        assert abs(g.status()["dt"] - sc["dt"]) <= 1e-12 * sc["dt"]
    o.close()


def _run_to_end(name, g, stop_at=None):
    steps = 0
    t = g.status()["t"]
    while case_running(name, t) and (stop_at is None or steps < stop_at):
        _, _, t = g.step()
        steps += 1
    return steps, t


@pytest.mark.parametrize("name", list(CASES))
def test_case_on_device(gpu_lib, name):
    fx = _fixtures()[name]
    with case_device(name) as g:
        gas0, mf0 = g.fetch("gas"), g.fetch("magflux")
        steps, t = _run_to_end(name, g)
        gas1, mf1 = g.fetch("gas"), g.fetch("magflux")
        props = case_properties(name, gas0, mf0, gas1, mf1)
        for key, val in props.items():
            if key.endswith("_max"):
                continue
            assert val <= props[key + "_max"], (name, key, val, props[key + "_max"])
        # the same run as the oracle's
        assert steps == fx["steps"], (steps, fx["steps"])
        assert abs(t - fx["t"]) <= 1e-12 * abs(fx["t"])
        field = case_field(name, gas1, mf1)
        ref = np.asarray(fx["field"])
        err = float(np.max(np.abs(field - ref)) / np.max(np.abs(ref)))
        print(f"{name}: {steps} steps, {props}, fingerprint vs oracle {err:.2e}")
        assert err <= CASE_FIELD_TOL[name], (name, err)
        for key, val in props.items():
            if not key.endswith("_max") and key != "dG":
                assert abs(val - fx["properties"][key]) <= 1e-6 * max(abs(fx["properties"][key]), 1e-12), key


@pytest.mark.parametrize("name", list(CASES))
def test_case_resync_step(gpu_lib, oracle_lib, name):
    """Half-way through the device's run, one step of the device and of the oracle from the same state."""
    from oracle.pyoracle import Oracle
    okw, model, _ = case_model(name)
    fx = _fixtures()[name]
    o = Oracle(model.Nip, model.Njp, model.Nkp, **okw)
    with case_device(name) as g:
        _run_to_end(name, g, stop_at=fx["steps"] // 2)
        device_to_oracle(g, o)
        o.step()
        dt, ts, t = g.step()
        sc = o.scalars()
        assert ts == sc["ts"]
        assert abs(dt - sc["dt"]) <= TOL * sc["dt"]
        for arr in ("gas", "magflux", "bxyz"):
            errs = per_var_rel(g.fetch(arr), o.get(arr))
            assert max(errs) <= TOL, (name, arr, errs)
    o.close()
