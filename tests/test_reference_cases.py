"""The oracle on the reference's accuracy cases (tests/cases/testCases.pf) at their deck sizes.

These properties are the reference's own answers for the flux / reconstruction / constrained-transport core
of the scheme (the known-answer vectors pin only C2P/P2C and the metrics). The oracle runs testAdv1D,
testAdv1D_8CENT, testAlfven and testOTSym here, at the decks' sizes and end times, with the reference's
thresholds, and must reproduce its recorded run (tests/golden/reference_cases.json, written by
tests/golden/make_case_fixtures.py) step for step. testAdv2D and testLoop2D (256^2 to t = 1, ~6200 steps)
take several CPU minutes each, so their oracle runs are the recorded ones: their thresholds are checked on
the record here, and the device's runs are compared with the record in tests/test_reference_cases_gpu.py.
"""
import json
import os

import numpy as np
import pytest

from helpers import CASES, case_field, case_model, case_properties, case_running

HERE = os.path.dirname(os.path.abspath(__file__))
LIVE = ("adv1d", "adv1d_8cent", "otsym", "alfven")


def _fixtures():
    with open(os.path.join(HERE, "golden", "reference_cases.json")) as f:
        return json.load(f)


def _check_thresholds(name, props):
    for key, val in props.items():
        if key.endswith("_max"):
            continue
        assert val <= props[key + "_max"], (name, key, val, props[key + "_max"])


@pytest.mark.parametrize("name", LIVE)
def test_oracle_case(oracle_lib, name):
    from oracle.pyoracle import Oracle
    okw, model, _ = case_model(name)
    o = Oracle(model.Nip, model.Njp, model.Nkp, **okw)
    gas0, mf0 = o.get("gas"), o.get("magflux")
    steps = 0
    while case_running(name, o.scalars()["t"]):
        o.step()
        steps += 1
    gas1, mf1 = o.get("gas"), o.get("magflux")
    props = case_properties(name, gas0, mf0, gas1, mf1)
    _check_thresholds(name, props)
    fx = _fixtures()[name]
    assert steps == fx["steps"]
    ref = np.asarray(fx["field"])
    assert np.max(np.abs(case_field(name, gas1, mf1) - ref)) <= 1e-13 * np.max(np.abs(ref))
    o.close()


@pytest.mark.parametrize("name", [c for c in CASES if c not in LIVE])
def test_recorded_oracle_case(name):
    fx = _fixtures()[name]
    _check_thresholds(name, fx["properties"])
    assert fx["t"] == pytest.approx(CASES[name]["tFin"], abs=1e-12)


def test_every_case_recorded():
    assert set(_fixtures()) == set(CASES)
