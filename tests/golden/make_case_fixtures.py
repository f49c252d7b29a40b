"""Run the oracle on the reference's accuracy cases at their deck sizes and write tests/golden/reference_cases.json.

The cases are the property tests of the reference's tests/cases/testCases.pf (testAdv1D, testAdv1D_8CENT,
testAdv2D, testLoop2D, testAlfven, testOTSym) with their decks (tests/cases/*.xml). For each, the file holds
the oracle's step count, final time, the quantities the reference test asserts on (with its thresholds) and
a block-sum fingerprint of the final state (tests/helpers.py: case_field), so that the device's full-length
runs can be compared with the oracle's without re-running the oracle. The 256^2 cases take several minutes
of CPU each, which is why they are recorded here instead of being re-run by the CPU test suite.

usage: python tests/golden/make_case_fixtures.py [case ...]   (default: every case)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from helpers import CASES, case_field, case_model, case_properties, case_running  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402

OUT = os.path.join(HERE, "reference_cases.json")


def run_case(name):
    okw, model, _ = case_model(name)
    t0 = time.time()
    o = Oracle(model.Nip, model.Njp, model.Nkp, **okw)
    gas0, mf0 = o.get("gas"), o.get("magflux")
    steps = 0
    while case_running(name, o.scalars()["t"]):
        o.step()
        steps += 1
    gas1, mf1 = o.get("gas"), o.get("magflux")
    sc = o.scalars()
    rec = dict(steps=steps, t=sc["t"], dt_last=sc["dt"], properties=case_properties(name, gas0, mf0, gas1, mf1),
               field=case_field(name, gas1, mf1).tolist(), oracle_seconds=round(time.time() - t0, 1),
               divb=o.divb())
    o.close()
    return rec


def main(names):
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names:
        rec = run_case(name)
        print(name, rec["steps"], rec["properties"], rec["oracle_seconds"], "s", flush=True)
        data[name] = rec
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
