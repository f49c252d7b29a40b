"""Extract the known-answer vectors of the reference's GAMERA unit tests into reference_kats.json.

Reads, as text, tests/gamera/testgamutils.pf (C2P/P2C known answers with their tolerances) and
tests/gamera/testmetric.pf (the unit box (1,1,1)-(2,3,4) and its cell/face/edge/corner answers) from a
kaiju checkout. Run once where the reference tree is available:

    python tests/golden/make_golden.py <kaiju checkout>

The JSON it writes is committed; the tests read only the JSON.
"""
import json
import os
import re
import sys

NUM = r"([-+]?\d+\.?\d*(?:[eEdD][-+]?\d+)?)(?:_rp|_dp)?"


def fnum(s: str) -> float:
    s = s.replace("_rp", "").replace("_dp", "")
    if "/" in s:
        a, b = s.split("/")
        return fnum(a) / fnum(b)
    return float(s.replace("d", "e").replace("D", "e"))


def parse_gamutils(text: str):
    out = {}
    blocks = re.split(r"@test\s*\n\s*subroutine\s+", text)[1:]
    for b in blocks:
        name = b.split("(")[0].strip()
        assigns = {}
        for m in re.finditer(r"(Prim|Con|CON)\((DEN|MOMX|MOMY|MOMZ|VELX|VELY|VELZ|PRESSURE|ENERGY)\)\s*=\s*([^\n!]+)", b):
            arr = m.group(1).capitalize()
            assigns.setdefault(arr, {})[m.group(2)] = fnum(m.group(3).strip())
        checks = []
        for m in re.finditer(r"@assertLessThanOrEqual\(abs\((\w+)\((\w+)\)\s*-\s*([^,]+?)\),\s*([^,]+?),", b):
            expect = m.group(3).strip()
            if expect.startswith("orig"):
                exp_val = {"orig": expect}
            else:
                exp_val = fnum(expect.strip("()"))
            checks.append({"array": m.group(1), "var": m.group(2), "expect": exp_val, "tol": fnum(m.group(4))})
        out[name] = {"inputs": assigns, "checks": checks}
    return out


def parse_metric(text: str):
    pts = {}
    for m in re.finditer(r"testGrid%xyz\((\d),(\d),(\d),(XDIR|YDIR|ZDIR)\)\s*=\s*(\S+?);", text):
        key = f"{m.group(1)}{m.group(2)}{m.group(3)}"
        pts.setdefault(key, [0.0, 0.0, 0.0])["XYZ".index(m.group(4)[0])] = float(m.group(5))
    centre = [float(x) for x in re.search(r"xc - ([\d.]+),.*\n.*yc - ([\d.]+),.*\n.*zc - ([\d.]+),", text).groups()]
    return {"corners_ijk": pts, "cell_center": centre, "face_coords": {
        "IDIR": [[1, 1, 1], [1, 3, 1], [1, 1, 4], [1, 3, 4]],
        "JDIR": [[1, 1, 1], [1, 1, 4], [2, 1, 1], [2, 1, 4]],
        "KDIR": [[1, 1, 1], [2, 1, 1], [1, 3, 1], [2, 3, 1]]},
        "face_centers": {"IDIR": [1, 2, 2.5], "JDIR": [1.5, 1, 2.5], "KDIR": [1.5, 2, 1]},
        "edge_coords": {"IDIR": [[1, 1, 1], [2, 1, 1]], "JDIR": [[1, 1, 1], [1, 3, 1]], "KDIR": [[1, 1, 1], [1, 1, 4]]}}


def main(root: str):
    g = open(os.path.join(root, "tests", "gamera", "testgamutils.pf")).read()
    m = open(os.path.join(root, "tests", "gamera", "testmetric.pf")).read()
    data = {"source": {"gamutils": "tests/gamera/testgamutils.pf", "metric": "tests/gamera/testmetric.pf"},
            "gamma": 5.0 / 3.0, "gamutils": parse_gamutils(g), "metric": parse_metric(m)}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_kats.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
