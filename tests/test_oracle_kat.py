"""The oracle against the reference's own known answers and properties (CPU only)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
IDX = {"DEN": 0, "MOMX": 1, "MOMY": 2, "MOMZ": 3, "ENERGY": 4, "VELX": 1, "VELY": 2, "VELZ": 3, "PRESSURE": 4}


def _vec(d):
    v = np.zeros(5)
    for k, x in d.items():
        v[IDX[k]] = x
    return v


@pytest.mark.parametrize("name", sorted(KATS["gamutils"]))
def test_gamutils_known_answers(oracle_lib, name):
    """tests/gamera/testgamutils.pf: C2P/P2C and the round trips, with the reference's tolerances."""
    case = KATS["gamutils"][name]
    gamma = KATS["gamma"]
    inp = case["inputs"]
    if name == "PrimitiveToConserved":
        out = {"Con": oracle_lib.p2c(_vec(inp["Prim"]), gamma)}
    elif name == "ConservedToPrimitive":
        out = {"Prim": oracle_lib.c2p(_vec(inp["Con"]), gamma)}
    elif name == "ConservedToConserved":
        orig = _vec(inp["Con"])
        out = {"Con": oracle_lib.p2c(oracle_lib.c2p(orig, gamma), gamma), "origCon": orig}
    elif name == "PrimitiveToPrimitive":
        orig = _vec(inp["Prim"])
        out = {"Prim": oracle_lib.c2p(oracle_lib.p2c(orig, gamma), gamma), "origPrim": orig}
    else:
        pytest.skip("no restatement needed")
    assert case["checks"], name
    for chk in case["checks"]:
        got = out[chk["array"]][IDX[chk["var"]]]
        exp = chk["expect"]
        if isinstance(exp, dict):
            exp = out[exp["orig"].split("(")[0]][IDX[chk["var"]]]
        assert abs(got - exp) <= chk["tol"], (name, chk, got)


def test_metric_box_quadrature(oracle_lib):
    """tests/gamera/testmetric.pf box (1,1,1)-(2,3,4): volume 6, barycentre, face areas and centres."""
    import ctypes as C
    m = KATS["metric"]
    P = {k: np.array(v, dtype=float) for k, v in m["corners_ijk"].items()}
    order = ["111", "211", "221", "121", "112", "212", "222", "122"]   # cellCoords order (metric.F90:133-148)
    xyzC = np.ascontiguousarray(np.stack([P[k] for k in order]))
    vol = C.c_double()
    ctr = np.zeros(3)
    L = oracle_lib.lib()
    L.orc_volume_integral(oracle_lib.dptr(xyzC), C.cast(C.pointer(vol), C.POINTER(C.c_double)), oracle_lib.dptr(ctr))
    assert abs(vol.value - 6.0) < 1e-13
    np.testing.assert_allclose(ctr, m["cell_center"], rtol=0, atol=1e-13)
    for d, pts in m["face_coords"].items():
        f = [np.ascontiguousarray(np.array(p, dtype=float)) for p in pts]
        area = C.c_double()
        fc = np.zeros(3)
        L.orc_face_integral_area(*[oracle_lib.dptr(x) for x in f], C.cast(C.pointer(area), C.POINTER(C.c_double)),
                                 oracle_lib.dptr(fc))
        sides = sorted(np.ptp(np.array(pts, dtype=float), axis=0))[1:]
        assert abs(area.value - sides[0] * sides[1]) < 1e-13, d
        np.testing.assert_allclose(fc, m["face_centers"][d], rtol=0, atol=1e-13)


def test_ot_symmetry_2d(oracle_lib):
    """testOTSym (tests/cases/testCases.pf:183-225) property: OT point-reflection symmetry at round-off."""
    o = oracle_lib.Oracle(32, 32, 1, ic="OT2D", bounds=(0, 1, 0, 1, -0.5, 0.5), CFL=0.3)
    while o.scalars()["t"] < 0.1:
        o.step()
    g = o.get("gas")[4:36, 4:36, 4, :]
    gp = g[::-1, ::-1, :].copy()
    gp[..., 1:3] *= -1
    dG = np.sqrt(((g - gp) ** 2).sum(-1)).sum() / (32 * 32)
    assert dG <= 1.0e-11


def test_divb_roundoff_blast(oracle_lib):
    """Constrained transport keeps div B at round-off on the warped, non-orthogonal grid."""
    o = oracle_lib.Oracle(16, 16, 16, ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5) * 3, CFL=0.3, bc=[1] * 6)
    d0 = o.divb()
    o.step(3)
    scale = np.abs(o.get("magflux")).max() * 16 ** 3
    assert o.divb() <= 1e-12 * scale + d0


def test_mass_conservation_periodic(oracle_lib):
    """Periodic OT: total mass and energy over active cells drift only by round-off."""
    o = oracle_lib.Oracle(16, 16, 4, ic="OT2D", bounds=(0, 1, 0, 1, 0, 0.125), CFL=0.3)
    vol = o.get("volume")[4:20, 4:20, 4:8]
    m0 = (o.get("gas")[4:20, 4:20, 4:8, 0] * vol).sum()
    o.step(5)
    m1 = (o.get("gas")[4:20, 4:20, 4:8, 0] * vol).sum()
    assert abs(m1 - m0) / m0 < 1e-13


def test_rejects_short_grid(oracle_lib):
    """Corners2Grid's checks (init.F90:825-834): Nip >= 16 and a multiple of 8."""
    with pytest.raises(ValueError):
        oracle_lib.Oracle(12, 16, 4)


def test_background_dipole_is_force_free(oracle_lib):
    """AddB0 (background.F90:20-167) of a curl-free dipole: the background momentum source dpB0 and the
    net B0 flux out of every cell vanish to round-off (12-point Gauss quadrature per face)."""
    o = oracle_lib.Oracle(16, 16, 16, ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5) * 3, CFL=0.3,
                          bc=[1] * 6, b0=("dipole", 0.05, (-1.0, 0.1, 0.2)))
    a = slice(4, 20)
    b0 = o.get("b0")[a, a, a]
    bf = o.get("bflux0")
    div = (bf[5:21, a, a, 0] - bf[a, a, a, 0] + bf[a, 5:21, a, 1] - bf[a, a, a, 1] + bf[a, a, 5:21, 2] - bf[a, a, a, 2])
    assert np.abs(div).max() <= 1e-13 * np.abs(bf).max()
    scale = (b0 ** 2).sum(-1).max() * 16   # |B0|^2 / dx
    assert np.abs(o.get("dpb0")[a, a, a]).max() <= 1e-12 * scale


def test_background_uniform_equilibrium(oracle_lib):
    """Uniform gas at rest in a uniform background field with no residual field stays at rest (Cartesian
    grid: on the warped grid the non-planar faces' area vectors do not close exactly, and uniform
    pressure alone drives a small flow)."""
    o = oracle_lib.Oracle(16, 16, 16, ic="BW", grid="uniform", bounds=(-0.5, 0.5) * 3, CFL=0.3,
                          bc=[1] * 6, b0=("uniform", 0.3, -0.2, 0.5))
    gas = o.get("gas")
    gas[..., 0] = 1.0
    gas[..., 1:4] = 0.0
    gas[..., 4] = 0.1 / (5.0 / 3.0 - 1.0)
    for nm in ("gas", "ogas"):
        o.set(nm, gas)
    o.step(3)
    g = o.get("gas")
    assert np.abs(g[..., 1:4]).max() <= 1e-13
    assert np.abs(g[..., 0] - 1.0).max() <= 1e-13
    assert np.abs(o.get("magflux")).max() <= 1e-15


def test_lfm_ring_k_periodicity(oracle_lib):
    """testFields (tests/gamera/testfields.pf) on the LFM blast wave with ring averaging: after the run the
    K faces of Tf, face and magFlux, the I/J edges of Te, Teb, edge and Efld, and the cell volumes at ks
    and ke+1 agree exactly; div B stays at round-off."""
    from helpers import problem
    n = (32, 24, 64)
    okw, _ = problem("lfmbw", n)
    o = oracle_lib.Oracle(*n, **okw)
    d0 = o.divb()
    o.step(20)
    G = 4
    i0, i1, j0, j1, ks, ke = G, G + n[0] - 1, G, G + n[1] - 1, G, G + n[2] - 1
    I, J, Ip, Jp = slice(i0, i1 + 1), slice(j0, j1 + 1), slice(i0, i1 + 2), slice(j0, j1 + 2)
    for name in ("tf", "face", "magflux"):
        a = o.get(name)[..., 2]
        assert np.abs(a[I, J, ks] - a[I, J, ke + 1]).max() == 0.0, name
    for name in ("te", "teb", "edge", "efld"):
        a = o.get(name)
        assert np.abs(a[..., 0][I, Jp, ks] - a[..., 0][I, Jp, ke + 1]).max() == 0.0, name
        assert np.abs(a[..., 1][Ip, J, ks] - a[..., 1][Ip, J, ke + 1]).max() == 0.0, name
    v = o.get("volume")
    assert np.abs(v[I, J, ks] - v[I, J, ke + 1]).max() == 0.0
    scale = np.abs(o.get("magflux")).max() * n[0] * n[1] * n[2]
    assert o.divb() <= d0 + 1e-13 * scale


def test_slice_current_of_uniform_field(oracle_lib):
    """writeSlc's current of the blast wave's uniform field is zero to round-off; DivB per cell too."""
    o = oracle_lib.Oracle(16, 16, 16, ic="BW", grid="uniform", bounds=(-0.5, 0.5) * 3, CFL=0.3, bc=[1] * 6)
    s = o.slice(fat=True)
    assert max(np.abs(s[c]).max() for c in ("Jx", "Jy", "Jz")) <= 1e-12
    assert np.abs(s["DivB"]).max() <= 1e-15
    assert np.allclose(s["Bx"], 0.5 ** 0.5, rtol=1e-6) and np.allclose(s["Bz"], 0.0, atol=1e-14)
