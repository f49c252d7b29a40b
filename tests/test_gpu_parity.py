"""Device step vs the CPU oracle on identical inputs (relative L-infinity per variable <= 1e-10).

Each case builds the problem with the oracle (Hatch-equivalent set-up on the CPU), mirrors the
oracle's Grid/State arrays onto the GPU through the C ABI (gam_gpu_create), advances both by one
stepGamera and compares the intermediates (predictor half state, E field, deltas) and the final state.
Multi-step cases re-synchronise the device to the oracle before every step so chaotic growth of
round-off differences does not mask kernel errors.
"""
import numpy as np
import pytest

from helpers import oracle_and_gpu, per_var_rel, rel_linf, resync

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _cmp(o, g, names, tol=TOL, where=""):
    for name in names:
        a, b = g.fetch(name), o.get(name)
        errs = per_var_rel(a, b)
        assert max(errs) <= tol, f"{where}{name}: {errs}"


CASES = [
    ("ot3d", "ot", (32, 32, 4), {}),
    ("ot25d", "ot", (32, 32, 1), {}),
    ("bw_warp", "bw", (32, 16, 16), {}),
    ("bw_7up", "bw", (32, 16, 16), dict(rmeth="7UP", pdmb=4.0)),
    ("bw_hydro", "bw", (16, 16, 16), dict(doMHD=False)),
    ("bw_boris", "bw", (16, 16, 16), dict(doBoris=True, Ca=2.0)),
    ("ot_nolfmlim", "ot", (32, 32, 4), dict(doLFMLim=False)),
    # background field: the blast-wave field held entirely as a uniform B0 (residual field starts at 0)
    ("bw_bg_uniform", "bw", (32, 16, 16), dict(b0=("uniform", 0.5 ** 0.5, 0.5 ** 0.5, 0.0))),
    # a dipole background centred off the domain on top of the blast-wave field, with Boris
    ("bw_bg_dipole", "bw", (32, 16, 16), dict(b0=("dipole", 0.05, (-1.0, 0.1, 0.2)))),
    ("bw_bg_dipole_boris", "bw", (16, 16, 16), dict(b0=("dipole", 0.05, (-1.0, 0.1, 0.2)), doBoris=True, Ca=2.0)),
    # LFM-type spherical grid with ring averaging about the axis, the axis BCs and the LFM blast wave's
    # fixed shells and predictor fix (the reference's lfmbw test problem)
    ("lfmbw", "lfmbw", (32, 24, 64), {}),
    # the spherical configuration's physics together: LFM grid, rings, axis BCs, Boris, and a dipole
    # background centred on the grid's axis (the magnetosphere-like set-up without its wind/ionosphere BCs)
    ("lfmbw_dipole", "lfmbw", (32, 24, 64), dict(b0=("dipole", 2000.0))),
]


@pytest.mark.parametrize("name,kind,n,kw", CASES, ids=[c[0] for c in CASES])
def test_one_step_intermediates(gpu_lib, oracle_lib, name, kind, n, kw):
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu(kind, n, **kw)
    with g:
        g.set_tile(gm.GAM_TILE_FUSED_UPDATE, 0)   # keep the dGasH/dGasM planes for inspection
        # inputs mirrored exactly
        _cmp(o, g, ["gas", "magflux", "bxyz", "ogas", "omagflux"], tol=0.0, where="input ")
        o.step()
        dt, ts, t = g.step()
        sc = o.scalars()
        assert ts == sc["ts"] == 1
        assert abs(dt - sc["dt"]) <= TOL * sc["dt"]
        assert abs(t - sc["t"]) <= TOL * abs(sc["t"])
        inter = ["hgas"]
        if kw.get("doMHD", True):
            inter += ["hmagflux", "hbxyz", "efld"]
        _cmp(o, g, inter, where=f"{name} ")
        # deltas: judge the increment dt*dGasH (dt*dGasM) against the size of the state it updates;
        # a delta that is zero in exact arithmetic (OT's initial dRho/dt) carries only round-off
        gas0 = o.get("ogas")
        dts = sc["time"] - sc["otime"]   # the dt this step used
        gmax = np.abs(gas0).reshape(-1, 5, order="F").max(0)
        # momentum scale: the larger of the momenta present and sqrt(rho*E), the momentum the cell would
        # carry were its energy all kinetic (the blast wave starts at rest)
        mscale = max(gmax[1:4].max(), np.sqrt(gmax[0] * gmax[4]))
        for nm, ref_scale in (("dgash", np.array([gmax[0], mscale, mscale, mscale, gmax[4]])),
                              ("dgasm", np.full(3, mscale))):
            if nm == "dgasm" and not kw.get("doMHD", True):
                continue
            a, b = g.fetch(nm), o.get(nm)
            nv = a.shape[-1]
            for v in range(nv):
                err = np.abs(a[..., v] - b[..., v]).max() * dts / ref_scale[v]
                assert err <= TOL, (name, nm, v, err)
        _cmp(o, g, ["gas", "magflux", "bxyz"], where=f"{name} ")


@pytest.mark.parametrize("name,kind,n,kw", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_resynced_steps(gpu_lib, oracle_lib, name, kind, n, kw):
    o, g = oracle_and_gpu(kind, n, **kw)
    with g:
        for s in range(6):
            o.step()
            dt, ts, t = g.step()
            sc = o.scalars()
            assert abs(dt - sc["dt"]) <= TOL * sc["dt"], (s, dt, sc["dt"])
            _cmp(o, g, ["gas", "magflux"], where=f"step {s} ")
            resync(o, g)


def test_free_running_trajectory(gpu_lib, oracle_lib):
    """Without re-synchronisation the trajectories stay together to near round-off over 20 steps."""
    o, g = oracle_and_gpu("bw", (32, 16, 16))
    with g:
        o.step(20)
        g.run_steps(20)
        st = g.status()
        assert st["ts"] == 20
        for v, e in enumerate(per_var_rel(g.fetch("gas"), o.get("gas"))):
            assert e < 1e-8, (v, e)


def test_divb_roundoff(gpu_lib, oracle_lib):
    o, g = oracle_and_gpu("bw", (32, 16, 16))
    with g:
        g.run_steps(10)
        mf = g.fetch("magflux")
        scale = np.abs(mf).max() * 32 * 16 * 16
        assert g.divb() <= 1e-12 * scale


def test_device_grid_matches_oracle(gpu_lib, oracle_lib):
    """Corners2Grid + IC + Hatch tail on the device vs the oracle's host set-up, same corners."""
    from helpers import problem
    from kaiju_b200 import gamera as gm
    for kind, n in (("bw", (32, 16, 16)), ("ot", (32, 32, 4))):
        okw, model = problem(kind, n)
        o = oracle_lib.Oracle(*n, **okw)
        xyz = o.get("xyz")
        with gm.GameraGPU.from_corners(model, xyz, "BW" if kind == "bw" else "OT2D") as g:
            for name in ("volume", "xyzcc", "xfc", "face", "edge", "di", "dj", "dk", "tf", "te", "teb"):
                errs = per_var_rel(g.fetch(name), o.get(name))
                assert max(errs) <= 1e-12, (kind, name, errs)
            for name in ("gas", "magflux", "bxyz"):
                errs = per_var_rel(g.fetch(name), o.get(name))
                assert max(errs) <= 1e-12, (kind, name, errs)
            st = g.status()
            sc = o.scalars()
            assert abs(st["dt"] - sc["dt"]) <= 1e-12 * sc["dt"]
            assert abs(st["otime"] - sc["otime"]) <= 1e-12 * sc["dt"]


def test_fp32_flux_error(gpu_lib, oracle_lib):
    """FP32 reconstruction/limiter/fluxes, FP64 state: L1 error against the FP64 oracle after 10 steps."""
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (32, 16, 16))
    with g:
        g.set_precision(gm.GAM_FP32FLUX)
        o.step(10)
        g.run_steps(10)
        a, b = g.fetch("gas")[4:36, 4:20, 4:20], o.get("gas")[4:36, 4:20, 4:20]
        for v in range(5):
            l1 = np.abs(a[..., v] - b[..., v]).sum() / np.abs(b[..., v]).sum() if np.abs(b[..., v]).sum() > 0 else \
                np.abs(a[..., v]).mean()
            assert l1 <= 1e-5, (v, l1)


@pytest.mark.parametrize("b0", [("uniform", 0.5 ** 0.5, 0.5 ** 0.5, 0.0), ("dipole", 0.05, (-1.0, 0.1, 0.2))],
                         ids=["uniform", "dipole"])
def test_device_background_matches_oracle(gpu_lib, oracle_lib, b0):
    """AddB0 on the device (12x12 face, 12 edge, 12^3 volume quadrature of the built-in B0) vs the
    oracle's host AddB0 on the same corners; then two steps of the background-field scheme."""
    from helpers import problem
    from kaiju_b200 import gamera as gm
    n = (32, 16, 16)
    okw, model = problem("bw", n, b0=b0)
    o = oracle_lib.Oracle(*n, **okw)
    with gm.GameraGPU.from_corners(model, o.get("xyz"), "BW", b0=b0) as g:
        b0c = o.get("b0")
        scale = float((b0c ** 2).sum(-1).max()) * n[0]   # |B0|^2 / dx: the size of a stress divergence
        for name in ("fcb0", "edgb0", "b0", "bflux0"):
            errs = per_var_rel(g.fetch(name), o.get(name))
            assert max(errs) <= 1e-12, (name, errs)
        assert np.abs(g.fetch("dpb0") - o.get("dpb0")).max() <= 1e-12 * scale
        for name in ("gas", "magflux", "bxyz"):
            a, b = g.fetch(name), o.get(name)
            if np.abs(b).max() == 0.0:
                assert np.abs(a).max() == 0.0, name
            else:
                assert max(per_var_rel(a, b)) <= 1e-12, name
        sc = o.scalars()
        assert abs(g.status()["dt"] - sc["dt"]) <= 1e-12 * sc["dt"]
        o.step(2)
        g.run_steps(2)
        _cmp(o, g, ["gas"], tol=1e-9, where="after 2 steps ")


def test_fp32_flux_error_background(gpu_lib, oracle_lib):
    """FP32-flux path with a dipole background (float copies of fcB0, bFlux0/face, edgB0)."""
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (32, 16, 16), b0=("dipole", 0.05, (-1.0, 0.1, 0.2)))
    with g:
        g.set_precision(gm.GAM_FP32FLUX)
        o.step(10)
        g.run_steps(10)
        a, b = g.fetch("gas")[4:36, 4:20, 4:20], o.get("gas")[4:36, 4:20, 4:20]
        for v in range(5):
            den = np.abs(b[..., v]).sum()
            l1 = np.abs(a[..., v] - b[..., v]).sum() / den if den > 0 else np.abs(a[..., v]).mean()
            assert l1 <= 1e-5, (v, l1)


def test_lfmbw_resynced_steps(gpu_lib, oracle_lib):
    """Ring averaging, axis BCs and the LFM blast wave's shells over re-synchronised steps."""
    o, g = oracle_and_gpu("lfmbw", (32, 24, 64))
    with g:
        for s in range(4):
            o.step()
            dt, ts, t = g.step()
            sc = o.scalars()
            assert abs(dt - sc["dt"]) <= TOL * sc["dt"], (s, dt, sc["dt"])
            _cmp(o, g, ["gas", "magflux", "bxyz", "efld"], where=f"step {s} ")
            resync(o, g)


def test_lfmbw_k_periodicity(gpu_lib, oracle_lib):
    """The reference's testFields (tests/gamera/testfields.pf) on the device run: after free-running steps
    the K faces of magFlux and the I/J edges of Efld at ks and ke+1 agree exactly, and the trajectory
    follows the oracle's."""
    o, g = oracle_and_gpu("lfmbw", (32, 24, 64))
    Ni, Nj, Nk, G = 32, 24, 64, 4
    i0, i1, j0, j1, ks, ke = G, G + Ni - 1, G, G + Nj - 1, G, G + Nk - 1
    with g:
        o.step(10)
        g.run_steps(10)
        mf, e = g.fetch("magflux"), g.fetch("efld")
        assert np.abs(mf[i0:i1 + 1, j0:j1 + 1, ks, 2] - mf[i0:i1 + 1, j0:j1 + 1, ke + 1, 2]).max() == 0.0
        assert np.abs(e[i0:i1 + 1, j0:j1 + 2, ks, 0] - e[i0:i1 + 1, j0:j1 + 2, ke + 1, 0]).max() == 0.0
        assert np.abs(e[i0:i1 + 2, j0:j1 + 1, ks, 1] - e[i0:i1 + 2, j0:j1 + 1, ke + 1, 1]).max() == 0.0
        for v, err in enumerate(per_var_rel(g.fetch("gas"), o.get("gas"))):
            assert err < 1e-8, (v, err)


def test_device_lfm_grid_matches_oracle(gpu_lib, oracle_lib):
    """Corners2Grid with RingGridFix, the LFM blast-wave IC and the Hatch tail on the device vs the oracle's
    host set-up, same corners."""
    from helpers import problem
    from kaiju_b200 import gamera as gm
    n = (32, 24, 64)
    okw, model = problem("lfmbw", n)
    o = oracle_lib.Oracle(*n, **okw)
    with gm.GameraGPU.from_corners(model, o.get("xyz"), "LFMBW") as g:
        for name in ("volume", "xyzcc", "xfc", "face", "edge", "di", "dj", "dk", "tf", "te", "teb",
                     "gas", "magflux", "bxyz"):
            errs = per_var_rel(g.fetch(name), o.get(name))
            assert max(errs) <= 1e-12, (name, errs)
        sc = o.scalars()
        assert abs(g.status()["dt"] - sc["dt"]) <= 1e-12 * sc["dt"]
        o.step(2)
        g.run_steps(2)
        _cmp(o, g, ["gas", "magflux"], tol=1e-9, where="after 2 steps ")


def test_lfm_dipole_fp32_flux_l1(gpu_lib, oracle_lib):
    """FP32-flux path on the spherical set-up (LFM grid, rings, Boris, dipole background): L1 error of the
    state after re-synchronised steps within the FP32 path's 1e-5 bound."""
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("lfmbw", (32, 24, 64), b0=("dipole", 2000.0))
    with g:
        g.set_precision(gm.GAM_FP32FLUX)
        for s in range(3):
            o.step()
            g.step()
            a, b = g.fetch("gas"), o.get("gas")
            for v in range(5):
                l1 = np.abs(a[..., v] - b[..., v]).mean() / np.abs(b[..., v]).mean()
                assert l1 <= 1e-5, (s, v, l1)
            resync(o, g)


@pytest.mark.parametrize("prec", ["fp64", "fp32flux"])
def test_fused_update_equals_separate_deltas(gpu_lib, oracle_lib, prec):
    """The update computing Flux2Deltas itself gives bit-identical states to the separate kernel."""
    from kaiju_b200 import gamera as gm
    for kw in ({}, dict(doBoris=True, Ca=2.0)):
        o, a = oracle_and_gpu("bw", (32, 16, 16), **kw)
        _, b = oracle_and_gpu("bw", (32, 16, 16), **kw)
        with a, b:
            if prec == "fp32flux":
                a.set_precision(gm.GAM_FP32FLUX)
                b.set_precision(gm.GAM_FP32FLUX)
            b.set_tile(gm.GAM_TILE_FUSED_UPDATE, 0)
            a.run_steps(5)
            b.run_steps(5)
            for name in ("gas", "magflux", "bxyz"):
                assert np.array_equal(a.fetch(name), b.fetch(name)), (kw, name)


@pytest.mark.parametrize("prec", ["fp64", "fp32flux"])
@pytest.mark.parametrize("name", ["bw_warp", "bw_hydro", "bw_7up", "ot25d", "lfmbw_dipole"])
def test_tma_staging_equals_cp_async(gpu_lib, oracle_lib, name, prec):
    """The flux and E-field kernels' footprints staged by tensor copies (one thread per tile) give
    bit-identical states to per-element cp.async staging: the widened boxes along i, the J/K boxes, hydro
    (no B planes), the 2.5D slab and a background field on the LFM grid."""
    from kaiju_b200 import gamera as gm
    _, kind, n, kw = next(c for c in CASES if c[0] == name)
    o, a = oracle_and_gpu(kind, n, **kw)
    _, b = oracle_and_gpu(kind, n, **kw)
    with a, b:
        if prec == "fp32flux":
            a.set_precision(gm.GAM_FP32FLUX)
            b.set_precision(gm.GAM_FP32FLUX)
        b.set_tile(gm.GAM_TILE_TMA, 0)
        a.run_steps(4)
        b.run_steps(4)
        assert a.status()["status"] == 0
        for nm in ("gas", "magflux", "bxyz"):
            assert np.array_equal(a.fetch(nm), b.fetch(nm)), (name, prec, nm)

