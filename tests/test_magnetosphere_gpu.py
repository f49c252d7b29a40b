"""The magnetosphere problem on the device against the oracle (relative L-infinity <= 1e-10 per variable).

The Earth deck's Gamera part with a constant solar wind and no ionospheric coupling, on a small LFM-type grid
(r from 2 to 30, rings about the axis): the device's own set-up (cut-dipole background, elliptically cut
initial field, uniform gas, gravity) against the oracle's; one step from the oracle's state through every hook
(EFix with IonEFix/WindEFix/DiffuseOuter/FixEFieldLFM, IonFlux, gravity, PushIon and NudgeSW, the ionospheric
and solar-wind boundaries), intermediates included; re-synchronised steps; and the FP32-flux path's L1 error.
"""
import numpy as np
import pytest

from helpers import BACKGROUND_NAMES, oracle_and_gpu, per_var_rel, problem, resync

pytestmark = pytest.mark.gpu
TOL = 1e-10
N = (32, 24, 16)


def _params():
    from kaiju_b200 import magnetosphere as ms
    return ms.Magnetosphere().code_params()


def test_device_setup_matches_oracle(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm, magnetosphere as ms
    from oracle.pyoracle import Oracle
    okw, model = problem("msph", N)
    o = Oracle(*N, **okw)
    with ms.magnetosphere_problem(N) as g:
        for name in ("gas", "magflux", "bxyz") + BACKGROUND_NAMES:
            errs = per_var_rel(g.fetch(name), o.get(name))
            assert max(errs) <= 1e-12, (name, errs)
        assert abs(g.status()["dt"] - o.scalars()["dt"]) <= 1e-12 * o.scalars()["dt"]
    o.close()


def _mirrored(**kw):
    o, g = oracle_and_gpu("msph", N, **kw)
    g.set_magnetosphere(_params())
    return o, g


def test_one_step_with_hooks(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    o, g = _mirrored()
    with g:
        g.set_tile(gm.GAM_TILE_FUSED_UPDATE, 0)
        o.step()
        dt, ts, t = g.step()
        sc = o.scalars()
        assert ts == sc["ts"] == 1 and abs(dt - sc["dt"]) <= TOL * sc["dt"]
        for name in ("hgas", "hmagflux", "efld", "gas", "magflux", "bxyz"):
            errs = per_var_rel(g.fetch(name), o.get(name))
            assert max(errs) <= TOL, (name, errs)
    o.close()


def test_resynced_steps(gpu_lib, oracle_lib):
    o, g = _mirrored()
    with g:
        for s in range(8):
            o.step()
            g.step()
            for name in ("gas", "magflux", "bxyz"):
                errs = per_var_rel(g.fetch(name), o.get(name))
                assert max(errs) <= TOL, (s, name, errs)
            resync(o, g)
    o.close()


def test_fp32_flux_error(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    o, g = _mirrored()
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
    o.close()
