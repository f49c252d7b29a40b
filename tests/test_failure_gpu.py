"""Failure detection of the device step, driven by host-made failures (no GPU fault, trap or hang).

The reference detects failures in CalcDT (src/gamera/step.F90:96-168): a NaN timestep, a timestep that
dropped 10x or below limDT0 of the initial one (isBad), or one below TINY (isDisaster), after which it
calls BlackBox and stops. The device step reports the same conditions as status codes:
  * a NaN poisoned into State on the host gives GAM_ERR_NAN with the NaN cells counted;
  * negative pressure or density in State is floored in C2P (pFloor/dFloor), as in the reference; a density
    floored to TINY collapses the next dt, which CalcDT flags as isBad on both sides; the floored step itself
    is checked against the oracle's;
  * a forced dt collapse (dt0 set so that dtMin/dt0 <= limDT0) gives GAM_ERR_DT_COLLAPSE, as the oracle's
    isBad;
  * the flux and E-field kernels' bounded wait on their staged tiles, made to give up at once
    (GAM_TILE_STAGE_WAIT = 0), gives GAM_ERR_TIMEOUT; the CTAs still let their own copies land before
    exiting, and the same handle steps normally again once the bound is restored.
"""
import numpy as np
import pytest

from helpers import oracle_and_gpu, per_var_rel, resync

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _push_state(o, g, gas):
    sc = o.scalars()
    g.sync_to_device(gas=gas, magflux=o.get("magflux"), ogas=o.get("ogas"), omagflux=o.get("omagflux"),
                     time=sc["time"], otime=sc["otime"], bxyz=o.get("bxyz"), obxyz=o.get("obxyz"))
    g.set_scalars(sc["t"], sc["dt"], sc["dt0"], sc["ts"], sc["time"], sc["otime"])


def test_nan_state_reports_nan(gpu_lib, oracle_lib):
    """A NaN momentum reaches CellDT as a NaN speed. (A NaN energy or density would not: the C2P floors,
    max(P, pFloor) and max(rho, dFloor), replace a NaN by the floor, in the reference as on the device.)"""
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (16, 16, 16))
    with g:
        gas = o.get("gas")
        gas[10, 9, 8, 1] = np.nan   # one active cell's x momentum
        _push_state(o, g, gas)
        with pytest.raises(gm.GamError) as err:
            g.step()
        assert err.value.code == gm.GAM_ERR_NAN
        assert g.status()["nanCells"] > 0
    o.close()


@pytest.mark.parametrize("what", ["pressure", "density"])
def test_negative_state_is_floored_like_the_oracle(gpu_lib, oracle_lib, what):
    """Negative pressure or density is floored in C2P. A density floored to dFloor = TINY makes that cell's
    sound speed, and so CalcDT's next dt, collapse: the reference's isBad (a 10x drop), reported by the
    device as GAM_ERR_DT_COLLAPSE after completing the step, as the oracle flags it."""
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (16, 16, 16))
    with g:
        gas = o.get("gas")
        if what == "pressure":   # energy below the kinetic energy: P < 0 before the floor
            gas[10, 9, 8, 4] = -0.5 * abs(gas[10, 9, 8, 4])
        else:
            gas[10, 9, 8, 0] = -abs(gas[10, 9, 8, 0])
        o.set("gas", gas)
        _push_state(o, g, gas)
        o.step()
        bad = o.scalars()["status"] & 3
        if bad:
            with pytest.raises(gm.GamError) as err:
                g.step()
            assert err.value.code == gm.GAM_ERR_DT_COLLAPSE
        else:
            g.step()
        assert bool(bad) == (what == "density")
        for name in ("gas", "magflux"):
            errs = per_var_rel(g.fetch(name), o.get(name))
            assert max(errs) <= TOL, (what, name, errs)
    o.close()


def test_dt_collapse_reports_like_calcdt(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (16, 16, 16))
    with g:
        o.step()
        resync(o, g)
        sc = o.scalars()
        dt0 = sc["dt"] / 1.0e-4   # dtMin/dt0 ~ 1e-4 <= limDT0 = 1e-3
        o.set_scalars(sc["t"], sc["dt"], dt0, sc["time"], sc["otime"], sc["ts"])
        g.set_scalars(sc["t"], sc["dt"], dt0, sc["ts"], sc["time"], sc["otime"])
        o.step()
        assert o.scalars()["status"] & 2   # the oracle's isBad
        with pytest.raises(gm.GamError) as err:
            g.step()
        assert err.value.code == gm.GAM_ERR_DT_COLLAPSE
    o.close()


def test_staging_wait_timeout_is_reported_and_recoverable(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    o, g = oracle_and_gpu("bw", (32, 16, 16))
    with g:
        g.set_tile(gm.GAM_TILE_STAGE_WAIT, 0)
        with pytest.raises(gm.GamError) as err:
            g.step()
        assert err.value.code == gm.GAM_ERR_TIMEOUT
        rc = g.run_steps(2, check=False)   # graph-replayed steps report it too
        assert rc == gm.GAM_ERR_TIMEOUT
        g.set_tile(gm.GAM_TILE_STAGE_WAIT, 1)
        resync(o, g)   # the timed-out steps' state is not valid; start again from the oracle's
        o.step()
        g.step()
        for name in ("gas", "magflux"):
            assert max(per_var_rel(g.fetch(name), o.get(name))) <= TOL
    o.close()
