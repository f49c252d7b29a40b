"""The oracle's magnetosphere problem (the Earth deck's Gamera part with a constant solar wind and no
ionospheric coupling): properties its set-up and boundaries must have by construction.

* The cut dipole (apps/msphutils.F90:561-579) is the dipole itself inside rCut, so the background's cell
  average there follows 1/r^3 with the moment M0, and the initial residual field (the elliptically cut
  dipole's vector-potential fluxes minus the background's face fluxes) is quadrature-small inside both cuts.
* WindBC (apps/wind.F90:206-374): on the sunward side (weight 1) the outer ghost cells hold the wind's state.
* IonInner (voltron/ICs/earthcmi.F90:378-522) with no ionospheric E field: the inner ghosts carry the mirrored
  active cell's density and pressure at rest, their faces no residual flux.
* div B stays at round-off and the wind brings mass in.
"""
import numpy as np
import pytest

from helpers import problem

N = (32, 24, 16)


@pytest.fixture(scope="module")
def msph(oracle_lib):
    from oracle.pyoracle import Oracle
    okw, model = problem("msph", N)
    o = Oracle(*N, **okw)
    yield o, okw, model
    o.close()


def test_cut_dipole_background(msph):
    from kaiju_b200 import magnetosphere as ms
    o, okw, model = msph
    M0 = ms.Magnetosphere().code_params()[0]
    xc, B0 = o.get("xyzcc"), o.get("b0")
    a = (slice(4, 4 + N[0]), slice(4, 4 + N[1]), slice(4, 4 + N[2]))
    r = np.sqrt(np.sum(xc[a] ** 2, axis=-1))
    inner = r < 6.0
    bmag = np.sqrt(np.sum(B0[a] ** 2, axis=-1))
    # a dipole's |B| lies between |M0|/r^3 (equator) and 2|M0|/r^3 (pole)
    ratio = bmag[inner] * r[inner] ** 3 / abs(M0)
    assert ratio.min() > 0.95 and ratio.max() < 2.05
    # the initial residual field inside both cuts is the difference of two quadratures of the same dipole
    mf, bf0 = o.get("magflux"), o.get("bflux0")
    res = np.abs(mf[a][inner]).max()
    assert res <= 1e-6 * np.abs(bf0[a][inner]).max()


def test_wind_and_ionosphere_ghosts(msph):
    from kaiju_b200 import magnetosphere as ms
    o, okw, model = msph
    par = ms.Magnetosphere().code_params()
    o.step(3)
    gas, xc = o.get("gas"), o.get("xyzcc")
    ie = 4 + N[0] - 1
    # sunward outer ghosts (the wind's weight is 1 where the angle to -V is at most 90 degrees)
    gh = gas[ie + 1, 4:4 + N[1], 4:4 + N[2], :]
    x = xc[ie + 1, 4:4 + N[1], 4:4 + N[2], 0]
    sun = x > 0
    assert sun.any()
    D, P, Vx = par[9], par[10], par[11]
    np.testing.assert_allclose(gh[sun][:, 0], D, rtol=1e-14)
    np.testing.assert_allclose(gh[sun][:, 1], D * Vx, rtol=1e-14)
    kin = 0.5 * D * Vx * Vx
    np.testing.assert_allclose(gh[sun][:, 4], kin + P / (model.gamma - 1), rtol=1e-13)
    # inner ghosts: the mirrored active cell's density at rest, no residual face flux
    is_ = 4
    for n in range(1, 5):
        ig, ip = is_ - n, is_ + n - 1
        np.testing.assert_array_equal(gas[ig, 4:4 + N[1], 4:4 + N[2], 0], gas[ip, 4:4 + N[1], 4:4 + N[2], 0])
        assert np.all(gas[ig, 4:4 + N[1], 4:4 + N[2], 1:4] == 0.0)
    mf = o.get("magflux")
    assert np.all(mf[:is_, :, :, :] == 0.0)


def test_divb_and_inflow(msph):
    o, okw, model = msph
    vol = o.get("volume")
    a = (slice(4, 4 + N[0]), slice(4, 4 + N[1]), slice(4, 4 + N[2]))
    m0 = float(np.sum(o.get("gas")[a][..., 0] * vol[a]))
    o.step(5)
    m1 = float(np.sum(o.get("gas")[a][..., 0] * vol[a]))
    assert m1 > m0
    assert np.isfinite(o.get("gas")).all()
    flux_scale = float(np.abs(o.get("magflux")).max() + np.abs(o.get("bflux0")).max()) * np.prod(N)
    assert o.divb() <= 1e-12 * flux_scale
