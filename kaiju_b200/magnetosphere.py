"""The magnetosphere problem: units, parameters and the device problem.

The Gamera part of the reference's Earth deck (tests/voltron/cmriD_Earth.xml: 7UP, pdmb 0.75, floors
1e-4 / 1e-6 nPa, Boris Ca = 10, ring averaging about the LFM axis, planet Earth) set up by
voltron/ICs/earthcmi.F90's initUser, without the Voltron coupling: the solar wind is a constant state instead
of a time series, and the ionospheric boundary sees no REMIX potential. Not carried over from the deck: the
ring-average velocity cleaning (ringknobs/doVClean) and the plasma ingestion (source/doSource, which needs
RAIJU); CalcDT's CPR stays inert because dt0 stays 0 without console output.

Units follow setMagsphere (src/gamera/apps/msphutils.F90:65-185) with getGamPlanetNorms
(src/base/planethelper.F90:96-123) and the constants of src/base/kdefs.F90 and src/base/defs/cmidefs.F90;
the wind's conversion follows readWind (src/gamera/apps/wind.F90:620-700).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import gamera as gm

# src/base/kdefs.F90
RE_CGS = 6.3781e8                    # Earth's radius [cm]
REARTH = RE_CGS * 1.0e-2             # [m]
MU0 = 4 * math.pi * 1.0e-7           # [T m / A]
KBLTZ = 1.380649e-16                 # [erg / K]
DALTON = 1.6605390666e-27            # [kg]
# src/base/defs/cmidefs.F90:19-22
DEF_D0 = DALTON * 1.0e6              # 1 amu/cc in kg/m^3
DEF_V0 = 1.0e5                       # 100 km/s in m/s
DEF_B0 = math.sqrt(MU0 * DEF_D0) * DEF_V0 * 1.0e9   # [nT]
DEF_P0 = DEF_D0 * DEF_V0 * DEF_V0 * 1.0e9            # [nPa]
EARTH_GRAV = 9.807                   # planethelper.F90:42 [m/s^2]
ERGCC2NPA = 1.0e8                    # wind.F90 readWind


@dataclass
class Magnetosphere:
    """Physical inputs of the configuration; code_params() gives the device's / oracle's GAM_NMSPH vector."""
    moment_gauss: float = 0.31       # equatorial field at r = 1: 3.1e4 nT (prob/M0 in Gauss)
    wind_density: float = 5.0        # [#/cc]
    wind_velocity: tuple = (-400.0e3, 0.0, 0.0)   # [m/s]
    wind_field: tuple = (0.0, 0.0, -5.0)          # [nT]
    wind_temperature: float = 1.0e5  # [K]
    rho0: float = 0.2                # initial density (prob/Rho0) [#/cc]
    p0: float = 0.001                # initial pressure (prob/P0) [nPa]
    dt_couple: float = 5.0           # PushIon's coupling time (voltron/coupling/dt) [s]
    rCut: float = 16.0               # cut dipole (msphutils.F90:47-50)
    lCut: float = 8.0
    dcScl: float = 4.0
    xSun: float = 20.0               # initial-field ellipse (msphutils.F90:440-444)
    xTail: float = -225.0
    yMax: float = 75.0
    sInner: float = 0.96
    nIonP: int = 1
    doIonPush: bool = True

    @property
    def gT0(self) -> float:          # time unit [s]
        return REARTH / DEF_V0

    def code_params(self) -> np.ndarray:
        gv0, gB0, gP0 = DEF_V0, DEF_B0, DEF_P0
        M0 = -self.moment_gauss * 1.0e5 / gB0
        GM0 = EARTH_GRAV * REARTH / (gv0 * gv0)
        D = self.wind_density / 1.0
        V = [v / gv0 for v in self.wind_velocity]
        B = [b / gB0 for b in self.wind_field]
        P = (1 / gP0) * D * KBLTZ * self.wind_temperature * ERGCC2NPA
        par = [M0, GM0, self.rCut, self.lCut, self.dcScl, self.xSun, self.xTail, self.yMax, self.sInner,
               D, P, V[0], V[1], V[2], B[0], B[1], B[2], float(np.float32(self.dt_couple)) / self.gT0, self.gT0,
               self.rho0, self.p0 / gP0, float(self.nIonP), 1.0 if self.doIonPush else 0.0]
        assert len(par) == 23
        return np.array(par, dtype=np.float64)


def magnetosphere_model(Nip: int = 96, Njp: int = 96, Nkp: int = 128, tFin: float = 1.0e30) -> gm.Model:
    """Model_T of the Earth deck on an LFM-type grid: 7UP, pdmb 0.75, dFloor 1e-4, pFloor 1e-6 nPa in code
    units (setMagsphere reinterprets the pressure floor in nPa), Boris Ca = 10, rings, dt over the active
    cells (initUser's DT bounds), the cut-dipole background."""
    return gm.Model(Nip, Njp, Nkp, pdmb=0.75, rmeth="7UP", dFloor=1.0e-4, pFloor=1.0e-6 / DEF_P0, doBoris=True,
                    Ca=10.0, tFin=tFin, bc=(gm.GAM_BC_ION, gm.GAM_BC_WIND, gm.GAM_BC_LFMPOLE, gm.GAM_BC_LFMPOLE,
                                            gm.GAM_BC_PERIODIC, gm.GAM_BC_PERIODIC),
                    ring=dict(recon="PPM"), dtActive=True, doBackground=True)


# The configuration's grid: r from 2 to 30 planet radii (geometric spacing), theta from 0.05 to pi - 0.05, the
# full circle in phi, about the x axis (LFM-type)
GRID = (2.0, 30.0, 1.03, 0.05)


def magnetosphere_problem(n=(96, 96, 128), ms: Magnetosphere | None = None, tFin: float = 1.0e30):
    """The device problem built on the device: grid, cut dipole, initial state, gravity, boundaries."""
    ms = ms or Magnetosphere()
    model = magnetosphere_model(*n, tFin=tFin)
    xyz = gm.corners_lfm(model, *GRID)
    return gm.GameraGPU.from_corners(model, xyz, "MAGSPHERE", ic_par=ms.code_params())
