// Device-side problem set-up: grid metrics from corners and the built-in initial conditions.
#pragma once
#include "gam_step.cuh"

namespace gam {
// Corners2Grid (src/gamera/init.F90:801-1145) from the corner planes h.xyz[3] already on the device.
int init_grid_from_corners(Handle& h);
// A built-in background field: type 1 uniform par[0..2]; type 2 dipole of moment par[3] along z
// centred at par[0..2]; type 3 the magnetosphere's cut dipole (moment par[3] at the origin, ramped down
// beyond cut = {rCut, lCut, dcScl})
struct BgSpec { int type; double par[4]; double cut[3] = {0.0, 0.0, 1.0}; };
// the magnetosphere problem (GAM_IC_MAGSPHERE): its parameters into h.p.msph, the gravity planes and AddGrav
int msph_setup(Handle& h, const double* par, int n);
// AddB0 (src/gamera/background.F90:20-167) of bg into the background planes
int add_background(Handle& h, const BgSpec& bg);
// Initial condition ic (0 = OT2D, 1 = BW) into State n, AddB0 when bg is given, then the end of
// CalcGridInfo (init.F90:204-244): bFlux2Fld, EnforceBCs, oState = State, CalcDT,
// oState%time = State%time - dt.
// icPar: the IC's parameters (GAM_IC_KH: a, Bx, amp, seed)
int init_problem(Handle& h, int ic, const BgSpec* bg = nullptr, const double* icPar = nullptr);
}  // namespace gam
