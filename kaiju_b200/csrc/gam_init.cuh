// Device-side problem set-up: grid metrics from corners and the built-in initial conditions.
#pragma once
#include "gam_step.cuh"

namespace gam {
// Corners2Grid (src/gamera/init.F90:801-1145) from the corner planes h.xyz[3] already on the device.
int init_grid_from_corners(Handle& h);
// Initial condition ic (0 = OT2D, 1 = BW) into State n, then the end of CalcGridInfo
// (init.F90:204-244): bFlux2Fld, EnforceBCs, oState = State, CalcDT, oState%time = State%time - dt.
int init_problem(Handle& h, int ic);
}  // namespace gam
