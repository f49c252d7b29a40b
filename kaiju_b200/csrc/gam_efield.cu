// Constrained-transport electric field (fields.F90:70-232) with shared-memory staging.
//
// For each edge direction eD with transverse pair (dT1, dT2) = (J,K), (K,I), (I,J):
//  1. k_mom2face: Vf on the dT1 faces, the volume-weighted Central8 of the cell values
//     vol*rho*v/max(rho,dFloor) (precomputed once per cell by the predictor) over max(Central8(vol),TINY).
//  2. k_edge_tile: a CTA of 256 threads owns a 32 x TJ x TK tile of eD edges. It stages with cp.async
//     the stencil footprints -- along dT2: Vf, the dT1 face areas and the dT1 face field (flux/area,
//     half state for the reconstruction, n state for the limiter); along dT1: the dT2 face areas and
//     field; the 2x2 corner densities -- and evaluates GetCornerV, GetCornerD, GetCornerB (two limited
//     EdgeLRs) and the EMF for its edge from shared memory.
#include "gam_efield_tile.cuh"

namespace gam {

// ------------------------------------------------------------------ Mom2Face (fields.F90:235-285)
struct Vec3F { float* v[3]; };
// VP is Vec3P (FP64: double summands) or Vec3F (FP32-flux: float summands, summed in double)
template <typename VP>
__global__ void k_mom2face2(Lay L, GridP g, VP VdV, Vec3P Vf, Vec3F Vf32, Reg r, int dT1) {
    int i, j, k;
    if (!reg3(r, i, j, k)) return;
    long long c = L.at(i, j, k), s = L.stride(dT1);
    double sV = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        long long cn = c + (n - 4) * s;
        double w = wC8(n);
        sV = sV + w * __ldg(&g.volume[cn]);
        s0 = s0 + w * double(__ldg(&VdV.v[0][cn]));
        s1 = s1 + w * double(__ldg(&VdV.v[1][cn]));
        s2 = s2 + w * double(__ldg(&VdV.v[2][cn]));
    }
    double dV = dmax(sV, TINY);
    if (Vf32.v[0]) {   // FP32-flux path stores the face velocities as float
        Vf32.v[0][c] = float(s0 / dV); Vf32.v[1][c] = float(s1 / dV); Vf32.v[2][c] = float(s2 / dV);
        return;
    }
    Vf.v[0][c] = s0 / dV;
    Vf.v[1][c] = s1 / dV;
    Vf.v[2][c] = s2 / dV;
}


void efield_kernels_init() {
    set_edge_smem<double, double, 0>(); set_edge_smem<double, double, 1>(); set_edge_smem<double, double, 2>();
    efield_kernels_init_f32();
}

// CalcElecField (fields.F90:70-232): E = 0, then for eD = I, J, K: Mom2Face along dT1, EMF on the edges
void enqueue_efield(Handle& h, const StateP& nS, cudaStream_t st) {
    (void)nS;   // the limiter values come from the precomputed nbA planes
    const Lay& L = h.L;
    cudaMemsetAsync(h.E[0], 0, sizeof(double) * L.E * 3, st);   // E planes are contiguous in the pool
    Vec3P Vf = {{h.Vf[0], h.Vf[1], h.Vf[2]}}, VdV = {{h.VdV[0], h.VdV[1], h.VdV[2]}};
    GridP g = h.gridP();
    Vec3F Vf32{};
    EdgeSrc<double> in64;
    EdgeSrc<float> in32;
    if (h.prec == PREC_FP32FLUX) {
        const F32Planes& f = h.f32;
        for (int x = 0; x < 3; ++x) { Vf32.v[x] = f.Vf[x]; in32.Vf[x] = f.Vf[x]; }
        for (int d = 0; d < 3; ++d) {
            in32.face[d] = f.face[d]; in32.hbA[d] = f.hbA[d]; in32.nbA[d] = f.nbA[d]; in32.edge[d] = f.edge[d];
            for (int c = 0; c < 6; ++c) in32.Te[d][c] = f.Te[d][c];
            for (int c = 0; c < 4; ++c) in32.Teb[d][c] = f.Teb[d][c];
            for (int c = 0; c < 2; ++c) in32.edgB0[d][c] = f.edgB0[d][c];
        }
        in32.rho = f.rho;
    } else {
        for (int x = 0; x < 3; ++x) in64.Vf[x] = h.Vf[x];
        for (int d = 0; d < 3; ++d) {
            in64.face[d] = h.face[d]; in64.hbA[d] = h.hbA[d]; in64.nbA[d] = h.nbA[d]; in64.edge[d] = h.edge[d];
            for (int c = 0; c < 6; ++c) in64.Te[d][c] = h.Te[d][3 + c];
            for (int c = 0; c < 4; ++c) in64.Teb[d][c] = h.Teb[d][c];
            for (int c = 0; c < 2; ++c) in64.edgB0[d][c] = h.edgB0[d][c];
        }
        in64.rho = h.H.gas[0];
    }
    int is = L.is(), ie = L.ie(), js = L.js(), je = L.je(), ks = L.ks(), ke = L.ke();
    bool f32 = h.prec == PREC_FP32FLUX;
    for (int eD = 0; eD < 3; ++eD) {
        Reg rv, re;
        int dT1;
        if (eD == IDIR) {
            dT1 = JDIR;
            rv = mkreg(0, L.Ni - 1, js, je + 1, 0, L.Nk - 1);
            re = mkreg(is, ie, js, je + 1, ks, ke + 1);
        } else if (eD == JDIR) {
            dT1 = KDIR;
            rv = mkreg(0, L.Ni - 1, 0, L.Nj - 1, ks, ke + 1);
            re = mkreg(is, ie + 1, js, je, ks, ke + 1);
        } else {
            dT1 = IDIR;
            rv = mkreg(is, ie + 1, 0, L.Nj - 1, 0, L.Nk - 1);
            re = mkreg(is, ie + 1, js, je + 1, ks, ke);
        }
        dim3 bv = dT1 == 2 ? dim3(32, 1, 4) : dim3(32, 4, 1);
        if (f32) {
            Vec3F VdV32 = {{h.f32.VdV[0], h.f32.VdV[1], h.f32.VdV[2]}};
            k_mom2face2<<<grid3(rv, bv), bv, 0, st>>>(L, g, VdV32, Vf, Vf32, rv, dT1);
        } else {
            k_mom2face2<<<grid3(rv, bv), bv, 0, st>>>(L, g, VdV, Vf, Vf32, rv, dT1);
        }
        h.launches++;
        if (f32) launch_edge_dir_f32(h, in32, eD, re, st);
        else launch_edge_dir<double, double>(h, in64, eD, re, st);
    }
}

}  // namespace gam
