// Constrained-transport electric field (fields.F90:70-232) with shared-memory staging.
//
// For each edge direction eD with transverse pair (dT1, dT2) = (J,K), (K,I), (I,J):
//  1. Vf on the dT1 faces, the volume-weighted Central8 of the cell values vol*rho*v/max(rho,dFloor)
//     (precomputed once per cell by the predictor) over max(Central8(vol),TINY) -- one pass,
//     k_mom2face3, for all three directions.
//  2. k_edge_tile: a CTA of 256 threads owns a 32 x TJ x TK tile of eD edges. It stages (TMA tensor copies,
//     or cp.async) the stencil footprints -- along dT2: Vf, the dT1 face areas and the dT1 face field
//     (flux/area, half state for the reconstruction, n state for the limiter); along dT1: the dT2 face
//     areas and field; the 2x2 corner densities -- and evaluates GetCornerV, GetCornerD, GetCornerB (two
//     limited EdgeLRs) and the EMF for its edge from shared memory.
#include "gam_efield_tile.cuh"

namespace gam {

// ------------------------------------------------------------------ Mom2Face (fields.F90:235-285)
struct Vec3F { float* v[3]; };
// Vf at one face (explicit fused multiply-adds): the Central8 sums along dT1 of the summands
// vol*rho*v/max(rho,dFloor) over the Central8 sum of the volumes (clamped at TINY). A is the accumulation type: double on the FP64 path, float on the
// FP32-flux path, whose summands and volumes are float copies and whose Vf is stored as float.
template <typename A>
__device__ __forceinline__ void mom2face_sum(const A* wV, const A* w0, const A* w1, const A* w2, A& f0, A& f1, A& f2) {
    A sV = A(0), s0 = A(0), s1 = A(0), s2 = A(0);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        A w = A(wC8(n));
        sV = fma(w, wV[n], sV);
        s0 = fma(w, w0[n], s0);
        s1 = fma(w, w1[n], s1);
        s2 = fma(w, w2[n], s2);
    }
    const A idV = A(1) / (sV > A(TINY) ? sV : A(TINY));   // one reciprocal for the three quotients
    f0 = s0 * idV; f1 = s1 * idV; f2 = s2 * idV;
}

// All three Mom2Face directions in one pass over the cells: a thread reads its cell's stencils along i, j
// and k (neighbouring threads share them through the caches) and writes the face velocities of every
// direction whose region holds the cell, so the volumes and summands cross HBM once instead of three
// times. out.v[eD]: the three component planes the edges of direction eD read (dT1 = J, K, I for
// eD = I, J, K). Against three one-direction passes (the J/K ones with register windows along dT1) it
// measured the same in FP64 and slightly faster in FP32, with two launches fewer per step.
template <typename A> struct Vf9 { A* v[3][3]; };

template <typename A, typename VS, typename GS>
__global__ void k_mom2face3(Lay L, const GS* vol, VS v0, VS v1, VS v2, Vf9<A> out, Reg rI, Reg rJ, Reg rK) {
    int i, j, k;
    if (!reg_plane(Reg{0, L.Ni, 0, L.Nj, 0, L.Nk}, i, j, k)) return;
    const long long c = L.at(i, j, k);
    auto in = [&](const Reg& r) {
        return i >= r.i0 && i < r.i0 + r.ni && j >= r.j0 && j < r.j0 + r.nj && k >= r.k0 && k < r.k0 + r.nk;
    };
    auto face = [&](long long s, A* const* o) {
        A wV[8], w0[8], w1[8], w2[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const long long cn = c + (long long)(n - 4) * s;
            wV[n] = A(__ldg(&vol[cn])); w0[n] = A(__ldg(&v0[cn])); w1[n] = A(__ldg(&v1[cn])); w2[n] = A(__ldg(&v2[cn]));
        }
        A f0, f1, f2;
        mom2face_sum<A>(wV, w0, w1, w2, f0, f1, f2);
        o[0][c] = f0; o[1][c] = f1; o[2][c] = f2;
    };
    if (in(rJ)) face(L.P, out.v[0]);
    if (in(rK)) face((long long)L.P * L.Q, out.v[1]);
    if (in(rI)) face(1, out.v[2]);
}

void efield_kernels_init() {
    set_edge_smem<double, double, 0>(); set_edge_smem<double, double, 1>(); set_edge_smem<double, double, 2>();
    efield_kernels_init_f32();
}

// CalcElecField (fields.F90:70-232): E = 0, then for eD = I, J, K: Mom2Face along dT1, EMF on the edges
void enqueue_efield(Handle& h, const StateP& nS, cudaStream_t st) {
    (void)nS;   // the limiter values come from the precomputed nbA planes
    const Lay& L = h.L;
    // E = 0 (fields.F90:88) needs no pass per step: the edge kernels rewrite the same edges every step, and
    // every edge outside them stays zero from the pool's zeroing (initialisation clears its scratch use)
    Vec3P VdV = {{h.VdV[0], h.VdV[1], h.VdV[2]}};
    GridP g = h.gridP();
    EdgeSrc<double> in64;
    EdgeSrc<float> in32;
    if (h.prec == PREC_FP32FLUX) {
        const F32Planes& f = h.f32;
        for (int x = 0; x < 3; ++x) in32.Vf[x] = f.Vf[x];
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
    // Mom2Face regions (dT1 = J, K, I for the I, J, K edges) and the edge regions
    const Reg rv[3] = {mkreg(0, L.Ni - 1, js, je + 1, 0, L.Nk - 1), mkreg(0, L.Ni - 1, 0, L.Nj - 1, ks, ke + 1),
                       mkreg(is, ie + 1, 0, L.Nj - 1, 0, L.Nk - 1)};
    const Reg re[3] = {mkreg(is, ie, js, je + 1, ks, ke + 1), mkreg(is, ie + 1, js, je, ks, ke + 1),
                       mkreg(is, ie + 1, js, je + 1, ks, ke)};
    const Reg cells = {0, L.Ni, 0, L.Nj, 0, L.Nk};
    if (f32) {
        Vf9<float> o;
        for (int x = 0; x < 3; ++x) { o.v[0][x] = h.f32.VfE[0][x]; o.v[1][x] = h.f32.VfE[1][x]; o.v[2][x] = h.f32.Vf[x]; }
        const float* const* q = h.f32.VdV;
        k_mom2face3<float, const float*, float><<<grid_plane(cells, 128), 128, 0, st>>>(
            L, h.f32.volume, q[0], q[1], q[2], o, rv[2], rv[0], rv[1]);
    } else {
        Vf9<double> o;
        for (int x = 0; x < 3; ++x) { o.v[0][x] = h.VfE[0][x]; o.v[1][x] = h.VfE[1][x]; o.v[2][x] = h.Vf[x]; }
        k_mom2face3<double, const double*, double><<<grid_plane(cells, 128), 128, 0, st>>>(
            L, g.volume, VdV.v[0], VdV.v[1], VdV.v[2], o, rv[2], rv[0], rv[1]);
    }
    h.launches++;
    for (int eD = 0; eD < 3; ++eD) {
        for (int x = 0; x < 3; ++x) {
            in32.Vf[x] = eD < 2 ? h.f32.VfE[eD][x] : h.f32.Vf[x];
            in64.Vf[x] = eD < 2 ? h.VfE[eD][x] : h.Vf[x];
        }
        if (f32) launch_edge_dir_f32(h, in32, eD, re[eD], st);
        else launch_edge_dir<double, double>(h, in64, eD, re[eD], st);
    }
}

}  // namespace gam
