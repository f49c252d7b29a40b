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
// Vf at one face (fused multiply-adds, as in the windowed kernel): the Central8 sums along dT1 of the summands vol*rho*v/max(rho,dFloor) over the Central8
// sum of the volumes (clamped at TINY). A is the accumulation type: double on the FP64 path, float on the
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

// Faces along i (dT1 = I): one face per thread; the stencil runs along the warp, so neighbouring lanes
// share their loads through L1
template <typename A, typename VS, typename GS>
__global__ void k_mom2face_i(Lay L, const GS* vol, VS v0, VS v1, VS v2, A* o0, A* o1, A* o2, Reg r) {
    int i, j, k;
    if (!reg3(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    A wV[8], w0[8], w1[8], w2[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        long long cn = c + n - 4;
        wV[n] = A(__ldg(&vol[cn])); w0[n] = A(__ldg(&v0[cn])); w1[n] = A(__ldg(&v1[cn])); w2[n] = A(__ldg(&v2[cn]));
    }
    A f0, f1, f2;
    mom2face_sum<A>(wV, w0, w1, w2, f0, f1, f2);
    o0[c] = f0; o1[c] = f1; o2[c] = f2;
}

// Faces along j or k (dT1 = J, K): a thread computes NW consecutive faces along dT1 from a window of
// NW + 7 cells held in registers (8 loads per face become (NW + 7) / NW). Threads run along i (x) and
// along dT1 in steps of NW (y); z is the remaining axis. The sums keep the one-face order, so the FP64
// result is the same bit for bit.
template <typename A, typename VS, typename GS, int NW>
__global__ void k_mom2face_run(Lay L, const GS* vol, VS v0, VS v1, VS v2, A* o0, A* o1, A* o2, Reg r, int dT1) {
    const int i = r.i0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int a0 = (int)(blockIdx.y * blockDim.y + threadIdx.y) * NW;   // first face of the run, from the region start
    const int t2 = (int)blockIdx.z;
    const int n1 = dT1 == 1 ? r.nj : r.nk;
    if (i >= r.i0 + r.ni || a0 >= n1) return;
    const int j = dT1 == 1 ? r.j0 + a0 : r.j0 + t2, k = dT1 == 1 ? r.k0 + t2 : r.k0 + a0;
    const long long c = L.at(i, j, k), s = L.stride(dT1);
    // cells a0-4 .. a0+NW+2 of the run; the stencils of faces past the region end are not loaded. One
    // quantity at a time: the volume sums first, then each summand's sums over them.
    const int nload = (n1 - a0 + 7 < NW + 7) ? n1 - a0 + 7 : NW + 7;
    auto window = [&](const auto* src, A* w) {
#pragma unroll
        for (int m = 0; m < NW + 7; ++m) w[m] = m < nload ? A(__ldg(&src[c + (long long)(m - 4) * s])) : A(0);
    };
    // explicit fused multiply-adds: the weights are symmetric, so neighbouring faces' sums share products
    // (c3*w[4] is term 4 of one face and term 3 of the next); left to contraction, a shared product may be
    // rounded on its own and a face's result would depend on its place in the run
    auto sum8 = [&](const A* w) {
        A acc = A(0);
#pragma unroll
        for (int n = 0; n < 8; ++n) acc = fma(A(wC8(n)), w[n], acc);
        return acc;
    };
    A w[NW + 7], idV[NW];   // the reciprocal of each face's volume sum serves its three quotients
    window(vol, w);
#pragma unroll
    for (int q = 0; q < NW; ++q) { A sV = sum8(w + q); idV[q] = A(1) / (sV > A(TINY) ? sV : A(TINY)); }
    A* const out[3] = {o0, o1, o2};
    VS const src[3] = {v0, v1, v2};
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        window(src[x], w);
#pragma unroll
        for (int q = 0; q < NW; ++q)
            if (a0 + q < n1) out[x][c + (long long)q * s] = sum8(w + q) * idV[q];
    }
}

constexpr int M2F_RUN = 4;   // faces per thread along dT1 = J, K

template <typename A, typename VS, typename GS>
static void launch_mom2face(const Lay& L, const GS* vol, VS v0, VS v1, VS v2, A* const* o, const Reg& r, int dT1,
                            cudaStream_t st) {
    if (dT1 == IDIR) {
        dim3 b(32, 4, 1);
        k_mom2face_i<A, VS, GS><<<grid3(r, b), b, 0, st>>>(L, vol, v0, v1, v2, o[0], o[1], o[2], r);
    } else {
        const int n1 = dT1 == JDIR ? r.nj : r.nk, n2 = dT1 == JDIR ? r.nk : r.nj;
        const int runs = (n1 + M2F_RUN - 1) / M2F_RUN;
        dim3 b(32, 4, 1), grid((unsigned)((r.ni + 31) / 32), (unsigned)((runs + 3) / 4), (unsigned)n2);
        k_mom2face_run<A, VS, GS, M2F_RUN><<<grid, b, 0, st>>>(L, vol, v0, v1, v2, o[0], o[1], o[2], r, dT1);
    }
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
        if (f32) {
            const float* const* q = h.f32.VdV;
            launch_mom2face<float, const float*, float>(L, h.f32.volume, q[0], q[1], q[2], Vf32.v, rv, dT1, st);
        } else {
            launch_mom2face<double, const double*, double>(L, g.volume, VdV.v[0], VdV.v[1], VdV.v[2], Vf.v, rv, dT1, st);
        }
        h.launches++;
        if (f32) launch_edge_dir_f32(h, in32, eD, re, st);
        else launch_edge_dir<double, double>(h, in64, eD, re, st);
    }
}

}  // namespace gam
