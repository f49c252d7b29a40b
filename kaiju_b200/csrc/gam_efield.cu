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
#include <cstdio>
#include <type_traits>
#include "gam_common.cuh"
#include "gam_kern.cuh"
#include "gam_step.cuh"

namespace gam {

// ------------------------------------------------------------------ Mom2Face (fields.F90:235-285)
struct Vec3F { float* v[3]; };
__global__ void k_mom2face2(Lay L, GridP g, Vec3P VdV, Vec3P Vf, Vec3F Vf32, Reg r, int dT1) {
    int i, j, k;
    if (!reg3(r, i, j, k)) return;
    long long c = L.at(i, j, k), s = L.stride(dT1);
    double sV = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        long long cn = c + (n - 4) * s;
        double w = wC8(n);
        sV = sV + w * __ldg(&g.volume[cn]);
        s0 = s0 + w * __ldg(&VdV.v[0][cn]);
        s1 = s1 + w * __ldg(&VdV.v[1][cn]);
        s2 = s2 + w * __ldg(&VdV.v[2][cn]);
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

// ------------------------------------------------------------------ tile geometry
struct BoxC { int oi, oj, ok, ni, nj, nk; };
template <int ED> struct ETile {
    static constexpr int dT1 = ED == 0 ? 1 : (ED == 1 ? 2 : 0);
    static constexpr int dT2 = ED == 0 ? 2 : (ED == 1 ? 0 : 1);
    static constexpr int TI = 32;
    static constexpr int TJ = ED == 0 ? 2 : (ED == 1 ? 1 : 8);
    static constexpr int TK = ED == 0 ? 4 : (ED == 1 ? 8 : 1);
    // stencil box along s with offsets [lo, lo+len) beyond the tile (8-pt: lo -4 len 7; 4-pt: -2, 3)
    static constexpr BoxC box(int s, int lo, int extra) {
        return BoxC{s == 0 ? lo : 0, s == 1 ? lo : 0, s == 2 ? lo : 0, TI + (s == 0 ? extra : 0),
                    TJ + (s == 1 ? extra : 0), TK + (s == 2 ? extra : 0)};
    }
    static constexpr BoxC b8t2 = box(dT2, -4, 7), b4t2 = box(dT2, -2, 3);
    static constexpr BoxC b8t1 = box(dT1, -4, 7), b4t1 = box(dT1, -2, 3);
    // corner densities: offsets -1 along dT1 and dT2
    static constexpr BoxC bR = BoxC{(dT1 == 0 || dT2 == 0) ? -1 : 0, (dT1 == 1 || dT2 == 1) ? -1 : 0,
                                    (dT1 == 2 || dT2 == 2) ? -1 : 0, TI + ((dT1 == 0 || dT2 == 0) ? 1 : 0),
                                    TJ + ((dT1 == 1 || dT2 == 1) ? 1 : 0), TK + ((dT1 == 2 || dT2 == 2) ? 1 : 0)};
    static constexpr int n8t2 = b8t2.ni * b8t2.nj * b8t2.nk, n4t2 = b4t2.ni * b4t2.nj * b4t2.nk;
    static constexpr int n8t1 = b8t1.ni * b8t1.nj * b8t1.nk, n4t1 = b4t1.ni * b4t1.nj * b4t1.nk;
    static constexpr int nR = bR.ni * bR.nj * bR.nk;
    // layout: Vf[3], A1, B1 (b8t2) | N1 (b4t2) | A2, B2 (b8t1) | N2 (b4t1) | rho (bR)
    static constexpr int oVf = 0, oA1 = 3 * n8t2, oB1 = 4 * n8t2, oN1 = 5 * n8t2, oA2 = 5 * n8t2 + n4t2,
                         oB2 = oA2 + n8t1, oN2 = oA2 + 2 * n8t1, oR = oN2 + n4t1, total = oR + nR;
};
__device__ __forceinline__ int bidx(BoxC b, int di, int dj, int dk) {
    return (di - b.oi) + b.ni * ((dj - b.oj) + b.nj * (dk - b.ok));
}

template <typename T, typename S, int ED>
__global__ void __launch_bounds__(256, 2) k_edge_tile(Lay L, Par p, EdgeSrc<S> in, double* Eout, Reg r, const Scal* sc) {
    using TL = ETile<ED>;
    constexpr int dT1 = TL::dT1, dT2 = TL::dT2;
    extern __shared__ __align__(16) unsigned char smraw[];
    S* sm = reinterpret_cast<S*>(smraw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ti = lane, tj = (tid >> 5) % TL::TJ, tk = (tid >> 5) / TL::TJ;
    const int i0 = r.i0 + blockIdx.x * TL::TI, j0 = r.j0 + blockIdx.y * TL::TJ, k0 = r.k0 + blockIdx.z * TL::TK;
    constexpr BoxC b8t2 = TL::b8t2, b4t2 = TL::b4t2, b8t1 = TL::b8t1, b4t1 = TL::b4t1, bR = TL::bR;
    auto stage = [&](S* dst, const S* src, BoxC b) {
        stage_rows<S>(dst, src, L, i0 + b.oi, b.ni, j0 + b.oj, b.nj, k0 + b.ok, b.nk, warp, 8, lane);
    };
#pragma unroll
    for (int x = 0; x < 3; ++x) stage(sm + TL::oVf + x * TL::n8t2, in.Vf[x], b8t2);
    stage(sm + TL::oA1, in.face[dT1], b8t2);
    stage(sm + TL::oB1, in.hbA[dT1], b8t2);
    stage(sm + TL::oN1, in.nbA[dT1], b4t2);
    stage(sm + TL::oA2, in.face[dT2], b8t1);
    stage(sm + TL::oB2, in.hbA[dT2], b8t1);
    stage(sm + TL::oN2, in.nbA[dT2], b4t1);
    stage(sm + TL::oR, in.rho, bR);
    cp_async_wait_all();
    __syncthreads();
    const int i = i0 + ti, j = j0 + tj, k = k0 + tk;
    if (!(i < r.i0 + r.ni && j < r.j0 + r.nj && k < r.k0 + r.nk)) return;
    const long long c = L.at(i, j, k);
    auto off = [&](int s, int m, int& di, int& dj, int& dk) {
        di = ti + (s == 0 ? m : 0); dj = tj + (s == 1 ? m : 0); dk = tk + (s == 2 ? m : 0);
    };
    // GetCornerV (fields.F90:457-517): area-weighted Central8 of Vf along dT2, mapped with Te
    T Ab[8], Bb[8], nBb[4];
    T Vc0 = T(0), Vc1 = T(0), Vc2 = T(0);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        int di, dj, dk;
        off(dT2, m - 4, di, dj, dk);
        int q = bidx(b8t2, di, dj, dk);
        Ab[m] = T(sm[TL::oA1 + q]);
        Bb[m] = T(sm[TL::oB1 + q]);
        T w = T(wC8(m));
        Vc0 = Vc0 + w * (Ab[m] * T(sm[TL::oVf + q]));
        Vc1 = Vc1 + w * (Ab[m] * T(sm[TL::oVf + TL::n8t2 + q]));
        Vc2 = Vc2 + w * (Ab[m] * T(sm[TL::oVf + 2 * TL::n8t2 + q]));
    }
    T fA1 = central8<T>(Ab);
    T dA = fA1 > T(TINY) ? fA1 : T(TINY);
    Vc0 = Vc0 / dA; Vc1 = Vc1 / dA; Vc2 = Vc2 / dA;
    T v1 = Vc0 * T(__ldg(&in.Te[ED][0][c])) + Vc1 * T(__ldg(&in.Te[ED][1][c])) + Vc2 * T(__ldg(&in.Te[ED][2][c]));
    T v2 = Vc0 * T(__ldg(&in.Te[ED][3][c])) + Vc1 * T(__ldg(&in.Te[ED][4][c])) + Vc2 * T(__ldg(&in.Te[ED][5][c]));
    T vDiff = sqrt(v1 * v1 + v2 * v2);
    // GetCornerD (fields.F90:427-454), getNormalPlane order: e1 = first transverse of (I,J,K) \ eD
    constexpr int e1 = ED == 0 ? 1 : 0, e2 = ED == 2 ? 1 : 2;
    int a0i, a0j, a0k;
    off(0, 0, a0i, a0j, a0k);
    auto rho = [&](int d1, int d2) {
        int di = a0i - (e1 == 0 ? d1 : 0) - (e2 == 0 ? d2 : 0);
        int dj = a0j - (e1 == 1 ? d1 : 0) - (e2 == 1 ? d2 : 0);
        int dk = a0k - (e1 == 2 ? d1 : 0) - (e2 == 2 ? d2 : 0);
        return sm[TL::oR + bidx(bR, di, dj, dk)];
    };
    T Dc;
    if constexpr (std::is_same<S, double>::value) Dc = T(0.25 * (rho(0, 0) + rho(1, 0) + rho(0, 1) + rho(1, 1)));
    else Dc = T(0.25) * (T(rho(0, 0)) + T(rho(1, 0)) + T(rho(0, 1)) + T(rho(1, 1)));
    // GetCornerB (fields.F90:365-424): EdgeLRs of the dT1 faces along dT2 ...
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        int di, dj, dk;
        off(dT2, m - 2, di, dj, dk);
        nBb[m] = T(sm[TL::oN1 + bidx(b4t2, di, dj, dk)]);
    }
    T pdmb = T(p.pdmb);
    T l1, r1;
    getLR<T>(p.rmeth, pdmb, Ab, Bb, nBb, fA1, l1, r1);
    T bT1L = l1 * fA1, bT1R = r1 * fA1;
    // ... and of the dT2 faces along dT1
    T A2[8], B2[8], nB2[4];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        int di, dj, dk;
        off(dT1, m - 4, di, dj, dk);
        int q = bidx(b8t1, di, dj, dk);
        A2[m] = T(sm[TL::oA2 + q]);
        B2[m] = T(sm[TL::oB2 + q]);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        int di, dj, dk;
        off(dT1, m - 2, di, dj, dk);
        nB2[m] = T(sm[TL::oN2 + bidx(b4t1, di, dj, dk)]);
    }
    T fA2 = central8<T>(A2);
    T l2, r2;
    getLR<T>(p.rmeth, pdmb, A2, B2, nB2, fA2, l2, r2);
    T bT2L = l2 * fA2, bT2R = r2 * fA2;
    T xni = T(__ldg(&in.Teb[ED][0][c])), yni = T(__ldg(&in.Teb[ED][1][c]));
    T xnj = T(__ldg(&in.Teb[ED][2][c])), ynj = T(__ldg(&in.Teb[ED][3][c]));
    T detT = T(1) / (xni * ynj - xnj * yni);
    T bT1 = T(0.5) * (bT1L + bT1R) / fA1;
    T bT2 = T(0.5) * (bT2L + bT2R) / fA2;
    T db1 = (bT1R - bT1L) / fA1;
    T db2 = (bT2R - bT2L) / fA2;
    T Jd = db2 - db1;
    T b1 = detT * (ynj * bT1 - yni * bT2);
    T b2 = detT * (-(xnj * bT1) + xni * bT2);
    if (p.doBackground) {   // total corner field (fields.F90:417-420)
        b1 = b1 + T(__ldg(&in.edgB0[ED][0][c]));
        b2 = b2 + T(__ldg(&in.edgB0[ED][1][c]));
    }
    // diffusive speed and EMF (fields.F90:204-221)
    T vA = sqrt(b1 * b1 + b2 * b2) / sqrt(Dc);
    if (p.doBoris) { T Ca = T(p.Ca); vA = Ca * vA / sqrt(Ca * Ca + vA * vA); }
    vDiff = vDiff + vA;
    double edg = double(__ldg(&in.edge[ED][c]));
    T lim = T(p.CFL * edg / sc->dt);
    vDiff = vDiff < lim ? vDiff : lim;
    T e = -(v1 * b2 - v2 * b1) + T(p.Vd0) * vDiff * Jd;
    Eout[c] = double(e) * edg;
}

template <typename T, typename S, int ED>
static void launch_edge(Handle& h, const EdgeSrc<S>& in, const Reg& re, cudaStream_t st) {
    using TL = ETile<ED>;
    dim3 grid((unsigned)((re.ni + TL::TI - 1) / TL::TI), (unsigned)((re.nj + TL::TJ - 1) / TL::TJ),
              (unsigned)((re.nk + TL::TK - 1) / TL::TK));
    k_edge_tile<T, S, ED><<<grid, 256, sizeof(S) * TL::total, st>>>(h.L, h.p, in, h.E[ED], re, h.dScal);
    h.launches++;
}

template <typename T, typename S, int ED>
static void set_edge_smem() {
    cudaFuncSetAttribute(k_edge_tile<T, S, ED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(S) * ETile<ED>::total));
}
void efield_kernels_init() {
    set_edge_smem<double, double, 0>(); set_edge_smem<double, double, 1>(); set_edge_smem<double, double, 2>();
    set_edge_smem<float, float, 0>(); set_edge_smem<float, float, 1>(); set_edge_smem<float, float, 2>();
}

template <typename T, typename S>
static void launch_edge_dir(Handle& h, const EdgeSrc<S>& in, int eD, const Reg& re, cudaStream_t st) {
    if (eD == 0) launch_edge<T, S, 0>(h, in, re, st);
    else if (eD == 1) launch_edge<T, S, 1>(h, in, re, st);
    else launch_edge<T, S, 2>(h, in, re, st);
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
        k_mom2face2<<<grid3(rv, bv), bv, 0, st>>>(L, g, VdV, Vf, Vf32, rv, dT1);
        h.launches++;
        if (f32) launch_edge_dir<float, float>(h, in32, eD, re, st);
        else launch_edge_dir<double, double>(h, in64, eD, re, st);
    }
}

}  // namespace gam
