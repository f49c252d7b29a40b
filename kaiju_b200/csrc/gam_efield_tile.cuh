// Edge-EMF tile kernel of the constrained-transport electric field (fields.F90:70-232) and its launch
// helpers; gam_efield.cu instantiates the FP64 path and gam_efield_f32.cu, compiled with approximate
// single-precision division and square root, the FP32 path.
#pragma once
#include <cstdio>
#include <cstring>
#include <type_traits>
#include "gam_common.cuh"
#include "gam_kern.cuh"
#include "gam_step.cuh"
#include "gam_tma.cuh"

namespace gam {

// the FP32 instantiation lives in gam_efield_f32.cu
void launch_edge_dir_f32(Handle& h, const EdgeSrc<float>& in, int eD, const Reg& re, cudaStream_t st);

// ------------------------------------------------------------------ tile geometry
struct BoxC { int oi, oj, ok, ni, nj, nk; };
// TMA: a box that reaches below the tile along i starts at i0-4 (a copy's x coordinate must be a multiple of
// 16 bytes) and every box row is a multiple of 4 elements; each box's region in shared memory starts on a
// 128-byte boundary (regions padded to 32 elements), with the mbarrier after the last
template <int ED, bool TMA = false> struct ETile {
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
    static constexpr BoxC widen(BoxC b) {
        if (!TMA) return b;
        const int oi = b.oi < 0 ? -4 : 0;
        return BoxC{oi, b.oj, b.ok, (b.ni + b.oi - oi + 3) / 4 * 4, b.nj, b.nk};
    }
    static constexpr BoxC b8t2 = widen(box(dT2, -4, 7)), b4t2 = widen(box(dT2, -2, 3));
    static constexpr BoxC b8t1 = widen(box(dT1, -4, 7)), b4t1 = widen(box(dT1, -2, 3));
    // corner densities: offsets -1 along dT1 and dT2
    static constexpr BoxC bR = widen(BoxC{(dT1 == 0 || dT2 == 0) ? -1 : 0, (dT1 == 1 || dT2 == 1) ? -1 : 0,
                                          (dT1 == 2 || dT2 == 2) ? -1 : 0, TI + ((dT1 == 0 || dT2 == 0) ? 1 : 0),
                                          TJ + ((dT1 == 1 || dT2 == 1) ? 1 : 0), TK + ((dT1 == 2 || dT2 == 2) ? 1 : 0)});
    static constexpr int n8t2 = b8t2.ni * b8t2.nj * b8t2.nk, n4t2 = b4t2.ni * b4t2.nj * b4t2.nk;
    static constexpr int n8t1 = b8t1.ni * b8t1.nj * b8t1.nk, n4t1 = b4t1.ni * b4t1.nj * b4t1.nk;
    static constexpr int nR = bR.ni * bR.nj * bR.nk;
    static constexpr int pad(int n) { return TMA ? (n + 31) / 32 * 32 : n; }
    // layout: Vf[3], A1, B1 (b8t2) | N1 (b4t2) | A2, B2 (b8t1) | N2 (b4t1) | rho (bR); sVf: Vf plane stride
    static constexpr int sVf = pad(n8t2);
    static constexpr int oVf = 0, oA1 = 3 * sVf, oB1 = 4 * sVf, oN1 = 5 * sVf, oA2 = oN1 + pad(n4t2),
                         oB2 = oA2 + pad(n8t1), oN2 = oB2 + pad(n8t1), oR = oN2 + pad(n4t1), total = oR + pad(nR);
    static constexpr int boxed = 5 * n8t2 + n4t2 + 2 * n8t1 + n4t1 + nR;   // elements the copies deliver
};
// Tensor maps of the staged planes in layout order: Vf 0-2, face/hbA/nbA of dT1, face/hbA/nbA of dT2, rho
struct EdgeMaps { CUtensorMap m[10]; };
__device__ __forceinline__ int bidx(BoxC b, int di, int dj, int dk) {
    return (di - b.oi) + b.ni * ((dj - b.oj) + b.nj * (dk - b.ok));
}

// TMA: the footprint arrives by tensor copies issued by one thread; otherwise by cp.async row copies. The
// FP64 I-edge tile's 59 KB footprint allows three CTAs per SM whatever their registers, so that kernel gets the
// 80 registers three CTAs leave (it spills at 64); the J and K edges keep four CTAs at 64.
template <typename T, typename S, int ED, bool TMA>
__global__ void __launch_bounds__(256, sizeof(S) == 4 ? 6 : (ED == 0 && TMA ? 3 : 4))
k_edge_tile(Lay L, Par p, const __grid_constant__ EdgeMaps maps, EdgeSrc<S> in, double* Eout, Reg r, Scal* sc) {
    using TL = ETile<ED, TMA>;
    constexpr int dT1 = TL::dT1, dT2 = TL::dT2;
    extern __shared__ __align__(128) unsigned char smraw[];
    S* sm = reinterpret_cast<S*>(smraw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ti = lane, tj = (tid >> 5) % TL::TJ, tk = (tid >> 5) / TL::TJ;
    const int i0 = r.i0 + blockIdx.x * TL::TI, j0 = r.j0 + blockIdx.y * TL::TJ, k0 = r.k0 + blockIdx.z * TL::TK;
    constexpr BoxC b8t2 = TL::b8t2, b4t2 = TL::b4t2, b8t1 = TL::b8t1, b4t1 = TL::b4t1, bR = TL::bR;
    if constexpr (TMA) {
        static_assert((TL::total * sizeof(S)) % 16 == 0, "mbarrier alignment");
        uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + TL::total * sizeof(S));
        if (tid == 0) {
            tc::mbar_init(bar, 1);
            tma::fence_barrier_init();
        }
        __syncthreads();
        if (tid == 0) {
            tma::arrive_expect_tx(bar, (uint32_t)(TL::boxed * sizeof(S)));
            auto ld = [&](int q, int off, BoxC b) { tma::load3(sm + off, &maps.m[q], i0 + b.oi, j0 + b.oj, k0 + b.ok, bar); };
#pragma unroll
            for (int x = 0; x < 3; ++x) ld(x, TL::oVf + x * TL::sVf, b8t2);
            ld(3, TL::oA1, b8t2);
            ld(4, TL::oB1, b8t2);
            ld(5, TL::oN1, b4t2);
            ld(6, TL::oA2, b8t1);
            ld(7, TL::oB2, b8t1);
            ld(8, TL::oN2, b4t1);
            ld(9, TL::oR, bR);
        }
        if constexpr (sizeof(S) == 8) {
            // while the tile lands, prefetch this edge's metric values (read from HBM after the wait) into L1:
            // the FP64 kernel otherwise stalls on their latency (measured 6-7% of the FP64 E-field phase; the
            // FP32 kernel measured slower with it)
            const int pi = i0 + ti, pj = j0 + tj, pk = k0 + tk;
            if (pi < r.i0 + r.ni && pj < r.j0 + r.nj && pk < r.k0 + r.nk) {
                const long long pc = L.at(pi, pj, pk);
                auto pf = [](const S* a) { asm volatile("prefetch.global.L1 [%0];" :: "l"(a)); };
#pragma unroll
                for (int q = 0; q < 6; ++q) pf(&in.Te[ED][q][pc]);
#pragma unroll
                for (int q = 0; q < 4; ++q) pf(&in.Teb[ED][q][pc]);
                pf(&in.edge[ED][pc]);
            }
        }
        if (!tc::mbar_wait(bar, 0u, p.stageWait)) {
            if (tid == 0) atomicOr(&sc->waitFail, 1u);
            tc::mbar_wait(bar, 0u, STAGE_DRAIN);   // let copies in flight land before the CTA's shared memory goes
            return;
        }
    } else {
        auto stage = [&](S* dst, const S* src, BoxC b) {
            stage_rows<S>(dst, src, L, i0 + b.oi, b.ni, j0 + b.oj, b.nj, k0 + b.ok, b.nk, warp, 8, lane);
        };
#pragma unroll
        for (int x = 0; x < 3; ++x) stage(sm + TL::oVf + x * TL::sVf, in.Vf[x], b8t2);
        stage(sm + TL::oA1, in.face[dT1], b8t2);
        stage(sm + TL::oB1, in.hbA[dT1], b8t2);
        stage(sm + TL::oN1, in.nbA[dT1], b4t2);
        stage(sm + TL::oA2, in.face[dT2], b8t1);
        stage(sm + TL::oB2, in.hbA[dT2], b8t1);
        stage(sm + TL::oN2, in.nbA[dT2], b4t1);
        stage(sm + TL::oR, in.rho, bR);
        cp_async_wait_all();
        __syncthreads();
    }
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
        Vc1 = Vc1 + w * (Ab[m] * T(sm[TL::oVf + TL::sVf + q]));
        Vc2 = Vc2 + w * (Ab[m] * T(sm[TL::oVf + 2 * TL::sVf + q]));
    }
    T fA1 = central8<T>(Ab);
    // 1 / max(fA1, TINY), where the reference divides three times; for fA1 > TINY it is the 1 / fA1 the
    // face-field reconstruction uses as well
    const T ifA1 = T(1) / fA1;
    T idA = fA1 > T(TINY) ? ifA1 : T(1.0 / TINY);
    Vc0 = Vc0 * idA; Vc1 = Vc1 * idA; Vc2 = Vc2 * idA;
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
    getLR<T>(p.rmeth, pdmb, Ab, Bb, nBb, ifA1, l1, r1);
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
    const T ifA2 = T(1) / fA2;
    T l2, r2;
    getLR<T>(p.rmeth, pdmb, A2, B2, nB2, ifA2, l2, r2);
    T bT2L = l2 * fA2, bT2R = r2 * fA2;
    T xni = T(__ldg(&in.Teb[ED][0][c])), yni = T(__ldg(&in.Teb[ED][1][c]));
    T xnj = T(__ldg(&in.Teb[ED][2][c])), ynj = T(__ldg(&in.Teb[ED][3][c]));
    T detT = T(1) / (xni * ynj - xnj * yni);
    T bT1 = T(0.5) * (bT1L + bT1R) * ifA1;
    T bT2 = T(0.5) * (bT2L + bT2R) * ifA2;
    T db1 = (bT1R - bT1L) * ifA1;
    T db2 = (bT2R - bT2L) * ifA2;
    T Jd = db2 - db1;
    T b1 = detT * (ynj * bT1 - yni * bT2);
    T b2 = detT * (-(xnj * bT1) + xni * bT2);
    if (p.doBackground) {   // total corner field (fields.F90:417-420)
        b1 = b1 + T(__ldg(&in.edgB0[ED][0][c]));
        b2 = b2 + T(__ldg(&in.edgB0[ED][1][c]));
    }
    // diffusive speed and EMF (fields.F90:204-221)
    T vA = sqrt(b1 * b1 + b2 * b2) * rsq(Dc);
    if (p.doBoris) { T Ca = T(p.Ca); vA = Ca * vA * rsq(Ca * Ca + vA * vA); }
    vDiff = vDiff + vA;
    double edg = double(__ldg(&in.edge[ED][c]));
    T lim = T(p.CFL * edg / sc->dt);
    vDiff = vDiff < lim ? vDiff : lim;
    T e = -(v1 * b2 - v2 * b1) + T(p.Vd0) * vDiff * Jd;
    Eout[c] = double(e) * edg;
}

// Tensor maps of the staged planes of edge direction ED; false when a plane cannot be mapped or the boxes'
// x origins (i0 and i0-4; tiles step by 32) would not be 16-byte aligned
template <typename S, int ED>
static bool edge_maps(const Handle& h, const EdgeSrc<S>& in, const Reg& re, EdgeMaps& m) {
    using TL = ETile<ED, true>;
    if ((re.i0 * (int)sizeof(S)) % 16 != 0) return false;
    const S* src[10] = {in.Vf[0], in.Vf[1], in.Vf[2], in.face[TL::dT1], in.hbA[TL::dT1], in.nbA[TL::dT1],
                        in.face[TL::dT2], in.hbA[TL::dT2], in.nbA[TL::dT2], in.rho};
    const BoxC box[10] = {TL::b8t2, TL::b8t2, TL::b8t2, TL::b8t2, TL::b8t2, TL::b4t2, TL::b8t1, TL::b8t1, TL::b4t1, TL::bR};
    for (int q = 0; q < 10; ++q)
        if (!tma::plane_map(&m.m[q], src[q], (int)sizeof(S), h.L, box[q].ni, box[q].nj, box[q].nk)) return false;
    return true;
}

template <typename T, typename S, int ED>
static void launch_edge(Handle& h, const EdgeSrc<S>& in, const Reg& re, cudaStream_t st) {
    using TL = ETile<ED>;
    dim3 grid((unsigned)((re.ni + TL::TI - 1) / TL::TI), (unsigned)((re.nj + TL::TJ - 1) / TL::TJ),
              (unsigned)((re.nk + TL::TK - 1) / TL::TK));
    EdgeMaps maps;
    memset(&maps, 0, sizeof(maps));
    if (h.tileTma && edge_maps<S, ED>(h, in, re, maps))
        k_edge_tile<T, S, ED, true><<<grid, 256, sizeof(S) * ETile<ED, true>::total + 16, st>>>(h.L, h.p, maps, in, h.E[ED], re, h.dScal);
    else
        k_edge_tile<T, S, ED, false><<<grid, 256, sizeof(S) * TL::total, st>>>(h.L, h.p, maps, in, h.E[ED], re, h.dScal);
    h.launches++;
}

template <typename T, typename S, int ED>
static void set_edge_smem() {
    cudaFuncSetAttribute(k_edge_tile<T, S, ED, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(S) * ETile<ED>::total));
    cudaFuncSetAttribute(k_edge_tile<T, S, ED, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(S) * ETile<ED, true>::total + 16));
}

template <typename T, typename S>
static void launch_edge_dir(Handle& h, const EdgeSrc<S>& in, int eD, const Reg& re, cudaStream_t st) {
    if (eD == 0) launch_edge<T, S, 0>(h, in, re, st);
    else if (eD == 1) launch_edge<T, S, 1>(h, in, re, st);
    else launch_edge<T, S, 2>(h, in, re, st);
}

}  // namespace gam
