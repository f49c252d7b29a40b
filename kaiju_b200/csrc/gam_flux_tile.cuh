// Interface fluxes (stress.F90:204-429) with shared-memory staging.
//
// A CTA of 256 threads owns a 32 x 8 tile of interfaces: 32 consecutive i (one warp per row) by 8
// rows, the rows running along the sweep direction d for J/K sweeps and along j for the I sweep. It
// first copies, with coalesced row loads, the stencil footprint -- the tile plus the 4-cell halo of
// the reconstruction stencil (half-state primitives, half-state B, volumes) and the 2-cell halo of
// the limiter stencil (state-n primitives and B) -- into shared memory, then every thread
// reconstructs, limits and evaluates the kinetic fluxes of its interface from shared memory. The
// per-interface data (face triad, area, normal flux) is read once, coalesced, from HBM.
//
// The arithmetic type T is double for the plain path and float for the FP32-flux path (staged
// values are converted while they are copied in).
//
// This header holds the tile kernel and its launch helpers; gam_flux.cu instantiates the FP64 path and
// gam_flux_f32.cu, compiled with approximate single-precision division and square root, the FP32 path.
#pragma once
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>
#include "gam_common.cuh"
#include "gam_kern.cuh"
#include "gam_step.cuh"
#include "gam_tma.cuh"

namespace gam {

constexpr int FL = 32;   // interfaces per tile along i
// FR: rows per tile (one warp per row), 8 by default; 4 gives twice the CTAs, which the ensemble
// autotuner picks for members too small to fill the GPU

template <int D, int FR> __host__ __device__ constexpr int rec_box() { return D == 0 ? (FL + 8) * FR : FL * (FR + 7); }
// TMA: the I-sweep limiter box starts at i0-4 like the reconstruction box (its x coordinate must be a
// multiple of 16 bytes), so its rows are FL+8 wide with the stencil 2 cells in
template <int D, int FR, bool TMA = false> __host__ __device__ constexpr int lim_box() {
    return D == 0 ? (TMA ? FL + 8 : FL + 4) * FR : FL * (FR + 3);
}
template <typename S, int D, int FR, bool TMA = false> constexpr size_t flux_smem() {
    return sizeof(S) * (9 * rec_box<D, FR>() + 8 * lim_box<D, FR, TMA>()) + (TMA ? 16 : 0);   // + the mbarrier
}

// Tensor maps of the staged planes: the reconstruction planes (W 0-4, volume, B 0-2) and the limiter
// planes (W 0-4, B 0-2), each with the box of the sweep direction
struct FluxMaps { CUtensorMap rec[9]; CUtensorMap lim[8]; };

// A flux times the face area in the storage type: for float storage a float product, which is the double
// product of the two floats (exact) rounded once, so the same value without the conversions
template <typename S, typename T>
__device__ __forceinline__ S area_scaled(double faB, T f) {
    if constexpr (std::is_same<S, float>::value) return float(faB) * float(f);
    else return S(faB * double(f));
}

// One tile (bx, by, bz) of interfaces: the body of the per-problem flux kernel and of the ensembles'
// persistent tile-queue kernel. Every thread of the CTA calls it for the same tile.
template <typename T, typename S, int D, bool MHD, bool BG, int FR>
__device__ __forceinline__ void flux_tile_body(const Lay& L, const Par& p, const FluxSrc<S>& in, const StateP& h,
                                               const FluxOut<S>& F, const Reg& r, int bx, int by, int bz,
                                               unsigned char* smraw) {
    S* sRec = reinterpret_cast<S*>(smraw);   // staged in the storage type, converted to T on use
    constexpr int RB = rec_box<D, FR>(), LB = lim_box<D, FR>();
    S* sLim = sRec + 9 * RB;
    const int tid = threadIdx.x, lane = tid & 31, row = tid >> 5;
    const int i0 = r.i0 + bx * FL;
    int i = i0 + lane, j, k, a0;
    if (D == 2) { a0 = r.k0 + by * FR; k = a0 + row; j = r.j0 + bz; }
    else { a0 = r.j0 + by * FR; j = a0 + row; k = r.k0 + bz; }

    // ---- stage the stencil footprint (rows of 32..40 doubles, one warp per row)
    const int warp = tid >> 5;
    auto stage_rec = [&](S* dst, const S* src) {
        if (D == 0) stage_rows<S>(dst, src, L, i0 - 4, FL + 8, a0, FR, k, 1, warp, FR, lane);
        else if (D == 1) stage_rows<S>(dst, src, L, i0, FL, a0 - 4, FR + 7, k, 1, warp, FR, lane);
        else stage_rows<S>(dst, src, L, i0, FL, j, 1, a0 - 4, FR + 7, warp, FR, lane);
    };
    auto stage_lim = [&](S* dst, const S* src) {
        if (D == 0) stage_rows<S>(dst, src, L, i0 - 2, FL + 4, a0, FR, k, 1, warp, FR, lane);
        else if (D == 1) stage_rows<S>(dst, src, L, i0, FL, a0 - 2, FR + 3, k, 1, warp, FR, lane);
        else stage_rows<S>(dst, src, L, i0, FL, j, 1, a0 - 2, FR + 3, warp, FR, lane);
    };
#pragma unroll
    for (int q = 0; q < 5; ++q) stage_rec(sRec + q * RB, in.W[q]);
    stage_rec(sRec + 5 * RB, in.vol);
#pragma unroll
    for (int q = 0; q < 5; ++q) stage_lim(sLim + q * LB, in.Wl[q]);
    if (MHD) {
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            stage_rec(sRec + (6 + x) * RB, in.B[x]);
            stage_lim(sLim + (5 + x) * LB, in.Bl[x]);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    bool valid = (i < r.i0 + r.ni) && (j >= r.j0) && (j < r.j0 + r.nj) && (k >= r.k0) && (k < r.k0 + r.nk);
    if (!valid) return;

    // stencil offsets in the staged boxes: recon cell m = f-4+m, limiter cell m = f-2+m
    auto ro = [&](int m) { return D == 0 ? (lane + m) + (FL + 8) * row : lane + FL * (row + m); };
    auto lo = [&](int m) { return D == 0 ? (lane + m) + (FL + 4) * row : lane + FL * (row + m); };
    const long long c = L.at(i, j, k), s = L.stride(D);
    // the Central8 weights applied to the stencil volumes once for all the variables (8CENT); 7UP reads
    // the volumes again where it needs them
    T c8[8], Vi = T(0);
#pragma unroll
    for (int m = 0; m < 8; ++m) { c8[m] = T(wC8(m)) * T(sRec[5 * RB + ro(m)]); Vi = Vi + c8[m]; }
    const T iVi = T(1) / Vi;
    const T pdmb = T(p.pdmb);
    auto recon = [&](const T* Q, const T* nQ, T& Ql, T& Qr) {
        if (p.rmeth == RM_8CENT) getLR8<T>(pdmb, c8, Q, nQ, iVi, Ql, Qr);
        else {
            T Vol[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) Vol[m] = T(sRec[5 * RB + ro(m)]);
            getLR<T>(p.rmeth, pdmb, Vol, Q, nQ, iVi, Ql, Qr);
        }
    };
    T WL[5], WR[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        T Q[8], nQ[4];
#pragma unroll
        for (int m = 0; m < 8; ++m) Q[m] = T(sRec[v * RB + ro(m)]);
#pragma unroll
        for (int m = 0; m < 4; ++m) nQ[m] = T(sLim[v * LB + lo(m)]);
        recon(Q, nQ, WL[v], WR[v]);
    }
    T Tf[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Tf[q] = T(__ldg(&in.Tf[D][q][c]));
    double faB = double(__ldg(&in.face[D][c]));
    T VaD = T(0), bbD = T(0);
    if (MHD) {
        T BL[3], BR[3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            T Q[8], nQ[4];
#pragma unroll
            for (int m = 0; m < 8; ++m) Q[m] = T(sRec[(6 + x) * RB + ro(m)]);
#pragma unroll
            for (int m = 0; m < 4; ++m) nQ[m] = T(sLim[(5 + x) * LB + lo(m)]);
            recon(Q, nQ, BL[x], BR[x]);
        }
        // FP64: the half-state flux over the area (stress.F90:301); FP32: the stored flux/area
        T Bn;
        if constexpr (std::is_same<S, double>::value) Bn = T(__ldg(&in.bn[D][c]) / faB);
        else Bn = T(__ldg(&in.bn[D][c]));
        T mF[3] = {T(0), T(0), T(0)};
        if constexpr (BG) {   // background field on the face (stress.F90:302-305)
            T B0[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) B0[x] = T(__ldg(&in.fcB0[D][x][c]));
            T B0n;
            if constexpr (std::is_same<S, double>::value) B0n = T(__ldg(&in.b0[D][c]) / faB);
            else B0n = T(__ldg(&in.b0[D][c]));
            magKin<T, true>(p, T(-1), WL, BL, Bn, Tf, mF, bbD, VaD, B0, B0n);
            magKin<T, true>(p, T(1), WR, BR, Bn, Tf, mF, bbD, VaD, B0, B0n);
        } else {
            magKin<T>(p, T(-1), WL, BL, Bn, Tf, mF, bbD, VaD);
            magKin<T>(p, T(1), WR, BR, Bn, Tf, mF, bbD, VaD);
        }
        if (p.doBoris) {
            T Ca2 = T(p.Ca) * T(p.Ca);
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                T deeV = WR[1 + x] - WL[1 + x];
                T deeP = bbD * deeV / Ca2;
                mF[x] = mF[x] - T(p.cHogM) * VaD * deeP;
            }
        }
#pragma unroll
        for (int x = 0; x < 3; ++x) F.m[x][c] = area_scaled<S>(faB, mF[x]);
    }
    T gF[5] = {T(0), T(0), T(0), T(0), T(0)}, dW[5] = {T(0), T(0), T(0), T(0), T(0)};
    const T igm1 = T(1.0 / (p.gamma - 1));
    gasKin<T>(igm1, T(-1), WL, Tf, gF, dW);
    gasKin<T>(igm1, T(1), WR, Tf, gF, dW);
    T cH = T(p.cHogH);
#pragma unroll
    for (int v = 0; v < 5; ++v) gF[v] = gF[v] - cH * VaD * dW[v];
    if (p.doBoris) {  // nuclear option, stress.F90:399-417 (cLim = 1.5)
        T vL = sqrt(WL[1] * WL[1] + WL[2] * WL[2] + WL[3] * WL[3]);
        T vR = sqrt(WR[1] * WR[1] + WR[2] * WR[2] + WR[3] * WR[3]);
        T Vn = sqrt(vL * vL + vR * vR) / T(1.41421353816986083984375);   // sqrt(2.0) of a default-real literal
        if (Vn >= T(1.5) * T(p.Ca)) {
#pragma unroll
            for (int v = 0; v < 5; ++v) gF[v] = gF[v] - T(p.Ca) * T(h.gas[v][c] - h.gas[v][c - s]);
        }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) F.g[v][c] = area_scaled<S>(faB, gF[v]);
}

// The per-problem kernel keeps its own copy of the tile body: calling flux_tile_body from the kernel
// (by reference or by value) measured 8% slower on the 256^3 FP64 step (7.37 vs 6.83 ms of fluxes).
// TMA: the footprint arrives by tensor copies issued by one thread (no per-element address arithmetic);
// otherwise by cp.async row copies.
template <typename T, typename S, int D, bool MHD, bool BG, int FR, bool TMA>
__global__ void __launch_bounds__(32 * FR, (sizeof(S) == 4 ? 32 : 24) / FR)
k_flux_tile(Lay L, Par p, const __grid_constant__ FluxMaps maps, FluxSrc<S> in, StateP h, FluxOut<S> F, Reg r,
            Scal* sc) {
    extern __shared__ __align__(128) unsigned char smraw[];
    S* sRec = reinterpret_cast<S*>(smraw);   // staged in the storage type, converted to T on use
    constexpr int RB = rec_box<D, FR>(), LB = lim_box<D, FR, TMA>();
    static_assert(!TMA || ((RB * sizeof(S)) % 128 == 0 && (LB * sizeof(S)) % 128 == 0), "box alignment");
    S* sLim = sRec + 9 * RB;
    const int tid = threadIdx.x, lane = tid & 31, row = tid >> 5;
    const int i0 = r.i0 + blockIdx.x * FL;
    int i = i0 + lane, j, k, a0;
    if (D == 2) { a0 = r.k0 + blockIdx.y * FR; k = a0 + row; j = r.j0 + blockIdx.z; }
    else { a0 = r.j0 + blockIdx.y * FR; j = a0 + row; k = r.k0 + blockIdx.z; }

    if constexpr (TMA) {
        // ---- stage the stencil footprint by tensor copies: one box per plane, one mbarrier for all
        uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + (9 * RB + 8 * LB) * sizeof(S));
        constexpr int NR = MHD ? 9 : 6, NL = MHD ? 8 : 5;
        if (tid == 0) {
            tc::mbar_init(bar, 1);
            tma::fence_barrier_init();
        }
        __syncthreads();
        if (tid == 0) {
            tma::arrive_expect_tx(bar, (uint32_t)((NR * RB + NL * LB) * sizeof(S)));
            int rx, ry, rz, ly, lz;   // box origins; the limiter box shares x with the reconstruction box
            if (D == 0) { rx = i0 - 4; ry = a0; rz = k; ly = a0; lz = k; }
            else if (D == 1) { rx = i0; ry = a0 - 4; rz = k; ly = a0 - 2; lz = k; }
            else { rx = i0; ry = j; rz = a0 - 4; ly = j; lz = a0 - 2; }
#pragma unroll
            for (int q = 0; q < NR; ++q) tma::load3(sRec + q * RB, &maps.rec[q], rx, ry, rz, bar);
#pragma unroll
            for (int q = 0; q < NL; ++q) tma::load3(sLim + q * LB, &maps.lim[q], rx, ly, lz, bar);
        }
        if (!tc::mbar_wait(bar, 0u, p.stageWait)) {
            if (tid == 0) atomicOr(&sc->waitFail, 1u);
            tc::mbar_wait(bar, 0u, STAGE_DRAIN);   // let copies in flight land before the CTA's shared memory goes
            return;
        }
    } else {
        // ---- stage the stencil footprint (rows of 32..40 doubles, one warp per row)
        const int warp = tid >> 5;
        auto stage_rec = [&](S* dst, const S* src) {
            if (D == 0) stage_rows<S>(dst, src, L, i0 - 4, FL + 8, a0, FR, k, 1, warp, FR, lane);
            else if (D == 1) stage_rows<S>(dst, src, L, i0, FL, a0 - 4, FR + 7, k, 1, warp, FR, lane);
            else stage_rows<S>(dst, src, L, i0, FL, j, 1, a0 - 4, FR + 7, warp, FR, lane);
        };
        auto stage_lim = [&](S* dst, const S* src) {
            if (D == 0) stage_rows<S>(dst, src, L, i0 - 2, FL + 4, a0, FR, k, 1, warp, FR, lane);
            else if (D == 1) stage_rows<S>(dst, src, L, i0, FL, a0 - 2, FR + 3, k, 1, warp, FR, lane);
            else stage_rows<S>(dst, src, L, i0, FL, j, 1, a0 - 2, FR + 3, warp, FR, lane);
        };
#pragma unroll
        for (int q = 0; q < 5; ++q) stage_rec(sRec + q * RB, in.W[q]);
        stage_rec(sRec + 5 * RB, in.vol);
#pragma unroll
        for (int q = 0; q < 5; ++q) stage_lim(sLim + q * LB, in.Wl[q]);
        if (MHD) {
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                stage_rec(sRec + (6 + x) * RB, in.B[x]);
                stage_lim(sLim + (5 + x) * LB, in.Bl[x]);
            }
        }
        cp_async_wait_all();
        __syncthreads();
    }
    bool valid = (i < r.i0 + r.ni) && (j >= r.j0) && (j < r.j0 + r.nj) && (k >= r.k0) && (k < r.k0 + r.nk);
    if (!valid) return;

    // stencil offsets in the staged boxes: recon cell m = f-4+m, limiter cell m = f-2+m
    auto ro = [&](int m) { return D == 0 ? (lane + m) + (FL + 8) * row : lane + FL * (row + m); };
    constexpr int LW = TMA ? FL + 8 : FL + 4, LX = TMA ? 2 : 0;   // I-sweep limiter row width and stencil shift
    auto lo = [&](int m) { return D == 0 ? (lane + m + LX) + LW * row : lane + FL * (row + m); };
    const long long c = L.at(i, j, k), s = L.stride(D);
    // the Central8 weights applied to the stencil volumes once for all the variables (8CENT); 7UP reads
    // the volumes again where it needs them
    T c8[8], Vi = T(0);
#pragma unroll
    for (int m = 0; m < 8; ++m) { c8[m] = T(wC8(m)) * T(sRec[5 * RB + ro(m)]); Vi = Vi + c8[m]; }
    const T iVi = T(1) / Vi;
    const T pdmb = T(p.pdmb);
    auto recon = [&](const T* Q, const T* nQ, T& Ql, T& Qr) {
        if (p.rmeth == RM_8CENT) getLR8<T>(pdmb, c8, Q, nQ, iVi, Ql, Qr);
        else {
            T Vol[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) Vol[m] = T(sRec[5 * RB + ro(m)]);
            getLR<T>(p.rmeth, pdmb, Vol, Q, nQ, iVi, Ql, Qr);
        }
    };
    T WL[5], WR[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        T Q[8], nQ[4];
#pragma unroll
        for (int m = 0; m < 8; ++m) Q[m] = T(sRec[v * RB + ro(m)]);
#pragma unroll
        for (int m = 0; m < 4; ++m) nQ[m] = T(sLim[v * LB + lo(m)]);
        recon(Q, nQ, WL[v], WR[v]);
    }
    T Tf[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Tf[q] = T(__ldg(&in.Tf[D][q][c]));
    double faB = double(__ldg(&in.face[D][c]));
    T VaD = T(0), bbD = T(0);
    if (MHD) {
        T BL[3], BR[3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            T Q[8], nQ[4];
#pragma unroll
            for (int m = 0; m < 8; ++m) Q[m] = T(sRec[(6 + x) * RB + ro(m)]);
#pragma unroll
            for (int m = 0; m < 4; ++m) nQ[m] = T(sLim[(5 + x) * LB + lo(m)]);
            recon(Q, nQ, BL[x], BR[x]);
        }
        // FP64: the half-state flux over the area (stress.F90:301); FP32: the stored flux/area
        T Bn;
        if constexpr (std::is_same<S, double>::value) Bn = T(__ldg(&in.bn[D][c]) / faB);
        else Bn = T(__ldg(&in.bn[D][c]));
        T mF[3] = {T(0), T(0), T(0)};
        if constexpr (BG) {   // background field on the face (stress.F90:302-305)
            T B0[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) B0[x] = T(__ldg(&in.fcB0[D][x][c]));
            T B0n;
            if constexpr (std::is_same<S, double>::value) B0n = T(__ldg(&in.b0[D][c]) / faB);
            else B0n = T(__ldg(&in.b0[D][c]));
            magKin<T, true>(p, T(-1), WL, BL, Bn, Tf, mF, bbD, VaD, B0, B0n);
            magKin<T, true>(p, T(1), WR, BR, Bn, Tf, mF, bbD, VaD, B0, B0n);
        } else {
            magKin<T>(p, T(-1), WL, BL, Bn, Tf, mF, bbD, VaD);
            magKin<T>(p, T(1), WR, BR, Bn, Tf, mF, bbD, VaD);
        }
        if (p.doBoris) {
            T Ca2 = T(p.Ca) * T(p.Ca);
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                T deeV = WR[1 + x] - WL[1 + x];
                T deeP = bbD * deeV / Ca2;
                mF[x] = mF[x] - T(p.cHogM) * VaD * deeP;
            }
        }
#pragma unroll
        for (int x = 0; x < 3; ++x) F.m[x][c] = area_scaled<S>(faB, mF[x]);
    }
    T gF[5] = {T(0), T(0), T(0), T(0), T(0)}, dW[5] = {T(0), T(0), T(0), T(0), T(0)};
    const T igm1 = T(1.0 / (p.gamma - 1));
    gasKin<T>(igm1, T(-1), WL, Tf, gF, dW);
    gasKin<T>(igm1, T(1), WR, Tf, gF, dW);
    T cH = T(p.cHogH);
#pragma unroll
    for (int v = 0; v < 5; ++v) gF[v] = gF[v] - cH * VaD * dW[v];
    if (p.doBoris) {  // nuclear option, stress.F90:399-417 (cLim = 1.5)
        T vL = sqrt(WL[1] * WL[1] + WL[2] * WL[2] + WL[3] * WL[3]);
        T vR = sqrt(WR[1] * WR[1] + WR[2] * WR[2] + WR[3] * WR[3]);
        T Vn = sqrt(vL * vL + vR * vR) / T(1.41421353816986083984375);   // sqrt(2.0) of a default-real literal
        if (Vn >= T(1.5) * T(p.Ca)) {
#pragma unroll
            for (int v = 0; v < 5; ++v) gF[v] = gF[v] - T(p.Ca) * T(h.gas[v][c] - h.gas[v][c - s]);
        }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) F.g[v][c] = area_scaled<S>(faB, gF[v]);
}

// Tensor maps of the staged planes of sweep D; false when a plane cannot be mapped or the tiles' x origins
// (i0-4 for the I sweep, i0 otherwise; tiles step by FL) would not be 16-byte aligned
template <typename S, int D, int FR>
static bool flux_maps(const Handle& h, const FluxSrc<S>& in, const Reg& r, bool mhd, FluxMaps& m) {
    const int x0 = D == 0 ? r.i0 - 4 : r.i0;
    if ((x0 * (int)sizeof(S)) % 16 != 0) return false;
    const int rb[3] = {D == 0 ? FL + 8 : FL, D == 0 ? FR : (D == 1 ? FR + 7 : 1), D == 2 ? FR + 7 : 1};
    const int lb[3] = {D == 0 ? FL + 8 : FL, D == 0 ? FR : (D == 1 ? FR + 3 : 1), D == 2 ? FR + 3 : 1};
    const S* rec[9] = {in.W[0], in.W[1], in.W[2], in.W[3], in.W[4], in.vol, in.B[0], in.B[1], in.B[2]};
    const S* lim[8] = {in.Wl[0], in.Wl[1], in.Wl[2], in.Wl[3], in.Wl[4], in.Bl[0], in.Bl[1], in.Bl[2]};
    for (int q = 0; q < (mhd ? 9 : 6); ++q)
        if (!tma::plane_map(&m.rec[q], rec[q], (int)sizeof(S), h.L, rb[0], rb[1], rb[2])) return false;
    for (int q = 0; q < (mhd ? 8 : 5); ++q)
        if (!tma::plane_map(&m.lim[q], lim[q], (int)sizeof(S), h.L, lb[0], lb[1], lb[2])) return false;
    return true;
}

template <typename T, typename S, int D, int FR>
static void launch_flux_rows(Handle& h, const FluxSrc<S>& in, const FluxOut<S>& F, const Reg& r, cudaStream_t st) {
    const Par& p = h.p;
    dim3 grid((unsigned)((r.ni + FL - 1) / FL), 0, 0);
    if (D == 2) { grid.y = (unsigned)((r.nk + FR - 1) / FR); grid.z = (unsigned)r.nj; }
    else { grid.y = (unsigned)((r.nj + FR - 1) / FR); grid.z = (unsigned)r.nk; }
    FluxMaps maps;
    memset(&maps, 0, sizeof(maps));
    if (h.tileTma && flux_maps<S, D, FR>(h, in, r, p.doMHD != 0, maps)) {
        const size_t sm = flux_smem<S, D, FR, true>();
        if (p.doMHD && p.doBackground)
            k_flux_tile<T, S, D, true, true, FR, true><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
        else if (p.doMHD)
            k_flux_tile<T, S, D, true, false, FR, true><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
        else k_flux_tile<T, S, D, false, false, FR, true><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
        return;
    }
    const size_t sm = flux_smem<S, D, FR>();
    if (p.doMHD && p.doBackground)
        k_flux_tile<T, S, D, true, true, FR, false><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
    else if (p.doMHD) k_flux_tile<T, S, D, true, false, FR, false><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
    else k_flux_tile<T, S, D, false, false, FR, false><<<grid, 32 * FR, sm, st>>>(h.L, p, maps, in, h.H, F, r, h.dScal);
}

template <typename T, typename S, int D>
static void launch_flux_dir(Handle& h, const FluxSrc<S>& in, const Reg& r, cudaStream_t st) {
    FluxOut<S> F;
    if constexpr (std::is_same<S, double>::value) {
        for (int v = 0; v < 5; ++v) F.g[v] = h.gflx[D][v];
        for (int x = 0; x < 3; ++x) F.m[x] = h.mflx[D][x];
    } else {   // FP32-flux path: the area-scaled fluxes are stored as floats
        for (int v = 0; v < 5; ++v) F.g[v] = h.f32.gflx[D][v];
        for (int x = 0; x < 3; ++x) F.m[x] = h.f32.mflx[D][x];
    }
    if (h.fluxRows == 4) launch_flux_rows<T, S, D, 4>(h, in, F, r, st);
    else launch_flux_rows<T, S, D, 8>(h, in, F, r, st);
    h.launches++;
}

template <typename T, typename S, int D, int FR, bool TMA>
static void set_flux_smem_kind() {
    const int sm = (int)flux_smem<S, D, FR, TMA>();
    cudaFuncSetAttribute(k_flux_tile<T, S, D, true, true, FR, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_flux_tile<T, S, D, true, false, FR, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_flux_tile<T, S, D, false, false, FR, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}
template <typename T, typename S, int D, int FR>
static void set_flux_smem_rows() {
    set_flux_smem_kind<T, S, D, FR, false>();
    set_flux_smem_kind<T, S, D, FR, true>();
}
template <typename T, typename S, int D>
static void set_flux_smem() {
    set_flux_smem_rows<T, S, D, 4>();
    set_flux_smem_rows<T, S, D, 8>();
}
// ------------------------------------------------------------------ ensembles: one tile queue for all members
// A job is one flux direction of one problem; its tiles are numbered from `first` in a single sequence
// over all jobs. The persistent kernel's CTAs take tile numbers from a counter until the sequence is done,
// find the job (jobs are sorted by `first`) and run the tile body of that problem and direction.
template <typename T, typename S, int D>
__device__ __forceinline__ void flux_job_tile(const FluxJob<S>& J, int bx, int by, int bz, unsigned char* sm) {
    if (J.kind == 2) flux_tile_body<T, S, D, true, true, 8>(J.L, J.p, J.in, J.h, J.F, J.r, bx, by, bz, sm);
    else if (J.kind == 1) flux_tile_body<T, S, D, true, false, 8>(J.L, J.p, J.in, J.h, J.F, J.r, bx, by, bz, sm);
    else flux_tile_body<T, S, D, false, false, 8>(J.L, J.p, J.in, J.h, J.F, J.r, bx, by, bz, sm);
}

template <typename T, typename S>
__global__ void __launch_bounds__(256, (sizeof(S) == 4 ? 4 : 3)) k_flux_queue(const FluxJob<S>* jobs, int njobs,
                                                                             long long ntiles,
                                                                             unsigned long long* counter) {
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ long long item;
    for (;;) {
        if (threadIdx.x == 0) item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long t = item;
        if (t >= ntiles) break;
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].first <= t) lo = mid;
            else hi = mid - 1;
        }
        const FluxJob<S>& J = jobs[lo];
        const long long u = t - J.first;
        const int bx = (int)(u % J.gx), by = (int)((u / J.gx) % J.gy), bz = (int)(u / ((long long)J.gx * J.gy));
        if (J.D == 0) flux_job_tile<T, S, 0>(J, bx, by, bz, smraw);
        else if (J.D == 1) flux_job_tile<T, S, 1>(J, bx, by, bz, smraw);
        else flux_job_tile<T, S, 2>(J, bx, by, bz, smraw);
        __syncthreads();   // every thread is done with the staged tile (and has read `item`)
    }
}

template <typename S> constexpr size_t flux_queue_smem() {
    return flux_smem<S, 1, 8>() > flux_smem<S, 0, 8>() ? flux_smem<S, 1, 8>() : flux_smem<S, 0, 8>();
}

// the jobs of one problem's flux directions, tiles numbered on from `first`
template <typename S>
static void flux_jobs_of(Handle& h, const FluxSrc<S>& in, const FluxOut<S> F[3], std::vector<FluxJob<S>>& jobs,
                         long long& first) {
    const Lay& L = h.L;
    int is = L.is(), ie = L.ie(), js = L.js(), je = L.je(), ks = L.ks(), ke = L.ke();
    if (h.p.do25D) ke = ks;
    const Reg regs[3] = {mkreg(is, ie + 1, js, je, ks, ke), mkreg(is, ie, js, je + 1, ks, ke),
                         mkreg(is, ie, js, je, ks, ke + 1)};
    for (int D = 0; D < (h.p.do25D ? 2 : 3); ++D) {
        FluxJob<S> J;
        J.L = L; J.p = h.p; J.in = in; J.h = h.H; J.F = F[D]; J.r = regs[D]; J.D = D;
        J.kind = h.p.doMHD ? (h.p.doBackground ? 2 : 1) : 0;
        const Reg& r = regs[D];
        J.gx = (r.ni + FL - 1) / FL;
        int gz;
        if (D == 2) { J.gy = (r.nk + 8 - 1) / 8; gz = r.nj; }
        else { J.gy = (r.nj + 8 - 1) / 8; gz = r.nk; }
        J.first = first;
        first += (long long)J.gx * J.gy * gz;
        jobs.push_back(J);
    }
}

// CalcStress flux loop (stress.F90:84-128): I, J and (unless 2.5D) K interfaces
template <typename T, typename S>
static void fluxes_all(Handle& h, const FluxSrc<S>& in, cudaStream_t st) {
    const Lay& L = h.L;
    int is = L.is(), ie = L.ie(), js = L.js(), je = L.je(), ks = L.ks(), ke = L.ke();
    if (h.p.do25D) ke = ks;
    launch_flux_dir<T, S, 0>(h, in, mkreg(is, ie + 1, js, je, ks, ke), st);
    launch_flux_dir<T, S, 1>(h, in, mkreg(is, ie, js, je + 1, ks, ke), st);
    if (!h.p.do25D) launch_flux_dir<T, S, 2>(h, in, mkreg(is, ie, js, je, ks, ke + 1), st);
}

}  // namespace gam
