// Kernel-side helpers shared by the step kernels: launch regions, pointer bundles, the one-sided
// kinetic fluxes, and row-wise cp.async staging of a box of a pencil plane into shared memory (the
// variant the tile kernels use where tensor copies do not apply; gam_tma.cuh has the tensor copies).
#pragma once
#include <vector>
#include "gam_common.cuh"

namespace gam {

struct Reg {
    int i0, ni, j0, nj, k0, nk;
    __host__ __device__ long long n() const { return (long long)ni * nj * nk; }
};
__device__ __forceinline__ bool reg_ijk(const Reg& r, long long t, int& i, int& j, int& k) {
    if (t >= r.n()) return false;
    i = r.i0 + (int)(t % r.ni);
    long long q = t / r.ni;
    j = r.j0 + (int)(q % r.nj);
    k = r.k0 + (int)(q / r.nj);
    return true;
}
// 3-D launch over a region: threadIdx.x runs along i (coalesced)
__device__ __forceinline__ bool reg3(const Reg& r, int& i, int& j, int& k) {
    i = r.i0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    j = r.j0 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    k = r.k0 + (int)(blockIdx.z * blockDim.z + threadIdx.z);
    return (i < r.i0 + r.ni) && (j < r.j0 + r.nj) && (k < r.k0 + r.nk);
}
// Launch over a region as (i, j) planes: blockIdx.y is k and the threads run linearly over the plane, i
// fastest -- one 32-bit division per thread, and idle lanes only in the last block of each plane
__device__ __forceinline__ bool reg_plane(const Reg& r, int& i, int& j, int& k) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)r.ni * (unsigned)r.nj) return false;
    const unsigned jj = t / (unsigned)r.ni;
    i = r.i0 + (int)(t - jj * (unsigned)r.ni);
    j = r.j0 + (int)jj;
    k = r.k0 + (int)blockIdx.y;
    return true;
}
static inline dim3 grid_plane(const Reg& r, int tpb) {
    return dim3((unsigned)(((long long)r.ni * r.nj + tpb - 1) / tpb), (unsigned)r.nk);
}
static inline dim3 grid3(const Reg& r, dim3 b) {
    return dim3((unsigned)((r.ni + b.x - 1) / b.x), (unsigned)((r.nj + b.y - 1) / b.y), (unsigned)((r.nk + b.z - 1) / b.z));
}
static inline Reg mkreg(int i0, int i1, int j0, int j1, int k0, int k1) {
    Reg r;
    r.i0 = i0; r.ni = i1 - i0 + 1; r.j0 = j0; r.nj = j1 - j0 + 1; r.k0 = k0; r.nk = k1 - k0 + 1;
    return r;
}
static inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

struct PrimP { double* w[5]; };
// Inputs of the flux kernels in storage type S (double planes for FP64, float copies for FP32-flux)
template <typename S> struct FluxSrc {
    const S* W[5];      // half-state primitives (reconstruction)
    const S* Wl[5];     // limiter primitives (state n, or the half state without LFM limiting)
    const S* B[3];      // half-state B
    const S* Bl[3];     // limiter B
    const S* vol;
    const S* Tf[3][9];
    const S* face[3];
    const S* bn[3];     // normal field on the face: half-state flux / area
    const S* fcB0[3][3];  // background: face-averaged B0 per face direction
    const S* b0[3];       // background normal field: bFlux0 (divided by the area in the kernel) for
                          // double storage, bFlux0/area for float storage
};
// Inputs of the edge kernels
template <typename S> struct EdgeSrc {
    const S* Vf[3];
    const S* face[3];
    const S* hbA[3];
    const S* nbA[3];
    const S* rho;       // half-state density
    const S* Te[3][6];  // T1 (x,y,z), T2 (x,y,z) of each edge direction
    const S* Teb[3][4];
    const S* edge[3];
    const S* edgB0[3][2]; // background: edge-frame B0 (tangents 1, 2) per edge direction
};
struct Vec3P { double* v[3]; };
// interface fluxes (area-scaled) of one direction: double planes, or float planes on the FP32-flux path
template <typename O> struct FluxOut { O* g[5]; O* m[3]; };
using FluxP = FluxOut<double>;

// one flux direction of one problem in the ensembles' tile queue (gam_flux_tile.cuh)
template <typename S> struct FluxJob {
    Lay L;
    Par p;
    FluxSrc<S> in;
    StateP h;
    FluxOut<S> F;
    Reg r;
    int D, kind;   // kind: 0 hydro, 1 MHD, 2 MHD with a background field
    int gx, gy;
    long long first;
};
struct Handle;
void flux_jobs64(Handle& h, int cur, std::vector<FluxJob<double>>& jobs, long long& first);
void flux_jobs32(Handle& h, std::vector<FluxJob<float>>& jobs, long long& first);
void launch_flux_queue64(const FluxJob<double>* jobs, int njobs, long long ntiles, unsigned long long* counter,
                         int grid, cudaStream_t st);
void launch_flux_queue32(const FluxJob<float>* jobs, int njobs, long long ntiles, unsigned long long* counter,
                         int grid, cudaStream_t st);

// 1 / sqrt(x) from the math library's reciprocal square root, in the precision of T
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }

// erfc of the kinetic flux splitting. Near zero -- where the flow is slow against the thermal or magnetosonic
// speed, most interfaces of a problem -- it is 1 - erf(x) with erf from its Maclaurin series
// (Abramowitz & Stegun 7.1.5: erf(x) = 2/sqrt(pi) sum_n (-1)^n x^(2n+1) / (n! (2n+1))), evaluated by Horner in
// x^2: 13 terms reach double precision for |x| <= 1/2 (the first term left out is below 5e-18 of the sum), 8
// terms single precision. That is 15 fused multiply-adds where the library's double-precision erfc costs
// about 84 of this GPU's FP64 operations; above 1/2 the library's erfc is used. erfc stays above 0.47 on
// |x| <= 1/2, so 1 - erf loses no relative precision.
template <typename T> struct ErfcSeries;
template <> struct ErfcSeries<double> { static constexpr int N = 13; };
template <> struct ErfcSeries<float> { static constexpr int N = 8; };
__host__ __device__ constexpr double erf_series_coef(int n) {
    // (-1)^n / (n! (2n+1))
    return n == 0 ? 1.0 : n == 1 ? -1.0 / 3.0 : n == 2 ? 1.0 / 10.0 : n == 3 ? -1.0 / 42.0 : n == 4 ? 1.0 / 216.0
         : n == 5 ? -1.0 / 1320.0 : n == 6 ? 1.0 / 9360.0 : n == 7 ? -1.0 / 75600.0 : n == 8 ? 1.0 / 685440.0
         : n == 9 ? -1.0 / 6894720.0 : n == 10 ? 1.0 / 76204800.0 : n == 11 ? -1.0 / 918086400.0
         : 1.0 / 11975040000.0;
}
template <typename T>
__device__ __forceinline__ T erfc_k(T x) {
    if (fabs(x) <= T(0.5)) {
        const T z = x * x;
        constexpr int N = ErfcSeries<T>::N;
        T s = T(erf_series_coef(N - 1));
#pragma unroll
        for (int n = N - 2; n >= 0; --n) s = fma(s, z, T(erf_series_coef(n)));
        return fma(T(-1.1283791670955125739) * x, s, T(1));   // 1 - (2/sqrt(pi)) x s
    }
    return erfc(x);
}

// One-sided gas kinetic flux (stress.F90:432-511). igm1 = 1 / (gamma - 1). The reference's sqrt(lambda)
// and 1 / sqrt(pi lambda) come from one reciprocal square root of lambda (divisions are the FP64 flux
// kernel's costliest operations; the results differ by an ulp or so).
template <typename T>
__device__ __forceinline__ void gasKin(T igm1, T sg, const T* W, const T* Tf, T* gF, T* dW) {
    T D = W[0], Vx = W[1], Vy = W[2], Vz = W[3], P = W[4];
    T E = T(0.5) * D * (Vx * Vx + Vy * Vy + Vz * Vz) + P * igm1;
    T lambda = D / (T(2) * P);
    T rl = rsq(lambda);   // 1 / sqrt(lambda)
    T Vn = Tf[0] * Vx + Tf[1] * Vy + Tf[2] * Vz;
    T Vt1 = Tf[3] * Vx + Tf[4] * Vy + Tf[5] * Vz;
    T Vt2 = Tf[6] * Vx + Tf[7] * Vy + Tf[8] * Vz;
    T Vn0 = T(0.5) * erfc_k<T>(sg * (lambda * rl) * Vn);
    T Vn1 = Vn * Vn0 - T(0.5) * sg * exp(-(lambda * Vn * Vn)) * (rl * T(0.56418958354775628695));   // 1/sqrt(pi)
    gF[0] = gF[0] + D * Vn1;
    gF[4] = gF[4] + (E + T(0.5) * P) * Vn1 + T(0.5) * P * Vn0 * Vn;
    T fMn = D * Vn * Vn1 + P * Vn0;
    T fMt1 = D * Vt1 * Vn1;
    T fMt2 = D * Vt2 * Vn1;
    gF[1] = gF[1] + (Tf[0] * fMn + Tf[3] * fMt1 + Tf[6] * fMt2);
    gF[2] = gF[2] + (Tf[1] * fMn + Tf[4] * fMt1 + Tf[7] * fMt2);
    gF[3] = gF[3] + (Tf[2] * fMn + Tf[5] * fMt1 + Tf[8] * fMt2);
    dW[0] = dW[0] + sg * D;
    dW[1] = dW[1] + sg * D * Vx;
    dW[2] = dW[2] + sg * D * Vy;
    dW[3] = dW[3] + sg * D * Vz;
    dW[4] = dW[4] + sg * E;
}
// One-sided magnetic stress (stress.F90:513-599). With a background field (BG) the Alfven speed and
// bbD use the total field and the stress gains the B0 cross terms; B0 is the face-averaged background
// and B0n its normal component.
template <typename T, bool BG = false>
__device__ __forceinline__ void magKin(const Par& p, T sg, const T* W, const T* B, T Bn, const T* Tf, T* mF, T& bbD,
                                       T& VaD, const T* B0 = nullptr, T B0n = T(0)) {
    T D = W[0], P = W[4];
    T iD = T(1) / D;   // one reciprocal for the reference's three divisions by rho
    T dPb = T(0.5) * (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    T Va2;
    if constexpr (BG) {
        T Bt0 = B[0] + B0[0], Bt1 = B[1] + B0[1], Bt2 = B[2] + B0[2];
        Va2 = (Bt0 * Bt0 + Bt1 * Bt1 + Bt2 * Bt2) * iD;
        bbD = bbD + T(0.5) * (Bt0 * Bt0 + Bt1 * Bt1 + Bt2 * Bt2);
    } else {
        Va2 = T(2) * dPb * iD;
        bbD = bbD + T(0.5) * (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    }
    T Vac2 = Va2;
    if (p.doBoris) Vac2 = Va2 / (T(1) + Va2 * T(1.0 / (p.Ca * p.Ca)));
    T Vn = Tf[0] * W[1] + Tf[1] * W[2] + Tf[2] * W[3];
    // lambda = 1 / (2P/rho + Va^2) enters only as sqrt(lambda): one reciprocal square root
    T Vn0 = T(0.5) * erfc_k<T>(sg * rsq(T(2) * P * iD + Vac2) * Vn);
    VaD = VaD + T(0.5) * sqrt(Vac2);
    mF[0] = mF[0] + Vn0 * (dPb * Tf[0] - B[0] * Bn);
    mF[1] = mF[1] + Vn0 * (dPb * Tf[1] - B[1] * Bn);
    mF[2] = mF[2] + Vn0 * (dPb * Tf[2] - B[2] * Bn);
    if constexpr (BG) {
        T BdB0 = B0[0] * B[0] + B0[1] * B[1] + B0[2] * B[2];
        mF[0] = mF[0] + Vn0 * (-B0[0] * Bn - B[0] * B0n + BdB0 * Tf[0]);
        mF[1] = mF[1] + Vn0 * (-B0[1] * Bn - B[1] * B0n + BdB0 * Tf[1]);
        mF[2] = mF[2] + Vn0 * (-B0[2] * Bn - B[2] * B0n + BdB0 * Tf[2]);
    }
}

// Asynchronous global->shared copies (cp.async, 8 bytes each): every thread keeps all of its copies in
// flight at once instead of one load at a time.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
template <typename S> __device__ __forceinline__ void cp_async_elem(S* smem, const S* gmem);
template <> __device__ __forceinline__ void cp_async_elem<double>(double* smem, const double* gmem) { cp_async8(smem, gmem); }
template <> __device__ __forceinline__ void cp_async_elem<float>(float* smem, const float* gmem) { cp_async4(smem, gmem); }

// Row-wise staging: the box [gi0,gi0+ni) x [gj0,gj0+nj) x [gk0,gk0+nk) (absolute pencil indices) is
// copied row by row, one warp per row, lanes along i, one cp.async per element; each row's address is
// computed once. Out-of-range elements are zero.
template <typename S>
__device__ __forceinline__ void stage_rows(S* dst, const S* __restrict__ src, const Lay& L, int gi0, int ni,
                                           int gj0, int nj, int gk0, int nk, int warp, int nwarp, int lane) {
    const int nrow = nj * nk;
    for (int rr = warp; rr < nrow; rr += nwarp) {
        int b = rr % nj, c = rr / nj;
        int j = gj0 + b, k = gk0 + c;
        S* drow = dst + rr * ni;
        bool ok = (j >= 0) && (j <= L.Nj) && (k >= 0) && (k <= L.Nk);
        const S* srow = src + L.at(0, ok ? j : 0, ok ? k : 0);
        for (int a = lane; a < ni; a += 32) {
            int i = gi0 + a;
            if (ok && i >= 0 && i <= L.Ni) cp_async_elem<S>(drow + a, srow + i);
            else drow[a] = S(0);
        }
    }
}

}  // namespace gam
