// DivB without any allocation, for callers that cannot call cudaMalloc.
//
// Some hosts of this step cannot allocate device memory themselves: a Fortran code whose device
// arrays are owned by another runtime (OpenACC/CUDA Fortran data regions, a coupler's memory pool), or
// a caller running inside a section where allocation is forbidden because it would synchronise the
// device or break its memory accounting. gam_gpu_divb needs a handle, and the handle owns a pool
// allocated with cudaMalloc. gam_divb_noalloc computes the same diagnostic straight from caller-provided
// device copies of magFlux (and of the background face fluxes bFlux0 when the problem has a background
// field) and writes the total to a caller-provided device double. The formula is the reference's DivB
// (src/gamera/gridutils.F90:717-770; the function itself has no counterpart there). Its only scratch --
// one partial sum per 256-cell block -- lives in the file-scope array below, which every GPU that loads
// this library holds until the process exits (512 KiB).
#include <cstdio>
#include <mutex>
#include <cuda_runtime.h>
#include "gamgpu.h"

namespace {

constexpr int kThreads = 256;
constexpr long long kMaxCells = GAM_DIVB_NOALLOC_MAX_CELLS;
constexpr int kMaxBlocks = (int)(kMaxCells / kThreads);
static_assert(kMaxCells % kThreads == 0, "the cell limit is a whole number of blocks");

// One partial sum per block. Shared by every call on a device and kept between calls; every call
// writes the partials of all the blocks it reads, so nothing has to start at zero.
static __device__ __align__(256) double g_divb_partials[kMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {nullptr};   // host-side device address of g_divb_partials, per device

// magFlux(isg:ieg+1, jsg:jeg+1, ksg:keg+1, 1:3) and, when given, Grid%bFlux0(isg:ieg, jsg:jeg, ksg:keg, 1:3)
// in the Fortran layout; active cells only. Per cell |dFi + dFj + dFk + dFi0 + dFj0 + dFk0| as DivB sums it.
__global__ void k_divb_blocks(const double* __restrict__ mf, const double* __restrict__ bf0, int Nip, int Njp,
                              int Nkp, int nG, double* partials) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long n = (long long)Nip * Njp * Nkp;
    double v = 0.0;
    if (t < n) {
        int i = (int)(t % Nip) + nG;
        long long q = t / Nip;
        int j = (int)(q % Njp) + nG, k = (int)(q / Njp) + nG;
        long long fi = Nip + 2 * nG + 1, fj = Njp + 2 * nG + 1, fk = Nkp + 2 * nG + 1;
        long long plane = fi * fj * fk;
        long long c = i + fi * (j + fj * k);
        double dFi = mf[c] - mf[c + 1];
        double dFj = mf[plane + c] - mf[plane + c + fi];
        double dFk = mf[2 * plane + c] - mf[2 * plane + c + fi * fj];
        double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
        if (bf0) {
            long long ci = fi - 1, cj = fj - 1, cplane = ci * cj * (fk - 1);
            long long b = i + ci * (j + cj * k);
            dFi0 = bf0[b] - bf0[b + 1];
            dFj0 = bf0[cplane + b] - bf0[cplane + b + ci];
            dFk0 = bf0[2 * cplane + b] - bf0[2 * cplane + b + ci * cj];
        }
        v = fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
    }
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __shared__ double ws[kThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < kThreads / 32 ? ws[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) partials[blockIdx.x] = v;
    }
}

// Fixed-order sum of the nb partials (deterministic across calls)
__global__ void k_divb_total(const double* partials, int nb, double* out) {
    __shared__ double ws[32];
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v += partials[b];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        v = lane < nw ? ws[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) *out = v;
    }
}

// Device address of the static scratch on the current device, looked up once per device and kept for the
// life of the process (a cudaDeviceReset of that device invalidates it; the entry point is not for use on
// a device after a reset).
int scratch_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { std::fprintf(stderr, "gam_divb_noalloc: cudaGetDevice: %s\n", cudaGetErrorString(e)); return GAM_ERR_CUDA; }
    if (dev < 0 || dev >= kMaxDevices) return GAM_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_divb_partials);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "gam_divb_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
            return GAM_ERR_CUDA;
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return GAM_OK;
}

}  // namespace

extern "C" int gam_divb_noalloc(const double* magflux_dev, const double* bflux0_dev, int Nip, int Njp, int Nkp,
                                int nG, double* tot_dev) {
    if (!magflux_dev || !tot_dev || Nip < 1 || Njp < 1 || Nkp < 1 || nG < 0) return GAM_ERR_ARG;
    // an error left pending by the caller's own work is reported, not cleared, and nothing is launched
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        std::fprintf(stderr, "gam_divb_noalloc: an earlier CUDA error is pending: %s\n", cudaGetErrorString(pending));
        return GAM_ERR_CUDA;
    }
    long long n = (long long)Nip * Njp * Nkp;
    if (n > kMaxCells) {
        std::fprintf(stderr, "gam_divb_noalloc: %lld active cells exceed the static limit of %lld\n", n, kMaxCells);
        return GAM_ERR_ARG;
    }
    double* partials = nullptr;
    int rc = scratch_address(&partials);
    if (rc) return rc;
    int nb = (int)((n + kThreads - 1) / kThreads);
    k_divb_blocks<<<nb, kThreads>>>(magflux_dev, bflux0_dev, Nip, Njp, Nkp, nG, partials);
    k_divb_total<<<1, 1024>>>(partials, nb, tot_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { std::fprintf(stderr, "gam_divb_noalloc: launch: %s\n", cudaGetErrorString(e)); return GAM_ERR_CUDA; }
    return GAM_OK;
}
