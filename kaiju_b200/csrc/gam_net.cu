// The closure network's kernels: weight packing, the tcgen05 implicit-GEMM convolution (forward and
// backward-data), the weight gradient, the bias gradient and Adam. Layout and GEMM mapping: gam_net.cuh.
#include <cstdio>

#include "gam_net.cuh"
#include "gam_tc.cuh"

namespace gam {
namespace {

constexpr uint32_t WAIT_LIMIT = 1u << 24;   // mbarrier polls before a wait gives up (well above any MMA time)

__device__ __forceinline__ float bf2f(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}
__host__ __device__ __forceinline__ long long tap_off(int t, int P, int Q) {
    int di = t % 3 - 1, dj = (t / 3) % 3 - 1, dk = t / 9 - 1;
    return (long long)di + (long long)P * (dj + (long long)Q * dk);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);   // a at the lower address
    return *reinterpret_cast<uint32_t*>(&h);
}

enum { MODE_HIDDEN = 0, MODE_OUT = 1, MODE_BWD = 2 };

struct ConvArgs {
    const __nv_bfloat16* x;    // input planes [cin][E]
    const __nv_bfloat16* gz;   // MODE_BWD: the A operand is x * gelu'(gz) when non-null
    const __nv_bfloat16* w;    // packed weights, 27 taps of [COUTP x CINP] K-major blocks
    const float* bias;         // [cout] (MODE_HIDDEN, MODE_OUT)
    __nv_bfloat16* y;          // MODE_HIDDEN: GELU(z); MODE_BWD: the input gradient
    __nv_bfloat16* z;          // MODE_HIDDEN: pre-activation (null: not kept)
    float* yf;                 // MODE_OUT: output planes [cout][E]
    long long E, c0, c1;
    int P, Q, cin, cout;
    int* err;
};

template <int CINP, int COUTP>
struct ConvSmem {
    static constexpr int TAPB = COUTP * CINP * 2;
    static constexpr int WB = 27 * TAPB;
    static constexpr int WBA = (WB + 1023) / 1024 * 1024;
    static constexpr int AB = 128 * CINP * 2;
    static constexpr int BYTES = WBA + 2 * AB + 1024;
};

__device__ __forceinline__ unsigned char* align1k(unsigned char* p) {
    uint32_t s = tc::smem_u32(p);
    return p + ((1024u - (s & 1023u)) & 1023u);
}

// out[cell][n] = sum over taps t and input channels c of A_t[cell][c] * W_t[n][c], 128 cells per tile
template <int CINP, int COUTP, int MODE>
__global__ void __launch_bounds__(128) k_conv(ConvArgs a) {
    static_assert(CINP % 16 == 0 && COUTP % 16 == 0 && COUTP <= 32, "tile shape");
    using S = ConvSmem<CINP, COUTP>;
    extern __shared__ unsigned char smraw[];
    unsigned char* sW = align1k(smraw);
    unsigned char* sA = sW + S::WBA;
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmemBase;
    const int tid = threadIdx.x, warp = tid >> 5;

    for (int q = tid; q < S::WB / 16; q += 128)
        reinterpret_cast<uint4*>(sW)[q] = reinterpret_cast<const uint4*>(a.w)[q];
    if (tid == 0) {
        tc::mbar_init(&mbar[0], 1);
        tc::mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmemBase, 32);
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmemBase;
    const uint32_t idesc = tc::idesc_bf16_f32(128, COUTP);
    constexpr uint32_t SBO = CINP / 8 * 128;
    const unsigned short* xs = reinterpret_cast<const unsigned short*>(a.x);
    const bool gated = MODE == MODE_BWD && a.gz != nullptr;

    uint32_t use0 = 0, use1 = 0;
    int ok = 1, it = 0;
    const long long ntiles = (a.c1 - a.c0 + 127) / 128;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long cell0 = a.c0 + tile * 128;
        for (int t = 0; t < 27; ++t, ++it) {
            const int b = it & 1;
            const uint32_t use = b ? use1 : use0;
            bool fine = true;
            if (use > 0) fine = tc::mbar_wait(&mbar[b], (use - 1) & 1u, WAIT_LIMIT);
            unsigned char* dA = sA + b * S::AB;
            if (fine) {
                const long long cell = cell0 + tid + tap_off(t, a.P, a.Q);
                const bool inb = cell >= 0 && cell < a.E;
#pragma unroll
                for (int kc = 0; kc < CINP / 8; ++kc) {
                    uint32_t pk[4];
#pragma unroll
                    for (int e = 0; e < 8; e += 2) {
                        const int c = kc * 8 + e;
                        if (!gated) {
                            uint32_t lo = (inb && c < a.cin) ? xs[(long long)c * a.E + cell] : 0u;
                            uint32_t hi = (inb && c + 1 < a.cin) ? xs[(long long)(c + 1) * a.E + cell] : 0u;
                            pk[e / 2] = lo | (hi << 16);
                        } else {
                            float f0 = 0.f, f1 = 0.f;
                            if (inb && c < a.cin)
                                f0 = bf2f(a.x[(long long)c * a.E + cell]) * gelu_d(bf2f(a.gz[(long long)c * a.E + cell]));
                            if (inb && c + 1 < a.cin)
                                f1 = bf2f(a.x[(long long)(c + 1) * a.E + cell]) *
                                     gelu_d(bf2f(a.gz[(long long)(c + 1) * a.E + cell]));
                            pk[e / 2] = pack2(f0, f1);
                        }
                    }
                    *reinterpret_cast<uint4*>(dA + tc::kmajor_off(tid, kc * 8, CINP)) =
                        make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
            }
            tc::fence_smem_async();
            if (!__syncthreads_and(fine)) { ok = 0; break; }
            if (tid == 0) {
                tc::fence_after_sync();
#pragma unroll
                for (int ks = 0; ks < CINP / 16; ++ks) {
                    uint64_t ad = tc::desc_kmajor(tc::smem_u32(dA) + ks * 256, 128, SBO);
                    uint64_t bd = tc::desc_kmajor(tc::smem_u32(sW + t * S::TAPB) + ks * 256, 128, SBO);
                    tc::mma_bf16(tbase, ad, bd, idesc, t > 0 || ks > 0);
                }
                tc::mma_commit(&mbar[b]);
            }
            if (b) ++use1; else ++use0;
        }
        if (!ok) break;
        const int bl = (it - 1) & 1;
        const uint32_t ul = bl ? use1 : use0;
        bool fine = tc::mbar_wait(&mbar[bl], (ul - 1) & 1u, WAIT_LIMIT);
        if (!__syncthreads_and(fine)) { ok = 0; break; }
        tc::fence_after_sync();
        float acc[32];
        tc::tmem_ld32(tbase + ((uint32_t)(warp * 32) << 16), acc);
        const long long cell = cell0 + tid;
        if (cell < a.c1) {
#pragma unroll
            for (int co = 0; co < 32; ++co) {
                if (co >= a.cout) break;
                const long long o = (long long)co * a.E + cell;
                if (MODE == MODE_HIDDEN) {
                    float zf = acc[co] + a.bias[co];
                    if (a.z) a.z[o] = __float2bfloat16_rn(zf);
                    a.y[o] = __float2bfloat16_rn(gelu(zf));
                } else if (MODE == MODE_OUT) {
                    a.yf[o] = acc[co] + a.bias[co];
                } else {
                    a.y[o] = __float2bfloat16_rn(acc[co]);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    if (!ok) {
        if (tid == 0) atomicExch(a.err, 1);
        // MMAs still in flight read this CTA's shared memory and write its TMEM: let them finish
        if (use0) tc::mbar_wait(&mbar[0], (use0 - 1) & 1u, WAIT_LIMIT);
        if (use1) tc::mbar_wait(&mbar[1], (use1 - 1) & 1u, WAIT_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, 32);
}

// ------------------------------------------------------------------ weight gradient
struct DwArgs {
    const __nv_bfloat16* x;    // layer input planes [cin][E]
    const __nv_bfloat16* dy;   // gradient w.r.t. the layer output [cout][E]
    const __nv_bfloat16* z;    // pre-activation of a hidden layer (the gradient is gated by gelu'(z)), or null
    float* partial;            // [gridDim.x][NG][128][COUTP]
    long long E, c0, c1;
    int P, Q, cin, cout;
    int* err;
};

template <int CINP, int COUTP>
struct DwShape {
    static constexpr int G = 128 / CINP;                  // taps per 128-row group
    static constexpr int NG = (27 + G - 1) / G;
    static constexpr int AB = 128 * 16 * 2;               // one group's A: 128 rows x 16 cells
    static constexpr int BB = COUTP * 16 * 2;
    static constexpr int STAGE = (NG * AB + BB + 1023) / 1024 * 1024;
    static constexpr int COLS = NG * COUTP <= 32 ? 32 : NG * COUTP <= 64 ? 64 : NG * COUTP <= 128 ? 128 : 256;
    // request enough shared memory that TMEM (512 columns per SM) always covers the resident CTAs
    static constexpr int BYTES_MIN = 2 * STAGE + 1024;
    static constexpr int PER_SM = 512 / COLS;
    static constexpr int BYTES = BYTES_MIN > (228 * 1024 / PER_SM - 2048) ? BYTES_MIN : (228 * 1024 / PER_SM - 2048);
};

// D[(tap, ci)][co] = sum over cells of x[ci][cell + off(tap)] * dy'[co][cell], 16 cells per MMA
template <int CINP, int COUTP>
__global__ void __launch_bounds__(128) k_conv_dw(DwArgs a) {
    using S = DwShape<CINP, COUTP>;
    extern __shared__ unsigned char smraw[];
    unsigned char* sbase = align1k(smraw);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmemBase;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        tc::mbar_init(&mbar[0], 1);
        tc::mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmemBase, S::COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmemBase;
    const uint32_t idesc = tc::idesc_bf16_f32(128, COUTP);
    const unsigned short* xs = reinterpret_cast<const unsigned short*>(a.x);

    uint32_t use0 = 0, use1 = 0;
    int ok = 1, it = 0;
    const long long nsteps = (a.c1 - a.c0 + 15) / 16;
    for (long long s = blockIdx.x; s < nsteps; s += gridDim.x, ++it) {
        const long long cell0 = a.c0 + s * 16;
        const int b = it & 1;
        const uint32_t use = b ? use1 : use0;
        bool fine = true;
        if (use > 0) fine = tc::mbar_wait(&mbar[b], (use - 1) & 1u, WAIT_LIMIT);
        unsigned char* st = sbase + b * S::STAGE;
        if (fine) {
            // A: row m = tid of every group: x[ci][cell0 + k + off(tap)] for k = 0..15
            const int ci = tid % CINP;
#pragma unroll 1
            for (int g = 0; g < S::NG; ++g) {
                const int t = g * S::G + tid / CINP;
                uint32_t pk[8];
                const bool live = t < 27 && ci < a.cin;
                const long long base = (long long)ci * a.E + cell0 + (live ? tap_off(t, a.P, a.Q) : 0);
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    const long long c = cell0 + k + (live ? tap_off(t, a.P, a.Q) : 0);
                    uint32_t lo = (live && c >= 0 && c < a.E) ? xs[base + k] : 0u;
                    uint32_t hi = (live && c + 1 >= 0 && c + 1 < a.E) ? xs[base + k + 1] : 0u;
                    pk[k / 2] = lo | (hi << 16);
                }
                unsigned char* dA = st + g * S::AB;
                *reinterpret_cast<uint4*>(dA + tc::kmajor_off(tid, 0, 16)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *reinterpret_cast<uint4*>(dA + tc::kmajor_off(tid, 8, 16)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            // B: row n = output channel, 16 cells of the (gated) output gradient
            if (tid < COUTP * 2) {
                const int n = tid >> 1, h = tid & 1;
                uint32_t pk[4];
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    float f[2];
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const long long c = cell0 + h * 8 + k + q;
                        f[q] = 0.f;
                        if (n < a.cout && c < a.c1) {
                            const long long o = (long long)n * a.E + c;
                            f[q] = bf2f(a.dy[o]);
                            if (a.z) f[q] *= gelu_d(bf2f(a.z[o]));
                        }
                    }
                    pk[k / 2] = pack2(f[0], f[1]);
                }
                *reinterpret_cast<uint4*>(st + S::NG * S::AB + tc::kmajor_off(n, h * 8, 16)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
        }
        tc::fence_smem_async();
        if (!__syncthreads_and(fine)) { ok = 0; break; }
        if (tid == 0) {
            tc::fence_after_sync();
            const uint64_t bd = tc::desc_kmajor(tc::smem_u32(st + S::NG * S::AB), 128, 256);
#pragma unroll 1
            for (int g = 0; g < S::NG; ++g) {
                const uint64_t ad = tc::desc_kmajor(tc::smem_u32(st + g * S::AB), 128, 256);
                tc::mma_bf16(tbase + g * COUTP, ad, bd, idesc, it > 0);
            }
            tc::mma_commit(&mbar[b]);
        }
        if (b) ++use1; else ++use0;
    }
    if (ok && it > 0) {
        const int bl = (it - 1) & 1;
        const uint32_t ul = bl ? use1 : use0;
        bool fine = tc::mbar_wait(&mbar[bl], (ul - 1) & 1u, WAIT_LIMIT);
        ok = __syncthreads_and(fine);
    }
    float* part = a.partial + (long long)blockIdx.x * S::NG * 128 * COUTP;
    if (ok) {
        tc::fence_after_sync();
#pragma unroll 1
        for (int g = 0; g < S::NG; ++g) {
            float acc[32];
            if (it > 0) tc::tmem_ld32(tbase + ((uint32_t)(warp * 32) << 16) + g * COUTP, acc);
            else for (int q = 0; q < 32; ++q) acc[q] = 0.f;
            float* row = part + ((long long)g * 128 + tid) * COUTP;
#pragma unroll
            for (int n = 0; n < COUTP; ++n) row[n] = acc[n];
        }
    } else {
        if (tid == 0) atomicExch(a.err, 1);
        if (use0) tc::mbar_wait(&mbar[0], (use0 - 1) & 1u, WAIT_LIMIT);
        if (use1) tc::mbar_wait(&mbar[1], (use1 - 1) & 1u, WAIT_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, S::COLS);
}

// grads W[t][co][ci] of one layer = the fixed-order sum of the CTAs' partials
template <int CINP, int COUTP>
__global__ void k_dw_reduce(const float* partial, int nblk, float* gW, int cin, int cout) {
    using S = DwShape<CINP, COUTP>;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= 27 * cout * cin) return;
    const int ci = id % cin, co = (id / cin) % cout, t = id / (cin * cout);
    const int g = t / S::G, m = (t % S::G) * CINP + ci;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += partial[(((long long)b * S::NG + g) * 128 + m) * COUTP + co];
    gW[id] = (float)s;
}

// bias gradient: per-block partial sums of the (gated) output gradient over the cell range, then a fixed-order sum
__global__ void k_bias_partial(const __nv_bfloat16* dy, const __nv_bfloat16* z, long long E, long long c0,
                               long long c1, int cout, float* part) {
    __shared__ float red[256];
    for (int co = 0; co < cout; ++co) {
        float s = 0.f;
        for (long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < c1;
             c += (long long)gridDim.x * blockDim.x) {
            const long long o = (long long)co * E + c;
            float v = bf2f(dy[o]);
            if (z) v *= gelu_d(bf2f(z[o]));
            s += v;
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * cout + co] = red[0];
        __syncthreads();
    }
}
__global__ void k_bias_reduce(const float* part, int nblk, int cout, float* gb) {
    const int co = threadIdx.x;
    if (co >= cout) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(long long)b * cout + co];
    gb[co] = (float)s;
}

// ------------------------------------------------------------------ packing and Adam
// forward blocks: tap t, row n = output channel, K = input channel; backward-data blocks: tap 26 - t
// (the mirrored offset), row n = input channel, K = output channel
__global__ void k_pack(const float* W, int cin, int cout, __nv_bfloat16* fwd, int fCinP, int fCoutP,
                       __nv_bfloat16* bwd, int bCinP, int bCoutP) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= 27 * cout * cin) return;
    const int ci = id % cin, co = (id / cin) % cout, t = id / (cin * cout);
    const __nv_bfloat16 w = __float2bfloat16_rn(W[id]);
    fwd[((long long)t * fCoutP * fCinP * 2 + tc::kmajor_off(co, ci, fCinP)) / 2] = w;
    if (bwd) bwd[((long long)(26 - t) * bCoutP * bCinP * 2 + tc::kmajor_off(ci, co, bCinP)) / 2] = w;
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline int pad16(int c) { return (c + 15) / 16 * 16; }

template <typename K>
void set_smem(K kern, int bytes) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

int g_sms = 0;
int sm_count() {
    if (!g_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_sms <= 0) g_sms = 148;
    }
    return g_sms;
}

template <int CINP, int COUTP, int MODE>
void launch_conv(const ConvArgs& a, cudaStream_t st) {
    using S = ConvSmem<CINP, COUTP>;
    long long ntiles = (a.c1 - a.c0 + 127) / 128;
    long long grid = sm_count() * 3;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    k_conv<CINP, COUTP, MODE><<<(unsigned)grid, 128, S::BYTES, st>>>(a);
}

}  // namespace

// shared-memory limits of every kernel instance (set once, outside any stream capture)
int net_init() {
    set_smem(k_conv<16, 32, MODE_HIDDEN>, ConvSmem<16, 32>::BYTES);
    set_smem(k_conv<32, 32, MODE_HIDDEN>, ConvSmem<32, 32>::BYTES);
    set_smem(k_conv<32, 32, MODE_OUT>, ConvSmem<32, 32>::BYTES);
    set_smem(k_conv<32, 32, MODE_BWD>, ConvSmem<32, 32>::BYTES);
    set_smem(k_conv_dw<16, 32>, DwShape<16, 32>::BYTES);
    set_smem(k_conv_dw<32, 32>, DwShape<32, 32>::BYTES);
    sm_count();
    return (int)cudaGetLastError();
}

int net_dw_blocks() { return sm_count() * 2; }
long long net_partial_floats(int nblocks) {
    // the largest layer: CINP 32 -> 7 groups of 128 x 32
    return (long long)nblocks * 7 * 128 * 32;
}
size_t net_act_bytes(long long E) { return (size_t)E * sizeof(__nv_bfloat16); }

int net_pack_weights(const float* params, __nv_bfloat16* wfwd[NET_LAYERS], __nv_bfloat16* wbwd[NET_LAYERS],
                     cudaStream_t st) {
    NetShape s = net_shape();
    for (int l = 0; l < NET_LAYERS; ++l) {
        const int fCinP = pad16(s.cin[l]), fCoutP = 32, bCinP = pad16(s.cout[l]), bCoutP = 32;
        cudaMemsetAsync(wfwd[l], 0, sizeof(__nv_bfloat16) * 27 * fCinP * fCoutP, st);
        if (wbwd[l]) cudaMemsetAsync(wbwd[l], 0, sizeof(__nv_bfloat16) * 27 * bCinP * bCoutP, st);
        const int n = 27 * s.cin[l] * s.cout[l];
        k_pack<<<(n + 255) / 256, 256, 0, st>>>(params + net_param_offset(l), s.cin[l], s.cout[l], wfwd[l], fCinP,
                                                fCoutP, wbwd[l], bCinP, bCoutP);
    }
    return (int)cudaGetLastError();
}

int net_forward(const NetBox& b, __nv_bfloat16* const wfwd[NET_LAYERS], const float* params, NetBuffers& nb,
                bool keepPre, int* err, cudaStream_t st) {
    NetShape s = net_shape();
    for (int l = 0; l < NET_LAYERS; ++l) {
        ConvArgs a{};
        a.x = nb.act[l];
        a.w = wfwd[l];
        a.bias = params + net_param_offset(l) + 27LL * s.cout[l] * s.cin[l];
        a.E = b.E; a.c0 = b.c0; a.c1 = b.c1; a.P = b.P; a.Q = b.Q;
        a.cin = s.cin[l]; a.cout = s.cout[l];
        a.err = err;
        if (l < NET_LAYERS - 1) {
            a.y = nb.act[l + 1];
            a.z = keepPre ? nb.pre[l] : nullptr;
            if (l == 0) launch_conv<16, 32, MODE_HIDDEN>(a, st);
            else launch_conv<32, 32, MODE_HIDDEN>(a, st);
        } else {
            a.yf = nb.out;
            launch_conv<32, 32, MODE_OUT>(a, st);
        }
    }
    return (int)cudaGetLastError();
}

template <int CINP, int COUTP>
static void launch_dw(const DwArgs& a, int nblk, float* gW, cudaStream_t st) {
    using S = DwShape<CINP, COUTP>;
    k_conv_dw<CINP, COUTP><<<nblk, 128, S::BYTES, st>>>(a);
    const int n = 27 * a.cin * a.cout;
    k_dw_reduce<CINP, COUTP><<<(n + 255) / 256, 256, 0, st>>>(a.partial, nblk, gW, a.cin, a.cout);
}

// gradients of every parameter from the output gradient nb.gact[0] (planar bf16, NET_OUT planes), given
// the activations and pre-activations of the last forward (keepPre)
int net_backward(const NetBox& b, __nv_bfloat16* const wbwd[NET_LAYERS], NetBuffers& nb, float* grads, int* err,
                 cudaStream_t st) {
    NetShape s = net_shape();
    const int nblk = net_dw_blocks();
    for (int l = NET_LAYERS - 1; l >= 0; --l) {
        // gradient w.r.t. this layer's output, and the gate (its pre-activation) for hidden layers
        const __nv_bfloat16* dy = l == NET_LAYERS - 1 ? nb.gact[0] : nb.gact[l + 1];
        const __nv_bfloat16* z = l == NET_LAYERS - 1 ? nullptr : nb.pre[l];
        DwArgs d{};
        d.x = nb.act[l]; d.dy = dy; d.z = z; d.partial = nb.partial;
        d.E = b.E; d.c0 = b.c0; d.c1 = b.c1; d.P = b.P; d.Q = b.Q; d.cin = s.cin[l]; d.cout = s.cout[l]; d.err = err;
        float* gW = grads + net_param_offset(l);
        if (l == 0) launch_dw<16, 32>(d, nblk, gW, st);
        else launch_dw<32, 32>(d, nblk, gW, st);
        k_bias_partial<<<nblk, 256, 0, st>>>(dy, z, b.E, b.c0, b.c1, s.cout[l], nb.partial);
        k_bias_reduce<<<1, 32, 0, st>>>(nb.partial, nblk, s.cout[l], gW + 27LL * s.cout[l] * s.cin[l]);
        if (l > 0) {   // gradient w.r.t. this layer's input (the previous layer's GELU output)
            ConvArgs a{};
            a.x = dy; a.gz = z; a.w = wbwd[l];
            a.y = nb.gact[l];
            a.E = b.E; a.c0 = b.c0; a.c1 = b.c1; a.P = b.P; a.Q = b.Q;
            a.cin = s.cout[l]; a.cout = s.cin[l]; a.err = err;
            launch_conv<32, 32, MODE_BWD>(a, st);
        }
    }
    return (int)cudaGetLastError();
}

int net_adam(float* params, const float* grads, float* m, float* v, long long n, float lr, float b1, float b2,
             float eps, int step, cudaStream_t st) {
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(params, grads, m, v, n, lr, b1, b2, eps, c1, c2);
    return (int)cudaGetLastError();
}

}  // namespace gam
