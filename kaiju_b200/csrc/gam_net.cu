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
    const __nv_bfloat16* x;    // input activations, channels-last with pitch CINP
    const __nv_bfloat16* gz;   // MODE_BWD: pre-activation of the previous layer (pitch 32): the epilogue
                               // multiplies the input gradient by its GELU derivative
    const __nv_bfloat16* w;    // packed weights, 27 taps of [32 x CINP] K-major blocks
    const float* bias;         // [cout] (MODE_HIDDEN, MODE_OUT)
    __nv_bfloat16* y;          // MODE_HIDDEN: GELU(z); MODE_BWD: the previous layer's gradient (pitch 32)
    __nv_bfloat16* z;          // MODE_HIDDEN: pre-activation (null: not kept), pitch 32
    float* yf;                 // MODE_OUT: output planes [cout][E]
    long long E, c0, c1;
    int P, Q, cout;
    int* err;
};

template <int CINP>
struct ConvShape {
    static constexpr int COUTP = 32;
    static constexpr int ROWS = 130;                   // 128 cells and one on each side (di = -1, +1)
    static constexpr int KCH = CINP / 8;               // 16-byte channel chunks per cell
    static constexpr int LBO = ROWS * 16;              // bytes between the channel-chunk blocks of a window
    static constexpr int WIN = KCH * LBO;
    static constexpr int TAPB = COUTP * CINP * 2;      // one tap's packed weights
    static constexpr int WB = (27 * TAPB + 1023) / 1024 * 1024;   // all taps, resident for the CTA's life
    static constexpr int STAGE = (WIN + 127) / 128 * 128;
    static constexpr int NS = 5;                       // window stages in the ring
    static constexpr int BYTES = WB + NS * STAGE + 1024;
    static constexpr int THREADS = 160;                // 4 worker warps (copies, epilogue) + 1 MMA warp
};

__device__ __forceinline__ unsigned char* align1k(unsigned char* p) {
    uint32_t s = tc::smem_u32(p);
    return p + ((1024u - (s & 1023u)) & 1023u);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(tc::smem_u32(dst)), "l"(src), "r"(bytes)
                 : "memory");
}
// arrive on the mbarrier once every cp.async this thread issued so far has landed
__device__ __forceinline__ void cp_async_arrive(uint64_t* mbar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"(tc::smem_u32(mbar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" :: "r"(tc::smem_u32(mbar))
                 : "memory");
}

// out[cell][n] = sum over taps t and input channels c of in[cell + off(t)][c] * W_t[n][c], 128 cells per tile.
// The weights of all 27 taps stay in shared memory. Warps 0-3 copy windows into a ring of NS stages (full[s] completes when the 128 threads' copies of a
// window have landed) and run the epilogue of each finished tile (warp w reads TMEM lanes 32w..32w+31);
// one thread of warp 4 issues the MMAs of a window once its stage is full and commits them to empty[s]
// (the stage may be refilled) and, after a tile's last window, to tfull[a] (accumulator a is ready).
// Two TMEM accumulators alternate between tiles; tempty[a] completes when the workers have read one.
template <int CINP, int MODE>
__global__ void __launch_bounds__(160) k_conv(ConvArgs a) {
    using S = ConvShape<CINP>;
    static_assert(CINP % 16 == 0, "K step");
    extern __shared__ unsigned char smraw[];
    unsigned char* sW = align1k(smraw);
    unsigned char* sStage = sW + S::WB;
    __shared__ __align__(8) uint64_t full[S::NS], empty[S::NS], tfull[2], tempty[2], wready;
    __shared__ uint32_t tmemBase;
    __shared__ int failed;
    __shared__ float sBias[32];
    const int tid = threadIdx.x, warp = tid >> 5;

    // the bias, once per CTA: the epilogue reads it from shared memory instead of 32 global loads per tile
    if (tid < 32) sBias[tid] = (MODE != MODE_BWD && tid < a.cout) ? a.bias[tid] : 0.f;
    if (tid == 0) {
        for (int q = 0; q < S::NS; ++q) { tc::mbar_init(&full[q], 128); tc::mbar_init(&empty[q], 1); }
        for (int q = 0; q < 2; ++q) { tc::mbar_init(&tfull[q], 1); tc::mbar_init(&tempty[q], 128); }
        tc::mbar_init(&wready, 128);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmemBase, 64);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmemBase;

    const long long ntiles = (a.c1 - a.c0 + 127) / 128;
    const long long myTiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp < 4) {
        // ---------------- workers: copies and epilogues
        auto epilogue = [&](long long T) -> bool {
            const int acc = (int)(T & 1);
            if (!tc::mbar_wait(&tfull[acc], (uint32_t)((T >> 1) & 1), WAIT_LIMIT)) return false;
            tc::fence_after_sync();
            float v[32];
            tc::tmem_ld32(tbase + ((uint32_t)(warp * 32) << 16) + acc * 32, v);
            tc::fence_before_sync();
            mbar_arrive(&tempty[acc]);
            const long long cell = a.c0 + (blockIdx.x + T * (long long)gridDim.x) * 128 + tid;
            if (cell >= a.c1) return true;
            if (MODE == MODE_OUT) {
#pragma unroll
                for (int co = 0; co < 32; ++co)
                    if (co < a.cout) a.yf[(long long)co * a.E + cell] = v[co] + sBias[co];
                return true;
            }
            uint32_t py[16], pz[16];
            if (MODE == MODE_BWD) {
                const uint4* g4 = reinterpret_cast<const uint4*>(a.gz + cell * NET_PITCH);
                uint32_t gz[16];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint4 u = g4[q];
                    gz[4 * q] = u.x; gz[4 * q + 1] = u.y; gz[4 * q + 2] = u.z; gz[4 * q + 3] = u.w;
                }
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&gz[q]);
                    py[q] = pack2(v[2 * q] * gelu_d(__low2float(h)), v[2 * q + 1] * gelu_d(__high2float(h)));
                }
            } else {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int c0 = 2 * q, c1 = 2 * q + 1;
                    const float z0 = c0 < a.cout ? v[c0] + sBias[c0] : 0.f;
                    const float z1 = c1 < a.cout ? v[c1] + sBias[c1] : 0.f;
                    pz[q] = pack2(z0, z1);
                    py[q] = pack2(gelu(z0), gelu(z1));
                }
            }
            uint4* y4 = reinterpret_cast<uint4*>(a.y + cell * NET_PITCH);
#pragma unroll
            for (int q = 0; q < 4; ++q) y4[q] = make_uint4(py[4 * q], py[4 * q + 1], py[4 * q + 2], py[4 * q + 3]);
            if (MODE == MODE_HIDDEN && a.z) {
                uint4* z4 = reinterpret_cast<uint4*>(a.z + cell * NET_PITCH);
#pragma unroll
                for (int q = 0; q < 4; ++q) z4[q] = make_uint4(pz[4 * q], pz[4 * q + 1], pz[4 * q + 2], pz[4 * q + 3]);
            }
            return true;
        };
        // the weights of all taps, once
        for (int id = tid; id < 27 * S::TAPB / 16; id += 128)
            cp_async16(sW + id * 16, reinterpret_cast<const unsigned char*>(a.w) + id * 16, 16u);
        cp_async_arrive(&wready);
        bool ok = true;
        for (long long T = 0; T < myTiles && ok; ++T) {
            const long long cell0 = a.c0 + (blockIdx.x + T * (long long)gridDim.x) * 128;
            for (int w = 0; w < 9 && ok; ++w) {
                const long long it = T * 9 + w;
                const int st = (int)(it % S::NS);
                const long long use = it / S::NS;
                if (use > 0 && !tc::mbar_wait(&empty[st], (uint32_t)((use - 1) & 1), WAIT_LIMIT)) { ok = false; break; }
                const int dj = w % 3 - 1, dk = w / 3 - 1;
                const long long base = cell0 - 1 + (long long)a.P * (dj + (long long)a.Q * dk);
                unsigned char* dst = sStage + st * S::STAGE;
                for (int id = tid; id < S::ROWS * S::KCH; id += 128) {
                    const int row = id / S::KCH, kc = id % S::KCH;
                    const long long cell = base + row;
                    const bool inb = cell >= 0 && cell < a.E;
                    cp_async16(dst + kc * S::LBO + row * 16, a.x + (inb ? cell : 0) * CINP + kc * 8, inb ? 16u : 0u);
                }
                cp_async_arrive(&full[st]);
            }
            if (ok && T > 0) ok = epilogue(T - 1);
        }
        if (ok && myTiles > 0) ok = epilogue(myTiles - 1);
        if (!ok) failed = 1;
        cp_async_wait_all();
    } else if (tid == 128) {
        // ---------------- MMA issue
        const uint32_t idesc = tc::idesc_bf16_f32(128, S::COUTP);
        constexpr uint32_t SBO_W = CINP / 8 * 128;
        long long issued = 0;   // windows whose MMAs were committed
        bool ok = myTiles == 0 || tc::mbar_wait(&wready, 0u, WAIT_LIMIT);
        for (long long T = 0; T < myTiles && ok; ++T) {
            const int acc = (int)(T & 1);
            if (T >= 2 && !tc::mbar_wait(&tempty[acc], (uint32_t)(((T >> 1) - 1) & 1), WAIT_LIMIT)) { ok = false; break; }
            for (int w = 0; w < 9; ++w) {
                const long long it = T * 9 + w;
                const int st = (int)(it % S::NS);
                if (!tc::mbar_wait(&full[st], (uint32_t)((it / S::NS) & 1), WAIT_LIMIT)) { ok = false; break; }
                tc::fence_smem_async();   // the generic-proxy copies, to the tensor core
                tc::fence_after_sync();
                const uint32_t win = tc::smem_u32(sStage + st * S::STAGE);
                const uint32_t wt = tc::smem_u32(sW) + (3 * (w % 3) + 9 * (w / 3)) * S::TAPB;   // taps of (dj, dk)
#pragma unroll
                for (int di = -1; di <= 1; ++di) {
#pragma unroll
                    for (int ks = 0; ks < CINP / 16; ++ks) {
                        const uint64_t ad = tc::desc_kmajor(win + (di + 1) * 16 + ks * 2 * S::LBO, S::LBO, 128);
                        const uint64_t bd = tc::desc_kmajor(wt + (di + 1) * S::TAPB + ks * 256, 128, SBO_W);
                        tc::mma_bf16(tbase + acc * 32, ad, bd, idesc, !(w == 0 && di == -1 && ks == 0));
                    }
                }
                tc::mma_commit(&empty[st]);
                if (w == 8) tc::mma_commit(&tfull[acc]);
                ++issued;
            }
        }
        if (!ok) {
            failed = 1;
            // the MMAs already issued read shared memory and write TMEM: wait for the last commit
            if (issued > 0) {
                const long long it = issued - 1;
                tc::mbar_wait(&empty[(int)(it % S::NS)], (uint32_t)((it / S::NS) & 1), WAIT_LIMIT);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0 && failed) atomicExch(a.err, 1);
    if (warp == 0) tc::tmem_free(tbase, 64);
}

// ------------------------------------------------------------------ weight gradient
struct DwArgs {
    const __nv_bfloat16* x;    // layer input activations, channels-last with pitch CINP
    const __nv_bfloat16* dy;   // gradient w.r.t. the layer's pre-activation, channels-last pitch 32
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
                const long long c0 = cell0 + (live ? tap_off(t, a.P, a.Q) : 0);
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    const long long c = c0 + k;
                    uint32_t lo = (live && c >= 0 && c < a.E) ? xs[c * CINP + ci] : 0u;
                    uint32_t hi = (live && c + 1 >= 0 && c + 1 < a.E) ? xs[(c + 1) * CINP + ci] : 0u;
                    pk[k / 2] = lo | (hi << 16);
                }
                unsigned char* dA = st + g * S::AB;
                *reinterpret_cast<uint4*>(dA + tc::kmajor_off(tid, 0, 16)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *reinterpret_cast<uint4*>(dA + tc::kmajor_off(tid, 8, 16)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            // B: row n = output channel, 16 cells of the gradient w.r.t. the pre-activation
            if (tid < COUTP * 2) {
                const int n = tid >> 1, h = tid & 1;
                const unsigned short* dys = reinterpret_cast<const unsigned short*>(a.dy);
                uint32_t pk[4];
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    const long long c = cell0 + h * 8 + k;
                    uint32_t lo = (n < a.cout && c < a.c1) ? dys[c * NET_PITCH + n] : 0u;
                    uint32_t hi = (n < a.cout && c + 1 < a.c1) ? dys[(c + 1) * NET_PITCH + n] : 0u;
                    pk[k / 2] = lo | (hi << 16);
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

// bias gradient: per-block partial sums of the gradient w.r.t. the pre-activation over the cell range, then
// a fixed-order sum
__global__ void k_bias_partial(const __nv_bfloat16* dy, long long c0, long long c1, int cout, float* part) {
    __shared__ float red[256];
    for (int co = 0; co < cout; ++co) {
        float s = 0.f;
        for (long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < c1;
             c += (long long)gridDim.x * blockDim.x)
            s += bf2f(dy[c * NET_PITCH + co]);
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

template <int CINP, int MODE>
void launch_conv(const ConvArgs& a, cudaStream_t st) {
    using S = ConvShape<CINP>;
    long long ntiles = (a.c1 - a.c0 + 127) / 128;
    long long grid = sm_count() * (CINP == 16 ? 4 : 2);
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    k_conv<CINP, MODE><<<(unsigned)grid, S::THREADS, S::BYTES, st>>>(a);
}

}  // namespace

// shared-memory limits of every kernel instance (set once, outside any stream capture)
int net_init() {
    set_smem(k_conv<16, MODE_HIDDEN>, ConvShape<16>::BYTES);
    set_smem(k_conv<32, MODE_HIDDEN>, ConvShape<32>::BYTES);
    set_smem(k_conv<32, MODE_OUT>, ConvShape<32>::BYTES);
    set_smem(k_conv<32, MODE_BWD>, ConvShape<32>::BYTES);
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
        a.cout = s.cout[l];
        a.err = err;
        if (l < NET_LAYERS - 1) {
            a.y = nb.act[l + 1];
            a.z = keepPre ? nb.pre[l] : nullptr;
            if (l == 0) launch_conv<16, MODE_HIDDEN>(a, st);
            else launch_conv<32, MODE_HIDDEN>(a, st);
        } else {
            a.yf = nb.out;
            launch_conv<32, MODE_OUT>(a, st);
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

// gradients of every parameter from the output gradient nb.grad[3] (channels-last, pitch 32), given the
// activations and pre-activations of the last forward (keepPre)
int net_backward(const NetBox& b, __nv_bfloat16* const wbwd[NET_LAYERS], NetBuffers& nb, float* grads, int* err,
                 cudaStream_t st) {
    NetShape s = net_shape();
    const int nblk = net_dw_blocks();
    for (int l = NET_LAYERS - 1; l >= 0; --l) {
        DwArgs d{};
        d.x = nb.act[l]; d.dy = nb.grad[l]; d.partial = nb.partial;
        d.E = b.E; d.c0 = b.c0; d.c1 = b.c1; d.P = b.P; d.Q = b.Q; d.cin = s.cin[l]; d.cout = s.cout[l]; d.err = err;
        float* gW = grads + net_param_offset(l);
        if (l == 0) launch_dw<16, 32>(d, nblk, gW, st);
        else launch_dw<32, 32>(d, nblk, gW, st);
        k_bias_partial<<<nblk, 256, 0, st>>>(nb.grad[l], b.c0, b.c1, s.cout[l], nb.partial);
        k_bias_reduce<<<1, 32, 0, st>>>(nb.partial, nblk, s.cout[l], gW + 27LL * s.cout[l] * s.cin[l]);
        if (l > 0) {   // gradient w.r.t. the previous layer's pre-activation: through this layer, then GELU'
            ConvArgs a{};
            a.x = nb.grad[l]; a.gz = nb.pre[l - 1]; a.w = wbwd[l];
            a.y = nb.grad[l - 1];
            a.E = b.E; a.c0 = b.c0; a.c1 = b.c1; a.P = b.P; a.Q = b.Q;
            a.cout = s.cin[l]; a.err = err;
            launch_conv<32, MODE_BWD>(a, st);
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
