// The learned flux closure's network on the device: a 3D convolution net over the solver's cell box
// (the pencil index space of gam_common.cuh, ghosts included), activations channels-last in BF16
// (cell-major, 16 or 32 channels per cell, so the channels of one cell are one to four 16-byte chunks),
// FP32 master weights.
//
//   input 8 (normalised primitives rho, v, P, B; padded to 16) -> 32 -> 32 -> 32 -> 27 (8 face-flux
//   corrections per direction: the 5 gas fluxes and the 3 magnetic-stress momentum fluxes of each cell's
//   lower face; then one EMF correction per direction on each cell's lower I, J and K edge), 3x3x3 kernels,
//   GELU between layers.
//
// Every convolution is an implicit GEMM on the tensor cores (tcgen05.mma kind::f16, BF16 x BF16 -> FP32
// in TMEM): a CTA owns 128 consecutive cells (M = 128) and all output channels (N = 32). For each of the
// 9 (dj, dk) offsets it copies (cp.async, 16-byte chunks) a window of 130 cells x input channels into
// shared memory, one block of rows per channel chunk with the rows 16 bytes apart, so the A operand of
// the three taps di = -1, 0, +1 is the same window read from row 0, 1 or 2 (a 16-byte shift of the
// descriptor's start address). Windows are triple-buffered: the copy of window w+2 overlaps the MMAs of
// window w. The weight gradient contracts over cells instead (M = 128 rows of (tap, input channel),
// N = output channels, K = 16 cells per MMA), each CTA accumulating all taps in TMEM over its cells and
// writing one partial that a fixed-order reduction sums.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace gam {

constexpr int NET_LAYERS = 4;
constexpr int NET_IN = 8, NET_WIDTH = 32, NET_OUT = 27;
constexpr int NET_FACE_OUT = 24;   // outputs 0..23: face fluxes (direction d, flux v at d*8+v); 24..26: edge EMFs

struct NetShape {
    int cin[NET_LAYERS], cout[NET_LAYERS];
};
__host__ __device__ inline NetShape net_shape() {
    NetShape s{};
    s.cin[0] = NET_IN; s.cout[0] = NET_WIDTH;
    s.cin[1] = NET_WIDTH; s.cout[1] = NET_WIDTH;
    s.cin[2] = NET_WIDTH; s.cout[2] = NET_WIDTH;
    s.cin[3] = NET_WIDTH; s.cout[3] = NET_OUT;
    return s;
}
// parameters of layer l: W[27][cout][cin] then b[cout], layers back to back
inline long long net_layer_params(int l) {
    NetShape s = net_shape();
    return 27LL * s.cout[l] * s.cin[l] + s.cout[l];
}
inline long long net_param_offset(int l) {
    long long o = 0;
    for (int q = 0; q < l; ++q) o += net_layer_params(q);
    return o;
}
inline long long net_num_params() { return net_param_offset(NET_LAYERS); }

// the cell box the net runs over: the solver's pencil layout of one grid
struct NetBox {
    int P, Q;          // pencil strides (cells per row incl. padding, rows per plane)
    long long E;       // cells per plane
    long long c0, c1;  // GEMM cell range: every tap of every cell in it stays inside [0, E)
};

constexpr int NET_IN_PITCH = 16;     // channels per cell of the input activations (8 used)
constexpr int NET_PITCH = 32;        // channels per cell of every other activation and gradient

struct NetBuffers {
    __nv_bfloat16* act[NET_LAYERS];     // act[0] = input (pitch 16); act[l] = GELU output of layer l-1 (pitch 32)
    __nv_bfloat16* pre[NET_LAYERS];     // pre-activation of layer l (l < NET_LAYERS - 1), pitch 32
    float* out;                         // the output layer, planar fp32: NET_OUT planes
    __nv_bfloat16* grad[NET_LAYERS];    // gradient w.r.t. layer l's pre-activation (grad[3]: the output), pitch 32
    float* partial;                     // weight-gradient partials
    long long partialFloats;
};

// host launchers (gam_net.cu); each returns 0 or a CUDA error code
int net_pack_weights(const float* params, __nv_bfloat16* wfwd[NET_LAYERS], __nv_bfloat16* wbwd[NET_LAYERS],
                     cudaStream_t st);
int net_forward(const NetBox& b, __nv_bfloat16* const wfwd[NET_LAYERS], const float* params, NetBuffers& nb,
                bool keepPre, int* err, cudaStream_t st);
int net_backward(const NetBox& b, __nv_bfloat16* const wbwd[NET_LAYERS], NetBuffers& nb, float* grads, int* err,
                 cudaStream_t st);
int net_adam(float* params, const float* grads, float* m, float* v, long long n, float lr, float b1, float b2,
             float eps, int step, cudaStream_t st);
int net_init();
long long net_partial_floats(int nblocks);
int net_dw_blocks();
size_t net_act_bytes(long long E);

}  // namespace gam
