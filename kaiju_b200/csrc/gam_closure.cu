// The learned flux closure object: the network's parameters (FP32 master copy, Adam moments, BF16 packed
// weights), its activation planes over one grid's cell box, and the entry points that run it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "gam_net.cuh"
#include "gam_step.cuh"
#include "gamgpu.h"

using namespace gam;

struct gam_closure {
    Lay L;                       // the grid's pencil layout (as a solver handle of that grid has it)
    NetBox box;
    int device = 0;
    cudaStream_t stream = nullptr;
    long long np = 0;
    float* params = nullptr;     // device FP32 master parameters
    float* grads = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    int adamStep = 0;
    __nv_bfloat16* wfwd[NET_LAYERS] = {};
    __nv_bfloat16* wbwd[NET_LAYERS] = {};
    NetBuffers nb{};
    void* pool = nullptr;        // activation planes
    float* stage = nullptr;      // host-layout staging (largest: NET_OUT or NET_IN planes of the box)
    int* err = nullptr;
    bool packed = false;
};

namespace {

#define CKC(x)                                                                               \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess) {                                                             \
            std::fprintf(stderr, "gamgpu closure: %s: %s\n", #x, cudaGetErrorString(e_));    \
            return GAM_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

Lay make_lay(int Nip, int Njp, int Nkp) {
    Lay L{};
    L.Nip = Nip; L.Njp = Njp; L.Nkp = Nkp; L.nG = 4;
    L.Ni = Nip + 8; L.Nj = Njp + 8; L.Nk = Nkp + 8;
    L.P = ((L.Ni + 1) + 7) / 8 * 8;
    L.Q = L.Nj + 1; L.R = L.Nk + 1;
    L.E = (long long)L.P * L.Q * L.R;
    return L;
}

// Fortran (Ni,Nj,Nk,nc) host layout -> planar bf16 planes at the pencil index
__global__ void k_in_from_fortran(Lay L, const float* src, int nc, __nv_bfloat16* dst) {
    const long long n = (long long)L.Ni * L.Nj * L.Nk;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % L.Ni), j = (int)((t / L.Ni) % L.Nj), k = (int)(t / ((long long)L.Ni * L.Nj));
    const long long c = L.at(i, j, k);
    for (int q = 0; q < nc; ++q) dst[(long long)q * L.E + c] = __float2bfloat16_rn(src[t + q * n]);
}
// active cells of fp32 planes -> Fortran (Nip,Njp,Nkp,nc)
__global__ void k_out_to_fortran(Lay L, const float* src, int nc, float* dst) {
    const long long n = (long long)L.Nip * L.Njp * L.Nkp;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % L.Nip), j = (int)((t / L.Nip) % L.Njp), k = (int)(t / ((long long)L.Nip * L.Njp));
    const long long c = L.at(i + 4, j + 4, k + 4);
    for (int q = 0; q < nc; ++q) dst[t + q * n] = src[(long long)q * L.E + c];
}
// Fortran (Nip,Njp,Nkp,nc) gradient of the active cells -> bf16 planes (zero elsewhere)
__global__ void k_gout_from_fortran(Lay L, const float* src, int nc, __nv_bfloat16* dst) {
    const long long n = (long long)L.Nip * L.Njp * L.Nkp;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % L.Nip), j = (int)((t / L.Nip) % L.Njp), k = (int)(t / ((long long)L.Nip * L.Njp));
    const long long c = L.at(i + 4, j + 4, k + 4);
    for (int q = 0; q < nc; ++q) dst[(long long)q * L.E + c] = __float2bfloat16_rn(src[t + q * n]);
}

int closure_pack(gam_closure* C) {
    if (net_pack_weights(C->params, C->wfwd, C->wbwd, C->stream) != 0) return GAM_ERR_CUDA;
    C->packed = true;
    return GAM_OK;
}

int check_err(gam_closure* C) {
    int e = 0;
    CKC(cudaMemcpyAsync(&e, C->err, sizeof(int), cudaMemcpyDeviceToHost, C->stream));
    CKC(cudaStreamSynchronize(C->stream));
    return e ? GAM_ERR_TIMEOUT : GAM_OK;
}

}  // namespace

extern "C" {

int gam_closure_create(gam_closure_t** out, int Nip, int Njp, int Nkp, unsigned long long seed) {
    if (!out || Nip < 8 || Njp < 1 || Nkp < 1) return GAM_ERR_ARG;
    *out = nullptr;
    gam_closure* C = new (std::nothrow) gam_closure();
    if (!C) return GAM_ERR_ARG;
    C->L = make_lay(Nip, Njp, Nkp);
    const Lay& L = C->L;
    C->box.P = L.P; C->box.Q = L.Q; C->box.E = L.E;
    const long long margin = (long long)L.P * L.Q + L.P + 1;
    C->box.c0 = margin;
    C->box.c1 = L.E - margin;
    cudaGetDevice(&C->device);
    C->np = net_num_params();
    int rc = GAM_OK;
    auto fail = [&](int r) { gam_closure_destroy(C); return r; };
    if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(GAM_ERR_CUDA);
    const size_t pbytes = sizeof(float) * C->np;
    if (cudaMalloc(&C->params, pbytes) || cudaMalloc(&C->grads, pbytes) || cudaMalloc(&C->m, pbytes) ||
        cudaMalloc(&C->v, pbytes) || cudaMalloc(&C->err, sizeof(int)))
        return fail(GAM_ERR_CUDA);
    NetShape s = net_shape();
    for (int l = 0; l < NET_LAYERS; ++l) {
        const int fc = (s.cin[l] + 15) / 16 * 16, bc = (s.cout[l] + 15) / 16 * 16;
        if (cudaMalloc(&C->wfwd[l], sizeof(__nv_bfloat16) * 27 * fc * 32) ||
            cudaMalloc(&C->wbwd[l], sizeof(__nv_bfloat16) * 27 * bc * 32))
            return fail(GAM_ERR_CUDA);
    }
    // activation planes: act (8 + 3*32), pre (3*32), gact (24 + 3*32) bf16; out (24) fp32
    const long long E = L.E;
    const long long bfPlanes = NET_IN + 3 * NET_WIDTH + 3 * NET_WIDTH + NET_OUT + 3 * NET_WIDTH;
    const size_t bytes = sizeof(__nv_bfloat16) * E * bfPlanes + sizeof(float) * E * NET_OUT;
    if (cudaMalloc(&C->pool, bytes) != cudaSuccess) return fail(GAM_ERR_CUDA);
    cudaMemsetAsync(C->pool, 0, bytes, C->stream);
    __nv_bfloat16* q = static_cast<__nv_bfloat16*>(C->pool);
    C->nb.act[0] = q; q += E * NET_IN;
    for (int l = 1; l < NET_LAYERS; ++l) { C->nb.act[l] = q; q += E * NET_WIDTH; }
    for (int l = 0; l < NET_LAYERS - 1; ++l) { C->nb.pre[l] = q; q += E * NET_WIDTH; }
    C->nb.pre[NET_LAYERS - 1] = nullptr;
    C->nb.gact[0] = q; q += E * NET_OUT;
    for (int l = 1; l < NET_LAYERS; ++l) { C->nb.gact[l] = q; q += E * NET_WIDTH; }
    C->nb.out = reinterpret_cast<float*>(q);
    C->nb.partialFloats = net_partial_floats(net_dw_blocks());
    if (cudaMalloc(&C->nb.partial, sizeof(float) * C->nb.partialFloats) != cudaSuccess) return fail(GAM_ERR_CUDA);
    const long long stageFloats = (long long)L.Ni * L.Nj * L.Nk * NET_OUT;
    if (cudaMalloc(&C->stage, sizeof(float) * stageFloats) != cudaSuccess) return fail(GAM_ERR_CUDA);
    cudaMemsetAsync(C->err, 0, sizeof(int), C->stream);
    cudaMemsetAsync(C->m, 0, pbytes, C->stream);
    cudaMemsetAsync(C->v, 0, pbytes, C->stream);
    // initial parameters: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) for the hidden layers, biases 0, and
    // the output layer at a tenth of that, so an untrained closure is a small correction
    std::vector<float> h(C->np, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < NET_LAYERS; ++l) {
        const double bound = (l == NET_LAYERS - 1 ? 0.1 : 1.0) / std::sqrt(27.0 * s.cin[l]);
        std::uniform_real_distribution<double> U(-bound, bound);
        float* w = h.data() + net_param_offset(l);
        for (long long k = 0; k < 27LL * s.cout[l] * s.cin[l]; ++k) w[k] = (float)U(rng);
    }
    if (cudaMemcpyAsync(C->params, h.data(), pbytes, cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
        return fail(GAM_ERR_CUDA);
    rc = closure_pack(C);
    if (rc) return fail(rc);
    if (cudaStreamSynchronize(C->stream) != cudaSuccess) return fail(GAM_ERR_CUDA);
    *out = C;
    return GAM_OK;
}

void gam_closure_destroy(gam_closure_t* C) {
    if (!C) return;
    if (C->stream) cudaStreamSynchronize(C->stream);
    cudaFree(C->params); cudaFree(C->grads); cudaFree(C->m); cudaFree(C->v); cudaFree(C->err);
    for (int l = 0; l < NET_LAYERS; ++l) { cudaFree(C->wfwd[l]); cudaFree(C->wbwd[l]); }
    cudaFree(C->pool); cudaFree(C->nb.partial); cudaFree(C->stage);
    if (C->stream) cudaStreamDestroy(C->stream);
    delete C;
}

long long gam_closure_num_params(const gam_closure_t* C) { return C ? C->np : -1; }

int gam_closure_set_params(gam_closure_t* C, const float* p, long long n) {
    if (!C || !p || n != C->np) return GAM_ERR_ARG;
    CKC(cudaMemcpyAsync(C->params, p, sizeof(float) * n, cudaMemcpyHostToDevice, C->stream));
    int rc = closure_pack(C);
    if (rc) return rc;
    CKC(cudaStreamSynchronize(C->stream));
    return GAM_OK;
}

int gam_closure_get_params(gam_closure_t* C, float* p, long long n) {
    if (!C || !p || n != C->np) return GAM_ERR_ARG;
    CKC(cudaMemcpyAsync(p, C->params, sizeof(float) * n, cudaMemcpyDeviceToHost, C->stream));
    CKC(cudaStreamSynchronize(C->stream));
    return GAM_OK;
}

int gam_closure_get_grads(gam_closure_t* C, float* g, long long n) {
    if (!C || !g || n != C->np) return GAM_ERR_ARG;
    CKC(cudaMemcpyAsync(g, C->grads, sizeof(float) * n, cudaMemcpyDeviceToHost, C->stream));
    CKC(cudaStreamSynchronize(C->stream));
    return GAM_OK;
}

int gam_closure_forward_host(gam_closure_t* C, const float* in, float* out) {
    if (!C || !in || !out) return GAM_ERR_ARG;
    const Lay& L = C->L;
    const long long nAll = (long long)L.Ni * L.Nj * L.Nk, nAct = (long long)L.Nip * L.Njp * L.Nkp;
    CKC(cudaMemcpyAsync(C->stage, in, sizeof(float) * nAll * NET_IN, cudaMemcpyHostToDevice, C->stream));
    k_in_from_fortran<<<(unsigned)((nAll + 255) / 256), 256, 0, C->stream>>>(L, C->stage, NET_IN, C->nb.act[0]);
    if (net_forward(C->box, C->wfwd, C->params, C->nb, true, C->err, C->stream) != 0) return GAM_ERR_CUDA;
    k_out_to_fortran<<<(unsigned)((nAct + 255) / 256), 256, 0, C->stream>>>(L, C->nb.out, NET_OUT, C->stage);
    CKC(cudaMemcpyAsync(out, C->stage, sizeof(float) * nAct * NET_OUT, cudaMemcpyDeviceToHost, C->stream));
    return check_err(C);
}

int gam_closure_backward_host(gam_closure_t* C, const float* in, const float* gout) {
    if (!C || !in || !gout) return GAM_ERR_ARG;
    const Lay& L = C->L;
    const long long nAll = (long long)L.Ni * L.Nj * L.Nk, nAct = (long long)L.Nip * L.Njp * L.Nkp;
    CKC(cudaMemcpyAsync(C->stage, in, sizeof(float) * nAll * NET_IN, cudaMemcpyHostToDevice, C->stream));
    k_in_from_fortran<<<(unsigned)((nAll + 255) / 256), 256, 0, C->stream>>>(L, C->stage, NET_IN, C->nb.act[0]);
    if (net_forward(C->box, C->wfwd, C->params, C->nb, true, C->err, C->stream) != 0) return GAM_ERR_CUDA;
    CKC(cudaStreamSynchronize(C->stream));
    CKC(cudaMemcpyAsync(C->stage, gout, sizeof(float) * nAct * NET_OUT, cudaMemcpyHostToDevice, C->stream));
    k_gout_from_fortran<<<(unsigned)((nAct + 255) / 256), 256, 0, C->stream>>>(L, C->stage, NET_OUT, C->nb.gact[0]);
    if (net_backward(C->box, C->wbwd, C->nb, C->grads, C->err, C->stream) != 0) return GAM_ERR_CUDA;
    return check_err(C);
}

}  // extern "C"
