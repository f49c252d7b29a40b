// The learned flux closure object: the network's parameters (FP32 master copy, Adam moments, BF16 packed
// weights), its activation planes over one grid's cell box, and the entry points that run it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "gam_kern.cuh"
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
    // normalisation: net input (rho, vx, vy, vz, P, Bx, By, Bz) = (prim - inMean) / inScale; face
    // correction of variable v = net output * fluxScale[v] * face area; loss terms / resScale[v]
    float inMean[8] = {0, 0, 0, 0, 0, 0, 0, 0}, inScale[8] = {1, 1, 1, 1, 1, 1, 1, 1};
    float fluxScale[8] = {1, 1, 1, 1, 1, 1, 1, 1}, resScale[5] = {1, 1, 1, 1, 1};
    // EMF corrections: the EMF of an edge of direction e gains output 24+e times emfScale[e] times the edge
    // length (all zero: no EMF corrections), and the cell loss adds the magnetic-flux residual of the faces of
    // each direction over resScaleB[d]. Only on grids periodic in all three directions (the edge owner map
    // below assumes it); elsewhere the EMF outputs are left unused.
    float emfScale[3] = {0, 0, 0}, resScaleB[3] = {1, 1, 1};
    int periodic[3] = {0, 0, 0};
    float* corr = nullptr;       // 24 face-correction planes (area-scaled), then 3 edge EMF-correction planes
    float* geom = nullptr;       // volume, face I, J, K, edge I, J, K (float planes, copied from a solver handle)
    bool haveGeom = false;
    float* wts = nullptr;        // loss weights: w_v = dL/d(dU_v) * dt / V (5 planes), u_d = dL/d(curl_d) (3)
    double* lossAcc = nullptr;   // device loss accumulators [2]
    float* lossPart = nullptr;   // per-block loss partials
    // training samples: net input (8 bf16 planes) and residual (5 float planes) per slot, and its dt
    std::vector<__nv_bfloat16*> sIn;
    std::vector<float*> sRes;
    std::vector<double> sDt;
    __nv_bfloat16* act0 = nullptr;   // the net's own input planes (act[0] is pointed at a sample in training)
    // face targets: per slot the area-scaled correction that turns the plain coarse step's face fluxes into
    // the restricted, time-integrated fine fluxes (24 float planes, made when the sample's fine steps were
    // accumulated); fAcc sums dt_f x the restricted fine fluxes of those steps (24 double planes)
    std::vector<float*> sFace;
    double* fAcc = nullptr;
    int fAccSteps = 0;
    int lossMode = 0;   // GAM_CLOSURE_LOSS_CELL or GAM_CLOSURE_LOSS_FACE
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

// Fortran (Ni,Nj,Nk,nc) host layout -> the net's channels-last input at the pencil index
__global__ void k_in_from_fortran(Lay L, const float* src, int nc, __nv_bfloat16* dst) {
    const long long n = (long long)L.Ni * L.Nj * L.Nk;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % L.Ni), j = (int)((t / L.Ni) % L.Nj), k = (int)(t / ((long long)L.Ni * L.Nj));
    const long long c = L.at(i, j, k);
    for (int q = 0; q < nc; ++q) dst[c * NET_IN_PITCH + q] = __float2bfloat16_rn(src[t + q * n]);
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
// Fortran (Nip,Njp,Nkp,nc) gradient of the active cells -> channels-last bf16 (zero elsewhere)
__global__ void k_gout_from_fortran(Lay L, const float* src, int nc, __nv_bfloat16* dst) {
    const long long n = (long long)L.Nip * L.Njp * L.Nkp;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % L.Nip), j = (int)((t / L.Nip) % L.Njp), k = (int)(t / ((long long)L.Nip * L.Njp));
    const long long c = L.at(i + 4, j + 4, k + 4);
    for (int q = 0; q < nc; ++q) dst[c * NET_PITCH + q] = __float2bfloat16_rn(src[t + q * n]);
}


struct NormP {
    float inMean[8], inScale[8], fluxScale[8], resScale[5];
    float emfScale[3], resScaleB[3];
    int per[3];
    int emf;   // EMF corrections and the magnetic-flux loss terms on
};
NormP norm_of(const gam_closure* C) {
    NormP n;
    for (int q = 0; q < 8; ++q) { n.inMean[q] = C->inMean[q]; n.inScale[q] = C->inScale[q]; n.fluxScale[q] = C->fluxScale[q]; }
    for (int q = 0; q < 5; ++q) n.resScale[q] = C->resScale[q];
    for (int d = 0; d < 3; ++d) { n.per[d] = C->periodic[d]; n.emfScale[d] = C->emfScale[d]; n.resScaleB[d] = C->resScaleB[d]; }
    n.emf = (C->emfScale[0] != 0.f || C->emfScale[1] != 0.f || C->emfScale[2] != 0.f) && C->periodic[0] &&
            C->periodic[1] && C->periodic[2];
    return n;
}

// the net's input from a state: normalised rho, v, P, B of every cell (ghosts included), channels-last
// launched over (i, j) planes (gam_kern.cuh reg_plane); the 8 channels of a cell go out as one 16-byte store
__global__ void k_closure_input(Lay L, double gamma, StateP s, NormP n, __nv_bfloat16* in) {
    int i, j, k;
    if (!reg_plane(Reg{0, L.Ni, 0, L.Nj, 0, L.Nk}, i, j, k)) return;
    const long long c = L.at(i, j, k);
    const double rho = s.gas[0][c];
    const double vx = s.gas[1][c] / rho, vy = s.gas[2][c] / rho, vz = s.gas[3][c] / rho;
    const double P = (gamma - 1.0) * (s.gas[4][c] - 0.5 * rho * (vx * vx + vy * vy + vz * vz));
    const double w[8] = {rho, vx, vy, vz, P, s.b[0][c], s.b[1][c], s.b[2][c]};
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        f[q] = (float)((w[q] - n.inMean[q]) / n.inScale[q]);
        if (!(f[q] == f[q]) || fabsf(f[q]) > 1e4f) f[q] = 0.f;   // keep the net's input finite
    }
    uint32_t pk[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);   // channel 2q at the lower address
        pk[q] = *reinterpret_cast<uint32_t*>(&h2);
    }
    *reinterpret_cast<uint4*>(in + c * NET_IN_PITCH) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
}

// face corrections (area-scaled): plane d*8+v at the index of the lower d-face of the owner cell, for the
// faces of the active cells and the upper boundary faces. A boundary face of a non-periodic direction gets
// none; across a periodic one the upper boundary face repeats the lower boundary face.
__global__ void k_closure_corr(Lay L, const float* out, NormP n, const float* geom, float* corr) {
    int i, j, k;
    if (!reg_plane(Reg{L.is(), L.Nip + 1, L.js(), L.Njp + 1, L.ks(), L.Nkp + 1}, i, j, k)) return;
    const long long c = L.at(i, j, k);
    const int idx[3] = {i, j, k};
    const int lo[3] = {L.is(), L.js(), L.ks()}, hi[3] = {L.ie(), L.je(), L.ke()};
    for (int d = 0; d < 3; ++d) {
        // the other two indices must be active for a d-face of an active cell
        bool ok = true;
        for (int e = 0; e < 3; ++e)
            if (e != d && idx[e] > hi[e]) ok = false;
        if (!ok) continue;
        long long own = c;
        bool zero = false;
        if (idx[d] == hi[d] + 1) {
            if (n.per[d]) own = c - (long long)(hi[d] - lo[d] + 1) * (d == 0 ? 1 : d == 1 ? L.P : (long long)L.P * L.Q);
            else zero = true;
        } else if (idx[d] == lo[d] && !n.per[d]) {
            zero = true;
        }
        const float A = geom[(long long)(1 + d) * L.E + c];
        for (int v = 0; v < 8; ++v) {
            const long long o = (long long)(d * 8 + v) * L.E;
            corr[o + c] = zero ? 0.f : out[o + own] * n.fluxScale[v] * A;
        }
    }
    // EMF corrections (edge-integrated, like the solver's E) on the edges of direction e: the edges of the
    // active cells and, across the periodic boundaries, the upper boundary edges repeating the lower ones
    const long long st[3] = {1, L.P, (long long)L.P * L.Q};
    const int cnt[3] = {L.Nip, L.Njp, L.Nkp};
    for (int e = 0; e < 3; ++e) {
        const long long o = (long long)(NET_FACE_OUT + e) * L.E;
        if (!n.emf || idx[e] > hi[e]) { corr[o + c] = 0.f; continue; }
        long long own = c;
        for (int d = 0; d < 3; ++d)
            if (d != e && idx[d] == hi[d] + 1) own -= (long long)cnt[d] * st[d];
        corr[o + c] = out[o + own] * n.emfScale[e] * geom[(long long)(4 + e) * L.E + c];
    }
}

// the closure's EMF corrections added to the step's edge EMFs (before E2Flux), unless this step's corrected
// update failed positivity (the plain step is then taken whole)
__global__ void k_closure_emf(Lay L, const float* corr, Vec3P E, const Scal* sc) {
    if (sc->closureReject) return;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ni = L.Nip + 1, nj = L.Njp + 1, nk = L.Nkp + 1;
    if (t >= (long long)ni * nj * nk) return;
    const int idx[3] = {L.is() + (int)(t % ni), L.js() + (int)((t / ni) % nj), L.ks() + (int)(t / ((long long)ni * nj))};
    const int hi[3] = {L.ie(), L.je(), L.ke()};
    const long long c = L.at(idx[0], idx[1], idx[2]);
    for (int e = 0; e < 3; ++e)
        if (idx[e] <= hi[e]) E.v[e][c] += (double)corr[(long long)(NET_FACE_OUT + e) * L.E + c];
}

// closure positivity: the Reynolds stage of the corrected update must keep rho > 0 and P > 0 (before floors)
__global__ void k_closure_check(Lay L, double gamma, StateP nS, PrimP dGH, const Scal* scIn, Scal* sc) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nip * L.Njp * L.Nkp) return;
    const int i = L.is() + (int)(t % L.Nip), j = L.js() + (int)((t / L.Nip) % L.Njp),
              k = L.ks() + (int)(t / ((long long)L.Nip * L.Njp));
    const long long c = L.at(i, j, k);
    const double dt = scIn->dt;
    double U[5];
    for (int v = 0; v < 5; ++v) U[v] = nS.gas[v][c] + dt * dGH.w[v][c];
    bool bad = !(U[0] > 0.0);
    if (!bad) {
        const double P = (gamma - 1.0) * (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]);
        bad = !(P > 0.0);
    }
    if (bad) atomicExch(&sc->closureReject, 1);
}
__global__ void k_closure_count(Scal* sc) {
    if (sc->closureReject) sc->closureRejects++;
}

// the residual of one coarse step: the volume-weighted restriction of the fine state minus the coarse
// state, gas variables, active coarse cells (fine cells 2x2x2 per coarse cell)
__global__ void k_closure_residual(Lay Lc, Lay Lf, StateP fine, const double* fineVol, StateP coarse, float* res) {
    // (planes 5..7: the magnetic-flux residual of each active cell's lower I, J, K face: the sum of the 2 x 2
    // fine sub-face fluxes minus the coarse flux)
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)Lc.Nip * Lc.Njp * Lc.Nkp) return;
    const int I = (int)(t % Lc.Nip), J = (int)((t / Lc.Nip) % Lc.Njp), K = (int)(t / ((long long)Lc.Nip * Lc.Njp));
    const long long cc = Lc.at(Lc.is() + I, Lc.js() + J, Lc.ks() + K);
    double sum[5] = {0, 0, 0, 0, 0}, vol = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const long long cf = Lf.at(Lf.is() + 2 * I + di, Lf.js() + 2 * J + dj, Lf.ks() + 2 * K + dk);
                const double V = fineVol[cf];
                vol += V;
                for (int v = 0; v < 5; ++v) sum[v] += fine.gas[v][cf] * V;
            }
    for (int v = 0; v < 5; ++v) res[(long long)v * Lc.E + cc] = (float)(sum[v] / vol - coarse.gas[v][cc]);
    const int fi = Lf.is() + 2 * I, fj = Lf.js() + 2 * J, fk = Lf.ks() + 2 * K;
    const double f0 = fine.mf[0][Lf.at(fi, fj, fk)] + fine.mf[0][Lf.at(fi, fj + 1, fk)] +
                      fine.mf[0][Lf.at(fi, fj, fk + 1)] + fine.mf[0][Lf.at(fi, fj + 1, fk + 1)];
    const double f1 = fine.mf[1][Lf.at(fi, fj, fk)] + fine.mf[1][Lf.at(fi + 1, fj, fk)] +
                      fine.mf[1][Lf.at(fi, fj, fk + 1)] + fine.mf[1][Lf.at(fi + 1, fj, fk + 1)];
    const double f2 = fine.mf[2][Lf.at(fi, fj, fk)] + fine.mf[2][Lf.at(fi + 1, fj, fk)] +
                      fine.mf[2][Lf.at(fi, fj + 1, fk)] + fine.mf[2][Lf.at(fi + 1, fj + 1, fk)];
    res[5LL * Lc.E + cc] = (float)(f0 - coarse.mf[0][cc]);
    res[6LL * Lc.E + cc] = (float)(f1 - coarse.mf[1][cc]);
    res[7LL * Lc.E + cc] = (float)(f2 - coarse.mf[2][cc]);
}

// restriction into a coarse state: gas volume-weighted, magnetic fluxes summed over the 4 fine faces of
// each coarse face (so the coarse field stays divergence-free)
__global__ void k_restrict_gas(Lay Lc, Lay Lf, StateP fine, const double* fineVol, StateP coarse) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)Lc.Nip * Lc.Njp * Lc.Nkp) return;
    const int I = (int)(t % Lc.Nip), J = (int)((t / Lc.Nip) % Lc.Njp), K = (int)(t / ((long long)Lc.Nip * Lc.Njp));
    const long long cc = Lc.at(Lc.is() + I, Lc.js() + J, Lc.ks() + K);
    double sum[5] = {0, 0, 0, 0, 0}, vol = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const long long cf = Lf.at(Lf.is() + 2 * I + di, Lf.js() + 2 * J + dj, Lf.ks() + 2 * K + dk);
                const double V = fineVol[cf];
                vol += V;
                for (int v = 0; v < 5; ++v) sum[v] += fine.gas[v][cf] * V;
            }
    for (int v = 0; v < 5; ++v) coarse.gas[v][cc] = sum[v] / vol;
}
__global__ void k_restrict_flux(Lay Lc, Lay Lf, StateP fine, StateP coarse) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ni = Lc.Nip + 1, nj = Lc.Njp + 1, nk = Lc.Nkp + 1;
    if (t >= (long long)ni * nj * nk) return;
    const int I = (int)(t % ni), J = (int)((t / ni) % nj), K = (int)(t / ((long long)ni * nj));
    const long long cc = Lc.at(Lc.is() + I, Lc.js() + J, Lc.ks() + K);
    const int fi = Lf.is() + 2 * I, fj = Lf.js() + 2 * J, fk = Lf.ks() + 2 * K;
    if (J < Lc.Njp && K < Lc.Nkp)
        coarse.mf[0][cc] = fine.mf[0][Lf.at(fi, fj, fk)] + fine.mf[0][Lf.at(fi, fj + 1, fk)] +
                           fine.mf[0][Lf.at(fi, fj, fk + 1)] + fine.mf[0][Lf.at(fi, fj + 1, fk + 1)];
    if (I < Lc.Nip && K < Lc.Nkp)
        coarse.mf[1][cc] = fine.mf[1][Lf.at(fi, fj, fk)] + fine.mf[1][Lf.at(fi + 1, fj, fk)] +
                           fine.mf[1][Lf.at(fi, fj, fk + 1)] + fine.mf[1][Lf.at(fi + 1, fj, fk + 1)];
    if (I < Lc.Nip && J < Lc.Njp)
        coarse.mf[2][cc] = fine.mf[2][Lf.at(fi, fj, fk)] + fine.mf[2][Lf.at(fi + 1, fj, fk)] +
                           fine.mf[2][Lf.at(fi, fj + 1, fk)] + fine.mf[2][Lf.at(fi + 1, fj + 1, fk)];
}

__global__ void k_to_float(const double* src, float* dst, long long n) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) dst[t] = (float)src[t];
}

// loss of one sample: dU = dt / V * (sum of corrections in - out) (momentum also from the magnetic-stress
// corrections), L = mean over active cells of sum_v ((dU_v - r_v) / resScale_v)^2; stores
// w_v = dL/d(dU_v) * dt / V for the gradient and per-block partial sums of L
__global__ void k_loss_w(Lay L, const float* corr, const float* res, const float* geom, NormP n, double dt,
                         float* w, float* part) {
    __shared__ float red[256];
    const long long nact = (long long)L.Nip * L.Njp * L.Nkp;
    float acc = 0.f;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nact; t += (long long)gridDim.x * blockDim.x) {
        const int i = L.is() + (int)(t % L.Nip), j = L.js() + (int)((t / L.Nip) % L.Njp),
                  k = L.ks() + (int)(t / ((long long)L.Nip * L.Njp));
        const long long c = L.at(i, j, k);
        const long long nb[3] = {c + 1, c + L.P, c + (long long)L.P * L.Q};
        const float f = (float)dt / geom[c];
        float dU[5];
        for (int v = 0; v < 5; ++v) {
            float s = 0.f;
            for (int d = 0; d < 3; ++d) {
                const float* q = corr + (long long)(d * 8 + v) * L.E;
                s += q[c] - q[nb[d]];
            }
            dU[v] = s;
        }
        for (int x = 0; x < 3; ++x)
            for (int d = 0; d < 3; ++d) {
                const float* q = corr + (long long)(d * 8 + 5 + x) * L.E;
                dU[1 + x] += q[c] - q[nb[d]];
            }
        for (int v = 0; v < 5; ++v) {
            const float e = (f * dU[v] - res[(long long)v * L.E + c]) / n.resScale[v];
            acc += e * e;
            w[(long long)v * L.E + c] = 2.f * e / n.resScale[v] / (float)nact * f;
        }
        if (n.emf) {   // magnetic flux of the lower faces: -dt x the curl of the EMF corrections (E2Flux's stencil)
            const float* Ei = corr + (long long)NET_FACE_OUT * L.E;
            const float* Ej = Ei + L.E;
            const float* Ek = Ej + L.E;
            const long long cj = c + L.P, ck = c + (long long)L.P * L.Q;
            const float df[3] = {Ek[cj] - Ek[c] - Ej[ck] + Ej[c], Ei[ck] - Ei[c] - Ek[c + 1] + Ek[c],
                                 Ej[c + 1] - Ej[c] - Ei[cj] + Ei[c]};
            for (int d = 0; d < 3; ++d) {
                const float e = (-(float)dt * df[d] - res[(long long)(5 + d) * L.E + c]) / n.resScaleB[d];
                acc += e * e;
                w[(long long)(5 + d) * L.E + c] = 2.f * e / n.resScaleB[d] / (float)nact * (-(float)dt);
            }
        }
    }
    red[threadIdx.x] = acc / (float)nact;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}
__global__ void k_loss_sum(const float* part, int nblk, double* acc) {
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[b];
    acc[0] += s;
}

// output gradient: dL/dy for the lower d-face of each active cell = fluxScale * A * (w(cell) - w(cell below)),
// the cell below wrapping across a periodic boundary; a non-periodic boundary face has no correction
__global__ void k_loss_grad(Lay L, const float* w, const float* geom, NormP n, __nv_bfloat16* gout) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nip * L.Njp * L.Nkp) return;
    const int i = L.is() + (int)(t % L.Nip), j = L.js() + (int)((t / L.Nip) % L.Njp),
              k = L.ks() + (int)(t / ((long long)L.Nip * L.Njp));
    const long long c = L.at(i, j, k);
    const int idx[3] = {i, j, k};
    const int lo[3] = {L.is(), L.js(), L.ks()}, cnt[3] = {L.Nip, L.Njp, L.Nkp};
    const long long st[3] = {1, L.P, (long long)L.P * L.Q};
    for (int d = 0; d < 3; ++d) {
        bool zero = false;
        long long below = c - st[d];
        if (idx[d] == lo[d]) {
            if (n.per[d]) below = c + (long long)(cnt[d] - 1) * st[d];
            else zero = true;
        }
        const float A = geom[(long long)(1 + d) * L.E + c];
        for (int v = 0; v < 8; ++v) {
            const int u = v < 5 ? v : v - 4;   // the magnetic-stress corrections act on the momentum
            const float g = zero ? 0.f
                                 : n.fluxScale[v] * A * (w[(long long)u * L.E + c] - w[(long long)u * L.E + below]);
            gout[c * NET_PITCH + d * 8 + v] = __float2bfloat16_rn(g);
        }
    }
    // EMF outputs: the transpose of the curl (E2Flux's stencil), u_d = dL/d(curl_d) on the lower faces of the
    // active cells, the neighbours below wrapping across the periodic boundaries
    float ge[3] = {0.f, 0.f, 0.f};
    if (n.emf) {
        auto below = [&](int d) { return idx[d] == lo[d] ? c + (long long)(cnt[d] - 1) * st[d] : c - st[d]; };
        auto u = [&](int d, long long x) { return w[(long long)(5 + d) * L.E + x]; };
        const long long bi = below(0), bj = below(1), bk = below(2);
        ge[0] = -u(1, c) + u(1, bk) + u(2, c) - u(2, bj);
        ge[1] = u(0, c) - u(0, bk) + u(2, bi) - u(2, c);
        ge[2] = u(0, bj) - u(0, c) - u(1, bi) + u(1, c);
    }
    for (int e = 0; e < 3; ++e)
        gout[c * NET_PITCH + NET_FACE_OUT + e] =
            __float2bfloat16_rn(n.emf ? n.emfScale[e] * geom[(long long)(4 + e) * L.E + c] * ge[e] : 0.f);
}

inline unsigned nblk256(long long n) { return (unsigned)((n + 255) / 256); }

// ---------------------------------------------------------------- face targets
// Area-scaled interface fluxes of a solver, plane d*8+v: the 5 gas fluxes, then the 3 magnetic-stress
// momentum fluxes, of direction d
struct FluxPlanes { const double* f[24]; };
FluxPlanes flux_planes(const Handle& h) {
    FluxPlanes F;
    for (int d = 0; d < 3; ++d) {
        for (int v = 0; v < 5; ++v) F.f[d * 8 + v] = h.gflx[d][v];
        for (int x = 0; x < 3; ++x) F.f[d * 8 + 5 + x] = h.mflx[d][x];
    }
    return F;
}

// the coarse face sites: lower faces of the active cells and the upper boundary faces; a d-face needs the
// other two indices active
__device__ __forceinline__ bool face_site(const Lay& L, long long t, int& i, int& j, int& k) {
    const int ni = L.Nip + 1, nj = L.Njp + 1, nk = L.Nkp + 1;
    if (t >= (long long)ni * nj * nk) return false;
    i = L.is() + (int)(t % ni); j = L.js() + (int)((t / ni) % nj); k = L.ks() + (int)(t / ((long long)ni * nj));
    return true;
}
__device__ __forceinline__ bool face_of_active(const Lay& L, int d, int i, int j, int k) {
    return (d == 0 || i <= L.ie()) && (d == 1 || j <= L.je()) && (d == 2 || k <= L.ke());
}

// w x the fine fluxes through each coarse face (the sum over its 2 x 2 fine sub-faces) added into acc
__global__ void k_accum_fine(Lay Lc, Lay Lf, FluxPlanes F, int nv, double w, double* acc) {
    int i, j, k;
    if (!face_site(Lc, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    const long long c = Lc.at(i, j, k);
    const int fi = Lf.is() + 2 * (i - Lc.is()), fj = Lf.js() + 2 * (j - Lc.js()), fk = Lf.ks() + 2 * (k - Lc.ks());
    for (int d = 0; d < 3; ++d) {
        if (!face_of_active(Lc, d, i, j, k)) continue;
        long long sub[4];
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                sub[2 * a + b] = d == 0 ? Lf.at(fi, fj + a, fk + b) : d == 1 ? Lf.at(fi + a, fj, fk + b)
                                                                           : Lf.at(fi + a, fj + b, fk);
        for (int v = 0; v < nv; ++v) {
            const double* q = F.f[d * 8 + v];
            acc[(long long)(d * 8 + v) * Lc.E + c] += w * (q[sub[0]] + q[sub[1]] + q[sub[2]] + q[sub[3]]);
        }
    }
}

// target = acc / dt - (the plain coarse step's flux), per face site and direction
__global__ void k_face_target(Lay L, const double* acc, double dt, FluxPlanes F, int nv, float* tgt) {
    int i, j, k;
    if (!face_site(L, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    const long long c = L.at(i, j, k);
    for (int d = 0; d < 3; ++d) {
        if (!face_of_active(L, d, i, j, k)) continue;
        for (int v = 0; v < 8; ++v) {
            const long long o = (long long)(d * 8 + v) * L.E + c;
            tgt[o] = v < nv ? (float)(acc[o] / dt - F.f[d * 8 + v][c]) : 0.f;
        }
    }
}

// face-target loss of one sample: over the lower d-faces of the active cells (a non-periodic boundary face
// carries no correction), e = y - target / (fluxScale_v * area), L = mean of e^2 over faces and the 8
// variables of 3 directions; the net-output gradient dL/dy = 2e / N goes to gout (when given); y = 0
// without a net output
__global__ void k_loss_face(Lay L, const float* out, const float* tgt, const float* geom, NormP n,
                            __nv_bfloat16* gout, float* part) {
    __shared__ float red[256];
    const long long nact = (long long)L.Nip * L.Njp * L.Nkp;
    const float N = (float)nact * 24.f;
    float acc = 0.f;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nact; t += (long long)gridDim.x * blockDim.x) {
        const int idx[3] = {L.is() + (int)(t % L.Nip), L.js() + (int)((t / L.Nip) % L.Njp),
                            L.ks() + (int)(t / ((long long)L.Nip * L.Njp))};
        const int lo[3] = {L.is(), L.js(), L.ks()};
        const long long c = L.at(idx[0], idx[1], idx[2]);
        for (int d = 0; d < 3; ++d) {
            const bool none = idx[d] == lo[d] && !n.per[d];
            const float A = geom[(long long)(1 + d) * L.E + c];
            for (int v = 0; v < 8; ++v) {
                const long long o = (long long)(d * 8 + v) * L.E + c;
                float e = 0.f;
                if (!none) {
                    const float y = out ? out[o] : 0.f;
                    e = y - tgt[o] / (n.fluxScale[v] * A);
                    acc += e * e;
                }
                if (gout) gout[c * NET_PITCH + d * 8 + v] = __float2bfloat16_rn(2.f * e / N);
            }
        }
        if (gout)   // the face targets carry no EMF; those outputs get no gradient
            for (int e = 0; e < 3; ++e) gout[c * NET_PITCH + NET_FACE_OUT + e] = __float2bfloat16_rn(0.f);
    }
    red[threadIdx.x] = acc / N;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// statistics of one sample's face targets: acc[0..7] sums of (target_v / area)^2 over the lower faces of the
// active cells; acc[8..12] sums of (dt / V * div(target)_v - residual_v)^2 and acc[13..17] of residual_v^2
// (how closely the face targets account for the cell residual)
__global__ void k_face_stats(Lay L, const float* tgt, const float* res, const float* geom, double dt, double* acc) {
    __shared__ double red[18][128];
    double s[18];
    for (int q = 0; q < 18; ++q) s[q] = 0.0;
    const long long nact = (long long)L.Nip * L.Njp * L.Nkp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nact; t += (long long)gridDim.x * blockDim.x) {
        const int i = L.is() + (int)(t % L.Nip), j = L.js() + (int)((t / L.Nip) % L.Njp),
                  k = L.ks() + (int)(t / ((long long)L.Nip * L.Njp));
        const long long c = L.at(i, j, k);
        const long long nb[3] = {c + 1, c + L.P, c + (long long)L.P * L.Q};
        for (int d = 0; d < 3; ++d) {
            const double A = geom[(long long)(1 + d) * L.E + c];
            for (int v = 0; v < 8; ++v) {
                const double y = tgt[(long long)(d * 8 + v) * L.E + c] / A;
                s[v] += y * y;
            }
        }
        double dU[5];
        for (int v = 0; v < 5; ++v) {
            double q = 0.0;
            for (int d = 0; d < 3; ++d) {
                const float* f = tgt + (long long)(d * 8 + v) * L.E;
                q += (double)f[c] - (double)f[nb[d]];
            }
            dU[v] = q;
        }
        for (int x = 0; x < 3; ++x)
            for (int d = 0; d < 3; ++d) {
                const float* f = tgt + (long long)(d * 8 + 5 + x) * L.E;
                dU[1 + x] += (double)f[c] - (double)f[nb[d]];
            }
        const double fV = dt / geom[c];
        for (int v = 0; v < 5; ++v) {
            const double r = res[(long long)v * L.E + c], e = fV * dU[v] - r;
            s[8 + v] += e * e;
            s[13 + v] += r * r;
        }
    }
    for (int q = 0; q < 18; ++q) red[q][threadIdx.x] = s[q];
    __syncthreads();
    if (threadIdx.x < 18) {
        double a = 0.0;
        for (int b = 0; b < (int)blockDim.x; ++b) a += red[threadIdx.x][b];
        atomicAdd(&acc[threadIdx.x], a);
    }
}

// sums of the residual squares per plane (nv <= 5 planes from res) over the active cells (statistics for the
// normalisation)
__global__ void k_res_sq(Lay L, const float* res, int nv, double* acc) {
    __shared__ double red[5][256];
    double s[5] = {0, 0, 0, 0, 0};
    const long long nact = (long long)L.Nip * L.Njp * L.Nkp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nact; t += (long long)gridDim.x * blockDim.x) {
        const long long c = L.at(L.is() + (int)(t % L.Nip), L.js() + (int)((t / L.Nip) % L.Njp),
                                 L.ks() + (int)(t / ((long long)L.Nip * L.Njp)));
        for (int v = 0; v < nv; ++v) { const double r = res[(long long)v * L.E + c]; s[v] += r * r; }
    }
    for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = s[v];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int v = 0; v < 5; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 5; ++v) atomicAdd(&acc[v], red[v][0]);
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
    if (net_init() != 0) { delete C; return GAM_ERR_CUDA; }
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
    // channels-last activations: act (16 + 3*32), pre (3*32), grad (4*32) bf16 per cell; out (24) fp32 planes
    const long long E = L.E;
    const long long bfPerCell = NET_IN_PITCH + 3 * NET_PITCH + 3 * NET_PITCH + 4 * NET_PITCH;
    const size_t bytes = sizeof(__nv_bfloat16) * E * bfPerCell + sizeof(float) * E * NET_OUT;
    if (cudaMalloc(&C->pool, bytes) != cudaSuccess) return fail(GAM_ERR_CUDA);
    cudaMemsetAsync(C->pool, 0, bytes, C->stream);
    __nv_bfloat16* q = static_cast<__nv_bfloat16*>(C->pool);
    C->nb.act[0] = q; q += E * NET_IN_PITCH;
    for (int l = 1; l < NET_LAYERS; ++l) { C->nb.act[l] = q; q += E * NET_PITCH; }
    for (int l = 0; l < NET_LAYERS - 1; ++l) { C->nb.pre[l] = q; q += E * NET_PITCH; }
    C->nb.pre[NET_LAYERS - 1] = nullptr;
    for (int l = 0; l < NET_LAYERS; ++l) { C->nb.grad[l] = q; q += E * NET_PITCH; }
    C->nb.out = reinterpret_cast<float*>(q);
    C->nb.partialFloats = net_partial_floats(net_dw_blocks());
    if (cudaMalloc(&C->nb.partial, sizeof(float) * C->nb.partialFloats) != cudaSuccess) return fail(GAM_ERR_CUDA);
    C->act0 = C->nb.act[0];
    if (cudaMalloc(&C->corr, sizeof(float) * E * NET_OUT) || cudaMalloc(&C->geom, sizeof(float) * E * 7) ||
        cudaMalloc(&C->wts, sizeof(float) * E * 8) || cudaMalloc(&C->lossAcc, sizeof(double) * 2) ||
        cudaMalloc(&C->lossPart, sizeof(float) * 2 * 4096))
        return fail(GAM_ERR_CUDA);
    cudaMemsetAsync(C->corr, 0, sizeof(float) * E * NET_OUT, C->stream);
    cudaMemsetAsync(C->wts, 0, sizeof(float) * E * 8, C->stream);
    cudaMemsetAsync(C->geom, 0, sizeof(float) * E * 7, C->stream);
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
    cudaFree(C->corr); cudaFree(C->geom); cudaFree(C->wts); cudaFree(C->lossAcc); cudaFree(C->lossPart);
    for (auto* q : C->sIn) cudaFree(q);
    for (auto* q : C->sRes) cudaFree(q);
    for (auto* q : C->sFace) cudaFree(q);
    cudaFree(C->fAcc);
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
    k_gout_from_fortran<<<(unsigned)((nAct + 255) / 256), 256, 0, C->stream>>>(L, C->stage, NET_OUT, C->nb.grad[NET_LAYERS - 1]);
    if (net_backward(C->box, C->wbwd, C->nb, C->grads, C->err, C->stream) != 0) return GAM_ERR_CUDA;
    return check_err(C);
}

}  // extern "C"

// ================================================================================ the closure in the step
namespace gam {

const float* closure_enqueue_corr(Handle& h, const StateP& nS, cudaStream_t st) {
    gam_closure* C = h.closure;
    const Lay& L = h.L;
    NormP n = norm_of(C);
    C->nb.act[0] = C->act0;
    k_closure_input<<<grid_plane(Reg{0, L.Ni, 0, L.Nj, 0, L.Nk}, 256), 256, 0, st>>>(L, h.p.gamma, nS, n, C->act0);
    net_forward(C->box, C->wfwd, C->params, C->nb, false, C->err, st);
    k_closure_corr<<<grid_plane(Reg{L.is(), L.Nip + 1, L.js(), L.Njp + 1, L.ks(), L.Nkp + 1}, 256), 256, 0, st>>>(
        L, C->nb.out, n, C->geom, C->corr);
    h.launches += 2 + NET_LAYERS;
    return C->corr;
}

void closure_enqueue_check(Handle& h, const StateP& nS, cudaStream_t st) {
    const Lay& L = h.L;
    PrimP dGH;
    for (int v = 0; v < 5; ++v) dGH.w[v] = h.dGasH[v];
    k_closure_check<<<nblk256((long long)L.Nip * L.Njp * L.Nkp), 256, 0, st>>>(L, h.p.gamma, nS, dGH, h.dScal, h.dScal);
    k_closure_count<<<1, 1, 0, st>>>(h.dScal);
    h.launches += 2;
}

void closure_enqueue_emf(Handle& h, cudaStream_t st) {
    gam_closure* C = h.closure;
    if (!norm_of(C).emf) return;
    const Lay& L = h.L;
    Vec3P E = {{h.E[0], h.E[1], h.E[2]}};
    k_closure_emf<<<nblk256((long long)(L.Nip + 1) * (L.Njp + 1) * (L.Nkp + 1)), 256, 0, st>>>(L, C->corr, E, h.dScal);
    h.launches++;
}

int closure_kernels_per_step(const Handle& h) {
    return h.closure ? 2 + NET_LAYERS + 2 + (norm_of(h.closure).emf ? 1 : 0) : 0;
}

// shape check and geometry for a handle the closure is attached to
int closure_attach(Handle& h, gam_closure* C) {
    const Lay& L = h.L;
    if (C->L.Nip != L.Nip || C->L.Njp != L.Njp || C->L.Nkp != L.Nkp || C->device != h.device) return GAM_ERR_ARG;
    if (h.p.doRing) return GAM_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; ++d) C->periodic[d] = h.p.bc[2 * d] == BC_PERIODIC && h.p.bc[2 * d + 1] == BC_PERIODIC;
    k_to_float<<<nblk256(L.E), 256, 0, h.stream>>>(h.volume, C->geom, L.E);
    for (int d = 0; d < 3; ++d) k_to_float<<<nblk256(L.E), 256, 0, h.stream>>>(h.face[d], C->geom + (1 + d) * L.E, L.E);
    for (int d = 0; d < 3; ++d) k_to_float<<<nblk256(L.E), 256, 0, h.stream>>>(h.edge[d], C->geom + (4 + d) * L.E, L.E);
    C->haveGeom = true;
    return cudaStreamSynchronize(h.stream) == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

}  // namespace gam

namespace gam {
Handle& capi_handle(gam_gpu* G);
int capi_download_scalars(gam_gpu* G);
}  // namespace gam

extern "C" {

int gam_closure_set_norm(gam_closure_t* C, const float* inMean, const float* inScale, const float* fluxScale,
                         const float* resScale) {
    if (!C || !inMean || !inScale || !fluxScale || !resScale) return GAM_ERR_ARG;
    for (int q = 0; q < 8; ++q) {
        if (!(inScale[q] > 0.f) || !(fluxScale[q] > 0.f)) return GAM_ERR_ARG;
        C->inMean[q] = inMean[q]; C->inScale[q] = inScale[q]; C->fluxScale[q] = fluxScale[q];
    }
    for (int q = 0; q < 5; ++q) {
        if (!(resScale[q] > 0.f)) return GAM_ERR_ARG;
        C->resScale[q] = resScale[q];
    }
    return GAM_OK;
}

int gam_closure_reserve(gam_closure_t* C, int n) {
    if (!C || n < 0) return GAM_ERR_ARG;
    const long long E = C->L.E;
    while ((int)C->sIn.size() < n) {
        __nv_bfloat16* in = nullptr;
        float* res = nullptr;
        if (cudaMalloc(&in, sizeof(__nv_bfloat16) * E * NET_IN_PITCH) != cudaSuccess) return GAM_ERR_CUDA;
        if (cudaMalloc(&res, sizeof(float) * E * 8) != cudaSuccess) { cudaFree(in); return GAM_ERR_CUDA; }
        cudaMemsetAsync(in, 0, sizeof(__nv_bfloat16) * E * NET_IN_PITCH, C->stream);
        cudaMemsetAsync(res, 0, sizeof(float) * E * 8, C->stream);
        C->sIn.push_back(in);
        C->sRes.push_back(res);
        C->sDt.push_back(0.0);
        C->sFace.push_back(nullptr);   // made by a capture that follows accumulated fine steps
    }
    CKC(cudaStreamSynchronize(C->stream));
    return GAM_OK;
}

int gam_closure_capture(gam_closure_t* C, int slot, gam_gpu_t* coarse, gam_gpu_t* fine) {
    if (!C || !coarse || !fine || slot < 0 || slot >= (int)C->sIn.size()) return GAM_ERR_ARG;
    Handle& hc = capi_handle(coarse);
    Handle& hf = capi_handle(fine);
    if (hc.closure || hf.L.Nip != 2 * hc.L.Nip || hf.L.Njp != 2 * hc.L.Njp || hf.L.Nkp != 2 * hc.L.Nkp ||
        hc.device != hf.device)
        return GAM_ERR_ARG;
    int rc = closure_attach(hc, C);
    if (rc) return rc;
    const Lay& L = hc.L;
    NormP n = norm_of(C);
    k_closure_input<<<grid_plane(Reg{0, L.Ni, 0, L.Nj, 0, L.Nk}, 256), 256, 0, hc.stream>>>(L, hc.p.gamma,
                                                                                           hc.S[hc.cur], n, C->sIn[slot]);
    rc = capi_download_scalars(coarse);
    if (rc) return rc;
    C->sDt[slot] = hc.hScal->dt;
    double dt = 0.0, t = 0.0;
    int ts = 0;
    rc = gam_gpu_step(coarse, &dt, &ts, &t);   // the plain coarse step
    if (rc) return rc;
    CKC(cudaStreamSynchronize(hf.stream));
    k_closure_residual<<<nblk256((long long)L.Nip * L.Njp * L.Nkp), 256, 0, hc.stream>>>(
        L, hf.L, hf.S[hf.cur], hf.volume, hc.S[hc.cur], C->sRes[slot]);
    if (C->fAccSteps > 0) {   // the fine steps of this sample were accumulated: its face target
        if (hc.prec != PREC_FP64) return GAM_ERR_ARG;
        if (!C->sFace[slot]) {
            CKC(cudaMalloc(&C->sFace[slot], sizeof(float) * L.E * NET_OUT));
            CKC(cudaMemsetAsync(C->sFace[slot], 0, sizeof(float) * L.E * NET_OUT, hc.stream));
        }
        CKC(cudaStreamSynchronize(C->stream));
        k_face_target<<<nblk256((long long)(L.Nip + 1) * (L.Njp + 1) * (L.Nkp + 1)), 256, 0, hc.stream>>>(
            L, C->fAcc, C->sDt[slot], flux_planes(hc), hc.p.doMHD ? 8 : 5, C->sFace[slot]);
        C->fAccSteps = 0;
    }
    CKC(cudaStreamSynchronize(hc.stream));
    return GAM_OK;
}

// dt_f x the fine fluxes of the fine handle's last step, restricted to the coarse faces, added to the
// accumulation of the next capture's sample (reset: start a new sample)
int gam_closure_accum_fine(gam_closure_t* C, gam_gpu_t* fine, double weight, int reset) {
    if (!C || !fine) return GAM_ERR_ARG;
    Handle& hf = capi_handle(fine);
    const Lay& L = C->L;
    if (hf.L.Nip != 2 * L.Nip || hf.L.Njp != 2 * L.Njp || hf.L.Nkp != 2 * L.Nkp || hf.prec != PREC_FP64)
        return GAM_ERR_ARG;
    if (!C->fAcc) {
        CKC(cudaMalloc(&C->fAcc, sizeof(double) * L.E * NET_OUT));
        reset = 1;
    }
    CKC(cudaStreamSynchronize(hf.stream));
    if (reset || C->fAccSteps == 0) CKC(cudaMemsetAsync(C->fAcc, 0, sizeof(double) * L.E * NET_OUT, C->stream));
    k_accum_fine<<<nblk256((long long)(L.Nip + 1) * (L.Njp + 1) * (L.Nkp + 1)), 256, 0, C->stream>>>(
        L, hf.L, flux_planes(hf), hf.p.doMHD ? 8 : 5, weight, C->fAcc);
    C->fAccSteps = (reset ? 0 : C->fAccSteps) + 1;
    CKC(cudaStreamSynchronize(C->stream));
    return GAM_OK;
}

int gam_closure_set_loss(gam_closure_t* C, int mode) {
    if (!C || (mode != GAM_CLOSURE_LOSS_CELL && mode != GAM_CLOSURE_LOSS_FACE)) return GAM_ERR_ARG;
    C->lossMode = mode;
    return GAM_OK;
}

// rms[0..7]: rms of the slot's face targets over area (per variable, lower faces of the active cells);
// rel[0..4]: || dt / V * div(target) - residual || / || residual || per gas variable
int gam_closure_face_stats(gam_closure_t* C, int slot, double* rms, double* rel) {
    if (!C || !rms || !rel || slot < 0 || slot >= (int)C->sIn.size() || !C->sFace[slot] || !C->haveGeom)
        return GAM_ERR_ARG;
    double* acc = nullptr;
    CKC(cudaMalloc(&acc, sizeof(double) * 18));
    cudaMemsetAsync(acc, 0, sizeof(double) * 18, C->stream);
    k_face_stats<<<256, 128, 0, C->stream>>>(C->L, C->sFace[slot], C->sRes[slot], C->geom, C->sDt[slot], acc);
    double h[18];
    cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, C->stream);
    cudaError_t e = cudaStreamSynchronize(C->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return GAM_ERR_CUDA;
    const double n = 3.0 * C->L.Nip * C->L.Njp * C->L.Nkp;
    for (int v = 0; v < 8; ++v) rms[v] = std::sqrt(h[v] / n);
    for (int v = 0; v < 5; ++v) rel[v] = h[13 + v] > 0 ? std::sqrt(h[8 + v] / h[13 + v]) : 0.0;
    return GAM_OK;
}

// forward, loss and (train) gradient + Adam for one sample, on the closure's stream
static int closure_sample_pass(gam_closure* C, int slot, bool train, float lr) {
    const Lay& L = C->L;
    NormP n = norm_of(C);
    C->nb.act[0] = C->sIn[slot];
    if (net_forward(C->box, C->wfwd, C->params, C->nb, train, C->err, C->stream) != 0) return GAM_ERR_CUDA;
    const int nb = 1024;
    if (C->lossMode == GAM_CLOSURE_LOSS_FACE) {
        k_loss_face<<<nb, 256, 0, C->stream>>>(L, C->nb.out, C->sFace[slot], C->geom, n,
                                               train ? C->nb.grad[NET_LAYERS - 1] : nullptr, C->lossPart);
        k_loss_sum<<<1, 32, 0, C->stream>>>(C->lossPart, nb, C->lossAcc);
    } else {
        k_closure_corr<<<grid_plane(Reg{L.is(), L.Nip + 1, L.js(), L.Njp + 1, L.ks(), L.Nkp + 1}, 256), 256, 0,
                         C->stream>>>(L, C->nb.out, n, C->geom, C->corr);
        k_loss_w<<<nb, 256, 0, C->stream>>>(L, C->corr, C->sRes[slot], C->geom, n, C->sDt[slot], C->wts, C->lossPart);
        k_loss_sum<<<1, 32, 0, C->stream>>>(C->lossPart, nb, C->lossAcc);
    }
    if (train) {
        if (C->lossMode != GAM_CLOSURE_LOSS_FACE)
            k_loss_grad<<<nblk256((long long)L.Nip * L.Njp * L.Nkp), 256, 0, C->stream>>>(L, C->wts, C->geom, n,
                                                                                           C->nb.grad[NET_LAYERS - 1]);
        if (net_backward(C->box, C->wbwd, C->nb, C->grads, C->err, C->stream) != 0) return GAM_ERR_CUDA;
        C->adamStep++;
        if (net_adam(C->params, C->grads, C->m, C->v, C->np, lr, 0.9f, 0.999f, 1e-8f, C->adamStep, C->stream) != 0)
            return GAM_ERR_CUDA;
        if (closure_pack(C)) return GAM_ERR_CUDA;
    }
    C->nb.act[0] = C->act0;
    return GAM_OK;
}

// one Adam step per listed sample, in order; meanLoss = the mean of their losses before each step
int gam_closure_train(gam_closure_t* C, const int* slots, int n, float lr, double* meanLoss) {
    if (!C || !slots || n < 1 || !(lr > 0.f) || !C->haveGeom) return GAM_ERR_ARG;
    for (int q = 0; q < n; ++q)
        if (slots[q] < 0 || slots[q] >= (int)C->sIn.size() ||
            (C->lossMode == GAM_CLOSURE_LOSS_FACE && !C->sFace[slots[q]]))
            return GAM_ERR_ARG;
    CKC(cudaMemsetAsync(C->lossAcc, 0, sizeof(double) * 2, C->stream));
    for (int q = 0; q < n; ++q) {
        int rc = closure_sample_pass(C, slots[q], true, lr);
        if (rc) return rc;
    }
    double acc[2];
    CKC(cudaMemcpyAsync(acc, C->lossAcc, sizeof(acc), cudaMemcpyDeviceToHost, C->stream));
    int rc = check_err(C);
    if (rc) return rc;
    if (meanLoss) *meanLoss = acc[0] / n;
    return GAM_OK;
}

// mean loss over the listed samples with the net (loss) and without any correction (lossNone)
int gam_closure_eval(gam_closure_t* C, const int* slots, int n, double* loss, double* lossNone) {
    if (!C || !slots || n < 1 || !C->haveGeom) return GAM_ERR_ARG;
    for (int q = 0; q < n; ++q)
        if (slots[q] < 0 || slots[q] >= (int)C->sIn.size() ||
            (C->lossMode == GAM_CLOSURE_LOSS_FACE && !C->sFace[slots[q]]))
            return GAM_ERR_ARG;
    const Lay& L = C->L;
    NormP nrm = norm_of(C);
    double acc[2] = {0, 0};
    for (int pass = 0; pass < 2; ++pass) {
        CKC(cudaMemsetAsync(C->lossAcc, 0, sizeof(double) * 2, C->stream));
        for (int q = 0; q < n; ++q) {
            if (pass == 0) {
                int rc = closure_sample_pass(C, slots[q], false, 0.f);
                if (rc) return rc;
            } else if (C->lossMode == GAM_CLOSURE_LOSS_FACE) {   // no correction: the targets alone
                k_loss_face<<<1024, 256, 0, C->stream>>>(L, nullptr, C->sFace[slots[q]], C->geom, nrm, nullptr,
                                                         C->lossPart);
                k_loss_sum<<<1, 32, 0, C->stream>>>(C->lossPart, 1024, C->lossAcc);
            } else {   // no correction: the residual alone
                CKC(cudaMemsetAsync(C->corr, 0, sizeof(float) * L.E * NET_OUT, C->stream));
                k_loss_w<<<1024, 256, 0, C->stream>>>(L, C->corr, C->sRes[slots[q]], C->geom, nrm, C->sDt[slots[q]],
                                                       C->wts, C->lossPart);
                k_loss_sum<<<1, 32, 0, C->stream>>>(C->lossPart, 1024, C->lossAcc);
            }
        }
        double a[2];
        CKC(cudaMemcpyAsync(a, C->lossAcc, sizeof(a), cudaMemcpyDeviceToHost, C->stream));
        CKC(cudaStreamSynchronize(C->stream));
        acc[pass] = a[0] / n;
    }
    if (loss) *loss = acc[0];
    if (lossNone) *lossNone = acc[1];
    return check_err(C);
}

// restriction of a fine problem's State into a coarse problem's State (what = GAM_SYNC_STATE) or oState
// (GAM_SYNC_OSTATE), then the coarse BCs and Bxyz; the fine grid has 2x the coarse cells per direction
int gam_gpu_restrict(gam_gpu_t* fine, gam_gpu_t* coarse, unsigned what) {
    if (!fine || !coarse || (what != GAM_SYNC_STATE && what != GAM_SYNC_OSTATE)) return GAM_ERR_ARG;
    Handle& hf = capi_handle(fine);
    Handle& hc = capi_handle(coarse);
    if (hf.L.Nip != 2 * hc.L.Nip || hf.L.Njp != 2 * hc.L.Njp || hf.L.Nkp != 2 * hc.L.Nkp || hf.device != hc.device)
        return GAM_ERR_ARG;
    CKC(cudaStreamSynchronize(hf.stream));
    const Lay& L = hc.L;
    StateP dst = what == GAM_SYNC_STATE ? hc.S[hc.cur] : hc.S[hc.cur ^ 1];
    k_restrict_gas<<<nblk256((long long)L.Nip * L.Njp * L.Nkp), 256, 0, hc.stream>>>(L, hf.L, hf.S[hf.cur], hf.volume, dst);
    k_restrict_flux<<<nblk256((long long)(L.Nip + 1) * (L.Njp + 1) * (L.Nkp + 1)), 256, 0, hc.stream>>>(L, hf.L,
                                                                                                        hf.S[hf.cur], dst);
    launch_bcs(hc, dst, hc.stream);
    launch_bflux2fld(hc, dst, hc.stream);
    hc.launches += 2;
    CKC(cudaStreamSynchronize(hc.stream));
    return GAM_OK;
}

int gam_closure_residual_rms(gam_closure_t* C, int slot, double* rms) {
    if (!C || !rms || slot < 0 || slot >= (int)C->sIn.size()) return GAM_ERR_ARG;
    double* acc = nullptr;
    CKC(cudaMalloc(&acc, sizeof(double) * 5));
    cudaMemsetAsync(acc, 0, sizeof(double) * 5, C->stream);
    k_res_sq<<<256, 256, 0, C->stream>>>(C->L, C->sRes[slot], 5, acc);
    double h[5];
    cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, C->stream);
    cudaError_t e = cudaStreamSynchronize(C->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return GAM_ERR_CUDA;
    const double n = (double)C->L.Nip * C->L.Njp * C->L.Nkp;
    for (int v = 0; v < 5; ++v) rms[v] = std::sqrt(h[v] / n);
    rms[5] = C->sDt[slot];
    return GAM_OK;
}

int gam_closure_set_norm_emf(gam_closure_t* C, const float* emfScale, const float* resScaleB) {
    if (!C || !emfScale || !resScaleB) return GAM_ERR_ARG;
    for (int d = 0; d < 3; ++d)
        if (!(emfScale[d] >= 0.f) || !(resScaleB[d] > 0.f)) return GAM_ERR_ARG;
    for (int d = 0; d < 3; ++d) { C->emfScale[d] = emfScale[d]; C->resScaleB[d] = resScaleB[d]; }
    return GAM_OK;
}

// rms of a sample's magnetic-flux residual over the lower faces of the active cells, per face direction
int gam_closure_residual_rms_b(gam_closure_t* C, int slot, double* rms) {
    if (!C || !rms || slot < 0 || slot >= (int)C->sIn.size()) return GAM_ERR_ARG;
    double* acc = nullptr;
    CKC(cudaMalloc(&acc, sizeof(double) * 5));
    cudaMemsetAsync(acc, 0, sizeof(double) * 5, C->stream);
    k_res_sq<<<256, 256, 0, C->stream>>>(C->L, C->sRes[slot] + 5LL * C->L.E, 3, acc);   // planes 5..7
    double h[5];
    cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, C->stream);
    cudaError_t e = cudaStreamSynchronize(C->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return GAM_ERR_CUDA;
    const double n = (double)C->L.Nip * C->L.Njp * C->L.Nkp;
    for (int d = 0; d < 3; ++d) rms[d] = std::sqrt(h[d] / n);
    return GAM_OK;
}

int gam_gpu_closure_rejects(gam_gpu_t* G, int* n) {
    if (!G || !n) return GAM_ERR_ARG;
    int rc = capi_download_scalars(G);
    if (rc) return rc;
    *n = capi_handle(G).hScal->closureRejects;
    return GAM_OK;
}

}  // extern "C"
