// C ABI (include/gamgpu.h): handle lifetime, Fortran-layout mirroring, step / advance entry points.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>
#include <cstdlib>
#include <new>
#include <string>
#include "gamgpu.h"
#include "gam_common.cuh"
#include "gam_step.cuh"
#include "gam_kern.cuh"
#include "gam_init.cuh"

using namespace gam;

struct gam_gpu {
    Handle h;
    double* stage = nullptr;        // contiguous staging for Fortran<->pencil repacking (two buffers that
    double* stage2 = nullptr;       // alternate, copies on xfer, repacking on the step stream)
    size_t stagePlanes = 0;
    cudaStream_t xfer = nullptr;
    cudaEvent_t xferEv[2] = {}, packEv[2] = {};
    double* scratch = nullptr;      // reduction partials
    size_t scratchDoubles = 0;
    int lastStatus = 0;
    // slice output: device staging, scratch planes, the copy stream and its events (allocated on first use)
    double* iobuf = nullptr;
    double* ioscratch = nullptr;
    size_t iobufDoubles = 0;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t ioReady = nullptr, ioDone = nullptr;
    bool ioPending = false;
    bool haveCorners = false;
};

namespace {

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            std::fprintf(stderr, "gamgpu: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_),  \
                         __FILE__, __LINE__);                                                  \
            return GAM_ERR_CUDA;                                                               \
        }                                                                                      \
    } while (0)

__global__ void k_pack_in(Lay L, double* dst, const double* src, int ni, int nj, int nk) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long n = (long long)ni * nj * nk;
    if (t >= n) return;
    int i = (int)(t % ni);
    long long q = t / ni;
    int j = (int)(q % nj), k = (int)(q / nj);
    dst[L.at(i, j, k)] = src[t];
}
__global__ void k_pack_out(Lay L, double* dst, const double* src, int ni, int nj, int nk) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long n = (long long)ni * nj * nk;
    if (t >= n) return;
    int i = (int)(t % ni);
    long long q = t / ni;
    int j = (int)(q % nj), k = (int)(q / nj);
    dst[t] = src[L.at(i, j, k)];
}

// Per-plane extents in the Fortran arrays: cell (Ni,Nj,Nk) or face/edge/corner (Ni+1,Nj+1,Nk+1)
struct Ext { int ni, nj, nk; long long n() const { return (long long)ni * nj * nk; } };
Ext cellExt(const Lay& L) { return {L.Ni, L.Nj, L.Nk}; }
Ext faceExt(const Lay& L) { return {L.Ni + 1, L.Nj + 1, L.Nk + 1}; }

// Host <-> device planes: the host copies run on their own stream through two staging buffers that
// alternate, so the repacking of one plane (on the step stream) overlaps the host copy of the next; events
// order each buffer's copy after its previous reader and each repack after its copy. When these return,
// the step stream is ordered after every copy.
int h2d_planes(gam_gpu* G, double* const* planes, int np, const double* host, Ext e) {
    Handle& h = G->h;
    double* const st[2] = {G->stage, G->stage2};
    const size_t bytes = sizeof(double) * e.n();
    // a buffer's last reader so far is earlier work on the step stream
    CK(cudaEventRecord(G->packEv[0], h.stream));
    CK(cudaEventRecord(G->packEv[1], h.stream));
    for (int q = 0; q < np; ++q) {
        const int b = q & 1;
        CK(cudaStreamWaitEvent(G->xfer, G->packEv[b], 0));
        CK(cudaMemcpyAsync(st[b], host + q * e.n(), bytes, cudaMemcpyHostToDevice, G->xfer));
        CK(cudaEventRecord(G->xferEv[b], G->xfer));
        CK(cudaStreamWaitEvent(h.stream, G->xferEv[b], 0));
        k_pack_in<<<(unsigned)((e.n() + 255) / 256), 256, 0, h.stream>>>(h.L, planes[q], st[b], e.ni, e.nj, e.nk);
        CK(cudaEventRecord(G->packEv[b], h.stream));
        h.launches++;
    }
    CK(cudaGetLastError());
    return GAM_OK;
}
int d2h_planes(gam_gpu* G, double* const* planes, int np, double* host, Ext e) {
    Handle& h = G->h;
    double* const st[2] = {G->stage, G->stage2};
    const size_t bytes = sizeof(double) * e.n();
    for (int q = 0; q < np; ++q) {
        const int b = q & 1;
        if (q >= 2) CK(cudaStreamWaitEvent(h.stream, G->xferEv[b], 0));   // the buffer's copy of plane q-2 is done
        k_pack_out<<<(unsigned)((e.n() + 255) / 256), 256, 0, h.stream>>>(h.L, st[b], planes[q], e.ni, e.nj, e.nk);
        CK(cudaEventRecord(G->packEv[b], h.stream));
        h.launches++;
        CK(cudaStreamWaitEvent(G->xfer, G->packEv[b], 0));
        CK(cudaMemcpyAsync(host + q * e.n(), st[b], bytes, cudaMemcpyDeviceToHost, G->xfer));
        CK(cudaEventRecord(G->xferEv[b], G->xfer));
    }
    for (int b = 0; b < 2 && b < np; ++b) CK(cudaStreamWaitEvent(h.stream, G->xferEv[b], 0));
    CK(cudaGetLastError());
    return GAM_OK;
}

// Grid_T background arrays (Fortran layout, cell-sized) into the background planes
int upload_background(gam_gpu* G, const double* fcB0, const double* edgB0, const double* B0, const double* bFlux0,
                      const double* dpB0) {
    Handle& h = G->h;
    if (!h.bgpool) return GAM_ERR_ARG;
    Ext ce = cellExt(h.L);
    double* pl[9];
    for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) pl[d * 3 + x] = h.fcB0[d][x];
    int rc = h2d_planes(G, pl, 9, fcB0, ce);
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 2; ++c) pl[d * 2 + c] = h.edgB0[d][c];
    if (!rc) rc = h2d_planes(G, pl, 6, edgB0, ce);
    if (!rc) rc = h2d_planes(G, h.B0, 3, B0, ce);
    if (!rc) rc = h2d_planes(G, h.bFlux0, 3, bFlux0, ce);
    if (!rc) rc = h2d_planes(G, h.dpB0, 3, dpB0, ce);
    if (!rc) refresh_f32_background(h);
    return rc;
}

int check_model(const gam_model_c* m) {
    if (!m) return GAM_ERR_ARG;
    if (m->doGrav || m->doResistive || m->doMultiF || m->doAB3 || m->nSpc != 0 ||
        m->hasHooks)
        return GAM_ERR_UNSUPPORTED;
    if (m->nG != 4 || m->Nip < 16 || m->Njp < 1 || m->Nkp < 1) return GAM_ERR_ARG;
    for (int n = 0; n < 6; ++n) {
        int b = m->bc[n];
        bool ok = b == GAM_BC_PERIODIC || b == GAM_BC_ZEROGRAD || (b == GAM_BC_LFMPOLE && (n == 2 || n == 3)) ||
                  (b == GAM_BC_LFMBW && n < 2) || (b == GAM_BC_HALO && n >= 4) || (b == GAM_BC_ION && n == 0) ||
                  (b == GAM_BC_WIND && n == 1);
        // the magnetosphere's boundaries work across the LFM axis (its ring maps)
        if ((b == GAM_BC_ION || b == GAM_BC_WIND) && !m->doRing) return GAM_ERR_ARG;
        if (!ok) return GAM_ERR_UNSUPPORTED;
        // k tiles: ring averaging needs whole rings in k, 2.5D replicates the single k layer
        if (b == GAM_BC_HALO && (m->doRing || m->do25D)) return GAM_ERR_UNSUPPORTED;
        if (b == GAM_BC_HALO && m->Nkp < m->nG) return GAM_ERR_ARG;
        if (b == GAM_BC_LFMPOLE && !m->doRing) return GAM_ERR_ARG;   // the axis maps need Model%Ring
    }
    if (m->doRing) {   // InitRings checks (ringutils.F90:203-225) and the device ring sizes
        int Np = m->Nkp;
        if (Np < 8 || Np > 512 || (Np & (Np - 1)) != 0) return GAM_ERR_ARG;
        if (m->ringNumR < 1 || m->ringNumR > 32 || m->ringNumR >= m->Njp) return GAM_ERR_ARG;
        for (int r = 0; r < m->ringNumR; ++r)
            if (m->ringNch[r] < 1 || (Np % m->ringNch[r]) != 0) return GAM_ERR_ARG;
        if (m->ringRecon < GAM_RING_PLM || m->ringRecon > GAM_RING_PCM) return GAM_ERR_ARG;
        if (!m->ringDoS && !m->ringDoE) return GAM_ERR_ARG;
    }
    if (m->rmeth != GAM_RM_8CENT && m->rmeth != GAM_RM_7UP) return GAM_ERR_ARG;
    return GAM_OK;
}

// Allocate the pool and carve the planes
int alloc_handle(gam_gpu* G, const gam_model_c* m) {
    Handle& h = G->h;
    Lay& L = h.L;
    L.Nip = m->Nip; L.Njp = m->Njp; L.Nkp = m->Nkp; L.nG = m->nG;
    L.Ni = L.Nip + 2 * L.nG; L.Nj = L.Njp + 2 * L.nG; L.Nk = L.Nkp + 2 * L.nG;
    L.P = ((L.Ni + 1) + 7) / 8 * 8;
    L.Q = L.Nj + 1; L.R = L.Nk + 1;
    L.E = (long long)L.P * L.Q * L.R;
    Par& p = h.p;
    p.gamma = m->gamma; p.CFL = m->CFL; p.pdmb = m->pdmb; p.Vd0 = m->Vd0; p.cHogH = m->cHogH; p.cHogM = m->cHogM;
    p.Ca = m->Ca; p.dFloor = m->dFloor; p.pFloor = m->pFloor; p.limDT0 = m->limDT0; p.tFin = m->tFin;
    p.doMHD = m->doMHD; p.doBoris = m->doBoris; p.do25D = m->do25D; p.doLFMLim = m->doLFMLim; p.rmeth = m->rmeth;
    p.fixedTimestep = m->fixedTimestep;
    p.doBackground = m->doBackground ? 1 : 0;
    for (int n = 0; n < 6; ++n) p.bc[n] = m->bc[n];
    p.doRing = m->doRing ? 1 : 0;
    p.ringDoS = m->doRing && m->ringDoS ? 1 : 0;
    p.ringDoE = m->doRing && m->ringDoE ? 1 : 0;
    p.predFixLFM = m->predFixLFM ? 1 : 0;
    p.dtActive = m->dtActive ? 1 : 0;
    p.bwD0 = m->bwD0; p.bwP0 = m->bwP0;
    p.stageWait = STAGE_WAIT;
    p.msph = MsphPar{};
    if (m->doRing) {
        h.ring.NumR = m->ringNumR;
        for (int r = 0; r < 32; ++r) h.ring.Nch[r] = r < m->ringNumR ? m->ringNch[r] : 0;
        h.ring.recon = m->ringRecon;
    }

    CK(cudaGetDevice(&h.device));
    flux_kernels_init();
    efield_kernels_init();
    ring_kernels_init();
    CK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    h.ownStream = true;
    const size_t planes = 11 * 3 + 10 + 14 + 9 + 24 + 91 + 6;   // + the I and J edges' face velocities
    h.poolPlanes = planes;
    CK(cudaMalloc(&h.pool, sizeof(double) * L.E * planes));
    CK(cudaMemsetAsync(h.pool, 0, sizeof(double) * L.E * planes, h.stream));
    double* q = h.pool;
    auto take = [&]() { double* r = q; q += L.E; return r; };
    for (int s = 0; s < 2; ++s) {
        for (int v = 0; v < 5; ++v) h.S[s].gas[v] = take();
        for (int x = 0; x < 3; ++x) h.S[s].mf[x] = take();
        for (int x = 0; x < 3; ++x) h.S[s].b[x] = take();
    }
    for (int v = 0; v < 5; ++v) h.H.gas[v] = take();
    for (int x = 0; x < 3; ++x) h.H.mf[x] = take();
    for (int x = 0; x < 3; ++x) h.H.b[x] = take();
    for (int v = 0; v < 5; ++v) h.Wh[v] = take();
    for (int v = 0; v < 5; ++v) h.Wn[v] = take();
    for (int x = 0; x < 3; ++x) h.E[x] = take();   // contiguous: memset as one range
    for (int x = 0; x < 3; ++x) h.Vf[x] = take();
    for (int e = 0; e < 2; ++e) for (int x = 0; x < 3; ++x) h.VfE[e][x] = take();
    for (int x = 0; x < 3; ++x) h.VdV[x] = take();
    for (int x = 0; x < 3; ++x) h.hbA[x] = take();
    for (int x = 0; x < 3; ++x) h.nbA[x] = take();
    for (int v = 0; v < 5; ++v) h.dGasH[v] = take();
    for (int x = 0; x < 3; ++x) h.dGasM[x] = take();
    for (int d = 0; d < 3; ++d) for (int v = 0; v < 5; ++v) h.gflx[d][v] = take();
    for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) h.mflx[d][x] = take();
    h.volume = take();
    for (int x = 0; x < 3; ++x) h.xyzcc[x] = take();
    for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) h.xfc[d][x] = take();
    h.di = take(); h.dj = take(); h.dk = take();
    for (int d = 0; d < 3; ++d) h.face[d] = take();
    for (int d = 0; d < 3; ++d) h.edge[d] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 9; ++c) h.Tf[d][c] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 9; ++c) h.Te[d][c] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 4; ++c) h.Teb[d][c] = take();
    for (int x = 0; x < 3; ++x) h.xyz[x] = take();
    if ((size_t)(q - h.pool) != (size_t)L.E * planes) return GAM_ERR_ARG;
    if (p.doRing) {   // ring-average smoothing E field, 3 contiguous planes
        CK(cudaMalloc(&h.ringpool, sizeof(double) * L.E * 3));
        CK(cudaMemsetAsync(h.ringpool, 0, sizeof(double) * L.E * 3, h.stream));
        for (int x = 0; x < 3; ++x) h.SmoothE[x] = h.ringpool + (size_t)x * L.E;
    }
    if (p.doBackground) {   // fcB0 (9), edgB0 (6), B0, bFlux0, dpB0 (3 each)
        const size_t bgPlanes = 24;
        CK(cudaMalloc(&h.bgpool, sizeof(double) * L.E * bgPlanes));
        CK(cudaMemsetAsync(h.bgpool, 0, sizeof(double) * L.E * bgPlanes, h.stream));
        q = h.bgpool;
        for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) h.fcB0[d][x] = take();
        for (int d = 0; d < 3; ++d) for (int c = 0; c < 2; ++c) h.edgB0[d][c] = take();
        for (int x = 0; x < 3; ++x) h.B0[x] = take();
        for (int d = 0; d < 3; ++d) h.bFlux0[d] = take();
        for (int x = 0; x < 3; ++x) h.dpB0[x] = take();
    }

    Ext fe = faceExt(L);
    CK(cudaMalloc(&G->stage, sizeof(double) * fe.n()));
    CK(cudaMalloc(&G->stage2, sizeof(double) * fe.n()));
    CK(cudaStreamCreateWithFlags(&G->xfer, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        CK(cudaEventCreateWithFlags(&G->xferEv[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&G->packEv[b], cudaEventDisableTiming));
    }
    G->scratchDoubles = (size_t)((long long)L.Nip * L.Njp * L.Nkp / 256 + 1024);
    CK(cudaMalloc(&G->scratch, sizeof(double) * G->scratchDoubles));
    CK(cudaMalloc(&h.dScal, sizeof(Scal)));
    CK(cudaMallocHost(&h.hScal, sizeof(Scal)));
    std::memset(h.hScal, 0, sizeof(Scal));
    h.hScal->t = m->t; h.hScal->dt = m->dt; h.hScal->dt0 = m->dt0; h.hScal->ts = m->ts;
    h.hScal->dtMinBits = 0x7FF0000000000000ull;
    CK(cudaMemcpyAsync(h.dScal, h.hScal, sizeof(Scal), cudaMemcpyHostToDevice, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int upload_scalars(gam_gpu* G) {
    Handle& h = G->h;
    CK(cudaMemcpyAsync(h.dScal, h.hScal, sizeof(Scal), cudaMemcpyHostToDevice, h.stream));
    return GAM_OK;
}
int download_scalars(gam_gpu* G) {
    Handle& h = G->h;
    CK(cudaMemcpyAsync(h.hScal, h.dScal, sizeof(Scal), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int status_code(int st) {
    if (st & 8) return GAM_ERR_TIMEOUT;
    if (st & 4) return GAM_ERR_NAN;
    if (st & 3) return GAM_ERR_DT_COLLAPSE;
    return GAM_OK;
}

void destroy_graphs(Handle& h) {
    for (int c = 0; c < 2; ++c)
        if (h.graph[c]) { cudaGraphExecDestroy(h.graph[c]); h.graph[c] = nullptr; }
}

int build_graphs(gam_gpu* G) {
    Handle& h = G->h;
    destroy_graphs(h);
    for (int c = 0; c < 2; ++c) {
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
        int rc = step_enqueue(h, c);
        cudaError_t e = cudaStreamEndCapture(h.stream, &gr);
        if (rc != 0 || e != cudaSuccess) {
            std::fprintf(stderr, "gamgpu: step capture failed: %s\n", cudaGetErrorString(e));
            if (e == cudaSuccess) cudaGraphDestroy(gr);
            return GAM_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&h.graph[c], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return GAM_ERR_CUDA;
    }
    return GAM_OK;
}

int launch_one_step(gam_gpu* G) {
    Handle& h = G->h;
    // the magnetosphere's boundaries need its parameters (gam_gpu_set_magnetosphere or GAM_IC_MAGSPHERE)
    if ((h.p.bc[0] == BC_ION || h.p.bc[1] == BC_WIND) && !h.p.msph.on) return GAM_ERR_ARG;
    if (h.useGraph) {
        if (!h.graph[0]) {
            int rc = build_graphs(G);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(h.graph[h.cur], h.stream));
        h.launches += kernels_per_step(h);
    } else {
        if (step_enqueue(h, h.cur) != 0) return GAM_ERR_CUDA;
    }
    h.cur ^= 1;
    return GAM_OK;
}

}  // namespace

// Shared with gam_init.cu
namespace gam {
int capi_alloc(gam_gpu* G, const gam_model_c* m) { return alloc_handle(G, m); }
int capi_upload_scalars(gam_gpu* G) { return upload_scalars(G); }
int capi_download_scalars(gam_gpu* G) { return download_scalars(G); }
Handle& capi_handle(gam_gpu* G) { return G->h; }
double* capi_scratch(gam_gpu* G) { return G->scratch; }
}  // namespace gam

extern "C" {

const char* gam_gpu_errstr(int code) {
    switch (code) {
    case GAM_OK: return "ok";
    case GAM_ERR_NAN: return "NaN in the state (CellDT)";
    case GAM_ERR_DT_COLLAPSE: return "timestep collapse (CalcDT isDisaster/isBad)";
    case GAM_ERR_CUDA: return "CUDA error";
    case GAM_ERR_TIMEOUT: return "bounded device wait timed out";
    case GAM_ERR_UNSUPPORTED: return "Model option not supported on the device path";
    case GAM_ERR_ARG: return "bad argument";
    default: return "unknown";
    }
}

int gam_gpu_create(gam_gpu_t** out, const gam_model_c* m, const gam_grid_c* g, const double* gas,
                   const double* magflux, const double* bxyz, const double* ogas, const double* omagflux,
                   const double* obxyz, double time, double otime) {
    if (!out || !g || !gas || !magflux || !ogas || !omagflux) return GAM_ERR_ARG;
    *out = nullptr;
    int rc = check_model(m);
    if (rc) return rc;
    if (!g->xyzcc || !g->xfc || !g->di || !g->dj || !g->dk || !g->volume || !g->face || !g->edge || !g->Tf ||
        !g->Te || !g->Teb)
        return GAM_ERR_ARG;
    if (m->doBackground && (!g->fcB0 || !g->edgB0 || !g->B0 || !g->bFlux0 || !g->dpB0)) return GAM_ERR_ARG;
    gam_gpu* G = new (std::nothrow) gam_gpu();
    if (!G) return GAM_ERR_ARG;
    rc = alloc_handle(G, m);
    if (rc) { gam_gpu_destroy(G); return rc; }
    Handle& h = G->h;
    const Lay& L = h.L;
    Ext ce = cellExt(L), fe = faceExt(L);
    double* pl[27];
    rc = h2d_planes(G, &h.volume, 1, g->volume, ce);
    if (!rc) rc = h2d_planes(G, h.xyzcc, 3, g->xyzcc, ce);
    if (!rc) { for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) pl[d * 3 + x] = h.xfc[d][x]; rc = h2d_planes(G, pl, 9, g->xfc, fe); }
    if (!rc) rc = h2d_planes(G, &h.di, 1, g->di, ce);
    if (!rc) rc = h2d_planes(G, &h.dj, 1, g->dj, ce);
    if (!rc) rc = h2d_planes(G, &h.dk, 1, g->dk, ce);
    if (!rc) rc = h2d_planes(G, h.face, 3, g->face, fe);
    if (!rc) rc = h2d_planes(G, h.edge, 3, g->edge, fe);
    if (!rc) { for (int d = 0; d < 3; ++d) for (int c = 0; c < 9; ++c) pl[d * 9 + c] = h.Tf[d][c]; rc = h2d_planes(G, pl, 27, g->Tf, fe); }
    if (!rc) { for (int d = 0; d < 3; ++d) for (int c = 0; c < 9; ++c) pl[d * 9 + c] = h.Te[d][c]; rc = h2d_planes(G, pl, 27, g->Te, fe); }
    if (!rc) { for (int d = 0; d < 3; ++d) for (int c = 0; c < 4; ++c) pl[d * 4 + c] = h.Teb[d][c]; rc = h2d_planes(G, pl, 12, g->Teb, fe); }
    if (!rc && m->doBackground) rc = upload_background(G, g->fcB0, g->edgB0, g->B0, g->bFlux0, g->dpB0);
    if (!rc && g->xyz) { rc = h2d_planes(G, h.xyz, 3, g->xyz, fe); G->haveCorners = true; }
    if (rc) { gam_gpu_destroy(G); return rc; }
    rc = gam_gpu_sync_to_device(G, GAM_SYNC_STATE | GAM_SYNC_OSTATE, gas, magflux, bxyz, ogas, omagflux, obxyz, time,
                                otime);
    if (rc) { gam_gpu_destroy(G); return rc; }
    *out = G;
    return GAM_OK;
}

static int create_from_corners(gam_gpu_t** out, const gam_model_c* m, const double* xyz, int ic, const BgSpec* bg,
                               const double* icPar = nullptr) {
    if (!out || !xyz) return GAM_ERR_ARG;
    *out = nullptr;
    int rc = check_model(m);
    if (rc) return rc;
    bool caseIC = ic == GAM_IC_ADV1D || ic == GAM_IC_ADV2D || ic == GAM_IC_LOOP2D || ic == GAM_IC_ALFVEN ||
                  ic == GAM_IC_MAGSPHERE;
    if (ic != GAM_IC_OT2D && ic != GAM_IC_BW && ic != GAM_IC_LFMBW && !((ic == GAM_IC_KH || caseIC) && icPar))
        return GAM_ERR_ARG;
    if (ic == GAM_IC_MAGSPHERE && (m->bc[0] != GAM_BC_ION || m->bc[1] != GAM_BC_WIND)) return GAM_ERR_ARG;
    if ((m->Nip % 8) != 0) return GAM_ERR_ARG;   // Corners2Grid divisibility check (init.F90:830-834)
    if ((bg != nullptr) != (m->doBackground != 0)) return GAM_ERR_ARG;
    gam_gpu* G = new (std::nothrow) gam_gpu();
    if (!G) return GAM_ERR_ARG;
    rc = alloc_handle(G, m);
    if (rc) { gam_gpu_destroy(G); return rc; }
    Handle& h = G->h;
    rc = h2d_planes(G, h.xyz, 3, xyz, faceExt(h.L));
    if (rc) { gam_gpu_destroy(G); return rc; }
    G->haveCorners = true;
    h.hScal->time = m->t;   // allocState: State%time = Model%t
    h.hScal->otime = m->t;
    rc = upload_scalars(G);
    if (!rc && init_grid_from_corners(h) != 0) rc = GAM_ERR_CUDA;
    if (!rc && init_problem(h, ic, bg, icPar) != 0) rc = GAM_ERR_CUDA;
    if (!rc) rc = download_scalars(G);
    if (rc) { gam_gpu_destroy(G); return rc; }
    *out = G;
    return GAM_OK;
}

int gam_gpu_create_from_corners(gam_gpu_t** out, const gam_model_c* m, const double* xyz, int ic) {
    return create_from_corners(out, m, xyz, ic, nullptr);
}

int gam_gpu_create_from_corners_ic(gam_gpu_t** out, const gam_model_c* m, const double* xyz, int ic,
                                   const double* icPar, int nPar) {
    if (ic == GAM_IC_KH && (!icPar || nPar < 4 || !(icPar[0] > 0.0) || icPar[3] < 0.0)) return GAM_ERR_ARG;
    if (ic == GAM_IC_MAGSPHERE) {   // its background is the cut dipole (genCutDipole)
        if (!icPar || nPar < GAM_NMSPH || !m || !m->doBackground) return GAM_ERR_ARG;
        BgSpec bg;
        bg.type = 3;
        bg.par[0] = bg.par[1] = bg.par[2] = 0.0; bg.par[3] = icPar[0];
        bg.cut[0] = icPar[2]; bg.cut[1] = icPar[3]; bg.cut[2] = icPar[4];
        return create_from_corners(out, m, xyz, ic, &bg, icPar);
    }
    static const int casePars[4] = {0, 7, 9, 5};   // ADV1D, ADV2D, LOOP2D, ALFVEN
    if (ic >= GAM_IC_ADV1D && ic <= GAM_IC_ALFVEN) {
        int need = casePars[ic - GAM_IC_ADV1D];
        if (nPar < need || (need > 0 && !icPar) || nPar > 10) return GAM_ERR_ARG;
        double par[10] = {0.0};
        for (int n = 0; n < nPar; ++n) par[n] = icPar[n];
        return create_from_corners(out, m, xyz, ic, nullptr, par);
    }
    return create_from_corners(out, m, xyz, ic, nullptr, icPar);
}

int gam_gpu_create_from_corners_b0(gam_gpu_t** out, const gam_model_c* m, const double* xyz, int ic, int b0Kind,
                                   const double* b0Par) {
    if (!b0Par || (b0Kind != GAM_B0_UNIFORM && b0Kind != GAM_B0_DIPOLE)) return GAM_ERR_ARG;
    BgSpec bg;
    bg.type = b0Kind;
    for (int n = 0; n < 4; ++n) bg.par[n] = b0Par[n];
    return create_from_corners(out, m, xyz, ic, &bg);
}

int gam_gpu_sync_to_device(gam_gpu_t* G, unsigned what, const double* gas, const double* magflux, const double* bxyz,
                           const double* ogas, const double* omagflux, const double* obxyz, double time, double otime) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = G->h;
    const Lay& L = h.L;
    Ext ce = cellExt(L), fe = faceExt(L);
    int rc = GAM_OK;
    StateP n = h.S[h.cur], o = h.S[h.cur ^ 1];
    if ((what & GAM_SYNC_STATE) && gas) rc = h2d_planes(G, n.gas, 5, gas, ce);
    if (!rc && (what & GAM_SYNC_STATE) && magflux) rc = h2d_planes(G, n.mf, 3, magflux, fe);
    if (!rc && (what & GAM_SYNC_OSTATE) && ogas) rc = h2d_planes(G, o.gas, 5, ogas, ce);
    if (!rc && (what & GAM_SYNC_OSTATE) && omagflux) rc = h2d_planes(G, o.mf, 3, omagflux, fe);
    if (rc) return rc;
    // Bxyz as given, else from the fluxes (bFlux2Fld), as after a restart read (init.F90:204-210)
    if (what & GAM_SYNC_STATE) {
        if (bxyz) rc = h2d_planes(G, n.b, 3, bxyz, ce);
        else launch_bflux2fld(h, n, h.stream);
    }
    if (!rc && (what & GAM_SYNC_OSTATE)) {
        if (obxyz) rc = h2d_planes(G, o.b, 3, obxyz, ce);
        else launch_bflux2fld(h, o, h.stream);
    }
    if (rc) return rc;
    // State%time / oState%time travel with the arrays; the other scalars stay as they are on the device
    rc = download_scalars(G);
    if (rc) return rc;
    if (what & GAM_SYNC_STATE) h.hScal->time = time;
    if (what & GAM_SYNC_OSTATE) h.hScal->otime = otime;
    rc = upload_scalars(G);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int gam_gpu_sync_to_host(gam_gpu_t* G, unsigned what, double* gas, double* magflux, double* bxyz, double* ogas,
                         double* omagflux) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = G->h;
    const Lay& L = h.L;
    Ext ce = cellExt(L), fe = faceExt(L);
    StateP n = h.S[h.cur], o = h.S[h.cur ^ 1];
    int rc = GAM_OK;
    if ((what & GAM_SYNC_STATE) && gas) rc = d2h_planes(G, n.gas, 5, gas, ce);
    if (!rc && (what & GAM_SYNC_STATE) && magflux) rc = d2h_planes(G, n.mf, 3, magflux, fe);
    if (!rc && (what & GAM_SYNC_STATE) && bxyz) rc = d2h_planes(G, n.b, 3, bxyz, ce);
    if (!rc && (what & GAM_SYNC_OSTATE) && ogas) rc = d2h_planes(G, o.gas, 5, ogas, ce);
    if (!rc && (what & GAM_SYNC_OSTATE) && omagflux) rc = d2h_planes(G, o.mf, 3, omagflux, fe);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int gam_gpu_set_scalars(gam_gpu_t* G, double t, double dt, double dt0, int ts, double time, double otime) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = G->h;
    h.hScal->t = t; h.hScal->dt = dt; h.hScal->dt0 = dt0; h.hScal->ts = ts; h.hScal->time = time;
    h.hScal->otime = otime; h.hScal->dtMinBits = 0x7FF0000000000000ull; h.hScal->nanCount = 0;
    h.hScal->status = 0; h.hScal->sticky = 0; h.hScal->waitFail = 0u;
    int rc = upload_scalars(G);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int gam_gpu_get_status(gam_gpu_t* G, gam_status_c* s) {
    if (!G || !s) return GAM_ERR_ARG;
    int rc = download_scalars(G);
    if (rc) return rc;
    Handle& h = G->h;
    s->t = h.hScal->t; s->dt = h.hScal->dt; s->dt0 = h.hScal->dt0; s->time = h.hScal->time; s->otime = h.hScal->otime;
    s->ts = h.hScal->ts; s->status = status_code(h.hScal->status); s->nanCells = (int)h.hScal->lastNan;
    s->precision = h.prec; s->kernelLaunches = h.launches;
    return GAM_OK;
}

int gam_gpu_step(gam_gpu_t* G, double* dt, int* ts, double* t) {
    if (!G) return GAM_ERR_ARG;
    int rc = launch_one_step(G);
    if (rc) return rc;
    rc = download_scalars(G);
    if (rc) return rc;
    Handle& h = G->h;
    if (dt) *dt = h.hScal->dt;
    if (ts) *ts = h.hScal->ts;
    if (t) *t = h.hScal->t;
    G->lastStatus = status_code(h.hScal->status);
    return G->lastStatus;
}

int gam_gpu_advance(gam_gpu_t* G, double dtAdvance) {
    if (!G) return GAM_ERR_ARG;
    int rc = download_scalars(G);
    if (rc) return rc;
    double target = G->h.hScal->t + dtAdvance;
    double t = 0.0;
    rc = gam_gpu_step(G, nullptr, nullptr, &t);
    if (rc) return rc;
    while (t < target) {
        rc = gam_gpu_step(G, nullptr, nullptr, &t);
        if (rc) return rc;
    }
    return GAM_OK;
}

int gam_gpu_run_steps(gam_gpu_t* G, int n) {
    if (!G || n < 0) return GAM_ERR_ARG;
    for (int s = 0; s < n; ++s) {
        int rc = launch_one_step(G);
        if (rc) return rc;
    }
    int rc = download_scalars(G);
    if (rc) return rc;
    G->lastStatus = status_code(G->h.hScal->sticky);
    return G->lastStatus;
}

int gam_gpu_run_steps_timed(gam_gpu_t* G, int n, double* ms) {
    if (!G || n < 0 || !ms) return GAM_ERR_ARG;
    Handle& h = G->h;
    if (h.useGraph && !h.graph[0]) {
        int rc = build_graphs(G);
        if (rc) return rc;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaStreamSynchronize(h.stream));
    CK(cudaEventRecord(e0, h.stream));
    for (int s = 0; s < n; ++s) {
        int rc = launch_one_step(G);
        if (rc) return rc;
    }
    CK(cudaEventRecord(e1, h.stream));
    CK(cudaEventSynchronize(e1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, e0, e1));
    *ms = (double)f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = download_scalars(G);
    if (rc) return rc;
    G->lastStatus = status_code(G->h.hScal->sticky);
    return G->lastStatus;
}

int gam_gpu_profile_phases(gam_gpu_t* G, int nsteps, double* ms, int nphase) {
    if (!G || nsteps <= 0 || !ms || nphase < NPHASE) return GAM_ERR_ARG;
    Handle& h = G->h;
    cudaEvent_t ev[NPHASE + 1];
    for (int q = 0; q <= NPHASE; ++q) CK(cudaEventCreate(&ev[q]));
    for (int q = 0; q < NPHASE; ++q) ms[q] = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        if (step_enqueue(h, h.cur, ev) != 0) return GAM_ERR_CUDA;
        h.cur ^= 1;
        CK(cudaEventSynchronize(ev[NPHASE]));
        for (int q = 0; q < NPHASE; ++q) {
            float f = 0.f;
            CK(cudaEventElapsedTime(&f, ev[q], ev[q + 1]));
            ms[q] += f / nsteps;
        }
    }
    for (int q = 0; q <= NPHASE; ++q) cudaEventDestroy(ev[q]);
    int rc = download_scalars(G);
    if (rc) return rc;
    return status_code(G->h.hScal->sticky);
}

int gam_gpu_set_tile(gam_gpu_t* G, int what, int value) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = G->h;
    if (what == GAM_TILE_FUSED_UPDATE) {
        if (value != 0 && value != 1) return GAM_ERR_ARG;
        if (h.fuseUpdate != (value != 0)) { h.fuseUpdate = value != 0; destroy_graphs(h); }
        return GAM_OK;
    }
    if (what == GAM_TILE_TMA) {
        if (value != 0 && value != 1) return GAM_ERR_ARG;
        if (h.tileTma != (value != 0)) { h.tileTma = value != 0; destroy_graphs(h); }
        return GAM_OK;
    }
    if (what == GAM_TILE_STAGE_WAIT) {   // 1: the normal bound; 0: give up at once (tests the timeout path)
        if (value != 0 && value != 1) return GAM_ERR_ARG;
        unsigned int polls = value ? STAGE_WAIT : 0u;
        if (h.p.stageWait != polls) { h.p.stageWait = polls; destroy_graphs(h); }
        return GAM_OK;
    }
    if (what != GAM_TILE_FLUX_ROWS || (value != 4 && value != 8)) return GAM_ERR_ARG;
    if (h.fluxRows != value) {
        h.fluxRows = value;
        destroy_graphs(h);
    }
    return GAM_OK;
}

int gam_gpu_set_magnetosphere(gam_gpu_t* G, const double* par, int n) {
    if (!G || !par || n < GAM_NMSPH) return GAM_ERR_ARG;
    Handle& h = G->h;
    // WindEFix needs Grid%xyz (gam_grid_c.xyz)
    if (h.p.bc[0] != BC_ION || h.p.bc[1] != BC_WIND || !h.p.doBackground || !G->haveCorners) return GAM_ERR_ARG;
    if (h.closure) return GAM_ERR_UNSUPPORTED;
    int rc = msph_setup(h, par, n);
    if (rc) return GAM_ERR_CUDA;
    destroy_graphs(h);
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

int gam_gpu_set_closure(gam_gpu_t* G, gam_closure_t* c) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = G->h;
    if (c) {
        int rc = closure_attach(h, c);
        if (rc) return rc;
    }
    destroy_graphs(h);   // the step graphs are captured with or without the closure's kernels
    h.closure = c;
    return GAM_OK;
}

int gam_gpu_divb(gam_gpu_t* G, double* tot) {
    if (!G || !tot) return GAM_ERR_ARG;
    *tot = launch_divb(G->h, G->scratch, G->h.stream);
    CK(cudaGetLastError());
    return GAM_OK;
}

int gam_gpu_set_precision(gam_gpu_t* G, int mode) {
    if (!G) return GAM_ERR_ARG;
    if (mode != GAM_FP64 && mode != GAM_FP32FLUX) return GAM_ERR_ARG;
    if (mode == GAM_FP32FLUX && ensure_f32(G->h) != 0) return GAM_ERR_CUDA;
    if (mode != G->h.prec) {
        G->h.prec = mode;
        destroy_graphs(G->h);
    }
    return GAM_OK;
}

int gam_gpu_fetch(gam_gpu_t* G, const char* name, double* out, long long n) {
    if (!G || !name || !out) return GAM_ERR_ARG;
    Handle& h = G->h;
    const Lay& L = h.L;
    Ext ce = cellExt(L), fe = faceExt(L);
    double* pl[27];
    int np = 0;
    Ext e = ce;
    std::string s(name);
    StateP cS = h.S[h.cur], oS = h.S[h.cur ^ 1];
    auto put = [&](double* const* src, int k) { for (int q = 0; q < k; ++q) pl[np++] = src[q]; };
    if (s == "gas") put(cS.gas, 5);
    else if (s == "magflux") { put(cS.mf, 3); e = fe; }
    else if (s == "bxyz") put(cS.b, 3);
    else if (s == "ogas") put(oS.gas, 5);
    else if (s == "omagflux") { put(oS.mf, 3); e = fe; }
    else if (s == "obxyz") put(oS.b, 3);
    else if (s == "hgas") put(h.H.gas, 5);
    else if (s == "hmagflux") { put(h.H.mf, 3); e = fe; }
    else if (s == "hbxyz") put(h.H.b, 3);
    else if (s == "efld") put(h.E, 3);
    else if (s == "vf") put(h.Vf, 3);
    else if (s == "dgash") put(h.dGasH, 5);
    else if (s == "dgasm") put(h.dGasM, 3);
    else if (s == "gflx") { for (int d = 0; d < 3; ++d) put(h.gflx[d], 5); }
    else if (s == "mflx") { for (int d = 0; d < 3; ++d) put(h.mflx[d], 3); }
    else if (s == "volume") put(&h.volume, 1);
    else if (s == "xyzcc") put(h.xyzcc, 3);
    else if (s == "xfc") { for (int d = 0; d < 3; ++d) put(h.xfc[d], 3); e = fe; }
    else if (s == "di") put(&h.di, 1);
    else if (s == "dj") put(&h.dj, 1);
    else if (s == "dk") put(&h.dk, 1);
    else if (s == "face") { put(h.face, 3); e = fe; }
    else if (s == "edge") { put(h.edge, 3); e = fe; }
    else if (s == "tf") { for (int d = 0; d < 3; ++d) put(h.Tf[d], 9); e = fe; }
    else if (s == "te") { for (int d = 0; d < 3; ++d) put(h.Te[d], 9); e = fe; }
    else if (s == "teb") { for (int d = 0; d < 3; ++d) put(h.Teb[d], 4); e = fe; }
    else if (s == "xyz") { put(h.xyz, 3); e = fe; }
    else if (h.bgpool && s == "fcb0") { for (int d = 0; d < 3; ++d) put(h.fcB0[d], 3); }
    else if (h.bgpool && s == "edgb0") { for (int d = 0; d < 3; ++d) put(h.edgB0[d], 2); }
    else if (h.bgpool && s == "b0") put(h.B0, 3);
    else if (h.bgpool && s == "bflux0") put(h.bFlux0, 3);
    else if (h.bgpool && s == "dpb0") put(h.dpB0, 3);
    else if (h.ringpool && s == "smoothe") put(h.SmoothE, 3);
    else return GAM_ERR_ARG;
    if (n < (long long)np * e.n()) return GAM_ERR_ARG;
    int rc = d2h_planes(G, pl, np, out, e);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h.stream));
    return GAM_OK;
}

long long gam_gpu_slice_count(gam_gpu_t* G, unsigned flags) {
    if (!G) return -1;
    return slice_count(G->h, (flags & GAM_SLICE_FAT) ? 1 : 0);
}

static int slice_prepare(gam_gpu* G, unsigned flags, long long n, double* out) {
    Handle& h = G->h;
    if (!out) return GAM_ERR_ARG;
    if (!G->haveCorners) return GAM_ERR_ARG;   // J and E need Grid%xyz
    long long need = slice_count(h, (flags & GAM_SLICE_FAT) ? 1 : 0);
    if (n < need) return GAM_ERR_ARG;
    if (!G->copyStream) {
        CK(cudaStreamCreateWithFlags(&G->copyStream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&G->ioReady, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&G->ioDone, cudaEventDisableTiming));
        CK(cudaMalloc(&G->ioscratch, sizeof(double) * h.L.E * 6));
    }
    if ((size_t)need > G->iobufDoubles) {
        if (G->ioPending) CK(cudaEventSynchronize(G->ioDone));
        if (G->iobuf) cudaFree(G->iobuf);
        G->iobuf = nullptr;
        CK(cudaMalloc(&G->iobuf, sizeof(double) * (size_t)need));
        G->iobufDoubles = (size_t)need;
    }
    if (G->ioPending) CK(cudaStreamWaitEvent(h.stream, G->ioDone, 0));   // the staging buffer is free again
    return GAM_OK;
}

int gam_gpu_slice_begin(gam_gpu_t* G, unsigned flags, double* out, long long n) {
    if (!G) return GAM_ERR_ARG;
    int rc = slice_prepare(G, flags, n, out);
    if (rc) return rc;
    Handle& h = G->h;
    int fat = (flags & GAM_SLICE_FAT) ? 1 : 0;
    if (enqueue_slice(h, fat, G->iobuf, G->ioscratch, h.stream) != 0) return GAM_ERR_CUDA;
    CK(cudaEventRecord(G->ioReady, h.stream));
    CK(cudaStreamWaitEvent(G->copyStream, G->ioReady, 0));
    CK(cudaMemcpyAsync(out, G->iobuf, sizeof(double) * (size_t)slice_count(h, fat), cudaMemcpyDeviceToHost,
                       G->copyStream));
    CK(cudaEventRecord(G->ioDone, G->copyStream));
    G->ioPending = true;
    return GAM_OK;
}

int gam_gpu_slice_wait(gam_gpu_t* G) {
    if (!G) return GAM_ERR_ARG;
    if (G->ioPending) {
        CK(cudaEventSynchronize(G->ioDone));
        G->ioPending = false;
    }
    return GAM_OK;
}

int gam_gpu_slice(gam_gpu_t* G, unsigned flags, double* out, long long n) {
    int rc = gam_gpu_slice_begin(G, flags, out, n);
    if (rc) return rc;
    return gam_gpu_slice_wait(G);
}

void gam_gpu_destroy(gam_gpu_t* G) {
    if (!G) return;
    Handle& h = G->h;
    if (h.stream) cudaStreamSynchronize(h.stream);
    destroy_graphs(h);
    if (h.pool) cudaFree(h.pool);
    if (h.bgpool) cudaFree(h.bgpool);
    if (h.ringpool) cudaFree(h.ringpool);
    if (h.f32pool) cudaFree(h.f32pool);
    if (G->xfer) cudaStreamSynchronize(G->xfer);
    if (G->stage) cudaFree(G->stage);
    if (G->stage2) cudaFree(G->stage2);
    for (int b = 0; b < 2; ++b) {
        if (G->xferEv[b]) cudaEventDestroy(G->xferEv[b]);
        if (G->packEv[b]) cudaEventDestroy(G->packEv[b]);
    }
    if (G->xfer) cudaStreamDestroy(G->xfer);
    if (G->scratch) cudaFree(G->scratch);
    if (G->copyStream) cudaStreamSynchronize(G->copyStream);
    if (G->iobuf) cudaFree(G->iobuf);
    if (G->ioscratch) cudaFree(G->ioscratch);
    if (G->ioReady) cudaEventDestroy(G->ioReady);
    if (G->ioDone) cudaEventDestroy(G->ioDone);
    if (G->copyStream) cudaStreamDestroy(G->copyStream);
    if (h.dScal) cudaFree(h.dScal);
    if (h.hScal) cudaFreeHost(h.hScal);
    if (h.stream && h.ownStream) cudaStreamDestroy(h.stream);
    if (h.msphpool) cudaFree(h.msphpool);
    delete G;
}

}  // extern "C"

// ================================================================================ ensembles
// A batch of independent problems advanced together. One step of the batch is one CUDA graph launch
// that holds every active member's whole step as its own branch: the branches run concurrently, so many
// small grids fill the GPU that one of them alone would leave mostly idle, and the host launches once
// per batch step instead of once per kernel per member. Each member keeps its own time step. Every step
// flips each member's buffer parity, so two graphs (the current parities and their complement) cover a
// run; they are rebuilt when the set of active members changes.
struct gam_ensemble {
    std::vector<gam_gpu*> members;
    std::vector<char> active;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int phase = 0;   // which of the two graphs runs next
    // tile queue: the members' flux kernels replaced by one persistent launch per precision
    bool queue = false;
    FluxJob<double>* jobs64[2] = {nullptr, nullptr};
    FluxJob<float>* jobs32[2] = {nullptr, nullptr};
    int n64 = 0, n32 = 0;
    long long tiles64[2] = {0, 0}, tiles32[2] = {0, 0};
    unsigned long long* counter = nullptr;   // [2]: FP64 and FP32 queues
};

namespace {
void ens_destroy_graphs(gam_ensemble* E) {
    for (int c = 0; c < 2; ++c)
        if (E->graph[c]) { cudaGraphExecDestroy(E->graph[c]); E->graph[c] = nullptr; }
}
// capture the batch step with member m at parity cur[m] ^ flip
void ens_free_jobs(gam_ensemble* E) {
    for (int c = 0; c < 2; ++c) {
        if (E->jobs64[c]) { cudaFree(E->jobs64[c]); E->jobs64[c] = nullptr; }
        if (E->jobs32[c]) { cudaFree(E->jobs32[c]); E->jobs32[c] = nullptr; }
    }
    E->n64 = E->n32 = 0;
}
// the queue's jobs for both parities of the active members
int ens_build_jobs(gam_ensemble* E) {
    ens_free_jobs(E);
    for (int flip = 0; flip < 2; ++flip) {
        std::vector<FluxJob<double>> j64;
        std::vector<FluxJob<float>> j32;
        long long f64 = 0, f32 = 0;
        for (size_t m = 0; m < E->members.size(); ++m) {
            if (!E->active[m]) continue;
            Handle& h = E->members[m]->h;
            if (h.prec == PREC_FP32FLUX) flux_jobs32(h, j32, f32);
            else flux_jobs64(h, h.cur ^ flip, j64, f64);
        }
        E->n64 = (int)j64.size();
        E->n32 = (int)j32.size();
        E->tiles64[flip] = f64;
        E->tiles32[flip] = f32;
        if (E->n64) {
            CK(cudaMalloc(&E->jobs64[flip], sizeof(FluxJob<double>) * E->n64));
            CK(cudaMemcpy(E->jobs64[flip], j64.data(), sizeof(FluxJob<double>) * E->n64, cudaMemcpyHostToDevice));
        }
        if (E->n32) {
            CK(cudaMalloc(&E->jobs32[flip], sizeof(FluxJob<float>) * E->n32));
            CK(cudaMemcpy(E->jobs32[flip], j32.data(), sizeof(FluxJob<float>) * E->n32, cudaMemcpyHostToDevice));
        }
    }
    return GAM_OK;
}
int ens_capture(gam_ensemble* E, int flip, cudaGraphExec_t* out) {
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(E->root, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    // the members' steps as concurrent branches; with the queue, the branches stop before the fluxes and
    // continue after one persistent flux launch that covers every member's tiles
    const int parts[2] = {E->queue ? STEP_PRE : STEP_ALL, STEP_POST};
    for (int pi = 0; pi < (E->queue ? 2 : 1); ++pi) {
        if (pi == 1) {
            int sms = 148, dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaMemsetAsync(E->counter, 0, 2 * sizeof(unsigned long long), E->root);
            if (E->n64) launch_flux_queue64(E->jobs64[flip], E->n64, E->tiles64[flip], E->counter, sms * 3, E->root);
            if (E->n32) launch_flux_queue32(E->jobs32[flip], E->n32, E->tiles32[flip], E->counter + 1, sms * 4, E->root);
        }
        cudaEventRecord(E->fork, E->root);
        for (size_t m = 0; m < E->members.size(); ++m) {
            if (!E->active[m]) continue;
            Handle& h = E->members[m]->h;
            cudaStreamWaitEvent(h.stream, E->fork, 0);
            if (step_enqueue(h, h.cur ^ flip, nullptr, false, parts[pi]) != 0) rc = GAM_ERR_CUDA;
            cudaEventRecord(E->join[m], h.stream);
            cudaStreamWaitEvent(E->root, E->join[m], 0);
        }
    }
    cudaError_t e = cudaStreamEndCapture(E->root, &gr);
    if (rc || e != cudaSuccess) {
        std::fprintf(stderr, "gamgpu: ensemble capture failed: %s\n", cudaGetErrorString(e));
        if (e == cudaSuccess) cudaGraphDestroy(gr);
        return GAM_ERR_CUDA;
    }
    e = cudaGraphInstantiate(out, gr, 0);
    cudaGraphDestroy(gr);
    return e == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}
int ens_build(gam_ensemble* E) {
    ens_destroy_graphs(E);
    for (auto* G : E->members) CK(cudaStreamSynchronize(G->h.stream));
    if (E->queue) {
        int rc = ens_build_jobs(E);
        if (rc) return rc;
    }
    int rc = ens_capture(E, 0, &E->graph[0]);
    if (!rc) rc = ens_capture(E, 1, &E->graph[1]);
    E->phase = 0;
    return rc;
}
int ens_launch(gam_ensemble* E) {
    CK(cudaGraphLaunch(E->graph[E->phase], E->root));
    E->phase ^= 1;
    bool first = true;
    for (size_t m = 0; m < E->members.size(); ++m) {
        if (!E->active[m]) continue;
        Handle& h = E->members[m]->h;
        h.cur ^= 1;
        h.launches += kernels_per_step(h);
        if (E->queue) {   // its flux launches are the shared queue launches, counted on the first member
            h.launches -= h.p.do25D ? 2 : 3;
            if (first) h.launches += (E->n64 ? 1 : 0) + (E->n32 ? 1 : 0) + 1;
            first = false;
        }
    }
    return GAM_OK;
}
int ens_collect(gam_ensemble* E) {   // scalars of every member back to the host; OR of their statuses
    CK(cudaStreamSynchronize(E->root));
    bool nan = false, collapse = false;
    for (auto* G : E->members) {
        int rc = download_scalars(G);
        if (rc) return rc;
        G->lastStatus = status_code(G->h.hScal->sticky);
        nan = nan || G->lastStatus == GAM_ERR_NAN;
        collapse = collapse || G->lastStatus == GAM_ERR_DT_COLLAPSE;
    }
    return nan ? GAM_ERR_NAN : (collapse ? GAM_ERR_DT_COLLAPSE : GAM_OK);
}
}  // namespace

extern "C" {

int gam_gpu_ensemble_create(gam_ensemble_t** out, gam_gpu_t* const* members, int n) {
    if (!out || !members || n < 1) return GAM_ERR_ARG;
    *out = nullptr;
    int dev0 = members[0] ? members[0]->h.device : -1;
    for (int m = 0; m < n; ++m) {
        if (!members[m] || members[m]->h.device != dev0) return GAM_ERR_ARG;
        for (int q = 0; q < m; ++q)
            if (members[q] == members[m]) return GAM_ERR_ARG;
    }
    gam_ensemble* E = new (std::nothrow) gam_ensemble();
    if (!E) return GAM_ERR_ARG;
    E->members.assign(members, members + n);
    E->active.assign(n, 1);
    E->join.assign(n, nullptr);
    bool ok = cudaStreamCreateWithFlags(&E->root, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int m = 0; ok && m < n; ++m) ok = cudaEventCreateWithFlags(&E->join[m], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { gam_gpu_ensemble_destroy(E); return GAM_ERR_CUDA; }
    *out = E;
    return GAM_OK;
}

int gam_gpu_ensemble_run_steps(gam_ensemble_t* E, int nsteps) {
    if (!E || nsteps < 0) return GAM_ERR_ARG;
    if (!E->graph[0]) { int rc = ens_build(E); if (rc) return rc; }
    for (int s = 0; s < nsteps; ++s) { int rc = ens_launch(E); if (rc) return rc; }
    return ens_collect(E);
}

int gam_gpu_ensemble_run_steps_timed(gam_ensemble_t* E, int nsteps, double* ms) {
    if (!E || nsteps < 0 || !ms) return GAM_ERR_ARG;
    if (!E->graph[0]) { int rc = ens_build(E); if (rc) return rc; }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaStreamSynchronize(E->root));
    CK(cudaEventRecord(e0, E->root));
    for (int s = 0; s < nsteps; ++s) { int rc = ens_launch(E); if (rc) return rc; }
    CK(cudaEventRecord(e1, E->root));
    CK(cudaEventSynchronize(e1));
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = f;
    return ens_collect(E);
}

int gam_gpu_ensemble_advance(gam_ensemble_t* E, double tEnd, int chunk, int maxSteps, int* steps) {
    if (!E || chunk < 1 || maxSteps < 0) return GAM_ERR_ARG;
    int taken = 0, st = GAM_OK;
    while (taken < maxSteps) {
        int rc = ens_collect(E);
        if (rc == GAM_ERR_CUDA) return rc;
        st = rc ? rc : st;
        bool changed = false, any = false;
        for (size_t m = 0; m < E->members.size(); ++m) {
            bool act = E->members[m]->h.hScal->t < tEnd;
            if ((char)act != E->active[m]) { E->active[m] = act; changed = true; }
            any = any || act;
        }
        if (!any) break;
        if (changed || !E->graph[0]) { rc = ens_build(E); if (rc) return rc; }
        int n = chunk < maxSteps - taken ? chunk : maxSteps - taken;
        for (int s = 0; s < n; ++s) { rc = ens_launch(E); if (rc) return rc; }
        taken += n;
    }
    if (steps) *steps = taken;
    int rc = ens_collect(E);
    for (size_t m = 0; m < E->members.size(); ++m) E->active[m] = 1;   // later runs step every member again
    ens_destroy_graphs(E);
    return rc ? rc : st;
}

// Autotuner: members grouped by grid shape; for each group, largest first, every flux tile height is timed
// over `steps` batch steps with the other groups fixed, and the fastest kept. The tile height does not
// change any result (each interface is computed from the same staged values), so the steps it takes are
// ordinary steps of the run.
int gam_gpu_ensemble_autotune(gam_ensemble_t* E, int steps, int* fluxRows, int* queue) {
    if (!E || steps < 1) return GAM_ERR_ARG;
    const size_t n = E->members.size();
    std::vector<long long> key(n);
    std::vector<long long> groups;
    for (size_t m = 0; m < n; ++m) {
        const Lay& L = E->members[m]->h.L;
        key[m] = ((long long)L.Nip << 40) | ((long long)L.Njp << 20) | (long long)L.Nkp;
        bool seen = false;
        for (long long g : groups) seen = seen || g == key[m];
        if (!seen) groups.push_back(key[m]);
    }
    auto cells = [](long long k) { return (k >> 40) * ((k >> 20) & 0xFFFFF) * (k & 0xFFFFF); };
    std::sort(groups.begin(), groups.end(), [&](long long a, long long b) { return cells(a) > cells(b); });
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (long long g : groups) {
        int best = 8;
        float bestMs = 0.f;
        const int cand[2] = {8, 4};
        for (int c : cand) {
            for (size_t m = 0; m < n; ++m)
                if (key[m] == g) gam_gpu_set_tile(E->members[m], GAM_TILE_FLUX_ROWS, c);
            int rc = ens_build(E);
            if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
            rc = ens_launch(E);   // untimed: first launch of the new graphs
            if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
            CK(cudaEventRecord(e0, E->root));
            for (int s = 0; s < steps; ++s) {
                rc = ens_launch(E);
                if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
            }
            CK(cudaEventRecord(e1, E->root));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (c == cand[0] || ms < bestMs) { best = c; bestMs = ms; }
        }
        for (size_t m = 0; m < n; ++m)
            if (key[m] == g) gam_gpu_set_tile(E->members[m], GAM_TILE_FLUX_ROWS, best);
    }
    // then the flux phase as per-member launches or as one tile-queue launch, whichever is faster
    {
        float msMode[2] = {0.f, 0.f};
        for (int on = 0; on < 2; ++on) {
            int rc = gam_gpu_ensemble_set_queue(E, on);
            if (!rc) rc = ens_build(E);
            if (!rc) rc = ens_launch(E);
            if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
            CK(cudaEventRecord(e0, E->root));
            for (int s = 0; s < steps; ++s) {
                rc = ens_launch(E);
                if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
            }
            CK(cudaEventRecord(e1, E->root));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&msMode[on], e0, e1));
        }
        int rc = gam_gpu_ensemble_set_queue(E, msMode[1] < msMode[0] ? 1 : 0);
        if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = ens_build(E);
    if (rc) return rc;
    if (fluxRows)
        for (size_t m = 0; m < n; ++m) fluxRows[m] = E->members[m]->h.fluxRows;
    if (queue) *queue = E->queue ? 1 : 0;
    return ens_collect(E);
}

void gam_gpu_ensemble_destroy(gam_ensemble_t* E) {
    if (!E) return;
    if (E->root) cudaStreamSynchronize(E->root);
    ens_destroy_graphs(E);
    ens_free_jobs(E);
    if (E->counter) cudaFree(E->counter);
    for (auto ev : E->join) if (ev) cudaEventDestroy(ev);
    if (E->fork) cudaEventDestroy(E->fork);
    if (E->root) cudaStreamDestroy(E->root);
    delete E;
}

int gam_gpu_ensemble_set_queue(gam_ensemble_t* E, int on) {
    if (!E || (on != 0 && on != 1)) return GAM_ERR_ARG;
    if (on && !E->counter) CK(cudaMalloc(&E->counter, 2 * sizeof(unsigned long long)));
    if (E->queue != (on != 0)) {
        for (auto* G : E->members) CK(cudaStreamSynchronize(G->h.stream));
        ens_destroy_graphs(E);
        E->queue = on != 0;
    }
    return GAM_OK;
}

}  // extern "C"
