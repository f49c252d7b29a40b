// Tiled runs: one problem split along k into tiles, each an ordinary handle whose k faces between tiles
// carry GAM_BC_HALO (the reference's MPI decomposition, src/gamera/mpi/gamapp_mpi.F90).
//
// A tiled step is the reference's stepGamera_mpi (:665-692): every tile advances its own cells and takes
// the per-cell CalcDT minimum; the minimum over all tiles becomes every tile's dt (CalcDT_mpi, :501-518);
// each tile runs its physical BCs, its 4-layer k halos are filled from its neighbours (haloUpdate,
// :694-794) and Bxyz of its ghost cells is recomputed from the fluxes (updateMpiBCs, :579-663).
//
// Halo messages. In the pencil layout a k layer of a plane is one contiguous run of P*Q doubles, so a
// halo is a fixed sequence of contiguous runs: per plane (Gas 5, optionally Bxyz 3, magFlux 3) the cells
// ks-4..ks-1 come from the lower neighbour's ke-3..ke; the cells ke+1..ke+4 and their I/J faces from the
// upper neighbour's ks..ks+3, and the K faces ke+1..ke+5 from its K faces ks..ks+4, so the face two tiles
// share is the upper tile's (calcDatatypeFC, :1518-1664: nG+1 K-face layers for kData=1). Layers span the
// full i/j extent, ghosts included; i and j are not decomposed, so the edge and corner pieces of the
// reference's neighbour datatypes come from the same neighbour.
//
// Two ways to drive the tiles:
//  * gam_tiles_*: all tiles in one process (one GPU, or several GPUs of a node with peer access). A tile's
//    halo fill reads its neighbours' planes directly (over NVLink when the neighbour is on another GPU);
//    the tiles' dt minimum is one kernel over their scalars. With all tiles on one GPU a step is one CUDA
//    graph whose tile branches run concurrently.
//  * gam_gpu_step_local / _bcs / _ghosts with gam_gpu_halo_pack / _unpack: the pieces a host with one
//    process per GPU (NCCL send/recv and an all-reduce MIN over two 64-bit words) strings together.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "gam_step.cuh"
#include "gamgpu.h"

struct gam_gpu;

namespace gam {
Handle& capi_handle(gam_gpu* G);
int capi_download_scalars(gam_gpu* G);
}  // namespace gam

using namespace gam;

namespace {

#define CKT(x)                                                                                        \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) {                                                                      \
            std::fprintf(stderr, "gamgpu: %s: %s\n", #x, cudaGetErrorString(e_));                    \
            return GAM_ERR_CUDA;                                                                      \
        }                                                                                             \
    } while (0)

constexpr int kPlanes = 11;                 // Gas 5, Bxyz 3, magFlux 3
constexpr int kMaxChunks = 2 * 2 * kPlanes;  // two sides, State and oState

// one contiguous run of k layers of one plane
struct Seg { int plane, k0, nl; };

double* plane_ptr(const StateP& s, int pl) {
    return pl < 5 ? s.gas[pl] : (pl < 8 ? s.b[pl - 5] : s.mf[pl - 8]);
}

// The runs of one halo side, in message order. recv: the halo of a tile with nk active k cells on
// `side` (0 lower, 1 upper); send: what this tile gives its neighbour on `side`.
int halo_segs(const Lay& L, int side, bool recv, bool withB, Seg* out) {
    const int G = L.nG, nk = L.Nkp;
    int n = 0;
    for (int pl = 0; pl < kPlanes; ++pl) {
        if (!withB && pl >= 5 && pl < 8) continue;
        bool kface = pl == 10;
        Seg s;
        if (recv) s = side == 0 ? Seg{pl, 0, G} : Seg{pl, G + nk, kface ? G + 1 : G};
        else s = side == 0 ? Seg{pl, G, kface ? G + 1 : G} : Seg{pl, nk, G};
        out[n++] = s;
    }
    return n;
}

long long seg_doubles(const Lay& L, const Seg* s, int n) {
    long long t = 0;
    for (int q = 0; q < n; ++q) t += (long long)s[q].nl * L.P * L.Q;
    return t;
}

struct Chunk { const double* src; double* dst; long long n; };   // n doubles, even, 16-byte aligned
struct ChunkTab { Chunk c[kMaxChunks]; int n; };

__global__ void k_copy_chunks(ChunkTab t) {
    const Chunk c = t.c[blockIdx.y];
    const double2* s = reinterpret_cast<const double2*>(c.src);
    double2* d = reinterpret_cast<double2*>(c.dst);
    long long n2 = c.n >> 1;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n2;
         x += (long long)gridDim.x * blockDim.x)
        d[x] = s[x];
}

void launch_chunks(Handle& h, const ChunkTab& t, cudaStream_t st) {
    if (t.n == 0) return;
    long long mx = 0;
    for (int q = 0; q < t.n; ++q) mx = t.c[q].n > mx ? t.c[q].n : mx;
    long long gx = (mx / 2 + 255) / 256;
    if (gx > 96) gx = 96;
    if (gx < 1) gx = 1;
    k_copy_chunks<<<dim3((unsigned)gx, (unsigned)t.n), 256, 0, st>>>(t);
    h.launches++;
}

// append the runs that fill side `side` of tile d (state ds) from its neighbour n (state ns)
void add_fill(const Lay& Ld, const StateP& ds, const Lay& Ln, const StateP& ns, int side, bool withB, ChunkTab& t) {
    Seg r[kPlanes], s[kPlanes];
    int nr = halo_segs(Ld, side, true, withB, r);
    halo_segs(Ln, side ^ 1, false, withB, s);
    const long long PQd = (long long)Ld.P * Ld.Q, PQn = (long long)Ln.P * Ln.Q;
    for (int q = 0; q < nr; ++q)
        t.c[t.n++] = Chunk{plane_ptr(ns, s[q].plane) + s[q].k0 * PQn, plane_ptr(ds, r[q].plane) + r[q].k0 * PQd,
                           (long long)r[q].nl * PQd};
}

// which state buffers a halo call touches: bit 0 State, bit 1 oState; mid-step "State" is the new state
int halo_states(const Handle& h, unsigned what, StateP* out) {
    int cs = h.tilePhase == 2 ? (h.cur ^ 1) : h.cur;
    int n = 0;
    if (what & GAM_HALO_STATE) out[n++] = h.S[cs];
    if (what & GAM_HALO_OSTATE) out[n++] = h.S[cs ^ 1];
    return n;
}

__global__ void k_red_pack(Scal* sc, long long* words) {
    // both words order like their values as signed 64-bit integers, so a MIN reduction works on either
    words[0] = (long long)sc->dtMinBits;
    words[1] = 0x7FFFFFFFFFFFFFFFll - (long long)sc->nanCount;
}
__global__ void k_red_unpack(Scal* sc, const long long* words) {
    sc->dtMinBits = (unsigned long long)words[0];
    sc->nanCount = (unsigned)(0x7FFFFFFFFFFFFFFFll - words[1]);
}
__global__ void k_red_reset(Scal* sc) {
    sc->dtMinBits = 0x7FF0000000000000ull;
    sc->nanCount = 0u;
}
__global__ void k_tiles_set_otime(Scal* sc) { sc->otime = sc->time - sc->dt; }   // init.F90's oState%time

// the tiles' CalcDT minimum and NaN count, written back to every tile (CalcDT_mpi)
__global__ void k_tiles_dtmin(Scal* const* sc, int n) {
    if (threadIdx.x != 0) return;
    unsigned long long b = ~0ull;
    unsigned nan = 0u;
    for (int q = 0; q < n; ++q) {
        unsigned long long v = sc[q]->dtMinBits;
        b = v < b ? v : b;
        nan += sc[q]->nanCount;
    }
    for (int q = 0; q < n; ++q) { sc[q]->dtMinBits = b; sc[q]->nanCount = nan; }
}

int status_of(int st) {
    if (st & 8) return GAM_ERR_TIMEOUT;
    if (st & 4) return GAM_ERR_NAN;
    if (st & 3) return GAM_ERR_DT_COLLAPSE;
    return GAM_OK;
}

}  // namespace

// ================================================================================ tile group
struct gam_tiles {
    std::vector<gam_gpu*> t;
    bool periodic = false;
    bool oneDevice = true;
    int dev0 = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    Scal** dScals = nullptr;   // the tiles' device scalars, on dev0
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int phase = 0;
    std::vector<int> launchesPerStep;
};

namespace {

Handle& H(gam_tiles* T, int q) { return capi_handle(T->t[q]); }

int lower_of(const gam_tiles* T, int q) {
    int n = (int)T->t.size();
    return q > 0 ? q - 1 : (T->periodic ? n - 1 : -1);
}
int upper_of(const gam_tiles* T, int q) {
    int n = (int)T->t.size();
    return q < n - 1 ? q + 1 : (T->periodic ? 0 : -1);
}

// halo fill of tile q from its neighbours, state buffers at parity offset `flip` from each tile's cur
void enqueue_fill(gam_tiles* T, int q, int flip, bool withB, bool bothStates) {
    Handle& h = H(T, q);
    ChunkTab tab;
    tab.n = 0;
    for (int which = 0; which < (bothStates ? 2 : 1); ++which) {
        int lo = lower_of(T, q), up = upper_of(T, q);
        StateP ds = h.S[h.cur ^ flip ^ which];
        if (lo >= 0) { Handle& n = H(T, lo); add_fill(h.L, ds, n.L, n.S[n.cur ^ flip ^ which], 0, withB, tab); }
        if (up >= 0) { Handle& n = H(T, up); add_fill(h.L, ds, n.L, n.S[n.cur ^ flip ^ which], 1, withB, tab); }
    }
    launch_chunks(h, tab, h.stream);
}

// fork from root to every tile stream, run f(q) on each, join back to root
template <typename F>
void fan(gam_tiles* T, F f) {
    cudaSetDevice(T->dev0);
    cudaEventRecord(T->fork, T->root);
    for (size_t q = 0; q < T->t.size(); ++q) {
        Handle& h = H(T, (int)q);
        cudaSetDevice(h.device);
        cudaStreamWaitEvent(h.stream, T->fork, 0);
        f((int)q);
        cudaEventRecord(T->join[q], h.stream);
    }
    cudaSetDevice(T->dev0);
    for (size_t q = 0; q < T->t.size(); ++q) cudaStreamWaitEvent(T->root, T->join[q], 0);
}

// one tiled step, every tile at parity cur ^ flip
int enqueue_tiled_step(gam_tiles* T, int flip) {
    int rc = 0;
    fan(T, [&](int q) { Handle& h = H(T, q); if (step_enqueue(h, h.cur ^ flip, nullptr, true) != 0) rc = GAM_ERR_CUDA; });
    k_tiles_dtmin<<<1, 32, 0, T->root>>>(T->dScals, (int)T->t.size());
    fan(T, [&](int q) { Handle& h = H(T, q); step_enqueue_bcs(h, h.cur ^ flip); });
    // the new states are at parity cur ^ flip ^ 1; Bxyz of the halo is recomputed, so it is not copied
    fan(T, [&](int q) {
        enqueue_fill(T, q, flip ^ 1, false, false);
        step_enqueue_ghosts(H(T, q), H(T, q).cur ^ flip);
    });
    return rc ? rc : (cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA);
}

void tiles_destroy_graphs(gam_tiles* T) {
    for (int c = 0; c < 2; ++c)
        if (T->graph[c]) { cudaGraphExecDestroy(T->graph[c]); T->graph[c] = nullptr; }
}

int tiles_build(gam_tiles* T) {
    tiles_destroy_graphs(T);
    cudaSetDevice(T->dev0);
    for (int c = 0; c < 2; ++c) {
        cudaGraph_t gr;
        CKT(cudaStreamBeginCapture(T->root, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_tiled_step(T, c);
        cudaError_t e = cudaStreamEndCapture(T->root, &gr);
        if (rc || e != cudaSuccess) {
            std::fprintf(stderr, "gamgpu: tiled step capture failed: %s\n", cudaGetErrorString(e));
            if (e == cudaSuccess) cudaGraphDestroy(gr);
            return GAM_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&T->graph[c], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return GAM_ERR_CUDA;
    }
    T->phase = 0;
    return GAM_OK;
}

int tiles_launch(gam_tiles* T) {
    if (T->oneDevice) {
        if (!T->graph[0]) { int rc = tiles_build(T); if (rc) return rc; }
        cudaSetDevice(T->dev0);
        CKT(cudaGraphLaunch(T->graph[T->phase], T->root));
        T->phase ^= 1;
        for (size_t q = 0; q < T->t.size(); ++q) H(T, (int)q).launches += T->launchesPerStep[q];
    } else {
        int rc = enqueue_tiled_step(T, 0);
        if (rc) return rc;
    }
    for (size_t q = 0; q < T->t.size(); ++q) H(T, (int)q).cur ^= 1;
    return GAM_OK;
}

int tiles_collect(gam_tiles* T) {
    cudaSetDevice(T->dev0);
    CKT(cudaStreamSynchronize(T->root));
    int worst = GAM_OK;
    for (auto* G : T->t) {
        cudaSetDevice(capi_handle(G).device);
        int rc = capi_download_scalars(G);
        if (rc) return rc;
        int s = status_of(capi_handle(G).hScal->sticky);
        if (s == GAM_ERR_NAN || (s && !worst)) worst = s;
    }
    cudaSetDevice(T->dev0);
    return worst;
}

// kernels of one tiled step per tile: those of an ordinary step plus the halo fill (and the tiles'
// dt minimum, counted on tile 0)
void count_launches(gam_tiles* T) {
    T->launchesPerStep.assign(T->t.size(), 0);
    for (size_t q = 0; q < T->t.size(); ++q) T->launchesPerStep[q] = kernels_per_step(H(T, (int)q)) + 1 + (q == 0);
}

}  // namespace

extern "C" {

int gam_tiles_create(gam_tiles_t** out, gam_gpu_t* const* tiles, int n, int periodicK) {
    if (!out || !tiles || n < 2) return GAM_ERR_ARG;
    *out = nullptr;
    for (int q = 0; q < n; ++q) {
        if (!tiles[q]) return GAM_ERR_ARG;
        for (int r = 0; r < q; ++r)
            if (tiles[r] == tiles[q]) return GAM_ERR_ARG;
    }
    const Handle& h0 = capi_handle(tiles[0]);
    for (int q = 0; q < n; ++q) {
        const Handle& h = capi_handle(tiles[q]);
        if (h.L.Nip != h0.L.Nip || h.L.Njp != h0.L.Njp || h.L.Nkp < h.L.nG) return GAM_ERR_ARG;
        if (h.cur != h0.cur || h.tilePhase != 0) return GAM_ERR_ARG;
        bool loHalo = q > 0 || periodicK, upHalo = q < n - 1 || periodicK;
        if ((h.p.bc[4] == BC_HALO) != loHalo || (h.p.bc[5] == BC_HALO) != upHalo) return GAM_ERR_ARG;
    }
    gam_tiles* T = new (std::nothrow) gam_tiles();
    if (!T) return GAM_ERR_ARG;
    T->t.assign(tiles, tiles + n);
    T->periodic = periodicK != 0;
    T->dev0 = h0.device;
    for (int q = 0; q < n; ++q) T->oneDevice = T->oneDevice && capi_handle(tiles[q]).device == T->dev0;
    T->join.assign(n, nullptr);
    int rc = GAM_OK;
    // peer access: dev0 reads every tile's scalars, a tile reads its neighbours' planes
    if (!T->oneDevice) {
        for (int q = 0; q < n && !rc; ++q) {
            int dq = capi_handle(tiles[q]).device;
            int nbr[3] = {T->dev0, capi_handle(tiles[lower_of(T, q) >= 0 ? lower_of(T, q) : q]).device,
                          capi_handle(tiles[upper_of(T, q) >= 0 ? upper_of(T, q) : q]).device};
            for (int a = 0; a < 3 && !rc; ++a) {
                int pairs[2][2] = {{dq, nbr[a]}, {nbr[a], dq}};
                for (auto& pr : pairs) {
                    if (pr[0] == pr[1]) continue;
                    int can = 0;
                    cudaDeviceCanAccessPeer(&can, pr[0], pr[1]);
                    if (!can) { rc = GAM_ERR_UNSUPPORTED; break; }
                    cudaSetDevice(pr[0]);
                    cudaError_t e = cudaDeviceEnablePeerAccess(pr[1], 0);
                    if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
                    else if (e != cudaSuccess) { rc = GAM_ERR_CUDA; break; }
                }
            }
        }
    }
    cudaSetDevice(T->dev0);
    if (!rc && (cudaStreamCreateWithFlags(&T->root, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&T->fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaMalloc(&T->dScals, sizeof(Scal*) * n) != cudaSuccess))
        rc = GAM_ERR_CUDA;
    for (int q = 0; q < n && !rc; ++q) {
        cudaSetDevice(capi_handle(tiles[q]).device);
        if (cudaEventCreateWithFlags(&T->join[q], cudaEventDisableTiming) != cudaSuccess) rc = GAM_ERR_CUDA;
    }
    cudaSetDevice(T->dev0);
    if (!rc) {
        std::vector<Scal*> sc(n);
        for (int q = 0; q < n; ++q) sc[q] = capi_handle(tiles[q]).dScal;
        if (cudaMemcpy(T->dScals, sc.data(), sizeof(Scal*) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = GAM_ERR_CUDA;
    }
    if (rc) { gam_tiles_destroy(T); return rc; }
    count_launches(T);
    // set-up as Hatch_mpi leaves it: halos of State and oState, Bxyz included, then the tiles' initial dt
    for (int q = 0; q < n; ++q) {
        cudaSetDevice(H(T, q).device);
        cudaStreamSynchronize(H(T, q).stream);
    }
    fan(T, [&](int q) { enqueue_fill(T, q, 0, true, true); });
    fan(T, [&](int q) {
        Handle& h = H(T, q);
        k_red_reset<<<1, 1, 0, h.stream>>>(h.dScal);
        launch_calcdt_partial(h, h.S[h.cur], h.stream);
    });
    k_tiles_dtmin<<<1, 32, 0, T->root>>>(T->dScals, n);
    fan(T, [&](int q) {
        Handle& h = H(T, q);
        launch_dt_finalize(h, 1, h.stream);
        k_tiles_set_otime<<<1, 1, 0, h.stream>>>(h.dScal);
    });
    rc = tiles_collect(T);
    if (rc == GAM_ERR_CUDA) { gam_tiles_destroy(T); return rc; }
    *out = T;
    return GAM_OK;
}

int gam_tiles_run_steps(gam_tiles_t* T, int nsteps) {
    if (!T || nsteps < 0) return GAM_ERR_ARG;
    for (int s = 0; s < nsteps; ++s) {
        int rc = tiles_launch(T);
        if (rc) return rc;
    }
    return tiles_collect(T);
}

int gam_tiles_run_steps_timed(gam_tiles_t* T, int nsteps, double* ms) {
    if (!T || nsteps < 0 || !ms) return GAM_ERR_ARG;
    if (T->oneDevice && !T->graph[0]) { int rc = tiles_build(T); if (rc) return rc; }
    cudaSetDevice(T->dev0);
    cudaEvent_t e0, e1;
    CKT(cudaEventCreate(&e0));
    CKT(cudaEventCreate(&e1));
    for (size_t q = 0; q < T->t.size(); ++q) {
        cudaSetDevice(H(T, (int)q).device);
        CKT(cudaStreamSynchronize(H(T, (int)q).stream));
    }
    cudaSetDevice(T->dev0);
    CKT(cudaEventRecord(e0, T->root));
    for (int s = 0; s < nsteps; ++s) {
        int rc = tiles_launch(T);
        if (rc) return rc;
    }
    CKT(cudaEventRecord(e1, T->root));
    CKT(cudaEventSynchronize(e1));
    float f = 0.f;
    CKT(cudaEventElapsedTime(&f, e0, e1));
    *ms = (double)f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return tiles_collect(T);
}

void gam_tiles_destroy(gam_tiles_t* T) {
    if (!T) return;
    cudaSetDevice(T->dev0);
    if (T->root) cudaStreamSynchronize(T->root);
    tiles_destroy_graphs(T);
    for (size_t q = 0; q < T->join.size(); ++q)
        if (T->join[q]) cudaEventDestroy(T->join[q]);
    if (T->fork) cudaEventDestroy(T->fork);
    if (T->root) cudaStreamDestroy(T->root);
    if (T->dScals) cudaFree(T->dScals);
    delete T;
}

// ================================================================================ split step, one process per GPU
int gam_gpu_stream(gam_gpu_t* G, void** stream) {
    if (!G || !stream) return GAM_ERR_ARG;
    *stream = (void*)capi_handle(G).stream;
    return GAM_OK;
}

// Hatch's initial dt (init.F90:204-244) for a state placed on the device afterwards (gam_gpu_sync_to_device):
// CalcDT on State, then oState%time = State%time - dt
int gam_gpu_init_dt(gam_gpu_t* G) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 0) return GAM_ERR_ARG;
    k_red_reset<<<1, 1, 0, h.stream>>>(h.dScal);
    launch_calcdt_partial(h, h.S[h.cur], h.stream);
    launch_dt_finalize(h, 1, h.stream);
    k_tiles_set_otime<<<1, 1, 0, h.stream>>>(h.dScal);
    h.launches += 2;
    int rc = capi_download_scalars(G);
    if (rc) return rc;
    return status_of(h.hScal->status);
}

int gam_gpu_calcdt_local(gam_gpu_t* G, long long* dtWords) {
    if (!G || !dtWords) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 0) return GAM_ERR_ARG;
    k_red_reset<<<1, 1, 0, h.stream>>>(h.dScal);
    launch_calcdt_partial(h, h.S[h.cur], h.stream);
    k_red_pack<<<1, 1, 0, h.stream>>>(h.dScal, dtWords);
    h.launches += 2;
    h.tilePhase = 3;
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

int gam_gpu_calcdt_finish(gam_gpu_t* G, const long long* dtWords) {
    if (!G || !dtWords) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 3) return GAM_ERR_ARG;
    k_red_unpack<<<1, 1, 0, h.stream>>>(h.dScal, dtWords);
    launch_dt_finalize(h, 1, h.stream);
    k_tiles_set_otime<<<1, 1, 0, h.stream>>>(h.dScal);
    h.launches += 2;
    h.tilePhase = 0;
    int rc = capi_download_scalars(G);
    if (rc) return rc;
    return status_of(h.hScal->status);
}

int gam_gpu_step_local(gam_gpu_t* G, long long* dtWords) {
    if (!G || !dtWords) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 0) return GAM_ERR_ARG;
    if (step_enqueue(h, h.cur, nullptr, true) != 0) return GAM_ERR_CUDA;
    k_red_pack<<<1, 1, 0, h.stream>>>(h.dScal, dtWords);
    h.launches++;
    h.tilePhase = 1;
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

int gam_gpu_step_bcs(gam_gpu_t* G, const long long* dtWords) {
    if (!G || !dtWords) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 1) return GAM_ERR_ARG;
    k_red_unpack<<<1, 1, 0, h.stream>>>(h.dScal, dtWords);
    h.launches++;
    step_enqueue_bcs(h, h.cur);
    h.tilePhase = 2;
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

int gam_gpu_step_ghosts(gam_gpu_t* G) {
    if (!G) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase != 2) return GAM_ERR_ARG;
    step_enqueue_ghosts(h, h.cur);
    h.cur ^= 1;
    h.tilePhase = 0;
    int rc = capi_download_scalars(G);
    if (rc) return rc;
    return status_of(h.hScal->status);
}

int gam_gpu_halo_bytes(gam_gpu_t* G, int side, unsigned what, long long* sendBytes, long long* recvBytes) {
    if (!G || (side != 0 && side != 1) || !(what & (GAM_HALO_STATE | GAM_HALO_OSTATE))) return GAM_ERR_ARG;
    const Handle& h = capi_handle(G);
    bool withB = (what & GAM_HALO_BXYZ) != 0;
    int ns = ((what & GAM_HALO_STATE) ? 1 : 0) + ((what & GAM_HALO_OSTATE) ? 1 : 0);
    Seg s[kPlanes];
    int n = halo_segs(h.L, side, false, withB, s);
    if (sendBytes) *sendBytes = ns * seg_doubles(h.L, s, n) * (long long)sizeof(double);
    n = halo_segs(h.L, side, true, withB, s);
    if (recvBytes) *recvBytes = ns * seg_doubles(h.L, s, n) * (long long)sizeof(double);
    return GAM_OK;
}

int gam_gpu_halo_pack(gam_gpu_t* G, int side, unsigned what, void* dst) {
    if (!G || !dst || (side != 0 && side != 1) || ((uintptr_t)dst & 15)) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase == 1 || h.tilePhase == 3) return GAM_ERR_ARG;
    StateP st[2];
    int ns = halo_states(h, what, st);
    if (!ns) return GAM_ERR_ARG;
    Seg s[kPlanes];
    int n = halo_segs(h.L, side, false, (what & GAM_HALO_BXYZ) != 0, s);
    const long long PQ = (long long)h.L.P * h.L.Q;
    ChunkTab tab;
    tab.n = 0;
    double* o = static_cast<double*>(dst);
    for (int w = 0; w < ns; ++w)
        for (int q = 0; q < n; ++q) {
            long long len = (long long)s[q].nl * PQ;
            tab.c[tab.n++] = Chunk{plane_ptr(st[w], s[q].plane) + s[q].k0 * PQ, o, len};
            o += len;
        }
    launch_chunks(h, tab, h.stream);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

int gam_gpu_halo_unpack(gam_gpu_t* G, int side, unsigned what, const void* src) {
    if (!G || !src || (side != 0 && side != 1) || ((uintptr_t)src & 15)) return GAM_ERR_ARG;
    Handle& h = capi_handle(G);
    if (h.tilePhase == 1 || h.tilePhase == 3) return GAM_ERR_ARG;
    if (h.p.bc[4 + side] != BC_HALO) return GAM_ERR_ARG;   // only a tile face takes a halo
    StateP st[2];
    int ns = halo_states(h, what, st);
    if (!ns) return GAM_ERR_ARG;
    Seg s[kPlanes];
    int n = halo_segs(h.L, side, true, (what & GAM_HALO_BXYZ) != 0, s);
    const long long PQ = (long long)h.L.P * h.L.Q;
    ChunkTab tab;
    tab.n = 0;
    const double* i = static_cast<const double*>(src);
    for (int w = 0; w < ns; ++w)
        for (int q = 0; q < n; ++q) {
            long long len = (long long)s[q].nl * PQ;
            tab.c[tab.n++] = Chunk{i, plane_ptr(st[w], s[q].plane) + s[q].k0 * PQ, len};
            i += len;
        }
    launch_chunks(h, tab, h.stream);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ERR_CUDA;
}

}  // extern "C"
