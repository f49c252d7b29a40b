// Host-side handle of one GAMERA problem on one GPU and the step launcher.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "gam_common.cuh"

struct gam_closure;

namespace gam {

enum Prec { PREC_FP64 = 0, PREC_FP32FLUX = 1 };

// float copies used by the FP32-flux path: stencil inputs written by the predictor each step and
// metric planes converted once
struct F32Planes {
    float* Wh[5]; float* Wn[5]; float* hb[3]; float* nb[3]; float* hbA[3]; float* nbA[3]; float* Vf[3]; float* rho;
    float* VfE[2][3];   // face velocities for the I and J edges (Vf: the K edges')
    float* VdV[3];
    float* gflx[3][5]; float* mflx[3][3];   // area-scaled interface fluxes
    float* volume; float* face[3]; float* edge[3]; float* Tf[3][9]; float* Te[3][6]; float* Teb[3][4];
    // background field: fcB0, bFlux0/face and edgB0 (only with a background)
    float* fcB0[3][3]; float* b0n[3]; float* edgB0[3][2];
};

// Ring-average configuration for the LFM axis (Model%Ring, ringutils.F90:37-226)
struct RingCfg {
    int NumR = 0;
    int Nch[32] = {0};
    int recon = 1;            // 0 PLM, 1 PPM, 2 PCM
    int NFTMAG = 1;           // Fourier modes (beyond the 0th) removed from the face fluxes
    int doCleanLoop = 1, doFastLoop = 1, doMassRA = 0;
};

struct Handle {
    Lay L;
    Par p;
    RingCfg ring;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    int prec = PREC_FP64;

    // one pool holds every plane; planes are E doubles each
    double* pool = nullptr;
    size_t poolPlanes = 0;

    StateP S[2];          // State n and oState, roles swap each step (cur indexes State n)
    StateP H;             // predictor half state (Solver%StateHf)
    double* Wh[5];        // primitives of the half state (BlockCon2Prim), for reconstruction
    double* Wn[5];        // primitives of state n, for the limiter
    double* E[3];         // Efld (edge-centred, times edge length)
    double* VdV[3];       // half-state volume * momentum / max(rho, dFloor) per cell (Mom2Face summand)
    double* hbA[3];       // half-state face flux / max(face area, TINY) (EdgeLRs reconstruction values)
    double* nbA[3];       // limiter-state face flux / max(face area, TINY) (EdgeLRs limiter values)
    double* Vf[3];        // face velocities pushed along dT1 for the K edges (the last direction, as the reference leaves it)
    double* VfE[2][3];    // the same for the I and J edges (all three come from one Mom2Face pass)
    double* dGasH[5];
    double* dGasM[3];
    double* gflx[3][5];   // interface gas fluxes per direction (area-scaled)
    double* mflx[3][3];   // interface magnetic stresses per direction
    // grid metrics (owned)
    double* volume; double* xyzcc[3]; double* xfc[3][3]; double* di; double* dj; double* dk;
    double* face[3]; double* edge[3]; double* Tf[3][9]; double* Te[3][9]; double* Teb[3][4];
    double* xyz[3];       // corners (only kept when the grid was built on the device)
    // background field planes (own allocation, only with Model%doBackground), Grid_T layout per plane
    double* bgpool = nullptr;
    double* fcB0[3][3] = {}; double* edgB0[3][2] = {}; double* B0[3] = {}; double* bFlux0[3] = {}; double* dpB0[3] = {};
    // ring-average smoothing E field (own allocation, only with Model%doRing)
    double* ringpool = nullptr;
    double* SmoothE[3] = {};
    // gravitational acceleration (own allocation, only with the magnetosphere's gravity), Grid_T gxyz
    double* msphpool = nullptr;
    double* gxyz[3] = {};
    // FP32 copies for the FP32-flux mode (allocated on first use)
    float* f32pool = nullptr;
    F32Planes f32{};

    Scal* dScal = nullptr;   // device scalars
    Scal* hScal = nullptr;   // pinned host mirror
    int cur = 0;
    bool fuseUpdate = true;  // the update computes Flux2Deltas itself (off: dGasH/dGasM planes kept for inspection)
    int fluxRows = 8;        // rows per flux tile (4 or 8), chosen per problem by the ensemble autotuner
    bool tileTma = true;     // flux and E-field kernels stage by tensor copies (off: per-element cp.async)
    int tilePhase = 0;       // split-step position of a tile (gam_tiles.cu): 0 between steps
    ::gam_closure* closure = nullptr;   // learned flux closure applied in the step (gam_closure.cu)

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool useGraph = true;
    long long launches = 0;  // kernel launches issued (for accounting)

    GridP gridP() const;
    StateP cur_state() const { return S[cur]; }
    StateP old_state() const { return S[cur ^ 1]; }
};

// Enqueue one full stepGamera on h.stream with State n = S[cur]. Does not flip cur.
// part: the whole step, or the part before the fluxes (predictor, E field) / after them (Flux2Deltas on),
// for the ensembles' tile-queue flux kernel that runs between the two for all members at once
enum { STEP_ALL = 0, STEP_PRE = 1, STEP_POST = 2 };
int step_enqueue(Handle& h, int cur, cudaEvent_t* phaseEv = nullptr, bool split = false, int part = STEP_ALL);
// split = true stops after the per-cell CalcDT minimum (into Scal::dtMinBits); a tiled run then reduces
// the minimum over its tiles and continues with step_enqueue_bcs, the halo fill and step_enqueue_ghosts
void step_enqueue_bcs(Handle& h, int cur, cudaEvent_t* phaseEv = nullptr);
void step_enqueue_ghosts(Handle& h, int cur);
void launch_calcdt_partial(Handle& h, const StateP& s, cudaStream_t st);
void launch_dt_finalize(Handle& h, int mode, cudaStream_t st);
// phases recorded by step_enqueue when phaseEv is given (NPHASE+1 events)
enum { PH_PREDICT = 0, PH_EFIELD, PH_FLUXES, PH_DELTAS, PH_UPDATE, PH_DT, PH_BCS, NPHASE };
// Kernels used outside the step
void launch_bflux2fld(Handle& h, const StateP& s, cudaStream_t st);
void launch_bcs(Handle& h, const StateP& s, cudaStream_t st);
void launch_calcdt(Handle& h, const StateP& s, int mode, cudaStream_t st);   // mode 0: in-step, 1: initial (no time advance)
double launch_divb(Handle& h, double* scratchDev, cudaStream_t st);
int kernels_per_step(const Handle& h);
// learned closure in the step (gam_closure.cu): the net on State n and its face corrections (24 float
// planes, area-scaled) before Flux2Deltas; after it the positivity check that sets Scal::closureReject
const float* closure_enqueue_corr(Handle& h, const StateP& nS, cudaStream_t st);
void closure_enqueue_check(Handle& h, const StateP& nS, cudaStream_t st);
// the closure's EMF corrections added to the edge EMFs before E2Flux (skipped when the step fell back)
void closure_enqueue_emf(Handle& h, cudaStream_t st);
int closure_kernels_per_step(const Handle& h);
int closure_attach(Handle& h, ::gam_closure* c);   // shape check, geometry and periodicity from h
// interface fluxes of all directions (gam_flux.cu)
void enqueue_fluxes(Handle& h, const StateP& nS, cudaStream_t st);
void flux_kernels_init();
void enqueue_fluxes_f32(Handle& h, const StateP& nS, cudaStream_t st);   // gam_flux_f32.cu
void flux_kernels_init_f32();
// E field of all edge directions (gam_efield.cu): Mom2Face + tiled EMF
void enqueue_efield(Handle& h, const StateP& nS, cudaStream_t st);
void efield_kernels_init();
void efield_kernels_init_f32();   // gam_efield_f32.cu
// ring averaging about the LFM axis (gam_ring.cu)
// withF32: the FP32-flux half state, whose B exists only as the float copies
void launch_ring_bfix(Handle& h, const StateP& s, cudaStream_t st, bool withF32 = false);  // RingFlux2FieldFix
void launch_predfix_lfm(Handle& h, const StateP& s, cudaStream_t st, bool withF32 = false);  // lfmbw PredFix
void launch_ring_flux(Handle& h, cudaStream_t st);                              // RingFlux + FixGasFluxLFM
void launch_pole_e(Handle& h, double* const* E, cudaStream_t st);               // PoleE + FixEFieldLFM
void launch_fix_e_lfm(Handle& h, double* const* E, cudaStream_t st);            // FixEFieldLFM alone
// the magnetosphere problem (gam_msph.cu): its I boundaries, EFix, IonFlux, gravity and PerStep hooks
void launch_msph_bcs(Handle& h, const StateP& s, cudaStream_t st);
void launch_msph_efix(Handle& h, const StateP& nS, cudaStream_t st);
void launch_ion_flux(Handle& h, cudaStream_t st);
void launch_apply_grav(Handle& h, const StateP& S, const StateP& O, cudaStream_t st);
void launch_msph_perstep(Handle& h, const StateP& S, cudaStream_t st);
void launch_add_grav(Handle& h, double GM0, cudaStream_t st);
int msph_kernels_per_step(const Handle& h);
void launch_ring_average(Handle& h, const StateP& s, cudaStream_t st);          // RingAverage
int ring_kernels_per_step(const Handle& h);
// slice output (gam_io.cu): doubles of a slice, and the kernels that compute one into dst (device) from
// State n with 6 scratch planes
long long slice_count(const Handle& h, int fat);
int enqueue_slice(Handle& h, int fat, double* dst, double* scratch, cudaStream_t st);
void launch_ring_grid_fix(Handle& h, cudaStream_t st);                          // RingGridFix
void ring_kernels_init();
// allocate the float planes and convert the metrics (first switch to GAM_FP32FLUX)
int ensure_f32(Handle& h);
// re-convert the background planes into the float copies (after the background changed)
void refresh_f32_background(Handle& h);

}  // namespace gam
