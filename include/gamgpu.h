/* gamgpu.h -- C ABI of the B200 GAMERA ideal-MHD step.
 *
 * This is the drop-in boundary for the reference's step call. A Fortran host keeps its Model_T,
 * Grid_T and State_T (src/base/types/gamtypes.F90:71-286), runs Hatch (src/gamera/init.F90:38-59)
 * as before, and hands the arrays to gam_gpu_create; stepGamera (src/gamera/gamapp.F90:73-94)
 * becomes gam_gpu_step and gamAdvanceModel (src/gamera/gamtypessub.F90:78-94) becomes
 * gam_gpu_advance. Every array argument is a plain double* in the reference's Fortran layout:
 * column-major, i fastest, ghosts included, lower bounds isg/jsg/ksg, the trailing dimension(s)
 * being the variable / vector component / transform index exactly as declared in gamtypes.F90.
 * No torch or CUDA types appear here.
 *
 * Return codes are GAM_OK (0) or one of GAM_ERR_*; nothing traps on the device.
 */
#ifndef GAMGPU_H
#define GAMGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define GAM_OK 0
#define GAM_ERR_NAN 1          /* a CellDT evaluation produced NaN (bad state)                    */
#define GAM_ERR_DT_COLLAPSE 2  /* CalcDT's isDisaster / isBad (src/gamera/step.F90:103-135)      */
#define GAM_ERR_CUDA 3         /* a CUDA call failed; the handle should be destroyed              */
#define GAM_ERR_TIMEOUT 4      /* a bounded device wait gave up                                   */
#define GAM_ERR_UNSUPPORTED 5  /* a Model option this library does not run on the device         */
#define GAM_ERR_ARG 6          /* bad argument (null pointer, size, name)                          */

/* precision modes (gam_gpu_set_precision) */
#define GAM_FP64 0             /* everything in FP64: the parity path                              */
#define GAM_FP32FLUX 1         /* FP32 reconstruction, limiter, kinetic fluxes and EMF arithmetic;
                                  FP64 state, accumulation, CT update, C2P with floors and dt      */

/* boundary kinds for gam_model_c.bc[] in the reference's order INI,OUTI,INJ,OUTJ,INK,OUTK
   (src/base/defs/gdefs.F90:43-45) */
#define GAM_BC_PERIODIC 0      /* src/gamera/bcs.F90:279-450 */
#define GAM_BC_ZEROGRAD 1      /* src/gamera/bcs.F90:799-930 */
#define GAM_BC_LFMPOLE 2       /* INJ/OUTJ across the LFM axis: lfmIn/lfmOut, src/gamera/bcs.F90:1020-1106 */
#define GAM_BC_LFMBW 3         /* INI/OUTI fixed-gas shells of the LFM blast wave: bw_ibcI/bw_obcI,
                                  src/gamera/ICs/lfmbw.F90:141-225 (gas state gam_model_c.bwD0/bwP0) */
#define GAM_BC_ION 5           /* INI: the magnetosphere's ionospheric boundary (IonInner, src/voltron/ICs/earthcmi.F90:378-522) */
#define GAM_BC_WIND 6          /* OUTI: the magnetosphere's solar-wind boundary (WindBC, src/gamera/apps/wind.F90:206-374) */
#define GAM_BC_HALO 4          /* INK/OUTK of a k-tile inside a decomposed problem: no physical BC, the ghost
                                  layers are filled from the neighbouring tile (the reference's mpiNullBc_T,
                                  src/gamera/mpi/gamapp_mpi.F90:428-463); not with doRing or do25D */

/* ring reconstruction (ring/rngrec, src/gamera/init.F90:466-478) */
#define GAM_RING_PLM 0
#define GAM_RING_PPM 1
#define GAM_RING_PCM 2

/* reconstruction (Model sim/rmeth, src/gamera/init.F90:447-462) */
#define GAM_RM_8CENT 0
#define GAM_RM_7UP 1

/* sync masks */
#define GAM_SYNC_STATE 1u      /* State%Gas, State%magFlux (and State%Bxyz on the way out) */
#define GAM_SYNC_OSTATE 2u     /* oState%Gas, oState%magFlux                                */

typedef struct gam_gpu gam_gpu_t;

/* The Model_T fields the step reads (src/base/types/gamtypes.F90:71-146). */
typedef struct {
    int Nip, Njp, Nkp;         /* active cells (Grid_T Nip,Njp,Nkp)                     */
    int nG;                    /* ghosts per side (Model%nG, 4)                         */
    double gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, dFloor, pFloor, limDT0;
    double t, tFin, dt, dt0;   /* Model%t, tFin, dt, dt0                                 */
    int ts;                    /* Model%ts                                              */
    int doMHD, doBoris, do25D, doLFMLim, rmeth, fixedTimestep;
    /* doBackground: a background field B0 (gam_grid_c fcB0..dpB0) enters the fluxes, E field, CalcDT and
     * Boris update (src/gamera/background.F90). doRing: ring averaging about the LFM axis (the ring
     * fields below). The other options are not run on the device; nonzero -> GAM_ERR_UNSUPPORTED */
    int doBackground, doGrav, doResistive, doRing, doMultiF, doAB3, nSpc, hasHooks;
    int bc[6];                 /* GAM_BC_* per face                                      */
    /* ring averaging about the LFM axis (doRing with ring/gid = lfm; src/gamera/ringav.F90,
     * ringutils.F90): Model%Ring%NumR and Nch(1:NumR) as InitRings set them (ringutils.F90:37-226),
     * the ring reconstruction, and Model%Ring%doS/doE (both 1 on an untiled grid) */
    int ringNumR;
    int ringNch[32];
    int ringRecon;             /* GAM_RING_*                                              */
    int ringDoS, ringDoE;
    /* problem pieces the LFM blast wave (src/gamera/ICs/lfmbw.F90) sets: its predictor fix
     * (HackPredictor => PredFix, :227-248), the gas state of its GAM_BC_LFMBW shells, and its
     * timestep domain (DT bounds = active cells, :86-92) */
    int predFixLFM;
    double bwD0, bwP0;
    int dtActive;              /* 1: CalcDT over the active cells only; 0: one ghost layer more */
} gam_model_c;

/* The Grid_T metric arrays the step reads (gamtypes.F90:163-245), Fortran layout. */
typedef struct {
    const double* xyzcc;   /* (Ni,Nj,Nk,3)            cell centres              */
    const double* xfc;     /* (Ni+1,Nj+1,Nk+1,3,3)    face centres              */
    const double* di;      /* (Ni,Nj,Nk)              dt lengths                */
    const double* dj;
    const double* dk;
    const double* volume;  /* (Ni,Nj,Nk)                                       */
    const double* face;    /* (Ni+1,Nj+1,Nk+1,3)      face areas                */
    const double* edge;    /* (Ni+1,Nj+1,Nk+1,3)      edge lengths              */
    const double* Tf;      /* (Ni+1,Nj+1,Nk+1,9,3)    face triads               */
    const double* Te;      /* (Ni+1,Nj+1,Nk+1,9,3)    edge triads               */
    const double* Teb;     /* (Ni+1,Nj+1,Nk+1,4,3)    edge B transforms         */
    /* background field from AddB0 (src/gamera/background.F90:20-167); NULL unless Model%doBackground */
    const double* fcB0;    /* (Ni,Nj,Nk,3,3)          face-averaged B0 [xyz, face dir]   */
    const double* edgB0;   /* (Ni,Nj,Nk,2,3)          edge-frame B0 [tangent, edge dir]  */
    const double* B0;      /* (Ni,Nj,Nk,3)            cell-averaged B0                   */
    const double* bFlux0;  /* (Ni,Nj,Nk,3)            B0 flux through the lower faces    */
    const double* dpB0;    /* (Ni,Nj,Nk,3)            background momentum source          */
    /* Grid%xyz corners (Ni+1,Nj+1,Nk+1,3); optional, needed only by the slice output (current, E) */
    const double* xyz;
} gam_grid_c;

typedef struct {
    double t, dt, dt0, time, otime; /* Model%t/dt/dt0, State%time, oState%time */
    int ts;
    int status;                     /* GAM_ERR_* of the last step, 0 if fine    */
    int nanCells;                   /* cells with NaN CellDT in the last step    */
    int precision;
    long long kernelLaunches;       /* kernels launched by this handle so far    */
} gam_status_c;

/* Mirror a Hatch-ed problem onto the current CUDA device. gas/ogas are State%Gas/oState%Gas
 * (Ni,Nj,Nk,5); magflux/omagflux are (Ni+1,Nj+1,Nk+1,3); bxyz/obxyz are State%Bxyz/oState%Bxyz
 * (Ni,Nj,Nk,3) -- pass them as Hatch left them (its EnforceBCs runs after bFlux2Fld, so ghost cells
 * may differ from a fresh bFlux2Fld); NULL recomputes them with bFlux2Fld. time/otime are
 * State%time/oState%time. Replaces: the arrays Hatch leaves in gamApp_T (src/gamera/init.F90:150-260). */
int gam_gpu_create(gam_gpu_t** h, const gam_model_c* m, const gam_grid_c* g, const double* gas,
                   const double* magflux, const double* bxyz, const double* ogas, const double* omagflux,
                   const double* obxyz, double time, double otime);

/* Build the grid metrics and the initial state on the device from corner coordinates
 * xyz (Ni+1,Nj+1,Nk+1,3): Corners2Grid (src/gamera/init.F90:801-1145) and the problem set-up that
 * ends CalcGridInfo (init.F90:204-244: bFlux2Fld, EnforceBCs, CalcDT, oState = State).
 * ic: GAM_IC_OT2D (src/gamera/prob.F90:74-119) or GAM_IC_BW (prob.F90:190-298, deck defaults). */
#define GAM_IC_OT2D 0
#define GAM_IC_BW 1
#define GAM_IC_LFMBW 2   /* the LFM blast wave with the deck of tests/gamera/lfmbw.xml (x0=-50, y0=30, z0=0,
                            rC=20, P0=0.1, pRat=10, D0=1, B0=1): ICs/lfmbw.F90:33-104 */
int gam_gpu_create_from_corners(gam_gpu_t** h, const gam_model_c* m, const double* xyz, int ic);

/* gam_gpu_create_from_corners for initial conditions with parameters:
 *   GAM_IC_KH: the Kelvin-Helmholtz shear layer of the batched-ensemble problem (no counterpart in the
 *   reference), sampled at cell centres: rho = 1, P = 1, Vx = 0.5 tanh((y-0.5)/a), Vy = amp*(2u-1) with u
 *   a counter-based hash of (seed, i, j, k), B = (Bx, 0, 0). icPar = {a, Bx, amp, seed}, nPar >= 4. */
#define GAM_IC_KH 3
/*   The accuracy cases of the reference's tests/cases/testCases.pf, with the values of their decks
 *   (tests/cases/*.xml) in icPar and Model%gamma as the deck leaves it (1.4 for ADV1D):
 *   GAM_IC_ADV1D:  initADV1D (src/gamera/prob.F90:671-736), four density shapes at Vx = 1, no field; nPar 0.
 *   GAM_IC_ADV2D:  initADV2D (prob.F90:739-797), icPar = {d0, P0, V0, alpha, R0, x0, y0}.
 *   GAM_IC_LOOP2D: initLoop (prob.F90:436-500), icPar = {d0, P0, V0, Vz0, alpha, A0, R0, x0, y0}.
 *   GAM_IC_ALFVEN: initALFVEN (prob.F90:1027-1083), icPar = {d0, P0, B_para, V_para, alp}. */
#define GAM_IC_ADV1D 4
#define GAM_IC_ADV2D 5
#define GAM_IC_LOOP2D 6
#define GAM_IC_ALFVEN 7
/*   GAM_IC_MAGSPHERE: the magnetosphere of the reference's Earth deck (tests/voltron/cmriD_Earth.xml, its Gamera
 *   part: voltron/ICs/earthcmi.F90 initUser) with a constant solar wind and no ionospheric coupling -- the cut
 *   dipole as background field with the elliptically cut initial field (apps/msphutils.F90:419-532), uniform gas
 *   at rest, gravity (background.F90:170-252), the ionospheric inner boundary with zero potential and the
 *   solar-wind outer boundary (bc {GAM_BC_ION, GAM_BC_WIND, GAM_BC_LFMPOLE x2, GAM_BC_PERIODIC x2} on an LFM
 *   grid with rings; Model%doBackground = 1), and the hooks EFix, IonFlux and PerStep. icPar (GAM_NMSPH values,
 *   code units) = {M0, GM0, rCut, lCut, dcScl, xSun, xTail, yMax, sInner, wind D, P, Vx, Vy, Vz, Bx, By, Bz,
 *   dtCpl, gT0 [s], Rho0, P0, nIonP, doIonPush}; kaiju_b200/magnetosphere.py computes them from physical units
 *   as setMagsphere and readWind do (apps/msphutils.F90:65-185, apps/wind.F90:620-700). */
#define GAM_IC_MAGSPHERE 8
#define GAM_NMSPH 23
int gam_gpu_create_from_corners_ic(gam_gpu_t** h, const gam_model_c* m, const double* xyz, int ic,
                                   const double* icPar, int nPar);

/* gam_gpu_create_from_corners with a background field (Model%doBackground must be set): AddB0
 * (src/gamera/background.F90:20-167) runs on the device after the IC, as CalcGridInfo does
 * (init.F90:180-184), with a built-in Model%B0:
 *   GAM_B0_UNIFORM: B0 = (par[0], par[1], par[2]), the blast wave's BlastB0 (prob.F90:261-269). With
 *                   GAM_IC_BW it replaces the blast field (prob/doBack: residual field starts at 0).
 *   GAM_B0_DIPOLE:  B0 = 3 (m.r) r/|r|^5 - m/|r|^3, m = (0, 0, par[3]), r measured from
 *                   (par[0], par[1], par[2]) (Dipole, apps/msphutils.F90:534-551, centred at the origin
 *                   there). */
#define GAM_B0_UNIFORM 1
#define GAM_B0_DIPOLE 2
int gam_gpu_create_from_corners_b0(gam_gpu_t** h, const gam_model_c* m, const double* xyz, int ic, int b0Kind,
                                   const double* b0Par);

/* One stepGamera (src/gamera/gamapp.F90:73-94): AdvanceMHD, ts/t update, CalcDT, EnforceBCs,
 * bFlux2Fld. Outputs (may be NULL): the new Model%dt, Model%ts, Model%t. */
int gam_gpu_step(gam_gpu_t* h, double* dt, int* ts, double* t);

/* gamAdvanceModel (src/gamera/gamtypessub.F90:78-94): step at least once, until t >= t0 + dtAdvance. */
int gam_gpu_advance(gam_gpu_t* h, double dtAdvance);

/* n steps back to back without a host round trip per step (device-resident dt); status is the OR of
 * the steps' statuses. */
int gam_gpu_run_steps(gam_gpu_t* h, int n);

/* n steps like gam_gpu_run_steps, timed with CUDA events on the handle's stream; *ms = elapsed time. */
int gam_gpu_run_steps_timed(gam_gpu_t* h, int n, double* ms);

/* Average per-step device time of each phase of the step over nsteps eager (non-graph) steps, in
 * the order predictor, E field, fluxes, flux divergence, update (CT + Reynolds/Maxwell), CalcDT,
 * boundaries + bFlux2Fld. nphase must be >= 7. The steps advance the state. */
#define GAM_NPHASE 7
int gam_gpu_profile_phases(gam_gpu_t* h, int nsteps, double* ms, int nphase);

/* Copy state to / from the caller's Fortran arrays (NULL pointers are skipped; on the way in a NULL
 * Bxyz is recomputed from the fluxes with bFlux2Fld, as after a restart read, init.F90:204-210). */
int gam_gpu_sync_to_host(gam_gpu_t* h, unsigned what, double* gas, double* magflux, double* bxyz,
                         double* ogas, double* omagflux);
int gam_gpu_sync_to_device(gam_gpu_t* h, unsigned what, const double* gas, const double* magflux,
                           const double* bxyz, const double* ogas, const double* omagflux,
                           const double* obxyz, double time, double otime);

/* Model/state scalars, e.g. to resume from a restart (Model%t, dt, dt0, ts; State%time, oState%time) */
int gam_gpu_get_status(gam_gpu_t* h, gam_status_c* s);
int gam_gpu_set_scalars(gam_gpu_t* h, double t, double dt, double dt0, int ts, double time, double otime);

/* DivB (src/gamera/gridutils.F90:717-770): sum over active cells of |net face flux| */
int gam_gpu_divb(gam_gpu_t* h, double* tot);

/* GAM_FP64 or GAM_FP32FLUX */
int gam_gpu_set_precision(gam_gpu_t* h, int mode);

/* Fetch an internal or grid array in the reference's Fortran layout, by the reference's name:
 * "gas","magflux","bxyz","ogas","omagflux","obxyz","hgas","hmagflux","hbxyz" (Solver%StateHf),
 * "efld","vf","dgash","dgasm","gflx","mflx", "volume","xyzcc","xfc","di","dj","dk","face","edge",
 * "tf","te","teb","xyz". n = number of doubles the caller's buffer holds. */
int gam_gpu_fetch(gam_gpu_t* h, const char* name, double* out, long long n);

void gam_gpu_destroy(gam_gpu_t* h);

/* Slice output: the variables writeSlc computes from State (src/gamera/gioH5.F90:255-602) for the active
 * cells of a single-fluid problem: D, Vx, Vy, Vz, P, Cs, Bx, By, Bz (total field), Pb, Jx, Jy, Jz (the
 * current of bFld2Jxyz, gridutils.F90:314-478) and, with GAM_SLICE_FAT (output/doFatIO), Ex, Ey, Ez
 * (Eijk2xyz) and DivB (plus DivdB with a background field). Each variable is one Fortran-ordered
 * (is:ie, js:je, ks:ke) block of out, in that order; gam_gpu_slice_count gives the doubles needed. The
 * handle must know Grid%xyz (gam_grid_c.xyz, or a handle built from corners).
 * gam_gpu_slice_begin computes the slice of the current State on the step stream and copies it to out on a
 * separate copy stream, returning at once: steps issued afterwards run while the copy proceeds (with
 * page-locked out; pageable memory makes the copy synchronous). gam_gpu_slice_wait waits for that copy;
 * gam_gpu_slice does both. Replaces: the State copy-back and the host loops of writeSlc. */
#define GAM_SLICE_FAT 1u
long long gam_gpu_slice_count(gam_gpu_t* h, unsigned flags);
int gam_gpu_slice_begin(gam_gpu_t* h, unsigned flags, double* out, long long n);
int gam_gpu_slice_wait(gam_gpu_t* h);
int gam_gpu_slice(gam_gpu_t* h, unsigned flags, double* out, long long n);

/* Ensembles: independent problems (any sizes, on one device) advanced together. Each batch step is one
 * CUDA graph launch holding every active member's stepGamera as a concurrent branch; every member keeps
 * its own dt. No counterpart in the reference, which runs one problem per process. The members stay
 * owned by the caller and usable on their own between ensemble calls. */
typedef struct gam_ensemble gam_ensemble_t;
int gam_gpu_ensemble_create(gam_ensemble_t** e, gam_gpu_t* const* members, int n);
/* nsteps batch steps; returns the worst member status (GAM_ERR_NAN before GAM_ERR_DT_COLLAPSE) */
int gam_gpu_ensemble_run_steps(gam_ensemble_t* e, int nsteps);
/* the same, with the device time of the batch steps (ms) from CUDA events on the ensemble stream */
int gam_gpu_ensemble_run_steps_timed(gam_ensemble_t* e, int nsteps, double* ms);
/* advance until every member's Model%t >= tEnd (members drop out as they get there; the host checks
 * every `chunk` batch steps, so a member may take up to chunk-1 steps past tEnd, of the tiny dt CalcDT
 * gives once t reaches the member's tFin) or maxSteps batch steps; *steps = batch steps taken */
int gam_gpu_ensemble_advance(gam_ensemble_t* e, double tEnd, int chunk, int maxSteps, int* steps);
void gam_gpu_ensemble_destroy(gam_ensemble_t* e);   /* the members are not destroyed */
/* Tile shapes. GAM_TILE_FLUX_ROWS: rows of interfaces per flux-kernel CTA, 8 (default) or 4; results do
 * not depend on it. The ensemble autotuner times whole batch steps for each member shape (largest first)
 * with each height and keeps the fastest, then times per-member flux launches against the tile queue
 * (gam_gpu_ensemble_set_queue) and keeps the faster (the timed steps are ordinary steps of the run);
 * fluxRows (optional, one per member) and queue (optional) receive the choices. */
/* Tile queue: with on = 1 every batch step runs the members' predictor and E field as concurrent branches,
 * then ONE persistent flux kernel whose CTAs take tiles of every member and direction from a shared
 * counter, then the rest of each member's step as branches (on = 0: each member launches its own flux
 * kernels). Results do not depend on it. */
int gam_gpu_ensemble_set_queue(gam_ensemble_t* e, int on);
#define GAM_TILE_FLUX_ROWS 1
/* GAM_TILE_FUSED_UPDATE: 1 (default) the update kernel computes Flux2Deltas itself; 0 keeps the separate
 * Flux2Deltas kernel, whose dGasH/dGasM planes gam_gpu_fetch can then read. Results do not depend on it. */
#define GAM_TILE_FUSED_UPDATE 2
/* GAM_TILE_TMA: 1 (default) the flux and E-field kernels stage their stencil footprints with
 * tensor-memory-accelerator copies (cp.async.bulk.tensor, one thread per tile); 0 with per-element
 * cp.async. Results do not depend on it. */
#define GAM_TILE_TMA 3
/* GAM_TILE_STAGE_WAIT: 1 (default) the flux and E-field kernels wait for their staged tile up to a bound of
 * 2^20 mbarrier polls; 0 makes that wait give up at once. Either way a CTA whose wait gave up still waits
 * (with a far larger bound) for its own tensor copies to land before it exits, writes nothing, and the step
 * returns GAM_ERR_TIMEOUT. Setting 0 exercises a host's handling of that error without a hung GPU; the
 * state of that step is not valid. */
#define GAM_TILE_STAGE_WAIT 4
int gam_gpu_set_tile(gam_gpu_t* h, int what, int value);
int gam_gpu_ensemble_autotune(gam_ensemble_t* e, int steps, int* fluxRows, int* queue);

/* DivB for callers that cannot allocate device memory. This entry point has no counterpart in the
 * reference; its formula is the reference's DivB (src/gamera/gridutils.F90:717-770).
 * Some hosts cannot call cudaMalloc: device arrays owned by another runtime (OpenACC or CUDA Fortran
 * data regions, a coupler's memory pool) or code running where an allocation would synchronise the
 * device or upset its memory accounting. This entry point needs no handle and allocates nothing: it
 * reads magflux_dev, a device copy of State%magFlux in the Fortran layout (Ni+1,Nj+1,Nk+1,3) with
 * Ni = Nip+2*nG etc., and bflux0_dev, a device copy of Grid%bFlux0 (Ni,Nj,Nk,3) for a problem with a
 * background field (Model%doBackground) or NULL without one, and writes the sum over active cells of
 * |net face flux| (magFlux plus bFlux0, as DivB sums it with doTot) to the device double *tot_dev. Its
 * only scratch is a file-scope device array sized for GAM_DIVB_NOALLOC_MAX_CELLS active cells (512 KiB
 * per GPU that loads the library, held until exit); larger grids are rejected with GAM_ERR_ARG. The
 * first call on a device looks up that array's device address, so make it before capturing a stream;
 * the address is kept until exit, so the entry point is not for use on a device after cudaDeviceReset.
 * Kernels run on the legacy default stream; synchronise before reading *tot_dev. A CUDA error already
 * pending when it is called is returned as GAM_ERR_CUDA (and left pending) and nothing is launched. All
 * calls share the scratch array, so calls that overlap on the GPU (from several host threads or
 * streams) race. */
#define GAM_DIVB_NOALLOC_MAX_CELLS (256LL * 256LL * 256LL)
int gam_divb_noalloc(const double* magflux_dev, const double* bflux0_dev, int Nip, int Njp, int Nkp, int nG,
                     double* tot_dev);
/* ---- tiled runs: one problem split along k into tiles (src/gamera/mpi/gamapp_mpi.F90) ----
 * A tile is a handle created for its k range (its corners with 4 ghost layers of the global grid)
 * with GAM_BC_HALO on every k face that borders another tile (both k faces of every tile when the
 * global K boundary is periodic). Tiles need the same Nip and Njp and at least 4 active k cells. */
typedef struct gam_tiles gam_tiles_t;

/* All tiles in this process, ordered along k, on one GPU or on GPUs with peer access. Fills the tiles'
 * halos of State and oState (Bxyz included) from their neighbours and sets every tile's dt to the
 * minimum over the tiles, as Hatch_mpi leaves a decomposed problem. The tiles stay owned by the caller
 * and are stepped only through the group from then on. Replaces: Hatch_mpi's halo set-up and
 * CalcDT_mpi (gamapp_mpi.F90:79-497, :501-518). */
int gam_tiles_create(gam_tiles_t** g, gam_gpu_t* const* tiles, int n, int periodicK);
/* nsteps of stepGamera_mpi (gamapp_mpi.F90:665-692) over all tiles; returns the worst status */
int gam_tiles_run_steps(gam_tiles_t* g, int nsteps);
int gam_tiles_run_steps_timed(gam_tiles_t* g, int nsteps, double* ms);
void gam_tiles_destroy(gam_tiles_t* g);   /* the tiles are not destroyed */

/* One process per GPU: the pieces of stepGamera_mpi for a host that moves the halos itself (NCCL
 * send/recv, MPI). All work is enqueued on the handle's stream (gam_gpu_stream). The dt words are
 * two 64-bit integers in device memory; the host reduces them with MIN over the tiles between
 * gam_gpu_step_local and gam_gpu_step_bcs (one all-reduce replaces CalcDT_mpi's MPI_AllReduce,
 * gamapp_mpi.F90:501-518). A step is:
 *   step_local(words) ; allreduce MIN(words) ; step_bcs(words) ;
 *   halo_pack(side 0 and 1, GAM_HALO_STATE) ; exchange ; halo_unpack(side 0 and 1) ; step_ghosts
 * where side 0 is the lower k neighbour, side 1 the upper, and the message packed for side s is the one
 * the neighbour there unpacks on side 1-s. Initial set-up: halo_pack/unpack with
 * GAM_HALO_STATE|GAM_HALO_OSTATE|GAM_HALO_BXYZ, then calcdt_local ; allreduce ; calcdt_finish.
 * Replaces: haloUpdate and updateMpiBCs (gamapp_mpi.F90:579-663, :694-794). */
#define GAM_HALO_STATE 1u      /* State (between step_bcs and step_ghosts: the new state)            */
#define GAM_HALO_OSTATE 2u     /* oState                                                             */
#define GAM_HALO_BXYZ 4u       /* include Bxyz (set-up only: a step recomputes the halo's Bxyz)       */
int gam_gpu_stream(gam_gpu_t* h, void** stream);   /* the cudaStream_t the handle enqueues on */
int gam_gpu_step_local(gam_gpu_t* h, long long* dtWordsDev);
int gam_gpu_step_bcs(gam_gpu_t* h, const long long* dtWordsDev);
int gam_gpu_step_ghosts(gam_gpu_t* h);     /* completes the step; returns its status */
int gam_gpu_calcdt_local(gam_gpu_t* h, long long* dtWordsDev);
int gam_gpu_calcdt_finish(gam_gpu_t* h, const long long* dtWordsDev);
/* bytes of the message this tile sends to / receives from its neighbour on `side` */
int gam_gpu_halo_bytes(gam_gpu_t* h, int side, unsigned what, long long* sendBytes, long long* recvBytes);
int gam_gpu_halo_pack(gam_gpu_t* h, int side, unsigned what, void* dstDev);          /* 16-byte aligned */
int gam_gpu_halo_unpack(gam_gpu_t* h, int side, unsigned what, const void* srcDev);  /* 16-byte aligned */

/* ---- learned flux closure (no counterpart in the reference; the device analogue of its HackFlux hook,
 * src/base/types/gamtypes.F90:137-144) ----
 * A 3D convolution net over a grid's cells: 8 normalised primitives (rho, v, P, B) in, 4 layers of 3x3x3
 * kernels with 32 channels and GELU, 27 outputs = corrections to the 5 gas fluxes and the 3 magnetic-stress
 * momentum fluxes through each cell's lower I, J and K face (outputs 0..23, direction d and flux v at d*8+v),
 * then to the EMF on each cell's lower I, J and K edge (24..26). BF16 weights and activations, FP32
 * accumulation on the tensor cores (tcgen05); FP32 master weights and Adam moments. Parameters are
 * W[27][cout][cin] (tap = (di+1) + 3(dj+1) + 9(dk+1)) then b[cout], layer after layer. */
typedef struct gam_closure gam_closure_t;
int gam_closure_create(gam_closure_t** c, int Nip, int Njp, int Nkp, unsigned long long seed);
void gam_closure_destroy(gam_closure_t* c);
long long gam_closure_num_params(const gam_closure_t* c);
int gam_closure_set_params(gam_closure_t* c, const float* p, long long n);
int gam_closure_get_params(gam_closure_t* c, float* p, long long n);
int gam_closure_get_grads(gam_closure_t* c, float* g, long long n);
/* the net on host inputs (Ni,Nj,Nk,8), ghosts included, Fortran layout; out: (Nip,Njp,Nkp,27) */
int gam_closure_forward_host(gam_closure_t* c, const float* in, float* out);
/* parameter gradients (gam_closure_get_grads) of sum(out * gout) for gout (Nip,Njp,Nkp,27) */
int gam_closure_backward_host(gam_closure_t* c, const float* in, const float* gout);
/* normalisation: net input q = (primitive q - inMean[q]) / inScale[q] for rho, vx, vy, vz, P, Bx, By, Bz;
 * the face correction of flux v (rho, 3 momenta, energy, 3 magnetic-stress momenta) is the net output times
 * fluxScale[v] times the face area; the loss divides the residual of each gas variable by resScale[v] */
int gam_closure_set_norm(gam_closure_t* c, const float* inMean, const float* inScale, const float* fluxScale,
                         const float* resScale);
/* training data: n sample slots; a capture stores the net input from the coarse problem's State, takes one
 * plain coarse step (its dt as set) and stores the residual restrict(fine State) - coarse State of the
 * 5 gas variables. The fine problem has 2x the cells per direction and sits one coarse step later. */
int gam_closure_reserve(gam_closure_t* c, int n);
int gam_closure_capture(gam_closure_t* c, int slot, gam_gpu_t* coarse, gam_gpu_t* fine);
/* one Adam step per listed slot (forward, loss, backward through the network, Adam) on the loss
 * mean over active cells of sum_v ((dt/V * div(corrections)_v - residual_v) / resScale_v)^2 */
int gam_closure_train(gam_closure_t* c, const int* slots, int n, float lr, double* meanLoss);
int gam_closure_eval(gam_closure_t* c, const int* slots, int n, double* loss, double* lossNone);
/* rms over the active cells of a sample's residual per gas variable (rms[0..4]) and its dt (rms[5]) */
int gam_closure_residual_rms(gam_closure_t* c, int slot, double* rms);
/* EMF corrections (grids periodic in all three directions): the edge EMF of direction e gains net output 24+e
 * times emfScale[e] times the edge length, before E2Flux (so div B stays at round-off); the cell loss adds,
 * per face direction d, ((-dt curl(EMF corrections))_d - magnetic-flux residual_d) / resScaleB[d] squared over
 * the lower faces of the active cells. emfScale all zero (the default) turns both off. */
int gam_closure_set_norm_emf(gam_closure_t* c, const float* emfScale, const float* resScaleB);
/* rms over the lower faces of the active cells of a sample's magnetic-flux residual (restricted fine minus plain
 * coarse face flux), per face direction (rms[0..2]) */
int gam_closure_residual_rms_b(gam_closure_t* c, int slot, double* rms);
/* Face targets. After each fine step of a sample (reset = 1 on its first), add weight (that step's dt) times
 * the fine problem's interface fluxes, summed over the 2 x 2 fine sub-faces of every coarse face; the next
 * capture then also stores the face target: the accumulation over the coarse dt minus the plain coarse
 * step's flux, the correction that gives the coarse faces the restricted fine fluxes (exact for density and
 * momentum, whose updates are flux divergences). The fine problem must run FP64. */
int gam_closure_accum_fine(gam_closure_t* c, gam_gpu_t* fine, double weight, int reset);
/* the loss gam_closure_train and gam_closure_eval minimise: the cell residual (default) or, with
 * GAM_CLOSURE_LOSS_FACE, the mean over the lower faces of the active cells and the 24 outputs of
 * (output - target / (fluxScale[v] * area))^2 */
#define GAM_CLOSURE_LOSS_CELL 0
#define GAM_CLOSURE_LOSS_FACE 1
int gam_closure_set_loss(gam_closure_t* c, int mode);
/* a slot's face targets: rms[0..7] the rms of target / area per flux; rel[0..4] the relative rms mismatch
 * of dt / V * div(target) against the cell residual per gas variable */
int gam_closure_face_stats(gam_closure_t* c, int slot, double* rms, double* rel);
/* attach (c) or detach (NULL) the closure: every step adds its face corrections to the fluxes of State n
 * before Flux2Deltas; a step whose corrected update would make rho or P non-positive uses the plain
 * fluxes instead (counted by gam_gpu_closure_rejects). One handle per closure at a time. */
int gam_gpu_set_closure(gam_gpu_t* h, gam_closure_t* c);
/* The magnetosphere's hooks and gravity for a problem created with gam_gpu_create (its Grid and State as the
 * reference's Hatch leaves them: bc {GAM_BC_ION, GAM_BC_WIND, ...}, the cut-dipole background arrays and
 * gam_grid_c.xyz given): par = the GAM_NMSPH values of GAM_IC_MAGSPHERE. AddGrav runs on the device from the
 * grid's metrics. Replaces: initUser's hooks and Model%Phi of voltron/ICs/earthcmi.F90:150-177 for one problem
 * without ionospheric coupling. */
int gam_gpu_set_magnetosphere(gam_gpu_t* h, const double* par, int n);
int gam_gpu_closure_rejects(gam_gpu_t* h, int* n);
/* restriction of a fine problem's State (2x the cells per direction) into a coarse problem's State
 * (GAM_SYNC_STATE) or oState (GAM_SYNC_OSTATE): gas volume-weighted, magnetic fluxes summed per face
 * (divergence-free), then the coarse BCs and Bxyz */
int gam_gpu_restrict(gam_gpu_t* fine, gam_gpu_t* coarse, unsigned what);
/* Hatch's initial dt for a state placed with gam_gpu_sync_to_device: CalcDT, oState%time = time - dt */
int gam_gpu_init_dt(gam_gpu_t* h);

const char* gam_gpu_errstr(int code);

#ifdef __cplusplus
}
#endif
#endif /* GAMGPU_H */
