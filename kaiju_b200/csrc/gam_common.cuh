// Device-side layout, pointer bundles and per-cell arithmetic shared by the GAMERA step kernels.
//
// Layout in HBM. Every field -- cell-centred (Gas, Bxyz, volume, ...), face-centred (magFlux, face,
// Tf, ...) and edge-centred (Efld, edge, Te, Teb) -- lives in one "pencil" index space
//     at(i,j,k) = i + P*(j + Q*k),   0 <= i <= Ni, 0 <= j <= Nj, 0 <= k <= Nk,
// with i,j,k counted from the first ghost (Fortran isg,jsg,ksg), P = Ni+1 rounded up to 8 doubles
// (64-byte rows), Q = Nj+1, R = Nk+1. Cell arrays leave the last i/j/k slot unused. One index
// expression therefore addresses a cell, its lower faces and its lower edges, so a stencil along
// direction d is a fixed stride (1, P or P*Q) and every kernel reads i-contiguous, coalesced rows.
// Each vector component / variable is its own plane (structure of arrays), like the reference's
// Fortran arrays Gas(i,j,k,v), so host<->device mirroring is one strided copy per plane.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gam {

constexpr double TINY = 1.0e-12;   // kdefs.F90:23
constexpr double HUGEV = 1.0e12;
constexpr double PI = 3.14159265358979323846264338327950288;

enum { IDIR = 0, JDIR = 1, KDIR = 2 };
enum { RM_8CENT = 0, RM_7UP = 1 };
// BC_HALO: a face between two k-tiles of one problem; no physical BC runs there, its ghost layers are
// filled from the neighbouring tile after the step (the reference's mpiNullBc_T, gamapp_mpi.F90:428-463)
// BC_ION / BC_WIND: the magnetosphere's ionospheric inner and solar-wind outer I boundaries (gam_msph.cu)
enum { BC_PERIODIC = 0, BC_ZEROGRAD = 1, BC_LFMPOLE = 2, BC_LFMBW = 3, BC_HALO = 4, BC_ION = 5, BC_WIND = 6 };

// The magnetosphere problem (voltron/ICs/earthcmi.F90 initUser with a constant solar wind and no
// ionospheric coupling), code units: the wind, PushIon's coupling time, NudgeSW's time unit, gravity
struct MsphPar {
    int on;
    double wD, wP, wV[3], wB[3];   // the solar wind
    double dtCpl, gT0;             // ibc dtCpl; the time unit in seconds
    int nIonP, doIonPush;
    int doGrav;                    // gravitational acceleration planes present (AddGrav)
};

struct Lay {
    int Nip, Njp, Nkp;     // active cells
    int nG;                // ghosts per side
    int Ni, Nj, Nk;        // cells including ghosts
    int P, Q, R;           // pencil extents (P padded)
    long long E;           // elements per plane = P*Q*R
    __host__ __device__ long long at(int i, int j, int k) const { return i + (long long)P * (j + (long long)Q * k); }
    __host__ __device__ long long stride(int d) const { return d == 0 ? 1 : (d == 1 ? (long long)P : (long long)P * Q); }
    __host__ __device__ int is() const { return nG; }
    __host__ __device__ int ie() const { return nG + Nip - 1; }
    __host__ __device__ int js() const { return nG; }
    __host__ __device__ int je() const { return nG + Njp - 1; }
    __host__ __device__ int ks() const { return nG; }
    __host__ __device__ int ke() const { return nG + Nkp - 1; }
};

// Model scalars that stay constant across a run (init.F90:312-492 defaults, overridable)
struct Par {
    double gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, dFloor, pFloor, limDT0, tFin;
    int doMHD, doBoris, do25D, doLFMLim, rmeth, fixedTimestep;
    int doBackground;      // background field B0 present (Model%doBackground)
    int bc[6];
    int doRing, ringDoS, ringDoE;   // ring averaging about the LFM axis (Model%doRing, Ring%doS/doE)
    int predFixLFM;                 // the LFM blast wave's predictor fix
    int dtActive;                   // CalcDT over the active cells only
    double bwD0, bwP0;              // gas of the LFM blast wave's fixed shells
    // mbarrier polls before the flux and E-field kernels' wait on their staged tile gives up (GAM_TILE_STAGE_WAIT;
    // default STAGE_WAIT). After giving up a CTA still waits, with the far larger STAGE_DRAIN bound, for its own
    // copies to land before it exits, and the step reports GAM_ERR_TIMEOUT.
    unsigned int stageWait;
    MsphPar msph;
};
constexpr unsigned int STAGE_WAIT = 1u << 20;
constexpr unsigned int STAGE_DRAIN = 1u << 28;

// Time-dependent scalars kept on the device so a whole step can be captured and replayed.
struct Scal {
    double t, dt, dt0, time, otime;   // Model%t, Model%dt, Model%dt0, State%time, oState%time
    double pdt, odt;                  // predictor half-step and state separation of this step
    unsigned long long dtMinBits;     // running min of CellDT (bit pattern of a non-negative double)
    unsigned int nanCount;            // cells whose CellDT was NaN
    int ts;
    int status;                       // status bits of the last CalcDT (1 disaster, 2 bad, 4 NaN, 8 wait gave up)
    int sticky;                       // OR of status over steps since the last reset
    unsigned int lastNan;             // nanCount of the last CalcDT
    int pad;
    // tiled runs: {dtMinBits, ~nanCount} of this tile, reduced with MIN across the tiles (so the second
    // word carries the largest NaN count) before the dt is finalized
    unsigned long long red[2];
    // learned closure: 1 when this step's corrected update failed positivity and the plain fluxes were used
    int closureReject;
    int closureRejects;               // steps that fell back, since the handle was created
    // nonzero once a kernel's bounded wait on its own asynchronous copies gave up (the step's results are
    // not valid); CalcDT reports it as status bit 8
    unsigned int waitFail;
};

// Device field bundle. Planes are contiguous arrays of Lay::E doubles.
struct StateP {
    double* gas[5];
    double* mf[3];
    double* b[3];
};

struct GridP {
    const double* volume;
    const double* xyzcc[3];
    const double* xfc[3][3];   // [dir][xyz]
    const double* di; const double* dj; const double* dk;
    const double* face[3];
    const double* edge[3];
    const double* Tf[3][9];    // [dir][component]
    const double* Te[3][9];
    const double* Teb[3][4];
    // background field (Grid_T fcB0, edgB0, B0, bFlux0, dpB0; gamtypes.F90:225-236); null without one
    const double* fcB0[3][3];  // [face dir][xyz] face-averaged B0
    const double* edgB0[3][2]; // [edge dir][tangent 1, 2] edge-averaged B0 in the edge frame
    const double* B0[3];       // cell-averaged B0
    const double* bFlux0[3];   // B0 flux through the lower faces
    const double* dpB0[3];     // -div(B0 Maxwell stress)/volume, the background momentum source
};

// ------------------------------------------------------------------------------------------------ helpers
__device__ __forceinline__ double sq(double x) { return x * x; }
__device__ __forceinline__ double fsign1(double b) { return copysign(1.0, b); }
__device__ __forceinline__ double dmax(double a, double b) { return (a > b) ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return (a < b) ? a : b; }

// recon.F90:22-32 -- weights are integer/840 (exact sum 1) and integer/420
__device__ __forceinline__ double wC8(int n) {
    const double c[8] = {-3.0 / 840.0, 29.0 / 840.0, -139.0 / 840.0, 533.0 / 840.0,
                         533.0 / 840.0, -139.0 / 840.0, 29.0 / 840.0, -3.0 / 840.0};
    return c[n];
}
__device__ __forceinline__ double wU7(int n) {
    const double c[7] = {-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0, 319.0 / 420.0, 214.0 / 420.0, -38.0 / 420.0, 4.0 / 420.0};
    return c[n];
}

// Cell conversions (gamutils.F90:301-321, 362-383). Where the reference divides several values by the same
// density or volume, one reciprocal serves them all here (FP64 divisions are long instruction sequences;
// the results differ by an ulp or so).
__device__ __forceinline__ void cellC2P(const Par& p, const double* Con, double* Prim) {
    double rho = Con[0], ir = 1.0 / rho;
    double Vx = Con[1] * ir, Vy = Con[2] * ir, Vz = Con[3] * ir;
    double KinE = 0.5 * rho * (sq(Vx) + sq(Vy) + sq(Vz));
    Prim[0] = dmax(rho, p.dFloor);
    Prim[1] = Vx; Prim[2] = Vy; Prim[3] = Vz;
    Prim[4] = dmax((p.gamma - 1) * (Con[4] - KinE), p.pFloor);
}
__device__ __forceinline__ void cellP2C(const Par& p, const double* Prim, double* Con) {
    double rho = dmax(Prim[0], p.dFloor);
    double IntE = dmax(Prim[4], p.pFloor) / (p.gamma - 1);
    double KinE = 0.5 * rho * (sq(Prim[1]) + sq(Prim[2]) + sq(Prim[3]));
    Con[0] = rho; Con[1] = rho * Prim[1]; Con[2] = rho * Prim[2]; Con[3] = rho * Prim[3]; Con[4] = IntE + KinE;
}
// BlockCon2Prim (recon.F90:66-92): density floored first, kinetic energy from momenta
__device__ __forceinline__ void blockC2P(const Par& p, const double* Con, double* W) {
    double D = dmax(Con[0], p.dFloor), iD = 1.0 / D;
    double KinE = 0.5 * (sq(Con[1]) + sq(Con[2]) + sq(Con[3])) * iD;
    double P = dmax((p.gamma - 1) * (Con[4] - KinE), p.pFloor);
    W[0] = D; W[1] = Con[1] * iD; W[2] = Con[2] * iD; W[3] = Con[3] * iD; W[4] = P;
}

// The limiter's max and min: a > b ? a : b and a < b ? a : b. In single precision fmaxf/fminf, one instruction
// each and the same value for every non-NaN input (the FP32 flux kernel measured 1-3% faster); in double
// precision the comparisons measured faster than fmax/fmin.
template <typename T> __device__ __forceinline__ T lmax(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T lmin(T a, T b) { return a < b ? a : b; }
template <> __device__ __forceinline__ float lmax<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ float lmin<float>(float a, float b) { return fminf(a, b); }

// pdmLR (recon.F90:231-272) on one interface
template <typename T>
__device__ __forceinline__ void pdmLR(T pdmb, T v0, T v1, T v2, T v3, T Qi, T& Ql, T& Qr) {
    T maxV = lmax(v1, v2), minV = lmin(v1, v2);
    T c = lmin(Qi, maxV);
    T vN = lmax(minV, c);
    T dv0 = pdmb * (v1 - v0), dv1 = pdmb * (v2 - v1), dv2 = pdmb * (v3 - v2);
    T s0 = copysign(T(1), dv0), s1 = copysign(T(1), dv1), s2 = copysign(T(1), dv2);
    T q0 = fabs(s0 + s1), q1 = fabs(s1 + s2);
    T dvL = vN - v1, dvR = v2 - vN;
    T aL = fabs(dvL) - q0 * fabs(dv0), aR = fabs(dvR) - q1 * fabs(dv2);
    Ql = vN - s1 * lmax(T(0), aL);
    Qr = vN + s1 * lmax(T(0), aR);
}
// PDM (recon.F90:275-301)
template <typename T>
__device__ __forceinline__ T PDM(T pdmb, T q0, T q1, T q2, T qI) {
    T maxQ = lmax(q1, q2), minQ = lmin(q1, q2);
    T c = lmin(qI, maxQ);
    T qN = lmax(minQ, c);
    T dq0 = pdmb * (q1 - q0), dq1 = pdmb * (q2 - q1);
    T s0 = copysign(T(1), dq0), s1 = copysign(T(1), dq1);
    T s01 = fabs(s0 + s1);
    T dqL = qN - q1;
    T a = fabs(dqL) - s01 * fabs(dq0);
    return qN - s1 * lmax(T(0), a);
}

// GetLRs on one interface: dV[8] volumes, Q[8] values (stencil cells f-4..f+3), nQ[4] limiter values
// (cells f-2..f+1), iVi = 1 / Central8(dV): the reference divides each variable's sum by Central8(dV);
// here one reciprocal per interface serves all of them (the results differ by an ulp or so).
// Cen8LRs (recon.F90:125-158) or Up7LRs (:162-198).
template <typename T>
__device__ __forceinline__ void getLR(int rmeth, T pdmb, const T* dV, const T* Q, const T* nQ, T iVi, T& Ql, T& Qr) {
    T QdV[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) QdV[n] = dV[n] * Q[n];
    if (rmeth == RM_8CENT) {
        T s = T(0);
#pragma unroll
        for (int n = 0; n < 8; ++n) s = s + T(wC8(n)) * QdV[n];
        T Qi = s * iVi;
        pdmLR<T>(pdmb, nQ[0], nQ[1], nQ[2], nQ[3], Qi, Ql, Qr);
    } else {
        T l = QdV[0] * T(wU7(0)) + QdV[1] * T(wU7(1)) + QdV[2] * T(wU7(2)) + QdV[3] * T(wU7(3)) +
              QdV[4] * T(wU7(4)) + QdV[5] * T(wU7(5)) + QdV[6] * T(wU7(6));
        T r = QdV[7] * T(wU7(0)) + QdV[6] * T(wU7(1)) + QdV[5] * T(wU7(2)) + QdV[4] * T(wU7(3)) +
              QdV[3] * T(wU7(4)) + QdV[2] * T(wU7(5)) + QdV[1] * T(wU7(6));
        Ql = PDM<T>(pdmb, nQ[0], nQ[1], nQ[2], l * iVi);
        Qr = PDM<T>(pdmb, nQ[3], nQ[2], nQ[1], r * iVi);
    }
}

// Cen8LRs with the stencil weights already applied to the volumes: c8[n] = w8[n] * dV[n], shared by all the
// variables of an interface (the reference weights dV[n] * Q[n] per variable), iVi = 1 / sum(c8)
template <typename T>
__device__ __forceinline__ void getLR8(T pdmb, const T* c8, const T* Q, const T* nQ, T iVi, T& Ql, T& Qr) {
    T s = T(0);
#pragma unroll
    for (int n = 0; n < 8; ++n) s = s + c8[n] * Q[n];
    pdmLR<T>(pdmb, nQ[0], nQ[1], nQ[2], nQ[3], s * iVi, Ql, Qr);
}

template <typename T>
__device__ __forceinline__ T central8(const T* q) {
    T s = T(0);
#pragma unroll
    for (int n = 0; n < 8; ++n) s = s + T(wC8(n)) * q[n];
    return s;
}

// gamCellBxyz (gridutils.F90:648-680): second-order cell field from the six face fluxes
__device__ __forceinline__ void cellBxyz(const Lay& L, const GridP& g, double* const* mf, long long c, double* B) {
    double idV = 1.0 / g.volume[c];
    double fI = mf[0][c], fJ = mf[1][c], fK = mf[2][c];
    long long ci = c + 1, cj = c + L.P, ck = c + (long long)L.P * L.Q;
    double fIp = mf[0][ci], fJp = mf[1][cj], fKp = mf[2][ck];
    double Div = fIp - fI + fJp - fJ + fKp - fK;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        double b = (fIp * g.xfc[0][x][ci] + fJp * g.xfc[1][x][cj] + fKp * g.xfc[2][x][ck] - fI * g.xfc[0][x][c] -
                    fJ * g.xfc[1][x][c] - fK * g.xfc[2][x][c]) * idV;
        B[x] = b - Div * g.xyzcc[x][c] * idV;
    }
}

}  // namespace gam
