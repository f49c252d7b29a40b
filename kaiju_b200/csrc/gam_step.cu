// GAMERA ideal-MHD step on sm_100a: predictor, constrained-transport E field, interface fluxes,
// update, CFL dt and boundary conditions. One stepGamera (src/gamera/gamapp.F90:73-94) is a fixed
// sequence of kernels on one stream; with the time scalars on the device the sequence is captured
// once per buffer parity as a CUDA graph and replayed.
//
// The flux and E-field kernels compute the reconstruction, limiter and kinetic fluxes in the
// arithmetic type T (double for the plain path, float for the FP32-flux path); state, accumulation,
// CT update, C2P with floors and the dt reduction stay FP64 in both.
#include <cstdio>
#include <cmath>
#include <nvtx3/nvToolsExt.h>
#include "gam_common.cuh"
#include "gam_step.cuh"
#include "gam_lfm.cuh"
#include "gam_kern.cuh"

namespace gam {

// ================================================================================ step scalars
// AdvanceMHD trap (mhdgroup.F90:26-28) and the predictor time factors (:459)
__global__ void k_step_begin(Scal* sc) {
    if (fabs(sc->otime - sc->time) < TINY) sc->otime = sc->time - sc->dt;
    sc->pdt = 0.5 * sc->dt;
    sc->odt = sc->time - sc->otime;
    sc->dtMinBits = 0x7FF0000000000000ull;  // +inf
    sc->nanCount = 0u;
    sc->closureReject = 0;
}

// ================================================================================ predictor
// Predictor magFlux part (mhdgroup.F90:466-488): AB2 on every face element, ghosts included. Also the
// per-face values EdgeLRs divides out at every stencil point (fields.F90:335-336): flux/max(area,TINY)
// for the half state (reconstruction) and for the limiting state.
struct F32FaceOut { float* hbA[3]; float* nbA[3]; };
struct F32CellOut { float* Wh[5]; float* Wn[5]; float* hb[3]; float* nb[3]; float* rho; float* VdV[3]; };

// Two consecutive face elements per thread with 16-byte loads and stores (E = P*Q*R is a multiple of 8 and
// every plane starts 16-byte aligned), twice the bytes in flight per thread of a one-element loop; the
// arithmetic per element is unchanged.
__global__ void k_predict_faces(long long E, Par p, GridP g, Vec3P mf, Vec3P omf, Vec3P hmf, Vec3P hbA, Vec3P nbA,
                                F32FaceOut o, const Scal* sc) {
    long long l = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
    if (l >= E) return;
    const double pdt = sc->pdt, iodt = 1.0 / sc->odt;   // reciprocals where the reference divides repeatedly
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double2 Q2 = *reinterpret_cast<const double2*>(mf.v[c] + l);
        const double2 oQ2 = *reinterpret_cast<const double2*>(omf.v[c] + l);
        const double2 a2 = *reinterpret_cast<const double2*>(g.face[c] + l);
        double H[2], hb[2], nb[2];
        const double Q[2] = {Q2.x, Q2.y}, oQ[2] = {oQ2.x, oQ2.y}, A[2] = {a2.x, a2.y};
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            double dQ = (Q[e] - oQ[e]) * iodt;
            H[e] = Q[e] + pdt * dQ;
            const double ia = 1.0 / dmax(A[e], TINY);
            hb[e] = H[e] * ia;
            nb[e] = (p.doLFMLim ? Q[e] : H[e]) * ia;
        }
        // the half-state flux: bFlux2Fld of the half state reads it
        *reinterpret_cast<double2*>(hmf.v[c] + l) = make_double2(H[0], H[1]);
        if (o.hbA[0]) {
            *reinterpret_cast<float2*>(o.hbA[c] + l) = make_float2(float(hb[0]), float(hb[1]));
            *reinterpret_cast<float2*>(o.nbA[c] + l) = make_float2(float(nb[0]), float(nb[1]));
        } else {
            *reinterpret_cast<double2*>(hbA.v[c] + l) = make_double2(hb[0], hb[1]);
            *reinterpret_cast<double2*>(nbA.v[c] + l) = make_double2(nb[0], nb[1]);
        }
    }
}

// bFlux2Fld of the half state + PredictCell (mhdgroup.F90:492-518, 529-563) on every cell, plus the
// BlockCon2Prim primitives of the half state and of state n used by the interface reconstruction.
__global__ void k_predict_cells(Lay L, Par p, GridP g, StateP n, StateP o, StateP h, PrimP Wh, PrimP Wn, Vec3P VdV,
                                F32CellOut f, const Scal* sc) {
    Reg r = {0, L.Ni, 0, L.Nj, 0, L.Nk};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    double B[3] = {0.0, 0.0, 0.0};
    const bool f32 = f.Wh[0] != nullptr;
    cellBxyz(L, g, h.mf, c, B);
    if (!f32) { h.b[0][c] = B[0]; h.b[1][c] = B[1]; h.b[2][c] = B[2]; }
    double Q[5], oQ[5], W[5], oW[5], pW[5], pQ[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) { Q[v] = n.gas[v][c]; oQ[v] = o.gas[v][c]; }
    cellC2P(p, oQ, oW);
    cellC2P(p, Q, W);
    double pdt = sc->pdt, iodt = 1.0 / sc->odt;
#pragma unroll
    for (int v = 0; v < 5; ++v) { double dQ = (W[v] - oW[v]) * iodt; pW[v] = W[v] + pdt * dQ; }
    pW[0] = dmax(pW[0], p.dFloor);
    pW[4] = dmax(pW[4], p.pFloor);
    cellP2C(p, pW, pQ);
    // the FP32-flux path keeps the half state as floats only; the double gas half state feeds its
    // Boris flux correction
    if (!f32 || p.doBoris) {
#pragma unroll
        for (int v = 0; v < 5; ++v) h.gas[v][c] = pQ[v];
    }
    // Mom2Face summand VolB*MomB/max(DenB,dFloor) (fields.F90:265-271), a pointwise cell value
    {
        double vol = g.volume[c], iden = 1.0 / dmax(pQ[0], p.dFloor);
        double v0 = vol * pQ[1] * iden, v1 = vol * pQ[2] * iden, v2 = vol * pQ[3] * iden;
        if (f32) { f.VdV[0][c] = float(v0); f.VdV[1][c] = float(v1); f.VdV[2][c] = float(v2); }
        else { VdV.v[0][c] = v0; VdV.v[1][c] = v1; VdV.v[2][c] = v2; }
    }
    double w[5];
    if (f32) {   // FP32-flux path: float copies of every stencil input
        blockC2P(p, pQ, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) f.Wh[v][c] = float(w[v]);
        blockC2P(p, Q, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) f.Wn[v][c] = float(w[v]);
#pragma unroll
        for (int x = 0; x < 3; ++x) { f.hb[x][c] = float(B[x]); f.nb[x][c] = float(n.b[x][c]); }
        f.rho[c] = float(pQ[0]);
        return;
    }
    blockC2P(p, pQ, w);
#pragma unroll
    for (int v = 0; v < 5; ++v) Wh.w[v][c] = w[v];
    blockC2P(p, Q, w);
#pragma unroll
    for (int v = 0; v < 5; ++v) Wn.w[v][c] = w[v];
}

// Flux2Deltas (stress.F90:150-196); O is the flux storage type (float on the FP32-flux path), the sums
// run in double
// Flux2Deltas of one active cell: dGasH (5) and dGasM (3). corr: the learned closure's face corrections
// (24 float planes: direction d, variable v at d*8+v; the 5 gas fluxes then the 3 magnetic-stress momentum
// fluxes), added to the face fluxes, or null.
template <typename O>
__device__ __forceinline__ void cellDeltas(const Lay& L, const Par& p, const GridP& g, const FluxOut<O>& FI,
                                           const FluxOut<O>& FJ, const FluxOut<O>& FK, const float* corr,
                                           long long c, double* dh, double* dm) {
    long long cj = c + L.P, ck = c + (long long)L.P * L.Q;
    double idV = 1.0 / g.volume[c];
    auto cr = [&](int d, int v, long long lo, long long hi) {
        if (!corr) return 0.0;
        const float* q = corr + (long long)(d * 8 + v) * L.E;
        return double(q[lo]) - double(q[hi]);
    };
#pragma unroll
    for (int v = 0; v < 5; ++v)
        dh[v] = (double(FI.g[v][c]) - double(FI.g[v][c + 1]) + double(FJ.g[v][c]) - double(FJ.g[v][cj]) +
                 double(FK.g[v][c]) - double(FK.g[v][ck]) +
                 (cr(0, v, c, c + 1) + cr(1, v, c, cj) + cr(2, v, c, ck))) * idV;
    if (p.doMHD) {
#pragma unroll
        for (int x = 0; x < 3; ++x)
            dm[x] = (double(FI.m[x][c]) - double(FI.m[x][c + 1]) + double(FJ.m[x][c]) - double(FJ.m[x][cj]) +
                     double(FK.m[x][c]) - double(FK.m[x][ck]) +
                     (cr(0, 5 + x, c, c + 1) + cr(1, 5 + x, c, cj) + cr(2, 5 + x, c, ck))) * idV;
        if (p.doBackground) {   // background momentum source (stress.F90:185-188)
#pragma unroll
            for (int x = 0; x < 3; ++x) dm[x] = dm[x] + g.dpB0[x][c];
        }
    }
}

// Flux2Deltas (stress.F90:150-196) into the dGasH/dGasM planes; O is the flux storage type (float on the
// FP32-flux path), the sums run in double. With cond set the kernel runs only when the closure's
// positivity check rejected this step (the plain fallback).
template <typename O>
__global__ void k_flux2deltas(Lay L, Par p, GridP g, FluxOut<O> FI, FluxOut<O> FJ, FluxOut<O> FK, PrimP dGH,
                              Vec3P dGM, const float* corr, const Scal* cond) {
    if (cond && !cond->closureReject) return;
    Reg r = {L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    double dh[5], dm[3] = {0.0, 0.0, 0.0};
    cellDeltas<O>(L, p, g, FI, FJ, FK, corr, c, dh, dm);
#pragma unroll
    for (int v = 0; v < 5; ++v) dGH.w[v][c] = dh[v];
    if (p.doMHD) {
#pragma unroll
        for (int x = 0; x < 3; ++x) dGM.v[x][c] = dm[x];
    }
}

// ================================================================================ update
// E2Flux (fields.F90:18-51) on the active faces; every other face element carries State n over
// (the reference updates State in place after copying it to oState).
__global__ void k_e2flux(Lay L, Par p, Vec3P E, StateP nS, StateP oNew, const Scal* sc) {
    Reg r = {0, L.Ni + 1, 0, L.Nj + 1, 0, L.Nk + 1};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    double m0 = nS.mf[0][c], m1 = nS.mf[1][c], m2 = nS.mf[2][c];
    bool act = p.doMHD && i >= L.is() && i <= L.ie() + 1 && j >= L.js() && j <= L.je() + 1 && k >= L.ks() &&
               k <= L.ke() + 1;
    if (act) {
        double dt = sc->dt;
        long long cj = c + L.P, ck = c + (long long)L.P * L.Q;
        const double* Ei = E.v[0]; const double* Ej = E.v[1]; const double* Ek = E.v[2];
        double dfi = Ek[cj] - Ek[c] - Ej[ck] + Ej[c];
        double dfj = Ei[ck] - Ei[c] - Ek[c + 1] + Ek[c];
        double dfk = Ej[c + 1] - Ej[c] - Ei[cj] + Ei[c];
        m0 = m0 - dt * dfi;
        m1 = m1 - dt * dfj;
        m2 = m2 - dt * dfk;
    }
    oNew.mf[0][c] = m0; oNew.mf[1][c] = m1; oNew.mf[2][c] = m2;
}

__global__ void k_bflux2fld(Lay L, GridP g, StateP s) {
    Reg r = {0, L.Ni, 0, L.Nj, 0, L.Nk};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    double B[3];
    cellBxyz(L, g, s.mf, c, B);
    s.b[0][c] = B[0]; s.b[1][c] = B[1]; s.b[2][c] = B[2];
}
__global__ void k_copy_b(Lay L, StateP src, StateP dst) {
    long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (l >= L.E) return;
    dst.b[0][l] = src.b[0][l]; dst.b[1][l] = src.b[1][l]; dst.b[2][l] = src.b[2][l];
}

__device__ __forceinline__ void normVec3(const double* a, double* o) {
    double nA = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    if (nA <= TINY) { o[0] = o[1] = o[2] = 0.0; }
    else { o[0] = a[0] / nA; o[1] = a[1] / nA; o[2] = a[2] / nA; }
}
// CellBoris (mhdgroup.F90:337-390), single fluid
__device__ void cellBoris(const Par& p, double* U2, const double* U0, const double* B2, const double* B0,
                          const double* dGH, const double* dGM, double dt) {
    double W2[5];
    cellC2P(p, U2, W2);
    double D2 = dmax(W2[0], p.dFloor), P2 = dmax(W2[4], p.pFloor);
    double D0 = dmax(U0[0], p.dFloor);
    double V0[3] = {U0[1] / D0, U0[2] / D0, U0[3] / D0};
    double B1[3] = {0.5 * (B2[0] + B0[0]), 0.5 * (B2[1] + B0[1]), 0.5 * (B2[2] + B0[2])};
    double Ca = p.Ca;
    double alpha = (B1[0] * B1[0] + B1[1] * B1[1] + B1[2] * B1[2]) / (D2 * Ca * Ca);
    double dRho = dt * dGH[0];
    double dPGas[3], dPMag[3], dMom[3];
    for (int c = 0; c < 3; ++c) { dPGas[c] = dt * dGH[1 + c]; dPMag[c] = dt * dGM[c]; }
    double pCon = 1.0 / (1.0 + alpha);
    double bh[3];
    normVec3(B1, bh);
    if (alpha > TINY) {
        double s[3] = {dPGas[0] + dPMag[0], dPGas[1] + dPMag[1], dPGas[2] + dPMag[2]};
        double pg = dPGas[0] * bh[0] + dPGas[1] * bh[1] + dPGas[2] * bh[2];
        double ps = s[0] * bh[0] + s[1] * bh[1] + s[2] * bh[2];
        double pv = V0[0] * bh[0] + V0[1] * bh[1] + V0[2] * bh[2];
        for (int c = 0; c < 3; ++c) {
            double para = pg * bh[c];
            double perpS = s[c] - ps * bh[c];
            double perpV = V0[c] - pv * bh[c];
            dMom[c] = (para + pCon * perpS) + alpha * pCon * dRho * perpV;
        }
    } else {
        for (int c = 0; c < 3; ++c) dMom[c] = dPGas[c] + dPMag[c];
    }
    double Wn[5] = {D2, (D0 * V0[0] + dMom[0]) / D2, (D0 * V0[1] + dMom[1]) / D2, (D0 * V0[2] + dMom[2]) / D2, P2};
    cellP2C(p, Wn, U2);
}

// CellReynolds + CellMaxwell/CellBoris (mhdgroup.F90:113-126, 170-197, 263-330) on active cells;
// ghost cells carry State n over.
// FUSED: the deltas are computed here from the face fluxes (Flux2Deltas of the same cell, same arithmetic)
// instead of read from the dGasH/dGasM planes
template <typename O, bool FUSED>
__global__ void k_update_gas(Lay L, Par p, GridP g, StateP nS, StateP oNew, PrimP dGH, Vec3P dGM, FluxOut<O> FI,
                             FluxOut<O> FJ, FluxOut<O> FK, const Scal* sc) {
    Reg r = {0, L.Ni, 0, L.Nj, 0, L.Nk};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    long long c = L.at(i, j, k);
    double U[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) U[v] = nS.gas[v][c];
    bool act = i >= L.is() && i <= L.ie() && j >= L.js() && j <= L.je() && k >= L.ks() && k <= L.ke();
    if (act) {
        double dt = sc->dt;
        double dh[5], dm[3] = {0.0, 0.0, 0.0};
        if (FUSED) cellDeltas<O>(L, p, g, FI, FJ, FK, nullptr, c, dh, dm);
        else {
#pragma unroll
            for (int v = 0; v < 5; ++v) dh[v] = dGH.w[v][c];
            if (p.doMHD) { dm[0] = dGM.v[0][c]; dm[1] = dGM.v[1][c]; dm[2] = dGM.v[2][c]; }
        }
        double U0[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) { U0[v] = U[v]; U[v] = U[v] + dt * dh[v]; }
        if (p.doMHD) {
            double dPm[3] = {dm[0], dm[1], dm[2]};
            if (p.doBoris) {
                double B2[3] = {oNew.b[0][c], oNew.b[1][c], oNew.b[2][c]};
                double B0[3] = {nS.b[0][c], nS.b[1][c], nS.b[2][c]};
                if (p.doBackground) {   // total fields (mhdgroup.F90:180-183)
#pragma unroll
                    for (int x = 0; x < 3; ++x) { B2[x] = B2[x] + g.B0[x][c]; B0[x] = B0[x] + g.B0[x][c]; }
                }
                cellBoris(p, U, U0, B2, B0, dh, dPm, dt);
            } else {
                double D = dmax(U[0], p.dFloor), Mx = U[1], My = U[2], Mz = U[3], TotE = U[4];
                const double iD = 1.0 / D;
                double KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) * iD;
                double P = dmax((p.gamma - 1) * (TotE - KinE), p.pFloor);
                Mx = Mx + dt * dPm[0];
                My = My + dt * dPm[1];
                Mz = Mz + dt * dPm[2];
                KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) * iD;
                U[0] = D; U[1] = Mx; U[2] = My; U[3] = Mz; U[4] = KinE + P / (p.gamma - 1);
            }
        }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) oNew.gas[v][c] = U[v];
}

// bFlux2Fld after EnforceBCs restricted to ghost cells: outside 2.5D the BCs only rewrite faces of
// ghost cells (outer I/J/K faces from ie+2/je+2/ke+2 on, inner ones below is/js/ks), so active cells
// keep the B of the update.
// The ghost cells are enumerated as five slabs so the launch covers only them: k below and above the active
// range (all i, j), then j below and above (all i, active k), then the i ghosts of the active rows (both
// ends of a row next to each other, so a warp reads whole ghost runs of neighbouring rows). i runs fastest
// in every slab.
__host__ __device__ inline long long ghost_cells(const Lay& L) {
    return (long long)L.Ni * L.Nj * L.Nk - (long long)L.Nip * L.Njp * L.Nkp;
}
__device__ __forceinline__ void ghost_ijk(const Lay& L, long long t, int& i, int& j, int& k) {
    const long long sK = (long long)L.Ni * L.Nj, sJ = (long long)L.Ni * L.Nkp;
    const long long nK = sK * (L.Nk - L.Nkp), nJ = sJ * (L.Nj - L.Njp);
    if (t < nK) {   // k slabs: whole (i, j) planes
        const int kk = (int)(t / sK), rem = (int)(t % sK);
        k = kk < L.ks() ? kk : L.ke() + 1 + (kk - L.ks());
        j = rem / L.Ni; i = rem % L.Ni;
        return;
    }
    t -= nK;
    if (t < nJ) {   // j slabs within the active k: whole rows
        const int jj = (int)(t / sJ), rem = (int)(t % sJ);
        j = jj < L.js() ? jj : L.je() + 1 + (jj - L.js());
        k = L.ks() + rem / L.Ni; i = rem % L.Ni;
        return;
    }
    t -= nJ;        // the i ghosts of the active rows: nGi = Ni - Nip cells per row
    const int nGi = L.Ni - L.Nip, ii = (int)(t % nGi), q = (int)(t / nGi);
    i = ii < L.is() ? ii : L.ie() + 1 + (ii - L.is());
    j = L.js() + q % L.Njp; k = L.ks() + q / L.Njp;
}
__global__ void k_bflux2fld_ghost(Lay L, GridP g, StateP s) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ghost_cells(L)) return;
    int i, j, k;
    ghost_ijk(L, t, i, j, k);
    long long c = L.at(i, j, k);
    double B[3];
    cellBxyz(L, g, s.mf, c, B);
    s.b[0][c] = B[0]; s.b[1][c] = B[1]; s.b[2][c] = B[2];
}

// ================================================================================ timestep
// CellDT (gridutils.F90:49-106) over the dt domain (one ghost layer at physical boundaries), min-reduced
// The dt domain: one ghost layer at physical boundaries (init.F90:531-537), the active cells with dtActive;
// a tile face has no ghost layer in it (ksDT = ks, keDT = ke; gamapp_mpi.F90:441-462)
__host__ __device__ inline Reg reg_dt(const Lay& L, const Par& p) {
    Reg r = {L.is() - 1, L.Nip + 2, L.js() - 1, L.Njp + 2, L.ks() - 1, L.Nkp + 2};
    if (p.dtActive) r = Reg{L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    if (!p.dtActive && p.bc[4] == BC_HALO) { r.k0 += 1; r.nk -= 1; }
    if (!p.dtActive && p.bc[5] == BC_HALO) r.nk -= 1;
    return r;
}

__global__ void k_calcdt(Lay L, Par p, GridP g, StateP s, Scal* sc) {
    const Reg r = reg_dt(L, p);
    int i, j, k;
    double dtijk = HUGEV * 2.0;
    bool isnan_ = false;
    if (reg_plane(r, i, j, k)) {
        long long c = L.at(i, j, k);
        double rho = s.gas[0][c], ir = 1.0 / rho;   // one reciprocal for the reference's divisions by rho
        double Vx = s.gas[1][c] * ir, Vy = s.gas[2][c] * ir, Vz = s.gas[3][c] * ir;
        double MagV = sqrt(sq(Vx) + sq(Vy) + sq(Vz));
        double ke = 0.5 * rho * sq(MagV);
        double e = s.gas[4][c] - ke;
        double P = (p.gamma - 1) * e;
        double Cs = sqrt(p.gamma * P * ir);
        double Valf = 0.0;
        if (p.doMHD) {
            double Bx = s.b[0][c], By = s.b[1][c], Bz = s.b[2][c];
            if (p.doBackground) { Bx = Bx + g.B0[0][c]; By = By + g.B0[1][c]; Bz = Bz + g.B0[2][c]; }  // gridutils.F90:82-86
            double MagB = sqrt(sq(Bx) + sq(By) + sq(Bz));
            Valf = MagB * rsq(rho);
            if (p.doBoris) Valf = p.Ca * Valf * rsq(p.Ca * p.Ca + Valf * Valf);
        }
        double vCFL = MagV + sqrt(sq(Cs) + sq(Valf)) + 0.0;
        double dl = g.di[c];
        if (g.dj[c] < dl) dl = g.dj[c];
        if (g.dk[c] < dl) dl = g.dk[c];
        dtijk = p.CFL * dl / vCFL;
        if (dtijk != dtijk) { isnan_ = true; dtijk = HUGEV * 2.0; }
    }
    // bit patterns of non-negative doubles order like the values
    unsigned long long bits = __double_as_longlong(dtijk);
    if (dtijk < 0.0) bits = 0ull;
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_down_sync(0xffffffffu, bits, off);
        bits = o < bits ? o : bits;
    }
    unsigned nn = __popc(__ballot_sync(0xffffffffu, isnan_));
    __shared__ unsigned long long wmin[32];
    __shared__ unsigned wnan[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { wmin[w] = bits; wnan[w] = nn; }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        bits = lane < nw ? wmin[lane] : ~0ull;
        nn = lane < nw ? wnan[lane] : 0u;
        for (int off = 16; off > 0; off >>= 1) {
            unsigned long long o = __shfl_down_sync(0xffffffffu, bits, off);
            bits = o < bits ? o : bits;
            nn += __shfl_down_sync(0xffffffffu, nn, off);
        }
        if (lane == 0) {
            atomicMin(&sc->dtMinBits, bits);
            if (nn) atomicAdd(&sc->nanCount, nn);
        }
    }
}

// UpdateStateData time bookkeeping (gamapp.F90:113-114, mhdgroup.F90:104-105) and the rest of CalcDT
// (step.F90:103-166): checks, the tFin clamp and the 10*dt0 clamp. mode 1 = initial dt (Hatch).
__global__ void k_dt_finalize(Par p, Scal* sc, int mode) {
    if (mode == 0) {
        sc->otime = sc->time;
        sc->time = sc->time + sc->dt;
        sc->ts = sc->ts + 1;
        sc->t = sc->t + sc->dt;
    }
    if (p.fixedTimestep) { sc->status = 0; return; }
    double dtOld = sc->dt;
    double dtMin = __longlong_as_double((long long)sc->dtMinBits);
    if (sc->dtMinBits >= 0x7FF0000000000000ull || dtMin > HUGEV) dtMin = HUGEV;
    int st = 0;
    if (dtMin == HUGEV) st |= 1;
    if (sc->ts > 0) {
        if (dtOld / dtMin >= 10) st |= 2;
        if ((sc->dt0 > TINY) && (dtMin / sc->dt0 <= p.limDT0)) st |= 2;
        if (dtMin <= TINY) st |= 1;
    }
    if (sc->nanCount) st |= 4;
    if (sc->waitFail) st |= 8;
    double r = dtMin;
    if ((sc->t + r) > p.tFin) r = dmax(p.tFin - sc->t, TINY);
    if (sc->dt0 > TINY && r > 10.0 * sc->dt0) r = 10.0 * sc->dt0;
    sc->dt = r;
    sc->status = st;
    sc->sticky |= st;
    sc->lastNan = sc->nanCount;
    sc->dtMinBits = 0x7FF0000000000000ull;
    sc->nanCount = 0u;
    sc->waitFail = 0u;   // reported in this step's status (and the sticky OR); the next step starts clear
}

// ================================================================================ boundary conditions
__device__ __forceinline__ void cpcell(const StateP& s, long long dst, long long src, bool withB) {
#pragma unroll
    for (int v = 0; v < 5; ++v) s.gas[v][dst] = s.gas[v][src];
    if (withB) { s.b[0][dst] = s.b[0][src]; s.b[1][dst] = s.b[1][src]; s.b[2][dst] = s.b[2][src]; }
}
__device__ __forceinline__ void cpmf(const StateP& s, long long dst, long long src) {
    s.mf[0][dst] = s.mf[0][src]; s.mf[1][dst] = s.mf[1][src]; s.mf[2][dst] = s.mf[2][src];
}

// I faces: periodic (bcs.F90:279-327) or zero gradient (bcs.F90:799-843), inner and outer side
__global__ void k_bc_i(Lay L, Par p, GridP g, StateP s) {
    // one thread per ghost layer n and (j, k) row: the layers are independent (each writes its own ghost
    // cell and faces, from active cells only)
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nG = L.nG, nj = L.Nj + 1;
    if (t >= (long long)nG * nj * (L.Nk + 1)) return;
    const int n = 1 + (int)(t % nG);
    const long long row = t / nG;
    const int j = (int)(row % nj), k = (int)(row / nj);
    const bool cell = (j < L.Nj) && (k < L.Nk);
    const int is = L.is(), ie = L.ie();
    // the LFM blast wave's fixed shells (ICs/lfmbw.F90:141-225): fixed gas; ghost face fluxes are the
    // conjugate active-shell fluxes scaled by the face areas (J/K signs flip across the axis)
    auto lfmbwShell = [&](bool inner) {
        double dApm[3] = {1.0, 1.0, 1.0};
        if (p.ringDoS && j < L.js()) dApm[1] = dApm[2] = -1.0;
        if (p.ringDoE && j >= L.je() + 1) dApm[1] = dApm[2] = -1.0;
        int ig = inner ? is - n : ie + n;
        if (cell) {
            long long c = L.at(ig, j, k);
            s.gas[0][c] = p.bwD0; s.gas[1][c] = 0.0; s.gas[2][c] = 0.0; s.gas[3][c] = 0.0;
            s.gas[4][c] = p.bwP0 / (p.gamma - 1.0);
        }
        for (int d = 0; d < 3; ++d) {
            int di = (!inner && d == 0) ? 1 : 0;
            int ia = inner ? is : ie + di;
            int jp, kp;
            lfmFC(L, p.ringDoS, p.ringDoE, d, j, k, jp, kp);
            long long cg = L.at(ig + di, j, k), ca = L.at(ia, jp, kp);
            double dA = g.face[d][cg] / g.face[d][ca];
            s.mf[d][cg] = dApm[d] * dA * s.mf[d][ca];
        }
    };
    if (p.bc[0] == BC_LFMBW) lfmbwShell(true);
    else if (p.bc[0] == BC_PERIODIC) {
        long long d = L.at(is - n, j, k), sidx = L.at(ie - n + 1, j, k);
        if (cell) cpcell(s, d, sidx, true);
        cpmf(s, d, sidx);
    } else if (p.bc[0] != BC_ION && cell) {   // BC_ION: launch_msph_bcs
        long long d = L.at(is - n, j, k), sidx = L.at(is, j, k);
        cpcell(s, d, sidx, false);
        cpmf(s, d, sidx);
    }
    if (p.bc[1] == BC_LFMBW) lfmbwShell(false);
    else if (p.bc[1] == BC_PERIODIC) {
        long long d = L.at(ie + n, j, k), sidx = L.at(is + n - 1, j, k);
        if (cell) cpcell(s, d, sidx, true);
        s.mf[1][d] = s.mf[1][sidx];
        s.mf[2][d] = s.mf[2][sidx];
        s.mf[0][d + 1] = s.mf[0][L.at(is + n, j, k)];
    } else if (p.bc[1] != BC_WIND && cell) {   // BC_WIND: launch_msph_bcs
        double B[3];
        cellBxyz(L, g, s.mf, L.at(ie, j, k), B);
        int ig = ie + n;
        long long d = L.at(ig, j, k);
        cpcell(s, d, L.at(ie, j, k), false);
        long long dI = d + 1;
        s.mf[0][dI] = g.face[0][dI] * (B[0] * g.Tf[0][0][dI] + B[1] * g.Tf[0][1][dI] + B[2] * g.Tf[0][2][dI]);
        s.mf[1][d] = g.face[1][d] * (B[0] * g.Tf[1][0][d] + B[1] * g.Tf[1][1][d] + B[2] * g.Tf[1][2][d]);
        s.mf[2][d] = g.face[2][d] * (B[0] * g.Tf[2][0][d] + B[1] * g.Tf[2][1][d] + B[2] * g.Tf[2][2][d]);
    }
}

// J faces: periodic (bcs.F90:329-378) or zero gradient (bcs.F90:845-888)
__global__ void k_bc_j(Lay L, Par p, StateP s) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int ni = L.Ni + 1;
    if (t >= (long long)ni * (L.Nk + 1)) return;
    int i = (int)(t % ni), k = (int)(t / ni);
    bool cell = (i < L.Ni) && (k < L.Nk);
    int js = L.js(), je = L.je(), nG = L.nG;
    // lfmIn / lfmOut (bcs.F90:1020-1106): ghosts across the axis from their conjugates
    auto lfmPole = [&](bool in) {
        for (int n = 1; n <= nG; ++n) {
            int jg = in ? js - n : je + n, jp, kp;
            if (cell) {
                lfmCC(L, p.ringDoS, p.ringDoE, jg, k, jp, kp);
                cpcell(s, L.at(i, jg, k), L.at(i, jp, kp), true);
            }
            lfmFC(L, p.ringDoS, p.ringDoE, 0, jg, k, jp, kp);
            s.mf[0][L.at(i, jg, k)] = s.mf[0][L.at(i, jp, kp)];
            int jf = in ? jg : jg + 1;   // the first outer J ghost face is je+2
            lfmFC(L, p.ringDoS, p.ringDoE, 1, jf, k, jp, kp);
            s.mf[1][L.at(i, jf, k)] = -s.mf[1][L.at(i, jp, kp)];
            lfmFC(L, p.ringDoS, p.ringDoE, 2, jg, k, jp, kp);
            s.mf[2][L.at(i, jg, k)] = -s.mf[2][L.at(i, jp, kp)];
        }
    };
    if (p.bc[2] == BC_LFMPOLE) lfmPole(true);
    else if (p.bc[2] == BC_PERIODIC) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, js - n, k), sidx = L.at(i, je - n + 1, k);
            if (cell) cpcell(s, d, sidx, true);
            cpmf(s, d, sidx);
        }
    } else if (cell) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, js - n, k), sidx = L.at(i, js, k);
            cpcell(s, d, sidx, false);
            cpmf(s, d, sidx);
        }
    }
    if (p.bc[3] == BC_LFMPOLE) lfmPole(false);
    else if (p.bc[3] == BC_PERIODIC) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, je + n, k), sidx = L.at(i, js + n - 1, k);
            if (cell) cpcell(s, d, sidx, true);
            s.mf[0][d] = s.mf[0][sidx];
            s.mf[2][d] = s.mf[2][sidx];
            s.mf[1][L.at(i, je + n + 1, k)] = s.mf[1][L.at(i, js + n, k)];
        }
    } else if (cell) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, je + n, k), sidx = L.at(i, je, k);
            cpcell(s, d, sidx, false);
            s.mf[0][d] = s.mf[0][sidx];
            s.mf[2][d] = s.mf[2][sidx];
            s.mf[1][L.at(i, je + n + 1, k)] = s.mf[1][L.at(i, je + 1, k)];
        }
    }
}

// K faces: periodic (bcs.F90:380-450, 2.5D replication included) or zero gradient (bcs.F90:890-930)
__global__ void k_bc_k(Lay L, Par p, StateP s) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int ni = L.Ni + 1;
    if (t >= (long long)ni * (L.Nj + 1)) return;
    int i = (int)(t % ni), j = (int)(t / ni);
    bool cell = (i < L.Ni) && (j < L.Nj);
    int ks = L.ks(), ke = L.ke(), nG = L.nG;
    if (p.bc[4] == BC_HALO) {
        // filled from the lower tile after the step
    } else if (p.bc[4] == BC_PERIODIC) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, j, ks - n), sidx = p.do25D ? L.at(i, j, ks) : L.at(i, j, ke - n + 1);
            if (cell) cpcell(s, d, sidx, true);
            cpmf(s, d, sidx);
        }
    } else if (cell) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, j, ks - n), sidx = L.at(i, j, ks);
            cpcell(s, d, sidx, false);
            cpmf(s, d, sidx);
        }
    }
    if (p.bc[5] == BC_HALO) {
        // filled from the upper tile after the step
    } else if (p.bc[5] == BC_PERIODIC) {
        for (int n = 1; n <= nG; ++n) {
            if (p.do25D) {
                long long d = L.at(i, j, ks + n), sidx = L.at(i, j, ks);
                if (cell) cpcell(s, d, sidx, true);
                cpmf(s, d, sidx);
            } else {
                long long d = L.at(i, j, ke + n), sidx = L.at(i, j, ks + n - 1);
                if (cell) cpcell(s, d, sidx, true);
                s.mf[0][d] = s.mf[0][sidx];
                s.mf[1][d] = s.mf[1][sidx];
                s.mf[2][L.at(i, j, ke + n + 1)] = s.mf[2][L.at(i, j, ks + n)];
            }
        }
    } else if (cell) {
        for (int n = 1; n <= nG; ++n) {
            long long d = L.at(i, j, ke + n), sidx = L.at(i, j, ke);
            cpcell(s, d, sidx, false);
            s.mf[0][d] = s.mf[0][sidx];
            s.mf[1][d] = s.mf[1][sidx];
            // bcs.F90:924 writes the J component of face ke+1 into the K faces above it; kept for parity
            s.mf[2][L.at(i, j, ke + n + 1)] = s.mf[1][L.at(i, j, ke + 1)];
        }
    }
}

// DivB (gridutils.F90:717-770) partial sums, one per block, reduced in a fixed order afterwards
__global__ void k_divb_partial(Lay L, GridP g, int bg, StateP s, double* partial) {
    Reg r = {L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    int i, j, k;
    double v = 0.0;
    if (reg_ijk(r, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) {
        long long c = L.at(i, j, k);
        double dFi = s.mf[0][c] - s.mf[0][c + 1];
        double dFj = s.mf[1][c] - s.mf[1][c + L.P];
        double dFk = s.mf[2][c] - s.mf[2][c + (long long)L.P * L.Q];
        double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
        if (bg) {   // total divergence includes the background flux (gridutils.F90:754-758)
            dFi0 = g.bFlux0[0][c] - g.bFlux0[0][c + 1];
            dFj0 = g.bFlux0[1][c] - g.bFlux0[1][c + L.P];
            dFk0 = g.bFlux0[2][c] - g.bFlux0[2][c + (long long)L.P * L.Q];
        }
        v = fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
    }
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __shared__ double ws[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        v = lane < nw ? ws[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) partial[blockIdx.x] = v;
    }
}
__global__ void k_sum_partials(const double* partial, int n, double* out) {
    __shared__ double ws[32];
    double v = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) v += partial[b];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        v = lane < nw ? ws[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) *out = v;
    }
}

// ================================================================================ host side
GridP Handle::gridP() const {
    GridP g;
    g.volume = volume;
    for (int x = 0; x < 3; ++x) g.xyzcc[x] = xyzcc[x];
    for (int d = 0; d < 3; ++d) for (int x = 0; x < 3; ++x) g.xfc[d][x] = xfc[d][x];
    g.di = di; g.dj = dj; g.dk = dk;
    for (int d = 0; d < 3; ++d) {
        g.face[d] = face[d]; g.edge[d] = edge[d];
        for (int q = 0; q < 9; ++q) { g.Tf[d][q] = Tf[d][q]; g.Te[d][q] = Te[d][q]; }
        for (int q = 0; q < 4; ++q) g.Teb[d][q] = Teb[d][q];
        for (int x = 0; x < 3; ++x) g.fcB0[d][x] = fcB0[d][x];
        for (int q = 0; q < 2; ++q) g.edgB0[d][q] = edgB0[d][q];
        g.B0[d] = B0[d]; g.bFlux0[d] = bFlux0[d]; g.dpB0[d] = dpB0[d];
    }
    return g;
}

static const int TPB = 128;

void launch_bflux2fld(Handle& h, const StateP& s, cudaStream_t st) {
    k_bflux2fld<<<grid_plane(Reg{0, h.L.Ni, 0, h.L.Nj, 0, h.L.Nk}, TPB), TPB, 0, st>>>(h.L, h.gridP(), s);
    h.launches++;
    if (h.p.doRing) launch_ring_bfix(h, s, st);   // gridutils.F90:298-300
}

void launch_bcs(Handle& h, const StateP& s, cudaStream_t st) {
    const Lay& L = h.L;
    k_bc_i<<<nblk((long long)L.nG * (L.Nj + 1) * (L.Nk + 1), TPB), TPB, 0, st>>>(L, h.p, h.gridP(), s);
    if (h.p.bc[0] == BC_ION || h.p.bc[1] == BC_WIND) launch_msph_bcs(h, s, st);   // IonInner, WindBC
    k_bc_j<<<nblk((long long)(L.Ni + 1) * (L.Nk + 1), TPB), TPB, 0, st>>>(L, h.p, s);
    k_bc_k<<<nblk((long long)(L.Ni + 1) * (L.Nj + 1), TPB), TPB, 0, st>>>(L, h.p, s);
    h.launches += 3;
}

void launch_calcdt_partial(Handle& h, const StateP& s, cudaStream_t st) {
    const Lay& L = h.L;
    k_calcdt<<<grid_plane(reg_dt(L, h.p), 256), 256, 0, st>>>(L, h.p, h.gridP(), s, h.dScal);
    h.launches++;
}

void launch_dt_finalize(Handle& h, int mode, cudaStream_t st) {
    k_dt_finalize<<<1, 1, 0, st>>>(h.p, h.dScal, mode);
    h.launches++;
}

void launch_calcdt(Handle& h, const StateP& s, int mode, cudaStream_t st) {
    launch_calcdt_partial(h, s, st);
    launch_dt_finalize(h, mode, st);
}

__global__ void k_to_f32(const double* src, float* dst, long long n) {
    long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (l < n) dst[l] = float(src[l]);
}

__global__ void k_ratio_f32(const double* num, const double* den, float* dst, long long n) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) { double d = den[t]; dst[t] = d != 0.0 ? float(num[t] / d) : 0.0f; }
}

// float copies of the background planes (fcB0, bFlux0/face, edgB0)
void refresh_f32_background(Handle& h) {
    if (!h.f32pool || !h.p.doBackground) return;
    const long long E = h.L.E;
    F32Planes& f = h.f32;
    for (int d = 0; d < 3; ++d) {
        for (int x = 0; x < 3; ++x) { k_to_f32<<<nblk(E, 256), 256, 0, h.stream>>>(h.fcB0[d][x], f.fcB0[d][x], E); }
        for (int c = 0; c < 2; ++c) { k_to_f32<<<nblk(E, 256), 256, 0, h.stream>>>(h.edgB0[d][c], f.edgB0[d][c], E); }
        k_ratio_f32<<<nblk(E, 256), 256, 0, h.stream>>>(h.bFlux0[d], h.face[d], f.b0n[d], E);
        h.launches += 6;
    }
}

int ensure_f32(Handle& h) {
    if (h.f32pool) return 0;
    const long long E = h.L.E;
    const int nplanes = 29 + 24 + 64 + 6 + (h.p.doBackground ? 18 : 0);   // 6: the I and J edges' face velocities
    if (cudaMalloc(&h.f32pool, sizeof(float) * E * nplanes) != cudaSuccess) return 3;
    cudaMemsetAsync(h.f32pool, 0, sizeof(float) * E * nplanes, h.stream);
    float* q = h.f32pool;
    auto take = [&]() { float* r = q; q += E; return r; };
    F32Planes& f = h.f32;
    for (int v = 0; v < 5; ++v) f.Wh[v] = take();
    for (int v = 0; v < 5; ++v) f.Wn[v] = take();
    for (int x = 0; x < 3; ++x) f.hb[x] = take();
    for (int x = 0; x < 3; ++x) f.nb[x] = take();
    for (int x = 0; x < 3; ++x) f.hbA[x] = take();
    for (int x = 0; x < 3; ++x) f.nbA[x] = take();
    for (int x = 0; x < 3; ++x) f.Vf[x] = take();
    for (int e = 0; e < 2; ++e) for (int x = 0; x < 3; ++x) f.VfE[e][x] = take();
    f.rho = take();
    for (int x = 0; x < 3; ++x) f.VdV[x] = take();
    for (int d = 0; d < 3; ++d) {
        for (int v = 0; v < 5; ++v) f.gflx[d][v] = take();
        for (int x = 0; x < 3; ++x) f.mflx[d][x] = take();
    }
    f.volume = take();
    for (int d = 0; d < 3; ++d) f.face[d] = take();
    for (int d = 0; d < 3; ++d) f.edge[d] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 9; ++c) f.Tf[d][c] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 6; ++c) f.Te[d][c] = take();
    for (int d = 0; d < 3; ++d) for (int c = 0; c < 4; ++c) f.Teb[d][c] = take();
    if (h.p.doBackground) {
        for (int d = 0; d < 3; ++d) {
            for (int x = 0; x < 3; ++x) f.fcB0[d][x] = take();
            for (int c = 0; c < 2; ++c) f.edgB0[d][c] = take();
            f.b0n[d] = take();
        }
    }
    auto cv = [&](const double* s_, float* d_) { k_to_f32<<<nblk(E, 256), 256, 0, h.stream>>>(s_, d_, E); h.launches++; };
    cv(h.volume, f.volume);
    for (int d = 0; d < 3; ++d) {
        cv(h.face[d], f.face[d]);
        cv(h.edge[d], f.edge[d]);
        for (int c = 0; c < 9; ++c) cv(h.Tf[d][c], f.Tf[d][c]);
        for (int c = 0; c < 6; ++c) cv(h.Te[d][3 + c], f.Te[d][c]);
        for (int c = 0; c < 4; ++c) cv(h.Teb[d][c], f.Teb[d][c]);
    }
    refresh_f32_background(h);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

int kernels_per_step(const Handle& h) {
    int n = 1 + 1;                      // begin, predict cells
    if (h.p.doMHD) n += 1 + 1 + 3;      // predict faces, Mom2Face (all directions), 3 edge kernels
    n += (h.p.do25D ? 2 : 3) + ((h.fuseUpdate && !h.closure) ? 0 : 1);   // fluxes + flux2deltas
    n += 1 + 1 + 1;                     // e2flux/copy, bflux2fld, update gas
    n += 2 + 3 + 1;                     // calcdt + finalize, 3 BC kernels, final bflux2fld
    n += ring_kernels_per_step(h);
    n += msph_kernels_per_step(h);
    if (h.closure) n += closure_kernels_per_step(h) + 1;   // + the conditional Flux2Deltas
    return n;
}

// NVTX ranges named after the reference's timers of the step (mhdgroup.F90:30-70, stress.F90:78-150,
// gamapp.F90:76-99): a profiler attached to an eager (non-graph) step sees its kernels under the same
// names as the reference's printClocks tree (Advance > Gamera > Predictor, E-Field, Fluxes, ...).
static const char* const kPhaseRange[NPHASE] = {"Predictor", "E-Field", "Fluxes", "Flux2Deltas", "Update", "DT",
                                                "BCs"};   // BCs is pushed by step_enqueue_bcs

int step_enqueue(Handle& h, int cur, cudaEvent_t* ev, bool split, int part) {
    cudaStream_t st = h.stream;
    int openRange = -1;
    auto mark = [&](int ph) {
        if (ev) cudaEventRecord(ev[ph], st);
        if (openRange >= 0) nvtxRangePop();
        openRange = ph < NPHASE ? ph : -1;
        if (openRange >= 0) nvtxRangePushA(kPhaseRange[ph]);
    };
    struct Outer {   // "Advance" around the whole enqueue, closing any open phase range on return
        int& open;
        explicit Outer(int& o) : open(o) { nvtxRangePushA("Advance"); }
        ~Outer() { if (open >= 0) nvtxRangePop(); nvtxRangePop(); }
    } outer(openRange);
    const Lay& L = h.L;
    const Par& p = h.p;
    GridP g = h.gridP();
    StateP nS = h.S[cur], oS = h.S[cur ^ 1];
    const Reg cells = {0, L.Ni, 0, L.Nj, 0, L.Nk}, act = {L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    if (part != STEP_POST) {
    mark(PH_PREDICT);
    k_step_begin<<<1, 1, 0, st>>>(h.dScal);
    if (p.doMHD) {
        Vec3P mf = {{nS.mf[0], nS.mf[1], nS.mf[2]}}, omf = {{oS.mf[0], oS.mf[1], oS.mf[2]}},
              hmf = {{h.H.mf[0], h.H.mf[1], h.H.mf[2]}}, hbA = {{h.hbA[0], h.hbA[1], h.hbA[2]}},
              nbA = {{h.nbA[0], h.nbA[1], h.nbA[2]}};
        F32FaceOut fo{};
        if (h.prec == PREC_FP32FLUX)
            for (int x = 0; x < 3; ++x) { fo.hbA[x] = h.f32.hbA[x]; fo.nbA[x] = h.f32.nbA[x]; }
        k_predict_faces<<<nblk(L.E / 2, 256), 256, 0, st>>>(L.E, p, g, mf, omf, hmf, hbA, nbA, fo, h.dScal);
        h.launches++;
    }
    PrimP Wh, Wn;
    for (int v = 0; v < 5; ++v) { Wh.w[v] = h.Wh[v]; Wn.w[v] = h.Wn[v]; }
    Vec3P VdV = {{h.VdV[0], h.VdV[1], h.VdV[2]}};
    F32CellOut fc{};
    if (h.prec == PREC_FP32FLUX) {
        for (int v = 0; v < 5; ++v) { fc.Wh[v] = h.f32.Wh[v]; fc.Wn[v] = h.f32.Wn[v]; }
        for (int x = 0; x < 3; ++x) { fc.hb[x] = h.f32.hb[x]; fc.nb[x] = h.f32.nb[x]; fc.VdV[x] = h.f32.VdV[x]; }
        fc.rho = h.f32.rho;
    }
    k_predict_cells<<<grid_plane(Reg{0, L.Ni, 0, L.Nj, 0, L.Nk}, TPB), TPB, 0, st>>>(L, p, g, nS, oS, h.H, Wh, Wn, VdV, fc, h.dScal);
    h.launches += 2;
    if (p.doRing) launch_ring_bfix(h, h.H, st, h.prec == PREC_FP32FLUX);   // bFlux2Fld's ring fix
    if (p.predFixLFM) launch_predfix_lfm(h, h.H, st, h.prec == PREC_FP32FLUX);   // HackPredictor
    mark(PH_EFIELD);
    if (p.doMHD) {
        enqueue_efield(h, nS, st);
        if (p.msph.on) launch_msph_efix(h, nS, st);   // HackE (mhdgroup.F90:40-44)
    }
    }
    if (part == STEP_PRE) return (int)cudaGetLastError();
    if (part == STEP_ALL) {
        mark(PH_FLUXES);
        enqueue_fluxes(h, nS, st);
    }
    if (p.doRing) launch_ring_flux(h, st);   // stress.F90:134-139
    if (p.msph.on) launch_ion_flux(h, st);    // HackFlux (stress.F90:141-143)
    mark(PH_DELTAS);
    PrimP dGH;
    for (int v = 0; v < 5; ++v) dGH.w[v] = h.dGasH[v];
    Vec3P dGM = {{h.dGasM[0], h.dGasM[1], h.dGasM[2]}};
    FluxOut<float> F32[3];
    FluxP F64[3];
    for (int d = 0; d < 3; ++d) {
        for (int v = 0; v < 5; ++v) { F32[d].g[v] = h.f32.gflx[d][v]; F64[d].g[v] = h.gflx[d][v]; }
        for (int x = 0; x < 3; ++x) { F32[d].m[x] = h.f32.mflx[d][x]; F64[d].m[x] = h.mflx[d][x]; }
    }
    // without a closure the update computes the deltas itself (no dGasH/dGasM round trip through HBM)
    const bool fuse = h.fuseUpdate && !h.closure;
    // learned closure: face corrections from the net on State n; a corrected update that fails positivity
    // falls back to the plain fluxes (the second, conditional Flux2Deltas)
    const float* corr = h.closure ? closure_enqueue_corr(h, nS, st) : nullptr;
    for (int pass = 0; pass < (fuse ? 0 : (corr ? 2 : 1)); ++pass) {
        const float* cq = pass == 0 ? corr : nullptr;
        const Scal* cond = pass == 0 ? nullptr : h.dScal;
        if (h.prec == PREC_FP32FLUX)
            k_flux2deltas<float><<<grid_plane(act, TPB), TPB, 0, st>>>(L, p, g, F32[0], F32[1], F32[2], dGH, dGM, cq, cond);
        else
            k_flux2deltas<double><<<grid_plane(act, TPB), TPB, 0, st>>>(L, p, g, F64[0], F64[1], F64[2], dGH, dGM, cq, cond);
        if (pass == 0 && corr) closure_enqueue_check(h, nS, st);
        if (pass == 1) h.launches++;
    }
    mark(PH_UPDATE);
    // applyUpdate into the oState buffer (which becomes State n+1)
    Vec3P E = {{h.E[0], h.E[1], h.E[2]}};
    if (p.doRing && p.doMHD) launch_pole_e(h, h.E, st);   // mhdgroup.F90:139-142
    if (h.closure && p.doMHD) closure_enqueue_emf(h, st);
    k_e2flux<<<grid_plane(Reg{0, L.Ni + 1, 0, L.Nj + 1, 0, L.Nk + 1}, TPB), TPB, 0, st>>>(L, p, E, nS, oS, h.dScal);
    // bFlux2Fld of the update; with ring averaging its ring fix is left to the RingAverage bFlux2Fld,
    // which recomputes every cell before anything reads a ghost B
    if (p.doMHD) k_bflux2fld<<<grid_plane(cells, TPB), TPB, 0, st>>>(L, g, oS);
    else k_copy_b<<<nblk(L.E, 256), 256, 0, st>>>(L, nS, oS);
    if (h.prec == PREC_FP32FLUX) {
        if (fuse) k_update_gas<float, true><<<grid_plane(cells, TPB), TPB, 0, st>>>(L, p, g, nS, oS, dGH, dGM, F32[0], F32[1], F32[2], h.dScal);
        else k_update_gas<float, false><<<grid_plane(cells, TPB), TPB, 0, st>>>(L, p, g, nS, oS, dGH, dGM, F32[0], F32[1], F32[2], h.dScal);
    } else {
        if (fuse) k_update_gas<double, true><<<grid_plane(cells, TPB), TPB, 0, st>>>(L, p, g, nS, oS, dGH, dGM, F64[0], F64[1], F64[2], h.dScal);
        else k_update_gas<double, false><<<grid_plane(cells, TPB), TPB, 0, st>>>(L, p, g, nS, oS, dGH, dGM, F64[0], F64[1], F64[2], h.dScal);
    }
    h.launches += 4;
    if (p.msph.on) launch_apply_grav(h, oS, nS, st);   // mhdgroup.F90:60-65 (oS holds the new state)
    if (p.doRing) launch_ring_average(h, oS, st);   // mhdgroup.F90:68-74
    if (p.msph.on) launch_msph_perstep(h, oS, st);   // HackStep (gamapp.F90:104-109)
    // CalcDT (the per-cell minimum; finalized below, or after the tiles' minimum for a tiled run)
    mark(PH_DT);
    launch_calcdt_partial(h, oS, st);
    if (!split) {
        step_enqueue_bcs(h, cur, ev);
        step_enqueue_ghosts(h, cur);
        mark(NPHASE);
    }
    return (int)cudaGetLastError();
}

// The rest of CalcDT, then EnforceBCs on the new state S[cur ^ 1]
void step_enqueue_bcs(Handle& h, int cur, cudaEvent_t* ev) {
    cudaStream_t st = h.stream;
    launch_dt_finalize(h, 0, st);
    if (ev) cudaEventRecord(ev[PH_BCS], st);
    nvtxRangePushA("BCs");
    launch_bcs(h, h.S[cur ^ 1], st);
    nvtxRangePop();
}

// bFlux2Fld of the ghost cells of the new state S[cur ^ 1], after the BCs (and the halo fill of a tile)
void step_enqueue_ghosts(Handle& h, int cur) {
    cudaStream_t st = h.stream;
    const Lay& L = h.L;
    StateP s = h.S[cur ^ 1];
    if (h.p.do25D) launch_bflux2fld(h, s, st);   // the 2.5D K replication rewrites an active cell's upper face
    else {
        k_bflux2fld_ghost<<<nblk(ghost_cells(L), TPB), TPB, 0, st>>>(L, h.gridP(), s);
        h.launches++;
        if (h.p.doRing) launch_ring_bfix(h, s, st);
    }
}

double launch_divb(Handle& h, double* scratchDev, cudaStream_t st) {
    const Lay& L = h.L;
    long long n = (long long)L.Nip * L.Njp * L.Nkp;
    int nb = (int)nblk(n, 256);
    StateP s = h.S[h.cur];
    k_divb_partial<<<nb, 256, 0, st>>>(L, h.gridP(), h.p.doBackground, s, scratchDev);
    k_sum_partials<<<1, 1024, 0, st>>>(scratchDev, nb, scratchDev + nb);
    h.launches += 2;
    double out = 0.0;
    cudaMemcpyAsync(&out, scratchDev + nb, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return out;
}

}  // namespace gam
