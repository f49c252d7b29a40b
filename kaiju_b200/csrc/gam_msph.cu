// The magnetosphere problem on the device: its ionospheric inner and solar-wind outer I boundaries, its
// E-field, flux and per-step hooks, and gravity -- the pieces voltron/ICs/earthcmi.F90's initUser plugs into
// the step (HackE = EFix, HackFlux = IonFlux, HackStep = PerStep; IonInnerBC_T and WindBC_T), for a constant
// solar wind and no ionospheric coupling (IonInnerBC_T%inExyz = inEijk = 0: no REMIX potential reaches the
// inner boundary). One thread per cell, face, edge or ghost; all FP64 (they act on the state, not the fluxes,
// except IonFlux, which runs on the flux planes in their storage type).
#include <cstdio>
#include "gam_common.cuh"
#include "gam_step.cuh"
#include "gam_lfm.cuh"
#include "gam_kern.cuh"

namespace gam {

namespace {

constexpr int TB = 256;
inline unsigned nblkM(long long n, int b) { return (unsigned)((n + b - 1) / b); }

__device__ __forceinline__ double dot3v(const double* a, const double* b) {
    double s = 0.0;
    for (int c = 0; c < 3; ++c) s = s + a[c] * b[c];
    return s;
}
// normVec (math.F90:332-343)
__device__ __forceinline__ void normVecD(const double* a, double* o) {
    double nA = sqrt(dot3v(a, a));
    if (nA <= TINY) { o[0] = o[1] = o[2] = 0.0; }
    else { o[0] = a[0] / nA; o[1] = a[1] / nA; o[2] = a[2] / nA; }
}
// gfortran's NORM2 (scaled sum of squares)
__device__ __forceinline__ double norm2D(const double* a) {
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < 3; ++i) {
        if (a[i] != 0.0) {
            double ax = fabs(a[i]);
            if (scale < ax) { ssq = 1.0 + ssq * sq(scale / ax); scale = ax; }
            else ssq = ssq + sq(ax / scale);
        }
    }
    return scale * sqrt(ssq);
}
// RampDown (math.F90:97-111)
__device__ __forceinline__ double rampDown(double r, double rC, double lC) {
    if (r <= rC) return 1.0;
    if (r >= rC + lC) return 0.0;
    double rScl = (r - rC) / lC;
    double eArg = -1.0 / (1.0 - rScl * rScl);
    return exp(eArg + 1.0);
}
// wgtWind (apps/wind.F90:185-203) for the constant wind: 1 on the sunward half, ramping to 0 tailward
__device__ __forceinline__ double wgtWind(const MsphPar& m, const double* xyz) {
    double nHat[3], vHat[3];
    normVecD(xyz, nHat);
    normVecD(m.wV, vHat);
    double d = 0.0;
    for (int c = 0; c < 3; ++c) d = d + (-vHat[c]) * nHat[c];
    double dTh = acos(d) * 180.0 / PI;
    return rampDown(dTh, 90.0, 90.0);
}
// Con2Fast with CellPress2Cs (gamutils.F90:324-360)
__device__ __forceinline__ double con2Fast(const Par& p, const double* gCon, const double* B) {
    double rho = dmax(gCon[0], p.dFloor), ir = 1.0 / rho;
    double Vx = gCon[1] * ir, Vy = gCon[2] * ir, Vz = gCon[3] * ir;
    double KinE = 0.5 * rho * (sq(Vx) + sq(Vy) + sq(Vz));
    double P = dmax((p.gamma - 1) * (gCon[4] - KinE), p.pFloor);
    double Cs = sqrt(p.gamma * P / rho);
    double Va = norm2D(B) / sqrt(gCon[0]);
    if (p.doBoris) Va = p.Ca * Va / sqrt(sq(p.Ca) + sq(Va));
    return sqrt(sq(Cs) + sq(Va));
}
__device__ __forceinline__ void loadCon(const StateP& s, long long c, double* U) {
    for (int v = 0; v < 5; ++v) U[v] = s.gas[v][c];
}
__device__ __forceinline__ void storeCon(const StateP& s, long long c, const double* U) {
    for (int v = 0; v < 5; ++v) s.gas[v][c] = U[v];
}

// ------------------------------------------------------------------ boundaries
// Gas and face fluxes of the I ghost shells. One thread per ghost layer n and (j, k) row, j in [0, Nj], k in
// [0, Nk] (the +1 rows carry faces only). side 0: IonInner (earthcmi.F90:397-456) with CellPlasmaBC
// (apps/msphingest.F90:354-368) for one fluid and Veb = 0: the ghost is the mirrored active cell's density and
// pressure at rest, its faces carry no residual flux. side 1: WindBC (apps/wind.F90:224-319): the ghost is
// the wind blended with an outflow copy of the last active cell (at least MinMach = 1 fast speed outward), its
// faces the wind's flux blended with the last active face's.
__global__ void k_bc_ionwind(Lay L, Par p, GridP g, StateP s, int side) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nG = L.nG, nj = L.Nj + 1;
    if (t >= (long long)nG * nj * (L.Nk + 1)) return;
    const int n = 1 + (int)(t % nG);
    const long long row = t / nG;
    const int j = (int)(row % nj), k = (int)(row / nj);
    const bool cell = (j < L.Nj) && (k < L.Nk);
    if (side == 0) {
        const int ig = L.is() - n, ip = L.is() + n - 1;
        if (cell) {
            int jp, kp;
            lfmCC(L, p.ringDoS, p.ringDoE, j, k, jp, kp);
            double pU[5], pW[5], gW[5], gU[5];
            loadCon(s, L.at(ip, jp, kp), pU);
            cellC2P(p, pU, pW);
            gW[0] = pW[0]; gW[1] = 0.0; gW[2] = 0.0; gW[3] = 0.0; gW[4] = pW[4];
            cellP2C(p, gW, gU);
            storeCon(s, L.at(ig, j, k), gU);
        }
        const long long c = L.at(ig, j, k);
        if (j < L.Nj && k < L.Nk) s.mf[0][c] = 0.0;   // isGoodFaceIJK (gridutils.F90:985-1009)
        if (k < L.Nk) s.mf[1][c] = 0.0;
        if (j < L.Nj) s.mf[2][c] = 0.0;
        return;
    }
    const MsphPar& m = p.msph;
    const int ip = L.ie(), ig = L.ie() + n;
    if (cell) {
        const long long c = L.at(ig, j, k);
        double xcc[3] = {g.xyzcc[0][c], g.xyzcc[1][c], g.xyzcc[2][c]};
        double wSW = wgtWind(m, xcc), wMHD = 1.0 - wSW;
        double gW_sw[5] = {0, 0, 0, 0, 0}, gW_in[5] = {0, 0, 0, 0, 0};
        if (wSW > TINY) {
            gW_sw[0] = m.wD; gW_sw[4] = m.wP;
            for (int q = 0; q < 3; ++q) gW_sw[1 + q] = m.wV[q];
        }
        if (wMHD > TINY) {
            const long long a = L.at(ip, j, k);
            double gCon[5], B_in[3] = {s.b[0][a], s.b[1][a], s.b[2][a]};
            loadCon(s, a, gCon);
            cellC2P(p, gCon, gW_in);
            double Cx = con2Fast(p, gCon, B_in);
            double V[3] = {gW_in[1], gW_in[2], gW_in[3]};
            const long long f = a + 1;   // face ip+1
            double nHat[3] = {g.Tf[0][0][f], g.Tf[0][1][f], g.Tf[0][2][f]};
            if (dot3v(V, nHat) < 1.0 * Cx) {
                double vn = dot3v(V, nHat);
                for (int q = 0; q < 3; ++q) V[q] = V[q] - vn * nHat[q] + 1.0 * Cx * nHat[q];
            }
            for (int q = 0; q < 3; ++q) gW_in[1 + q] = V[q];
        }
        double gW[5], gCon[5];
        for (int v = 0; v < 5; ++v) gW[v] = wSW * gW_sw[v] + wMHD * gW_in[v];
        cellP2C(p, gW, gCon);
        storeCon(s, c, gCon);
    }
    for (int d = 0; d < 3; ++d) {
        const int fi = d == 0 ? ig + 1 : ig, si = d == 0 ? ip + 1 : ip;
        const long long f = L.at(fi, j, k);
        double xf[3] = {g.xfc[d][0][f], g.xfc[d][1][f], g.xfc[d][2][f]};
        double wSW = wgtWind(m, xf);
        double nHat[3] = {g.Tf[d][0][f], g.Tf[d][1][f], g.Tf[d][2][f]};
        double swFlx = g.face[d][f] * dot3v(nHat, m.wB);   // Project2Face (bcs.F90:250-263)
        double inFlx = s.mf[d][L.at(si, j, k)];
        s.mf[d][f] = wSW * swFlx + (1 - wSW) * inFlx;
    }
}
// Bxyz of the ghost shell from the (conjugate) cell's faces (the second loops of IonInner and WindBC)
__global__ void k_bc_ionwind_b(Lay L, Par p, GridP g, StateP s, int side) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nG = L.nG;
    if (t >= (long long)nG * L.Nj * L.Nk) return;
    const int n = 1 + (int)(t % nG);
    const long long row = t / nG;
    const int j = (int)(row % L.Nj), k = (int)(row / L.Nj);
    const int ig = side == 0 ? L.is() - n : L.ie() + n;
    int jp, kp;
    lfmCC(L, p.ringDoS, p.ringDoE, j, k, jp, kp);
    double B[3];
    cellBxyz(L, g, s.mf, L.at(ig, jp, kp), B);
    const long long c = L.at(ig, j, k);
    s.b[0][c] = B[0]; s.b[1][c] = B[1]; s.b[2][c] = B[2];
}
// the ghost shell's cells across the axis take their conjugates' Bxyz (the third loops)
__global__ void k_bc_ionwind_bfix(Lay L, Par p, StateP s, int side) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nG = L.nG;
    if (t >= (long long)nG * L.Nk) return;
    const int n = 1 + (int)(t % nG), k = (int)(t / nG);
    for (int q = 0; q < nG; ++q) {
        const int i = side == 0 ? q : L.ie() + 1 + q;   // isg..is-1 or ie+1..ieg
        int jp, kp;
        if (p.ringDoS) {
            int jg = L.js() - n;
            lfmCC(L, true, p.ringDoE, jg, k, jp, kp);
            long long d = L.at(i, jg, k), a = L.at(i, jp, kp);
            s.b[0][d] = s.b[0][a]; s.b[1][d] = s.b[1][a]; s.b[2][d] = s.b[2][a];
        }
        if (p.ringDoE) {
            int jg = L.je() + n;
            lfmCC(L, p.ringDoS, true, jg, k, jp, kp);
            long long d = L.at(i, jg, k), a = L.at(i, jp, kp);
            s.b[0][d] = s.b[0][a]; s.b[1][d] = s.b[1][a]; s.b[2][d] = s.b[2][a];
        }
    }
}

// ------------------------------------------------------------------ E field (HackE = EFix)
// IonEFix (apps/msphutils.F90:214-240) with zero ionospheric E: the first shell's J and K edges
__global__ void k_ion_efix(Lay L, GridP g, Vec3P E) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nj * L.Nk) return;
    const int j = (int)(t % L.Nj), k = (int)(t / L.Nj);
    const long long c = L.at(L.is(), j, k);
    E.v[1][c] = g.edge[1][c] * 0.0;
    E.v[2][c] = g.edge[2][c] * 0.0;
}
// WindEFix (apps/wind.F90:489-565): edges i = ie-2 .. ie+1 blended toward the wind's -V x B, plus the
// diffusive E of DiffuseOuter (:568-618) on the outermost edges
struct Xyz3 { const double* x[3]; };
__global__ void k_wind_efix(Lay L, Par p, GridP g, Xyz3 X, StateP n, Vec3P E, const Scal* sc) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ni = 4, nj = L.Njp + 1, nk = L.Nkp + 1;
    if (t >= (long long)ni * nj * nk) return;
    const int i = L.ie() - 2 + (int)(t % ni);
    const long long q = t / ni;
    const int j = L.js() + (int)(q % nj), k = L.ks() + (int)(q / nj);
    const MsphPar& m = p.msph;
    double swE[3] = {-(m.wV[1] * m.wB[2] - m.wV[2] * m.wB[1]), -(m.wV[2] * m.wB[0] - m.wV[0] * m.wB[2]),
                     -(m.wV[0] * m.wB[1] - m.wV[1] * m.wB[0])};
    const long long c = L.at(i, j, k);
    double wSW = 0.0;
    for (int d = 0; d < 3; ++d) {
        const long long c2 = c + L.stride(d);
        double e1[3] = {X.x[0][c], X.x[1][c], X.x[2][c]}, e2[3] = {X.x[0][c2], X.x[1][c2], X.x[2][c2]};
        double ecc[3] = {0.5 * (e1[0] + e2[0]), 0.5 * (e1[1] + e2[1]), 0.5 * (e1[2] + e2[2])};
        wSW = wgtWind(m, ecc);
        if (wSW > TINY) {
            if (i <= L.ie()) wSW = wSW / (1.0 + L.ie() + 1 - i);
            double de[3] = {e2[0] - e1[0], e2[1] - e1[1], e2[2] - e1[2]};
            E.v[d][c] = (1.0 - wSW) * E.v[d][c] + wSW * dot3v(swE, de);
        }
    }
    if (i == L.ie() + 1) {   // DiffuseOuter with the weight of the last (K) edge
        const double vSW = dmin(norm2D(m.wV), p.Ca);
        const long long cj = L.stride(1), ck = L.stride(2);
        double bP = n.mf[1][c] / dmax(g.face[1][c], TINY), bM = n.mf[1][c - 1] / dmax(g.face[1][c - 1], TINY);
        double db2 = bP - bM;
        bP = n.mf[0][c] / g.face[0][c]; bM = n.mf[0][c - cj] / g.face[0][c - cj];
        double db1 = bP - bM;
        const double JdK = db2 - db1;
        bP = n.mf[0][c] / g.face[0][c]; bM = n.mf[0][c - ck] / g.face[0][c - ck];
        db2 = bP - bM;
        bP = n.mf[2][c] / g.face[2][c]; bM = n.mf[2][c - 1] / g.face[2][c - 1];
        db1 = bP - bM;
        const double JdJ = db2 - db1;
        double dl = sqrt(g.edge[1][c] * g.edge[2][c]);
        double Vd = dmin(vSW, p.CFL * dl / sc->dt);
        E.v[0][c] = E.v[0][c] + wSW * 0.0;
        E.v[1][c] = E.v[1][c] + wSW * (Vd * JdJ * dl);
        E.v[2][c] = E.v[2][c] + wSW * (Vd * JdK * dl);
    }
}
// WindEFix's touch-up next to the axis: the I edges of the axis rows take their k average, the K edges 0
__global__ void k_wind_efix_ring(Lay L, Par p, Vec3P E) {
    const int t = threadIdx.x;   // 4 shells x 2 sides
    if (t >= 8) return;
    const int nS = L.ie() - 2 + (t >> 1), side = t & 1;   // side 0: doE (je+1), 1: doS (js)
    if ((side == 0 && !p.ringDoE) || (side == 1 && !p.ringDoS)) return;
    const int j = side == 0 ? L.je() + 1 : L.js();
    double s = 0.0;
    for (int k = L.ks(); k <= L.ke(); ++k) s = s + E.v[0][L.at(nS, j, k)];
    const double avg = s / L.Nkp;
    for (int k = 0; k < L.Nk; ++k) { E.v[0][L.at(nS, j, k)] = avg; E.v[2][L.at(nS, j, k)] = 0.0; }
}

// ------------------------------------------------------------------ fluxes (HackFlux = IonFlux)
// IonFlux (earthcmi.F90:282-331): the first shell's I fluxes at the two cells next to the axis replaced by
// their average over k. One thread per side and variable (5 gas, 3 magnetic); doE before doS as there.
template <typename O>
__global__ void k_ion_flux(Lay L, Par p, FluxOut<O> FI) {
    const int t = threadIdx.x;
    if (t >= 16) return;
    const int side = t / 8, v = t % 8;   // side 0: je (doE), 1: js (doS)
    if ((side == 0 && !p.ringDoE) || (side == 1 && !p.ringDoS)) return;
    const int j = side == 0 ? L.je() : L.js();
    O* q = v < 5 ? FI.g[v] : FI.m[v - 5];
    double s = 0.0;
    for (int k = L.ks(); k <= L.ke(); ++k) s = s + double(q[L.at(L.is(), j, k)]);
    const O avg = O(s / L.Nkp);
    for (int k = L.ks(); k <= L.ke(); ++k) q[L.at(L.is(), j, k)] = avg;
}

// ------------------------------------------------------------------ gravity
// AddGrav (background.F90:170-252) with Phi = -GM0/r and doSphGrav (the radial part only), active cells
__global__ void k_add_grav(Lay L, GridP g, double GM0, Vec3P gx) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nip * L.Njp * L.Nkp) return;
    const int i = L.is() + (int)(t % L.Nip);
    const long long q = t / L.Nip;
    const int j = L.js() + (int)(q % L.Njp), k = L.ks() + (int)(q / L.Njp);
    const long long c = L.at(i, j, k);
    const long long f[6] = {c, c, c, c + 1, c + L.stride(1), c + L.stride(2)};
    const int fd[6] = {0, 1, 2, 0, 1, 2};
    double Phi[6], da[6], nn[6][3];
    for (int u = 0; u < 6; ++u) {
        double x = g.xfc[fd[u]][0][f[u]], y = g.xfc[fd[u]][1][f[u]], z = g.xfc[fd[u]][2][f[u]];
        Phi[u] = -GM0 / sqrt(sq(x) + sq(y) + sq(z));   // PhiGrav (msphutils.F90:626-633)
        da[u] = g.face[fd[u]][f[u]];
        for (int x3 = 0; x3 < 3; ++x3) nn[u][x3] = g.Tf[fd[u]][x3][f[u]];
    }
    const double dV = g.volume[c];
    double gv[3], rhat[3], xc[3] = {g.xyzcc[0][c], g.xyzcc[1][c], g.xyzcc[2][c]};
    for (int x3 = 0; x3 < 3; ++x3)
        gv[x3] = -(Phi[3] * da[3] * nn[3][x3] - Phi[0] * da[0] * nn[0][x3] + Phi[4] * da[4] * nn[4][x3] -
                   Phi[1] * da[1] * nn[1][x3] + Phi[5] * da[5] * nn[5][x3] - Phi[2] * da[2] * nn[2][x3]) / dV;
    normVecD(xc, rhat);
    const double gr = dot3v(gv, rhat);
    for (int x3 = 0; x3 < 3; ++x3) gx.v[x3][c] = gr * rhat[x3];
}
// applyGrav (mhdgroup.F90:620-705), one fluid, classical momentum: S is the updated state, O the previous
__global__ void k_apply_grav(Lay L, Par p, Vec3P gx, StateP S, StateP O, const Scal* sc) {
    Reg r = {L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    int i, j, k;
    if (!reg_plane(r, i, j, k)) return;
    const long long c = L.at(i, j, k);
    if (!(S.gas[0][c] >= 0.0)) return;
    double U[5], W[5];
    loadCon(S, c, U);
    cellC2P(p, U, W);
    const double IntE = W[4] / (p.gamma - 1);
    const double Dhf = 0.5 * (S.gas[0][c] + O.gas[0][c]);
    const double dt = sc->dt;
    double cM[3];
    for (int q = 0; q < 3; ++q) cM[q] = U[1 + q] + dt * Dhf * gx.v[q][c];
    for (int q = 0; q < 3; ++q) U[1 + q] = cM[q];
    U[4] = IntE + 0.5 * dot3v(cM, cM) / U[0];
    storeCon(S, c, U);
}

// ------------------------------------------------------------------ per step (HackStep = PerStep)
// PushIon (earthcmi.F90:524-606): the first nIonP shells' velocity pushed toward the (zero) E x B drift
__global__ void k_push_ion(Lay L, Par p, StateP S, const Scal* sc) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nI = p.msph.nIonP;
    if (t >= (long long)nI * L.Njp * L.Nkp) return;
    const int i = L.is() + (int)(t % nI);
    const long long q = t / nI;
    const int j = L.js() + (int)(q % L.Njp), k = L.ks() + (int)(q / L.Njp);
    const long long c = L.at(i, j, k);
    double U[5], W[5];
    loadCon(S, c, U);
    cellC2P(p, U, W);
    if (U[0] < 0.0) return;
    const int dN = i - L.is() + 1;
    const double dt = dmin(sc->dt / (dN * p.msph.dtCpl), 1.0);
    for (int v = 1; v <= 3; ++v) W[v] = W[v] + dt * (0.0 - W[v]);
    cellP2C(p, W, U);
    storeCon(S, c, U);
}
// NudgeSW (apps/wind.F90:392-447): the outermost active shell nudged toward the wind over one minute
__global__ void k_nudge_sw(Lay L, Par p, GridP g, StateP S, const Scal* sc) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Njp * L.Nkp) return;
    const int j = L.js() + (int)(t % L.Njp), k = L.ks() + (int)(t / L.Njp);
    const long long c = L.at(L.ie(), j, k);
    const MsphPar& m = p.msph;
    double xcc[3] = {g.xyzcc[0][c], g.xyzcc[1][c], g.xyzcc[2][c]};
    const double wSW = wgtWind(m, xcc);
    if (!(wSW > TINY)) return;
    const double dt = sc->dt;
    const double dtSW = dmax((60.0 / m.gT0) / wSW, dt);
    const double gW_sw[5] = {m.wD, m.wV[0], m.wV[1], m.wV[2], m.wP};
    double U[5], W[5], gW[5];
    loadCon(S, c, U);
    cellC2P(p, U, W);
    for (int v = 0; v < 5; ++v) gW[v] = W[v] + (dt / dtSW) * (gW_sw[v] - W[v]);
    cellP2C(p, gW, U);
    storeCon(S, c, U);
}
// NudgeSW's back-of-grid fix (:449-484): the two rows at the axis end (je, je+1) of the last shell flow out
__global__ void k_nudge_ring(Lay L, Par p, StateP S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= 2LL * L.Nkp) return;
    const int nn = (int)(t % 2), k = L.ks() + (int)(t / 2);
    const long long c = L.at(L.ie(), L.je() + nn, k);
    if (!(S.gas[1][c] > 0)) return;
    double U[5], W[5], B[3] = {S.b[0][c], S.b[1][c], S.b[2][c]};
    loadCon(S, c, U);
    const double Cx = con2Fast(p, U, B);
    cellC2P(p, U, W);
    W[1] = -Cx;
    cellP2C(p, W, U);
    storeCon(S, c, U);
}

}  // namespace

// ------------------------------------------------------------------ launch helpers
void launch_msph_bcs(Handle& h, const StateP& s, cudaStream_t st) {
    const Lay& L = h.L;
    GridP g = h.gridP();
    for (int side = 0; side < 2; ++side) {
        if (h.p.bc[side] != (side == 0 ? BC_ION : BC_WIND)) continue;
        k_bc_ionwind<<<nblkM((long long)L.nG * (L.Nj + 1) * (L.Nk + 1), TB), TB, 0, st>>>(L, h.p, g, s, side);
        k_bc_ionwind_b<<<nblkM((long long)L.nG * L.Nj * L.Nk, TB), TB, 0, st>>>(L, h.p, g, s, side);
        k_bc_ionwind_bfix<<<nblkM((long long)L.nG * L.Nk, TB), TB, 0, st>>>(L, h.p, s, side);
        h.launches += 3;
    }
}
void launch_msph_efix(Handle& h, const StateP& nS, cudaStream_t st) {
    const Lay& L = h.L;
    GridP g = h.gridP();
    Vec3P E = {{h.E[0], h.E[1], h.E[2]}};
    if (h.p.bc[0] == BC_ION) { k_ion_efix<<<nblkM((long long)L.Nj * L.Nk, TB), TB, 0, st>>>(L, g, E); h.launches++; }
    if (h.p.bc[1] == BC_WIND) {
        Xyz3 X = {{h.xyz[0], h.xyz[1], h.xyz[2]}};
        k_wind_efix<<<nblkM(4LL * (L.Njp + 1) * (L.Nkp + 1), TB), TB, 0, st>>>(L, h.p, g, X, nS, E, h.dScal);
        h.launches++;
        if (h.p.doRing) { k_wind_efix_ring<<<1, 32, 0, st>>>(L, h.p, E); h.launches++; }
    }
    launch_fix_e_lfm(h, h.E, st);   // FixEFieldLFM, EFix's last call
}
void launch_ion_flux(Handle& h, cudaStream_t st) {
    if (h.p.bc[0] != BC_ION || !h.p.doRing) return;
    FluxOut<float> F32;
    FluxOut<double> F64;
    for (int v = 0; v < 5; ++v) { F32.g[v] = h.f32.gflx[0][v]; F64.g[v] = h.gflx[0][v]; }
    for (int x = 0; x < 3; ++x) { F32.m[x] = h.f32.mflx[0][x]; F64.m[x] = h.mflx[0][x]; }
    if (h.prec == PREC_FP32FLUX) k_ion_flux<float><<<1, 32, 0, st>>>(h.L, h.p, F32);
    else k_ion_flux<double><<<1, 32, 0, st>>>(h.L, h.p, F64);
    h.launches++;
}
void launch_apply_grav(Handle& h, const StateP& S, const StateP& O, cudaStream_t st) {
    if (!h.p.msph.doGrav) return;
    const Lay& L = h.L;
    Vec3P gx = {{h.gxyz[0], h.gxyz[1], h.gxyz[2]}};
    k_apply_grav<<<grid_plane(Reg{L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp}, TB), TB, 0, st>>>(L, h.p, gx, S, O, h.dScal);
    h.launches++;
}
void launch_msph_perstep(Handle& h, const StateP& S, cudaStream_t st) {
    const Lay& L = h.L;
    if (h.p.bc[0] == BC_ION && h.p.msph.doIonPush) {
        k_push_ion<<<nblkM((long long)h.p.msph.nIonP * L.Njp * L.Nkp, TB), TB, 0, st>>>(L, h.p, S, h.dScal);
        h.launches++;
    }
    if (h.p.bc[1] == BC_WIND) {
        k_nudge_sw<<<nblkM((long long)L.Njp * L.Nkp, TB), TB, 0, st>>>(L, h.p, h.gridP(), S, h.dScal);
        h.launches++;
        if (h.p.doRing && h.p.ringDoE) { k_nudge_ring<<<nblkM(2LL * L.Nkp, TB), TB, 0, st>>>(L, h.p, S); h.launches++; }
    }
}
int msph_kernels_per_step(const Handle& h) {
    if (!h.p.msph.on) return 0;
    int n = 0;
    for (int side = 0; side < 2; ++side) if (h.p.bc[side] == (side == 0 ? BC_ION : BC_WIND)) n += 3;
    n += (h.p.bc[0] == BC_ION) + (h.p.bc[1] == BC_WIND) * (1 + (h.p.doRing ? 1 : 0)) + 1;   // EFix
    n += (h.p.bc[0] == BC_ION && h.p.doRing) ? 1 : 0;                                         // IonFlux
    n += h.p.msph.doGrav ? 1 : 0;
    n += (h.p.bc[0] == BC_ION && h.p.msph.doIonPush) ? 1 : 0;
    n += (h.p.bc[1] == BC_WIND) ? 1 + ((h.p.doRing && h.p.ringDoE) ? 1 : 0) : 0;
    return n;
}
void launch_add_grav(Handle& h, double GM0, cudaStream_t st) {
    const Lay& L = h.L;
    Vec3P gx = {{h.gxyz[0], h.gxyz[1], h.gxyz[2]}};
    k_add_grav<<<nblkM((long long)L.Nip * L.Njp * L.Nkp, TB), TB, 0, st>>>(L, h.gridP(), GM0, gx);
    h.launches++;
}

}  // namespace gam
