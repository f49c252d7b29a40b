// CPU FP64 restatement of the GAMERA ideal-MHD step (kaiju v1.25.1) -- TEST INFRASTRUCTURE ONLY.
//
// This file is the oracle: the parity tests, the smoke check and the bench's CPU-baseline leg check the
// device results against it. The product path (kaiju_b200/csrc, libgamgpu.so) never links or calls it.
//
// It restates, routine by routine and in the Fortran evaluation order, the reference's
//   src/gamera/mhdgroup.F90   AdvanceMHD :16-76, applyUpdate :79-259, CellReynolds :263-297,
//                             CellMaxwell :300-330, CellBoris :337-442, Predictor :445-525,
//                             PredictCell :529-616, ExtrapAB2 :710-718
//   src/gamera/stress.F90     CalcStress :41-198, Fluxes :204-429, GasKinFlux :432-511, MagKinFlux :513-599
//   src/gamera/recon.F90      weights :22-32, BlockStateLRs :39-93, BlockLRs :96-122, Cen8LRs :125-158,
//                             Up7LRs :162-198, Central8 :202-214, pdmLR :231-272, PDM :275-301, Up7 :303-310
//   src/gamera/fields.F90     E2Flux :18-51, CalcElecField :70-232, Mom2Face :235-285, EdgeLRs :288-362,
//                             GetCornerB :365-424, GetCornerD :427-454, GetCornerV :457-517
//   src/gamera/gamutils.F90   gamLoadBlock/gamLoadBlockI :63-130, CellC2P :301-321, CellP2C :362-383
//   src/gamera/gridutils.F90  CellDT :49-106, GasIC2State :144-189, VectorPot2Flux :193-237,
//                             bFlux2Fld :281-301, gamCellBxyz :648-680, DivB :717-770
//   src/gamera/step.F90       EnforceBCs :17-55, CalcDT :58-168
//   src/gamera/bcs.F90        periodic :279-450, zeroGrad :799-930
//   src/gamera/init.F90       CalcGridInfo :150-260, initModel defaults :312-492, SetDomain :519-538,
//                             genGridXML :572-798, Corners2Grid :801-1080, ebGeom :1083-1145
//   src/gamera/quadrature.F90 Gauss-Legendre 12-point tables :9-26, GaussianVolumeIntegral :42-100,
//                             GaussianFaceIntegral :159-221, GaussianEdgeIntegral :345-370, faceDeltas :373-389
//   src/gamera/metric.F90     faceCoords :79-108, cellCoords :133-148, CellDV/rVec/IdVec :298-328
//   src/gamera/prob.F90       initOT2D :74-119, initBW :190-298
//   src/base/math.F90         cross :265-274, normVec :332-343, Vec2Para/Perp :364-376, DetJ :470-478
//   src/gamera/gamapp.F90     stepGamera :73-94, UpdateStateData :96-116
//
// Build: -O2 -fno-fast-math -ffp-contract=off (no FMA contraction, no reassociation).
// Assumptions written down where Fortran leaves the compiler a choice:
//   * x**2.0 is evaluated as x*x (gfortran lowers real exponents equal to 2 that way);
//   * NORM2 follows gfortran's scaled sum-of-squares expansion;
//   * DOT_PRODUCT is a left-to-right sum starting from zero;
//   * real(4) literals (0.3 MaxCFL, sqrt(2.0) in initBW) keep their single-precision values.
// Parity against the reference binary itself is not pinned (no Fortran compiler is available); the
// restatement is pinned by the reference's known-answer tests (testgamutils.pf, testmetric.pf) and the
// property tests of tests/cases/testCases.pf.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const double PI = 3.14159265358979323846264338327950288;   // kdefs.F90:21 (4*atan(1))
static const double TINY = 1.0e-12, HUGEV = 1.0e12;                 // kdefs.F90:23
enum { NVAR = 5, NDIM = 3, recLen = 8, limLen = 4, vecLen = 16, Nr2 = 4, Nl2 = 2 };
enum { DEN = 1, MOMX, MOMY, MOMZ, ENERGY };
enum { VELX = 2, VELY, VELZ, PRESSURE };
enum { XDIR = 1, YDIR, ZDIR };
enum { IDIR = 1, JDIR, KDIR };
enum { NORMX = 1, NORMY, NORMZ, TAN1X, TAN1Y, TAN1Z, TAN2X, TAN2Y, TAN2Z };
enum { XNQI = 1, YNQI, XNQJ, YNQJ };
enum { INI = 1, OUTI, INJ, OUTJ, INK, OUTK };
// Boundary classes: periodic, zero-gradient, the LFM axis (lfmIn/lfmOut, bcs.F90:1020-1106) for INJ/OUTJ,
// and the LFM blast-wave problem's fixed inner/outer shells (ICs/lfmbw.F90:141-249) for INI/OUTI
// BC_HALO: a tile face inside a decomposed domain (no physical BC; gamapp_mpi.F90's halo exchange fills
// the ghosts, and the dt domain takes no ghost layer there, init.F90:519-538)
// BC_ION / BC_WIND: the magnetosphere's ionospheric inner boundary (IonInner, voltron/ICs/earthcmi.F90:378-522)
// and solar-wind outer boundary (WindBC, apps/wind.F90:206-374)
enum { BC_PERIODIC = 0, BC_ZEROGRAD = 1, BC_LFMPOLE = 2, BC_LFMBW = 3, BC_HALO = 4, BC_ION = 5, BC_WIND = 6 };
enum { SPOLE = 1, EPOLE = 2 };
enum { RR_PLM = 0, RR_PPM = 1, RR_PCM = 2, RR_WENO = 3 };
static const int NFTMAX = 2;

// Ring-average configuration for an LFM-type grid (ringutils.F90:37-226, Model%Ring)
struct Ring {
    int NumR = 0;
    int Nch[32] = {0};
    int Np = 0, nSi = 0, nSe = 0;
    bool doS = true, doE = true, doMassRA = false;
    int recon = RR_PPM;                 // ring/rngrec (init.F90:466-478)
    int NFTMAG = 1;                     // Fourier modes removed from the face fluxes
    bool doCleanLoop = true, doFastLoop = true;
};
enum { RM_8CENT = 0, RM_7UP = 1 };

static inline int ijkD(int a, int b) { return a == b ? 1 : 0; }

// Fortran-ordered array with arbitrary lower bounds (column-major, first index fastest).
struct Arr {
    std::vector<double> d;
    int lb[5] = {0, 0, 0, 0, 0};
    int n[5] = {1, 1, 1, 1, 1};
    long st[5] = {1, 1, 1, 1, 1};
    void alloc(int nd, const int* lo, const int* hi) {
        long s = 1;
        for (int a = 0; a < 5; ++a) {
            if (a < nd) { lb[a] = lo[a]; n[a] = hi[a] - lo[a] + 1; } else { lb[a] = 0; n[a] = 1; }
            st[a] = s; s *= n[a];
        }
        d.assign((size_t)s, 0.0);
    }
    long size() const { return (long)d.size(); }
    double* data() { return d.data(); }
    inline long off(int i, int j, int k, int l = 0, int m = 0) const {
        return (long)(i - lb[0]) + st[1] * (j - lb[1]) + st[2] * (k - lb[2]) + st[3] * (l - lb[3]) + st[4] * (m - lb[4]);
    }
    inline double& operator()(int i, int j, int k) { return d[off(i, j, k, lb[3], lb[4])]; }
    inline double& operator()(int i, int j, int k, int l) { return d[off(i, j, k, l, lb[4])]; }
    inline double& operator()(int i, int j, int k, int l, int m) { return d[off(i, j, k, l, m)]; }
    inline double operator()(int i, int j, int k) const { return d[off(i, j, k, lb[3], lb[4])]; }
    inline double operator()(int i, int j, int k, int l) const { return d[off(i, j, k, l, lb[4])]; }
    inline double operator()(int i, int j, int k, int l, int m) const { return d[off(i, j, k, l, m)]; }
};

struct Model {
    int nSpc = 0, nG = 4;
    double CFL = 0.3, gamma = 5.0 / 3.0, Vd0 = 0.5;
    double t = 0.0, tFin = 1.0, dt = 0.0, dt0 = 0.0;
    bool fixedTimestep = false;
    int ts = 0;
    bool doMHD = true, do25D = false, doBoris = false, doHogs = true, doLFMLim = true;
    double cHogH = 0.25, cHogM = 0.25, Ca = HUGEV;
    double limDT0 = 1.0e-3;
    double pdmb = 0.75, dFloor = TINY, pFloor = TINY;
    int rmeth = RM_8CENT;
    int status = 0;   // bit0: disaster (dt<=TINY or no dt<HUGE), bit1: bad (10x drop / limDT0)
    bool doBackground = false;
    bool doRing = false;
    Ring R;
    bool predFixLFM = false;   // the LFM blast-wave problem's HackPredictor (ICs/lfmbw.F90:227-248)
    double bwD0 = 1.0, bwP0 = 0.1;   // its fixed-shell gas state (prob/D0, prob/P0)
    // gravity (Model%doGrav, doSphGrav; background.F90:170-252, mhdgroup.F90:620-705)
    bool doGrav = false, doSphGrav = false;
    // the magnetosphere problem's hooks (voltron/ICs/earthcmi.F90 initUser): HackE = EFix, HackFlux = IonFlux,
    // HackStep = PerStep, with a constant solar wind and no ionospheric coupling (inExyz = inEijk = 0)
    struct Msph {
        bool on = false;
        double M0 = 0.0, GM0 = 0.0;   // dipole moment and gravity coefficient in code units (setMagsphere)
        double rCut = 16.0, lCut = 8.0, dcScl = 4.0;   // cut dipole (msphutils.F90:47-50)
        double xSun = 20.0, xTail = -225.0, yMax = 75.0, sInner = 0.96;   // initial-field cut (:440-444)
        double wD = 0.0, wP = 0.0, wV[3] = {0, 0, 0}, wB[3] = {0, 0, 0};   // the wind, code units
        double dtCpl = 0.0;   // PushIon coupling time scale (ibc dtCpl, earthcmi.F90:368-369)
        double gT0 = 1.0;     // the time unit in seconds (NudgeSW's one-minute nudge time)
        int nIonP = 1;        // ibc/nIonP
        bool doIonPush = true;
    } W;
};

struct Grid {
    int Nip, Njp, Nkp, Ni, Nj, Nk;
    int is, ie, js, je, ks, ke, isg, ieg, jsg, jeg, ksg, keg;
    int isDT, ieDT, jsDT, jeDT, ksDT, keDT;
    Arr xyz, xyzcc, xfc, di, dj, dk, volume, Tf, Te, Teb, face, edge;
    Arr fcB0, edgB0, B0, bFlux0, dpB0;   // background field (background.F90:20-167), cell-sized arrays
    Arr gxyz;                            // gravitational acceleration (AddGrav, background.F90:170-252)
    int bc[6] = {BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC};
};

struct State {
    double time = 0.0;
    Arr Gas, magFlux, Efld, Bxyz;
};

struct Solver {
    Arr gFlx, mFlx, Vf, dGasH, dGasM;
    Arr SmoothE;   // ring-average smoothing E field (ringav.F90:30)
    State StateHf;
};

struct App {
    Model M;
    Grid G;
    State S, oS;
    Solver V;
};

// ---------------------------------------------------------------- helpers (math.F90, gfortran intrinsics)
static inline double sq(double x) { return x * x; }   // x**2.0
static inline double fsign1(double b) { return std::copysign(1.0, b); }  // sign(1.0_rp,b)
static inline double fmaxd(double a, double b) { return (a > b) ? a : b; }
static inline double fmind(double a, double b) { return (a < b) ? a : b; }

// gfortran NORM2: scaled sum of squares (avoids overflow), then scale*sqrt(ssq).
static double norm2v(const double* a, int n) {
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        if (a[i] != 0.0) {
            double ax = std::fabs(a[i]);
            if (scale < ax) { ssq = 1.0 + ssq * sq(scale / ax); scale = ax; }
            else { ssq = ssq + sq(ax / scale); }
        }
    }
    return scale * std::sqrt(ssq);
}
static inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot(const double* a, const double* b, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
    return s;
}

// recon.F90:22-32 weights, initialised from integers / 840 so the sum is exactly one
static double interpWgt[8], interpWgt6[8], Up7C[7];
static void initWeights() {
    const int w8[8] = {-3, 29, -139, 533, 533, -139, 29, -3};
    const int w6[8] = {0, 1, -8, 37, 37, -8, 1, 0};
    const int u7[7] = {-3, 25, -101, 319, 214, -38, 4};
    for (int n = 0; n < 8; ++n) { interpWgt[n] = (double)w8[n] / 840.0; interpWgt6[n] = (double)w6[n] / 60.0; }
    for (int n = 0; n < 7; ++n) Up7C[n] = (double)u7[n] / 420.0;
}

// ---------------------------------------------------------------- cell conversions (gamutils.F90)
static void CellC2P(const Model& M, const double* Con, double* Prim) {  // gamutils.F90:301-321
    double rho = Con[0];
    double Vx = Con[1] / rho, Vy = Con[2] / rho, Vz = Con[3] / rho;
    double E = Con[4];
    double KinE = 0.5 * rho * (sq(Vx) + sq(Vy) + sq(Vz));
    Prim[0] = fmaxd(rho, M.dFloor);
    Prim[1] = Vx; Prim[2] = Vy; Prim[3] = Vz;
    Prim[4] = fmaxd((M.gamma - 1) * (E - KinE), M.pFloor);
}
static void CellP2C(const Model& M, const double* Prim, double* Con) {  // gamutils.F90:362-383
    double rho = fmaxd(Prim[0], M.dFloor);
    double Vx = Prim[1], Vy = Prim[2], Vz = Prim[3];
    double IntE = fmaxd(Prim[4], M.pFloor) / (M.gamma - 1);
    double KinE = 0.5 * rho * (sq(Vx) + sq(Vy) + sq(Vz));
    Con[0] = rho; Con[1] = rho * Vx; Con[2] = rho * Vy; Con[3] = rho * Vz; Con[4] = IntE + KinE;
}

// ---------------------------------------------------------------- block loaders (gamutils.F90:63-130)
// Qb(vecLen, -Nx2:Nx2-1) stored as Qb[n+Nx2][i]; zero beyond iMax.
static void loadBlock(const Grid& G, double (*Qb)[vecLen], const double* Q, int iS, int j, int k, int iMax,
                      int d, int Nx2, bool iface) {
    long nSi = 1, nSj, nSk;
    long l0;
    if (iface) {
        nSj = G.Ni + 1; nSk = (long)(G.Ni + 1) * (G.Nj + 1);
        l0 = (iS - G.isg) + nSj * (j - G.jsg) + nSk * (k - G.ksg);
    } else {
        nSj = G.Ni; nSk = (long)G.Ni * G.Nj;
        l0 = (iS - G.isg) + nSj * (j - G.jsg) + nSk * (k - G.ksg);
    }
    long nSt = nSi * ijkD(d, IDIR) + nSj * ijkD(d, JDIR) + nSk * ijkD(d, KDIR);
    for (int n = -Nx2; n <= Nx2 - 1; ++n) {
        long l = l0 + nSt * n;
        for (int i = 0; i < vecLen; ++i) Qb[n + Nx2][i] = (i < iMax) ? Q[l + i] : 0.0;
    }
}

// ---------------------------------------------------------------- reconstruction (recon.F90)
static double pdmb_g = 0.75;

static void pdmLR(const double (*Qb)[vecLen], const double* Qi, double* Ql, double* Qr) {  // recon.F90:231-272
    for (int i = 0; i < vecLen; ++i) {
        double v0 = Qb[0][i], v1 = Qb[1][i], v2 = Qb[2][i], v3 = Qb[3][i];
        double maxV = fmaxd(v1, v2), minV = fmind(v1, v2);
        double vN = fmaxd(minV, fmind(Qi[i], maxV));
        double dv0 = pdmb_g * (v1 - v0), dv1 = pdmb_g * (v2 - v1), dv2 = pdmb_g * (v3 - v2);
        double s0 = fsign1(dv0), s1 = fsign1(dv1), s2 = fsign1(dv2);
        double q0 = std::fabs(s0 + s1), q1 = std::fabs(s1 + s2);
        double dvL = vN - v1, dvR = v2 - vN;
        Ql[i] = vN - s1 * fmaxd(0.0, std::fabs(dvL) - q0 * std::fabs(dv0));
        Qr[i] = vN + s1 * fmaxd(0.0, std::fabs(dvR) - q1 * std::fabs(dv2));
    }
}
static double PDM(double q0, double q1, double q2, double qI) {  // recon.F90:275-301
    double maxQ = fmaxd(q1, q2), minQ = fmind(q1, q2);
    double qN = fmaxd(minQ, fmind(qI, maxQ));
    double dq0 = pdmb_g * (q1 - q0), dq1 = pdmb_g * (q2 - q1);
    double s0 = fsign1(dq0), s1 = fsign1(dq1);
    double s01 = std::fabs(s0 + s1);
    double dqL = qN - q1;
    return qN - s1 * fmaxd(0.0, std::fabs(dqL) - s01 * std::fabs(dq0));
}
static double Up7(double q0, double q1, double q2, double q3, double q4, double q5, double q6) {  // recon.F90:303-310
    return q0 * Up7C[0] + q1 * Up7C[1] + q2 * Up7C[2] + q3 * Up7C[3] + q4 * Up7C[4] + q5 * Up7C[5] + q6 * Up7C[6];
}
static void Central8(const double (*Qb)[vecLen], double* Qi) {  // recon.F90:202-214
    for (int i = 0; i < vecLen; ++i) {
        double s = 0.0;
        for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * Qb[n][i];
        Qi[i] = s;
    }
}
// GetLRs: Cen8LRs (recon.F90:125-158) or Up7LRs (:162-198)
static void GetLRs(int rmeth, const double (*dV)[vecLen], const double (*nQ)[vecLen], const double (*Q)[vecLen],
                   const double* Vi, double* Ql, double* Qr) {
    double QdV[recLen][vecLen];
    for (int n = 0; n < recLen; ++n)
        for (int i = 0; i < vecLen; ++i) QdV[n][i] = dV[n][i] * Q[n][i];
    if (rmeth == RM_8CENT) {
        double Qi[vecLen];
        Central8(QdV, Qi);
        for (int i = 0; i < vecLen; ++i) Qi[i] = Qi[i] / Vi[i];
        pdmLR(nQ, Qi, Ql, Qr);
    } else {
        for (int i = 0; i < vecLen; ++i) {
            Ql[i] = Up7(QdV[0][i], QdV[1][i], QdV[2][i], QdV[3][i], QdV[4][i], QdV[5][i], QdV[6][i]) / Vi[i];
            Qr[i] = Up7(QdV[7][i], QdV[6][i], QdV[5][i], QdV[4][i], QdV[3][i], QdV[2][i], QdV[1][i]) / Vi[i];
            Ql[i] = PDM(nQ[0][i], nQ[1][i], nQ[2][i], Ql[i]);
            Qr[i] = PDM(nQ[3][i], nQ[2][i], nQ[1][i], Qr[i]);
        }
    }
}
// BlockLRs (recon.F90:96-122): Qb[nv][n][i]
static void BlockLRs(int rmeth, const double (*VolB)[vecLen], const double (*nQb)[limLen][vecLen],
                     const double (*Qb)[recLen][vecLen], double (*Ql)[vecLen], double (*Qr)[vecLen], int NumV) {
    double Vi[vecLen];
    Central8(VolB, Vi);
    for (int nv = 0; nv < NumV; ++nv) GetLRs(rmeth, VolB, nQb[nv], Qb[nv], Vi, Ql[nv], Qr[nv]);
}
// BlockCon2Prim (recon.F90:66-92)
static void BlockCon2Prim(const Model& M, const double (*inCon)[vecLen], double (*oPrim)[vecLen], int xLen,
                          int stride /* per-variable stride in rows */) {
    // inCon[nv*stride + n][i]
    for (int n = 0; n < xLen; ++n)
        for (int i = 0; i < vecLen; ++i) {
            double D = fmaxd(inCon[0 * stride + n][i], M.dFloor);
            double Mx = inCon[1 * stride + n][i], My = inCon[2 * stride + n][i], Mz = inCon[3 * stride + n][i];
            double E = inCon[4 * stride + n][i];
            double KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) / D;
            double P = fmaxd((M.gamma - 1) * (E - KinE), M.pFloor);
            oPrim[0 * stride + n][i] = D;
            oPrim[1 * stride + n][i] = Mx / D;
            oPrim[2 * stride + n][i] = My / D;
            oPrim[3 * stride + n][i] = Mz / D;
            oPrim[4 * stride + n][i] = P;
        }
}

// ---------------------------------------------------------------- kinetic fluxes (stress.F90)
static const int SgnLR[2] = {-1, 1};

static void GasKinFlux(const Model& M, int q, const double (*Prim)[vecLen], const double (*TfB)[vecLen],
                       double (*gFlxB)[vecLen], double (*dW)[vecLen]) {  // stress.F90:432-511
    double sg = (double)SgnLR[q];
    for (int i = 0; i < vecLen; ++i) {
        double D = Prim[0][i], P = Prim[4][i], Vx = Prim[1][i], Vy = Prim[2][i], Vz = Prim[3][i];
        double E = 0.5 * D * (sq(Vx) + sq(Vy) + sq(Vz)) + P / (M.gamma - 1);
        double lambda = D / (2 * P);
        double Vn = TfB[NORMX - 1][i] * Vx + TfB[NORMY - 1][i] * Vy + TfB[NORMZ - 1][i] * Vz;
        double Vt1 = TfB[TAN1X - 1][i] * Vx + TfB[TAN1Y - 1][i] * Vy + TfB[TAN1Z - 1][i] * Vz;
        double Vt2 = TfB[TAN2X - 1][i] * Vx + TfB[TAN2Y - 1][i] * Vy + TfB[TAN2Z - 1][i] * Vz;
        double Vn0 = 0.5 * std::erfc(sg * std::sqrt(lambda) * Vn);
        double Vn1 = Vn * Vn0 - 0.5 * sg * std::exp(-(lambda * Vn * Vn)) / std::sqrt(PI * lambda);
        gFlxB[DEN - 1][i] = gFlxB[DEN - 1][i] + D * Vn1;
        gFlxB[ENERGY - 1][i] = gFlxB[ENERGY - 1][i] + (E + 0.5 * P) * Vn1 + 0.5 * P * Vn0 * Vn;
        double fMn = D * Vn * Vn1 + P * Vn0;
        double fMt1 = D * Vt1 * Vn1;
        double fMt2 = D * Vt2 * Vn1;
        double fMx = TfB[NORMX - 1][i] * fMn + TfB[TAN1X - 1][i] * fMt1 + TfB[TAN2X - 1][i] * fMt2;
        double fMy = TfB[NORMY - 1][i] * fMn + TfB[TAN1Y - 1][i] * fMt1 + TfB[TAN2Y - 1][i] * fMt2;
        double fMz = TfB[NORMZ - 1][i] * fMn + TfB[TAN1Z - 1][i] * fMt1 + TfB[TAN2Z - 1][i] * fMt2;
        gFlxB[MOMX - 1][i] = gFlxB[MOMX - 1][i] + fMx;
        gFlxB[MOMY - 1][i] = gFlxB[MOMY - 1][i] + fMy;
        gFlxB[MOMZ - 1][i] = gFlxB[MOMZ - 1][i] + fMz;
        dW[DEN - 1][i] = dW[DEN - 1][i] + sg * D;
        dW[MOMX - 1][i] = dW[MOMX - 1][i] + sg * D * Vx;
        dW[MOMY - 1][i] = dW[MOMY - 1][i] + sg * D * Vy;
        dW[MOMZ - 1][i] = dW[MOMZ - 1][i] + sg * D * Vz;
        dW[ENERGY - 1][i] = dW[ENERGY - 1][i] + sg * E;
    }
}

static void MagKinFlux(const Model& M, int q, const double (*Prim)[vecLen], const double (*Mag)[vecLen],
                       const double* Bn, const double (*TfB)[vecLen], double (*mFlxB)[vecLen], double* bbD,
                       double* VaD, const double (*B0)[vecLen], const double* B0n) {  // stress.F90:513-599
    double sg = (double)SgnLR[q];
    for (int i = 0; i < vecLen; ++i) {
        double D = Prim[0][i], P = Prim[4][i];
        double Bx = Mag[0][i], By = Mag[1][i], Bz = Mag[2][i];
        double B0x = B0[0][i], B0y = B0[1][i], B0z = B0[2][i];
        double dPb = 0.5 * (sq(Bx) + sq(By) + sq(Bz));
        double Va2;
        if (M.doBackground) {
            Va2 = (sq(Bx + B0x) + sq(By + B0y) + sq(Bz + B0z)) / D;
            bbD[i] = bbD[i] + 0.5 * (sq(Bx + B0x) + sq(By + B0y) + sq(Bz + B0z));
        } else {
            Va2 = 2 * dPb / D;
            bbD[i] = bbD[i] + 0.5 * (sq(Bx) + sq(By) + sq(Bz));
        }
        double Vac2;
        if (M.doBoris) Vac2 = Va2 / (1 + (Va2 / sq(M.Ca)));
        else Vac2 = Va2;
        double Vx = Prim[1][i], Vy = Prim[2][i], Vz = Prim[3][i];
        double Nx = TfB[NORMX - 1][i], Ny = TfB[NORMY - 1][i], Nz = TfB[NORMZ - 1][i];
        double Vn = Nx * Vx + Ny * Vy + Nz * Vz;
        double lambda = 1 / (2 * P / D + Vac2);
        double Vn0 = 0.5 * std::erfc(sg * std::sqrt(lambda) * Vn);
        VaD[i] = VaD[i] + 0.5 * std::sqrt(Vac2);
        mFlxB[0][i] = mFlxB[0][i] + Vn0 * (dPb * Nx - Bx * Bn[i]);
        mFlxB[1][i] = mFlxB[1][i] + Vn0 * (dPb * Ny - By * Bn[i]);
        mFlxB[2][i] = mFlxB[2][i] + Vn0 * (dPb * Nz - Bz * Bn[i]);
        if (M.doBackground) {
            double BdB0 = B0x * Bx + B0y * By + B0z * Bz;
            mFlxB[0][i] = mFlxB[0][i] + Vn0 * (-B0x * Bn[i] - Bx * B0n[i] + BdB0 * Nx);
            mFlxB[1][i] = mFlxB[1][i] + Vn0 * (-B0y * Bn[i] - By * B0n[i] + BdB0 * Ny);
            mFlxB[2][i] = mFlxB[2][i] + Vn0 * (-B0z * Bn[i] - Bz * B0n[i] + BdB0 * Nz);
        }
    }
}

// Fluxes (stress.F90:204-429) for one brick (iB:iB+vecLen-1, j, k) in direction dN
static void Fluxes(const Model& M, const Grid& G, const State& nS, const State& hS, int iB, int j, int k, int dN,
                   Arr& gFlx, Arr& mFlx) {
    double VolB[recLen][vecLen];
    double ConB[NVAR][recLen][vecLen];
    double MagB[NDIM][recLen][vecLen];
    double TfB[9][vecLen];
    double faB[vecLen];
    double nConB[NVAR][limLen][vecLen];
    double nMagB[NDIM][limLen][vecLen];
    double PrimL[NVAR][vecLen], PrimR[NVAR][vecLen], MagL[NDIM][vecLen], MagR[NDIM][vecLen];
    double gFlxB[NVAR][vecLen], mFlxB[NDIM][vecLen], dW[NVAR][vecLen], VaD[vecLen], Bn[vecLen], bbD[vecLen];
    double B0[NDIM][vecLen], B0n[vecLen];

    int ie = G.ie + ijkD(dN, IDIR);
    int iMax = std::min((int)vecLen, ie - iB + 1);
    int isB = iB;
    std::memset(gFlxB, 0, sizeof gFlxB); std::memset(mFlxB, 0, sizeof mFlxB); std::memset(dW, 0, sizeof dW);
    std::memset(VaD, 0, sizeof VaD); std::memset(bbD, 0, sizeof bbD); std::memset(TfB, 0, sizeof TfB);
    std::memset(Bn, 0, sizeof Bn); std::memset(faB, 0, sizeof faB);
    std::memset(B0, 0, sizeof B0); std::memset(B0n, 0, sizeof B0n);

    loadBlock(G, VolB, G.volume.d.data(), iB, j, k, iMax, dN, Nr2, false);
    for (int i = 0; i < iMax; ++i) {
        for (int c = 0; c < 9; ++c) TfB[c][i] = G.Tf(isB + i, j, k, c + 1, dN);
        faB[i] = G.face(isB + i, j, k, dN);
    }
    const long cellN = (long)G.Ni * G.Nj * G.Nk;
    const long faceN = (long)(G.Ni + 1) * (G.Nj + 1) * (G.Nk + 1);
    if (M.doMHD) {
        for (int nv = 0; nv < NDIM; ++nv) {
            loadBlock(G, MagB[nv], hS.Bxyz.d.data() + nv * cellN, iB, j, k, iMax, dN, Nr2, false);
            const State& lS = M.doLFMLim ? nS : hS;
            loadBlock(G, nMagB[nv], lS.Bxyz.d.data() + nv * cellN, iB, j, k, iMax, dN, Nl2, false);
        }
        BlockLRs(M.rmeth, VolB, nMagB, MagB, MagL, MagR, NDIM);
        for (int i = 0; i < iMax; ++i) Bn[i] = hS.magFlux(isB + i, j, k, dN) / faB[i];
        if (M.doBackground) {
            for (int i = 0; i < iMax; ++i) {
                for (int c = 0; c < 3; ++c) B0[c][i] = G.fcB0(isB + i, j, k, c + 1, dN);
                B0n[i] = G.bFlux0(isB + i, j, k, dN) / faB[i];
            }
        }
        (void)faceN;
    }
    for (int nv = 0; nv < NVAR; ++nv) {
        loadBlock(G, ConB[nv], hS.Gas.d.data() + nv * cellN, iB, j, k, iMax, dN, Nr2, false);
        const State& lS = M.doLFMLim ? nS : hS;
        loadBlock(G, nConB[nv], lS.Gas.d.data() + nv * cellN, iB, j, k, iMax, dN, Nl2, false);
    }
    // BlockStateLRs (recon.F90:39-93)
    {
        double PrimB[NVAR][recLen][vecLen], nPrimB[NVAR][limLen][vecLen];
        BlockCon2Prim(M, &nConB[0][0], &nPrimB[0][0], limLen, limLen);
        BlockCon2Prim(M, &ConB[0][0], &PrimB[0][0], recLen, recLen);
        BlockLRs(M.rmeth, VolB, nPrimB, PrimB, PrimL, PrimR, NVAR);
    }
    if (M.doMHD) {
        MagKinFlux(M, 0, PrimL, MagL, Bn, TfB, mFlxB, bbD, VaD, B0, B0n);
        MagKinFlux(M, 1, PrimR, MagR, Bn, TfB, mFlxB, bbD, VaD, B0, B0n);
        if (M.doBoris) {
            for (int i = 0; i < iMax; ++i) {
                double deeV[3], deeP[3];
                for (int c = 0; c < 3; ++c) deeV[c] = PrimR[1 + c][i] - PrimL[1 + c][i];
                for (int c = 0; c < 3; ++c) deeP[c] = bbD[i] * deeV[c] / sq(M.Ca);
                for (int c = 0; c < 3; ++c) mFlxB[c][i] = mFlxB[c][i] - M.cHogM * VaD[i] * deeP[c];
            }
        }
        for (int nv = 0; nv < NDIM; ++nv)
            for (int i = 0; i < iMax; ++i) mFlx(isB + i, j, k, nv + 1, dN) = faB[i] * mFlxB[nv][i];
    }
    std::memset(gFlxB, 0, sizeof gFlxB); std::memset(dW, 0, sizeof dW);
    GasKinFlux(M, 0, PrimL, TfB, gFlxB, dW);
    GasKinFlux(M, 1, PrimR, TfB, gFlxB, dW);
    for (int nv = 0; nv < NVAR; ++nv)
        for (int i = 0; i < iMax; ++i) {
            double alphaS = 1.0;
            gFlxB[nv][i] = gFlxB[nv][i] - alphaS * M.cHogH * VaD[i] * dW[nv][i];
        }
    if (M.doBoris) {  // nuclear option (stress.F90:399-417), cLim = 1.5 (single precision literal)
        const double cLim = 1.5;
        for (int i = 0; i < iMax; ++i) {
            double a[3] = {PrimL[1][i], PrimL[2][i], PrimL[3][i]}, b[3] = {PrimR[1][i], PrimR[2][i], PrimR[3][i]};
            double vL = norm2v(a, 3), vR = norm2v(b, 3);
            double Vn = std::sqrt(sq(vL) + sq(vR)) / (double)std::sqrt(2.0f);
            if (Vn >= cLim * M.Ca) {
                for (int nv = 0; nv < NVAR; ++nv) {
                    double dCon = ConB[nv][Nr2][i] - ConB[nv][Nr2 - 1][i];
                    gFlxB[nv][i] = gFlxB[nv][i] - M.Ca * dCon;
                }
            }
        }
    }
    for (int nv = 0; nv < NVAR; ++nv)
        for (int i = 0; i < iMax; ++i) gFlx(isB + i, j, k, nv + 1, dN) = faB[i] * gFlxB[nv][i];
}

// RingFlux (ringutils.F90:663-680): no flux through the faces on the axis; FixGasFluxLFM
// (gamdebug.F90:91-124) makes the K fluxes at ks and ke+1 agree
static void RingFlux(const Model& M, const Grid& G, Arr& gFlx, Arr& mFlx) {
    auto zeroJ = [&](int j) {
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int i = G.isg; i <= G.ieg; ++i) {
                for (int v = 1; v <= NVAR; ++v) gFlx(i, j, k, v, JDIR) = 0.0;
                if (M.doMHD)
                    for (int c = 1; c <= NDIM; ++c) mFlx(i, j, k, c, JDIR) = 0.0;
            }
    };
    if (M.R.doS) zeroJ(G.js);
    if (M.R.doE) zeroJ(G.je + 1);
    if (!M.doMHD) return;
    for (int j = G.js; j <= G.je; ++j)
        for (int i = G.is; i <= G.ie; ++i) {
            for (int v = 1; v <= NVAR; ++v) {
                double gF = 0.5 * (gFlx(i, j, G.ks, v, KDIR) + gFlx(i, j, G.ke + 1, v, KDIR));
                gFlx(i, j, G.ks, v, KDIR) = gF;
                gFlx(i, j, G.ke + 1, v, KDIR) = gF;
            }
            for (int c = 1; c <= NDIM; ++c) {
                double mF = 0.5 * (mFlx(i, j, G.ks, c, KDIR) + mFlx(i, j, G.ke + 1, c, KDIR));
                mFlx(i, j, G.ks, c, KDIR) = mF;
                mFlx(i, j, G.ke + 1, c, KDIR) = mF;
            }
        }
}

// IonFlux, the magnetosphere's HackFlux (voltron/ICs/earthcmi.F90:282-331): the I fluxes of the first shell at
// the two cells next to the axis (js, je) replaced by their average over k
static void IonFlux(const Model& M, const Grid& G, Arr& gFlx, Arr& mFlx) {
    if (!M.doRing) return;
    const int Np = M.R.Np;
    auto avg = [&](int j) {
        double im[3] = {0, 0, 0}, ig[5] = {0, 0, 0, 0, 0};
        for (int c = 1; c <= 3; ++c) {
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; ++k) s = s + mFlx(G.is, j, k, c, IDIR);
            im[c - 1] = s / Np;
        }
        for (int v = 1; v <= NVAR; ++v) {
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; ++k) s = s + gFlx(G.is, j, k, v, IDIR);
            ig[v - 1] = s / Np;
        }
        for (int k = G.ks; k <= G.ke; ++k) {
            for (int c = 1; c <= 3; ++c) mFlx(G.is, j, k, c, IDIR) = im[c - 1];
            for (int v = 1; v <= NVAR; ++v) gFlx(G.is, j, k, v, IDIR) = ig[v - 1];
        }
    };
    if (M.R.doE) avg(G.je);
    if (M.R.doS) avg(G.js);
}

static void CalcStress(const Model& M, const Grid& G, const State& nS, const State& hS, Arr& gFlx, Arr& mFlx,
                       Arr& dGasH, Arr& dGasM) {  // stress.F90:41-198
    int nFlx = NDIM, ks = G.ks, ke = G.ke;
    if (M.do25D) { nFlx = 2; ks = G.ks; ke = G.ks; }
    for (int d = 1; d <= nFlx; ++d) {
        if (d == IDIR) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = ks; k <= ke; ++k)
                for (int j = G.js; j <= G.je; ++j)
                    for (int iB = G.is; iB <= G.ie + 1; iB += vecLen) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
        } else if (d == JDIR) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = ks; k <= ke; ++k)
                for (int iB = G.is; iB <= G.ie; iB += vecLen)
                    for (int j = G.js; j <= G.je + 1; ++j) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
        } else {
#pragma omp parallel for collapse(2) schedule(static)
            for (int j = G.js; j <= G.je; ++j)
                for (int iB = G.is; iB <= G.ie; iB += vecLen)
                    for (int k = ks; k <= ke + 1; ++k) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
        }
    }
    if (M.doRing) RingFlux(M, G, gFlx, mFlx);   // stress.F90:134-139
    if (M.W.on) IonFlux(M, G, gFlx, mFlx);      // HackFlux, stress.F90:141-143
    bool doMaxwell = M.doMHD;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double dV = G.volume(i, j, k);
                for (int nv = 1; nv <= NVAR; ++nv)
                    dGasH(i, j, k, nv) = (gFlx(i, j, k, nv, IDIR) - gFlx(i + 1, j, k, nv, IDIR) + gFlx(i, j, k, nv, JDIR) -
                                          gFlx(i, j + 1, k, nv, JDIR) + gFlx(i, j, k, nv, KDIR) - gFlx(i, j, k + 1, nv, KDIR)) / dV;
                if (doMaxwell) {
                    for (int c = 1; c <= NDIM; ++c)
                        dGasM(i, j, k, c) = (mFlx(i, j, k, c, IDIR) - mFlx(i + 1, j, k, c, IDIR) + mFlx(i, j, k, c, JDIR) -
                                             mFlx(i, j + 1, k, c, JDIR) + mFlx(i, j, k, c, KDIR) - mFlx(i, j, k + 1, c, KDIR)) / dV;
                    if (M.doBackground)
                        for (int c = 1; c <= NDIM; ++c) dGasM(i, j, k, c) = dGasM(i, j, k, c) + G.dpB0(i, j, k, c);
                }
            }
}

// ---------------------------------------------------------------- LFM axis index maps (ringutils.F90:482-660)
static int WrapK(int k, int Np) {   // ringutils.F90:652-660
    int kp = k + Np / 2;
    if (kp > Np) kp = kp - Np;
    return kp;
}
// cell-centred conjugate across the axis (lfmIJKcc, ringutils.F90:482-514)
static void lfmIJKcc(const Model& M, const Grid& G, int i, int j, int k, int& ip, int& jp, int& kp) {
    int Np = G.Nkp;
    ip = i;
    if (k < G.ks) kp = k + Np;
    else if (k > G.ke) kp = k - Np;
    else kp = k;
    jp = j;
    if (M.R.doS && j < G.js) { jp = G.js + (G.js - j) - 1; kp = WrapK(kp, Np); }
    if (M.R.doE && j > G.je) { jp = G.je - (j - G.je) + 1; kp = WrapK(kp, Np); }
}
// face-centred conjugate (lfmIJKfc, ringutils.F90:517-575)
static void lfmIJKfc(const Model& M, const Grid& G, int d, int i, int j, int k, int& ip, int& jp, int& kp) {
    int Np = G.Nkp;
    ip = i;
    if (d == IDIR) { lfmIJKcc(M, G, i, j, k, ip, jp, kp); return; }
    kp = k;
    if (k < G.ks) kp = k + Np;
    if (d == JDIR && k > G.ke) kp = k - Np;
    if (d == KDIR && k > G.ke + 1) kp = k - Np;
    jp = j;
    if (d == JDIR) {
        if (M.R.doS && j < G.js) { jp = G.js + (G.js - j); kp = WrapK(k, Np); }
        if (M.R.doE && j > G.je + 1) { jp = G.je + 1 - (j - G.je) + 1; kp = WrapK(k, Np); }
    } else {
        if (M.R.doS && j < G.js) { jp = G.js + (G.js - j) - 1; kp = WrapK(k, Np); }
        if (M.R.doE && j > G.je) { jp = G.je - (j - G.je) + 1; kp = WrapK(k, Np); }
    }
}
// RingFlux2FieldFix (ringutils.F90:380-433): Bxyz of the cells across the axis from their conjugates
static void RingFlux2FieldFix(const Model& M, const Grid& G, Arr& B) {
    if (!M.doRing || (!M.R.doS && !M.R.doE)) return;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int i = G.isg; i <= G.ieg; ++i)
            for (int n = 1; n <= M.nG; ++n) {
                int ip, jp, kp;
                if (M.R.doS) {
                    int jg = G.js - n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) B(i, jg, k, c) = B(ip, jp, kp, c);
                }
                if (M.R.doE) {
                    int jg = G.je + n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) B(i, jg, k, c) = B(ip, jp, kp, c);
                }
            }
}

// ---------------------------------------------------------------- B from flux (gridutils.F90:281-301,648-680)
static void gamCellBxyz(const Grid& G, const Arr& mf, int i, int j, int k, double* B) {
    double dV = G.volume(i, j, k);
    double fI = mf(i, j, k, IDIR), fJ = mf(i, j, k, JDIR), fK = mf(i, j, k, KDIR);
    double fIp = mf(i + 1, j, k, IDIR), fJp = mf(i, j + 1, k, JDIR), fKp = mf(i, j, k + 1, KDIR);
    double Div = fIp - fI + fJp - fJ + fKp - fK;
    for (int c = 1; c <= 3; ++c) {
        double xfI = G.xfc(i, j, k, c, IDIR), xfJ = G.xfc(i, j, k, c, JDIR), xfK = G.xfc(i, j, k, c, KDIR);
        double xfIp = G.xfc(i + 1, j, k, c, IDIR), xfJp = G.xfc(i, j + 1, k, c, JDIR), xfKp = G.xfc(i, j, k + 1, c, KDIR);
        double b = (fIp * xfIp + fJp * xfJp + fKp * xfKp - fI * xfI - fJ * xfJ - fK * xfK) / dV;
        b = b - Div * G.xyzcc(i, j, k, c) / dV;
        B[c - 1] = b;
    }
}
static void bFlux2Fld(const Model& M, const Grid& G, const Arr& mf, Arr& B) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i) {
                double b[3];
                gamCellBxyz(G, mf, i, j, k, b);
                for (int c = 0; c < 3; ++c) B(i, j, k, c + 1) = b[c];
            }
    if (M.doRing) RingFlux2FieldFix(M, G, B);   // gridutils.F90:298-300
}

// ---------------------------------------------------------------- predictor (mhdgroup.F90:445-616)
static void Predictor(const Model& M, const Grid& G, const State& S, const State& oS, State& pS, double pdt) {
    double odt = S.time - oS.time;
    if (M.doMHD) {
        long N = S.magFlux.size();
#pragma omp parallel for schedule(static)
        for (long l = 0; l < N; ++l) {
            double Q = S.magFlux.d[l], oQ = oS.magFlux.d[l];
            double dQ = (Q - oQ) / odt;
            pS.magFlux.d[l] = Q + pdt * dQ;
        }
    }
    bFlux2Fld(M, G, pS.magFlux, pS.Bxyz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i) {
                double Q[5], oQ[5], W[5], oW[5], pW[5], pQ[5];
                for (int v = 0; v < 5; ++v) { Q[v] = S.Gas(i, j, k, v + 1); oQ[v] = oS.Gas(i, j, k, v + 1); }
                CellC2P(M, oQ, oW);
                CellC2P(M, Q, W);
                for (int v = 0; v < 5; ++v) { double dQ = (W[v] - oW[v]) / odt; pW[v] = W[v] + pdt * dQ; }
                pW[0] = fmaxd(pW[0], M.dFloor);
                pW[4] = fmaxd(pW[4], M.pFloor);
                CellP2C(M, pW, pQ);
                for (int v = 0; v < 5; ++v) pS.Gas(i, j, k, v + 1) = pQ[v];
            }
    if (M.predFixLFM) {   // HackPredictor of the LFM blast wave, PredFix (ICs/lfmbw.F90:227-248)
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int j = G.jsg; j <= G.jeg; ++j)
                for (int n = 1; n <= M.nG; ++n) {
                    int ig = G.is - n, ix, jp, kp;
                    lfmIJKcc(M, G, ig, j, k, ix, jp, kp);
                    for (int c = 1; c <= 3; ++c) pS.Bxyz(ig, j, k, c) = pS.Bxyz(G.is, jp, kp, c);
                }
    }
}

// ---------------------------------------------------------------- electric field (fields.F90)
static void Mom2Face(const Model& M, const Grid& G, const State& hS, double (*VfB)[vecLen], int iB, int j, int k,
                     int iMax, int dT) {  // fields.F90:235-285
    double VolB[recLen][vecLen], DenB[recLen][vecLen], MomB[3][recLen][vecLen], VelB[3][recLen][vecLen];
    const long cellN = (long)G.Ni * G.Nj * G.Nk;
    loadBlock(G, VolB, G.volume.d.data(), iB, j, k, iMax, dT, Nr2, false);
    loadBlock(G, DenB, hS.Gas.d.data() + 0 * cellN, iB, j, k, iMax, dT, Nr2, false);
    for (int c = 0; c < 3; ++c) loadBlock(G, MomB[c], hS.Gas.d.data() + (1 + c) * cellN, iB, j, k, iMax, dT, Nr2, false);
    for (int n = 0; n < recLen; ++n)
        for (int i = 0; i < iMax; ++i)
            for (int c = 0; c < 3; ++c) VelB[c][n][i] = VolB[n][i] * MomB[c][n][i] / fmaxd(DenB[n][i], M.dFloor);
    for (int c = 0; c < 3; ++c) for (int i = 0; i < vecLen; ++i) VfB[c][i] = 0.0;
    double dV[vecLen];
    for (int i = 0; i < iMax; ++i) {
        double s = 0.0;
        for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * VolB[n][i];
        dV[i] = fmaxd(s, TINY);
    }
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < iMax; ++i) {
            double s = 0.0;
            for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * VelB[c][n][i];
            VfB[c][i] = s / dV[i];
        }
}

static void EdgeLRs(const Model& M, const Grid& G, const Arr& bFluxn, const Arr& bFluxHf, double* bL, double* bR,
                    double* fA, int iB, int j, int k, int iMax, int dN, int dT1, int dT2) {  // fields.F90:288-362
    (void)dN;
    double AreaB[recLen][vecLen], VolB[recLen][vecLen], nAreaB[limLen][vecLen];
    double MagB[1][recLen][vecLen], nMagB[1][limLen][vecLen], MagLB[1][vecLen], MagRB[1][vecLen];
    const long faceN = (long)(G.Ni + 1) * (G.Nj + 1) * (G.Nk + 1);
    for (int i = 0; i < vecLen; ++i) { fA[i] = 0.0; bL[i] = 0.0; bR[i] = 0.0; }
    for (int n = 0; n < recLen; ++n) for (int i = 0; i < vecLen; ++i) VolB[n][i] = 0.0;
    loadBlock(G, AreaB, G.face.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nr2, true);
    loadBlock(G, MagB[0], bFluxHf.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nr2, true);
    loadBlock(G, nAreaB, G.face.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nl2, true);
    const Arr& lim = M.doLFMLim ? bFluxn : bFluxHf;
    loadBlock(G, nMagB[0], lim.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nl2, true);
    for (int i = 0; i < iMax; ++i) {
        for (int n = 0; n < recLen; ++n) {
            VolB[n][i] = AreaB[n][i];
            MagB[0][n][i] = MagB[0][n][i] / fmaxd(AreaB[n][i], TINY);
        }
        for (int n = 0; n < limLen; ++n) nMagB[0][n][i] = nMagB[0][n][i] / fmaxd(nAreaB[n][i], TINY);
    }
    BlockLRs(M.rmeth, VolB, nMagB, MagB, MagLB, MagRB, 1);
    for (int i = 0; i < vecLen; ++i) { bL[i] = MagLB[0][i]; bR[i] = MagRB[0][i]; }
    for (int i = 0; i < iMax; ++i) {
        double s = 0.0;
        for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * AreaB[n][i];
        fA[i] = s;
        bL[i] = bL[i] * fA[i];
        bR[i] = bR[i] * fA[i];
    }
}

static void GetCornerB(const Model& M, const Grid& G, const Arr& bFluxn, const Arr& bFluxHf, double* b1, double* b2,
                       double* Jd, int iB, int j, int k, int iMax, int dN, int dT1, int dT2) {  // fields.F90:365-424
    double bT1L[vecLen], bT1R[vecLen], fA1[vecLen], bT2L[vecLen], bT2R[vecLen], fA2[vecLen];
    EdgeLRs(M, G, bFluxn, bFluxHf, bT1L, bT1R, fA1, iB, j, k, iMax, dN, dT1, dT2);
    EdgeLRs(M, G, bFluxn, bFluxHf, bT2L, bT2R, fA2, iB, j, k, iMax, dN, dT2, dT1);
    for (int i = 0; i < iMax; ++i) {
        int iG = iB + i;
        double xni = G.Teb(iG, j, k, XNQI, dN), yni = G.Teb(iG, j, k, YNQI, dN);
        double xnj = G.Teb(iG, j, k, XNQJ, dN), ynj = G.Teb(iG, j, k, YNQJ, dN);
        double detT = 1.0 / (xni * ynj - xnj * yni);
        double bT1 = 0.5 * (bT1L[i] + bT1R[i]) / fA1[i];
        double bT2 = 0.5 * (bT2L[i] + bT2R[i]) / fA2[i];
        double db1 = (bT1R[i] - bT1L[i]) / fA1[i];
        double db2 = (bT2R[i] - bT2L[i]) / fA2[i];
        Jd[i] = db2 - db1;
        b1[i] = detT * (ynj * bT1 - yni * bT2);
        b2[i] = detT * (-(xnj * bT1) + xni * bT2);
        if (M.doBackground) {
            b1[i] = b1[i] + G.edgB0(iG, j, k, 1, dN);
            b2[i] = b2[i] + G.edgB0(iG, j, k, 2, dN);
        }
    }
}

static void GetCornerD(const Grid& G, const Arr& Gas, double* Dc, int iB, int j, int k, int iMax, int dN) {
    int e1[3], e2[3];  // metric.F90:151-167 getNormalPlane
    if (dN == IDIR) { e1[0] = 0; e1[1] = 1; e1[2] = 0; e2[0] = 0; e2[1] = 0; e2[2] = 1; }
    else if (dN == JDIR) { e1[0] = 1; e1[1] = 0; e1[2] = 0; e2[0] = 0; e2[1] = 0; e2[2] = 1; }
    else { e1[0] = 1; e1[1] = 0; e1[2] = 0; e2[0] = 0; e2[1] = 1; e2[2] = 0; }
    for (int i = 0; i < iMax; ++i) {
        int iG = iB + i;
        Dc[i] = 0.25 * (Gas(iG, j, k, DEN) + Gas(iG - e1[0], j - e1[1], k - e1[2], DEN) +
                        Gas(iG - e2[0], j - e2[1], k - e2[2], DEN) +
                        Gas(iG - e1[0] - e2[0], j - e1[1] - e2[1], k - e1[2] - e2[2], DEN));
    }
}

static void GetCornerV(const Grid& G, const Arr& Vf, double* v1, double* v2, double* vDiff, int iB, int j, int k,
                       int iMax, int dN, int dT1, int dT2) {  // fields.F90:457-517
    double VelB[3][recLen][vecLen], AreaB[recLen][vecLen], VxyzC[3][vecLen], dA[vecLen];
    const long faceN = (long)(G.Ni + 1) * (G.Nj + 1) * (G.Nk + 1);
    const long cellN = (long)G.Ni * G.Nj * G.Nk;
    loadBlock(G, AreaB, G.face.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nr2, true);
    for (int i = 0; i < iMax; ++i) {
        double s = 0.0;
        for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * AreaB[n][i];
        dA[i] = fmaxd(s, TINY);
    }
    for (int d = 0; d < 3; ++d) {
        loadBlock(G, VelB[d], Vf.d.data() + d * cellN, iB, j, k, iMax, dT2, Nr2, false);
        for (int i = 0; i < iMax; ++i) {
            double s = 0.0;
            for (int n = 0; n < recLen; ++n) s = s + interpWgt[n] * (AreaB[n][i] * VelB[d][n][i]);
            VxyzC[d][i] = s / dA[i];
        }
    }
    for (int i = 0; i < iMax; ++i) {
        int iG = iB + i;
        v1[i] = VxyzC[0][i] * G.Te(iG, j, k, TAN1X, dN) + VxyzC[1][i] * G.Te(iG, j, k, TAN1Y, dN) +
                VxyzC[2][i] * G.Te(iG, j, k, TAN1Z, dN);
        v2[i] = VxyzC[0][i] * G.Te(iG, j, k, TAN2X, dN) + VxyzC[1][i] * G.Te(iG, j, k, TAN2Y, dN) +
                VxyzC[2][i] * G.Te(iG, j, k, TAN2Z, dN);
        vDiff[i] = std::sqrt(sq(v1[i]) + sq(v2[i]));
    }
}

static void CalcElecField(const Model& M, const Grid& G, const State& nS, const State& hS, Arr& Vf, Arr& E) {
    std::fill(E.d.begin(), E.d.end(), 0.0);
    for (int eD = 1; eD <= NDIM; ++eD) {
        int dT1, dT2, ie, je, ke;
        if (eD == IDIR) {
            dT1 = JDIR; dT2 = KDIR; ie = G.ie; je = G.je + 1; ke = G.ke + 1;
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = G.ksg; k <= G.keg; ++k)
                for (int iB = G.isg; iB <= G.ieg; iB += vecLen)
                    for (int j = G.js; j <= G.je + 1; ++j) {
                        int iMax = std::min((int)vecLen, G.ieg - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(M, G, hS, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; ++i) for (int c = 0; c < 3; ++c) Vf(iB + i, j, k, c + 1) = VelB[c][i];
                    }
        } else if (eD == JDIR) {
            dT1 = KDIR; dT2 = IDIR; ie = G.ie + 1; je = G.je; ke = G.ke + 1;
#pragma omp parallel for collapse(2) schedule(static)
            for (int j = G.jsg; j <= G.jeg; ++j)
                for (int iB = G.isg; iB <= G.ieg; iB += vecLen)
                    for (int k = G.ks; k <= G.ke + 1; ++k) {
                        int iMax = std::min((int)vecLen, G.ieg - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(M, G, hS, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; ++i) for (int c = 0; c < 3; ++c) Vf(iB + i, j, k, c + 1) = VelB[c][i];
                    }
        } else {
            dT1 = IDIR; dT2 = JDIR; ie = G.ie + 1; je = G.je + 1; ke = G.ke;
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = G.ksg; k <= G.keg; ++k)
                for (int j = G.jsg; j <= G.jeg; ++j)
                    for (int iB = G.is; iB <= G.ie + 1; iB += vecLen) {
                        int iMax = std::min((int)vecLen, G.ie + 1 - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(M, G, hS, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; ++i) for (int c = 0; c < 3; ++c) Vf(iB + i, j, k, c + 1) = VelB[c][i];
                    }
        }
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = G.ks; k <= ke; ++k)
            for (int j = G.js; j <= je; ++j)
                for (int iB = G.is; iB <= ie; iB += vecLen) {
                    int iMax = std::min((int)vecLen, ie - iB + 1);
                    double v1[vecLen], v2[vecLen], b1[vecLen], b2[vecLen], Jd[vecLen], Dc[vecLen], vDiff[vecLen];
                    for (int i = 0; i < vecLen; ++i) vDiff[i] = 0.0;
                    GetCornerV(G, Vf, v1, v2, vDiff, iB, j, k, iMax, eD, dT1, dT2);
                    GetCornerD(G, hS.Gas, Dc, iB, j, k, iMax, eD);
                    GetCornerB(M, G, nS.magFlux, hS.magFlux, b1, b2, Jd, iB, j, k, iMax, eD, dT1, dT2);
                    for (int i = 0; i < iMax; ++i) {
                        int iG = iB + i;
                        double vA = std::sqrt(sq(b1[i]) + sq(b2[i])) / std::sqrt(Dc[i]);
                        if (M.doBoris) vA = M.Ca * vA / std::sqrt(sq(M.Ca) + sq(vA));
                        vDiff[i] = vDiff[i] + vA;
                        vDiff[i] = fmind(vDiff[i], M.CFL * G.edge(iG, j, k, eD) / M.dt);
                        double e = -(v1[i] * b2[i] - v2[i] * b1[i]) + M.Vd0 * vDiff[i] * Jd[i];
                        E(iG, j, k, eD) = e * G.edge(iG, j, k, eD);
                    }
                }
    }
}

static void E2Flux(const Grid& G, Arr& mf, const Arr& E, double dt) {  // fields.F90:18-51
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double dfi = E(i, j + 1, k, KDIR) - E(i, j, k, KDIR) - E(i, j, k + 1, JDIR) + E(i, j, k, JDIR);
                double dfj = E(i, j, k + 1, IDIR) - E(i, j, k, IDIR) - E(i + 1, j, k, KDIR) + E(i, j, k, KDIR);
                double dfk = E(i + 1, j, k, JDIR) - E(i, j, k, JDIR) - E(i, j + 1, k, IDIR) + E(i, j, k, IDIR);
                mf(i, j, k, IDIR) = mf(i, j, k, IDIR) - dt * dfi;
                mf(i, j, k, JDIR) = mf(i, j, k, JDIR) - dt * dfj;
                mf(i, j, k, KDIR) = mf(i, j, k, KDIR) - dt * dfk;
            }
}

// ---------------------------------------------------------------- update (mhdgroup.F90:79-442)
static inline double dot3(const double* a, const double* b) { return dot(a, b, 3); }
static void normVec3(const double* a, double* o) {
    double nA = std::sqrt(dot3(a, a));
    if (nA <= TINY) { o[0] = o[1] = o[2] = 0.0; }
    else { o[0] = a[0] / nA; o[1] = a[1] / nA; o[2] = a[2] / nA; }
}
static void Vec2Para(const double* A, const double* n, double* o) {
    double s = dot3(A, n);
    for (int c = 0; c < 3; ++c) o[c] = s * n[c];
}
static void Vec2Perp(const double* A, const double* n, double* o) {
    double p[3];
    Vec2Para(A, n, p);
    for (int c = 0; c < 3; ++c) o[c] = A[c] - p[c];
}
static void CellMaxwell(const Model& M, double* U, const double* dGasM, double dt) {  // mhdgroup.F90:300-330
    double D = fmaxd(U[0], M.dFloor), Mx = U[1], My = U[2], Mz = U[3], TotE = U[4];
    double KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) / D;
    double P = fmaxd((M.gamma - 1) * (TotE - KinE), M.pFloor);
    Mx = Mx + dt * dGasM[0];
    My = My + dt * dGasM[1];
    Mz = Mz + dt * dGasM[2];
    KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) / D;
    U[0] = D; U[1] = Mx; U[2] = My; U[3] = Mz; U[4] = KinE + P / (M.gamma - 1);
}
static void CellBoris(const Model& M, double* U2, const double* U0, const double* B2, const double* B0,
                      const double* dGasH, const double* dGasM, double Ca, double dt) {  // mhdgroup.F90:337-390
    double W2[5];
    CellC2P(M, U2, W2);
    double D2 = fmaxd(W2[0], M.dFloor), P2 = fmaxd(W2[4], M.pFloor);
    double D0 = U0[0];
    D0 = fmaxd(D0, M.dFloor);
    double V0[3] = {U0[1] / D0, U0[2] / D0, U0[3] / D0};
    double B1[3];
    for (int c = 0; c < 3; ++c) B1[c] = 0.5 * (B2[c] + B0[c]);
    double alpha = dot3(B1, B1) / (D2 * Ca * Ca);
    double dRho = dt * dGasH[0];
    double dPGas[3], dPMag[3], dMom[3];
    for (int c = 0; c < 3; ++c) { dPGas[c] = dt * dGasH[1 + c]; dPMag[c] = dt * dGasM[c]; }
    double pCon = 1.0 / (1.0 + alpha);
    double bhat1[3];
    normVec3(B1, bhat1);
    if (alpha > TINY) {
        double a[3], s[3], b[3], c3[3], d[3];
        Vec2Para(dPGas, bhat1, a);
        for (int c = 0; c < 3; ++c) s[c] = dPGas[c] + dPMag[c];
        Vec2Perp(s, bhat1, b);
        Vec2Perp(V0, bhat1, c3);
        for (int c = 0; c < 3; ++c) { d[c] = a[c] + pCon * b[c]; dMom[c] = d[c] + alpha * pCon * dRho * c3[c]; }
    } else {
        for (int c = 0; c < 3; ++c) dMom[c] = dPGas[c] + dPMag[c];
    }
    double V2[3];
    for (int c = 0; c < 3; ++c) V2[c] = (D0 * V0[c] + dMom[c]) / D2;
    W2[0] = D2; W2[1] = V2[0]; W2[2] = V2[1]; W2[3] = V2[2]; W2[4] = P2;
    CellP2C(M, W2, U2);
}

static void PoleE(const Model& M, const Grid& G, Arr& E);

// applyUpdate with the buffer roles of the reference: CopyState(State->oState) then in-place update of State
static void applyUpdate(Model& M, const Grid& G, State& S, State& oS, double dt, const Arr& dGasH, const Arr& dGasM,
                        Arr& E) {
    oS.Gas.d = S.Gas.d;
    oS.Bxyz.d = S.Bxyz.d;
    oS.magFlux.d = S.magFlux.d;
    oS.time = S.time;
    S.time = S.time + dt;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i)
                for (int v = 1; v <= NVAR; ++v) S.Gas(i, j, k, v) = S.Gas(i, j, k, v) + M.dt * dGasH(i, j, k, v);
    if (!M.doMHD) return;
    if (M.doRing && (M.R.doS || M.R.doE)) PoleE(M, G, E);   // mhdgroup.F90:139-142
    E2Flux(G, S.magFlux, E, dt);
    bFlux2Fld(M, G, S.magFlux, S.Bxyz);
    bool Boris = M.doBoris;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double U[5], dPm[3];
                for (int v = 0; v < 5; ++v) U[v] = S.Gas(i, j, k, v + 1);
                for (int c = 0; c < 3; ++c) dPm[c] = dGasM(i, j, k, c + 1);
                if (Boris) {
                    double oU[5], B[3], oB[3], dPg[5];
                    for (int v = 0; v < 5; ++v) { oU[v] = oS.Gas(i, j, k, v + 1); dPg[v] = dGasH(i, j, k, v + 1); }
                    for (int c = 0; c < 3; ++c) { B[c] = S.Bxyz(i, j, k, c + 1); oB[c] = oS.Bxyz(i, j, k, c + 1); }
                    if (M.doBackground)
                        for (int c = 0; c < 3; ++c) { B[c] = B[c] + G.B0(i, j, k, c + 1); oB[c] = oB[c] + G.B0(i, j, k, c + 1); }
                    CellBoris(M, U, oU, B, oB, dPg, dPm, M.Ca, dt);
                } else {
                    CellMaxwell(M, U, dPm, dt);
                }
                for (int v = 0; v < 5; ++v) S.Gas(i, j, k, v + 1) = U[v];
            }
}

// ---------------------------------------------------------------- dt (gridutils.F90:49-106, step.F90:58-168)
static double CellDT(const Model& M, const Grid& G, const State& S, int i, int j, int k) {
    double rho = S.Gas(i, j, k, DEN);
    double Vx = S.Gas(i, j, k, MOMX) / rho, Vy = S.Gas(i, j, k, MOMY) / rho, Vz = S.Gas(i, j, k, MOMZ) / rho;
    double MagV = std::sqrt(sq(Vx) + sq(Vy) + sq(Vz));
    double ke = 0.5 * rho * sq(MagV);
    double e = S.Gas(i, j, k, ENERGY) - ke;
    double P = (M.gamma - 1) * e;
    double Cs = std::sqrt(M.gamma * P / rho);
    double Vfl = MagV, Valf = 0.0, Vdiff = 0.0;
    if (M.doMHD) {
        double Bx = S.Bxyz(i, j, k, XDIR), By = S.Bxyz(i, j, k, YDIR), Bz = S.Bxyz(i, j, k, ZDIR);
        if (M.doBackground) {
            Bx = Bx + G.B0(i, j, k, XDIR);
            By = By + G.B0(i, j, k, YDIR);
            Bz = Bz + G.B0(i, j, k, ZDIR);
        }
        double MagB = std::sqrt(sq(Bx) + sq(By) + sq(Bz));
        Valf = MagB / std::sqrt(rho);
        if (M.doBoris) Valf = M.Ca * Valf / std::sqrt(M.Ca * M.Ca + Valf * Valf);
    }
    double vCFL = Vfl + std::sqrt(sq(Cs) + sq(Valf)) + Vdiff;
    double dl = G.di(i, j, k);
    if (G.dj(i, j, k) < dl) dl = G.dj(i, j, k);
    if (G.dk(i, j, k) < dl) dl = G.dk(i, j, k);
    return M.CFL * dl / vCFL;
}

static double CalcDT(Model& M, const Grid& G, const State& S) {
    if (M.fixedTimestep) return M.dt;
    double dtOld = M.dt;
    double dtMin = HUGEV;
    bool isDisaster = false, isBad = false;
#pragma omp parallel for collapse(2) reduction(min : dtMin) schedule(static)
    for (int k = G.ksDT; k <= G.keDT; ++k)
        for (int j = G.jsDT; j <= G.jeDT; ++j)
            for (int i = G.isDT; i <= G.ieDT; ++i) {
                double dtijk = CellDT(M, G, S, i, j, k);
                dtMin = fmind(dtijk, dtMin);
            }
    if (dtMin == HUGEV) isDisaster = true;
    double r = dtMin;
    if (M.ts > 0) {
        if (dtOld / dtMin >= 10) isBad = true;
        if ((M.dt0 > TINY) && (dtMin / M.dt0 <= M.limDT0)) isBad = true;
        if (dtMin <= TINY) isDisaster = true;
    }
    M.status = (isDisaster ? 1 : 0) | (isBad ? 2 : 0);
    if ((M.t + r) > M.tFin) r = fmaxd(M.tFin - M.t, TINY);
    if (M.dt0 > TINY && r > (10.0 * M.dt0)) r = 10.0 * M.dt0;
    return r;
}

// ---------------------------------------------------------------- boundary conditions (bcs.F90)
static void copyCellVec(Arr& A, int i, int j, int k, int si, int sj, int sk, int nc) {
    for (int c = 1; c <= nc; ++c) A(i, j, k, c) = A(si, sj, sk, c);
}
static void periodicBC(const Model& M, const Grid& G, State& S, int dir) {  // bcs.F90:279-450
    const int nG = M.nG;
    switch (dir) {
    case INI:
        for (int k = G.ksg; k <= G.keg + 1; ++k)
            for (int j = G.jsg; j <= G.jeg + 1; ++j)
                for (int n = 1; n <= nG; ++n) {
                    int ig = G.is - n;
                    if (j <= G.jeg && k <= G.keg) {
                        copyCellVec(S.Gas, ig, j, k, G.ie - n + 1, j, k, 5);
                        copyCellVec(S.Bxyz, ig, j, k, G.ie - n + 1, j, k, 3);
                    }
                    copyCellVec(S.magFlux, ig, j, k, G.ie - n + 1, j, k, 3);
                }
        break;
    case OUTI:
        for (int k = G.ksg; k <= G.keg + 1; ++k)
            for (int j = G.jsg; j <= G.jeg + 1; ++j)
                for (int n = 1; n <= nG; ++n) {
                    int ig = G.ie + n;
                    if (j <= G.jeg && k <= G.keg) {
                        copyCellVec(S.Gas, ig, j, k, G.is + n - 1, j, k, 5);
                        copyCellVec(S.Bxyz, ig, j, k, G.is + n - 1, j, k, 3);
                    }
                    S.magFlux(ig, j, k, JDIR) = S.magFlux(G.is + n - 1, j, k, JDIR);
                    S.magFlux(ig, j, k, KDIR) = S.magFlux(G.is + n - 1, j, k, KDIR);
                    S.magFlux(ig + 1, j, k, IDIR) = S.magFlux(G.is + n, j, k, IDIR);
                }
        break;
    case INJ:
        for (int k = G.ksg; k <= G.keg + 1; ++k)
            for (int i = G.isg; i <= G.ieg + 1; ++i)
                for (int n = 1; n <= nG; ++n) {
                    int jg = G.js - n;
                    if (i <= G.ieg && k <= G.keg) {
                        copyCellVec(S.Gas, i, jg, k, i, G.je - n + 1, k, 5);
                        copyCellVec(S.Bxyz, i, jg, k, i, G.je - n + 1, k, 3);
                    }
                    copyCellVec(S.magFlux, i, jg, k, i, G.je - n + 1, k, 3);
                }
        break;
    case OUTJ:
        for (int k = G.ksg; k <= G.keg + 1; ++k)
            for (int i = G.isg; i <= G.ieg + 1; ++i)
                for (int n = 1; n <= nG; ++n) {
                    int jg = G.je + n;
                    if (i <= G.ieg && k <= G.keg) {
                        copyCellVec(S.Gas, i, jg, k, i, G.js + n - 1, k, 5);
                        copyCellVec(S.Bxyz, i, jg, k, i, G.js + n - 1, k, 3);
                    }
                    S.magFlux(i, jg, k, IDIR) = S.magFlux(i, G.js + n - 1, k, IDIR);
                    S.magFlux(i, jg, k, KDIR) = S.magFlux(i, G.js + n - 1, k, KDIR);
                    S.magFlux(i, jg + 1, k, JDIR) = S.magFlux(i, G.js + n, k, JDIR);
                }
        break;
    case INK:
        if (M.do25D) {
            for (int n = 1; n <= nG; ++n)
                for (int j = G.jsg; j <= G.jeg + 1; ++j)
                    for (int i = G.isg; i <= G.ieg + 1; ++i) {
                        if (i <= G.ieg && j <= G.jeg) {
                            copyCellVec(S.Gas, i, j, G.ks - n, i, j, G.ks, 5);
                            copyCellVec(S.Bxyz, i, j, G.ks - n, i, j, G.ks, 3);
                        }
                        copyCellVec(S.magFlux, i, j, G.ks - n, i, j, G.ks, 3);
                    }
        } else {
            for (int j = G.jsg; j <= G.jeg + 1; ++j)
                for (int i = G.isg; i <= G.ieg + 1; ++i)
                    for (int n = 1; n <= nG; ++n) {
                        int kg = G.ks - n;
                        if (i <= G.ieg && j <= G.jeg) {
                            copyCellVec(S.Gas, i, j, kg, i, j, G.ke - n + 1, 5);
                            copyCellVec(S.Bxyz, i, j, kg, i, j, G.ke - n + 1, 3);
                        }
                        copyCellVec(S.magFlux, i, j, kg, i, j, G.ke - n + 1, 3);
                    }
        }
        break;
    case OUTK:
        if (M.do25D) {
            for (int n = 1; n <= nG; ++n)
                for (int j = G.jsg; j <= G.jeg + 1; ++j)
                    for (int i = G.isg; i <= G.ieg + 1; ++i) {
                        if (i <= G.ieg && j <= G.jeg) {
                            copyCellVec(S.Gas, i, j, G.ks + n, i, j, G.ks, 5);
                            copyCellVec(S.Bxyz, i, j, G.ks + n, i, j, G.ks, 3);
                        }
                        copyCellVec(S.magFlux, i, j, G.ks + n, i, j, G.ks, 3);
                    }
        } else {
            for (int j = G.jsg; j <= G.jeg + 1; ++j)
                for (int i = G.isg; i <= G.ieg + 1; ++i)
                    for (int n = 1; n <= nG; ++n) {
                        int kg = G.ke + n;
                        if (i <= G.ieg && j <= G.jeg) {
                            copyCellVec(S.Gas, i, j, kg, i, j, G.ks + n - 1, 5);
                            copyCellVec(S.Bxyz, i, j, kg, i, j, G.ks + n - 1, 3);
                        }
                        S.magFlux(i, j, kg, IDIR) = S.magFlux(i, j, G.ks + n - 1, IDIR);
                        S.magFlux(i, j, kg, JDIR) = S.magFlux(i, j, G.ks + n - 1, JDIR);
                        S.magFlux(i, j, kg + 1, KDIR) = S.magFlux(i, j, G.ks + n, KDIR);
                    }
        }
        break;
    }
}
// isCellCenterG is true for cell-centred indices inside the allocated cell range; the guards above
// (i<=ieg, j<=jeg, k<=keg) restate it for the loops that run to the +1 face index.

static void zeroGradBC(const Model& M, const Grid& G, State& S, int dir) {  // bcs.F90:799-930
    const int nG = M.nG;
    switch (dir) {
    case INI:
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int j = G.jsg; j <= G.jeg; ++j)
                for (int n = 1; n <= nG; ++n) {
                    copyCellVec(S.Gas, G.is - n, j, k, G.is, j, k, 5);
                    copyCellVec(S.magFlux, G.is - n, j, k, G.is, j, k, 3);
                }
        break;
    case OUTI:
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int j = G.jsg; j <= G.jeg; ++j) {
                double B[3];
                gamCellBxyz(G, S.magFlux, G.ie, j, k, B);
                for (int n = 1; n <= nG; ++n) {
                    int ig = G.ie + n;
                    copyCellVec(S.Gas, ig, j, k, G.ie, j, k, 5);
                    double t1[3] = {G.Tf(ig + 1, j, k, NORMX, IDIR), G.Tf(ig + 1, j, k, NORMY, IDIR), G.Tf(ig + 1, j, k, NORMZ, IDIR)};
                    double t2[3] = {G.Tf(ig, j, k, NORMX, JDIR), G.Tf(ig, j, k, NORMY, JDIR), G.Tf(ig, j, k, NORMZ, JDIR)};
                    double t3[3] = {G.Tf(ig, j, k, NORMX, KDIR), G.Tf(ig, j, k, NORMY, KDIR), G.Tf(ig, j, k, NORMZ, KDIR)};
                    S.magFlux(ig + 1, j, k, IDIR) = G.face(ig + 1, j, k, IDIR) * dot3(B, t1);
                    S.magFlux(ig, j, k, JDIR) = G.face(ig, j, k, JDIR) * dot3(B, t2);
                    S.magFlux(ig, j, k, KDIR) = G.face(ig, j, k, KDIR) * dot3(B, t3);
                }
            }
        break;
    case INJ:
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int n = 1; n <= nG; ++n)
                for (int i = G.isg; i <= G.ieg; ++i) {
                    copyCellVec(S.Gas, i, G.js - n, k, i, G.js, k, 5);
                    copyCellVec(S.magFlux, i, G.js - n, k, i, G.js, k, 3);
                }
        break;
    case OUTJ:
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int n = 1; n <= nG; ++n)
                for (int i = G.isg; i <= G.ieg; ++i) {
                    copyCellVec(S.Gas, i, G.je + n, k, i, G.je, k, 5);
                    S.magFlux(i, G.je + n, k, IDIR) = S.magFlux(i, G.je, k, IDIR);
                    S.magFlux(i, G.je + n, k, KDIR) = S.magFlux(i, G.je, k, KDIR);
                    S.magFlux(i, G.je + n + 1, k, JDIR) = S.magFlux(i, G.je + 1, k, JDIR);
                }
        break;
    case INK:
        for (int n = 1; n <= nG; ++n)
            for (int j = G.jsg; j <= G.jeg; ++j)
                for (int i = G.isg; i <= G.ieg; ++i) {
                    copyCellVec(S.Gas, i, j, G.ks - n, i, j, G.ks, 5);
                    copyCellVec(S.magFlux, i, j, G.ks - n, i, j, G.ks, 3);
                }
        break;
    case OUTK:
        for (int n = 1; n <= nG; ++n)
            for (int j = G.jsg; j <= G.jeg; ++j)
                for (int i = G.isg; i <= G.ieg; ++i) {
                    copyCellVec(S.Gas, i, j, G.ke + n, i, j, G.ke, 5);
                    S.magFlux(i, j, G.ke + n, XDIR) = S.magFlux(i, j, G.ke, IDIR);
                    S.magFlux(i, j, G.ke + n, YDIR) = S.magFlux(i, j, G.ke, JDIR);
                    // bcs.F90:924 copies the J component of face ke+1 into the K faces above it; kept as is.
                    S.magFlux(i, j, G.ke + n + 1, ZDIR) = S.magFlux(i, j, G.ke + 1, JDIR);
                }
        break;
    }
}

// lfmIn / lfmOut (bcs.F90:1020-1106): ghost cells and faces across the axis from their conjugates
static void lfmPoleBC(const Model& M, const Grid& G, State& S, int dir) {
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int i = G.isg; i <= G.ieg + 1; ++i)
            for (int n = 1; n <= M.nG; ++n) {
                int ig = i, kg = k, jg = (dir == INJ) ? G.js - n : G.je + n;
                int ip, jp, kp;
                if (ig <= G.ieg && kg <= G.keg) {   // isCellCenterG
                    lfmIJKcc(M, G, ig, jg, kg, ip, jp, kp);
                    for (int v = 1; v <= NVAR; ++v) S.Gas(ig, jg, kg, v) = S.Gas(ip, jp, kp, v);
                    for (int c = 1; c <= NDIM; ++c) S.Bxyz(ig, jg, kg, c) = S.Bxyz(ip, jp, kp, c);
                }
                lfmIJKfc(M, G, IDIR, ig, jg, kg, ip, jp, kp);
                S.magFlux(ig, jg, kg, IDIR) = S.magFlux(ip, jp, kp, IDIR);
                int jf = (dir == INJ) ? jg : jg + 1;   // the first outer J ghost face is je+2
                lfmIJKfc(M, G, JDIR, ig, jf, kg, ip, jp, kp);
                S.magFlux(ig, jf, kg, JDIR) = -S.magFlux(ip, jp, kp, JDIR);
                lfmIJKfc(M, G, KDIR, ig, jg, kg, ip, jp, kp);
                S.magFlux(ig, jg, kg, KDIR) = -S.magFlux(ip, jp, kp, KDIR);
            }
}
// bw_ibcI / bw_obcI of the LFM blast wave (ICs/lfmbw.F90:141-225): fixed gas in the ghost shells, face
// fluxes mirrored from the first/last active shell scaled by the face areas
static void lfmbwShellBC(const Model& M, const Grid& G, State& S, int dir) {
    const bool inner = (dir == INI);
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int j = G.jsg; j <= G.jeg + 1; ++j)
            for (int n = 1; n <= M.nG; ++n) {
                int ig = inner ? G.is - n : G.ie + n;
                if (j <= G.jeg && k <= G.keg) {
                    S.Gas(ig, j, k, DEN) = M.bwD0;
                    S.Gas(ig, j, k, MOMX) = 0.0; S.Gas(ig, j, k, MOMY) = 0.0; S.Gas(ig, j, k, MOMZ) = 0.0;
                    S.Gas(ig, j, k, ENERGY) = M.bwP0 / (M.gamma - 1.0);
                }
                double dApm[3] = {1.0, 1.0, 1.0};
                if (M.R.doS && j < G.js) dApm[1] = dApm[2] = -1.0;
                if (M.R.doE && j >= G.je + 1) dApm[1] = dApm[2] = -1.0;
                for (int d = IDIR; d <= KDIR; ++d) {
                    int di = (!inner && d == IDIR) ? 1 : 0;
                    int ia = inner ? G.is : G.ie + di;   // the active shell the ghost face copies
                    int ip, jp, kp;
                    lfmIJKfc(M, G, d, ig + di, j, k, ip, jp, kp);
                    double dA = G.face(ig + di, j, k, d) / G.face(ia, jp, kp, d);
                    S.magFlux(ig + di, j, k, d) = dApm[d - 1] * dA * S.magFlux(ia, jp, kp, d);
                }
            }
}

// ---------------------------------------------------------------- the magnetosphere problem's boundaries
// A constant solar wind (its GetWindAt is the same state everywhere: RefreshWind's front velocity is along x
// with ByC = BzC = 0, wind.F90:112-161) and no ionospheric coupling (IonInnerBC_T%inExyz = inEijk = 0).
static double RampDownE(double r, double rC, double lC) {   // RampDown, math.F90:97-111
    if (r <= rC) return 1.0;
    if (r >= rC + lC) return 0.0;
    double rScl = (r - rC) / lC;
    double eArg = -1.0 / (1.0 - rScl * rScl);
    return std::exp(eArg + 1.0);
}
// wgtWind (wind.F90:185-203): the weight of the solar wind at a point, 1 on the sunward half
static double wgtWind(const Model& M, const double* xyz) {
    double nHat[3], vHat[3];
    normVec3(xyz, nHat);
    normVec3(M.W.wV, vHat);
    double d = 0.0;
    for (int c = 0; c < 3; ++c) d = d + (-vHat[c]) * nHat[c];
    double dTh = std::acos(d) * 180.0 / PI;
    return RampDownE(dTh, 90.0, 90.0);
}
// Con2Fast (gamutils.F90:343-360) with CellPress2Cs (:324-341): fast magnetosonic speed of a cell
static double Con2Fast(const Model& M, const double* gCon, const double* B) {
    double rho = fmaxd(gCon[0], M.dFloor);
    double Vx = gCon[1] / rho, Vy = gCon[2] / rho, Vz = gCon[3] / rho;
    double KinE = 0.5 * rho * (sq(Vx) + sq(Vy) + sq(Vz));
    double P = fmaxd((M.gamma - 1) * (gCon[4] - KinE), M.pFloor);
    double Cs = std::sqrt(M.gamma * P / rho);
    double D = gCon[0];
    double MagB = norm2v(B, 3);
    double Va = MagB / std::sqrt(D);
    if (M.doBoris) Va = M.Ca * Va / std::sqrt(sq(M.Ca) + sq(Va));
    return std::sqrt(sq(Cs) + sq(Va));
}
static double Project2Face(const Grid& G, const double* V, int d, int i, int j, int k) {   // bcs.F90:250-263
    double n[3] = {G.Tf(i, j, k, NORMX, d), G.Tf(i, j, k, NORMY, d), G.Tf(i, j, k, NORMZ, d)};
    return G.face(i, j, k, d) * dot3(n, V);
}
// WindBC (wind.F90:206-374), outer I shells
static void WindBC(const Model& M, const Grid& G, State& S) {
    const double MinMach = 1.0;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int j = G.jsg; j <= G.jeg + 1; ++j) {
            const int ip = G.ie;
            for (int n = 1; n <= M.nG; ++n) {
                const int ig = G.ie + n;
                if (j <= G.jeg && k <= G.keg) {   // isCellCenterG
                    double xcc[3] = {G.xyzcc(ig, j, k, 1), G.xyzcc(ig, j, k, 2), G.xyzcc(ig, j, k, 3)};
                    double wSW = wgtWind(M, xcc), wMHD = 1.0 - wSW;
                    double gW_sw[5] = {0, 0, 0, 0, 0}, gW_in[5] = {0, 0, 0, 0, 0};
                    if (wSW > TINY) {
                        gW_sw[0] = M.W.wD; gW_sw[4] = M.W.wP;
                        for (int c = 0; c < 3; ++c) gW_sw[1 + c] = M.W.wV[c];
                    }
                    if (wMHD > TINY) {
                        double gCon[5], B_in[3];
                        for (int v = 0; v < 5; ++v) gCon[v] = S.Gas(ip, j, k, v + 1);
                        for (int c = 0; c < 3; ++c) B_in[c] = S.Bxyz(ip, j, k, c + 1);
                        CellC2P(M, gCon, gW_in);
                        double Cx = Con2Fast(M, gCon, B_in);
                        double V[3] = {gW_in[1], gW_in[2], gW_in[3]};
                        double nHat[3] = {G.Tf(ip + 1, j, k, NORMX, IDIR), G.Tf(ip + 1, j, k, NORMY, IDIR),
                                          G.Tf(ip + 1, j, k, NORMZ, IDIR)};
                        if (dot3(V, nHat) < MinMach * Cx) {
                            double Vp[3];
                            Vec2Para(V, nHat, Vp);
                            for (int c = 0; c < 3; ++c) V[c] = V[c] - Vp[c] + MinMach * Cx * nHat[c];
                        }
                        for (int c = 0; c < 3; ++c) gW_in[1 + c] = V[c];
                    }
                    double gW[5], gCon[5];
                    for (int v = 0; v < 5; ++v) gW[v] = wSW * gW_sw[v] + wMHD * gW_in[v];
                    CellP2C(M, gW, gCon);
                    for (int v = 0; v < 5; ++v) S.Gas(ig, j, k, v + 1) = gCon[v];
                }
                // face fluxes: the wind's flux blended with the last active face's
                for (int d = 1; d <= 3; ++d) {
                    int fi = d == IDIR ? ig + 1 : ig, si = d == IDIR ? ip + 1 : ip;
                    double xf[3] = {G.xfc(fi, j, k, 1, d), G.xfc(fi, j, k, 2, d), G.xfc(fi, j, k, 3, d)};
                    double wSW = wgtWind(M, xf);
                    double swFlx = Project2Face(G, M.W.wB, d, fi, j, k);
                    double inFlx = S.magFlux(si, j, k, d);
                    S.magFlux(fi, j, k, d) = wSW * swFlx + (1 - wSW) * inFlx;
                }
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int n = 1; n <= M.nG; ++n) {
                int ig = G.ie + n, ip, jp, kp;
                lfmIJKcc(M, G, ig, j, k, ip, jp, kp);
                double B[3];
                gamCellBxyz(G, S.magFlux, ip, jp, kp, B);
                for (int c = 0; c < 3; ++c) S.Bxyz(ig, j, k, c + 1) = B[c];
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int i = G.ie + 1; i <= G.ieg; ++i)
            for (int n = 1; n <= M.nG; ++n) {
                int ip, jp, kp;
                if (M.R.doS) {
                    int jg = G.js - n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) S.Bxyz(i, jg, k, c) = S.Bxyz(ip, jp, kp, c);
                }
                if (M.R.doE) {
                    int jg = G.je + n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) S.Bxyz(i, jg, k, c) = S.Bxyz(ip, jp, kp, c);
                }
            }
}
// IonInner (voltron/ICs/earthcmi.F90:378-522) with CellPlasmaBC (apps/msphingest.F90:268-372) for one fluid
// without ingestion or ionospheric E field: the ghost takes the mirrored active cell's density and pressure at
// rest (Veb = 0), the ghost face fluxes are zero (the dipole is the background field), the ghost B comes from
// the (conjugate) cell's faces
static void IonInnerBC(const Model& M, const Grid& G, State& S) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int j = G.jsg; j <= G.jeg + 1; ++j)
            for (int n = 1; n <= M.nG; ++n) {
                const int ig = G.is - n, ip = G.is + n - 1;
                if (j <= G.jeg && k <= G.keg) {   // isCellCenterG
                    int idip, jp, kp;
                    lfmIJKcc(M, G, ig, j, k, idip, jp, kp);
                    double pU[5], pW[5], gW[5], gU[5];
                    for (int v = 0; v < 5; ++v) pU[v] = S.Gas(ip, jp, kp, v + 1);
                    CellC2P(M, pU, pW);
                    gW[0] = pW[0]; gW[4] = pW[4];
                    gW[1] = gW[2] = gW[3] = 0.0;   // Vec2Perp(Veb, rHat) + min(Vr, 0) rHat with Veb = 0
                    CellP2C(M, gW, gU);
                    for (int v = 0; v < 5; ++v) S.Gas(ig, j, k, v + 1) = gU[v];
                }
                for (int d = 1; d <= 3; ++d) {   // isGoodFaceIJK (gridutils.F90:985-1009)
                    bool good = (d == IDIR) ? (j <= G.jeg && k <= G.keg)
                                            : (d == JDIR) ? (k <= G.keg) : (j <= G.jeg);
                    if (good) S.magFlux(ig, j, k, d) = 0.0;
                }
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int n = 1; n <= M.nG; ++n) {
                int ig = G.is - n, ip, jp, kp;
                lfmIJKcc(M, G, ig, j, k, ip, jp, kp);
                double B[3];
                gamCellBxyz(G, S.magFlux, ip, jp, kp, B);
                for (int c = 0; c < 3; ++c) S.Bxyz(ig, j, k, c + 1) = B[c];
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int i = G.isg; i <= G.is - 1; ++i)
            for (int n = 1; n <= M.nG; ++n) {
                int ip, jp, kp;
                if (M.R.doS) {
                    int jg = G.js - n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) S.Bxyz(i, jg, k, c) = S.Bxyz(ip, jp, kp, c);
                }
                if (M.R.doE) {
                    int jg = G.je + n;
                    lfmIJKcc(M, G, i, jg, k, ip, jp, kp);
                    for (int c = 1; c <= 3; ++c) S.Bxyz(i, jg, k, c) = S.Bxyz(ip, jp, kp, c);
                }
            }
}

static void EnforceBCs(const Model& M, const Grid& G, State& S) {  // step.F90:17-55
    for (int n = 1; n <= 6; ++n) {
        int kind = G.bc[n - 1];
        if (kind == BC_HALO) continue;
        if (kind == BC_PERIODIC) periodicBC(M, G, S, n);
        else if (kind == BC_LFMPOLE) lfmPoleBC(M, G, S, n);
        else if (kind == BC_LFMBW) lfmbwShellBC(M, G, S, n);
        else if (kind == BC_ION) { if (n == INI) IonInnerBC(M, G, S); }
        else if (kind == BC_WIND) { if (n == OUTI) WindBC(M, G, S); }
        else zeroGradBC(M, G, S, n);
    }
}

// ---------------------------------------------------------------- ring average (ringav.F90, ringrecon.F90)
static double minmod(double x, double y) {   // math.F90:192-197
    return 0.5 * (fsign1(x) + fsign1(y)) * fmind(std::fabs(x), std::fabs(y));
}
static void RingLR(int meth, double fm2, double fm1, double f, double fp1, double fp2, double& vm, double& vp) {
    if (meth == RR_PCM) { vm = f; vp = f; return; }   // ringrecon.F90:239-246
    if (meth == RR_PLM) {                             // ringrecon.F90:251-270
        double dwL = f - fm1, dwR = fp1 - f, dwC = (fp1 - fm1) / 2.0;
        double min1 = fmind(2 * std::fabs(dwL), 2 * std::fabs(dwR));
        double min2 = fmind(min1, std::fabs(dwC));
        double dwM = std::copysign(min2, dwC);
        vp = f + 0.5 * dwM; vm = f - 0.5 * dwM;
        return;
    }
    // PPM (ringrecon.F90:282-322)
    double dvm2 = fm1 - fm2, dvm1 = f - fm1, dvp1 = fp1 - f, dvp2 = fp2 - fp1;
    double dvc = 0.5 * (dvm2 + dvm1), SM = 2.0 * minmod(dvm2, dvm1), Sm1 = minmod(dvc, SM);
    dvc = 0.5 * (dvm1 + dvp1); SM = 2.0 * minmod(dvm1, dvp1); double Sp1 = minmod(dvc, SM);
    dvc = 0.5 * (dvp2 + dvp1); SM = 2.0 * minmod(dvp2, dvp1); double Sp2 = minmod(dvc, SM);
    vp = 0.5 * (f + fp1) - (Sp2 - Sp1) / 6.0;
    vm = 0.5 * (f + fm1) - (Sp1 - Sm1) / 6.0;
    double ap = vp - f, am = vm - f;
    if (ap * am >= 0.0) { ap = 0.0; am = 0.0; }
    else {
        if (std::fabs(ap) >= 2.0 * std::fabs(am)) ap = -2.0 * am;
        if (std::fabs(am) >= 2.0 * std::fabs(ap)) am = -2.0 * ap;
    }
    vp = f + ap; vm = f + am;
}
// ReconstructRing (ringrecon.F90:34-98): parabolic interpolant of each chunk from its chunk neighbours
static void ReconstructRing(const Model& M, double* rW, int Nc) {
    const int Np = M.R.Np, dJ = Np / Nc, Ng = 2;
    std::vector<double> chW(Nc + 2 * Ng);
    auto ch = [&](int n) -> double& { return chW[n - 1 + Ng]; };
    for (int n = 1; n <= Nc; ++n) ch(n) = rW[(n - 1) * dJ];
    for (int n = 1; n <= Ng; ++n) { ch(1 - n) = ch(Nc - n + 1); ch(Nc + n) = ch(n); }
    for (int n = 1; n <= Nc; ++n) {
        int mS = 1 + (n - 1) * dJ;
        double fL, fR, f = ch(n);
        RingLR(M.R.recon, ch(n - 2), ch(n - 1), f, ch(n + 1), ch(n + 2), fL, fR);
        double a = 3 * (fL + fR - 2 * f), b = 2 * (3 * f - fR - 2 * fL), c = fL;
        for (int m = 1; m <= dJ; ++m) {
            double fI = (a / 3.0) * (double)(3 * m * m - 3 * m + 1) / (double)(dJ * dJ) + 0.5 * b * (double)(2 * m - 1) / (double)dJ + c;
            rW[mS + m - 2] = fI;
        }
    }
}
// CleanRing / DirtyRing (ringav.F90:416-458): remove / restore the 0..numFT Fourier modes of a ring
static void CleanRing(const Model& M, double* Q, double cFT[NFTMAX + 1][2], int numFT) {
    const int Np = M.R.Np;
    for (int m = 0; m <= NFTMAX; ++m) cFT[m][0] = cFT[m][1] = 0.0;
    double aScl = (double)(2.0f / (float)Np);   // 2.0/Np in default real
    double dp = 2.0 * PI / Np;
    for (int n = 1; n <= Np; ++n) {
        double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; ++m) {
            cFT[m][0] = cFT[m][0] + Q[n - 1] * std::cos(1.0 * m * phi);
            cFT[m][1] = cFT[m][1] + Q[n - 1] * std::sin(1.0 * m * phi);
        }
    }
    cFT[0][0] = 0.5 * aScl * cFT[0][0]; cFT[0][1] = 0.5 * aScl * cFT[0][1];
    for (int m = 1; m <= numFT; ++m) { cFT[m][0] = 1.0 * aScl * cFT[m][0]; cFT[m][1] = 1.0 * aScl * cFT[m][1]; }
    for (int n = 1; n <= Np; ++n) {
        double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; ++m)
            Q[n - 1] = Q[n - 1] - cFT[m][0] * std::cos(1.0 * m * phi) - cFT[m][1] * std::sin(1.0 * m * phi);
    }
}
static void DirtyRing(const Model& M, double* Q, const double cFT[NFTMAX + 1][2], int numFT) {
    const int Np = M.R.Np;
    double dp = 2.0 * PI / Np;
    for (int n = 1; n <= Np; ++n) {
        double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; ++m)
            Q[n - 1] = Q[n - 1] + cFT[m][0] * std::cos(1.0 * m * phi) + cFT[m][1] * std::sin(1.0 * m * phi);
    }
}
// chunk averages (ringav.F90:156-161, 266-273)
static void ChunkAverage(const double* in, double* out, int Np, int Nc) {
    int dC = Np / Nc;
    for (int n = 1; n <= Nc; ++n) {
        int lRs = 1 + (n - 1) * dC, lRe = lRs + dC - 1;
        double s = 0.0;
        for (int m = lRs; m <= lRe; ++m) s = s + in[m - 1];
        for (int m = lRs; m <= lRe; ++m) out[m - 1] = s / dC;
    }
}
// CalcSmoothE (ringav.F90:203-336) for the LFM axis
static void CalcSmoothE(const Model& M, const Grid& G, const State& S, Arr& SmoothE, int XPOLE) {
    const int Np = M.R.Np;
    const int fDIRS[2] = {JDIR, IDIR}, eDIRS[2] = {IDIR, JDIR};
    const double eScls[2] = {1.0, -1.0};
#pragma omp parallel for schedule(static)
    for (int nS = M.R.nSi; nS <= M.R.nSe + 1; ++nS) {
        std::vector<double> bFlx(3 * Np), dEr(3 * Np), rFlx(Np), raFlx(Np), dFlx(Np);
        for (int nR = 1; nR <= M.R.NumR; ++nR) {
            int NumCh = M.R.Nch[nR - 1], dC = Np / NumCh;
            for (int q = 0; q < Np; ++q) {   // PullRingI (ringutils.F90:753-787)
                int k = G.ks + q;
                if (XPOLE == SPOLE) {
                    bFlx[q] = S.magFlux(nS, G.js + nR - 1, k, IDIR);
                    bFlx[Np + q] = S.magFlux(nS, G.js + nR, k, JDIR);
                    bFlx[2 * Np + q] = S.magFlux(nS, G.js + nR - 1, k, KDIR);
                } else {
                    for (int d = 0; d < 3; ++d) bFlx[d * Np + q] = S.magFlux(nS, G.je - nR + 1, k, d + 1);
                }
            }
            std::fill(dEr.begin(), dEr.end(), 0.0);
            for (int d = 0; d < 2; ++d) {
                int fD = fDIRS[d], eD = eDIRS[d];
                double eScl = eScls[d], cFT[NFTMAX + 1][2];
                for (int q = 0; q < Np; ++q) rFlx[q] = bFlx[(fD - 1) * Np + q];
                CleanRing(M, rFlx.data(), cFT, M.R.NFTMAG);
                ChunkAverage(rFlx.data(), raFlx.data(), Np, NumCh);
                ReconstructRing(M, raFlx.data(), NumCh);
                DirtyRing(M, raFlx.data(), cFT, M.R.NFTMAG);
                for (int q = 0; q < Np; ++q) dFlx[q] = raFlx[q] - bFlx[(fD - 1) * Np + q];
                for (int n = 1; n <= NumCh; ++n) {
                    int lRs = 1 + (n - 1) * dC;
                    double cumFlx = -dFlx[lRs - 1];
                    for (int m = 2; m <= dC; ++m) {
                        dEr[(eD - 1) * Np + lRs + m - 2] = eScl * cumFlx;
                        cumFlx = cumFlx - dFlx[lRs + m - 2];
                    }
                }
            }
            for (int q = 0; q < Np; ++q) {
                int k = G.ks + q;
                if (XPOLE == SPOLE) {
                    SmoothE(nS, G.js + nR, k, IDIR) = dEr[q];
                    SmoothE(nS, G.js + nR - 1, k, JDIR) = dEr[Np + q];
                    SmoothE(nS, G.js + nR - 1, k, KDIR) = dEr[2 * Np + q];
                } else {
                    for (int d = 0; d < 3; ++d) SmoothE(nS, G.je - nR + 1, k, d + 1) = dEr[d * Np + q];
                }
            }
            if (XPOLE == SPOLE) {
                SmoothE(nS, G.js + nR, G.ke + 1, IDIR) = SmoothE(nS, G.js + nR, G.ks, IDIR);
                SmoothE(nS, G.js + nR - 1, G.ke + 1, JDIR) = SmoothE(nS, G.js + nR - 1, G.ks, JDIR);
            } else {
                SmoothE(nS, G.je - nR + 1, G.ke + 1, IDIR) = SmoothE(nS, G.je - nR + 1, G.ks, IDIR);
                SmoothE(nS, G.je - nR + 1, G.ke + 1, JDIR) = SmoothE(nS, G.je - nR + 1, G.ks, JDIR);
            }
        }
    }
}
// FixEFieldLFM (gamdebug.F90:149-175): the I and J edges of the periodic K seam take the average of the two copies
static void FixEFieldLFM(const Grid& G, Arr& E) {
    for (int j = G.js; j <= G.je + 1; ++j)
        for (int i = G.is; i <= G.ie + 1; ++i) {
            double Ei = 0.5 * (E(i, j, G.ks, IDIR) + E(i, j, G.ke + 1, IDIR));
            double Ej = 0.5 * (E(i, j, G.ks, JDIR) + E(i, j, G.ke + 1, JDIR));
            E(i, j, G.ks, IDIR) = Ei; E(i, j, G.ke + 1, IDIR) = Ei;
            E(i, j, G.ks, JDIR) = Ej; E(i, j, G.ke + 1, JDIR) = Ej;
        }
}
// PoleE (ringav.F90:376-411) for the LFM axis, then FixEFieldLFM (gamdebug.F90:149-175)
static void PoleE(const Model& M, const Grid& G, Arr& E) {
    const int Np = M.R.Np;
    for (int nS = M.R.nSi; nS <= M.R.nSe + 1; ++nS) {
        auto pole = [&](int j) {
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; ++k) s = s + E(nS, j, k, IDIR);
            double avg = s / Np;
            for (int k = G.ksg; k <= G.keg; ++k) { E(nS, j, k, KDIR) = 0.0; E(nS, j, k, IDIR) = avg; }
        };
        if (M.R.doS) pole(G.js);
        if (M.R.doE) pole(G.je + 1);
    }
    FixEFieldLFM(G, E);
}
// CleanLoops (ringav.F90:339-373): remove the net K flux around the first/last ring
static void CleanLoops(const Model& M, const Grid& G, State& S) {
    const int Np = M.R.Np;
    double tScl = M.R.doFastLoop ? 1.0 : 1.0 / Np;
    for (int nS = M.R.nSi; nS <= M.R.nSe + 1; ++nS) {
        auto clean = [&](int nR) {
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; ++k) s = s + S.magFlux(nS, nR, k, KDIR);
            double avgFlx = s / Np;
            for (int k = G.ks; k <= G.ke + 1; ++k) S.magFlux(nS, nR, k, KDIR) = S.magFlux(nS, nR, k, KDIR) - tScl * avgFlx;
        };
        if (M.R.doS) clean(G.js);
        if (M.R.doE) clean(G.je);
    }
}
// SmoothGas (ringav.F90:82-200), single fluid, no shift, no velocity cleaning
static void SmoothGas(const Model& M, const Grid& G, State& S, int XPOLE) {
    const int Np = M.R.Np;
#pragma omp parallel for schedule(static)
    for (int nS = M.R.nSi; nS <= M.R.nSe; ++nS) {
        std::vector<double> rW(NVAR * Np), raW(NVAR * Np);
        for (int nR = 1; nR <= M.R.NumR; ++nR) {
            int NumCh = M.R.Nch[nR - 1];
            int jR = (XPOLE == SPOLE) ? G.js + nR - 1 : G.je - nR + 1;
            for (int q = 0; q < Np; ++q)
                for (int v = 0; v < NVAR; ++v) rW[v * Np + q] = S.Gas(nS, jR, G.ks + q, v + 1);
            for (int q = 0; q < Np; ++q) {   // Gas2Ring (ringutils.F90:800-826)
                double D = fmaxd(rW[q], M.dFloor);
                double Mom[3] = {rW[Np + q], rW[2 * Np + q], rW[3 * Np + q]};
                double E = rW[4 * Np + q];
                double KinE = 0.5 * dot3(Mom, Mom) / D;
                double P = fmaxd((M.gamma - 1) * (E - KinE), M.pFloor);
                double IntE = P / (M.gamma - 1);
                rW[q] = D;
                rW[4 * Np + q] = M.R.doMassRA ? M.gamma * P : IntE;
            }
            for (int v = 0; v < NVAR; ++v) ChunkAverage(&rW[v * Np], &raW[v * Np], Np, NumCh);
            for (int v = 0; v < NVAR; ++v) ReconstructRing(M, &raW[v * Np], NumCh);
            for (int q = 0; q < Np; ++q) {   // Ring2Gas (ringutils.F90:829-856)
                double D = fmaxd(raW[q], M.dFloor);
                double Mom[3] = {raW[Np + q], raW[2 * Np + q], raW[3 * Np + q]};
                double P;
                if (!M.R.doMassRA) P = (M.gamma - 1) * raW[4 * Np + q];
                else P = (raW[4 * Np + q] / D) * D / M.gamma;
                P = fmaxd(P, M.pFloor);
                double KinE = 0.5 * dot3(Mom, Mom) / D;
                double IntE = P / (M.gamma - 1);
                raW[q] = D;
                raW[4 * Np + q] = KinE + IntE;
            }
            for (int q = 0; q < Np; ++q)
                for (int v = 0; v < NVAR; ++v) S.Gas(nS, jR, G.ks + q, v + 1) = raW[v * Np + q];
        }
    }
}
// RingAverage (ringav.F90:26-79)
static void RingAverage(const Model& M, const Grid& G, State& S, Arr& SmoothE) {
    std::fill(SmoothE.d.begin(), SmoothE.d.end(), 0.0);
    if (M.R.doS) CalcSmoothE(M, G, S, SmoothE, SPOLE);
    if (M.R.doE) CalcSmoothE(M, G, S, SmoothE, EPOLE);
    PoleE(M, G, SmoothE);
    E2Flux(G, S.magFlux, SmoothE, 1.0);
    if (M.R.doCleanLoop) CleanLoops(M, G, S);
    bFlux2Fld(M, G, S.magFlux, S.Bxyz);
    if (M.R.doS) SmoothGas(M, G, S, SPOLE);
    if (M.R.doE) SmoothGas(M, G, S, EPOLE);
}

// ---------------------------------------------------------------- the magnetosphere problem's hooks
// DiffuseOuter (wind.F90:568-618): diffusive E of the outermost I edge from the face-field current
static void DiffuseOuter(const Model& M, const Grid& G, const State& S, int i, int j, int k, double vSW, double* Ed) {
    double db2, db1, bP, bM, Jd[3] = {0.0, 0.0, 0.0};
    bP = S.magFlux(i, j, k, JDIR) / fmaxd(G.face(i, j, k, JDIR), TINY);
    bM = S.magFlux(i - 1, j, k, JDIR) / fmaxd(G.face(i - 1, j, k, JDIR), TINY);
    db2 = bP - bM;
    bP = S.magFlux(i, j, k, IDIR) / G.face(i, j, k, IDIR);
    bM = S.magFlux(i, j - 1, k, IDIR) / G.face(i, j - 1, k, IDIR);
    db1 = bP - bM;
    Jd[2] = db2 - db1;
    bP = S.magFlux(i, j, k, IDIR) / G.face(i, j, k, IDIR);
    bM = S.magFlux(i, j, k - 1, IDIR) / G.face(i, j, k - 1, IDIR);
    db2 = bP - bM;
    bP = S.magFlux(i, j, k, KDIR) / G.face(i, j, k, KDIR);
    bM = S.magFlux(i - 1, j, k, KDIR) / G.face(i - 1, j, k, KDIR);
    db1 = bP - bM;
    Jd[1] = db2 - db1;
    double dl = std::sqrt(G.edge(i, j, k, JDIR) * G.edge(i, j, k, KDIR));
    double Vd = fmind(vSW, M.CFL * dl / M.dt);
    Ed[0] = 0.0;
    Ed[1] = Vd * Jd[1] * dl;
    Ed[2] = Vd * Jd[2] * dl;
}
// WindEFix (wind.F90:489-565): the E of the outer shells' edges blended toward the wind's -V x B
static void WindEFix(const Model& M, const Grid& G, State& S) {
    const double vSW = fmind(norm2v(M.W.wV, 3), M.Ca);   // norm2 of the front velocity (-|V|, 0, 0)
    double swE[3];
    cross3(M.W.wV, M.W.wB, swE);
    for (int c = 0; c < 3; ++c) swE[c] = -swE[c];
    Arr& E = S.Efld;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.ie - 2; i <= G.ie + 1; ++i) {
                double wSW = 0.0;
                for (int n = IDIR; n <= KDIR; ++n) {
                    double e1[3], e2[3], ecc[3];
                    for (int c = 0; c < 3; ++c) {
                        e1[c] = G.xyz(i, j, k, c + 1);
                        e2[c] = G.xyz(i + (n == IDIR), j + (n == JDIR), k + (n == KDIR), c + 1);
                        ecc[c] = 0.5 * (e1[c] + e2[c]);
                    }
                    wSW = wgtWind(M, ecc);
                    if (wSW > TINY) {
                        if (i <= G.ie) wSW = wSW / (1.0 + G.ie + 1 - i);
                        double de[3] = {e2[0] - e1[0], e2[1] - e1[1], e2[2] - e1[2]};
                        E(i, j, k, n) = (1.0 - wSW) * E(i, j, k, n) + wSW * dot3(swE, de);
                    }
                }
                if (i == G.ie + 1) {   // doSWDiffuse, with the weight of the last (K) edge
                    double Ed[3];
                    DiffuseOuter(M, G, S, i, j, k, vSW, Ed);
                    for (int c = 0; c < 3; ++c) E(i, j, k, c + 1) = E(i, j, k, c + 1) + wSW * Ed[c];
                }
            }
    if (M.doRing) {
        const int Np = M.R.Np;
        for (int n = G.ie - 2; n <= G.ie + 1; ++n) {
            auto ring = [&](int j) {
                double s = 0.0;
                for (int k = G.ks; k <= G.ke; ++k) s = s + E(n, j, k, IDIR);
                double avg = s / Np;
                for (int k = G.ksg; k <= G.keg; ++k) { E(n, j, k, IDIR) = avg; E(n, j, k, KDIR) = 0.0; }
            };
            if (M.R.doE) ring(G.je + 1);
            if (M.R.doS) ring(G.js);
        }
    }
}
// EFix, the magnetosphere's HackE (earthcmi.F90:260-280): IonEFix (msphutils.F90:214-240) with zero
// ionospheric E on the first shell's J and K edges, WindEFix, FixEFieldLFM
static void EFix(const Model& M, const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j) {
            S.Efld(G.is, j, k, JDIR) = G.edge(G.is, j, k, JDIR) * 0.0;
            S.Efld(G.is, j, k, KDIR) = G.edge(G.is, j, k, KDIR) * 0.0;
        }
    WindEFix(M, G, S);
    FixEFieldLFM(G, S.Efld);
}
// PushIon (earthcmi.F90:524-606): the first nIonP shells' velocity pushed toward the (zero) E x B drift
static void PushIon(const Model& M, const Grid& G, State& S) {
    if (!M.W.doIonPush) return;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.is + M.W.nIonP - 1; ++i) {
                double pCon[5], pW[5];
                for (int v = 0; v < 5; ++v) pCon[v] = S.Gas(i, j, k, v + 1);
                CellC2P(M, pCon, pW);
                if (pCon[0] < 0.0) continue;
                int dN = i - G.is + 1;
                double dt = M.dt / (dN * M.W.dtCpl);
                dt = fmind(dt, 1.0);
                for (int c = 1; c <= 3; ++c) pW[c] = pW[c] + dt * (0.0 - pW[c]);
                CellP2C(M, pW, pCon);
                for (int v = 0; v < 5; ++v) S.Gas(i, j, k, v + 1) = pCon[v];
            }
}
// NudgeSW (wind.F90:392-486): the outermost active shell nudged toward the wind over a minute, and the cells
// next to the axis at the back of the grid kept flowing out
static void NudgeSW(const Model& M, const Grid& G, State& S) {
    const int ip = G.ie;
    const double dtSW0 = 60.0 / M.W.gT0;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j) {
            double xcc[3] = {G.xyzcc(ip, j, k, 1), G.xyzcc(ip, j, k, 2), G.xyzcc(ip, j, k, 3)};
            double wSW = wgtWind(M, xcc);
            if (wSW > TINY) {
                double dtSW = fmaxd(dtSW0 / wSW, M.dt);
                double gW_sw[5] = {M.W.wD, M.W.wV[0], M.W.wV[1], M.W.wV[2], M.W.wP};
                double gCon[5], gW_mhd[5], gW[5];
                for (int v = 0; v < 5; ++v) gCon[v] = S.Gas(ip, j, k, v + 1);
                CellC2P(M, gCon, gW_mhd);
                for (int v = 0; v < 5; ++v) gW[v] = gW_mhd[v] + (M.dt / dtSW) * (gW_sw[v] - gW_mhd[v]);
                CellP2C(M, gW, gCon);
                for (int v = 0; v < 5; ++v) S.Gas(ip, j, k, v + 1) = gCon[v];
            }
        }
    if (M.doRing && M.R.doE) {
        for (int k = G.ks; k <= G.ke; ++k)
            for (int n = 0; n <= 1; ++n) {
                int i = G.ie, j = G.je + n;
                if (S.Gas(i, j, k, MOMX) > 0) {
                    double gCon[5], B[3], gW[5];
                    for (int v = 0; v < 5; ++v) gCon[v] = S.Gas(i, j, k, v + 1);
                    for (int c = 0; c < 3; ++c) B[c] = S.Bxyz(i, j, k, c + 1);
                    double Cx = Con2Fast(M, gCon, B);
                    CellC2P(M, gCon, gW);
                    gW[1] = -Cx;
                    CellP2C(M, gW, gCon);
                    for (int v = 0; v < 5; ++v) S.Gas(i, j, k, v + 1) = gCon[v];
                }
            }
    }
}
// applyGrav (mhdgroup.F90:620-705), one fluid, classical momentum (doBorisGrav = .false.)
static void applyGrav(const Model& M, const Grid& G, State& S, const State& oS) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                if (!(S.Gas(i, j, k, DEN) >= 0.0)) continue;
                double pCon[5], pW[5];
                for (int v = 0; v < 5; ++v) pCon[v] = S.Gas(i, j, k, v + 1);
                CellC2P(M, pCon, pW);
                double IntE = pW[4] / (M.gamma - 1);
                double Dhf = 0.5 * (S.Gas(i, j, k, DEN) + oS.Gas(i, j, k, DEN));
                double cM[3];
                for (int c = 0; c < 3; ++c) cM[c] = pCon[1 + c] + M.dt * Dhf * G.gxyz(i, j, k, c + 1);
                for (int c = 0; c < 3; ++c) pCon[1 + c] = cM[c];
                pCon[4] = IntE + 0.5 * dot3(cM, cM) / pCon[0];
                for (int v = 0; v < 5; ++v) S.Gas(i, j, k, v + 1) = pCon[v];
            }
}

// ---------------------------------------------------------------- one step (gamapp.F90:73-116, mhdgroup.F90:16-76)
static void AdvanceMHD(App& A, double dt) {
    Model& M = A.M;
    if (std::fabs(A.oS.time - A.S.time) < TINY) A.oS.time = A.S.time - M.dt;
    Predictor(M, A.G, A.S, A.oS, A.V.StateHf, 0.5 * dt);
    if (M.doMHD) {
        CalcElecField(M, A.G, A.S, A.V.StateHf, A.V.Vf, A.S.Efld);
        if (M.W.on) EFix(M, A.G, A.S);   // HackE, mhdgroup.F90:40-44
    }
    CalcStress(M, A.G, A.S, A.V.StateHf, A.V.gFlx, A.V.mFlx, A.V.dGasH, A.V.dGasM);
    applyUpdate(M, A.G, A.S, A.oS, dt, A.V.dGasH, A.V.dGasM, A.S.Efld);
    if (M.doGrav) applyGrav(M, A.G, A.S, A.oS);   // mhdgroup.F90:60-65
    if (M.doRing && (M.R.doS || M.R.doE)) RingAverage(M, A.G, A.S, A.V.SmoothE);   // mhdgroup.F90:68-74
}
static void stepGamera(App& A) {
    AdvanceMHD(A, A.M.dt);
    if (A.M.W.on) { PushIon(A.M, A.G, A.S); NudgeSW(A.M, A.G, A.S); }   // HackStep, gamapp.F90:104-109
    A.M.ts = A.M.ts + 1;
    A.M.t = A.M.t + A.M.dt;
    A.M.dt = CalcDT(A.M, A.G, A.S);
    EnforceBCs(A.M, A.G, A.S);
    bFlux2Fld(A.M, A.G, A.S.magFlux, A.S.Bxyz);
}

// ---------------------------------------------------------------- setup (init.F90, quadrature.F90, metric.F90)
static const double gA[12] = {0.1252334085114689154724, 0.3678314989981801937527, 0.5873179542866174472967,
                              0.7699026741943046870369, 0.9041172563704748566785, 0.9815606342467192506906,
                              -0.1252334085114689154724, -0.3678314989981801937527, -0.5873179542866174472967,
                              -0.7699026741943046870369, -0.9041172563704748566785, -0.9815606342467192506906};
static const double gWgt[12] = {0.2491470458134027850006, 0.233492536538354808761, 0.203167426723065921749,
                                0.160078328543346226335, 0.1069393259953184309603, 0.0471753363865118271946,
                                0.2491470458134027850006, 0.233492536538354808761, 0.203167426723065921749,
                                0.160078328543346226335, 0.1069393259953184309603, 0.0471753363865118271946};

static void faceCoords(const Grid& G, int i, int j, int k, int d, double* f0, double* f1, double* f2, double* f3) {
    for (int c = 0; c < 3; ++c) {
        f0[c] = G.xyz(i, j, k, c + 1);
        if (d == IDIR) { f1[c] = G.xyz(i, j + 1, k, c + 1); f2[c] = G.xyz(i, j, k + 1, c + 1); f3[c] = G.xyz(i, j + 1, k + 1, c + 1); }
        else if (d == JDIR) { f1[c] = G.xyz(i, j, k + 1, c + 1); f2[c] = G.xyz(i + 1, j, k, c + 1); f3[c] = G.xyz(i + 1, j, k + 1, c + 1); }
        else { f1[c] = G.xyz(i + 1, j, k, c + 1); f2[c] = G.xyz(i, j + 1, k, c + 1); f3[c] = G.xyz(i + 1, j + 1, k, c + 1); }
    }
}
static void cellCoords(const Grid& G, int i, int j, int k, double xyzC[8][3]) {
    const int di[8] = {0, 1, 1, 0, 0, 1, 1, 0}, dj[8] = {0, 0, 1, 1, 0, 0, 1, 1}, dk[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    for (int p = 0; p < 8; ++p) for (int c = 0; c < 3; ++c) xyzC[p][c] = G.xyz(i + di[p], j + dj[p], k + dk[p], c + 1);
}

typedef void (*VecFun)(double, double, double, double*, void*);
typedef void (*GasFun)(double, double, double, double*, void*);

// GaussianFaceIntegral (quadrature.F90:159-221), returns fInt only (fInt2/fIntX are unused by the callers here)
static void GaussianFaceIntegral(const double* f0, const double* f1, const double* f2, const double* f3, VecFun A,
                                 void* ctx, double* fInt) {
    double dx[3], dy[3], dz[3];
    dx[0] = f1[0] - f0[0]; dx[1] = f2[0] - f0[0]; dx[2] = f3[0] + f0[0] - f2[0] - f1[0];
    dy[0] = f1[1] - f0[1]; dy[1] = f2[1] - f0[1]; dy[2] = f3[1] + f0[1] - f2[1] - f1[1];
    dz[0] = f1[2] - f0[2]; dz[1] = f2[2] - f0[2]; dz[2] = f3[2] + f0[2] - f2[2] - f1[2];
    fInt[0] = fInt[1] = fInt[2] = 0.0;
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            double eta = 0.5 * (1 + gA[i]), psi = 0.5 * (1 + gA[j]);
            double w = gWgt[i] * gWgt[j];
            double xp = f0[0] + dx[0] * eta + dx[1] * psi + dx[2] * eta * psi;
            double yp = f0[1] + dy[0] * eta + dy[1] * psi + dy[2] * eta * psi;
            double zp = f0[2] + dz[0] * eta + dz[1] * psi + dz[2] * eta * psi;
            double Ap[3];
            A(xp, yp, zp, Ap, ctx);
            double etaV[3] = {dx[0] + dx[2] * psi, dy[0] + dy[2] * psi, dz[0] + dz[2] * psi};
            double psiV[3] = {dx[1] + dx[2] * eta, dy[1] + dy[2] * eta, dz[1] + dz[2] * eta};
            double cr[3];
            cross3(etaV, psiV, cr);
            double area = 0.25 * norm2v(cr, 3) * w;
            fInt[0] = fInt[0] + area * Ap[0];
            fInt[1] = fInt[1] + area * Ap[1];
            fInt[2] = fInt[2] + area * Ap[2];
        }
}
static double DetJ(double J[3][3]) {  // math.F90:470-478, J[row][col]
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}
// GaussianVolumeIntegral (quadrature.F90:42-100)
static void GaussianVolumeIntegral(double xyzC[8][3], GasFun W, void* ctx, double* wInt) {
    const int iS[8] = {-1, +1, +1, -1, -1, +1, +1, -1}, jS[8] = {-1, -1, +1, +1, -1, -1, +1, +1},
              kS[8] = {-1, -1, -1, -1, +1, +1, +1, +1};
    for (int v = 0; v < 5; ++v) wInt[v] = 0.0;
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j)
            for (int k = 0; k < 12; ++k) {
                double wijk = gWgt[i] * gWgt[j] * gWgt[k];
                double iScl[8], jScl[8], kScl[8];
                for (int p = 0; p < 8; ++p) {
                    iScl[p] = (iS[p] < 0) ? (1 - gA[i]) : (1 + gA[i]);
                    jScl[p] = (jS[p] < 0) ? (1 - gA[j]) : (1 + gA[j]);
                    kScl[p] = (kS[p] < 0) ? (1 - gA[k]) : (1 + gA[k]);
                }
                double xp[3], Jac[3][3];
                for (int c = 0; c < 3; ++c) {
                    double s = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                    for (int p = 0; p < 8; ++p) s = s + xyzC[p][c] * (iScl[p] * jScl[p] * kScl[p]);
                    for (int p = 0; p < 8; ++p) s1 = s1 + xyzC[p][c] * (iS[p] * jScl[p] * kScl[p]);
                    for (int p = 0; p < 8; ++p) s2 = s2 + xyzC[p][c] * (iScl[p] * jS[p] * kScl[p]);
                    for (int p = 0; p < 8; ++p) s3 = s3 + xyzC[p][c] * (iScl[p] * jScl[p] * kS[p]);
                    xp[c] = 0.125 * s;
                    Jac[c][0] = 0.125 * s1; Jac[c][1] = 0.125 * s2; Jac[c][2] = 0.125 * s3;
                }
                double dJ = std::fabs(DetJ(Jac));
                double Wp[5];
                W(xp[0], xp[1], xp[2], Wp, ctx);
                for (int v = 0; v < 5; ++v) wInt[v] = wInt[v] + dJ * wijk * Wp[v];
            }
}
// GaussianEdgeIntegral (quadrature.F90:345-370)
static void GaussianEdgeIntegral(const double* e1, const double* e2, VecFun A, void* ctx, double* eInt) {
    double dR2[3], xBar[3];
    for (int c = 0; c < 3; ++c) { dR2[c] = 0.5 * (e2[c] - e1[c]); xBar[c] = 0.5 * (e2[c] + e1[c]); }
    eInt[0] = eInt[1] = eInt[2] = 0.0;
    for (int i = 0; i < 12; ++i) {
        double xp[3], Ap[3];
        for (int c = 0; c < 3; ++c) xp[c] = xBar[c] + gA[i] * dR2[c];
        A(xp[0], xp[1], xp[2], Ap, ctx);
        for (int c = 0; c < 3; ++c) eInt[c] = eInt[c] + 0.5 * gWgt[i] * Ap[c];
    }
}
static void IdVec(double, double, double, double* A, void*) { A[0] = A[1] = A[2] = 1.0; }
static void rVec(double x, double y, double z, double* A, void*) { A[0] = x; A[1] = y; A[2] = z; }
static void CellDV(double x, double y, double z, double* W, void*) { W[0] = 1; W[1] = x; W[2] = y; W[3] = z; W[4] = 0; }

static void allocGrid(const Model& M, Grid& G) {
    G.Ni = G.Nip + 2 * M.nG; G.Nj = G.Njp + 2 * M.nG; G.Nk = G.Nkp + 2 * M.nG;
    G.is = 1; G.ie = G.Nip; G.js = 1; G.je = G.Njp; G.ks = 1; G.ke = G.Nkp;
    G.isg = G.is - M.nG; G.ieg = G.ie + M.nG; G.jsg = G.js - M.nG; G.jeg = G.je + M.nG;
    G.ksg = G.ks - M.nG; G.keg = G.ke + M.nG;
    int lo4[4] = {G.isg, G.jsg, G.ksg, 1};
    int hi4p[4] = {G.ieg + 1, G.jeg + 1, G.keg + 1, 3};
    G.xyz.alloc(4, lo4, hi4p);
}

// SetDomain (init.F90:519-538) for a single untiled grid
static void SetDomain(Grid& G) {
    G.isDT = G.is - 1; G.ieDT = G.ie + 1; G.jsDT = G.js - 1; G.jeDT = G.je + 1; G.ksDT = G.ks - 1; G.keDT = G.ke + 1;
}

// InitRings for the LFM axis (ringutils.F90:37-226): Np = Nkp and the default chunking per ring
static int InitRingsLFM(Model& M, const Grid& G, int NumR, const int* Nch) {
    Ring& R = M.R;
    R.Np = G.Nkp; R.nSi = G.is; R.nSe = G.ie;
    R.doS = true; R.doE = true;   // untiled: both sides of the axis
    static const int c8[] = {4}, c16[] = {8}, c32[] = {8, 16}, c64[] = {8, 16, 32, 32},
                     c128[] = {8, 16, 32, 32, 64, 64, 64, 64}, c256[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128},
                     c512[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 256, 256, 256, 256};
    const int* NCr = nullptr;
    int Nr = 0;
    switch (R.Np) {
    case 8: NCr = c8; Nr = 1; break;
    case 16: NCr = c16; Nr = 1; break;
    case 32: NCr = c32; Nr = 2; break;
    case 64: NCr = c64; Nr = 4; break;
    case 128: NCr = c128; Nr = 8; break;
    case 256: NCr = c256; Nr = 12; break;
    case 512: NCr = c512; Nr = 16; break;
    default: return -1;
    }
    R.NumR = NumR > 0 ? NumR : Nr;
    if (R.NumR > 32) return -1;
    for (int iR = 1; iR <= R.NumR; ++iR) {
        int iLim = std::min(iR, Nr);
        R.Nch[iR - 1] = (Nch && Nch[iR - 1] > 0) ? Nch[iR - 1] : NCr[iLim - 1];
        if (R.Np % R.Nch[iR - 1] != 0) return -1;
    }
    if (R.NumR >= G.Njp) return -1;
    return 0;
}
// RingGridFix for the LFM axis (ringutils.F90:229-377): widen dk of the ring cells by the chunk size and copy
// the ghost metrics across the axis from the conjugate cells/faces (normals of J and K faces flip sign)
static void RingGridFix(const Model& M, Grid& G) {
    const int Np = M.R.Np;
    for (int iR = 1; iR <= M.R.NumR; ++iR) {
        int dJ = Np / M.R.Nch[iR - 1];
        for (int k = G.ksg; k <= G.keg; ++k)
            for (int i = G.isg; i <= G.ieg; ++i) {
                if (M.R.doS) G.dk(i, G.js + iR - 1, k) = dJ * G.dk(i, G.js + iR - 1, k);
                if (M.R.doE) G.dk(i, G.je - iR + 1, k) = dJ * G.dk(i, G.je - iR + 1, k);
            }
    }
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int i = G.isg; i <= G.ieg + 1; ++i)
            for (int n = 1; n <= M.nG; ++n)
                for (int side = 0; side < 2; ++side) {
                    if (side == 0 && !M.R.doS) continue;
                    if (side == 1 && !M.R.doE) continue;
                    int ig = i, kg = k, jg = side == 0 ? G.js - n : G.je + n, ip, jp, kp;
                    if (kg <= G.keg && ig <= G.ieg) {
                        lfmIJKcc(M, G, ig, jg, kg, ip, jp, kp);
                        G.volume(ig, jg, kg) = G.volume(ip, jp, kp);
                        G.di(ig, jg, kg) = G.di(ip, jp, kp);
                        G.dj(ig, jg, kg) = G.dj(ip, jp, kp);
                        G.dk(ig, jg, kg) = G.dk(ip, jp, kp);
                    }
                    lfmIJKfc(M, G, IDIR, ig, jg, kg, ip, jp, kp);
                    for (int c = 0; c < 3; ++c) G.Tf(ig, jg, kg, NORMX + c, IDIR) = G.Tf(ip, jp, kp, NORMX + c, IDIR);
                    G.face(ig, jg, kg, IDIR) = G.face(ip, jp, kp, IDIR);
                    int jf = side == 0 ? jg : jg + 1;   // the first outer J ghost face is je+2
                    lfmIJKfc(M, G, JDIR, ig, jf, kg, ip, jp, kp);
                    for (int c = 0; c < 3; ++c) G.Tf(ig, jf, kg, NORMX + c, JDIR) = -G.Tf(ip, jp, kp, NORMX + c, JDIR);
                    G.face(ig, jf, kg, JDIR) = G.face(ip, jp, kp, JDIR);
                    lfmIJKfc(M, G, KDIR, ig, jg, kg, ip, jp, kp);
                    for (int c = 0; c < 3; ++c) G.Tf(ig, jg, kg, NORMX + c, KDIR) = -G.Tf(ip, jp, kp, NORMX + c, KDIR);
                    G.face(ig, jg, kg, KDIR) = G.face(ip, jp, kp, KDIR);
                }
}

// The arrays Corners2Grid fills, allocated with its shapes but left for the caller to set (a grid whose
// metrics come from elsewhere, e.g. a slab of a device-built grid)
static void allocGridMetrics(Grid& G) {
    int lo[5] = {G.isg, G.jsg, G.ksg, 1, 1};
    int hi[5] = {G.ieg, G.jeg, G.keg, 3, 3};
    G.xyzcc.alloc(4, lo, hi);
    G.volume.alloc(3, lo, hi); G.di.alloc(3, lo, hi); G.dj.alloc(3, lo, hi); G.dk.alloc(3, lo, hi);
    hi[0] = G.ieg + 1; hi[1] = G.jeg + 1; hi[2] = G.keg + 1;
    G.xfc.alloc(5, lo, hi);
    G.face.alloc(4, lo, hi);
    G.edge.alloc(4, lo, hi);
    hi[3] = 9;
    G.Tf.alloc(5, lo, hi);
    G.Te.alloc(5, lo, hi);
    hi[3] = 4;
    G.Teb.alloc(5, lo, hi);
}

static int Corners2Grid(const Model& M, Grid& G) {  // init.F90:801-1080
    if ((G.ie - G.is + 1) < vecLen) return -1;
    if (((G.ie - G.is + 1) % 8) != 0) return -2;
    int lo[5], hi[5];
    lo[0] = G.isg; lo[1] = G.jsg; lo[2] = G.ksg; lo[3] = 1; lo[4] = 1;
    hi[0] = G.ieg; hi[1] = G.jeg; hi[2] = G.keg; hi[3] = 3;
    G.xyzcc.alloc(4, lo, hi);
    hi[0] = G.ieg + 1; hi[1] = G.jeg + 1; hi[2] = G.keg + 1; hi[3] = 3; hi[4] = 3;
    G.xfc.alloc(5, lo, hi);
    G.face.alloc(4, lo, hi);
    std::fill(G.face.d.begin(), G.face.d.end(), 1.0);
    hi[3] = 9; hi[4] = 3;
    G.Tf.alloc(5, lo, hi);
    for (int d = 1; d <= 3; ++d) {
        int DelI = ijkD(d, IDIR), DelJ = ijkD(d, JDIR), DelK = ijkD(d, KDIR);
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = G.ksg; k <= G.keg + DelK; ++k)
            for (int j = G.jsg; j <= G.jeg + DelJ; ++j)
                for (int i = G.isg; i <= G.ieg + DelI; ++i) {
                    double f0[3], f1[3], f2[3], f3[3], fInt[3];
                    faceCoords(G, i, j, k, d, f0, f1, f2, f3);
                    GaussianFaceIntegral(f0, f1, f2, f3, IdVec, nullptr, fInt);
                    double fA = fInt[0];
                    GaussianFaceIntegral(f0, f1, f2, f3, rVec, nullptr, fInt);
                    for (int c = 0; c < 3; ++c) G.xfc(i, j, k, c + 1, d) = fInt[c] / fA;
                    G.face(i, j, k, d) = fA;
                    double dT1[3], dT2[3];
                    for (int c = 1; c <= 3; ++c) {
                        if (d == IDIR) {
                            dT1[c - 1] = 0.5 * (G.xyz(i, j + 1, k + 1, c) - G.xyz(i, j, k + 1, c)) + 0.5 * (G.xyz(i, j + 1, k, c) - G.xyz(i, j, k, c));
                            dT2[c - 1] = 0.5 * (G.xyz(i, j + 1, k + 1, c) - G.xyz(i, j + 1, k, c)) + 0.5 * (G.xyz(i, j, k + 1, c) - G.xyz(i, j, k, c));
                        } else if (d == JDIR) {
                            dT1[c - 1] = 0.5 * (G.xyz(i + 1, j, k + 1, c) - G.xyz(i + 1, j, k, c)) + 0.5 * (G.xyz(i, j, k + 1, c) - G.xyz(i, j, k, c));
                            dT2[c - 1] = 0.5 * (G.xyz(i + 1, j, k + 1, c) - G.xyz(i, j, k + 1, c)) + 0.5 * (G.xyz(i + 1, j, k, c) - G.xyz(i, j, k, c));
                        } else {
                            dT1[c - 1] = 0.5 * (G.xyz(i + 1, j + 1, k, c) - G.xyz(i, j + 1, k, c)) + 0.5 * (G.xyz(i + 1, j, k, c) - G.xyz(i, j, k, c));
                            dT2[c - 1] = 0.5 * (G.xyz(i + 1, j + 1, k, c) - G.xyz(i + 1, j, k, c)) + 0.5 * (G.xyz(i, j + 1, k, c) - G.xyz(i, j, k, c));
                        }
                    }
                    double cr[3], eN[3], eT1[3], eT2[3];
                    cross3(dT1, dT2, cr);
                    double ncr = norm2v(cr, 3);
                    for (int c = 0; c < 3; ++c) eN[c] = cr[c] / ncr;
                    double nT2 = norm2v(dT2, 3);
                    for (int c = 0; c < 3; ++c) eT2[c] = dT2[c] / nT2;
                    cross3(eT2, eN, cr);
                    ncr = norm2v(cr, 3);
                    for (int c = 0; c < 3; ++c) eT1[c] = cr[c] / ncr;
                    for (int c = 0; c < 3; ++c) {
                        G.Tf(i, j, k, NORMX + c, d) = eN[c];
                        G.Tf(i, j, k, TAN1X + c, d) = eT1[c];
                        G.Tf(i, j, k, TAN2X + c, d) = eT2[c];
                    }
                }
    }
    hi[0] = G.ieg; hi[1] = G.jeg; hi[2] = G.keg;
    G.volume.alloc(3, lo, hi); G.di.alloc(3, lo, hi); G.dj.alloc(3, lo, hi); G.dk.alloc(3, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i) {
                double dI[3], dJ[3], dK[3];
                for (int c = 1; c <= 3; ++c) {
                    dI[c - 1] = G.xfc(i + 1, j, k, c, IDIR) - G.xfc(i, j, k, c, IDIR);
                    dJ[c - 1] = G.xfc(i, j + 1, k, c, JDIR) - G.xfc(i, j, k, c, JDIR);
                    dK[c - 1] = G.xfc(i, j, k + 1, c, KDIR) - G.xfc(i, j, k, c, KDIR);
                }
                G.di(i, j, k) = norm2v(dI, 3); G.dj(i, j, k) = norm2v(dJ, 3); G.dk(i, j, k) = norm2v(dK, 3);
                double xyzC[8][3], ijkDV[5];
                cellCoords(G, i, j, k, xyzC);
                GaussianVolumeIntegral(xyzC, CellDV, nullptr, ijkDV);
                G.volume(i, j, k) = ijkDV[0];
                for (int c = 0; c < 3; ++c) G.xyzcc(i, j, k, c + 1) = ijkDV[1 + c] / ijkDV[0];
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i) {
                double fA = fmaxd(G.face(i + 1, j, k, IDIR), G.face(i, j, k, IDIR));
                G.di(i, j, k) = G.volume(i, j, k) / fA;
                fA = fmaxd(G.face(i, j + 1, k, JDIR), G.face(i, j, k, JDIR));
                G.dj(i, j, k) = G.volume(i, j, k) / fA;
                fA = fmaxd(G.face(i, j, k + 1, KDIR), G.face(i, j, k, KDIR));
                G.dk(i, j, k) = G.volume(i, j, k) / fA;
            }
    if (M.doRing) RingGridFix(M, G);   // init.F90:967-968
    hi[0] = G.ieg + 1; hi[1] = G.jeg + 1; hi[2] = G.keg + 1; hi[3] = 3;
    G.edge.alloc(4, lo, hi);
    std::fill(G.edge.d.begin(), G.edge.d.end(), 1.0);
    hi[3] = 9; hi[4] = 3;
    G.Te.alloc(5, lo, hi);
    for (int d = 1; d <= 3; ++d) {
        int is = G.isg, ie = G.ieg + 1, js = G.jsg, je = G.jeg + 1, ks = G.ksg, ke = G.keg + 1;
        if (d == IDIR) { ie = G.ieg; ks = G.ksg + 1; ke = G.keg; }
        else if (d == JDIR) { je = G.jeg; is = G.isg + 1; ie = G.ieg; }
        else { ke = G.keg; js = G.jsg + 1; je = G.jeg; }
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = ks; k <= ke; ++k)
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) {
                    double dEdge[3], eAvg[3];
                    for (int c = 1; c <= 3; ++c) {
                        if (d == IDIR) {
                            dEdge[c - 1] = G.xyz(i + 1, j, k, c) - G.xyz(i, j, k, c);
                            eAvg[c - 1] = 0.5 * (G.xyz(i, j, k + 1, c) - G.xyz(i, j, k - 1, c) + G.xyz(i + 1, j, k + 1, c) - G.xyz(i + 1, j, k - 1, c));
                        } else if (d == JDIR) {
                            dEdge[c - 1] = G.xyz(i, j + 1, k, c) - G.xyz(i, j, k, c);
                            eAvg[c - 1] = 0.5 * (G.xyz(i + 1, j, k, c) - G.xyz(i - 1, j, k, c) + G.xyz(i + 1, j + 1, k, c) - G.xyz(i - 1, j + 1, k, c));
                        } else {
                            dEdge[c - 1] = G.xyz(i, j, k + 1, c) - G.xyz(i, j, k, c);
                            eAvg[c - 1] = 0.5 * (G.xyz(i, j + 1, k, c) - G.xyz(i, j - 1, k, c) + G.xyz(i, j + 1, k + 1, c) - G.xyz(i, j - 1, k + 1, c));
                        }
                    }
                    double nE = norm2v(dEdge, 3), eN[3], eT1[3], eT2[3], cr[3];
                    for (int c = 0; c < 3; ++c) eN[c] = dEdge[c] / nE;
                    cross3(eAvg, eN, cr);
                    double ncr = norm2v(cr, 3);
                    for (int c = 0; c < 3; ++c) eT1[c] = cr[c] / ncr;
                    cross3(eN, eT1, cr);
                    ncr = norm2v(cr, 3);
                    for (int c = 0; c < 3; ++c) eT2[c] = cr[c] / ncr;
                    G.edge(i, j, k, d) = norm2v(dEdge, 3);
                    for (int c = 0; c < 3; ++c) {
                        G.Te(i, j, k, NORMX + c, d) = eN[c];
                        G.Te(i, j, k, TAN1X + c, d) = eT1[c];
                        G.Te(i, j, k, TAN2X + c, d) = eT2[c];
                    }
                }
    }
    hi[3] = 4; hi[4] = 3;
    G.Teb.alloc(5, lo, hi);
    std::fill(G.Teb.d.begin(), G.Teb.d.end(), 1.0);   // ebGeom initialises nQ = 1.0 everywhere
    const long faceN = (long)(G.Ni + 1) * (G.Nj + 1) * (G.Nk + 1);
    for (int dNorm = 1; dNorm <= 3; ++dNorm) {
        int T1, T2;
        if (dNorm == IDIR) { T1 = JDIR; T2 = KDIR; } else if (dNorm == JDIR) { T1 = KDIR; T2 = IDIR; } else { T1 = IDIR; T2 = JDIR; }
        for (int pass = 0; pass < 2; ++pass) {  // ebGeom (init.F90:1083-1145)
            int dT1 = pass == 0 ? T1 : T2, dT2 = pass == 0 ? T2 : T1;
            int c0 = pass == 0 ? XNQI : XNQJ;
            int ie = G.ie + 1;
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = G.ks; k <= G.ke + 1; ++k)
                for (int j = G.js; j <= G.je + 1; ++j)
                    for (int iB = G.is; iB <= ie; iB += vecLen) {
                        int iMax = std::min((int)vecLen, ie - iB + 1);
                        double fArB[recLen][vecLen], NB[3][recLen][vecLen];
                        loadBlock(G, fArB, G.face.d.data() + (dT1 - 1) * faceN, iB, j, k, iMax, dT2, Nr2, true);
                        for (int c = 0; c < 3; ++c)
                            loadBlock(G, NB[c], G.Tf.d.data() + (long)(NORMX - 1 + c) * faceN + (long)(dT1 - 1) * 9 * faceN, iB, j, k, iMax, dT2, Nr2, true);
                        for (int i = 0; i < iMax; ++i) {
                            int iG = iB + i;
                            double fAi = 0.0;
                            for (int n = 0; n < recLen; ++n) fAi = fAi + interpWgt6[n] * fArB[n][i];
                            double Nec[3];
                            for (int c = 0; c < 3; ++c) {
                                double s = 0.0;
                                for (int n = 0; n < recLen; ++n) s = s + (NB[c][n][i] * fArB[n][i]) * interpWgt6[n];
                                Nec[c] = s / fAi;
                            }
                            double t1[3] = {G.Te(iG, j, k, TAN1X, dNorm), G.Te(iG, j, k, TAN1Y, dNorm), G.Te(iG, j, k, TAN1Z, dNorm)};
                            double t2[3] = {G.Te(iG, j, k, TAN2X, dNorm), G.Te(iG, j, k, TAN2Y, dNorm), G.Te(iG, j, k, TAN2Z, dNorm)};
                            double dxT = dot3(Nec, t1), dyT = dot3(Nec, t2);
                            double dScl = std::sqrt(sq(dxT) + sq(dyT));
                            if (dScl <= TINY) dScl = 1.0;
                            G.Teb(iG, j, k, c0, dNorm) = dxT / dScl;
                            G.Teb(iG, j, k, c0 + 1, dNorm) = dyT / dScl;
                        }
                    }
        }
    }
    return 0;
}

static void allocState(const Model& M, const Grid& G, State& S) {
    int lo[4] = {G.isg, G.jsg, G.ksg, 1};
    int hi[4] = {G.ieg, G.jeg, G.keg, 5};
    S.Gas.alloc(4, lo, hi);
    hi[3] = 3;
    S.Efld.alloc(4, lo, hi);
    S.Bxyz.alloc(4, lo, hi);
    int hip[4] = {G.ieg + 1, G.jeg + 1, G.keg + 1, 3};
    S.magFlux.alloc(4, lo, hip);
    S.time = M.t;
}

// ICs (prob.F90)
static void initOT2D(const Model& M, Grid& G, State& S) {  // prob.F90:74-119
    double Rho0 = 25.0 / (36.0 * PI), P0 = 5 / (12.0 * PI), B0 = 1 / std::sqrt(4.0 * PI);
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double xc = G.xyzcc(i, j, k, 1), yc = G.xyzcc(i, j, k, 2);
                S.Gas(i, j, k, DEN) = Rho0;
                double Vx = -std::sin(2 * PI * yc), Vy = std::sin(2 * PI * xc), Vz = 0.0;
                double KinE = 0.5 * Rho0 * (sq(Vx) + sq(Vy) + sq(Vz));
                S.Gas(i, j, k, MOMX) = Vx * Rho0;
                S.Gas(i, j, k, MOMY) = Vy * Rho0;
                S.Gas(i, j, k, MOMZ) = Vz * Rho0;
                S.Gas(i, j, k, ENERGY) = KinE + P0 / (M.gamma - 1);
                S.magFlux(i, j, k, XDIR) = (-B0 * std::sin(2 * PI * yc)) * G.face(i, j, k, XDIR);
                S.magFlux(i, j, k, YDIR) = (B0 * std::sin(4 * PI * xc)) * G.face(i, j, k, YDIR);
                S.magFlux(i, j, k, ZDIR) = 0.0;
            }
}

// Kelvin-Helmholtz shear layer of the batched-ensemble problem (no reference counterpart), sampled at cell
// centres: rho = 1, P = 1, Vx = 0.5 tanh((y-0.5)/a), Vy = amp*(2u-1) with u a counter-based hash of
// (seed, i, j, k), B = (Bx, 0, 0) as face fluxes Bx*n_x*area. kh = {a, Bx, amp, seed}.
static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double khNoise(uint64_t seed, int i, int j, int k) {   // u in [0,1), i,j,k counted from is = 1
    uint64_t key = (seed << 40) ^ (uint64_t)(uint32_t)(i + 4096 * (j + 4096 * k));
    return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}
static void initKH(const Model& M, Grid& G, State& S, const double* kh) {
    double a = kh[0], Bx = kh[1], amp = kh[2];
    uint64_t seed = (uint64_t)kh[3];
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double yc = G.xyzcc(i, j, k, 2);
                double D = 1.0, P = 1.0;
                double Vx = 0.5 * std::tanh((yc - 0.5) / a);
                double Vy = amp * (2.0 * khNoise(seed, i, j, k) - 1.0), Vz = 0.0;
                double KinE = 0.5 * D * (sq(Vx) + sq(Vy) + sq(Vz));
                S.Gas(i, j, k, DEN) = D;
                S.Gas(i, j, k, MOMX) = D * Vx; S.Gas(i, j, k, MOMY) = D * Vy; S.Gas(i, j, k, MOMZ) = D * Vz;
                S.Gas(i, j, k, ENERGY) = KinE + P / (M.gamma - 1);
                for (int d = 1; d <= 3; ++d) S.magFlux(i, j, k, d) = Bx * G.Tf(i, j, k, NORMX, d) * G.face(i, j, k, d);
            }
}

struct BWctx { double x0, y0, z0, Vx0, Vy0, Vz0, P0, pRat, dRat, D0, rC, bScl, bSclz; };
static void GasIC_BW(double x, double y, double z, double* W, void* c) {  // prob.F90:280-297
    BWctx* b = (BWctx*)c;
    double R = std::sqrt(sq(x - b->x0) + sq(y - b->y0) + sq(z - b->z0));
    double D = b->D0, P = b->P0;
    if (R <= b->rC) { D = b->dRat * D; P = b->pRat * P; }
    W[0] = D; W[1] = b->Vx0; W[2] = b->Vy0; W[3] = b->Vz0; W[4] = P;
}
static void VectorPot_BW(double x, double y, double z, double* A, void* c) {  // prob.F90:271-278
    (void)z;
    BWctx* b = (BWctx*)c;
    A[0] = 0.0; A[1] = b->bSclz * x; A[2] = b->bScl * (y - x);
}
static void GasIC2State(const Model& M, const Grid& G, State& S, GasFun W, void* ctx) {  // gridutils.F90:144-189
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double xyzC[8][3], ijkW[5];
                cellCoords(G, i, j, k, xyzC);
                double dV = G.volume(i, j, k);
                GaussianVolumeIntegral(xyzC, W, ctx, ijkW);
                for (int v = 0; v < 5; ++v) ijkW[v] = ijkW[v] / dV;
                double D = ijkW[0], Mx = D * ijkW[1], My = D * ijkW[2], Mz = D * ijkW[3], P = ijkW[4];
                double KinE = 0.5 * (sq(Mx) + sq(My) + sq(Mz)) / D;
                double IntE = P / (M.gamma - 1.0);
                S.Gas(i, j, k, DEN) = D; S.Gas(i, j, k, MOMX) = Mx; S.Gas(i, j, k, MOMY) = My;
                S.Gas(i, j, k, MOMZ) = Mz; S.Gas(i, j, k, ENERGY) = IntE + KinE;
            }
}
static void VectorPot2Flux(const Grid& G, State& S, VecFun Axyz, void* ctx) {  // gridutils.F90:193-237
    Arr lA;
    int lo[4] = {G.isg, G.jsg, G.ksg, 1}, hi[4] = {G.ieg, G.jeg, G.keg, 3};
    lA.alloc(4, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg - 1; ++k)
        for (int j = G.jsg; j <= G.jeg - 1; ++j)
            for (int i = G.isg; i <= G.ieg - 1; ++i) {
                double e0[3], eI[3], eJ[3], eK[3], I[3], d[3];
                for (int c = 0; c < 3; ++c) {
                    e0[c] = G.xyz(i, j, k, c + 1); eI[c] = G.xyz(i + 1, j, k, c + 1);
                    eJ[c] = G.xyz(i, j + 1, k, c + 1); eK[c] = G.xyz(i, j, k + 1, c + 1);
                }
                GaussianEdgeIntegral(eI, e0, Axyz, ctx, I);
                for (int c = 0; c < 3; ++c) d[c] = eI[c] - e0[c];
                lA(i, j, k, IDIR) = dot3(I, d);
                GaussianEdgeIntegral(eJ, e0, Axyz, ctx, I);
                for (int c = 0; c < 3; ++c) d[c] = eJ[c] - e0[c];
                lA(i, j, k, JDIR) = dot3(I, d);
                GaussianEdgeIntegral(eK, e0, Axyz, ctx, I);
                for (int c = 0; c < 3; ++c) d[c] = eK[c] - e0[c];
                lA(i, j, k, KDIR) = dot3(I, d);
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg - 1; ++k)
        for (int j = G.jsg; j <= G.jeg - 1; ++j)
            for (int i = G.isg; i <= G.ieg - 1; ++i) {
                S.magFlux(i, j, k, IDIR) = lA(i, j, k, JDIR) - lA(i, j, k + 1, JDIR) + lA(i, j + 1, k, KDIR) - lA(i, j, k, KDIR);
                S.magFlux(i, j, k, JDIR) = -(lA(i, j, k, IDIR) - lA(i, j, k + 1, IDIR) + lA(i + 1, j, k, KDIR) - lA(i, j, k, KDIR));
                S.magFlux(i, j, k, KDIR) = lA(i, j, k, IDIR) - lA(i, j + 1, k, IDIR) + lA(i + 1, j, k, JDIR) - lA(i, j, k, JDIR);
            }
}
// ---------------------------------------------------------------- background field (background.F90:20-167)
// type 1: uniform (bx,by,bz); 2: dipole of moment M0 along z centred at (bx,by,bz) (the reference's
// magnetosphere dipole is the centre-at-origin case; the offset keeps the singularity off a test domain)
struct B0ctx { int type; double bx, by, bz, M0; double rCut = 0, lCut = 0, dcScl = 1; };
static double RampUpE(double r, double rC, double lC) {   // RampUp, math.F90:174-189
    double rScl = (r - rC) / lC;
    if (rScl <= 0.0) return 0.0;
    if (rScl >= 1.0) return 1.0;
    double eArg = -1.0 / (rScl * rScl);
    return (double)std::exp(1.0f) * std::exp(eArg);   // exp(1.0) of a default-real literal
}
static double PenticRampDown(double r, double rC, double lC) {   // math.F90:156-172 (msphutils' magRampDown)
    double rScl = (r - rC) / lC;
    if (rScl <= 0.0) return 1.0;
    if (rScl >= 1.0) return 0.0;
    double Mc = 6 * std::pow(rScl, 5.0) - 15 * std::pow(rScl, 4.0) + 10 * std::pow(rScl, 3.0);
    return 1.0 - Mc;
}
static void B0fun(double x, double y, double z, double* A, void* c) {
    B0ctx* b = (B0ctx*)c;
    if (b->type == 1) { A[0] = b->bx; A[1] = b->by; A[2] = b->bz; return; }
    if (b->type == 3) {   // cutDipole (apps/msphutils.F90:561-579): the dipole at the origin, ramped down
        double r = std::sqrt(sq(x) + sq(y) + sq(z));
        B0ctx d = *b;
        d.type = 2; d.bx = d.by = d.bz = 0.0;
        B0fun(x, y, z, A, &d);
        double yp = std::sqrt(sq(y) + sq(z));
        double phid = std::atan2(yp, x) * 180.0 / PI;
        double rScl = 1.0 + RampUpE(phid, 0.0, 180.0) * (b->dcScl - 1.0);
        double M = PenticRampDown(r, b->rCut * rScl, b->lCut * rScl);
        A[0] = M * A[0]; A[1] = M * A[1]; A[2] = M * A[2];
        return;
    }
    // Dipole (apps/msphutils.F90:534-551): 3 (m.r) r / rad**5 - m / rad**3
    double r[3] = {x - b->bx, y - b->by, z - b->bz};
    double rad = norm2v(r, 3);
    double m[3] = {0.0, 0.0, b->M0};
    double mr = dot(m, r, 3);
    for (int c = 0; c < 3; ++c) A[c] = 3 * mr * r[c] / std::pow(rad, 5.0) - m[c] / std::pow(rad, 3.0);
}
static void B0Wrap(double x, double y, double z, double* W, void* c) {
    double A[3];
    B0fun(x, y, z, A, c);
    W[0] = A[0]; W[1] = A[1]; W[2] = A[2]; W[3] = 0.0; W[4] = 0.0;
}
static void faceDeltas(const double* f0, const double* f1, const double* f2, const double* f3, double* dx, double* dy,
                       double* dz) {  // quadrature.F90:373-389
    dx[0] = f1[0] - f0[0]; dx[1] = f2[0] - f0[0]; dx[2] = f3[0] + f0[0] - f2[0] - f1[0];
    dy[0] = f1[1] - f0[1]; dy[1] = f2[1] - f0[1]; dy[2] = f3[1] + f0[1] - f2[1] - f1[1];
    dz[0] = f1[2] - f0[2]; dz[1] = f2[2] - f0[2]; dz[2] = f3[2] + f0[2] - f2[2] - f1[2];
}
// GaussianFaceFlux (quadrature.F90:105-151) and GaussianFaceStress (:223-280) of A over one face
static void GaussianFaceFluxStress(const double* f0, const double* f1, const double* f2, const double* f3, VecFun A,
                                   void* ctx, double* flx, double* Mbb) {
    double dx[3], dy[3], dz[3];
    faceDeltas(f0, f1, f2, f3, dx, dy, dz);
    *flx = 0.0;
    Mbb[0] = Mbb[1] = Mbb[2] = 0.0;
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            double eta = 0.5 * (1 + gA[i]), psi = 0.5 * (1 + gA[j]);
            double w = gWgt[i] * gWgt[j];
            double xp = f0[0] + dx[0] * eta + dx[1] * psi + dx[2] * eta * psi;
            double yp = f0[1] + dy[0] * eta + dy[1] * psi + dy[2] * eta * psi;
            double zp = f0[2] + dz[0] * eta + dz[1] * psi + dz[2] * eta * psi;
            double Ap[3];
            A(xp, yp, zp, Ap, ctx);
            double etaV[3] = {dx[0] + dx[2] * psi, dy[0] + dy[2] * psi, dz[0] + dz[2] * psi};
            double psiV[3] = {dx[1] + dx[2] * eta, dy[1] + dy[2] * eta, dz[1] + dz[2] * eta};
            double cr[3], N[3];
            cross3(etaV, psiV, cr);
            for (int c = 0; c < 3; ++c) N[c] = 0.25 * w * cr[c];
            *flx = *flx + dot(N, Ap, 3);
            double B0B0 = dot(Ap, Ap, 3), B0dS = dot(Ap, N, 3);
            for (int c = 0; c < 3; ++c) Mbb[c] = Mbb[c] + 0.5 * B0B0 * N[c] - Ap[c] * B0dS;
        }
}
static void AddB0(const Model& M, Grid& G, B0ctx* ctx) {
    (void)M;
    int lo[5] = {G.isg, G.jsg, G.ksg, 1, 1}, hi[5] = {G.ieg, G.jeg, G.keg, 3, 3};
    G.fcB0.alloc(5, lo, hi);
    hi[3] = 2;
    G.edgB0.alloc(5, lo, hi);
    hi[3] = 3;
    G.B0.alloc(4, lo, hi); G.bFlux0.alloc(4, lo, hi); G.dpB0.alloc(4, lo, hi);
    Arr faceStress;
    faceStress.alloc(5, lo, hi);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i) {
                for (int d = 1; d <= 3; ++d) {
                    double f0[3], f1[3], f2[3], f3[3], fI[3], flx, Mbb[3];
                    faceCoords(G, i, j, k, d, f0, f1, f2, f3);
                    GaussianFaceFluxStress(f0, f1, f2, f3, B0fun, ctx, &flx, Mbb);
                    G.bFlux0(i, j, k, d) = flx;
                    GaussianFaceIntegral(f0, f1, f2, f3, B0fun, ctx, fI);
                    for (int c = 0; c < 3; ++c) G.fcB0(i, j, k, c + 1, d) = fI[c] / G.face(i, j, k, d);
                    for (int c = 0; c < 3; ++c) faceStress(i, j, k, d, c + 1) = Mbb[c];
                }
                for (int d = 1; d <= 3; ++d) {   // edge integrals mapped with the edge velocity triad
                    double e1[3], e2[3], eInt[3];
                    for (int c = 0; c < 3; ++c) {
                        e1[c] = G.xyz(i, j, k, c + 1);
                        e2[c] = G.xyz(i + (d == IDIR), j + (d == JDIR), k + (d == KDIR), c + 1);
                    }
                    GaussianEdgeIntegral(e1, e2, B0fun, ctx, eInt);
                    G.edgB0(i, j, k, 1, d) = eInt[0] * G.Te(i, j, k, TAN1X, d) + eInt[1] * G.Te(i, j, k, TAN1Y, d) +
                                             eInt[2] * G.Te(i, j, k, TAN1Z, d);
                    G.edgB0(i, j, k, 2, d) = eInt[0] * G.Te(i, j, k, TAN2X, d) + eInt[1] * G.Te(i, j, k, TAN2Y, d) +
                                             eInt[2] * G.Te(i, j, k, TAN2Z, d);
                }
                double xyzC[8][3], w[5];
                cellCoords(G, i, j, k, xyzC);
                GaussianVolumeIntegral(xyzC, B0Wrap, ctx, w);
                for (int c = 0; c < 3; ++c) G.B0(i, j, k, c + 1) = w[c] / G.volume(i, j, k);
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i)
                for (int c = 1; c <= 3; ++c)
                    G.dpB0(i, j, k, c) = -(faceStress(i + 1, j, k, IDIR, c) - faceStress(i, j, k, IDIR, c) +
                                           faceStress(i, j + 1, k, JDIR, c) - faceStress(i, j, k, JDIR, c) +
                                           faceStress(i, j, k + 1, KDIR, c) - faceStress(i, j, k, KDIR, c)) /
                                         G.volume(i, j, k);
}

static void initBW(const Model& M, Grid& G, State& S, bool fieldAsBackground) {  // prob.F90:190-255, deck defaults
    BWctx b;
    b.x0 = b.y0 = b.z0 = 0.0; b.Vx0 = b.Vy0 = b.Vz0 = 0.0;
    double B0_BW = 1.0;
    b.P0 = 0.1; b.pRat = 100.0; b.dRat = 1.0; b.D0 = 1.0; b.rC = 0.1;
    b.bScl = B0_BW / (double)std::sqrt(2.0f);   // sqrt(2.0) is a default-real (single precision) literal
    b.bSclz = 0.0;
    GasIC2State(M, G, S, GasIC_BW, &b);
    if (M.doMHD && !fieldAsBackground) VectorPot2Flux(G, S, VectorPot_BW, &b);   // prob/doBack = F
}

// LFM-type spherical corners about the x axis: i -> r (geometric), j -> theta, k -> phi; ghost corners continue
// the same formulas (theta < 0 or > pi reflects through the axis) and repeat exactly with period Nkp in k
static void lfmCorner(const double* lfm, const Grid& G, int i, int j, int k, double* x, double* y, double* z) {
    double rin = lfm[0], rout = lfm[1], q = lfm[2], th0 = lfm[3];
    double r;
    if (q == 1.0) r = rin + (rout - rin) * (double)(i - G.is) / G.Nip;
    else {
        double dr0 = (rout - rin) * (q - 1.0) / (std::pow(q, (double)G.Nip) - 1.0);
        r = rin + dr0 * (std::pow(q, (double)(i - G.is)) - 1.0) / (q - 1.0);
    }
    double th = th0 + (double)(j - G.js) * (PI - 2.0 * th0) / G.Njp;
    int kk = ((k - G.ks) % G.Nkp + G.Nkp) % G.Nkp;   // exactly periodic in k
    double ph = (double)kk * 2.0 * PI / G.Nkp;
    *x = r * std::cos(th);
    *y = r * std::sin(th) * std::cos(ph);
    *z = r * std::sin(th) * std::sin(ph);
}
// initUser of the LFM blast wave (ICs/lfmbw.F90:33-104): pressure sphere of radius rC at (x0,y0,z0) with
// pRat*P0, Az = B0/sqrt(2.0) * (y - x) (sqrt of a default-real literal)
static void initLFMBW(const Model& M, const Grid& G, State& S, const double* bw) {
    BWctx b;
    b.x0 = bw[0]; b.y0 = bw[1]; b.z0 = bw[2];
    b.Vx0 = b.Vy0 = b.Vz0 = 0.0;
    b.P0 = bw[3]; b.pRat = bw[4]; b.dRat = 1.0; b.D0 = bw[5]; b.rC = bw[6];
    b.bScl = bw[7] / (double)std::sqrt(2.0f);
    b.bSclz = 0.0;
    GasIC2State(M, G, S, GasIC_BW, &b);
    if (M.doMHD) VectorPot2Flux(G, S, VectorPot_BW, &b);
}

// ---------------------------------------------------------------- the accuracy cases of tests/cases/testCases.pf
// Single-precision (default-real) literals of the Fortran keep their float values: a literal such as 0.1 is
// written (double)0.1f, and 0.1**2 is evaluated in float, as gfortran does.
static const double F01 = (double)0.1f, F03 = (double)0.3f, F05 = (double)0.5f, F07 = (double)0.7f,
                    F005 = (double)0.05f;

// cell-centre primitive state written as conserved Gas on the cells is..ie+1 (the loops of prob.F90)
static void putPrim(const Model& M, State& S, int i, int j, int k, double Rho, double Vx, double Vy, double Vz, double P) {
    S.Gas(i, j, k, DEN) = Rho;
    S.Gas(i, j, k, MOMX) = Rho * Vx;
    S.Gas(i, j, k, MOMY) = Rho * Vy;
    S.Gas(i, j, k, MOMZ) = Rho * Vz;
    double KinE = 0.5 * Rho * (sq(Vx) + sq(Vy) + sq(Vz));
    S.Gas(i, j, k, ENERGY) = KinE + P / (M.gamma - 1);
}

// initADV1D (prob.F90:671-736): four density shapes advected at Vx = 1 on [-1, 1], P = 1, no field
static void initADV1D(const Model& M, Grid& G, State& S) {
    const double f01sq = (double)(0.1f * 0.1f);   // 0.1**2 of two default reals
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double xc = G.xyzcc(i, j, k, 1);
                double Rho0 = F01;
                double Rho1 = std::exp(-sq((xc + F07) / F005));
                double Rho2 = (std::fabs(xc + F03) <= F01) ? 1.0 : 0.0;
                double Rho3 = (std::fabs(xc - F01) <= F01) ? 1.0 - std::fabs(10.0 * (xc - F01)) : 0.0;
                double Rho4 = ((f01sq - sq(xc - F05)) >= 0) ? 10.0 * std::sqrt(f01sq - sq(xc - F05)) : 0.0;
                double Rho = Rho0 + Rho1 + Rho2 + Rho3 + Rho4;
                putPrim(M, S, i, j, k, Rho, 1.0, 0.0, 0.0, 1.0);
                S.magFlux(i, j, k, IDIR) = 0.0; S.magFlux(i, j, k, JDIR) = 0.0; S.magFlux(i, j, k, KDIR) = 0.0;
            }
}

// initADV2D (prob.F90:739-797): a disc of radius R0 with twice the density, advected at V0 along alpha
// degrees from +y; prob = {d0, P0, V0, alpha, R0, x0, y0}
static void initADV2D(const Model& M, Grid& G, State& S, const double* pr) {
    double Rho0 = pr[0], P0 = pr[1], V0 = pr[2], alpha = pr[3], R0 = pr[4], x0 = pr[5], y0 = pr[6];
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double xc = G.xyzcc(i, j, k, 1), yc = G.xyzcc(i, j, k, 2);
                double Vx = V0 * std::sin(alpha * PI / 180.0), Vy = V0 * std::cos(alpha * PI / 180.0);
                double r = std::sqrt(sq(xc - x0) + sq(yc - y0));
                double Rho = (r < R0) ? Rho0 * 2.0 : Rho0;
                putPrim(M, S, i, j, k, Rho, Vx, Vy, 0.0, P0);
                S.magFlux(i, j, k, IDIR) = 0.0; S.magFlux(i, j, k, JDIR) = 0.0; S.magFlux(i, j, k, KDIR) = 0.0;
            }
}

// initLoop (prob.F90:436-500): uniform flow along alpha, a field loop from Az = max(0, A0 (R0 - r));
// prob = {d0, P0, V0, Vz0, alpha, A0, R0, x0, y0}
struct LoopCtx { double A0, R0, x0, y0; };
static void VectorPot_Loop2D(double x, double y, double z, double* A, void* c) {   // prob.F90:489-499
    (void)z;
    LoopCtx* l = (LoopCtx*)c;
    double r = std::sqrt(sq(x - l->x0) + sq(y - l->y0));
    A[0] = 0.0; A[1] = 0.0;
    A[2] = fmaxd(0.0, l->A0 * (l->R0 - r));
}
static void initLoop2D(const Model& M, Grid& G, State& S, const double* pr) {
    double Rho0 = pr[0], P0 = pr[1], V0 = pr[2], Vz0 = pr[3], alpha = pr[4];
    for (int k = G.ks; k <= G.ke + 1; ++k)
        for (int j = G.js; j <= G.je + 1; ++j)
            for (int i = G.is; i <= G.ie + 1; ++i) {
                double Vx = V0 * std::sin(alpha * PI / 180.0), Vy = V0 * std::cos(alpha * PI / 180.0);
                putPrim(M, S, i, j, k, Rho0, Vx, Vy, Vz0, P0);
            }
    LoopCtx l = {pr[5], pr[6], pr[7], pr[8]};
    VectorPot2Flux(G, S, VectorPot_Loop2D, &l);
}

// initALFVEN (prob.F90:1027-1083): the nonlinear circularly polarised Alfven wave along angle alp;
// prob = {d0, P0, B_para, V_para, alp}
struct AlfCtx { double Rho0, P0, Bpar, Vpar, alp; };
static void GasIC_ALF(double x, double y, double z, double* W, void* c) {   // prob.F90:1072-1082
    (void)z;
    AlfCtx* a = (AlfCtx*)c;
    double ph = 2 * PI * (x * std::cos(a->alp) + y * std::sin(a->alp));
    W[0] = a->Rho0;
    W[1] = a->Vpar * std::cos(a->alp) - F01 * std::sin(ph) * std::sin(a->alp);
    W[2] = a->Vpar * std::sin(a->alp) + F01 * std::sin(ph) * std::cos(a->alp);
    W[3] = F01 * std::cos(ph);
    W[4] = a->P0;
}
static void VectorPot_ALF(double x, double y, double z, double* A, void* c) {   // prob.F90:1063-1070
    AlfCtx* a = (AlfCtx*)c;
    double ph = 2 * PI * (x * std::cos(a->alp) + y * std::sin(a->alp));
    A[0] = a->Bpar * std::sin(a->alp) * z;
    A[1] = -1.0 * a->Bpar * std::cos(a->alp) * z + F01 * std::sin(ph) / (2 * PI * std::cos(a->alp));
    A[2] = F01 * std::cos(ph) / (2 * PI);
}
static void initALFVEN(const Model& M, Grid& G, State& S, const double* pr) {
    AlfCtx a = {pr[0], pr[1], pr[2], pr[3], pr[4]};
    GasIC2State(M, G, S, GasIC_ALF, &a);
    VectorPot2Flux(G, S, VectorPot_ALF, &a);
}

// ---------------------------------------------------------------- the magnetosphere problem's set-up
// (voltron/ICs/earthcmi.F90 initUser with apps/msphutils.F90 genCutDipole, background.F90 AddGrav)
struct VPInitCtx { double M0, x0, Aq, Bq, sInner; };
static void VP_Init(double x, double y, double z, double* A, void* c) {   // msphutils.F90:503-532
    VPInitCtx* v = (VPInitCtx*)c;
    double r[3] = {x, y, z}, nr = norm2v(r, 3), rhat[3] = {x / nr, y / nr, z / nr};
    double m[3] = {0.0, 0.0, 1.0}, cr[3];
    cross3(m, rhat, cr);
    double rr = dot(r, r, 3);
    for (int c2 = 0; c2 < 3; ++c2) A[c2] = v->M0 * cr[c2] / rr;   // VP_Dipole
    double s = std::sqrt(sq((x + v->x0) / v->Aq) + (sq(y) + sq(z)) / sq(v->Bq));
    double M = PenticRampDown(s, v->sInner, 1.0 - v->sInner);
    A[0] = M * A[0]; A[1] = M * A[1]; A[2] = M * A[2];
}
struct PhiCtx { double GM0; };
static double PhiGrav(double x, double y, double z, double GM0) {   // msphutils.F90:626-633
    double rad = std::sqrt(sq(x) + sq(y) + sq(z));
    return -GM0 / rad;
}
// AddGrav (background.F90:170-252) with the spherical gravity of the magnetosphere (doSphGrav)
static void AddGrav(const Model& M, Grid& G) {
    int lo[4] = {G.isg, G.jsg, G.ksg, 1}, hi[4] = {G.ieg, G.jeg, G.keg, 3};
    G.gxyz.alloc(4, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double dV = G.volume(i, j, k);
                const int fi[6] = {i, i, i, i + 1, i, i}, fj[6] = {j, j, j, j, j + 1, j}, fk[6] = {k, k, k, k, k, k + 1};
                const int fd[6] = {IDIR, JDIR, KDIR, IDIR, JDIR, KDIR};
                double Phi[6], da[6], n[6][3];
                for (int f = 0; f < 6; ++f) {
                    Phi[f] = PhiGrav(G.xfc(fi[f], fj[f], fk[f], 1, fd[f]), G.xfc(fi[f], fj[f], fk[f], 2, fd[f]),
                                     G.xfc(fi[f], fj[f], fk[f], 3, fd[f]), M.W.GM0);
                    da[f] = G.face(fi[f], fj[f], fk[f], fd[f]);
                    for (int c = 0; c < 3; ++c) n[f][c] = G.Tf(fi[f], fj[f], fk[f], NORMX + c, fd[f]);
                }
                // g = -(PhiIp daIp nIp - PhiI daI nI + PhiJp daJp nJp - PhiJ daJ nJ + PhiKp daKp nKp - PhiK daK nK)/dV
                double g[3], rhat[3], xc[3] = {G.xyzcc(i, j, k, 1), G.xyzcc(i, j, k, 2), G.xyzcc(i, j, k, 3)};
                for (int c = 0; c < 3; ++c)
                    g[c] = -(Phi[3] * da[3] * n[3][c] - Phi[0] * da[0] * n[0][c] + Phi[4] * da[4] * n[4][c] -
                             Phi[1] * da[1] * n[1][c] + Phi[5] * da[5] * n[5][c] - Phi[2] * da[2] * n[2][c]) / dV;
                normVec3(xc, rhat);
                double gp[3];
                Vec2Para(g, rhat, gp);
                for (int c = 0; c < 3; ++c) G.gxyz(i, j, k, c + 1) = gp[c];
            }
}
struct GasConstCtx { double D, P; };
static void GasIC_Const(double, double, double, double* W, void* c) {   // earthcmi.F90:183-200 GasIC
    GasConstCtx* g = (GasConstCtx*)c;
    W[0] = g->D; W[1] = 0.0; W[2] = 0.0; W[3] = 0.0; W[4] = g->P;
}
// initUser's field and gas (earthcmi.F90:86-132): the cut dipole as background (genCutDipole, msphutils.F90:
// 419-498: AddB0, dpB0 zeroed inside rCut, the initial residual field = flux of the elliptically cut dipole's
// vector potential minus the background's face flux), uniform gas at rest, gravity
static void initMagsphere(Model& M, Grid& G, State& S, double Rho0, double P0) {
    B0ctx bc;
    bc.type = 3; bc.bx = bc.by = bc.bz = 0.0; bc.M0 = M.W.M0;
    bc.rCut = M.W.rCut; bc.lCut = M.W.lCut; bc.dcScl = M.W.dcScl;
    M.doBackground = true;
    AddB0(M, G, &bc);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double xyzC[8][3], rMin = 0.0;
                cellCoords(G, i, j, k, xyzC);
                for (int p = 0; p < 8; ++p) {
                    double r = norm2v(xyzC[p], 3);
                    rMin = (p == 0 || r < rMin) ? r : rMin;
                }
                if (rMin + TINY < M.W.rCut)
                    for (int c = 1; c <= 3; ++c) G.dpB0(i, j, k, c) = 0.0;
            }
    // VectorField2Flux (gridutils.F90:240-278) of the cut dipole: the background's face fluxes, cells isg..ieg
    Arr bF0 = S.magFlux;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = G.ksg; k <= G.keg; ++k)
        for (int j = G.jsg; j <= G.jeg; ++j)
            for (int i = G.isg; i <= G.ieg; ++i)
                for (int d = 1; d <= 3; ++d) {
                    double f0[3], f1[3], f2[3], f3[3], flx, Mbb[3];
                    faceCoords(G, i, j, k, d, f0, f1, f2, f3);
                    GaussianFaceFluxStress(f0, f1, f2, f3, B0fun, &bc, &flx, Mbb);
                    S.magFlux(i, j, k, d) = flx;
                }
    bF0.d = S.magFlux.d;
    VPInitCtx v;
    v.M0 = M.W.M0; v.Aq = 0.5 * (M.W.xSun - M.W.xTail); v.x0 = v.Aq - M.W.xSun; v.Bq = M.W.yMax;
    v.sInner = M.W.sInner;
    VectorPot2Flux(G, S, VP_Init, &v);
    for (size_t q = 0; q < S.magFlux.d.size(); ++q) S.magFlux.d[q] = S.magFlux.d[q] - bF0.d[q];
    GasConstCtx gc = {Rho0, P0};
    GasIC2State(M, G, S, GasIC_Const, &gc);
    M.doGrav = true;
    M.doSphGrav = true;
    AddGrav(M, G);
}

}  // namespace orc

// =========================================================================================== C ABI
using namespace orc;

extern "C" {

struct orc_params {
    int Nip, Njp, Nkp;
    int icType;            // 0 = OT2D, 1 = BW, 2 = LFM blast wave, 3 = KH, 4..7 = ADV1D, ADV2D, LOOP2D, ALFVEN
    int gridType;          // 0 = uniform Cartesian, 1 = sinusoidal warp x'=x+A sin(2 pi y) sin(2 pi z) (cyclic)
    double xyzBds[6];
    double warpAmp;
    double CFL, gamma, pdmb, Vd0, cHogH, cHogM, Ca, tFin;
    int doMHD, doBoris, rmeth, doLFMLim;
    int bc[6];             // 0 periodic, 1 zeroGrad
    int nThreads;
    int b0Type;            // 0 none, 1 uniform (b0[0..2]), 2 dipole (moment b0[3] along z, centre b0[0..2])
    double b0[4];
    // gridType 2: LFM-type spherical grid about the x axis, lfm = {r_in, r_out, radial stretch ratio, theta0}:
    // r geometric from r_in to r_out over Nip cells, theta uniform on [theta0, pi - theta0], phi uniform on [0, 2 pi)
    double lfm[4];
    double dFloor, pFloor;  // sim/dFloor, sim/pFloor (0: the TINY defaults)
    int doRing;             // ring averaging about the LFM axis (ring/doRing, gid = lfm)
    int ringNumR;           // ring/Nr (0: the default table for Nkp)
    int ringNch[32];        // ring/Nc1.. (0: default)
    int ringRecon;          // ring/rngrec: 0 PLM, 1 PPM (default), 2 PCM
    int dtActive;           // 1: the timestep domain is the active cells only (problem DT bounds)
    // icType 2: the LFM blast wave (ICs/lfmbw.F90), bw = {x0, y0, z0, P0, pRat, D0, rC, B0}; its INI/OUTI shells
    // are bc 3 and its predictor fix is on
    double bw[8];
    double kh[4];           // icType 3: Kelvin-Helmholtz shear layer {a, Bx, amp, seed}
    // icType 4 ADV1D, 5 ADV2D {d0, P0, V0, alpha, R0, x0, y0}, 6 LOOP2D {d0, P0, V0, Vz0, alpha, A0, R0, x0, y0},
    // 7 ALFVEN {d0, P0, B_para, V_para, alp}: the deck values of tests/cases/*.xml with prob.F90's defaults
    double prob[10];
    // 1: no set-up -- allocate the grid, State and Solver only; the caller sets the metrics, State, oState and
    // the scalars (orc_set, orc_set_scalars) before stepping. Used to step a slab of a grid built elsewhere.
    int noSetup;
    // icType 8, the magnetosphere (voltron/ICs/earthcmi.F90 initUser) with a constant solar wind, in code units:
    // {M0, GM0, rCut, lCut, dcScl, xSun, xTail, yMax, sInner, windD, windP, windVx, windVy, windVz, windBx,
    //  windBy, windBz, dtCpl, gT0, Rho0, P0, nIonP, doIonPush}; bc {BC_ION, BC_WIND, lfm, lfm, periodic x2}
    double msph[24];
    const double* xyzIn;    // corners (Ni+1,Nj+1,Nk+1,3), Fortran layout, replacing the generated ones (a tile)
};

void* orc_create(const orc_params* p) {
    initWeights();
    App* A = new App();
    Model& M = A->M;
    Grid& G = A->G;
    M.CFL = p->CFL; M.gamma = p->gamma; M.pdmb = p->pdmb; pdmb_g = p->pdmb;
    M.Vd0 = p->Vd0; M.cHogH = p->cHogH; M.cHogM = p->cHogM; M.Ca = p->Ca; M.tFin = p->tFin;
    M.doMHD = p->doMHD != 0; M.doBoris = p->doBoris != 0; M.rmeth = p->rmeth; M.doLFMLim = p->doLFMLim != 0;
#ifdef _OPENMP
    if (p->nThreads > 0) omp_set_num_threads(p->nThreads);
#endif
    G.Nip = p->Nip; G.Njp = p->Njp; G.Nkp = p->Nkp;
    M.do25D = (G.Nkp == 1);
    if (p->dFloor > 0) M.dFloor = p->dFloor;
    if (p->pFloor > 0) M.pFloor = p->pFloor;
    for (int n = 0; n < 6; ++n) G.bc[n] = p->bc[n];
    allocGrid(M, G);
    if (p->doRing) {   // SetRings before Corners2Grid (init.F90:164-165)
        M.doRing = true;
        M.R.recon = p->ringRecon == 0 ? RR_PLM : (p->ringRecon == 2 ? RR_PCM : RR_PPM);
        if (InitRingsLFM(M, G, p->ringNumR, p->ringNch) != 0) { delete A; return nullptr; }
    }
    // genGridXML (init.F90:572-798): uniform corners, then the optional warp
    double dx = (p->xyzBds[1] - p->xyzBds[0]) / G.Nip, dy = (p->xyzBds[3] - p->xyzBds[2]) / G.Njp,
           dz = (p->xyzBds[5] - p->xyzBds[4]) / G.Nkp;
    for (int k = G.ksg; k <= G.keg + 1; ++k)
        for (int j = G.jsg; j <= G.jeg + 1; ++j)
            for (int i = G.isg; i <= G.ieg + 1; ++i) {
                double x = p->xyzBds[0] + (i - 1) * dx, y = p->xyzBds[2] + (j - 1) * dy, z = p->xyzBds[4] + (k - 1) * dz;
                if (p->gridType == 1) {
                    double a = p->warpAmp;
                    double xw = x + a * std::sin(2 * PI * y) * std::sin(2 * PI * z);
                    double yw = y + a * std::sin(2 * PI * z) * std::sin(2 * PI * x);
                    double zw = z + a * std::sin(2 * PI * x) * std::sin(2 * PI * y);
                    x = xw; y = yw; z = zw;
                } else if (p->gridType == 2) {
                    lfmCorner(p->lfm, G, i, j, k, &x, &y, &z);
                }
                G.xyz(i, j, k, 1) = x; G.xyz(i, j, k, 2) = y; G.xyz(i, j, k, 3) = z;
                if (p->xyzIn) {
                    long nc = (long)(G.Ni + 1) * (G.Nj + 1) * (G.Nk + 1);
                    long q = (long)(i - G.isg) + (long)(G.Ni + 1) * ((j - G.jsg) + (long)(G.Nj + 1) * (k - G.ksg));
                    for (int c = 0; c < 3; ++c) G.xyz(i, j, k, c + 1) = p->xyzIn[q + c * nc];
                }
            }
    SetDomain(G);
    if (p->dtActive) { G.isDT = G.is; G.ieDT = G.ie; G.jsDT = G.js; G.jeDT = G.je; G.ksDT = G.ks; G.keDT = G.ke; }
    // tile faces: the dt domain stops at the active cells (SetDomain adds a ghost layer only at physical BCs)
    if (G.bc[0] == BC_HALO) G.isDT = G.is;
    if (G.bc[1] == BC_HALO) G.ieDT = G.ie;
    if (G.bc[2] == BC_HALO) G.jsDT = G.js;
    if (G.bc[3] == BC_HALO) G.jeDT = G.je;
    if (G.bc[4] == BC_HALO) G.ksDT = G.ks;
    if (G.bc[5] == BC_HALO) G.keDT = G.ke;
    if (p->noSetup) {
        if (p->doRing || p->b0Type != 0) { delete A; return nullptr; }
        allocGridMetrics(G);
        allocState(M, G, A->S);
        allocState(M, G, A->oS);
    } else {
        if (Corners2Grid(M, G) != 0) { delete A; return nullptr; }
        allocState(M, G, A->S);
        allocState(M, G, A->oS);
        if (p->icType == 0) initOT2D(M, G, A->S);
        else if (p->icType == 3) initKH(M, G, A->S, p->kh);
        else if (p->icType == 4) initADV1D(M, G, A->S);
        else if (p->icType == 5) initADV2D(M, G, A->S, p->prob);
        else if (p->icType == 6) initLoop2D(M, G, A->S, p->prob);
        else if (p->icType == 7) initALFVEN(M, G, A->S, p->prob);
        else if (p->icType == 8) {
            const double* w = p->msph;
            Model::Msph& W = M.W;
            W.on = true;
            W.M0 = w[0]; W.GM0 = w[1]; W.rCut = w[2]; W.lCut = w[3]; W.dcScl = w[4];
            W.xSun = w[5]; W.xTail = w[6]; W.yMax = w[7]; W.sInner = w[8];
            W.wD = w[9]; W.wP = w[10];
            for (int c = 0; c < 3; ++c) { W.wV[c] = w[11 + c]; W.wB[c] = w[14 + c]; }
            W.dtCpl = w[17]; W.gT0 = w[18]; W.nIonP = (int)w[21]; W.doIonPush = w[22] != 0.0;
            initMagsphere(M, G, A->S, w[19], w[20]);
        }
        else if (p->icType == 2) {
            M.predFixLFM = true;
            M.bwD0 = p->bw[5]; M.bwP0 = p->bw[3];
            initLFMBW(M, G, A->S, p->bw);
        }
        else initBW(M, G, A->S, p->b0Type == 1);
        if (p->b0Type != 0 && p->icType != 8) {   // CalcGridInfo: AddB0 after the IC (init.F90:180-184)
            M.doBackground = true;
            B0ctx bc;
            bc.type = p->b0Type; bc.bx = p->b0[0]; bc.by = p->b0[1]; bc.bz = p->b0[2]; bc.M0 = p->b0[3];
            AddB0(M, G, &bc);
        }
        // CalcGridInfo (init.F90:204-244)
        if (M.doMHD) bFlux2Fld(M, G, A->S.magFlux, A->S.Bxyz);
        EnforceBCs(M, G, A->S);
        A->oS.Gas.d = A->S.Gas.d; A->oS.magFlux.d = A->S.magFlux.d; A->oS.Bxyz.d = A->S.Bxyz.d;
        A->oS.time = A->S.time;
        M.dt = CalcDT(M, G, A->S);
        A->oS.time = A->S.time - M.dt;
    }
    // initSolver (init.F90:494-516)
    Solver& V = A->V;
    int lo[6] = {G.isg, G.jsg, G.ksg, 1, 1, 0};
    int hi[6] = {G.ieg, G.jeg, G.keg, 5, 3, 0};
    V.gFlx.alloc(5, lo, hi);
    hi[3] = 3;
    V.mFlx.alloc(5, lo, hi);
    V.Vf.alloc(4, lo, hi);
    V.dGasM.alloc(4, lo, hi);
    hi[3] = 5;
    V.dGasH.alloc(4, lo, hi);
    if (M.doRing) { hi[3] = 3; V.SmoothE.alloc(4, lo, hi); }
    allocState(M, G, V.StateHf);
    return A;
}

void orc_destroy(void* h) { delete (App*)h; }

void orc_step(void* h) { stepGamera(*(App*)h); }

void orc_get_scalars(void* h, double* out) {  // t, dt, dt0, S.time, oS.time, ts, status
    App* A = (App*)h;
    out[0] = A->M.t; out[1] = A->M.dt; out[2] = A->M.dt0; out[3] = A->S.time; out[4] = A->oS.time;
    out[5] = (double)A->M.ts; out[6] = (double)A->M.status;
}
void orc_set_scalars(void* h, const double* in) {
    App* A = (App*)h;
    A->M.t = in[0]; A->M.dt = in[1]; A->M.dt0 = in[2]; A->S.time = in[3]; A->oS.time = in[4]; A->M.ts = (int)in[5];
}

static Arr* lookup(App* A, const char* name) {
    struct { const char* n; Arr* a; } tab[] = {
        {"gas", &A->S.Gas}, {"magflux", &A->S.magFlux}, {"bxyz", &A->S.Bxyz}, {"efld", &A->S.Efld},
        {"ogas", &A->oS.Gas}, {"omagflux", &A->oS.magFlux}, {"obxyz", &A->oS.Bxyz},
        {"hgas", &A->V.StateHf.Gas}, {"hmagflux", &A->V.StateHf.magFlux}, {"hbxyz", &A->V.StateHf.Bxyz},
        {"gflx", &A->V.gFlx}, {"mflx", &A->V.mFlx}, {"vf", &A->V.Vf}, {"dgash", &A->V.dGasH}, {"dgasm", &A->V.dGasM},
        {"xyz", &A->G.xyz}, {"xyzcc", &A->G.xyzcc}, {"xfc", &A->G.xfc}, {"di", &A->G.di}, {"dj", &A->G.dj},
        {"dk", &A->G.dk}, {"volume", &A->G.volume}, {"tf", &A->G.Tf}, {"te", &A->G.Te}, {"teb", &A->G.Teb},
        {"face", &A->G.face}, {"edge", &A->G.edge},
        {"fcb0", &A->G.fcB0}, {"edgb0", &A->G.edgB0}, {"b0", &A->G.B0}, {"bflux0", &A->G.bFlux0}, {"dpb0", &A->G.dpB0},
        {"smoothe", &A->V.SmoothE},
    };
    for (auto& t : tab) if (std::strcmp(t.n, name) == 0) return t.a;
    return nullptr;
}
long orc_size(void* h, const char* name) { Arr* a = lookup((App*)h, name); return a ? a->size() : -1; }
int orc_get(void* h, const char* name, double* out) {
    Arr* a = lookup((App*)h, name);
    if (!a) return -1;
    std::memcpy(out, a->d.data(), sizeof(double) * a->size());
    return 0;
}
int orc_set(void* h, const char* name, const double* in) {
    Arr* a = lookup((App*)h, name);
    if (!a) return -1;
    std::memcpy(a->d.data(), in, sizeof(double) * a->size());
    return 0;
}
// Recompute State%Bxyz from State%magFlux (bFlux2Fld) after a host-side edit.
void orc_bflux2fld(void* h) {
    App* A = (App*)h;
    bFlux2Fld(A->M, A->G, A->S.magFlux, A->S.Bxyz);
    bFlux2Fld(A->M, A->G, A->oS.magFlux, A->oS.Bxyz);
}

double orc_divb(void* h) {  // gridutils.F90:717-770
    App* A = (App*)h;
    const Grid& G = A->G;
    const Arr& mf = A->S.magFlux;
    double tot = 0.0;
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double dFi = mf(i, j, k, IDIR) - mf(i + 1, j, k, IDIR);
                double dFj = mf(i, j, k, JDIR) - mf(i, j + 1, k, JDIR);
                double dFk = mf(i, j, k, KDIR) - mf(i, j, k + 1, KDIR);
                double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
                if (A->M.doBackground) {
                    dFi0 = G.bFlux0(i, j, k, IDIR) - G.bFlux0(i + 1, j, k, IDIR);
                    dFj0 = G.bFlux0(i, j, k, JDIR) - G.bFlux0(i, j + 1, k, JDIR);
                    dFk0 = G.bFlux0(i, j, k, KDIR) - G.bFlux0(i, j, k + 1, KDIR);
                }
                tot = tot + std::fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
            }
    return tot;
}

// ---------------------------------------------------------------- slice output (gioH5.F90:255-602)
// The variables writeSlc computes from State (active cells, no ghosts, single fluid, not a magnetosphere):
// D, Vx, Vy, Vz, P, Cs, Bx, By, Bz, Pb, Jx, Jy, Jz and, with fat output, Ex, Ey, Ez, DivB (and DivdB with a
// background field). Each variable is one (is:ie, js:je, ks:ke) Fortran block of out, in that order.
static void ijkVecC(const Grid& G, int i, int j, int k, int d, double* v) {   // metric.F90:172-201
    double p[3], m[3];
    for (int c = 1; c <= 3; ++c) {
        if (d == IDIR) {
            p[c - 1] = 0.25 * (G.xyz(i + 1, j, k, c) + G.xyz(i + 1, j + 1, k, c) + G.xyz(i + 1, j, k + 1, c) + G.xyz(i + 1, j + 1, k + 1, c));
            m[c - 1] = 0.25 * (G.xyz(i, j, k, c) + G.xyz(i, j + 1, k, c) + G.xyz(i, j, k + 1, c) + G.xyz(i, j + 1, k + 1, c));
        } else if (d == JDIR) {
            p[c - 1] = 0.25 * (G.xyz(i, j + 1, k, c) + G.xyz(i + 1, j + 1, k, c) + G.xyz(i, j + 1, k + 1, c) + G.xyz(i + 1, j + 1, k + 1, c));
            m[c - 1] = 0.25 * (G.xyz(i, j, k, c) + G.xyz(i + 1, j, k, c) + G.xyz(i, j, k + 1, c) + G.xyz(i + 1, j, k + 1, c));
        } else {
            p[c - 1] = 0.25 * (G.xyz(i, j, k + 1, c) + G.xyz(i + 1, j, k + 1, c) + G.xyz(i, j + 1, k + 1, c) + G.xyz(i + 1, j + 1, k + 1, c));
            m[c - 1] = 0.25 * (G.xyz(i, j, k, c) + G.xyz(i + 1, j, k, c) + G.xyz(i, j + 1, k, c) + G.xyz(i + 1, j + 1, k, c));
        }
    }
    for (int c = 0; c < 3; ++c) v[c] = p[c] - m[c];
    double n = norm2v(v, 3);
    for (int c = 0; c < 3; ++c) v[c] = v[c] / n;
}
// CellExyz (gridutils.F90:559-609) from edge fields (EMF / edge length)
static void cellExyz(const Grid& G, const Arr& Ef, int i, int j, int k, double* E) {
    auto ef = [&](int a, int b, int c, int d) {
        double e = G.edge(a, b, c, d);
        return e == 0.0 ? 0.0 : Ef(a, b, c, d) / e;
    };
    double cc[3];
    cc[0] = 0.25 * (ef(i, j, k, IDIR) + ef(i, j, k + 1, IDIR) + ef(i, j + 1, k, IDIR) + ef(i, j + 1, k + 1, IDIR));
    cc[1] = 0.25 * (ef(i, j, k, JDIR) + ef(i, j, k + 1, JDIR) + ef(i + 1, j, k, JDIR) + ef(i + 1, j, k + 1, JDIR));
    cc[2] = 0.25 * (ef(i, j, k, KDIR) + ef(i + 1, j, k, KDIR) + ef(i, j + 1, k, KDIR) + ef(i + 1, j + 1, k, KDIR));
    double iV[3], jV[3], kV[3], M[3][3];
    ijkVecC(G, i, j, k, IDIR, iV); ijkVecC(G, i, j, k, JDIR, jV); ijkVecC(G, i, j, k, KDIR, kV);
    M[0][0] = kV[2] * jV[1] - kV[1] * jV[2]; M[1][0] = kV[0] * jV[2] - kV[2] * jV[0]; M[2][0] = kV[1] * jV[0] - kV[0] * jV[1];
    M[0][1] = kV[1] * iV[2] - kV[2] * iV[1]; M[1][1] = kV[2] * iV[0] - kV[0] * iV[2]; M[2][1] = kV[0] * iV[1] - kV[1] * iV[0];
    M[0][2] = jV[2] * iV[1] - jV[1] * iV[2]; M[1][2] = jV[0] * iV[2] - jV[2] * iV[0]; M[2][2] = jV[1] * iV[0] - jV[0] * iV[1];
    double det = iV[0] * M[0][0] + jV[0] * M[0][1] + kV[0] * M[0][2];
    for (int r = 0; r < 3; ++r) E[r] = (M[r][0] * cc[0] + M[r][1] * cc[1] + M[r][2] * cc[2]) / det;
}
// bFld2Jxyz (gridutils.F90:314-478): B.dl on the edges, circulation per face, then the cell field of the
// face "fluxes" J.dS; on an LFM grid the two rings next to the axis are re-interpolated toward the pole
static void bFld2Jxyz(const Model& M, const Grid& G, const Arr& B, Arr& J) {
    int lo[4] = {G.isg, G.jsg, G.ksg, 1}, hiC[4] = {G.ieg, G.jeg, G.keg, 3}, hiF[4] = {G.ieg + 1, G.jeg + 1, G.keg + 1, 3};
    Arr bInt, JdS;
    bInt.alloc(4, lo, hiC);
    JdS.alloc(4, lo, hiF);
    std::fill(J.d.begin(), J.d.end(), 0.0);
    auto goodE = [&](int i, int j, int k, int d) {
        if (d == IDIR) return i >= G.isg && i <= G.ieg && j >= G.jsg && j <= G.jeg + 1 && k >= G.ksg && k <= G.keg + 1;
        if (d == JDIR) return i >= G.isg && i <= G.ieg + 1 && j >= G.jsg && j <= G.jeg && k >= G.ksg && k <= G.keg + 1;
        return i >= G.isg && i <= G.ieg + 1 && j >= G.jsg && j <= G.jeg + 1 && k >= G.ksg && k <= G.keg;
    };
    auto goodF = [&](int i, int j, int k, int d) {
        if (d == IDIR) return i >= G.isg && i <= G.ieg + 1 && j >= G.jsg && j <= G.jeg && k >= G.ksg && k <= G.keg;
        if (d == JDIR) return i >= G.isg && i <= G.ieg && j >= G.jsg && j <= G.jeg + 1 && k >= G.ksg && k <= G.keg;
        return i >= G.isg && i <= G.ieg && j >= G.jsg && j <= G.jeg && k >= G.ksg && k <= G.keg + 1;
    };
    for (int k = G.ksg + 1; k <= G.keg; ++k)
        for (int j = G.jsg + 1; j <= G.jeg; ++j)
            for (int i = G.isg + 1; i <= G.ieg; ++i) {
                double bA[3], dx[3];
                if (goodE(i + 1, j, k, IDIR)) {
                    for (int c = 1; c <= 3; ++c) {
                        bA[c - 1] = 0.25 * (B(i, j, k, c) + B(i, j - 1, k, c) + B(i, j, k - 1, c) + B(i, j - 1, k - 1, c));
                        dx[c - 1] = G.xyz(i + 1, j, k, c) - G.xyz(i, j, k, c);
                    }
                    bInt(i, j, k, IDIR) = dot3(bA, dx);
                }
                if (goodE(i, j + 1, k, JDIR)) {
                    for (int c = 1; c <= 3; ++c) {
                        bA[c - 1] = 0.25 * (B(i, j, k, c) + B(i, j, k - 1, c) + B(i - 1, j, k, c) + B(i - 1, j, k - 1, c));
                        dx[c - 1] = G.xyz(i, j + 1, k, c) - G.xyz(i, j, k, c);
                    }
                    bInt(i, j, k, JDIR) = dot3(bA, dx);
                }
                if (goodE(i, j, k + 1, KDIR)) {
                    for (int c = 1; c <= 3; ++c) {
                        bA[c - 1] = 0.25 * (B(i, j, k, c) + B(i - 1, j, k, c) + B(i, j - 1, k, c) + B(i - 1, j - 1, k, c));
                        dx[c - 1] = G.xyz(i, j, k + 1, c) - G.xyz(i, j, k, c);
                    }
                    bInt(i, j, k, KDIR) = dot3(bA, dx);
                }
            }
    for (int k = G.ksg + 1; k <= G.keg; ++k)
        for (int j = G.jsg + 1; j <= G.jeg; ++j)
            for (int i = G.isg + 1; i <= G.ieg; ++i) {
                if (goodF(i, j + 1, k + 1, IDIR))
                    JdS(i, j, k, IDIR) = bInt(i, j, k, JDIR) + bInt(i, j + 1, k, KDIR) - bInt(i, j, k + 1, JDIR) - bInt(i, j, k, KDIR);
                if (goodF(i + 1, j, k + 1, JDIR))
                    JdS(i, j, k, JDIR) = bInt(i, j, k, KDIR) + bInt(i, j, k + 1, IDIR) - bInt(i + 1, j, k, KDIR) - bInt(i, j, k, IDIR);
                if (goodF(i + 1, j + 1, k, KDIR))
                    JdS(i, j, k, KDIR) = bInt(i, j, k, IDIR) + bInt(i + 1, j, k, JDIR) - bInt(i, j + 1, k, IDIR) - bInt(i, j, k, JDIR);
            }
    for (int k = G.ksg + 1; k <= G.keg - 1; ++k)
        for (int j = G.jsg + 1; j <= G.jeg - 1; ++j)
            for (int i = G.isg + 1; i <= G.ieg - 1; ++i) {
                double b[3];
                gamCellBxyz(G, JdS, i, j, k, b);
                for (int c = 0; c < 3; ++c) J(i, j, k, c + 1) = 1.0 * b[c];
            }
    if (M.doRing) {   // gridutils.F90:414-470, active rings only (the ghost copies do not reach the output)
        const int Nk = G.ke - G.ks + 1;
        const double a8 = (double)0.8f, a2 = (double)0.2f, a4 = (double)0.4f, a6 = (double)0.6f;
        for (int i = G.isg + 1; i <= G.ieg - 1; ++i)
            for (int side = 0; side < 2; ++side) {
                if ((side == 0 && !M.R.doS) || (side == 1 && !M.R.doE)) continue;
                int j3 = side == 0 ? G.js + 2 : G.je - 2, j1 = side == 0 ? G.js : G.je, j2 = side == 0 ? G.js + 1 : G.je - 1;
                double J0[3] = {0.0, 0.0, 0.0};
                for (int k = G.ks; k <= G.ke; ++k)
                    for (int c = 0; c < 3; ++c) J0[c] = J0[c] + J(i, j3, k, c + 1);
                for (int c = 0; c < 3; ++c) J0[c] = J0[c] / Nk;
                for (int k = G.ks; k <= G.ke; ++k)
                    for (int c = 0; c < 3; ++c) {
                        double J3 = J(i, j3, k, c + 1);
                        J(i, j1, k, c + 1) = a8 * J0[c] + a2 * J3;
                        J(i, j2, k, c + 1) = a4 * J0[c] + a6 * J3;
                    }
            }
    }
}

static long sliceCount(const App& A, int fat) {
    long nv = 13 + (fat ? 4 + (A.M.doBackground ? 1 : 0) : 0);
    return nv * (long)A.G.Nip * A.G.Njp * A.G.Nkp;
}

// writeSlc's variables of the current State (see sliceCount for the layout); returns the doubles written
long orc_slice(void* h, int fat, double* out) {
    App* A = (App*)h;
    const Model& M = A->M;
    const Grid& G = A->G;
    const State& S = A->S;
    const long Na = (long)G.Nip * G.Njp * G.Nkp;
    auto o = [&](int v, int i, int j, int k) -> double& {
        return out[v * Na + (i - G.is) + (long)G.Nip * ((j - G.js) + (long)G.Njp * (k - G.ks))];
    };
    int lo[4] = {G.isg, G.jsg, G.ksg, 1}, hi[4] = {G.ieg, G.jeg, G.keg, 3};
    Arr J;
    J.alloc(4, lo, hi);
    if (M.doMHD) bFld2Jxyz(M, G, S.Bxyz, J);
    for (int k = G.ks; k <= G.ke; ++k)
        for (int j = G.js; j <= G.je; ++j)
            for (int i = G.is; i <= G.ie; ++i) {
                double D = S.Gas(i, j, k, DEN), Mx = S.Gas(i, j, k, MOMX), My = S.Gas(i, j, k, MOMY), Mz = S.Gas(i, j, k, MOMZ);
                double En = S.Gas(i, j, k, ENERGY);
                o(0, i, j, k) = D < 0.0 ? 0.0 : D;   // vacuum mask with the bulk floor 0
                double V[3] = {0.0, 0.0, 0.0}, P = 0.0;
                if (D > TINY) {
                    V[0] = Mx / D; V[1] = My / D; V[2] = Mz / D;
                    P = (M.gamma - 1) * (En - 0.5 * (Mx * Mx + My * My + Mz * Mz) / D);
                }
                o(1, i, j, k) = V[0]; o(2, i, j, k) = V[1]; o(3, i, j, k) = V[2]; o(4, i, j, k) = P;
                {   // CellPress2Cs (gamutils.F90:324-341)
                    double rho = fmaxd(D, M.dFloor);
                    double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
                    double KinE = 0.5 * rho * (sq(vx) + sq(vy) + sq(vz));
                    double Pc = fmaxd((M.gamma - 1) * (En - KinE), M.pFloor);
                    o(5, i, j, k) = std::sqrt(M.gamma * Pc / rho);
                }
                double B[3] = {0.0, 0.0, 0.0};
                if (M.doMHD)
                    for (int c = 0; c < 3; ++c) B[c] = S.Bxyz(i, j, k, c + 1) + (M.doBackground ? G.B0(i, j, k, c + 1) : 0.0);
                for (int c = 0; c < 3; ++c) o(6 + c, i, j, k) = B[c];
                o(9, i, j, k) = 0.5 * (sq(B[0]) + sq(B[1]) + sq(B[2]));
                for (int c = 0; c < 3; ++c) o(10 + c, i, j, k) = M.doMHD ? J(i, j, k, c + 1) : 0.0;
                if (!fat) continue;
                double E[3] = {0.0, 0.0, 0.0};
                if (M.doMHD) cellExyz(G, S.Efld, i, j, k, E);
                for (int c = 0; c < 3; ++c) o(13 + c, i, j, k) = E[c];
                const Arr& mf = S.magFlux;
                double dF = mf(i, j, k, IDIR) - mf(i + 1, j, k, IDIR) + mf(i, j, k, JDIR) - mf(i, j + 1, k, JDIR) +
                            mf(i, j, k, KDIR) - mf(i, j, k + 1, KDIR);
                double dFi = mf(i, j, k, IDIR) - mf(i + 1, j, k, IDIR), dFj = mf(i, j, k, JDIR) - mf(i, j + 1, k, JDIR),
                       dFk = mf(i, j, k, KDIR) - mf(i, j, k + 1, KDIR);
                (void)dF;
                double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
                if (M.doBackground) {
                    dFi0 = G.bFlux0(i, j, k, IDIR) - G.bFlux0(i + 1, j, k, IDIR);
                    dFj0 = G.bFlux0(i, j, k, JDIR) - G.bFlux0(i, j + 1, k, JDIR);
                    dFk0 = G.bFlux0(i, j, k, KDIR) - G.bFlux0(i, j, k + 1, KDIR);
                }
                o(16, i, j, k) = std::fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
                if (M.doBackground) o(17, i, j, k) = std::fabs(dFi + dFj + dFk + 0.0 + 0.0 + 0.0);
            }
    if (fat && M.doRing) {   // FixRAVec (gioH5.F90:577-601, metric.F90:227-300) on E
        const int Nk = G.ke - G.ks + 1;
        const double w1 = (double)(2.0f / 3.0f), w2 = (double)(1.0f / 3.0f);
        for (int i = G.is; i <= G.ie; ++i)
            for (int side = 0; side < 2; ++side) {
                if ((side == 0 && !M.R.doS) || (side == 1 && !M.R.doE)) continue;
                int jin = side == 0 ? G.js : G.je, jout = side == 0 ? G.js + 1 : G.je - 1;
                for (int c = 0; c < 3; ++c) {
                    double Q0 = 0.0;
                    for (int k = G.ks; k <= G.ke; ++k) Q0 = Q0 + o(13 + c, i, jout, k);
                    Q0 = Q0 / Nk;
                    for (int k = G.ks; k <= G.ke; ++k) o(13 + c, i, jin, k) = w1 * Q0 + w2 * o(13 + c, i, jout, k);
                }
            }
    }
    return sliceCount(*A, fat);
}

// Known-answer helpers for the reference's unit tests
void orc_c2p(double gamma, const double* con, double* prim) { Model M; M.gamma = gamma; CellC2P(M, con, prim); }
void orc_p2c(double gamma, const double* prim, double* con) { Model M; M.gamma = gamma; CellP2C(M, prim, con); }
double orc_norm2(const double* a, int n) { return norm2v(a, n); }
void orc_face_integral_area(const double* f0, const double* f1, const double* f2, const double* f3, double* area,
                            double* ctr) {
    double fI[3];
    GaussianFaceIntegral(f0, f1, f2, f3, IdVec, nullptr, fI);
    *area = fI[0];
    GaussianFaceIntegral(f0, f1, f2, f3, rVec, nullptr, fI);
    for (int c = 0; c < 3; ++c) ctr[c] = fI[c] / *area;
}
void orc_volume_integral(const double* xyzC /*8x3 row-major*/, double* vol, double* ctr) {
    double c8[8][3];
    for (int p = 0; p < 8; ++p) for (int c = 0; c < 3; ++c) c8[p][c] = xyzC[p * 3 + c];
    double w[5];
    GaussianVolumeIntegral(c8, CellDV, nullptr, w);
    *vol = w[0];
    for (int c = 0; c < 3; ++c) ctr[c] = w[1 + c] / w[0];
}
// PDM / reconstruction kernels on a single 8-point stencil (for unit tests of the limiter)
void orc_recon_lr(int rmeth, double pdmb, const double* vol8, const double* q8, const double* nq4, double* lr) {
    initWeights();
    double save = pdmb_g;
    pdmb_g = pdmb;
    double dV[recLen][vecLen], Q[recLen][vecLen], nQ[limLen][vecLen], Vi[vecLen], Ql[vecLen], Qr[vecLen];
    for (int n = 0; n < recLen; ++n) for (int i = 0; i < vecLen; ++i) { dV[n][i] = vol8[n]; Q[n][i] = q8[n]; }
    for (int n = 0; n < limLen; ++n) for (int i = 0; i < vecLen; ++i) nQ[n][i] = nq4[n];
    Central8(dV, Vi);
    GetLRs(rmeth, dV, nQ, Q, Vi, Ql, Qr);
    lr[0] = Ql[0]; lr[1] = Qr[0];
    pdmb_g = save;
}
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
