// Ring averaging about the axis of an LFM-type grid (ringav.F90, ringutils.F90, ringrecon.F90) and the
// axis fixes woven into the step: RingFlux2FieldFix after every bFlux2Fld, RingFlux after the fluxes,
// PoleE before the CT update, and RingAverage after the update.
//
// A ring is the Np = Nkp cells around the axis at one radius (slice i) and one distance from the axis
// (j = js+nR-1 or je-nR+1). One CTA owns one ring: the ring sits in shared memory, element-wise work is
// spread over the threads, and the few sequential sums of the reference (Fourier coefficients, chunk
// sums, the intra-chunk running flux) run on one thread each, in the reference's order.
#include <cstdio>
#include "gam_common.cuh"
#include "gam_kern.cuh"
#include "gam_lfm.cuh"
#include "gam_step.cuh"

namespace gam {

namespace {
constexpr int NFTMAX = 2;
constexpr int RTPB = 128;   // threads per ring CTA

struct RingDev {
    int Np, NumR, recon, NFTMAG, doMassRA, doFastLoop;
    int Nch[32];
};
struct F32B { float* v[3]; };

RingDev ringDev(const Handle& h) {
    RingDev r;
    r.Np = h.L.Nkp; r.NumR = h.ring.NumR; r.recon = h.ring.recon; r.NFTMAG = h.ring.NFTMAG;
    r.doMassRA = h.ring.doMassRA; r.doFastLoop = h.ring.doFastLoop;
    for (int n = 0; n < 32; ++n) r.Nch[n] = h.ring.Nch[n];
    return r;
}
inline unsigned nblk1(long long n, int b) { return (unsigned)((n + b - 1) / b); }
}  // namespace

// ------------------------------------------------------------------ RingFlux2FieldFix (ringutils.F90:380-433)
// With floatOnly (the FP32-flux half state, which exists only as floats) the float copies are the source.
__global__ void k_ring_bfix(Lay L, Par p, StateP s, F32B fb, int floatOnly) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nrow = (long long)L.Ni * L.Nk;
    if (t >= nrow * L.nG) return;
    int i = (int)(t % L.Ni);
    long long q = t / L.Ni;
    int k = (int)(q % L.Nk), n = 1 + (int)(q / L.Nk);
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && !p.ringDoS) continue;
        if (side == 1 && !p.ringDoE) continue;
        int jg = side == 0 ? L.js() - n : L.je() + n, jp, kp;
        lfmCC(L, p.ringDoS, p.ringDoE, jg, k, jp, kp);
        long long d = L.at(i, jg, k), src = L.at(i, jp, kp);
        for (int x = 0; x < 3; ++x) {
            if (floatOnly) { fb.v[x][d] = fb.v[x][src]; continue; }
            s.b[x][d] = s.b[x][src];
        }
    }
}

// ------------------------------------------------------------------ PredFix of the LFM blast wave (ICs/lfmbw.F90:227-248)
__global__ void k_predfix_lfm(Lay L, Par p, StateP s, F32B fb, int floatOnly) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nj * L.Nk * L.nG) return;
    int j = (int)(t % L.Nj);
    long long q = t / L.Nj;
    int k = (int)(q % L.Nk), n = 1 + (int)(q / L.Nk);
    int ig = L.is() - n, jp, kp;
    lfmCC(L, p.ringDoS, p.ringDoE, j, k, jp, kp);
    long long d = L.at(ig, j, k), src = L.at(L.is(), jp, kp);
    for (int x = 0; x < 3; ++x) {
        if (floatOnly) fb.v[x][d] = fb.v[x][src];
        else s.b[x][d] = s.b[x][src];
    }
}

// ------------------------------------------------------------------ RingFlux (ringutils.F90:663-680)
// J fluxes through the axis faces js and je+1 vanish (every i, k of the flux arrays)
template <typename O>
__global__ void k_ring_flux_zero(Lay L, Par p, FluxOut<O> FJ) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Ni * L.Nk) return;
    int i = (int)(t % L.Ni), k = (int)(t / L.Ni);
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && !p.ringDoS) continue;
        if (side == 1 && !p.ringDoE) continue;
        long long c = L.at(i, side == 0 ? L.js() : L.je() + 1, k);
        for (int v = 0; v < 5; ++v) FJ.g[v][c] = O(0);
        if (p.doMHD)
            for (int x = 0; x < 3; ++x) FJ.m[x][c] = O(0);
    }
}
// FixGasFluxLFM (gamdebug.F90:91-124): the K fluxes at ks and ke+1 take their mean
template <typename O>
__global__ void k_ring_flux_kavg(Lay L, FluxOut<O> FK) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Nip * L.Njp) return;
    int i = L.is() + (int)(t % L.Nip), j = L.js() + (int)(t / L.Nip);
    long long c0 = L.at(i, j, L.ks()), c1 = L.at(i, j, L.ke() + 1);
    for (int v = 0; v < 5; ++v) {
        O gF = O(0.5) * (FK.g[v][c0] + FK.g[v][c1]);
        FK.g[v][c0] = gF; FK.g[v][c1] = gF;
    }
    for (int x = 0; x < 3; ++x) {
        O mF = O(0.5) * (FK.m[x][c0] + FK.m[x][c1]);
        FK.m[x][c0] = mF; FK.m[x][c1] = mF;
    }
}

// ------------------------------------------------------------------ PoleE (ringav.F90:376-411) + FixEFieldLFM
// On the axis edges E_K = 0 and E_I is its ring mean (every k of the array)
__global__ void k_pole_e(Lay L, Par p, Vec3P E) {
    int nS = L.is() + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (nS > L.ie() + 1) return;
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && !p.ringDoS) continue;
        if (side == 1 && !p.ringDoE) continue;
        int j = side == 0 ? L.js() : L.je() + 1;
        double s = 0.0;
        for (int k = L.ks(); k <= L.ke(); ++k) s = s + E.v[0][L.at(nS, j, k)];
        double avg = s / L.Nkp;
        for (int k = 0; k < L.Nk; ++k) {
            long long c = L.at(nS, j, k);
            E.v[2][c] = 0.0;
            E.v[0][c] = avg;
        }
    }
}
// FixEFieldLFM (gamdebug.F90:149-175): E_I and E_J at ks and ke+1 take their mean
__global__ void k_fix_e_lfm(Lay L, Vec3P E) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int ni = L.Nip + 1, nj = L.Njp + 1;
    if (t >= (long long)ni * nj) return;
    int i = L.is() + (int)(t % ni), j = L.js() + (int)(t / ni);
    long long c0 = L.at(i, j, L.ks()), c1 = L.at(i, j, L.ke() + 1);
    double Ei = 0.5 * (E.v[0][c0] + E.v[0][c1]);
    double Ej = 0.5 * (E.v[1][c0] + E.v[1][c1]);
    E.v[0][c0] = Ei; E.v[0][c1] = Ei;
    E.v[1][c0] = Ej; E.v[1][c1] = Ej;
}

// ------------------------------------------------------------------ ring reconstruction (ringrecon.F90)
__device__ __forceinline__ double minmodR(double x, double y) {   // math.F90:192-197
    return 0.5 * (copysign(1.0, x) + copysign(1.0, y)) * fmin(fabs(x), fabs(y));
}
__device__ void ringLR(int meth, double fm2, double fm1, double f, double fp1, double fp2, double& vm, double& vp) {
    if (meth == 2) { vm = f; vp = f; return; }   // PCM
    if (meth == 0) {                             // PLM (ringrecon.F90:251-270)
        double dwL = f - fm1, dwR = fp1 - f, dwC = (fp1 - fm1) / 2.0;
        double min1 = fmin(2 * fabs(dwL), 2 * fabs(dwR));
        double min2 = fmin(min1, fabs(dwC));
        double dwM = copysign(min2, dwC);
        vp = f + 0.5 * dwM; vm = f - 0.5 * dwM;
        return;
    }
    // PPM (ringrecon.F90:282-322)
    double dvm2 = fm1 - fm2, dvm1 = f - fm1, dvp1 = fp1 - f, dvp2 = fp2 - fp1;
    double dvc = 0.5 * (dvm2 + dvm1), SM = 2.0 * minmodR(dvm2, dvm1), Sm1 = minmodR(dvc, SM);
    dvc = 0.5 * (dvm1 + dvp1); SM = 2.0 * minmodR(dvm1, dvp1);
    double Sp1 = minmodR(dvc, SM);
    dvc = 0.5 * (dvp2 + dvp1); SM = 2.0 * minmodR(dvp2, dvp1);
    double Sp2 = minmodR(dvc, SM);
    vp = 0.5 * (f + fp1) - (Sp2 - Sp1) / 6.0;
    vm = 0.5 * (f + fm1) - (Sp1 - Sm1) / 6.0;
    double ap = vp - f, am = vm - f;
    if (ap * am >= 0.0) { ap = 0.0; am = 0.0; }
    else {
        if (fabs(ap) >= 2.0 * fabs(am)) ap = -2.0 * am;
        if (fabs(am) >= 2.0 * fabs(ap)) am = -2.0 * ap;
    }
    vp = f + ap; vm = f + am;
}
// Chunk averages (each chunk's sum by one thread, in order)
__device__ void ringChunkAvg(const double* in, double* out, int Np, int Nc) {
    int dC = Np / Nc;
    for (int n = threadIdx.x; n < Nc; n += blockDim.x) {
        double s = 0.0;
        for (int m = 0; m < dC; ++m) s = s + in[n * dC + m];
        double a = s / dC;
        for (int m = 0; m < dC; ++m) out[n * dC + m] = a;
    }
}
// ReconstructRing (ringrecon.F90:34-98) of a chunk-averaged ring in place; every element evaluates the
// parabola of its chunk from the chunk values (periodic, two ghost chunks)
__device__ void ringReconstruct(double* rW, int Np, int Nc, int meth) {
    int dJ = Np / Nc;
    __syncthreads();
    double vals[8];   // Np / blockDim <= 512 / 128
    int cnt = 0;
    for (int e = threadIdx.x; e < Np; e += blockDim.x) {
        int n = e / dJ, m = e % dJ + 1;
        auto ch = [&](int q) { q = ((q % Nc) + Nc) % Nc; return rW[q * dJ]; };
        double f = ch(n), fL, fR;
        ringLR(meth, ch(n - 2), ch(n - 1), f, ch(n + 1), ch(n + 2), fL, fR);
        double a = 3 * (fL + fR - 2 * f), b = 2 * (3 * f - fR - 2 * fL), c = fL;
        vals[cnt++] = (a / 3.0) * (double)(3 * m * m - 3 * m + 1) / (double)(dJ * dJ) +
                      0.5 * b * (double)(2 * m - 1) / (double)dJ + c;
    }
    __syncthreads();
    cnt = 0;
    for (int e = threadIdx.x; e < Np; e += blockDim.x) rW[e] = vals[cnt++];
    __syncthreads();
}
// CleanRing / DirtyRing (ringav.F90:416-458) with the trigonometric table of the ring in shared memory
// (cosT[m*Np+n] = cos(m*phi_n), sinT likewise); cFT in shared memory
__device__ void ringClean(double* Q, const double* cosT, const double* sinT, double* cFT, int Np, int numFT) {
    __syncthreads();
    if (threadIdx.x == 0) {
        double aScl = (double)(2.0f / (float)Np);
        for (int m = 0; m <= NFTMAX; ++m) { cFT[2 * m] = 0.0; cFT[2 * m + 1] = 0.0; }
        for (int n = 0; n < Np; ++n)
            for (int m = 0; m <= numFT; ++m) {
                cFT[2 * m] = cFT[2 * m] + Q[n] * cosT[m * Np + n];
                cFT[2 * m + 1] = cFT[2 * m + 1] + Q[n] * sinT[m * Np + n];
            }
        cFT[0] = 0.5 * aScl * cFT[0]; cFT[1] = 0.5 * aScl * cFT[1];
        for (int m = 1; m <= numFT; ++m) { cFT[2 * m] = 1.0 * aScl * cFT[2 * m]; cFT[2 * m + 1] = 1.0 * aScl * cFT[2 * m + 1]; }
    }
    __syncthreads();
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        double q = Q[n];
        for (int m = 0; m <= numFT; ++m) q = q - cFT[2 * m] * cosT[m * Np + n] - cFT[2 * m + 1] * sinT[m * Np + n];
        Q[n] = q;
    }
    __syncthreads();
}
__device__ void ringDirty(double* Q, const double* cosT, const double* sinT, const double* cFT, int Np, int numFT) {
    __syncthreads();
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        double q = Q[n];
        for (int m = 0; m <= numFT; ++m) q = q + cFT[2 * m] * cosT[m * Np + n] + cFT[2 * m + 1] * sinT[m * Np + n];
        Q[n] = q;
    }
    __syncthreads();
}

// ------------------------------------------------------------------ CalcSmoothE (ringav.F90:203-336), LFM axis
// grid: (nS = is..ie+1) x (nR = 1..NumR); pole 0 = SPOLE (+x), 1 = EPOLE (-x)
__global__ void __launch_bounds__(RTPB) k_ring_smooth_e(Lay L, RingDev R, StateP s, Vec3P SE, int pole) {
    extern __shared__ __align__(16) double rsm[];
    const int Np = R.Np;
    double* cosT = rsm;                       // (NFTMAX+1)*Np
    double* sinT = cosT + (NFTMAX + 1) * Np;  // (NFTMAX+1)*Np
    double* bFlx = sinT + (NFTMAX + 1) * Np;  // 3*Np
    double* rFlx = bFlx + 3 * Np;             // Np
    double* raFlx = rFlx + Np;                // Np
    double* dEr = raFlx + Np;                 // 2*Np (I, J)
    double* cFT = dEr + 2 * Np;               // 2*(NFTMAX+1)
    const int nS = L.is() + blockIdx.x, nR = 1 + blockIdx.y;
    const int NumCh = R.Nch[nR - 1], dC = Np / NumCh;
    const double dp = 2.0 * PI / Np;
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        double phi = dp * (n + 1) - 0.5 * dp;
        for (int m = 0; m <= NFTMAX; ++m) { cosT[m * Np + n] = cos(1.0 * m * phi); sinT[m * Np + n] = sin(1.0 * m * phi); }
        int k = L.ks() + n;
        if (pole == 0) {   // PullRingI (ringutils.F90:753-787)
            bFlx[n] = s.mf[0][L.at(nS, L.js() + nR - 1, k)];
            bFlx[Np + n] = s.mf[1][L.at(nS, L.js() + nR, k)];
            bFlx[2 * Np + n] = s.mf[2][L.at(nS, L.js() + nR - 1, k)];
        } else {
            long long c = L.at(nS, L.je() - nR + 1, k);
            bFlx[n] = s.mf[0][c]; bFlx[Np + n] = s.mf[1][c]; bFlx[2 * Np + n] = s.mf[2][c];
        }
        dEr[n] = 0.0; dEr[Np + n] = 0.0;
    }
    for (int d = 0; d < 2; ++d) {
        const int fD = d == 0 ? 1 : 0, eD = d == 0 ? 0 : 1;   // (J flux -> E_I, I flux -> E_J)
        const double eScl = d == 0 ? 1.0 : -1.0;
        __syncthreads();
        for (int n = threadIdx.x; n < Np; n += blockDim.x) rFlx[n] = bFlx[fD * Np + n];
        ringClean(rFlx, cosT, sinT, cFT, Np, R.NFTMAG);
        ringChunkAvg(rFlx, raFlx, Np, NumCh);
        ringReconstruct(raFlx, Np, NumCh, R.recon);
        ringDirty(raFlx, cosT, sinT, cFT, Np, R.NFTMAG);
        // running flux change within each chunk -> ring E (one thread per chunk, in order)
        for (int n = threadIdx.x; n < NumCh; n += blockDim.x) {
            int lRs = n * dC;
            double cumFlx = -(raFlx[lRs] - bFlx[fD * Np + lRs]);
            for (int m = 1; m < dC; ++m) {
                dEr[eD * Np + lRs + m] = eScl * cumFlx;
                cumFlx = cumFlx - (raFlx[lRs + m] - bFlx[fD * Np + lRs + m]);
            }
        }
        __syncthreads();
    }
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        int k = L.ks() + n;
        if (pole == 0) {
            SE.v[0][L.at(nS, L.js() + nR, k)] = dEr[n];
            SE.v[1][L.at(nS, L.js() + nR - 1, k)] = dEr[Np + n];
            SE.v[2][L.at(nS, L.js() + nR - 1, k)] = 0.0;
            if (n == 0) {   // replicate at ke+1
                SE.v[0][L.at(nS, L.js() + nR, L.ke() + 1)] = dEr[0];
                SE.v[1][L.at(nS, L.js() + nR - 1, L.ke() + 1)] = dEr[Np];
            }
        } else {
            long long c = L.at(nS, L.je() - nR + 1, k);
            SE.v[0][c] = dEr[n]; SE.v[1][c] = dEr[Np + n]; SE.v[2][c] = 0.0;
            if (n == 0) {
                long long ce = L.at(nS, L.je() - nR + 1, L.ke() + 1);
                SE.v[0][ce] = dEr[0]; SE.v[1][ce] = dEr[Np];
            }
        }
    }
}

// ------------------------------------------------------------------ E2Flux with dt = 1 in place (fields.F90:18-51)
__global__ void k_e2flux_inplace(Lay L, Vec3P E, StateP s) {
    Reg r = {L.is(), L.Nip + 1, L.js(), L.Njp + 1, L.ks(), L.Nkp + 1};
    int i, j, k;
    if (!reg_ijk(r, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    long long c = L.at(i, j, k), cj = c + L.P, ck = c + (long long)L.P * L.Q;
    const double* Ei = E.v[0]; const double* Ej = E.v[1]; const double* Ek = E.v[2];
    double dfi = Ek[cj] - Ek[c] - Ej[ck] + Ej[c];
    double dfj = Ei[ck] - Ei[c] - Ek[c + 1] + Ek[c];
    double dfk = Ej[c + 1] - Ej[c] - Ei[cj] + Ei[c];
    s.mf[0][c] = s.mf[0][c] - 1.0 * dfi;
    s.mf[1][c] = s.mf[1][c] - 1.0 * dfj;
    s.mf[2][c] = s.mf[2][c] - 1.0 * dfk;
}

// ------------------------------------------------------------------ CleanLoops (ringav.F90:339-373), LFM axis
__global__ void k_clean_loops(Lay L, Par p, StateP s, double tScl) {
    int nS = L.is() + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (nS > L.ie() + 1) return;
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && !p.ringDoS) continue;
        if (side == 1 && !p.ringDoE) continue;
        int j = side == 0 ? L.js() : L.je();
        double sum = 0.0;
        for (int k = L.ks(); k <= L.ke(); ++k) sum = sum + s.mf[2][L.at(nS, j, k)];
        double avgFlx = sum / L.Nkp;
        for (int k = L.ks(); k <= L.ke() + 1; ++k) {
            long long c = L.at(nS, j, k);
            s.mf[2][c] = s.mf[2][c] - tScl * avgFlx;
        }
    }
}

// ------------------------------------------------------------------ SmoothGas (ringav.F90:82-200), single fluid
// grid: (nS = is..ie) x (nR = 1..NumR)
__global__ void __launch_bounds__(RTPB) k_ring_smooth_gas(Lay L, Par p, RingDev R, StateP s, int pole) {
    extern __shared__ __align__(16) double rsm[];
    const int Np = R.Np;
    double* rW = rsm;            // 5*Np
    double* raW = rW + 5 * Np;   // 5*Np
    const int nS = L.is() + blockIdx.x, nR = 1 + blockIdx.y;
    const int NumCh = R.Nch[nR - 1];
    const int jR = pole == 0 ? L.js() + nR - 1 : L.je() - nR + 1;
    const double gm1 = p.gamma - 1;
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {   // PullRingCC + Gas2Ring (ringutils.F90:800-826)
        long long c = L.at(nS, jR, L.ks() + n);
        double D = dmax(s.gas[0][c], p.dFloor);
        double Mx = s.gas[1][c], My = s.gas[2][c], Mz = s.gas[3][c], E = s.gas[4][c];
        double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
        double P = dmax(gm1 * (E - KinE), p.pFloor);
        rW[n] = D; rW[Np + n] = Mx; rW[2 * Np + n] = My; rW[3 * Np + n] = Mz;
        rW[4 * Np + n] = R.doMassRA ? p.gamma * P : P / gm1;
    }
    __syncthreads();
    for (int v = 0; v < 5; ++v) ringChunkAvg(rW + v * Np, raW + v * Np, Np, NumCh);
    for (int v = 0; v < 5; ++v) ringReconstruct(raW + v * Np, Np, NumCh, R.recon);
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {   // Ring2Gas (ringutils.F90:829-856) + PushRingCC
        double D = dmax(raW[n], p.dFloor);
        double Mx = raW[Np + n], My = raW[2 * Np + n], Mz = raW[3 * Np + n];
        double P = R.doMassRA ? (raW[4 * Np + n] / D) * D / p.gamma : gm1 * raW[4 * Np + n];
        P = dmax(P, p.pFloor);
        double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
        long long c = L.at(nS, jR, L.ks() + n);
        s.gas[0][c] = D; s.gas[1][c] = Mx; s.gas[2][c] = My; s.gas[3][c] = Mz;
        s.gas[4][c] = KinE + P / gm1;
    }
}

// ------------------------------------------------------------------ RingGridFix (ringutils.F90:229-377), LFM axis
// dk of the ring cells widened by the chunk size (dk counts in CalcDT)
__global__ void k_ring_dk_scale(Lay L, Par p, RingDev R, double* dk) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)L.Ni * L.Nk) return;
    int i = (int)(t % L.Ni), k = (int)(t / L.Ni);
    for (int iR = 1; iR <= R.NumR; ++iR) {
        int dJ = R.Np / R.Nch[iR - 1];
        if (p.ringDoS) { long long c = L.at(i, L.js() + iR - 1, k); dk[c] = dJ * dk[c]; }
        if (p.ringDoE) { long long c = L.at(i, L.je() - iR + 1, k); dk[c] = dJ * dk[c]; }
    }
}
struct GridW { double* vol; double* dl[3]; double* face[3]; double* Tn[3][3]; };
// ghost metrics across the axis from the conjugate cells / faces; J and K face normals flip sign
__global__ void k_ring_grid_fix(Lay L, Par p, GridW g) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int ni = L.Ni + 1, nk = L.Nk + 1;
    if (t >= (long long)ni * nk * L.nG) return;
    int i = (int)(t % ni);
    long long q = t / ni;
    int k = (int)(q % nk), n = 1 + (int)(q / nk);
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && !p.ringDoS) continue;
        if (side == 1 && !p.ringDoE) continue;
        int jg = side == 0 ? L.js() - n : L.je() + n, jp, kp;
        if (k < L.Nk && i < L.Ni) {
            lfmCC(L, p.ringDoS, p.ringDoE, jg, k, jp, kp);
            long long d = L.at(i, jg, k), src = L.at(i, jp, kp);
            g.vol[d] = g.vol[src];
            for (int x = 0; x < 3; ++x) g.dl[x][d] = g.dl[x][src];
        }
        for (int dir = 0; dir < 3; ++dir) {
            int jf = (dir == 1 && side == 1) ? jg + 1 : jg;   // the first outer J ghost face is je+2
            lfmFC(L, p.ringDoS, p.ringDoE, dir, jf, k, jp, kp);
            long long d = L.at(i, jf, k), src = L.at(i, jp, kp);
            double sgn = dir == 0 ? 1.0 : -1.0;
            for (int x = 0; x < 3; ++x) g.Tn[dir][x][d] = sgn * g.Tn[dir][x][src];
            g.face[dir][d] = g.face[dir][src];
        }
    }
}

void launch_ring_grid_fix(Handle& h, cudaStream_t st) {
    const Lay& L = h.L;
    RingDev R = ringDev(h);
    k_ring_dk_scale<<<nblk1((long long)L.Ni * L.Nk, 256), 256, 0, st>>>(L, h.p, R, h.dk);
    GridW g;
    g.vol = h.volume; g.dl[0] = h.di; g.dl[1] = h.dj; g.dl[2] = h.dk;
    for (int d = 0; d < 3; ++d) {
        g.face[d] = h.face[d];
        for (int x = 0; x < 3; ++x) g.Tn[d][x] = h.Tf[d][x];
    }
    k_ring_grid_fix<<<nblk1((long long)(L.Ni + 1) * (L.Nk + 1) * L.nG, 256), 256, 0, st>>>(L, h.p, g);
    h.launches += 2;
}

// ------------------------------------------------------------------ launchers
static size_t smoothESmem(int Np) { return sizeof(double) * ((size_t)2 * (NFTMAX + 1) * Np + 7 * (size_t)Np + 2 * (NFTMAX + 1)); }
static size_t smoothGasSmem(int Np) { return sizeof(double) * 10 * (size_t)Np; }

void ring_kernels_init() {
    cudaFuncSetAttribute(k_ring_smooth_e, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smoothESmem(512));
    cudaFuncSetAttribute(k_ring_smooth_gas, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smoothGasSmem(512));
}

void launch_ring_bfix(Handle& h, const StateP& s, cudaStream_t st, bool withF32) {
    const Lay& L = h.L;
    F32B fb{};
    if (withF32) for (int x = 0; x < 3; ++x) fb.v[x] = h.f32.hb[x];
    long long n = (long long)L.Ni * L.Nk * L.nG;
    k_ring_bfix<<<nblk1(n, 256), 256, 0, st>>>(L, h.p, s, fb, withF32 ? 1 : 0);
    h.launches++;
}
void launch_predfix_lfm(Handle& h, const StateP& s, cudaStream_t st, bool withF32) {
    const Lay& L = h.L;
    F32B fb{};
    if (withF32) for (int x = 0; x < 3; ++x) fb.v[x] = h.f32.hb[x];
    long long n = (long long)L.Nj * L.Nk * L.nG;
    k_predfix_lfm<<<nblk1(n, 256), 256, 0, st>>>(L, h.p, s, fb, withF32 ? 1 : 0);
    h.launches++;
}
template <typename O>
static void ring_flux(Handle& h, O* const (*g)[5], O* const (*m)[3], cudaStream_t st) {
    const Lay& L = h.L;
    FluxOut<O> FJ, FK;
    for (int v = 0; v < 5; ++v) { FJ.g[v] = g[1][v]; FK.g[v] = g[2][v]; }
    for (int x = 0; x < 3; ++x) { FJ.m[x] = m[1][x]; FK.m[x] = m[2][x]; }
    k_ring_flux_zero<O><<<nblk1((long long)L.Ni * L.Nk, 256), 256, 0, st>>>(L, h.p, FJ);
    h.launches++;
    if (h.p.doMHD) {
        k_ring_flux_kavg<O><<<nblk1((long long)L.Nip * L.Njp, 256), 256, 0, st>>>(L, FK);
        h.launches++;
    }
}
void launch_ring_flux(Handle& h, cudaStream_t st) {
    if (h.prec == PREC_FP32FLUX) ring_flux<float>(h, h.f32.gflx, h.f32.mflx, st);
    else ring_flux<double>(h, h.gflx, h.mflx, st);
}
void launch_pole_e(Handle& h, double* const* E, cudaStream_t st) {
    const Lay& L = h.L;
    Vec3P e = {{E[0], E[1], E[2]}};
    k_pole_e<<<nblk1(L.Nip + 1, 64), 64, 0, st>>>(L, h.p, e);
    k_fix_e_lfm<<<nblk1((long long)(L.Nip + 1) * (L.Njp + 1), 256), 256, 0, st>>>(L, e);
    h.launches += 2;
}
void launch_fix_e_lfm(Handle& h, double* const* E, cudaStream_t st) {
    const Lay& L = h.L;
    Vec3P e = {{E[0], E[1], E[2]}};
    k_fix_e_lfm<<<nblk1((long long)(L.Nip + 1) * (L.Njp + 1), 256), 256, 0, st>>>(L, e);
    h.launches++;
}
void launch_ring_average(Handle& h, const StateP& s, cudaStream_t st) {
    const Lay& L = h.L;
    const Par& p = h.p;
    RingDev R = ringDev(h);
    Vec3P SE = {{h.SmoothE[0], h.SmoothE[1], h.SmoothE[2]}};
    cudaMemsetAsync(h.SmoothE[0], 0, sizeof(double) * L.E * 3, st);   // InitRAVec: contiguous planes
    h.launches++;
    dim3 ge((unsigned)(L.Nip + 1), (unsigned)R.NumR);
    if (p.ringDoS) { k_ring_smooth_e<<<ge, RTPB, smoothESmem(R.Np), st>>>(L, R, s, SE, 0); h.launches++; }
    if (p.ringDoE) { k_ring_smooth_e<<<ge, RTPB, smoothESmem(R.Np), st>>>(L, R, s, SE, 1); h.launches++; }
    launch_pole_e(h, h.SmoothE, st);
    long long nf = (long long)(L.Nip + 1) * (L.Njp + 1) * (L.Nkp + 1);
    k_e2flux_inplace<<<nblk1(nf, 256), 256, 0, st>>>(L, SE, s);
    h.launches++;
    if (h.ring.doCleanLoop) {
        double tScl = h.ring.doFastLoop ? 1.0 : 1.0 / L.Nkp;
        k_clean_loops<<<nblk1(L.Nip + 1, 64), 64, 0, st>>>(L, p, s, tScl);
        h.launches++;
    }
    launch_bflux2fld(h, s, st);   // includes the ring fix
    dim3 gg((unsigned)L.Nip, (unsigned)R.NumR);
    if (p.ringDoS) { k_ring_smooth_gas<<<gg, RTPB, smoothGasSmem(R.Np), st>>>(L, p, R, s, 0); h.launches++; }
    if (p.ringDoE) { k_ring_smooth_gas<<<gg, RTPB, smoothGasSmem(R.Np), st>>>(L, p, R, s, 1); h.launches++; }
}

int ring_kernels_per_step(const Handle& h) {
    if (!h.p.doRing) return 0;
    const Par& p = h.p;
    int sides = (p.ringDoS ? 1 : 0) + (p.ringDoE ? 1 : 0);
    int n = 0;
    n += 1 + (p.predFixLFM ? 1 : 0);                    // predictor: ring fix (+ PredFix)
    n += 1 + (p.doMHD ? 1 : 0);                         // RingFlux
    if (p.doMHD) n += 2;                                // PoleE on the step E
    n += 1 + sides + 2 + 1 + (h.ring.doCleanLoop ? 1 : 0) + 2 + sides;   // RingAverage
    n += 1;                                             // ring fix after the final bFlux2Fld
    return n;
}

}  // namespace gam
