// Slice output on the device: the variables writeSlc (gioH5.F90:255-602) computes from State, for the
// active cells of a single-fluid, non-magnetosphere problem: D, Vx, Vy, Vz, P, Cs, Bx, By, Bz, Pb,
// Jx, Jy, Jz and, with fat output, Ex, Ey, Ez, DivB (and DivdB with a background field). Each variable is
// one Fortran-ordered (is:ie, js:je, ks:ke) block of the output, in that order.
//
// The current follows bFld2Jxyz (gridutils.F90:314-478): B.dl on the cell edges (one kernel), the
// circulation per face (one kernel), the cell field of those face "fluxes" (per cell, with the two
// rings next to an LFM axis re-interpolated toward the pole). The output is staged in an HBM buffer and
// copied to the host on a copy stream, so a caller can keep stepping while the copy runs.
#include <cstdio>
#include "gam_common.cuh"
#include "gam_kern.cuh"
#include "gam_step.cuh"

namespace gam {

namespace {
inline unsigned nb(long long n, int b) { return (unsigned)((n + b - 1) / b); }
struct Corn { const double* x[3]; };
// gfortran's NORM2 expansion (scaled sum of squares), as the oracle's
__device__ double norm2v3d(const double* a) {
    double scale = 0.0, ssq = 1.0;
    for (int q = 0; q < 3; ++q) {
        if (a[q] != 0.0) {
            double ax = fabs(a[q]);
            if (scale < ax) { ssq = 1.0 + ssq * sq(scale / ax); scale = ax; }
            else ssq = ssq + sq(ax / scale);
        }
    }
    return scale * sqrt(ssq);
}
__device__ __forceinline__ void corner(const Lay& L, const Corn& X, int i, int j, int k, double* v) {
    long long c = L.at(i, j, k);
    v[0] = X.x[0][c]; v[1] = X.x[1][c]; v[2] = X.x[2][c];
}
}  // namespace

// B.dl along the cell edges (gridutils.F90:339-373): bInt[d] at the edge of cell (i,j,k) along d
__global__ void k_io_bint(Lay L, StateP s, Corn X, Vec3P bInt) {
    Reg r = {1, L.Ni - 1, 1, L.Nj - 1, 1, L.Nk - 1};
    int i, j, k;
    if (!reg_ijk(r, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    long long c = L.at(i, j, k), ci = c - 1, cj = c - L.P, ck = c - (long long)L.P * L.Q;
    double p0[3], p1[3];
    corner(L, X, i, j, k, p0);
    if (i <= L.Ni - 2) {   // isGoodEdgeIJK(i+1,j,k,I)
        corner(L, X, i + 1, j, k, p1);
        double s_ = 0.0;
        for (int x = 0; x < 3; ++x) {
            double bA = 0.25 * (s.b[x][c] + s.b[x][cj] + s.b[x][ck] + s.b[x][cj - (long long)L.P * L.Q]);
            s_ = s_ + bA * (p1[x] - p0[x]);
        }
        bInt.v[0][c] = s_;
    }
    if (j <= L.Nj - 2) {   // isGoodEdgeIJK(i,j+1,k,J)
        corner(L, X, i, j + 1, k, p1);
        double s_ = 0.0;
        for (int x = 0; x < 3; ++x) {
            double bA = 0.25 * (s.b[x][c] + s.b[x][ck] + s.b[x][ci] + s.b[x][ci - (long long)L.P * L.Q]);
            s_ = s_ + bA * (p1[x] - p0[x]);
        }
        bInt.v[1][c] = s_;
    }
    if (k <= L.Nk - 2) {   // isGoodEdgeIJK(i,j,k+1,K)
        corner(L, X, i, j, k + 1, p1);
        double s_ = 0.0;
        for (int x = 0; x < 3; ++x) {
            double bA = 0.25 * (s.b[x][c] + s.b[x][ci] + s.b[x][cj] + s.b[x][cj - 1]);
            s_ = s_ + bA * (p1[x] - p0[x]);
        }
        bInt.v[2][c] = s_;
    }
}
// circulation of bInt around each face (gridutils.F90:376-398)
__global__ void k_io_jds(Lay L, Vec3P bInt, Vec3P JdS) {
    Reg r = {1, L.Ni - 1, 1, L.Nj - 1, 1, L.Nk - 1};
    int i, j, k;
    if (!reg_ijk(r, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    long long c = L.at(i, j, k), cj = c + L.P, ck = c + (long long)L.P * L.Q;
    const double* bI = bInt.v[0]; const double* bJ = bInt.v[1]; const double* bK = bInt.v[2];
    if (j <= L.Nj - 2 && k <= L.Nk - 2) JdS.v[0][c] = bJ[c] + bK[cj] - bJ[ck] - bK[c];
    if (i <= L.Ni - 2 && k <= L.Nk - 2) JdS.v[1][c] = bK[c] + bI[ck] - bK[c + 1] - bI[c];
    if (i <= L.Ni - 2 && j <= L.Nj - 2) JdS.v[2][c] = bI[c] + bJ[c + 1] - bI[cj] - bJ[c];
}

struct SliceOut { double* o; long long Na; int fat, bg, mhd; };
__device__ __forceinline__ double& sref(const SliceOut& S, const Lay& L, int v, int i, int j, int k) {
    return S.o[v * S.Na + (i - L.is()) + (long long)L.Nip * ((j - L.js()) + (long long)L.Njp * (k - L.ks()))];
}

// per active cell: D, V, P, Cs, B, Pb, J (cell field of J.dS), and with fat output E and DivB
__global__ void k_io_cells(Lay L, Par p, GridP g, StateP s, Vec3P JdS, Vec3P E, Corn X, SliceOut S) {
    Reg r = {L.is(), L.Nip, L.js(), L.Njp, L.ks(), L.Nkp};
    int i, j, k;
    if (!reg_ijk(r, blockIdx.x * (long long)blockDim.x + threadIdx.x, i, j, k)) return;
    long long c = L.at(i, j, k);
    double D = s.gas[0][c], Mx = s.gas[1][c], My = s.gas[2][c], Mz = s.gas[3][c], En = s.gas[4][c];
    sref(S, L, 0, i, j, k) = D < 0.0 ? 0.0 : D;
    double V0 = 0.0, V1 = 0.0, V2 = 0.0, P = 0.0;
    if (D > TINY) {
        V0 = Mx / D; V1 = My / D; V2 = Mz / D;
        P = (p.gamma - 1) * (En - 0.5 * (Mx * Mx + My * My + Mz * Mz) / D);
    }
    sref(S, L, 1, i, j, k) = V0; sref(S, L, 2, i, j, k) = V1; sref(S, L, 3, i, j, k) = V2; sref(S, L, 4, i, j, k) = P;
    {   // CellPress2Cs (gamutils.F90:324-341)
        double rho = dmax(D, p.dFloor);
        double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
        double KinE = 0.5 * rho * (sq(vx) + sq(vy) + sq(vz));
        double Pc = dmax((p.gamma - 1) * (En - KinE), p.pFloor);
        sref(S, L, 5, i, j, k) = sqrt(p.gamma * Pc / rho);
    }
    double B[3] = {0.0, 0.0, 0.0};
    if (S.mhd)
        for (int x = 0; x < 3; ++x) B[x] = s.b[x][c] + (S.bg ? g.B0[x][c] : 0.0);
    for (int x = 0; x < 3; ++x) sref(S, L, 6 + x, i, j, k) = B[x];
    sref(S, L, 9, i, j, k) = 0.5 * (sq(B[0]) + sq(B[1]) + sq(B[2]));
    double J[3] = {0.0, 0.0, 0.0};
    if (S.mhd) {
        double* jds[3] = {JdS.v[0], JdS.v[1], JdS.v[2]};
        cellBxyz(L, g, jds, c, J);
    }
    for (int x = 0; x < 3; ++x) sref(S, L, 10 + x, i, j, k) = 1.0 * J[x];
    if (!S.fat) return;
    double Ex[3] = {0.0, 0.0, 0.0};
    if (S.mhd) {   // CellExyz (gridutils.F90:559-609)
        auto ef = [&](int d, long long q) { double e = g.edge[d][q]; return e == 0.0 ? 0.0 : E.v[d][q] / e; };
        long long cj = c + L.P, ck = c + (long long)L.P * L.Q;
        double cc[3];
        cc[0] = 0.25 * (ef(0, c) + ef(0, ck) + ef(0, cj) + ef(0, cj + (long long)L.P * L.Q));
        cc[1] = 0.25 * (ef(1, c) + ef(1, ck) + ef(1, c + 1) + ef(1, ck + 1));
        cc[2] = 0.25 * (ef(2, c) + ef(2, c + 1) + ef(2, cj) + ef(2, cj + 1));
        double vec[3][3];
        for (int d = 0; d < 3; ++d) {   // ijkVec (metric.F90:172-201)
            double a[3], b[3], cc4[4][3], cm4[4][3];
            // corner orders of the reference's four-point sums
            if (d == 0) {
                corner(L, X, i + 1, j, k, cc4[0]); corner(L, X, i + 1, j + 1, k, cc4[1]);
                corner(L, X, i + 1, j, k + 1, cc4[2]); corner(L, X, i + 1, j + 1, k + 1, cc4[3]);
                corner(L, X, i, j, k, cm4[0]); corner(L, X, i, j + 1, k, cm4[1]);
                corner(L, X, i, j, k + 1, cm4[2]); corner(L, X, i, j + 1, k + 1, cm4[3]);
            } else if (d == 1) {
                corner(L, X, i, j + 1, k, cc4[0]); corner(L, X, i + 1, j + 1, k, cc4[1]);
                corner(L, X, i, j + 1, k + 1, cc4[2]); corner(L, X, i + 1, j + 1, k + 1, cc4[3]);
                corner(L, X, i, j, k, cm4[0]); corner(L, X, i + 1, j, k, cm4[1]);
                corner(L, X, i, j, k + 1, cm4[2]); corner(L, X, i + 1, j, k + 1, cm4[3]);
            } else {
                corner(L, X, i, j, k + 1, cc4[0]); corner(L, X, i + 1, j, k + 1, cc4[1]);
                corner(L, X, i, j + 1, k + 1, cc4[2]); corner(L, X, i + 1, j + 1, k + 1, cc4[3]);
                corner(L, X, i, j, k, cm4[0]); corner(L, X, i + 1, j, k, cm4[1]);
                corner(L, X, i, j + 1, k, cm4[2]); corner(L, X, i + 1, j + 1, k, cm4[3]);
            }
            for (int x = 0; x < 3; ++x) {
                a[x] = 0.25 * (cc4[0][x] + cc4[1][x] + cc4[2][x] + cc4[3][x]);
                b[x] = 0.25 * (cm4[0][x] + cm4[1][x] + cm4[2][x] + cm4[3][x]);
                vec[d][x] = a[x] - b[x];
            }
            double n = norm2v3d(vec[d]);
            for (int x = 0; x < 3; ++x) vec[d][x] = vec[d][x] / n;
        }
        const double* iV = vec[0]; const double* jV = vec[1]; const double* kV = vec[2];
        double M[3][3];   // ijkMatrix (metric.F90:203-221)
        M[0][0] = kV[2] * jV[1] - kV[1] * jV[2]; M[1][0] = kV[0] * jV[2] - kV[2] * jV[0]; M[2][0] = kV[1] * jV[0] - kV[0] * jV[1];
        M[0][1] = kV[1] * iV[2] - kV[2] * iV[1]; M[1][1] = kV[2] * iV[0] - kV[0] * iV[2]; M[2][1] = kV[0] * iV[1] - kV[1] * iV[0];
        M[0][2] = jV[2] * iV[1] - jV[1] * iV[2]; M[1][2] = jV[0] * iV[2] - jV[2] * iV[0]; M[2][2] = jV[1] * iV[0] - jV[0] * iV[1];
        double det = iV[0] * M[0][0] + jV[0] * M[0][1] + kV[0] * M[0][2];
        for (int q = 0; q < 3; ++q) Ex[q] = (M[q][0] * cc[0] + M[q][1] * cc[1] + M[q][2] * cc[2]) / det;
    }
    for (int x = 0; x < 3; ++x) sref(S, L, 13 + x, i, j, k) = Ex[x];
    long long cj = c + L.P, ck = c + (long long)L.P * L.Q;
    double dFi = s.mf[0][c] - s.mf[0][c + 1], dFj = s.mf[1][c] - s.mf[1][cj], dFk = s.mf[2][c] - s.mf[2][ck];
    double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
    if (S.bg) {
        dFi0 = g.bFlux0[0][c] - g.bFlux0[0][c + 1];
        dFj0 = g.bFlux0[1][c] - g.bFlux0[1][cj];
        dFk0 = g.bFlux0[2][c] - g.bFlux0[2][ck];
    }
    sref(S, L, 16, i, j, k) = fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
    if (S.bg) sref(S, L, 17, i, j, k) = fabs(dFi + dFj + dFk + 0.0 + 0.0 + 0.0);
}

// the two rings next to an LFM axis: J re-interpolated toward the pole value (gridutils.F90:414-470) and,
// with fat output, E (FixRAVec, gioH5.F90:577-601 / metric.F90:227-300); one thread per (i, side)
__global__ void k_io_ring(Lay L, Par p, SliceOut S) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.Nip * 2) return;
    int i = L.is() + t / 2, side = t % 2;
    if ((side == 0 && !p.ringDoS) || (side == 1 && !p.ringDoE)) return;
    const int Nk = L.Nkp;
    if (S.mhd) {
        const double a8 = (double)0.8f, a2 = (double)0.2f, a4 = (double)0.4f, a6 = (double)0.6f;
        int j3 = side == 0 ? L.js() + 2 : L.je() - 2, j1 = side == 0 ? L.js() : L.je(), j2 = side == 0 ? L.js() + 1 : L.je() - 1;
        for (int x = 0; x < 3; ++x) {
            double J0 = 0.0;
            for (int k = L.ks(); k <= L.ke(); ++k) J0 = J0 + sref(S, L, 10 + x, i, j3, k);
            J0 = J0 / Nk;
            for (int k = L.ks(); k <= L.ke(); ++k) {
                double J3 = sref(S, L, 10 + x, i, j3, k);
                sref(S, L, 10 + x, i, j1, k) = a8 * J0 + a2 * J3;
                sref(S, L, 10 + x, i, j2, k) = a4 * J0 + a6 * J3;
            }
        }
    }
    if (S.fat) {
        const double w1 = (double)(2.0f / 3.0f), w2 = (double)(1.0f / 3.0f);
        int jin = side == 0 ? L.js() : L.je(), jout = side == 0 ? L.js() + 1 : L.je() - 1;
        for (int x = 0; x < 3; ++x) {
            double Q0 = 0.0;
            for (int k = L.ks(); k <= L.ke(); ++k) Q0 = Q0 + sref(S, L, 13 + x, i, jout, k);
            Q0 = Q0 / Nk;
            for (int k = L.ks(); k <= L.ke(); ++k) sref(S, L, 13 + x, i, jin, k) = w1 * Q0 + w2 * sref(S, L, 13 + x, i, jout, k);
        }
    }
}

long long slice_count(const Handle& h, int fat) {
    long long nv = 13 + (fat ? 4 + (h.p.doBackground ? 1 : 0) : 0);
    return nv * (long long)h.L.Nip * h.L.Njp * h.L.Nkp;
}

// compute the slice of State n into dst (device, slice_count doubles) on stream st; scratch: 6 planes
int enqueue_slice(Handle& h, int fat, double* dst, double* scratch, cudaStream_t st) {
    const Lay& L = h.L;
    StateP s = h.S[h.cur];
    GridP g = h.gridP();
    Corn X = {{h.xyz[0], h.xyz[1], h.xyz[2]}};
    Vec3P bInt = {{scratch, scratch + L.E, scratch + 2 * L.E}};
    Vec3P JdS = {{scratch + 3 * L.E, scratch + 4 * L.E, scratch + 5 * L.E}};
    SliceOut S{dst, (long long)L.Nip * L.Njp * L.Nkp, fat, h.p.doBackground, h.p.doMHD};
    if (h.p.doMHD) {
        cudaMemsetAsync(scratch, 0, sizeof(double) * L.E * 6, st);   // allocGridVec wipes bInt and JdS
        long long n = (long long)(L.Ni - 1) * (L.Nj - 1) * (L.Nk - 1);
        k_io_bint<<<nb(n, 256), 256, 0, st>>>(L, s, X, bInt);
        k_io_jds<<<nb(n, 256), 256, 0, st>>>(L, bInt, JdS);
        h.launches += 3;
    }
    Vec3P E = {{h.E[0], h.E[1], h.E[2]}};
    k_io_cells<<<nb(S.Na, 128), 128, 0, st>>>(L, h.p, g, s, JdS, E, X, S);
    h.launches++;
    if (h.p.doRing) {
        k_io_ring<<<nb(L.Nip * 2, 64), 64, 0, st>>>(L, h.p, S);
        h.launches++;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // namespace gam
