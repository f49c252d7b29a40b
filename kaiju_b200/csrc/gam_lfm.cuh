// Index maps across the axis of an LFM-type grid (ringutils.F90:482-660), in device index space (i,j,k
// counted from the first ghost). Every relation of the reference is a difference of indices, so it reads
// the same here with js/je/ks/ke of the device layout; WrapK's "kp > Np" becomes "kp > ke".
#pragma once
#include "gam_common.cuh"

namespace gam {

__host__ __device__ __forceinline__ int lfmWrapK(const Lay& L, int k) {   // WrapK, ringutils.F90:652-660
    int kp = k + L.Nkp / 2;
    if (kp > L.ke()) kp = kp - L.Nkp;
    return kp;
}
// lfmIJKcc (ringutils.F90:482-514): conjugate cell across the axis
__host__ __device__ __forceinline__ void lfmCC(const Lay& L, bool doS, bool doE, int j, int k, int& jp, int& kp) {
    int Np = L.Nkp;
    if (k < L.ks()) kp = k + Np;
    else if (k > L.ke()) kp = k - Np;
    else kp = k;
    jp = j;
    if (doS && j < L.js()) { jp = L.js() + (L.js() - j) - 1; kp = lfmWrapK(L, kp); }
    if (doE && j > L.je()) { jp = L.je() - (j - L.je()) + 1; kp = lfmWrapK(L, kp); }
}
// lfmIJKfc (ringutils.F90:517-575): conjugate d-face
__host__ __device__ __forceinline__ void lfmFC(const Lay& L, bool doS, bool doE, int d, int j, int k, int& jp, int& kp) {
    if (d == 0) { lfmCC(L, doS, doE, j, k, jp, kp); return; }
    int Np = L.Nkp;
    kp = k;
    if (k < L.ks()) kp = k + Np;
    if (d == 1 && k > L.ke()) kp = k - Np;
    if (d == 2 && k > L.ke() + 1) kp = k - Np;
    jp = j;
    if (d == 1) {
        if (doS && j < L.js()) { jp = L.js() + (L.js() - j); kp = lfmWrapK(L, k); }
        if (doE && j > L.je() + 1) { jp = L.je() + 1 - (j - L.je()) + 1; kp = lfmWrapK(L, k); }
    } else {
        if (doS && j < L.js()) { jp = L.js() + (L.js() - j) - 1; kp = lfmWrapK(L, k); }
        if (doE && j > L.je()) { jp = L.je() - (j - L.je()) + 1; kp = lfmWrapK(L, k); }
    }
}

}  // namespace gam
