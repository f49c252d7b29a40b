// Interface fluxes (stress.F90:204-429), FP32-flux path: reconstruction, limiter and kinetic fluxes in
// single precision from the float copies of the stencil inputs; the fluxes are stored area-scaled in
// double. This file is compiled with approximate single-precision division and square root (the FP32
// path's error budget is the 1e-5 L1 bound against the FP64 oracle); the tile kernel is in
// gam_flux_tile.cuh.
#include "gam_flux_tile.cuh"

namespace gam {

void flux_kernels_init_f32() {
    set_flux_smem<float, float, 0>(); set_flux_smem<float, float, 1>(); set_flux_smem<float, float, 2>();
    cudaFuncSetAttribute(k_flux_queue<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)flux_queue_smem<float>());
}

static FluxSrc<float> flux_src32(Handle& h) {
    const bool lfm = h.p.doLFMLim != 0;
    const F32Planes& f = h.f32;
    FluxSrc<float> in;
    for (int v = 0; v < 5; ++v) { in.W[v] = f.Wh[v]; in.Wl[v] = lfm ? f.Wn[v] : f.Wh[v]; }
    for (int x = 0; x < 3; ++x) { in.B[x] = f.hb[x]; in.Bl[x] = lfm ? f.nb[x] : f.hb[x]; }
    in.vol = f.volume;
    for (int d = 0; d < 3; ++d) {
        for (int q = 0; q < 9; ++q) in.Tf[d][q] = f.Tf[d][q];
        in.face[d] = f.face[d];
        in.bn[d] = f.hbA[d];
        for (int x = 0; x < 3; ++x) in.fcB0[d][x] = f.fcB0[d][x];
        in.b0[d] = f.b0n[d];
    }
    return in;
}

void enqueue_fluxes_f32(Handle& h, const StateP& nS, cudaStream_t st) {
    (void)nS;
    fluxes_all<float, float>(h, flux_src32(h), st);
}

void flux_jobs32(Handle& h, std::vector<FluxJob<float>>& jobs, long long& first) {
    FluxOut<float> F[3];
    for (int d = 0; d < 3; ++d) {
        for (int v = 0; v < 5; ++v) F[d].g[v] = h.f32.gflx[d][v];
        for (int x = 0; x < 3; ++x) F[d].m[x] = h.f32.mflx[d][x];
    }
    flux_jobs_of<float>(h, flux_src32(h), F, jobs, first);
}

void launch_flux_queue32(const FluxJob<float>* jobs, int njobs, long long ntiles, unsigned long long* counter,
                         int grid, cudaStream_t st) {
    k_flux_queue<float, float><<<grid, 256, flux_queue_smem<float>(), st>>>(jobs, njobs, ntiles, counter);
}

}  // namespace gam
