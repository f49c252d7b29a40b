// Interface fluxes (stress.F90:204-429), FP64 path; the tile kernel is in gam_flux_tile.cuh.
#include "gam_flux_tile.cuh"

namespace gam {

void flux_kernels_init() {
    set_flux_smem<double, double, 0>(); set_flux_smem<double, double, 1>(); set_flux_smem<double, double, 2>();
    cudaFuncSetAttribute(k_flux_queue<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)flux_queue_smem<double>());
    flux_kernels_init_f32();
}

static FluxSrc<double> flux_src64(Handle& h, const StateP& nS) {
    const bool lfm = h.p.doLFMLim != 0;
    FluxSrc<double> in;
    for (int v = 0; v < 5; ++v) { in.W[v] = h.Wh[v]; in.Wl[v] = lfm ? h.Wn[v] : h.Wh[v]; }
    for (int x = 0; x < 3; ++x) { in.B[x] = h.H.b[x]; in.Bl[x] = lfm ? nS.b[x] : h.H.b[x]; }
    in.vol = h.volume;
    for (int d = 0; d < 3; ++d) {
        for (int q = 0; q < 9; ++q) in.Tf[d][q] = h.Tf[d][q];
        in.face[d] = h.face[d];
        in.bn[d] = h.H.mf[d];
        for (int x = 0; x < 3; ++x) in.fcB0[d][x] = h.fcB0[d][x];
        in.b0[d] = h.bFlux0[d];
    }
    return in;
}

void flux_jobs64(Handle& h, int cur, std::vector<FluxJob<double>>& jobs, long long& first) {
    FluxOut<double> F[3];
    for (int d = 0; d < 3; ++d) {
        for (int v = 0; v < 5; ++v) F[d].g[v] = h.gflx[d][v];
        for (int x = 0; x < 3; ++x) F[d].m[x] = h.mflx[d][x];
    }
    flux_jobs_of<double>(h, flux_src64(h, h.S[cur]), F, jobs, first);
}

void launch_flux_queue64(const FluxJob<double>* jobs, int njobs, long long ntiles, unsigned long long* counter,
                         int grid, cudaStream_t st) {
    k_flux_queue<double, double><<<grid, 256, flux_queue_smem<double>(), st>>>(jobs, njobs, ntiles, counter);
}

void enqueue_fluxes(Handle& h, const StateP& nS, cudaStream_t st) {
    if (h.prec == PREC_FP32FLUX) {
        enqueue_fluxes_f32(h, nS, st);
        return;
    }
    fluxes_all<double, double>(h, flux_src64(h, nS), st);
}

}  // namespace gam
