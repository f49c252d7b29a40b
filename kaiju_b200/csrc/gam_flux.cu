// Interface fluxes (stress.F90:204-429), FP64 path; the tile kernel is in gam_flux_tile.cuh.
#include "gam_flux_tile.cuh"

namespace gam {

void flux_kernels_init() {
    set_flux_smem<double, double, 0>(); set_flux_smem<double, double, 1>(); set_flux_smem<double, double, 2>();
    flux_kernels_init_f32();
}

void enqueue_fluxes(Handle& h, const StateP& nS, cudaStream_t st) {
    if (h.prec == PREC_FP32FLUX) {
        enqueue_fluxes_f32(h, nS, st);
        return;
    }
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
    fluxes_all<double, double>(h, in, st);
}

}  // namespace gam
