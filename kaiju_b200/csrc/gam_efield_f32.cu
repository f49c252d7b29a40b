// Edge EMFs of the FP32-flux path (fields.F90:70-232): the tile kernel in single precision from the
// float copies. Compiled with approximate single-precision division and square root; the tile kernel
// is in gam_efield_tile.cuh.
#include "gam_efield_tile.cuh"

namespace gam {

void efield_kernels_init_f32() {
    set_edge_smem<float, float, 0>(); set_edge_smem<float, float, 1>(); set_edge_smem<float, float, 2>();
}

void launch_edge_dir_f32(Handle& h, const EdgeSrc<float>& in, int eD, const Reg& re, cudaStream_t st) {
    launch_edge_dir<float, float>(h, in, eD, re, st);
}

}  // namespace gam
