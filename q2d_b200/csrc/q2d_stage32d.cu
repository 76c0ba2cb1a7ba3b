// Instantiations of the difference-form FP32-flux stage kernel (q2d_stage32d.cuh): HLLC, HLLE and
// LLF on 32x8 tiles of 256 threads, three CTAs per SM.
#include "q2d_stage32d.cuh"

namespace q2d {

cudaError_t launch_stage32d(const StageArgs& a, int riem, int grid, cudaStream_t s) {
    if (riem == 1) return launch_stage32d_t<1, 32, 8, 256, 3>(a, grid, s);
    if (riem == 2) return launch_stage32d_t<2, 32, 8, 256, 3>(a, grid, s);
    return launch_stage32d_t<0, 32, 8, 256, 3>(a, grid, s);
}

int stage32d_occupancy(int riem) {
    if (riem == 1) return stage32d_occupancy_t<1, 32, 8, 256, 3>();
    if (riem == 2) return stage32d_occupancy_t<2, 32, 8, 256, 3>();
    return stage32d_occupancy_t<0, 32, 8, 256, 3>();
}

}  // namespace q2d
