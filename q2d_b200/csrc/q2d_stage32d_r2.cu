// Instantiations of the difference-form FP32-flux stage kernel (q2d_stage32d.cuh) for Riemann
// solver 2 (LLF), every limiter, on 32x8 tiles of 256 threads, three CTAs per SM.
#include "q2d_stage32d.cuh"

namespace q2d {

cudaError_t launch_stage32d_r2(const StageArgs& a, int grid, cudaStream_t s) {
    return launch_stage32d_t<2, 32, 8, 256, 3>(a, grid, s);
}

int stage32d_occupancy_r2() { return stage32d_occupancy_t<2, 32, 8, 256, 3>(); }

}  // namespace q2d
