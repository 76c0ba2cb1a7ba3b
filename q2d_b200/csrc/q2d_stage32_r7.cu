// Instantiations of the FP32-flux stage kernel (tiles 0-2: 32x10, 32x8, 64x4 with 256 threads;
// tiles 3-4: 32x16, 64x8 with 512 threads) for the run-time selected Riemann solvers 7-14, which
// take their flux in FP64 from the FP32 face states (see q2d_stage32.cuh).
#include "q2d_stage32.cuh"

namespace q2d {

cudaError_t launch_stage32_r7(const StageArgs& a, int tile, int grid, cudaStream_t s) {
    switch (tile) {
        case 1: return launch_stage32_t<7, 32, 8, 256, 4>(a, grid, s);
        case 2: return launch_stage32_t<7, 64, 4, 256, 4>(a, grid, s);
        case 3: return launch_stage32_t<7, 32, 16, 512, 2>(a, grid, s);
        case 4: return launch_stage32_t<7, 64, 8, 512, 2>(a, grid, s);
        default: return launch_stage32_t<7, 32, 10, 256, 4>(a, grid, s);
    }
}

int stage32_occupancy_r7(int tile) {
    switch (tile) {
        case 1: return stage32_occupancy_t<7, 32, 8, 256, 4>();
        case 2: return stage32_occupancy_t<7, 64, 4, 256, 4>();
        case 3: return stage32_occupancy_t<7, 32, 16, 512, 2>();
        case 4: return stage32_occupancy_t<7, 64, 8, 512, 2>();
        default: return stage32_occupancy_t<7, 32, 10, 256, 4>();
    }
}

}  // namespace q2d
