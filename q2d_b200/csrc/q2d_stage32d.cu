// Dispatch of the difference-form FP32-flux stage kernel (q2d_stage32d.cuh) to its per-solver
// instantiation units q2d_stage32d_r{0,1,2}.cu (HLLC, HLLE, LLF).
#include "q2d_kernels.cuh"

namespace q2d {

cudaError_t launch_stage32d_r0(const StageArgs& a, int grid, cudaStream_t s);
cudaError_t launch_stage32d_r1(const StageArgs& a, int grid, cudaStream_t s);
cudaError_t launch_stage32d_r2(const StageArgs& a, int grid, cudaStream_t s);
int stage32d_occupancy_r0();
int stage32d_occupancy_r1();
int stage32d_occupancy_r2();

cudaError_t launch_stage32d(const StageArgs& a, int riem, int grid, cudaStream_t s) {
    if (riem == 1) return launch_stage32d_r1(a, grid, s);
    if (riem == 2) return launch_stage32d_r2(a, grid, s);
    return launch_stage32d_r0(a, grid, s);
}

int stage32d_occupancy(int riem) {
    if (riem == 1) return stage32d_occupancy_r1();
    if (riem == 2) return stage32d_occupancy_r2();
    return stage32d_occupancy_r0();
}

}  // namespace q2d
