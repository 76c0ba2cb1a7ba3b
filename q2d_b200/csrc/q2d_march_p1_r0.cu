// Instantiations of the warp-marching stage kernel: precision form 1, Riemann solver 0,
// all seven limiters (compiled in separate units so they build in parallel).
#include "q2d_march.cuh"

namespace q2d {
cudaError_t launch_march_p1_r0(const StageArgs& a, int lim, int grid, cudaStream_t s) {
    return launch_march_t<1, 0>(a, lim, grid, s);
}
int march_occupancy_p1_r0(int lim) { return march_occupancy_t<1, 0>(lim); }
}  // namespace q2d
