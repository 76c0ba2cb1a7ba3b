// Shock-sensor instantiations of the FP64 stage kernel (q2d_stage64.cuh): the sensor of
// Lib_Shock_Detector.f90:14-38 runs, for MUSCL-SD (it scales the face slopes) and for the
// sensor-driven Riemann solvers HLLC+ / HLLE++ (they blend by it). FP64 form only; the FP32-flux
// form runs on the FP32-flux kernel.
#include "q2d_stage64.cuh"

namespace q2d {

cudaError_t launch_stage_sd(const StageArgs& a, int prec, int riem, int tile, int grid, cudaStream_t s) {
    if (prec != 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaErrorInvalidValue;
#define Q2D_CALL(TX, TY, NT)                                                  \
    switch (riem) {                                                           \
        case 1: e = launch_stage_t<0, 1, TX, TY, NT, true>(a, grid, s); break; \
        case 2: e = launch_stage_t<0, 2, TX, TY, NT, true>(a, grid, s); break; \
        case 3: e = launch_stage_t<0, 3, TX, TY, NT, true>(a, grid, s); break; \
        case 4: e = launch_stage_t<0, 4, TX, TY, NT, true>(a, grid, s); break; \
        case 5: e = launch_stage_t<0, 5, TX, TY, NT, true>(a, grid, s); break; \
        case 6: e = launch_stage_t<0, 6, TX, TY, NT, true>(a, grid, s); break; \
        case 0: e = launch_stage_t<0, 0, TX, TY, NT, true>(a, grid, s); break; \
        default: e = launch_stage_t<0, 7, TX, TY, NT, true>(a, grid, s); break; \
    }
    switch (tile) {
        case 1: Q2D_CALL(32, 8, 256); break;
        case 2: Q2D_CALL(64, 4, 256); break;
        default: Q2D_CALL(32, 10, 256); break;
    }
#undef Q2D_CALL
    return e;
}

int stage_occupancy_sd(int prec, int riem, int tile) {
    if (prec != 0) return 0;
    int n = 0;
#define Q2D_CALL(TX, TY, NT)                                        \
    switch (riem) {                                                 \
        case 1: n = occupancy_t<0, 1, TX, TY, NT, true>(); break;   \
        case 2: n = occupancy_t<0, 2, TX, TY, NT, true>(); break;   \
        case 3: n = occupancy_t<0, 3, TX, TY, NT, true>(); break;   \
        case 4: n = occupancy_t<0, 4, TX, TY, NT, true>(); break;   \
        case 5: n = occupancy_t<0, 5, TX, TY, NT, true>(); break;   \
        case 6: n = occupancy_t<0, 6, TX, TY, NT, true>(); break;   \
        case 0: n = occupancy_t<0, 0, TX, TY, NT, true>(); break;   \
        default: n = occupancy_t<0, 7, TX, TY, NT, true>(); break;  \
    }
    switch (tile) {
        case 1: Q2D_CALL(32, 8, 256); break;
        case 2: Q2D_CALL(64, 4, 256); break;
        default: Q2D_CALL(32, 10, 256); break;
    }
#undef Q2D_CALL
    return n;
}

}  // namespace q2d
