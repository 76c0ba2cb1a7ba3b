// q2d_kernels.cuh — launch interface of the device code (q2d_kernels.cu and the stage kernels)
// for the host runtime (q2d_api.cu).
#pragma once
#include "q2d_dev.cuh"

namespace q2d {

// Tile configurations (tile id -> TX x TY cells, NT threads): 0: 32 x 10, 256; 1: 32 x 8, 256;
// 2: 64 x 4, 256 (every stage kernel); 3: 32 x 16, 512; 4: 64 x 8, 512 (FP32-flux kernel only)
constexpr int kNumTiles = 5;
void tile_dims(int tile, int* tx, int* ty, int* nt);

// FP64 stage kernel (q2d_stage64.cuh); a.sd selects the MUSCL-SD instantiation (FP64 form only).
cudaError_t launch_stage(const StageArgs& a, int prec, int riem, int tile, int grid, cudaStream_t s);
int stage_occupancy(int prec, int riem, int tile, int sd);
cudaError_t launch_stage_sd(const StageArgs& a, int prec, int riem, int tile, int grid, cudaStream_t s);
int stage_occupancy_sd(int prec, int riem, int tile);
// FP32-flux stage kernel (q2d_stage32.cuh) on the same tiles and work items.
cudaError_t launch_stage32(const StageArgs& a, int riem, int tile, int grid, cudaStream_t s);
int stage32_occupancy(int riem, int tile);
// FP32-flux stage kernel in difference form (q2d_stage32d.cuh): HLLC / HLLE / LLF on 32 x 8 tiles
// (tile id 1) of 256 threads, without MUSCL-SD or implicit residual smoothing.
cudaError_t launch_stage32d(const StageArgs& a, int riem, int grid, cudaStream_t s);
int stage32d_occupancy(int riem);
cudaError_t launch_dt(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_copy(const double* src, double* dst, long long n, int* flag, cudaStream_t s);
// cell-interleaved (rho, u, v, p) <-> 4 planes of stride pc, n cells (state upload / download)
cudaError_t launch_cells_to_planes(const double* in, double* out, long long n, long long pc, cudaStream_t s);
// One block of a many-block transfer: its staging offset and state-plane offset (doubles).
struct XferDesc {
    long long stage, plane, pc;
    int ni, nj;
};
cudaError_t launch_transfer_many(const XferDesc* d, int nd, long long max_cells, bool up, double* stage,
                                 double* pool, cudaStream_t s);
cudaError_t launch_planes_to_cells(const double* in, long long pc, double* out, long long n, cudaStream_t s);
cudaError_t launch_resume(CaseState* cs, int n, int* flag, cudaStream_t s);
cudaError_t launch_finalize(const StageArgs& a, cudaStream_t s);
cudaError_t launch_irs(const StageArgs& a, int tile, int grid, int dir, double beta, const double* Rin,
                       double* Rout, cudaStream_t s);

}  // namespace q2d
