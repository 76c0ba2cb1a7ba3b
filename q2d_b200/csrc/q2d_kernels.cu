// q2d_kernels.cu — the Q2D explicit path's device code besides the stage kernels (sm_100a): the
// launch dispatch of the FP64 stage kernel (q2d_stage64.cuh; its MUSCL-SD form is instantiated
// in q2d_stage64_sd.cu), the initial time step, the state copy for the single-stage scheme, case
// resumption, implicit residual smoothing, the end-of-step finalisation and the state transfers.
// No spin-waits: cross-CTA ordering uses only atomic counters observed by the last CTA.
#include "q2d_stage64.cuh"

#include <cfloat>
#include <type_traits>

namespace q2d {


// Initial time step (Compute_dt before the first step, or after a state upload).
template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) dt_kernel(const StageArgs a) {
    __shared__ double red[(NT / 32) * 5];
    __shared__ double tile_part[5];
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    if (tid == 0 && blockIdx.x == 0 && a.launch_flag) *a.launch_flag = 1;
    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x) {
        const WorkItem w = a.items[it];
        const DBlock B = a.blocks[w.block];
        CaseState* cs = &a.cstate[w.case_id];
        // a.first != 0: only cases admitted since the last pass (others keep their time step)
        if (__ldcg(&cs->status) != kStatus_Running || (a.first && !__ldcg(&cs->dt_pending))) continue;
        const long long iter_next = __ldcg(&cs->iter) + 1;
        const int ndir = a.cases[w.case_id].ndir;
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        for (int cidx = tid; cidx < TX * TY; cidx += NT) {
            const int row = cidx / TX, col = cidx - row * TX;
            const int ii = w.i0 + col, jj = w.j0 + row;
            if (ii >= B.ni || jj >= B.nj) continue;
            const long long cg = (long long)jj * B.ni + ii;
            double P[4];
            for (int v = 0; v < 4; ++v) P[v] = a.Pin[B.oc + v * B.pc + cg];
            const long long gidx = B.og + (long long)(jj + 2) * (B.ni + 4) + (ii + 2);
            const double* scb = a.sc + 2 * B.oc;
            const double dtn = cell_dt(a, a.gas, P, scb, cg, B.pc, a.dl[gidx], a.dl[gidx + B.pg], ndir, iter_next);
            if (!a.time_accurate) a.sc[2 * B.oc + B.pc + cg] = dtn;
            acc[4] = fmin(acc[4], dtn);
        }
        block_reduce_store<NT>(acc, red, tile_part);
        if (tid == 0)
            for (int k = 0; k < 5; ++k) a.part[5 * (size_t)it + k] = tile_part[k];
        item_done<NT>(a, w.case_id, false, true, false, red, &s_flag);
    }
}

// Copies the interior state B -> A for the single-stage (euler) scheme.
__global__ void copy_state_kernel(const double* src, double* dst, long long n, int* launch_flag) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && launch_flag) *launch_flag = 1;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        dst[k] = src[k];
}

// Resumes cases paused on TODO = IO at the start of a q2d_gpu_step call.
__global__ void resume_kernel(CaseState* cs, int n, int* launch_flag) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && launch_flag) *launch_flag = 1;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        if (cs[c].status == kStatus_Paused) cs[c].status = kStatus_Running;
}

// Residual_Smoothing along one grid direction (Lib_IRS.f90:45-119) for every running case: two
// Jacobi sweeps R*(p) = (R(p) + beta (R*(p-1) + R*(p+1))) / (1 + 2 beta) over the block's
// interior, R* = R at the start, evaluated per cell from R at p-2 .. p+2 (each first-sweep
// value with the same operations as the sweep). The first ghost layer is R of the donor cell
// for a connection and of the boundary cell otherwise (Ghost_Residual_Extrapolation,
// :125-177), taken from Rin, the residual before this direction. A 1-D case (ndir = 1) is
// copied through in direction 2.
template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) irs_kernel(const StageArgs a, int dir, double beta,
                                                 const double* __restrict__ Rin, double* __restrict__ Rout) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && a.launch_flag) *a.launch_flag = 1;
    const double den = 1.0 + 2.0 * beta;
    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x) {
        const WorkItem w = a.items[it];
        if (__ldcg(&a.cstate[w.case_id].status) != kStatus_Running) continue;
        const DBlock B = a.blocks[w.block];
        const int ni = B.ni, nj = B.nj;
        const int ndir = a.cases[w.case_id].ndir;
        for (int k = threadIdx.x; k < TX * TY; k += NT) {
            const int row = k / TX, col = k - row * TX;
            const int ii = w.i0 + col, jj = w.j0 + row;
            if (ii >= ni || jj >= nj) continue;
            const long long cg = (long long)jj * ni + ii;
            if (dir == 2 && ndir == 1) {
                for (int v = 0; v < 4; ++v) Rout[B.oc + v * B.pc + cg] = Rin[B.oc + v * B.pc + cg];
                continue;
            }
            const int n = dir == 1 ? ni : nj, p = dir == 1 ? ii : jj;
            const long long stride = dir == 1 ? 1 : ni;
            // the records of the two ghost cells of this line
            const EdgeRec elo = a.edges[B.eo[dir == 1 ? 0 : 2] + (dir == 1 ? jj : ii)];
            const EdgeRec ehi = a.edges[B.eo[dir == 1 ? 1 : 3] + (dir == 1 ? jj : ii)];
            for (int v = 0; v < 4; ++v) {
                const double* line = Rin + B.oc + v * B.pc + cg - (long long)p * stride;   // position 0
                auto ghost = [&](const EdgeRec& e, int bpos) -> double {
                    if (e.type == 101) {
                        const DBlock D = a.blocks[e.bs];
                        return Rin[D.oc + v * D.pc + (long long)(e.js - 1) * D.ni + (e.is - 1)];
                    }
                    return line[(long long)bpos * stride];
                };
                auto R = [&](int q) -> double {
                    if (q < 0) return ghost(elo, 0);
                    if (q >= n) return ghost(ehi, n - 1);
                    return line[(long long)q * stride];
                };
                const double sm = p - 1 >= 0 ? (R(p - 1) + beta * (R(p - 2) + R(p))) / den : R(p - 1);
                const double sp = p + 1 < n ? (R(p + 1) + beta * (R(p) + R(p + 2))) / den : R(p + 1);
                Rout[B.oc + v * B.pc + cg] = (R(p) + beta * (sm + sp)) / den;
            }
        }
    }
}

cudaError_t launch_irs(const StageArgs& a, int tile, int grid, int dir, double beta, const double* Rin,
                       double* Rout, cudaStream_t s) {
    switch (tile) {
        case 1: irs_kernel<32, 8, 256><<<grid, 256, 0, s>>>(a, dir, beta, Rin, Rout); break;
        case 2: irs_kernel<64, 4, 256><<<grid, 256, 0, s>>>(a, dir, beta, Rin, Rout); break;
        case 3: irs_kernel<32, 16, 512><<<grid, 512, 0, s>>>(a, dir, beta, Rin, Rout); break;
        case 4: irs_kernel<64, 8, 512><<<grid, 512, 0, s>>>(a, dir, beta, Rin, Rout); break;
        default: irs_kernel<32, 10, 256><<<grid, 256, 0, s>>>(a, dir, beta, Rin, Rout); break;
    }
    return cudaGetLastError();
}

// End-of-step finalisation of every running case (residual norm, time step, TODO: the tail of
// Explicit_Step, Mod_Explicit.f90:120-170) from the item partials the last stage wrote, one CTA
// per case. Run after the last stage when that stage does not count items itself (a.fin_sep):
// the stage's CTAs then end each item without a fence or an atomic.
__global__ void __launch_bounds__(256) finalize_kernel(const StageArgs a) {
    __shared__ double red[(256 / 32) * 5];
    if (threadIdx.x == 0 && blockIdx.x == 0 && a.launch_flag) *a.launch_flag = 1;
    for (int c = blockIdx.x; c < a.n_cases; c += gridDim.x) {
        const DCase dc = a.cases[c];
        if (dc.item_end <= dc.item_begin || __ldcg(&a.cstate[c].status) != kStatus_Running) continue;
        finalize_case<256>(a, c, true, true, a.first != 0 || a.dt_first != 0, red);
        __syncthreads();
    }
}

cudaError_t launch_finalize(const StageArgs& a, cudaStream_t s) {
    const int grid = std::max(1, std::min(a.n_cases, 148 * 8));
    finalize_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// launch helpers
// ------------------------------------------------------------------------------------------
#define Q2D_TILE_SWITCH(TILE, CALL)                                          \
    switch (TILE) {                                                          \
        case 1: CALL(32, 8, 256); break;                                     \
        case 2: CALL(64, 4, 256); break;                                     \
        default: CALL(32, 10, 256); break;                                   \
    }

cudaError_t launch_stage(const StageArgs& a, int prec, int riem, int tile, int grid, cudaStream_t s) {
    if (a.sd || riem == 5 || riem == 6) return launch_stage_sd(a, prec, riem, tile, grid, s);   // the sensor runs
    cudaError_t e = cudaErrorInvalidValue;
#define Q2D_CALL(TX, TY, NT)                                                                   \
    if (prec == 0 && a.gas.htab) {   /* thermally perfect gas: HLLC, HLLE, LLF */              \
        if (riem == 1) e = launch_stage_t<0, 1, TX, TY, NT, false, true>(a, grid, s);                \
        else if (riem == 2) e = launch_stage_t<0, 2, TX, TY, NT, false, true>(a, grid, s);           \
        else if (riem == 0) e = launch_stage_t<0, 0, TX, TY, NT, false, true>(a, grid, s);           \
    } else if (prec == 0) {                                                                    \
        if (riem == 1) e = launch_stage_t<0, 1, TX, TY, NT, false>(a, grid, s);                      \
        else if (riem == 2) e = launch_stage_t<0, 2, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem == 3) e = launch_stage_t<0, 3, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem == 4) e = launch_stage_t<0, 4, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem >= 7) e = launch_stage_t<0, 7, TX, TY, NT, false>(a, grid, s);                 \
        else e = launch_stage_t<0, 0, TX, TY, NT, false>(a, grid, s);                                \
    } else {                                                                                   \
        if (riem == 1) e = launch_stage_t<1, 1, TX, TY, NT, false>(a, grid, s);                      \
        else if (riem == 2) e = launch_stage_t<1, 2, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem == 3) e = launch_stage_t<1, 3, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem == 4) e = launch_stage_t<1, 4, TX, TY, NT, false>(a, grid, s);                 \
        else if (riem >= 7) e = launch_stage_t<1, 7, TX, TY, NT, false>(a, grid, s);                 \
        else e = launch_stage_t<1, 0, TX, TY, NT, false>(a, grid, s);                                \
    }
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
    return e;
}

int stage_occupancy(int prec, int riem, int tile, int sd) {
    if (sd || riem == 5 || riem == 6) return stage_occupancy_sd(prec, riem, tile);
    int n = 0;
#define Q2D_CALL(TX, TY, NT)                                                                   \
    if (prec == 0) {                                                                           \
        if (riem == 1) n = occupancy_t<0, 1, TX, TY, NT, false>();                                   \
        else if (riem == 2) n = occupancy_t<0, 2, TX, TY, NT, false>();                 \
        else if (riem == 3) n = occupancy_t<0, 3, TX, TY, NT, false>();                 \
        else if (riem == 4) n = occupancy_t<0, 4, TX, TY, NT, false>();                              \
        else if (riem >= 7) n = occupancy_t<0, 7, TX, TY, NT, false>();                              \
        else n = occupancy_t<0, 0, TX, TY, NT, false>();                                             \
    } else {                                                                                   \
        if (riem == 1) n = occupancy_t<1, 1, TX, TY, NT, false>();                                   \
        else if (riem == 2) n = occupancy_t<1, 2, TX, TY, NT, false>();                 \
        else if (riem == 3) n = occupancy_t<1, 3, TX, TY, NT, false>();                 \
        else if (riem == 4) n = occupancy_t<1, 4, TX, TY, NT, false>();                              \
        else if (riem >= 7) n = occupancy_t<1, 7, TX, TY, NT, false>();                              \
        else n = occupancy_t<1, 0, TX, TY, NT, false>();                                             \
    }
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
    return n;
}

void tile_dims(int tile, int* tx, int* ty, int* nt) {
    switch (tile) {
        case 1: *tx = 32; *ty = 8; *nt = 256; break;
        case 2: *tx = 64; *ty = 4; *nt = 256; break;
        case 3: *tx = 32; *ty = 16; *nt = 512; break;
        case 4: *tx = 64; *ty = 8; *nt = 512; break;
        default: *tx = 32; *ty = 10; *nt = 256; break;
    }
}

cudaError_t launch_dt(const StageArgs& a, int tile, int grid, cudaStream_t s) {
    switch (tile) {
        case 1: dt_kernel<32, 8, 256><<<grid, 256, 0, s>>>(a); break;
        case 2: dt_kernel<64, 4, 256><<<grid, 256, 0, s>>>(a); break;
        case 3: dt_kernel<32, 16, 512><<<grid, 512, 0, s>>>(a); break;
        case 4: dt_kernel<64, 8, 512><<<grid, 512, 0, s>>>(a); break;
        default: dt_kernel<32, 10, 256><<<grid, 256, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

// State transfer between the caller's cell-interleaved rows (rho, u, v, p per cell, the interior
// rows of the reference's P array packed by a strided copy) and the block's 4 state planes.
__global__ void cells_to_planes_kernel(const double2* __restrict__ in, double* __restrict__ out, long long n,
                                       long long pc) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const double2 a = in[2 * c], b = in[2 * c + 1];
        out[c] = a.x; out[pc + c] = a.y; out[2 * pc + c] = b.x; out[3 * pc + c] = b.y;
    }
}

__global__ void planes_to_cells_kernel(const double* __restrict__ in, long long pc, double2* __restrict__ out,
                                       long long n) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        out[2 * c] = make_double2(in[c], in[pc + c]);
        out[2 * c + 1] = make_double2(in[2 * pc + c], in[3 * pc + c]);
    }
}

// Many-block forms: one launch per staging segment, blockIdx.y over the segment's blocks.
// Upload: the staging holds each caller's whole ghosted array P(4, -1:ni+2, -1:nj+2); only its
// interior goes to the state planes. Download: the interior rows of each block, packed.
__global__ void ghosted_to_planes_kernel(const XferDesc* __restrict__ d, int nd, const double* __restrict__ stage,
                                         double* __restrict__ pool) {
    for (int b = blockIdx.y; b < nd; b += gridDim.y) {
        const XferDesc x = d[b];
        const long long n = (long long)x.ni * x.nj;
        const double2* in = reinterpret_cast<const double2*>(stage + x.stage);
        double* out = pool + x.plane;
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
             c += (long long)gridDim.x * blockDim.x) {
            const long long j = c / x.ni, i = c - j * x.ni;
            const long long g = (j + 2) * (x.ni + 4) + (i + 2);
            const double2 a = in[2 * g], q = in[2 * g + 1];
            out[c] = a.x; out[x.pc + c] = a.y; out[2 * x.pc + c] = q.x; out[3 * x.pc + c] = q.y;
        }
    }
}

__global__ void planes_to_rows_kernel(const XferDesc* __restrict__ d, int nd, const double* __restrict__ pool,
                                      double* __restrict__ stage) {
    for (int b = blockIdx.y; b < nd; b += gridDim.y) {
        const XferDesc x = d[b];
        const long long n = (long long)x.ni * x.nj;
        const double* in = pool + x.plane;
        double2* out = reinterpret_cast<double2*>(stage + x.stage);
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
             c += (long long)gridDim.x * blockDim.x) {
            out[2 * c] = make_double2(in[c], in[x.pc + c]);
            out[2 * c + 1] = make_double2(in[2 * x.pc + c], in[3 * x.pc + c]);
        }
    }
}

cudaError_t launch_transfer_many(const XferDesc* d, int nd, long long max_cells, bool up, double* stage,
                                 double* pool, cudaStream_t s) {
    if (nd <= 0) return cudaSuccess;
    const dim3 grid((unsigned)std::max<long long>(1, std::min<long long>((max_cells + 255) / 256, 64)),
                    (unsigned)std::min(nd, 65535));
    if (up) ghosted_to_planes_kernel<<<grid, 256, 0, s>>>(d, nd, stage, pool);
    else planes_to_rows_kernel<<<grid, 256, 0, s>>>(d, nd, pool, stage);
    return cudaGetLastError();
}

cudaError_t launch_cells_to_planes(const double* in, double* out, long long n, long long pc, cudaStream_t s) {
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 8));
    cells_to_planes_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<const double2*>(in), out, n, pc);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_cells(const double* in, long long pc, double* out, long long n, cudaStream_t s) {
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 8));
    planes_to_cells_kernel<<<grid, 256, 0, s>>>(in, pc, reinterpret_cast<double2*>(out), n);
    return cudaGetLastError();
}

cudaError_t launch_copy(const double* src, double* dst, long long n, int* flag, cudaStream_t s) {
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    copy_state_kernel<<<grid > 0 ? grid : 1, 256, 0, s>>>(src, dst, n, flag);
    return cudaGetLastError();
}

cudaError_t launch_resume(CaseState* cs, int n, int* flag, cudaStream_t s) {
    resume_kernel<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, s>>>(cs, n, flag);
    return cudaGetLastError();
}

cudaError_t launch_stage32_r0(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r1(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r2(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r3(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r4(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r5(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r6(const StageArgs& a, int tile, int grid, cudaStream_t s);
cudaError_t launch_stage32_r7(const StageArgs& a, int tile, int grid, cudaStream_t s);
int stage32_occupancy_r0(int tile);
int stage32_occupancy_r1(int tile);
int stage32_occupancy_r2(int tile);
int stage32_occupancy_r3(int tile);
int stage32_occupancy_r4(int tile);
int stage32_occupancy_r5(int tile);
int stage32_occupancy_r6(int tile);
int stage32_occupancy_r7(int tile);

cudaError_t launch_stage32(const StageArgs& a, int riem, int tile, int grid, cudaStream_t s) {
    if (riem == 1) return launch_stage32_r1(a, tile, grid, s);
    if (riem == 2) return launch_stage32_r2(a, tile, grid, s);
    if (riem == 3) return launch_stage32_r3(a, tile, grid, s);
    if (riem == 4) return launch_stage32_r4(a, tile, grid, s);
    if (riem == 5) return launch_stage32_r5(a, tile, grid, s);
    if (riem == 6) return launch_stage32_r6(a, tile, grid, s);
    if (riem >= 7) return launch_stage32_r7(a, tile, grid, s);   // the run-time selected solvers
    return launch_stage32_r0(a, tile, grid, s);
}

int stage32_occupancy(int riem, int tile) {
    if (riem == 1) return stage32_occupancy_r1(tile);
    if (riem == 2) return stage32_occupancy_r2(tile);
    if (riem == 3) return stage32_occupancy_r3(tile);
    if (riem == 4) return stage32_occupancy_r4(tile);
    if (riem == 5) return stage32_occupancy_r5(tile);
    if (riem == 6) return stage32_occupancy_r6(tile);
    if (riem >= 7) return stage32_occupancy_r7(tile);
    return stage32_occupancy_r0(tile);
}

}  // namespace q2d
