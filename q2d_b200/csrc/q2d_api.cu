// q2d_api.cu — host runtime behind include/q2d_gpu.h: contexts, device pools and their
// allocators, work lists, CUDA-graph execution of N explicit steps, state transfer, the
// schedule autotuner and the serving (continuous batching) entry points.
//
// Replaces, for one grid level: Assign_Setup (procedure-pointer binding -> kernel selection),
// Allocate_Block / Setup_Metrics (per-case device regions filled when the case is
// materialised), and the Explicit_Step loop (a captured graph of n_rk fused stage kernels per
// step; Mod_Explicit.f90:10-174). The reference's single domain becomes a "case"; a context
// holds many cases, each with its own dtglobal, time, iteration count, residual and TODO state.
//
// Batch contexts (q2d_gpu_create ... commit) size their pools exactly for the cases added
// before commit. Serving contexts (q2d_serve_create) size the pools from a byte budget and
// admit / retire cases between steps; admission does its host work (validation, metrics)
// at once and defers every device write to the next step call, after the work in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/q2d_gpu.h"
#include "q2d_kernels.cuh"
#include "q2d_setup.h"

using namespace q2d;

namespace {

// Device images of one block, built on the host when its case is prepared and copied to the
// block's regions when the case is uploaded.
// Host images of a block's device planes, in one buffer: a slice of the context's pinned
// staging area when it has room (serving), else a heap buffer of its own.
struct Staged {
    double *pa = nullptr, *sc = nullptr, *dl = nullptr, *fi = nullptr, *fj = nullptr;
    float *dl32 = nullptr, *fi4 = nullptr, *fj4 = nullptr;   // FP32 geometry of the FP32-flux form
    size_t n_pa = 0, n_sc = 0, n_dl = 0, n_fi = 0, n_fj = 0, n_dl32 = 0, n_fi4 = 0, n_fj4 = 0;
    std::unique_ptr<char[]> heap;
};

struct HBlock {
    int ni = 0, nj = 0, case_id = -1, local_b = 0;
    std::vector<double> nodes, area;
    std::vector<double> prim;      // 4 planes, interior (until the case is prepared)
    // a serving admission's caller arrays, read in place while the admission prepares the case
    // (the nodes, the cross-section and the ghosted state P): no host copies
    const double* nodes_ext = nullptr;
    const double* area_ext = nullptr;
    const double* P_ext = nullptr;
    std::vector<EdgeRec> edge[4];  // records of faces 1..4 (param: index into the case's params)
    Staged staged;
    DBlock d{};
    bool alive = false;            // holds device regions
    const double* nd() const { return nodes_ext ? nodes_ext : nodes.data(); }
    const double* ar() const { return area_ext ? area_ext : (area.empty() ? nullptr : area.data()); }
};

struct HCase {
    std::vector<int> blocks;       // global block ids
    std::vector<q2d_bc_rec> bc;
    std::vector<BCParam> params;
    double time0 = 0.0;
    int iter_end = 0;              // the case's own fixed end (q2d_gpu_set_case_end), 0 for none
    bool used = false;             // slot holds a case
    bool prepared = false;         // regions reserved, device images staged
    bool resident = false;         // device images and run state uploaded
    bool images_sent = false;      // device images queued on the copy stream at admission
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        n = count;
        return cudaMalloc(&p, sizeof(T) * (count ? count : 1));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// First-fit allocator over an index space [0, cap) of a pool (offsets in elements).
struct Arena {
    long long cap = 0;
    std::map<long long, long long> free;   // offset -> length, coalesced
    void init(long long c) {
        cap = c;
        free.clear();
        if (c > 0) free[0] = c;
    }
    bool alloc(long long n, long long* off) {
        for (auto it = free.begin(); it != free.end(); ++it)
            if (it->second >= n) {
                *off = it->first;
                const long long rest = it->second - n, o = it->first + n;
                free.erase(it);
                if (rest > 0) free[o] = rest;
                return true;
            }
        return false;
    }
    void release(long long off, long long n) {
        if (n <= 0) return;
        auto it = free.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free.erase(nx);
        }
        if (it != free.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free.erase(it);
            }
        }
    }
    long long free_total() const {
        long long t = 0;
        for (auto& kv : free) t += kv.second;
        return t;
    }
};

long long round32(long long n) { return (n + 31) / 32 * 32; }

// Element counts of one block's regions: 4-plane cell space, 2-plane ghost frame, 3-plane
// i-face and j-face spaces. Planes are padded to 32 elements (256 B).
struct Extents {
    long long pc, pg, pfi, pfj;
};
Extents block_extents(int ni, int nj) {
    return {round32((long long)ni * nj), round32((long long)(ni + 4) * (nj + 4)),
            round32((long long)(ni + 1) * nj), round32((long long)ni * (nj + 1))};
}

}  // namespace

struct q2d_ctx {
    q2d_options opt{};
    Gas gas{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // serving: admissions' image uploads during the steps
    bool copies_pending = false;
    std::vector<HBlock> blocks;
    std::vector<HCase> cases;     // slots
    bool serving = false;
    bool committed = false;
    bool dt_valid = false;        // every running case has its time step
    bool dt_new = false;          // some case was uploaded after the last time-step pass
    bool dirty = false;           // uploads, slot resets or list rebuild pending
    std::vector<int> reset_slots; // retired slots whose device run state still has to be reset
    int tile = 0;
    int kernel = 0;       // 0: FP64 tile stage kernel, 2: FP32-flux tile kernel, 3: FP32-flux
                          // tile kernel in difference form
    int grid = 0;
    // device pools and their allocators
    DevBuf<double> PA, PB, PC, SC, DL, FI, FJ, PART;
    DevBuf<double> RA, RB;          // scaled residuals for implicit residual smoothing (irs_beta > 0)
    DevBuf<double> XFER;            // staging rows of one block's state for upload / download
    DevBuf<XferDesc> XDESC;         // block descriptors of a many-block transfer segment
    DevBuf<float> DL32, FI4, FJ4;   // FP32 geometry (FP32-flux form only): same regions as DL/FI/FJ
    bool f4 = true;                 // FP32 face records kept (off in serving contexts that run only
                                    // the difference-form kernel, which reads the FP64 faces)
    Arena ac, ag, afi, afj;
    DevBuf<DBlock> dblocks;
    DevBuf<DCase> dcases;
    DevBuf<CaseState> cstate;
    DevBuf<WorkItem> items;
    DevBuf<EdgeRec> edges;
    DevBuf<BCParam> bcp;
    DevBuf<int> flag;
    DevBuf<double> TAB;             // thermally perfect gas table: h(T) then cp(T), ntab knots each
    CaseState* h_state = nullptr;   // pinned mirror
    CaseState* h_fresh = nullptr;   // pinned starting run states of the cases being uploaded
    char* pin = nullptr;            // pinned staging area of admissions (serving contexts)
    char* h_lists = nullptr;        // pinned staging of the device work lists
    size_t h_lists_cap = 0;
    // host geometry of the case being prepared, kept between cases: its pages stay mapped, so
    // the next admission's metrics do not fault them in again
    std::vector<HostGeom> geo_cache;
    size_t pin_cap = 0, pin_used = 0;
    int n_items = 0;
    std::map<int, cudaGraphExec_t> graphs;
    std::map<int, int> graph_kernels;
    long long launches = 0;
    std::string last_error;
};

namespace {

int fail(q2d_ctx* c, int code, const std::string& msg) {
    if (c) c->last_error = msg;
    return code;
}

int cuda_fail(q2d_ctx* c, cudaError_t e, const char* where) {
    if (c) c->last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return Q2D_ERR_CUDA;
}

#define CK(call)                                                 \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

StageArgs base_args(q2d_ctx* ctx) {
    StageArgs a{};
    a.blocks = ctx->dblocks.p;
    a.cases = ctx->dcases.p;
    a.cstate = ctx->cstate.p;
    a.items = ctx->items.p;
    a.n_items = ctx->n_items;
    a.n_cases = (int)ctx->cases.size();
    a.part_stride = 1;
    a.sc = ctx->SC.p;
    a.dl = ctx->DL.p;
    a.dl32 = ctx->DL32.p;
    a.fi4 = reinterpret_cast<const float4*>(ctx->FI4.p);
    a.fj4 = reinterpret_cast<const float4*>(ctx->FJ4.p);
    a.fi = ctx->FI.p;
    a.fj = ctx->FJ.p;
    a.edges = ctx->edges.p;
    a.bcp = ctx->bcp.p;
    a.part = ctx->PART.p;
    a.gas = ctx->gas;
    a.cfl = ctx->opt.cfl;
    a.n_rk = ctx->opt.n_rk;
    a.limiter = ctx->opt.limiter;
    a.sd = ctx->opt.shock_detector;
    a.source = ctx->opt.source;
    a.time_accurate = ctx->opt.time_accurate;
    a.rampa = ctx->opt.rampa_iter;
    a.res_diter = ctx->opt.res_diter;
    a.sol_diter = ctx->opt.sol_diter;
    a.res_relative = ctx->opt.res_relative;
    a.itermax = ctx->opt.itermax;
    a.res_threshold = ctx->opt.res_threshold;
    a.time_threshold = ctx->opt.time_threshold;
    a.sol_dtime = ctx->opt.sol_dtime;
    a.launch_flag = ctx->flag.p;
    return a;
}

// Local time stepping with the FP32-flux kernel computes each cell's time step in the first
// stage of the step, from the state the step starts from (as Explicit_Step calls Compute_dt,
// Mod_Explicit.f90:44-53); the other kernels, and global time stepping (which needs the minimum
// over the case before any cell updates), compute it in the last stage of the previous step and
// in the time-step passes of ensure_dt.
bool dt_in_first_stage(const q2d_ctx* ctx) { return ctx->kernel >= 2 && !ctx->opt.time_accurate; }

// Item partials per work item: one set per warp for the FP32-flux kernels (256 threads on tiles
// 0-2, 512 on tiles 3-4, as launch_stage32 / launch_stage32d instantiate them), which end their
// items without a CTA-wide reduction and leave the case finalisation to finalize_kernel; one
// otherwise.
int part_stride(const q2d_ctx* ctx) {
    int TX, TY, NT;
    tile_dims(ctx->tile, &TX, &TY, &NT);
    return ctx->kernel >= 2 ? NT / 32 : 1;
}

// RKcoeff (Lib_RK.f90:8-11)
double rk_coeff(int n_rk, int irk) {
    static const double C[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.5, 0.0}, {1.0, 0.25, 2.0 / 3.0}};
    return C[n_rk - 1][irk - 1];
}

// Enqueues one explicit step. Buffer plan: A holds the state between steps; stage 1 reads A
// (stencil and U^n) and writes B; stage 2 reads B and writes C (n_rk = 3) or A; the last
// stage of RK3 reads C and updates A in place (each cell reads only its own U^n from A).
int enqueue_step(q2d_ctx* ctx, cudaStream_t s, int* nk) {
    const int n_rk = ctx->opt.n_rk;
    if (ctx->n_items == 0) return Q2D_OK;
    for (int irk = 1; irk <= n_rk; ++irk) {
        StageArgs a = base_args(ctx);
        a.irk = irk;
        a.first = irk == 1;
        a.last = irk == n_rk;
        a.dt_first = dt_in_first_stage(ctx) ? 1 : 0;
        a.part_stride = part_stride(ctx);
        a.fin_sep = ctx->kernel >= 2 ? 1 : 0;
        a.rk_c = rk_coeff(n_rk, irk);
        a.PO = ctx->PA.p;
        if (n_rk == 1) { a.Pin = ctx->PA.p; a.Pout = ctx->PB.p; }
        else if (n_rk == 2) {
            if (irk == 1) { a.Pin = ctx->PA.p; a.Pout = ctx->PB.p; }
            else { a.Pin = ctx->PB.p; a.Pout = ctx->PA.p; }
        } else {
            if (irk == 1) { a.Pin = ctx->PA.p; a.Pout = ctx->PB.p; }
            else if (irk == 2) { a.Pin = ctx->PB.p; a.Pout = ctx->PC.p; }
            else { a.Pin = ctx->PC.p; a.Pout = ctx->PA.p; }
        }
        auto stage = [&](const StageArgs& x) -> int {
            if (ctx->kernel == 3)
                CK(launch_stage32d(x, ctx->opt.riemann, ctx->grid, s));
            else if (ctx->kernel == 2)
                CK(launch_stage32(x, ctx->opt.riemann, ctx->tile, ctx->grid, s));
            else
                CK(launch_stage(x, ctx->opt.precision, ctx->opt.riemann, ctx->tile, ctx->grid, s));
            ++*nk;
            return Q2D_OK;
        };
        if (ctx->opt.irs_beta > 0.0) {
            // Newstate_Conservative with IRS (Lib_Newstate.f90:36-66): the stage's scaled residual
            // (stage prologue and time steps as usual), smoothing along i then j, then the update
            // (item counting, residual partials and case finalisation as the stage's last pass)
            StageArgs r1 = a;
            r1.irs_mode = 1; r1.Rout = ctx->RA.p; r1.last = 0;
            if (int e = stage(r1)) return e;
            CK(launch_irs(a, ctx->tile, ctx->grid, 1, ctx->opt.irs_beta, ctx->RA.p, ctx->RB.p, s));
            CK(launch_irs(a, ctx->tile, ctx->grid, 2, ctx->opt.irs_beta, ctx->RB.p, ctx->RA.p, s));
            *nk += 2;
            a.irs_mode = 2; a.Rin = ctx->RA.p; a.first = 0;
        }
        if (int e = stage(a)) return e;
        if (a.last && a.fin_sep) {
            CK(launch_finalize(a, s));
            ++*nk;
        }
    }
    if (n_rk == 1) {
        CK(launch_copy(ctx->PB.p, ctx->PA.p, ctx->ac.cap, ctx->flag.p, s));
        ++*nk;
    }
    return Q2D_OK;
}

// Compute_dt for the cases that need it: every running case after a state upload, only the
// newly uploaded ones after an admission (the others keep the time step their last stage
// computed, so a case's trajectory does not depend on when other cases arrive).
// With time steps computed in the first stage no pass is needed, and the per-cell time steps
// left by a step are those it used, not the next step's: dt_valid is cleared so that a switch to
// another kernel (or `force`, the autotuner's baseline) runs a full pass first.
int ensure_dt(q2d_ctx* ctx, bool force = false) {
    if (!force && dt_in_first_stage(ctx)) {
        ctx->dt_valid = false;
        ctx->dt_new = false;
        return Q2D_OK;
    }
    if (ctx->dt_valid && !ctx->dt_new) return Q2D_OK;
    if (ctx->n_items > 0) {
        StageArgs a = base_args(ctx);
        a.Pin = ctx->PA.p;
        a.first = ctx->dt_valid ? 1 : 0;   // pending-only pass
        CK(launch_dt(a, ctx->tile, ctx->grid, ctx->stream));
        ctx->launches += 1;
    }
    ctx->dt_valid = true;
    ctx->dt_new = false;
    return Q2D_OK;
}

void drop_graphs(q2d_ctx* ctx) {
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
    ctx->graphs.clear();
    ctx->graph_kernels.clear();
}

int get_graph(q2d_ctx* ctx, int nsteps, cudaGraphExec_t* out) {
    auto it = ctx->graphs.find(nsteps);
    if (it != ctx->graphs.end()) { *out = it->second; return Q2D_OK; }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int nk = 0, st = Q2D_OK;
    for (int s = 0; s < nsteps && st == Q2D_OK; ++s) st = enqueue_step(ctx, ctx->stream, &nk);
    if (st == Q2D_OK) {
        cudaError_t e = cudaMemcpyAsync(ctx->h_state, ctx->cstate.p, sizeof(CaseState) * ctx->cases.size(),
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "cudaMemcpyAsync(state)");
    }
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st != Q2D_OK) { if (e == cudaSuccess) cudaGraphDestroy(g); return st; }
    CK(e);
    cudaGraphExec_t ge;
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    ctx->graphs[nsteps] = ge;
    ctx->graph_kernels[nsteps] = nk;
    *out = ge;
    return Q2D_OK;
}

void fill_info(const CaseState& s, q2d_step_info* o) {
    o->dtglobal = s.dtglobal;
    o->time = s.time;
    o->iter = s.iter;
    for (int k = 0; k < 4; ++k) o->residual[k] = s.res[k];
    o->residual0 = s.res0;
    o->todo = s.todo;
    o->err = s.err == 4 ? Q2D_ERR_NONPHYSICAL : (s.err == 5 ? Q2D_ERR_NAN : s.err);
    o->err_b = s.err_b; o->err_i = s.err_i; o->err_j = s.err_j; o->err_stage = s.err_stage;
}

bool rec_less(const q2d_bc_rec& a, const q2d_bc_rec& b) {
    return a.b != b.b ? a.b < b.b : a.f < b.f;
}

CaseState fresh_state(double time0, int iter_end) {
    CaseState s;
    std::memset(&s, 0, sizeof(s));
    s.iter_end = iter_end;
    s.res0 = -1.0;
    s.todo = Q2D_TODO_CONTINUE;
    s.status = kStatus_Running;
    s.time = time0;
    s.time_from_call = time0;
    s.dt_pending = 1;
    return s;
}

CaseState empty_state() {
    CaseState s;
    std::memset(&s, 0, sizeof(s));
    s.res0 = -1.0;
    s.todo = Q2D_TODO_END;
    s.status = kStatus_Done;
    return s;
}

// Grows a device buffer to at least n elements (contents are not kept).
template <typename T>
cudaError_t ensure_cap(DevBuf<T>& b, size_t n) {
    if (b.p && b.n >= n) return cudaSuccess;
    b.release();
    return b.alloc(std::max<size_t>(n, 1) + n / 4);
}

// Validates the boundary records of a case and derives per-block edge records and the
// parameters of its inflow / outflow faces.
int build_case_edges(q2d_ctx* ctx, int c) {
    HCase& cs = ctx->cases[c];
    cs.params.clear();
    for (int gb : cs.blocks) {
        HBlock& B = ctx->blocks[gb];
        const int len[4] = {B.nj, B.nj, B.ni, B.ni};
        for (int f = 0; f < 4; ++f) B.edge[f].assign(len[f], EdgeRec{-1, 0, 0, 0, 0, -1});
    }
    for (const q2d_bc_rec& r : cs.bc) {
        HBlock& B = ctx->blocks[cs.blocks[r.b - 1]];
        const bool pos_ok = (r.f == 1 && r.i == 1) || (r.f == 2 && r.i == B.ni) ||
                            (r.f == 3 && r.j == 1) || (r.f == 4 && r.j == B.nj);
        if (!pos_ok) return fail(ctx, Q2D_ERR_BADARG, "boundary record not on its face");
        const int k = (r.f <= 2) ? r.j - 1 : r.i - 1;
        EdgeRec& er = B.edge[r.f - 1][k];
        if (er.type != -1) return fail(ctx, Q2D_ERR_BADARG, "duplicate boundary record");
        // A periodic seam (201) is a connection on the device: Ghost_Connection and
        // BC_Connection_Eul serve both (Lib_Ghost.f90:63, Mod_BC_Fluxes.f90:99-102); only its
        // ghost metrics differ (ghost_metrics)
        er.type = r.type == 201 ? 101 : r.type;
        if (r.type == 101 || r.type == 201) {
            const HBlock& D = ctx->blocks[cs.blocks[r.bs - 1]];
            const int gi = r.fs == 1 ? 1 : (r.fs == 2 ? -1 : 0);
            const int gj = r.fs == 3 ? 1 : (r.fs == 4 ? -1 : 0);
            for (int g = 0; g < 2; ++g) {
                const int si = r.is + gi * g, sj = r.js + gj * g;
                if (si < 1 || si > D.ni || sj < 1 || sj > D.nj)
                    return fail(ctx, Q2D_ERR_BADARG, "connection donor cell outside its block");
            }
            er.bs = cs.blocks[r.bs - 1];
            er.is = r.is; er.js = r.js; er.fs = r.fs;
        }
        if (r.type == 401 || r.type == 405 || r.type == 406) {
            BCParam p{};
            p.T0 = r.T0; p.p0 = r.p0; p.pamb = r.pamb; p.mach = r.mach;
            p.alpha = r.alpha; p.rel_fac = r.rel_fac;
            face_tangent(r, B.ni, B.nd(), &p.t0, &p.t1);
            er.param = (int)cs.params.size();
            cs.params.push_back(p);
        }
    }
    for (int gb : cs.blocks) {
        const HBlock& B = ctx->blocks[gb];
        for (int f = 0; f < 4; ++f)
            for (const EdgeRec& e : B.edge[f])
                if (e.type == -1)
                    return fail(ctx, Q2D_ERR_BADARG, "boundary cell without a record (block " +
                                std::to_string(B.local_b) + ", face " + std::to_string(f + 1) + ")");
    }
    return Q2D_OK;
}

void release_regions(q2d_ctx* ctx, HBlock& b) {
    if (!b.alive) return;
    ctx->ac.release(b.d.oc, 4 * b.d.pc);
    ctx->ag.release(b.d.og, 2 * b.d.pg);
    ctx->afi.release(b.d.ofi, 3 * b.d.pfi);
    ctx->afj.release(b.d.ofj, 3 * b.d.pfj);
    b.alive = false;
}

// Reserves the device regions of every block of a case (all or nothing).
bool reserve_regions(q2d_ctx* ctx, int c) {
    HCase& cs = ctx->cases[c];
    for (size_t k = 0; k < cs.blocks.size(); ++k) {
        HBlock& b = ctx->blocks[cs.blocks[k]];
        DBlock& d = b.d;
        const Extents x = block_extents(b.ni, b.nj);
        d = DBlock{};
        d.ni = b.ni; d.nj = b.nj; d.case_id = c; d.local_b = b.local_b;
        d.pc = x.pc; d.pg = x.pg; d.pfi = x.pfi; d.pfj = x.pfj;
        long long oc, og, ofi, ofj;
        bool okc = ctx->ac.alloc(4 * x.pc, &oc);
        bool okg = okc && ctx->ag.alloc(2 * x.pg, &og);
        bool oki = okg && ctx->afi.alloc(3 * x.pfi, &ofi);
        bool okj = oki && ctx->afj.alloc(3 * x.pfj, &ofj);
        if (!okj) {
            if (oki) ctx->afi.release(ofi, 3 * x.pfi);
            if (okg) ctx->ag.release(og, 2 * x.pg);
            if (okc) ctx->ac.release(oc, 4 * x.pc);
            for (size_t q = 0; q < k; ++q) release_regions(ctx, ctx->blocks[cs.blocks[q]]);
            return false;
        }
        d.oc = oc; d.og = og; d.ofi = ofi; d.ofj = ofj;
        b.alive = true;
    }
    return true;
}

// Host half of materialising a case: edge records, device regions, metrics (Setup_Metrics
// restated on the host) and the device images of every block, staged for upload.
// Carves the images of one block out of the pinned staging area (bump allocation, reset once
// the uploads that read it have completed) or, when it is full, out of a heap buffer.
void stage_alloc(q2d_ctx* ctx, Staged& S, const DBlock& d, bool fp32) {
    auto al = [](size_t bytes) { return (bytes + 255) & ~size_t(255); };
    S.n_pa = 4 * (size_t)d.pc; S.n_sc = 8 * (size_t)d.pc; S.n_dl = 2 * (size_t)d.pg;
    S.n_fi = 3 * (size_t)d.pfi; S.n_fj = 3 * (size_t)d.pfj;
    S.n_dl32 = fp32 ? 2 * (size_t)d.pg : 0; S.n_fi4 = fp32 && ctx->f4 ? 4 * (size_t)d.pfi : 0;
    S.n_fj4 = fp32 ? 4 * (size_t)d.pfj : 0;
    const size_t sizes[8] = {al(8 * S.n_pa), al(8 * S.n_sc), al(8 * S.n_dl), al(8 * S.n_fi), al(8 * S.n_fj),
                             al(4 * S.n_dl32), al(4 * S.n_fi4), al(4 * S.n_fj4)};
    size_t total = 0;
    for (size_t s : sizes) total += s;
    char* base;
    if (ctx->pin && ctx->pin_used + total <= ctx->pin_cap) {
        base = ctx->pin + ctx->pin_used;
        ctx->pin_used += total;
    } else {
        S.heap.reset(new char[total]);
        base = S.heap.get();
    }
    char* p = base;
    S.pa = reinterpret_cast<double*>(p); p += sizes[0];
    S.sc = reinterpret_cast<double*>(p); p += sizes[1];
    S.dl = reinterpret_cast<double*>(p); p += sizes[2];
    S.fi = reinterpret_cast<double*>(p); p += sizes[3];
    S.fj = reinterpret_cast<double*>(p); p += sizes[4];
    S.dl32 = fp32 ? reinterpret_cast<float*>(p) : nullptr; p += sizes[5];
    S.fi4 = S.n_fi4 ? reinterpret_cast<float*>(p) : nullptr; p += sizes[6];
    S.fj4 = S.n_fj4 ? reinterpret_cast<float*>(p) : nullptr;
}

int prepare_case(q2d_ctx* ctx, int c) {
    HCase& cs = ctx->cases[c];
    if (int e = build_case_edges(ctx, c)) return e;
    std::vector<HostGeom>& geo = ctx->geo_cache;   // every array is rewritten by setup_block
    if (geo.size() < cs.blocks.size()) geo.resize(cs.blocks.size());
    // regions and staging images first: the face geometry is written straight into its images
    if (!reserve_regions(ctx, c)) return fail(ctx, Q2D_ERR_CAPACITY, "device memory budget exhausted");
    const bool fp32 = ctx->opt.precision == Q2D_PREC_FP32_FLUX;
    for (size_t lb = 0; lb < cs.blocks.size(); ++lb) {
        HBlock& b = ctx->blocks[cs.blocks[lb]];
        Staged& S = b.staged;
        stage_alloc(ctx, S, b.d, fp32);
        FaceOut fo;
        fo.fi = S.fi; fo.fj = S.fj; fo.pfi = b.d.pfi; fo.pfj = b.d.pfj; fo.fi4 = S.fi4; fo.fj4 = S.fj4;
        int e = setup_block(b.ni, b.nj, b.nd(), b.ar(), ctx->opt.source, geo[lb], &fo);
        if (e) return fail(ctx, e, "degenerate cell in block " + std::to_string(b.local_b));
    }
    for (const q2d_bc_rec& r : cs.bc) {
        HBlock& B = ctx->blocks[cs.blocks[r.b - 1]];
        const HBlock* D = (r.type == 101 || r.type == 201) ? &ctx->blocks[cs.blocks[r.bs - 1]] : nullptr;
        int e = ghost_metrics(r, B.ni, B.nj, B.nd(), geo[r.b - 1], D ? D->ni : 0, D ? D->nj : 0,
                              D ? D->nd() : nullptr);
        if (e) return fail(ctx, e, "ghost metrics failed for a boundary record");
    }
    for (size_t lb = 0; lb < cs.blocks.size(); ++lb) {
        HBlock& b = ctx->blocks[cs.blocks[lb]];
        const DBlock& d = b.d;
        const HostGeom& G = geo[lb];
        const long long n = (long long)b.ni * b.nj;
        const long long ngh = (long long)(b.ni + 4) * (b.nj + 4), nfi = (long long)(b.ni + 1) * b.nj,
                        nfj = (long long)b.ni * (b.nj + 1);
        const long long pc = d.pc, pg = d.pg, pfi = d.pfi, pfj = d.pfj;
        Staged& S = b.staged;
        // images of the device planes (the faces written by setup_block), filled in parallel;
        // padding and the dt plane are zero
        parallel_zero(S.sc, (size_t)pc, 2 * (size_t)pc);   // dt
        for (int v = 0; v < 8; ++v) parallel_zero(S.sc, v * (size_t)pc + n, (v + 1) * (size_t)pc);
        for (int v = 0; v < 4; ++v) parallel_zero(S.pa, v * (size_t)pc + n, (v + 1) * (size_t)pc);
        for (int v = 0; v < 2; ++v) parallel_zero(S.dl, v * (size_t)pg + ngh, (v + 1) * (size_t)pg);
        for (int q = 0; q < 3; ++q) parallel_zero(S.fi, q * (size_t)pfi + nfi, (q + 1) * (size_t)pfi);
        for (int q = 0; q < 3; ++q) parallel_zero(S.fj, q * (size_t)pfj + nfj, (q + 1) * (size_t)pfj);
        if (fp32) {
            parallel_zero(S.dl32, 2 * (size_t)ngh, 2 * (size_t)pg);
            if (S.fi4) {
                parallel_zero(S.fi4, 4 * (size_t)nfi, 4 * (size_t)pfi);
                parallel_zero(S.fj4, 4 * (size_t)nfj, 4 * (size_t)pfj);
            }
        }
        parallel_rows(b.nj, 160L * b.ni, [&](long long r0, long long r1) {
            for (int j = (int)r0; j < (int)r1; ++j)
                for (int i = 0; i < b.ni; ++i) {
                    const long long k = (long long)j * b.ni + i;
                    double v[4];
                    versors(G, i, j, v);
                    S.sc[k] = G.sur[G.g(i, j)];
                    S.sc[2 * pc + k] = v[0];
                    S.sc[3 * pc + k] = v[1];
                    S.sc[4 * pc + k] = v[2];
                    S.sc[5 * pc + k] = v[3];
                    S.sc[6 * pc + k] = G.src0[k];
                    S.sc[7 * pc + k] = G.src1[k];
                    if (b.P_ext) {   // the caller's P(4, -1:ni+2, -1:nj+2)
                        const double* src = &b.P_ext[4 * ((size_t)(i + 2) + (size_t)(b.ni + 4) * (j + 2))];
                        for (int q = 0; q < 4; ++q) S.pa[q * pc + k] = src[q];
                    } else {
                        for (int q = 0; q < 4; ++q) S.pa[q * pc + k] = b.prim[(size_t)q * n + k];
                    }
                }
        });
        parallel_rows(ngh, 32, [&](long long k0, long long k1) {
            for (long long k = k0; k < k1; ++k) {
                S.dl[k] = G.dl[2 * k];
                S.dl[pg + k] = G.dl[2 * k + 1];
                if (fp32) {
                    S.dl32[2 * k] = (float)G.dl[2 * k];   // interleaved: (dl(1), dl(2)) per frame cell
                    S.dl32[2 * k + 1] = (float)G.dl[2 * k + 1];
                }
            }
        });
        b.prim.clear();
        b.prim.shrink_to_fit();
    }
    cs.prepared = true;
    return Q2D_OK;
}

// Device half: copies the staged images into the case's regions (send_images; a serving
// admission queues them on the copy stream right away, while the steps in flight run: the
// regions belong to no listed case) and starts its run state (upload_case, called only while
// no work is in flight on the context's stream). Heap images wait for their copies; the caller
// synchronises both streams before the pinned staging area or the pinned run states are reused.
int send_images(q2d_ctx* ctx, int c, cudaStream_t s) {
    HCase& cs = ctx->cases[c];
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    for (int gb : cs.blocks) {
        HBlock& b = ctx->blocks[gb];
        const DBlock& d = b.d;
        Staged& S = b.staged;
        CK(cudaMemcpyAsync(ctx->PA.p + d.oc, S.pa, sizeof(double) * S.n_pa, h2d, s));
        CK(cudaMemcpyAsync(ctx->SC.p + 2 * d.oc, S.sc, sizeof(double) * S.n_sc, h2d, s));
        CK(cudaMemcpyAsync(ctx->DL.p + d.og, S.dl, sizeof(double) * S.n_dl, h2d, s));
        CK(cudaMemcpyAsync(ctx->FI.p + d.ofi, S.fi, sizeof(double) * S.n_fi, h2d, s));
        CK(cudaMemcpyAsync(ctx->FJ.p + d.ofj, S.fj, sizeof(double) * S.n_fj, h2d, s));
        if (ctx->DL32.p) {   // face offsets are multiples of 32, so float index 2*off is 16-byte aligned
            CK(cudaMemcpyAsync(ctx->DL32.p + d.og, S.dl32, sizeof(float) * S.n_dl32, h2d, s));
            if (ctx->FI4.p && S.fi4) {
                CK(cudaMemcpyAsync(ctx->FI4.p + 2 * d.ofi, S.fi4, sizeof(float) * S.n_fi4, h2d, s));
                CK(cudaMemcpyAsync(ctx->FJ4.p + 2 * d.ofj, S.fj4, sizeof(float) * S.n_fj4, h2d, s));
            }
        }
        if (S.heap) CK(cudaStreamSynchronize(s));   // a heap image is freed right away
        S = Staged{};
    }
    cs.images_sent = true;
    return Q2D_OK;
}

int upload_case(q2d_ctx* ctx, int c) {
    HCase& cs = ctx->cases[c];
    cudaStream_t s = ctx->stream;
    if (!cs.images_sent)
        if (int e = send_images(ctx, c, s)) return e;
    ctx->h_fresh[c] = fresh_state(cs.time0, cs.iter_end);   // one pinned entry per slot
    CK(cudaMemcpyAsync(ctx->cstate.p + c, ctx->h_fresh + c, sizeof(CaseState), cudaMemcpyHostToDevice, s));
    cs.resident = true;
    ctx->dt_new = true;
    return Q2D_OK;
}

// Device descriptor arrays (blocks, edge records, BC parameters, work items, per-case item
// ranges) of the resident cases, and the persistent grid size. Called only while no work is
// in flight on the context's stream.
int rebuild_device_lists(q2d_ctx* ctx) {
    int TX, TY, NT;
    tile_dims(ctx->tile, &TX, &TY, &NT);
    std::vector<DBlock> db(ctx->blocks.size());
    std::vector<EdgeRec> edges;
    std::vector<BCParam> params;
    std::vector<WorkItem> items;
    std::vector<DCase> dcases(ctx->cases.size(), DCase{0, 0, 2, 0});
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        HCase& cs = ctx->cases[c];
        dcases[c].item_begin = (int)items.size();
        if (cs.used && cs.resident) {
            const int pbase = (int)params.size();
            params.insert(params.end(), cs.params.begin(), cs.params.end());
            for (int gb : cs.blocks) {
                HBlock& B = ctx->blocks[gb];
                for (int f = 0; f < 4; ++f) {
                    B.d.eo[f] = (int)edges.size();
                    for (EdgeRec e : B.edge[f]) {
                        if (e.param >= 0) e.param += pbase;
                        edges.push_back(e);
                    }
                }
                for (int j0 = 0; j0 < B.nj; j0 += TY)
                    for (int i0 = 0; i0 < B.ni; i0 += TX) items.push_back(WorkItem{gb, i0, j0, (int)c, 0, 0});
            }
            dcases[c].ndir = ctx->blocks[cs.blocks[0]].nj == 1 ? 1 : 2;
        }
        dcases[c].item_end = (int)items.size();
    }
    for (size_t k = 0; k < ctx->blocks.size(); ++k) db[k] = ctx->blocks[k].d;
    CK(ensure_cap(ctx->dblocks, db.size()));
    CK(ensure_cap(ctx->edges, edges.size()));
    CK(ensure_cap(ctx->bcp, params.size()));
    CK(ensure_cap(ctx->items, items.size()));
    const size_t npart = 5 * (size_t)part_stride(ctx) * items.size();
    if (!ctx->PART.p || ctx->PART.n < npart) {
        CK(ensure_cap(ctx->PART, npart));
        CK(cudaMemsetAsync(ctx->PART.p, 0, sizeof(double) * ctx->PART.n, ctx->stream));
    }
    {   // one pinned staging buffer, copies queued on the context's stream (no work is in flight,
        // and the next rebuild comes after a synchronisation of the stream)
        auto al = [](size_t n) { return (n + 255) & ~size_t(255); };
        const size_t nb[5] = {sizeof(DBlock) * db.size(), sizeof(EdgeRec) * edges.size(),
                              sizeof(BCParam) * params.size(), sizeof(WorkItem) * items.size(),
                              sizeof(DCase) * dcases.size()};
        size_t need = 0;
        for (size_t n : nb) need += al(n);
        if (need > ctx->h_lists_cap) {
            if (ctx->h_lists) CK(cudaFreeHost(ctx->h_lists));
            ctx->h_lists = nullptr;
            ctx->h_lists_cap = 0;
            CK(cudaMallocHost(&ctx->h_lists, need + need / 2));
            ctx->h_lists_cap = need + need / 2;
        }
        const void* src[5] = {db.data(), edges.data(), params.data(), items.data(), dcases.data()};
        void* dst[5] = {ctx->dblocks.p, ctx->edges.p, ctx->bcp.p, ctx->items.p, ctx->dcases.p};
        size_t off = 0;
        for (int k = 0; k < 5; ++k) {
            if (nb[k] == 0) continue;
            std::memcpy(ctx->h_lists + off, src[k], nb[k]);
            CK(cudaMemcpyAsync(dst[k], ctx->h_lists + off, nb[k], cudaMemcpyHostToDevice, ctx->stream));
            off += al(nb[k]);
        }
    }
    ctx->n_items = (int)items.size();
    {
        const int occ = std::max(1, ctx->kernel == 3   ? stage32d_occupancy(ctx->opt.riemann)
                                    : ctx->kernel == 2 ? stage32_occupancy(ctx->opt.riemann, ctx->tile)
                                                       : stage_occupancy(ctx->opt.precision, ctx->opt.riemann,
                                                                         ctx->tile, ctx->opt.shock_detector));
        ctx->grid = (int)std::min<long long>((long long)items.size(), (long long)occ * ctx->num_sms);
    }
    if (ctx->grid < 1) ctx->grid = 1;
    drop_graphs(ctx);
    return Q2D_OK;
}

// Applies what admissions and retirements left for the device, after the work in flight.
int apply_pending(q2d_ctx* ctx) {
    if (!ctx->dirty) return Q2D_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->copies_pending) {   // the admissions' image copies (done during the steps, as a rule)
        CK(cudaStreamSynchronize(ctx->copy_stream));
        ctx->copies_pending = false;
    }
    for (int c : ctx->reset_slots) {
        if (ctx->cases[c].used) continue;   // slot taken again: the upload below starts it
        const CaseState s = empty_state();
        CK(cudaMemcpy(ctx->cstate.p + c, &s, sizeof(CaseState), cudaMemcpyHostToDevice));
    }
    ctx->reset_slots.clear();
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        HCase& cs = ctx->cases[c];
        if (cs.used && cs.prepared && !cs.resident)
            if (int e = upload_case(ctx, (int)c)) return e;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->pin_used = 0;   // every staged image has been uploaded
    if (int e = rebuild_device_lists(ctx)) return e;
    ctx->dirty = false;
    return Q2D_OK;
}

int allocate_pools(q2d_ctx* ctx, long long ec, long long eg, long long efi, long long efj, int ncases) {
    CK(ctx->PA.alloc(ec)); CK(ctx->PB.alloc(ec)); CK(ctx->PC.alloc(ec));
    if (ctx->opt.irs_beta > 0.0) { CK(ctx->RA.alloc(ec)); CK(ctx->RB.alloc(ec)); }
    CK(ctx->SC.alloc(2 * ec)); CK(ctx->DL.alloc(eg)); CK(ctx->FI.alloc(efi)); CK(ctx->FJ.alloc(efj));
    if (ctx->opt.precision == Q2D_PREC_FP32_FLUX) {
        CK(ctx->DL32.alloc(eg));
        if (ctx->f4) { CK(ctx->FI4.alloc(2 * efi)); CK(ctx->FJ4.alloc(2 * efj)); }
    }
    CK(cudaMemset(ctx->PB.p, 0, sizeof(double) * (ec ? ec : 1)));
    CK(cudaMemset(ctx->PC.p, 0, sizeof(double) * (ec ? ec : 1)));
    ctx->ac.init(ec); ctx->ag.init(eg); ctx->afi.init(efi); ctx->afj.init(efj);
    CK(ctx->dcases.alloc(ncases));
    CK(ctx->cstate.alloc(ncases));
    CK(ctx->flag.alloc(1));
    CK(cudaMallocHost(&ctx->h_state, sizeof(CaseState) * ncases));
    CK(cudaMallocHost(&ctx->h_fresh, sizeof(CaseState) * ncases));
    std::vector<CaseState> st(ncases, empty_state());   // empty slots read as finished
    CK(cudaMemcpy(ctx->cstate.p, st.data(), sizeof(CaseState) * ncases, cudaMemcpyHostToDevice));
    return Q2D_OK;
}

int commit(q2d_ctx* ctx) {
    if (ctx->committed) return Q2D_OK;
    if (ctx->cases.empty()) return fail(ctx, Q2D_ERR_BADARG, "no case");
    long long ec = 0, eg = 0, efi = 0, efj = 0;
    for (const HBlock& b : ctx->blocks) {
        const Extents x = block_extents(b.ni, b.nj);
        ec += 4 * x.pc; eg += 2 * x.pg; efi += 3 * x.pfi; efj += 3 * x.pfj;
    }
    for (size_t c = 0; c < ctx->cases.size(); ++c)
        if (ctx->cases[c].blocks.empty()) return fail(ctx, Q2D_ERR_BADARG, "case without blocks");
    if (int e = allocate_pools(ctx, ec, eg, efi, efj, (int)ctx->cases.size())) return e;
    // prepared and uploaded case by case: host memory stays at one case's images
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        ctx->cases[c].used = true;
        if (int e = prepare_case(ctx, (int)c)) return e;
        if (int e = upload_case(ctx, (int)c)) return e;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    if (int e = rebuild_device_lists(ctx)) return e;
    ctx->committed = true;
    ctx->dt_valid = false;
    return Q2D_OK;
}

// Committed / pending state brought up to date before device work.
int ready(q2d_ctx* ctx) {
    if (!ctx->serving) return commit(ctx);
    return apply_pending(ctx);
}

// ---- autotuner ------------------------------------------------------------------------------
// Times every schedule (stage kernel and tile shape) for `steps`
// explicit steps on the context's own workload and keeps the fastest. The state, the scalar
// planes (time steps) and the case states are saved before and restored after each candidate,
// so tuning leaves the results unchanged.
struct Schedule { int kernel, tile; };
// Candidate schedules, indexed like the autotuner's result: FP64 tile stage kernel on tiles
// 32x10, 32x8, 64x4; FP32-flux tile kernel on tiles 32x10, 32x8, 64x4 (256 threads) and 32x16,
// 64x8 (512 threads); FP32-flux tile kernel in difference form on 32x8 (FP32-flux form only).
const Schedule kSchedules[] = {{0, 0}, {0, 1}, {0, 2}, {2, 0}, {2, 1}, {2, 2}, {2, 3}, {2, 4}, {3, 1}};
constexpr int kNumSchedules = (int)(sizeof(kSchedules) / sizeof(kSchedules[0]));

bool schedule_allowed(const q2d_ctx* ctx, int k) {
    const bool sensor = ctx->opt.shock_detector || ctx->opt.riemann == Q2D_RIEMANN_HLLCP ||
                        ctx->opt.riemann == Q2D_RIEMANN_HLLEPP;
    if (kSchedules[k].kernel == 0 && sensor &&
        ctx->opt.precision != Q2D_PREC_FP64)
        return false;   // the shock sensor on the tile kernel: FP64 form only (FP32-flux: the FP32-flux kernel)
    if (kSchedules[k].kernel == 2 && !ctx->f4) return false;   // no FP32 face records
    if (kSchedules[k].kernel == 3)   // difference form: HLLC / HLLE / LLF, no sensor, no smoothing
        return ctx->opt.precision == Q2D_PREC_FP32_FLUX && ctx->opt.riemann <= 2 && !sensor &&
               !(ctx->opt.irs_beta > 0.0);
    return kSchedules[k].kernel != 2 || ctx->opt.precision == Q2D_PREC_FP32_FLUX;
}

// The FP32-flux form of HLLC / HLLE / LLF without MUSCL-SD or smoothing is the difference-form
// kernel: its error against FP64 stays at ~1e-9 relative L1 over thousands of steps where the
// tile kernels that round whole fluxes to FP32 reach ~1e-6. The autotuner does not trade that
// form for another one; q2d_gpu_set_schedule can still pin the others.
bool difference_form(const q2d_ctx* ctx) {
    for (int k = 0; k < kNumSchedules; ++k)
        if (kSchedules[k].kernel == 3 && schedule_allowed(ctx, k)) return true;
    return false;
}

int autotune(q2d_ctx* ctx, int steps, int* best_out, float* ms_out) {
    const Schedule* cands = kSchedules;
    const int ncand = kNumSchedules;
    const size_t nst = ctx->cases.size();
    const long long ec = ctx->ac.cap;
    DevBuf<double> saveP, saveSC;
    DevBuf<CaseState> saveCS;
    CK(saveP.alloc(ec));
    CK(saveSC.alloc(2 * ec));
    CK(saveCS.alloc(nst));
    if (int e = ensure_dt(ctx, true)) return e;   // every candidate starts from valid time steps
    CK(cudaMemcpyAsync(saveP.p, ctx->PA.p, sizeof(double) * ec, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(saveSC.p, ctx->SC.p, sizeof(double) * 2 * ec, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(saveCS.p, ctx->cstate.p, sizeof(CaseState) * nst, cudaMemcpyDeviceToDevice, ctx->stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int besti = 0;
    const bool df = difference_form(ctx);
    for (int k = 0; k < ncand; ++k) {
        if (!schedule_allowed(ctx, k) || (df && cands[k].kernel != 3)) continue;
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->kernel = cands[k].kernel;
        ctx->tile = cands[k].tile;
        if (int e = rebuild_device_lists(ctx)) return e;
        int nk = 0;
        if (int e = enqueue_step(ctx, ctx->stream, &nk)) return e;   // warm-up step
        CK(cudaEventRecord(e0, ctx->stream));
        for (int sidx = 0; sidx < steps; ++sidx)
            if (int e = enqueue_step(ctx, ctx->stream, &nk)) return e;
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        ctx->launches += nk;
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) { best = ms; besti = k; }
        CK(cudaMemcpyAsync(ctx->PA.p, saveP.p, sizeof(double) * ec, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->SC.p, saveSC.p, sizeof(double) * 2 * ec, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->cstate.p, saveCS.p, sizeof(CaseState) * nst, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->kernel = cands[besti].kernel;
    ctx->tile = cands[besti].tile;
    if (int e = rebuild_device_lists(ctx)) return e;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    saveP.release(); saveSC.release(); saveCS.release();
    if (best_out) *best_out = besti;
    if (ms_out) *ms_out = best / (float)steps;
    return Q2D_OK;
}

int check_options(const q2d_options* opt) {
    if (opt->n_rk < 1 || opt->n_rk > 3 || opt->limiter < 0 || opt->limiter > 6 || opt->riemann < 0 ||
        opt->riemann > Q2D_RIEMANN_AUSMP_UP2 || opt->source < 0 || opt->source > 2 || opt->precision < 0 ||
        opt->precision > 1 || !(opt->gas_gamma > 1.0) || !(opt->gas_R > 0.0) || opt->res_diter < 1 ||
        opt->sol_diter < 1 || !(opt->cfl > 0.0) || !(opt->irs_beta >= 0.0) || !(opt->irs_beta < 1e300) ||
        opt->shock_detector < 0 || opt->shock_detector > 1 || !(opt->riemann_minf >= 0.0) ||
        ((opt->riemann == Q2D_RIEMANN_AUSMP_UP || opt->riemann == Q2D_RIEMANN_AUSMP_UP2) && !(opt->riemann_minf > 0.0)))
        return Q2D_ERR_BADARG;   // AUSM+-up needs Minf (Assign_Setup.f90:108-112)
    return Q2D_OK;
}

// Input checks of Read_BC (Lib_IO.f90) and of the boundary kinds on this path.
int check_recs(q2d_ctx* ctx, const HCase& cs, const std::vector<q2d_bc_rec>& v) {
    for (const q2d_bc_rec& r : v) {
        if (r.b < 1 || r.b > (int)cs.blocks.size() || r.f < 1 || r.f > 4)
            return fail(ctx, Q2D_ERR_BADARG, "set_bcs: block or face out of range");
        const HBlock& B = ctx->blocks[cs.blocks[r.b - 1]];
        if (r.i < 1 || r.i > B.ni || r.j < 1 || r.j > B.nj)
            return fail(ctx, Q2D_ERR_BADARG, "set_bcs: cell out of range");
        switch (r.type) {
            case 400:
                if ((r.f <= 2 && B.ni < 3) || (r.f >= 3 && B.nj < 3))
                    return fail(ctx, Q2D_ERR_BADARG, "set_bcs: extrapolation needs 3 cells");
                break;
            case 0: case 300: case 401: case 405: case 406:
                if (r.f <= 2 && B.ni < 2) return fail(ctx, Q2D_ERR_BADARG, "set_bcs: block too thin");
                break;
            case 101: case 201: {   // connection / translational periodic seam (Mod_BC_Fluxes.f90:99-102)
                if (r.bs < 1 || r.bs > (int)cs.blocks.size() || r.fs < 1 || r.fs > 4)
                    return fail(ctx, Q2D_ERR_BADARG, "set_bcs: bad connection donor");
                const HBlock& D = ctx->blocks[cs.blocks[r.bs - 1]];
                if (r.is < 1 || r.is > D.ni || r.js < 1 || r.js > D.nj)
                    return fail(ctx, Q2D_ERR_BADARG, "set_bcs: connection donor cell out of range");
                break;
            }
            default:
                return fail(ctx, Q2D_ERR_UNSUPPORTED, "set_bcs: BC type " + std::to_string(r.type) +
                                                          " is not on the built path");
        }
    }
    return Q2D_OK;
}

// Fortran P(1:4, -1:ni+2, -1:nj+2) (ghost frame of 2) -> 4 interior planes
void fortran_to_planes(int ni, int nj, const double* P, std::vector<double>& planes) {
    const long long n = (long long)ni * nj;
    planes.resize(4 * n);
    double* out = planes.data();
    parallel_rows(nj, 64L * ni, [=](long long r0, long long r1) {
        for (long long j = r0; j < r1; ++j)
            for (int i = 0; i < ni; ++i) {
                const double* src = &P[4 * ((size_t)(i + 2) + (size_t)(ni + 4) * (j + 2))];
                for (int v = 0; v < 4; ++v) out[v * n + (size_t)j * ni + i] = src[v];
            }
    });
}

q2d_ctx* new_ctx(const q2d_options* opt) {
    q2d_ctx* ctx = new (std::nothrow) q2d_ctx();
    if (!ctx) return nullptr;
    ctx->opt = *opt;
    ctx->gas.R = opt->gas_R;
    ctx->gas.gamma = opt->gas_gamma;
    ctx->gas.gm1 = opt->gas_gamma - 1.0;
    ctx->gas.cp = opt->gas_gamma * opt->gas_R / (opt->gas_gamma - 1.0);
    ctx->gas.cv = opt->gas_R / (opt->gas_gamma - 1.0);
    ctx->gas.gfac = opt->gas_gamma / (opt->gas_gamma - 1.0);
    ctx->gas.igm1 = 1.0 / (opt->gas_gamma - 1.0);
    ctx->gas.rkind = opt->riemann;
    ctx->gas.minf = opt->riemann_minf;
    ctx->gas.iR = 1.0 / opt->gas_R;
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return nullptr;
    }
    if (opt->precision == Q2D_PREC_FP32_FLUX) {   // default schedules 0 / 8 (difference form) / 3
        const bool df = opt->riemann <= 2 && !opt->shock_detector && !(opt->irs_beta > 0.0);
        ctx->kernel = df ? 3 : 2;
        ctx->tile = df ? 1 : 0;
    }
    return ctx;
}

void free_case_blocks(q2d_ctx* ctx, HCase& cs) {
    for (int gb : cs.blocks) {
        release_regions(ctx, ctx->blocks[gb]);
        ctx->blocks[gb] = HBlock{};
    }
    cs = HCase{};
}

}  // namespace

extern "C" {

void q2d_options_default(q2d_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->limiter = Q2D_LIM_IORD;
    o->riemann = Q2D_RIEMANN_HLLC;
    o->n_rk = 1;
    o->time_accurate = 0;
    o->source = Q2D_SRC_NONE;
    o->precision = Q2D_PREC_FP64;
    o->rampa_iter = 0;
    o->res_diter = 1;
    o->sol_diter = 1000000000;
    o->res_relative = 0;
    o->itermax = 1000000000LL;
    o->cfl = 0.5;
    o->res_threshold = 1e-10;
    o->time_threshold = 1e30;
    o->sol_dtime = 1e30;
    o->gas_R = 287.0;
    o->gas_gamma = 1.4;
}

int q2d_gpu_create(q2d_ctx** out, const q2d_options* opt) {
    if (!out || !opt) return Q2D_ERR_BADARG;
    *out = nullptr;
    if (check_options(opt)) return Q2D_ERR_BADARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return Q2D_ERR_CUDA;
    q2d_ctx* ctx = new_ctx(opt);
    if (!ctx) return Q2D_ERR_OOM;
    *out = ctx;
    return Q2D_OK;
}

int q2d_gpu_add_case(q2d_ctx* ctx, int* case_id) {
    if (!ctx || ctx->committed || ctx->serving) return fail(ctx, Q2D_ERR_BADARG, "add_case after commit");
    ctx->cases.emplace_back();
    if (case_id) *case_id = (int)ctx->cases.size() - 1;
    return Q2D_OK;
}

int q2d_gpu_set_case_time(q2d_ctx* ctx, int case_id, double time) {
    if (!ctx || ctx->committed || ctx->serving || case_id < 0 || case_id >= (int)ctx->cases.size() ||
        !std::isfinite(time))
        return fail(ctx, Q2D_ERR_BADARG, "set_case_time: bad argument or after commit");
    ctx->cases[case_id].time0 = time;
    return Q2D_OK;
}

int q2d_gpu_set_thermo_table(q2d_ctx* ctx, int ntab, const double* h_tab, const double* cp_tab) {
    if (!ctx || ctx->committed || ctx->serving || ntab < 2 || ntab > (1 << 20) || !h_tab || !cp_tab)
        return fail(ctx, Q2D_ERR_BADARG, "set_thermo_table: bad argument or after commit");
    if (ctx->opt.precision != Q2D_PREC_FP64 || ctx->opt.riemann > Q2D_RIEMANN_LLF || ctx->opt.shock_detector)
        return fail(ctx, Q2D_ERR_BADARG, "set_thermo_table: plain FP64 form with HLLC, HLLE or LLF only");
    const double R = ctx->gas.R;
    for (int k = 0; k < ntab; ++k)
        if (!std::isfinite(h_tab[k]) || !(cp_tab[k] > R))
            return fail(ctx, Q2D_ERR_BADARG, "set_thermo_table: h not finite or cp <= R");
    for (int k = 0; k + 1 < ntab; ++k)
        if (!(h_tab[k + 1] - h_tab[k] > R))
            return fail(ctx, Q2D_ERR_BADARG, "set_thermo_table: internal energy not increasing");
    ctx->TAB.release();
    CK(ctx->TAB.alloc(2 * (size_t)ntab));
    CK(cudaMemcpy(ctx->TAB.p, h_tab, sizeof(double) * ntab, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->TAB.p + ntab, cp_tab, sizeof(double) * ntab, cudaMemcpyHostToDevice));
    ctx->gas.htab = ctx->TAB.p;
    ctx->gas.cptab = ctx->TAB.p + ntab;
    ctx->gas.ntab = ntab;
    return Q2D_OK;
}

int q2d_gpu_set_case_end(q2d_ctx* ctx, int case_id, long long iter_end) {
    if (!ctx || case_id < 0 || case_id >= (int)ctx->cases.size() ||
        (ctx->serving && !ctx->cases[case_id].used) || iter_end < 0 || iter_end > 2000000000LL)
        return fail(ctx, Q2D_ERR_BADARG, "set_case_end: bad argument");
    HCase& cs = ctx->cases[case_id];
    cs.iter_end = (int)iter_end;
    if (cs.resident) {   // stream-ordered after the steps in flight
        const int v = cs.iter_end;
        CK(cudaMemcpyAsync(&ctx->cstate.p[case_id].iter_end, &v, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return Q2D_OK;
}

int q2d_gpu_add_block(q2d_ctx* ctx, int case_id, int ni, int nj, const double* nodes_xy,
                      const double* cross_section, int* block_id) {
    if (!ctx || ctx->committed || ctx->serving || case_id < 0 || case_id >= (int)ctx->cases.size() ||
        ni < 1 || nj < 1 || !nodes_xy)
        return fail(ctx, Q2D_ERR_BADARG, "add_block: bad argument");
    HBlock b;
    b.ni = ni; b.nj = nj; b.case_id = case_id;
    b.local_b = (int)ctx->cases[case_id].blocks.size() + 1;
    b.nodes.assign(nodes_xy, nodes_xy + 2 * (size_t)(ni + 1) * (nj + 1));
    if (cross_section) b.area.assign(cross_section, cross_section + (size_t)(ni + 1) * (nj + 1));
    b.prim.assign(4 * (size_t)ni * nj, 0.0);
    ctx->blocks.push_back(std::move(b));
    ctx->cases[case_id].blocks.push_back((int)ctx->blocks.size() - 1);
    if (block_id) *block_id = (int)ctx->blocks.size() - 1;
    return Q2D_OK;
}

int q2d_gpu_set_bcs(q2d_ctx* ctx, int case_id, const q2d_bc_rec* recs, int n) {
    if (!ctx || ctx->committed || ctx->serving || case_id < 0 || case_id >= (int)ctx->cases.size() ||
        n < 0 || (n && !recs))
        return fail(ctx, Q2D_ERR_BADARG, "set_bcs: bad argument");
    HCase& cs = ctx->cases[case_id];
    std::vector<q2d_bc_rec> v(recs, recs + n);
    if (int e = check_recs(ctx, cs, v)) return e;
    std::stable_sort(v.begin(), v.end(), rec_less);
    cs.bc = std::move(v);
    return Q2D_OK;
}

int q2d_gpu_upload_prim(q2d_ctx* ctx, int block_id, const double* P) {
    if (!ctx || block_id < 0 || block_id >= (int)ctx->blocks.size() || !P || ctx->blocks[block_id].case_id < 0)
        return fail(ctx, Q2D_ERR_BADARG, "upload_prim: bad argument");
    HBlock& b = ctx->blocks[block_id];
    const HCase& hc = ctx->cases[b.case_id];
    if (hc.images_sent && !hc.resident && ctx->copy_stream)   // the admission's image copies first
        CK(cudaStreamSynchronize(ctx->copy_stream));
    if (hc.resident || hc.images_sent) {
        // the interior rows of P (4*ni doubles each, pitch 4*(ni+4)) by one strided copy into a
        // staging buffer, then into the state planes on the device (a serving admission's
        // region, whose images were copied at admission, takes the same path)
        const long long n = (long long)b.ni * b.nj;
        CK(ensure_cap(ctx->XFER, 4 * (size_t)n));
        const double* row0 = P + 4 * (2 + (size_t)(b.ni + 4) * 2);
        CK(cudaMemcpy2DAsync(ctx->XFER.p, sizeof(double) * 4 * b.ni, row0, sizeof(double) * 4 * (b.ni + 4),
                             sizeof(double) * 4 * b.ni, b.nj, cudaMemcpyHostToDevice, ctx->stream));
        CK(launch_cells_to_planes(ctx->XFER.p, ctx->PA.p + b.d.oc, n, b.d.pc, ctx->stream));
        ctx->launches += 1;
        CK(cudaStreamSynchronize(ctx->stream));   // P is the caller's: done before returning
        ctx->dt_valid = false;
        return Q2D_OK;
    }
    std::vector<double> planes;
    fortran_to_planes(b.ni, b.nj, P, planes);
    {
        if (ctx->cases[b.case_id].prepared) {
            for (int v = 0; v < 4; ++v)
                std::memcpy(&b.staged.pa[v * b.d.pc], &planes[v * (size_t)b.ni * b.nj],
                            sizeof(double) * b.ni * b.nj);
        } else {
            b.prim = std::move(planes);
        }
        return Q2D_OK;
    }
}

int q2d_gpu_download_prim(q2d_ctx* ctx, int block_id, double* P) {
    if (!ctx || block_id < 0 || block_id >= (int)ctx->blocks.size() || !P)
        return fail(ctx, Q2D_ERR_BADARG, "download_prim: bad argument");
    if (int e = ready(ctx)) return e;
    HBlock& b = ctx->blocks[block_id];
    if (!b.alive || b.case_id < 0 || !ctx->cases[b.case_id].resident)
        return fail(ctx, Q2D_ERR_BADARG, "download_prim: block not resident");
    // the state planes into interleaved rows on the device, then one strided copy into the
    // interior rows of P (its ghost layers are left as they are)
    const long long n = (long long)b.ni * b.nj;
    CK(ensure_cap(ctx->XFER, 4 * (size_t)n));
    CK(launch_planes_to_cells(ctx->PA.p + b.d.oc, b.d.pc, ctx->XFER.p, n, ctx->stream));
    ctx->launches += 1;
    double* row0 = P + 4 * (2 + (size_t)(b.ni + 4) * 2);
    CK(cudaMemcpy2DAsync(row0, sizeof(double) * 4 * (b.ni + 4), ctx->XFER.p, sizeof(double) * 4 * b.ni,
                         sizeof(double) * 4 * b.ni, b.nj, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return Q2D_OK;
}

// Many blocks per call: the strided copies and transposes of all blocks are queued on the
// context's stream through a staging ring of up to kXferRing doubles, synchronising only when
// the ring wraps and once at the end (the caller's arrays are done with when the call returns).
// Blocks of cases not yet on the device take the single-block path (staged on the host).
constexpr long long kXferRing = 16ll << 20;   // 128 MiB

static int transfer_many(q2d_ctx* ctx, int n, const int* ids, double* const* P, bool up) {
    if (!ctx) return Q2D_ERR_BADARG;
    if (n < 0 || (n && (!ids || !P))) return fail(ctx, Q2D_ERR_BADARG, "transfer: bad argument");
    for (int k = 0; k < n; ++k) {
        if (ids[k] < 0 || ids[k] >= (int)ctx->blocks.size() || !P[k] || ctx->blocks[ids[k]].case_id < 0)
            return fail(ctx, Q2D_ERR_BADARG, "transfer: bad block id or array");
    }
    if (!up) {   // a serving context reads resident cases without applying admissions first
        bool all_resident = ctx->serving;
        for (int k = 0; k < n && all_resident; ++k) {
            const HBlock& b = ctx->blocks[ids[k]];
            all_resident = b.alive && ctx->cases[b.case_id].resident;
        }
        if (!all_resident)
            if (int e = ready(ctx)) return e;
    }
    long long need_max = 0, total = 0;
    for (int k = 0; k < n; ++k) {
        const HBlock& b = ctx->blocks[ids[k]];
        if (!ctx->cases[b.case_id].resident || !b.alive) {
            if (!up) return fail(ctx, Q2D_ERR_BADARG, "download_prim: block not resident");
            if (int e = q2d_gpu_upload_prim(ctx, ids[k], P[k])) return e;
            continue;
        }
        const long long len = ((up ? 4ll * (b.ni + 4) * (b.nj + 4) : 4ll * b.ni * b.nj) + 31) / 32 * 32;
        need_max = std::max(need_max, len);
        total += len;
    }
    if (total == 0) return Q2D_OK;
    CK(ensure_cap(ctx->XFER, (size_t)std::max(need_max, std::min(kXferRing, total))));
    const long long cap = (long long)ctx->XFER.n;
    // Segments of the staging ring: upload = one contiguous copy of each caller's whole array,
    // then one transposing launch for the segment; download = one launch, then a strided copy
    // of each block's interior rows (the caller's ghost layers are not written). Work on the
    // one stream is ordered, so a segment reuses the ring without waiting on the host.
    std::vector<XferDesc> seg;
    std::vector<int> seg_k;
    long long off = 0, seg_cells = 0;
    auto flush = [&]() -> int {
        if (seg.empty()) return Q2D_OK;
        CK(ensure_cap(ctx->XDESC, seg.size()));
        CK(cudaMemcpyAsync(ctx->XDESC.p, seg.data(), sizeof(XferDesc) * seg.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
        if (!up) CK(launch_transfer_many(ctx->XDESC.p, (int)seg.size(), seg_cells, false, ctx->XFER.p, ctx->PA.p,
                                         ctx->stream));
        for (size_t q = 0; q < seg.size(); ++q) {
            const XferDesc& x = seg[q];
            const HBlock& b = ctx->blocks[ids[seg_k[q]]];
            if (!up) {
                double* row0 = P[seg_k[q]] + 4 * (2 + (size_t)(b.ni + 4) * 2);
                const size_t w = sizeof(double) * 4 * b.ni, pitch = sizeof(double) * 4 * (b.ni + 4);
                CK(cudaMemcpy2DAsync(row0, pitch, ctx->XFER.p + x.stage, w, w, b.nj, cudaMemcpyDeviceToHost,
                                     ctx->stream));
            }
        }
        if (up) CK(launch_transfer_many(ctx->XDESC.p, (int)seg.size(), seg_cells, true, ctx->XFER.p, ctx->PA.p,
                                        ctx->stream));
        ctx->launches += 1;
        seg.clear();
        seg_k.clear();
        off = 0;
        seg_cells = 0;
        return Q2D_OK;
    };
    for (int k = 0; k < n; ++k) {
        const HBlock& b = ctx->blocks[ids[k]];
        if (!ctx->cases[b.case_id].resident || !b.alive) continue;
        const long long cells = (long long)b.ni * b.nj;
        const long long len = up ? 4ll * (b.ni + 4) * (b.nj + 4) : 4 * cells;
        if (off + len > cap || seg.size() >= 65535) {
            if (int e = flush()) return e;
        }
        XferDesc x;
        x.stage = off; x.plane = b.d.oc; x.pc = b.d.pc; x.ni = b.ni; x.nj = b.nj;
        if (up)   // the whole array in one contiguous copy (its ghost values are not used)
            CK(cudaMemcpyAsync(ctx->XFER.p + off, P[k], sizeof(double) * len, cudaMemcpyHostToDevice, ctx->stream));
        seg.push_back(x);
        seg_k.push_back(k);
        seg_cells = std::max(seg_cells, cells);
        off += (len + 31) / 32 * 32;
    }
    if (int e = flush()) return e;
    CK(cudaStreamSynchronize(ctx->stream));
    if (up) ctx->dt_valid = false;
    return Q2D_OK;
}

int q2d_gpu_commit(q2d_ctx* ctx) {
    if (!ctx) return Q2D_ERR_BADARG;
    return ready(ctx);
}

int q2d_gpu_upload_prim_many(q2d_ctx* ctx, int n, const int* block_ids, const double* const* P) {
    return transfer_many(ctx, n, block_ids, const_cast<double* const*>(P), true);
}

int q2d_gpu_download_prim_many(q2d_ctx* ctx, int n, const int* block_ids, double* const* P) {
    return transfer_many(ctx, n, block_ids, P, false);
}

int q2d_gpu_step_async(q2d_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return fail(ctx, Q2D_ERR_BADARG, "step: bad argument");
    if (int e = ready(ctx)) return e;
    CK(launch_resume(ctx->cstate.p, (int)ctx->cases.size(), ctx->flag.p, ctx->stream));
    ctx->launches += 1;
    if (int e = ensure_dt(ctx)) return e;
    if (nsteps > 0 && ctx->n_items > 0) {
        cudaGraphExec_t ge;
        if (int e = get_graph(ctx, nsteps, &ge)) return e;
        CK(cudaGraphLaunch(ge, ctx->stream));
        ctx->launches += ctx->graph_kernels[nsteps];
    } else {
        CK(cudaMemcpyAsync(ctx->h_state, ctx->cstate.p, sizeof(CaseState) * ctx->cases.size(),
                           cudaMemcpyDeviceToHost, ctx->stream));
    }
    return Q2D_OK;
}

int q2d_gpu_wait(q2d_ctx* ctx, q2d_step_info* out) {
    if (!ctx) return Q2D_ERR_BADARG;
    CK(cudaStreamSynchronize(ctx->stream));
    int first = Q2D_OK;
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        q2d_step_info info;
        fill_info(ctx->h_state[c], &info);
        if (out) out[c] = info;
        if (!first && info.err && ctx->cases[c].used) first = info.err;
    }
    return first;
}

int q2d_gpu_step(q2d_ctx* ctx, int nsteps, q2d_step_info* out) {
    int e = q2d_gpu_step_async(ctx, nsteps);
    if (e) return e;
    return q2d_gpu_wait(ctx, out);
}

void* q2d_gpu_stream(const q2d_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int q2d_gpu_set_schedule(q2d_ctx* ctx, int schedule) {
    if (!ctx || schedule < 0 || schedule >= kNumSchedules || !schedule_allowed(ctx, schedule))
        return fail(ctx, Q2D_ERR_BADARG, "set_schedule: unknown schedule or not valid for this precision");
    if (int e = ready(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->kernel = kSchedules[schedule].kernel;
    ctx->tile = kSchedules[schedule].tile;
    return rebuild_device_lists(ctx);
}

int q2d_gpu_get_schedule(const q2d_ctx* ctx) {
    if (!ctx) return -1;
    for (int k = 0; k < kNumSchedules; ++k)
        if (kSchedules[k].kernel == ctx->kernel && kSchedules[k].tile == ctx->tile) return k;
    return -1;
}

int q2d_gpu_autotune(q2d_ctx* ctx, int steps, int* schedule, float* ms_per_step) {
    if (!ctx || steps < 1) return fail(ctx, Q2D_ERR_BADARG, "autotune: bad argument");
    if (int e = ready(ctx)) return e;
    return autotune(ctx, steps, schedule, ms_per_step);
}

int q2d_gpu_prepare(q2d_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 1) return fail(ctx, Q2D_ERR_BADARG, "prepare: bad argument");
    if (int e = ready(ctx)) return e;
    if (ctx->n_items == 0) return Q2D_OK;
    cudaGraphExec_t ge;
    return get_graph(ctx, nsteps, &ge);
}

int q2d_gpu_case_info(q2d_ctx* ctx, int case_id, q2d_step_info* out) {
    if (!ctx || !out || case_id < 0 || case_id >= (int)ctx->cases.size())
        return fail(ctx, Q2D_ERR_BADARG, "case_info: bad argument");
    if (int e = ready(ctx)) return e;
    CK(cudaMemcpyAsync(ctx->h_state, ctx->cstate.p, sizeof(CaseState) * ctx->cases.size(),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    fill_info(ctx->h_state[case_id], out);
    return Q2D_OK;
}

int q2d_gpu_num_cases(const q2d_ctx* ctx) { return ctx ? (int)ctx->cases.size() : 0; }

long long q2d_gpu_num_cells(const q2d_ctx* ctx) {
    if (!ctx) return 0;
    long long n = 0;
    for (const HCase& cs : ctx->cases)
        if (!ctx->serving || cs.used)
            for (int gb : cs.blocks) n += (long long)ctx->blocks[gb].ni * ctx->blocks[gb].nj;
    return n;
}

long long q2d_gpu_launch_count(const q2d_ctx* ctx) { return ctx ? ctx->launches : 0; }

// ---- serving ---------------------------------------------------------------------------------
int q2d_serve_create(q2d_ctx** out, const q2d_options* opt, unsigned long long device_bytes, int max_cases) {
    if (!out || !opt || max_cases < 1 || device_bytes < (1ull << 20)) return Q2D_ERR_BADARG;
    *out = nullptr;
    if (check_options(opt)) return Q2D_ERR_BADARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return Q2D_ERR_CUDA;
    q2d_ctx* ctx = new_ctx(opt);
    if (!ctx) return Q2D_ERR_OOM;
    ctx->serving = true;
    if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        ctx->copy_stream = nullptr;
        q2d_gpu_destroy(ctx);
        return Q2D_ERR_CUDA;
    }
    ctx->cases.resize(max_cases);
    ctx->f4 = !(opt->precision == Q2D_PREC_FP32_FLUX && difference_form(ctx));
    // Bytes per interior cell: states 3 x 4 planes + scalars 8 planes (160 B), ghost frame
    // 2 planes with up to 50 % halo (24 B), i- and j-faces 3 planes each with up to 15 %
    // extra faces (55 B); the FP32-flux form adds FP32 copies of the ghost-frame and face
    // geometry (12 B + 55 B), the face part only where a kernel other than the difference form
    // can run.
    const double per_cell = (opt->precision == Q2D_PREC_FP32_FLUX ? (ctx->f4 ? 306.4 : 251.2) : 239.2) +
                            (opt->irs_beta > 0.0 ? 64.0 : 0.0);   // two residual pools with IRS
    const long long cells = (long long)((double)device_bytes / per_cell);
    const long long ec = 4 * cells, eg = 3 * cells + 4096, efi = (long long)(3.45 * (double)cells) + 4096,
                    efj = efi;
    int e = allocate_pools(ctx, ec, eg, efi, efj, max_cases);
    if (!e) e = rebuild_device_lists(ctx);
    if (!e) {   // pinned staging of admissions; without it they stage in pageable memory
        const size_t cap = (size_t)std::min<unsigned long long>(2ull << 30, device_bytes / 2);
        if (cudaHostAlloc(&ctx->pin, cap, cudaHostAllocDefault) == cudaSuccess) ctx->pin_cap = cap;
        else { ctx->pin = nullptr; cudaGetLastError(); }
    }
    if (e) {
        q2d_gpu_destroy(ctx);
        return e;
    }
    ctx->committed = true;
    ctx->dt_valid = true;
    *out = ctx;
    return Q2D_OK;
}

int q2d_serve_admit(q2d_ctx* ctx, int nblocks, const int* ni, const int* nj, const double* const* nodes_xy,
                    const double* const* cross_sections, const double* const* P, const q2d_bc_rec* recs,
                    int nrecs, int* case_id) {
    if (!ctx || !ctx->serving || nblocks < 1 || !ni || !nj || !nodes_xy || !P || nrecs < 0 || (nrecs && !recs))
        return fail(ctx, Q2D_ERR_BADARG, "serve_admit: bad argument");
    for (int b = 0; b < nblocks; ++b)
        if (ni[b] < 1 || nj[b] < 1 || !nodes_xy[b] || !P[b])
            return fail(ctx, Q2D_ERR_BADARG, "serve_admit: bad block");
    int slot = -1;
    for (size_t c = 0; c < ctx->cases.size(); ++c)
        if (!ctx->cases[c].used) { slot = (int)c; break; }
    if (slot < 0) return fail(ctx, Q2D_ERR_CAPACITY, "serve_admit: no free case slot");
    HCase& cs = ctx->cases[slot];
    cs = HCase{};
    cs.used = true;
    for (int b = 0; b < nblocks; ++b) {
        int gid = -1;
        for (size_t k = 0; k < ctx->blocks.size(); ++k)
            if (ctx->blocks[k].case_id < 0 && !ctx->blocks[k].alive) { gid = (int)k; break; }
        if (gid < 0) { ctx->blocks.emplace_back(); gid = (int)ctx->blocks.size() - 1; }
        HBlock& hb = ctx->blocks[gid];
        hb = HBlock{};
        hb.ni = ni[b]; hb.nj = nj[b]; hb.case_id = slot; hb.local_b = b + 1;
        hb.nodes_ext = nodes_xy[b];   // read in place until this call returns
        if (cross_sections && cross_sections[b]) hb.area_ext = cross_sections[b];
        hb.P_ext = P[b];
        cs.blocks.push_back(gid);
    }
    std::vector<q2d_bc_rec> v(recs, recs + nrecs);
    int e = check_recs(ctx, cs, v);
    if (!e) {
        std::stable_sort(v.begin(), v.end(), rec_less);
        cs.bc = std::move(v);
        e = prepare_case(ctx, slot);
    }
    if (!e && ctx->copy_stream) {
        e = send_images(ctx, slot, ctx->copy_stream);
        ctx->copies_pending = true;
    }
    for (int gb : cs.blocks) {   // the caller's arrays are not kept past this call
        HBlock& hb = ctx->blocks[gb];
        hb.nodes_ext = hb.area_ext = hb.P_ext = nullptr;
    }
    if (e) {
        free_case_blocks(ctx, cs);
        return e;
    }
    ctx->dirty = true;
    if (case_id) *case_id = slot;
    return Q2D_OK;
}

int q2d_serve_retire(q2d_ctx* ctx, int case_id) {
    if (!ctx || !ctx->serving || case_id < 0 || case_id >= (int)ctx->cases.size() || !ctx->cases[case_id].used)
        return fail(ctx, Q2D_ERR_BADARG, "serve_retire: bad argument");
    // the freed regions may go to the next admission, whose images are copied at once: steps in
    // flight (which may still read this case) finish first
    if (cudaStreamQuery(ctx->stream) == cudaErrorNotReady) CK(cudaStreamSynchronize(ctx->stream));
    free_case_blocks(ctx, ctx->cases[case_id]);
    ctx->reset_slots.push_back(case_id);
    ctx->dirty = true;
    return Q2D_OK;
}

int q2d_serve_block_id(const q2d_ctx* ctx, int case_id, int b, int* block_id) {
    if (!ctx || case_id < 0 || case_id >= (int)ctx->cases.size() || !ctx->cases[case_id].used || b < 1 ||
        b > (int)ctx->cases[case_id].blocks.size() || !block_id)
        return Q2D_ERR_BADARG;
    *block_id = ctx->cases[case_id].blocks[b - 1];
    return Q2D_OK;
}

long long q2d_serve_free_cells(const q2d_ctx* ctx) {
    if (!ctx) return 0;
    const long long c = ctx->ac.free_total() / 4, g = ctx->ag.free_total() / 3,
                    f = std::min(ctx->afi.free_total(), ctx->afj.free_total()) * 100 / 345;
    return std::min(c, std::min(g, f));
}

const char* q2d_gpu_errstr(int status) {
    switch (status) {
        case Q2D_OK: return "ok";
        case Q2D_ERR_BADARG: return "invalid argument or call order";
        case Q2D_ERR_OOM: return "out of memory";
        case Q2D_ERR_CUDA: return "CUDA runtime error";
        case Q2D_ERR_NONPHYSICAL: return "non-physical state detected at an interface";
        case Q2D_ERR_NAN: return "NaN or p<0 detected";
        case Q2D_ERR_TIMEOUT: return "bounded device wait expired";
        case Q2D_ERR_UNSUPPORTED: return "unsupported option or boundary type";
        case Q2D_ERR_CAPACITY: return "request exceeds a fixed capacity";
        default: return "unknown status";
    }
}

const char* q2d_gpu_last_error(const q2d_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

void q2d_gpu_destroy(q2d_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
    ctx->PA.release(); ctx->PB.release(); ctx->PC.release(); ctx->SC.release(); ctx->DL.release();
    ctx->FI.release(); ctx->FJ.release(); ctx->PART.release(); ctx->dblocks.release(); ctx->XFER.release();
    ctx->XDESC.release();
    ctx->RA.release(); ctx->RB.release();
    ctx->DL32.release(); ctx->FI4.release(); ctx->FJ4.release();
    ctx->dcases.release(); ctx->cstate.release(); ctx->items.release(); ctx->edges.release();
    ctx->bcp.release(); ctx->flag.release(); ctx->TAB.release();
    if (ctx->h_state) cudaFreeHost(ctx->h_state);
    if (ctx->h_fresh) cudaFreeHost(ctx->h_fresh);
    if (ctx->h_lists) cudaFreeHost(ctx->h_lists);
    if (ctx->pin) cudaFreeHost(ctx->pin);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

}  // extern "C"
