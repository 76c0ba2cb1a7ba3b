// q2d_api.cu — host runtime behind include/q2d_gpu.h: contexts, device memory, work lists,
// CUDA-graph execution of N explicit steps, state transfer.
//
// Replaces, for one grid level: Assign_Setup (procedure-pointer binding -> kernel selection),
// Allocate_Block / Setup_Metrics (device pools built at commit), and the Explicit_Step loop
// (a captured graph of n_rk fused stage kernels per step; Mod_Explicit.f90:10-174).
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

struct HBlock {
    int ni, nj, case_id, local_b;
    std::vector<double> nodes, area;
    std::vector<double> prim;   // 4 planes, interior
    HostGeom geom;
    DBlock d{};
};

struct HCase {
    std::vector<int> blocks;
    std::vector<q2d_bc_rec> bc;
    double time0 = 0.0;
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

long long round32(long long n) { return (n + 31) / 32 * 32; }

}  // namespace

struct q2d_ctx {
    q2d_options opt{};
    Gas gas{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::vector<HBlock> blocks;
    std::vector<HCase> cases;
    bool committed = false;
    bool dt_valid = false;
    int tile = 0;
    int kernel = 0;       // 0: CTA-tile stage kernel, 1: warp-marching stage kernel
    int march_h = 16;     // rows per warp-marching item
    int grid = 0;
    // device pools
    DevBuf<double> PA, PB, PC, SC, DL, FI, FJ, PART;
    DevBuf<DBlock> dblocks;
    DevBuf<DCase> dcases;
    DevBuf<CaseState> cstate;
    DevBuf<WorkItem> items;
    DevBuf<EdgeRec> edges;
    DevBuf<BCParam> bcp;
    DevBuf<int> flag;
    CaseState* h_state = nullptr;   // pinned mirror
    long long total_cells = 0;
    long long pool4 = 0;            // elements of a 4-plane cell pool
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

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

StageArgs base_args(q2d_ctx* ctx) {
    StageArgs a{};
    a.blocks = ctx->dblocks.p;
    a.cases = ctx->dcases.p;
    a.cstate = ctx->cstate.p;
    a.items = ctx->items.p;
    a.n_items = (int)ctx->items.n;
    a.sc = ctx->SC.p;
    a.dl = ctx->DL.p;
    a.dl32 = nullptr;
    a.fi = ctx->FI.p;
    a.fj = ctx->FJ.p;
    a.edges = ctx->edges.p;
    a.bcp = ctx->bcp.p;
    a.part = ctx->PART.p;
    a.gas = ctx->gas;
    a.cfl = ctx->opt.cfl;
    a.n_rk = ctx->opt.n_rk;
    a.limiter = ctx->opt.limiter;
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
    for (int irk = 1; irk <= n_rk; ++irk) {
        StageArgs a = base_args(ctx);
        a.irk = irk;
        a.first = irk == 1;
        a.last = irk == n_rk;
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
        if (ctx->kernel == 1)
            CK(launch_march(a, ctx->opt.precision, ctx->opt.riemann, ctx->opt.limiter, ctx->grid, s));
        else
            CK(launch_stage(a, ctx->opt.precision, ctx->opt.riemann, ctx->tile, ctx->grid, s));
        ++*nk;
    }
    if (n_rk == 1) {
        CK(launch_copy(ctx->PB.p, ctx->PA.p, ctx->pool4, ctx->flag.p, s));
        ++*nk;
    }
    return Q2D_OK;
}

int ensure_dt(q2d_ctx* ctx) {
    if (ctx->dt_valid) return Q2D_OK;
    StageArgs a = base_args(ctx);
    a.Pin = ctx->PA.p;
    if (ctx->kernel == 1) CK(launch_dt_march(a, ctx->grid, ctx->stream));
    else CK(launch_dt(a, ctx->tile, ctx->grid, ctx->stream));
    ctx->launches += 1;
    ctx->dt_valid = true;
    return Q2D_OK;
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


// Work items of the current schedule (kernel / tile / rows per item), grouped by case, and
// the persistent grid size. Re-run by the autotuner for every candidate schedule.
int build_items(q2d_ctx* ctx) {
    int TX, TY, NT;
    tile_dims(ctx->tile, &TX, &TY, &NT);
    std::vector<WorkItem> items;
    std::vector<DCase> dcases(ctx->cases.size());
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        dcases[c].item_begin = (int)items.size();
        for (int gb : ctx->cases[c].blocks) {
            const HBlock& B = ctx->blocks[gb];
            if (ctx->kernel == 1) {
                for (int i0 = 0; i0 < B.ni; i0 += kMarchCols)
                    for (int j0 = 0; j0 < B.nj; j0 += ctx->march_h)
                        items.push_back(WorkItem{gb, i0, j0, (int)c, std::min(B.nj, j0 + ctx->march_h), 0});
            } else {
                for (int j0 = 0; j0 < B.nj; j0 += TY)
                    for (int i0 = 0; i0 < B.ni; i0 += TX) items.push_back(WorkItem{gb, i0, j0, (int)c, 0, 0});
            }
        }
        dcases[c].item_end = (int)items.size();
        dcases[c].ndir = ctx->blocks[ctx->cases[c].blocks[0]].nj == 1 ? 1 : 2;
    }
    ctx->items.release();
    ctx->PART.release();
    ctx->dcases.release();
    CK(ctx->items.alloc(items.size()));
    CK(ctx->PART.alloc(5 * items.size()));
    CK(ctx->dcases.alloc(dcases.size()));
    CK(cudaMemcpy(ctx->items.p, items.data(), sizeof(WorkItem) * items.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->dcases.p, dcases.data(), sizeof(DCase) * dcases.size(), cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->PART.p, 0, sizeof(double) * 5 * items.size()));
    if (ctx->kernel == 1) {
        const int occ = std::max(1, march_occupancy(ctx->opt.precision, ctx->opt.riemann, ctx->opt.limiter));
        ctx->grid = (int)std::min<long long>(((long long)items.size() + 3) / 4, (long long)occ * ctx->num_sms);
    } else {
        const int occ = std::max(1, stage_occupancy(ctx->opt.precision, ctx->opt.riemann, ctx->tile));
        ctx->grid = (int)std::min<long long>((long long)items.size(), (long long)occ * ctx->num_sms);
    }
    if (ctx->grid < 1) ctx->grid = 1;
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
    ctx->graphs.clear();
    ctx->graph_kernels.clear();
    return Q2D_OK;
}

int commit(q2d_ctx* ctx) {
    if (ctx->committed) return Q2D_OK;
    if (ctx->cases.empty()) return fail(ctx, Q2D_ERR_BADARG, "no case");
    // ---- boundary records -> edge arrays (geometry of ghost cells is added per block below) --
    std::vector<EdgeRec> edges;
    std::vector<BCParam> params;
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        HCase& cs = ctx->cases[c];
        if (cs.blocks.empty()) return fail(ctx, Q2D_ERR_BADARG, "case without blocks");
        for (int gb : cs.blocks) {
            HBlock& B = ctx->blocks[gb];
            const int len[4] = {B.nj, B.nj, B.ni, B.ni};
            for (int f = 0; f < 4; ++f) {
                B.d.eo[f] = (int)edges.size();
                edges.resize(edges.size() + len[f], EdgeRec{-1, 0, 0, 0, 0, -1});
            }
        }
        for (const q2d_bc_rec& r : cs.bc) {
            HBlock& B = ctx->blocks[cs.blocks[r.b - 1]];
            const bool pos_ok = (r.f == 1 && r.i == 1) || (r.f == 2 && r.i == B.ni) ||
                                (r.f == 3 && r.j == 1) || (r.f == 4 && r.j == B.nj);
            if (!pos_ok) return fail(ctx, Q2D_ERR_BADARG, "boundary record not on its face");
            const int k = (r.f <= 2) ? r.j - 1 : r.i - 1;
            EdgeRec& er = edges[B.d.eo[r.f - 1] + k];
            if (er.type != -1) return fail(ctx, Q2D_ERR_BADARG, "duplicate boundary record");
            er.type = r.type;
            if (r.type == 101) {
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
                face_tangent(r, B.ni, B.nodes.data(), &p.t0, &p.t1);
                er.param = (int)params.size();
                params.push_back(p);
            }
        }
        for (int gb : cs.blocks) {
            const HBlock& B = ctx->blocks[gb];
            const int len[4] = {B.nj, B.nj, B.ni, B.ni};
            for (int f = 0; f < 4; ++f)
                for (int k = 0; k < len[f]; ++k)
                    if (edges[B.d.eo[f] + k].type == -1)
                        return fail(ctx, Q2D_ERR_BADARG, "boundary cell without a record (block " +
                                    std::to_string(B.local_b) + ", face " + std::to_string(f + 1) + ")");
        }
    }
    // ---- pool layout ---------------------------------------------------------------------
    long long oc = 0, og = 0, ofi = 0, ofj = 0;
    for (HBlock& b : ctx->blocks) {
        DBlock& d = b.d;
        d.ni = b.ni; d.nj = b.nj; d.case_id = b.case_id; d.local_b = b.local_b;
        d.pc = round32((long long)b.ni * b.nj);
        d.pg = round32((long long)(b.ni + 4) * (b.nj + 4));
        d.pfi = round32((long long)(b.ni + 1) * b.nj);
        d.pfj = round32((long long)b.ni * (b.nj + 1));
        d.oc = oc; d.og = og; d.ofi = ofi; d.ofj = ofj; d.on = 0; d.pn = 0;
        oc += 4 * d.pc; og += 2 * d.pg; ofi += 3 * d.pfi; ofj += 3 * d.pfj;
    }
    ctx->pool4 = oc;
    // ---- device pools, filled block by block (host memory stays at one block) -------------
    CK(ctx->PA.alloc(oc)); CK(ctx->PB.alloc(oc)); CK(ctx->PC.alloc(oc));
    CK(ctx->SC.alloc(2 * oc)); CK(ctx->DL.alloc(og)); CK(ctx->FI.alloc(ofi)); CK(ctx->FJ.alloc(ofj));
    CK(cudaMemset(ctx->PB.p, 0, sizeof(double) * oc));
    CK(cudaMemset(ctx->PC.p, 0, sizeof(double) * oc));
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        HCase& cs = ctx->cases[c];
        for (int gb : cs.blocks) {
            HBlock& b = ctx->blocks[gb];
            int e = setup_block(b.ni, b.nj, b.nodes.data(), b.area.empty() ? nullptr : b.area.data(),
                                ctx->opt.source, b.geom);
            if (e) return fail(ctx, e, "degenerate cell in block " + std::to_string(b.local_b));
        }
        for (const q2d_bc_rec& r : cs.bc) {
            HBlock& B = ctx->blocks[cs.blocks[r.b - 1]];
            const HBlock* D = r.type == 101 ? &ctx->blocks[cs.blocks[r.bs - 1]] : nullptr;
            int e = ghost_metrics(r, B.ni, B.nj, B.nodes.data(), B.geom, D ? D->ni : 0, D ? D->nj : 0,
                                  D ? D->nodes.data() : nullptr);
            if (e) return fail(ctx, e, "ghost metrics failed for a boundary record");
        }
        for (int gb : cs.blocks) {
            HBlock& b = ctx->blocks[gb];
            const DBlock& d = b.d;
            const HostGeom& G = b.geom;
            const long long n = (long long)b.ni * b.nj;
            std::vector<double> sc(8 * (size_t)d.pc, 0.0), dl(2 * (size_t)d.pg, 0.0), fi(3 * (size_t)d.pfi, 0.0),
                fj(3 * (size_t)d.pfj, 0.0), pa(4 * (size_t)d.pc, 0.0);
            for (int j = 0; j < b.nj; ++j)
                for (int i = 0; i < b.ni; ++i) {
                    const long long k = (long long)j * b.ni + i;
                    double v[4];
                    versors(G, i, j, v);
                    sc[k] = G.sur[G.g(i, j)];
                    sc[2 * d.pc + k] = v[0];
                    sc[3 * d.pc + k] = v[1];
                    sc[4 * d.pc + k] = v[2];
                    sc[5 * d.pc + k] = v[3];
                    sc[6 * d.pc + k] = G.src0[k];
                    sc[7 * d.pc + k] = G.src1[k];
                }
            for (long long k = 0; k < (long long)(b.ni + 4) * (b.nj + 4); ++k) {
                dl[k] = G.dl[2 * k];
                dl[d.pg + k] = G.dl[2 * k + 1];
            }
            for (long long k = 0; k < (long long)(b.ni + 1) * b.nj; ++k)
                for (int q = 0; q < 3; ++q) fi[q * d.pfi + k] = G.fi[3 * k + q];
            for (long long k = 0; k < (long long)b.ni * (b.nj + 1); ++k)
                for (int q = 0; q < 3; ++q) fj[q * d.pfj + k] = G.fj[3 * k + q];
            for (int v = 0; v < 4; ++v) std::memcpy(&pa[v * d.pc], &b.prim[(size_t)v * n], sizeof(double) * n);
            CK(cudaMemcpy(ctx->PA.p + d.oc, pa.data(), sizeof(double) * pa.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ctx->SC.p + 2 * d.oc, sc.data(), sizeof(double) * sc.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ctx->DL.p + d.og, dl.data(), sizeof(double) * dl.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ctx->FI.p + d.ofi, fi.data(), sizeof(double) * fi.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ctx->FJ.p + d.ofj, fj.data(), sizeof(double) * fj.size(), cudaMemcpyHostToDevice));
            ctx->total_cells += n;
            b.prim.clear(); b.prim.shrink_to_fit();
            b.geom = HostGeom{};
        }
    }
    std::vector<DBlock> db(ctx->blocks.size());
    for (size_t k = 0; k < ctx->blocks.size(); ++k) db[k] = ctx->blocks[k].d;
    std::vector<CaseState> st(ctx->cases.size());
    for (size_t c = 0; c < ctx->cases.size(); ++c) {
        CaseState& s = st[c];
        std::memset(&s, 0, sizeof(s));
        s.res0 = -1.0;
        s.todo = Q2D_TODO_CONTINUE;
        s.status = kStatus_Running;
        s.time = ctx->cases[c].time0;
        s.time_from_call = s.time;
    }
    CK(ctx->dblocks.alloc(db.size()));
    CK(ctx->cstate.alloc(st.size()));
    CK(ctx->edges.alloc(edges.size())); CK(ctx->bcp.alloc(params.size())); CK(ctx->flag.alloc(1));
    CK(cudaMallocHost(&ctx->h_state, sizeof(CaseState) * st.size()));
    CK(cudaMemcpy(ctx->dblocks.p, db.data(), sizeof(DBlock) * db.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->cstate.p, st.data(), sizeof(CaseState) * st.size(), cudaMemcpyHostToDevice));
    if (!edges.empty()) CK(cudaMemcpy(ctx->edges.p, edges.data(), sizeof(EdgeRec) * edges.size(), cudaMemcpyHostToDevice));
    if (!params.empty()) CK(cudaMemcpy(ctx->bcp.p, params.data(), sizeof(BCParam) * params.size(), cudaMemcpyHostToDevice));
    {
        int e = build_items(ctx);
        if (e) return e;
    }
    ctx->committed = true;
    ctx->dt_valid = false;
    return Q2D_OK;
}

// ---- autotuner ------------------------------------------------------------------------------
// Times every schedule (stage-kernel tile shape or warp-marching rows per item) for `steps`
// explicit steps on the context's own workload and keeps the fastest. The state, the case
// states and the time steps are saved before and restored after, so tuning has no effect on
// the results.
struct Schedule { int kernel, tile, march_h; };

int autotune(q2d_ctx* ctx, int steps, int* best_out, float* ms_out) {
    static const Schedule cands[] = {{0, 0, 16}, {0, 1, 16}, {0, 2, 16}, {1, 0, 8}, {1, 0, 16}};
    const int ncand = (int)(sizeof(cands) / sizeof(cands[0]));
    const size_t nst = ctx->cases.size();
    DevBuf<double> saveP, saveSC;
    DevBuf<CaseState> saveCS;
    CK(saveP.alloc(ctx->pool4));
    CK(saveSC.alloc(2 * ctx->pool4));
    CK(saveCS.alloc(nst));
    if (int e = ensure_dt(ctx)) return e;
    CK(cudaMemcpyAsync(saveP.p, ctx->PA.p, sizeof(double) * ctx->pool4, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(saveSC.p, ctx->SC.p, sizeof(double) * 2 * ctx->pool4, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(saveCS.p, ctx->cstate.p, sizeof(CaseState) * nst, cudaMemcpyDeviceToDevice, ctx->stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int besti = 0;
    for (int k = 0; k < ncand; ++k) {
        ctx->kernel = cands[k].kernel;
        ctx->tile = cands[k].tile;
        ctx->march_h = cands[k].march_h;
        if (int e = build_items(ctx)) return e;
        int nk = 0;
        for (int w = 0; w < 1 && nk >= 0; ++w)
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
        // restore before the next candidate
        CK(cudaMemcpyAsync(ctx->PA.p, saveP.p, sizeof(double) * ctx->pool4, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->SC.p, saveSC.p, sizeof(double) * 2 * ctx->pool4, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->cstate.p, saveCS.p, sizeof(CaseState) * nst, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    ctx->kernel = cands[besti].kernel;
    ctx->tile = cands[besti].tile;
    ctx->march_h = cands[besti].march_h;
    if (int e = build_items(ctx)) return e;
    CK(cudaStreamSynchronize(ctx->stream));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    saveP.release(); saveSC.release(); saveCS.release();
    if (best_out) *best_out = besti;
    if (ms_out) *ms_out = best / (float)steps;
    return Q2D_OK;
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
    if (opt->n_rk < 1 || opt->n_rk > 3 || opt->limiter < 0 || opt->limiter > 6 || opt->riemann < 0 ||
        opt->riemann > 2 || opt->source < 0 || opt->source > 2 || opt->precision < 0 ||
        opt->precision > 1 || !(opt->gas_gamma > 1.0) || !(opt->gas_R > 0.0) || opt->res_diter < 1 ||
        opt->sol_diter < 1 || !(opt->cfl > 0.0))
        return Q2D_ERR_BADARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return Q2D_ERR_CUDA;
    q2d_ctx* ctx = new (std::nothrow) q2d_ctx();
    if (!ctx) return Q2D_ERR_OOM;
    ctx->opt = *opt;
    ctx->gas.R = opt->gas_R;
    ctx->gas.gamma = opt->gas_gamma;
    ctx->gas.gm1 = opt->gas_gamma - 1.0;
    ctx->gas.cp = opt->gas_gamma * opt->gas_R / (opt->gas_gamma - 1.0);
    ctx->gas.cv = opt->gas_R / (opt->gas_gamma - 1.0);
    ctx->gas.gfac = opt->gas_gamma / (opt->gas_gamma - 1.0);
    ctx->gas.igm1 = 1.0 / (opt->gas_gamma - 1.0);
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return Q2D_ERR_CUDA;
    }
    const char* t = getenv("Q2D_TILE");
    if (t) ctx->tile = std::max(0, std::min(kNumTiles - 1, atoi(t)));
    const char* kk = getenv("Q2D_KERNEL");
    if (kk) ctx->kernel = atoi(kk) == 0 ? 0 : 1;
    const char* mh = getenv("Q2D_MARCH_H");
    if (mh) ctx->march_h = std::max(1, std::min(4096, atoi(mh)));
    *out = ctx;
    return Q2D_OK;
}

int q2d_gpu_add_case(q2d_ctx* ctx, int* case_id) {
    if (!ctx || ctx->committed) return fail(ctx, Q2D_ERR_BADARG, "add_case after commit");
    ctx->cases.emplace_back();
    if (case_id) *case_id = (int)ctx->cases.size() - 1;
    return Q2D_OK;
}

int q2d_gpu_add_block(q2d_ctx* ctx, int case_id, int ni, int nj, const double* nodes_xy,
                      const double* cross_section, int* block_id) {
    if (!ctx || ctx->committed || case_id < 0 || case_id >= (int)ctx->cases.size() || ni < 1 ||
        nj < 1 || !nodes_xy)
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
    if (!ctx || ctx->committed || case_id < 0 || case_id >= (int)ctx->cases.size() || n < 0 ||
        (n && !recs))
        return fail(ctx, Q2D_ERR_BADARG, "set_bcs: bad argument");
    HCase& cs = ctx->cases[case_id];
    std::vector<q2d_bc_rec> v(recs, recs + n);
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
            case 101:
                if (r.bs < 1 || r.bs > (int)cs.blocks.size() || r.fs < 1 || r.fs > 4)
                    return fail(ctx, Q2D_ERR_BADARG, "set_bcs: bad connection donor");
                break;
            default:
                return fail(ctx, Q2D_ERR_UNSUPPORTED, "set_bcs: BC type " + std::to_string(r.type) +
                                                          " is not on the built path");
        }
    }
    std::stable_sort(v.begin(), v.end(), rec_less);
    cs.bc = std::move(v);
    return Q2D_OK;
}

int q2d_gpu_upload_prim(q2d_ctx* ctx, int block_id, const double* P) {
    if (!ctx || block_id < 0 || block_id >= (int)ctx->blocks.size() || !P)
        return fail(ctx, Q2D_ERR_BADARG, "upload_prim: bad argument");
    HBlock& b = ctx->blocks[block_id];
    const long long n = (long long)b.ni * b.nj;
    std::vector<double> planes(4 * n);
    for (int j = 0; j < b.nj; ++j)
        for (int i = 0; i < b.ni; ++i) {
            const double* src = &P[4 * ((size_t)(i + 2) + (size_t)(b.ni + 4) * (j + 2))];
            for (int v = 0; v < 4; ++v) planes[v * n + (size_t)j * b.ni + i] = src[v];
        }
    if (!ctx->committed) {
        b.prim = std::move(planes);
        return Q2D_OK;
    }
    std::vector<double> staged(4 * (size_t)b.d.pc, 0.0);
    for (int v = 0; v < 4; ++v) std::memcpy(&staged[v * b.d.pc], &planes[v * n], sizeof(double) * n);
    CK(cudaMemcpy(ctx->PA.p + b.d.oc, staged.data(), sizeof(double) * staged.size(), cudaMemcpyHostToDevice));
    ctx->dt_valid = false;
    return Q2D_OK;
}

int q2d_gpu_download_prim(q2d_ctx* ctx, int block_id, double* P) {
    if (!ctx || block_id < 0 || block_id >= (int)ctx->blocks.size() || !P)
        return fail(ctx, Q2D_ERR_BADARG, "download_prim: bad argument");
    int e = commit(ctx);
    if (e) return e;
    HBlock& b = ctx->blocks[block_id];
    std::vector<double> staged(4 * (size_t)b.d.pc);
    CK(cudaMemcpyAsync(staged.data(), ctx->PA.p + b.d.oc, sizeof(double) * staged.size(),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double* planes = staged.data();
    const long long pcs = b.d.pc;
    for (int j = 0; j < b.nj; ++j)
        for (int i = 0; i < b.ni; ++i) {
            double* dst = &P[4 * ((size_t)(i + 2) + (size_t)(b.ni + 4) * (j + 2))];
            for (int v = 0; v < 4; ++v) dst[v] = planes[v * pcs + (size_t)j * b.ni + i];
        }
    return Q2D_OK;
}

int q2d_gpu_commit(q2d_ctx* ctx) {
    if (!ctx) return Q2D_ERR_BADARG;
    return commit(ctx);
}

int q2d_gpu_step_async(q2d_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return fail(ctx, Q2D_ERR_BADARG, "step: bad argument");
    int e = commit(ctx);
    if (e) return e;
    CK(launch_resume(ctx->cstate.p, (int)ctx->cases.size(), ctx->flag.p, ctx->stream));
    ctx->launches += 1;
    if ((e = ensure_dt(ctx))) return e;
    if (nsteps > 0) {
        cudaGraphExec_t ge;
        if ((e = get_graph(ctx, nsteps, &ge))) return e;
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
        if (!first && info.err) first = info.err;
    }
    return first;
}

int q2d_gpu_step(q2d_ctx* ctx, int nsteps, q2d_step_info* out) {
    int e = q2d_gpu_step_async(ctx, nsteps);
    if (e) return e;
    return q2d_gpu_wait(ctx, out);
}

void* q2d_gpu_stream(const q2d_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int q2d_gpu_autotune(q2d_ctx* ctx, int steps, int* schedule, float* ms_per_step) {
    if (!ctx || steps < 1) return fail(ctx, Q2D_ERR_BADARG, "autotune: bad argument");
    int e = commit(ctx);
    if (e) return e;
    return autotune(ctx, steps, schedule, ms_per_step);
}

int q2d_gpu_prepare(q2d_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 1) return fail(ctx, Q2D_ERR_BADARG, "prepare: bad argument");
    int e = commit(ctx);
    if (e) return e;
    cudaGraphExec_t ge;
    return get_graph(ctx, nsteps, &ge);
}

int q2d_gpu_case_info(q2d_ctx* ctx, int case_id, q2d_step_info* out) {
    if (!ctx || !out || case_id < 0 || case_id >= (int)ctx->cases.size())
        return fail(ctx, Q2D_ERR_BADARG, "case_info: bad argument");
    int e = commit(ctx);
    if (e) return e;
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
    for (const HBlock& b : ctx->blocks) n += (long long)b.ni * b.nj;
    return n;
}
long long q2d_gpu_launch_count(const q2d_ctx* ctx) { return ctx ? ctx->launches : 0; }

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
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
    ctx->PA.release(); ctx->PB.release(); ctx->PC.release(); ctx->SC.release(); ctx->DL.release();
    ctx->FI.release(); ctx->FJ.release(); ctx->PART.release(); ctx->dblocks.release();
    ctx->dcases.release(); ctx->cstate.release(); ctx->items.release(); ctx->edges.release();
    ctx->bcp.release(); ctx->flag.release();
    if (ctx->h_state) cudaFreeHost(ctx->h_state);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

}  // extern "C"
