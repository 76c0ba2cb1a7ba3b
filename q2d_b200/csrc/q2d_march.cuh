// q2d_march.cuh — the warp-marching RK-stage kernel of the Q2D explicit path (sm_100a).
//
// One warp owns a strip of 32 consecutive columns of a block (28 updated columns plus a
// 2-column halo on each side, the stencil width of MUSCL) and marches up a range of rows
// with a 3-row register window. Per row it:
//   - loads the row two ahead (primitive state, mean lengths); block-edge ghost columns are
//     filled from neighbouring lanes by the Fill_Ghost_Cell rules (Lib_Ghost.f90:163-299) or,
//     for block interfaces (101), read from the donor block's HBM state — the device-side
//     block-interface copy that replaces the MPI halo exchange (Mod_GhostExchange.f90);
//   - j-direction: one new interface slope, one limited cell slope and the j-face flux above
//     the row (MUSCL reconstruction + Riemann, Convective_Flux, Lib_Convective.f90:15-82);
//   - i-direction: interface slopes, limited slopes and i-face fluxes of the row, neighbours
//     exchanged with warp shuffles;
//   - the residual of the row's cells in the reference accumulation order (interior i-faces,
//     interior j-faces, boundary faces 1..4; Mod_Fluxes.f90:122-232, Mod_BC_Fluxes.f90:79-84),
//     the geometric source, Newstate_Conservative with the RK stage and Check_And_Fix_State
//     (Lib_Newstate.f90:131-159, 316-350; Lib_RK.f90:15-27);
//   - on the last stage, the cell's time step for the next step (Compute_dt, Mod_dt.f90:59-104)
//     and its squared change (Compute_Residual, Mod_Diagnostic.f90:438-469).
// Warps are independent: no shared memory, no block barrier. Per-case reductions are summed
// in item order by the last warp to finish the case (atomic counter, no spin-wait).
#pragma once
#include "q2d_common.cuh"

namespace q2d {

constexpr unsigned kFull = 0xffffffffu;

template <typename T>
struct V4 { T v[4]; };

// Warp-level: the warp that completes the last item of a case finalises it.
__device__ __forceinline__ void warp_item_done(const StageArgs& a, int case_id, const double* part5,
                                               int item, bool with_res, bool with_dt, bool commit_begin) {
    const int lane = threadIdx.x & 31;
    if (with_res || with_dt) {
        if (lane == 0)
            for (int k = 0; k < 5; ++k) a.part[5 * (size_t)item + k] = part5[k];
    }
    __syncwarp();
    int last = 0;
    const DCase dc = a.cases[case_id];
    if (lane == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&a.cstate[case_id].counter, 1u);
        last = (prev == (unsigned)(dc.item_end - dc.item_begin - 1));
    }
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    CaseState* cs = &a.cstate[case_id];
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
    if (with_res || with_dt) {
        for (int it = dc.item_begin + lane; it < dc.item_end; it += 32) {
            const double* p = a.part + 5 * (size_t)it;
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] += __ldcg(p + k);
            acc[4] = fmin(acc[4], __ldcg(p + 4));
        }
#pragma unroll
        for (int k = 0; k < 5; ++k)
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(kFull, acc[k], o);
                acc[k] = (k < 4) ? acc[k] + w : fmin(acc[k], w);
            }
    }
    if (lane == 0) {
        if (commit_begin) {   // Explicit_Step prologue (Mod_Explicit.f90:38-55)
            cs->dtglobal = cs->dt_step;
            cs->iter += 1;
            cs->iter_from_call += 1;
            if (a.time_accurate) cs->time = cs->time + cs->dt_step;
        }
        if (with_dt) {
            cs->dt_step = fmin(acc[4], 1e5);
            cs->dt_pending = 0;
        }
        if (with_res) {   // Mod_Explicit.f90:120-170
            if (cs->iter_from_call == 1 || (cs->iter % a.res_diter) == 0) {
                for (int k = 0; k < 4; ++k) cs->res[k] = sqrt(acc[k]);
                if (cs->res0 < 0.0) cs->res0 = cs->res[0];
            }
            const double thr = a.res_relative ? a.res_threshold * cs->res0 : a.res_threshold;
            const bool endsim = (cs->iter_from_call >= a.itermax) || (cs->res[0] <= thr) ||
                                (cs->time >= a.time_threshold);
            const bool iosim = ((cs->iter % a.sol_diter) == 0) ||
                               (cs->time >= cs->time_from_call + a.sol_dtime);
            cs->todo = endsim ? 3 : (iosim ? 2 : 1);
            cs->status = endsim ? kStatus_Done : (iosim ? kStatus_Paused : kStatus_Running);
        }
        if (atomicAdd(&cs->err, 0) != 0) cs->status = kStatus_Error;
        cs->counter = 0;
        __threadfence();
    }
    __syncwarp();
}

// One row of the window: primitive state and mean lengths dl(1), dl(2) of this lane's column.
struct Row {
    double q[4];
    double dli, dlj;
};

template <int PREC, int RIEM, int LIM>
__global__ void __launch_bounds__(128, 2) march_kernel(const StageArgs a) {
    using ST = typename std::conditional<PREC == 0, double, float>::type;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const Gas& g = a.gas;

    for (int it = gw; it < a.n_items; it += nw) {
        const WorkItem w = a.items[it];
        const DBlock B = a.blocks[w.block];
        CaseState* cs = &a.cstate[w.case_id];
        if (__ldcg(&cs->status) != kStatus_Running) continue;   // warp-uniform
        const int ni = B.ni, nj = B.nj;
        const long long pc = B.pc;
        const double* Pin = a.Pin + B.oc;
        const double* scb = a.sc + 2 * B.oc;
        const int c = w.i0 - 2 + lane;                 // 0-based column of this lane
        const bool inI = (c >= 0 && c < ni);
        const bool useful = (lane >= 2 && lane < 30 && inI);
        const bool edgeStrip = (w.i0 == 0) || (w.i0 + 29 >= ni);   // a ghost column lies in the strip
        const bool inFrameI = (c >= -2 && c <= ni + 1);
        const int r0 = w.j0, r1 = w.j1;
        // j-edge records of this column (faces 3 and 4)
        EdgeRec eBot{-1, 0, 0, 0, 0, -1}, eTop{-1, 0, 0, 0, 0, -1};
        if (inI) { eBot = a.edges[B.eo[2] + c]; eTop = a.edges[B.eo[3] + c]; }

        // ---- loaders ----------------------------------------------------------------------
        auto load_dl = [&](int jr, Row& R) {
            if (inFrameI && jr >= -2 && jr <= nj + 1) {
                const double* d = a.dl + B.og + (long long)(jr + 2) * (ni + 4) + (c + 2);
                R.dli = d[0];
                R.dlj = d[B.pg];
            } else {
                R.dli = 1.0;
                R.dlj = 1.0;
            }
        };
        auto load_donor = [&](const EdgeRec& e, int gd, double* q) {   // Ghost_Connection
            const DBlock S = a.blocks[e.bs];
            const int si = e.is + guide_i(e.fs) * (gd - 1) - 1;
            const int sj = e.js + guide_j(e.fs) * (gd - 1) - 1;
            const double* src = a.Pin + S.oc + (long long)sj * S.ni + si;
#pragma unroll
            for (int v = 0; v < 4; ++v) q[v] = src[v * S.pc];
        };
        // Interior row jr in [0, nj): state + i-ghost columns of edge strips.
        auto load_row = [&](int jr, Row& R) {
            load_dl(jr, R);
            int etype = -2;   // i-ghost rule of this lane (-2: not an i-ghost)
            int gd = 0, f = 0;
            if (inI) {
                const double* src = Pin + (long long)jr * ni + c;
#pragma unroll
                for (int v = 0; v < 4; ++v) R.q[v] = src[v * pc];
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) R.q[v] = 0.0;
                if (c >= -2 && c < 0) { f = 1; gd = -c; }
                else if (c >= ni && c <= ni + 1) { f = 2; gd = c - ni + 1; }
                if (f) {
                    const EdgeRec e = a.edges[B.eo[f - 1] + jr];
                    etype = e.type;
                    if (etype == 101) load_donor(e, gd, R.q);
                }
            }
            if (edgeStrip) {   // warp-uniform: fill the non-connection i-ghosts by shuffles
                int sb = lane, s1 = lane, s2 = lane;
                if (f == 1) { sb = lane - c; s1 = sb + 1; s2 = sb + 2; }
                if (f == 2) { sb = lane - (c - (ni - 1)); s1 = sb - 1; s2 = sb - 2; }
                sb &= 31; s1 &= 31; s2 &= 31;
                double qb[4], q1[4], q2[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    qb[v] = __shfl_sync(kFull, R.q[v], sb);
                    q1[v] = __shfl_sync(kFull, R.q[v], s1);
                    q2[v] = __shfl_sync(kFull, R.q[v], s2);
                }
                if (f && etype != 101) {
                    if (etype == 300) {   // Ghost_Symmetry (Lib_Ghost.f90:163-196)
                        const long long fidx = B.ofi + (long long)jr * (ni + 1) + (f == 1 ? 0 : ni);
                        const double nx = a.fi[fidx], ny = a.fi[fidx + B.pfi];
                        const double udotn = qb[1] * nx + qb[2] * ny;
                        R.q[0] = qb[0];
                        R.q[1] = qb[1] - 2.0 * udotn * nx;
                        R.q[2] = qb[2] - 2.0 * udotn * ny;
                        R.q[3] = qb[3];
                    } else if (etype == 0 || etype == 401 || etype == 405 || etype == 406 || etype < 0) {
#pragma unroll
                        for (int v = 0; v < 4; ++v) R.q[v] = qb[v];   // Ghost_ZG_Extrapolate
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) {                  // Ghost_Extrapolate
                            const double g1 = 3.0 * qb[v] - 3.0 * q1[v] + q2[v];
                            R.q[v] = (gd == 1) ? g1 : 3.0 * g1 - 3.0 * qb[v] + q1[v];
                        }
                    }
                }
            }
        };
        // Ghost row of the bottom (face 3) or top (face 4) edge, layer gd, for this column:
        // b0 = boundary row, b1/b2 = the next interior rows inward.
        auto ghost_row = [&](const EdgeRec& e, int face, int gd, const double* b0, const double* b1,
                             const double* b2, Row& R) {
            if (!inI) {
#pragma unroll
                for (int v = 0; v < 4; ++v) R.q[v] = 0.0;
                return;
            }
            if (e.type == 101) { load_donor(e, gd, R.q); return; }
            if (e.type == 300) {
                const long long fidx = B.ofj + (long long)(face == 3 ? 0 : nj) * ni + c;
                const double nx = a.fj[fidx], ny = a.fj[fidx + B.pfj];
                const double udotn = b0[1] * nx + b0[2] * ny;
                R.q[0] = b0[0];
                R.q[1] = b0[1] - 2.0 * udotn * nx;
                R.q[2] = b0[2] - 2.0 * udotn * ny;
                R.q[3] = b0[3];
            } else if (e.type == 0 || e.type == 401 || e.type == 405 || e.type == 406 || e.type < 0) {
#pragma unroll
                for (int v = 0; v < 4; ++v) R.q[v] = b0[v];
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const double g1 = 3.0 * b0[v] - 3.0 * b1[v] + b2[v];
                    R.q[v] = (gd == 1) ? g1 : 3.0 * g1 - 3.0 * b0[v] + b1[v];
                }
            }
        };
        // Row jr of the window, for any jr in [-2, nj+1].

        // ---- j-direction helpers -------------------------------------------------------
        auto slope_j = [&](const Row& A_, const Row& B_, ST* s) {
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = iface_slope<ST>(A_.q[v], B_.q[v], A_.dlj, B_.dlj);
        };
        auto sigma = [&](const ST* fw, const ST* bw, ST* sg) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if constexpr (PREC == 0) sg[v] = lim64<LIM>(fw[v], bw[v]);
                else sg[v] = lim32<LIM>(fw[v], bw[v]);
            }
        };
        // j-face flux above row jb (1-based face G = jb+1) from rows jb (L) and jb+1 (R).
        auto jface = [&](int G, const Row& L_, const Row& R_, const ST* sgL, const ST* sgR, const double* intr,
                         double intr_dl, double* X) {
            // intr / intr_dl: the interior neighbour of the boundary row (BC faces only)
#pragma unroll
            for (int v = 0; v < 4; ++v) X[v] = 0.0;
            if (!inI) return;
            const long long fidx = B.ofj + (long long)G * ni + c;
            const double nx = a.fj[fidx], ny = a.fj[fidx + B.pfj], ln = a.fj[fidx + 2 * B.pfj];
            int etype = 101, Fm = 0;
            if (G == 0) { etype = eBot.type; Fm = 3; }
            else if (G == nj) { etype = eTop.type; Fm = 4; }
            if (etype == 101) {
                double QL[4], QR[4];
                const double lm = 0.5 * L_.dlj, lp = 0.5 * R_.dlj;
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    QL[v] = L_.q[v] + (double)(1.0 * sgL[v] * lm);
                    QR[v] = R_.q[v] - (double)(1.0 * sgR[v] * lp);
                }
                if (!face_flux<PREC, RIEM>(g, QL, QR, nx, ny, ln, X))
                    record_error(cs, 4, B.local_b, c + 1, G, a.irk);
            } else if (etype >= 0) {
                const Row& bnd = (Fm == 3) ? R_ : L_;
                Q4 Bp, Ip;
#pragma unroll
                for (int v = 0; v < 4; ++v) { Bp.v[v] = bnd.q[v]; Ip.v[v] = intr[v]; }
                const int prm = (Fm == 3) ? eBot.param : eTop.param;
                const Q4 q = bc_face<RIEM>(g, a.limiter, etype, Fm, Bp, Ip, bnd.dlj, intr_dl,
                                           nx, ny, ln, prm >= 0 ? a.bcp + prm : nullptr);
#pragma unroll
                for (int v = 0; v < 4; ++v) X[v] = q.v[v];
            }
        };

        // ---- warm-up: rows r0-2 .. r0+1 -------------------------------------------------
        Row rm2{{0.0, 0.0, 0.0, 0.0}, 1.0, 1.0}, rm1{{0.0, 0.0, 0.0, 0.0}, 1.0, 1.0};
        Row rA, rB, rC;
        if (r0 >= 2) {
            load_row(r0 - 2, rm2);
            load_row(r0 - 1, rm1);
        }
        load_row(r0, rA);
        if (r0 + 1 < nj) load_row(r0 + 1, rB);
        if (r0 + 2 < nj) load_row(r0 + 2, rC);
        if (r0 + 1 >= nj) {   // top ghost rows inside the warm-up window (thin blocks)
            ghost_row(eTop, 4, 1, rA.q, rm1.q, rm2.q, rB);
            load_dl(r0 + 1, rB);
        }
        if (r0 + 2 >= nj) {
            const Row& b0 = (r0 + 2 == nj) ? rB : rA;
            const Row& b1 = (r0 + 2 == nj) ? rA : rm1;
            const Row& b2 = (r0 + 2 == nj) ? rm1 : rm2;
            ghost_row(eTop, 4, r0 + 2 - nj + 1, b0.q, b1.q, b2.q, rC);
            load_dl(r0 + 2, rC);
        }
        if (r0 == 0) {   // bottom ghost rows from rows 0..2
            ghost_row(eBot, 3, 1, rA.q, rB.q, rC.q, rm1);
            ghost_row(eBot, 3, 2, rA.q, rB.q, rC.q, rm2);
            load_dl(-1, rm1);
            load_dl(-2, rm2);
        } else if (r0 == 1) {
            // row -1 is a ghost of layer 1 (rm2), row 0 interior (rm1)
            load_row(0, rm1);
            ghost_row(eBot, 3, 1, rm1.q, rA.q, rB.q, rm2);
            load_dl(-1, rm2);
        }
        ST s_m32[4], s_m12[4], s_p12[4], sg_m1[4], sg_0[4];
        slope_j(rm2, rm1, s_m32);
        slope_j(rm1, rA, s_m12);
        slope_j(rA, rB, s_p12);
        sigma(s_m12, s_m32, sg_m1);
        sigma(s_p12, s_m12, sg_0);
        double Gm[4];
        jface(r0, rm1, rA, sg_m1, sg_0, rB.q, rB.dlj, Gm);   // face below row r0 (BC face 3 when r0 == 0)
        // carried: s(j+1/2) = s_p12, sigma(j) = sg_0

        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        const double dt_case = __ldcg(&cs->dt_step);
        const long long iter_next = __ldcg(&cs->iter) + (a.first ? 1 : 0) + 1;
        const int ndir = a.cases[w.case_id].ndir;
        const bool iEdgeL = (w.i0 == 0), iEdgeR = (w.i0 + 29 >= ni);

        for (int j = r0; j < r1; ++j) {
            // ---- row j+2 (rC) : loaded ahead except in the warm-up step ----------------------
            if (j > r0) {
                const int jr = j + 2;
                if (jr < nj) load_row(jr, rC);
                else {
                    if (jr == nj) {
                        // extrapolation needs row nj-3 = j-1
                        double q3[4] = {0.0, 0.0, 0.0, 0.0};
                        if (inI && nj >= 3) {
                            const double* src = Pin + (long long)(nj - 3) * ni + c;
#pragma unroll
                            for (int v = 0; v < 4; ++v) q3[v] = src[v * pc];
                        }
                        ghost_row(eTop, 4, 1, rB.q, rA.q, q3, rC);
                    } else {
                        ghost_row(eTop, 4, 2, rA.q, rA.q, rA.q, rC);   // unused unless 101
                        if (eTop.type != 101) {
#pragma unroll
                            for (int v = 0; v < 4; ++v) rC.q[v] = rB.q[v];
                        }
                    }
                    load_dl(jr, rC);
                }
            }
            // ---- j-direction: slope, limited slope and the face above row j --------------
            ST s_p32[4], sg_1[4];
            slope_j(rB, rC, s_p32);
            sigma(s_p32, s_p12, sg_1);
            double Gp[4];
            {
                // interior neighbour for a top BC face (row nj-2)
                double intr[4] = {0.0, 0.0, 0.0, 0.0};
                double intr_dl = 1.0;
                if (j + 1 == nj && inI && eTop.type != 101 && eTop.type >= 0) {
                    // interior neighbour of the top boundary row (row nj-2; the top ghost for nj = 1,
                    // which is this window's row j+2)
                    if (nj >= 2) {
                        const double* src = Pin + (long long)(nj - 2) * ni + c;
#pragma unroll
                        for (int v = 0; v < 4; ++v) intr[v] = src[v * pc];
                        intr_dl = a.dl[B.og + (long long)(nj - 2 + 2) * (ni + 4) + (c + 2) + B.pg];
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) intr[v] = rC.q[v];
                        intr_dl = rC.dlj;
                    }
                }
                jface(j + 1, rA, rB, sg_0, sg_1, intr, intr_dl, Gp);
            }

            // ---- i-direction on row j ----------------------------------------------------
            double qR[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) qR[v] = __shfl_down_sync(kFull, rA.q[v], 1);
            const double dlR = __shfl_down_sync(kFull, rA.dli, 1);
            ST si[4], siL[4], sgi[4], sgiR[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) si[v] = iface_slope<ST>(rA.q[v], qR[v], rA.dli, dlR);
#pragma unroll
            for (int v = 0; v < 4; ++v) siL[v] = __shfl_up_sync(kFull, si[v], 1);
            sigma(si, siL, sgi);
#pragma unroll
            for (int v = 0; v < 4; ++v) sgiR[v] = __shfl_down_sync(kFull, sgi[v], 1);
            double Fi[4] = {0.0, 0.0, 0.0, 0.0};
            const int F = c + 1;   // 1-based index of the face between this lane's column and the next
            const bool faceValid = (F >= 0 && F <= ni);
            int ietype = 101, iFm = 0;
            if (faceValid && (F == 0 || F == ni)) {
                iFm = (F == 0) ? 1 : 2;
                ietype = a.edges[B.eo[iFm - 1] + j].type;
            }
            double nx = 0.0, ny = 0.0, ln = 0.0;
            if (faceValid) {
                const long long fidx = B.ofi + (long long)j * (ni + 1) + F;
                nx = a.fi[fidx]; ny = a.fi[fidx + B.pfi]; ln = a.fi[fidx + 2 * B.pfi];
            }
            if (faceValid && ietype == 101) {
                double QL[4], QR[4];
                const double lm = 0.5 * rA.dli, lp = 0.5 * dlR;
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    QL[v] = rA.q[v] + (double)(1.0 * sgi[v] * lm);
                    QR[v] = qR[v] - (double)(1.0 * sgiR[v] * lp);
                }
                if (!face_flux<PREC, RIEM>(g, QL, QR, nx, ny, ln, Fi) && lane >= 1 && lane < 30)
                    record_error(cs, 4, B.local_b, F, j + 1, a.irk);
            }
            if (iEdgeL || iEdgeR) {   // warp-uniform: boundary i-faces by their BC routine
                double q2R[4], qLn[4];
                double dl2R = __shfl_down_sync(kFull, rA.dli, 2);
                double dlLn = __shfl_up_sync(kFull, rA.dli, 1);
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    q2R[v] = __shfl_down_sync(kFull, rA.q[v], 2);
                    qLn[v] = __shfl_up_sync(kFull, rA.q[v], 1);
                }
                if (faceValid && ietype != 101 && ietype >= 0) {
                    Q4 Bp, Ip;
                    double dlb, dli;
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        Bp.v[v] = (iFm == 1) ? qR[v] : rA.q[v];
                        Ip.v[v] = (iFm == 1) ? q2R[v] : qLn[v];
                    }
                    dlb = (iFm == 1) ? dlR : rA.dli;
                    dli = (iFm == 1) ? dl2R : dlLn;
                    const int prm = a.edges[B.eo[iFm - 1] + j].param;
                    const Q4 q = bc_face<RIEM>(g, a.limiter, ietype, iFm, Bp, Ip, dlb, dli, nx, ny, ln,
                                               prm >= 0 ? a.bcp + prm : nullptr);
#pragma unroll
                    for (int v = 0; v < 4; ++v) Fi[v] = q.v[v];
                }
            }
            double FiL[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) FiL[v] = __shfl_up_sync(kFull, Fi[v], 1);

            // ---- residual, sources, RK update of row j --------------------------------------
            if (useful) {
                const int i1 = c + 1, j1 = j + 1;
                double r[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    double x = 0.0;
                    if (i1 > 1) x = x - FiL[v];
                    if (i1 < ni) x = x + Fi[v];
                    if (j1 > 1) x = x - Gm[v];
                    if (j1 < nj) x = x + Gp[v];
                    if (i1 == 1) x = x - FiL[v];
                    if (i1 == ni) x = x + Fi[v];
                    if (j1 == 1) x = x - Gm[v];
                    if (j1 == nj) x = x + Gp[v];
                    r[v] = x;
                }
                const long long cg = (long long)j * ni + c;
                const double sur = scb[cg];
                const double* P = rA.q;
                if (a.source == 1) {
                    const double invr = scb[6 * pc + cg];
                    const double mod_v = sqrt(P[1] * P[1] + P[2] * P[2]);
                    double S[4];
                    S[0] = -P[0] * P[2] * invr;
                    S[1] = -P[0] * P[1] * P[2] * invr;
                    S[2] = -P[0] * P[2] * P[2] * invr;
                    S[3] = -(P[0] * E0(g, P[3], P[0], mod_v) + P[3]) * P[2] * invr;
#pragma unroll
                    for (int v = 0; v < 4; ++v) r[v] = r[v] - S[v] * sur;
                } else if (a.source == 2) {
                    const double Gx = scb[6 * pc + cg], Gy = scb[7 * pc + cg];
                    const double mod_v = sqrt(P[1] * P[1] + P[2] * P[2]);
                    const double VG = P[1] * Gx + P[2] * Gy;
                    double S[4];
                    S[0] = P[0] * VG;
                    S[1] = P[0] * P[1] * VG;
                    S[2] = P[0] * P[2] * VG;
                    S[3] = (P[0] * E0(g, P[3], P[0], mod_v) + P[3]) * VG;
#pragma unroll
                    for (int v = 0; v < 4; ++v) r[v] = r[v] - S[v] * sur;
                }
                const double dt = a.time_accurate ? dt_case : scb[pc + cg];
                double PO[4];
                if (a.first) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) PO[v] = P[v];
                } else {
                    const double* po = a.PO + B.oc + cg;
#pragma unroll
                    for (int v = 0; v < 4; ++v) PO[v] = po[v * pc];
                }
                double res[4];
                if (PREC == 0) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) res[v] = -r[v] / sur * dt * 1.0;
                } else {
                    const double fct = -dt / sur;
#pragma unroll
                    for (int v = 0; v < 4; ++v) res[v] = r[v] * fct;
                }
                double U0[4], U[4];
                U0[0] = PO[0]; U0[1] = PO[0] * PO[1]; U0[2] = PO[0] * PO[2];
                U[0] = P[0]; U[1] = P[0] * P[1]; U[2] = P[0] * P[2];
                if (PREC == 0) {
                    U0[3] = PO[3] / g.gm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
                    U[3] = P[3] / g.gm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
                } else {
                    U0[3] = PO[3] * g.igm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
                    U[3] = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) U[v] = U0[v] + (U[v] - U0[v] + res[v]) * a.rk_c;
                double N[4];
                N[0] = U[0];
                if (PREC == 0) {
                    N[1] = U[1] / U[0];
                    N[2] = U[2] / U[0];
                } else {
                    const double ir = 1.0 / U[0];
                    N[1] = U[1] * ir;
                    N[2] = U[2] * ir;
                }
                N[3] = g.gm1 * (U[3] - 0.5 * U[0] * (N[1] * N[1] + N[2] * N[2]));
                if (isnan(N[0]) || isnan(N[1]) || isnan(N[2]) || isnan(N[3]) || N[3] < 0.0)
                    record_error(cs, 5, B.local_b, i1, j1, a.irk);
                if (N[0] < 1e-20) N[0] = 1e-20;
                double* po = a.Pout + B.oc + cg;
#pragma unroll
                for (int v = 0; v < 4; ++v) po[v * pc] = N[v];
                if (a.last) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const double d = fabs(N[v] - PO[v]);
                        acc[v] += d * d;
                    }
                    const double dtn = cell_dt(a, N, scb, cg, pc, rA.dli, rA.dlj, ndir, iter_next);
                    if (!a.time_accurate) a.sc[2 * B.oc + pc + cg] = dtn;
                    acc[4] = fmin(acc[4], dtn);
                }
            }
            // ---- shift the window ----------------------------------------------------------
            rA = rB;
            rB = rC;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                s_p12[v] = s_p32[v];
                sg_0[v] = sg_1[v];
                Gm[v] = Gp[v];
            }
        }
        // per-item partials (fixed shuffle tree), then the case finalisation
        if (a.last) {
#pragma unroll
            for (int k = 0; k < 5; ++k)
                for (int o = 16; o > 0; o >>= 1) {
                    const double wv = __shfl_down_sync(kFull, acc[k], o);
                    acc[k] = (k < 4) ? acc[k] + wv : fmin(acc[k], wv);
                }
        }
        warp_item_done(a, w.case_id, acc, it, a.last != 0, a.last != 0, a.first != 0);
    }
}

template <int PREC, int RIEM>
cudaError_t launch_march_t(const StageArgs& a, int lim, int grid, cudaStream_t s) {
    switch (lim) {
        case 0: march_kernel<PREC, RIEM, 0><<<grid, 128, 0, s>>>(a); break;
        case 1: march_kernel<PREC, RIEM, 1><<<grid, 128, 0, s>>>(a); break;
        case 2: march_kernel<PREC, RIEM, 2><<<grid, 128, 0, s>>>(a); break;
        case 3: march_kernel<PREC, RIEM, 3><<<grid, 128, 0, s>>>(a); break;
        case 4: march_kernel<PREC, RIEM, 4><<<grid, 128, 0, s>>>(a); break;
        case 5: march_kernel<PREC, RIEM, 5><<<grid, 128, 0, s>>>(a); break;
        default: march_kernel<PREC, RIEM, 6><<<grid, 128, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

template <int PREC, int RIEM>
int march_occupancy_t(int lim) {
    int n = 0;
    switch (lim) {
        case 0: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 0>, 128, 0); break;
        case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 1>, 128, 0); break;
        case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 2>, 128, 0); break;
        case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 3>, 128, 0); break;
        case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 4>, 128, 0); break;
        case 5: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 5>, 128, 0); break;
        default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, march_kernel<PREC, RIEM, 6>, 128, 0); break;
    }
    return n;
}

}  // namespace q2d
