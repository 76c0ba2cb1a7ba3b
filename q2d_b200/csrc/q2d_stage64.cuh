// q2d_stage64.cuh — the fused RK-stage kernel of the Q2D explicit path (sm_100a), FP64 form.
//
// One launch runs one RK stage for every running case of a context. Each CTA takes work items
// (a TX x TY tile of one block) in a grid-stride loop and, per tile:
//   1. stages the primitive state of the tile plus a 2-cell cross-shaped halo in shared memory;
//      halo cells outside the block are the ghost cells of Fill_Ghost_Cell
//      (Lib_Ghost.f90:16-299), computed on the fly: block-interface (101) ghosts are read from
//      the donor block's HBM state (the device-side block-interface copy that replaces the MPI
//      halo exchange of Mod_GhostExchange.f90), the others follow Ghost_Symmetry /
//      Ghost_ZG_Extrapolate / Ghost_Extrapolate from the tile's own cells;
//   2. computes every i- and j-face flux of the tile once (interior faces: MUSCL reconstruction
//      + Riemann solver, Convective_Flux, Lib_Convective.f90:15-82; block-boundary faces: the
//      BC_Fluxes routine of the face's record, Mod_BC_Fluxes.f90:79-269);
//   3. per cell, accumulates the residual in the reference order (interior i-faces, interior
//      j-faces, boundary faces 1..4; Mod_Fluxes.f90:122-232 then Mod_BC_Fluxes.f90:79-84),
//      subtracts the geometric source (Mod_Sources.f90:79-91), applies Newstate_Conservative
//      with the RK stage (Lib_Newstate.f90:131-159, Lib_RK.f90:15-27) and Check_And_Fix_State;
//   4. on the last stage, also computes the cell's time step for the next step (Compute_dt,
//      Mod_dt.f90:59-104) and its squared change (Compute_Residual, Mod_Diagnostic.f90:438-469),
//      reduced per tile with warp shuffles and per case by the last CTA to finish the case
//      (summed in item order, so the result does not depend on scheduling).
// No spin-waits: cross-CTA ordering uses only atomic counters observed by the last CTA.
#pragma once
#include "q2d_kernels.cuh"
#include "q2d_common.cuh"

#include <cfloat>
#include <type_traits>

namespace q2d {

// Shared-memory layout of one tile (offsets in doubles).
template <int PREC, int TX, int TY, bool SD>
struct Tile {
    using ST = typename std::conditional<PREC == 0, double, float>::type;
    static constexpr int W = TX + 4, H = TY + 4, AREA = W * H;
    static constexpr int NSI = (TX + 3) * TY, NSJ = TX * (TY + 3);   // interfaces
    static constexpr int NGI = (TX + 2) * TY, NGJ = TX * (TY + 2);   // limited cell slopes
    static constexpr int NFI = (TX + 1) * TY, NFJ = TX * (TY + 1);   // faces
    static constexpr int NC = TX * TY;                               // cells
    static constexpr int oP = 0;                        // [4][H][W] primitive state + ghosts
    static constexpr int oD = oP + 4 * AREA;            // [2][H][W] mean lengths dl(1), dl(2)
    static constexpr int oC = oD + 2 * AREA;            // [6][NC]   U^n (4), sur, dt
    static constexpr int oG = oC + 6 * NC;              // [3][NFI] + [3][NFJ] face nx, ny, len
    static constexpr int nS = (int)((4 * (NSI + NSJ) * sizeof(ST) + 7) / 8);
    static constexpr int nF = 4 * (NFI + NFJ);
    static constexpr int oS = oG + 3 * (NFI + NFJ);     // interface slopes (ST), then face fluxes
    static constexpr int oSG = oS + (nS > nF ? nS : nF);
    static constexpr int nSG = (int)((4 * (NGI + NGJ) * sizeof(ST) + 7) / 8);
    // MUSCL-SD: the shock sensor of the tile's cells and of the halo column / row on its left and
    // lower faces, [(TY+1)][(TX+1)] with offset 1
    static constexpr int NB = SD ? (TX + 1) * (TY + 1) : 0;
    static constexpr int oB = oSG + nSG;
    static constexpr int total = oB + NB;
    static constexpr size_t bytes = sizeof(double) * (size_t)total;
};

// Limited cell slopes of a tile (step 4 of the stage kernel), one limiter per instantiation.
template <int LIM, int NT, int TX, int TY, typename ST>
__device__ __forceinline__ void sigma_phase(const ST* sSi, const ST* sSj, ST* sGI, ST* sGJ) {
    constexpr int NSI = (TX + 3) * TY, NSJ = TX * (TY + 3);
    constexpr int NGI = (TX + 2) * TY, NGJ = TX * (TY + 2);
    for (int k = threadIdx.x; k < NGI; k += NT) {
        const int r = k / (TX + 2), c = k - r * (TX + 2);   // cell at smem column c+1
        const int sfw = r * (TX + 3) + c + 1;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if constexpr (sizeof(ST) == 8) sGI[v * NGI + k] = lim64<LIM>(sSi[v * NSI + sfw], sSi[v * NSI + sfw - 1]);
            else sGI[v * NGI + k] = lim32<LIM>(sSi[v * NSI + sfw], sSi[v * NSI + sfw - 1]);
        }
    }
    // the j slopes start on the warp after the one that took the last i slopes (no barrier in
    // between): no warp gets two partial rounds
    constexpr int NW = NT / 32, ROT = ((NGI + 31) / 32) % NW;
    for (int k = (((int)(threadIdx.x >> 5) - ROT + NW) % NW) * 32 + (int)(threadIdx.x & 31); k < NGJ; k += NT) {
        const int r = k / TX, c = k - r * TX;               // cell at smem row r+1
        const int sfw = (r + 1) * TX + c, sbw = r * TX + c;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if constexpr (sizeof(ST) == 8) sGJ[v * NGJ + k] = lim64<LIM>(sSj[v * NSJ + sfw], sSj[v * NSJ + sbw]);
            else sGJ[v * NGJ + k] = lim32<LIM>(sSj[v * NSJ + sfw], sSj[v * NSJ + sbw]);
        }
    }
}

// Face fluxes of one direction of a tile (step 5 of the stage kernel). IDIR: i-faces
// (F = i0..i0+TX on TY rows) or j-faces (G = j0..j0+TY on TX columns).
// SD: the shock sensor sB runs (MUSCL-SD or a sensor-driven Riemann solver); an interior face
// takes it from its left / lower cell (Mod_Fluxes.f90:140-204), a block-interface face from its
// boundary cell (Lib_BC_Fluxes_Connection.f90, beta_ = blk%beta(Im,Jm)). It scales both limited
// slopes under MUSCL-SD (a.sd) and goes to the Riemann solver.
template <int PREC, int RIEM, bool IDIR, int NT, int TX, int TY, bool SD, typename ST>
__device__ __forceinline__ void face_phase(const StageArgs& a, const Gas& g, const DBlock& B, CaseState* cs, int i0,
                                           int j0, const double* sP, const double* sD,
                                           const double* sG, const ST* sg, const double* sB, double* sF) {
    constexpr int W = TX + 4, AREA = W * (TY + 4);
    constexpr int NF = IDIR ? (TX + 1) * TY : TX * (TY + 1);
    constexpr int NG = IDIR ? (TX + 2) * TY : TX * (TY + 2);
    constexpr int ROWLEN = IDIR ? TX + 1 : TX;
    constexpr int DSTEP = IDIR ? 1 : W;
    const int ni = B.ni, nj = B.nj;
    const double* dlp = sD + (IDIR ? 0 : AREA);
    // j-faces start on the warp after the one that took the last i-faces (the two directions
    // run back to back with no barrier): every warp has at most ceil((NFI + NFJ) / NT) rounds
    constexpr int NW = NT / 32, ROT = IDIR ? 0 : (((TX + 1) * TY + 31) / 32) % NW;
    for (int f = (((int)(threadIdx.x >> 5) - ROT + NW) % NW) * 32 + (int)(threadIdx.x & 31); f < NF; f += NT) {
        const int row = f / ROWLEN, col = f - row * ROWLEN;
        int pos, lenn, k;        // face index along the direction, its limit, edge position
        if (IDIR) { pos = i0 + col; lenn = ni; k = j0 + row; if (k >= nj || pos > ni) continue; }
        else      { pos = j0 + row; lenn = nj; k = i0 + col; if (k >= ni || pos > nj) continue; }
        const double nx = sG[f], ny = sG[NF + f], ln = sG[2 * NF + f];
        const int pL = IDIR ? (row + 2) * W + col + 1 : (row + 1) * W + col + 2;   // left cell
        double X[4];
        int etype = 101, Fm = 0;
        if (pos == 0 || pos == lenn) {
            Fm = IDIR ? (pos == 0 ? 1 : 2) : (pos == 0 ? 3 : 4);
            etype = a.edges[B.eo[Fm - 1] + k].type;
        }
        if (etype == 101) {
            const int gL = IDIR ? row * (TX + 2) + col : row * TX + col;
            const int gR = gL + (IDIR ? 1 : TX);
            const double lm = 0.5 * dlp[pL], lp = 0.5 * dlp[pL + DSTEP];
            double beta = 1.0, beta_l = 1.0;   // the sensor; its value for the slopes (MUSCL-SD)
            if (SD) {   // cell (col - 1, row) for i-faces, (col, row - 1) for j-faces
                const int bL = IDIR ? (row + 1) * (TX + 1) + col : row * (TX + 1) + col + 1;
                beta = sB[Fm == 1 || Fm == 3 ? bL + (IDIR ? 1 : TX + 1) : bL];
                if (a.sd) beta_l = beta;
            }
            double QL[4], QR[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                QL[v] = sP[v * AREA + pL] + (double)(beta_l * sg[v * NG + gL] * lm);
                QR[v] = sP[v * AREA + pL + DSTEP] - (double)(beta_l * sg[v * NG + gR] * lp);
            }
            if (!face_flux<PREC, RIEM>(g, QL, QR, nx, ny, ln, X, beta))
                record_error(cs, 4, B.local_b, IDIR ? pos : k + 1, IDIR ? k + 1 : pos, a.irk);
        } else if (etype >= 0) {
            const bool minside = (Fm == 1 || Fm == 3);
            const int cb = minside ? pL + DSTEP : pL;         // boundary cell
            const int ci = minside ? cb + DSTEP : cb - DSTEP; // interior neighbour
            Q4 Bp, Ip;
#pragma unroll
            for (int v = 0; v < 4; ++v) { Bp.v[v] = sP[v * AREA + cb]; Ip.v[v] = sP[v * AREA + ci]; }
            const int prm = a.edges[B.eo[Fm - 1] + k].param;
            const Q4 q = bc_face<RIEM>(g, a.limiter, etype, Fm, Bp, Ip, dlp[cb], dlp[ci], nx, ny, ln,
                                       prm >= 0 ? a.bcp + prm : nullptr);
#pragma unroll
            for (int v = 0; v < 4; ++v) X[v] = q.v[v];
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) X[v] = 0.0;
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) sF[v * NF + f] = X[v];
    }
}

// TAB: the thermally perfect gas (a.gas.htab set); without it the calorically perfect closure
// is fixed at compile time.
template <int PREC, int RIEM, int TX, int TY, int NT, bool SD, bool TAB = false>
__global__ void __launch_bounds__(NT, 2) stage_kernel(const StageArgs a) {
    using L = Tile<PREC, TX, TY, SD>;
    using ST = typename L::ST;
    constexpr int W = L::W, AREA = L::AREA, NFI = L::NFI, NFJ = L::NFJ, NSI = L::NSI, NSJ = L::NSJ,
                  NGI = L::NGI, NC = L::NC;
    extern __shared__ double smem[];
    double* sP = smem + L::oP;
    double* sD = smem + L::oD;
    double* sC = smem + L::oC;
    double* sGi = smem + L::oG;            // i-face geometry [3][NFI]
    double* sGj = sGi + 3 * NFI;           // j-face geometry [3][NFJ]
    ST* sSi = reinterpret_cast<ST*>(smem + L::oS);   // [4][NSI]
    ST* sSj = sSi + 4 * NSI;                          // [4][NSJ]
    double* sFi = smem + L::oS;            // [4][NFI] (aliases the slopes once they are consumed)
    double* sFj = sFi + 4 * NFI;           // [4][NFJ]
    ST* sGI = reinterpret_cast<ST*>(smem + L::oSG);  // [4][NGI]
    ST* sGJ = sGI + 4 * NGI;                          // [4][NGJ]
    double* sB = smem + L::oB;                        // [(TY+1)][(TX+1)] shock sensor
    __shared__ double red[(NT / 32) * 5];
    __shared__ double tile_part[5];
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    Gas g = a.gas;
    if (!TAB) g.htab = nullptr;
    const int lim = a.limiter;

    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x) {
        const WorkItem w = a.items[it];
        const DBlock B = a.blocks[w.block];
        CaseState* cs = &a.cstate[w.case_id];
        if (__ldcg(&cs->status) != kStatus_Running) continue;   // uniform over the CTA
        const int ni = B.ni, nj = B.nj, i0 = w.i0, j0 = w.j0;
        const double* Pin = a.Pin + B.oc;
        const long long pc = B.pc;
        const double* scb = a.sc + 2 * B.oc;   // 8-plane scalar pool of the block

        const int irs = a.irs_mode;
        double* sR = sFi;   // mode 2: the smoothed residual [4][NC] (NFI >= NC), no faces computed
        if (irs == 2) {
            for (int k = tid; k < NC; k += NT) {
                const int row = k / TX, col = k - row * TX;
                const int ii = i0 + col, jj = j0 + row;
                if (ii >= ni || jj >= nj) continue;
                const long long cg = (long long)jj * ni + ii;
                const int sidx = (row + 2) * W + (col + 2);
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    cp_async8(sP + v * AREA + sidx, Pin + v * pc + cg);
                    cp_async8(sC + v * NC + k, a.PO + B.oc + v * pc + cg);
                    cp_async8(sR + v * NFI + k, a.Rin + B.oc + v * pc + cg);
                }
                if (a.last) {   // cell lengths of the next step's time step
                    const double* src = a.dl + B.og + (long long)(jj + 2) * (ni + 4) + (ii + 2);
                    cp_async8(sD + sidx, src);
                    cp_async8(sD + AREA + sidx, src + B.pg);
                }
            }
        } else {
            // ---- 1. asynchronous loads of everything the tile reads --------------------------
            for (int idx = tid; idx < AREA; idx += NT) {
                const int r = idx / W, c = idx - r * W;
                if ((r < 2 || r >= TY + 2) && (c < 2 || c >= TX + 2)) continue;
                const int ii = i0 - 2 + c, jj = j0 - 2 + r;
                const bool inI = (ii >= 0 && ii < ni), inJ = (jj >= 0 && jj < nj);
                if (ii >= -2 && ii <= ni + 1 && jj >= -2 && jj <= nj + 1) {
                    const double* src = a.dl + B.og + (long long)(jj + 2) * (ni + 4) + (ii + 2);
                    cp_async8(sD + idx, src);
                    cp_async8(sD + AREA + idx, src + B.pg);
                }
                if (inI && inJ) {
                    const double* src = Pin + (long long)jj * ni + ii;
#pragma unroll
                    for (int v = 0; v < 4; ++v) cp_async8(sP + v * AREA + idx, src + v * pc);
                } else if (inI != inJ) {   // every ghost the tile's faces read, from HBM
                    double q[4];
                    if (ghost_value(a, B, ii, jj, q)) {
#pragma unroll
                        for (int v = 0; v < 4; ++v) sP[v * AREA + idx] = q[v];
                    }
                }
            }
            if (SD && tid < 3) {   // the halo corners the sensor's edge cells read (pressure)
                const int ii = tid == 1 ? i0 + TX : i0 - 1, jj = tid == 2 ? j0 + TY : j0 - 1;
                const bool need = tid == 0 ? (i0 > 0 || j0 > 0)
                                : tid == 1 ? (j0 > 0 && i0 + TX <= ni) : (i0 > 0 && j0 + TY <= nj);
                const int idx = (jj - j0 + 2) * W + (ii - i0 + 2);
                if (need) {
                    if (ii >= 0 && ii < ni && jj >= 0 && jj < nj) {
                        cp_async8(sP + 3 * AREA + idx, Pin + 3 * pc + (long long)jj * ni + ii);
                    } else {
                        double q[4];
                        if (ghost_value(a, B, ii, jj, q)) sP[3 * AREA + idx] = q[3];
                    }
                }
            }
            for (int k = tid; k < NC; k += NT) {
                const int row = k / TX, col = k - row * TX;
                const int ii = i0 + col, jj = j0 + row;
                if (ii >= ni || jj >= nj) continue;
                const long long cg = (long long)jj * ni + ii;
                cp_async8(sC + 4 * NC + k, scb + cg);                                  // sur
                if (!a.time_accurate) cp_async8(sC + 5 * NC + k, scb + pc + cg);       // dt
                if (!a.first) {
                    const double* po = a.PO + B.oc + cg;
#pragma unroll
                    for (int v = 0; v < 4; ++v) cp_async8(sC + v * NC + k, po + v * pc);
                }
            }
            for (int f = tid; f < NFI + NFJ; f += NT) {
                if (f < NFI) {
                    const int row = f / (TX + 1), col = f - row * (TX + 1);
                    const int jj = j0 + row, F = i0 + col;
                    if (jj >= nj || F > ni) continue;
                    const double* src = a.fi + B.ofi + (long long)jj * (ni + 1) + F;
#pragma unroll
                    for (int q = 0; q < 3; ++q) cp_async8(sGi + q * NFI + f, src + q * B.pfi);
                } else {
                    const int ff = f - NFI;
                    const int row = ff / TX, col = ff - row * TX;
                    const int ii = i0 + col, G = j0 + row;
                    if (ii >= ni || G > nj) continue;
                    const double* src = a.fj + B.ofj + (long long)G * ni + ii;
#pragma unroll
                    for (int q = 0; q < 3; ++q) cp_async8(sGj + q * NFJ + ff, src + q * B.pfj);
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();

        if (irs != 2) {
            // ---- 3. interface slopes ---------------------------------------------------------
            for (int k = tid; k < NSI + NSJ; k += NT) {
                if (k < NSI) {
                    const int r = k / (TX + 3), c = k - r * (TX + 3);
                    const int p0 = (r + 2) * W + c;
                    const double da = sD[p0], db = sD[p0 + 1];
                    if constexpr (sizeof(ST) == 8) {   // one reciprocal of the interface distance
                        const double inv = 1.0 / (0.5 * (da + db));
#pragma unroll
                        for (int v = 0; v < 4; ++v) sSi[v * NSI + k] = (sP[v * AREA + p0 + 1] - sP[v * AREA + p0]) * inv;
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            sSi[v * NSI + k] = iface_slope<ST>(sP[v * AREA + p0], sP[v * AREA + p0 + 1], da, db);
                    }
                } else {
                    const int kk = k - NSI;
                    const int r = kk / TX, c = kk - r * TX;
                    const int p0 = r * W + c + 2;
                    const double da = sD[AREA + p0], db = sD[AREA + p0 + W];
                    if constexpr (sizeof(ST) == 8) {
                        const double inv = 1.0 / (0.5 * (da + db));
#pragma unroll
                        for (int v = 0; v < 4; ++v) sSj[v * NSJ + kk] = (sP[v * AREA + p0 + W] - sP[v * AREA + p0]) * inv;
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            sSj[v * NSJ + kk] = iface_slope<ST>(sP[v * AREA + p0], sP[v * AREA + p0 + W], da, db);
                    }
                }
            }
            if (SD) {   // SD_Tramel of the cells whose faces the tile computes (Mod_Fluxes.f90:132-138)
                for (int k = tid; k < L::NB; k += NT) {
                    const int r = k / (TX + 1) - 1, c = k - (r + 1) * (TX + 1) - 1;
                    if ((r < 0 && (c < 0 || j0 == 0)) || (c < 0 && i0 == 0) || i0 + c >= ni || j0 + r >= nj)
                        continue;
                    const double* pp = sP + 3 * AREA + (r + 2) * W + (c + 2);
                    sB[k] = sd_tramel(pp[0], pp[-1], pp[1], pp[-W], pp[W]);
                }
            }
            __syncthreads();

            // ---- 4. limited slope of every cell next to a face of the tile -------------------
            switch (lim) {
                case 0: sigma_phase<0, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                case 1: sigma_phase<1, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                case 2: sigma_phase<2, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                case 3: sigma_phase<3, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                case 4: sigma_phase<4, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                case 5: sigma_phase<5, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
                default: sigma_phase<6, NT, TX, TY>(sSi, sSj, sGI, sGJ); break;
            }
            __syncthreads();

            // ---- 5. face fluxes (interior: Riemann on MUSCL states; boundary: BC_Fluxes) -----
            face_phase<PREC, RIEM, true, NT, TX, TY, SD>(a, g, B, cs, i0, j0, sP, sD, sGi, sGI, sB, sFi);
            face_phase<PREC, RIEM, false, NT, TX, TY, SD>(a, g, B, cs, i0, j0, sP, sD, sGj, sGJ, sB, sFj);
        }
        __syncthreads();

        // ---- 6. residual, sources, RK update (+ next dt and residual norm) ----------------
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        const double dt_case = __ldcg(&cs->dt_step);
        const long long iter_next = __ldcg(&cs->iter) + (a.first ? 1 : 0) + 1;
        const int ndir = a.cases[w.case_id].ndir;
        for (int k = tid; k < NC; k += NT) {
            const int row = k / TX, col = k - row * TX;
            const int ii = i0 + col, jj = j0 + row;
            if (ii >= ni || jj >= nj) continue;
            const int i1 = ii + 1, j1 = jj + 1;
            const int sidx = (row + 2) * W + (col + 2);
            const int fi0 = row * (TX + 1) + col, fj0 = row * TX + col;
            const long long cg = (long long)jj * ni + ii;
            double P[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) P[v] = sP[v * AREA + sidx];
            double res[4];   // the scaled residual -R / sur * dt of the update
            if (irs == 2) {
#pragma unroll
                for (int v = 0; v < 4; ++v) res[v] = sR[v * NFI + k];
            } else {
            double r[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const double* Fi = sFi + v * NFI;
                const double* Fj = sFj + v * NFJ;
                double x = 0.0;
                if (i1 > 1) x = x - Fi[fi0];
                if (i1 < ni) x = x + Fi[fi0 + 1];
                if (j1 > 1) x = x - Fj[fj0];
                if (j1 < nj) x = x + Fj[fj0 + TX];
                if (i1 == 1) x = x - Fi[fi0];
                if (i1 == ni) x = x + Fi[fi0 + 1];
                if (j1 == 1) x = x - Fj[fj0];
                if (j1 == nj) x = x + Fj[fj0 + TX];
                r[v] = x;
            }
            const double sur = sC[4 * NC + k];
            if (a.source == 1) {   // Source_Axi_Eul_Blk (Lib_Source_Axisymmetry.f90:57-76)
                const double invr = scb[6 * pc + cg];
                const double mod_v = sqrt(P[1] * P[1] + P[2] * P[2]);
                double S[4];
                S[0] = -P[0] * P[2] * invr;
                S[1] = -P[0] * P[1] * P[2] * invr;
                S[2] = -P[0] * P[2] * P[2] * invr;
                S[3] = -(P[0] * E0(g, P[3], P[0], mod_v) + P[3]) * P[2] * invr;
#pragma unroll
                for (int v = 0; v < 4; ++v) r[v] = r[v] - S[v] * sur;
            } else if (a.source == 2) {   // Source_Area_Eul_Blk (Lib_Source_Areavariation.f90:120-142)
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
            // Compute_Cons_NoIRS (Lib_Newstate.f90:131-159)
            const double dt = a.time_accurate ? dt_case : sC[5 * NC + k];
            {   // -R / sur * dt with one division
                const double f = -dt / sur;
#pragma unroll
                for (int v = 0; v < 4; ++v) res[v] = r[v] * f;
            }
            if (irs == 1) {   // Scale_Residual_Cons (Lib_Newstate.f90:86-92): smoothed before the update
                double* ro = a.Rout + B.oc;
#pragma unroll
                for (int v = 0; v < 4; ++v) ro[v * pc + cg] = res[v];
                continue;
            }
            }
            double PO[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) PO[v] = a.first ? P[v] : sC[v * NC + k];
            double U0[4], U[4];
            U0[0] = PO[0]; U0[1] = PO[0] * PO[1]; U0[2] = PO[0] * PO[2];
            if (PREC == 0 && g.htab) {   // thermally perfect gas
                U0[3] = rhoE_tab(g, PO);
                U[3] = rhoE_tab(g, P);
            } else {
                U0[3] = PO[3] * g.igm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
                U[3] = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
            }
            U[0] = P[0]; U[1] = P[0] * P[1]; U[2] = P[0] * P[2];
#pragma unroll
            for (int v = 0; v < 4; ++v) U[v] = U0[v] + (U[v] - U0[v] + res[v]) * a.rk_c;
            double N[4];
            N[0] = U[0];
            {
                const double ir = 1.0 / U[0];
                N[1] = U[1] * ir;
                N[2] = U[2] * ir;
            }
            if (PREC == 0 && g.htab)   // cons2prim on the table, guess: the state before the update
                N[3] = N[0] * g.R *
                       T_of_e(g, U[3] / U[0] - 0.5 * (N[1] * N[1] + N[2] * N[2]), P[3] / (P[0] * g.R));
            else
                N[3] = g.gm1 * (U[3] - 0.5 * U[0] * (N[1] * N[1] + N[2] * N[2]));
            // Check_And_Fix_State (Lib_Newstate.f90:316-350)
            if (isnan(N[0]) || isnan(N[1]) || isnan(N[2]) || isnan(N[3]) || N[3] < 0.0)
                record_error(cs, 5, B.local_b, i1, j1, a.irk);
            if (N[0] < 1e-20) N[0] = 1e-20;
            double* po = a.Pout + B.oc;
#pragma unroll
            for (int v = 0; v < 4; ++v) po[v * pc + cg] = N[v];
            if (a.last) {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const double d = fabs(N[v] - PO[v]);
                    acc[v] += d * d;
                }
                const double dtn = cell_dt(a, g, N, scb, cg, pc, sD[sidx], sD[AREA + sidx], ndir, iter_next);
                if (!a.time_accurate) a.sc[2 * B.oc + pc + cg] = dtn;
                acc[4] = fmin(acc[4], dtn);
            }
        }
        if (a.last) {
            block_reduce_store<NT>(acc, red, tile_part);
            if (tid == 0)
                for (int k = 0; k < 5; ++k) a.part[5 * (size_t)it + k] = tile_part[k];
        }
        stage_item_end<NT>(a, it, w.case_id, red, &s_flag);
    }
}

// ------------------------------------------------------------------------------------------
// launch helpers (instantiated by q2d_kernels.cu, and by q2d_stage64_sd.cu for MUSCL-SD)
// ------------------------------------------------------------------------------------------
template <int PREC, int RIEM, int TX, int TY, int NT, bool SD, bool TAB = false>
cudaError_t launch_stage_t(const StageArgs& a, int grid, cudaStream_t s) {
    constexpr size_t smem = Tile<PREC, TX, TY, SD>::bytes;
    auto k = stage_kernel<PREC, RIEM, TX, TY, NT, SD, TAB>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int PREC, int RIEM, int TX, int TY, int NT, bool SD>
int occupancy_t() {
    constexpr size_t smem = Tile<PREC, TX, TY, SD>::bytes;
    auto k = stage_kernel<PREC, RIEM, TX, TY, NT, SD>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, smem);
    return n;
}

}  // namespace q2d
