// q2d_kernels.cu — the fused RK-stage kernel of the Q2D explicit path (sm_100a).
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
#include "q2d_kernels.cuh"
#include "q2d_common.cuh"
#include "q2d_march.cuh"

#include <cfloat>
#include <type_traits>

namespace q2d {


// ------------------------------------------------------------------------------------------
// The stage kernel
// ------------------------------------------------------------------------------------------

// Shared-memory layout of one tile (offsets in doubles).
template <int PREC, int TX, int TY>
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
    static constexpr int total = oSG + nSG;
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
    for (int k = threadIdx.x; k < NGJ; k += NT) {
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
template <int PREC, int RIEM, bool IDIR, int NT, int TX, int TY, typename ST>
__device__ __forceinline__ void face_phase(const StageArgs& a, const DBlock& B, CaseState* cs, int i0,
                                           int j0, const double* sP, const double* sD,
                                           const double* sG, const ST* sg, double* sF) {
    constexpr int W = TX + 4, AREA = W * (TY + 4);
    constexpr int NF = IDIR ? (TX + 1) * TY : TX * (TY + 1);
    constexpr int NG = IDIR ? (TX + 2) * TY : TX * (TY + 2);
    constexpr int ROWLEN = IDIR ? TX + 1 : TX;
    constexpr int DSTEP = IDIR ? 1 : W;
    const int ni = B.ni, nj = B.nj;
    const double* dlp = sD + (IDIR ? 0 : AREA);
    for (int f = threadIdx.x; f < NF; f += NT) {
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
            double QL[4], QR[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                QL[v] = sP[v * AREA + pL] + (double)(1.0 * sg[v * NG + gL] * lm);
                QR[v] = sP[v * AREA + pL + DSTEP] - (double)(1.0 * sg[v * NG + gR] * lp);
            }
            if (!face_flux<PREC, RIEM>(a.gas, QL, QR, nx, ny, ln, X))
                record_error(cs, 4, B.local_b, IDIR ? pos : k + 1, IDIR ? k + 1 : pos, a.irk);
        } else if (etype >= 0) {
            const bool minside = (Fm == 1 || Fm == 3);
            const int cb = minside ? pL + DSTEP : pL;         // boundary cell
            const int ci = minside ? cb + DSTEP : cb - DSTEP; // interior neighbour
            Q4 Bp, Ip;
#pragma unroll
            for (int v = 0; v < 4; ++v) { Bp.v[v] = sP[v * AREA + cb]; Ip.v[v] = sP[v * AREA + ci]; }
            const int prm = a.edges[B.eo[Fm - 1] + k].param;
            const Q4 q = bc_face<RIEM>(a.gas, a.limiter, etype, Fm, Bp, Ip, dlp[cb], dlp[ci], nx, ny, ln,
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

template <int PREC, int RIEM, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 2) stage_kernel(const StageArgs a) {
    using L = Tile<PREC, TX, TY>;
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
    __shared__ double red[(NT / 32) * 5];
    __shared__ double tile_part[5];
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    const Gas& g = a.gas;
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
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        sSi[v * NSI + k] = iface_slope<ST>(sP[v * AREA + p0], sP[v * AREA + p0 + 1], da, db);
                } else {
                    const int kk = k - NSI;
                    const int r = kk / TX, c = kk - r * TX;
                    const int p0 = r * W + c + 2;
                    const double da = sD[AREA + p0], db = sD[AREA + p0 + W];
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        sSj[v * NSJ + kk] = iface_slope<ST>(sP[v * AREA + p0], sP[v * AREA + p0 + W], da, db);
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
            face_phase<PREC, RIEM, true, NT, TX, TY>(a, B, cs, i0, j0, sP, sD, sGi, sGI, sFi);
            face_phase<PREC, RIEM, false, NT, TX, TY>(a, B, cs, i0, j0, sP, sD, sGj, sGJ, sFj);
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
            if (PREC == 0) {
#pragma unroll
                for (int v = 0; v < 4; ++v) res[v] = -r[v] / sur * dt * 1.0;
            } else {
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
            if (PREC == 0) {
                U0[3] = PO[3] / g.gm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
                U[3] = P[3] / g.gm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
            } else {
                U0[3] = PO[3] * g.igm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
                U[3] = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
            }
            U[0] = P[0]; U[1] = P[0] * P[1]; U[2] = P[0] * P[2];
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
                const double dtn = cell_dt(a, N, scb, cg, pc, sD[sidx], sD[AREA + sidx], ndir, iter_next);
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
            const double dtn = cell_dt(a, P, scb, cg, B.pc, a.dl[gidx], a.dl[gidx + B.pg], ndir, iter_next);
            if (!a.time_accurate) a.sc[2 * B.oc + B.pc + cg] = dtn;
            acc[4] = fmin(acc[4], dtn);
        }
        block_reduce_store<NT>(acc, red, tile_part);
        if (tid == 0)
            for (int k = 0; k < 5; ++k) a.part[5 * (size_t)it + k] = tile_part[k];
        item_done<NT>(a, w.case_id, false, true, false, red, &s_flag);
    }
}

// Initial time step for warp-marching items (a warp per item: strip columns x rows).
__global__ void __launch_bounds__(128) dt_march_kernel(const StageArgs a) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    for (int it = gw; it < a.n_items; it += nw) {
        const WorkItem w = a.items[it];
        const DBlock B = a.blocks[w.block];
        CaseState* cs = &a.cstate[w.case_id];
        // a.first != 0: only cases admitted since the last pass (others keep their time step)
        if (__ldcg(&cs->status) != kStatus_Running || (a.first && !__ldcg(&cs->dt_pending))) continue;
        const long long iter_next = __ldcg(&cs->iter) + 1;
        const int ndir = a.cases[w.case_id].ndir;
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        const int ii = w.i0 + lane;
        if (lane < kMarchCols && ii < B.ni) {
            for (int jj = w.j0; jj < w.j1; ++jj) {
                const long long cg = (long long)jj * B.ni + ii;
                double P[4];
                for (int v = 0; v < 4; ++v) P[v] = a.Pin[B.oc + v * B.pc + cg];
                const long long gidx = B.og + (long long)(jj + 2) * (B.ni + 4) + (ii + 2);
                const double* scb = a.sc + 2 * B.oc;
                const double dtn = cell_dt(a, P, scb, cg, B.pc, a.dl[gidx], a.dl[gidx + B.pg], ndir, iter_next);
                if (!a.time_accurate) a.sc[2 * B.oc + B.pc + cg] = dtn;
                acc[4] = fmin(acc[4], dtn);
            }
        }
        for (int o = 16; o > 0; o >>= 1) acc[4] = fmin(acc[4], __shfl_down_sync(kFull, acc[4], o));
        warp_item_done(a, w.case_id, acc, it, false, true, false);
    }
}

cudaError_t launch_dt_march(const StageArgs& a, int grid, cudaStream_t s) {
    dt_march_kernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
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
template <int PREC, int RIEM, int TX, int TY, int NT>
static cudaError_t launch_stage_t(const StageArgs& a, int grid, cudaStream_t s) {
    constexpr size_t smem = Tile<PREC, TX, TY>::bytes;
    auto k = stage_kernel<PREC, RIEM, TX, TY, NT>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int PREC, int RIEM, int TX, int TY, int NT>
static int occupancy_t() {
    constexpr size_t smem = Tile<PREC, TX, TY>::bytes;
    auto k = stage_kernel<PREC, RIEM, TX, TY, NT>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, smem);
    return n;
}

#define Q2D_TILE_SWITCH(TILE, CALL)                                          \
    switch (TILE) {                                                          \
        case 1: CALL(32, 8, 256); break;                                     \
        case 2: CALL(64, 4, 256); break;                                     \
        default: CALL(32, 10, 256); break;                                   \
    }

cudaError_t launch_stage(const StageArgs& a, int prec, int riem, int tile, int grid, cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
#define Q2D_CALL(TX, TY, NT)                                                                   \
    if (prec == 0) {                                                                           \
        if (riem == 1) e = launch_stage_t<0, 1, TX, TY, NT>(a, grid, s);                      \
        else if (riem == 2) e = launch_stage_t<0, 2, TX, TY, NT>(a, grid, s);                 \
        else if (riem == 3) e = launch_stage_t<0, 3, TX, TY, NT>(a, grid, s);                 \
        else if (riem == 4) e = launch_stage_t<0, 4, TX, TY, NT>(a, grid, s);                 \
        else e = launch_stage_t<0, 0, TX, TY, NT>(a, grid, s);                                \
    } else {                                                                                   \
        if (riem == 1) e = launch_stage_t<1, 1, TX, TY, NT>(a, grid, s);                      \
        else if (riem == 2) e = launch_stage_t<1, 2, TX, TY, NT>(a, grid, s);                 \
        else if (riem == 3) e = launch_stage_t<1, 3, TX, TY, NT>(a, grid, s);                 \
        else if (riem == 4) e = launch_stage_t<1, 4, TX, TY, NT>(a, grid, s);                 \
        else e = launch_stage_t<1, 0, TX, TY, NT>(a, grid, s);                                \
    }
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
    return e;
}

int stage_occupancy(int prec, int riem, int tile) {
    int n = 0;
#define Q2D_CALL(TX, TY, NT)                                                                   \
    if (prec == 0) {                                                                           \
        if (riem == 1) n = occupancy_t<0, 1, TX, TY, NT>();                                   \
        else if (riem == 2) n = occupancy_t<0, 2, TX, TY, NT>();                 \
        else if (riem == 3) n = occupancy_t<0, 3, TX, TY, NT>();                 \
        else if (riem == 4) n = occupancy_t<0, 4, TX, TY, NT>();                              \
        else n = occupancy_t<0, 0, TX, TY, NT>();                                             \
    } else {                                                                                   \
        if (riem == 1) n = occupancy_t<1, 1, TX, TY, NT>();                                   \
        else if (riem == 2) n = occupancy_t<1, 2, TX, TY, NT>();                 \
        else if (riem == 3) n = occupancy_t<1, 3, TX, TY, NT>();                 \
        else if (riem == 4) n = occupancy_t<1, 4, TX, TY, NT>();                              \
        else n = occupancy_t<1, 0, TX, TY, NT>();                                             \
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
int stage32_occupancy_r0(int tile);
int stage32_occupancy_r1(int tile);
int stage32_occupancy_r2(int tile);
int stage32_occupancy_r3(int tile);
int stage32_occupancy_r4(int tile);

cudaError_t launch_stage32(const StageArgs& a, int riem, int tile, int grid, cudaStream_t s) {
    if (riem == 1) return launch_stage32_r1(a, tile, grid, s);
    if (riem == 2) return launch_stage32_r2(a, tile, grid, s);
    if (riem == 3) return launch_stage32_r3(a, tile, grid, s);
    if (riem == 4) return launch_stage32_r4(a, tile, grid, s);
    return launch_stage32_r0(a, tile, grid, s);
}

int stage32_occupancy(int riem, int tile) {
    if (riem == 1) return stage32_occupancy_r1(tile);
    if (riem == 2) return stage32_occupancy_r2(tile);
    if (riem == 3) return stage32_occupancy_r3(tile);
    if (riem == 4) return stage32_occupancy_r4(tile);
    return stage32_occupancy_r0(tile);
}

#define Q2D_MARCH_DECL(P, R)                                                                  \
    cudaError_t launch_march_p##P##_r##R(const StageArgs& a, int lim, int grid, cudaStream_t s); \
    int march_occupancy_p##P##_r##R(int lim);
Q2D_MARCH_DECL(0, 0) Q2D_MARCH_DECL(0, 1) Q2D_MARCH_DECL(0, 2)
Q2D_MARCH_DECL(1, 0) Q2D_MARCH_DECL(1, 1) Q2D_MARCH_DECL(1, 2)
#undef Q2D_MARCH_DECL

cudaError_t launch_march(const StageArgs& a, int prec, int riem, int lim, int grid, cudaStream_t s) {
    if (riem > 2) return cudaErrorInvalidValue;   // the warp-marching schedule has no SLAU instantiation
    if (prec == 0) {
        if (riem == 1) return launch_march_p0_r1(a, lim, grid, s);
        if (riem == 2) return launch_march_p0_r2(a, lim, grid, s);
        return launch_march_p0_r0(a, lim, grid, s);
    }
    if (riem == 1) return launch_march_p1_r1(a, lim, grid, s);
    if (riem == 2) return launch_march_p1_r2(a, lim, grid, s);
    return launch_march_p1_r0(a, lim, grid, s);
}

int march_occupancy(int prec, int riem, int lim) {
    if (riem > 2) return 0;
    if (prec == 0) {
        if (riem == 1) return march_occupancy_p0_r1(lim);
        if (riem == 2) return march_occupancy_p0_r2(lim);
        return march_occupancy_p0_r0(lim);
    }
    if (riem == 1) return march_occupancy_p1_r1(lim);
    if (riem == 2) return march_occupancy_p1_r2(lim);
    return march_occupancy_p1_r0(lim);
}

}  // namespace q2d
