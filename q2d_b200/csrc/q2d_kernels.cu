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

#include <cfloat>
#include <type_traits>

namespace q2d {


__device__ __forceinline__ int guide_i(int f) { return f == 1 ? 1 : (f == 2 ? -1 : 0); }
__device__ __forceinline__ int guide_j(int f) { return f == 3 ? 1 : (f == 4 ? -1 : 0); }

__device__ __forceinline__ void record_error(CaseState* cs, int code, int b, int i, int j, int stage) {
    if (atomicCAS(&cs->err, 0, code) == 0) {
        cs->err_b = b;
        cs->err_i = i;
        cs->err_j = j;
        cs->err_stage = stage;
    }
}

// ------------------------------------------------------------------------------------------
// Boundary-face fluxes, FP64 (the oracle's restatement of Lib_BC_Fluxes_*.f90). Each returns
// the reference's `Flux` vector; the cell adds it with the sign of its face like an interior
// face (modfm2 = -1 on faces 1/3, +1 on faces 2/4).
// ------------------------------------------------------------------------------------------
template <int RIEM>
__device__ void bc_symmetry(const Gas& g, int lim, int Fm, const double* Bp, const double* Ip,
                            double Bound_Dl, double Int_Dl, double n0, double n1, double int_l,
                            double* X) {
    // BC_Symmetry_Eul (Lib_BC_Fluxes_Symmetry.f90:28-124), Un_wall = 0
    const int modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm;
    double Un = Bp[1] * n0 + Bp[2] * n1;
    double G[4] = {Bp[0], Bp[1], Bp[2], Bp[3]};
    G[1] = G[1] - 2.0 * Un * n0;
    G[2] = G[2] - 2.0 * Un * n1;
    const double Dist12 = 2.0 * Bound_Dl * modfm + (Bound_Dl + Int_Dl) * modfm1;
    const double Dist23 = (Bound_Dl + Int_Dl) * modfm + 2.0 * Bound_Dl * modfm1;
    const double Dist = Bound_Dl * modfm2;
    double Face[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double P1 = modfm * G[v] + modfm1 * Ip[v];
        const double P3 = modfm * Ip[v] + modfm1 * G[v];
        const double s32 = (P3 - Bp[v]) / Dist23;
        const double s21 = (Bp[v] - P1) / Dist12;
        Face[v] = Bp[v] + rlimiter(lim, s32, s21) * Dist;
    }
    const double Sound = f_ss(g, Face[3], Face[0]);
    Un = Face[1] * n0 + Face[2] * n1;
    const double vtx = Face[1] - Un * n0, vty = Face[2] - Un * n1;
    const double Un1 = Un * modfm2;
    const double L[4] = {Face[0], Un1 * n0 + vtx, Un1 * n1 + vty, Face[3]};
    const double R[4] = {Face[0], -Un1 * n0 + vtx, -Un1 * n1 + vty, Face[3]};
    const F4 F = riemann64<RIEM>(g, L, Sound, R, Sound, n0, n1);
    X[0] = 0.0;
    X[1] = F.u * int_l;
    X[2] = F.v * int_l;
    X[3] = 0.0;
}

__device__ void bc_extrapolation(const Gas& g, const double* P, double n0, double n1,
                                 double int_l, double* X) {
    // BC_Extrapolation (Lib_BC_Fluxes_Extrapolation.f90:18-49)
    const double Un = P[1] * n0 + P[2] * n1;
    X[0] = P[0] * Un * int_l;
    const double Fmass = X[0];
    X[1] = Fmass * P[1] + P[3] * int_l * n0;
    X[2] = Fmass * P[2] + P[3] * int_l * n1;
    X[3] = Fmass * H0(g, P[3], P[0], sqrt(P[1] * P[1] + P[2] * P[2]));
}

__device__ __forceinline__ double inflow_direction(double n0, double n1, double a) {
    // Compute_Inflow_Direction (Lib_BC_Fluxes_Inflow.f90:548-563)
    return a >= 0.5 * DBL_MAX ? atan(n1 / (n0 + 1e-20)) : a;
}

__device__ bool bc_stagnation(const Gas& g, int Fm, const double* Bp, double n0, double n1,
                              double int_l, const BCParam& bp, double* X) {
    // BC_Inlet_StagnCond + Stagn_Inflow (Lib_BC_Fluxes_Inflow.f90:64-120, 412-483)
    const double modfm2 = 1 - 2 * (Fm % 2);
    const double BC_Sign = modfm2;
    const double Un = Bp[1] * n0 + Bp[2] * n1;
    if (BC_Sign * Un >= 0.0) return false;
    const double Gamma = g.gamma;
    const double Sound = f_ss(g, Bp[3], Bp[0]);
    const double Riem = Sound + BC_Sign * 0.5 * (Gamma - 1.0) * Un;
    const double alpha = inflow_direction(n0, n1, bp.alpha);
    const double XA = n1 - n0 * tan(alpha);
    const double XB = bp.t1 - bp.t0 * tan(alpha);
    const double E1 = -XA / XB;
    double Discr = -1.0, p0try = bp.p0;
    double Sound0 = 0.0, Coef_D = 0.0, YA = 0.0, YB = 0.0;
    const double p = Bp[3];
    for (int iter = 1;; ++iter) {   // bounded: the reference exits after 1000 iterations
        Sound0 = sqrt(Gamma * g.R * bp.T0);
        Coef_D = (1.0 + E1 * E1) * (Gamma - 1.0) / 2.0;
        double Coef_C = pow(p0try / p, (Gamma - 1.0) / Gamma);
        const double ss = Sound / Sound0;
        Coef_C = Coef_C * (ss * ss);
        const double gh = (Gamma - 1.0) / 2.0;
        YA = gh * gh + Coef_C * Coef_D;
        YB = BC_Sign * Riem * ((Gamma - 1.0) / 2.0);
        const double YC = Riem * Riem - Coef_C * (Sound0 * Sound0);
        Discr = YB * YB - YA * YC;
        if (Discr < 0.0 && fabs(Discr) < 1e-2) Discr = 0.0;
        if (Discr < 0.0 && fabs(Discr) > 1e-2) p0try = bp.rel_fac * p0try + (1 - bp.rel_fac) * p;
        if (iter > 1000) { Discr = 0.0; break; }
        if (!(Discr < 0.0)) break;
    }
    const double Un_Sign = copysign(1.0, Un);
    const double Un3 = (YB + Un_Sign * sqrt(Discr)) / YA;
    const double Sound3 = sqrt(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
    const double p3 = p0try * pow(Sound3 / Sound0, 2.0 * Gamma / (Gamma - 1.0));
    const double Ut3 = Un3 * E1;
    const double Face_rho = Gamma * p3 / (Sound3 * Sound3);
    const double Face_r1 = 1.0 * Face_rho;
    const double fu = Un3 * n0 + Ut3 * bp.t0;
    const double fv = Un3 * n1 + Ut3 * bp.t1;
    const double Face_T = p3 / (g.R * Face_rho);
    const double Face_H = 0.0 + Face_r1 / Face_rho * (g.cp * Face_T);
    X[0] = Face_r1 * Un3 * int_l;
    const double Fmass = Face_rho * Un3 * int_l;
    X[1] = Fmass * fu + p3 * int_l * n0;
    X[2] = Fmass * fv + p3 * int_l * n1;
    X[3] = Fmass * (0.5 * (fu * fu + fv * fv) + Face_H);
    return true;
}

template <int RIEM>
__device__ bool bc_supersonic(const Gas& g, int lim, int Fm, const double* P2, const double* Ip,
                              double n0, double n1, double int_l, const BCParam& bp, double* X) {
    // BC_Inlet_Supersonic_Static + Supersonic_Inflow (Lib_BC_Fluxes_Inflow.f90:272-311, 321-403)
    const int modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm;
    const double Un = P2[1] * n0 + P2[2] * n1;
    if ((double)modfm2 * Un >= 0.0) return false;
    const double flow_Sound = f_ss(g, P2[3], P2[0]);
    const double flow_Mach = sqrt(P2[1] * P2[1] + P2[2] * P2[2]) / flow_Sound;
    const double Mloc = bp.rel_fac * bp.mach + (1 - bp.rel_fac) * flow_Mach;
    const double ploc = bp.rel_fac * bp.pamb + (1 - bp.rel_fac) * P2[3];
    const double alpha = inflow_direction(n0, n1, bp.alpha);
    double Sup[4];
    Sup[3] = ploc;
    const double Sup_rho = Sup[3] / (g.R * bp.T0);
    Sup[0] = Sup_rho * 1.0;
    const double Sup_Sound = f_ss(g, Sup[3], Sup_rho);
    Sup[1] = Mloc * Sup_Sound * cos(alpha);
    Sup[2] = Mloc * Sup_Sound * sin(alpha);
    double Face[4], PL[4], PR[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double P1 = modfm * Sup[v] + modfm1 * Ip[v];
        const double P3 = modfm * Ip[v] + modfm1 * Sup[v];
        const double s = rlimiter(lim, P3 - P2[v], P2[v] - P1);
        Face[v] = P2[v] + 0.5 * s * modfm2;
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        PL[v] = modfm * Sup[v] + modfm1 * Face[v];
        PR[v] = modfm * Face[v] + modfm1 * Sup[v];
    }
    const double aL = f_ss(g, PL[3], PL[0]);
    const double aR = f_ss(g, PR[3], PR[0]);
    const F4 F = riemann64<RIEM>(g, PL, aL, PR, aR, n0, n1);
    const double su = copysign(1.0, F.r);
    const double SelL = (1.0 + su) / 2.0, SelR = (su - 1.0) / 2.0;
    const double Fmass = F.r * int_l;
    X[0] = Fmass * (SelL * PL[0] / PL[0] - SelR * PR[0] / PR[0]);
    X[1] = F.u * int_l;
    X[2] = F.v * int_l;
    X[3] = F.e * int_l;
    return true;
}

__device__ bool bc_outflow(const Gas& g, int Fm, const double* Bp, double n0, double n1,
                           double int_l, const BCParam& bp, double* X) {
    // BC_Outflow + Outflow (Lib_BC_Fluxes_Outflow.f90:36-165)
    const double BC_Sign = 1 - 2 * (Fm % 2);
    const double Un = Bp[1] * n0 + Bp[2] * n1;
    if (BC_Sign * Un < 0.0) return false;
    const double rho = Bp[0];
    const double Sound = f_ss(g, Bp[3], rho);
    const double Gamma = g.gamma;
    const double Riem = Sound + BC_Sign * 0.5 * (Gamma - 1.0) * Un;
    const double vtx = Bp[1] - Un * n0, vty = Bp[2] - Un * n1;
    const double Mach_N = fabs(Un / Sound);
    double Face[4], Face_Un, Face_rho;
    if (Mach_N < 1.0 && bp.pamb > 0.0) {
        double p_exit = bp.pamb;
        const double delta = 0.5 * (Gamma - 1.0);
        const double den = 1.0 / pow(1 + delta, Gamma / (Gamma - 1.0));
        const double pstar = Bp[3] * den * pow(1 + delta * (Mach_N * Mach_N), Gamma / (Gamma - 1.0));
        if (pstar >= p_exit) p_exit = pstar;
        const double Isen = (Gamma - 1.0) / (2.0 * Gamma);
        Face[3] = p_exit * bp.rel_fac + Bp[3] * (1.0 - bp.rel_fac);
        const double Face_Sound = Sound * pow(Face[3] / Bp[3], Isen);
        Face_Un = (Riem - Face_Sound) / (BC_Sign * 0.5 * (Gamma - 1.0));
        Face_rho = Gamma * Face[3] / (Face_Sound * Face_Sound);
        Face[0] = Bp[0] / rho * Face_rho;
        Face[1] = vtx + Face_Un * n0;
        Face[2] = vty + Face_Un * n1;
    } else {
        Face[0] = Bp[0]; Face[1] = Bp[1]; Face[2] = Bp[2]; Face[3] = Bp[3];
        Face_Un = Un;
        Face_rho = rho;
    }
    const double Face_T = Face[3] / (g.R * Face_rho);
    const double Face_H = 0.0 + Face[0] / Face_rho * (g.cp * Face_T);
    X[0] = Face[0] * int_l * Face_Un;
    const double mdot = Face_rho * int_l * Face_Un;
    X[1] = Face[1] * mdot + Face[3] * int_l * n0;
    X[2] = Face[2] * mdot + Face[3] * int_l * n1;
    X[3] = mdot * (0.5 * (Face[1] * Face[1] + Face[2] * Face[2]) + Face_H);
    return true;
}

// Boundary face flux by record type, states passed by value so that the common interior path
// keeps its arrays in registers (BC_Fluxes dispatch, Mod_BC_Fluxes.f90:79-269; 401/405/406
// fall back to BC_Symmetry_Eul when the flow direction does not match, :176-227).
struct Q4 { double v[4]; };
template <int RIEM>
__device__ __noinline__ Q4 bc_face(const Gas g, int lim, int etype, int Fm, const Q4 Bp, const Q4 Ip,
                                   double dlb, double dli, double nx, double ny, double ln,
                                   const BCParam* bp) {
    Q4 X = {{0.0, 0.0, 0.0, 0.0}};
    bool done = true;
    if (etype == 400) bc_extrapolation(g, Bp.v, nx, ny, ln, X.v);
    else if (etype == 401) done = bc_stagnation(g, Fm, Bp.v, nx, ny, ln, *bp, X.v);
    else if (etype == 405) done = bc_supersonic<RIEM>(g, lim, Fm, Bp.v, Ip.v, nx, ny, ln, *bp, X.v);
    else if (etype == 406) done = bc_outflow(g, Fm, Bp.v, nx, ny, ln, *bp, X.v);
    else if (etype == 300) done = false;
    else if (etype != 0) return X;
    if (etype == 0) return X;
    if (!done) bc_symmetry<RIEM>(g, lim, Fm, Bp.v, Ip.v, 0.5 * dlb, 0.5 * dli, nx, ny, ln, X.v);
    return X;
}

// ------------------------------------------------------------------------------------------
// Interior face flux from two reconstructed face states, FP64 or FP32-flux form.
// ------------------------------------------------------------------------------------------
template <int PREC, int RIEM>
__device__ __forceinline__ bool face_flux(const Gas& g, const double* PL, const double* PR, double nx,
                                          double ny, double int_l, double* X) {
    if (PREC == 0) return flux_from_states64<RIEM>(g, PL, PR, nx, ny, int_l, X);
    const bool bad = gas_state_bad(PL[0], PL[3]) || gas_state_bad(PR[0], PR[3]);
    FluxState L, R;
    phys64(g, PL, nx, ny, L);
    phys64(g, PR, nx, ny, R);
    const F4 F = riemann32<RIEM>(g, L, R, (float)nx, (float)ny);
    X[0] = F.r * int_l;
    X[1] = F.u * int_l;
    X[2] = F.v * int_l;
    X[3] = F.e * int_l;
    return !bad;
}

// MUSCL pieces shared between faces (Lib_Reconstruction.f90:21-27): the slope of an
// interface between cells a and b, (q_b - q_a) / (0.5 (dl_a + dl_b)), and the limited slope
// of a cell, rlimiter(forward slope, backward slope). Every face of the reference recomputes
// both for its two cells; here each is computed once per interface / cell, with the same
// operations, so the face states are bitwise those of Convective_Flux.
template <typename ST>
__device__ __forceinline__ ST iface_slope(double qa, double qb, double dla, double dlb);
template <>
__device__ __forceinline__ double iface_slope<double>(double qa, double qb, double dla, double dlb) {
    return (qb - qa) / (0.5 * (dla + dlb));
}
template <>
__device__ __forceinline__ float iface_slope<float>(double qa, double qb, double dla, double dlb) {
    return (float)(qb - qa) * __frcp_rn(0.5f * (float)(dla + dlb));
}
__device__ __forceinline__ double cell_sigma(int lim, double fwd, double bwd) { return rlimiter(lim, fwd, bwd); }
__device__ __forceinline__ float cell_sigma(int lim, float fwd, float bwd) { return rlimiter32(lim, fwd, bwd); }

// ------------------------------------------------------------------------------------------
// Per-case finalisation by the last CTA of a case (called by all threads of the CTA).
// ------------------------------------------------------------------------------------------
template <int NT>
__device__ void finalize_case(const StageArgs& a, int case_id, bool with_res, bool with_dt,
                              bool commit_begin, double* red) {
    const DCase dc = a.cases[case_id];
    CaseState* cs = &a.cstate[case_id];
    const int tid = threadIdx.x;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
    if (with_res || with_dt) {
        for (int it = dc.item_begin + tid; it < dc.item_end; it += NT) {
            const double* p = a.part + 5 * (size_t)it;
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] += __ldcg(p + k);
            acc[4] = fmin(acc[4], __ldcg(p + 4));
        }
        // fixed-order tree: warp shuffles then warps in index order
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            double v = acc[k];
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(0xffffffffu, v, o);
                v = (k < 4) ? v + w : fmin(v, w);
            }
            if ((tid & 31) == 0) red[(tid >> 5) * 5 + k] = v;
        }
    }
    __syncthreads();
    if (tid == 0) {
        double tot[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        if (with_res || with_dt)
            for (int w = 0; w < NT / 32; ++w)
                for (int k = 0; k < 5; ++k)
                    tot[k] = (k < 4) ? tot[k] + red[w * 5 + k] : fmin(tot[k], red[w * 5 + k]);
        if (commit_begin) {   // Explicit_Step prologue (Mod_Explicit.f90:38-55)
            cs->dtglobal = cs->dt_step;
            cs->iter += 1;
            cs->iter_from_call += 1;
            if (a.time_accurate) cs->time = cs->time + cs->dt_step;
        }
        if (with_dt) cs->dt_step = fmin(tot[4], 1e5);
        if (with_res) {   // Mod_Explicit.f90:120-170
            if (cs->iter_from_call == 1 || (cs->iter % a.res_diter) == 0) {
                for (int k = 0; k < 4; ++k) cs->res[k] = sqrt(tot[k]);
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
}

// Marks the item done; the CTA that completes the last item of the case finalises it.
template <int NT>
__device__ void item_done(const StageArgs& a, int case_id, bool with_res, bool with_dt,
                          bool commit_begin, double* red, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const DCase dc = a.cases[case_id];
        const unsigned prev = atomicAdd(&a.cstate[case_id].counter, 1u);
        *s_flag = (prev == (unsigned)(dc.item_end - dc.item_begin - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (*s_flag) {
        __threadfence();
        finalize_case<NT>(a, case_id, with_res, with_dt, commit_begin, red);
    }
    __syncthreads();
}

template <int NT>
__device__ void block_reduce_store(double* acc, double* red, double* out) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, v, o);
            v = (k < 4) ? v + w : fmin(v, w);
        }
        if ((tid & 31) == 0) red[(tid >> 5) * 5 + k] = v;
    }
    __syncthreads();
    if (tid == 0) {
        double tot[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        for (int w = 0; w < NT / 32; ++w)
            for (int k = 0; k < 5; ++k)
                tot[k] = (k < 4) ? tot[k] + red[w * 5 + k] : fmin(tot[k], red[w * 5 + k]);
        for (int k = 0; k < 5; ++k) out[k] = tot[k];
    }
}

// Compute_dt body for one cell (Mod_dt.f90:59-104), model == 0, plus the CFL ramp (:43).
__device__ __forceinline__ double cell_dt(const StageArgs& a, const double* P, const double* sc,
                                          long long cidx, long long pc, double dl_i, double dl_j,
                                          int ndir, long long iter_next) {
    const double Sound = f_ss(a.gas, P[3], P[0]);
    double dtmin = 1e8;
    {
        const double v0 = sc[2 * pc + cidx], v1 = sc[3 * pc + cidx];
        const double vel_ = fabs(P[1] * v0 + P[2] * v1);
        const double dt = dl_i / (vel_ + Sound) * a.cfl;
        dtmin = dmin(dt, dtmin);
    }
    if (ndir == 2) {
        const double v0 = sc[4 * pc + cidx], v1 = sc[5 * pc + cidx];
        const double vel_ = fabs(P[1] * v0 + P[2] * v1);
        const double dt = dl_j / (vel_ + Sound) * a.cfl;
        dtmin = dmin(dt, dtmin);
    }
    if (iter_next < a.rampa) dtmin = dtmin * (double)iter_next / (double)a.rampa;
    return dtmin;
}

// ------------------------------------------------------------------------------------------
// The stage kernel
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
}

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
                  NGI = L::NGI, NGJ = L::NGJ, NC = L::NC;
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
            } else if (inI != inJ) {
                int f, gd, k;
                if (!inI) { f = ii < 0 ? 1 : 2; gd = ii < 0 ? -ii : ii - ni + 1; k = jj; }
                else      { f = jj < 0 ? 3 : 4; gd = jj < 0 ? -jj : jj - nj + 1; k = ii; }
                if (gd > 2) continue;
                const EdgeRec e = a.edges[B.eo[f - 1] + k];
                if (e.type == 101) {   // Ghost_Connection (Lib_Ghost.f90:143-160): donor cells
                    const DBlock S = a.blocks[e.bs];
                    const int si = e.is + guide_i(e.fs) * (gd - 1) - 1;
                    const int sj = e.js + guide_j(e.fs) * (gd - 1) - 1;
                    const double* src = a.Pin + S.oc + (long long)sj * S.ni + si;
#pragma unroll
                    for (int v = 0; v < 4; ++v) cp_async8(sP + v * AREA + idx, src + v * S.pc);
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
        cp_async_wait_all();
        __syncthreads();

        // ---- 2. ghost cells that follow from the tile's own cells --------------------------
        {
            const int nrow = min(TY, nj - j0), ncol = min(TX, ni - i0);
            const int nl = (i0 == 0) ? nrow : 0;
            const int nr = (i0 + TX >= ni) ? nrow : 0;
            const int nb = (j0 == 0) ? ncol : 0;
            const int nt = (j0 + TY >= nj) ? ncol : 0;
            for (int t = tid; t < nl + nr + nb + nt; t += NT) {
                int f, k, cb, rb, dc, dr, gidx;   // boundary cell, outward step, face geometry index
                const double* gn;
                int gstride;
                if (t < nl) {
                    f = 1; rb = 2 + t; cb = 2; k = j0 + t; dc = -1; dr = 0;
                    gn = sGi; gstride = NFI; gidx = t * (TX + 1);
                } else if (t < nl + nr) {
                    const int u = t - nl;
                    f = 2; rb = 2 + u; cb = (ni - 1 - i0) + 2; k = j0 + u; dc = 1; dr = 0;
                    gn = sGi; gstride = NFI; gidx = u * (TX + 1) + (ni - i0);
                } else if (t < nl + nr + nb) {
                    const int u = t - nl - nr;
                    f = 3; cb = 2 + u; rb = 2; k = i0 + u; dc = 0; dr = -1;
                    gn = sGj; gstride = NFJ; gidx = u;
                } else {
                    const int u = t - nl - nr - nb;
                    f = 4; cb = 2 + u; rb = (nj - 1 - j0) + 2; k = i0 + u; dc = 0; dr = 1;
                    gn = sGj; gstride = NFJ; gidx = (nj - j0) * TX + u;
                }
                const int type = a.edges[B.eo[f - 1] + k].type;
                if (type == 101) continue;
                const int b0 = rb * W + cb;
                const int s1 = b0 + dr * W + dc, s2 = s1 + dr * W + dc;
                const int in1 = b0 - dr * W - dc, in2 = in1 - dr * W - dc;
                if (type == 300) {   // Ghost_Symmetry (Lib_Ghost.f90:163-196)
                    const double nx = gn[gidx], ny = gn[gstride + gidx];
                    const double vx = sP[AREA + b0], vy = sP[2 * AREA + b0];
                    const double udotn = vx * nx + vy * ny;
                    const double gx = vx - 2.0 * udotn * nx, gy = vy - 2.0 * udotn * ny;
                    sP[s1] = sP[b0]; sP[AREA + s1] = gx; sP[2 * AREA + s1] = gy; sP[3 * AREA + s1] = sP[3 * AREA + b0];
                    sP[s2] = sP[b0]; sP[AREA + s2] = gx; sP[2 * AREA + s2] = gy; sP[3 * AREA + s2] = sP[3 * AREA + b0];
                } else if (type == 0 || type == 401 || type == 405 || type == 406 || type < 0) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {   // Ghost_ZG_Extrapolate (:199-219)
                        sP[v * AREA + s1] = sP[v * AREA + b0];
                        sP[v * AREA + s2] = sP[v * AREA + b0];
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {   // Ghost_Extrapolate (:270-299)
                        const double* q = sP + v * AREA;
                        const double g1 = 3.0 * q[b0] - 3.0 * q[in1] + q[in2];
                        sP[v * AREA + s1] = g1;
                        sP[v * AREA + s2] = 3.0 * g1 - 3.0 * q[b0] + q[in1];
                    }
                }
            }
        }
        __syncthreads();

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
            const long long cg = (long long)jj * ni + ii;
            const double sur = sC[4 * NC + k];
            double P[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) P[v] = sP[v * AREA + sidx];
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
            double PO[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) PO[v] = a.first ? P[v] : sC[v * NC + k];
            double res[4];
            if (PREC == 0) {
#pragma unroll
                for (int v = 0; v < 4; ++v) res[v] = -r[v] / sur * dt * 1.0;
            } else {
                const double f = -dt / sur;
#pragma unroll
                for (int v = 0; v < 4; ++v) res[v] = r[v] * f;
            }
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
        item_done<NT>(a, w.case_id, a.last != 0, a.last != 0, a.first != 0, red, &s_flag);
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
        if (__ldcg(&cs->status) != kStatus_Running) continue;
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
        else e = launch_stage_t<0, 0, TX, TY, NT>(a, grid, s);                                \
    } else {                                                                                   \
        if (riem == 1) e = launch_stage_t<1, 1, TX, TY, NT>(a, grid, s);                      \
        else if (riem == 2) e = launch_stage_t<1, 2, TX, TY, NT>(a, grid, s);                 \
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
        else if (riem == 2) n = occupancy_t<0, 2, TX, TY, NT>();                              \
        else n = occupancy_t<0, 0, TX, TY, NT>();                                             \
    } else {                                                                                   \
        if (riem == 1) n = occupancy_t<1, 1, TX, TY, NT>();                                   \
        else if (riem == 2) n = occupancy_t<1, 2, TX, TY, NT>();                              \
        else n = occupancy_t<1, 0, TX, TY, NT>();                                             \
    }
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
    return n;
}

void tile_dims(int tile, int* tx, int* ty, int* nt) {
#define Q2D_CALL(TX, TY, NT) { *tx = TX; *ty = TY; *nt = NT; }
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
}

cudaError_t launch_dt(const StageArgs& a, int tile, int grid, cudaStream_t s) {
#define Q2D_CALL(TX, TY, NT) dt_kernel<TX, TY, NT><<<grid, NT, 0, s>>>(a);
    Q2D_TILE_SWITCH(tile, Q2D_CALL)
#undef Q2D_CALL
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

}  // namespace q2d
