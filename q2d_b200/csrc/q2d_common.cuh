// q2d_common.cuh — device routines shared by the stage kernels: boundary-face fluxes
// (Lib_BC_Fluxes_*.f90 restated), face fluxes, MUSCL pieces, time step, per-case finalisation.
#pragma once
#include <cfloat>
#include <type_traits>
#include "q2d_dev.cuh"

namespace q2d {

// 8-byte asynchronous global -> shared copies (cp.async), completed by cp_async_wait_all.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
}

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
// Ghost cell (ii, jj) of block B outside exactly one of its index ranges (Fill_Ghost_Cell,
// Lib_Ghost.f90:16-299), evaluated from the stage's input state in HBM: gd = 1, 2 layers beyond
// face f at tangential index k. Returns false beyond the second layer.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ bool ghost_value(const StageArgs& a, const DBlock& B, int ii, int jj, double* q) {
    const int ni = B.ni, nj = B.nj;
    const bool inI = (ii >= 0 && ii < ni);
    int f, gd, k, bi, bj, di, dj;
    if (!inI) {
        f = ii < 0 ? 1 : 2; gd = ii < 0 ? -ii : ii - ni + 1; k = jj;
        bi = ii < 0 ? 0 : ni - 1; bj = jj; di = ii < 0 ? 1 : -1; dj = 0;
    } else {
        f = jj < 0 ? 3 : 4; gd = jj < 0 ? -jj : jj - nj + 1; k = ii;
        bi = ii; bj = jj < 0 ? 0 : nj - 1; di = 0; dj = jj < 0 ? 1 : -1;
    }
    if (gd > 2) return false;
    const long long pc = B.pc;
    const EdgeRec e = a.edges[B.eo[f - 1] + k];
    const double* pb = a.Pin + B.oc + (long long)bj * ni + bi;    // boundary cell
    if (e.type == 101) {   // Ghost_Connection (Lib_Ghost.f90:143-160): the donor block's cells
        const DBlock S = a.blocks[e.bs];
        const int si = e.is + guide_i(e.fs) * (gd - 1) - 1;
        const int sj = e.js + guide_j(e.fs) * (gd - 1) - 1;
        const double* src = a.Pin + S.oc + (long long)sj * S.ni + si;
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = __ldg(src + v * S.pc);
    } else if (e.type == 300) {   // Ghost_Symmetry (Lib_Ghost.f90:163-196)
        const double* gn = f <= 2 ? a.fi + B.ofi + (long long)bj * (ni + 1) + (f == 1 ? 0 : ni)
                                  : a.fj + B.ofj + (long long)(f == 3 ? 0 : nj) * ni + bi;
        const long long gs = f <= 2 ? B.pfi : B.pfj;
        const double nx = __ldg(gn), ny = __ldg(gn + gs);
        const double vx = __ldg(pb + pc), vy = __ldg(pb + 2 * pc);
        const double udotn = vx * nx + vy * ny;
        q[0] = __ldg(pb);
        q[1] = vx - 2.0 * udotn * nx;
        q[2] = vy - 2.0 * udotn * ny;
        q[3] = __ldg(pb + 3 * pc);
    } else if (e.type == 0 || e.type == 401 || e.type == 405 || e.type == 406 || e.type < 0) {
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = __ldg(pb + v * pc);   // Ghost_ZG_Extrapolate (:199-219)
    } else {   // Ghost_Extrapolate (Lib_Ghost.f90:270-299)
        const long long s1 = (long long)dj * ni + di;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double b0 = __ldg(pb + v * pc), i1 = __ldg(pb + v * pc + s1), i2 = __ldg(pb + v * pc + 2 * s1);
            const double g1 = 3.0 * b0 - 3.0 * i1 + i2;
            q[v] = gd == 1 ? g1 : 3.0 * g1 - 3.0 * b0 + i1;
        }
    }
    return true;
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

static __device__ void bc_extrapolation(const Gas& g, const double* P, double n0, double n1,
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

static __device__ bool bc_stagnation(const Gas& g, int Fm, const double* Bp, double n0, double n1,
                              double int_l, const BCParam& bp, double* X) {
    // BC_Inlet_StagnCond + Stagn_Inflow (Lib_BC_Fluxes_Inflow.f90:64-120, 412-483)
    const double modfm2 = 1 - 2 * (Fm % 2);
    const double BC_Sign = modfm2;
    const double Un = Bp[1] * n0 + Bp[2] * n1;
    if (BC_Sign * Un >= 0.0) return false;
    const double Gamma = f_gamma(g, Bp[3], Bp[0]);
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
    const double Face_H = 0.0 + Face_r1 / Face_rho * h_of_T(g, Face_T);
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

static __device__ bool bc_outflow(const Gas& g, int Fm, const double* Bp, double n0, double n1,
                           double int_l, const BCParam& bp, double* X) {
    // BC_Outflow + Outflow (Lib_BC_Fluxes_Outflow.f90:36-165)
    const double BC_Sign = 1 - 2 * (Fm % 2);
    const double Un = Bp[1] * n0 + Bp[2] * n1;
    if (BC_Sign * Un < 0.0) return false;
    const double rho = Bp[0];
    const double Sound = f_ss(g, Bp[3], rho);
    const double Gamma = f_gamma(g, Bp[3], rho);
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
    const double Face_H = 0.0 + Face[0] / Face_rho * h_of_T(g, Face_T);
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
                                          double ny, double int_l, double* X, double beta = 1.0) {
    if (PREC == 0) return flux_from_states64<RIEM>(g, PL, PR, nx, ny, int_l, X, beta);
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
// both for its two cells; here each is computed once per interface / cell (the FP64 kernel
// takes the interface distance's reciprocal once for the four variables: within an ulp of the
// reference's quotient). The FP32 form of the interface slope:
template <typename ST>
__device__ __forceinline__ ST iface_slope(double qa, double qb, double dla, double dlb);
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
    // with a.dt_first the partials' dt min is the time step of the step that ends here
    const DCase dc = a.cases[case_id];
    CaseState* cs = &a.cstate[case_id];
    const int tid = threadIdx.x;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
    if (with_res || with_dt) {
        const long long e1 = (long long)dc.item_end * a.part_stride;
        for (long long e = (long long)dc.item_begin * a.part_stride + tid; e < e1; e += NT) {
            const double* p = a.part + 5 * (size_t)e;
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
            if (a.dt_first) cs->dt_step = fmin(tot[4], 1e5);
            cs->dtglobal = cs->dt_step;
            cs->iter += 1;
            cs->iter_from_call += 1;
            if (a.time_accurate) cs->time = cs->time + cs->dt_step;
        }
        if (with_dt) {
            if (!a.dt_first) cs->dt_step = fmin(tot[4], 1e5);
            cs->dt_pending = 0;
        }
        if (with_res) {   // Mod_Explicit.f90:120-170
            if (cs->iter_from_call == 1 || (cs->iter % a.res_diter) == 0) {
                for (int k = 0; k < 4; ++k) cs->res[k] = sqrt(tot[k]);
                if (cs->res0 < 0.0) cs->res0 = cs->res[0];
            }
            const double thr = a.res_relative ? a.res_threshold * cs->res0 : a.res_threshold;
            const bool endsim = (cs->iter_from_call >= a.itermax) || (cs->res[0] <= thr) ||
                                (cs->time >= a.time_threshold) || (cs->iter_end > 0 && cs->iter >= cs->iter_end);
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

// Explicit_Step prologue of a case (Mod_Explicit.f90:38-55): done once per step, in the first
// stage, by the CTA that takes the case's first item. Nothing in the other items of that stage
// reads the fields it changes.
__device__ __forceinline__ void step_prologue(const StageArgs& a, int case_id) {
    CaseState* cs = &a.cstate[case_id];
    cs->dtglobal = cs->dt_step;
    cs->iter += 1;
    cs->iter_from_call += 1;
    if (a.time_accurate) cs->time = cs->time + cs->dt_step;
}

// End of one work item of a stage kernel. Only the last stage counts items to find the CTA that
// finalises the case (residual, next dt, TODO; with a fence so that the item partials are
// visible), unless a.fin_sep leaves that to finalize_kernel, launched after the stage. The step prologue runs in that finalisation when the time steps are computed in the
// first stage (its cells read the iteration count) or the step has one stage; otherwise the
// first stage runs it from the case's first item. Middle stages only need the barrier that
// protects the shared tile.
template <int NT>
__device__ void stage_item_end(const StageArgs& a, int it, int case_id, double* red, int* s_flag) {
    if (a.last && !a.fin_sep) {
        item_done<NT>(a, case_id, true, true, a.first != 0 || a.dt_first != 0, red, s_flag);
        return;
    }
    if (a.first && !a.dt_first && threadIdx.x == 0 && it == a.cases[case_id].item_begin)
        step_prologue(a, case_id);
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
__device__ __forceinline__ double cell_dt(const StageArgs& a, const Gas& g, const double* P, const double* sc,
                                          long long cidx, long long pc, double dl_i, double dl_j,
                                          int ndir, long long iter_next) {
    const double Sound = f_ss(g, P[3], P[0]);
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


}  // namespace q2d
