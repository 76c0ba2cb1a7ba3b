// q2d_dev.cuh — device data layout and the per-face / per-cell physics of the Q2D explicit
// path for sm_100a.
//
// Layout in HBM (all pools are structure-of-arrays planes, padded to 32 elements):
//   state pools A, B, C    4 cell planes per block (rho, u, v, p), cell (i,j) at j*ni + i
//   scalar pool            8 cell planes per block: sur, dtlocal, versor1 (x,y), versor2 (x,y),
//                          source 0/1 (1/r for axisymmetric; Gx, Gy for area variation)
//   dl pool                2 ghost-frame planes per block ((ni+4) x (nj+4), gc = 2); its FP32
//                          copy holds the same region with the two lengths interleaved per cell
//   i-face / j-face pools  3 planes (nx, ny, int_l) on (ni+1) x nj and ni x (nj+1) faces
//   node pool              2 planes (x, y) on (ni+1) x (nj+1) nodes
// Index conventions follow the reference: face F of a row (0..ni) separates 1-based cells F
// and F+1 (dir(1)%f(F,j), Lib_Metrics.f90:88-100); guide/face codes 1..4 as in
// Parameters_m.f90:13-18.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace q2d {

constexpr int kStatus_Running = 0;
constexpr int kStatus_Paused = 1;   // TODO = IO inside a multi-step call
constexpr int kStatus_Done = 2;     // TODO = END
constexpr int kStatus_Error = 3;

struct DBlock {
    int ni, nj;
    int case_id, local_b;
    long long oc;     // offset of the block in 4-plane cell pools (elements); plane stride pc
    long long pc;
    long long og;     // offset in 2-plane ghost-frame pools; plane stride pg
    long long pg;
    long long ofi, pfi;   // i-face pool offset / plane stride
    long long ofj, pfj;   // j-face pool offset / plane stride
    long long on, pn;     // node pool offset / plane stride
    int eo[4];            // offset of the edge records of faces 1..4
};

// One boundary-cell record as the kernels consume it.
struct EdgeRec {
    int type;        // BC code, or -1 when the face has no record
    int bs;          // 101: global id of the donor block
    int is, js, fs;  // 101: donor cell (1-based) and face
    int param;       // index into BCParam (401/405/406), -1 otherwise
};

struct BCParam {
    double T0, p0, pamb, mach, alpha, rel_fac;
    double t0, t1;   // unit tangent of the boundary face (Setup_Inflow_Geometry)
};

struct DCase {
    int item_begin, item_end;   // work items of the case (contiguous)
    int ndir;                   // 1 when block 1 of the case has nj == 1 (Check_Mesh_Type)
    int pad;
};

// Per-case run state, updated on the device by the last CTA that finishes a case's work in
// each stage (no host round trip per step).
struct CaseState {
    double dt_step;        // dt of the step being run / about to run (min over cells, <= 1e5)
    double dtglobal;       // reported dtglobal of the last started step
    double time;
    double time_from_call;
    double res[4];
    double res0;
    long long iter;
    long long iter_from_call;
    int todo;
    int status;
    int err, err_b, err_i, err_j, err_stage;
    unsigned int counter;  // items of the current stage finished (reset by the last CTA)
    int dt_pending;        // the case has no time step yet (admitted after the last dt pass)
    int iter_end;          // the case's own fixed end (iteration count), 0 for none
};
static_assert(sizeof(CaseState) == 128, "case state: 128 bytes");

struct WorkItem {
    int block;   // global block id
    int i0, j0;  // 0-based origin of the tile (tile kernel) or strip / first row (march kernel)
    int case_id;
    int j1;      // march kernel: one past the last row of the item
    int pad;
};

struct Gas {
    double R, gamma, gm1, cp, cv;
    double gfac;   // gamma / (gamma - 1)
    double igm1;   // 1 / (gamma - 1)
    int rkind;     // the Riemann solver (Q2D_RIEMANN_*): selects among the ones of the generic form
    double minf;   // riemann-options-Minf (AUSM+-up, AUSM+-up2)
    double iR;     // 1 / R
    const double* htab;    // thermally perfect gas: h(T) [J/kg] at T = 0, 1, .. ntab-1 K (null:
    const double* cptab;   //   calorically perfect); cp(T) [J/(kg K)] on the same knots
    int ntab;
};

struct StageArgs {
    const DBlock* blocks;
    const DCase* cases;
    CaseState* cstate;
    const WorkItem* items;
    int n_items;
    int n_cases;           // case slots (cstate / cases entries)
    const double* Pin;     // stencil state
    const double* PO;      // state at the start of the step
    double* Pout;
    double* sc;            // scalar pool
    const double* dl;
    const float* dl32;     // FP32 copy of the dl pool (FP32-flux form), the two lengths of a
                           // ghost-frame cell k interleaved at og + 2k (float2)
    const double* fi;
    const double* fj;
    const float4* fi4;     // FP32 copies of the face pools as (nx, ny, len, 0); a block's faces
    const float4* fj4;     // start at float4 index ofi / 2 (ofj / 2)
    const EdgeRec* edges;
    const BCParam* bcp;
    double* part;          // per-item partials: 4 residual sums + dt min, part_stride sets of 5
    int part_stride;       //   doubles per item (one per warp for the FP32-flux kernel)
    int fin_sep;           // the last stage leaves the case finalisation to finalize_kernel
    Gas gas;
    double rk_c;           // RKcoeff(n_rk, irk)
    double cfl;
    int irk, n_rk;
    int first, last;       // stage is the first / last of the step
    // implicit residual smoothing (Lib_Newstate.f90:36-66): 0 off; 1 the stage writes its scaled
    // residual -R dt / sur to Rout and stops there; 2 the stage updates the state from the
    // smoothed residual in Rin (no fluxes)
    int irs_mode;
    double* Rout;
    const double* Rin;
    int dt_first;          // local time steps computed in the first stage from the step's
                           // starting state (else in the last stage of the previous step)
    int limiter, source, time_accurate, rampa;
    int sd;                // MUSCL-SD: face slopes scaled by the Tramel sensor of the face's cell
    int res_diter, sol_diter, res_relative;
    long long itermax;
    double res_threshold, time_threshold, sol_dtime;
    int* launch_flag;      // set to 1 by every kernel launch (instrumentation, unused by math)
};

// ---------------------------------------------------------------------------------------
// Single-species closures (FLINT_Lib_Thermodynamic's roles; formulas of docs/theory/thermo.md:
// 39-99 of the reference). Calorically perfect: a = sqrt(gamma p / rho),
// E0 = p/((gamma-1) rho) + |V|^2/2, H0 = gamma p/((gamma-1) rho) + |V|^2/2, h = cp T.
// Thermally perfect (g.htab set): h(T), cp(T) interpolated linearly at int(T) on 1-K knots,
// T = p / (rho R), gamma(T) = cp / (cp - R), E0 = h(T) - p/rho + |V|^2/2, H0 = h(T) + |V|^2/2,
// and the state from the conserved variables by solving e(T) = h(T) - R T on the table.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int tab_knot(const Gas& g, double T) {   // int(T), kept in the table
    if (!(T >= 0.0)) return 0;
    if (T >= (double)(g.ntab - 2)) return g.ntab - 2;
    return (int)T;
}
__device__ __forceinline__ double tab_at(const Gas& g, const double* t, double T) {
    const int Ti = tab_knot(g, T);
    const double dT = T - Ti;
    const double a = __ldg(t + Ti), b = __ldg(t + Ti + 1);
    return a + (b - a) * dT;
}
__device__ __forceinline__ double h_of_T(const Gas& g, double T) {
    return g.htab ? tab_at(g, g.htab, T) : g.cp * T;
}
__device__ __forceinline__ double cp_of_T(const Gas& g, double T) {
    return g.htab ? tab_at(g, g.cptab, T) : g.cp;
}
__device__ __forceinline__ double f_gamma(const Gas& g, double p, double rho) {
    if (!g.htab) return g.gamma;
    const double cp = tab_at(g, g.cptab, p / (rho * g.R));
    return cp / (cp - g.R);
}
__device__ __forceinline__ double f_ss(const Gas& g, double p, double rho) {
    if (g.htab) return sqrt(f_gamma(g, p, rho) * p / rho);
    return sqrt(g.gamma * p * (1.0 / rho));   // 1 / rho shared with the Roe averages' reciprocal
}
__device__ __forceinline__ double E0(const Gas& g, double p, double rho, double modv) {
    if (g.htab) return tab_at(g, g.htab, p / (rho * g.R)) - p / rho + 0.5 * modv * modv;
    return p / (g.gm1 * rho) + 0.5 * modv * modv;
}
__device__ __forceinline__ double H0(const Gas& g, double p, double rho, double modv) {
    if (g.htab) return tab_at(g, g.htab, p / (rho * g.R)) + 0.5 * modv * modv;
    return g.gamma * p / (g.gm1 * rho) + 0.5 * modv * modv;
}
// rho E of a primitive state on the table: rho h(T) - p + rho |V|^2 / 2.
__device__ __forceinline__ double rhoE_tab(const Gas& g, const double* P) {
    return P[0] * tab_at(g, g.htab, P[3] / (P[0] * g.R)) - P[3] + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
}
// Temperature of the specific internal energy e on the table, from the knot interval of the
// guess T0 walked to the interval holding e (e(T) increases with T where cp > R), then solved
// exactly on that interval (e is linear between knots).
__device__ __forceinline__ double T_of_e(const Gas& g, double e, double T0) {
    int k = tab_knot(g, T0);
    double ek = __ldg(g.htab + k) - g.R * (double)k;
    for (int w = 0; w < g.ntab && k > 0 && e < ek; ++w) {
        --k;
        ek = __ldg(g.htab + k) - g.R * (double)k;
    }
    double ek1 = __ldg(g.htab + k + 1) - g.R * (double)(k + 1);
    for (int w = 0; w < g.ntab && k < g.ntab - 2 && e >= ek1; ++w) {
        ++k;
        ek = ek1;
        ek1 = __ldg(g.htab + k + 1) - g.R * (double)(k + 1);
    }
    return (double)k + (e - ek) / (ek1 - ek);
}
__device__ __forceinline__ bool gas_state_bad(double rho, double p) {
    return !(rho > 0.0) || !(p > 0.0);
}

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// SD_Tramel (Lib_Shock_Detector.f90:14-38): pressure sensor on the cross stencil p1 = p(i-1,j),
// p2 = p(i+1,j), p3 = p(i,j-1), p4 = p(i,j+1). 0 where max(kp1, kp2) >= 1/20 (a shock), else
// 1 - tanh(10 phi^3), phi = sw/20 (within 1.6e-7 of 1).
__device__ __forceinline__ double sd_tramel(double p, double p1, double p2, double p3, double p4) {
    const double kp1 = fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
    const double kp2 = fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
    const double sw = kp1 > kp2 ? kp1 : kp2;
    if (sw < 1.0 / 20.0) {
        const double phi = sw / 20.0 > 0.0 ? sw / 20.0 : 0.0;
        return 1.0 - tanh(10.0 * phi * phi * phi);
    }
    return 0.0;
}
__device__ __forceinline__ float sd_tramel32(float p, float p1, float p2, float p3, float p4) {
    const float kp1 = fabsf((p2 - 2.0f * p + p1) / (p2 + 2.0f * p + p1));
    const float kp2 = fabsf((p4 - 2.0f * p + p3) / (p4 + 2.0f * p + p3));
    const float sw = kp1 > kp2 ? kp1 : kp2;
    if (sw < 1.0f / 20.0f) {
        const float phi = sw / 20.0f > 0.0f ? sw / 20.0f : 0.0f;
        return 1.0f - tanhf(10.0f * phi * phi * phi);
    }
    return 0.0f;
}
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// Limiters, FP64, operation order of Lib_Limiters.f90:26-110.
__device__ __forceinline__ double rlimiter(int lim, double x, double y) {
    if (lim == 1) {                                   // minmod :36-46
        double r = 0.0;
        if (x * y < 0.0) return r;
        r = x;
        if (fabs(x) > fabs(y)) r = y;
        return r;
    }
    if (lim == 0) return 0.0;                         // IORD
    const double ru = y / (x + 1e-30);
    double phi;
    switch (lim) {
        case 2: phi = (ru + fabs(ru)) / (1.0 + fabs(ru)); break;                       // vanleer
        case 3: phi = (ru * ru + ru) / (1.0 + ru * ru); break;                          // vanalbada
        case 4: phi = dmax(0.0, dmin(dmin(2.0 * ru, 0.5 * (1.0 + ru)), 2.0)); break;   // MC
        case 5: phi = dmax(dmax(0.0, dmin(2.0 * ru, 1.0)), dmin(ru, 2.0)); break;       // superbee
        default: {                                                                      // LIMO3
            const double a = (2.0 + ru) / 3.0;
            const double inner = dmin(dmin(2.0 * ru, (2.0 + ru) / 3.0), 1.6);
            const double mid = dmax(dmax(-0.5 * ru, 0.0), inner);
            phi = dmax(0.0, dmin(a, mid));
        }
    }
    return phi * x;
}

// Limiters, FP32, division-free algebraic equivalents of phi(y/x)*x (x = 0 gives 0 like the
// reference's epsilon form).
__device__ __forceinline__ float rlimiter32(int lim, float x, float y) {
    switch (lim) {
        case 0: return 0.0f;
        case 1: {
            if (x * y < 0.0f) return 0.0f;
            return fabsf(x) > fabsf(y) ? y : x;
        }
        case 2: {   // 2xy/(x+y) when xy > 0
            const float xy = x * y;
            return xy > 0.0f ? __fdividef(2.0f * xy, x + y) : 0.0f;
        }
        case 3: {   // xy(x+y)/(x^2+y^2)
            const float d = x * x + y * y;
            return d > 0.0f ? __fdividef(x * y * (x + y), d) : 0.0f;
        }
        case 4: {   // MC
            const float a = fminf(fminf(2.0f * y, 0.5f * (x + y)), 2.0f * x);
            const float b = fmaxf(fmaxf(2.0f * y, 0.5f * (x + y)), 2.0f * x);
            return x > 0.0f ? fmaxf(0.0f, a) : (x < 0.0f ? fminf(0.0f, b) : 0.0f);
        }
        case 5: {   // superbee
            if (x > 0.0f) return fmaxf(fmaxf(0.0f, fminf(2.0f * y, x)), fminf(y, 2.0f * x));
            if (x < 0.0f) return fminf(fminf(0.0f, fmaxf(2.0f * y, x)), fmaxf(y, 2.0f * x));
            return 0.0f;
        }
        default: {  // LIMO3
            const float t = (2.0f * x + y) * (1.0f / 3.0f);
            if (x > 0.0f) {
                const float inner = fminf(fminf(2.0f * y, t), 1.6f * x);
                const float mid = fmaxf(fmaxf(-0.5f * y, 0.0f), inner);
                return fmaxf(0.0f, fminf(t, mid));
            }
            if (x < 0.0f) {
                const float inner = fmaxf(fmaxf(2.0f * y, t), 1.6f * x);
                const float mid = fminf(fminf(-0.5f * y, 0.0f), inner);
                return fminf(0.0f, fmaxf(t, mid));
            }
            return 0.0f;
        }
    }
}


// Compile-time limiter selection for the hot loops (same arithmetic as rlimiter/rlimiter32).
template <int LIM>
__device__ __forceinline__ double lim64(double x, double y) {
    if (LIM == 1) {
        double r = 0.0;
        if (x * y < 0.0) return r;
        r = x;
        if (fabs(x) > fabs(y)) r = y;
        return r;
    }
    if (LIM == 0) return 0.0;
    if (LIM == 2) {   // van Leer with one division: phi(ru) x = 2 x y / ((x + 1e-30) + y) for ru > 0
        const double xe = x + 1e-30;
        return y * xe > 0.0 ? (2.0 * x * y) / (xe + y) : 0.0;
    }
    const double ru = y / (x + 1e-30);
    double phi;
    if (LIM == 2) phi = (ru + fabs(ru)) / (1.0 + fabs(ru));
    else if (LIM == 3) phi = (ru * ru + ru) / (1.0 + ru * ru);
    else if (LIM == 4) phi = dmax(0.0, dmin(dmin(2.0 * ru, 0.5 * (1.0 + ru)), 2.0));
    else if (LIM == 5) phi = dmax(dmax(0.0, dmin(2.0 * ru, 1.0)), dmin(ru, 2.0));
    else {
        const double a = (2.0 + ru) / 3.0;
        const double inner = dmin(dmin(2.0 * ru, (2.0 + ru) / 3.0), 1.6);
        const double mid = dmax(dmax(-0.5 * ru, 0.0), inner);
        phi = dmax(0.0, dmin(a, mid));
    }
    return phi * x;
}
template <int LIM>
__device__ __forceinline__ float lim32(float x, float y) { return rlimiter32(LIM, x, y); }

struct F4 { double r, u, v, e; };

// roe_averages (Lib_Riemann_HLL.f90:229-317), constant-cp identities, same operation order
// as the oracle.
__device__ __forceinline__ void roe_averages(const Gas& g, double dltot, double drtot, double ul,
                                             double vl, double ur, double vr, double pl,
                                             double pr, double& h0l, double& h0r,
                                             double& u_roe, double& v_roe, double& a_roe,
                                             double& rho_roe, double& h0_roe) {
    const double inv_dltot = 1.0 / dltot;
    const double inv_drtot = 1.0 / drtot;
    const double Tl = pl * inv_dltot * g.iR;
    const double Tr = pr * inv_drtot * g.iR;
    const double srL = sqrt(dltot);
    const double srR = sqrt(drtot);
    const double inv_sr = 1.0 / (srL + srR);
    rho_roe = srL * srR;
    u_roe = (srR * ur + srL * ul) * inv_sr;
    v_roe = (srR * vr + srL * vl) * inv_sr;
    const double R_roe = (srR * g.R + srL * g.R) * inv_sr;
    const double T_roe = (srR * Tr + srL * Tl) * inv_sr;
    const double hl = h_of_T(g, Tl);
    const double hr = h_of_T(g, Tr);
    const double el = hl - g.R * Tl;
    const double er = hr - g.R * Tr;
    h0l = 0.0 + hl * dltot * inv_dltot;
    h0r = 0.0 + hr * drtot * inv_drtot;
    const double d_roe = (srR * drtot * inv_drtot + srL * dltot * inv_dltot) * inv_sr;
    const double cv_roe = 0.0 + d_roe * (0.5 * (cp_of_T(g, Tl) + cp_of_T(g, Tr)) - g.R);
    const double sum_ei = 0.0 + d_roe * (srR * er + srL * el) * inv_sr;
    h0l = h0l + 0.5 * (ul * ul + vl * vl);
    h0r = h0r + 0.5 * (ur * ur + vr * vr);
    h0_roe = (srR * h0r + srL * h0l) * inv_sr;
    const double gam_roe = 1.0 + R_roe / cv_roe;
    const double vel2 = u_roe * u_roe + v_roe * v_roe;
    a_roe = sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
}

// riemann_HLLC (Lib_Riemann_HLL.f90:34-123), FP64.
__device__ __forceinline__ F4 riemann_hllc(const Gas& g, const double* L, double al,
                                           const double* R, double ar, double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    F4 F;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe;
    roe_averages(g, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double e0l = h0l - pl * (1.0 / dltot);   // the Roe averages' reciprocals
    const double e0r = h0r - pr * (1.0 / drtot);
    const double S1 = dmin(dmin(0.0, unl - al), un_roe - a_roe);
    const double S4 = dmax(dmax(0.0, unr + ar), un_roe + a_roe);
    double inv_denom = 1.0 / (dltot * (S1 - unl) - drtot * (S4 - unr));
    const double Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
    const double pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    if (S1 >= 0.0) {
        F.r = dltot * unl;
        F.u = F.r * ul + pl * nx;
        F.v = F.r * vl + pl * ny;
        F.e = F.r * h0l;
    } else if (Sstar >= 0.0) {
        F.r = dltot * unl;
        F.u = F.r * ul + pl * nx;
        F.v = F.r * vl + pl * ny;
        F.e = F.r * h0l;
        inv_denom = 1.0 / (S1 - Sstar);
        const double U1S = dltot * (S1 - unl) * inv_denom;
        const double U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * inv_denom;
        const double U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * inv_denom;
        const double U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * inv_denom;
        F.r = F.r + S1 * (U1S - dltot);
        F.u = F.u + S1 * (U2S - dltot * ul);
        F.v = F.v + S1 * (U3S - dltot * vl);
        F.e = F.e + S1 * (U5S - dltot * e0l);
    } else if (S4 > 0.0) {
        F.r = drtot * unr;
        F.u = F.r * ur + pr * nx;
        F.v = F.r * vr + pr * ny;
        F.e = F.r * h0r;
        inv_denom = 1.0 / (S4 - Sstar);
        const double U1S = drtot * (S4 - unr) * inv_denom;
        const double U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * inv_denom;
        const double U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * inv_denom;
        const double U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * inv_denom;
        F.r = F.r + S4 * (U1S - drtot);
        F.u = F.u + S4 * (U2S - drtot * ur);
        F.v = F.v + S4 * (U3S - drtot * vr);
        F.e = F.e + S4 * (U5S - drtot * e0r);
    } else {
        F.r = drtot * unr;
        F.u = F.r * ur + pr * nx;
        F.v = F.r * vr + pr * ny;
        F.e = F.r * h0r;
    }
    return F;
}

// riemann_HLLE (Lib_Riemann_HLL.f90:126-169), FP64.
__device__ __forceinline__ F4 riemann_hlle(const Gas& g, const double* L, double al,
                                           const double* R, double ar, double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    F4 F;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe;
    roe_averages(g, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double S1 = dmin(dmin(0.0, unl - al), un_roe - a_roe);
    const double S4 = dmax(dmax(0.0, unr + ar), un_roe + a_roe);
    const double inv_denom = 1.0 / (S4 - S1);
    const double FrL = dltot * unl;
    const double FrR = drtot * unr;
    F.r = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
    F.u = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) +
           S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
    F.v = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) +
           S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
    F.e = (S4 * (FrL * h0l) - S1 * (FrR * h0r) +
           S1 * S4 * (drtot * (h0r - pr * (1.0 / drtot)) - dltot * (h0l - pl * (1.0 / dltot)))) * inv_denom;
    return F;
}

// riemann_LLF (Lib_Riemann_LF.f90:11-40) with fluxes (:101-118), FP64.
__device__ __forceinline__ F4 phys_flux(const Gas& g, double p, double r, double u, double v,
                                        double nx, double ny) {
    F4 F;
    F.r = r * (u * nx + v * ny);
    F.u = F.r * u + p * nx;
    F.v = F.r * v + p * ny;
    F.e = F.r * H0(g, p, r, sqrt(u * u + v * v));
    return F;
}
__device__ __forceinline__ F4 riemann_llf(const Gas& g, const double* L, double al,
                                          const double* R, double ar, double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    F4 F;
    const double uln = ul * nx + vl * ny;
    const double urn = ur * nx + vr * ny;
    const double A = dmax(dmax(dmax(fabs(uln - al), fabs(urn - ar)), fabs(uln + al)), fabs(urn + ar));
    const F4 Fr = phys_flux(g, pr, drtot, ur, vr, nx, ny);
    const F4 Fl = phys_flux(g, pl, dltot, ul, vl, nx, ny);
    F.r = 0.5 * (Fl.r + Fr.r - A * (drtot - dltot));
    F.u = 0.5 * (Fr.u + Fl.u - A * (drtot * ur - dltot * ul));
    F.v = 0.5 * (Fr.v + Fl.v - A * (drtot * vr - dltot * vl));
    F.e = 0.5 * (Fl.e + Fr.e - A * (drtot * E0(g, pr, drtot, sqrt(ur * ur + vr * vr)) -
                                    dltot * E0(g, pl, dltot, sqrt(ul * ul + vl * vl))));
    return F;
}

// riemann_SLAU_base + riemann_SLAU / riemann_SLAU2 (Lib_Riemann_SLAU.f90:10-124), FP64, the
// reference's operation order: mass flux from the density-weighted normal speed with the
// low-Mach pressure term, pressure flux by Mach-split weights (SLAU: (1 - chi) blend; SLAU2:
// |V| a_F scaling), momentum and total enthalpy upwinded on the mass flux.
template <bool SLAU2>
__device__ __forceinline__ F4 riemann_slau(const Gas& g, const double* L, double al, const double* R, double ar,
                                           double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double sq_veli = ul * ul + vl * vl;
    const double sq_velj = ur * ur + vr * vr;
    const double aF = 0.5 * (al + ar);
    const double mL = unl / aF;
    const double mR = unr / aF;
    const double Mach_tilde = dmin(1.0, sqrt(0.5 * (sq_veli + sq_velj)) / aF);
    const double Chi = (1.0 - Mach_tilde) * (1.0 - Mach_tilde);
    const double Vn_mag = (dltot * fabs(unl) + drtot * fabs(unr)) / (dltot + drtot);
    const double f_rho = -dmax(dmin(mL, 0.0), -1.0) * dmin(dmax(mR, 0.0), 1.0);
    const double Vn_magL = (1.0 - f_rho) * Vn_mag + f_rho * fabs(unl);
    const double Vn_magR = (1.0 - f_rho) * Vn_mag + f_rho * fabs(unr);
    F4 F;
    F.r = 0.5 * (dltot * (unl + Vn_magL) + drtot * (unr - Vn_magR) - (Chi / aF) * (pr - pl));
    double BetaL, BetaR;
    if (fabs(mL) < 1.0) BetaL = 0.25 * (2.0 - mL) * ((mL + 1.0) * (mL + 1.0));
    else BetaL = mL >= 0.0 ? 1.0 : 0.0;
    if (fabs(mR) < 1.0) BetaR = 0.25 * (2.0 + mR) * ((mR - 1.0) * (mR - 1.0));
    else BetaR = mR >= 0.0 ? 0.0 : 1.0;
    const double p_half = SLAU2
        ? 0.5 * (pl + pr) + 0.5 * (BetaL - BetaR) * (pl - pr) +
              sqrt(0.5 * (sq_veli + sq_velj)) * (BetaL + BetaR - 1.0) * aF * 0.5 * (dltot + drtot)
        : 0.5 * (pl + pr) + 0.5 * (BetaL - BetaR) * (pl - pr) +
              (1.0 - Chi) * (BetaL + BetaR - 1.0) * 0.5 * (pl + pr);
    const double H_L = H0(g, pl, dltot, sqrt(sq_veli));
    const double H_R = H0(g, pr, drtot, sqrt(sq_velj));
    if (F.r >= 0.0) {
        F.u = F.r * ul + nx * p_half;
        F.v = F.r * vl + ny * p_half;
        F.e = F.r * H_L;
    } else {
        F.u = F.r * ur + nx * p_half;
        F.v = F.r * vr + ny * p_half;
        F.e = F.r * H_R;
    }
    return F;
}

// riemann_HLLEpp (Lib_Riemann_HLL.f90:437-533), FP64: centred flux minus the wave sum of a
// Roe linearisation whose eigenvalues blend Roe's (Harten-Hyman fix on the acoustic waves,
// hartenHyman :320-331) and HLLE's by the shock sensor beta.
__device__ __forceinline__ double harten_hyman(double v, double e) {
    const double al = fabs(v);
    return al <= e ? (v * v + e * e) / (2.0 * e) : al;
}
__device__ __forceinline__ F4 riemann_hllepp(const Gas& g, const double* L, double al, const double* R,
                                             double ar, double beta, double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe;
    roe_averages(g, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double Sm = dmin(dmin(0.0, unl - al), un_roe - a_roe);
    const double Sp = dmax(dmax(0.0, unr + ar), un_roe + a_roe);
    const double inv_denom = 1.0 / (Sp - Sm);
    const double lam1_hlle = fabs((Sp + Sm) * un_roe * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double lam2_hlle = fabs((Sp + Sm) * (un_roe - a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double lam3_hlle = fabs((Sp + Sm) * (un_roe + a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double eps = 0.3 * (fabs(un_roe) + a_roe);
    const double lam1 = beta * fabs(un_roe) + (1.0 - beta) * lam1_hlle;
    const double lam2 = beta * harten_hyman(un_roe - a_roe, eps) + (1.0 - beta) * lam2_hlle;
    const double lam3 = beta * harten_hyman(un_roe + a_roe, eps) + (1.0 - beta) * lam3_hlle;
    const F4 FL = phys_flux(g, pl, dltot, ul, vl, nx, ny);   // fluxes_helper (:334-352)
    const F4 FR = phys_flux(g, pr, drtot, ur, vr, nx, ny);
    F4 F;
    F.r = 0.5 * (FL.r + FR.r);
    F.u = 0.5 * (FL.u + FR.u);
    F.v = 0.5 * (FL.v + FR.v);
    F.e = 0.5 * (FL.e + FR.e);
    const double drho = drtot - dltot, dp = pr - pl, du = ur - ul, dv = vr - vl, dun = unr - unl;
    const double tx = -ny, ty = nx;
    const double alpha_m = (dp - rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
    const double alpha_c = drho - dp / (a_roe * a_roe);
    const double alpha_s = rho_roe * (du * tx + dv * ty);
    const double alpha_p = (dp + rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
    F.r = F.r - 0.5 * (alpha_c * lam1 + alpha_m * lam2 + alpha_p * lam3);
    F.u = F.u - 0.5 * (alpha_c * lam1 * u_roe + alpha_s * lam1 * tx + alpha_m * lam2 * (u_roe - a_roe * nx) +
                       alpha_p * lam3 * (u_roe + a_roe * nx));
    F.v = F.v - 0.5 * (alpha_c * lam1 * v_roe + alpha_s * lam1 * ty + alpha_m * lam2 * (v_roe - a_roe * ny) +
                       alpha_p * lam3 * (v_roe + a_roe * ny));
    F.e = F.e - 0.5 * (alpha_c * lam1 * 0.5 * (u_roe * u_roe + v_roe * v_roe) +
                       alpha_s * lam1 * (u_roe * tx + v_roe * ty) + alpha_m * lam2 * (h0_roe - a_roe * un_roe) +
                       alpha_p * lam3 * (h0_roe + a_roe * un_roe));
    return F;
}

// The Riemann solvers the reference offers beside the ones above, FP64, in the oracle's operation
// order; riemann64<kRiemGeneric> selects among them at run time (Gas::rkind).
// riemann_HLLEM (Lib_Riemann_HLL.f90:355-434): HLL plus antidiffusion on contact and shear.
static __device__ __noinline__ F4 riemann_hllem(const Gas& g, const double* L, double al, const double* R, double ar,
                                         double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    double h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe;
    roe_averages(g, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, u_roe, v_roe, a_roe, rho_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double S1 = dmin(dmin(0.0, (ul * nx + vl * ny) - al), un_roe - a_roe);
    const double S4 = dmax(dmax(0.0, (ur * nx + vr * ny) + ar), un_roe + a_roe);
    const F4 FL = phys_flux(g, pl, dltot, ul, vl, nx, ny);
    const F4 FR = phys_flux(g, pr, drtot, ur, vr, nx, ny);
    const double e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
    const double inv_denom = 1.0 / (S4 - S1);
    F4 F;
    F.r = (S4 * FL.r - S1 * FR.r + S1 * S4 * (drtot - dltot)) * inv_denom;
    F.u = (S4 * FL.u - S1 * FR.u + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
    F.v = (S4 * FL.v - S1 * FR.v + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
    F.e = (S4 * FL.e - S1 * FR.e + S1 * S4 * (drtot * e0r - dltot * e0l)) * inv_denom;
    if (S1 < 0.0 && S4 > 0.0) {
        const double drho = drtot - dltot, dp = pr - pl, du = ur - ul, dv = vr - vl;
        const double tx = -ny, ty = nx;
        const double alpha_c = drho - dp / (a_roe * a_roe);
        const double alpha_s = rho_roe * (du * tx + dv * ty);
        const double delta = a_roe / (a_roe + fabs(0.5 * (S1 + S4)));
        const double C = (S1 * S4) * inv_denom;
        F.r = F.r - C * delta * alpha_c;
        F.u = F.u - C * delta * (alpha_c * u_roe + alpha_s * tx);
        F.v = F.v - C * delta * (alpha_c * v_roe + alpha_s * ty);
        F.e = F.e - C * delta * (alpha_c * 0.5 * (u_roe * u_roe + v_roe * v_roe) + alpha_s * (u_roe * tx + v_roe * ty));
    }
    return F;
}

// riemann_HLLCHLLE (Lib_Riemann_HLL.f90:172-226): HLLE along the velocity jump, HLLC across it.
static __device__ __noinline__ F4 riemann_hllc_rotated(const Gas& g, const double* L, double al, const double* R,
                                                double ar, double nx, double ny) {
    const double ul = L[1], vl = L[2], ur = R[1], vr = R[2];
    const double abs_dv = sqrt((ur - ul) * (ur - ul) + (vr - vl) * (vr - vl));
    const double dum = 0.5 * (sqrt(ul * ul + vl * vl) + sqrt(ur * ur + vr * vr));
    if (abs_dv / (dum + 1.0e-10) > 1.0e-12) {
        double nx1 = (ur - ul) / abs_dv, ny1 = (vr - vl) / abs_dv;
        double alfa1 = nx * nx1 + ny * ny1;
        const double s1 = copysign(1.0, alfa1);
        nx1 = s1 * nx1; ny1 = s1 * ny1; alfa1 = s1 * alfa1;
        double nx2 = -ny1, ny2 = nx1;
        double alfa2 = nx * nx2 + ny * ny2;
        const double s2 = copysign(1.0, alfa2);
        nx2 = s2 * nx2; ny2 = s2 * ny2; alfa2 = s2 * alfa2;
        const F4 E = riemann_hlle(g, L, al, R, ar, nx1, ny1);
        const F4 C = riemann_hllc(g, L, al, R, ar, nx2, ny2);
        F4 F;
        F.r = E.r * alfa1 + C.r * alfa2;
        F.u = E.u * alfa1 + C.u * alfa2;
        F.v = E.v * alfa1 + C.v * alfa2;
        F.e = E.e * alfa1 + C.e * alfa2;
        return F;
    }
    return riemann_hllc(g, L, al, R, ar, nx, ny);
}

// Riemann_PLLF (Lib_Riemann_LF.f90:44-98): Rusanov with the preconditioned dissipation speed.
static __device__ __noinline__ F4 riemann_pllf(const Gas& g, const double* L, double al, const double* R, double ar,
                                        double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double uln = ul * nx + vl * ny;
    const double urn = ur * nx + vr * ny;
    const double U_rl = dmax(1e-5 * al, dmin(fabs(uln), al));
    const double U_rr = dmax(1e-5 * ar, dmin(fabs(urn), ar));
    const double betal = 1.0 / (al * al), betar = 1.0 / (ar * ar);
    const double alphal = 0.5 * (1.0 - betal * (U_rl * U_rl));
    const double alphar = 0.5 * (1.0 - betar * (U_rr * U_rr));
    const double ul_mod = fabs(uln * (1.0 - alphal));
    const double ur_mod = fabs(urn * (1.0 - alphar));
    const double al_mod = sqrt((alphal * alphal) * (uln * uln) + U_rl * U_rl);
    const double ar_mod = sqrt((alphar * alphar) * (urn * urn) + U_rr * U_rr);
    const double A = dmax(ul_mod + al_mod, ur_mod + ar_mod);
    const F4 Fr = phys_flux(g, pr, drtot, ur, vr, nx, ny);
    const F4 Fl = phys_flux(g, pl, dltot, ul, vl, nx, ny);
    F4 F;
    F.r = 0.5 * (Fl.r + Fr.r - A * (drtot - dltot));
    F.u = 0.5 * (Fr.u + Fl.u - A * (drtot * ur - dltot * ul));
    F.v = 0.5 * (Fr.v + Fl.v - A * (drtot * vr - dltot * vl));
    F.e = 0.5 * (Fl.e + Fr.e - A * (drtot * E0(g, pr, drtot, sqrt(ur * ur + vr * vr)) -
                                    dltot * E0(g, pl, dltot, sqrt(ul * ul + vl * vl))));
    return F;
}

// riemann_exact (Lib_Riemann_Godunov.f90:14-248): Newton iteration on the contact velocity
// (|1 - p2/p3| < 1e-5, at most 1001 passes; bounded), the sampled state at x/t = 0, its flux.
__device__ __forceinline__ void ex_rare(double ps, double as, double us, double ud, double sgn, double gamma,
                                        double& pd, double& ad, double& dp, double& v1, double& v2) {
    // rareleft (sgn = +1): ad = as - delta (ud - us), v1 = us - as, v2 = ud - ad; rareright
    // (sgn = -1, with the roles of the two states exchanged): ad = as + delta (ud - us),
    // v1 = ud + ad, v2 = us + as
    const double delta = 0.5 * (gamma - 1.0);
    const double dum1 = 2.0 * gamma / (gamma - 1.0);
    ad = sgn > 0.0 ? as - delta * (ud - us) : as + delta * (ud - us);
    pd = ps * pow(ad / as, dum1);
    dp = sgn > 0.0 ? -gamma * pd / ad : gamma * pd / ad;
    v1 = sgn > 0.0 ? us - as : ud + ad;
    v2 = sgn > 0.0 ? ud - ad : us + as;
}
__device__ __forceinline__ void ex_shock(double us, double as, double ps, double ud, double sgn, double gamma,
                                         double& ad, double& pd, double& dp, double& ws) {
    // shockleft (sgn = +1): M = x - sqrt(1 + x^2); shockright (sgn = -1): M = x + sqrt(1 + x^2)
    const double x = (gamma + 1.0) * (ud - us) / (4.0 * as);
    const double M = sgn > 0.0 ? x - sqrt(1.0 + x * x) : x + sqrt(1.0 + x * x);
    const double C = gamma * ps / as;
    pd = ps + C * (ud - us) * M;
    dp = 2.0 * C * (M * M * M) / (1.0 + M * M);
    const double rp = pd / ps;
    ws = us + as * M;
    ad = as * sqrt((gamma + 1.0 + (gamma - 1.0) * rp) / (gamma + 1.0 + (gamma - 1.0) / rp));
}
static __device__ __noinline__ F4 riemann_exact(const Gas& g, const double* L, double a1, const double* R, double a4,
                                         double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], p1 = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], p4 = R[3];
    const double gam1 = g.gamma, gam4 = g.gamma;
    const double gm1_1 = gam1 - 1.0, gm1_4 = gam4 - 1.0;
    const double delta1 = 0.5 * gm1_1, delta4 = 0.5 * gm1_4;
    const double eta1 = gam1 / delta1, eta4 = gam4 / delta4;
    const double un1 = ul * nx + vl * ny;
    const double ut1 = ul - un1 * nx, vt1 = vl - un1 * ny;
    const double un4 = ur * nx + vr * ny;
    const double ut4 = ur - un4 * nx, vt4 = vr - un4 * ny;
    const double R2I = un1 + (2.0 / gm1_1) * a1;
    const double R1IV = un4 - (2.0 / gm1_4) * a4;
    const double dum = p1 < p4 ? gm1_4 / (2.0 * gam4) : gm1_1 / (2.0 * gam1);
    const double z = (gm1_1 / gm1_4) * (a4 / a1) * pow(p1 / p4, dum);
    double vel = (z * R2I + R1IV) / (1.0 + z);
    double p3 = 1.0, p2 = 2.0 * p3, a2 = 0.0, a3 = 0.0, dpr = 0.0, dpl = 0.0;
    double sw_l = 0.0, sw_r = 0.0, vw1 = 0.0, vw2 = 0.0, vw3 = 0.0, vw4 = 0.0;
    for (int iter = 0; fabs(1.0 - (p2 / p3)) >= 1e-5 && iter <= 1000; ++iter) {
        if (vel < un1) ex_shock(un1, a1, p1, vel, 1.0, gam1, a2, p2, dpr, sw_l);
        else ex_rare(p1, a1, un1, vel, 1.0, gam1, p2, a2, dpr, vw1, vw2);
        if (vel > un4) ex_shock(un4, a4, p4, vel, -1.0, gam4, a3, p3, dpl, sw_r);
        else ex_rare(p4, a4, un4, vel, -1.0, gam4, p3, a3, dpl, vw3, vw4);
        vel = vel - ((p2 - p3) / (dpr - dpl));
    }
    double af, pf, rhof, uf, vf;
    if (vel > 0.0) {
        af = a2; pf = p2;
        if (vel <= un1) {
            if (sw_l > 0.0) { af = a1; vel = un1; pf = p1; }
        } else if (vw1 > 0.0) {
            vel = un1; af = a1; pf = p1;
        } else if (vw2 > 0.0) {
            af = (un1 + a1 / delta1) / (1.0 + 1.0 / delta1);
            vel = af;
            pf = p1 * pow(af / a1, eta1);
        }
        rhof = gam1 * pf / (af * af);
        rhof = dltot / dltot * rhof;
        uf = vel * nx + ut1;
        vf = vel * ny + vt1;
    } else {
        af = a3; pf = p3;
        if (vel >= un4) {
            if (sw_r < 0.0) { af = a4; vel = un4; pf = p4; }
        } else if (vw4 < 0.0) {
            af = a4; vel = un4; pf = p4;
        } else if (vw3 < 0.0) {
            af = -(un4 - a4 / delta4) / (1.0 + 1.0 / delta4);
            vel = -af;
            pf = p4 * pow(af / a4, eta4);
        }
        rhof = gam4 * pf / (af * af);
        rhof = drtot / drtot * rhof;
        uf = vel * nx + ut4;
        vf = vel * ny + vt4;
    }
    return phys_flux(g, pf, rhof, uf, vf, nx, ny);
}

// riemann_Hanel (Lib_Riemann_AUSM.f90:18-70): van Leer splitting of velocity and pressure.
static __device__ __noinline__ F4 riemann_hanel(const Gas& g, const double* L, double al, const double* R, double ar,
                                         double nx, double ny) {
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dltot, sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, drtot, sqrt(ur * ur + vr * vr));
    const double uLp = fabs(unl) <= al ? (unl + al) * (unl + al) / (4.0 * al) : 0.5 * (unl + fabs(unl));
    const double uRm = fabs(unr) <= ar ? (-((unr - ar) * (unr - ar))) / (4.0 * ar) : 0.5 * (unr - fabs(unr));
    const double pLp = fabs(unl) <= al ? pl * uLp * (2.0 - unl / al) / al : pl * uLp / unl;
    const double pRm = fabs(unr) <= ar ? pr * uRm * (-2.0 - unr / ar) / ar : pr * uRm / unr;
    const double phalf = pLp + pRm;
    F4 F;
    F.r = uLp * dltot + uRm * drtot;
    F.u = uLp * (dltot * ul) + uRm * (drtot * ur) + phalf * nx;
    F.v = uLp * (dltot * vl) + uRm * (drtot * vr) + phalf * ny;
    F.e = uLp * (dltot * H_L) + uRm * (drtot * H_R);
    return F;
}

// riemann_AUSMp (Lib_Riemann_AUSM.f90:73-128).
static __device__ __noinline__ F4 riemann_ausmp(const Gas& g, const double* L, double al, const double* R, double ar,
                                         double nx, double ny) {
    const double betap = 0.125, alpha = 0.1875;
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dltot, sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, drtot, sqrt(ur * ur + vr * vr));
    const double a_half = sqrt(al * ar);
    const double ML = unl / a_half, MR = unr / a_half;
    double MplusL, pplusL, MminusR, pminusR;
    if (fabs(ML) < 1.0) {
        const double q = (ML + 1.0) * (ML + 1.0), w = (ML * ML - 1.0) * (ML * ML - 1.0);
        MplusL = 0.25 * q + betap * w;
        pplusL = 0.25 * q * (2.0 - ML) + alpha * ML * w;
    } else {
        MplusL = 0.5 * (ML + fabs(ML));
        pplusL = 0.5 * (1.0 + copysign(1.0, ML));
    }
    if (fabs(MR) < 1.0) {
        const double q = (MR - 1.0) * (MR - 1.0), w = (MR * MR - 1.0) * (MR * MR - 1.0);
        MminusR = -0.25 * q - betap * w;
        pminusR = 0.25 * q * (2.0 + MR) - alpha * MR * w;
    } else {
        MminusR = 0.5 * (MR - fabs(MR));
        pminusR = 0.5 * (1.0 - copysign(1.0, MR));
    }
    const double Mhalf = MplusL + MminusR;
    const double phalf = pplusL * pl + pminusR * pr;
    const double mdotp = dltot * a_half * 0.5 * (Mhalf + fabs(Mhalf));
    const double mdotm = drtot * a_half * 0.5 * (Mhalf - fabs(Mhalf));
    F4 F;
    F.r = mdotp + mdotm;
    F.u = mdotp * ul + mdotm * ur + nx * phalf;
    F.v = mdotp * vl + mdotm * vr + ny * phalf;
    F.e = mdotp * H_L + mdotm * H_R;
    return F;
}

// riemann_AUSMp_up / riemann_AUSMp_up2 (Lib_Riemann_AUSM.f90:131-321).
static __device__ __noinline__ F4 riemann_ausmp_up(const Gas& g, bool up2, const double* L, const double* R, double nx,
                                            double ny) {
    const double Kp = 0.25, Ku = 0.75, sigma = 1.0, betap = 0.125;
    const double dltot = L[0], ul = L[1], vl = L[2], pl = L[3];
    const double drtot = R[0], ur = R[1], vr = R[2], pr = R[3];
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dltot, sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, drtot, sqrt(ur * ur + vr * vr));
    const double gamma_L = g.gamma, gamma_R = g.gamma;
    const double astarL2 = 2.0 * (gamma_L - 1.0) / (gamma_L + 1.0) * H_L;
    const double astarR2 = 2.0 * (gamma_R - 1.0) / (gamma_R + 1.0) * H_R;
    const double astarL = sqrt(astarL2), astarR = sqrt(astarR2);
    const double atildeL = astarL2 / dmax(astarL, unl);
    const double atildeR = astarR2 / dmax(astarR, -unr);
    const double aF = dmin(atildeL, atildeR);
    const double mL = unl / aF, mR = unr / aF;
    const double MFsq = 0.5 * (mL * mL + mR * mR);
    const double Mrefsq = dmin(1.0, dmax(MFsq, g.minf * g.minf));
    const double fa = 2.0 * sqrt(Mrefsq) - Mrefsq;
    const double alpha = 0.1875 * (-4.0 + 5.0 * fa * fa);
    double mLP, bLP, mRM, bRM;
    if (fabs(mL) <= 1.0) {
        const double p1 = 0.25 * ((mL + 1.0) * (mL + 1.0)), p2 = (mL * mL - 1.0) * (mL * mL - 1.0);
        mLP = p1 + betap * p2;
        bLP = p1 * (2.0 - mL) + alpha * mL * p2;
    } else {
        mLP = 0.5 * (mL + fabs(mL));
        bLP = mLP / mL;
    }
    if (fabs(mR) <= 1.0) {
        const double p1 = 0.25 * ((mR - 1.0) * (mR - 1.0)), p2 = (mR * mR - 1.0) * (mR * mR - 1.0);
        mRM = -p1 - betap * p2;
        bRM = p1 * (2.0 + mR) - alpha * mR * p2;
    } else {
        mRM = 0.5 * (mR - fabs(mR));
        bRM = mRM / mR;
    }
    const double rhoF = 0.5 * (dltot + drtot);
    const double Mp = -(Kp / fa) * dmax(0.0, 1.0 - sigma * MFsq) * (pr - pl) / (rhoF * aF * aF);
    const double mF = mLP + mRM + Mp;
    const double mdot = aF * (dmax(mF, 0.0) * dltot + dmin(mF, 0.0) * drtot);
    double phalf;
    if (up2) {
        const double sq_vel = 0.5 * ((ul * ul + vl * vl) + (ur * ur + vr * vr));
        phalf = 0.5 * (pr + pl) + 0.5 * (bLP - bRM) * (pl - pr) + sqrt(sq_vel) * (bLP + bRM - 1.0) * rhoF * aF;
    } else {
        const double Pu = -Ku * fa * bLP * bRM * 2.0 * rhoF * aF * (unr - unl);
        phalf = bLP * pl + bRM * pr + Pu;
    }
    const bool upw = mF >= 0.0;
    F4 F;
    F.r = mdot;
    F.u = mdot * (upw ? ul : ur) + nx * phalf;
    F.v = mdot * (upw ? vl : vr) + ny * phalf;
    F.e = mdot * (upw ? H_L : H_R);
    return F;
}

constexpr int kRiemGeneric = 7;   // instantiation id of the run-time selected solvers (ids 7-14)
static __device__ __noinline__ F4 riemann_generic(const Gas& g, const double* L, double al, const double* R, double ar,
                                           double nx, double ny) {
    switch (g.rkind) {
        case 8: return riemann_hllc_rotated(g, L, al, R, ar, nx, ny);
        case 9: return riemann_pllf(g, L, al, R, ar, nx, ny);
        case 10: return riemann_exact(g, L, al, R, ar, nx, ny);
        case 11: return riemann_hanel(g, L, al, R, ar, nx, ny);
        case 12: return riemann_ausmp(g, L, al, R, ar, nx, ny);
        case 13: return riemann_ausmp_up(g, false, L, R, nx, ny);
        case 14: return riemann_ausmp_up(g, true, L, R, nx, ny);
        default: return riemann_hllem(g, L, al, R, ar, nx, ny);
    }
}

// beta: the shock sensor of the face's cell for the sensor-driven solvers (HLLC+ blends HLLC and
// HLLE by it, riemann_HLLCSD, Lib_Riemann_HLL.f90:572-605; HLLE++); 1 from walls and inflows.
template <int RIEM>
__device__ __forceinline__ F4 riemann64(const Gas& g, const double* L, double al, const double* R,
                                        double ar, double nx, double ny, double beta = 1.0) {
    if (RIEM == 5) {
        if (beta == 0.0) return riemann_hlle(g, L, al, R, ar, nx, ny);
        if (beta >= 1.0) return riemann_hllc(g, L, al, R, ar, nx, ny);
        const F4 E = riemann_hlle(g, L, al, R, ar, nx, ny);
        const F4 C = riemann_hllc(g, L, al, R, ar, nx, ny);
        F4 F;
        F.r = beta * C.r + (1.0 - beta) * E.r;
        F.u = beta * C.u + (1.0 - beta) * E.u;
        F.v = beta * C.v + (1.0 - beta) * E.v;
        F.e = beta * C.e + (1.0 - beta) * E.e;
        return F;
    }
    if (RIEM == 6) return riemann_hllepp(g, L, al, R, ar, beta, nx, ny);
    if (RIEM == kRiemGeneric) return riemann_generic(g, L, al, R, ar, nx, ny);
    if (RIEM == 1) return riemann_hlle(g, L, al, R, ar, nx, ny);
    if (RIEM == 2) return riemann_llf(g, L, al, R, ar, nx, ny);
    if (RIEM == 3) return riemann_slau<false>(g, L, al, R, ar, nx, ny);
    if (RIEM == 4) return riemann_slau<true>(g, L, al, R, ar, nx, ny);
    return riemann_hllc(g, L, al, R, ar, nx, ny);
}

// Face flux from two reconstructed states (Lib_Convective.f90:56-80), FP64. Returns false on
// a non-physical state (check_gas_state).
template <int RIEM>
__device__ __forceinline__ bool flux_from_states64(const Gas& g, const double* P1, const double* P4,
                                                   double nx, double ny, double int_l, double* fl,
                                                   double beta = 1.0) {
    const bool bad = gas_state_bad(P1[0], P1[3]) || gas_state_bad(P4[0], P4[3]);
    const double a1 = f_ss(g, P1[3], P1[0]);
    const double a4 = f_ss(g, P4[3], P4[0]);
    const F4 F = riemann64<RIEM>(g, P1, a1, P4, a4, nx, ny, beta);
    // single species: sp*(rho1/rho1) - sm*(rho4/rho4) == 1 exactly
    fl[0] = F.r * int_l;
    fl[1] = F.u * int_l;
    fl[2] = F.v * int_l;
    fl[3] = F.e * int_l;
    return !bad;
}

// ---------------------------------------------------------------------------------------
// FP32-flux form. Reconstruction, limiter and the Riemann wave structure run in FP32; the
// physical fluxes of the two face states, the state jumps and the sum F = F_K + S_K (U*_K -
// U_K) stay FP64. (U*_K - U_K) is rewritten so that every FP32 product multiplies a state
// jump (S* - un_K, p* - p_K): FP32 rounding then scales with the jump, not with |F|.
// ---------------------------------------------------------------------------------------
struct FluxState {   // FP64 face state plus its physical flux (per unit normal)
    double r, u, v, p, un;
    F4 F;
};

__device__ __forceinline__ void phys64(const Gas& g, const double* q, double nx, double ny,
                                       FluxState& s) {
    s.r = q[0]; s.u = q[1]; s.v = q[2]; s.p = q[3];
    s.un = s.u * nx + s.v * ny;
    const double m = s.r * s.un;
    s.F.r = m;
    s.F.u = m * s.u + s.p * nx;
    s.F.v = m * s.v + s.p * ny;
    // un * (rho E + p) = un * (gamma/(gamma-1) p + rho |V|^2 / 2): no division
    s.F.e = s.un * (g.gfac * s.p + 0.5 * s.r * (s.u * s.u + s.v * s.v));
}

__device__ __forceinline__ float frcp(float x) { return __fdividef(1.0f, x); }

template <int RIEM>
__device__ __forceinline__ F4 riemann32(const Gas& g, const FluxState& L, const FluxState& R,
                                        float nx, float ny) {
    if (RIEM >= 3) {   // no FP32 wave structure of their own here: the FP64 solver on the face states
        const double ql[4] = {L.r, L.u, L.v, L.p}, qr[4] = {R.r, R.u, R.v, R.p};
        return riemann64<RIEM>(g, ql, f_ss(g, L.p, L.r), qr, f_ss(g, R.p, R.r), (double)nx, (double)ny);
    }
    // FP32 wave structure
    const float rl = (float)L.r, rr = (float)R.r;
    const float ul = (float)L.u, vl = (float)L.v, ur = (float)R.u, vr = (float)R.v;
    const float pl = (float)L.p, pr = (float)R.p;
    const float gam = (float)g.gamma;
    const float igm1 = (float)(1.0 / g.gm1);
    const float irl = frcp(rl), irr = frcp(rr);
    const float al = sqrtf(gam * pl * irl), ar = sqrtf(gam * pr * irr);
    const float unl = (float)L.un, unr = (float)R.un;
    // jumps, formed in FP64
    const float dp = (float)(R.p - L.p);
    const float dun = (float)(R.un - L.un);
    if (RIEM == 2) {   // LLF: F = (F_L + F_R)/2 - A/2 (U_R - U_L)
        const float A = fmaxf(fmaxf(fabsf(unl - al), fabsf(unr - ar)), fmaxf(fabsf(unl + al), fabsf(unr + ar)));
        const double dU0 = R.r - L.r;
        const double dU1 = R.r * R.u - L.r * L.u;
        const double dU2 = R.r * R.v - L.r * L.v;
        const double dU3 = (R.p * g.igm1 + 0.5 * R.r * (R.u * R.u + R.v * R.v)) -
                           (L.p * g.igm1 + 0.5 * L.r * (L.u * L.u + L.v * L.v));
        const double hA = 0.5 * (double)A;
        F4 F;
        F.r = 0.5 * (L.F.r + R.F.r) - hA * (double)(float)dU0;
        F.u = 0.5 * (L.F.u + R.F.u) - hA * (double)(float)dU1;
        F.v = 0.5 * (L.F.v + R.F.v) - hA * (double)(float)dU2;
        F.e = 0.5 * (L.F.e + R.F.e) - hA * (double)(float)dU3;
        return F;
    }
    // Roe averages (constant cp: gamma_roe = gamma, a^2 = (gamma-1)(h0 - |V|^2/2))
    const float srL = sqrtf(rl), srR = sqrtf(rr);
    const float isr = frcp(srL + srR);
    const float u_roe = (srR * ur + srL * ul) * isr;
    const float v_roe = (srR * vr + srL * vl) * isr;
    const float gf = (float)g.gfac;
    const float h0l = gf * pl * irl + 0.5f * (ul * ul + vl * vl);
    const float h0r = gf * pr * irr + 0.5f * (ur * ur + vr * vr);
    const float h0_roe = (srR * h0r + srL * h0l) * isr;
    const float a_roe = sqrtf(fmaxf((gam - 1.0f) * (h0_roe - 0.5f * (u_roe * u_roe + v_roe * v_roe)), 0.0f));
    const float un_roe = u_roe * nx + v_roe * ny;
    const float S1 = fminf(fminf(0.0f, unl - al), un_roe - a_roe);
    const float S4 = fmaxf(fmaxf(0.0f, unr + ar), un_roe + a_roe);
    if (RIEM == 1) {   // HLLE: F = Fbar - (S4+S1)/(2(S4-S1)) dF + S1 S4/(S4-S1) dU
        const float inv = frcp(S4 - S1);
        const float c1 = 0.5f * (S4 + S1) * inv;
        const float c2 = S1 * S4 * inv;
        const double dU0 = R.r - L.r;
        const double dU1 = R.r * R.u - L.r * L.u;
        const double dU2 = R.r * R.v - L.r * L.v;
        const double dU3 = (R.p * g.igm1 + 0.5 * R.r * (R.u * R.u + R.v * R.v)) -
                           (L.p * g.igm1 + 0.5 * L.r * (L.u * L.u + L.v * L.v));
        F4 F;
        F.r = 0.5 * (L.F.r + R.F.r) + (double)(c2 * (float)dU0 - c1 * (float)(R.F.r - L.F.r));
        F.u = 0.5 * (L.F.u + R.F.u) + (double)(c2 * (float)dU1 - c1 * (float)(R.F.u - L.F.u));
        F.v = 0.5 * (L.F.v + R.F.v) + (double)(c2 * (float)dU2 - c1 * (float)(R.F.v - L.F.v));
        F.e = 0.5 * (L.F.e + R.F.e) + (double)(c2 * (float)dU3 - c1 * (float)(R.F.e - L.F.e));
        return F;
    }
    // HLLC (Batten), jump form
    if (S1 >= 0.0f) return L.F;
    const float D = rl * (S1 - unl) - rr * (S4 - unr);
    const float sm_unl = (dp - rr * (S4 - unr) * dun) * frcp(D);   // S* - un_L
    const float Sstar = unl + sm_unl;
    if (Sstar >= 0.0f) {
        const float inv = frcp(S1 - Sstar);
        const float q = sm_unl * inv;
        const float dps = rl * (S1 - unl) * sm_unl;                      // p* - p_L
        const float e0l = pl * irl * igm1 + 0.5f * (ul * ul + vl * vl);
        const float d0 = rl * q;
        const float d1 = rl * ul * q + dps * nx * inv;
        const float d2 = rl * vl * q + dps * ny * inv;
        const float d3 = rl * e0l * q + (dps * Sstar + pl * sm_unl) * inv;
        F4 F;
        F.r = L.F.r + (double)(S1 * d0);
        F.u = L.F.u + (double)(S1 * d1);
        F.v = L.F.v + (double)(S1 * d2);
        F.e = L.F.e + (double)(S1 * d3);
        return F;
    }
    if (S4 > 0.0f) {
        const float inv = frcp(S4 - Sstar);
        const float sm_unr = sm_unl - dun;                               // S* - un_R
        const float q = sm_unr * inv;
        const float dps = rr * (S4 - unr) * sm_unr;                      // p* - p_R
        const float e0r = pr * irr * igm1 + 0.5f * (ur * ur + vr * vr);
        const float d0 = rr * q;
        const float d1 = rr * ur * q + dps * nx * inv;
        const float d2 = rr * vr * q + dps * ny * inv;
        const float d3 = rr * e0r * q + (dps * Sstar + pr * sm_unr) * inv;
        F4 F;
        F.r = R.F.r + (double)(S4 * d0);
        F.u = R.F.u + (double)(S4 * d1);
        F.v = R.F.v + (double)(S4 * d2);
        F.e = R.F.e + (double)(S4 * d3);
        return F;
    }
    return R.F;
}

}  // namespace q2d
