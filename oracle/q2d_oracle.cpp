// q2d_oracle.cpp — CPU oracle: C++ restatement of Q2D's explicit residual + update path.
//
// TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline). Each routine names the
// reference Fortran file:line it restates (paths relative to the open-hydra/Q2D tree).
// Loop nesting, accumulation order and operation order follow the Fortran so that the
// oracle is the reference's arithmetic up to the thermodynamic closure (FLINT is absent;
// the calorically perfect single-species closure implied by the constant-cp tables is
// used, see the THERMO section). OpenMP parallelises the cell loops the way the
// reference's `!$omp do` does; every reduction is summed in a fixed order.
#include "q2d_oracle.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <cfloat>
#include <vector>
#include <algorithm>
#include <new>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int GC = 2;      // Global_m.f90:25
constexpr int NPRIM = 4;   // rho, u, v, p (nsc = 1)

// guide(f,:) for faces 1..4 (Parameters_m.f90:13-18)
constexpr int GUIDE[5][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}};

// ---------------------------------------------------------------------------------------
// THERMO: single-species closures standing in for FLINT_Lib_Thermodynamic (an un-vendored
// submodule of the reference; its documented formulas are in docs/theory/thermo.md:39-99).
// Calorically perfect (the default, what the reference's constant-cp gas tables give):
//   co_rotot_Rtot -> rho = rho_1, R = gas_R ; f_ss -> sqrt(gamma p / rho) ; f_gamma -> gamma
//   E0(p,rho,|V|) = p/((gamma-1) rho) + |V|^2/2 ; H0 = gamma p/((gamma-1) rho) + |V|^2/2
//   h_tab/cp_tab lerp -> h = cp T, cp = gamma R/(gamma-1)
//   prim2cons -> (rho, rho u, rho v, p/(gamma-1) + rho |V|^2/2)
//   cons2prim -> p = (gamma-1)(rho E - rho |V|^2/2)
// Thermally perfect (a table set by q2d_oracle_set_thermo_table): h(T) and cp(T) on 1-K knots,
// interpolated linearly at int(T) (f_tabT_expr, as called at Lib_Riemann_HLL.f90:258-291 and
// Lib_Newstate.f90:281-282), T = p / (rho R):
//   gamma(T) = cp / (cp - R) ; f_ss -> sqrt(gamma(T) p / rho) ; e(T) = h(T) - R T
//   E0 = h(T) - p/rho + |V|^2/2 ; H0 = h(T) + |V|^2/2 ; prim2cons -> rho E = rho h(T) - p + ..
//   cons2prim -> T solving e(T) = E - |V|^2/2 on the interpolated table (e is linear between
//   knots: the knot interval is found from the temperature guess, then solved exactly),
//   p = rho R T.
// ---------------------------------------------------------------------------------------
struct Gas {
    double R, gamma, gm1, cp, cv;
    double minf = 0.0;   // riemann-options-Minf (AUSM+-up, AUSM+-up2)
    const double* htab = nullptr;    // thermally perfect: h(T) [J/kg] at T = 0, 1, .. ntab-1 K
    const double* cptab = nullptr;   //   cp(T) [J/(kg K)] on the same knots
    int ntab = 0;
};

// Knot interval of T: int(T) (truncation, T >= 0), kept inside the table; a T past either end
// extrapolates its end interval.
inline int tab_knot(const Gas& g, double T) {
    if (!(T >= 0.0)) return 0;
    if (T >= (double)(g.ntab - 2)) return g.ntab - 2;
    return (int)T;
}
inline double tab_at(const Gas& g, const double* t, double T) {
    const int Ti = tab_knot(g, T);
    const double dT = T - Ti;
    return t[Ti] + (t[Ti + 1] - t[Ti]) * dT;
}
inline double h_of_T(const Gas& g, double T) { return g.htab ? tab_at(g, g.htab, T) : g.cp * T; }
inline double cp_of_T(const Gas& g, double T) { return g.htab ? tab_at(g, g.cptab, T) : g.cp; }
inline double f_gamma(const Gas& g, double p, double rho) {
    if (!g.htab) return g.gamma;
    const double cp = tab_at(g, g.cptab, p / (rho * g.R));
    return cp / (cp - g.R);
}
inline double f_ss(const Gas& g, double p, double rho) {
    if (!g.htab) return std::sqrt(g.gamma * p / rho);
    return std::sqrt(f_gamma(g, p, rho) * p / rho);
}
inline double E0(const Gas& g, double p, double rho, double modv) {
    if (g.htab) return tab_at(g, g.htab, p / (rho * g.R)) - p / rho + 0.5 * modv * modv;
    return p / (g.gm1 * rho) + 0.5 * modv * modv;
}
inline double H0(const Gas& g, double p, double rho, double modv) {
    if (g.htab) return tab_at(g, g.htab, p / (rho * g.R)) + 0.5 * modv * modv;
    return g.gamma * p / (g.gm1 * rho) + 0.5 * modv * modv;
}
inline void prim2cons(const Gas& g, const double* P, double* U) {
    U[0] = P[0];
    U[1] = P[0] * P[1];
    U[2] = P[0] * P[2];
    if (g.htab)
        U[3] = P[0] * tab_at(g, g.htab, P[3] / (P[0] * g.R)) - P[3] + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
    else
        U[3] = P[3] / g.gm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
}
// Temperature of the specific internal energy e on the interpolated table, from the knot
// interval of the guess T0 (walked to the interval holding e; e(T) = h(T) - R T increases
// with T for cp > R).
inline double T_of_e(const Gas& g, double e, double T0) {
    int k = tab_knot(g, T0);
    auto ek = [&](int n) { return g.htab[n] - g.R * (double)n; };
    for (int w = 0; w < g.ntab && k > 0 && e < ek(k); ++w) --k;
    for (int w = 0; w < g.ntab && k < g.ntab - 2 && e >= ek(k + 1); ++w) ++k;
    return (double)k + (e - ek(k)) / (ek(k + 1) - ek(k));
}
// cons2prim(cons, temperature): the guess is the temperature of the state before the update.
inline void cons2prim(const Gas& g, const double* U, double* P, double Tguess = 0.0) {
    const double rho = U[0];
    const double u = U[1] / rho;
    const double v = U[2] / rho;
    P[0] = rho;
    P[1] = u;
    P[2] = v;
    if (g.htab) {
        const double T = T_of_e(g, U[3] / rho - 0.5 * (u * u + v * v), Tguess);
        P[3] = rho * g.R * T;
    } else {
        P[3] = g.gm1 * (U[3] - 0.5 * rho * (u * u + v * v));
    }
}
// check_gas_state (Lib_Convective.f90:49-54): non-physical when rho<=0, p<=0 or NaN.
inline bool gas_state_bad(double rho, double p) { return !(rho > 0.0) || !(p > 0.0); }

// ---------------------------------------------------------------------------------------
// Limiters (Lib_Limiters.f90:26-110)
// ---------------------------------------------------------------------------------------
inline double lim_minmod(double x, double y) {          // :36-46
    double r = 0.0;
    if (x * y < 0.0) return r;
    r = x;
    if (std::fabs(x) > std::fabs(y)) r = y;
    return r;
}
inline double lim_vanleer(double x, double y) {         // :49-58
    double ru = y / (x + 1e-30);
    double phi = (ru + std::fabs(ru)) / (1.0 + std::fabs(ru));
    return phi * x;
}
inline double lim_vanalbada(double x, double y) {       // :61-70
    double ru = y / (x + 1e-30);
    double phi = (ru * ru + ru) / (1.0 + ru * ru);
    return phi * x;
}
inline double fmax_(double a, double b) { return a > b ? a : b; }   // Fortran max on non-NaN
inline double fmin_(double a, double b) { return a < b ? a : b; }
inline double lim_mc(double x, double y) {              // :73-82
    double ru = y / (x + 1e-30);
    double phi = fmax_(0.0, fmin_(fmin_(2.0 * ru, 0.5 * (1.0 + ru)), 2.0));
    return phi * x;
}
inline double lim_superbee(double x, double y) {        // :85-94
    double ru = y / (x + 1e-30);
    double phi = fmax_(fmax_(0.0, fmin_(2.0 * ru, 1.0)), fmin_(ru, 2.0));
    return phi * x;
}
inline double lim_limo3(double x, double y) {           // :98-110
    double ru = y / (x + 1e-30);
    double a = (2.0 + ru) / 3.0;
    double inner = fmin_(fmin_(2.0 * ru, (2.0 + ru) / 3.0), 1.6);
    double mid = fmax_(fmax_(-0.5 * ru, 0.0), inner);
    double phi = fmax_(0.0, fmin_(a, mid));
    return phi * x;
}
inline double rlimiter(int lim, double x, double y) {
    switch (lim) {
        case Q2D_LIM_MINMOD: return lim_minmod(x, y);
        case Q2D_LIM_VANLEER: return lim_vanleer(x, y);
        case Q2D_LIM_VANALBADA: return lim_vanalbada(x, y);
        case Q2D_LIM_MC: return lim_mc(x, y);
        case Q2D_LIM_SUPERBEE: return lim_superbee(x, y);
        case Q2D_LIM_LIMO3: return lim_limo3(x, y);
        default: return 0.0;                             // rlimiter_IORD :26-33
    }
}

// ---------------------------------------------------------------------------------------
// Riemann solvers. Arguments follow riemann_if (Mod_Riemann.f90:11-20) for nsc = 1:
// (rho_s, u, v, p, a, rho_tot) for L and R, then nx, ny.
// ---------------------------------------------------------------------------------------
struct Flux4 { double r, u, v, e; };

// roe_averages (Lib_Riemann_HLL.f90:229-317); the table lerps at int(Tl), int(Tr) (constant cp:
// h = cp T, cp).
inline void roe_averages(const Gas& g, double dl, double dr, double dltot, double drtot,
                         double ul, double vl, double ur, double vr, double pl, double pr,
                         double& h0l, double& h0r, double& rho_roe, double& u_roe,
                         double& v_roe, double& a_roe, double& h0_roe) {
    const double Rl = g.R, Rr = g.R;                        // f_Rtot
    const double inv_dltot = 1.0 / dltot;
    const double inv_drtot = 1.0 / drtot;
    const double Tl = pl * inv_dltot / Rl;
    const double Tr = pr * inv_drtot / Rr;
    const double srL = std::sqrt(dltot);
    const double srR = std::sqrt(drtot);
    const double inv_sr = 1.0 / (srL + srR);
    rho_roe = srL * srR;
    u_roe = (srR * ur + srL * ul) * inv_sr;
    v_roe = (srR * vr + srL * vl) * inv_sr;
    const double R_roe = (srR * Rr + srL * Rl) * inv_sr;
    const double T_roe = (srR * Tr + srL * Tl) * inv_sr;
    const double invW = g.R;                                // Runiv / Wm_tab
    const double hl = h_of_T(g, Tl);                        // h_tab lerp at Tl
    const double hr = h_of_T(g, Tr);
    const double el = hl - invW * Tl;
    const double er = hr - invW * Tr;
    h0l = 0.0 + hl * dl * inv_dltot;
    h0r = 0.0 + hr * dr * inv_drtot;
    const double d_roe = (srR * dr * inv_drtot + srL * dl * inv_dltot) * inv_sr;
    const double cv_roe = 0.0 + d_roe * (0.5 * (cp_of_T(g, Tl) + cp_of_T(g, Tr)) - invW);
    const double sum_ei = 0.0 + d_roe * (srR * er + srL * el) * inv_sr;
    h0l = h0l + 0.5 * (ul * ul + vl * vl);
    h0r = h0r + 0.5 * (ur * ur + vr * vr);
    h0_roe = (srR * h0r + srL * h0l) * inv_sr;
    const double gam_roe = 1.0 + R_roe / cv_roe;
    const double vel2 = u_roe * u_roe + v_roe * v_roe;
    a_roe = std::sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
}

// riemann_HLLC (Lib_Riemann_HLL.f90:34-123)
inline Flux4 riemann_hllc(const Gas& g, double dl, double ul, double vl, double pl, double al,
                          double dltot, double dr, double ur, double vr, double pr, double ar,
                          double drtot, double nx, double ny) {
    Flux4 F;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, rho_roe, u_roe, v_roe, a_roe, h0_roe;
    roe_averages(g, dl, dr, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, rho_roe, u_roe,
                 v_roe, a_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double e0l = h0l - pl / dltot;
    const double e0r = h0r - pr / drtot;
    const double S1 = fmin_(fmin_(0.0, unl - al), un_roe - a_roe);
    const double S4 = fmax_(fmax_(0.0, unr + ar), un_roe + a_roe);
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

// riemann_HLLE (Lib_Riemann_HLL.f90:126-169)
inline Flux4 riemann_hlle(const Gas& g, double dl, double ul, double vl, double pl, double al,
                          double dltot, double dr, double ur, double vr, double pr, double ar,
                          double drtot, double nx, double ny) {
    Flux4 F;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, rho_roe, u_roe, v_roe, a_roe, h0_roe;
    roe_averages(g, dl, dr, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, rho_roe, u_roe,
                 v_roe, a_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double S1 = fmin_(fmin_(0.0, unl - al), un_roe - a_roe);
    const double S4 = fmax_(fmax_(0.0, unr + ar), un_roe + a_roe);
    const double inv_denom = 1.0 / (S4 - S1);
    const double FrL = dltot * unl;
    const double FrR = drtot * unr;
    F.r = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
    F.u = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) +
           S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
    F.v = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) +
           S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
    F.e = (S4 * (FrL * h0l) - S1 * (FrR * h0r) +
           S1 * S4 * (drtot * (h0r - pr / drtot) - dltot * (h0l - pl / dltot))) * inv_denom;
    return F;
}

// fluxes (Lib_Riemann_LF.f90:101-118)
inline Flux4 physical_flux(const Gas& g, double p, double r, double u, double v, double nx,
                           double ny) {
    Flux4 F;
    F.r = r * (u * nx + v * ny);
    F.u = F.r * u + p * nx;
    F.v = F.r * v + p * ny;
    F.e = F.r * H0(g, p, r, std::sqrt(u * u + v * v));
    return F;
}

// riemann_LLF (Lib_Riemann_LF.f90:11-40)
inline Flux4 riemann_llf(const Gas& g, double dl, double ul, double vl, double pl, double al,
                         double dltot, double dr, double ur, double vr, double pr, double ar,
                         double drtot, double nx, double ny) {
    Flux4 F;
    const double uln = ul * nx + vl * ny;
    const double urn = ur * nx + vr * ny;
    const double A = fmax_(fmax_(fmax_(std::fabs(uln - al), std::fabs(urn - ar)),
                                 std::fabs(uln + al)), std::fabs(urn + ar));
    const Flux4 Fr = physical_flux(g, pr, dr, ur, vr, nx, ny);
    const Flux4 Fl = physical_flux(g, pl, dl, ul, vl, nx, ny);
    F.r = 0.5 * (Fl.r + Fr.r - A * (drtot - dltot));
    F.u = 0.5 * (Fr.u + Fl.u - A * (drtot * ur - dltot * ul));
    F.v = 0.5 * (Fr.v + Fl.v - A * (drtot * vr - dltot * vl));
    F.e = 0.5 * (Fl.e + Fr.e - A * (drtot * E0(g, pr, dr, std::sqrt(ur * ur + vr * vr)) -
                                    dltot * E0(g, pl, dl, std::sqrt(ul * ul + vl * vl))));
    return F;
}

// riemann_SLAU_base + riemann_SLAU / riemann_SLAU2 (Lib_Riemann_SLAU.f90:10-124): mass flux
// from the density-weighted normal speed with the low-Mach pressure term, the pressure flux by
// Mach-split weights (SLAU: (1 - chi) blend; SLAU2: |V| a_F scaling), upwinded momentum and
// total enthalpy.
inline Flux4 riemann_slau(const Gas& g, bool slau2, double dltot, double ul, double vl, double pl, double al,
                          double drtot, double ur, double vr, double pr, double ar, double nx, double ny) {
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double sq_veli = ul * ul + vl * vl;
    const double sq_velj = ur * ur + vr * vr;
    const double aF = 0.5 * (al + ar);
    const double mL = unl / aF;
    const double mR = unr / aF;
    const double Mach_tilde = fmin_(1.0, std::sqrt(0.5 * (sq_veli + sq_velj)) / aF);
    const double Chi = (1.0 - Mach_tilde) * (1.0 - Mach_tilde);
    const double Vn_mag = (dltot * std::fabs(unl) + drtot * std::fabs(unr)) / (dltot + drtot);
    const double f_rho = -fmax_(fmin_(mL, 0.0), -1.0) * fmin_(fmax_(mR, 0.0), 1.0);
    const double Vn_magL = (1.0 - f_rho) * Vn_mag + f_rho * std::fabs(unl);
    const double Vn_magR = (1.0 - f_rho) * Vn_mag + f_rho * std::fabs(unr);
    Flux4 F;
    F.r = 0.5 * (dltot * (unl + Vn_magL) + drtot * (unr - Vn_magR) - (Chi / aF) * (pr - pl));
    double BetaL, BetaR;
    if (std::fabs(mL) < 1.0) BetaL = 0.25 * (2.0 - mL) * ((mL + 1.0) * (mL + 1.0));
    else BetaL = mL >= 0.0 ? 1.0 : 0.0;
    if (std::fabs(mR) < 1.0) BetaR = 0.25 * (2.0 + mR) * ((mR - 1.0) * (mR - 1.0));
    else BetaR = mR >= 0.0 ? 0.0 : 1.0;
    const double p_half = slau2
        ? 0.5 * (pl + pr) + 0.5 * (BetaL - BetaR) * (pl - pr) +
              std::sqrt(0.5 * (sq_veli + sq_velj)) * (BetaL + BetaR - 1.0) * aF * 0.5 * (dltot + drtot)
        : 0.5 * (pl + pr) + 0.5 * (BetaL - BetaR) * (pl - pr) +
              (1.0 - Chi) * (BetaL + BetaR - 1.0) * 0.5 * (pl + pr);
    const double H_L = H0(g, pl, dltot, std::sqrt(sq_veli));
    const double H_R = H0(g, pr, drtot, std::sqrt(sq_velj));
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

// the solvers that run the shock sensor (obj_riemann%SD, Mod_Riemann.f90:70-80)
inline bool riemann_sd(int kind) { return kind == Q2D_RIEMANN_HLLCP || kind == Q2D_RIEMANN_HLLEPP; }

// hartenHyman (Lib_Riemann_HLL.f90:320-331): entropy fix of an acoustic eigenvalue
inline double harten_hyman(double v, double e) {
    const double al = std::fabs(v);
    return al <= e ? (v * v + e * e) / (2.0 * e) : al;
}

// riemann_HLLEpp (Lib_Riemann_HLL.f90:437-533): centred flux minus the wave sum of a Roe
// linearisation whose eigenvalues blend Roe's (Harten-Hyman fix on the acoustic waves, |un| on
// the contact and the shear) and HLLE's by the shock sensor beta.
inline Flux4 riemann_hllepp(const Gas& g, double dl, double ul, double vl, double pl, double al,
                            double dltot, double dr, double ur, double vr, double pr, double ar,
                            double drtot, double beta, double nx, double ny) {
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    double h0l, h0r, rho_roe, u_roe, v_roe, a_roe, h0_roe;
    roe_averages(g, dl, dr, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, rho_roe, u_roe,
                 v_roe, a_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double Sm = fmin_(fmin_(0.0, unl - al), un_roe - a_roe);
    const double Sp = fmax_(fmax_(0.0, unr + ar), un_roe + a_roe);
    const double inv_denom = 1.0 / (Sp - Sm);
    const double lam1_hlle = std::fabs((Sp + Sm) * un_roe * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double lam2_hlle = std::fabs((Sp + Sm) * (un_roe - a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double lam3_hlle = std::fabs((Sp + Sm) * (un_roe + a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
    const double eps = 0.3 * (std::fabs(un_roe) + a_roe);
    const double lam1_roe = std::fabs(un_roe);
    const double lam2_roe = harten_hyman(un_roe - a_roe, eps);
    const double lam3_roe = harten_hyman(un_roe + a_roe, eps);
    const double lam1 = beta * lam1_roe + (1.0 - beta) * lam1_hlle;
    const double lam2 = beta * lam2_roe + (1.0 - beta) * lam2_hlle;
    const double lam3 = beta * lam3_roe + (1.0 - beta) * lam3_hlle;
    const Flux4 FL = physical_flux(g, pl, dl, ul, vl, nx, ny);   // fluxes_helper (:334-352)
    const Flux4 FR = physical_flux(g, pr, dr, ur, vr, nx, ny);
    Flux4 F;
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

// riemann_HLLEM (Lib_Riemann_HLL.f90:355-434): HLL flux plus Einfeldt's antidiffusion on the
// contact and the shear wave when S1 < 0 < S4.
inline Flux4 riemann_hllem(const Gas& g, double dl, double ul, double vl, double pl, double al,
                           double dltot, double dr, double ur, double vr, double pr, double ar,
                           double drtot, double nx, double ny) {
    double h0l, h0r, rho_roe, u_roe, v_roe, a_roe, h0_roe;
    roe_averages(g, dl, dr, dltot, drtot, ul, vl, ur, vr, pl, pr, h0l, h0r, rho_roe, u_roe,
                 v_roe, a_roe, h0_roe);
    const double un_roe = u_roe * nx + v_roe * ny;
    const double S1 = fmin_(fmin_(0.0, (ul * nx + vl * ny) - al), un_roe - a_roe);
    const double S4 = fmax_(fmax_(0.0, (ur * nx + vr * ny) + ar), un_roe + a_roe);
    const Flux4 FL = physical_flux(g, pl, dl, ul, vl, nx, ny);
    const Flux4 FR = physical_flux(g, pr, dr, ur, vr, nx, ny);
    const double e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
    const double inv_denom = 1.0 / (S4 - S1);
    Flux4 F;
    F.r = (S4 * FL.r - S1 * FR.r + S1 * S4 * (drtot - dltot)) * inv_denom;
    F.u = (S4 * FL.u - S1 * FR.u + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
    F.v = (S4 * FL.v - S1 * FR.v + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
    F.e = (S4 * FL.e - S1 * FR.e + S1 * S4 * (drtot * e0r - dltot * e0l)) * inv_denom;
    if (S1 < 0.0 && S4 > 0.0) {
        const double drho = drtot - dltot, dp = pr - pl, du = ur - ul, dv = vr - vl;
        const double tx = -ny, ty = nx;
        const double alpha_c = drho - dp / (a_roe * a_roe);
        const double alpha_s = rho_roe * (du * tx + dv * ty);
        const double delta = a_roe / (a_roe + std::fabs(0.5 * (S1 + S4)));
        const double C = (S1 * S4) * inv_denom;
        F.r = F.r - C * delta * alpha_c;
        F.u = F.u - C * delta * (alpha_c * u_roe + alpha_s * tx);
        F.v = F.v - C * delta * (alpha_c * v_roe + alpha_s * ty);
        F.e = F.e - C * delta * (alpha_c * 0.5 * (u_roe * u_roe + v_roe * v_roe) + alpha_s * (u_roe * tx + v_roe * ty));
    }
    return F;
}

// riemann_HLLCHLLE (Lib_Riemann_HLL.f90:172-226): HLLE along the velocity-jump direction and
// HLLC across it, weighted by their projections on the face normal; HLLC when the jump vanishes.
inline Flux4 riemann_hllc_rotated(const Gas& g, double dl, double ul, double vl, double pl, double al,
                                  double dltot, double dr, double ur, double vr, double pr, double ar,
                                  double drtot, double nx, double ny) {
    const double abs_dv = std::sqrt((ur - ul) * (ur - ul) + (vr - vl) * (vr - vl));
    const double dum = 0.5 * (std::sqrt(ul * ul + vl * vl) + std::sqrt(ur * ur + vr * vr));
    if (abs_dv / (dum + 1.0e-10) > 1.0e-12) {
        double nx1 = (ur - ul) / abs_dv, ny1 = (vr - vl) / abs_dv;
        double alfa1 = nx * nx1 + ny * ny1;
        const double s1 = std::copysign(1.0, alfa1);
        nx1 = s1 * nx1; ny1 = s1 * ny1; alfa1 = s1 * alfa1;
        double nx2 = -ny1, ny2 = nx1;
        double alfa2 = nx * nx2 + ny * ny2;
        const double s2 = std::copysign(1.0, alfa2);
        nx2 = s2 * nx2; ny2 = s2 * ny2; alfa2 = s2 * alfa2;
        const Flux4 E = riemann_hlle(g, dl, ul, vl, pl, al, dltot, dr, ur, vr, pr, ar, drtot, nx1, ny1);
        const Flux4 C = riemann_hllc(g, dl, ul, vl, pl, al, dltot, dr, ur, vr, pr, ar, drtot, nx2, ny2);
        Flux4 F;
        F.r = E.r * alfa1 + C.r * alfa2;
        F.u = E.u * alfa1 + C.u * alfa2;
        F.v = E.v * alfa1 + C.v * alfa2;
        F.e = E.e * alfa1 + C.e * alfa2;
        return F;
    }
    return riemann_hllc(g, dl, ul, vl, pl, al, dltot, dr, ur, vr, pr, ar, drtot, nx, ny);
}

// Riemann_PLLF (Lib_Riemann_LF.f90:44-98): Rusanov flux with the dissipation speed of the
// low-Mach preconditioned system (reference speed clipped to [1e-5 a, a]).
inline Flux4 riemann_pllf(const Gas& g, double dl, double ul, double vl, double pl, double al,
                          double dltot, double dr, double ur, double vr, double pr, double ar,
                          double drtot, double nx, double ny) {
    const double uln = ul * nx + vl * ny;
    const double urn = ur * nx + vr * ny;
    const double U_rl = fmax_(1e-5 * al, fmin_(std::fabs(uln), al));
    const double U_rr = fmax_(1e-5 * ar, fmin_(std::fabs(urn), ar));
    const double betal = 1.0 / (al * al), betar = 1.0 / (ar * ar);
    const double alphal = 0.5 * (1.0 - betal * (U_rl * U_rl));
    const double alphar = 0.5 * (1.0 - betar * (U_rr * U_rr));
    const double ul_mod = std::fabs(uln * (1.0 - alphal));
    const double ur_mod = std::fabs(urn * (1.0 - alphar));
    const double al_mod = std::sqrt((alphal * alphal) * (uln * uln) + U_rl * U_rl);
    const double ar_mod = std::sqrt((alphar * alphar) * (urn * urn) + U_rr * U_rr);
    const double A = fmax_(ul_mod + al_mod, ur_mod + ar_mod);
    const Flux4 Fr = physical_flux(g, pr, dr, ur, vr, nx, ny);
    const Flux4 Fl = physical_flux(g, pl, dl, ul, vl, nx, ny);
    Flux4 F;
    F.r = 0.5 * (Fl.r + Fr.r - A * (drtot - dltot));
    F.u = 0.5 * (Fr.u + Fl.u - A * (drtot * ur - dltot * ul));
    F.v = 0.5 * (Fr.v + Fl.v - A * (drtot * vr - dltot * vl));
    F.e = 0.5 * (Fl.e + Fr.e - A * (drtot * E0(g, pr, dr, std::sqrt(ur * ur + vr * vr)) -
                                    dltot * E0(g, pl, dl, std::sqrt(ul * ul + vl * vl))));
    return F;
}

// riemann_exact (Lib_Riemann_Godunov.f90:14-152) with its wave routines (:177-248): Newton
// iteration on the contact velocity (|1 - p2/p3| < 1e-5, at most 1001 passes) from the
// two-rarefaction guess, then the sampled state at x/t = 0 and its physical flux. Integer
// powers are products; the wave-family flags keep the values of their last evaluation (0
// before any).
inline void ex_rareleft(double ps, double as, double us, double ud, double& pd, double& ad,
                        double& dpr, double& v1, double& v2, double gamma) {
    const double delta = 0.5 * (gamma - 1.0);
    const double dum1 = 2.0 * gamma / (gamma - 1.0);
    ad = as - delta * (ud - us);
    pd = ps * std::pow(ad / as, dum1);
    dpr = -gamma * pd / ad;
    v1 = us - as;
    v2 = ud - ad;
}
inline void ex_rareright(double pd, double ad, double ud, double us, double& ps, double& as,
                         double& dpl, double& v3, double& v4, double gamma) {
    const double delta = 0.5 * (gamma - 1.0);
    const double dum1 = 2.0 * gamma / (gamma - 1.0);
    as = ad + delta * (us - ud);
    ps = pd * std::pow(as / ad, dum1);
    dpl = gamma * ps / as;
    v3 = us + as;
    v4 = ud + ad;
}
inline void ex_shockleft(double us, double as, double ps, double ud, double& ad, double& pd,
                         double& dpr, double& ws, double gamma) {
    const double x1 = (gamma + 1.0) * (ud - us) / (4.0 * as);
    const double M = x1 - std::sqrt(1.0 + x1 * x1);
    const double C1 = gamma * ps / as;
    pd = ps + C1 * (ud - us) * M;
    dpr = 2.0 * C1 * (M * M * M) / (1.0 + M * M);
    const double rpd = pd / ps;
    ws = us + as * M;
    ad = as * std::sqrt((gamma + 1.0 + (gamma - 1.0) * rpd) / (gamma + 1.0 + (gamma - 1.0) / rpd));
}
inline void ex_shockright(double ud, double ad, double pd, double us, double& as, double& ps,
                          double& dpl, double& ws, double gamma) {
    const double x4 = (gamma + 1.0) * (us - ud) / (4.0 * ad);
    const double M = x4 + std::sqrt(1.0 + x4 * x4);
    const double C4 = gamma * pd / ad;
    ps = pd + C4 * (us - ud) * M;
    dpl = 2.0 * C4 * (M * M * M) / (1.0 + M * M);
    const double rps = ps / pd;
    ws = ud + ad * M;
    as = ad * std::sqrt((gamma + 1.0 + (gamma - 1.0) * rps) / (gamma + 1.0 + (gamma - 1.0) / rps));
}
inline Flux4 riemann_exact(const Gas& g, double dl, double ul, double vl, double p1, double a1,
                           double dltot, double dr, double ur, double vr, double p4, double a4,
                           double drtot, double nx, double ny) {
    const double gam1 = g.gamma, gam4 = g.gamma;   // f_gamma
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
    const double z = (gm1_1 / gm1_4) * (a4 / a1) * std::pow(p1 / p4, dum);
    double vel = (z * R2I + R1IV) / (1.0 + z);
    double p3 = 1.0, p2 = 2.0 * p3, a2 = 0.0, a3 = 0.0, dpr = 0.0, dpl = 0.0;
    double sw_l = 0.0, sw_r = 0.0, vw1 = 0.0, vw2 = 0.0, vw3 = 0.0, vw4 = 0.0;
    int iter = 0;
    while (std::fabs(1.0 - (p2 / p3)) >= 1e-5 && iter <= 1000) {
        if (vel < un1) ex_shockleft(un1, a1, p1, vel, a2, p2, dpr, sw_l, gam1);
        else ex_rareleft(p1, a1, un1, vel, p2, a2, dpr, vw1, vw2, gam1);
        if (vel > un4) ex_shockright(un4, a4, p4, vel, a3, p3, dpl, sw_r, gam4);
        else ex_rareright(p4, a4, un4, vel, p3, a3, dpl, vw3, vw4, gam4);
        vel = vel - ((p2 - p3) / (dpr - dpl));
        ++iter;
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
            pf = p1 * std::pow(af / a1, eta1);
        }
        rhof = gam1 * pf / (af * af);
        rhof = dl / dltot * rhof;
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
            pf = p4 * std::pow(af / a4, eta4);
        }
        rhof = gam4 * pf / (af * af);
        rhof = dr / drtot * rhof;
        uf = vel * nx + ut4;
        vf = vel * ny + vt4;
    }
    return physical_flux(g, pf, rhof, uf, vf, nx, ny);   // fluxes (:155-174)
}

// riemann_Hanel (Lib_Riemann_AUSM.f90:18-70): van Leer splitting of the normal velocity and
// the pressure, total enthalpy convected.
inline Flux4 riemann_hanel(const Gas& g, double dl, double ul, double vl, double pl, double al,
                           double dltot, double dr, double ur, double vr, double pr, double ar,
                           double drtot, double nx, double ny) {
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dl, std::sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, dr, std::sqrt(ur * ur + vr * vr));
    const double uLp = std::fabs(unl) <= al ? (unl + al) * (unl + al) / (4.0 * al) : 0.5 * (unl + std::fabs(unl));
    const double uRm = std::fabs(unr) <= ar ? (-((unr - ar) * (unr - ar))) / (4.0 * ar) : 0.5 * (unr - std::fabs(unr));
    const double pLp = std::fabs(unl) <= al ? pl * uLp * (2.0 - unl / al) / al : pl * uLp / unl;
    const double pRm = std::fabs(unr) <= ar ? pr * uRm * (-2.0 - unr / ar) / ar : pr * uRm / unr;
    const double phalf = pLp + pRm;
    Flux4 F;
    F.r = uLp * dltot + uRm * drtot;
    F.u = uLp * (dltot * ul) + uRm * (drtot * ur) + phalf * nx;
    F.v = uLp * (dltot * vl) + uRm * (drtot * vr) + phalf * ny;
    F.e = uLp * (dltot * H_L) + uRm * (drtot * H_R);
    return F;
}

// riemann_AUSMp (Lib_Riemann_AUSM.f90:73-128): AUSM+ with the geometric-mean interface sound
// speed, quartic Mach and quintic pressure polynomials (beta 1/8, alpha 3/16).
inline Flux4 riemann_ausmp(const Gas& g, double dl, double ul, double vl, double pl, double al,
                           double dltot, double dr, double ur, double vr, double pr, double ar,
                           double drtot, double nx, double ny) {
    const double betap = 0.125, alpha = 0.1875;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dl, std::sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, dr, std::sqrt(ur * ur + vr * vr));
    const double a_half = std::sqrt(al * ar);
    const double ML = unl / a_half, MR = unr / a_half;
    double MplusL, pplusL, MminusR, pminusR;
    if (std::fabs(ML) < 1.0) {
        const double q = (ML + 1.0) * (ML + 1.0), w = (ML * ML - 1.0) * (ML * ML - 1.0);
        MplusL = 0.25 * q + betap * w;
        pplusL = 0.25 * q * (2.0 - ML) + alpha * ML * w;
    } else {
        MplusL = 0.5 * (ML + std::fabs(ML));
        pplusL = 0.5 * (1.0 + std::copysign(1.0, ML));
    }
    if (std::fabs(MR) < 1.0) {
        const double q = (MR - 1.0) * (MR - 1.0), w = (MR * MR - 1.0) * (MR * MR - 1.0);
        MminusR = -0.25 * q - betap * w;
        pminusR = 0.25 * q * (2.0 + MR) - alpha * MR * w;
    } else {
        MminusR = 0.5 * (MR - std::fabs(MR));
        pminusR = 0.5 * (1.0 - std::copysign(1.0, MR));
    }
    const double Mhalf = MplusL + MminusR;
    const double phalf = pplusL * pl + pminusR * pr;
    const double mdotp = dltot * a_half * 0.5 * (Mhalf + std::fabs(Mhalf));
    const double mdotm = drtot * a_half * 0.5 * (Mhalf - std::fabs(Mhalf));
    Flux4 F;
    F.r = mdotp + mdotm;
    F.u = mdotp * ul + mdotm * ur + nx * phalf;
    F.v = mdotp * vl + mdotm * vr + ny * phalf;
    F.e = mdotp * H_L + mdotm * H_R;
    return F;
}

// riemann_AUSMp_up / riemann_AUSMp_up2 (Lib_Riemann_AUSM.f90:131-321): AUSM+-up with the
// critical-speed interface sound speed, the reference Mach number from max(M_F^2, Minf^2),
// pressure diffusion in the mass flux (Kp 1/4, sigma 1) and, for AUSM+-up, velocity diffusion
// in the pressure flux (Ku 3/4); AUSM+-up2 takes its pressure flux in Kitamura-Shima form.
inline Flux4 riemann_ausmp_up(const Gas& g, bool up2, double minf, double dl, double ul, double vl,
                              double pl, double dltot, double dr, double ur, double vr, double pr,
                              double drtot, double nx, double ny) {
    const double Kp = 0.25, Ku = 0.75, sigma = 1.0, betap = 0.125;
    const double unl = ul * nx + vl * ny;
    const double unr = ur * nx + vr * ny;
    const double H_L = H0(g, pl, dl, std::sqrt(ul * ul + vl * vl));
    const double H_R = H0(g, pr, dr, std::sqrt(ur * ur + vr * vr));
    const double gamma_L = g.gamma, gamma_R = g.gamma;   // f_gamma
    const double astarL2 = 2.0 * (gamma_L - 1.0) / (gamma_L + 1.0) * H_L;
    const double astarR2 = 2.0 * (gamma_R - 1.0) / (gamma_R + 1.0) * H_R;
    const double astarL = std::sqrt(astarL2), astarR = std::sqrt(astarR2);
    const double atildeL = astarL2 / fmax_(astarL, unl);
    const double atildeR = astarR2 / fmax_(astarR, -unr);
    const double aF = fmin_(atildeL, atildeR);
    const double mL = unl / aF, mR = unr / aF;
    const double MFsq = 0.5 * (mL * mL + mR * mR);
    const double Mrefsq = fmin_(1.0, fmax_(MFsq, minf * minf));
    const double fa = 2.0 * std::sqrt(Mrefsq) - Mrefsq;
    const double alpha = 0.1875 * (-4.0 + 5.0 * fa * fa);
    double mLP, bLP, mRM, bRM;
    if (std::fabs(mL) <= 1.0) {
        const double p1 = 0.25 * ((mL + 1.0) * (mL + 1.0)), p2 = (mL * mL - 1.0) * (mL * mL - 1.0);
        mLP = p1 + betap * p2;
        bLP = p1 * (2.0 - mL) + alpha * mL * p2;
    } else {
        mLP = 0.5 * (mL + std::fabs(mL));
        bLP = mLP / mL;
    }
    if (std::fabs(mR) <= 1.0) {
        const double p1 = 0.25 * ((mR - 1.0) * (mR - 1.0)), p2 = (mR * mR - 1.0) * (mR * mR - 1.0);
        mRM = -p1 - betap * p2;
        bRM = p1 * (2.0 + mR) - alpha * mR * p2;
    } else {
        mRM = 0.5 * (mR - std::fabs(mR));
        bRM = mRM / mR;
    }
    const double rhoF = 0.5 * (dltot + drtot);
    const double Mp = -(Kp / fa) * fmax_(0.0, 1.0 - sigma * MFsq) * (pr - pl) / (rhoF * aF * aF);
    const double mF = mLP + mRM + Mp;
    const double mdot = aF * (fmax_(mF, 0.0) * dltot + fmin_(mF, 0.0) * drtot);
    double phalf;
    if (up2) {
        const double sq_vel = 0.5 * ((ul * ul + vl * vl) + (ur * ur + vr * vr));
        phalf = 0.5 * (pr + pl) + 0.5 * (bLP - bRM) * (pl - pr) + std::sqrt(sq_vel) * (bLP + bRM - 1.0) * rhoF * aF;
    } else {
        const double Pu = -Ku * fa * bLP * bRM * 2.0 * rhoF * aF * (unr - unl);
        phalf = bLP * pl + bRM * pr + Pu;
    }
    const bool upw = mF >= 0.0;
    Flux4 F;
    F.r = mdot;
    F.u = mdot * (upw ? ul : ur) + nx * phalf;
    F.v = mdot * (upw ? vl : vr) + ny * phalf;
    F.e = mdot * (upw ? H_L : H_R);
    return F;
}

// beta: the shock sensor of the face's cell for the sensor-driven solvers (HLLC+, HLLE++;
// Convective_Flux passes it, Lib_Convective.f90:62-64), 1 from the wall and inflow boundaries.
inline Flux4 riemann(int kind, const Gas& g, const double* L, double aL, const double* R,
                     double aR, double nx, double ny, double beta = 1.0) {
    switch (kind) {
        case Q2D_RIEMANN_HLLCP: {   // riemann_HLLCSD (Lib_Riemann_HLL.f90:572-605)
            if (beta == 0.0)
                return riemann_hlle(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
            if (beta >= 1.0)
                return riemann_hllc(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
            const Flux4 E = riemann_hlle(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
            const Flux4 C = riemann_hllc(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
            Flux4 F;
            F.r = beta * C.r + (1.0 - beta) * E.r;
            F.u = beta * C.u + (1.0 - beta) * E.u;
            F.v = beta * C.v + (1.0 - beta) * E.v;
            F.e = beta * C.e + (1.0 - beta) * E.e;
            return F;
        }
        case Q2D_RIEMANN_HLLEPP:
            return riemann_hllepp(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], beta, nx, ny);
        case Q2D_RIEMANN_HLLEM:
            return riemann_hllem(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_HLLC_ROTATED:
            return riemann_hllc_rotated(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_PLLF:
            return riemann_pllf(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_EXACT:
            return riemann_exact(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_HANEL:
            return riemann_hanel(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_AUSMP:
            return riemann_ausmp(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR, R[0], nx, ny);
        case Q2D_RIEMANN_AUSMP_UP:
        case Q2D_RIEMANN_AUSMP_UP2:
            return riemann_ausmp_up(g, kind == Q2D_RIEMANN_AUSMP_UP2, g.minf, L[0], L[1], L[2], L[3], L[0], R[0], R[1],
                                    R[2], R[3], R[0], nx, ny);
        case Q2D_RIEMANN_SLAU:
        case Q2D_RIEMANN_SLAU2:
            return riemann_slau(g, kind == Q2D_RIEMANN_SLAU2, L[0], L[1], L[2], L[3], aL, R[0], R[1], R[2],
                                R[3], aR, nx, ny);
        case Q2D_RIEMANN_HLLE:
            return riemann_hlle(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR,
                                R[0], nx, ny);
        case Q2D_RIEMANN_LLF:
            return riemann_llf(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR,
                               R[0], nx, ny);
        default:
            return riemann_hllc(g, L[0], L[1], L[2], L[3], aL, L[0], R[0], R[1], R[2], R[3], aR,
                                R[0], nx, ny);
    }
}

// ---------------------------------------------------------------------------------------
// Data structures (Advanced_Types_m.f90:17-89)
// ---------------------------------------------------------------------------------------
struct Block {
    int ni = 0, nj = 0, case_id = 0, local_b = 0;
    std::vector<double> node;     // (0:ni,0:nj) x,y
    std::vector<double> area;     // (0:ni,0:nj) or empty
    std::vector<double> P, PO, R; // (4, -1:ni+2, -1:nj+2)
    std::vector<double> M;        // (4) per ghost-frame cell: M11 M12 M21 M22
    std::vector<double> dl;       // (2) per ghost-frame cell
    std::vector<double> sur;      // per ghost-frame cell
    std::vector<double> f1;       // i-faces (0:ni,1:nj): nx ny len
    std::vector<double> f2;       // j-faces (1:ni,0:nj): nx ny len
    std::vector<double> dtlocal;  // (1:ni,1:nj)
    std::vector<double> inv_r, Gx, Gy;   // (1:ni,1:nj)
    std::vector<double> beta;     // (1:ni,1:nj) shock sensor of the stage (MUSCL-SD only)

    int c(int i, int j) const { return (i + 1) + (ni + 4) * (j + 1); }
    double nx_(int i, int j) const { return node[2 * (i + (ni + 1) * j)]; }
    double ny_(int i, int j) const { return node[2 * (i + (ni + 1) * j) + 1]; }
    double* p(int i, int j) { return &P[4 * c(i, j)]; }
    const double* pc(int i, int j) const { return &P[4 * c(i, j)]; }
    double* r(int i, int j) { return &R[4 * c(i, j)]; }
    const double* face1(int i, int j) const { return &f1[3 * (i + (ni + 1) * (j - 1))]; }
    const double* face2(int i, int j) const { return &f2[3 * ((i - 1) + ni * j)]; }
    const double* face(int dir, int i, int j) const { return dir == 1 ? face1(i, j) : face2(i, j); }
    double dlc(int i, int j, int d) const { return dl[2 * c(i, j) + (d - 1)]; }
    double sd(int i, int j) const { return beta[(i - 1) + ni * (j - 1)]; }
};

struct Case {
    std::vector<int> blocks;      // global ids, local order
    std::vector<q2d_bc_rec> bc;
    double time = 0.0, dtglobal = 0.0, time_from_call = 0.0;
    long long iter = 0, iter_from_call = 0;
    double res[4] = {0, 0, 0, 0};
    double res0 = -1.0;
    int todo = Q2D_TODO_CONTINUE;
    int err = Q2D_OK, err_b = 0, err_i = 0, err_j = 0, err_stage = 0;
    bool done = false;
    long long iter_end = 0;       // the case's own fixed end, 0 for none
};

}  // namespace

struct q2d_oracle {
    q2d_options opt;
    Gas gas;
    std::vector<double> htab, cptab;   // thermally perfect table (empty: constant cp)
    std::vector<Block> blk;
    std::vector<Case> cases;
    bool committed = false;
};

namespace {

// ---------------------------------------------------------------------------------------
// Metrics (Lib_Metrics.f90)
// ---------------------------------------------------------------------------------------
struct V2 { double x, y; };

// Compute_Metric_Tensor (Lib_Metrics.f90:125-189)
int metric_tensor(V2 N1, V2 N2, V2 N3, V2 N4, double* M, double* dl, double* sur) {
    double A[2][2];
    A[0][0] = N4.x - N2.x + N3.x - N1.x;
    A[0][1] = N4.y - N2.y + N3.y - N1.y;
    A[1][0] = N4.x - N3.x + N2.x - N1.x;
    A[1][1] = N4.y - N3.y + N2.y - N1.y;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) A[a][b] = 0.5 * A[a][b];
    const double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    if (std::fabs(det) == 0.0) return Q2D_ERR_BADARG;
    M[0] = A[1][1] / det;     // cofactor(1,1)/det
    M[1] = -A[1][0] / det;    // cofactor(1,2)/det
    M[2] = -A[0][1] / det;    // cofactor(2,1)/det
    M[3] = A[0][0] / det;     // cofactor(2,2)/det
    for (int h = 0; h < 2; ++h) dl[h] = std::sqrt(A[h][0] * A[h][0] + A[h][1] * A[h][1]);
    // tsurface(vx,vy,1,2,3,4): d1 = N4-N1, d2 = N3-N2
    const double d1x = N4.x - N1.x, d1y = N4.y - N1.y;
    const double d2x = N3.x - N2.x, d2y = N3.y - N2.y;
    const double cross = d1x * d2y - d1y * d2x;
    *sur = 0.5 * std::fabs(cross);
    if (*sur <= 0.0) return Q2D_ERR_BADARG;
    return Q2D_OK;
}

int metric_into(Block& B, int i, int j, V2 N1, V2 N2, V2 N3, V2 N4) {
    const int k = B.c(i, j);
    return metric_tensor(N1, N2, N3, N4, &B.M[4 * k], &B.dl[2 * k], &B.sur[k]);
}

V2 nodev(const Block& B, int i, int j) { return V2{B.nx_(i, j), B.ny_(i, j)}; }
V2 quad_ex(V2 a, V2 b, V2 c) {   // 3a - 3b + c
    return V2{3.0 * a.x - 3.0 * b.x + c.x, 3.0 * a.y - 3.0 * b.y + c.y};
}
V2 lin_ex(V2 a, V2 b) { return V2{2.0 * a.x - b.x, 2.0 * a.y - b.y}; }

// Compute_Norm_Area (Lib_Metrics.f90:41-122)
void norm_area(Block& B) {
    const int im = B.ni, jm = B.nj;
    auto sgn = [](double a) { return std::copysign(1.0, a); };
    double d1x = B.nx_(1, 1) - B.nx_(1, 0), d1y = B.ny_(1, 1) - B.ny_(1, 0);
    double snixx = d1y, sniyy = -d1x;
    double ax = 0.5 * (B.nx_(1, 1) + B.nx_(1, 0)), ay = 0.5 * (B.ny_(1, 1) + B.ny_(1, 0));
    double bx = 0.5 * (B.nx_(0, 1) + B.nx_(0, 0)), by = 0.5 * (B.ny_(0, 1) + B.ny_(0, 0));
    double scal = (ax - bx) * snixx + (ay - by) * sniyy;
    const double signi = sgn(scal);
    d1x = B.nx_(0, 1) - B.nx_(1, 1);
    d1y = B.ny_(0, 1) - B.ny_(1, 1);
    double snjxx = d1y, snjyy = -d1x;
    ax = 0.5 * (B.nx_(1, 1) + B.nx_(0, 1));
    ay = 0.5 * (B.ny_(1, 1) + B.ny_(0, 1));
    bx = 0.5 * (B.nx_(1, 0) + B.nx_(0, 0));
    by = 0.5 * (B.ny_(1, 0) + B.ny_(0, 0));
    scal = (ax - bx) * snjxx + (ay - by) * snjyy;
    const double signj = sgn(scal);
    B.f1.assign(3 * (im + 1) * jm, 0.0);
    B.f2.assign(3 * im * (jm + 1), 0.0);
    for (int j = 1; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
            const double dx = B.nx_(i, j) - B.nx_(i, j - 1), dy = B.ny_(i, j) - B.ny_(i, j - 1);
            const double d3x = dy, d3y = -dx;
            const double Ai = std::sqrt(d3x * d3x + d3y * d3y);
            double* f = &B.f1[3 * (i + (im + 1) * (j - 1))];
            f[0] = Ai == 0.0 ? 0.0 : d3x / Ai * signi;
            f[1] = Ai == 0.0 ? 0.0 : d3y / Ai * signi;
            f[2] = Ai;
        }
    for (int j = 0; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
            const double dx = B.nx_(i - 1, j) - B.nx_(i, j), dy = B.ny_(i - 1, j) - B.ny_(i, j);
            const double d3x = dy, d3y = -dx;
            const double Aj = std::sqrt(d3x * d3x + d3y * d3y);
            double* f = &B.f2[3 * ((i - 1) + im * j)];
            f[0] = Aj == 0.0 ? 0.0 : d3x / Aj * signj;
            f[1] = Aj == 0.0 ? 0.0 : d3y / Aj * signj;
            f[2] = Aj;
        }
}

// BC_Extrapolate_Metrics (Lib_Metrics.f90:285-395)
int extrapolate_metrics(Block& B, int Im, int Jm, int Fm) {
    V2 N1[2 * GC + 1], N2[2 * GC + 1], N3[2 * GC + 1], N4[2 * GC + 1];
    auto at = [](V2* a, int g) -> V2& { return a[g + GC]; };
    int e = Q2D_OK;
    switch (Fm) {
        case 1:
            for (int g = 0; g <= GC; ++g) {
                at(N1, g) = nodev(B, Im + g - 1, Jm - 1);
                at(N2, g) = nodev(B, Im + g - 1, Jm);
            }
            for (int g = -1; g >= -GC; --g) {
                at(N1, g) = quad_ex(at(N1, g + 1), at(N1, g + 2), at(N1, g + 3));
                at(N2, g) = quad_ex(at(N2, g + 1), at(N2, g + 2), at(N2, g + 3));
                e |= metric_into(B, Im + g, Jm, at(N1, g), at(N2, g), at(N1, g + 1), at(N2, g + 1));
            }
            break;
        case 2:
            for (int g = 0; g >= -GC; --g) {
                at(N3, g) = nodev(B, Im + g, Jm - 1);
                at(N4, g) = nodev(B, Im + g, Jm);
            }
            for (int g = 1; g <= GC; ++g) {
                at(N3, g) = quad_ex(at(N3, g - 1), at(N3, g - 2), at(N3, g - 3));
                at(N4, g) = quad_ex(at(N4, g - 1), at(N4, g - 2), at(N4, g - 3));
                e |= metric_into(B, Im + g, Jm, at(N3, g - 1), at(N4, g - 1), at(N3, g), at(N4, g));
            }
            break;
        case 3:
            if (B.nj > 2) {
                for (int g = 0; g <= GC; ++g) {
                    at(N1, g) = nodev(B, Im - 1, Jm + g - 1);
                    at(N3, g) = nodev(B, Im, Jm + g - 1);
                }
                for (int g = -1; g >= -GC; --g) {
                    at(N1, g) = quad_ex(at(N1, g + 1), at(N1, g + 2), at(N1, g + 3));
                    at(N3, g) = quad_ex(at(N3, g + 1), at(N3, g + 2), at(N3, g + 3));
                    e |= metric_into(B, Im, Jm + g, at(N1, g), at(N1, g + 1), at(N3, g), at(N3, g + 1));
                }
            } else {
                for (int g = 0; g <= 1; ++g) {
                    at(N1, g) = nodev(B, Im - 1, Jm + g - 1);
                    at(N3, g) = nodev(B, Im, Jm + g - 1);
                }
                for (int g = -1; g >= -GC; --g) {
                    at(N1, g) = lin_ex(at(N1, g + 1), at(N1, g + 2));
                    at(N3, g) = lin_ex(at(N3, g + 1), at(N3, g + 2));
                    e |= metric_into(B, Im, Jm + g, at(N1, g), at(N1, g + 1), at(N3, g), at(N3, g + 1));
                }
            }
            break;
        case 4:
            if (B.nj > 2) {
                for (int g = 0; g >= -GC; --g) {
                    at(N2, g) = nodev(B, Im - 1, Jm + g);
                    at(N4, g) = nodev(B, Im, Jm + g);
                }
                for (int g = 1; g <= GC; ++g) {
                    at(N2, g) = quad_ex(at(N2, g - 1), at(N2, g - 2), at(N2, g - 3));
                    at(N4, g) = quad_ex(at(N4, g - 1), at(N4, g - 2), at(N4, g - 3));
                    e |= metric_into(B, Im, Jm + g, at(N2, g - 1), at(N2, g), at(N4, g - 1), at(N4, g));
                }
            } else {
                for (int g = 0; g >= -1; --g) {
                    at(N2, g) = nodev(B, Im - 1, Jm + g);
                    at(N4, g) = nodev(B, Im, Jm + g);
                }
                for (int g = 1; g <= GC; ++g) {
                    at(N2, g) = lin_ex(at(N2, g - 1), at(N2, g - 2));
                    at(N4, g) = lin_ex(at(N4, g - 1), at(N4, g - 2));
                    e |= metric_into(B, Im, Jm + g, at(N2, g - 1), at(N2, g), at(N4, g - 1), at(N4, g));
                }
            }
            break;
    }
    return e;
}

// BC_Symmetry_Metrics (Lib_Metrics.f90:398-441)
void symmetry_metrics(Block& B, int Im, int Jm, int Fm) {
    for (int g = 1; g <= GC; ++g) {
        int di = 0, dj = 0, si = 0, sj = 0;
        switch (Fm) {
            case 1: di = Im - g; dj = Jm; si = Im + g - 1; sj = Jm; break;
            case 2: di = Im + g; dj = Jm; si = Im - g + 1; sj = Jm; break;
            case 3: di = Im; dj = Jm - g; si = Im; sj = Jm + g - 1; break;
            case 4: di = Im; dj = Jm + g; si = Im; sj = Jm - g + 1; break;
        }
        const int kd = B.c(di, dj), ks = B.c(si, sj);
        for (int q = 0; q < 4; ++q) B.M[4 * kd + q] = B.M[4 * ks + q];
        for (int q = 0; q < 2; ++q) B.dl[2 * kd + q] = B.dl[2 * ks + q];
        B.sur[kd] = B.sur[ks];
    }
}

// BC_Connect_Metrics (Lib_Metrics.f90:444-553); with periodic, BC_Connect_Metrics_Periodic
// (:556-700): every donor node read is moved by the rigid translation T that maps the donor's
// seam nodes of step g = 0 onto this block's seam nodes (T from both seam nodes must agree).
int connect_metrics(Block& Bm, int Im, int Jm, int Fm, const Block& Bs, int Is, int Js, int Fs,
                    int d11s, int d21s, bool periodic = false) {
    static const int guides[5][2] = {{0, 0}, {0, 0}, {-1, 0}, {0, 0}, {0, -1}};
    static const int guides2[5][2] = {{0, 0}, {1, 0}, {-2, 0}, {0, 1}, {0, -2}};
    V2 N1[GC + 1], N2[GC + 1], N3[GC + 1], N4[GC + 1];
    switch (Fm) {
        case 1: N1[0] = nodev(Bm, Im - 1, Jm - 1); N2[0] = nodev(Bm, Im - 1, Jm); break;
        case 2: N3[0] = nodev(Bm, Im, Jm - 1); N4[0] = nodev(Bm, Im, Jm); break;
        case 3: N1[0] = nodev(Bm, Im - 1, Jm - 1); N3[0] = nodev(Bm, Im, Jm - 1); break;
        case 4: N2[0] = nodev(Bm, Im - 1, Jm); N4[0] = nodev(Bm, Im, Jm); break;
    }
    int e = Q2D_OK;
    V2 T{0.0, 0.0};
    if (periodic) {
        const int Is1 = Is + GC * guides[Fs][0] - guides2[Fs][0];
        const int Js1 = Js + GC * guides[Fs][1] - guides2[Fs][1];
        int II0, JJ0, III0, JJJ0;
        if (Fs <= 2) { II0 = Is1; JJ0 = (2 * Js1 + d11s + d21s) / 2; III0 = II0; JJJ0 = JJ0 - d11s; }
        else { II0 = (2 * Is1 + d11s + d21s) / 2; JJ0 = Js1; III0 = II0 - d11s; JJJ0 = JJ0; }
        if (II0 < 0 || II0 > Bs.ni || JJ0 < 0 || JJ0 > Bs.nj || III0 < 0 || III0 > Bs.ni || JJJ0 < 0 ||
            JJJ0 > Bs.nj)
            return Q2D_ERR_BADARG;
        const V2 a0 = nodev(Bs, II0, JJ0), b0 = nodev(Bs, III0, JJJ0);
        V2 T2;
        switch (Fm) {
            case 1: T = {N2[0].x - a0.x, N2[0].y - a0.y}; T2 = {N1[0].x - b0.x, N1[0].y - b0.y}; break;
            case 2: T = {N4[0].x - a0.x, N4[0].y - a0.y}; T2 = {N3[0].x - b0.x, N3[0].y - b0.y}; break;
            case 3: T = {N3[0].x - a0.x, N3[0].y - a0.y}; T2 = {N1[0].x - b0.x, N1[0].y - b0.y}; break;
            default: T = {N4[0].x - a0.x, N4[0].y - a0.y}; T2 = {N2[0].x - b0.x, N2[0].y - b0.y}; break;
        }
        const double big = 1.0 + std::max(std::fabs(T.x), std::fabs(T.y));
        if (std::max(std::fabs(T.x - T2.x), std::fabs(T.y - T2.y)) > 1e-10 * big) return Q2D_ERR_BADARG;
    }
    for (int g = 1; g <= GC; ++g) {
        const int Is1 = Is + (GC - g) * guides[Fs][0] + (g - 1) * guides2[Fs][0];
        const int Js1 = Js + (GC - g) * guides[Fs][1] + (g - 1) * guides2[Fs][1];
        int II, JJ, III, JJJ;
        if (Fs <= 2) { II = Is1; JJ = (2 * Js1 + d11s + d21s) / 2; }
        else { II = (2 * Is1 + d11s + d21s) / 2; JJ = Js1; }
        if (II < 0 || II > Bs.ni || JJ < 0 || JJ > Bs.nj) return Q2D_ERR_BADARG;
        V2 a = nodev(Bs, II, JJ);
        a = {a.x + T.x, a.y + T.y};
        switch (Fm) { case 1: N2[g] = a; break; case 2: N4[g] = a; break;
                      case 3: N3[g] = a; break; case 4: N4[g] = a; break; }
        if (Fs <= 2) { III = II; JJJ = JJ - d11s; } else { III = II - d11s; JJJ = JJ; }
        if (III < 0 || III > Bs.ni || JJJ < 0 || JJJ > Bs.nj) return Q2D_ERR_BADARG;
        V2 b = nodev(Bs, III, JJJ);
        b = {b.x + T.x, b.y + T.y};
        switch (Fm) { case 1: N1[g] = b; break; case 2: N3[g] = b; break;
                      case 3: N1[g] = b; break; case 4: N2[g] = b; break; }
        switch (Fm) {
            case 1: e |= metric_into(Bm, Im - g, Jm, N1[g], N2[g], N1[g - 1], N2[g - 1]); break;
            case 2: e |= metric_into(Bm, Im + g, Jm, N3[g - 1], N4[g - 1], N3[g], N4[g]); break;
            case 3: e |= metric_into(Bm, Im, Jm - g, N1[g], N1[g - 1], N3[g], N3[g - 1]); break;
            case 4: e |= metric_into(Bm, Im, Jm + g, N2[g - 1], N2[g], N4[g - 1], N4[g]); break;
        }
    }
    return e;
}

// ---------------------------------------------------------------------------------------
// Ghost cells (Lib_Ghost.f90:16-299)
// ---------------------------------------------------------------------------------------
void ghost_fill(q2d_oracle* o, Case& cs) {
    for (const q2d_bc_rec& rec : cs.bc) {
        Block& B = o->blk[cs.blocks[rec.b - 1]];
        const int Im = rec.i, Jm = rec.j, Fm = rec.f;
        switch (rec.type) {
            case 101: case 201: {   // Ghost_Connection :143-160 (201: Lib_Ghost.f90:63)
                const Block& S = o->blk[cs.blocks[rec.bs - 1]];
                for (int g = 1; g <= GC; ++g) {
                    const int Ig = Im - GUIDE[Fm][0] * g, Jg = Jm - GUIDE[Fm][1] * g;
                    const double* src = S.pc(rec.is + GUIDE[rec.fs][0] * (g - 1),
                                             rec.js + GUIDE[rec.fs][1] * (g - 1));
                    std::memcpy(B.p(Ig, Jg), src, sizeof(double) * NPRIM);
                }
                break;
            }
            case 300: {   // Ghost_Symmetry :163-196
                const int Ig = Im - GUIDE[Fm][0], Jg = Jm - GUIDE[Fm][1];
                const double* n;
                if (Fm <= 2) n = B.face1(Im - (Fm % 2), Jm);
                else n = B.face2(Im, Jm - (Fm % 2));
                const double* Pm = B.pc(Im, Jm);
                double vx = Pm[1], vy = Pm[2];
                const double udotn = vx * n[0] + vy * n[1];
                vx = vx - 2.0 * udotn * n[0];
                vy = vy - 2.0 * udotn * n[1];
                double* Pg = B.p(Ig, Jg);
                Pg[1] = vx;
                Pg[2] = vy;
                Pg[0] = Pm[0];
                Pg[3] = Pm[3];
                break;
            }
            case 0: case 401: case 405: case 406: {   // Ghost_ZG_Extrapolate :199-219
                for (int g = 1; g <= GC; ++g) {
                    const int Ig = Im - GUIDE[Fm][0] * g, Jg = Jm - GUIDE[Fm][1] * g;
                    std::memcpy(B.p(Ig, Jg), B.pc(Im, Jm), sizeof(double) * NPRIM);
                }
                break;
            }
            default: {    // Ghost_Extrapolate :270-299 (400 and every other code)
                const int si = -GUIDE[Fm][0], sj = -GUIDE[Fm][1];   // outward step
                for (int g = 1; g <= GC; ++g) {
                    double* dst = B.p(Im + si * g, Jm + sj * g);
                    const double* a = B.pc(Im + si * (g - 1), Jm + sj * (g - 1));
                    const double* b = B.pc(Im + si * (g - 2), Jm + sj * (g - 2));
                    const double* c = B.pc(Im + si * (g - 3), Jm + sj * (g - 3));
                    for (int v = 0; v < NPRIM; ++v) dst[v] = 3.0 * a[v] - 3.0 * b[v] + c[v];
                }
                break;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Face fluxes
// ---------------------------------------------------------------------------------------
struct FaceErr { bool bad = false; };

// Reconstruction (Lib_Reconstruction.f90:10-29), elemental over the 4 primitives.
inline void reconstruct(int lim, const double* prev, const double* loc, const double* next,
                        const double* next2, double dl0, double dl1, double dl2, double dll,
                        double dlr, double beta, double* pl, double* pr) {
    for (int v = 0; v < NPRIM; ++v) {
        const double s0 = (loc[v] - prev[v]) / dl0;
        const double s1 = (next[v] - loc[v]) / dl1;
        const double s2 = (next2[v] - next[v]) / dl2;
        const double sl = rlimiter(lim, s1, s0);
        const double sr = rlimiter(lim, s2, s1);
        pl[v] = loc[v] + beta * sl * dll;
        pr[v] = next[v] - beta * sr * dlr;
    }
}

// Flux from two reconstructed states: Lib_Convective.f90:56-80 (also used by the connection
// BC, Lib_BC_Fluxes_Connection.f90:97-130, which has the same body).
inline bool face_flux_from_states(const q2d_oracle* o, const double* P1, const double* P4,
                                  double nx, double ny, double int_l, double beta, double* flux) {
    if (gas_state_bad(P1[0], P1[3]) || gas_state_bad(P4[0], P4[3])) return false;
    const Gas& g = o->gas;
    const double rotot1 = P1[0], rotot4 = P4[0];
    const double a1 = f_ss(g, P1[3], rotot1);
    const double a4 = f_ss(g, P4[3], rotot4);
    const Flux4 F = riemann(o->opt.riemann, g, P1, a1, P4, a4, nx, ny, beta);
    const double su = std::copysign(0.5, F.r);
    const double sp = 0.5 + su, sm = su - 0.5;
    flux[0] = F.r * int_l * (sp * (P1[0] / rotot1) - sm * (P4[0] / rotot4));
    flux[1] = F.u * int_l;
    flux[2] = F.v * int_l;
    flux[3] = F.e * int_l;
    return true;
}

// Convective_Flux (Lib_Convective.f90:15-82): dl[-1..2], Prim[-1..2] along the direction; beta_l
// scales both limited slopes (the SD_limiter branch, :40-47; 1 without MUSCL-SD), beta_r goes to
// the Riemann solver (the cell's sensor whenever the sensor runs, :62-64).
inline bool convective_flux(const q2d_oracle* o, const double* dlm1, const double* const* pr,
                            double nx, double ny, double int_l, double beta_l, double beta_r,
                            double* flux) {
    const double l0 = 0.5 * (dlm1[0] + dlm1[1]);
    const double l1 = 0.5 * (dlm1[1] + dlm1[2]);
    const double l2 = 0.5 * (dlm1[2] + dlm1[3]);
    const double lm = 0.5 * dlm1[1];
    const double lp = 0.5 * dlm1[2];
    double P1[4], P4[4];
    reconstruct(o->opt.limiter, pr[0], pr[1], pr[2], pr[3], l0, l1, l2, lm, lp, beta_l, P1, P4);
    return face_flux_from_states(o, P1, P4, nx, ny, int_l, beta_r, flux);
}

// SD_Tramel (Lib_Shock_Detector.f90:14-38): Jameson-type pressure sensor on the cross stencil
// p(i+-1, j), p(i, j+-1); 0 in shock cells, 1 - tanh(10 phi^3) (within 1.6e-7 of 1) elsewhere.
inline double sd_tramel(double p, double p1, double p2, double p3, double p4) {
    const double kp1 = std::fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
    const double kp2 = std::fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
    const double sw = std::max(kp1, kp2);
    if (sw < 1.0 / 20.0) {
        const double phi = std::max(sw / 20.0, 0.0);
        return 1.0 - std::tanh(10.0 * phi * phi * phi);
    }
    return 0.0;
}

// beta(i,j) of every interior cell from the ghost-filled stage state (Mod_Fluxes.f90:132-138).
void shock_sensor(Block& B) {
    B.beta.resize((size_t)B.ni * B.nj);
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i)
            B.beta[(i - 1) + B.ni * (j - 1)] = sd_tramel(B.pc(i, j)[3], B.pc(i - 1, j)[3], B.pc(i + 1, j)[3],
                                                         B.pc(i, j - 1)[3], B.pc(i, j + 1)[3]);
}

// Fluxes_blk_omp_do (Mod_Fluxes.f90:97-234), Euler part. Returns false on a bad state.
bool block_fluxes(const q2d_oracle* o, Block& B, int& eb_i, int& eb_j) {
    const int n1 = B.ni, n2 = B.nj;
    // obj_shock_detector%SD: MUSCL-SD or a sensor-driven Riemann solver (Assign_Setup.f90:49-53)
    const bool sdl = o->opt.shock_detector != 0;
    const bool sd = sdl || riemann_sd(o->opt.riemann);
    if (sd) shock_sensor(B);
    bool ok = true;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= n2; ++j)
        for (int i = 1; i <= n1; ++i) {
            double* r = B.r(i, j);
            r[0] = r[1] = r[2] = r[3] = 0.0;
        }
    int bi = 0, bj = 0;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= n2; ++j) {
        for (int i = 1; i <= n1 - 1; ++i) {
            const double dl4[4] = {B.dlc(i - 1, j, 1), B.dlc(i, j, 1), B.dlc(i + 1, j, 1),
                                   B.dlc(i + 2, j, 1)};
            const double* pr[4] = {B.pc(i - 1, j), B.pc(i, j), B.pc(i + 1, j), B.pc(i + 2, j)};
            const double* f = B.face1(i, j);
            double fl[4];
            if (!convective_flux(o, dl4, pr, f[0], f[1], f[2], sdl ? B.sd(i, j) : 1.0, sd ? B.sd(i, j) : 1.0,
                                 fl)) {
#pragma omp critical
                { if (ok) { ok = false; bi = i; bj = j; } }
                continue;
            }
            double* r0 = B.r(i, j);
            double* r1 = B.r(i + 1, j);
            for (int v = 0; v < 4; ++v) { r0[v] = r0[v] + fl[v]; r1[v] = r1[v] - fl[v]; }
        }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= n1; ++i) {
        for (int j = 1; j <= n2 - 1; ++j) {
            const double dl4[4] = {B.dlc(i, j - 1, 2), B.dlc(i, j, 2), B.dlc(i, j + 1, 2),
                                   B.dlc(i, j + 2, 2)};
            const double* pr[4] = {B.pc(i, j - 1), B.pc(i, j), B.pc(i, j + 1), B.pc(i, j + 2)};
            const double* f = B.face2(i, j);
            double fl[4];
            if (!convective_flux(o, dl4, pr, f[0], f[1], f[2], sdl ? B.sd(i, j) : 1.0, sd ? B.sd(i, j) : 1.0,
                                 fl)) {
#pragma omp critical
                { if (ok) { ok = false; bi = i; bj = j; } }
                continue;
            }
            double* r0 = B.r(i, j);
            double* r1 = B.r(i, j + 1);
            for (int v = 0; v < 4; ++v) { r0[v] = r0[v] + fl[v]; r1[v] = r1[v] - fl[v]; }
        }
    }
    if (!ok) { eb_i = bi; eb_j = bj; }
    return ok;
}

// Face_Index (Lib_BC_Fluxes.f90:34-50)
inline void face_index(int f, int ci, int cj, int& dir, int& fi, int& fj) {
    if (f <= 2) { dir = 1; fi = ci - (f % 2); fj = cj; }
    else { dir = 2; fi = ci; fj = cj - (f % 2); }
}

// BC_Symmetry_Eul (Lib_BC_Fluxes_Symmetry.f90:28-124), Un_wall = 0.
void bc_symmetry(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm) {
    const int modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm;
    const int Int_i = Im + GUIDE[Fm][0], Int_j = Jm + GUIDE[Fm][1];
    int dir, Fi, Fj;
    face_index(Fm, Im, Jm, dir, Fi, Fj);
    const double* fc = B.face(dir, Fi, Fj);
    const double n0 = fc[0], n1 = fc[1], int_l = fc[2];
    const double Bound_Dl = 0.5 * B.dlc(Im, Jm, dir);
    const double Int_Dl = 0.5 * B.dlc(Int_i, Int_j, dir);
    const double* Bp = B.pc(Im, Jm);
    const double* Ip = B.pc(Int_i, Int_j);
    double Un = Bp[1] * n0 + Bp[2] * n1;
    double G[4] = {Bp[0], Bp[1], Bp[2], Bp[3]};
    G[1] = G[1] - 2.0 * Un * n0;
    G[2] = G[2] - 2.0 * Un * n1;
    double P1[4], P3[4];
    for (int v = 0; v < 4; ++v) {
        P1[v] = modfm * G[v] + modfm1 * Ip[v];
        P3[v] = modfm * Ip[v] + modfm1 * G[v];
    }
    const double Dist12 = 2.0 * Bound_Dl * modfm + (Bound_Dl + Int_Dl) * modfm1;
    const double Dist23 = (Bound_Dl + Int_Dl) * modfm + 2.0 * Bound_Dl * modfm1;
    double Face[4];
    const double Dist = Bound_Dl * modfm2;
    for (int v = 0; v < 4; ++v) {
        const double s32 = (P3[v] - Bp[v]) / Dist23;
        const double s21 = (Bp[v] - P1[v]) / Dist12;
        const double s = rlimiter(o->opt.limiter, s32, s21);
        Face[v] = Bp[v] + s * Dist;
    }
    const Gas& g = o->gas;
    const double rotot = Face[0];
    const double Sound = f_ss(g, Face[3], rotot);
    Un = Face[1] * n0 + Face[2] * n1;
    const double vtx = Face[1] - Un * n0, vty = Face[2] - Un * n1;
    const double Un1 = Un * modfm2;
    const double U1[2] = {Un1 * n0 + vtx, Un1 * n1 + vty};
    const double U4[2] = {-Un1 * n0 + vtx, -Un1 * n1 + vty};
    const double L[4] = {Face[0], U1[0], U1[1], Face[3]};
    const double R[4] = {Face[0], U4[0], U4[1], Face[3]};
    const Flux4 F = riemann(o->opt.riemann, g, L, Sound, R, Sound, n0, n1);
    double* r = B.r(Im, Jm);
    r[1] = r[1] + modfm2 * (F.u * int_l);
    r[2] = r[2] + modfm2 * (F.v * int_l);
}

// BC_Extrapolation (Lib_BC_Fluxes_Extrapolation.f90:18-49)
void bc_extrapolation(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm) {
    int dir, Fi, Fj;
    face_index(Fm, Im, Jm, dir, Fi, Fj);
    const double* fc = B.face(dir, Fi, Fj);
    const double n0 = fc[0], n1 = fc[1], int_l = fc[2];
    const double* P = B.pc(Im, Jm);
    const double Un = P[1] * n0 + P[2] * n1;
    double F[4];
    F[0] = P[0] * Un * int_l;
    const double Fmass = F[0];
    F[1] = Fmass * P[1] + P[3] * int_l * n0;
    F[2] = Fmass * P[2] + P[3] * int_l * n1;
    F[3] = Fmass * H0(o->gas, P[3], P[0], std::sqrt(P[1] * P[1] + P[2] * P[2]));
    const double sgn = 1 - 2 * (Fm % 2);
    double* r = B.r(Im, Jm);
    for (int v = 0; v < 4; ++v) r[v] = r[v] + sgn * F[v];
}

struct InflowGeom {
    int modfm, modfm1, modfm2;
    double n0, n1, int_l, t0, t1, BC_Sign, Un, rho, Sound, Gamma, Riem;
    const double* Bp;
    const double* Ip;
};

// Setup_Inflow_Geometry (Lib_BC_Fluxes_Inflow.f90:489-541)
InflowGeom inflow_geometry(const q2d_oracle* o, const Block& B, int Im, int Jm, int Fm) {
    InflowGeom G;
    G.modfm = Fm % 2; G.modfm1 = 1 - G.modfm; G.modfm2 = 1 - 2 * G.modfm;
    const int Int_i = Im + GUIDE[Fm][0], Int_j = Jm + GUIDE[Fm][1];
    int dir, Fi, Fj;
    face_index(Fm, Im, Jm, dir, Fi, Fj);
    G.Bp = B.pc(Im, Jm);
    G.Ip = B.pc(Int_i, Int_j);
    const double* fc = B.face(dir, Fi, Fj);
    G.n0 = fc[0]; G.n1 = fc[1]; G.int_l = fc[2];
    double tx, ty;
    if (Fm <= 2) { tx = B.nx_(Fi, Fj) - B.nx_(Fi, Fj - 1); ty = B.ny_(Fi, Fj) - B.ny_(Fi, Fj - 1); }
    else { tx = B.nx_(Fi, Fj) - B.nx_(Fi - 1, Fj); ty = B.ny_(Fi, Fj) - B.ny_(Fi - 1, Fj); }
    const double tmod = std::sqrt(tx * tx + ty * ty);
    G.t0 = tx / tmod; G.t1 = ty / tmod;
    G.BC_Sign = (double)G.modfm2;
    G.Un = G.Bp[1] * G.n0 + G.Bp[2] * G.n1;
    G.rho = G.Bp[0];
    G.Sound = f_ss(o->gas, G.Bp[3], G.rho);
    G.Gamma = f_gamma(o->gas, G.Bp[3], G.rho);
    G.Riem = G.Sound + G.BC_Sign * 0.5 * (G.Gamma - 1.0) * G.Un;
    return G;
}

// Compute_Inflow_Direction (Lib_BC_Fluxes_Inflow.f90:548-563)
inline double inflow_direction(double n0, double n1, double alpha_in) {
    if (alpha_in >= 0.5 * DBL_MAX) return std::atan(n1 / (n0 + 1e-20));
    return alpha_in;
}

// BC_Inlet_StagnCond + Stagn_Inflow (Lib_BC_Fluxes_Inflow.f90:64-120, 412-483).
// Returns false when the flow leaves the domain (caller falls back to symmetry).
bool bc_stagnation(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm, const q2d_bc_rec& rec) {
    const InflowGeom G = inflow_geometry(o, B, Im, Jm, Fm);
    if (G.BC_Sign * G.Un >= 0.0) return false;
    const double alpha = inflow_direction(G.n0, G.n1, rec.alpha);
    const double Gamma = G.Gamma, Rg = o->gas.R;
    const double XA = G.n1 - G.n0 * std::tan(alpha);
    const double XB = G.t1 - G.t0 * std::tan(alpha);
    const double E1 = -XA / XB;
    double Discr = -1.0, p0try = rec.p0;
    int iter = 0;
    double Sound0 = 0, Coef_D = 0, YA = 0, YB = 0;
    const double p = G.Bp[3];
    while (Discr < 0.0) {
        ++iter;
        Sound0 = std::sqrt(Gamma * Rg * rec.T0);
        Coef_D = (1.0 + E1 * E1) * (Gamma - 1.0) / 2.0;
        double Coef_C = std::pow(p0try / p, (Gamma - 1.0) / Gamma);
        const double ss = G.Sound / Sound0;
        Coef_C = Coef_C * (ss * ss);
        const double gh = (Gamma - 1.0) / 2.0;
        YA = gh * gh + Coef_C * Coef_D;
        YB = G.BC_Sign * G.Riem * ((Gamma - 1.0) / 2.0);
        const double YC = G.Riem * G.Riem - Coef_C * (Sound0 * Sound0);
        Discr = YB * YB - YA * YC;
        if (Discr < 0.0 && std::fabs(Discr) < 1e-2) Discr = 0.0;
        if (Discr < 0.0 && std::fabs(Discr) > 1e-2) p0try = rec.rel_fac * p0try + (1 - rec.rel_fac) * p;
        if (iter > 1000) { Discr = 0.0; break; }
    }
    const double Un_Sign = std::copysign(1.0, G.Un);
    const double Un3 = (YB + Un_Sign * std::sqrt(Discr)) / YA;
    const double Sound3 = std::sqrt(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
    const double p3 = p0try * std::pow(Sound3 / Sound0, 2.0 * Gamma / (Gamma - 1.0));
    const double Ut3 = Un3 * E1;
    const double Face_rho = Gamma * p3 / (Sound3 * Sound3);
    const double Face_r1 = 1.0 * Face_rho;
    const double fu = Un3 * G.n0 + Ut3 * G.t0;
    const double fv = Un3 * G.n1 + Ut3 * G.t1;
    const double Face_T = p3 / (Rg * Face_rho);
    const double Face_H = 0.0 + Face_r1 / Face_rho * h_of_T(o->gas, Face_T);
    double F[4];
    F[0] = Face_r1 * Un3 * G.int_l;
    const double Fmass = Face_rho * Un3 * G.int_l;
    F[1] = Fmass * fu + p3 * G.int_l * G.n0;
    F[2] = Fmass * fv + p3 * G.int_l * G.n1;
    F[3] = Fmass * (0.5 * (fu * fu + fv * fv) + Face_H);
    double* r = B.r(Im, Jm);
    for (int v = 0; v < 4; ++v) r[v] = r[v] + G.modfm2 * F[v];
    return true;
}

// BC_Inlet_Supersonic_Static + Supersonic_Inflow (Lib_BC_Fluxes_Inflow.f90:272-311, 321-403)
bool bc_supersonic(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm, const q2d_bc_rec& rec) {
    const InflowGeom G = inflow_geometry(o, B, Im, Jm, Fm);
    if (G.BC_Sign * G.Un >= 0.0) return false;
    const Gas& g = o->gas;
    const double* P2 = G.Bp;
    const double flow_Sound = f_ss(g, P2[3], P2[0]);
    const double flow_Mach = std::sqrt(P2[1] * P2[1] + P2[2] * P2[2]) / flow_Sound;
    const double Mloc = rec.rel_fac * rec.mach + (1 - rec.rel_fac) * flow_Mach;
    const double ploc = rec.rel_fac * rec.pamb + (1 - rec.rel_fac) * P2[3];
    const double alpha = inflow_direction(G.n0, G.n1, rec.alpha);
    double Sup[4];
    Sup[3] = ploc;
    const double Sup_rho = Sup[3] / (g.R * rec.T0);
    Sup[0] = Sup_rho * 1.0;
    const double Sup_Sound = f_ss(g, Sup[3], Sup_rho);
    Sup[1] = Mloc * Sup_Sound * std::cos(alpha);
    Sup[2] = Mloc * Sup_Sound * std::sin(alpha);
    double P1[4], P3[4], Face[4];
    for (int v = 0; v < 4; ++v) {
        P1[v] = G.modfm * Sup[v] + G.modfm1 * G.Ip[v];
        P3[v] = G.modfm * G.Ip[v] + G.modfm1 * Sup[v];
    }
    for (int v = 0; v < 4; ++v) {
        const double d32 = P3[v] - P2[v], d21 = P2[v] - P1[v];
        const double s = rlimiter(o->opt.limiter, d32, d21);
        Face[v] = P2[v] + 0.5 * s * G.modfm2;
    }
    double PL[4], PR[4];
    for (int v = 0; v < 4; ++v) {
        PL[v] = G.modfm * Sup[v] + G.modfm1 * Face[v];
        PR[v] = G.modfm * Face[v] + G.modfm1 * Sup[v];
    }
    const double aL = f_ss(g, PL[3], PL[0]);
    const double aR = f_ss(g, PR[3], PR[0]);
    const Flux4 F = riemann(o->opt.riemann, g, PL, aL, PR, aR, G.n0, G.n1);
    const double su = std::copysign(1.0, F.r);
    const double SelL = (1.0 + su) / 2.0, SelR = (su - 1.0) / 2.0;
    const double Fmass = F.r * G.int_l;
    double Fl[4];
    Fl[0] = Fmass * (SelL * PL[0] / PL[0] - SelR * PR[0] / PR[0]);
    Fl[1] = F.u * G.int_l;
    Fl[2] = F.v * G.int_l;
    Fl[3] = F.e * G.int_l;
    double* r = B.r(Im, Jm);
    for (int v = 0; v < 4; ++v) r[v] = r[v] + G.modfm2 * Fl[v];
    return true;
}

// BC_Outflow + Outflow (Lib_BC_Fluxes_Outflow.f90:36-165)
bool bc_outflow(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm, const q2d_bc_rec& rec) {
    const int modfm = Fm % 2, modfm2 = 1 - 2 * modfm;
    int dir, Fi, Fj;
    face_index(Fm, Im, Jm, dir, Fi, Fj);
    const double* Bp = B.pc(Im, Jm);
    const double* fc = B.face(dir, Fi, Fj);
    const double n0 = fc[0], n1 = fc[1], int_l = fc[2];
    const double BC_Sign = (double)modfm2;
    const double Un = Bp[1] * n0 + Bp[2] * n1;
    if (BC_Sign * Un < 0.0) return false;
    const Gas& g = o->gas;
    const double rho = Bp[0];
    const double Sound = f_ss(g, Bp[3], rho);
    const double Gamma = f_gamma(g, Bp[3], rho);
    const double Riem = Sound + BC_Sign * 0.5 * (Gamma - 1.0) * Un;
    const double vtx = Bp[1] - Un * n0, vty = Bp[2] - Un * n1;
    const double Mach_N = std::fabs(Un / Sound);
    double Face[4], Face_Un, Face_rho;
    if (Mach_N < 1.0 && rec.pamb > 0.0) {
        double p_exit = rec.pamb;
        const double delta = 0.5 * (Gamma - 1.0);
        const double den = 1.0 / std::pow(1 + delta, Gamma / (Gamma - 1.0));
        const double pstar = Bp[3] * den * std::pow(1 + delta * (Mach_N * Mach_N), Gamma / (Gamma - 1.0));
        if (pstar >= p_exit) p_exit = pstar;
        const double Isen = (Gamma - 1.0) / (2.0 * Gamma);
        Face[3] = p_exit * rec.rel_fac + Bp[3] * (1.0 - rec.rel_fac);
        const double Face_Sound = Sound * std::pow(Face[3] / Bp[3], Isen);
        Face_Un = (Riem - Face_Sound) / (BC_Sign * 0.5 * (Gamma - 1.0));
        Face_rho = Gamma * Face[3] / (Face_Sound * Face_Sound);
        Face[0] = Bp[0] / rho * Face_rho;
        Face[1] = vtx + Face_Un * n0;
        Face[2] = vty + Face_Un * n1;
    } else {
        for (int v = 0; v < 4; ++v) Face[v] = Bp[v];
        Face_Un = Un;
        Face_rho = rho;
    }
    const double Face_T = Face[3] / (g.R * Face_rho);
    const double Face_H = 0.0 + Face[0] / Face_rho * h_of_T(g, Face_T);
    double F[4];
    F[0] = Face[0] * int_l * Face_Un;
    const double mdot = Face_rho * int_l * Face_Un;
    F[1] = Face[1] * mdot + Face[3] * int_l * n0;
    F[2] = Face[2] * mdot + Face[3] * int_l * n1;
    F[3] = mdot * (0.5 * (Face[1] * Face[1] + Face[2] * Face[2]) + Face_H);
    double* r = B.r(Im, Jm);
    for (int v = 0; v < 4; ++v) r[v] = r[v] + modfm2 * F[v];
    return true;
}

// BC_Connection_Eul (Lib_BC_Fluxes_Connection.f90:24-133)
bool bc_connection(const q2d_oracle* o, Block& B, int Im, int Jm, int Fm) {
    const int modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm;
    int dir, Fi, Fj;
    face_index(Fm, Im, Jm, dir, Fi, Fj);
    const int gx = GUIDE[Fm][0], gy = GUIDE[Fm][1];
    const int I1 = modfm * (Im - gx * GC) + modfm1 * (Im + gx);
    const int J1 = modfm * (Jm - gy * GC) + modfm1 * (Jm + gy);
    const int I2 = modfm1 * Im + modfm * (Im - gx);
    const int J2 = modfm1 * Jm + modfm * (Jm - gy);
    const int I3 = modfm1 * (Im - gx) + modfm * Im;
    const int J3 = modfm1 * (Jm - gy) + modfm * Jm;
    const int I4 = modfm1 * (Im - gx * GC) + modfm * (Im + gx);
    const int J4 = modfm1 * (Jm - gy * GC) + modfm * (Jm + gy);
    const double* fc = B.face(dir, Fi, Fj);
    const double Dl1 = B.dlc(I1, J1, dir) * 0.5;
    const double Dl2 = B.dlc(I2, J2, dir) * 0.5;
    const double Dl3 = B.dlc(I3, J3, dir) * 0.5;
    const double Dl4 = B.dlc(I4, J4, dir) * 0.5;
    const double Dist23 = Dl2 + Dl3, Dist12 = Dl1 + Dl2, Dist34 = Dl3 + Dl4;
    double PL[4], PR[4];
    // SD_limiter / SD_riemann: beta of the boundary cell (Lib_BC_Fluxes_Connection.f90,
    // beta_ = blk%beta(Im,Jm)) for the reconstruction / the Riemann solver
    const double beta_l = o->opt.shock_detector ? B.sd(Im, Jm) : 1.0;
    const double beta_r = riemann_sd(o->opt.riemann) ? B.sd(Im, Jm) : 1.0;
    reconstruct(o->opt.limiter, B.pc(I1, J1), B.pc(I2, J2), B.pc(I3, J3), B.pc(I4, J4), Dist12,
                Dist23, Dist34, Dl2, Dl3, beta_l, PL, PR);
    double F[4];
    if (!face_flux_from_states(o, PL, PR, fc[0], fc[1], fc[2], beta_r, F)) return false;
    double* r = B.r(Im, Jm);
    for (int v = 0; v < 4; ++v) r[v] = r[v] + F[v] * modfm2;
    return true;
}

// BC_Fluxes (Mod_BC_Fluxes.f90:49-271), record order.
bool bc_fluxes(q2d_oracle* o, Case& cs, int& eb, int& ei, int& ej) {
    for (const q2d_bc_rec& rec : cs.bc) {
        Block& B = o->blk[cs.blocks[rec.b - 1]];
        const int Im = rec.i, Jm = rec.j, Fm = rec.f;
        switch (rec.type) {
            case 101: case 201:   // connection and periodic seam (Mod_BC_Fluxes.f90:99-102)
                if (!bc_connection(o, B, Im, Jm, Fm)) { eb = rec.b; ei = Im; ej = Jm; return false; }
                break;
            case 300: bc_symmetry(o, B, Im, Jm, Fm); break;
            case 400: bc_extrapolation(o, B, Im, Jm, Fm); break;
            case 401: if (!bc_stagnation(o, B, Im, Jm, Fm, rec)) bc_symmetry(o, B, Im, Jm, Fm); break;
            case 405: if (!bc_supersonic(o, B, Im, Jm, Fm, rec)) bc_symmetry(o, B, Im, Jm, Fm); break;
            case 406: if (!bc_outflow(o, B, Im, Jm, Fm, rec)) bc_symmetry(o, B, Im, Jm, Fm); break;
            default: break;   // type 0: no flux
        }
    }
    return true;
}

// Source_Axi_Eul_Blk (Lib_Source_Axisymmetry.f90:40-78) and
// Source_Area_Eul_Blk (Lib_Source_Areavariation.f90:104-144)
void sources(const q2d_oracle* o, Block& B) {
    const Gas& g = o->gas;
    const int src = o->opt.source;
    if (src == Q2D_SRC_NONE) return;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
            const double* P = B.pc(i, j);
            const double rho = P[0];
            const double mod_v = std::sqrt(P[1] * P[1] + P[2] * P[2]);
            const int k = (i - 1) + B.ni * (j - 1);
            double S[4];
            if (src == Q2D_SRC_AXI) {
                const double invr = B.inv_r[k];
                S[0] = -P[0] * P[2] * invr;
                S[1] = -rho * P[1] * P[2] * invr;
                S[2] = -rho * P[2] * P[2] * invr;
                S[3] = -(rho * E0(g, P[3], P[0], mod_v) + P[3]) * P[2] * invr;
            } else {
                const double Gx = B.Gx[k], Gy = B.Gy[k];
                const double VG = P[1] * Gx + P[2] * Gy;
                S[0] = P[0] * VG;
                S[1] = rho * P[1] * VG;
                S[2] = rho * P[2] * VG;
                S[3] = (rho * E0(g, P[3], P[0], mod_v) + P[3]) * VG;
            }
            double* r = B.r(i, j);
            const double s = B.sur[B.c(i, j)];
            for (int v = 0; v < 4; ++v) r[v] = r[v] - S[v] * s;
        }
}

// RKcoeff (Lib_RK.f90:8-11)
inline double rk_coeff(int n_rk, int irk) {
    static const double C[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.5, 0.0}, {1.0, 0.25, 2.0 / 3.0}};
    return C[n_rk - 1][irk - 1];
}

// Newstate_Conservative / Compute_Cons_NoIRS + Check_And_Fix_State
// (Lib_Newstate.f90:14-161, 316-350)
bool newstate(const q2d_oracle* o, Block& B, int irk, int& ei, int& ej, bool scaled) {
    const Gas& g = o->gas;
    const double c = rk_coeff(o->opt.n_rk, irk);
    const double strangcoeff = 1.0;
    bool ok = true;
    int bi = 0, bj = 0;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
            double* prim = B.p(i, j);
            const double* primold = &B.PO[4 * B.c(i, j)];
            double* res = B.r(i, j);
            const double surface = B.sur[B.c(i, j)];
            const double dt = B.dtlocal[(i - 1) + B.ni * (j - 1)];
            if (!scaled)   // Compute_Cons_NoIRS; with IRS the residual was scaled before smoothing
                for (int v = 0; v < 4; ++v) res[v] = -res[v] / surface * dt * strangcoeff;
            double consold[4], cons[4];
            prim2cons(g, primold, consold);
            prim2cons(g, prim, cons);
            for (int v = 0; v < 4; ++v) cons[v] = consold[v] + (cons[v] - consold[v] + res[v]) * c;
            cons2prim(g, cons, prim, prim[3] / (prim[0] * g.R));   // guess: the state before
            bool bad = false;
            for (int v = 0; v < 4; ++v) bad = bad || std::isnan(prim[v]);
            if (bad || prim[3] < 0.0) {
#pragma omp critical
                { if (ok) { ok = false; bi = i; bj = j; } }
            }
            if (prim[0] < 1e-20) prim[0] = 1e-20;
        }
    if (!ok) { ei = bi; ej = bj; }
    return ok;
}

// Residual_Smoothing (Lib_IRS.f90:17-177): per grid direction, the first ghost layer of the
// (scaled) residual is filled by Ghost_Residual_Extrapolation (connections copy the donor cell,
// every other record the boundary cell), then two Jacobi sweeps of
// R*(i) = (R(i) + beta (R*(i-1) + R*(i+1))) / (1 + 2 beta) along that direction replace R.
void residual_smoothing(q2d_oracle* o, Case& cs, double beta) {
    const int ndir = (o->blk[cs.blocks[0]].nj == 1) ? 1 : 2;
    for (int d = 1; d <= ndir; ++d) {
        for (const q2d_bc_rec& r : cs.bc) {   // Ghost_Residual_Extrapolation (:125-177)
            Block& B = o->blk[cs.blocks[r.b - 1]];
            const int gi = r.i - (r.f == 1 ? 1 : r.f == 2 ? -1 : 0);
            const int gj = r.j - (r.f == 3 ? 1 : r.f == 4 ? -1 : 0);
            const double* src = (r.type == 101 || r.type == 201) ? o->blk[cs.blocks[r.bs - 1]].r(r.is, r.js) : B.r(r.i, r.j);
            double* g = B.r(gi, gj);
            for (int v = 0; v < 4; ++v) g[v] = src[v];
        }
        for (int bid : cs.blocks) {   // Residual_Smoothing_Blk (:45-119)
            Block& B = o->blk[bid];
            std::vector<double> S(B.R), Sn(B.R);
            for (int it = 0; it < 2; ++it) {
#pragma omp parallel for schedule(static)
                for (int j = 1; j <= B.nj; ++j)
                    for (int i = 1; i <= B.ni; ++i) {
                        const int i1 = d == 1 ? i - 1 : i, j1 = d == 1 ? j : j - 1;
                        const int i2 = d == 1 ? i + 1 : i, j2 = d == 1 ? j : j + 1;
                        const double* r0 = B.r(i, j);
                        const double* rm = &S[4 * B.c(i1, j1)];
                        const double* rp = &S[4 * B.c(i2, j2)];
                        double* out = &Sn[4 * B.c(i, j)];
                        for (int v = 0; v < 4; ++v) out[v] = (r0[v] + beta * (rm[v] + rp[v])) / (1.0 + 2.0 * beta);
                    }
                for (int j = 1; j <= B.nj; ++j)
                    for (int i = 1; i <= B.ni; ++i)
                        std::memcpy(&S[4 * B.c(i, j)], &Sn[4 * B.c(i, j)], sizeof(double) * 4);
            }
            for (int j = 1; j <= B.nj; ++j)
                for (int i = 1; i <= B.ni; ++i) std::memcpy(B.r(i, j), &S[4 * B.c(i, j)], sizeof(double) * 4);
        }
    }
}

// Compute_dt (Mod_dt.f90:10-106), Euler model (model == 0).
void compute_dt(q2d_oracle* o, Case& cs, int ndir) {
    const Gas& g = o->gas;
    double dtglobal = cs.dtglobal;
    for (int bid : cs.blocks) {
        Block& B = o->blk[bid];
        double dmin = dtglobal;
#pragma omp parallel for schedule(static) reduction(min : dmin)
        for (int j = 1; j <= B.nj; ++j)
            for (int i = 1; i <= B.ni; ++i) {
                const double* P = B.pc(i, j);
                const double* M = &B.M[4 * B.c(i, j)];
                const double Sound = f_ss(g, P[3], P[0]);
                double dtmin = 1e8;
                for (int d = 1; d <= ndir; ++d) {
                    const double m0 = M[2 * (d - 1)], m1 = M[2 * (d - 1) + 1];   // M(d,:)
                    const double nrm = std::sqrt(m0 * m0 + m1 * m1);
                    const double v0 = m0 / nrm, v1 = m1 / nrm;
                    const double vel_ = std::fabs(P[1] * v0 + P[2] * v1);
                    const double lambda = vel_ + Sound;
                    const double dt = B.dlc(i, j, d) / lambda * o->opt.cfl;
                    dtmin = fmin_(dt, dtmin);
                }
                double dtcell = dtmin;
                if (cs.iter < o->opt.rampa_iter) dtcell = dtcell * (double)cs.iter / (double)o->opt.rampa_iter;
                B.dtlocal[(i - 1) + B.ni * (j - 1)] = dtcell;
                dmin = fmin_(dtcell, dmin);
            }
        dtglobal = dmin;
    }
    cs.dtglobal = dtglobal;
}

// Compute_Residual (Mod_Diagnostic.f90:438-469): sum of squares in (j, i) order.
void compute_residual(q2d_oracle* o, Case& cs, double* total) {
    for (int bid : cs.blocks) {
        Block& B = o->blk[bid];
        std::vector<double> rows(4 * (size_t)B.nj, 0.0);
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= B.nj; ++j) {
            double acc[4] = {0, 0, 0, 0};
            for (int i = 1; i <= B.ni; ++i) {
                const double* nw = B.pc(i, j);
                const double* od = &B.PO[4 * B.c(i, j)];
                for (int v = 0; v < 4; ++v) {
                    const double rn = std::fabs(nw[v] - od[v]);
                    acc[v] = acc[v] + rn * rn;
                }
            }
            for (int v = 0; v < 4; ++v) rows[4 * (j - 1) + v] = acc[v];
        }
        for (int j = 0; j < B.nj; ++j)
            for (int v = 0; v < 4; ++v) total[v] = total[v] + rows[4 * j + v];
    }
}

// Explicit_Step (Mod_Explicit.f90:10-174) for one case.
void explicit_step(q2d_oracle* o, Case& cs) {
    const q2d_options& op = o->opt;
    cs.iter += 1;
    cs.iter_from_call += 1;
    const int ndir = (o->blk[cs.blocks[0]].nj == 1) ? 1 : 2;   // Check_Mesh_Type
    cs.dtglobal = 1e5;
    compute_dt(o, cs, ndir);
    if (op.time_accurate) {
        for (int bid : cs.blocks) {   // Set_Global_dt
            Block& B = o->blk[bid];
            std::fill(B.dtlocal.begin(), B.dtlocal.end(), cs.dtglobal);
        }
        cs.time = cs.time + cs.dtglobal;
    }
    for (int bid : cs.blocks) {   // Copy_State
        Block& B = o->blk[bid];
        for (int j = 1; j <= B.nj; ++j)
            for (int i = 1; i <= B.ni; ++i)
                std::memcpy(&B.PO[4 * B.c(i, j)], B.pc(i, j), sizeof(double) * 4);
    }
    for (int irk = 1; irk <= op.n_rk; ++irk) {
        ghost_fill(o, cs);
        for (size_t lb = 0; lb < cs.blocks.size(); ++lb) {
            int ei = 0, ej = 0;
            if (!block_fluxes(o, o->blk[cs.blocks[lb]], ei, ej)) {
                cs.err = Q2D_ERR_NONPHYSICAL; cs.err_b = (int)lb + 1; cs.err_i = ei; cs.err_j = ej;
                cs.err_stage = irk; cs.done = true; return;
            }
        }
        int eb = 0, ei = 0, ej = 0;
        if (!bc_fluxes(o, cs, eb, ei, ej)) {
            cs.err = Q2D_ERR_NONPHYSICAL; cs.err_b = eb; cs.err_i = ei; cs.err_j = ej;
            cs.err_stage = irk; cs.done = true; return;
        }
        for (int bid : cs.blocks) sources(o, o->blk[bid]);
        const bool irs = op.irs_beta > 0.0;
        if (irs) {   // Newstate_Conservative IRS branch (Lib_Newstate.f90:36-66): scale, smooth, update
            for (int bid : cs.blocks) {
                Block& B = o->blk[bid];
                for (int j = 1; j <= B.nj; ++j)
                    for (int i = 1; i <= B.ni; ++i) {
                        double* res = B.r(i, j);
                        const double surface = B.sur[B.c(i, j)];
                        const double dt = B.dtlocal[(i - 1) + B.ni * (j - 1)];
                        for (int v = 0; v < 4; ++v) res[v] = -res[v] / surface * dt * 1.0;
                    }
            }
            residual_smoothing(o, cs, op.irs_beta);
        }
        for (size_t lb = 0; lb < cs.blocks.size(); ++lb) {
            if (!newstate(o, o->blk[cs.blocks[lb]], irk, ei, ej, irs)) {
                cs.err = Q2D_ERR_NAN; cs.err_b = (int)lb + 1; cs.err_i = ei; cs.err_j = ej;
                cs.err_stage = irk; cs.done = true; return;
            }
        }
    }
    if (cs.iter_from_call == 1 || (cs.iter % op.res_diter) == 0) {
        double tot[4] = {0, 0, 0, 0};
        compute_residual(o, cs, tot);
        for (int v = 0; v < 4; ++v) cs.res[v] = std::sqrt(tot[v]);
        if (cs.res0 < 0.0) cs.res0 = cs.res[0];
    }
    const double thr = op.res_relative ? op.res_threshold * cs.res0 : op.res_threshold;
    const bool endsim = (cs.iter_from_call >= op.itermax) || (cs.res[0] <= thr) ||
                        (cs.time >= op.time_threshold) || (cs.iter_end > 0 && cs.iter >= cs.iter_end);
    const bool iosim = ((cs.iter % op.sol_diter) == 0) || (cs.time >= cs.time_from_call + op.sol_dtime);
    if (endsim) { cs.todo = Q2D_TODO_END; cs.done = true; }
    else if (iosim) cs.todo = Q2D_TODO_IO;
    else cs.todo = Q2D_TODO_CONTINUE;
}

void fill_info(const Case& cs, q2d_step_info* out) {
    out->dtglobal = cs.dtglobal;
    out->time = cs.time;
    out->iter = cs.iter;
    for (int v = 0; v < 4; ++v) out->residual[v] = cs.res[v];
    out->residual0 = cs.res0;
    out->todo = cs.todo;
    out->err = cs.err;
    out->err_b = cs.err_b; out->err_i = cs.err_i; out->err_j = cs.err_j; out->err_stage = cs.err_stage;
}

int commit(q2d_oracle* o) {
    if (o->committed) return Q2D_OK;
    for (Block& B : o->blk) {
        const size_t ng = (size_t)(B.ni + 4) * (B.nj + 4);
        B.M.assign(4 * ng, 0.0);
        B.dl.assign(2 * ng, 0.0);
        B.sur.assign(ng, 0.0);
        B.R.assign(4 * ng, 0.0);
        B.PO.assign(4 * ng, 0.0);
        B.dtlocal.assign((size_t)B.ni * B.nj, 0.0);
        for (int j = 1; j <= B.nj; ++j)          // Setup_Metrics interior (Mod_Metrics.f90:41-56)
            for (int i = 1; i <= B.ni; ++i) {
                const int e = metric_into(B, i, j, nodev(B, i - 1, j - 1), nodev(B, i - 1, j),
                                          nodev(B, i, j - 1), nodev(B, i, j));
                if (e) return e;
            }
        norm_area(B);
        const size_t n = (size_t)B.ni * B.nj;
        if (o->opt.source == Q2D_SRC_AXI) {      // Precompute_Axisymmetric_Geometry :19-37
            B.inv_r.assign(n, 0.0);
            for (int j = 1; j <= B.nj; ++j)
                for (int i = 1; i <= B.ni; ++i) {
                    const double r_ave = 0.25 * (B.ny_(i, j) + B.ny_(i - 1, j) + B.ny_(i, j - 1) +
                                                 B.ny_(i - 1, j - 1));
                    B.inv_r[(i - 1) + B.ni * (j - 1)] = 1.0 / fmax_(r_ave, 1e-12);
                }
        }
        if (o->opt.source == Q2D_SRC_AREA) {     // Precompute_Area_Geometry :26-50
            B.Gx.assign(n, 0.0);
            B.Gy.assign(n, 0.0);
            if (!B.area.empty()) {
                auto A = [&](int i, int j) { return B.area[i + (B.ni + 1) * j]; };
                for (int j = 1; j <= B.nj; ++j)
                    for (int i = 1; i <= B.ni; ++i) {
                        const double dAij0 = 0.5 * ((A(i, j) - A(i - 1, j)) + (A(i, j - 1) - A(i - 1, j - 1)));
                        const double dAij1 = 0.5 * ((A(i, j) - A(i, j - 1)) + (A(i - 1, j) - A(i - 1, j - 1)));
                        const double* M = &B.M[4 * B.c(i, j)];
                        const double dA0 = dAij0 * M[0] + dAij1 * M[2];
                        const double dA1 = dAij0 * M[1] + dAij1 * M[3];
                        const double Ac = 0.25 * (A(i, j) + A(i - 1, j) + A(i, j - 1) + A(i - 1, j - 1));
                        B.Gx[(i - 1) + B.ni * (j - 1)] = -dA0 / fmax_(Ac, 1e-12);
                        B.Gy[(i - 1) + B.ni * (j - 1)] = -dA1 / fmax_(Ac, 1e-12);
                    }
            }
        }
    }
    for (Case& cs : o->cases) {                   // ghost metrics (Mod_Metrics.f90:97-146)
        for (const q2d_bc_rec& rec : cs.bc) {
            Block& B = o->blk[cs.blocks[rec.b - 1]];
            int e = Q2D_OK;
            if (rec.type == 101 || rec.type == 201) {
                const Block& S = o->blk[cs.blocks[rec.bs - 1]];
                e = connect_metrics(B, rec.i, rec.j, rec.f, S, rec.is, rec.js, rec.fs, rec.d11, rec.d21,
                                    rec.type == 201);
            } else if (rec.type == 300) {
                symmetry_metrics(B, rec.i, rec.j, rec.f);
            } else {
                e = extrapolate_metrics(B, rec.i, rec.j, rec.f);
            }
            if (e) return e;
        }
        cs.time_from_call = cs.time;
    }
    o->committed = true;
    return Q2D_OK;
}

bool rec_less(const q2d_bc_rec& a, const q2d_bc_rec& b) {
    if (a.b != b.b) return a.b < b.b;
    return a.f < b.f;
}

}  // namespace

extern "C" {

int q2d_oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int q2d_oracle_create(q2d_oracle** out, const q2d_options* opt) {
    if (!out || !opt) return Q2D_ERR_BADARG;
    if (opt->n_rk < 1 || opt->n_rk > 3 || !(opt->gas_gamma > 1.0) || !(opt->gas_R > 0.0) || !(opt->irs_beta >= 0.0) ||
        opt->res_diter < 1 || opt->sol_diter < 1 || opt->shock_detector < 0 || opt->shock_detector > 1 ||
        opt->riemann < 0 || opt->riemann > Q2D_RIEMANN_AUSMP_UP2 || !(opt->riemann_minf >= 0.0) ||
        ((opt->riemann == Q2D_RIEMANN_AUSMP_UP || opt->riemann == Q2D_RIEMANN_AUSMP_UP2) && !(opt->riemann_minf > 0.0)))
        return Q2D_ERR_BADARG;
    q2d_oracle* o = new (std::nothrow) q2d_oracle();
    if (!o) return Q2D_ERR_OOM;
    o->opt = *opt;
    o->gas.R = opt->gas_R;
    o->gas.gamma = opt->gas_gamma;
    o->gas.gm1 = opt->gas_gamma - 1.0;
    o->gas.cp = opt->gas_gamma * opt->gas_R / (opt->gas_gamma - 1.0);
    o->gas.cv = opt->gas_R / (opt->gas_gamma - 1.0);
    o->gas.minf = opt->riemann_minf;
    *out = o;
    return Q2D_OK;
}

int q2d_oracle_add_case(q2d_oracle* o, int* case_id) {
    if (!o || o->committed) return Q2D_ERR_BADARG;
    o->cases.emplace_back();
    if (case_id) *case_id = (int)o->cases.size() - 1;
    return Q2D_OK;
}

int q2d_oracle_add_block(q2d_oracle* o, int case_id, int ni, int nj, const double* nodes_xy,
                         const double* cross_section, int* block_id) {
    if (!o || o->committed || case_id < 0 || case_id >= (int)o->cases.size() || ni < 1 || nj < 1 ||
        !nodes_xy)
        return Q2D_ERR_BADARG;
    Block B;
    B.ni = ni; B.nj = nj; B.case_id = case_id;
    B.local_b = (int)o->cases[case_id].blocks.size() + 1;
    B.node.assign(nodes_xy, nodes_xy + 2 * (size_t)(ni + 1) * (nj + 1));
    if (cross_section) B.area.assign(cross_section, cross_section + (size_t)(ni + 1) * (nj + 1));
    B.P.assign(4 * (size_t)(ni + 4) * (nj + 4), 0.0);
    o->blk.push_back(std::move(B));
    o->cases[case_id].blocks.push_back((int)o->blk.size() - 1);
    if (block_id) *block_id = (int)o->blk.size() - 1;
    return Q2D_OK;
}

int q2d_oracle_set_bcs(q2d_oracle* o, int case_id, const q2d_bc_rec* recs, int n) {
    if (!o || o->committed || case_id < 0 || case_id >= (int)o->cases.size() || n < 0 || (n && !recs))
        return Q2D_ERR_BADARG;
    Case& cs = o->cases[case_id];
    std::vector<q2d_bc_rec> v(recs, recs + n);
    for (const q2d_bc_rec& r : v) {
        if (r.b < 1 || r.b > (int)cs.blocks.size() || r.f < 1 || r.f > 4) return Q2D_ERR_BADARG;
        const Block& B = o->blk[cs.blocks[r.b - 1]];
        if (r.i < 1 || r.i > B.ni || r.j < 1 || r.j > B.nj) return Q2D_ERR_BADARG;
        switch (r.type) {
            case 400:
                if ((r.f <= 2 && B.ni < 3) || (r.f >= 3 && B.nj < 3)) return Q2D_ERR_BADARG;
                break;
            case 0: case 300: case 401: case 405: case 406:
                if (r.f <= 2 && B.ni < 2) return Q2D_ERR_BADARG;
                break;
            case 101: case 201:
                if (r.bs < 1 || r.bs > (int)cs.blocks.size() || r.fs < 1 || r.fs > 4) return Q2D_ERR_BADARG;
                break;
            default: return Q2D_ERR_UNSUPPORTED;
        }
    }
    std::stable_sort(v.begin(), v.end(), rec_less);
    cs.bc = std::move(v);
    return Q2D_OK;
}

int q2d_oracle_upload_prim(q2d_oracle* o, int block_id, const double* P) {
    if (!o || block_id < 0 || block_id >= (int)o->blk.size() || !P) return Q2D_ERR_BADARG;
    Block& B = o->blk[block_id];
    for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i)
            std::memcpy(B.p(i, j), &P[4 * B.c(i, j)], sizeof(double) * 4);
    return Q2D_OK;
}

int q2d_oracle_set_case_time(q2d_oracle* o, int case_id, double time) {
    if (!o || o->committed || case_id < 0 || case_id >= (int)o->cases.size() || !std::isfinite(time))
        return Q2D_ERR_BADARG;
    o->cases[case_id].time = time;   // Wrap_Setup.f90:141-144: time = solutiontime, counters at 0
    return Q2D_OK;
}

int q2d_oracle_set_thermo_table(q2d_oracle* o, int ntab, const double* h_tab, const double* cp_tab) {
    if (!o || o->committed || ntab < 2 || !h_tab || !cp_tab) return Q2D_ERR_BADARG;
    if (o->opt.precision != Q2D_PREC_FP64 || o->opt.riemann > Q2D_RIEMANN_LLF || o->opt.shock_detector)
        return Q2D_ERR_BADARG;   // HLLC, HLLE and LLF in the FP64 form
    for (int k = 0; k < ntab; ++k)
        if (!std::isfinite(h_tab[k]) || !(cp_tab[k] > o->gas.R)) return Q2D_ERR_BADARG;
    for (int k = 0; k + 1 < ntab; ++k)   // e(T) = h - R T increasing: an invertible energy
        if (!(h_tab[k + 1] - h_tab[k] > o->gas.R)) return Q2D_ERR_BADARG;
    o->htab.assign(h_tab, h_tab + ntab);
    o->cptab.assign(cp_tab, cp_tab + ntab);
    o->gas.htab = o->htab.data();
    o->gas.cptab = o->cptab.data();
    o->gas.ntab = ntab;
    return Q2D_OK;
}

int q2d_oracle_set_case_end(q2d_oracle* o, int case_id, long long iter_end) {
    if (!o || case_id < 0 || case_id >= (int)o->cases.size() || iter_end < 0) return Q2D_ERR_BADARG;
    o->cases[case_id].iter_end = iter_end;
    return Q2D_OK;
}

int q2d_oracle_download_prim(q2d_oracle* o, int block_id, double* P) {
    if (!o || block_id < 0 || block_id >= (int)o->blk.size() || !P) return Q2D_ERR_BADARG;
    Block& B = o->blk[block_id];
    for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i)
            std::memcpy(&P[4 * B.c(i, j)], B.pc(i, j), sizeof(double) * 4);
    return Q2D_OK;
}

int q2d_oracle_commit(q2d_oracle* o) {
    if (!o) return Q2D_ERR_BADARG;
    return commit(o);
}

int q2d_oracle_step(q2d_oracle* o, int nsteps, q2d_step_info* out) {
    if (!o || nsteps < 0) return Q2D_ERR_BADARG;
    int e = commit(o);
    if (e) return e;
    std::vector<char> paused(o->cases.size(), 0);
    for (int s = 0; s < nsteps; ++s) {
        bool any = false;
        for (size_t c = 0; c < o->cases.size(); ++c) {
            Case& cs = o->cases[c];
            if (cs.done || paused[c]) continue;
            explicit_step(o, cs);
            if (cs.todo == Q2D_TODO_IO) paused[c] = 1;
            any = true;
        }
        if (!any) break;
    }
    int first = Q2D_OK;
    for (size_t c = 0; c < o->cases.size(); ++c) {
        if (out) fill_info(o->cases[c], &out[c]);
        if (!first && o->cases[c].err) first = o->cases[c].err;
    }
    return first;
}

int q2d_oracle_case_info(q2d_oracle* o, int case_id, q2d_step_info* out) {
    if (!o || !out || case_id < 0 || case_id >= (int)o->cases.size()) return Q2D_ERR_BADARG;
    fill_info(o->cases[case_id], out);
    return Q2D_OK;
}

int q2d_oracle_get_geometry(q2d_oracle* o, int block_id, double* dl, double* sur, double* fi,
                            double* fj) {
    if (!o || block_id < 0 || block_id >= (int)o->blk.size()) return Q2D_ERR_BADARG;
    int e = commit(o);
    if (e) return e;
    const Block& B = o->blk[block_id];
    if (dl) std::memcpy(dl, B.dl.data(), sizeof(double) * B.dl.size());
    if (sur)
        for (int j = 1; j <= B.nj; ++j)
            for (int i = 1; i <= B.ni; ++i) sur[(i - 1) + B.ni * (j - 1)] = B.sur[B.c(i, j)];
    if (fi) std::memcpy(fi, B.f1.data(), sizeof(double) * B.f1.size());
    if (fj) std::memcpy(fj, B.f2.data(), sizeof(double) * B.f2.size());
    return Q2D_OK;
}

void q2d_oracle_destroy(q2d_oracle* o) { delete o; }

double q2d_oracle_limiter(int limiter, double x, double y) { return rlimiter(limiter, x, y); }

double q2d_oracle_sd_tramel(double p, double p1, double p2, double p3, double p4) {
    return sd_tramel(p, p1, p2, p3, p4);
}

int q2d_oracle_shock_sensor(q2d_oracle* o, int block_id, double* beta) {
    if (!o || block_id < 0 || block_id >= (int)o->blk.size() || !beta) return Q2D_ERR_BADARG;
    int e = commit(o);
    if (e) return e;
    ghost_fill(o, o->cases[o->blk[block_id].case_id]);
    Block& B = o->blk[block_id];
    shock_sensor(B);
    std::memcpy(beta, B.beta.data(), sizeof(double) * B.beta.size());
    return Q2D_OK;
}

void q2d_oracle_riemann(int kind, const q2d_options* opt, const double* L, const double* R,
                        double nx, double ny, double* flux4) {
    Gas g;
    g.R = opt->gas_R; g.gamma = opt->gas_gamma; g.gm1 = g.gamma - 1.0;
    g.cp = g.gamma * g.R / g.gm1; g.cv = g.R / g.gm1;
    g.minf = opt->riemann_minf;
    const double aL = f_ss(g, L[3], L[0]), aR = f_ss(g, R[3], R[0]);
    const Flux4 F = riemann(kind, g, L, aL, R, aR, nx, ny);
    flux4[0] = F.r; flux4[1] = F.u; flux4[2] = F.v; flux4[3] = F.e;
}

int q2d_oracle_thermo_tab(int kind, const q2d_options* opt, int ntab, const double* h_tab, const double* cp_tab,
                          const double* L, const double* R, double nx, double ny, double* out) {
    if (!opt || ntab < 2 || !h_tab || !cp_tab || !L || !R || !out || kind < 0 || kind > Q2D_RIEMANN_LLF)
        return Q2D_ERR_BADARG;
    Gas g;
    g.R = opt->gas_R; g.gamma = opt->gas_gamma; g.gm1 = g.gamma - 1.0;
    g.cp = g.gamma * g.R / g.gm1; g.cv = g.R / g.gm1;
    g.htab = h_tab; g.cptab = cp_tab; g.ntab = ntab;
    const double aL = f_ss(g, L[3], L[0]), aR = f_ss(g, R[3], R[0]);
    const Flux4 F = riemann(kind, g, L, aL, R, aR, nx, ny);
    out[0] = F.r; out[1] = F.u; out[2] = F.v; out[3] = F.e;
    double h0l, h0r, rho_roe, u_roe, v_roe, a_roe, h0_roe;
    roe_averages(g, L[0], R[0], L[0], R[0], L[1], L[2], R[1], R[2], L[3], R[3], h0l, h0r, rho_roe, u_roe,
                 v_roe, a_roe, h0_roe);
    out[4] = aL; out[5] = aR; out[6] = a_roe; out[7] = h0_roe;
    double U[4], P[4];
    prim2cons(g, L, U);
    cons2prim(g, U, P, 0.5 * L[3] / (L[0] * g.R));   // a guess far from the answer
    out[8] = U[3]; out[9] = P[3];
    return Q2D_OK;
}

void q2d_oracle_riemann_sd(int kind, const q2d_options* opt, const double* L, const double* R,
                           double beta, double nx, double ny, double* flux4) {
    Gas g;
    g.R = opt->gas_R; g.gamma = opt->gas_gamma; g.gm1 = g.gamma - 1.0;
    g.cp = g.gamma * g.R / g.gm1; g.cv = g.R / g.gm1;
    g.minf = opt->riemann_minf;
    const double aL = f_ss(g, L[3], L[0]), aR = f_ss(g, R[3], R[0]);
    const Flux4 F = riemann(kind, g, L, aL, R, aR, nx, ny, beta);
    flux4[0] = F.r; flux4[1] = F.u; flux4[2] = F.v; flux4[3] = F.e;
}

}  // extern "C"
