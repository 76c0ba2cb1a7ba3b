// q2d_stage32.cuh — the fused RK-stage kernel of the FP32-flux / FP64-state form (sm_100a).
//
// Same work per launch as the FP64 stage kernel (q2d_kernels.cu): one RK stage for every
// running case, CTAs taking TX x TY tiles of blocks in a grid-stride loop. The precision split
// follows the form's definition: MUSCL reconstruction, limiters and the interior Riemann fluxes
// run in FP32 and the face fluxes are kept in FP32; the residual accumulation (flux
// differences), sources, RK stage combination, positivity checks, the new state and the
// residual norms are FP64. Wall (symmetry) and extrapolation boundary fluxes are FP32 like the
// interior ones; inflow and outflow records (Lib_BC_Fluxes_Inflow/Outflow.f90) are evaluated in
// FP64 from the FP64 state.
//
// Per tile there are two CTA barriers:
//   1. loads: the FP64 cell data of the tile (U^n, sur, dt, source geometry) by cp.async;
//      the stencil state of the tile and its cross-shaped 2-cell halo converted to FP32, with
//      every ghost cell (Fill_Ghost_Cell, Lib_Ghost.f90:16-299) evaluated from HBM by the thread
//      that stores it; mean cell lengths and face geometry converted to FP32;
//   2. faces: each interior face reconstructs its two states from its 4-cell stencil
//      (Lib_Reconstruction.f90:10-29: three slopes, two limited slopes) and solves the Riemann
//      problem (Convective_Flux, Lib_Convective.f90:15-82); boundary faces follow BC_Fluxes;
//   3. cells: residual in the reference's accumulation order, sources, Newstate_Conservative
//      + RK_stage + Check_And_Fix_State in FP64 and, on the last stage, the cell's next time
//      step (FP32 arithmetic) and its squared change for the residual norm.
#pragma once
#include "q2d_common.cuh"
#include "q2d_kernels.cuh"
#include "../../include/q2d_gpu.h"

namespace q2d {

// Shared-memory layout of one tile (byte offsets): FP64 cell planes, then FP32 records of 16
// bytes (one shared-memory access per cell state, face geometry or face flux) and the mean
// cell lengths of both directions as pairs.
template <int TX, int TY>
struct Tile32 {
    static constexpr int W = TX + 4, H = TY + 4, AREA = W * H;
    static constexpr int NFI = (TX + 1) * TY, NFJ = TX * (TY + 1), NF = NFI + NFJ;
    static constexpr int NC = TX * TY;
    // FP64 cell planes: 0-3 state at the start of the step, 4 sur, 5 dt, 6-7 source geometry,
    // 8-11 state
    static constexpr int NCD = 12;
    static constexpr size_t bP = sizeof(double) * NCD * NC;   // float4 [AREA]  rho, u, v, p
    // float4 [NF]: a face's geometry (nx, ny, length, packed boundary record) until its thread
    // computes the face, then its flux times length in the same slot
    static constexpr size_t bG = bP + 16 * (size_t)AREA;
    static constexpr size_t bF = bG;
    static constexpr size_t bD = bF + 16 * (size_t)NF;        // float2 [AREA]  dl(1), dl(2)
    static constexpr size_t bytes = bD + 8 * (size_t)AREA;
};

__device__ __forceinline__ float comp(const float4& q, int v) {
    return v == 0 ? q.x : (v == 1 ? q.y : (v == 2 ? q.z : q.w));
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 1/x in FP64 from the FP32 hardware reciprocal and two Newton-Raphson steps (each doubles the
// number of correct bits: 2^-22 -> 2^-44 -> below the FP64 rounding). Valid for |x| in the
// normal FP32 range, which holds for cell volumes and densities.
__device__ __forceinline__ double rcp64(double x) {
    double y = (double)rcp_approx((float)x);
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// FP32 face state with its physical flux per unit normal.
struct FS32 {
    float r, u, v, p, un;
    float Fr, Fu, Fv, Fe;
};

__device__ __forceinline__ FS32 phys32(float r, float u, float v, float p, float nx, float ny, float gf) {
    FS32 s;
    s.r = r; s.u = u; s.v = v; s.p = p;
    s.un = u * nx + v * ny;
    const float m = r * s.un;
    s.Fr = m;
    s.Fu = m * u + p * nx;
    s.Fv = m * v + p * ny;
    s.Fe = s.un * (gf * p + 0.5f * r * (u * u + v * v));
    return s;
}

// Riemann solvers in FP32 (riemann_HLLC / riemann_HLLE, Lib_Riemann_HLL.f90:34-169; riemann_LLF,
// Lib_Riemann_LF.f90:11-40): clamped Einfeldt speeds from constant-cp Roe averages, HLLC star
// states written through the jumps (S* - un_K, p* - p_K). Returns the flux per unit length.
// beta: the shock sensor the sensor-driven solvers blend by (HLLC+, HLLE++).
template <int RIEM>
__device__ __forceinline__ void riemann_f32(const FS32& L, const FS32& R, float nx, float ny, float gam,
                                            float gm1, float gf, float* F, float beta = 1.0f,
                                            const Gas* gp = nullptr) {
    if (RIEM == kRiemGeneric) {   // the run-time selected solvers: FP64 on the FP32 face states
        const double ql[4] = {L.r, L.u, L.v, L.p}, qr[4] = {R.r, R.u, R.v, R.p};
        const F4 X = riemann_generic(*gp, ql, f_ss(*gp, ql[3], ql[0]), qr, f_ss(*gp, qr[3], qr[0]), nx, ny);
        F[0] = (float)X.r; F[1] = (float)X.u; F[2] = (float)X.v; F[3] = (float)X.e;
        return;
    }
    if (RIEM == 5) {   // HLLC+ (riemann_HLLCSD, Lib_Riemann_HLL.f90:572-605)
        if (beta == 0.0f) { riemann_f32<1>(L, R, nx, ny, gam, gm1, gf, F); return; }
        if (beta >= 1.0f) { riemann_f32<0>(L, R, nx, ny, gam, gm1, gf, F); return; }
        float E[4], Cf[4];
        riemann_f32<1>(L, R, nx, ny, gam, gm1, gf, E);
        riemann_f32<0>(L, R, nx, ny, gam, gm1, gf, Cf);
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] = beta * Cf[v] + (1.0f - beta) * E[v];
        return;
    }
    const float irl = rcp_approx(L.r), irr = rcp_approx(R.r);
    const float al = sqrtf(gam * L.p * irl), ar = sqrtf(gam * R.p * irr);
    if (RIEM == 3 || RIEM == 4) {   // SLAU / SLAU2 (Lib_Riemann_SLAU.f90:10-124)
        const float sqi = L.u * L.u + L.v * L.v, sqj = R.u * R.u + R.v * R.v;
        const float aF = 0.5f * (al + ar), iaF = rcp_approx(aF);
        const float mL = L.un * iaF, mR = R.un * iaF;
        const float vbar = sqrtf(0.5f * (sqi + sqj));
        const float Mt = fminf(1.0f, vbar * iaF);
        const float Chi = (1.0f - Mt) * (1.0f - Mt);
        const float Vn = (L.r * fabsf(L.un) + R.r * fabsf(R.un)) * rcp_approx(L.r + R.r);
        const float frho = -fmaxf(fminf(mL, 0.0f), -1.0f) * fminf(fmaxf(mR, 0.0f), 1.0f);
        const float VnL = (1.0f - frho) * Vn + frho * fabsf(L.un);
        const float VnR = (1.0f - frho) * Vn + frho * fabsf(R.un);
        const float m = 0.5f * (L.r * (L.un + VnL) + R.r * (R.un - VnR) - Chi * iaF * (R.p - L.p));
        const float BL = fabsf(mL) < 1.0f ? 0.25f * (2.0f - mL) * (mL + 1.0f) * (mL + 1.0f) : (mL >= 0.0f ? 1.0f : 0.0f);
        const float BR = fabsf(mR) < 1.0f ? 0.25f * (2.0f + mR) * (mR - 1.0f) * (mR - 1.0f) : (mR >= 0.0f ? 0.0f : 1.0f);
        const float pm = 0.5f * (L.p + R.p);
        const float ph = RIEM == 4 ? pm + 0.5f * (BL - BR) * (L.p - R.p) + vbar * (BL + BR - 1.0f) * aF * 0.5f * (L.r + R.r)
                                   : pm + 0.5f * (BL - BR) * (L.p - R.p) + (1.0f - Chi) * (BL + BR - 1.0f) * pm;
        const bool up = m >= 0.0f;
        const float h0 = up ? gf * L.p * irl + 0.5f * sqi : gf * R.p * irr + 0.5f * sqj;
        F[0] = m;
        F[1] = m * (up ? L.u : R.u) + nx * ph;
        F[2] = m * (up ? L.v : R.v) + ny * ph;
        F[3] = m * h0;
        return;
    }
    if (RIEM == 2) {
        const float A = fmaxf(fmaxf(fabsf(L.un - al), fabsf(R.un - ar)), fmaxf(fabsf(L.un + al), fabsf(R.un + ar)));
        const float igm1 = 1.0f / gm1;
        const float eL = L.p * igm1 + 0.5f * L.r * (L.u * L.u + L.v * L.v);
        const float eR = R.p * igm1 + 0.5f * R.r * (R.u * R.u + R.v * R.v);
        F[0] = 0.5f * (L.Fr + R.Fr - A * (R.r - L.r));
        F[1] = 0.5f * (L.Fu + R.Fu - A * (R.r * R.u - L.r * L.u));
        F[2] = 0.5f * (L.Fv + R.Fv - A * (R.r * R.v - L.r * L.v));
        F[3] = 0.5f * (L.Fe + R.Fe - A * (eR - eL));
        return;
    }
    const float srL = sqrtf(L.r), srR = sqrtf(R.r);
    const float isr = rcp_approx(srL + srR);
    const float u_roe = (srR * R.u + srL * L.u) * isr;
    const float v_roe = (srR * R.v + srL * L.v) * isr;
    const float h0l = gf * L.p * irl + 0.5f * (L.u * L.u + L.v * L.v);
    const float h0r = gf * R.p * irr + 0.5f * (R.u * R.u + R.v * R.v);
    const float h0_roe = (srR * h0r + srL * h0l) * isr;
    const float a_roe = sqrtf(fmaxf(gm1 * (h0_roe - 0.5f * (u_roe * u_roe + v_roe * v_roe)), 0.0f));
    const float un_roe = u_roe * nx + v_roe * ny;
    const float S1 = fminf(fminf(0.0f, L.un - al), un_roe - a_roe);
    const float S4 = fmaxf(fmaxf(0.0f, R.un + ar), un_roe + a_roe);
    if (RIEM == 6) {   // HLLE++ (riemann_HLLEpp, Lib_Riemann_HLL.f90:437-533)
        const float inv = rcp_approx(S4 - S1);
        const float ps = (S4 + S1) * inv, pp = 2.0f * S4 * S1 * inv;
        const float eps = 0.3f * (fabsf(un_roe) + a_roe);
        const float v2 = un_roe - a_roe, v3 = un_roe + a_roe;
        const float l2r = fabsf(v2) <= eps ? (v2 * v2 + eps * eps) * rcp_approx(2.0f * eps) : fabsf(v2);
        const float l3r = fabsf(v3) <= eps ? (v3 * v3 + eps * eps) * rcp_approx(2.0f * eps) : fabsf(v3);
        const float l1 = beta * fabsf(un_roe) + (1.0f - beta) * fabsf(ps * un_roe - pp);
        const float l2 = beta * l2r + (1.0f - beta) * fabsf(ps * v2 - pp);
        const float l3 = beta * l3r + (1.0f - beta) * fabsf(ps * v3 - pp);
        const float rho_roe = srL * srR;
        const float dp = R.p - L.p, dun = R.un - L.un, tx = -ny, ty = nx;
        const float ia2 = rcp_approx(a_roe * a_roe);
        const float am = 0.5f * (dp - rho_roe * a_roe * dun) * ia2;
        const float ac = (R.r - L.r) - dp * ia2;
        const float as = rho_roe * ((R.u - L.u) * tx + (R.v - L.v) * ty);
        const float ap = 0.5f * (dp + rho_roe * a_roe * dun) * ia2;
        const float w1 = ac * l1, ws = as * l1, w2 = am * l2, w3 = ap * l3;
        F[0] = 0.5f * (L.Fr + R.Fr - (w1 + w2 + w3));
        F[1] = 0.5f * (L.Fu + R.Fu - (w1 * u_roe + ws * tx + w2 * (u_roe - a_roe * nx) + w3 * (u_roe + a_roe * nx)));
        F[2] = 0.5f * (L.Fv + R.Fv - (w1 * v_roe + ws * ty + w2 * (v_roe - a_roe * ny) + w3 * (v_roe + a_roe * ny)));
        F[3] = 0.5f * (L.Fe + R.Fe - (w1 * 0.5f * (u_roe * u_roe + v_roe * v_roe) + ws * (u_roe * tx + v_roe * ty) +
                                      w2 * (h0_roe - a_roe * un_roe) + w3 * (h0_roe + a_roe * un_roe)));
        return;
    }
    if (RIEM == 1) {
        const float inv = rcp_approx(S4 - S1);
        const float c = S1 * S4;
        const float eL = L.r * h0l - L.p, eR = R.r * h0r - R.p;
        F[0] = (S4 * L.Fr - S1 * R.Fr + c * (R.r - L.r)) * inv;
        F[1] = (S4 * L.Fu - S1 * R.Fu + c * (R.r * R.u - L.r * L.u)) * inv;
        F[2] = (S4 * L.Fv - S1 * R.Fv + c * (R.r * R.v - L.r * L.v)) * inv;
        F[3] = (S4 * L.Fe - S1 * R.Fe + c * (eR - eL)) * inv;
        return;
    }
    if (S1 >= 0.0f) { F[0] = L.Fr; F[1] = L.Fu; F[2] = L.Fv; F[3] = L.Fe; return; }
    const float D = L.r * (S1 - L.un) - R.r * (S4 - R.un);
    const float sm_unl = ((R.p - L.p) - R.r * (S4 - R.un) * (R.un - L.un)) * rcp_approx(D);   // S* - un_L
    const float Sstar = L.un + sm_unl;
    if (Sstar >= 0.0f) {
        const float inv = rcp_approx(S1 - Sstar);
        const float q = sm_unl * inv;
        const float dps = L.r * (S1 - L.un) * sm_unl;                               // p* - p_L
        const float e0l = h0l - L.p * irl;
        F[0] = L.Fr + S1 * (L.r * q);
        F[1] = L.Fu + S1 * (L.r * L.u * q + dps * nx * inv);
        F[2] = L.Fv + S1 * (L.r * L.v * q + dps * ny * inv);
        F[3] = L.Fe + S1 * (L.r * e0l * q + (dps * Sstar + L.p * sm_unl) * inv);
        return;
    }
    if (S4 > 0.0f) {
        const float inv = rcp_approx(S4 - Sstar);
        const float sm_unr = sm_unl - (R.un - L.un);                                // S* - un_R
        const float q = sm_unr * inv;
        const float dps = R.r * (S4 - R.un) * sm_unr;                               // p* - p_R
        const float e0r = h0r - R.p * irr;
        F[0] = R.Fr + S4 * (R.r * q);
        F[1] = R.Fu + S4 * (R.r * R.u * q + dps * nx * inv);
        F[2] = R.Fv + S4 * (R.r * R.v * q + dps * ny * inv);
        F[3] = R.Fe + S4 * (R.r * e0r * q + (dps * Sstar + R.p * sm_unr) * inv);
        return;
    }
    F[0] = R.Fr; F[1] = R.Fu; F[2] = R.Fv; F[3] = R.Fe;
}

// One interior face: stencil cells m (= L-1), L, R, p (= R+1) at shared positions base + k*step;
// dlp is the cell-length pair array viewed as floats, offset to the face's direction.
// beta_l: the shock sensor scaling both limited slopes (1 without MUSCL-SD; Lib_Convective.f90:
// 40-47); beta_r: the sensor the Riemann solver receives (:62-64)
template <int RIEM, int LIM>
__device__ __forceinline__ bool face32(const float4* sP, const float* dlp, int base, int step, float nx,
                                      float ny, float len, float gam, float gm1, float gf, float beta_l,
                                      float beta_r, float* out, const Gas& g) {
    const float dm = dlp[2 * base], d0 = dlp[2 * (base + step)], d1 = dlp[2 * (base + 2 * step)],
                d2 = dlp[2 * (base + 3 * step)];
    const float il0 = rcp_approx(0.5f * (dm + d0));
    const float il1 = rcp_approx(0.5f * (d0 + d1));
    const float il2 = rcp_approx(0.5f * (d1 + d2));
    const float lm = 0.5f * d0, lp = 0.5f * d1;
    float QL[4], QR[4];
    const float4 Cm = sP[base], C0 = sP[base + step], C1 = sP[base + 2 * step], C2 = sP[base + 3 * step];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float qm = comp(Cm, v), q0 = comp(C0, v), q1 = comp(C1, v), q2 = comp(C2, v);
        const float s0 = (q0 - qm) * il0, s1 = (q1 - q0) * il1, s2 = (q2 - q1) * il2;
        QL[v] = q0 + beta_l * lim32<LIM>(s1, s0) * lm;
        QR[v] = q1 - beta_l * lim32<LIM>(s2, s1) * lp;
    }
    const bool ok = QL[0] > 0.0f && QL[3] > 0.0f && QR[0] > 0.0f && QR[3] > 0.0f;
    const FS32 L = phys32(QL[0], QL[1], QL[2], QL[3], nx, ny, gf);
    const FS32 R = phys32(QR[0], QR[1], QR[2], QR[3], nx, ny, gf);
    float F[4];
    riemann_f32<RIEM>(L, R, nx, ny, gam, gm1, gf, F, beta_r, &g);
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v] = F[v] * len;
    return ok;
}

// SD_Tramel (Lib_Shock_Detector.f90:14-38) of the tile cell at slot c, from the FP32 pressures of
// its cross stencil.
template <int W>
__device__ __forceinline__ float sd_cell32(const float4* sP, int c) {
    return sd_tramel32(sP[c].w, sP[c - 1].w, sP[c + 1].w, sP[c - W].w, sP[c + W].w);
}

// Interior faces of a tile (i faces, then j faces); boundary positions are left to the
// boundary-face loop. With MUSCL-SD a face takes the sensor of its left / lower cell
// (Mod_Fluxes.f90:140-204).
template <int RIEM, int LIM, int NT, int TX, int TY, bool SD>
__device__ __forceinline__ void interior_faces32(const StageArgs& a, const DBlock& B, CaseState* cs, int i0,
                                                 int j0, const float4* sP, const float* sD, const float4* sG,
                                                 float4* sF, float gam, float gm1, float gf) {
    using L = Tile32<TX, TY>;
    constexpr int W = L::W, NFI = L::NFI, NF = L::NF;
    const int ni = B.ni, nj = B.nj;
    for (int f = threadIdx.x; f < NF; f += NT) {
        int base, step, pos, lenn, k, kmax, ii, jj;
        const float* dlp;
        if (f < NFI) {
            const int row = f / (TX + 1), col = f - row * (TX + 1);
            pos = i0 + col; lenn = ni; k = j0 + row; kmax = nj;
            base = (row + 2) * W + col; step = 1; dlp = sD;
            ii = pos; jj = k + 1;
        } else {
            const int ff = f - NFI;
            const int row = ff / TX, col = ff - row * TX;
            pos = j0 + row; lenn = nj; k = i0 + col; kmax = ni;
            base = row * W + col + 2; step = W; dlp = sD + 1;
            ii = k + 1; jj = pos;
        }
        if (k >= kmax || pos <= 0 || pos >= lenn) continue;
        float out[4];
        const float4 gq = sG[f];
        const float beta = SD ? sd_cell32<W>(sP, base + step) : 1.0f;
        const bool ok = face32<RIEM, LIM>(sP, dlp, base, step, gq.x, gq.y, gq.z, gam, gm1, gf, a.sd ? beta : 1.0f,
                                          beta, out, a.gas);
        if (!ok) record_error(cs, 4, B.local_b, ii, jj, a.irk);
        sF[f] = make_float4(out[0], out[1], out[2], out[3]);
    }
}

template <int RIEM>
__device__ __forceinline__ bool face32_lim(int lim, const float4* sP, const float* dlp, int base, int step,
                                          float nx, float ny, float len, float gam, float gm1, float gf,
                                          float beta_l, float beta_r, float* out, const Gas& g) {
    switch (lim) {
        case 0: return face32<RIEM, 0>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        case 1: return face32<RIEM, 1>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        case 2: return face32<RIEM, 2>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        case 3: return face32<RIEM, 3>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        case 4: return face32<RIEM, 4>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        case 5: return face32<RIEM, 5>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
        default: return face32<RIEM, 6>(sP, dlp, base, step, nx, ny, len, gam, gm1, gf, beta_l, beta_r, out, g);
    }
}

// Boundary faces of the FP32-flux form in FP32 (the FP64 restatements are in q2d_common.cuh).
// BC_Symmetry_Eul (Lib_BC_Fluxes_Symmetry.f90:28-124): mirrored ghost, limited slope of the
// boundary cell, Riemann problem between the face state and its mirror; momentum flux only.
template <int RIEM, int LIM>
__device__ __forceinline__ void bc_symmetry32(int Fm, const float* B, const float* I, float dlb, float dli,
                                              float nx, float ny, float len, float gam, float gm1, float gf,
                                              float* out, const Gas& g) {
    const bool minside = (Fm & 1) != 0;   // faces 1 and 3
    const float bd = 0.5f * dlb, id = 0.5f * dli;
    const float un = B[1] * nx + B[2] * ny;
    const float G[4] = {B[0], B[1] - 2.0f * un * nx, B[2] - 2.0f * un * ny, B[3]};
    const float i12 = rcp_approx(minside ? 2.0f * bd : bd + id);
    const float i23 = rcp_approx(minside ? bd + id : 2.0f * bd);
    const float dist = minside ? -bd : bd;
    float Fc[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float P1 = minside ? G[v] : I[v], P3 = minside ? I[v] : G[v];
        Fc[v] = B[v] + lim32<LIM>((P3 - B[v]) * i23, (B[v] - P1) * i12) * dist;
    }
    const float Un = Fc[1] * nx + Fc[2] * ny;
    const float vtx = Fc[1] - Un * nx, vty = Fc[2] - Un * ny;
    const float Un1 = minside ? -Un : Un;
    const FS32 L = phys32(Fc[0], Un1 * nx + vtx, Un1 * ny + vty, Fc[3], nx, ny, gf);
    const FS32 R = phys32(Fc[0], -Un1 * nx + vtx, -Un1 * ny + vty, Fc[3], nx, ny, gf);
    float F[4];
    riemann_f32<RIEM>(L, R, nx, ny, gam, gm1, gf, F, 1.0f, &g);
    out[0] = 0.0f;
    out[1] = F[1] * len;
    out[2] = F[2] * len;
    out[3] = 0.0f;
}

// BC_Extrapolation (Lib_BC_Fluxes_Extrapolation.f90:18-49): exact flux of the boundary cell.
__device__ __forceinline__ void bc_extrapolation32(const float* B, float nx, float ny, float len, float gf,
                                                   float* out) {
    const float m = B[0] * (B[1] * nx + B[2] * ny) * len;
    out[0] = m;
    out[1] = m * B[1] + B[3] * len * nx;
    out[2] = m * B[2] + B[3] * len * ny;
    out[3] = m * (gf * B[3] * rcp_approx(B[0]) + 0.5f * (B[1] * B[1] + B[2] * B[2]));
}

// BC_Inlet_StagnCond + Stagn_Inflow (Lib_BC_Fluxes_Inflow.f90:64-120, 412-483) in FP32 for the
// common case: inflow through the face and a discriminant clearly above zero, where the
// reference takes the first iterate (p0 itself). The face state is the isentropic state on the
// outgoing Riemann invariant a + sign (gamma-1)/2 Un of the boundary cell, at the flow angle of
// the record ('normal': the face normal, so that tan(alpha) = n1 / n0). Returns 0 with the
// flux in out, 1 when the flow leaves through the inlet (the symmetry flux applies, :176-227),
// 2 when the discriminant is negative or too close to zero for FP32 to decide (the FP64
// routine then runs the reference's relaxation of p0).
__device__ __forceinline__ int bc_stagnation32(int Fm, const float* B, float n0, float n1, float len,
                                               float gam, float R, const BCParam& bp, float* out) {
    const float sgn = (Fm & 1) ? -1.0f : 1.0f;
    const float Un = B[1] * n0 + B[2] * n1;
    if (sgn * Un >= 0.0f) return 1;
    const float gh = 0.5f * (gam - 1.0f);
    const float Sound = sqrtf(gam * B[3] * rcp_approx(B[0]));
    const float Riem = Sound + sgn * gh * Un;
    const float ta = bp.alpha >= 0.5 * DBL_MAX ? n1 * rcp_approx(n0 + 1e-20f) : tanf((float)bp.alpha);
    const float t0 = (float)bp.t0, t1 = (float)bp.t1;
    const float E1 = -(n1 - n0 * ta) * rcp_approx(t1 - t0 * ta);
    const float Sound0 = sqrtf(gam * R * (float)bp.T0);
    const float CoefD = (1.0f + E1 * E1) * gh;
    const float p0 = (float)bp.p0;
    const float ss = Sound * rcp_approx(Sound0);
    const float CoefC = __powf(p0 * rcp_approx(B[3]), (gam - 1.0f) * rcp_approx(gam)) * (ss * ss);
    const float YA = gh * gh + CoefC * CoefD;
    const float YB = sgn * Riem * gh;
    const float R2 = Riem * Riem, C2 = CoefC * (Sound0 * Sound0);
    const float YC = R2 - C2;
    const float Discr = YB * YB - YA * YC;
    // FP32 error of Discr: a few ulps of its largest terms, plus the reference's 1e-2 band
    const float tol = 1e-5f * (YB * YB + YA * (R2 + C2)) + 2e-2f;
    if (!(Discr > tol)) return 2;
    const float Un3 = (YB + copysignf(1.0f, Un) * sqrtf(Discr)) * rcp_approx(YA);
    const float Sound3 = sqrtf(Sound0 * Sound0 - CoefD * (Un3 * Un3));
    const float p3 = p0 * __powf(Sound3 * rcp_approx(Sound0), 2.0f * gam * rcp_approx(gam - 1.0f));
    const float Ut3 = Un3 * E1;
    const float rho = gam * p3 * rcp_approx(Sound3 * Sound3);
    const float fu = Un3 * n0 + Ut3 * t0, fv = Un3 * n1 + Ut3 * t1;
    const float H = gam * rcp_approx(gam - 1.0f) * p3 * rcp_approx(rho);   // cp T
    const float m = rho * Un3 * len;
    out[0] = m;
    out[1] = m * fu + p3 * len * n0;
    out[2] = m * fv + p3 * len * n1;
    out[3] = m * (0.5f * (fu * fu + fv * fv) + H);
    return 0;
}

template <int RIEM>
__device__ __forceinline__ void bc_symmetry32_lim(int lim, int Fm, const float* B, const float* I, float dlb,
                                                  float dli, float nx, float ny, float len, float gam,
                                                  float gm1, float gf, float* out, const Gas& g) {
    switch (lim) {
        case 0: bc_symmetry32<RIEM, 0>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        case 1: bc_symmetry32<RIEM, 1>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        case 2: bc_symmetry32<RIEM, 2>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        case 3: bc_symmetry32<RIEM, 3>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        case 4: bc_symmetry32<RIEM, 4>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        case 5: bc_symmetry32<RIEM, 5>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
        default: bc_symmetry32<RIEM, 6>(Fm, B, I, dlb, dli, nx, ny, len, gam, gm1, gf, out, g); break;
    }
}

// Compute_dt body for one cell (Mod_dt.f90:59-104, model 0) in FP32: the CFL time step of each
// grid direction, dl / (|V.e| + a), the smaller of the two (one direction when ndir == 1).
__device__ __forceinline__ float cell_dt32(float rho, float u, float v, float p, float gam, float cfl, int ndir,
                                           float dli, float dlj, float ei0, float ei1, float ej0, float ej1) {
    const float snd = sqrtf(gam * p * rcp_approx(rho));
    float dtmin = fminf(1e8f, dli * rcp_approx(fabsf(u * ei0 + v * ei1) + snd) * cfl);
    if (ndir == 2) dtmin = fminf(dtmin, dlj * rcp_approx(fabsf(u * ej0 + v * ej1) + snd) * cfl);
    return dtmin;
}

// Boundary record of a face packed into one 32-bit word: the BC type as a 3-bit code and its
// BC parameter index + 1 above it.
__device__ __forceinline__ float pack_record(int type, int param) {
    const unsigned code = type == 101 ? 1u : type == 300 ? 2u : type == 400 ? 3u : type == 401 ? 4u
                        : type == 405 ? 5u : type == 406 ? 6u : type == 0 ? 7u : 0u;
    return __uint_as_float(((unsigned)(param + 1) << 3) | code);
}

__device__ __forceinline__ void unpack_record(float w, int& type, int& param) {
    const unsigned u = __float_as_uint(w);
    static constexpr int kTypes[8] = {-1, 101, 300, 400, 401, 405, 406, 0};
    type = kTypes[u & 7u];
    param = (int)(u >> 3) - 1;
}

// Boundary face t of a tile (nl faces on block face 1, nr on face 2, nb on face 3, then face 4):
// its block face Fm, its cell index k along that face and its slot f among the tile's faces.
template <int TX>
__device__ __forceinline__ void boundary_face_slot(int t, int nl, int nr, int nb, int i0, int j0, int ni,
                                                   int nj, int NFI, int& Fm, int& k, int& f) {
    if (t < nl) {
        Fm = 1; k = j0 + t; f = t * (TX + 1);
    } else if (t < nl + nr) {
        const int u = t - nl;
        Fm = 2; k = j0 + u; f = u * (TX + 1) + (ni - i0);
    } else if (t < nl + nr + nb) {
        const int u = t - nl - nr;
        Fm = 3; k = i0 + u; f = NFI + u;
    } else {
        const int u = t - nl - nr - nb;
        Fm = 4; k = i0 + u; f = NFI + (nj - j0) * TX + u;
    }
}

template <int RIEM, int TX, int TY, int NT, int MB, bool SD>
__global__ void __launch_bounds__(NT, MB) stage32_kernel(const StageArgs a) {
    using L = Tile32<TX, TY>;
    constexpr int W = L::W, AREA = L::AREA, NFI = L::NFI, NF = L::NF, NC = L::NC;
    static_assert(L::bG % 16 == 0 && L::bF % 16 == 0 && L::bD % 8 == 0, "shared layout alignment");
    static_assert(L::bF == L::bG, "a face's flux replaces its geometry in the same slot");
    extern __shared__ double smem[];
    double* sC = smem;
    unsigned char* sb = reinterpret_cast<unsigned char*>(smem);
    float4* sP = reinterpret_cast<float4*>(sb + L::bP);
    float4* sG = reinterpret_cast<float4*>(sb + L::bG);
    float4* sF = reinterpret_cast<float4*>(sb + L::bF);
    float2* sD2 = reinterpret_cast<float2*>(sb + L::bD);
    const float* sD = reinterpret_cast<const float*>(sD2);
    __shared__ double red[(NT / 32) * 5];
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    if (a.part_stride != NT / 32) {
        // the partials are laid out one set per warp: a host / kernel mismatch of that layout
        // fails every case of the launch with Q2D_ERR_BADARG instead of skipping the stage
        if (tid == 0)
            for (int it = blockIdx.x; it < a.n_items; it += gridDim.x)
                record_error(&a.cstate[__ldg(&a.items[it].case_id)], Q2D_ERR_BADARG, -1, -1, -1, a.irk);
        return;
    }
    const Gas& g = a.gas;
    const float gam = (float)g.gamma, gm1 = (float)g.gm1, gf = (float)g.gfac;

    // Work-item descriptors (item, block, case status), double-buffered in shared memory: warp 0
    // fetches the next item's while the CTA works on the current one.
    __shared__ WorkItem sW[2];
    __shared__ DBlock sBk[2];
    __shared__ int sSt[2];
    static_assert(sizeof(WorkItem) == 24 && sizeof(DBlock) % 4 == 0 && sizeof(DBlock) <= 128, "descriptor words");
    constexpr int NWW = (int)(sizeof(WorkItem) / 4), NBW = (int)(sizeof(DBlock) / 4);
    const int lane = tid & 31;
    const bool w0 = tid < 32;
    if (w0 && blockIdx.x < a.n_items) {
        const int wv = lane < NWW ? __ldg(reinterpret_cast<const int*>(a.items + blockIdx.x) + lane) : 0;
        const int blk = __shfl_sync(0xffffffffu, wv, 0), cid = __shfl_sync(0xffffffffu, wv, 3);
        const int bv = lane < NBW ? __ldg(reinterpret_cast<const int*>(a.blocks + blk) + lane) : 0;
        if (lane < NWW) reinterpret_cast<int*>(&sW[0])[lane] = wv;
        if (lane < NBW) reinterpret_cast<int*>(&sBk[0])[lane] = bv;
        if (lane == 0) sSt[0] = __ldcg(&a.cstate[cid].status);
    }
    __syncthreads();
    int cur = 0;
    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x, cur ^= 1) {
        const int nit = it + gridDim.x;
        const bool pre = w0 && nit < a.n_items;
        int pw = 0, pb = 0, ps = 0;   // the next item's descriptor words held by warp 0
        if (pre && lane < NWW) pw = __ldg(reinterpret_cast<const int*>(a.items + nit) + lane);
        const WorkItem w = sW[cur];
        const DBlock B = sBk[cur];
        CaseState* cs = &a.cstate[w.case_id];
        if (sSt[cur] != kStatus_Running) {   // uniform over the CTA: finish the prefetch, next item
            if (pre) {
                const int blk = __shfl_sync(0xffffffffu, pw, 0), cid = __shfl_sync(0xffffffffu, pw, 3);
                pb = lane < NBW ? __ldg(reinterpret_cast<const int*>(a.blocks + blk) + lane) : 0;
                if (lane < NWW) reinterpret_cast<int*>(&sW[cur ^ 1])[lane] = pw;
                if (lane < NBW) reinterpret_cast<int*>(&sBk[cur ^ 1])[lane] = pb;
                if (lane == 0) sSt[cur ^ 1] = __ldcg(&a.cstate[cid].status);
            }
            __syncthreads();
            continue;
        }
        const int ni = B.ni, nj = B.nj, i0 = w.i0, j0 = w.j0;
        const double* Pin = a.Pin + B.oc;
        const long long pc = B.pc;
        const double* scb = a.sc + 2 * B.oc;
        const int ndir = a.cases[w.case_id].ndir;
        const bool dt_here = a.dt_first && a.first;   // this stage computes the local time steps

        const int irs = a.irs_mode;
        if (irs == 2) {   // update from the smoothed residual: the tile's own cells only
            for (int k = tid; k < NC; k += NT) {
                const int row = k / TX, col = k - row * TX;
                const int ii = i0 + col, jj = j0 + row;
                if (ii >= ni || jj >= nj) continue;
                const long long cg = (long long)jj * ni + ii;
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    cp_async8(sC + (8 + v) * NC + k, Pin + v * pc + cg);
                    cp_async8(sC + v * NC + k, a.PO + B.oc + v * pc + cg);
                    cp_async8(sC + (4 + v) * NC + k, a.Rin + B.oc + v * pc + cg);
                }
                if (a.last && !a.dt_first) {   // cell lengths of the next step's time step
                    const float2* dsrc = reinterpret_cast<const float2*>(a.dl32 + B.og) +
                                         (long long)(jj + 2) * (ni + 4) + (ii + 2);
                    sD2[(row + 2) * W + (col + 2)] = __ldg(dsrc);
                }
            }
        } else {
            // ---- 1. loads ------------------------------------------------------------------------
            for (int k = tid; k < NC; k += NT) {   // FP64 cell data, asynchronous
                const int row = k / TX, col = k - row * TX;
                const int ii = i0 + col, jj = j0 + row;
                if (ii >= ni || jj >= nj) continue;
                const long long cg = (long long)jj * ni + ii;
                if (!a.first) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) cp_async8(sC + v * NC + k, a.PO + B.oc + v * pc + cg);
                } else if (dt_here) {   // the dt directions, into the planes U^n leaves free in stage 1
                    cp_async8(sC + k, scb + 2 * pc + cg);
                    cp_async8(sC + NC + k, scb + 3 * pc + cg);
                    if (ndir == 2) {
                        cp_async8(sC + 2 * NC + k, scb + 4 * pc + cg);
                        cp_async8(sC + 3 * NC + k, scb + 5 * pc + cg);
                    }
                }
                cp_async8(sC + 4 * NC + k, scb + cg);                                 // sur
                if (!a.time_accurate && !dt_here) cp_async8(sC + 5 * NC + k, scb + pc + cg);   // dt
                if (a.source) {
                    cp_async8(sC + 6 * NC + k, scb + 6 * pc + cg);
                    if (a.source == 2) cp_async8(sC + 7 * NC + k, scb + 7 * pc + cg);
                }
            }
            // face geometry and the state / lengths of the cross-shaped halo: branch-free address
            // selection so that every load of a thread is in flight before the first use
            const float4* gi4 = a.fi4 + B.ofi / 2;
            const float4* gj4 = a.fj4 + B.ofj / 2;
#pragma unroll
            for (int u = 0; u < (NF + NT - 1) / NT; ++u) {
                const int f = tid + u * NT;
                bool ok;
                const float4* src;
                const EdgeRec* er = a.edges;   // the face's boundary record, if it is on the block's edge
                bool edge;
                if (f < NFI) {
                    const int row = f / (TX + 1), col = f - row * (TX + 1);
                    const int jj = j0 + row, F = i0 + col;
                    ok = jj < nj && F <= ni;
                    src = gi4 + (ok ? (long long)jj * (ni + 1) + F : 0);
                    edge = ok && (F == 0 || F == ni);
                    if (edge) er += B.eo[F == 0 ? 0 : 1] + jj;
                } else {
                    const int ff = f - NFI;
                    const int row = ff / TX, col = ff - row * TX;
                    const int ii = i0 + col, G = j0 + row;
                    ok = f < NF && ii < ni && G <= nj;
                    src = gj4 + (ok ? (long long)G * ni + ii : 0);
                    edge = ok && (G == 0 || G == nj);
                    if (edge) er += B.eo[G == 0 ? 2 : 3] + ii;
                }
                float4 gq = __ldg(src);
                if (edge) gq.w = pack_record(__ldg(&er->type), __ldg(&er->param));
                if (ok) sG[f] = gq;
            }
            bool ghosts = false;   // the tile's halo reaches a ghost layer: second pass below
#pragma unroll
            for (int u = 0; u < (AREA + NT - 1) / NT; ++u) {
                const int idx = tid + u * NT;
                const int r = idx / W, c = idx - r * W;
                const int ii = i0 - 2 + c, jj = j0 - 2 + r;
                const bool cross = idx < AREA && !((r < 2 || r >= TY + 2) && (c < 2 || c >= TX + 2));
                const bool inI = ii >= 0 && ii < ni, inJ = jj >= 0 && jj < nj;
                const bool inner = cross && inI && inJ;
                const bool indl = cross && ii >= -2 && ii <= ni + 1 && jj >= -2 && jj <= nj + 1;
                const double* src = Pin + (inner ? (long long)jj * ni + ii : 0);
                const float2* dsrc = reinterpret_cast<const float2*>(a.dl32 + B.og) +
                                     (indl ? (long long)(jj + 2) * (ni + 4) + (ii + 2) : 0);
                const double q0 = __ldg(src), q1 = __ldg(src + pc), q2 = __ldg(src + 2 * pc), q3 = __ldg(src + 3 * pc);
                const float2 d01 = __ldg(dsrc);
                if (indl) sD2[idx] = d01;
                if (inner) sP[idx] = make_float4((float)q0, (float)q1, (float)q2, (float)q3);
                if (inner && r >= 2 && r < TY + 2 && c >= 2 && c < TX + 2) {   // the tile's own cells, FP64
                    const int kk = (r - 2) * TX + (c - 2);
                    sC[8 * NC + kk] = q0; sC[9 * NC + kk] = q1; sC[10 * NC + kk] = q2; sC[11 * NC + kk] = q3;
                }
                // A ghost a face stencil of the tile reads: one of the two ghost layers, an i-ghost in
                // a tile row or a j-ghost in a tile column (the boundary cell and its two inward
                // neighbours are then in the same row or column of the tile and its halo). Its record
                // type and boundary-face normal are parked in its own slot until the second pass.
                const bool ghost = cross && inI != inJ && (!inI ? (r >= 2 && r < TY + 2) : (c >= 2 && c < TX + 2)) &&
                                   ii >= -2 && ii <= ni + 1 && jj >= -2 && jj <= nj + 1;
                if (ghost) {
                    int f, k, bi, bj;
                    if (!inI) { f = ii < 0 ? 1 : 2; k = jj; bi = ii < 0 ? 0 : ni - 1; bj = jj; }
                    else { f = jj < 0 ? 3 : 4; k = ii; bi = ii; bj = jj < 0 ? 0 : nj - 1; }
                    const int type = __ldg(&a.edges[B.eo[f - 1] + k].type);
                    const float4 gq = f <= 2 ? __ldg(gi4 + (long long)bj * (ni + 1) + (f == 1 ? 0 : ni))
                                             : __ldg(gj4 + (long long)(f == 3 ? 0 : nj) * ni + bi);
                    sP[idx] = make_float4(__int_as_float(type), gq.x, gq.y, 0.0f);
                    ghosts = true;
                }
            }
            if (SD && tid < 3) {
                // pressures the sensor of the halo column / row on the tile's left / lower faces
                // reads outside the cross the loads above fill: the corner (i0-1, j0-1), and
                // (i0-1, min(j0+TY, nj)) / (min(i0+TX, ni), j0-1), a corner or, on a ragged tile, a
                // ghost beside the cross
                const int ii = tid == 1 ? min(i0 + TX, ni) : i0 - 1;
                const int jj = tid == 2 ? min(j0 + TY, nj) : j0 - 1;
                const bool need = tid == 0 ? (i0 > 0 || j0 > 0) : (tid == 1 ? j0 > 0 : i0 > 0);
                if (need) {
                    float p;
                    if (ii >= 0 && ii < ni && jj >= 0 && jj < nj) {
                        p = (float)__ldg(Pin + 3 * pc + (long long)jj * ni + ii);
                    } else {
                        double qd[4] = {0.0, 0.0, 0.0, 0.0};
                        ghost_value(a, B, ii, jj, qd);
                        p = (float)qd[3];
                    }
                    sP[(jj - j0 + 2) * W + (ii - i0 + 2)] = make_float4(0.0f, 0.0f, 0.0f, p);
                }
            }
            if (__syncthreads_or(ghosts)) {
                // ghost cells (Fill_Ghost_Cell, Lib_Ghost.f90:16-299) from the tile's FP32 state:
                // symmetry mirrors the boundary cell's velocity about the face normal (:163-196),
                // types 0 and 401-406 copy it (Ghost_ZG_Extrapolate, :199-219), the rest extrapolate
                // quadratically (Ghost_Extrapolate, :270-299); connection ghosts copy the donor
                // block's cells (Ghost_Connection, :143-160) from HBM
#pragma unroll 1
                for (int u = 0; u < (AREA + NT - 1) / NT; ++u) {
                    const int idx = tid + u * NT;
                    const int r = idx / W, c = idx - r * W;
                    const int ii = i0 - 2 + c, jj = j0 - 2 + r;
                    const bool inI = ii >= 0 && ii < ni, inJ = jj >= 0 && jj < nj;
                    if (idx >= AREA || inI == inJ || !(!inI ? (r >= 2 && r < TY + 2) : (c >= 2 && c < TX + 2)) ||
                        ii < -2 || ii > ni + 1 || jj < -2 || jj > nj + 1)
                        continue;
                    int gd, bi, bj, s1, nn;
                    if (!inI) {
                        gd = ii < 0 ? -ii : ii - ni + 1; bi = ii < 0 ? 0 : ni - 1; bj = jj;
                        s1 = ii < 0 ? 1 : -1; nn = ni;
                    } else {
                        gd = jj < 0 ? -jj : jj - nj + 1; bi = ii; bj = jj < 0 ? 0 : nj - 1;
                        s1 = jj < 0 ? W : -W; nn = nj;
                    }
                    const float4 park = sP[idx];
                    const int type = __float_as_int(park.x);
                    float4 q;
                    if (type == 101) {
                        double qd[4] = {0.0, 0.0, 0.0, 0.0};
                        ghost_value(a, B, ii, jj, qd);
                        q = make_float4((float)qd[0], (float)qd[1], (float)qd[2], (float)qd[3]);
                    } else {
                        const int sb = (bj - j0 + 2) * W + (bi - i0 + 2);
                        const int d1 = nn >= 2 ? s1 : 0, d2 = nn >= 3 ? 2 * s1 : d1;
                        const float4 b = sP[sb], c1 = sP[sb + d1], c2 = sP[sb + d2];
                        if (type == 300) {
                            const float nx = park.y, ny = park.z;
                            const float un = b.y * nx + b.z * ny;
                            q = make_float4(b.x, b.y - 2.0f * un * nx, b.z - 2.0f * un * ny, b.w);
                        } else if (type == 0 || type == 401 || type == 405 || type == 406 || type < 0) {
                            q = b;
                        } else {
                            const float4 g1 = make_float4(3.0f * b.x - 3.0f * c1.x + c2.x, 3.0f * b.y - 3.0f * c1.y + c2.y,
                                                          3.0f * b.z - 3.0f * c1.z + c2.z, 3.0f * b.w - 3.0f * c1.w + c2.w);
                            q = gd == 1 ? g1
                                        : make_float4(3.0f * g1.x - 3.0f * b.x + c1.x, 3.0f * g1.y - 3.0f * b.y + c1.y,
                                                      3.0f * g1.z - 3.0f * b.z + c1.z, 3.0f * g1.w - 3.0f * b.w + c1.w);
                        }
                    }
                    sP[idx] = q;
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (pre) {   // next descriptor: block record and case status (the item arrived meanwhile)
            const int blk = __shfl_sync(0xffffffffu, pw, 0), cid = __shfl_sync(0xffffffffu, pw, 3);
            pb = lane < NBW ? __ldg(reinterpret_cast<const int*>(a.blocks + blk) + lane) : 0;
            ps = lane == 0 ? __ldcg(&a.cstate[cid].status) : 0;
        }

        if (irs != 2) {
            // ---- 2. face fluxes ------------------------------------------------------------------
            switch (a.limiter) {
                case 0: interior_faces32<RIEM, 0, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                case 1: interior_faces32<RIEM, 1, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                case 2: interior_faces32<RIEM, 2, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                case 3: interior_faces32<RIEM, 3, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                case 4: interior_faces32<RIEM, 4, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                case 5: interior_faces32<RIEM, 5, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
                default: interior_faces32<RIEM, 6, NT, TX, TY, SD>(a, B, cs, i0, j0, sP, sD, sG, sF, gam, gm1, gf); break;
            }
            {   // boundary faces (BC_Fluxes, Mod_BC_Fluxes.f90:79-269), on the threads with the fewest
                // interior faces (the highest thread indices)
                const int nrow = min(TY, nj - j0), ncol = min(TX, ni - i0);
                const int nl = (i0 == 0) ? nrow : 0;
                const int nr = (i0 + TX >= ni) ? nrow : 0;
                const int nb = (j0 == 0) ? ncol : 0;
                const int nt = (j0 + TY >= nj) ? ncol : 0;
                for (int t = NT - 1 - tid; t < nl + nr + nb + nt; t += NT) {
                    int Fm, k, f;
                    boundary_face_slot<TX>(t, nl, nr, nb, i0, j0, ni, nj, NFI, Fm, k, f);
                    const int bi = Fm == 1 ? 0 : (Fm == 2 ? ni - 1 : k), bj = Fm == 3 ? 0 : (Fm == 4 ? nj - 1 : k);
                    const int di = Fm == 1 ? 1 : (Fm == 2 ? -1 : 0), dj = Fm == 3 ? 1 : (Fm == 4 ? -1 : 0);
                    struct { int type, param; } e;   // the record packed with the face geometry
                    const float4 gq = sG[f];
                    unpack_record(gq.w, e.type, e.param);
                    const int cb = (bj - j0 + 2) * W + (bi - i0 + 2);     // boundary cell
                    const int ci = cb + dj * W + di;                       // its inward neighbour
                    const float* dlp = Fm <= 2 ? sD : sD + 1;
                    const float nx = gq.x, ny = gq.y, ln = gq.z;
                    float X[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    if (e.type == 101) {   // BC_Connection_Eul: the interior scheme on the ghost stencil
                        const int step = Fm <= 2 ? 1 : W;
                        const int base = (Fm == 1 || Fm == 3) ? cb - 2 * step : cb - step;
                        // the sensor of the boundary cell (beta_ = blk%beta(Im,Jm))
                        const float beta = SD ? sd_cell32<W>(sP, cb) : 1.0f;
                        const bool ok = face32_lim<RIEM>(a.limiter, sP, dlp, base, step, nx, ny, ln, gam, gm1, gf,
                                                         a.sd ? beta : 1.0f, beta, X, g);
                        if (!ok) record_error(cs, 4, B.local_b, bi + 1, bj + 1, a.irk);
                    } else if (e.type == 300 || e.type == 400) {
                        const float4 Bc = sP[cb], Ic = sP[ci];
                        const float Bq[4] = {Bc.x, Bc.y, Bc.z, Bc.w}, Iq[4] = {Ic.x, Ic.y, Ic.z, Ic.w};
                        if (e.type == 300)
                            bc_symmetry32_lim<RIEM>(a.limiter, Fm, Bq, Iq, dlp[2 * cb], dlp[2 * ci], nx, ny, ln, gam, gm1,
                                                    gf, X, g);
                        else
                            bc_extrapolation32(Bq, nx, ny, ln, gf, X);
                    } else if (e.type > 0) {   // inflow / outflow records
                        int path = 2;
                        if (e.type == 401 && e.param >= 0) {   // stagnation inflow: FP32 when it decides, else FP64
                            const float4 Bc = sP[cb], Ic = sP[ci];
                            const float Bq[4] = {Bc.x, Bc.y, Bc.z, Bc.w}, Iq[4] = {Ic.x, Ic.y, Ic.z, Ic.w};
                            path = bc_stagnation32(Fm, Bq, nx, ny, ln, gam, (float)g.R, a.bcp[e.param], X);
                            if (path == 1) {
                                bc_symmetry32_lim<RIEM>(a.limiter, Fm, Bq, Iq, dlp[2 * cb], dlp[2 * ci], nx, ny, ln, gam,
                                                        gm1, gf, X, g);
                                path = 0;
                            }
                        }
                        if (path == 2) {   // FP64 from the FP64 state
                            const double* pb = Pin + (long long)bj * ni + bi;
                            const int ni2 = bi + di, nj2 = bj + dj;
                            Q4 Bp, Ip;
#pragma unroll
                            for (int v = 0; v < 4; ++v) Bp.v[v] = __ldg(pb + v * pc);
                            if (ni2 >= 0 && ni2 < ni && nj2 >= 0 && nj2 < nj) {
                                const double* pi = Pin + (long long)nj2 * ni + ni2;
#pragma unroll
                                for (int v = 0; v < 4; ++v) Ip.v[v] = __ldg(pi + v * pc);
                            } else {   // one-cell-thick block: the neighbour is the opposite ghost
                                const float4 Ic = sP[ci];
                                Ip.v[0] = Ic.x; Ip.v[1] = Ic.y; Ip.v[2] = Ic.z; Ip.v[3] = Ic.w;
                            }
                            const double* dlb = a.dl + B.og + (long long)(Fm <= 2 ? 0 : 1) * B.pg;
                            const double dlbv = __ldg(dlb + (long long)(bj + 2) * (ni + 4) + (bi + 2));
                            const double dli = __ldg(dlb + (long long)(nj2 + 2) * (ni + 4) + (ni2 + 2));
                            const double* gsrc = Fm <= 2 ? a.fi + B.ofi + (long long)bj * (ni + 1) + (Fm == 1 ? 0 : ni)
                                                         : a.fj + B.ofj + (long long)(Fm == 3 ? 0 : nj) * ni + bi;
                            const long long gs = Fm <= 2 ? B.pfi : B.pfj;
                            const Q4 q = bc_face<RIEM>(a.gas, a.limiter, e.type, Fm, Bp, Ip, dlbv, dli, __ldg(gsrc),
                                                       __ldg(gsrc + gs), __ldg(gsrc + 2 * gs),
                                                       e.param >= 0 ? a.bcp + e.param : nullptr);
#pragma unroll
                            for (int v = 0; v < 4; ++v) X[v] = (float)q.v[v];
                        }
                    }
                    sF[f] = make_float4(X[0], X[1], X[2], X[3]);
                }
            }
        }
        __syncthreads();
        if (pre) {   // store the next descriptor; the end-of-item barrier publishes it
            if (lane < NWW) reinterpret_cast<int*>(&sW[cur ^ 1])[lane] = pw;
            if (lane < NBW) reinterpret_cast<int*>(&sBk[cur ^ 1])[lane] = pb;
            if (lane == 0) sSt[cur ^ 1] = ps;
        }

        // ---- 3. residual, sources, RK update (+ next dt and residual norm) -----------------------
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        const double dt_case = __ldcg(&cs->dt_step);
        // iteration whose time step is computed: this one (dt_here; the prologue has not run) or
        // the next one (last stage)
        const long long iter_dt = __ldcg(&cs->iter) + (dt_here || a.first ? 1 : 0) + (dt_here ? 0 : 1);
        for (int k = tid; k < NC; k += NT) {
            const int row = k / TX, col = k - row * TX;
            const int ii = i0 + col, jj = j0 + row;
            if (ii >= ni || jj >= nj) continue;
            const long long cg = (long long)jj * ni + ii;
            double P[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) P[v] = sC[(8 + v) * NC + k];
            const int i1 = ii + 1, j1 = jj + 1;
            const int fi0 = row * (TX + 1) + col, fj0 = NFI + row * TX + col;
            double q[4];   // the scaled residual -R dt / sur of the update
            if (irs == 2) {
#pragma unroll
                for (int v = 0; v < 4; ++v) q[v] = sC[(4 + v) * NC + k];
            } else {
            double r[4];
            const float4 Fw = sF[fi0], Fe = sF[fi0 + 1], Fs = sF[fj0], Fn = sF[fj0 + TX];
#pragma unroll
            for (int v = 0; v < 4; ++v) {   // interior i, interior j, then boundary faces 1..4
                const double w = comp(Fw, v), e = comp(Fe, v), so = comp(Fs, v), no = comp(Fn, v);
                double x = 0.0;
                if (i1 > 1) x = x - w;
                if (i1 < ni) x = x + e;
                if (j1 > 1) x = x - so;
                if (j1 < nj) x = x + no;
                if (i1 == 1) x = x - w;
                if (i1 == ni) x = x + e;
                if (j1 == 1) x = x - so;
                if (j1 == nj) x = x + no;
                r[v] = x;
            }
            const double sur = sC[4 * NC + k];
            if (a.source) {
                // S = [rho, rho u, rho v, rho E0 + p] * f0 with f0 = -v/r (Lib_Source_Axisymmetry.f90:
                // 65-76) or V.G (Lib_Source_Areavariation.f90:120-142); Res -= S * sur
                const double rE0 = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
                const double f0 = a.source == 1 ? -P[2] * sC[6 * NC + k]
                                                : P[1] * sC[6 * NC + k] + P[2] * sC[7 * NC + k];
                const double fs = f0 * sur;
                r[0] = r[0] - P[0] * fs;
                r[1] = r[1] - P[0] * P[1] * fs;
                r[2] = r[2] - P[0] * P[2] * fs;
                r[3] = r[3] - (rE0 + P[3]) * fs;
            }
            double dt;
            if (dt_here) {
                // Compute_dt (Mod_dt.f90:59-104) from the step's starting state, FP32 arithmetic
                const int sidx = (row + 2) * W + (col + 2);
                const float dtc = cell_dt32((float)P[0], (float)P[1], (float)P[2], (float)P[3], gam,
                                            (float)a.cfl, ndir, sD[2 * sidx], sD[2 * sidx + 1],
                                            (float)sC[k], (float)sC[NC + k], (float)sC[2 * NC + k],
                                            (float)sC[3 * NC + k]);
                dt = (double)dtc;
                if (iter_dt < a.rampa) dt = dt * (double)iter_dt / (double)a.rampa;
                if (!a.last) a.sc[2 * B.oc + pc + cg] = dt;   // for the later stages
                acc[4] = fmin(acc[4], dt);
            } else {
                dt = a.time_accurate ? dt_case : sC[5 * NC + k];
            }
            const double fr = -dt * rcp64(sur);
#pragma unroll
            for (int v = 0; v < 4; ++v) q[v] = r[v] * fr;
            if (irs == 1) {   // Scale_Residual_Cons (Lib_Newstate.f90:86-92): smoothed before the update
                double* ro = a.Rout + B.oc;
#pragma unroll
                for (int v = 0; v < 4; ++v) ro[v * pc + cg] = q[v];
                continue;
            }
            }
            double PO[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) PO[v] = a.first ? P[v] : sC[v * NC + k];
            double U0[4], U[4];
            U0[0] = PO[0]; U0[1] = PO[0] * PO[1]; U0[2] = PO[0] * PO[2];
            U0[3] = PO[3] * g.igm1 + 0.5 * PO[0] * (PO[1] * PO[1] + PO[2] * PO[2]);
            U[0] = P[0]; U[1] = P[0] * P[1]; U[2] = P[0] * P[2];
            U[3] = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
#pragma unroll
            for (int v = 0; v < 4; ++v) U[v] = U0[v] + (U[v] - U0[v] + q[v]) * a.rk_c;
            double N[4];
            N[0] = U[0];
            const double ir = rcp64(U[0]);
            N[1] = U[1] * ir;
            N[2] = U[2] * ir;
            N[3] = g.gm1 * (U[3] - 0.5 * U[0] * (N[1] * N[1] + N[2] * N[2]));
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
                if (!a.dt_first) {
                    // Compute_dt (Mod_dt.f90:59-104) for the next step, FP32 arithmetic
                    const int sidx = (row + 2) * W + (col + 2);
                    const float dtc = cell_dt32((float)N[0], (float)N[1], (float)N[2], (float)N[3], gam,
                                                (float)a.cfl, ndir, sD[2 * sidx], sD[2 * sidx + 1],
                                                (float)scb[2 * pc + cg], (float)scb[3 * pc + cg],
                                                ndir == 2 ? (float)scb[4 * pc + cg] : 0.0f,
                                                ndir == 2 ? (float)scb[5 * pc + cg] : 0.0f);
                    double dtn = (double)dtc;
                    if (iter_dt < a.rampa) dtn = dtn * (double)iter_dt / (double)a.rampa;
                    if (!a.time_accurate) a.sc[2 * B.oc + pc + cg] = dtn;
                    acc[4] = fmin(acc[4], dtn);
                }
            }
        }
        if (a.last || dt_here) {   // per-warp partials: residual sums (last stage), dt min
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                double v = acc[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double u = __shfl_down_sync(0xffffffffu, v, o);
                    v = (k < 4) ? v + u : fmin(v, u);
                }
                acc[k] = v;
            }
            if (lane == 0) {
                double* pp = a.part + ((size_t)it * (NT / 32) + (tid >> 5)) * 5;
                if (a.last)
                    for (int k = 0; k < 4; ++k) pp[k] = acc[k];
                if (a.dt_first ? dt_here : a.last) pp[4] = acc[4];
            }
        }
        stage_item_end<NT>(a, it, w.case_id, red, &s_flag);
    }
}

// SD: the MUSCL-SD instantiation (the shock sensor in the face phase), a separate kernel so that
// the plain form keeps its register allocation.
template <int RIEM, int TX, int TY, int NT, int MB, bool SD>
cudaError_t launch_stage32_sd(const StageArgs& a, int grid, cudaStream_t s) {
    constexpr size_t smem = Tile32<TX, TY>::bytes;
    auto k = stage32_kernel<RIEM, TX, TY, NT, MB, SD>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

// The sensor-driven Riemann solvers (HLLC+, HLLE++) run the sensor whatever the reconstruction.
template <int RIEM, int TX, int TY, int NT, int MB>
cudaError_t launch_stage32_t(const StageArgs& a, int grid, cudaStream_t s) {
    if constexpr (RIEM == 5 || RIEM == 6) {
        return launch_stage32_sd<RIEM, TX, TY, NT, MB, true>(a, grid, s);
    } else {
        return a.sd ? launch_stage32_sd<RIEM, TX, TY, NT, MB, true>(a, grid, s)
                    : launch_stage32_sd<RIEM, TX, TY, NT, MB, false>(a, grid, s);
    }
}

template <int RIEM, int TX, int TY, int NT, int MB>
int stage32_occupancy_t() {
    constexpr size_t smem = Tile32<TX, TY>::bytes;
    auto k = stage32_kernel<RIEM, TX, TY, NT, MB, (RIEM == 5 || RIEM == 6)>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, smem);
    return n;
}

}  // namespace q2d
