// q2d_stage32d.cuh — the RK-stage kernel of the FP32-flux / FP64-state form in difference form
// (sm_100a), for the HLLC, HLLE and LLF Riemann solvers without MUSCL-SD or implicit residual
// smoothing.
//
// Precision split. A face flux is written as the physical flux of a face state plus the
// Riemann solver's upwind correction, F = F_K + corr. The face states (the FP64 cell value plus
// the limited FP32 slope times the half cell length), the physical fluxes F_K and the face
// geometry are FP64, so the large terms of the flux balance of a cell carry FP64 rounding; the
// slopes (from FP64 differences), the limiters, the Roe averages, the wave speeds and the
// correction terms are FP32, so the FP32 rounding scales with the jumps at the face instead of
// with the flux itself. The state, the flux sums, sources, RK combination, positivity checks
// and residual norms are FP64; the local time step is FP32 arithmetic.
//
// Tiles of TX x TY cells, one CTA of NT threads per tile in a grid-stride loop over the work
// items. Per tile:
//   1. loads: one bulk asynchronous copy (cp.async.bulk, completion on an mbarrier) per row of
//      each array the tile reads: the FP64 state of the tile and its 2-cell halo (4 planes),
//      the FP32 cell lengths on the ghost frame, the FP64 geometry of the tile's i and j faces
//      (3 planes each), and the FP64 per-cell data of the tile's own cells (U^n or the time-step
//      directions, volume, time step, source geometry). Rows whose start is not 16-byte aligned
//      are copied from the aligned element before it, and each row records that shift;
//   2. ghost cells of block edges the tile's stencils reach (Fill_Ghost_Cell,
//      Lib_Ghost.f90:16-299) in FP64 from the staged state, connection ghosts from the donor
//      block in HBM;
//   3. faces: each thread takes the west face and then the south face of its cell; the east
//      faces of the last column, the north faces of the top row and the boundary faces
//      (BC_Fluxes, Mod_BC_Fluxes.f90:79-269) go to separate warps in a third pass;
//   4. cells: residual in the reference's accumulation order, sources, Newstate_Conservative +
//      RK_stage + Check_And_Fix_State, the cell's time step (first stage) and the squared state
//      change of the residual norm (last stage), per-warp partials.
#pragma once
#include "q2d_stage32.cuh"

namespace q2d {
namespace dform {

// ---- bulk copies and transaction barriers ------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// 16-byte aligned global -> shared copy of `bytes` (a multiple of 16) completing on `bar`
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(1000000u)   // suspend for up to 1 ms per try
        : "memory");
    return ok != 0;
}
// Waits for the phase of `parity` to complete, for about a second of SM clocks at most.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (2LL << 30)) return false;
    return true;
}
// Orders this thread's generic-proxy shared-memory accesses before later bulk copies into them.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- tile layout ---------------------------------------------------------------------------
// Every staged row starts on a 16-byte boundary; element x of a row sits at column
// (x - first) + shift, the shift (0 or 1) recorded per row.
template <int TX, int TY>
struct TileD {
    static constexpr int HR = TY + 4;      // halo rows (state, cell lengths)
    static constexpr int RW = TX + 6;      // halo row: columns i0-2 .. i0+TX+1, shift, 16-byte rounding
    static constexpr int RGI = TX + 4;     // i-face row: faces i0 .. i0+TX
    static constexpr int RGJ = TX + 2;     // j-face row: faces of columns i0 .. i0+TX-1
    static constexpr int RO = TX + 2;      // own-cell row
    static constexpr int NOWN = 8;         // own-cell planes: 0-3 U^n or the time-step directions,
                                           // 4 volume, 5 time step, 6-7 source geometry
    static constexpr int NFI = (TX + 1) * TY, NFJ = TX * (TY + 1), NF = NFI + NFJ, NC = TX * TY;
    static constexpr int PS = HR * RW;                 // state plane (doubles)
    static constexpr int PGI = TY * RGI, PGJ = (TY + 1) * RGJ, PO = TY * RO;
    static constexpr size_t bS = 0;                                   // double [4][HR][RW]
    static constexpr size_t bD = bS + 8ull * 4 * PS;                  // float2 [HR][RW]
    static constexpr size_t bGI = bD + 8ull * PS;                     // double [3][TY][RGI]
    static constexpr size_t bGJ = bGI + 8ull * 3 * PGI;               // double [3][TY+1][RGJ]
    static constexpr size_t bO = bGJ + 8ull * 3 * PGJ;                // double [NOWN][TY][RO]
    static constexpr size_t bF = bO + 8ull * NOWN * PO;               // double [4][NF] face fluxes
    static constexpr size_t bytes = bF + 8ull * 4 * NF;
    // copies per tile: state 4 x HR, lengths HR, i faces 3 x TY, j faces 3 x (TY+1), own NOWN x TY
    static constexpr int NCOPY = 4 * HR + HR + 3 * TY + 3 * (TY + 1) + NOWN * TY;
    static_assert(RW % 2 == 0 && RGI % 2 == 0 && RGJ % 2 == 0 && RO % 2 == 0, "16-byte rows");
    static_assert(bD % 16 == 0 && bGI % 16 == 0 && bGJ % 16 == 0 && bO % 16 == 0 && bF % 16 == 0, "alignment");
};

// One row copy: n elements of `esz` bytes from element e0 of a plane whose base is 16-byte
// aligned, into a 16-byte aligned shared row; returns the byte count (0: nothing) and the
// row's shift.
struct RowCopy {
    const void* src;
    unsigned bytes;
    int shift;
};
__device__ __forceinline__ RowCopy row_copy(const char* plane, long long e0, int n, int esz) {
    // esz is 8 (double, float2): 16 bytes hold 2 elements
    const long long a0 = e0 & ~1LL, a1 = (e0 + n + 1) & ~1LL;
    RowCopy r;
    r.src = plane + a0 * esz;
    r.bytes = n > 0 ? (unsigned)((a1 - a0) * esz) : 0u;
    r.shift = (int)(e0 & 1);
    return r;
}

// ---- conversions ----------------------------------------------------------------------------
// FP64 <-> FP32 conversions as single cvt instructions (round to nearest, subnormals kept): the
// flush-to-zero forms the FP32 arithmetic is compiled with have no single-instruction
// conversion. The values converted here (states, jumps, slopes, flux corrections) are far from
// the subnormal range or are flushed by the FP32 arithmetic that follows.
__device__ __forceinline__ float f32(double x) {
    float y;
    asm("cvt.rn.f32.f64 %0, %1;" : "=f"(y) : "d"(x));
    return y;
}
__device__ __forceinline__ double f64(float x) {
    double y;
    asm("cvt.f64.f32 %0, %1;" : "=d"(y) : "f"(x));
    return y;
}

// ---- difference-form Riemann fluxes ---------------------------------------------------------
// Physical flux of an FP64 face state per unit length, normal velocity un.
__device__ __forceinline__ void phys_flux64(const double* Q, double un, double nx, double ny, double gf,
                                            double* F) {
    const double m = Q[0] * un;
    F[0] = m;
    F[1] = m * Q[1] + Q[3] * nx;
    F[2] = m * Q[2] + Q[3] * ny;
    F[3] = un * (gf * Q[3] + 0.5 * Q[0] * (Q[1] * Q[1] + Q[2] * Q[2]));
}

__device__ __forceinline__ void cons64(const double* Q, double igm1, double* U) {
    U[0] = Q[0];
    U[1] = Q[0] * Q[1];
    U[2] = Q[0] * Q[2];
    U[3] = Q[3] * igm1 + 0.5 * Q[0] * (Q[1] * Q[1] + Q[2] * Q[2]);
}

// Flux per unit length between FP64 face states QL, QR across the normal (nx, ny):
// riemann_HLLC (RIEM 0, Lib_Riemann_HLL.f90:34-123), riemann_HLLE (1, :126-169), riemann_LLF
// (2, Lib_Riemann_LF.f90:11-40), with the clamped Einfeldt speeds from constant-cp Roe
// averages. HLLC: F = F_K + S_K (U*_K - U_K) with K the side of the contact (the clamped speeds
// make S_K = 0 the supersonic cases); HLLE: F = F_L + S1 / (S4 - S1) (F_L - F_R + S4 (U_R - U_L));
// LLF: F = (F_L + F_R) / 2 - A (U_R - U_L) / 2. The jumps are FP64 differences rounded to FP32.
template <int RIEM>
__device__ __forceinline__ void riemann_df(const double* QL, const double* QR, double nx, double ny, const Gas& g,
                                           float gam, float gm1, float gf, double* F) {
    const double unL = QL[1] * nx + QL[2] * ny, unR = QR[1] * nx + QR[2] * ny;
    const float rl = f32(QL[0]), ul = f32(QL[1]), vl = f32(QL[2]), pl = f32(QL[3]);
    const float rr = f32(QR[0]), ur = f32(QR[1]), vr = f32(QR[2]), pr = f32(QR[3]);
    const float unl = f32(unL), unr = f32(unR);
    const float irl = rcp_approx(rl), irr = rcp_approx(rr);
    const float al = sqrtf(gam * pl * irl), ar = sqrtf(gam * pr * irr);
    if (RIEM == 2) {
        const float A = fmaxf(fmaxf(fabsf(unl - al), fabsf(unr - ar)), fmaxf(fabsf(unl + al), fabsf(unr + ar)));
        double FL[4], FR[4], UL[4], UR[4];
        phys_flux64(QL, unL, nx, ny, g.gfac, FL);
        phys_flux64(QR, unR, nx, ny, g.gfac, FR);
        cons64(QL, g.igm1, UL);
        cons64(QR, g.igm1, UR);
        const float hA = 0.5f * A;
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] = 0.5 * (FL[v] + FR[v]) - f64(hA * f32(UR[v] - UL[v]));
        return;
    }
    const float srL = sqrtf(rl), srR = sqrtf(rr);
    const float isr = rcp_approx(srL + srR);
    const float u_roe = (srR * ur + srL * ul) * isr;
    const float v_roe = (srR * vr + srL * vl) * isr;
    const float h0l = gf * pl * irl + 0.5f * (ul * ul + vl * vl);
    const float h0r = gf * pr * irr + 0.5f * (ur * ur + vr * vr);
    const float h0_roe = (srR * h0r + srL * h0l) * isr;
    const float a_roe = sqrtf(fmaxf(gm1 * (h0_roe - 0.5f * (u_roe * u_roe + v_roe * v_roe)), 0.0f));
    const float un_roe = u_roe * f32(nx) + v_roe * f32(ny);
    const float S1 = fminf(fminf(0.0f, unl - al), un_roe - a_roe);
    const float S4 = fmaxf(fmaxf(0.0f, unr + ar), un_roe + a_roe);
    if (RIEM == 1) {
        double FL[4], FR[4], UL[4], UR[4];
        phys_flux64(QL, unL, nx, ny, g.gfac, FL);
        phys_flux64(QR, unR, nx, ny, g.gfac, FR);
        cons64(QL, g.igm1, UL);
        cons64(QR, g.igm1, UR);
        const float w = S4 > S1 ? S1 * rcp_approx(S4 - S1) : 0.0f;
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] = FL[v] + f64(w * (f32(FL[v] - FR[v]) + S4 * f32(UR[v] - UL[v])));
        return;
    }
    const float dun = f32(unR - unL), dp = f32(QR[3] - QL[3]);
    const float D = rl * (S1 - unl) - rr * (S4 - unr);
    const float sm_unl = (dp - rr * (S4 - unr) * dun) * rcp_approx(D);   // S* - un_L
    const float Sstar = unl + sm_unl;
    const bool left = Sstar >= 0.0f;
    const double* QK = left ? QL : QR;
    const double unK64 = left ? unL : unR;
    const float SK = left ? S1 : S4;
    const float rK = left ? rl : rr, uK = left ? ul : ur, vK = left ? vl : vr, pK = left ? pl : pr;
    const float unK = left ? unl : unr, irK = left ? irl : irr, h0K = left ? h0l : h0r;
    const float smK = left ? sm_unl : sm_unl - dun;                      // S* - un_K
    double FK[4];
    phys_flux64(QK, unK64, nx, ny, g.gfac, FK);
    if (SK == 0.0f) {
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] = FK[v];
        return;
    }
    const float inv = rcp_approx(SK - Sstar);
    const float q = smK * inv;
    const float dps = rK * (SK - unK) * smK;                             // p* - p_K
    const float e0K = h0K - pK * irK;
    F[0] = FK[0] + f64(SK * (rK * q));
    F[1] = FK[1] + f64(SK * (rK * uK * q + dps * f32(nx) * inv));
    F[2] = FK[2] + f64(SK * (rK * vK * q + dps * f32(ny) * inv));
    F[3] = FK[3] + f64(SK * (rK * e0K * q + (dps * Sstar + pK * smK) * inv));
}

// One face from its 4-cell stencil m, 0, 1, p: the FP64 states at st[v * PS + o_k], the FP32
// cell lengths of the face's direction at dlf[2 * d_k] (dlf points at component 0 of the length
// pairs for an i face, 1 for a j face). Reconstruction (Lib_Reconstruction.f90:10-29) in
// difference form: the three slopes from FP64 differences, limited in FP32, added to the FP64
// cell values. Returns false when a face state has a non-positive density or pressure
// (check_gas_state, Lib_Convective.f90:49-54).
template <int RIEM, int LIM, int PS>
__device__ __forceinline__ bool face_df(const double* st, int o0, int o1, int o2, int o3, const float* dlf, int d0_,
                                        int d1_, int d2_, int d3_, double nx, double ny, double len, const Gas& g,
                                        float gam, float gm1, float gf, double* F) {
    const float dm = dlf[2 * d0_], d0 = dlf[2 * d1_], d1 = dlf[2 * d2_], d2 = dlf[2 * d3_];
    const float il0 = rcp_approx(0.5f * (dm + d0));
    const float il1 = rcp_approx(0.5f * (d0 + d1));
    const float il2 = rcp_approx(0.5f * (d1 + d2));
    const float lm = 0.5f * d0, lp = 0.5f * d1;
    double QL[4], QR[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double* p = st + v * PS;
        const double qm = p[o0], q0 = p[o1], q1 = p[o2], q2 = p[o3];
        const float s0 = f32(q0 - qm) * il0, s1 = f32(q1 - q0) * il1, s2 = f32(q2 - q1) * il2;
        QL[v] = q0 + f64(lim32<LIM>(s1, s0) * lm);
        QR[v] = q1 - f64(lim32<LIM>(s2, s1) * lp);
    }
    const bool ok = QL[0] > 0.0 && QL[3] > 0.0 && QR[0] > 0.0 && QR[3] > 0.0;
    riemann_df<RIEM>(QL, QR, nx, ny, g, gam, gm1, gf, F);
#pragma unroll
    for (int v = 0; v < 4; ++v) F[v] *= len;
    return ok;
}

// BC_Symmetry_Eul (Lib_BC_Fluxes_Symmetry.f90:28-124) in difference form: the mirrored ghost,
// the limited slope of the boundary cell (FP32, from FP64 differences) added to its FP64 value,
// the Riemann problem between the face state and its mirror; momentum flux only.
template <int RIEM, int LIM>
__device__ __forceinline__ void bc_symmetry_df(int Fm, const double* Bp, const double* Ip, float dlb, float dli,
                                               double nx, double ny, double len, const Gas& g, float gam,
                                               float gm1, float gf, double* out) {
    const bool minside = (Fm & 1) != 0;   // faces 1 and 3
    const float bd = 0.5f * dlb, id = 0.5f * dli;
    const double un = Bp[1] * nx + Bp[2] * ny;
    const double G[4] = {Bp[0], Bp[1] - 2.0 * un * nx, Bp[2] - 2.0 * un * ny, Bp[3]};
    const float i12 = rcp_approx(minside ? 2.0f * bd : bd + id);
    const float i23 = rcp_approx(minside ? bd + id : 2.0f * bd);
    const float dist = minside ? -bd : bd;
    double Fc[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double P1 = minside ? G[v] : Ip[v], P3 = minside ? Ip[v] : G[v];
        Fc[v] = Bp[v] + f64(lim32<LIM>(f32(P3 - Bp[v]) * i23, f32(Bp[v] - P1) * i12) * dist);
    }
    const double Un = Fc[1] * nx + Fc[2] * ny;
    const double vtx = Fc[1] - Un * nx, vty = Fc[2] - Un * ny;
    const double Un1 = minside ? -Un : Un;
    const double L[4] = {Fc[0], Un1 * nx + vtx, Un1 * ny + vty, Fc[3]};
    const double R[4] = {Fc[0], -Un1 * nx + vtx, -Un1 * ny + vty, Fc[3]};
    double F[4];
    riemann_df<RIEM>(L, R, nx, ny, g, gam, gm1, gf, F);
    out[0] = 0.0;
    out[1] = F[1] * len;
    out[2] = F[2] * len;
    out[3] = 0.0;
}

}  // namespace dform

template <int RIEM, int LIM, int TX, int TY, int NT, int MB>
__global__ void __launch_bounds__(NT, MB) stage32d_kernel(const StageArgs a) {
    using namespace dform;
    using L = TileD<TX, TY>;
    constexpr int HR = L::HR, RW = L::RW, RGI = L::RGI, RGJ = L::RGJ, RO = L::RO, PS = L::PS;
    constexpr int NFI = L::NFI, NF = L::NF, NC = L::NC;
    static_assert(TX == 32 && NT % 32 == 0 && NT >= NC && 5 * HR + 3 * TY + 3 * (TY + 1) <= NT && L::NOWN * TY < NT,
                  "one cell and at most one copy of each group per thread");
    static_assert(NT / 32 >= TY && NT / 32 >= 4, "a warp per tile row, and warps for the third face pass");
    static_assert(4 * TY + 4 * TX <= NT, "one ghost slot per thread");
    extern __shared__ __align__(16) unsigned char sb[];
    double* sS = reinterpret_cast<double*>(sb + L::bS);
    float2* sD = reinterpret_cast<float2*>(sb + L::bD);
    double* sGI = reinterpret_cast<double*>(sb + L::bGI);
    double* sGJ = reinterpret_cast<double*>(sb + L::bGJ);
    double* sO = reinterpret_cast<double*>(sb + L::bO);
    double* sF = reinterpret_cast<double*>(sb + L::bF);
    // stencil copies (state, lengths, face geometry) and own-cell copies complete on separate
    // barriers: a tile's stencil is issued after the previous tile's faces, its own-cell data
    // after the previous tile's end, so both usually land before they are needed
    __shared__ unsigned long long barS, barO;
    __shared__ int shS[2][HR], shD[2][HR], shGI[2][TY], shGJ[2][TY + 1], shO[2][TY];   // row shifts by slot
    // the first 80 bytes of the item's CaseState (dt_step at 0, iter at 72), copied with the own rows
    __shared__ __align__(16) double sCase[2][10];
    static_assert(sizeof(CaseState) % 16 == 0 && offsetof(CaseState, dt_step) == 0 && offsetof(CaseState, iter) == 72,
                  "CaseState head copied in one 80-byte bulk copy");
    __shared__ WorkItem sW[2];
    __shared__ DBlock sBk[2];
    __shared__ int sSt[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (a.part_stride != NT / 32 || !a.fin_sep) {   // host / kernel mismatch of the partials layout
        if (tid == 0)
            for (int it = blockIdx.x; it < a.n_items; it += gridDim.x)
                record_error(&a.cstate[__ldg(&a.items[it].case_id)], Q2D_ERR_BADARG, -1, -1, -1, a.irk);
        return;
    }
    const Gas& g = a.gas;
    const float gam = (float)g.gamma, gm1 = (float)g.gm1, gf = (float)g.gfac;
    if (tid == 0) {
        mbar_init(&barS, NT);
        mbar_init(&barO, NT);
        mbar_init_fence();
    }
    const bool dt_here = a.dt_first && a.first;
    // Bulk copies of the stencil rows of the item in descriptor slot `sl` (every thread arrives
    // once on barS, with the byte count of its copy if it has one).
    auto issue_stencil = [&](const WorkItem& w, const DBlock& B, int sl) {
        const int ni = B.ni, nj = B.nj, i0 = w.i0, j0 = w.j0;
        const int nrow = min(TY, nj - j0), ncol = min(TX, ni - i0);
        RowCopy rc{nullptr, 0u, 0};
        void* dst = nullptr;
        // copy index of the thread: consecutive copies go to different warps, so that the lanes
        // each warp issues one after another are spread over all of them
        const int t = lane * (NT / 32) + warp;
        if (t < 4 * HR) {                                   // state rows j0-2 .. j0+TY+1
            const int v = t / HR, r = t - v * HR, jj = j0 - 2 + r;
            const int cs0 = max(i0 - 2, 0), ce = min(i0 + TX + 2, ni);
            if (jj >= 0 && jj < nj)
                rc = row_copy(reinterpret_cast<const char*>(a.Pin + B.oc + v * B.pc), (long long)jj * ni + cs0,
                              ce - cs0, 8);
            // column of element cs0 is cs0 - (i0 - 2) + shift; the copy starts one element
            // before it when the shift is 1
            dst = sS + v * PS + r * RW + (cs0 - (i0 - 2));
            if (v == 0) shS[sl][r] = rc.bytes ? rc.shift : 0;
        } else if (t < 5 * HR) {                            // cell lengths on the ghost frame
            const int r = t - 4 * HR, jj = j0 - 2 + r;
            const int ce = min(i0 + TX + 2, ni + 2);
            if (jj <= nj + 1)
                rc = row_copy(reinterpret_cast<const char*>(a.dl32 + B.og),
                              (long long)(jj + 2) * (ni + 4) + i0, ce - (i0 - 2), 8);
            dst = sD + r * RW;
            shD[sl][r] = rc.bytes ? rc.shift : 0;
        } else if (t < 5 * HR + 3 * TY) {                   // i-face geometry rows
            const int u = t - 5 * HR, q = u / TY, r = u - q * TY;
            if (r < nrow)
                rc = row_copy(reinterpret_cast<const char*>(a.fi + B.ofi + q * B.pfi),
                              (long long)(j0 + r) * (ni + 1) + i0, ncol + 1, 8);
            dst = sGI + q * L::PGI + r * RGI;
            if (q == 0) shGI[sl][r] = rc.bytes ? rc.shift : 0;
        } else if (t < 5 * HR + 3 * TY + 3 * (TY + 1)) {    // j-face geometry rows
            const int u = t - 5 * HR - 3 * TY, q = u / (TY + 1), r = u - q * (TY + 1);
            if (r <= nrow)
                rc = row_copy(reinterpret_cast<const char*>(a.fj + B.ofj + q * B.pfj),
                              (long long)(j0 + r) * ni + i0, ncol, 8);
            dst = sGJ + q * L::PGJ + r * RGJ;
            if (q == 0) shGJ[sl][r] = rc.bytes ? rc.shift : 0;
        }
        if (rc.bytes) {
            mbar_arrive_expect_tx(&barS, rc.bytes);
            bulk_copy(dst, rc.src, rc.bytes, &barS);
        } else {
            mbar_arrive(&barS);
        }
    };
    // Bulk copies of the own-cell rows (U^n or the time-step directions, volume, time step,
    // source geometry) of the item in slot `sl`, completing on barO.
    auto issue_own = [&](const WorkItem& w, const DBlock& B, int sl) {
        const int ni = B.ni, nj = B.nj, i0 = w.i0, j0 = w.j0;
        const int nrow = min(TY, nj - j0), ncol = min(TX, ni - i0);
        const long long pc = B.pc;
        const double* scb = a.sc + 2 * B.oc;
        RowCopy rc{nullptr, 0u, 0};
        void* dst = nullptr;
        const int t = lane * (NT / 32) + warp;   // spread over the warps like the stencil copies
        if (t < L::NOWN * TY) {
            const int k = t / TY, r = t - k * TY;
            const double* plane = nullptr;
            if (k < 4) {
                if (!a.first) plane = a.PO + B.oc + k * pc;
                else if (dt_here && (k < 2 || a.cases[w.case_id].ndir == 2)) plane = scb + (2 + k) * pc;
            } else if (k == 4) {
                plane = scb;
            } else if (k == 5) {
                if (!a.time_accurate && !dt_here) plane = scb + pc;
            } else if (a.source && (k == 6 || a.source == 2)) {
                plane = scb + (k == 6 ? 6 : 7) * pc;
            }
            if (plane && r < nrow)
                rc = row_copy(reinterpret_cast<const char*>(plane), (long long)(j0 + r) * ni + i0, ncol, 8);
            dst = sO + k * L::PO + r * RO;
            if (k == 4) shO[sl][r] = rc.bytes ? rc.shift : 0;
        } else if (t == L::NOWN * TY) {   // the case's time step and iteration
            rc.src = &a.cstate[w.case_id];
            rc.bytes = 80u;
            dst = sCase[sl];
        }
        if (rc.bytes) {
            mbar_arrive_expect_tx(&barO, rc.bytes);
            bulk_copy(dst, rc.src, rc.bytes, &barO);
        } else {
            mbar_arrive(&barO);
        }
    };
    static_assert(sizeof(WorkItem) == 24 && sizeof(DBlock) % 4 == 0 && sizeof(DBlock) <= 128, "descriptor words");
    constexpr int NWW = (int)(sizeof(WorkItem) / 4), NBW = (int)(sizeof(DBlock) / 4);
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
    unsigned phS = 0, phO = 0;          // completed phases of barS / barO
    bool s_pre = false, o_pre = false;  // the current item's copies were issued by the last iteration
    const int row = warp, col = lane;   // the thread's cell in the tile (row < TY)
    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x, cur ^= 1) {
        const int nit = it + gridDim.x;
        const bool pre = w0 && nit < a.n_items;
        int pw = 0, pb = 0, ps = 0;
        if (pre && lane < NWW) pw = __ldg(reinterpret_cast<const int*>(a.items + nit) + lane);
        const WorkItem w = sW[cur];
        const DBlock B = sBk[cur];
        CaseState* cs = &a.cstate[w.case_id];
        if (sSt[cur] != kStatus_Running) {
            if (pre) {
                const int blk = __shfl_sync(0xffffffffu, pw, 0), cid = __shfl_sync(0xffffffffu, pw, 3);
                pb = lane < NBW ? __ldg(reinterpret_cast<const int*>(a.blocks + blk) + lane) : 0;
                if (lane < NWW) reinterpret_cast<int*>(&sW[cur ^ 1])[lane] = pw;
                if (lane < NBW) reinterpret_cast<int*>(&sBk[cur ^ 1])[lane] = pb;
                if (lane == 0) sSt[cur ^ 1] = __ldcg(&a.cstate[cid].status);
            }
            __syncthreads();
            s_pre = o_pre = false;
            continue;
        }
        const int ni = B.ni, nj = B.nj, i0 = w.i0, j0 = w.j0;
        const long long pc = B.pc;
        const double* scb = a.sc + 2 * B.oc;
        const int ndir = a.cases[w.case_id].ndir;
        const int nrow = min(TY, nj - j0), ncol = min(TX, ni - i0);

        // ---- 1. loads: one bulk copy per staged row (unless the last iteration issued them) ----
        if (!s_pre) issue_stencil(w, B, cur);
        if (!o_pre) issue_own(w, B, cur);
        // The thread's ghost slot (one ghost cell the tile's stencils read beyond a block edge:
        // two layers of i-ghosts beside the tile rows, two of j-ghosts beside its columns), its
        // boundary record and boundary-face normal, and a connection ghost's donor value, while
        // the copies are in flight.
        int g_ii = 0, g_jj = 0, g_type = -2, g_f = 0, g_gd = 0;
        double g_q[4] = {0.0, 0.0, 0.0, 0.0}, g_nx = 0.0, g_ny = 0.0;
        if (i0 == 0 || j0 == 0 || i0 + TX + 2 > ni || j0 + TY + 2 > nj) {
            const int t = tid;
            bool valid = false;
            if (t < 4 * TY) {                                     // i-ghosts: left (t < 2 TY), right
                const int side = t / (2 * TY), u = t - side * 2 * TY, gd = 1 + u / TY, r = u - (gd - 1) * TY;
                const int ii = side == 0 ? -gd : ni - 1 + gd;
                valid = r < nrow && (side == 0 ? i0 == 0 : ii <= i0 + TX + 1);
                g_ii = ii; g_jj = j0 + r; g_f = side == 0 ? 1 : 2; g_gd = gd;
            } else if (t < 4 * TY + 4 * TX) {                     // j-ghosts: bottom, top
                const int u0 = t - 4 * TY, side = u0 / (2 * TX), u = u0 - side * 2 * TX, gd = 1 + u / TX,
                          c = u - (gd - 1) * TX;
                const int jj = side == 0 ? -gd : nj - 1 + gd;
                valid = c < ncol && (side == 0 ? j0 == 0 : jj <= j0 + TY + 1);
                g_ii = i0 + c; g_jj = jj; g_f = side == 0 ? 3 : 4; g_gd = gd;
            }
            if (valid) {
                const int k = g_f <= 2 ? g_jj : g_ii;
                const int bi = g_f == 1 ? 0 : (g_f == 2 ? ni - 1 : g_ii), bj = g_f == 3 ? 0 : (g_f == 4 ? nj - 1 : g_jj);
                g_type = __ldg(&a.edges[B.eo[g_f - 1] + k].type);
                const double* gn = g_f <= 2 ? a.fi + B.ofi + (long long)bj * (ni + 1) + (g_f == 1 ? 0 : ni)
                                            : a.fj + B.ofj + (long long)(g_f == 3 ? 0 : nj) * ni + bi;
                const long long gs = g_f <= 2 ? B.pfi : B.pfj;
                g_nx = __ldg(gn);
                g_ny = __ldg(gn + gs);
                if (g_type == 101) ghost_value(a, B, g_ii, g_jj, g_q);   // Ghost_Connection: the donor's cells
            }
        }
        const bool arrived = mbar_wait(&barS, phS & 1u);
        phS += 1;
        // staged positions: state / lengths of cell (ii, jj) of the halo, face geometry
        const int* shSc = shS[cur];
        const int* shDc = shD[cur];
        const int* shGIc = shGI[cur];
        const int* shGJc = shGJ[cur];
        auto sidx = [&](int r, int ii) { return r * RW + (ii - i0 + 2) + shSc[r]; };   // r = jj - j0 + 2
        auto didx = [&](int r, int ii) { return r * RW + (ii - i0 + 2) + shDc[r]; };

        // ---- 2. ghost cells of the block edges the tile's stencils reach (Fill_Ghost_Cell) ------
        {
            if (g_type != -2) {
                double q[4];
                if (g_type == 101) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) q[v] = g_q[v];
                } else {
                    const int bi = g_f == 1 ? 0 : (g_f == 2 ? ni - 1 : g_ii), bj = g_f == 3 ? 0 : (g_f == 4 ? nj - 1 : g_jj);
                    const int di = g_f == 1 ? 1 : (g_f == 2 ? -1 : 0), dj = g_f == 3 ? 1 : (g_f == 4 ? -1 : 0);
                    const int rb = bj - j0 + 2;
                    const int sbc = sidx(rb, bi);
                    if (g_type == 300) {   // Ghost_Symmetry (Lib_Ghost.f90:163-196)
                        const double vx = sS[PS + sbc], vy = sS[2 * PS + sbc];
                        const double udotn = vx * g_nx + vy * g_ny;
                        q[0] = sS[sbc];
                        q[1] = vx - 2.0 * udotn * g_nx;
                        q[2] = vy - 2.0 * udotn * g_ny;
                        q[3] = sS[3 * PS + sbc];
                    } else if (g_type == 0 || g_type == 401 || g_type == 405 || g_type == 406 || g_type < 0) {
#pragma unroll
                        for (int v = 0; v < 4; ++v) q[v] = sS[v * PS + sbc];   // Ghost_ZG_Extrapolate
                    } else {   // Ghost_Extrapolate (Lib_Ghost.f90:270-299)
                        const int s1 = sidx(rb + dj, bi + di), s2 = sidx(rb + 2 * dj, bi + 2 * di);
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            const double b0 = sS[v * PS + sbc], i1 = sS[v * PS + s1], i2 = sS[v * PS + s2];
                            const double g1 = 3.0 * b0 - 3.0 * i1 + i2;
                            q[v] = g_gd == 1 ? g1 : 3.0 * g1 - 3.0 * b0 + i1;
                        }
                    }
                }
                const int sg = sidx(g_jj - j0 + 2, g_ii);
#pragma unroll
                for (int v = 0; v < 4; ++v) sS[v * PS + sg] = q[v];
                fence_proxy_async();   // before the next tile's bulk copies into these rows
            }
            if (__syncthreads_or(!arrived)) {
                // the copies did not complete within the wait: fail the case, let them land, stop
                if (tid == 0) record_error(cs, Q2D_ERR_TIMEOUT, B.local_b, i0 + 1, j0 + 1, a.irk);
                mbar_wait(&barS, (phS - 1) & 1u);
                mbar_wait(&barO, phO & 1u);
                return;
            }
        }
        if (pre) {   // next descriptor: block record and case status (the item arrived meanwhile)
            const int blk = __shfl_sync(0xffffffffu, pw, 0), cid = __shfl_sync(0xffffffffu, pw, 3);
            pb = lane < NBW ? __ldg(reinterpret_cast<const int*>(a.blocks + blk) + lane) : 0;
            ps = lane == 0 ? __ldcg(&a.cstate[cid].status) : 0;
        }

        // ---- 3. faces ---------------------------------------------------------------------------
        // Face tasks of a thread: 0 the west face of its cell, 1 its south face, 2 the north face
        // of a top-row cell (warp 0), the east face of a last-column cell (warp 1) or a boundary
        // face (warps 2 and up; block-interface faces run the interior scheme here, the other
        // boundary types below). One call site of the face routine serves every task.
        const int nl = (i0 == 0) ? nrow : 0;
        const int nr = (i0 + TX >= ni) ? nrow : 0;
        const int nb = (j0 == 0) ? ncol : 0;
        const int nt = (j0 + TY >= nj) ? ncol : 0;
        const int nbf = nl + nr + nb + nt;
        int bFm = 0, bk = 0, bslot = -1, btype = -1, bparam = -1;   // the boundary face of task 2
        if (warp >= 2 && tid - 64 < nbf) {
            boundary_face_slot<TX>(tid - 64, nl, nr, nb, i0, j0, ni, nj, NFI, bFm, bk, bslot);
            const EdgeRec* er = &a.edges[B.eo[bFm - 1] + bk];
            btype = __ldg(&er->type);
            bparam = __ldg(&er->param);
        }
        static_assert(2 * TY + 4 * TX <= NT - 64, "one boundary face per thread of warps 2 and up");
#pragma unroll 1
        for (int task = 0; task < 3; ++task) {
            bool idir, on;
            int fr, fc, slot, ei, ej;   // face row / column in the tile, flux slot, error cell
            if (task == 0) {
                idir = true; fr = row; fc = col; on = j0 + row < nj && i0 + col > 0 && i0 + col < ni;
            } else if (task == 1) {
                idir = false; fr = row; fc = col; on = i0 + col < ni && j0 + row > 0 && j0 + row < nj;
            } else if (warp == 0) {
                idir = false; fr = TY; fc = lane; on = i0 + lane < ni && j0 + TY < nj;
            } else if (warp == 1) {
                idir = true; fr = lane; fc = TX; on = lane < TY && j0 + lane < nj && i0 + TX < ni;
            } else {
                on = btype == 101;
                idir = bFm <= 2;
                fr = bFm <= 2 ? bk - j0 : (bFm == 3 ? 0 : nj - j0);
                fc = bFm <= 2 ? (bFm == 1 ? 0 : ni - i0) : bk - i0;
            }
            if (!on) continue;
            int o0, o1, o2, o3, e0, e1, e2, e3, gk;
            const double* gb;
            int gp;
            if (idir) {   // i face F = i0 + fc of tile row fr: cells F-2 .. F+1 of staged row fr + 2
                const int sr = fr + 2, F = i0 + fc;
                o1 = sidx(sr, F - 1); o0 = o1 - 1; o2 = o1 + 1; o3 = o1 + 2;
                e1 = didx(sr, F - 1); e0 = e1 - 1; e2 = e1 + 1; e3 = e1 + 2;
                gk = fr * RGI + fc + shGIc[fr];
                gb = sGI; gp = L::PGI;
                slot = fr * (TX + 1) + fc;
                ei = F; ej = j0 + fr + 1;
            } else {      // j face G = j0 + fr of tile column fc: rows G-2 .. G+1 (staged rows fr .. fr+3)
                const int ii = i0 + fc;
                o0 = sidx(fr, ii); o1 = sidx(fr + 1, ii); o2 = sidx(fr + 2, ii); o3 = sidx(fr + 3, ii);
                e0 = didx(fr, ii); e1 = didx(fr + 1, ii); e2 = didx(fr + 2, ii); e3 = didx(fr + 3, ii);
                gk = fr * RGJ + fc + shGJc[fr];
                gb = sGJ; gp = L::PGJ;
                slot = NFI + fr * TX + fc;
                ei = ii + 1; ej = j0 + fr;
            }
            if (task == 2 && warp >= 2) { slot = bslot; ei = (bFm == 2 ? ni : (bFm == 1 ? 1 : bk + 1)); ej = (bFm == 4 ? nj : (bFm == 3 ? 1 : bk + 1)); }
            const double nx = gb[gk], ny = gb[gp + gk], ln = gb[2 * gp + gk];
            const float* dlf = reinterpret_cast<const float*>(sD) + (idir ? 0 : 1);
            double X[4];
            bool ok;
            ok = face_df<RIEM, LIM, PS>(sS, o0, o1, o2, o3, dlf, e0, e1, e2, e3, nx, ny, ln, g, gam, gm1, gf, X);
            if (!ok) record_error(cs, 4, B.local_b, ei, ej, a.irk);
#pragma unroll
            for (int v = 0; v < 4; ++v) sF[v * NF + slot] = X[v];
        }
        if (btype >= 0 && btype != 101) {   // the other boundary faces (BC_Fluxes dispatch)
            const int Fm = bFm, k = bk;
            const int bi = Fm == 1 ? 0 : (Fm == 2 ? ni - 1 : k), bj = Fm == 3 ? 0 : (Fm == 4 ? nj - 1 : k);
            const int di = Fm == 1 ? 1 : (Fm == 2 ? -1 : 0), dj = Fm == 3 ? 1 : (Fm == 4 ? -1 : 0);
            double nx, ny, ln;
            if (Fm <= 2) {
                const int gk = (bj - j0) * RGI + ((Fm == 1 ? 0 : ni) - i0) + shGIc[bj - j0];
                nx = sGI[gk]; ny = sGI[L::PGI + gk]; ln = sGI[2 * L::PGI + gk];
            } else {
                const int gr = (Fm == 3 ? 0 : nj) - j0;
                const int gk = gr * RGJ + (bi - i0) + shGJc[gr];
                nx = sGJ[gk]; ny = sGJ[L::PGJ + gk]; ln = sGJ[2 * L::PGJ + gk];
            }
            const int rb = bj - j0 + 2;
            const int cb = sidx(rb, bi), ci = sidx(rb + dj, bi + di);
            const int db = didx(rb, bi), dci = didx(rb + dj, bi + di);
            double Bq[4], Iq[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { Bq[v] = sS[v * PS + cb]; Iq[v] = sS[v * PS + ci]; }
            const float dlb = Fm <= 2 ? sD[db].x : sD[db].y, dli = Fm <= 2 ? sD[dci].x : sD[dci].y;
            double X[4] = {0.0, 0.0, 0.0, 0.0};
            bool sym = btype == 300;
            if (btype == 400) {
                bc_extrapolation(g, Bq, nx, ny, ln, X);
            } else if (btype == 401) {   // stagnation inflow, or the symmetry flux on reverse flow
                const double un = Bq[1] * nx + Bq[2] * ny;
                const double sgn = (Fm & 1) ? -1.0 : 1.0;
                if (sgn * un >= 0.0) sym = true;
            }
            if (sym) {
                bc_symmetry_df<RIEM, LIM>(Fm, Bq, Iq, dlb, dli, nx, ny, ln, g, gam, gm1, gf, X);
            } else if (btype != 400 && btype > 0) {
                // inflow / outflow records in FP64 from the FP64 state (the reference's routines);
                // the flux through an inlet is the large term of a nozzle's balance
                Q4 Bp, Ip;
#pragma unroll
                for (int v = 0; v < 4; ++v) { Bp.v[v] = Bq[v]; Ip.v[v] = Iq[v]; }
                const double* dlp = a.dl + B.og + (long long)(Fm <= 2 ? 0 : 1) * B.pg;
                const int ni2 = bi + di, nj2 = bj + dj;
                const double dlbv = __ldg(dlp + (long long)(bj + 2) * (ni + 4) + (bi + 2));
                const double dliv = __ldg(dlp + (long long)(nj2 + 2) * (ni + 4) + (ni2 + 2));
                const Q4 qf = bc_face<RIEM>(a.gas, a.limiter, btype, Fm, Bp, Ip, dlbv, dliv, nx, ny, ln,
                                            bparam >= 0 ? a.bcp + bparam : nullptr);
#pragma unroll
                for (int v = 0; v < 4; ++v) X[v] = qf.v[v];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) sF[v * NF + bslot] = X[v];
        }
        // the cell's own state and lengths leave the staged rows before the next tile's copies
        const bool mine = row < TY && row < nrow && col < ncol;
        double P[4] = {0.0, 0.0, 0.0, 0.0};
        float2 dd = make_float2(0.0f, 0.0f);
        if (mine) {
            const int sc0 = sidx(row + 2, i0 + col);
#pragma unroll
            for (int v = 0; v < 4; ++v) P[v] = sS[v * PS + sc0];
            dd = sD[didx(row + 2, i0 + col)];
        }
        if (pre) {   // store the next descriptor; the barrier below publishes it
            if (lane < NWW) reinterpret_cast<int*>(&sW[cur ^ 1])[lane] = pw;
            if (lane < NBW) reinterpret_cast<int*>(&sBk[cur ^ 1])[lane] = pb;
            if (lane == 0) sSt[cur ^ 1] = ps;
        }
        __syncthreads();
        // the next item's stencil rows, while this tile's cells update
        const bool next_run = nit < a.n_items && sSt[cur ^ 1] == kStatus_Running;
        if (next_run) issue_stencil(sW[cur ^ 1], sBk[cur ^ 1], cur ^ 1);
        // each thread reads only its own cell's rows: no CTA barrier needed before the cell phase
        // (a copy that did not land fails the case at the end of the tile)
        const bool own_ok = mbar_wait(&barO, phO & 1u);
        phO += 1;

        // ---- 4. residual, sources, RK update (+ time step and residual norm) --------------------
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 1e300};
        const double dt_case = sCase[cur][0];   // CaseState.dt_step
        const long long iter_dt = *reinterpret_cast<const long long*>(&sCase[cur][9]) + (dt_here || a.first ? 1 : 0) +
                                  (dt_here ? 0 : 1);   // CaseState.iter
        if (mine) {
            const int ii = i0 + col, jj = j0 + row;
            const long long cg = (long long)jj * ni + ii;
            const int ok0 = row * RO + col + shO[cur][row];
            const int i1 = ii + 1, j1 = jj + 1;
            const int fi0 = row * (TX + 1) + col, fj0 = NFI + row * TX + col;
            double r[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {   // interior i, interior j, then boundary faces 1..4
                const double* Fv = sF + v * NF;
                const double wv = Fv[fi0], ev = Fv[fi0 + 1], so = Fv[fj0], no = Fv[fj0 + TX];
                double x = 0.0;
                if (i1 > 1) x = x - wv;
                if (i1 < ni) x = x + ev;
                if (j1 > 1) x = x - so;
                if (j1 < nj) x = x + no;
                if (i1 == 1) x = x - wv;
                if (i1 == ni) x = x + ev;
                if (j1 == 1) x = x - so;
                if (j1 == nj) x = x + no;
                r[v] = x;
            }
            const double sur = sO[4 * L::PO + ok0];
            if (a.source) {
                // S = [rho, rho u, rho v, rho E0 + p] * f0 with f0 = -v/r (Lib_Source_Axisymmetry.f90:
                // 65-76) or V.G (Lib_Source_Areavariation.f90:120-142); Res -= S * sur
                const double rE0 = P[3] * g.igm1 + 0.5 * P[0] * (P[1] * P[1] + P[2] * P[2]);
                const double f0 = a.source == 1 ? -P[2] * sO[6 * L::PO + ok0]
                                                : P[1] * sO[6 * L::PO + ok0] + P[2] * sO[7 * L::PO + ok0];
                const double fs = f0 * sur;
                r[0] = r[0] - P[0] * fs;
                r[1] = r[1] - P[0] * P[1] * fs;
                r[2] = r[2] - P[0] * P[2] * fs;
                r[3] = r[3] - (rE0 + P[3]) * fs;
            }
            double dt;
            if (dt_here) {
                // Compute_dt (Mod_dt.f90:59-104) from the step's starting state, FP32 arithmetic
                const float dtc = cell_dt32((float)P[0], (float)P[1], (float)P[2], (float)P[3], gam, (float)a.cfl,
                                            ndir, dd.x, dd.y, (float)sO[ok0], (float)sO[L::PO + ok0],
                                            ndir == 2 ? (float)sO[2 * L::PO + ok0] : 0.0f,
                                            ndir == 2 ? (float)sO[3 * L::PO + ok0] : 0.0f);
                dt = (double)dtc;
                if (iter_dt < a.rampa) dt = dt * (double)iter_dt / (double)a.rampa;
                if (!a.last) a.sc[2 * B.oc + pc + cg] = dt;   // for the later stages
                acc[4] = fmin(acc[4], dt);
            } else {
                dt = a.time_accurate ? dt_case : sO[5 * L::PO + ok0];
            }
            const double fr = -dt * rcp64(sur);
            double q[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) q[v] = r[v] * fr;
            double PO[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) PO[v] = a.first ? P[v] : sO[v * L::PO + ok0];
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
                    const float dtc = cell_dt32((float)N[0], (float)N[1], (float)N[2], (float)N[3], gam,
                                                (float)a.cfl, ndir, dd.x, dd.y, (float)scb[2 * pc + cg],
                                                (float)scb[3 * pc + cg], ndir == 2 ? (float)scb[4 * pc + cg] : 0.0f,
                                                ndir == 2 ? (float)scb[5 * pc + cg] : 0.0f);
                    double dtn = (double)dtc;
                    if (iter_dt < a.rampa) dtn = dtn * (double)iter_dt / (double)a.rampa;
                    if (!a.time_accurate) a.sc[2 * B.oc + pc + cg] = dtn;
                    acc[4] = fmin(acc[4], dtn);
                }
            }
        }
        // per-warp partials: residual sums (last stage), dt min (the stage that computes it)
        const bool need_dt = a.dt_first ? dt_here : a.last;
        if (a.last) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                double v = acc[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                acc[k] = v;
            }
        }
        if (need_dt) {
            double v = acc[4];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
            acc[4] = v;
        }
        if (lane == 0 && (a.last || need_dt)) {
            double* pp = a.part + ((size_t)it * (NT / 32) + warp) * 5;
            if (a.last)
                for (int k = 0; k < 4; ++k) pp[k] = acc[k];
            if (need_dt) pp[4] = acc[4];
        }
        // end of the item (stage_item_end for a kernel whose case finalisation is separate): the
        // step prologue from the case's first item when the time steps are not computed in the
        // first stage, then the barrier that frees the tile's buffers
        if (a.first && !a.dt_first && tid == 0 && it == a.cases[w.case_id].item_begin) step_prologue(a, w.case_id);
        if (__syncthreads_or(!own_ok)) {
            if (tid == 0) record_error(cs, Q2D_ERR_TIMEOUT, B.local_b, i0 + 1, j0 + 1, a.irk);
            mbar_wait(&barO, (phO - 1) & 1u);
            if (next_run) mbar_wait(&barS, phS & 1u);
            return;
        }
        // the next item's own-cell rows, once every cell of this tile has read its own
        if (next_run) issue_own(sW[cur ^ 1], sBk[cur ^ 1], cur ^ 1);
        s_pre = o_pre = next_run;
    }
}

template <int RIEM, int LIM, int TX, int TY, int NT, int MB>
cudaError_t launch_stage32d_l(const StageArgs& a, int grid, cudaStream_t s) {
    constexpr size_t smem = dform::TileD<TX, TY>::bytes;
    auto k = stage32d_kernel<RIEM, LIM, TX, TY, NT, MB>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

// One instantiation per limiter (a.limiter), so that each kernel holds one copy of the face code.
template <int RIEM, int TX, int TY, int NT, int MB>
cudaError_t launch_stage32d_t(const StageArgs& a, int grid, cudaStream_t s) {
    switch (a.limiter) {
        case 0: return launch_stage32d_l<RIEM, 0, TX, TY, NT, MB>(a, grid, s);
        case 1: return launch_stage32d_l<RIEM, 1, TX, TY, NT, MB>(a, grid, s);
        case 2: return launch_stage32d_l<RIEM, 2, TX, TY, NT, MB>(a, grid, s);
        case 3: return launch_stage32d_l<RIEM, 3, TX, TY, NT, MB>(a, grid, s);
        case 4: return launch_stage32d_l<RIEM, 4, TX, TY, NT, MB>(a, grid, s);
        case 5: return launch_stage32d_l<RIEM, 5, TX, TY, NT, MB>(a, grid, s);
        default: return launch_stage32d_l<RIEM, 6, TX, TY, NT, MB>(a, grid, s);
    }
}

template <int RIEM, int TX, int TY, int NT, int MB>
int stage32d_occupancy_t() {
    constexpr size_t smem = dform::TileD<TX, TY>::bytes;
    auto k = stage32d_kernel<RIEM, 2, TX, TY, NT, MB>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, smem);
    return n;
}

}  // namespace q2d
