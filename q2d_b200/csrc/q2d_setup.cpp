// q2d_setup.cpp — host-side geometry setup (Setup_Metrics and the ghost-cell metrics of
// Lib_Metrics.f90). Built with -ffp-contract=off: setup arithmetic is plain IEEE double.
#include "q2d_setup.h"

#include <algorithm>
#include <cmath>

namespace q2d {
namespace {

struct P2 { double x, y; };

inline P2 node(const double* nodes, int ni, int i, int j) {
    const double* p = nodes + 2 * ((long long)i + (long long)(ni + 1) * j);
    return P2{p[0], p[1]};
}

// Compute_Metric_Tensor (Lib_Metrics.f90:125-189)
int metric(P2 N1, P2 N2, P2 N3, P2 N4, double* M, double* dl, double* sur) {
    double a00 = N4.x - N2.x + N3.x - N1.x, a01 = N4.y - N2.y + N3.y - N1.y;
    double a10 = N4.x - N3.x + N2.x - N1.x, a11 = N4.y - N3.y + N2.y - N1.y;
    a00 = 0.5 * a00; a01 = 0.5 * a01; a10 = 0.5 * a10; a11 = 0.5 * a11;
    const double det = a00 * a11 - a01 * a10;
    if (std::fabs(det) == 0.0) return Q2D_ERR_BADARG;
    M[0] = a11 / det;
    M[1] = -a10 / det;
    M[2] = -a01 / det;
    M[3] = a00 / det;
    dl[0] = std::sqrt(a00 * a00 + a01 * a01);
    dl[1] = std::sqrt(a10 * a10 + a11 * a11);
    const double cross = (N4.x - N1.x) * (N3.y - N2.y) - (N4.y - N1.y) * (N3.x - N2.x);
    *sur = 0.5 * std::fabs(cross);
    return *sur <= 0.0 ? Q2D_ERR_BADARG : Q2D_OK;
}

int metric_at(HostGeom& G, int i1, int j1, P2 N1, P2 N2, P2 N3, P2 N4) {
    // i1, j1 are 1-based cell indices (ghosts allowed)
    const int k = G.g(i1 - 1, j1 - 1);
    return metric(N1, N2, N3, N4, &G.M[4 * k], &G.dl[2 * k], &G.sur[k]);
}

inline P2 q3(P2 a, P2 b, P2 c) { return P2{3.0 * a.x - 3.0 * b.x + c.x, 3.0 * a.y - 3.0 * b.y + c.y}; }
inline P2 l2(P2 a, P2 b) { return P2{2.0 * a.x - b.x, 2.0 * a.y - b.y}; }

}  // namespace

SetupPool& SetupPool::get() {
    static SetupPool pool;
    return pool;
}

SetupPool::SetupPool() {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int n = std::min(15, hw - 1);
    for (int k = 0; k < n; ++k) th_.emplace_back([this] { loop(); });
}

SetupPool::~SetupPool() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
}

void SetupPool::loop() {
    unsigned long long seen = 0;
    for (;;) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        while (next_ < T_) {   // take chunks 1..T-1 of this generation
            const int t = next_++;
            const std::function<void(int)>* fn = fn_;
            lk.unlock();
            (*fn)(t);
            lk.lock();
            if (--pending_ == 0) done_cv_.notify_one();
        }
    }
}

void SetupPool::run(int T, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> serial(run_mu_);
    {
        std::lock_guard<std::mutex> lk(mu_);
        fn_ = &fn;
        T_ = T;
        next_ = 1;
        pending_ = T - 1;
        ++gen_;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    while (next_ < T_) {   // help with chunks no worker has taken yet
        const int t = next_++;
        lk.unlock();
        fn(t);
        lk.lock();
        --pending_;
    }
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    fn_ = nullptr;
    T_ = 0;
}

int setup_block(int ni, int nj, const double* nodes, const double* area, int source, HostGeom& G,
                const FaceOut* out) {
    G.ni = ni;
    G.nj = nj;
    const size_t ng = (size_t)(ni + 4) * (nj + 4);
    G.M.resize(4 * ng);
    G.dl.resize(2 * ng);
    G.sur.resize(ng);
    // ghost-frame rows in parallel: zeroed, then the interior cells' metrics
    std::vector<int> row_err((size_t)nj + 4, Q2D_OK);
    parallel_rows(nj + 4, 8L * (ni + 4), [&](long long r0, long long r1) {
        for (long long r = r0; r < r1; ++r) {
            const size_t k0 = (size_t)r * (ni + 4), k1 = k0 + (ni + 4);
            std::fill(G.M.begin() + 4 * k0, G.M.begin() + 4 * k1, 0.0);
            std::fill(G.dl.begin() + 2 * k0, G.dl.begin() + 2 * k1, 0.0);
            std::fill(G.sur.begin() + k0, G.sur.begin() + k1, 0.0);
            const int j = (int)r - 1;   // 1-based interior row of frame row r
            if (j < 1 || j > nj) continue;
            for (int i = 1; i <= ni; ++i) {
                const int e = metric_at(G, i, j, node(nodes, ni, i - 1, j - 1), node(nodes, ni, i - 1, j),
                                        node(nodes, ni, i, j - 1), node(nodes, ni, i, j));
                if (e) { row_err[(size_t)r] = e; break; }
            }
        }
    });
    for (int e : row_err)
        if (e) return e;
    // Compute_Norm_Area (Lib_Metrics.f90:41-122): one orientation sign per direction
    auto X = [&](int i, int j) { return node(nodes, ni, i, j); };
    double sgn_i, sgn_j;
    {
        const double dx = X(1, 1).x - X(1, 0).x, dy = X(1, 1).y - X(1, 0).y;
        const double sx = dy, sy = -dx;
        const double cx = 0.5 * (X(1, 1).x + X(1, 0).x) - 0.5 * (X(0, 1).x + X(0, 0).x);
        const double cy = 0.5 * (X(1, 1).y + X(1, 0).y) - 0.5 * (X(0, 1).y + X(0, 0).y);
        sgn_i = std::copysign(1.0, cx * sx + cy * sy);
    }
    {
        const double dx = X(0, 1).x - X(1, 1).x, dy = X(0, 1).y - X(1, 1).y;
        const double sx = dy, sy = -dx;
        const double cx = 0.5 * (X(1, 1).x + X(0, 1).x) - 0.5 * (X(1, 0).x + X(0, 0).x);
        const double cy = 0.5 * (X(1, 1).y + X(0, 1).y) - 0.5 * (X(1, 0).y + X(0, 0).y);
        sgn_j = std::copysign(1.0, cx * sx + cy * sy);
    }
    // a face's (nx, ny, len) into G's AoS arrays, or into the device images (planes + float4)
    auto put = [](double* aos, double* planes, long long pstride, float* f4, long long k, double nx, double ny,
                  double len) {
        if (planes) {
            planes[k] = nx;
            planes[pstride + k] = ny;
            planes[2 * pstride + k] = len;
            if (f4) {
                f4[4 * k] = (float)nx;
                f4[4 * k + 1] = (float)ny;
                f4[4 * k + 2] = (float)len;
                f4[4 * k + 3] = 0.0f;
            }
        } else {
            aos[3 * k] = nx;
            aos[3 * k + 1] = ny;
            aos[3 * k + 2] = len;
        }
    };
    if (out) {
        G.fi.clear();
        G.fj.clear();
    } else {
        G.fi.resize(3 * (size_t)(ni + 1) * nj);
        G.fj.resize(3 * (size_t)ni * (nj + 1));
    }
    parallel_rows(nj, 24L * (ni + 1), [&](long long r0, long long r1) {
        for (int j = (int)r0 + 1; j <= (int)r1; ++j)
            for (int F = 0; F <= ni; ++F) {
                const double dx = X(F, j).x - X(F, j - 1).x, dy = X(F, j).y - X(F, j - 1).y;
                const double sx = dy, sy = -dx;
                const double A = std::sqrt(sx * sx + sy * sy);
                put(G.fi.data(), out ? out->fi : nullptr, out ? out->pfi : 0, out ? out->fi4 : nullptr,
                    (long long)(j - 1) * (ni + 1) + F, A == 0.0 ? 0.0 : sx / A * sgn_i,
                    A == 0.0 ? 0.0 : sy / A * sgn_i, A);
            }
    });
    parallel_rows(nj + 1, 24L * ni, [&](long long r0, long long r1) {
        for (int Gf = (int)r0; Gf < (int)r1; ++Gf)
            for (int i = 1; i <= ni; ++i) {
                const double dx = X(i - 1, Gf).x - X(i, Gf).x, dy = X(i - 1, Gf).y - X(i, Gf).y;
                const double sx = dy, sy = -dx;
                const double A = std::sqrt(sx * sx + sy * sy);
                put(G.fj.data(), out ? out->fj : nullptr, out ? out->pfj : 0, out ? out->fj4 : nullptr,
                    (long long)Gf * ni + (i - 1), A == 0.0 ? 0.0 : sx / A * sgn_j, A == 0.0 ? 0.0 : sy / A * sgn_j,
                    A);
            }
    });
    // source geometry (Precompute_Axisymmetric_Geometry / Precompute_Area_Geometry)
    const size_t n = (size_t)ni * nj;
    G.src0.resize(n);
    G.src1.resize(n);
    parallel_rows(nj, 16L * ni, [&](long long r0, long long r1) {
        for (int j = (int)r0 + 1; j <= (int)r1; ++j)
            for (int i = 1; i <= ni; ++i) {
                const size_t k = (size_t)(j - 1) * ni + (i - 1);
                double s0 = 0.0, s1 = 0.0;
                if (source == Q2D_SRC_AXI) {
                    const double r = 0.25 * (X(i, j).y + X(i - 1, j).y + X(i, j - 1).y + X(i - 1, j - 1).y);
                    s0 = 1.0 / (r > 1e-12 ? r : 1e-12);
                } else if (source == Q2D_SRC_AREA && area) {
                    auto A = [&](int a, int b) { return area[(size_t)a + (size_t)(ni + 1) * b]; };
                    const double d0 = 0.5 * ((A(i, j) - A(i - 1, j)) + (A(i, j - 1) - A(i - 1, j - 1)));
                    const double d1 = 0.5 * ((A(i, j) - A(i, j - 1)) + (A(i - 1, j) - A(i - 1, j - 1)));
                    const double* M = &G.M[4 * G.g(i - 1, j - 1)];
                    const double g0 = d0 * M[0] + d1 * M[2];
                    const double g1 = d0 * M[1] + d1 * M[3];
                    const double Ac = 0.25 * (A(i, j) + A(i - 1, j) + A(i, j - 1) + A(i - 1, j - 1));
                    const double den = Ac > 1e-12 ? Ac : 1e-12;
                    s0 = -g0 / den;
                    s1 = -g1 / den;
                }
                G.src0[k] = s0;
                G.src1[k] = s1;
            }
    });
    return Q2D_OK;
}

int ghost_metrics(const q2d_bc_rec& r, int ni, int nj, const double* nodes, HostGeom& G,
                  int dni, int dnj, const double* donor) {
    const int Im = r.i, Jm = r.j, Fm = r.f;
    auto X = [&](int i, int j) { return node(nodes, ni, i, j); };
    int e = Q2D_OK;
    if (r.type == 300) {   // BC_Symmetry_Metrics (Lib_Metrics.f90:398-441)
        for (int g = 1; g <= 2; ++g) {
            int di, dj, si, sj;
            switch (Fm) {
                case 1: di = Im - g; dj = Jm; si = Im + g - 1; sj = Jm; break;
                case 2: di = Im + g; dj = Jm; si = Im - g + 1; sj = Jm; break;
                case 3: di = Im; dj = Jm - g; si = Im; sj = Jm + g - 1; break;
                default: di = Im; dj = Jm + g; si = Im; sj = Jm - g + 1; break;
            }
            const int kd = G.g(di - 1, dj - 1), ks = G.g(si - 1, sj - 1);
            for (int q = 0; q < 4; ++q) G.M[4 * kd + q] = G.M[4 * ks + q];
            for (int q = 0; q < 2; ++q) G.dl[2 * kd + q] = G.dl[2 * ks + q];
            G.sur[kd] = G.sur[ks];
        }
        return Q2D_OK;
    }
    if (r.type == 101 || r.type == 201) {
        // BC_Connect_Metrics (Lib_Metrics.f90:444-553); for a translational periodic seam (201)
        // BC_Connect_Metrics_Periodic (:556-700): the donor nodes moved by the rigid offset T
        // that brings the donor's seam onto this block's, so that the ghost cells are the
        // donor's cells, not a quadrilateral folded across the domain
        static const int gd[5][2] = {{0, 0}, {0, 0}, {-1, 0}, {0, 0}, {0, -1}};
        static const int gd2[5][2] = {{0, 0}, {1, 0}, {-2, 0}, {0, 1}, {0, -2}};
        auto D = [&](int i, int j) { return node(donor, dni, i, j); };
        P2 A0, B0;   // the two seam nodes of this block (roles per face below)
        switch (Fm) {
            case 1: A0 = X(Im - 1, Jm - 1); B0 = X(Im - 1, Jm); break;
            case 2: A0 = X(Im, Jm - 1); B0 = X(Im, Jm); break;
            case 3: A0 = X(Im - 1, Jm - 1); B0 = X(Im, Jm - 1); break;
            default: A0 = X(Im - 1, Jm); B0 = X(Im, Jm); break;
        }
        // donor nodes of step g of the recurrence: a pairs with B0's role, b with A0's
        auto donor_nodes = [&](int g, int& II, int& JJ, int& III, int& JJJ) {
            const int Is1 = r.is + (2 - g) * gd[r.fs][0] + (g - 1) * gd2[r.fs][0];
            const int Js1 = r.js + (2 - g) * gd[r.fs][1] + (g - 1) * gd2[r.fs][1];
            if (r.fs <= 2) { II = Is1; JJ = (2 * Js1 + r.d11 + r.d21) / 2; III = II; JJJ = JJ - r.d11; }
            else { II = (2 * Is1 + r.d11 + r.d21) / 2; JJ = Js1; III = II - r.d11; JJJ = JJ; }
            return !(II < 0 || II > dni || JJ < 0 || JJ > dnj || III < 0 || III > dni || JJJ < 0 || JJJ > dnj);
        };
        P2 T{0.0, 0.0};
        if (r.type == 201) {   // T from the seam (step g = 0); it must be one rigid translation
            int II, JJ, III, JJJ;
            if (!donor_nodes(0, II, JJ, III, JJJ)) return Q2D_ERR_BADARG;
            const P2 a = D(II, JJ), b = D(III, JJJ);
            T = P2{B0.x - a.x, B0.y - a.y};
            const P2 T2{A0.x - b.x, A0.y - b.y};
            const double big = 1.0 + std::max(std::fabs(T.x), std::fabs(T.y));
            if (std::max(std::fabs(T.x - T2.x), std::fabs(T.y - T2.y)) > 1e-10 * big) return Q2D_ERR_BADARG;
        }
        P2 Ap = A0, Bp = B0;
        for (int g = 1; g <= 2; ++g) {
            int II, JJ, III, JJJ;
            if (!donor_nodes(g, II, JJ, III, JJJ)) return Q2D_ERR_BADARG;
            P2 a = D(II, JJ), b = D(III, JJJ);
            if (r.type == 201) {
                a = P2{a.x + T.x, a.y + T.y};
                b = P2{b.x + T.x, b.y + T.y};
            }
            // a replaces the node paired with B0, b the node paired with A0 (N2/N1, N4/N3, ...)
            switch (Fm) {
                case 1: e |= metric_at(G, Im - g, Jm, b, a, Ap, Bp); break;   // (N1g,N2g,N1g-1,N2g-1)
                case 2: e |= metric_at(G, Im + g, Jm, Ap, Bp, b, a); break;   // (N3g-1,N4g-1,N3g,N4g)
                case 3: e |= metric_at(G, Im, Jm - g, b, Ap, a, Bp); break;   // (N1g,N1g-1,N3g,N3g-1)
                default: e |= metric_at(G, Im, Jm + g, Ap, b, Bp, a); break;  // (N2g-1,N2g,N4g-1,N4g)
            }
            Ap = b;
            Bp = a;
        }
        return e;
    }
    // BC_Extrapolate_Metrics (Lib_Metrics.f90:285-395): every other type
    P2 U[5], V[5];   // index g+2, g in [-2, 2]
    auto u = [&](int g) -> P2& { return U[g + 2]; };
    auto v = [&](int g) -> P2& { return V[g + 2]; };
    switch (Fm) {
        case 1:
            for (int g = 0; g <= 2; ++g) { u(g) = X(Im + g - 1, Jm - 1); v(g) = X(Im + g - 1, Jm); }
            for (int g = -1; g >= -2; --g) {
                u(g) = q3(u(g + 1), u(g + 2), u(g + 3));
                v(g) = q3(v(g + 1), v(g + 2), v(g + 3));
                e |= metric_at(G, Im + g, Jm, u(g), v(g), u(g + 1), v(g + 1));
            }
            break;
        case 2:
            for (int g = 0; g >= -2; --g) { u(g) = X(Im + g, Jm - 1); v(g) = X(Im + g, Jm); }
            for (int g = 1; g <= 2; ++g) {
                u(g) = q3(u(g - 1), u(g - 2), u(g - 3));
                v(g) = q3(v(g - 1), v(g - 2), v(g - 3));
                e |= metric_at(G, Im + g, Jm, u(g - 1), v(g - 1), u(g), v(g));
            }
            break;
        case 3:
            if (nj > 2) {
                for (int g = 0; g <= 2; ++g) { u(g) = X(Im - 1, Jm + g - 1); v(g) = X(Im, Jm + g - 1); }
                for (int g = -1; g >= -2; --g) {
                    u(g) = q3(u(g + 1), u(g + 2), u(g + 3));
                    v(g) = q3(v(g + 1), v(g + 2), v(g + 3));
                    e |= metric_at(G, Im, Jm + g, u(g), u(g + 1), v(g), v(g + 1));
                }
            } else {
                for (int g = 0; g <= 1; ++g) { u(g) = X(Im - 1, Jm + g - 1); v(g) = X(Im, Jm + g - 1); }
                for (int g = -1; g >= -2; --g) {
                    u(g) = l2(u(g + 1), u(g + 2));
                    v(g) = l2(v(g + 1), v(g + 2));
                    e |= metric_at(G, Im, Jm + g, u(g), u(g + 1), v(g), v(g + 1));
                }
            }
            break;
        default:
            if (nj > 2) {
                for (int g = 0; g >= -2; --g) { u(g) = X(Im - 1, Jm + g); v(g) = X(Im, Jm + g); }
                for (int g = 1; g <= 2; ++g) {
                    u(g) = q3(u(g - 1), u(g - 2), u(g - 3));
                    v(g) = q3(v(g - 1), v(g - 2), v(g - 3));
                    e |= metric_at(G, Im, Jm + g, u(g - 1), u(g), v(g - 1), v(g));
                }
            } else {
                for (int g = 0; g >= -1; --g) { u(g) = X(Im - 1, Jm + g); v(g) = X(Im, Jm + g); }
                for (int g = 1; g <= 2; ++g) {
                    u(g) = l2(u(g - 1), u(g - 2));
                    v(g) = l2(v(g - 1), v(g - 2));
                    e |= metric_at(G, Im, Jm + g, u(g - 1), u(g), v(g - 1), v(g));
                }
            }
            break;
    }
    return e;
}

void face_tangent(const q2d_bc_rec& r, int ni, const double* nodes, double* t0, double* t1) {
    double tx, ty;
    if (r.f <= 2) {
        const int Fi = r.i - (r.f % 2), Fj = r.j;
        const P2 a = node(nodes, ni, Fi, Fj), b = node(nodes, ni, Fi, Fj - 1);
        tx = a.x - b.x; ty = a.y - b.y;
    } else {
        const int Fi = r.i, Fj = r.j - (r.f % 2);
        const P2 a = node(nodes, ni, Fi, Fj), b = node(nodes, ni, Fi - 1, Fj);
        tx = a.x - b.x; ty = a.y - b.y;
    }
    const double m = std::sqrt(tx * tx + ty * ty);
    *t0 = tx / m;
    *t1 = ty / m;
}

void versors(const HostGeom& G, int i, int j, double* v) {
    const double* M = &G.M[4 * G.g(i, j)];
    for (int d = 0; d < 2; ++d) {
        const double m0 = M[2 * d], m1 = M[2 * d + 1];
        const double nrm = std::sqrt(m0 * m0 + m1 * m1);
        v[2 * d] = m0 / nrm;
        v[2 * d + 1] = m1 / nrm;
    }
}

}  // namespace q2d
