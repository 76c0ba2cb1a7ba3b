// q2d_setup.h — host-side geometry setup of one block (Setup_Metrics, Mod_Metrics.f90:11-148).
// Setup runs once per block on the host, in IEEE double arithmetic without FMA contraction,
// and produces the SoA planes the device kernels read.
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>
#include "../../include/q2d_gpu.h"

namespace q2d {

// Vector whose resize() leaves new elements uninitialised: the setup arrays are written (or
// zeroed) by the parallel loops that fill them, not first by a serial zero fill.
template <class T>
struct DefaultInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = DefaultInitAlloc<U>; };
    DefaultInitAlloc() = default;
    template <class U>
    DefaultInitAlloc(const DefaultInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) { ::new ((void*)p) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
};
using dvec = std::vector<double, DefaultInitAlloc<double>>;
using fvec = std::vector<float, DefaultInitAlloc<float>>;

// Host worker threads of the setup loops (created on first use, up to 15 besides the caller).
// run(T, fn) calls fn(t) for t in [0, T) with t = 0 on the calling thread and returns when
// every call has finished; concurrent run() calls from different host threads are serialised.
class SetupPool {
public:
    static SetupPool& get();
    int workers() const { return (int)th_.size(); }
    void run(int T, const std::function<void(int)>& fn);
    ~SetupPool();
private:
    SetupPool();
    std::vector<std::thread> th_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    int T_ = 0, next_ = 0, pending_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
    void loop();
};

// Runs body(r0, r1) over contiguous ranges covering [0, n): on up to 16 host threads when
// n * cost_per_row is large, else on the calling thread. Every range is independent of the
// others, so the results do not depend on the split. body must not throw.
template <class F>
void parallel_rows(long long n, long long cost_per_row, F&& body) {
    SetupPool& pool = SetupPool::get();
    const long long T = std::min({(long long)pool.workers() + 1, n * cost_per_row / 200000 + 1, std::max(n, 1LL)});
    if (T <= 1) {
        body(0LL, n);
        return;
    }
    const std::function<void(int)> fn = [&body, n, T](int t) { body(n * t / T, n * (t + 1) / T); };
    pool.run((int)T, fn);
}

// Zeroes a[lo, hi) in parallel chunks.
template <class T>
void parallel_zero(T* a, size_t lo, size_t hi) {
    if (hi <= lo) return;
    T* p = a + lo;
    parallel_rows((long long)(hi - lo), 8, [p](long long r0, long long r1) {
        std::memset((void*)(p + r0), 0, sizeof(T) * (size_t)(r1 - r0));
    });
}

struct HostGeom {
    int ni = 0, nj = 0;
    // ghost-frame arrays (i, j in [-2, n+1], 0-based): index (j+2)*(ni+4) + (i+2)
    dvec M;     // 4 per cell: M11 M12 M21 M22
    dvec dl;    // 2 per cell
    dvec sur;   // 1 per cell
    dvec fi;    // (ni+1)*nj i-faces x (nx, ny, len), face F of row j at j*(ni+1)+F
    dvec fj;    // ni*(nj+1) j-faces x (nx, ny, len), face G of column i at G*ni+i
    dvec src0, src1;   // interior: 1/r (axi) or Gx, Gy (area)
    int g(int i, int j) const { return (j + 2) * (ni + 4) + (i + 2); }
};

// Where setup_block writes the face geometry instead of G.fi / G.fj: the device images of the
// face planes (plane q of i-face k at fi[q * pfi + k], j-faces alike) and, when given, their
// FP32 float4 records (fi4[4 k + q], the 4th component 0).
struct FaceOut {
    double* fi = nullptr;
    double* fj = nullptr;
    long long pfi = 0, pfj = 0;
    float* fi4 = nullptr;
    float* fj4 = nullptr;
};

// Interior metrics, face normals and source geometry of a block. nodes: (2, 0:ni, 0:nj)
// Fortran order; area: nodal cross-section or nullptr. With out, the faces go there (and
// G.fi / G.fj stay empty). Returns a Q2D_* status.
int setup_block(int ni, int nj, const double* nodes, const double* area, int source, HostGeom& G,
                const FaceOut* out = nullptr);

// Ghost-cell metrics of one boundary record (BC_Connect_Metrics / BC_Symmetry_Metrics /
// BC_Extrapolate_Metrics, Lib_Metrics.f90:285-553). donor/donor_nodes only for type 101.
int ghost_metrics(const q2d_bc_rec& r, int ni, int nj, const double* nodes, HostGeom& G,
                  int dni, int dnj, const double* donor_nodes);

// Unit tangent of the boundary face of a record (Setup_Inflow_Geometry, Lib_BC_Fluxes_Inflow.f90:521-531).
void face_tangent(const q2d_bc_rec& r, int ni, const double* nodes, double* t0, double* t1);

// versor(d,:) = M(d,:)/norm2(M(d,:)) of an interior cell (Mod_dt.f90:83).
void versors(const HostGeom& G, int i, int j, double* v);

}  // namespace q2d
