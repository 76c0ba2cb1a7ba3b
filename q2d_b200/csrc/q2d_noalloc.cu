// q2d_noalloc.cu — residual norm (Compute_Residual) of two caller-owned device states, for
// callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc at the point where they need the
// residual: a host whose device memory is entirely reserved by its own pool allocator (a
// Fortran/OpenACC or CUDA-Fortran driver that owns all arrays), or code running on a latency
// path where the implicit synchronisation of an allocation is not acceptable. This entry point
// takes only their input and output pointers: its scratch (one partial sum per chunk of cells)
// lives in the fixed-size device array below, which every GPU that loads the library holds
// until the process exits.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "../../include/q2d_gpu.h"

namespace {

constexpr int kCellsPerPartial = Q2D_NOALLOC_CELLS_PER_PARTIAL;
constexpr int kMaxPartials = Q2D_NOALLOC_MAX_PARTIALS;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// 4 partial sums of squares (rho, u, v, p) per chunk: 8192 * 4 * 8 B = 256 KiB per device.
static __device__ __align__(256) double g_noalloc_scratch[4 * kMaxPartials];

// Device address of g_noalloc_scratch per device, resolved once per device under g_scratch_mu
// and published with release / acquire ordering, so that host threads making their first calls
// at the same time resolve it once and never see a half-written slot. The cache is not rebuilt
// after cudaDeviceReset: a process that resets a device must not call this entry point on it
// afterwards.
std::atomic<double*> g_scratch_ptr[kMaxDevices];
std::mutex g_scratch_mu;

// The device address of the scratch array on the current device `dev`, or nullptr when the
// runtime cannot resolve it.
double* scratch_on(int dev) {
    double* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (p) return p;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!p) {
        // First call on this device (its device is current): the host-side name of the array
        // is only a stand-in, so fetch its device address once.
        if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) return nullptr;
        g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
    return p;
}

// Sum over cells of |new - old|^2 per variable, one chunk of kCellsPerPartial cells per CTA,
// in a fixed order (thread-strided sums, then a fixed shuffle/warp tree), as in
// Compute_Residual (Mod_Diagnostic.f90:457-462).
__global__ void __launch_bounds__(kThreads) residual_partials(const double* __restrict__ pn,
                                                              const double* __restrict__ po,
                                                              long long n, long long stride,
                                                              double* scratch) {
    __shared__ double red[(kThreads / 32) * 4];
    const long long c0 = (long long)blockIdx.x * kCellsPerPartial;
    const long long c1 = c0 + kCellsPerPartial < n ? c0 + kCellsPerPartial : n;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = c0 + threadIdx.x; c < c1; c += kThreads)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double d = fabs(pn[v * stride + c] - po[v * stride + c]);
            acc[v] += d * d;
        }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o);
        if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * 4 + v] = acc[v];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w * 4 + threadIdx.x];
        scratch[4 * (long long)blockIdx.x + threadIdx.x] = t;   // every slot used is rewritten
    }
}

// Sums the partials in index order and writes the L2 norms sqrt(sum) (Mod_Explicit.f90:132).
__global__ void __launch_bounds__(kThreads) residual_final(const double* scratch, int nparts, double* out) {
    __shared__ double red[(kThreads / 32) * 4];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < nparts; k += kThreads)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[v] += scratch[4 * k + v];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o);
        if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * 4 + v] = acc[v];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w * 4 + threadIdx.x];
        out[threadIdx.x] = sqrt(t);
    }
}

}  // namespace

extern "C" int q2d_gpu_residual_norm_noalloc(const double* p_new, const double* p_old, long long ncells,
                                             long long plane_stride, double* norms_out, void* stream) {
    if (!p_new || !p_old || !norms_out || ncells < 1 || plane_stride < ncells) return Q2D_ERR_BADARG;
    if (ncells > (long long)kMaxPartials * kCellsPerPartial) return Q2D_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return Q2D_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return Q2D_ERR_CAPACITY;
    // An error the caller left pending is theirs: report it without launching and without
    // clearing it, so that the launch check below sees only this call's own launches.
    if (cudaPeekAtLastError() != cudaSuccess) return Q2D_ERR_CUDA;
    double* scratch = scratch_on(dev);
    if (!scratch) return Q2D_ERR_CUDA;
    const int nparts = (int)((ncells + kCellsPerPartial - 1) / kCellsPerPartial);
    cudaStream_t s = (cudaStream_t)stream;
    residual_partials<<<nparts, kThreads, 0, s>>>(p_new, p_old, ncells, plane_stride, scratch);
    residual_final<<<1, kThreads, 0, s>>>(scratch, nparts, norms_out);
    return cudaGetLastError() == cudaSuccess ? Q2D_OK : Q2D_ERR_CUDA;
}
