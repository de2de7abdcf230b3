// k_noalloc.cu - divergence norm of caller-owned velocity arrays that allocates
// no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands out all
// device memory from its own fixed budget (a game engine or renderer with a
// VRAM cap), or a per-frame callback in which an allocation and the device
// synchronisation it can imply would stall the frame.  Such a caller cannot
// create an ss_sim either (that allocates the grid), so this entry point takes
// plain device pointers.  It is the same computation as the divergence norm
// the solver reports (ss_stats.div_before): the discrete divergence of every
// fluid cell with solid neighbours' faces replaced by their velocity (0 here:
// obstacles at rest), squared and summed in FP64.  Its scratch - one FP64
// partial sum per block - lives in a static device array instead of a buffer
// owned by a handle.
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "ss_internal.h"

namespace ss {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 16;
constexpr long long kCellsPerBlock = (long long)kThreads * kCellsPerThread;   // 4096
constexpr int kMaxPartials = 16384;                                          // 128 KiB
constexpr long long kMaxCells = kCellsPerBlock * kMaxPartials;               // 67,108,864

// Shared by every call on a device and kept until the process exits; each
// call writes every slot it later reads, so nothing needs clearing.
__device__ __align__(256) double g_noalloc_partials[kMaxPartials];

std::mutex g_setup_mu;
// Device address of g_noalloc_partials per device ordinal, with the CUDA
// context it was looked up in: after cudaDeviceReset (or under another
// context on that device) the module is loaded again, possibly elsewhere, so
// a changed context means a new look-up.
double* g_partials_addr[256] = {};
void* g_partials_ctx[256] = {};

// The calling thread's current CUDA context (driver cuCtxGetCurrent, found
// through the runtime so that no driver library is linked); null if unknown.
void* current_context() {
    using Fn = int (*)(void**);
    static Fn fn = []() -> Fn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<Fn>(p);
        return nullptr;
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

__device__ __forceinline__ double block_sum_noalloc(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ double warp_part[kThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < kThreads / 32 ? warp_part[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// One block per 4096 consecutive cells (x fastest); per cell the same
// operations, in the same order, as k_divergence.
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_div_norm_noalloc(int nx, int ny, int nz, const float* __restrict__ u,
                                                              const float* __restrict__ v, const float* __restrict__ w,
                                                              const uint8_t* __restrict__ solid,
                                                              double* __restrict__ partials) {
    const long long ncell = (long long)nx * ny * nz;
    const long long base = (long long)blockIdx.x * kCellsPerBlock;
    double acc = 0.0;
    for (int j = 0; j < kCellsPerThread; ++j) {
        const long long cl = base + (long long)j * kThreads + threadIdx.x;
        if (cl >= ncell) break;
        const int c = (int)cl;
        if (solid[c]) continue;
        const int x = c % nx, t = c / nx, y = t % ny, z = t / ny;
        // out of grid counts as fluid; a solid neighbour's face moves with it (velocity 0)
        const bool s_top = y + 1 < ny && solid[c + nx];
        const bool s_bottom = y > 0 && solid[c - nx];
        const bool s_right = x + 1 < nx && solid[c + 1];
        const bool s_left = x > 0 && solid[c - 1];
        const float v_top = s_top ? 0.f : __ldg(v + idx3(x, y + 1, z, nx, ny + 1));
        const float v_bottom = s_bottom ? 0.f : __ldg(v + idx3(x, y, z, nx, ny + 1));
        const float v_right = s_right ? 0.f : __ldg(u + idx3(x + 1, y, z, nx + 1, ny));
        const float v_left = s_left ? 0.f : __ldg(u + idx3(x, y, z, nx + 1, ny));
        float d = v_right - v_left + v_top - v_bottom;
        if constexpr (DIM == 3) {
            const int pl = nx * ny;
            const bool s_front = z + 1 < nz && solid[c + pl];
            const bool s_back = z > 0 && solid[c - pl];
            const float v_front = s_front ? 0.f : __ldg(w + idx3(x, y, z + 1, nx, ny));
            const float v_back = s_back ? 0.f : __ldg(w + idx3(x, y, z, nx, ny));
            d = d + v_front - v_back;
        }
        acc += (double)d * (double)d;
    }
    const double bs = block_sum_noalloc(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

// Fixed-order sum of the partials of this call, then the square root.
__global__ void __launch_bounds__(1024) k_div_norm_noalloc_final(const double* __restrict__ partials, int n,
                                                                 double* __restrict__ out) {
    __shared__ double sh[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(sh[0]);
}

// Set-up, once per device (and again only if that device's context changed),
// with the device current: the host-side name g_noalloc_partials is only a
// stand-in, so look up the array's device address.
int scratch_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= 256) return set_error(SS_E_UNSUPPORTED, "device ordinal out of range");
    const void* ctx = current_context();
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_partials_addr[dev] || !ctx || ctx != g_partials_ctx[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);   // also makes the device's context current
        if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(g_noalloc_partials)");
        g_partials_addr[dev] = static_cast<double*>(p);
        g_partials_ctx[dev] = current_context();
    }
    *out = g_partials_addr[dev];
    return SS_OK;
}

}  // namespace
}  // namespace ss

extern "C" int ss_divergence_norm_noalloc(int dim, const int n[3], const float* u, const float* v, const float* w,
                                          const uint8_t* solid, double* out_norm, void* stream) {
    using namespace ss;
    if (dim != 2 && dim != 3) return set_error(SS_E_INVALID, "dim must be 2 or 3");
    if (!n || !u || !v || !solid || !out_norm || (dim == 3 && !w))
        return set_error(SS_E_INVALID, "NULL argument");
    const int nz = dim == 2 ? 1 : n[2];
    if (n[0] < 1 || n[1] < 1 || nz < 1) return set_error(SS_E_INVALID, "grid sizes must be positive");
    const long long ncell = (long long)n[0] * n[1] * nz;
    if (ncell > kMaxCells || (long long)(n[0] + 1) * (n[1] + 1) * (nz + 1) >= 2147483647LL)
        return set_error(SS_E_INVALID, "grid too large for the allocation-free divergence norm: at most 67108864 "
                                       "cells (16384 partial sums of 4096 cells)");
    double* partials = nullptr;
    int rc = scratch_address(&partials);
    if (rc != SS_OK) return rc;
    const int nblocks = (int)((ncell + kCellsPerBlock - 1) / kCellsPerBlock);
    cudaStream_t st = (cudaStream_t)stream;
    if (dim == 3) k_div_norm_noalloc<3><<<nblocks, kThreads, 0, st>>>(n[0], n[1], nz, u, v, w, solid, partials);
    else k_div_norm_noalloc<2><<<nblocks, kThreads, 0, st>>>(n[0], n[1], nz, u, v, w, solid, partials);
    rc = check_cuda(cudaGetLastError(), "k_div_norm_noalloc");
    if (rc != SS_OK) return rc;
    k_div_norm_noalloc_final<<<1, 1024, 0, st>>>(partials, nblocks, out_norm);
    return check_cuda(cudaGetLastError(), "k_div_norm_noalloc_final");
}
