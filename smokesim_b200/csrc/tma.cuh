// tma.cuh - mbarrier and TMA (cp.async.bulk.tensor) helpers shared by the
// tile-fed sweep kernels, plus the host-side tensor-map cache.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"

struct ss_sim;

namespace ss {

SS_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

SS_D void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
SS_D void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
SS_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
SS_D void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
SS_D bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
SS_D void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait on an mbarrier phase: polls with back-off for at most about a
// second and reports whether the phase completed.
SS_D bool wait_bounded(uint64_t* bar, uint32_t phase) {
    for (int k = 0; k < (1 << 22); ++k) {
        if (mbar_try_wait(bar, phase)) return true;
        if (k > 64) __nanosleep(32);
    }
    return false;
}

// Block-uniform wait for a tile: every thread waits (bounded), then the block
// agrees; on failure the error word is set and every thread sees false, so no
// thread is left behind at a later barrier.
SS_D bool wait_tile(uint64_t* bar, uint32_t phase, int* err) {
    const bool ok = wait_bounded(bar, phase);
    const bool all = __syncthreads_and(ok) != 0;
    if (!all && threadIdx.x == 0) atomicOr(err, 1);
    return all;
}

// host (k_rbgs_tma.cu): the driver's tensor-map encoder, and a 3D tiled map
// of an x-fastest FP32 (bytes = false) or byte array, cached per simulation
PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn();
int tma_tensor_map(ss_sim* s, const void* ptr, bool bytes, const int dims[3], const int box[3], CUtensorMap* out);

}  // namespace ss
