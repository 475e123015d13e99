// Tensor Memory Accelerator (TMA) staging for the pass kernels, sm_100a.
//
// A pass stages the lines it transforms from HBM into shared memory with one elected thread:
// cp.async.bulk.tensor (a tile of a tensor map: strided gathers such as "rows y of every kx
// record") or cp.async.bulk (one contiguous run), both completing on a shared-memory mbarrier
// that counts the bytes delivered.  The other threads only wait on the barrier, so the staging
// costs no per-thread address arithmetic or registers.  Loads only, never with
// .multicast::cluster: every tensor map covers one buffer of this GPU's own memory.
//
// Every wait is bounded: after kWaitLimit polls the waiting thread records an error code in the
// handle's error word (read by the host after the batch) and gives up, so a lost completion can
// never hang the GPU.  A kernel that gave up waits once more, also bounded, before it exits, so
// that no copy is left writing into shared memory of a block that has finished.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bastr {

// Polls of an mbarrier before a wait gives up (each poll may suspend the thread for a while in
// hardware; far above any real staging latency, far below a second's worth of polls).
constexpr uint32_t kWaitLimit = 1u << 22;

// Error codes recorded in the handle's error word.
enum TmaErr : unsigned int { TMA_ERR_TIMEOUT = 1u };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barrier visible to the asynchronous (TMA) proxy; call after mbar_init,
// before the __syncthreads that publishes it.
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The elected thread announces `bytes` of asynchronous copies on the barrier's current phase.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// True once the phase with parity `phase` of the barrier has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait for a phase; on giving up, records TMA_ERR_TIMEOUT in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, unsigned int* err) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    if (err) atomicOr(err, (unsigned int)TMA_ERR_TIMEOUT);
    return false;
}

// One tile of a 3- or 4-dimensional tensor map into shared memory (coordinates innermost first,
// in elements; the innermost times the element size is a multiple of 16 bytes).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// One contiguous run (both addresses 16-byte aligned, size a multiple of 16 bytes).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Byte offset within a swizzled tile: the 16-byte chunk index (address bits 4..) is XORed with
// the 128-byte row index (address bits 7..), over 1, 2 or 3 bits for the 32-, 64- and 128-byte
// swizzle modes of the tensor map.  The tile must start at a multiple of 1024 bytes.
template <int SWZ_BYTES> __host__ __device__ __forceinline__ uint32_t swz(uint32_t o) {
    if constexpr (SWZ_BYTES == 32) return o ^ (((o >> 7) & 1u) << 4);
    else if constexpr (SWZ_BYTES == 64) return o ^ (((o >> 7) & 3u) << 4);
    else if constexpr (SWZ_BYTES == 128) return o ^ (((o >> 7) & 7u) << 4);
    else return o;
}

}  // namespace bastr
