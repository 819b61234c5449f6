// Tensor-memory-accelerator (TMA) bulk copies between global and shared memory.
//
// Loads are tiled, non-multicast loads of this GPU's own memory
// (cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes; a CTA launched
// without a cluster is a cluster of one), completed on mbarriers. Stores are tiled bulk stores
// tracked by bulk groups. Every mbarrier wait is bounded: mbar_wait gives up after kWaitNs of
// global-timer time and returns false, so a kernel can record the failure and drain its copies
// instead of spinning.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace mhdb {

// Tensor maps of one strip-march stage: 3D views (x, y, plane) of the stage input and output
// buffers. For a mixed state (stage_mixed.cuh) they span its 18 float planes (9 hi, then 9 lo):
//   in_halo: stage input, box {kTmaHaloW, 1, 9}    (hi planes of one row, x halo included)
//   in_own:  stage input, box {kTmaOwnW, 1, 18}    (hi and lo of a warp's owned columns)
//   out_own: stage output, box {kTmaOwnW, 1, 18}   (stage 2 only: U^n, updated in place)
// For an FP64 state they span its 9 double planes and every box holds all 9. In the increment
// form (stage_delta.cuh) stage 2 reads U* = U^n + delta from two tensors: in_halo is U^n's hi
// planes, delta_halo the increment's 9 planes (box {kTmaHaloW, 1, 9}), in_own the increment
// (box {kTmaOwnW, 1, 9}) and out_own U^n's own cells (box {kTmaOwnW, 1, 18}; read, since stage 2
// writes U^{n+1} to the other state buffer); stage 1 uses in_halo only.
struct MarchTmaMaps {
    CUtensorMap in_halo;
    CUtensorMap in_own;
    CUtensorMap out_own;
    CUtensorMap delta_halo;
};

constexpr int kTmaOwnW = 28;  // owned columns of a warp (a multiple of 4: 16-byte x offsets)
constexpr int kTmaHaloW = 36; // columns x0 - 4 .. x0 + 31 (x0 - 4 is a multiple of 4)
constexpr unsigned long long kWaitNs = 500000000ull; // 0.5 s per bounded wait

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Ends an mbarrier's life (before its shared memory is initialised as a new one).
__device__ __forceinline__ void mbar_inval(uint32_t bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

// Orders earlier generic-proxy writes of a tensor map in global memory (the host's copy of the
// batch descriptors) before this thread's TMA copies through it.
__device__ __forceinline__ void tensormap_acquire(const void* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// Makes mbarrier initialisation visible to the async proxy (the TMA unit).
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with the given parity to complete; false after kWaitNs without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) {
        return true;
    }
    const unsigned long long t0 = global_ns();
#pragma unroll 1
    while (true) {
#pragma unroll 1
        for (int i = 0; i < 64; ++i) {
            if (mbar_try_wait(bar, parity)) {
                return true;
            }
        }
        if (global_ns() - t0 > kWaitNs) {
            return false;
        }
    }
}

// 3D tiled load of one box at (x, y, z) of the tensor map into shared memory at dst; completion
// is signalled on the mbarrier bar as transaction bytes.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

// 3D tiled store of one box from shared memory at src to (x, y, z) of the tensor map; elements
// outside the tensor's extent are not written. Completion is tracked by bulk groups.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int x, int y,
                                             int z)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(src), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// All but the N most recent committed bulk stores of this thread have finished reading their
// shared-memory source.
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// All committed bulk stores of this thread are complete (their global writes performed).
__device__ __forceinline__ void bulk_wait_all()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later async-proxy (TMA) reads.
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

} // namespace mhdb
