/*
 * Shared-memory plane ring plumbing of the tiled substep kernels: mbarrier
 * waits with an iteration bound, and the 4-D TMA plane load
 * (cp.async.bulk.tensor into this CTA only) completing on an mbarrier.
 */
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "internal.h"

namespace tma_ring {

/* try_wait may suspend the thread for a short, implementation-defined time per
 * call; 2^22 calls bound a wait to seconds even if a copy never lands. */
constexpr long long kWaitLimit = 1LL << 22;
/* The bound under the fault-path test switch (a load that never lands). */
constexpr long long kDebugWaitLimit = 1LL << 12;

__device__ __forceinline__ uint32_t
smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void
mbar_init(uint64_t* bar, const unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void
fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void
mbar_arrive_expect_tx(uint64_t* bar, const unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool
mbar_try_wait(uint64_t* bar, const unsigned parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool
mbar_wait_bounded(uint64_t* bar, const unsigned parity, const long long limit = kWaitLimit)
{
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

/* Before a block exits: waits (bounded) until the last load issued into each of
 * the ring's `ring` slots has landed, so that no copy into this block's shared
 * memory is in flight even when an earlier wait gave up.  issued(s) is the
 * number of loads issued into slot s; each completed one phase of its
 * barrier. */
template <typename F>
__device__ __forceinline__ void
drain_ring(uint64_t* bars, const int ring, F issued)
{
    for (int s = 0; s < ring; ++s) {
        const int n = issued(s);
        if (n > 0)
            mbar_wait_bounded(&bars[s], (unsigned)((n - 1) & 1));
    }
}

/* One box of the 4-D (x, y, z, field) map at (x, y, z, 0) into dst; x is in
 * elements and must be a multiple of 16 bytes (negative starts are allowed
 * for loads: the part outside the tensor is not read). */
__device__ __forceinline__ void
tma_load_plane(void* dst, const CUtensorMap* map, uint64_t* bar, const int x, const int y,
               const int z)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
                 "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_addr(bar))
                 : "memory");
}

} // namespace tma_ring

/* Host: cuTensorMapEncodeTiled through the runtime's driver entry point, and
 * a 4-D map over the 8 field arrays of one buffer block (field stride
 * g.cells) with a (box_x, box_y, 1, 8) box.  Defined in solve_tiled.cu. */
bool ac_encode_field_map(void* map_out, void* base, const Geom& g, const int precision,
                         const unsigned box_x, const unsigned box_y);
