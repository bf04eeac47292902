/*
 * Tensor memory (TMEM) as per-cell storage of the substep kernels (sm_100a).
 *
 * TMEM is 128 lanes x 512 columns of 32-bit words per SM.  A warp reaches the
 * 32 lanes of its quarter (warp index mod 4) and each thread reads and writes
 * only its own lane, so a lane is private storage of the cells its threads
 * own.  Loads move up to ~420 B/clk per SM, about three times the shared-memory
 * bandwidth, on a path of their own; wide accesses (16 or 32 columns) are the
 * efficient ones.
 *
 * Every tcgen05 instruction below is warp-collective (.sync.aligned): all 32
 * threads of a warp execute it together.  Allocation is by one whole warp; the
 * allocating warp frees the columns before the block exits.
 */
#pragma once

#include <stdint.h>

namespace tmem {

__device__ __forceinline__ uint32_t
smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* Allocates ncols columns (a power of two, 32..512) and writes the base
 * address to *dst (shared memory).  Called by one whole warp. */
__device__ __forceinline__ void
alloc(uint32_t* dst, const uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void
dealloc(const uint32_t taddr, const uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

/* Orders tcgen05 operations around a block-wide barrier. */
__device__ __forceinline__ void
fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void
fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

/* Waits until this thread's earlier loads (stores) have completed. */
__device__ __forceinline__ void
wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
/* (no memory clobber: it orders tensor-memory stores only) */
__device__ __forceinline__ void
wait_st()
{
    asm volatile("tcgen05.wait::st.sync.aligned;");
}

/* Lane address of this warp's quarter: the lane field is bits 31..16. */
__device__ __forceinline__ uint32_t
lane_base(const uint32_t tbase, const int warp)
{
    return tbase + ((uint32_t)(32 * (warp & 3)) << 16);
}

/* ---- loads and stores of consecutive 32-bit columns of this thread's lane ----
 * They touch tensor memory only, so they carry no memory clobber and ordinary
 * loads may be scheduled across them; being volatile, they keep their order
 * among themselves and with the waits.  A load's registers are valid only after
 * wait_ld_tied() on them. */

__device__ __forceinline__ void
st1(const uint32_t a, const uint32_t v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(a), "r"(v));
}
__device__ __forceinline__ void
st2(const uint32_t a, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a), "r"(v[0]),
                 "r"(v[1])
                 );
}
__device__ __forceinline__ void
st4(const uint32_t a, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]));
}
__device__ __forceinline__ void
st8(const uint32_t a, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(
                     a),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
                 "r"(v[7]));
}
__device__ __forceinline__ void
st16(const uint32_t a, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
                 "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(a),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
                 "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
                 "r"(v[14]), "r"(v[15])
                 );
}
__device__ __forceinline__ void
st32(const uint32_t a, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
                 "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
                 "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(a),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
                 "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
                 "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]),
                 "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]),
                 "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
                 );
}

__device__ __forceinline__ void
ld1(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v[0]) : "r"(a)
                 );
}
__device__ __forceinline__ void
ld2(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(v[0]), "=r"(v[1])
                 : "r"(a)
                 );
}
__device__ __forceinline__ void
ld4(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(a));
}
__device__ __forceinline__ void
ld8(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7])
                 : "r"(a));
}
__device__ __forceinline__ void
ld16(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(a)
                 );
}
__device__ __forceinline__ void
ld32(const uint32_t a, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                   "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                   "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                   "=r"(v[30]), "=r"(v[31])
                 : "r"(a)
                 );
}

/* N consecutive columns from a, as the widest shapes first (x32, x16, ... x1). */
template <int N>
__device__ __forceinline__ void
st_n(const uint32_t a, const uint32_t* v)
{
    if constexpr (N >= 32) {
        st32(a, v);
        st_n<N - 32>(a + 32, v + 32);
    }
    else if constexpr (N >= 16) {
        st16(a, v);
        st_n<N - 16>(a + 16, v + 16);
    }
    else if constexpr (N >= 8) {
        st8(a, v);
        st_n<N - 8>(a + 8, v + 8);
    }
    else if constexpr (N >= 4) {
        st4(a, v);
        st_n<N - 4>(a + 4, v + 4);
    }
    else if constexpr (N >= 2) {
        st2(a, v);
        st_n<N - 2>(a + 2, v + 2);
    }
    else if constexpr (N == 1) {
        st1(a, v[0]);
    }
}
template <int N>
__device__ __forceinline__ void
ld_n(const uint32_t a, uint32_t* v)
{
    if constexpr (N >= 32) {
        ld32(a, v);
        ld_n<N - 32>(a + 32, v + 32);
    }
    else if constexpr (N >= 16) {
        ld16(a, v);
        ld_n<N - 16>(a + 16, v + 16);
    }
    else if constexpr (N >= 8) {
        ld8(a, v);
        ld_n<N - 8>(a + 8, v + 8);
    }
    else if constexpr (N >= 4) {
        ld4(a, v);
        ld_n<N - 4>(a + 4, v + 4);
    }
    else if constexpr (N >= 2) {
        ld2(a, v);
        ld_n<N - 2>(a + 2, v + 2);
    }
    else if constexpr (N == 1) {
        ld1(a, v);
    }
}

/* Waits for this thread's loads, then ties the loaded words to the wait (an
 * empty volatile statement per word, after the wait in program order) so that
 * no use of them can be scheduled before it. */
template <int N>
__device__ __forceinline__ void
wait_ld_tied(uint32_t* w)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int i = 0; i < N; ++i)
        asm volatile("" : "+r"(w[i]));
}

/* A record of N values of type T as 32-bit words: N * sizeof(T) / 4 columns. */
template <typename T, int N>
struct Words {
    static constexpr int W = N * (int)sizeof(T) / 4;
    uint32_t w[W];
    __device__ __forceinline__ void set(const int i, const T v)
    {
        if constexpr (sizeof(T) == 8) {
            const unsigned long long b = (unsigned long long)__double_as_longlong((double)v);
            w[2 * i]                   = (uint32_t)b;
            w[2 * i + 1]               = (uint32_t)(b >> 32);
        }
        else {
            w[i] = __float_as_uint((float)v);
        }
    }
    __device__ __forceinline__ T get(const int i) const
    {
        if constexpr (sizeof(T) == 8)
            return (T)__longlong_as_double((long long)(((unsigned long long)w[2 * i + 1] << 32) |
                                                       (unsigned long long)w[2 * i]));
        else
            return (T)__uint_as_float(w[i]);
    }
    __device__ __forceinline__ void store(const uint32_t a) const { st_n<W>(a, w); }
    __device__ __forceinline__ void load(const uint32_t a) { ld_n<W>(a, w); }
    /* after this thread's wait::ld: ties the words to it */
    __device__ __forceinline__ void tie()
    {
#pragma unroll
        for (int i = 0; i < W; ++i)
            asm volatile("" : "+r"(w[i]));
    }
};

} // namespace tmem
