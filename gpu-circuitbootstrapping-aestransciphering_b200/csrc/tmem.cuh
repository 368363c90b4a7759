// tmem.cuh -- tensor memory (TMEM, sm_100a) as per-thread storage.
//
// TMEM is 128 lanes x 512 columns of 32-bit cells per SM.  A warp reaches only the 32 lanes of
// its quadrant (warp id mod 4): with the 32x32b shape each thread reads or writes its own lane,
// `num` consecutive columns starting at the address's column.  Address: lane << 16 | column.
// These helpers keep thread-private data (a kernel's accumulator) there, off shared memory.
// Every call is warp-collective (.sync.aligned): all 32 lanes execute it with the same address.
#pragma once

#include <cstdint>

namespace cbs {

// allocate ncols columns (a power of two, 32..512) for this CTA; the base address lands in
// *slot (shared memory).  Executed by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(slot));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// free what tmem_alloc returned; one whole warp, after every thread's last access (ordered by
// tmem_fence_before / a CTA barrier / tmem_fence_after)
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// the TMEM address of column `col` in the calling warp's lane quadrant
__device__ __forceinline__ uint32_t tmem_quadrant_addr(uint32_t base, uint32_t col) {
    const uint32_t quadrant = (threadIdx.x >> 5) & 3u;
    return base + ((quadrant * 32u) << 16) + col;
}

// 16 consecutive columns of this thread's lane <-> r[0..15]; the load waits for its data
__device__ __forceinline__ void tmem_load16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_store16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

// the stores issued so far by this thread have completed (before TMEM is read again or freed)
__device__ __forceinline__ void tmem_wait_store() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace cbs
