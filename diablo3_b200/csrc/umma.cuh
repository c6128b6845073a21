// umma.cuh -- 5th-generation tensor core (tcgen05) primitives for sm_100a,
// as inline PTX: tensor-memory allocation, BF16 MMA with FP32 accumulation
// from shared-memory operands, completion through an mbarrier, and
// tensor-memory loads into registers.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout: the
// tile is cut into core matrices of 8 rows x 16 bytes (8 bf16 along K),
// each stored as 128 contiguous bytes (row r at +16 r).  Core matrices that
// follow each other along K are LBO bytes apart, groups of 8 rows SBO bytes
// apart.  kmajor_offset() gives the byte offset of element (row, k) for a
// tile of K columns stored [row / 8][k / 8][row % 8][k % 8], i.e. LBO = 128,
// SBO = K * 16; one MMA consumes K = 16 (two core matrices along K), so the
// s-th K step starts 256 s bytes further.
//
// Every wait is bounded: a wait that gives up sets an error flag and the
// kernel returns after releasing its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace db {

__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k, int K) {
  return (uint32_t)((row >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (sm100): start >> 4 at [0,14), LBO >> 4 at
// [16,30), SBO >> 4 at [32,46), version 1 at [46,48), base offset 0,
// legacy LBO mode, layout type 0 (no swizzle) at [61,64)
__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor, kind::f16: D = F32 (1 at [4,6)), A = B = BF16
// (1 at [7,10) and [10,13)), both K-major, N >> 3 at [17,23), M >> 4 at [24,29)
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// tensor memory: allocate / free ncols columns (power of two, >= 32); one
// whole warp calls each
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          bool accumulate) {
  const uint32_t acc = accumulate ? 1u : 0u;
  const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;   // no output lane disabled
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc), "r"(m0), "r"(m1), "r"(m2), "r"(m3)
      : "memory");
}

// the mbarrier arrives once every MMA issued so far by this thread is done
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for phase `parity` of the mbarrier; false when it gave up
// up to `polls` non-blocking checks (mbarrier.test_wait) of the phase with
// this parity; unlike try_wait no check suspends the thread
__device__ __forceinline__ bool mbar_poll(uint64_t* mbar, uint32_t parity, uint32_t polls) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < polls; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// the first wait on a copy: the built-in bound, or `limit` non-blocking
// polls when a limit is set (db_set_wait_limit)
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_iter);
__device__ __forceinline__ bool mbar_wait_first(uint64_t* mbar, uint32_t parity, uint32_t limit, uint32_t max_iter) {
  return limit ? mbar_poll(mbar, parity, limit) : mbar_wait(mbar, parity, max_iter);
}

__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_iter) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < max_iter; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// arm the mbarrier's current phase with one arrival and `bytes` of expected
// asynchronous transactions
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// TMA bulk copy global -> shared of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing on the mbarrier; no multicast
__device__ __forceinline__ void bulk_g2s(void* smem, const void* gmem, uint32_t bytes, uint64_t* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(smem)),
               "l"(gmem), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// per-thread asynchronous copies global -> shared of 4, 8 or 16 bytes
// (both addresses aligned to the size), grouped and waited for with
// commit_group / wait_group (hardware-completed; no spin)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(smem)), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane
// (warp w reads lanes 32 (w % 4) .. 32 (w % 4) + 31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace db
