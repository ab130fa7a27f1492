// Blackwell (sm_100a) tensor-core building blocks: TMEM allocation,
// tcgen05.mma with BF16 operands from shared memory and FP32 accumulators in
// TMEM, commit to an mbarrier, TMEM loads, and the exact three-piece BF16
// split of an FP32 value that the mixed form's compensated products use.
//
// Operand layout ("K-major, no swizzle"): an operand of R rows (M or N) and
// K = 16 BF16 columns occupies R * 32 bytes as 8-row x 16-byte core matrices;
// core (g, kc) (rows 8g..8g+7, columns 8kc..8kc+7) starts at g * 256 + kc * 128
// bytes and holds its 8 rows 16 bytes apart.  Descriptor: leading (K)
// byte offset 128, stride (8-row) byte offset 256.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fgtb {
namespace tc {

constexpr uint32_t kLBO = 128;  // bytes between the two K halves of a 16-column operand row group
constexpr uint32_t kSBO = 256;  // bytes between consecutive 8-row groups

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row r, column k < 16) in the operand layout above
__device__ __forceinline__ uint32_t op_off(int r, int k) {
  return (uint32_t)((r >> 3) * kSBO + (k >> 3) * kLBO + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (sm_100 format, no swizzle)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((kLBO >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((kSBO >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                 // base offset 0, relative LBO mode, no swizzle
}

// instruction descriptor of kind::f16 with BF16 A and B (both K-major), FP32
// accumulation, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- TMEM allocation (one full warp) ----
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy writes to shared memory become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- MMA: D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread ----
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// arrive once on the mbarrier when every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

// ---- mbarrier ----
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase of parity `parity` to complete; gives up after
// `limit` polls and returns false (the caller records the timeout).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---- TMEM -> registers: this warp's 32 lanes, 16 consecutive FP32 columns ----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// The same without the wait, for several loads in flight: the registers are
// valid only after tmem_wait_ld(); tmem_fix() then ties each register to a
// point after the wait, so that no use of it is scheduled before.
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_fix(uint32_t* r) {
#pragma unroll
  for (int i = 0; i < 16; i++) asm volatile("" : "+r"(r[i])::"memory");
}

// ---- exact three-piece BF16 split: v = f0 + f1 + f2 with each fi a BF16 value ----
// f0 keeps the top 8 significant bits of v (truncation), f1 the next 8 of the
// exact remainder, f2 the rest (at most 8 significant bits), so no rounding
// happens anywhere.  Returned as the BF16 bit patterns.
__device__ __forceinline__ void split3(float v, uint16_t& b0, uint16_t& b1, uint16_t& b2) {
  const uint32_t h0 = __float_as_uint(v) & 0xFFFF0000u;
  const float r1 = v - __uint_as_float(h0);
  const uint32_t h1 = __float_as_uint(r1) & 0xFFFF0000u;
  const float r2 = r1 - __uint_as_float(h1);
  b0 = (uint16_t)(h0 >> 16);
  b1 = (uint16_t)(h1 >> 16);
  b2 = (uint16_t)(__float_as_uint(r2) >> 16);
}

// The compensated product of split operands: the six piece products whose
// orders sum to <= 2 (the dropped ones are below 2^-22 of the product),
// smallest first, accumulated in TMEM.
struct SplitPair {
  int a, b;
};
__device__ __forceinline__ SplitPair split_pair(int i) {
  // (2,0) (1,1) (0,2) (1,0) (0,1) (0,0)
  const int pa[6] = {2, 1, 0, 1, 0, 0}, pb[6] = {0, 1, 2, 0, 1, 0};
  return {pa[i], pb[i]};
}

}  // namespace tc
}  // namespace fgtb
