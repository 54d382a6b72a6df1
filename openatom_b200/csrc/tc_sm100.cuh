// Small wrappers for the sm_100a tensor-core (tcgen05) path: TMEM allocation,
// shared-memory matrix and instruction descriptors, the MMA, its commit to an
// mbarrier, bounded mbarrier waits and TMEM loads.  Field layouts follow the
// PTX ISA descriptions of tcgen05 (the same fields CuTe's UMMA::SmemDescriptor
// and UMMA::InstrDescriptor name).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle ("interleave"): 8-row
// core matrices of 16 bytes per row; lbo = byte distance between the two
// 16-byte K units of a core, sbo = byte distance between 8-row groups.
// Bits: [0,14) start >> 4, [16,30) lbo >> 4, [32,46) sbo >> 4, [46,48)
// version 1 (sm_100), [49,52) base offset 0, [52] lbo mode 0, [61,64) layout 0.
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D,
// M = m (64 or 128), N = n (multiple of 8, <= 256).
// Bits: [4,6) D format (1 = F32), [7,10) A format (1 = BF16), [10,13) B
// format (1 = BF16), [15] A major, [16] B major (0 = K), [17,23) N >> 3,
// [24,29) M >> 4.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

// The same, FP16 A and B (format 0), FP32 D.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int m, int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D (+)= A B^T, issued by one thread (no output lanes disabled).
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
      "}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z));
}

// The mbarrier receives one arrival when every MMA issued before by this
// thread has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Shared-memory writes of the generic proxy made visible to the tensor core.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity to complete: returns
// false once limit_ns have passed without it (the caller reports an error).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint64_t limit_ns = 1000000000ull) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
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
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// One test of the phase with the given parity; the thread may sleep up to
// hint_ns waiting for it (woken when the phase completes).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t done;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return done != 0;
}

// Bounded wait that also gives up as soon as *stop is set (another role of
// the CTA reported an error): false on either.  Sleeps between tests.
__device__ __forceinline__ bool mbar_wait_or(uint64_t* bar, uint32_t parity, const volatile int* stop,
                                             uint64_t limit_ns = 1000000000ull,
                                             uint32_t hint_ns = 20000u) {
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    if (mbar_test(bar, parity, hint_ns)) return true;
    if (*stop) return false;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}
// The same with short sleeps, for hand-overs on the critical path of a
// pipeline (a long suspend hint can leave the waiter asleep after the phase
// completed).
__device__ __forceinline__ bool mbar_wait_fast(uint64_t* bar, uint32_t parity,
                                               const volatile int* stop) {
  return mbar_wait_or(bar, parity, stop, 1000000000ull, 200u);
}

// Arrival (release, CTA scope) of this thread.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Arrival that also announces `bytes` of asynchronous copies to land.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bulk copy (no tensor map, no multicast) of `bytes` from global memory into
// this CTA's shared memory, completing on *bar.  Both addresses 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Named barrier `id` over `n` threads (whole warps) with an OR of v.
__device__ __forceinline__ int bar_or(int id, int n, int v) {
  uint32_t r;
  asm volatile(
      "{\n\t"
      ".reg .pred p, q;\n\t"
      "setp.ne.s32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(r)
      : "r"(v), "r"(id), "r"(n)
      : "memory");
  return (int)r;
}
__device__ __forceinline__ void bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// cp.async of 16 bytes; the first src_bytes (0, 8 or 16) come from global
// memory, the rest of the 16 is zero-filled.
__device__ __forceinline__ void cp16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// TMEM allocation by one full warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 32 consecutive FP32 columns of TMEM lane (warp's 32-lane slice + lane).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 or 8 consecutive 32-bit TMEM columns (raw words), loads and a store; a
// store is complete for the storing thread after tmem_wait_st.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmem_ld8u(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(
                   taddr),
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
               "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Two FP32 values rounded to nearest even BF16, packed: a in the low half
// (the lower address).
__device__ __forceinline__ uint32_t cvt_bf16x2(float a, float b) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Three-level BF16 split of a pair of FP32 values, packed per level:
// a = h + m + l exactly (the remainders are exact in FP32; after two levels
// at most 8 significant bits are left, so the third rounding is exact).
__device__ __forceinline__ void split3_pair(float a, float b, uint32_t& h, uint32_t& m, uint32_t& l) {
  h = cvt_bf16x2(a, b);
  const float ra = a - bf16_lo(h), rb = b - bf16_hi(h);
  m = cvt_bf16x2(ra, rb);
  l = cvt_bf16x2(ra - bf16_lo(m), rb - bf16_hi(m));
}

// Two FP32 values rounded to nearest even FP16, packed: a in the low half.
__device__ __forceinline__ uint32_t cvt_f16x2(float a, float b) {
  uint32_t r;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}
__device__ __forceinline__ float f16_lo(uint32_t w) {
  return __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu)));
}
__device__ __forceinline__ float f16_hi(uint32_t w) {
  return __half2float(__ushort_as_half((unsigned short)(w >> 16)));
}

// Two-level FP16 split of a pair of FP32 values already scaled by a power of
// two into |x| < 2^15: x = h + m + r with h the nearest FP16 (11 significant
// bits), m the nearest FP16 to the exact FP32 remainder x - h; |r| is at most
// 2^-22 |x| (or an FP16 subnormal step, 2^-25, for the smallest values).
__device__ __forceinline__ void split2h_pair(float a, float b, uint32_t& h, uint32_t& m) {
  h = cvt_f16x2(a, b);
  m = cvt_f16x2(a - f16_lo(h), b - f16_hi(h));
}

// The power of two that brings a largest magnitude `mx` to [2^13, 2^14)
// (1 for mx = 0 or not finite): the FP16 levels then keep 22 bits of every
// value within 2^-14 of the largest.
__host__ __device__ __forceinline__ float pow2_scale(float mx) {
  if (!(mx > 0.f) || !(mx < 3.0e38f)) return 1.f;
  int e = 0;
  frexpf(mx, &e);  // mx in [2^(e-1), 2^e)
  return ldexpf(1.f, 14 - (e < -80 ? -80 : e));
}

// Core-matrix image of one K step (16 reals) of a 128-row operand tile,
// K-major without swizzle: 8-row x 16-byte core matrices, the two 8-element K
// halves 128 bytes apart, 8-row groups 256 bytes apart; one level is 4 KB
// (CM_TILE) and the levels of a K step follow each other.  Byte offset of
// (row r, k) in one level (k < 16).
constexpr int CM_TILE = 128 * 16 * 2;
__host__ __device__ __forceinline__ int core_off(int r, int k) {
  return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// 8 FP32 values of one row (8 consecutive K) times a power of two `sc` -> two
// FP16 levels, stored as 16 bytes at dst and at dst + CM_TILE
__device__ __forceinline__ void split_store_h(uint8_t* dst, const float (&f)[8], float sc) {
  uint32_t lv[2][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) split2h_pair(f[2 * e] * sc, f[2 * e + 1] * sc, lv[0][e], lv[1][e]);
#pragma unroll
  for (int v = 0; v < 2; ++v)
    *reinterpret_cast<uint4*>(dst + v * CM_TILE) = make_uint4(lv[v][0], lv[v][1], lv[v][2], lv[v][3]);
}

}  // namespace tc
