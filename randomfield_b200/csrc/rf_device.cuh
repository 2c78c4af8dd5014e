// rf_device.cuh -- device helpers shared by the table, tcgen05 and FP32
// kernels: sm_100a PTX wrappers (mbarrier, bulk copy, tcgen05), bounded
// waits, the rnglib jump-ahead and the Cody-Waite phase reduction.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "rf_plan.h"

namespace rfb {

// Device error word written by kernels whose bounded waits expire, and (in
// the RF_DEBUG_BOUNDS build) by a failed index check.
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrBounds = 2u;

// Index checks of the RF_DEBUG_BOUNDS build (the stand-in for a memory
// checker): RF_IN_BOUNDS(i, n, err) is true when 0 <= i < n; otherwise it
// records kErrBounds in *err and is false, and the caller skips the access.
// In the normal build it is `true` and compiles away.
#ifdef RF_DEBUG_BOUNDS
__device__ __forceinline__ bool bounds_ok(int64_t i, int64_t n, uint32_t* err) {
  if (i >= 0 && i < n) return true;
  if (err) atomicOr(err, kErrBounds);
  return false;
}
#define RF_IN_BOUNDS(i, n, err) ::rfb::bounds_ok((int64_t)(i), (int64_t)(n), (err))
#else
#define RF_IN_BOUNDS(i, n, err) true
#endif
// Wall-clock limit of one device wait (globaltimer nanoseconds).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Blocking probe: the thread is suspended in hardware until the phase of the
// given parity completes or about suspendNs nanoseconds pass, without issuing
// instructions meanwhile (a waiting warp leaves the issue slots of its
// sub-partition to the warps that work).
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t suspendNs) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(suspendNs)
      : "memory");
  return ok != 0;
}
// Suspension of one probe of the bounded waits: the abort flag and the time
// limit are checked between suspensions.
constexpr uint32_t kWaitSuspendNs = 20000u;

// Non-blocking probe of the phase of the given parity.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity.  Returns false once the
// wall-clock limit passes, or at once when *abort is already set.  A cheap
// non-blocking probe first: most waits on the hot path find the phase done.
// The limit counts as passed only when the SM's own cycle counter agrees
// (at least limitNs / 2 cycles, i.e. the limit at an SM clock of 0.5 GHz or
// more), so a step of the global timer alone cannot end a wait early.
// The probes between the checks suspend the thread in hardware
// (mbar_try_wait_suspend), so a warp that waits long issues almost nothing.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, volatile int* abort, uint64_t limitNs) {
  if (mbar_test_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  const long long c0 = clock64();
  const long long minCycles = (long long)(limitNs / 2);
  const uint32_t suspend = limitNs < (uint64_t)kWaitSuspendNs ? (uint32_t)limitNs : kWaitSuspendNs;
  while (true) {
    if (mbar_try_wait_suspend(bar, parity, suspend)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limitNs && clock64() - c0 > minCycles) return false;
  }
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  return mbar_wait_for(bar, parity, abort, kWaitLimitNs);
}

// Warp-wide bounded wait: lane 0 alone polls the barrier (256 threads
// spinning on one mbarrier word would contend its shared-memory bank and slow
// every barrier operation of the CTA), then the result is broadcast and the
// warp reconverges.  Call from all 32 lanes.
// With lanes_acquire set, every lane then probes the (completed) phase once
// itself, which gives each lane acquire ordering on data the barrier guards
// (bulk-copied shared memory).
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort,
                                               bool lanes_acquire = false) {
  bool ok = true;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort);
  ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
  if (ok && lanes_acquire) ok = mbar_test_wait(bar, parity);
  return __all_sync(0xffffffffu, ok);
}

// ------------------------------------------------------------ bulk copy (TMA)
// 1-D bulk copy global -> shared; completes transaction bytes on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------------ tcgen05
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D[tmem] (+)= A[tmem] x B[smem descriptor], kind::f16, FP32 accumulate.
__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// D[tmem] (+)= A[smem descriptor] x B[smem descriptor], kind::f16, FP32 accumulate.
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The same MMA of kind::tf32 (K = 8: rows of 32 bytes, two TF32 core-matrix
// columns, as one K = 16 step of the 16-bit kinds).
__device__ __forceinline__ void mma_ss_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The same MMA issued only when `issue` is nonzero, through a guard predicate
// (no branch between the MMAs of a K-step).
__device__ __forceinline__ void mma_ss_if(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate, uint32_t issue) {
  asm volatile(
      "{\n\t.reg .pred p, g;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "setp.ne.b32 g, %5, 0;\n\t"
      "@g tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(issue)
      : "memory");
}
// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy reads (tcgen05.mma operands) of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One lane of a converged warp (elect.sync over all 32 lanes), for code that
// runs a loop on the whole warp and issues single-thread instructions from
// the elected lane.
__device__ __forceinline__ bool elect_one() {
  uint32_t e;
  asm volatile(
      "{\n\t.reg .pred p;\n\t.reg .b32 l;\n\t"
      "elect.sync l|p, 0xffffffff;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(e));
  return e != 0;
}
// D[tmem] (+)= A[tmem] x B[smem descriptor], kind::f8f6f4 (A and B e4m3,
// K = 32 per instruction), FP32 accumulate.
__device__ __forceinline__ void mma_ts_f8(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive once on `bar` when all prior tcgen05 async ops of this thread finish.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x 4 / 8 / 16 consecutive 32-bit columns, one lane per thread.
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
               "r"(v[2]), "r"(v[3])
               : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}

// Instruction descriptor, kind::f16: D FP32, A and B both BF16 (ab=1) or
// both F16 (ab=0), K-major, dense.  Bits: [4,6) D fmt, [7,10) A fmt,
// [10,13) B fmt, [17,23) N>>3, [24,29) M>>4.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t ab, uint32_t M, uint32_t N) {
  return (1u << 4) | (ab << 7) | (ab << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; lbo = byte stride between the two K halves of one MMA
// (adjacent 8-element K groups), sbo = byte stride between 8-row groups.
__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout SWIZZLE_NONE (0)
}

// --------------------------------------------------------------- math
// Cody-Waite two-constant reduction of a phase to [-pi, pi] (W. J. Cody and
// W. Waite, Software Manual for the Elementary Functions, 1980): q = rint(x /
// 2pi); r = (x - q*C1) - q*C2 with C1 = 2pi rounded to double and C2 the
// remainder, each product fused so that the subtraction is exact for
// |q| < 2^20.
__device__ __forceinline__ double reduce_2pi(double x) {
  const double kInv2Pi = 0.15915494309189535;
  const double kC1 = 6.283185307179586;
  const double kC2 = 2.4492935982947064e-16;
  double q = rint(x * kInv2Pi);
  double r = fma(-q, kC1, x);
  return fma(-q, kC2, r);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
// Four e4m3 values (round to nearest, saturating) in K order: byte 0 = c0,
// byte 1 = s0, byte 2 = c1, byte 3 = s1.
__device__ __forceinline__ uint32_t pack_e4m3x4(float c0, float s0, float c1, float s1) {
  uint16_t lo, hi;
  asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(lo) : "f"(s0), "f"(c0));
  asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(hi) : "f"(s1), "f"(c1));
  return (uint32_t)lo | ((uint32_t)hi << 16);
}
__device__ __forceinline__ uint32_t pack_f16x2(float lo, float hi) {
  __half2 v = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
// x rounded to TF32 (10 mantissa bits; nearest, ties away from zero) in its
// 32-bit container: half a TF32 unit added to the magnitude bits, the low
// 13 bits cleared.  Finite |x| below the largest float only.
__device__ __forceinline__ uint32_t tf32_bits(float x) { return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u; }

// --------------------------------------------------------------- rnglib
// a^(2^j) mod m for j = 0..63, filled by the host (64-bit arithmetic).
struct JumpTable {
  int64_t p1[64];
  int64_t p2[64];
};

__device__ __forceinline__ int64_t mulmod(int64_t a, int64_t b, int64_t m) {
  return (int64_t)(((unsigned long long)a * (unsigned long long)b) % (unsigned long long)m);
}

// State (cg1, cg2) of generator 1 seeded (s1, s2) after p calls:
// cg = a^p * s mod m for each component (rnglib.f90:600-619).
__device__ __forceinline__ void uni_state_at(const JumpTable& jt, int64_t s1, int64_t s2, uint64_t p, int64_t& c1,
                                             int64_t& c2) {
  c1 = s1;
  c2 = s2;
  int j = 0;
  while (p) {
    if (p & 1ull) {
      c1 = mulmod(jt.p1[j], c1, kM1);
      c2 = mulmod(jt.p2[j], c2, kM2);
    }
    p >>= 1;
    ++j;
  }
}
// One call further: cg = a * cg mod m (a = jt.p*[0]).
__device__ __forceinline__ void uni_state_next(const JumpTable& jt, int64_t& c1, int64_t& c2) {
  c1 = mulmod(jt.p1[0], c1, kM1);
  c2 = mulmod(jt.p2[0], c2, kM2);
}
// i4_uni's value of a state: z = cg1 - cg2 folded to 1..m1-1 (:627-631).
__device__ __forceinline__ int32_t uni_value(int64_t c1, int64_t c2) {
  int64_t z = c1 - c2;
  if (z < 1) z += kM1 - 1;
  return (int32_t)z;
}

// i4_uni value of the p-th call (p >= 1) of generator 1 seeded (s1, s2).
__device__ __forceinline__ int32_t i4_uni_at(const JumpTable& jt, int64_t s1, int64_t s2, uint64_t p) {
  int64_t c1, c2;
  uni_state_at(jt, s1, s2, p, c1, c2);
  return uni_value(c1, c2);
}
__device__ __forceinline__ double r8_uni_at(const JumpTable& jt, int64_t s1, int64_t s2, uint64_t p) {
  return (double)i4_uni_at(jt, s1, s2, p) * kR8Scale;
}

}  // namespace rfb
