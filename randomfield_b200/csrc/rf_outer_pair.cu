// rf_outer_pair.cu -- the outer-group contraction (rf_outer.cu) on a CTA
// pair: one tcgen05 MMA of M = 256 covers both CTAs' 128-point tiles.
//
// Replaces the hot loop of gen_Std_Gauss_Shinozuka (randomFieldND.f90:276-330)
// for 3-D requests whose wavevectors form the set_kPoints tensor grid
// (spectra_RF.f90:87-133), with the factorisation of rf_outer.cu: f(x, r) =
// ampMult sum_i3 [c3 Yc + s3 Ys], Y = A (points x 2G) B (2G x N), A the outer
// phasors E1(i1) E2(i2)^{s2} generated on chip.
//
// Two kernels share one body: rf_outer_pair_kernel for a single request (of
// at least two items and two realizations) and rf_outer_pair_group_kernel
// for the outer-group units of a batch (each pair its own slice of the
// batch's items, each unit its own plan and stage table).
//
// A cluster of two CTAs works on a 256-point item, one 128-point tile per CTA.
// An N chunk is two halves of oRc realizations (N = 2 lPad oRc <= 256 each);
// the even CTA issues, per K-step and half, one tcgen05.mma.cta_group::2 of
// M = 256: each CTA contributes its tile's A (its own shared memory) and half
// of the half's B rows (lPad oRc rows each, the same shared-memory offset in
// both), and each CTA's TMEM receives its tile's 128 x N accumulator.  Against
// the one-CTA kernel a chunk covers twice the realizations at the same MMA
// count per K-step, so the generators build A for half as many chunks, the
// MMAs issued per flop halve, and a CTA's ring stage (one tile's A, half of
// B) is 46 KB instead of 62: four stages instead of three.
//
// BF16 plans (oTf32) carry the K-steps of the largest variance share as
// TF32: both A units of such a K-step hold its 16 K values in FP32
// containers (groups 0-3, then 4-7), both B blocks likewise, and the issuer
// runs two kind::tf32 MMAs (K = 8) per half where a BF16 K-step takes one.
//
// Warp roles (448 threads, in each CTA: 14 warps leave a thread 128
// registers):
//   warp 0      rank 0: MMA issuer (tcgen05.mma.cta_group::2, commits
//               multicast to both CTAs); rank 1: forwards each completed
//               stage of its own ring to rank 0's stage barrier (one
//               cluster-scope arrive), so that rank 0's barrier completes
//               when both CTAs' stages are full;
//   warp 1      producer (one thread): 1-D bulk copy (TMA, no multicast) of
//               the CTA's part of a stage's B blocks from HBM/L2;
//   warps 2-5   generators: one thread per point of the CTA's tile, the
//               K-step's 8 outer phasors (E1 of block 0 and the block step
//               from FP64-reduced phases once per item, later blocks and E2
//               by angle addition), rounded to 16 bits or, on a TF32
//               K-step, to TF32; driven by the stage table, four 16-bit
//               K-steps (or two TF32 ones) straight-line
//               (8 generator warps with half the phasors each measured 3 %
//               slower);
//   warps 6-13  epilogue: tcgen05.ld of one N half's accumulator (warp % 4
//               picks the TMEM lane quarter), the i3 sum, ampMult, marginal
//               map, FP64 stores; rank 1's release the accumulators to rank
//               0's issuer with cluster-scope arrives.
// Every wait is bounded (globaltimer); a final cluster barrier keeps each CTA
// alive until its peer no longer addresses its shared memory.
#include "rf_blend.cuh"
#include "rf_device.cuh"
#include "rf_gen.cuh"
#include "rf_launch.h"

namespace rfb {

namespace {

constexpr int kPIssuerWarp = 0, kPProducerWarp = 1, kPGenWarp0 = 2, kPGenWarps = 4;
constexpr int kPEpiWarp0 = kPGenWarp0 + kPGenWarps, kPEpiWarps = 8;
constexpr int kPThreads = (kPEpiWarp0 + kPEpiWarps) * 32;
constexpr int kPMaxSlots = 8;
constexpr int kPAUnitBytes = kTileM * 16 * 2;  // one tile's hi A of one K-step: 128 rows x 16 K x 16 bits
constexpr int kPStageABytes = kOuterStageUnits * kPAUnitBytes;
constexpr uint32_t kPTmemCols = 512;
constexpr int kPAccCols = 256;  // accumulator columns per N half

struct PairBars {
  uint64_t full[kPMaxSlots];   // rank 0: 8 generators + producer + rank 1's forward; rank 1: 8 + producer
  uint64_t empty[kPMaxSlots];  // the issuer's commit, multicast to both CTAs
  uint64_t acc_full;           // the issuer's commit after a chunk, multicast
  uint64_t acc_empty[2];       // rank 0: the 4 epilogue warps of a half in each CTA
  uint64_t done;               // rank 0: the issuer's last commit
  uint64_t dealloc_ok;         // rank 1: rank 0's MMAs have drained
  uint32_t tmem_base;
  int abort_flag;
  int32_t nStages;
  uint32_t stab[kOuterMaxKsteps];  // the issuer's stage table (rf_outer.cu's layout)
};
constexpr int kPHeader = 2048;
static_assert(sizeof(PairBars) <= kPHeader, "header");

struct OuterPairArgs {
  Plan P;
  const double* x;
  const unsigned char* B;
  double* out;
  uint32_t* err;
  int64_t row0, rows;
  int32_t S;          // ring stages
  int32_t slotBytes;  // one stage: A area (kPStageABytes), then kOuterStageUnits B units
};

// ------------------------------------------------------------ cluster helpers
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The shared::cluster address of this CTA's shared-memory word `p` in CTA `rank`.
__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// Arrive on an mbarrier of another CTA of the cluster, releasing this thread's
// prior writes (and what it has acquired) at cluster scope.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t clusterAddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(clusterAddr) : "memory");
}
__device__ __forceinline__ bool mbar_test_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity, uint32_t suspendNs) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(suspendNs)
      : "memory");
  return ok != 0;
}
// Bounded wait with cluster-scope acquire (barriers that remote arrivals
// complete), the same limits as mbar_wait_for.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, volatile int* abort,
                                                  uint64_t limitNs = kWaitLimitNs) {
  if (mbar_test_wait_cluster(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  const long long c0 = clock64();
  const long long minCycles = (long long)(limitNs / 2);
  while (true) {
    if (mbar_try_wait_cluster(bar, parity, kWaitSuspendNs)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limitNs && clock64() - c0 > minCycles) return false;
  }
}
__device__ __forceinline__ bool mbar_wait_cluster_warp(uint64_t* bar, uint32_t parity, volatile int* abort) {
  bool ok = true;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait_cluster(bar, parity, abort);
  return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc_pair(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (both CTAs' TMEM) (+)= A (256 rows: 128 from each CTA) x B (N rows: N/2
// from each CTA), kind::f16, FP32 accumulate; issued by one thread of rank 0.
__device__ __forceinline__ void mma_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The same MMA of kind::tf32 (K = 8: A and B rows of 32 bytes, two TF32
// core-matrix columns, as one K = 16 step of the 16-bit kinds).
__device__ __forceinline__ void mma_pair_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive once on `bar` in both CTAs (the same offset) when the issuing
// thread's prior tcgen05 operations have completed.
__device__ __forceinline__ void mma_commit_pair_both(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}
// The same, on this CTA's barrier only.
__device__ __forceinline__ void mma_commit_pair_local(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void pair_abort(PairBars* bars, uint32_t* err) {
  *reinterpret_cast<volatile int*>(&bars->abort_flag) = 1;
  atomicOr(err, kErrTimeout);
}

__device__ __forceinline__ float2 cmulf(float2 p, float2 q) {
  return make_float2(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x);
}
// One tile row's hi A unit of a K-step: the 8 groups E1(u) E, (re, im) as
// 16-bit pairs, groups 0-3 in the first core-matrix column, 4-7 in the
// second (2048 bytes on).
template <int PREC>
__device__ __forceinline__ void gen_hi(unsigned char* A, const float2* e1, float2 E) {
  uint32_t h[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const float2 v = cmulf(e1[u], E);
    h[u] = PREC == PREC_FP16 ? pack_f16x2(v.x, v.y) : pack_bf16x2(v.x, v.y);
  }
  *reinterpret_cast<uint4*>(A) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(A + 2048) = make_uint4(h[4], h[5], h[6], h[7]);
}
// A TF32 K-step's two units: unit 0 groups 0-3 (K 0-7), unit 1 groups 4-7,
// each unit's core-matrix columns two groups (re, im) in FP32 containers.
__device__ __forceinline__ void gen_tf32(unsigned char* A, const float2* e1, float2 E) {
#pragma unroll
  for (int h2 = 0; h2 < 4; ++h2) {
    const float2 p0 = cmulf(e1[2 * h2], E), p1 = cmulf(e1[2 * h2 + 1], E);
    *reinterpret_cast<uint4*>(A + (h2 >> 1) * kPAUnitBytes + (h2 & 1) * 2048) =
        make_uint4(tf32_bits(p0.x), tf32_bits(p0.y), tf32_bits(p1.x), tf32_bits(p1.y));
  }
}


// The stage table of a plan (issuer and generators): per stage its first
// K-step (9 bits), K-steps (3 bits) and per K-step two TF32 flags (B, A).  A
// stage must not span the end of an i2 run (outer_stage_layout closes one
// there); false when the plan's marks break that.
__host__ __device__ inline bool pair_stage_table(const Plan& P, uint32_t* stab, int32_t* nStages) {
  int32_t ns = 0, j0 = 0, n = 0;
  uint32_t fl = 0;
  bool bad = false;
  for (int32_t j = 0; j < P.oNK; ++j) {
    fl |= ((outer_b_lo(P, j) ? 1u : 0u) | (outer_a_lo(P, j) ? 2u : 0u)) << (2 * n);
    ++n;
    if (outer_stage_end(P, j) || j + 1 == P.oNK) {
      bad |= (j0 % P.kNStep[1]) + n > P.kNStep[1] || n > 4;
      stab[ns++] = (uint32_t)j0 | ((uint32_t)n << 9) | (fl << 12);
      j0 = j + 1;
      n = 0;
      fl = 0;
    }
  }
  *nStages = ns;
  return !bad;
}

// One 256-point item (one 128-point tile per CTA) as every role sees it.
struct PairView {
  const Plan* P;
  const double* x;
  double* out;
  const unsigned char* B;
  int64_t row0, rows;     // point range of the request covered by the launch
  int64_t item;           // 256-point item inside that range
  const uint32_t* stab;   // the plan's stage table
  int32_t nSt;
};

// The items pairIdx, pairIdx + nPairs, ... of one request; its stage table
// is built into shared memory at kernel start.
struct SinglePairWork {
  const OuterPairArgs* a;
  const uint32_t* stab;
  int64_t items;
  __device__ __forceinline__ int64_t count() const {
    const int64_t pairIdx = blockIdx.x >> 1, nPairs = gridDim.x >> 1;
    return pairIdx < items ? (items - 1 - pairIdx) / nPairs + 1 : 0;
  }
  __device__ __forceinline__ bool prepare(PairBars* bars) const {
    return pair_stage_table(a->P, bars->stab, &bars->nStages);
  }
  __device__ __forceinline__ void get(int64_t i, const PairBars* bars, PairView& v) const {
    v.P = &a->P;
    v.x = a->x;
    v.out = a->out;
    v.B = a->B;
    v.row0 = a->row0;
    v.rows = a->rows;
    v.item = (int64_t)(blockIdx.x >> 1) + i * (int64_t)(gridDim.x >> 1);
    v.stab = stab;
    v.nSt = bars->nStages;
  }
};

// This pair's slice [ctaStart[b], ctaStart[b+1]) of a grouped work list (b
// the pair's index); an item's `tile` field holds its 256-point item, and
// each unit's stage table comes with the launch's descriptors.
struct GroupPairWork {
  const OuterPairGroupArgs* g;
  int64_t begin, end;
  __device__ __forceinline__ int64_t count() const { return end - begin; }
  __device__ __forceinline__ bool prepare(PairBars*) const { return true; }
  __device__ __forceinline__ void get(int64_t i, const PairBars*, PairView& v) const {
    const GroupItem it = g->items[begin + i];
    const GroupSub& s = g->subs[it.sub];
    v.P = &s.P;
    v.x = s.x;
    v.out = s.out;
    v.B = s.B;
    v.row0 = 0;
    v.rows = s.P.n;
    v.item = it.tile;
    v.stab = g->stabs + (size_t)it.sub * kOuterMaxKsteps;
    v.nSt = g->nStages[it.sub];
  }
};

// The pipeline of one CTA pair over the items of `w`.  LPAD: axis-3 length
// padded to 8, 16, 24 or 32 (every item of a launch has this lPad).
template <int PREC, int LPAD, bool TF32, class Work>
__device__ __forceinline__ void pair_body(const Work& w, int S, int32_t slotBytes, uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  PairBars* bars = reinterpret_cast<PairBars*>(smem);
  unsigned char* slots = smem + kPHeader;
  volatile int* abort_flag = &bars->abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const int64_t count = w.count();
  PairView v;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&bars->full[s], kPGenWarps + 1 + (rank == 0 ? 1 : 0));
      mbar_init(&bars->empty[s], 1);
    }
    mbar_init(&bars->acc_full, 1);
    mbar_init(&bars->acc_empty[0], 8);
    mbar_init(&bars->acc_empty[1], 8);
    mbar_init(&bars->done, 1);
    mbar_init(&bars->dealloc_ok, 1);
    bars->abort_flag = 0;
    if (!w.prepare(bars)) {  // not a layout of outer_stage_layout: no stage runs
      bars->abort_flag = 1;
      atomicOr(err, kErrBounds);
    }
    mbar_fence_init();
  }
  if (warp == kPIssuerWarp) {
    tmem_alloc_pair(&bars->tmem_base, kPTmemCols);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();  // both CTAs' barriers and TMEM allocation before any remote arrive or MMA
  tc_fence_after();
  const uint32_t tbase = bars->tmem_base;

  if (warp == kPProducerWarp) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t s = 0, ph = 0;
      bool ok = true;
      for (int64_t i = 0; i < count && ok; ++i) {
        w.get(i, bars, v);
        const Plan& P = *v.P;
        const int32_t oNK = P.oNK, oNR = P.oNR;
        const int64_t kstepBytes = P.oKstepBytes, chunkBytes = P.oChunkBytes, opBytes = operand_bytes(P);
        for (int32_t c = 0; c < oNR && ok; ++c) {
          int64_t off = (int64_t)c * chunkBytes + (int64_t)rank * (chunkBytes / 2);
          for (int32_t j = 0; j < oNK;) {
            if (!mbar_wait(&bars->empty[s], ph ^ 1, abort_flag)) {
              ok = false;
              break;
            }
            uint32_t bytes = 0;
            bool end = false;
            for (; j < oNK && !end; ++j) {
              bytes += (uint32_t)(outer_b_lo(P, j) ? 2 * kstepBytes : kstepBytes);
              end = outer_stage_end(P, j);
            }
            if (!RF_IN_BOUNDS(off + bytes - 1, opBytes, err)) {
              ok = false;  // no copy: the stage stays empty, and the waits on it end the kernel
              break;
            }
            mbar_arrive_expect_tx(&bars->full[s], bytes);
            bulk_g2s(slots + (size_t)s * slotBytes + kPStageABytes, v.B + off, bytes, &bars->full[s]);
            off += bytes;
            if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
          }
        }
      }
      if (!ok) pair_abort(bars, err);
      if (*abort_flag) {
        // copies still in flight complete_tx on full barriers whose other
        // arrivals may never come: wait for them by time before going on
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < 1000000ull) {
        }
      }
    }
    __syncwarp();
  } else if (warp == kPIssuerWarp && rank == 1) {
    // ----------------------------------------------- rank 1: stage forwarder
    // Each stage of this CTA's ring, once full (its generators' and its bulk
    // copy's arrivals, acquired here), completes rank 0's barrier of the same
    // stage through one cluster-scope release.
    uint32_t s = 0, ph = 0;
    bool ok = true;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, bars, v);
      const int32_t oNR = v.P->oNR, nSt = v.nSt;
      for (int32_t c = 0; c < oNR && ok; ++c) {
        for (int32_t st = 0; st < nSt; ++st) {
          if (!mbar_wait_warp(&bars->full[s], ph, abort_flag)) { ok = false; break; }
          if (lane == 0) mbar_arrive_remote(map_to_rank(&bars->full[s], 0));
          __syncwarp();
          if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
        }
      }
    }
    if (!ok && lane == 0) pair_abort(bars, err);
    // rank 0's MMAs write this CTA's TMEM: free it only after they drained
    // (rank 0 arrives after its last commit completed, on every path)
    volatile int never = 0;
    mbar_wait_cluster_warp(&bars->dealloc_ok, 0, &never);
  } else if (warp == kPIssuerWarp) {
    // ------------------------------------------------ rank 0: MMA issuer
    // As rf_outer.cu's issuer, the two tiles' MMAs replaced by the two N
    // halves' MMAs of M = 256 (both tiles at once).  The stage barriers
    // complete only with rank 1's forwarded arrival, so their waits acquire
    // at cluster scope.
    const bool leader = elect_one();
    uint32_t s = 0, ph = 0, accPh = 0;
    bool ok = true, ready = false;
    const uint32_t ab = PREC == PREC_FP16 ? 0u : 1u;
    const uint64_t aU = (uint64_t)(kPAUnitBytes >> 4);  // descriptor step of one A unit
    const uint32_t t0 = tbase, t1 = tbase + (uint32_t)kPAccCols;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, bars, v);
      // the item's loop bounds in registers: every tcgen05 and mbarrier
      // statement clobbers memory, and a plan field read inside the loop
      // would be loaded again after each of them
      const Plan& P = *v.P;
      const int32_t oNR = P.oNR, oRc = P.oRc, lPad = P.lPad, nSt = v.nSt;
      const int32_t halfRows = lPad * oRc;  // B rows of a half in one CTA
      const uint64_t bU = (uint64_t)((uint32_t)P.oKstepBytes >> 4);    // descriptor step of one B unit
      const uint64_t bH = (uint64_t)((uint32_t)(halfRows * 32) >> 4);  // to the second half's rows
      const uint32_t idesc = make_idesc(ab, 256u, (uint32_t)(2 * lPad * oRc));
      const uint32_t idescT = make_idesc(2u, 256u, (uint32_t)(2 * lPad * oRc));  // A, B TF32
      const uint32_t* stab = v.stab;
      for (int32_t c = 0; c < oNR && ok; ++c) {
        // both halves' accumulators are free once both CTAs' epilogues read the last chunk
        if (!mbar_wait_cluster_warp(&bars->acc_empty[0], accPh ^ 1, abort_flag) ||
            !mbar_wait_cluster_warp(&bars->acc_empty[1], accPh ^ 1, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint32_t eNext = stab[0];
        for (int32_t st = 0; st < nSt; ++st) {
          if (!ready && !mbar_wait_cluster_warp(&bars->full[s], ph, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t e = eNext;
          if (st + 1 < nSt) eNext = stab[st + 1];
          const uint32_t n = (e >> 9) & 7u, fl = e >> 12;
          const uint32_t acc = (e & 0x1ffu) ? 1u : 0u;
          const uint32_t base = smem_u32(slots + (size_t)s * slotBytes);
          const uint64_t aD = make_sdesc(base, 2048u, 128u);
          const uint64_t bD = make_sdesc(base + (uint32_t)kPStageABytes, (uint32_t)halfRows * 16u, 128u);
          const uint32_t sn = (s + 1 == (uint32_t)S) ? 0u : s + 1;
          const uint32_t phn = (s + 1 == (uint32_t)S) ? ph ^ 1 : ph;
          const bool more = (st + 1 < nSt) || (c + 1 < oNR) || (i + 1 < count);
          const bool quad = fl == 0u && n == 4u, pair = fl == 0xFu && n == 2u;
          if (leader) {
            if (quad) {
              mma_pair(t0, aD, bD, idesc, acc);
              mma_pair(t1, aD, bD + bH, idesc, acc);
              mma_pair(t0, aD + aU, bD + bU, idesc, 1u);
              mma_pair(t1, aD + aU, bD + bU + bH, idesc, 1u);
              mma_pair(t0, aD + 2 * aU, bD + 2 * bU, idesc, 1u);
              mma_pair(t1, aD + 2 * aU, bD + 2 * bU + bH, idesc, 1u);
              mma_pair(t0, aD + 3 * aU, bD + 3 * bU, idesc, 1u);
            } else if (TF32 && pair) {
              // K-step 0 in units 0-1 (K 0-7, 8-15 as TF32) of A and B, K-step 1 in units 2-3
              mma_pair_tf32(t0, aD, bD, idescT, acc);
              mma_pair_tf32(t0, aD + aU, bD + bU, idescT, 1u);
              mma_pair_tf32(t1, aD, bD + bH, idescT, acc);
              mma_pair_tf32(t1, aD + aU, bD + bU + bH, idescT, 1u);
              mma_pair_tf32(t0, aD + 2 * aU, bD + 2 * bU, idescT, 1u);
              mma_pair_tf32(t0, aD + 3 * aU, bD + 3 * bU, idescT, 1u);
              mma_pair_tf32(t1, aD + 2 * aU, bD + 2 * bU + bH, idescT, 1u);
            } else {
              uint64_t ad = aD, bd = bD;
              for (uint32_t k = 0; k < n; ++k) {
                const uint32_t f = (fl >> (2 * k)) & 3u;  // both set on a TF32 K-step
                const uint32_t ak = k == 0 ? acc : 1u;
                if (TF32 && f) {
                  mma_pair_tf32(t0, ad, bd, idescT, ak);
                  mma_pair_tf32(t0, ad + aU, bd + bU, idescT, 1u);
                  mma_pair_tf32(t1, ad, bd + bH, idescT, ak);
                  mma_pair_tf32(t1, ad + aU, bd + bU + bH, idescT, 1u);
                  ad += 2 * aU;
                  bd += 2 * bU;
                } else {
                  mma_pair(t0, ad, bd, idesc, ak);
                  mma_pair(t1, ad, bd + bH, idesc, ak);
                  ad += aU;
                  bd += bU;
                }
              }
            }
          }
          ready = __all_sync(0xffffffffu, more && mbar_test_wait_cluster(&bars->full[sn], phn));
          if (leader) {
            if (quad) mma_pair(t1, aD + 3 * aU, bD + 3 * bU + bH, idesc, 1u);
            else if (TF32 && pair) mma_pair_tf32(t1, aD + 3 * aU, bD + 3 * bU + bH, idescT, 1u);
            mma_commit_pair_both(&bars->empty[s]);
          }
          __syncwarp();
          s = sn;
          ph = phn;
        }
        if (!ok) break;
        if (leader) mma_commit_pair_both(&bars->acc_full);
        __syncwarp();
        accPh ^= 1;
      }
    }
    if (!ok && lane == 0) pair_abort(bars, err);
    if (leader) mma_commit_pair_local(&bars->done);
    __syncwarp();
    volatile int never = 0;
    mbar_wait(&bars->done, 0, &never);  // every MMA issued, drained
    if (lane == 0) mbar_arrive_remote(map_to_rank(&bars->dealloc_ok, 1));
    __syncwarp();
  } else if (warp < kPEpiWarp0) {
    // ---------------------------------------------------------- generators
    // Stage by stage from the stage table.  A stage lies inside one i2 run
    // (fixed s2 and axis-1 block), so its K-steps' E2 powers follow by angle
    // addition from the run's walk; four hi-only K-steps (and two TF32 ones)
    // run straight-line.  The padded axis-1 groups (i1 >= n1) keep their
    // phasors: their B rows are zero.
    const int gi = threadIdx.x - kPGenWarp0 * 32;  // 0 .. 127
    const int row = gi;
    const uint32_t rowOff = (uint32_t)((row >> 3) * 128 + (row & 7) * 16);
    uint32_t s = 0, ph = 0;
    bool ok = !*abort_flag;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, bars, v);
      const Plan& P = *v.P;
      const int32_t n2 = P.kNStep[1], oNR = P.oNR, nSt = v.nSt;
      const uint32_t* stab = v.stab;
      const int64_t p = v.row0 + v.item * 2 * kTileM + (int64_t)rank * kTileM + row;
      const bool valid = p < v.row0 + v.rows;
      double x0 = 0.0, x1 = 0.0;
      if (valid && RF_IN_BOUNDS(p * 3 + 2, P.n * 3, err)) {
        x0 = v.x[p * 3 + 0] / P.corrL[0];
        x1 = v.x[p * 3 + 1] / P.corrL[1];
      }
      const float2 e2step = axis_phasor(P.kDelta[1], 1, x1);
      // E1(u) of block 0 and the block step E1(8), from FP64-reduced phases
      // once per item; later blocks by angle addition
      float2 e1base[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) e1base[u] = axis_phasor(P.kDelta[0], u, x0);
      const float2 e1step = axis_phasor(P.kDelta[0], 8, x0);
      for (int32_t c = 0; c < oNR && ok; ++c) {
        float2 e1[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) e1[u] = e1base[u];
        float2 e2 = make_float2(1.f, 0.f);
        int32_t jjCur = 0;
        for (int32_t st = 0; st < nSt; ++st) {
          const uint32_t e = stab[st];
          const int32_t j0 = (int32_t)(e & 0x1ffu), n = (int32_t)((e >> 9) & 7u);
          const uint32_t fl = e >> 12;
          const int32_t run = j0 / n2, jj = run >> 1;
          if (j0 - run * n2 == 0) e2 = make_float2(1.f, 0.f);  // a new i2 run
          if (jj != jjCur) {  // the next axis-1 block (blocks come in order)
            jjCur = jj;
#pragma unroll
            for (int u = 0; u < 8; ++u) e1[u] = cmulf(e1[u], e1step);
          }
          const float sg = (run & 1) ? -1.f : 1.f;  // s2 = 1: the conjugate of E2
          if (!mbar_wait_warp(&bars->empty[s], ph ^ 1, abort_flag)) {
            ok = false;
            break;
          }
          unsigned char* A = slots + (size_t)s * slotBytes + rowOff;
          if (fl == 0u && n == 4) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              gen_hi<PREC>(A + k * kPAUnitBytes, e1, make_float2(e2.x, sg * e2.y));
              e2 = cmulf(e2, e2step);
            }
          } else if (TF32 && fl == 0xFu && n == 2) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              gen_tf32(A + 2 * k * kPAUnitBytes, e1, make_float2(e2.x, sg * e2.y));
              e2 = cmulf(e2, e2step);
            }
          } else {
            uint32_t ua = 0;  // A units of the stage already written
            for (int32_t k = 0; k < n; ++k) {
              const bool tf = (fl >> (2 * k + 1)) & 1u;  // a TF32 K-step
              const float2 E = make_float2(e2.x, sg * e2.y);
              if (TF32 && tf) gen_tf32(A + ua * kPAUnitBytes, e1, E);
              else gen_hi<PREC>(A + ua * kPAUnitBytes, e1, E);
              ua += tf ? 2u : 1u;
              e2 = cmulf(e2, e2step);
            }
          }
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&bars->full[s]);
          if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
        }
      }
    }
    if (!ok) pair_abort(bars, err);
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3, h = (warp - kPEpiWarp0) >> 2;  // lane quarter, N half
    const int row = q * 32 + lane;
    const uint32_t taddr0 = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * kPAccCols);
    constexpr int LH = LPAD / 8;
    uint32_t accPh = 0;
    bool ok = true;
    const uint32_t releaseAddr = map_to_rank(&bars->acc_empty[h], 0);
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, bars, v);
      const Plan& P = *v.P;
      const int32_t oNR = P.oNR, oRc = P.oRc, nmcBlk = P.nmcBlk;
      const int64_t rOff = P.rOff, n = P.n, nOut = P.blend ? P.gTotal : P.n;
      [[maybe_unused]] const int64_t outLen = (int64_t)P.Nmc * nOut;  // the index checks' bound
      const bool blend = P.blend, marg = P.applyMarginal, logn = P.lognormal;
      const double outScale = P.outScale, margSd = P.margSd, margAvg = P.margAvg;
      double* out = v.out;
      const int64_t p = v.row0 + v.item * 2 * kTileM + (int64_t)rank * kTileM + row;
      const bool valid = p < v.row0 + v.rows;
      const double x2 = valid ? v.x[p * 3 + 2] / P.corrL[2] : 0.0;
      double bw = 0.0;
      int64_t bg = 0;
      if (blend && valid) bw = blend_weight(P, p, &bg);
      float2 e3[LPAD];
#pragma unroll
      for (int u = 0; u < LPAD; ++u)
        e3[u] = (u < P.kNStep[2]) ? axis_phasor(P.kDelta[2], u, x2) : make_float2(0.f, 0.f);
      for (int32_t c = 0; c < oNR; ++c) {
        if (!mbar_wait_warp(&bars->acc_full, accPh, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const int32_t r0 = c * 2 * oRc + h * oRc;  // the half's first realization of the block
        const int32_t rc = min(oRc, nmcBlk - r0);
        for (int32_t rl = 0; rl < rc; ++rl) {
          float acc = 0.f;
#pragma unroll
          for (int hh = 0; hh < LH; hh += 2) {
            uint32_t y[32];
            const uint32_t col = taddr0 + (uint32_t)(rl * 2 * LPAD + 16 * hh);
            if (hh + 1 < LH) tmem_ld32(col, y);
            else tmem_ld16(col, y);
            tmem_ld_wait();
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              if (hh + (u >> 3) < LH) {
                acc = fmaf(e3[8 * hh + u].x, __uint_as_float(y[2 * u]), acc);
                acc = fmaf(e3[8 * hh + u].y, __uint_as_float(y[2 * u + 1]), acc);
              }
            }
          }
          if (valid) {
            const int64_t r = rOff + r0 + rl;
            if (blend) {
              if (RF_IN_BOUNDS(r * nOut + bg, outLen, err)) atomicAdd(&out[r * nOut + bg], bw * ((double)acc * outScale));
            } else if (RF_IN_BOUNDS(r * n + p, outLen, err)) {
              double f = (double)acc * outScale;
              if (marg) {
                f = f * margSd + margAvg;
                if (logn) f = exp(f);
              }
              out[r * n + p] = f;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(releaseAddr);  // rank 0's barrier (its own CTA's too)
        accPh ^= 1;
      }
    }
    if (!ok) pair_abort(bars, err);
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kPIssuerWarp) tmem_dealloc_pair(tbase, kPTmemCols);
  cluster_sync_all();  // neither CTA leaves while its peer may still address its shared memory
}

template <int PREC, int LPAD, bool TF32>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    rf_outer_pair_kernel(const __grid_constant__ OuterPairArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const SinglePairWork w{&a, reinterpret_cast<const PairBars*>(smem)->stab, ((a.rows + kTileM - 1) / kTileM + 1) / 2};
  pair_body<PREC, LPAD, TF32>(w, a.S, a.slotBytes, a.err);
}

template <int PREC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    rf_outer_pair_group_kernel(const __grid_constant__ OuterPairGroupArgs g) {
  const int64_t b = blockIdx.x >> 1;
  const GroupPairWork w{&g, g.ctaStart[b], g.ctaStart[b + 1]};
  pair_body<PREC, kGroupLPad, PREC == PREC_BF16>(w, g.S, g.slotBytes, g.err);
}

template <int PREC, int LPAD>
cudaError_t launch_pair_t(const OuterPairArgs& a, size_t smem, int grid, cudaStream_t st) {
  auto fn = a.P.oTf32 ? rf_outer_pair_kernel<PREC, LPAD, PREC == PREC_BF16> : rf_outer_pair_kernel<PREC, LPAD, false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, kPThreads, smem, st>>>(a);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_pair_p(const OuterPairArgs& a, size_t smem, int grid, cudaStream_t st) {
  switch (a.P.lPad) {
    case 8: return launch_pair_t<PREC, 8>(a, smem, grid, st);
    case 16: return launch_pair_t<PREC, 16>(a, smem, grid, st);
    case 24: return launch_pair_t<PREC, 24>(a, smem, grid, st);
    case 32: return launch_pair_t<PREC, 32>(a, smem, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

// Stage bytes of a CTA-pair plan: one tile's A units, then this CTA's part of
// kOuterStageUnits B units.
size_t outer_pair_smem_bytes(const Plan& P, int* stages) {
  const int64_t slot = (kPStageABytes + kOuterStageUnits * P.oKstepBytes + 127) / 128 * 128;
  const size_t limit = 227 * 1024, floor = 120 * 1024;
  int S = (int)((limit - kPHeader) / (size_t)slot);
  if (S > kPMaxSlots) S = kPMaxSlots;
  if (stages) *stages = S;
  if (S < 2) return 0;
  const size_t total = (size_t)kPHeader + (size_t)S * (size_t)slot;
  return total < floor ? floor : total;
}

bool pair_group_stage_table(const Plan& P, uint32_t* stab, int32_t* nStages) {
  return pair_stage_table(P, stab, nStages);
}

size_t outer_pair_group_layout(const Plan* const* plans, size_t count, int maxStages, OuterPairGroupArgs* g) {
  int64_t bMax = 0;
  for (size_t i = 0; i < count; ++i) bMax = plans[i]->oKstepBytes > bMax ? plans[i]->oKstepBytes : bMax;
  const int64_t slot = (kPStageABytes + kOuterStageUnits * bMax + 127) / 128 * 128;
  const size_t limit = 227 * 1024, floor = 120 * 1024;
  int S = (int)((limit - kPHeader) / (size_t)slot);
  if (S > kPMaxSlots) S = kPMaxSlots;
  if (maxStages > 0 && S > maxStages) S = maxStages;
  g->S = S;
  g->slotBytes = (int32_t)slot;
  if (S < 2) return 0;
  const size_t total = (size_t)kPHeader + (size_t)S * (size_t)slot;
  return total < floor ? floor : total;
}

cudaError_t outer_pair_group_set_smem(int prec, size_t smem) {
  const int b = (int)smem;
  if (prec == PREC_FP16)
    return cudaFuncSetAttribute(rf_outer_pair_group_kernel<PREC_FP16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  return cudaFuncSetAttribute(rf_outer_pair_group_kernel<PREC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

cudaError_t launch_outer_pair_group(int prec, const OuterPairGroupArgs& g, size_t smem, int grid, cudaStream_t st) {
  if (prec == PREC_FP16) rf_outer_pair_group_kernel<PREC_FP16><<<grid, kPThreads, smem, st>>>(g);
  else rf_outer_pair_group_kernel<PREC_BF16><<<grid, kPThreads, smem, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_outer_pair(const Plan& P, const double* dX, const void* dB, double* dOut, int64_t row0,
                              int64_t rows, uint32_t* dErr, int numSMs, cudaStream_t st) {
  OuterPairArgs a;
  a.P = P;
  a.x = dX;
  a.B = reinterpret_cast<const unsigned char*>(dB);
  a.out = dOut;
  a.err = dErr;
  a.row0 = row0;
  a.rows = rows;
  a.slotBytes = (int32_t)((kPStageABytes + kOuterStageUnits * P.oKstepBytes + 127) / 128 * 128);
  int S = 0;
  const size_t smem = outer_pair_smem_bytes(P, &S);
  if (smem == 0) return cudaErrorInvalidValue;
  a.S = S;
  const int64_t items = ((rows + kTileM - 1) / kTileM + 1) / 2;
  int64_t pairs = items < numSMs / 2 ? items : numSMs / 2;
  if (pairs < 1) pairs = 1;
  const int grid = (int)(2 * pairs);
  if (P.prec == PREC_FP16) return launch_pair_p<PREC_FP16>(a, smem, grid, st);
  return launch_pair_p<PREC_BF16>(a, smem, grid, st);
}

}  // namespace rfb
