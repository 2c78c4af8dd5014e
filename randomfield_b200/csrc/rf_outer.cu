// rf_outer.cu -- the Shinozuka sum over 3-D tensor-grid wavevectors as an
// outer-group contraction on tcgen05 tensor cores.
//
// Replaces the hot loop of gen_Std_Gauss_Shinozuka (randomFieldND.f90:276-330)
// for 3-D requests whose wavevectors form the set_kPoints tensor grid
// (spectra_RF.f90:87-133): k = (k1(i1), s2 k2(i2), s3 k3(i3)).  With the
// outer phasor P_g(x) = exp(i (k1 x1 + s2 k2 x2)) of the group g = (i1, i2,
// s2) and E3 = exp(i k3 x3) = c3 + i s3, the field is
//
//   f(x, r) = ampMult sum_{i3} [ c3(i3) Yc(x, i3, r) + s3(i3) Ys(x, i3, r) ],
//   Y (points x (r, i3, cos|sin)) = A (points x 2G) B (2G x N),
//
// with A = (Re P_g, Im P_g) generated on chip and B built from the phases
// (rf_tables.cu, outer_run).  Against the plain contraction
// [cos Kx | sin Kx] x [a cos phi; -a sin phi] this is the same number of
// multiply-adds and the same operand bytes, but the generated operand shrinks
// from 2K = 8 n1 n2 n3 to 2G = 4 n1 n2 values per point and chunk, the MMAs
// run at N = 2 lPad x (realizations per chunk), up to 256, and the last
// contraction over i3 (2 lPad multiply-adds per output) runs in the epilogue
// in FP32 with FP64-reduced per-point phasors.
//
// This one-CTA form serves the single requests that the CTA-pair form
// (rf_outer_pair.cu) does not take: fewer than 512 points, or one
// realization.  One persistent CTA per SM; a work item is a pair of 128-point tiles that
// share every B stage (M = 256 per operand byte streamed from L2).  The
// realization block is cut into N chunks of oRc realizations (TMEM: one
// 256-column accumulator per tile); for each chunk the K-steps (16 K = 8
// outer groups of consecutive i1) stream through a ring of shared-memory
// stages, each holding two to four consecutive K-steps: both tiles' A and
// B's K-step blocks.  BF16 plans carry the K-steps of the largest variance
// share as TF32 (Plan::oTf32): two A units and two B blocks hold the K-step's
// 16 K values in 32-bit containers, and two kind::tf32 MMAs (K = 8) per tile
// replace the one BF16 MMA.
//
// Warp roles (576 threads):
//   warp 0      MMA issuer: the warp runs the stage loop, one elected lane
//               issues tcgen05.mma (A and B by shared-memory descriptor, D in
//               TMEM) and tcgen05.commit;
//   warp 1      producer (one thread): 1-D bulk copies (TMA, no multicast) of
//               a stage's B blocks from HBM/L2 into the ring;
//   warps 2-9   generators: one point each (256 = two tiles); per K-step the
//               8 outer phasors E1(i1) E2(i2)^{s2} of the point, rounded to
//               16 bits (or to TF32), stored in the K-major core-
//               matrix layout; the K-steps run axis-1 block by block (E1 of
//               the block's 8 i1 from FP64-reduced phases), E2 walked by
//               angle addition over i2;
//   warps 10-17 epilogue: tcgen05.ld of a tile's accumulator (warp % 4 picks
//               the TMEM lane quarter), the i3 sum with the point's own
//               E3 phasors, ampMult, the marginal map, FP64 stores.
// Every wait is bounded (globaltimer); on expiry the kernel raises the error
// word, drains its own async work, frees TMEM and returns.
#include "rf_blend.cuh"
#include "rf_device.cuh"
#include "rf_gen.cuh"
#include "rf_launch.h"

namespace rfb {

namespace {

constexpr int kIssuerWarp = 0, kProducerWarp = 1, kGenWarp0 = 2, kGenWarps = 8;
constexpr int kEpiWarp0 = kGenWarp0 + kGenWarps, kEpiWarps = 8;
constexpr int kOuterThreads = (kEpiWarp0 + kEpiWarps) * 32;
constexpr int kPairRows = 2 * kTileM;
constexpr int kOuterMaxSlots = 8;
constexpr int kATileBytes = kTileM * 16 * 2;  // one tile's K-step of A: 128 rows x 16 K x 16 bits
constexpr uint32_t kOuterTmemCols = 512;
constexpr int kAccCols = 256;  // accumulator columns per tile
// Ring stages of kOuterStageUnits units (rf_plan.h): one full/empty barrier
// pair, one bulk copy, one generator fence and one commit serve a stage of
// two to four K-steps.  The issuing thread keeps the tensor pipe fed only
// when it issues about eight or more MMAs per loop pass (measured on this
// kernel's MMA shape: 4 MMAs per pass ran at 1.4x the pipe's time per MMA,
// 8 at 1.03x, 12 at 1.0x, whatever the pass did besides), and a stage of
// four 16-bit K-steps carries 8, one of two TF32 K-steps 8 of twice the
// length.
constexpr int kAUnitBytes = 2 * kATileBytes;                    // both tiles' hi A of one K-step
constexpr int kStageABytes = kOuterStageUnits * kAUnitBytes;    // A area of a stage

struct OuterBars {
  uint64_t full[kOuterMaxSlots];   // per stage: 8 generator warps + producer (bytes)
  uint64_t empty[kOuterMaxSlots];  // per stage: MMA commit
  uint64_t acc_full;               // MMA commit after a chunk's last K-step
  uint64_t acc_empty[2];           // the 4 epilogue warps of a tile
  uint64_t done;
  uint32_t tmem_base;
  int abort_flag;
  int32_t nStages;                 // stages per chunk of the current item
  // the issuer's table of the current item's stages: first K-step (bits
  // 0-8), K-steps (bits 9-11), per K-step k bits 12+2k (B lo) and 13+2k (A lo)
  uint32_t stab[kOuterMaxKsteps];
};
constexpr int kOuterHeader = 2048;
static_assert(sizeof(OuterBars) <= kOuterHeader, "header");

struct OuterArgs {
  Plan P;
  const double* x;
  const unsigned char* B;
  double* out;
  uint32_t* err;
  int64_t row0, rows;
  int32_t S;          // ring stages
  int32_t slotBytes;  // one stage: A area (kStageABytes), then kOuterStageUnits B units; 128-byte multiple
  int32_t aBytes;     // A area of a stage (kStageABytes)
};

// One work item (a pair of 128-point tiles of one request) as every role sees it.
struct OuterView {
  const Plan* P;
  const double* x;
  double* out;
  const unsigned char* B;
  int64_t row0, rows;  // point range of the request covered by the launch
  int64_t pair;        // pair of tiles inside that range
};

// The pairs blockIdx.x, blockIdx.x + gridDim.x, ... of one request.
struct SingleOuterWork {
  const OuterArgs* a;
  int64_t pairs;
  __device__ __forceinline__ int64_t count() const {
    return (int64_t)blockIdx.x < pairs ? (pairs - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  }
  __device__ __forceinline__ void get(int64_t i, OuterView& v) const {
    v.P = &a->P;
    v.x = a->x;
    v.out = a->out;
    v.B = a->B;
    v.row0 = a->row0;
    v.rows = a->rows;
    v.pair = blockIdx.x + i * gridDim.x;
  }
};


__device__ __forceinline__ void outer_abort(OuterBars* bars, uint32_t* err) {
  *reinterpret_cast<volatile int*>(&bars->abort_flag) = 1;
  atomicOr(err, kErrTimeout);
}

template <int PREC>
__device__ __forceinline__ uint32_t pack16(float lo, float hi) {
  return PREC == PREC_FP16 ? pack_f16x2(lo, hi) : pack_bf16x2(lo, hi);
}

// The pipeline of one CTA over the work items of `w`.  LPAD: axis-3 length
// padded to 8, 16, 24 or 32 (every item of a launch has this lPad).
template <int PREC, int LPAD, class Work>
__device__ __forceinline__ void outer_body(const Work& w, int S, int32_t slotBytes, int32_t aBytes, uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  OuterBars* bars = reinterpret_cast<OuterBars*>(smem);
  unsigned char* slots = smem + kOuterHeader;
  volatile int* abort_flag = &bars->abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t count = w.count();
  // BF16 plans carry their high-variance K-steps as TF32 (Plan::oTf32)
  constexpr bool TF32 = PREC == PREC_BF16;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&bars->full[s], kGenWarps + 1);
      mbar_init(&bars->empty[s], 1);
    }
    mbar_init(&bars->acc_full, 1);
    mbar_init(&bars->acc_empty[0], 4);
    mbar_init(&bars->acc_empty[1], 4);
    mbar_init(&bars->done, 1);
    bars->abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == kIssuerWarp) {
    tmem_alloc(&bars->tmem_base, kOuterTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = bars->tmem_base;
  OuterView v;

  if (warp == kProducerWarp) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t s = 0, ph = 0;
      bool ok = true;
      for (int64_t i = 0; i < count && ok; ++i) {
        w.get(i, v);
        const Plan& P = *v.P;
        const int32_t oNK = P.oNK, oNR = P.oNR;
        const int64_t chunkBytes = P.oChunkBytes, opBytes = operand_bytes(P);
        for (int32_t c = 0; c < oNR && ok; ++c) {
          const unsigned char* src = v.B + (int64_t)c * chunkBytes;
          for (int32_t j = 0; j < oNK;) {
            if (!mbar_wait(&bars->empty[s], ph ^ 1, abort_flag)) {
              ok = false;
              break;
            }
            // the stage's B blocks lie back to back in the operand
            uint32_t bytes = 0;
            bool end = false;
            for (; j < oNK && !end; ++j) {
              bytes += (uint32_t)(outer_b_lo(P, j) ? 2 * P.oKstepBytes : P.oKstepBytes);
              end = outer_stage_end(P, j);
            }
            if (!RF_IN_BOUNDS((src - v.B) + bytes - 1, opBytes, err)) {
              ok = false;  // no copy: the stage stays empty, and the waits on it end the kernel
              break;
            }
            mbar_arrive_expect_tx(&bars->full[s], bytes);
            bulk_g2s(slots + (size_t)s * slotBytes + kStageABytes, src, bytes, &bars->full[s]);
            src += bytes;
            if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
          }
        }
      }
      if (!ok) outer_abort(bars, err);
      if (*abort_flag) {
        // copies still in flight complete_tx on full barriers whose generator
        // arrivals may never come: wait for them by time before the CTA exits
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < 1000000ull) {
        }
      }
    }
    __syncwarp();
  } else if (warp == kIssuerWarp) {
    // ---------------------------------------------------------- MMA issuer
    // The whole warp runs the loop (warp-uniform state); one elected lane
    // issues.  A stage's MMAs go out back to back, and the next stage's
    // barrier is probed before the last MMA so that the wait proper runs only
    // when the probe failed.  Stages of four 16-bit K-steps and of two TF32
    // ones (nearly all of them: the TF32 K-steps are the top of a variance
    // ranking and come in runs) take straight paths, whose last MMA is a
    // tile-1 MMA that may accumulate in any order (acc = 1) and so goes after
    // the probe; other stages loop over their K-steps.
    const bool leader = elect_one();
    uint32_t s = 0, ph = 0, accPh = 0;
    bool ok = true, ready = false;  // ready: full[s] of the next stage already observed
    const uint32_t ab = PREC == PREC_FP16 ? 0u : 1u;
    const uint64_t aT = (uint64_t)(kATileBytes >> 4);  // descriptor step to tile 1's A
    const uint64_t aU = (uint64_t)(kAUnitBytes >> 4);  // descriptor step of one A unit
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      // the item's loop bounds in registers: every tcgen05 and mbarrier
      // statement clobbers memory, and a plan field read inside the loop
      // would be loaded again after each of them
      const int32_t oNK = P.oNK, oNR = P.oNR, oRc = P.oRc, nmcBlk = P.nmcBlk, lPad = P.lPad;
      const uint64_t bU = (uint64_t)(P.oKstepBytes >> 4);  // descriptor step of one B unit
      if (lane == 0) {
        int32_t ns = 0, j0 = 0, n = 0;
        uint32_t fl = 0;
        for (int32_t j = 0; j < oNK; ++j) {
          fl |= ((outer_b_lo(P, j) ? 1u : 0u) | (outer_a_lo(P, j) ? 2u : 0u)) << (2 * n);
          ++n;
          if (outer_stage_end(P, j) || j + 1 == oNK) {
            bars->stab[ns++] = (uint32_t)j0 | ((uint32_t)n << 9) | (fl << 12);
            j0 = j + 1;
            n = 0;
            fl = 0;
          }
        }
        bars->nStages = ns;
      }
      __syncwarp();
      const int32_t nSt = *reinterpret_cast<volatile int32_t*>(&bars->nStages);
      const uint32_t nRows = (uint32_t)(2 * lPad * oRc);  // B rows (N) of a full chunk
      for (int32_t c = 0; c < oNR && ok; ++c) {
        const int32_t rc = min(oRc, nmcBlk - c * oRc);
        const uint32_t idesc = make_idesc(ab, 128u, (uint32_t)(2 * lPad * rc));
        const uint32_t idescT = make_idesc(2u, 128u, (uint32_t)(2 * lPad * rc));  // A, B TF32
        // both accumulators are free once the epilogue has read the last chunk
        if (!mbar_wait_warp(&bars->acc_empty[0], accPh ^ 1, abort_flag) ||
            !mbar_wait_warp(&bars->acc_empty[1], accPh ^ 1, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint32_t eNext = bars->stab[0];
        for (int32_t st = 0; st < nSt; ++st) {
          if (!ready && !mbar_wait_warp(&bars->full[s], ph, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t e = eNext;  // read one stage ahead
          if (st + 1 < nSt) eNext = bars->stab[st + 1];
          const uint32_t n = (e >> 9) & 7u, fl = e >> 12;
          const uint32_t acc = (e & 0x1ffu) ? 1u : 0u;  // the chunk's first K-step starts the accumulators
          const uint32_t base = smem_u32(slots + (size_t)s * slotBytes);
          const uint64_t aD = make_sdesc(base, 2048u, 128u);
          const uint64_t bD = make_sdesc(base + (uint32_t)kStageABytes, nRows * 16u, 128u);
          const uint32_t sn = (s + 1 == (uint32_t)S) ? 0u : s + 1;
          const uint32_t phn = (s + 1 == (uint32_t)S) ? ph ^ 1 : ph;
          const bool more = (st + 1 < nSt) || (c + 1 < oNR) || (i + 1 < count);
          const bool quad = fl == 0u && n == 4u, pair = fl == 0xFu && n == 2u;
          if (leader) {
            if (quad) {
              mma_ss(tbase, aD, bD, idesc, acc);
              mma_ss(tbase + (uint32_t)kAccCols, aD + aT, bD, idesc, acc);
              mma_ss(tbase, aD + aU, bD + bU, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aD + aU + aT, bD + bU, idesc, 1u);
              mma_ss(tbase, aD + 2 * aU, bD + 2 * bU, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aD + 2 * aU + aT, bD + 2 * bU, idesc, 1u);
              mma_ss(tbase, aD + 3 * aU, bD + 3 * bU, idesc, 1u);
            } else if (TF32 && pair) {
              // K-step 0 in units 0-1 (K 0-7, 8-15 as TF32) of A and B, K-step 1 in units 2-3
              mma_ss_tf32(tbase, aD, bD, idescT, acc);
              mma_ss_tf32(tbase, aD + aU, bD + bU, idescT, 1u);
              mma_ss_tf32(tbase + (uint32_t)kAccCols, aD + aT, bD, idescT, acc);
              mma_ss_tf32(tbase + (uint32_t)kAccCols, aD + aU + aT, bD + bU, idescT, 1u);
              mma_ss_tf32(tbase, aD + 2 * aU, bD + 2 * bU, idescT, 1u);
              mma_ss_tf32(tbase, aD + 3 * aU, bD + 3 * bU, idescT, 1u);
              mma_ss_tf32(tbase + (uint32_t)kAccCols, aD + 2 * aU + aT, bD + 2 * bU, idescT, 1u);
            } else {
              uint64_t a = aD, b = bD;
              for (uint32_t k = 0; k < n; ++k) {
                const uint32_t f = (fl >> (2 * k)) & 3u;  // both set on a TF32 K-step
                const uint32_t ak = k == 0 ? acc : 1u;
                if (TF32 && f) {
                  mma_ss_tf32(tbase, a, b, idescT, ak);
                  mma_ss_tf32(tbase, a + aU, b + bU, idescT, 1u);
                  mma_ss_tf32(tbase + (uint32_t)kAccCols, a + aT, b, idescT, ak);
                  mma_ss_tf32(tbase + (uint32_t)kAccCols, a + aU + aT, b + bU, idescT, 1u);
                  a += 2 * aU;
                  b += 2 * bU;
                } else {
                  mma_ss(tbase, a, b, idesc, ak);
                  mma_ss(tbase + (uint32_t)kAccCols, a + aT, b, idesc, ak);
                  a += aU;
                  b += bU;
                }
              }
            }
          }
          ready = __all_sync(0xffffffffu, more && mbar_test_wait(&bars->full[sn], phn));
          if (leader) {
            if (quad) mma_ss(tbase + (uint32_t)kAccCols, aD + 3 * aU + aT, bD + 3 * bU, idesc, 1u);
            else if (TF32 && pair) mma_ss_tf32(tbase + (uint32_t)kAccCols, aD + 3 * aU + aT, bD + 3 * bU, idescT, 1u);
            mma_commit(&bars->empty[s]);
          }
          __syncwarp();
          s = sn;
          ph = phn;
        }
        if (!ok) break;
        if (leader) mma_commit(&bars->acc_full);
        __syncwarp();
        accPh ^= 1;
      }
    }
    if (!ok && lane == 0) outer_abort(bars, err);
    if (leader) mma_commit(&bars->done);
    __syncwarp();
    volatile int never = 0;
    mbar_wait(&bars->done, 0, &never);
    __syncwarp();
  } else if (warp < kEpiWarp0) {
    // ---------------------------------------------------------- generators
    const int gi = threadIdx.x - kGenWarp0 * 32;  // 0 .. 255
    const int t = gi >> 7, row = gi & 127;
    const uint32_t rowOff = (uint32_t)((row >> 3) * 128 + (row & 7) * 16);
    uint32_t s = 0, ph = 0;
    uint32_t ua = 0;  // A units of the current stage already written
    bool ok = true;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      const int32_t n1 = P.kNStep[0], n2 = P.kNStep[1], nJJ = P.n1p >> 3;
      const int64_t p = v.row0 + v.pair * kPairRows + t * kTileM + row;
      const bool valid = p < v.row0 + v.rows;
      double x0 = 0.0, x1 = 0.0;
      if (valid && RF_IN_BOUNDS(p * 3 + 2, P.n * 3, err)) {
        x0 = v.x[p * 3 + 0] / P.corrL[0];
        x1 = v.x[p * 3 + 1] / P.corrL[1];
      }
      const float2 e2step = axis_phasor(P.kDelta[1], 1, x1);
      const int32_t oNR = P.oNR;
      // E1(u) of block 0 and the block step E1(8), from FP64-reduced phases
      // once per work item; block jj follows from block jj-1 by one complex
      // product per phasor (the direct FP64 reduction and sincos of 8
      // phasors per block and chunk took 13 % of the kernel's time)
      float2 e1base[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) e1base[u] = axis_phasor(P.kDelta[0], u, x0);
      const float2 e1step = axis_phasor(P.kDelta[0], 8, x0);
      for (int32_t c = 0; c < oNR && ok; ++c) {
        // K-steps in order j = 0, 1, ... (i2 fastest, then s2, then jj);
        // the TF32 and stage-end flags read 32 at a time
        int32_t j = 0;
        uint32_t aw = 0, ew = 0;
        float2 e1cur[8];
        for (int32_t jj = 0; jj < nJJ && ok; ++jj) {
          // the block's 8 axis-1 phasors E1(8 jj + u), zero past n1
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (jj > 0) {
              const float2 q = e1cur[u];
              e1cur[u] = make_float2(q.x * e1step.x - q.y * e1step.y, q.x * e1step.y + q.y * e1step.x);
            } else {
              e1cur[u] = e1base[u];
            }
          }
          float2 e1[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) e1[u] = (8 * jj + u < n1) ? e1cur[u] : make_float2(0.f, 0.f);
          for (int32_t s2 = 0; s2 < 2 && ok; ++s2) {
            float2 e2 = make_float2(1.f, 0.f);  // E2(i2), walked by angle addition
            for (int32_t i2 = 0; i2 < n2; ++i2) {
              const float2 E = make_float2(e2.x, s2 ? -e2.y : e2.y);
              if ((j & 31) == 0) {
                aw = P.aLoMask[j >> 5];
                ew = P.oStageEnd[j >> 5];
              }
              const bool tf = (aw >> (j & 31)) & 1u, end = (ew >> (j & 31)) & 1u;  // a TF32 K-step
              // A stage is written once its barrier says the MMAs have
              // released it; the proxy fence and the arrival are paid once
              // per stage, after its last K-step.
              if (ua == 0 && !mbar_wait_warp(&bars->empty[s], ph ^ 1, abort_flag)) {
                ok = false;
                break;
              }
              float2 pv[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                const float2 q = e1[u];
                pv[u] = make_float2(q.x * E.x - q.y * E.y, q.x * E.y + q.y * E.x);
              }
              unsigned char* A = slots + (size_t)s * slotBytes + ua * kAUnitBytes + t * kATileBytes + rowOff;
              if (TF32 && tf) {
                // TF32 K-step: unit 0 holds groups 0-3 (K 0-7), unit 1 groups
                // 4-7, each unit's core-matrix columns two groups (re, im)
#pragma unroll
                for (int h2 = 0; h2 < 4; ++h2) {
                  const float2 p0 = pv[2 * h2], p1 = pv[2 * h2 + 1];
                  *reinterpret_cast<uint4*>(A + (h2 >> 1) * kAUnitBytes + (h2 & 1) * 2048) =
                      make_uint4(tf32_bits(p0.x), tf32_bits(p0.y), tf32_bits(p1.x), tf32_bits(p1.y));
                }
              } else {
                uint32_t hi[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) hi[u] = pack16<PREC>(pv[u].x, pv[u].y);
                *reinterpret_cast<uint4*>(A) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<uint4*>(A + 2048) = make_uint4(hi[4], hi[5], hi[6], hi[7]);
              }
              ua += tf ? 2u : 1u;
              if (end) {
                ua = 0;
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars->full[s]);
                if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
              }
              e2 = make_float2(e2.x * e2step.x - e2.y * e2step.y, e2.x * e2step.y + e2.y * e2step.x);
              ++j;
            }
          }
        }
      }
    }
    if (!ok) outer_abort(bars, err);
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3, t = (warp - kEpiWarp0) >> 2;
    const int row = q * 32 + lane;
    const uint32_t taddr0 = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(t * kAccCols);
    constexpr int LH = LPAD / 8;  // 16-column pieces per realization
    uint32_t accPh = 0;
    bool ok = true;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      const int64_t p = v.row0 + v.pair * kPairRows + t * kTileM + row;
      const bool valid = p < v.row0 + v.rows;
      const double x2 = valid ? v.x[p * 3 + 2] / P.corrL[2] : 0.0;
      double bw = 0.0;  // localization blend: weight and group index of this point
      int64_t bg = 0;
      if (P.blend && valid) bw = blend_weight(P, p, &bg);
      float2 e3[LPAD];
#pragma unroll
      for (int u = 0; u < LPAD; ++u)
        e3[u] = (u < P.kNStep[2]) ? axis_phasor(P.kDelta[2], u, x2) : make_float2(0.f, 0.f);
      const int32_t oNR = P.oNR, oRc = P.oRc, nmcBlk = P.nmcBlk;
      const int64_t rOff = P.rOff, n = P.n, nOut = P.blend ? P.gTotal : P.n;
      [[maybe_unused]] const int64_t outLen = (int64_t)P.Nmc * nOut;  // the index checks' bound
      const bool blend = P.blend, marg = P.applyMarginal, logn = P.lognormal;
      const double outScale = P.outScale, margSd = P.margSd, margAvg = P.margAvg;
      for (int32_t c = 0; c < oNR; ++c) {
        if (!mbar_wait_warp(&bars->acc_full, accPh, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const int32_t rc = min(oRc, nmcBlk - c * oRc);
        for (int32_t rl = 0; rl < rc; ++rl) {
          // the realization's 2 LPAD columns in 32-column round trips (a load
          // then a wait for it; the last piece of an odd LH is 16 columns)
          float acc = 0.f;
#pragma unroll
          for (int h = 0; h < LH; h += 2) {
            uint32_t y[32];
            const uint32_t col = taddr0 + (uint32_t)(rl * 2 * LPAD + 16 * h);
            if (h + 1 < LH) tmem_ld32(col, y);
            else tmem_ld16(col, y);
            tmem_ld_wait();
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              if (h + (u >> 3) < LH) {
                acc = fmaf(e3[8 * h + u].x, __uint_as_float(y[2 * u]), acc);
                acc = fmaf(e3[8 * h + u].y, __uint_as_float(y[2 * u + 1]), acc);
              }
            }
          }
          if (valid) {
            const int64_t r = rOff + (int64_t)c * oRc + rl;
            if (blend) {
              if (RF_IN_BOUNDS(r * nOut + bg, outLen, err))
                atomicAdd(&v.out[r * nOut + bg], bw * ((double)acc * outScale));
            } else if (RF_IN_BOUNDS(r * n + p, outLen, err)) {
              double f = (double)acc * outScale;
              if (marg) {
                f = f * margSd + margAvg;
                if (logn) f = exp(f);
              }
              v.out[r * n + p] = f;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars->acc_empty[t]);
        accPh ^= 1;
      }
    }
    if (!ok) outer_abort(bars, err);
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kIssuerWarp) tmem_dealloc(tbase, kOuterTmemCols);
}

template <int PREC, int LPAD>
__global__ void __launch_bounds__(kOuterThreads, 1) rf_outer_kernel(const __grid_constant__ OuterArgs a) {
  const int64_t tiles = (a.rows + kTileM - 1) / kTileM;
  const SingleOuterWork w{&a, (tiles + 1) / 2};
  outer_body<PREC, LPAD>(w, a.S, a.slotBytes, a.aBytes, a.err);
}


// Stage layout: the A area (kOuterStageUnits units of kAUnitBytes), then
// kOuterStageUnits B units of bUnit bytes (one K-step block of B).
int32_t outer_stage_bytes(int64_t bUnit) {
  return (int32_t)((kStageABytes + kOuterStageUnits * bUnit + 127) / 128 * 128);
}

template <int PREC, int LPAD>
cudaError_t launch_outer_t(const OuterArgs& a, size_t smem, int grid, cudaStream_t st) {
  auto fn = rf_outer_kernel<PREC, LPAD>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, kOuterThreads, smem, st>>>(a);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_outer_p(const OuterArgs& a, size_t smem, int grid, cudaStream_t st) {
  switch (a.P.lPad) {
    case 8: return launch_outer_t<PREC, 8>(a, smem, grid, st);
    case 16: return launch_outer_t<PREC, 16>(a, smem, grid, st);
    case 24: return launch_outer_t<PREC, 24>(a, smem, grid, st);
    case 32: return launch_outer_t<PREC, 32>(a, smem, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

// Stages of slotBytes that fit the shared memory, and the bytes to request
// (0 when fewer than two fit).  More than half of the SM's shared memory is
// requested so that one CTA (and its 512 TMEM columns) sits on an SM.
size_t outer_fit(int32_t slotBytes, int* stages, int maxStages = 0) {
  const size_t limit = 227 * 1024, floor = 120 * 1024;
  int S = (int)((limit - kOuterHeader) / (size_t)slotBytes);
  if (S > kOuterMaxSlots) S = kOuterMaxSlots;
  if (maxStages > 0 && S > maxStages) S = maxStages;
  if (stages) *stages = S;
  if (S < 2) return 0;
  const size_t total = (size_t)kOuterHeader + (size_t)S * slotBytes;
  return total < floor ? floor : total;
}

}  // namespace

size_t outer_smem_bytes(const Plan& P, int* stages) {
  if (P.oPair) return outer_pair_smem_bytes(P, stages);
  return outer_fit(outer_stage_bytes(P.oKstepBytes), stages);
}

cudaError_t launch_outer(const Plan& P, const double* dX, const void* dB, double* dOut, int64_t row0, int64_t rows,
                         uint32_t* dErr, int numSMs, cudaStream_t st) {
  if (P.oPair) return launch_outer_pair(P, dX, dB, dOut, row0, rows, dErr, numSMs, st);
  OuterArgs a;
  a.P = P;
  a.x = dX;
  a.B = reinterpret_cast<const unsigned char*>(dB);
  a.out = dOut;
  a.err = dErr;
  a.row0 = row0;
  a.rows = rows;
  a.aBytes = kStageABytes;
  a.slotBytes = outer_stage_bytes(P.oKstepBytes);
  int S = 0;
  const size_t smem = outer_smem_bytes(P, &S);
  if (smem == 0) return cudaErrorInvalidValue;
  a.S = S;
  const int64_t tiles = (rows + kTileM - 1) / kTileM;
  const int64_t pairs = (tiles + 1) / 2;
  const int grid = (int)(pairs < numSMs ? pairs : numSMs);
  if (P.prec == PREC_FP16) return launch_outer_p<PREC_FP16>(a, smem, grid, st);
  return launch_outer_p<PREC_BF16>(a, smem, grid, st);
}

}  // namespace rfb
