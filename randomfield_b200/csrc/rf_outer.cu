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
// (rf_tables.cu, outer_element).  Against the plain contraction
// [cos Kx | sin Kx] x [a cos phi; -a sin phi] this is the same number of
// multiply-adds and the same operand bytes, but the generated operand shrinks
// from 2K = 8 n1 n2 n3 to 2G = 4 n1 n2 values per point and chunk, the MMAs
// run at N = 2 lPad x (realizations per chunk), up to 256, and the last
// contraction over i3 (2 lPad multiply-adds per output) runs in the epilogue
// in FP32 with FP64-reduced per-point phasors.
//
// One persistent CTA per SM; a work item is a pair of 128-point tiles that
// share every B stage (M = 256 per operand byte streamed from L2).  The
// realization block is cut into N chunks of oRc realizations (TMEM: one
// 256-column accumulator per tile); for each chunk the K-steps (16 K = 8
// outer groups of consecutive i1) stream through a ring of shared-memory
// stages of two K-steps, each K-step with both tiles' A (hi, and lo where the
// plan keeps it) and B's K-step block (hi, and lo).
//
// Warp roles (576 threads):
//   warp 0      MMA issuer: the warp runs the stage loop, one elected lane
//               issues tcgen05.mma (A and B by shared-memory descriptor, D in
//               TMEM) and tcgen05.commit;
//   warp 1      producer (one thread): 1-D bulk copies (TMA, no multicast) of
//               a stage's B blocks from HBM/L2 into the ring;
//   warps 2-9   generators: one point each (256 = two tiles); per K-step the
//               8 outer phasors E1(i1) E2(i2)^{s2} of the point, rounded to
//               16 bits (and the lo residual), stored in the K-major core-
//               matrix layout; E1 from FP64-reduced phases per work item, E2
//               walked by angle addition per chunk;
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
// K-steps per ring stage: one full/empty barrier pair, one bulk copy, one
// generator fence and one commit serve kStageK K-steps.  A K-step's MMAs keep
// the tensor pipe busy for about as long as the issuing thread takes to issue
// them, so the per-stage bookkeeping (barrier probe, commit, loop control)
// shows up directly in the kernel's time; two K-steps per stage halve it.
// A chunk's K-step count 2 n2 nJJ is always even.
constexpr int kStageK = 2;

struct OuterBars {
  uint64_t full[kOuterMaxSlots];   // per stage: 8 generator warps + producer (bytes)
  uint64_t empty[kOuterMaxSlots];  // per stage: MMA commit
  uint64_t acc_full;               // MMA commit after a chunk's last K-step
  uint64_t acc_empty[2];           // the 4 epilogue warps of a tile
  uint64_t done;
  uint32_t tmem_base;
  int abort_flag;
  // the issuer's table of the current item's K-steps: bit 0 B lo, bit 1 A lo
  uint8_t kflags[kOuterMaxKsteps];
};
constexpr int kOuterHeader = 512;
static_assert(sizeof(OuterBars) <= kOuterHeader, "header");

struct OuterArgs {
  Plan P;
  const double* x;
  const unsigned char* B;
  double* out;
  uint32_t* err;
  int64_t row0, rows;
  int32_t S;          // ring stages
  int32_t slotBytes;  // one stage: kStageK A areas, then kStageK B blocks; 128-byte multiple
  int32_t aBytes;     // one K-step's A area: two tiles x 4 KB, twice with a lo term
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

// This CTA's slice [ctaStart[b], ctaStart[b+1]) of a grouped work list; an
// item's `tile` field holds its pair index.
struct GroupOuterWork {
  const OuterGroupArgs* g;
  int64_t begin, end;
  __device__ __forceinline__ int64_t count() const { return end - begin; }
  __device__ __forceinline__ void get(int64_t i, OuterView& v) const {
    const GroupItem it = g->items[begin + i];
    const GroupSub& s = g->subs[it.sub];
    v.P = &s.P;
    v.x = s.x;
    v.out = s.out;
    v.B = s.B;
    v.row0 = 0;
    v.rows = s.P.n;
    v.pair = it.tile;
  }
};

__device__ __forceinline__ void outer_abort(OuterBars* bars, uint32_t* err) {
  *reinterpret_cast<volatile int*>(&bars->abort_flag) = 1;
  atomicOr(err, kErrTimeout);
}

__device__ __forceinline__ double outer_finish(const Plan& P, float acc) {
  double v = (double)acc * P.outScale;
  if (P.applyMarginal) {
    v = v * P.margSd + P.margAvg;
    if (P.lognormal) v = exp(v);
  }
  return v;
}

template <int PREC>
__device__ __forceinline__ uint32_t pack16(float lo, float hi) {
  return PREC == PREC_FP16 ? pack_f16x2(lo, hi) : pack_bf16x2(lo, hi);
}
// The 16-bit values of a packed pair back in FP32.
template <int PREC>
__device__ __forceinline__ float2 unpack16(uint32_t w) {
  if (PREC == PREC_FP16) {
    const __half2 h = *reinterpret_cast<const __half2*>(&w);
    return __half22float2(h);
  }
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
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
        for (int32_t c = 0; c < P.oNR && ok; ++c) {
          const unsigned char* src = v.B + (int64_t)c * P.oChunkBytes;
          for (int32_t j = 0; j < P.oNK; j += kStageK) {
            if (!mbar_wait(&bars->empty[s], ph ^ 1, abort_flag)) {
              ok = false;
              break;
            }
            // the stage's B blocks lie back to back in the operand
            uint32_t bytes = 0;
            for (int g = 0; g < kStageK; ++g)
              bytes += (uint32_t)(outer_b_lo(P, j + g) ? 2 * P.oKstepBytes : P.oKstepBytes);
            if (!RF_IN_BOUNDS((src - v.B) + bytes - 1, operand_bytes(P), err)) {
              ok = false;  // no copy: the stage stays empty, and the waits on it end the kernel
              break;
            }
            mbar_arrive_expect_tx(&bars->full[s], bytes);
            bulk_g2s(slots + (size_t)s * slotBytes + kStageK * aBytes, src, bytes, &bars->full[s]);
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
    // when the probe failed.  K-step 1 of a stage accumulates in any order
    // (acc = 1), so its tile-1 hi MMA goes last, after the probe, in every
    // case.  The lo K-steps are the top of a variance ranking and come in
    // runs: stages whose K-steps both have or both lack every lo term take a
    // straight path; the others issue the lo terms through a guard predicate
    // from the item's flag table (no branch between MMAs; a branch per MMA
    // costs the issuing thread a resolution it cannot hide).
    static_assert(kStageK == 2, "the issuer writes out two K-steps per stage");
    const bool leader = elect_one();
    uint32_t s = 0, ph = 0, accPh = 0;
    bool ok = true, ready = false;  // ready: full[s] of the next stage already observed
    const uint32_t ab = PREC == PREC_FP16 ? 0u : 1u;
    const uint64_t aStepLo = (uint64_t)((2 * kATileBytes) >> 4);  // descriptor step to the lo A tiles
    const uint64_t aStepT = (uint64_t)(kATileBytes >> 4);         // descriptor step to tile 1's A
    const uint64_t aStepK = (uint64_t)((uint32_t)aBytes >> 4);    // descriptor step to the next K-step's A
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      for (int32_t j = lane; j < P.oNK; j += 32)
        bars->kflags[j] = (uint8_t)((outer_b_lo(P, j) ? 1u : 0u) | (outer_a_lo(P, j) ? 2u : 0u));
      __syncwarp();
      const uint64_t bStepLo = (uint64_t)(P.oKstepBytes >> 4);
      const uint32_t nRows = (uint32_t)(2 * P.lPad * P.oRc);  // B rows (N) of a full chunk
      for (int32_t c = 0; c < P.oNR && ok; ++c) {
        const int32_t rc = min(P.oRc, P.nmcBlk - c * P.oRc);
        const uint32_t idesc = make_idesc(ab, 128u, (uint32_t)(2 * P.lPad * rc));
        // both accumulators are free once the epilogue has read the last chunk
        if (!mbar_wait_warp(&bars->acc_empty[0], accPh ^ 1, abort_flag) ||
            !mbar_wait_warp(&bars->acc_empty[1], accPh ^ 1, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int32_t j = 0; j < P.oNK; j += kStageK) {
          if (!ready && !mbar_wait_warp(&bars->full[s], ph, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t base = smem_u32(slots + (size_t)s * slotBytes);
          const uint64_t aDesc = make_sdesc(base, 2048u, 128u);
          const uint64_t bDesc = make_sdesc(base + (uint32_t)(kStageK * aBytes), nRows * 16u, 128u);
          // both K-steps' flags in one load (j is even)
          const uint32_t f = *reinterpret_cast<const uint16_t*>(&bars->kflags[j]);
          const uint32_t bLo0 = f & 1u, aLo0 = f & 2u, bLo1 = f & 0x100u, aLo1 = f & 0x200u;
          const uint32_t acc = j > 0 ? 1u : 0u;
          const uint64_t aDesc1 = aDesc + aStepK;
          const uint64_t bDesc1 = bDesc + (bLo0 ? 2 * bStepLo : bStepLo);
          const uint32_t sn = (s + 1 == (uint32_t)S) ? 0u : s + 1;
          const uint32_t phn = (s + 1 == (uint32_t)S) ? ph ^ 1 : ph;
          const bool more = (j + kStageK < P.oNK) || (c + 1 < P.oNR) || (i + 1 < count);
          if (leader) {
            if (f == 0u) {
              mma_ss(tbase, aDesc, bDesc, idesc, acc);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc + aStepT, bDesc, idesc, acc);
              mma_ss(tbase, aDesc1, bDesc1, idesc, 1u);
            } else if (f == 0x0303u) {
              mma_ss(tbase, aDesc, bDesc, idesc, acc);
              mma_ss(tbase, aDesc, bDesc + bStepLo, idesc, 1u);
              mma_ss(tbase, aDesc + aStepLo, bDesc, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc + aStepT, bDesc, idesc, acc);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc + aStepT, bDesc + bStepLo, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc + aStepT + aStepLo, bDesc, idesc, 1u);
              mma_ss(tbase, aDesc1, bDesc1, idesc, 1u);
              mma_ss(tbase, aDesc1, bDesc1 + bStepLo, idesc, 1u);
              mma_ss(tbase, aDesc1 + aStepLo, bDesc1, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc1 + aStepT, bDesc1 + bStepLo, idesc, 1u);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc1 + aStepT + aStepLo, bDesc1, idesc, 1u);
            } else {
              mma_ss(tbase, aDesc, bDesc, idesc, acc);
              mma_ss_if(tbase, aDesc, bDesc + bStepLo, idesc, 1u, bLo0);
              mma_ss_if(tbase, aDesc + aStepLo, bDesc, idesc, 1u, aLo0);
              mma_ss(tbase + (uint32_t)kAccCols, aDesc + aStepT, bDesc, idesc, acc);
              mma_ss_if(tbase + (uint32_t)kAccCols, aDesc + aStepT, bDesc + bStepLo, idesc, 1u, bLo0);
              mma_ss_if(tbase + (uint32_t)kAccCols, aDesc + aStepT + aStepLo, bDesc, idesc, 1u, aLo0);
              mma_ss(tbase, aDesc1, bDesc1, idesc, 1u);
              mma_ss_if(tbase, aDesc1, bDesc1 + bStepLo, idesc, 1u, bLo1);
              mma_ss_if(tbase, aDesc1 + aStepLo, bDesc1, idesc, 1u, aLo1);
              mma_ss_if(tbase + (uint32_t)kAccCols, aDesc1 + aStepT, bDesc1 + bStepLo, idesc, 1u, bLo1);
              mma_ss_if(tbase + (uint32_t)kAccCols, aDesc1 + aStepT + aStepLo, bDesc1, idesc, 1u, aLo1);
            }
          }
          ready = __all_sync(0xffffffffu, more && mbar_test_wait(&bars->full[sn], phn));
          if (leader) {
            mma_ss(tbase + (uint32_t)kAccCols, aDesc1 + aStepT, bDesc1, idesc, 1u);
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
    int g = 0;  // the next K-step's place in its stage
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
      float2 e1[kOuterMaxN1P];
#pragma unroll
      for (int u = 0; u < kOuterMaxN1P; ++u)
        e1[u] = (u < n1) ? axis_phasor(P.kDelta[0], u, x0) : make_float2(0.f, 0.f);
      const float2 e2step = axis_phasor(P.kDelta[1], 1, x1);
      for (int32_t c = 0; c < P.oNR && ok; ++c) {
        for (int32_t s2 = 0; s2 < 2 && ok; ++s2) {
          float2 e2 = make_float2(1.f, 0.f);  // E2(i2), walked by angle addition
          for (int32_t i2 = 0; i2 < n2 && ok; ++i2) {
            const float2 E = make_float2(e2.x, s2 ? -e2.y : e2.y);
            // A stage is written once its barrier says the MMAs have
            // released it; the proxy fence and the arrival are paid once per
            // stage, after its last K-step (stages run across the blocks).
#pragma unroll
            for (int jj = 0; jj < kOuterMaxN1P / 8; ++jj) {
              if (jj < nJJ) {
                const int32_t j = jj + nJJ * (i2 + n2 * s2);
                if (g == 0 && !mbar_wait_warp(&bars->empty[s], ph ^ 1, abort_flag)) {
                  ok = false;
                  break;
                }
                float2 pv[8];
                uint32_t hi[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                  const float2 q = e1[8 * jj + u];
                  pv[u] = make_float2(q.x * E.x - q.y * E.y, q.x * E.y + q.y * E.x);
                  hi[u] = pack16<PREC>(pv[u].x, pv[u].y);
                }
                unsigned char* A = slots + (size_t)s * slotBytes + g * aBytes + t * kATileBytes + rowOff;
                *reinterpret_cast<uint4*>(A) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<uint4*>(A + 2048) = make_uint4(hi[4], hi[5], hi[6], hi[7]);
                if (outer_a_lo(P, j)) {  // the residual of the 16-bit rounding, rounded again
                  uint32_t lo[8];
#pragma unroll
                  for (int u = 0; u < 8; ++u) {
                    const float2 h = unpack16<PREC>(hi[u]);
                    lo[u] = pack16<PREC>(pv[u].x - h.x, pv[u].y - h.y);
                  }
                  *reinterpret_cast<uint4*>(A + 2 * kATileBytes) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
                  *reinterpret_cast<uint4*>(A + 2 * kATileBytes + 2048) = make_uint4(lo[4], lo[5], lo[6], lo[7]);
                }
                if (++g == kStageK) {
                  g = 0;
                  fence_proxy_async_smem();
                  __syncwarp();
                  if (lane == 0) mbar_arrive(&bars->full[s]);
                  if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
                }
              }
            }
            e2 = make_float2(e2.x * e2step.x - e2.y * e2step.y, e2.x * e2step.y + e2.y * e2step.x);
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
      for (int32_t c = 0; c < P.oNR; ++c) {
        if (!mbar_wait_warp(&bars->acc_full, accPh, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const int32_t rc = min(P.oRc, P.nmcBlk - c * P.oRc);
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
            const int64_t r = (int64_t)P.rOff + c * P.oRc + rl;
            if (P.blend) {
              if (RF_IN_BOUNDS(r * P.gTotal + bg, (int64_t)P.Nmc * P.gTotal, err))
                atomicAdd(&v.out[r * P.gTotal + bg], bw * ((double)acc * P.outScale));
            } else if (RF_IN_BOUNDS(r * P.n + p, (int64_t)P.Nmc * P.n, err)) {
              v.out[r * P.n + p] = outer_finish(P, acc);
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

template <int PREC>
__global__ void __launch_bounds__(kOuterThreads, 1) rf_outer_group_kernel(const __grid_constant__ OuterGroupArgs g) {
  const GroupOuterWork w{&g, g.ctaStart[blockIdx.x], g.ctaStart[blockIdx.x + 1]};
  outer_body<PREC, kGroupLPad>(w, g.S, g.slotBytes, g.aBytes, g.err);
}

// Stage layout of a plan: per K-step an A area (two tiles, twice with a lo
// term somewhere) and a B block (twice with a lo block somewhere); a stage
// holds kStageK A areas and then kStageK B blocks.
void outer_slot(const Plan& P, int32_t* aBytes, int32_t* bBytes) {
  bool aLo = false, bLo = false;
  for (int32_t j = 0; j < P.oNK; ++j) {
    aLo = aLo || outer_a_lo(P, j);
    bLo = bLo || outer_b_lo(P, j);
  }
  *aBytes = 2 * kATileBytes * (aLo ? 2 : 1);
  *bBytes = (int32_t)(P.oKstepBytes * (bLo ? 2 : 1));
}

int32_t outer_stage_bytes(int32_t aBytes, int32_t bBytes) {
  return (kStageK * (aBytes + bBytes) + 127) / 128 * 128;
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
  int32_t aBytes = 0, bBytes = 0;
  outer_slot(P, &aBytes, &bBytes);
  return outer_fit(outer_stage_bytes(aBytes, bBytes), stages);
}

size_t outer_group_layout(const Plan* const* plans, size_t count, int maxStages, OuterGroupArgs* g) {
  int32_t aMax = 2 * kATileBytes, bMax = 0;
  for (size_t i = 0; i < count; ++i) {
    int32_t a = 0, b = 0;
    outer_slot(*plans[i], &a, &b);
    aMax = a > aMax ? a : aMax;
    bMax = b > bMax ? b : bMax;
  }
  g->aBytes = aMax;
  g->slotBytes = outer_stage_bytes(aMax, bMax);
  int S = 0;
  const size_t smem = outer_fit(g->slotBytes, &S, maxStages);
  g->S = S;
  return smem;
}

cudaError_t outer_group_set_smem(int prec, size_t smem) {
  const int b = (int)smem;
  if (prec == PREC_FP16) return cudaFuncSetAttribute(rf_outer_group_kernel<PREC_FP16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  return cudaFuncSetAttribute(rf_outer_group_kernel<PREC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

cudaError_t launch_outer_group(int prec, const OuterGroupArgs& g, size_t smem, int grid, cudaStream_t st) {
  if (prec == PREC_FP16) rf_outer_group_kernel<PREC_FP16><<<grid, kOuterThreads, smem, st>>>(g);
  else rf_outer_group_kernel<PREC_BF16><<<grid, kOuterThreads, smem, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_outer(const Plan& P, const double* dX, const void* dB, double* dOut, int64_t row0, int64_t rows,
                         uint32_t* dErr, int numSMs, cudaStream_t st) {
  OuterArgs a;
  a.P = P;
  a.x = dX;
  a.B = reinterpret_cast<const unsigned char*>(dB);
  a.out = dOut;
  a.err = dErr;
  a.row0 = row0;
  a.rows = rows;
  int32_t bBytes = 0;
  outer_slot(P, &a.aBytes, &bBytes);
  a.slotBytes = outer_stage_bytes(a.aBytes, bBytes);
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
