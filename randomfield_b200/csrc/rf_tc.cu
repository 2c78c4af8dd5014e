// rf_tc.cu -- the spectral-sum contraction on tcgen05 tensor cores.
//
// Replaces the hot loop of gen_Std_Gauss_Shinozuka (randomFieldND.f90:276-330:
// DGEMM k.x + phi, cos, DGEMM with sqrt(S)) and of the isotropic generator
// (:456-490) by one persistent kernel per launch:
//
//   D (128 points x Nmc, FP32 in TMEM) += A (128 x 16, trig tile in TMEM)
//                                         x B (16 x Nmc, amplitude/phase in SMEM)
//
// Two launches share one pipeline body: rf_tc_kernel runs the tiles of one
// request, rf_group_kernel runs a list of (request block, tile) work items of
// many requests per CTA (the batched and serving forms), choosing the
// generator per tile.
//
// Warp roles (one CTA per SM; 320 threads, 576 for GEN_TABLE kernels):
//   warp 0      MMA issuer: the warp runs the stage loop, one elected lane
//               issues tcgen05.mma kind::f16 (A from TMEM, B by descriptor
//               from SMEM) and tcgen05.commit, which frees stages;
//   warps 1-G   generators (G = 8, or 16 for GEN_TABLE): build the trig tile
//               of each stage straight into TMEM (tcgen05.st), lane = point;
//               the G/4 warps of a TMEM lane quarter split the columns; after
//               the last stage of a tile they run the fused epilogue
//               (tcgen05.ld, ampMult, marginal map, FP64 stores; or the
//               localization blend's weighted add into the group field);
//   warp G+1    producer (one thread): 1-D bulk copies (TMA) of B stages from
//               HBM/L2 into SMEM; no multicast.
// The issuing thread can run only about one MMA ahead of the tensor core, so
// anything it does between MMAs idles the tensor pipe: it waits on one
// barrier per stage (the bulk copy completes on the same barrier the
// generators arrive on), probes the next stage's barrier while the last MMA
// of the current stage runs, and issues the MMAs of a stage as straight-line
// code (the kernel is specialised on the padded axis-3 length LPAD, which
// fixes the MMAs per stage; a runtime-guarded unrolled loop cost a branch
// resolution per MMA and halved the tensor throughput).
// Measured balance (128^3 workload, BF16): the MMAs of a stage take about
// 770 cycles; the generators of the three sub-partitions without a service
// warp need about 750, those sharing a sub-partition with the issuer about
// 880, which sets the stage period (about 1130 cycles with the barriers).
// TMEM: accumulator columns [0, aCol0), then the A slots (SlotLayout).
// Every wait is bounded (globaltimer); on expiry the kernel raises an error
// word, drains its own async work, frees TMEM and returns.
#include "rf_blend.cuh"
#include "rf_device.cuh"
#include "rf_gen.cuh"
#include "rf_launch.h"

namespace rfb {

namespace {

constexpr int kMmaWarp = 0;
constexpr int kGenWarp0 = 1;  // generators: warps 1 .. Roles::kGen
// Warp roles of a kernel variant.  GEN_TABLE kernels run 16 generator warps
// (four per TMEM lane quarter, each a quarter of the stage's columns): their
// generators are latency-bound on the FP64 -> SFU chain of each pair, and
// four warps per sub-partition hide what two could not (200k points,
// isotropic 64 x 64 wavevectors: 1.08 -> 0.96 ms).  GEN_GRID3 kernels keep 8: at 16 the
// 128^3 workload ran 3 % slower (it is held at the 1000 W power cap, where
// more warps only spend more energy per stage), and the grouped kernel holds
// both generators' state, more registers than 576 threads have.
template <int GEN>
struct Roles {
  static constexpr int kGen = GEN == GEN_TABLE ? 16 : 8;
  static constexpr int kParts = kGen / 4;  // column parts per lane quarter
  static constexpr int kProd = kGenWarp0 + kGen;
  static constexpr int kThreads = (kProd + 1) * 32;
};
constexpr int kMaxStages = 8;
constexpr uint32_t kTmemCols = 512;
constexpr int kTableSteps = kTableChunk / 8;  // MMAs (K = 16) per GEN_TABLE stage

struct Bars {
  uint64_t full[kMaxStages];   // generators (8 warps) + producer (bytes)
  uint64_t kfull[kMaxStages];  // GEN_TABLE wavevector chunk (bytes)
  uint64_t empty[kMaxStages];
  uint64_t acc_full;
  uint64_t acc_empty;
  uint64_t done;
  uint32_t tmem_base;
  int abort_flag;
};
constexpr int kHeaderBytes = 512;
static_assert(sizeof(Bars) <= kHeaderBytes, "header");

struct TcArgs {
  Plan P;
  const double* x;
  const unsigned char* B;
  const double* ktab;
  double* out;
  uint32_t* err;
  int64_t row0, rows;
  SlotLayout L;
};

// One tile of work as every role sees it.
struct TileView {
  const Plan* P;
  const double* x;
  double* out;
  const unsigned char* B;
  const double* ktab;
  int64_t row0, rows;  // point range of the request covered by the launch
  int64_t tile;        // tile (128 points) inside that range
};

// The tiles blockIdx.x, blockIdx.x + gridDim.x, ... of one request.
struct SingleWork {
  const TcArgs* a;
  int64_t numTiles;
  __device__ __forceinline__ int64_t count() const {
    return (int64_t)blockIdx.x < numTiles ? (numTiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  }
  __device__ __forceinline__ void get(int64_t i, TileView& v) const {
    v.P = &a->P;
    v.x = a->x;
    v.out = a->out;
    v.B = a->B;
    v.ktab = a->ktab;
    v.row0 = a->row0;
    v.rows = a->rows;
    v.tile = blockIdx.x + i * gridDim.x;
  }
};

// This CTA's slice [ctaStart[b], ctaStart[b+1]) of a grouped work list.
struct GroupWork {
  const GroupArgs* g;
  int64_t begin, end;
  __device__ __forceinline__ int64_t count() const { return end - begin; }
  __device__ __forceinline__ void get(int64_t i, TileView& v) const {
    const GroupItem it = g->items[begin + i];
    const GroupSub& s = g->subs[it.sub];
    v.P = &s.P;
    v.x = s.x;
    v.out = s.out;
    v.B = s.B;
    v.ktab = s.ktab;
    v.row0 = 0;
    v.rows = s.P.n;
    v.tile = it.tile;
  }
};

__device__ __forceinline__ void raise_abort(Bars* bars, uint32_t* err) {
  *reinterpret_cast<volatile int*>(&bars->abort_flag) = 1;
  atomicOr(err, kErrTimeout);
}

// Epilogue value: ampMult (and FP16 unscale), then multiVariateTransformation
// (randomFieldND.f90:171-176) unless a normalisation pass follows.
__device__ __forceinline__ double finish_value(const Plan& P, float acc) {
  double v = (double)acc * P.outScale;
  if (P.applyMarginal) {
    v = v * P.margSd + P.margAvg;
    if (P.lognormal) v = exp(v);
  }
  return v;
}

// The MMAs of one stage from the elected lane, with the probe of the next
// stage's full barrier between the last two; returns the probe (warp-uniform).
// F8: kind::f8f6f4 (e4m3, K = 32 per MMA) instead of kind::f16 (K = 16); both
// consume 8 TMEM columns of A and 32 bytes of each B row per MMA.
template <bool F8>
__device__ __forceinline__ void mma_one(uint32_t tbase, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  if (F8) mma_ts_f8(tbase, a, b, idesc, acc);
  else mma_ts(tbase, a, b, idesc, acc);
}

// aLo > 0: the stage's A tile also holds its lo term aLo columns after the
// hi term, multiplied by the same B rows (one more MMA per K-step).
template <int STEPS, bool F8>
__device__ __forceinline__ bool issue_stage(bool leader, uint32_t tbase, uint32_t aBase, uint64_t d0, uint64_t jStep,
                                            uint32_t idesc, uint32_t acc0, bool more, uint64_t* fullNext,
                                            uint32_t phn, uint64_t* emptyBar, uint32_t aLo = 0) {
  static_assert(STEPS >= 2, "a stage holds at least two MMAs");
  if (leader) {
    mma_one<F8>(tbase, aBase, d0, idesc, acc0);  // the tile's first MMA overwrites D
#pragma unroll
    for (int j = 1; j < STEPS - 1; ++j) mma_one<F8>(tbase, aBase + 8u * j, d0 + jStep * j, idesc, 1u);
    if (aLo) {
#pragma unroll
      for (int j = 0; j < STEPS; ++j) mma_one<F8>(tbase, aBase + aLo + 8u * j, d0 + jStep * j, idesc, 1u);
    }
  }
  const bool ready = __all_sync(0xffffffffu, more && mbar_test_wait(fullNext, phn));
  if (leader) {
    mma_one<F8>(tbase, aBase + 8u * (STEPS - 1), d0 + jStep * (STEPS - 1), idesc, 1u);
    mma_commit(emptyBar);
  }
  __syncwarp();
  return ready;
}

// The pipeline of one CTA over the work items of `w`.
// GEN: GEN_TABLE, GEN_GRID3 (axis-3 length padded to LPAD) or GEN_MIXED
// (chosen per tile; its GEN_GRID3 tiles have lPad == LPAD).  TALO: a
// GEN_TABLE BF16 kernel whose plans carry the trig tile's lo term
// (tableALo); single-request kernels compile it apart, because the residual
// code in the generator loop cost the other GEN_TABLE requests 2.5 % even
// when skipped (the grouped kernel keeps it: its small table requests take
// the lo term).
template <int GEN, int PREC, int LPAD, bool TALO, class Work>
__device__ __forceinline__ void tc_body(const Work& w, const SlotLayout& L, uint32_t* err) {
  constexpr bool kHasGrid = GEN != GEN_TABLE;
  constexpr bool kHasTable = GEN != GEN_GRID3;
  constexpr bool kF8 = PREC == PREC_FP8;
  constexpr bool kHiLo = PREC == PREC_BF16 || PREC == PREC_FP8;
  // MMAs per stage: a GEN_GRID3 stage holds 2 groups x 2*LPAD (cos, sin) pairs,
  // a GEN_TABLE stage kTableChunk pairs; K = 16 (16-bit) or 32 (e4m3) per MMA
  constexpr int kGridSteps = (LPAD > 0 ? LPAD / 2 : 4) / (kF8 ? 2 : 1);
  constexpr int kTabSteps = kTableSteps / (kF8 ? 2 : 1);
  constexpr int kGenWarps = Roles<GEN>::kGen, kParts = Roles<GEN>::kParts, kProdWarp = Roles<GEN>::kProd;
  static_assert(!kHasGrid || kParts == 2, "GEN_GRID3 tiles: two column halves per lane quarter");
  extern __shared__ __align__(1024) unsigned char smem[];
  Bars* bars = reinterpret_cast<Bars*>(smem);
  unsigned char* sB = smem + kHeaderBytes;
  double* sK = reinterpret_cast<double*>(sB + L.ktabOff);
  volatile int* abort_flag = &bars->abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = L.S;
  const int64_t count = w.count();

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&bars->full[s], kGenWarps + 1);
      mbar_init(&bars->kfull[s], 1);
      mbar_init(&bars->empty[s], 1);
    }
    mbar_init(&bars->acc_full, 1);
    mbar_init(&bars->acc_empty, kGenWarps);
    mbar_init(&bars->done, 1);
    bars->abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(&bars->tmem_base, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = bars->tmem_base;

  if (warp == kProdWarp) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t s = 0, ph = 0;
      uint32_t ktabSlots = 0;  // slots whose last copy carried a wavevector chunk
      uint32_t kph = 0;        // per slot: parity of the kfull phase its next wavevector copy completes
      int64_t issued = 0;
      TileView v;
      for (int64_t i = 0; i < count && !*abort_flag; ++i) {
        w.get(i, v);
        const Plan& P = *v.P;
        const bool table = kHasTable && (GEN == GEN_TABLE || P.gen != GEN_GRID3);
        const int64_t nChunks = P.nChunks;
        int64_t off = 0;  // byte offset of stage ch in B (hi-only stages are half size)
        for (int64_t ch = 0; ch < nChunks; ++ch) {
          if (!mbar_wait(&bars->empty[s], ph ^ 1, abort_flag)) {
            raise_abort(bars, err);
            break;
          }
          const uint32_t bytes = (uint32_t)(stage_has_lo(P, ch) ? P.stageBytes : P.stageBytes / 2);
          if (!RF_IN_BOUNDS(off + bytes - 1, operand_bytes(P), err)) {
            raise_abort(bars, err);  // no copy: the waits on the slot end the kernel
            break;
          }
          mbar_arrive_expect_tx(&bars->full[s], bytes);
          bulk_g2s(sB + (size_t)s * L.slotBytes, v.B + off, bytes, &bars->full[s]);
          off += bytes;
          if (table) {
            mbar_arrive_expect_tx(&bars->kfull[s], (uint32_t)kKtabStageBytes);
            bulk_g2s(sK + s * kKtabStageDoubles, v.ktab + ch * kKtabStageDoubles, kKtabStageBytes, &bars->kfull[s]);
            ktabSlots |= 1u << s;
            kph ^= 1u << s;
          } else {
            ktabSlots &= ~(1u << s);
          }
          ++issued;
          if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
        }
      }
      if (*abort_flag) {
        // Drain: wait (bounded, ignoring the abort flag) for the copies still
        // in flight so that no bulk copy lands after the CTA exits.  A slot's
        // wavevector copy is done once its kfull phase completes; the B
        // copies complete_tx on full[s], whose generator arrivals may never
        // come, so those are waited for by time.
        volatile int never = 0;
        for (int k = 0; k < S && issued > 0; ++k, --issued) {
          if (s == 0) { s = S; ph ^= 1; }
          --s;
          if (ktabSlots & (1u << s)) mbar_wait(&bars->kfull[s], ((kph >> s) & 1u) ^ 1u, &never);
        }
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < 1000000ull) {
        }
      }
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------- MMA issuer
    // The whole warp runs the loop (its state stays warp-uniform; every
    // branch condition is made uniform by a warp vote); the lane elected once
    // here issues every MMA and commit, so that its commits cover its MMAs.
    // One elect for the kernel, not one per MMA: a warp-collective
    // instruction per MMA slowed the generator warps sharing this warp's
    // sub-partition by a fifth.  The hi/lo amplitude rows sit one above the
    // other in each B stage, so one MMA with N = bRows computes both products
    // into 2*nmcPad accumulator columns; the epilogue adds the halves.
    // Descriptors are advanced by plain adds of the start address field (it
    // cannot overflow: shared memory is below 256 KB).
    const bool leader = elect_one();
    const uint64_t sStep = (uint64_t)(L.slotBytes >> 4);
    uint32_t s = 0, ph = 0, accPh = 0;
    bool ok = true, ready = false;  // ready: full[s] of the next stage already observed
    TileView v;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      const bool grid = kHasGrid && (GEN == GEN_GRID3 || P.gen == GEN_GRID3);
      // A/B type field: F16 (0) or BF16 (1) for kind::f16, E4M3 (0) for kind::f8f6f4
      const uint32_t idescAll = make_idesc((PREC == PREC_FP16 || kF8) ? 0u : 1u, 128u, (uint32_t)P.bRows);
      const uint32_t lbo = (uint32_t)P.bRows * 16u, sbo = 128u;
      const uint64_t descAll = make_sdesc(smem_u32(sB), lbo, sbo);
      const uint64_t jStepAll = (uint64_t)((2u * lbo) >> 4);
      // hi-only stages (loSkip): N = nmcPad rows laid out for nmcPad
      const uint32_t idescHi = make_idesc((PREC == PREC_FP16 || kF8) ? 0u : 1u, 128u, (uint32_t)P.nmcPad);
      const uint64_t descHi = make_sdesc(smem_u32(sB), (uint32_t)P.nmcPad * 16u, sbo);
      const uint64_t jStepHi = (uint64_t)(((uint32_t)P.nmcPad * 32u) >> 4);
      const int64_t nChunks = P.nChunks;
      if (!mbar_wait_warp(&bars->acc_empty, accPh ^ 1, abort_flag)) { ok = false; break; }
      tc_fence_after();
      for (int64_t ch = 0; ch < nChunks; ++ch) {
        if (!ready && !mbar_wait_warp(&bars->full[s], ph, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t aBase = tbase + (uint32_t)L.aCol0 + s * (uint32_t)L.aStride;
        const bool lo = stage_has_lo(P, ch);
        const uint32_t idesc = lo ? idescAll : idescHi;
        const uint64_t jStep = lo ? jStepAll : jStepHi;
        const uint64_t d0 = (lo ? descAll : descHi) + sStep * s;
        const uint32_t sn = (s + 1 == (uint32_t)S) ? 0u : s + 1;
        const uint32_t phn = (s + 1 == (uint32_t)S) ? ph ^ 1 : ph;
        const bool more = (ch + 1 < nChunks) || (i + 1 < count);
        const uint32_t acc0 = ch != 0 ? 1u : 0u;
        if (kHasGrid && grid)
          ready = issue_stage<kGridSteps, kF8>(leader, tbase, aBase, d0, jStep, idesc, acc0, more, &bars->full[sn],
                                               phn, &bars->empty[s]);
        else
          ready = issue_stage<kTabSteps, kF8>(leader, tbase, aBase, d0, jStep, idesc, acc0, more, &bars->full[sn],
                                              phn, &bars->empty[s], (TALO && P.tableALo) ? (uint32_t)P.chunkK : 0u);
        s = sn;
        ph = phn;
      }
      if (!ok) break;
      if (leader) mma_commit(&bars->acc_full);
      __syncwarp();
      accPh ^= 1;
    }
    if (!ok && lane == 0) raise_abort(bars, err);
    // Drain every MMA the elected lane issued before TMEM is released.
    if (leader) mma_commit(&bars->done);
    __syncwarp();
    volatile int never = 0;
    mbar_wait(&bars->done, 0, &never);
    __syncwarp();
  } else {
    // ------------------------------------------------- generators + epilogue
    // TMEM lane quarter = warp % 4 (the sub-partition's lanes); the
    // generator warps of each quarter take the column parts h.
    const int q = warp & 3, h = (warp - kGenWarp0) >> 2;
    const int row = q * 32 + lane;
    const uint32_t laneOff = (uint32_t)(q * 32) << 16;
    uint32_t s = 0, ph = 0, accPh = 0;
    // Per slot, the parity of the kfull phase the next wavevector chunk
    // completes.  Only table stages arrive on kfull, so in a grouped launch
    // whose tiles mix both generators this parity and the ring's differ.
    uint32_t kph = 0;
    bool ok = true;
    TileView v;
    for (int64_t i = 0; i < count && ok; ++i) {
      w.get(i, v);
      const Plan& P = *v.P;
      const bool grid = kHasGrid && (GEN == GEN_GRID3 || P.gen == GEN_GRID3);
      const int64_t nChunks = P.nChunks;
      const int64_t p = v.row0 + v.tile * kTileM + row;
      const bool valid = (p < v.row0 + v.rows);
      double x[3] = {0.0, 0.0, 0.0};
      if (valid && RF_IN_BOUNDS(p * P.nDim + P.nDim - 1, P.n * P.nDim, err)) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (d < P.nDim) x[d] = v.x[p * P.nDim + d] / P.corrL[d];
      }

      const bool fastPhase = table_fast_phase(x, P.kMax);
      const bool f32Phase = table_f32_phase(x, P.kMax);
      const float xf[3] = {(float)x[0], (float)x[1], (float)x[2]};
      const FxpPoint fxp = fxp_point(x, P.kMax);
      Grid3Thread g3;
      Grid3Walk walk;
      if (kHasGrid && grid) {
        grid3_thread_setup<LPAD>(g3, P, h, x);
        walk.init(P, x);
      }

      // A full barrier wait costs a warp a couple of hundred cycles even when
      // the phase is already complete, so lane 0 probes the next stage's
      // slot at the start of the current stage and the answer is read after
      // the stage's work; the wait proper runs only when the probe failed.
      bool freeSeen = false;
      for (int64_t ch = 0; ch < nChunks; ++ch) {
        const uint32_t sc = s, phc = ph;
        if (++s == (uint32_t)S) { s = 0; ph ^= 1; }
        bool wt = freeSeen || mbar_wait_warp(&bars->empty[sc], phc ^ 1, abort_flag);
        if (kHasTable && !grid) {
          wt = wt && mbar_wait_warp(&bars->kfull[sc], (kph >> sc) & 1u, abort_flag, true);
          kph ^= 1u << sc;
        }
        if (!wt) { ok = false; break; }
        tc_fence_after();
        uint32_t probe = 0;
        if (lane == 0 && ch + 1 < nChunks) probe = mbar_test_wait(&bars->empty[s], ph ^ 1) ? 1u : 0u;
        const uint32_t aAddr = tbase + laneOff + (uint32_t)L.aCol0 + sc * (uint32_t)L.aStride;
        if (kHasGrid && grid) {
          // Two groups per stage; a thread takes its half (h) of both.
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const float2 Pq = walk.outer();
            walk.next(P, x);
            // one TMEM column per (cos, sin) pair, or per two pairs for e4m3
            constexpr int NW = kF8 ? (LPAD > 0 ? LPAD / 2 : 1) : (LPAD > 0 ? LPAD : 1);
            uint32_t words[NW];
            float pc0 = 0.f, ps0 = 0.f;  // e4m3: the even pair waits for the odd one
            auto emit = [&](int idx, float c, float sn) {
              if (kF8) {
                if ((idx & 1) == 0) {
                  pc0 = c;
                  ps0 = sn;
                } else {
                  words[idx >> 1] = pack_e4m3x4(pc0, ps0, c, sn);
                }
              } else {
                words[idx] = (PREC == PREC_FP16) ? pack_f16x2(c, sn) : pack_bf16x2(c, sn);
              }
            };
            grid3_pairs<LPAD>(g3, Pq, emit);
            // LPAD is a multiple of 8: 16-bit stores cover 8 columns at
            // 8-aligned offsets, e4m3 stores 4 columns at 4-aligned offsets.
            const uint32_t col = aAddr + (uint32_t)(u * 2 * NW + h * NW);
            if (kF8) {
#pragma unroll
              for (int pc = 0; pc < NW / 4; ++pc) tmem_st4(col + pc * 4, &words[pc * 4]);
            } else {
#pragma unroll
              for (int pc = 0; pc < NW / 8; ++pc) tmem_st8(col + pc * 8, &words[pc * 8]);
            }
          }
        } else if (kHasTable) {
          constexpr int T = kTableChunk / kParts;  // pairs of this thread
          constexpr int NW = kF8 ? T / 2 : T;
          uint32_t words[NW];
          uint32_t lows[(TALO && PREC == PREC_BF16) ? NW : 1];  // the BF16 residuals (tableALo)
          const bool aLo = TALO && PREC == PREC_BF16 && P.tableALo;
          float pc0 = 0.f, ps0 = 0.f;
          auto emit = [&](int idx, float c, float sn) {
            if (kF8) {
              if ((idx & 1) == 0) {
                pc0 = c;
                ps0 = sn;
              } else {
                words[idx >> 1] = pack_e4m3x4(pc0, ps0, c, sn);
              }
            } else {
              words[idx] = (PREC == PREC_FP16) ? pack_f16x2(c, sn) : pack_bf16x2(c, sn);
              if (PREC == PREC_BF16 && aLo) {
                const uint32_t w = words[idx];
                lows[idx] = pack_bf16x2(c - __uint_as_float(w << 16), sn - __uint_as_float(w & 0xffff0000u));
              }
            }
          };
          const double* kt = sK + sc * kKtabStageDoubles;
          if (f32Phase) table_pairs_f32<T>(kt, h, xf, emit);
          else if (fxp.ok) table_pairs_fxp<T>(kt, h, fxp, emit);
          else if (fastPhase) table_pairs<true, T>(kt, h, x, emit);
          else table_pairs<false, T>(kt, h, x, emit);
          const uint32_t col = aAddr + (uint32_t)(h * NW);
#pragma unroll
          for (int pc = 0; pc < NW / 8; ++pc) tmem_st8(col + pc * 8, &words[pc * 8]);
          if (PREC == PREC_BF16 && aLo) {
#pragma unroll
            for (int pc = 0; pc < NW / 8; ++pc) tmem_st8(col + (uint32_t)P.chunkK + pc * 8, &lows[pc * 8]);
          }
        }
        freeSeen = __shfl_sync(0xffffffffu, probe, 0) != 0;
        tmem_st_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars->full[sc]);
      }
      if (!ok) break;

      // ---------------------------------------------------------- epilogue
      if (!mbar_wait_warp(&bars->acc_full, accPh, abort_flag)) { ok = false; break; }
      tc_fence_after();
      double bw = 0.0;  // localization blend: weight and group index of this point
      int64_t bg = 0;
      if (P.blend && valid) bw = blend_weight(P, p, &bg);
      for (int cb = h * 8; cb < P.nmcPad; cb += 8 * kParts) {  // 8-column blocks, round robin over the parts
        uint32_t va[8], lo[8];
        tmem_ld8(tbase + laneOff + cb, va);
        if (kHiLo) tmem_ld8(tbase + laneOff + P.nmcPad + cb, lo);
        tmem_ld_wait();
        if (valid) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int r = cb + j;
            float acc = __uint_as_float(va[j]);
            if (kHiLo) acc += __uint_as_float(lo[j]);
            if (r >= P.nmcBlk) continue;
            if (P.blend) {
              if (RF_IN_BOUNDS((int64_t)(P.rOff + r) * P.gTotal + bg, (int64_t)P.Nmc * P.gTotal, err))
                atomicAdd(&v.out[(int64_t)(P.rOff + r) * P.gTotal + bg], bw * ((double)acc * P.outScale));
            } else if (RF_IN_BOUNDS((int64_t)(P.rOff + r) * P.n + p, (int64_t)P.Nmc * P.n, err)) {
              v.out[(int64_t)(P.rOff + r) * P.n + p] = finish_value(P, acc);
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->acc_empty);
      accPh ^= 1;
    }
    if (!ok) raise_abort(bars, err);
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tbase, kTmemCols);
}

// LPAD: GEN_GRID3 axis-3 length padded to 8/16/24/32 (0 for GEN_TABLE).
template <int GEN, int PREC, int LPAD, bool TALO>
__global__ void __launch_bounds__(Roles<GEN>::kThreads, 1) rf_tc_kernel(const __grid_constant__ TcArgs a) {
  const SingleWork w{&a, (a.rows + kTileM - 1) / kTileM};
  tc_body<GEN, PREC, LPAD, TALO>(w, a.L, a.err);
}

template <int PREC>
__global__ void __launch_bounds__(Roles<GEN_MIXED>::kThreads, 1) rf_group_kernel(const __grid_constant__ GroupArgs g) {
  const GroupWork w{&g, g.ctaStart[blockIdx.x], g.ctaStart[blockIdx.x + 1]};
  tc_body<GEN_MIXED, PREC, kGroupLPad, true>(w, g.L, g.err);
}

template <int GEN, int PREC, int LPAD, bool TALO = false>
cudaError_t launch_one(const TcArgs& args, size_t smem, int grid, cudaStream_t st) {
  auto fn = rf_tc_kernel<GEN, PREC, LPAD, TALO>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, Roles<GEN>::kThreads, smem, st>>>(args);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_prec(const Plan& P, const TcArgs& args, size_t smem, int grid, cudaStream_t st) {
  if (P.gen != GEN_GRID3) {
    if constexpr (PREC == PREC_BF16) {
      if (P.tableALo) return launch_one<GEN_TABLE, PREC, 0, true>(args, smem, grid, st);
    }
    return launch_one<GEN_TABLE, PREC, 0>(args, smem, grid, st);
  }
  switch (P.lPad) {
    case 8: return launch_one<GEN_GRID3, PREC, 8>(args, smem, grid, st);
    case 16: return launch_one<GEN_GRID3, PREC, 16>(args, smem, grid, st);
    case 24: return launch_one<GEN_GRID3, PREC, 24>(args, smem, grid, st);
    case 32: return launch_one<GEN_GRID3, PREC, 32>(args, smem, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int PREC>
cudaError_t launch_group_prec(const GroupArgs& g, size_t smem, int grid, cudaStream_t st) {
  rf_group_kernel<PREC><<<grid, Roles<GEN_MIXED>::kThreads, smem, st>>>(g);
  return cudaGetLastError();
}

// Shared-memory bytes of a layout (with the wavevector slots when `table`).
size_t layout_bytes(const SlotLayout& L, bool table) {
  return (size_t)kHeaderBytes + (size_t)L.S * (size_t)L.slotBytes + (table ? (size_t)L.S * kKtabStageBytes : 0);
}

// Deepest pipeline (2..maxS stages) that fits TMEM and shared memory; S = 0
// when none does.  The kernel allocates all 512 TMEM columns, so two CTAs
// must never share an SM: asking for more than half of the SM's shared
// memory guarantees it.
size_t fit_layout(SlotLayout& L, bool table, int maxS = kMaxStages) {
  const size_t limit = 227 * 1024, floor = 120 * 1024;
  int tmemS = (int)((kTmemCols - (uint32_t)L.aCol0) / (uint32_t)L.aStride);
  if (maxS > tmemS) maxS = tmemS;
  if (maxS > kMaxStages) maxS = kMaxStages;
  for (int s = maxS; s >= 2; --s) {
    L.S = s;
    L.ktabOff = (int32_t)((size_t)s * (size_t)L.slotBytes);
    const size_t total = layout_bytes(L, table);
    if (total <= limit) return total < floor ? floor : total;
  }
  L.S = 0;
  return 0;
}

}  // namespace

size_t tc_smem_bytes(const Plan& P, int* stages) {
  if (P.gen == GEN_OUTER) return outer_smem_bytes(P, stages);
  SlotLayout L;
  L.aCol0 = P.bRows;
  L.aStride = a_cols(P);
  L.slotBytes = P.stageBytes;
  const size_t smem = fit_layout(L, P.gen == GEN_TABLE);
  if (stages) *stages = L.S;
  return smem;
}

cudaError_t launch_tc(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                      int64_t row0, int64_t rows, uint32_t* dErr, int numSMs, cudaStream_t st) {
  if (P.gen == GEN_OUTER) return launch_outer(P, dX, dB, dOut, row0, rows, dErr, numSMs, st);
  TcArgs args;
  args.P = P;
  args.x = dX;
  args.B = reinterpret_cast<const unsigned char*>(dB);
  args.ktab = dKtab;
  args.out = dOut;
  args.err = dErr;
  args.row0 = row0;
  args.rows = rows;
  args.L.aCol0 = P.bRows;
  args.L.aStride = a_cols(P);
  args.L.slotBytes = P.stageBytes;
  const size_t smem = fit_layout(args.L, P.gen == GEN_TABLE);
  if (smem == 0) return cudaErrorInvalidValue;
  const int64_t tiles = (rows + kTileM - 1) / kTileM;
  const int grid = (int)(tiles < numSMs ? tiles : numSMs);
  if (P.prec == PREC_FP16) return launch_prec<PREC_FP16>(P, args, smem, grid, st);
  if (P.prec == PREC_BF16_FAST) return launch_prec<PREC_BF16_FAST>(P, args, smem, grid, st);
  if (P.prec == PREC_FP8) return launch_prec<PREC_FP8>(P, args, smem, grid, st);
  return launch_prec<PREC_BF16>(P, args, smem, grid, st);
}

size_t group_layout(int32_t maxBRows, int64_t maxStageBytes, int32_t maxStages, SlotLayout* L) {
  L->aCol0 = maxBRows;
  L->aStride = 2 * (2 * kGroupLPad);  // a GEN_GRID3 stage (two groups); GEN_TABLE stages use 32 of its columns
  L->slotBytes = maxStageBytes;
  return fit_layout(*L, true, maxStages > 0 ? maxStages : kMaxStages);
}

cudaError_t group_set_smem(int prec, size_t smem) {
  const int b = (int)smem;
  if (prec == PREC_FP16) return cudaFuncSetAttribute(rf_group_kernel<PREC_FP16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (prec == PREC_BF16_FAST)
    return cudaFuncSetAttribute(rf_group_kernel<PREC_BF16_FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (prec == PREC_BF16) return cudaFuncSetAttribute(rf_group_kernel<PREC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (prec == PREC_FP8) return cudaFuncSetAttribute(rf_group_kernel<PREC_FP8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  return cudaErrorInvalidValue;
}

cudaError_t launch_group(int prec, const GroupArgs& g, size_t smem, int grid, cudaStream_t st) {
  if (prec == PREC_FP16) return launch_group_prec<PREC_FP16>(g, smem, grid, st);
  if (prec == PREC_BF16_FAST) return launch_group_prec<PREC_BF16_FAST>(g, smem, grid, st);
  if (prec == PREC_BF16) return launch_group_prec<PREC_BF16>(g, smem, grid, st);
  if (prec == PREC_FP8) return launch_group_prec<PREC_FP8>(g, smem, grid, st);
  return cudaErrorInvalidValue;
}

}  // namespace rfb
