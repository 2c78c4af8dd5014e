// rf_plan.h -- host/device description of one generation request as the
// kernels consume it.  Plain C++ (no CUDA types) so the host code and every
// .cu file share it.
#pragma once
#include <stdint.h>

namespace rfb {

// constants_RF.f90:5 -- the reference's PI, used wherever PI enters a formula
// (kDelta, S(k), ampMult, phase = 2*PI*U).  Range reduction of a phase uses the
// true 2*pi instead, because cos is periodic in the true 2*pi.
constexpr double kRefPi = 3.1415926535898;

// rnglib.f90:548-659 moduli and multipliers of the combined MLCG.
constexpr int64_t kM1 = 2147483563, kM2 = 2147483399;
constexpr int64_t kA1 = 40014, kA2 = 40692;
constexpr double kR8Scale = 4.656613057E-10;  // rnglib.f90:1517

enum Generator : int32_t {
  GEN_TABLE = 0,  // explicit wavevector table, one FP64 phase + SFU sincos per (point, k)
  GEN_GRID3 = 1,  // 3-D tensor-grid wavevectors: per-axis tables and angle addition
  GEN_MIXED = 2,  // kernel variant only: the generator is chosen per tile (grouped launch)
  GEN_OUTER = 3,  // 3-D tensor grid, outer-group contraction (rf_outer.cu): A = outer phasors
                  // E1 E2^{s2}, N = (realization, i3, cos|sin), the i3 sum in the epilogue
};

enum Precision : int32_t { PREC_BF16 = 0, PREC_FP16 = 1, PREC_FP32 = 2, PREC_BF16_FAST = 3, PREC_FP8 = 4 };

// Forms whose amplitude side is split into hi and lo rows (N = 2 * nmcPad).
inline bool prec_hilo(int32_t prec) { return prec == PREC_BF16 || prec == PREC_FP8; }

constexpr int kTileM = 128;        // points per tile (MMA M)
constexpr int kStageCols = 64;     // max k-values (TMEM columns) per GEN_GRID3 group or FP32 stage
constexpr int kMaxStageCols = 128; // max k-values per tcgen05 stage (two groups)
constexpr int kTableChunk = 64;    // k-values per stage for GEN_TABLE
// The GEN_TABLE wavevector chunk of one stage: three [3][kTableChunk] arrays,
// k / 2 pi in FP64, round(k / 2 pi * 2^30) in int32 and k in FP32.
constexpr int kKtabStageDoubles = 6 * kTableChunk;
constexpr int kKtabStageBytes = 8 * kKtabStageDoubles;
constexpr int kMaxGridN = 32;      // GEN_GRID3: max wavenumbers per axis
constexpr int kMaxNmcPad = 256;    // realizations per launch (MMA N <= 256)
constexpr int kLoMaskWords = 32;   // stages of a plan that can drop the lo rows: up to 1024

struct Plan {
  // request
  int32_t nDim, Nmc, method, corrMod, margiFirst, literal, normalize, prec;
  int64_t n;
  double corrL[3];
  double fieldAvg, fieldVar;
  // geometry (spectra_RF.f90 / randomFieldND.f90)
  int64_t K;                  // wavevectors in the reference's count
  int32_t kNStep[3];          // Shinozuka per axis; isotropic [0]=n_r, [1]=n_dir
  double kDelta[3];           // Shinozuka per axis; isotropic [0]=dr
  double kMax, ampMult;
  int32_t ig1, ig2;           // rnglib generator-1 seed words
  // realization block of this launch: columns [rOff, rOff + nmcBlk) of Nmc
  int32_t rOff, nmcBlk;
  // kernel layout
  int32_t gen;                // Generator
  int32_t nmcPad;             // nmcBlk padded (16 for tcgen05, 8 * 2^j for FP32)
  int32_t bRows;              // rows of B per stage (nmcPad, or 2*nmcPad with hi/lo)
  int32_t chunkK;             // k-values per stage
  int32_t lPad;               // GEN_GRID3: inner (axis 3) length padded to a multiple of 8
  int32_t gps;                // GEN_GRID3: outer groups (i1, i2, s2) per stage
  int32_t forceTable;         // 1: GEN_TABLE even where GEN_GRID3 applies
  // BF16 hi/lo, single GEN_GRID3 requests: with loSkip, B stage s carries
  // the lo rows only where bit s of loMask is set (stage_has_lo); the other
  // stages hold the hi rows alone (half the bytes, MMA N = nmcPad)
  int32_t loSkip;
  uint32_t loMask[kLoMaskWords];
  int64_t nChunks;            // stages per tile
  int64_t stageBytes;         // bytes of one B stage
  int32_t bScaleLog2;         // FP16: B stored times 2^bScaleLog2
  double outScale;            // epilogue factor: ampMult * 2^-bScaleLog2
  // marginal map (randomFieldND.f90:139-178), applied in the epilogue
  int32_t applyMarginal;      // 0 when a normalisation pass follows
  int32_t lognormal;
  double margSd, margAvg;
  // localization blend (localization_RF.f90:199-263, 705-857): the request
  // is subdomain of a structured group grid; its points are the subdomain's
  // grid points (axis 1 fastest) and the epilogue adds the partition-of-unity
  // weight times the Gaussian field into the group field at bOrigin
  int32_t blend;
  int32_t bDims[3];           // subdomain grid points per axis
  int32_t bOrigin[3];         // subdomain origin in group grid indices
  int32_t gDims[3];           // group grid points per axis
  int32_t bRamp[3];           // overlapNPoints per axis (< 1: no ramp)
  int64_t gTotal;             // group grid points
  // GEN_OUTER layout (rf_outer.cu; single 3-D Shinozuka requests on the
  // tensor-core forms).  K = 2 x outer groups g = (i1, i2, s2) (re, im of
  // E1 E2^{s2}), in K-steps of 16 = 8 groups of consecutive i1; N chunk c
  // = realizations [c oRc, (c+1) oRc) of the block, each 2 lPad columns
  // (i3, cos|sin).  B of chunk c is oNK K-step blocks of oKstepBytes, each
  // followed by a second block where bit j of loMask is set; A takes two
  // units on the K-steps of aLoMask.  The BF16 form sets both masks on its
  // TF32 K-steps (oTf32): the two blocks and units hold K 0-7 and K 8-15 in
  // 32-bit containers.
  int32_t n1p;                // axis-1 wavenumbers padded to a multiple of 8 (8, 16, 24)
  int32_t oRc;                // realizations per N chunk
  int32_t oNR;                // N chunks of the realization block
  int32_t oNK;                // K-steps per chunk
  int64_t oKstepBytes;        // bytes of one K-step block of B: 16 x (2 lPad oRc) x 2
  int64_t oChunkBytes;        // bytes of one chunk of B, lo blocks included
  uint32_t aLoMask[8];        // K-steps whose A tile carries the lo term (up to 256)
  uint32_t oStageEnd[8];      // K-steps that close a ring stage (outer_stage_layout)
  // CTA-pair form (rf_outer_pair.cu; single requests, and every
  // outer-group unit of a batch): N chunk c is two
  // halves of oRc realizations each, [c 2 oRc + h oRc, + oRc); a CTA pair
  // computes a 256-point item (one tile per CTA), each CTA holding its half
  // (lPad oRc rows) of both halves' B rows.  B of chunk c is rank 0's part
  // then rank 1's, each its oNK K-step blocks of oKstepBytes (half 0's rows,
  // then half 1's), each followed by its lo block where loMask says.
  int32_t oPair;
  // BF16: the K-steps of aLoMask (= loMask) carry A and B as TF32
  // (kind::tf32, two MMAs of K = 8 over the K-step's two units and blocks)
  int32_t oTf32;
  int64_t oStepM1, oStepM2;   // rnglib multipliers a^(n1 n2 n3) mod m: the s3 = - draw from the s3 = + one
  // GEN_TABLE, BF16 single requests: the trig tile also carries its lo term
  // (the stage's A columns twice, one more MMA per K-step)
  int32_t tableALo;
  // caller-supplied uniform draws (device copy of rf_options.draws): draw p
  // (1-based) of the request is dDraws[p - 1]; null: the rnglib stream
  const double* dDraws;
  int64_t nDraws;
  // error word of the launch's context: the RF_DEBUG_BOUNDS build records
  // failed index checks in it (the normal build never reads it)
  uint32_t* dbgErr;
};

// Draws a request consumes, in the reference's order of random_number calls:
// Shinozuka Nmc K phases; randomization nDim kn base-wavevector draws first;
// isotropic the direction blocks (two in 3-D, one in 2-D), then per
// realization a gamma and a psi block.
__host__ __device__ inline int64_t draws_needed(const Plan& P) {
  if (P.method == 1) return (int64_t)(P.nDim == 3 ? 2 : 1) * P.K + (int64_t)P.Nmc * 2 * P.K;
  const int64_t skip = (P.method == 3) ? (P.K >> (P.nDim - 1)) * P.nDim : 0;
  return skip + (int64_t)P.Nmc * P.K;
}

__host__ __device__ inline int popcount32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}
// Whether B stage s of the plan carries the lo rows.
__host__ __device__ inline bool stage_has_lo(const Plan& P, int64_t s) {
  return !P.loSkip || ((P.loMask[s >> 5] >> (s & 31)) & 1u);
}
// Byte offset of B stage s: hi-only stages take half of stageBytes.
__host__ __device__ inline int64_t stage_offset(const Plan& P, int64_t s) {
  if (!P.loSkip) return s * P.stageBytes;
  int64_t lo = 0;
  for (int64_t w = 0; w < (s >> 5); ++w) lo += popcount32(P.loMask[w]);
  if (s & 31) lo += popcount32(P.loMask[s >> 5] & ((1u << (s & 31)) - 1u));
  return (s + lo) * (P.stageBytes / 2);
}

constexpr int kOuterMaxN1P = 24;  // GEN_OUTER: axis-1 wavenumbers (register table of the generators)
constexpr int kOuterMaxKsteps = 256;

__host__ __device__ inline bool mask_bit(const uint32_t* m, int64_t j) { return (m[j >> 5] >> (j & 31)) & 1u; }
// Set bits of m below bit j.
__host__ __device__ inline int64_t mask_rank(const uint32_t* m, int64_t j) {
  int64_t c = 0;
  for (int64_t w = 0; w < (j >> 5); ++w) c += popcount32(m[w]);
  if (j & 31) c += popcount32(m[j >> 5] & ((1u << (j & 31)) - 1u));
  return c;
}
// K-step j of a GEN_OUTER chunk holds the 8 outer groups (i1 = 8 jj ..
// 8 jj + 7, i2, s2) with j = i2 + n2 (s2 + 2 jj): the axis-1 block jj is the
// slowest index, so that a generator needs the 8 axis-1 phasors of one block
// at a time, and the K-steps that keep lo terms (small k1 and k2) come in
// runs.
__host__ __device__ inline int64_t outer_kstep(const Plan& P, int32_t jj, int32_t i2, int32_t s2) {
  return (int64_t)i2 + (int64_t)P.kNStep[1] * (s2 + 2 * (int64_t)jj);
}
__host__ __device__ inline void outer_kstep_groups(const Plan& P, int64_t j, int32_t* jj, int32_t* i2, int32_t* s2) {
  const int64_t n2 = P.kNStep[1];
  *i2 = (int32_t)(j % n2);
  *s2 = (int32_t)((j / n2) % 2);
  *jj = (int32_t)(j / (2 * n2));
}
// GEN_OUTER: byte offset of K-step j's hi block inside a chunk of B.
__host__ __device__ inline int64_t outer_kstep_offset(const Plan& P, int64_t j) {
  return (j + (P.loSkip ? mask_rank(P.loMask, j) : 0)) * P.oKstepBytes;
}
__host__ __device__ inline bool outer_b_lo(const Plan& P, int64_t j) { return P.loSkip && mask_bit(P.loMask, j); }
__host__ __device__ inline bool outer_a_lo(const Plan& P, int64_t j) { return mask_bit(P.aLoMask, j); }
// GEN_OUTER ring stages (rf_outer.cu): a stage holds kOuterStageUnits A
// units (one unit: both tiles' hi K-step; a K-step with an A lo term takes
// two) and as many B units (one K-step block of B; two with its lo block).
// The K-steps of a chunk fill stages in order, a stage closing before the
// K-step that would overflow either side: four K-steps without lo terms, or
// two with both, per stage.
constexpr int kOuterStageUnits = 4;
__host__ __device__ inline bool outer_stage_end(const Plan& P, int64_t j) { return mask_bit(P.oStageEnd, j); }

// Bytes of the contraction operand of a plan (one realization block).
__host__ __device__ inline int64_t operand_bytes(const Plan& P) {
  if (P.gen == GEN_OUTER) return (int64_t)P.oNR * P.oChunkBytes;
  return stage_offset(P, P.nChunks);
}

// Table builder threads (rf_tables.cu): one per (run, realization column).
// A run is n1 wavevectors of one GEN_GRID3 column (consecutive i1) or kRun
// consecutive wavevectors of the other generators.
constexpr int kRun = 32;
__host__ __device__ inline int64_t table_runs(const Plan& P) {
  if (P.gen == GEN_OUTER) return (int64_t)P.lPad * P.kNStep[1] * 2;  // (i3, i2, s2), a run over i1
  if (P.gen == GEN_GRID3) return (int64_t)(2 * P.lPad) * (P.nChunks * P.gps / P.kNStep[0]);
  return (P.nChunks * P.chunkK + kRun - 1) / kRun;
}
// Realization columns of the builder: GEN_OUTER lays out whole N chunks.
__host__ __device__ inline int32_t table_cols(const Plan& P) {
  return P.gen == GEN_OUTER ? P.oNR * P.oRc * (P.oPair ? 2 : 1) : P.nmcPad;
}
__host__ __device__ inline int64_t table_threads(const Plan& P) { return table_runs(P) * table_cols(P); }

// Shared-memory and TMEM slot layout of one tcgen05 launch: B slot s at
// byte slotBytes*s of the slot area, its wavevector chunk (GEN_TABLE) at
// ktabOff + s*768, its A tile at TMEM column aCol0 + s*aStride (the
// accumulator occupies the columns below aCol0).
struct SlotLayout {
  int32_t S;
  int32_t aCol0;
  int32_t aStride;
  int32_t ktabOff;
  int64_t slotBytes;
};

// One unit of a grouped launch: a request's realization block with its own
// plan, operands and output (device pointers).
struct GroupSub {
  Plan P;
  const double* x;      // n x nDim points
  double* out;          // Nmc x n field (realization-major)
  unsigned char* B;     // contraction operand, nChunks stages
  double* ktab;         // GEN_TABLE wavevector chunks
};

// Work item of a grouped launch: tile `tile` (128 points) of unit `sub`.
struct GroupItem {
  int32_t sub;
  int32_t tile;
};

// TMEM columns of one stage's A tile: one 32-bit column holds a (cos, sin)
// pair of 16-bit values, or two pairs of 8-bit values.
inline int32_t a_cols(const Plan& P) { return (P.prec == PREC_FP8 ? P.chunkK / 2 : P.chunkK) * (P.tableALo ? 2 : 1); }

}  // namespace rfb
