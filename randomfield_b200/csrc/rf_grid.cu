// rf_grid.cu -- the Shinozuka sum on a structured grid, by separable stages.
//
// The reference evaluates f(x, r) = ampMult * sum_k a_k cos(k.x + phi_{k,r})
// point by point (gen_Std_Gauss_Shinozuka, randomFieldND.f90:184-337) with
// k on the tensor grid k = (i1 d1, s2 i2 d2, s3 i3 d3) of set_kPoints
// (spectra_RF.f90:87-133; s2, s3 the sign rows of set_kSign, :267-286).
// When the points themselves form a tensor grid x = (x1(j1), x2(j2), x3(j3))
// (setGrid, math_RF.f90:16-92, as set_XPoints builds them, mesh_RF.f90:17-64)
// the phasor factorises, exp(i k.x) = E1(i1, j1) E2(s2 i2, j2) E3(s3 i3, j3)
// with E_d(i, j) = exp(i k_d(i) x_d(j)), and the sum runs axis by axis:
//   C(k)            = a_k exp(i phi_{k,r})                      (coefficients)
//   G(i1,i2,s2; j3) = sum_{i3,s3} C E3^{+-}  = sum_i3 P c3 + i Q s3   (axis 3)
//   H(i1; j2, j3)   = sum_{i2,s2} G E2^{+-}  = sum_i2 u c2 + i v s2   (axis 2)
//   f(j1, j2, j3)   = ampMult Re sum_i1 H E1 = sum_i1 Hr c1 - Hi s1   (axis 1)
// where the two signs of an axis share one cosine and one sine:
// P = C(s3=+) + C(s3=-), Q = C(s3=+) - C(s3=-), u = G(s2=+) + G(s2=-),
// v = G(s2=+) - G(s2=-).  Per realization that is
//   8 n1 n2 n3 N3 + 4 n1 n2 N2 N3 + 2 n1 N1 N2 N3
// FP64 multiply-adds (axis 3 for both sign rows of axis 2) instead of the reference's N1 N2 N3 x 4 n1 n2 n3 cosines
// (128^3 points, 24^3 x 4 wavevectors: 1.5e8 instead of 1.2e11), so the
// whole computation stays in FP64: the field equals the reference's sum to
// FP64 rounding, with no reduced-precision operand anywhere.
//
// Every stage is a small dense product on the FP64 tensor path (mma.sync
// m8n8k4 .f64, the only FP64 tensor-core instruction of sm_100a): operands
// staged in shared memory with rows padded against bank conflicts, k padded
// to a multiple of 4 with zero rows, FP64 accumulators in registers.
//   rf_sep_phasors  E_d(i, j) for the three axes (FP64 sincos);
//   rf_sep_coeffs   P, Q for every (r, s2, i2, i1, i3) from the rnglib stream;
//   rf_sep_axis3    tiles (r, 64 rows j3, 32 pairs (i1,i2)) -> u, v;
//   rf_sep_axes21   persistent: item (r, j3, 64 or 128 rows j2, 128 columns
//                   j1): H into shared memory, then f, the marginal map and
//                   the store of the item's field values.
// Axes the request does not have are carried as length-1 axes with k = 0 and
// one sign row, so 1-D and 2-D grids take the same kernels.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <chrono>

#include "rf_internal.h"

using namespace rfb;
using namespace rfh;

namespace {

constexpr int kSepThreads = 256;
constexpr int kAxesThreads = 512, kAxesWarps = kAxesThreads / 32;  // rf_sep_axes21
constexpr int kRows = 64;     // rows of a tile
constexpr int kMaxSepN = 32;  // wavenumbers per axis
constexpr size_t kSepScratch = (size_t)512 << 20;  // P/Q and u/v of one realization block

struct SepSpec {
  int32_t nDim;
  int32_t N[3];   // grid points per axis (1 where the request has no axis)
  int32_t kn[3];  // wavenumbers per axis (1 where absent)
  int32_t S2, S3; // sign rows of axes 2 and 3
  int32_t corrMod;
  int32_t ig1, ig2;
  int32_t r0, nr;  // realizations [r0, r0 + nr) of this block
  int32_t applyMarginal, lognormal;
  int64_t K, n;
  double kDelta[3];
  double xMin[3], xStep[3], corrL[3];
  double ampMult, margSd, margAvg;
};

// D += A B on the FP64 tensor path: one 8 x 8 x 4 product per warp
// (mma.sync m8n8k4 .f64).  Lane l = 4 g + t holds A[g][t], B[t][g] and
// D[g][2 t], D[g][2 t + 1].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Row padding (doubles) of the 8 x 4 fragment operands: a stride of 4 mod 16
// doubles puts the four k rows t of a half-warp's load (lanes 4 g + t, g < 4)
// on four different 32-byte bank groups.
constexpr int kPadLd = 4;

// E_d(i, j) = (cos, sin)(k_d(i) x_d(j)), k_d(i) = 0 + kDelta_d i (setGrid from
// 0, spectra_RF.f90:118), x_d(j) = (xMin_d + xStep_d j) / corrL_d
// (randomFieldND.f90:58-73).  Table d holds kn_d x N_d entries, i major.
__global__ void rf_sep_phasors(const SepSpec sp, double2* __restrict__ E) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t off = 0;
  for (int d = 0; d < 3; ++d) {
    const int64_t sz = (int64_t)sp.kn[d] * sp.N[d];
    if (t < off + sz) {
      const int64_t e = t - off;
      const int32_t i = (int32_t)(e / sp.N[d]), j = (int32_t)(e % sp.N[d]);
      double c = 1.0, s = 0.0;
      if (d < sp.nDim) {
        const double k = 0.0 + sp.kDelta[d] * (double)i;
        const double x = (sp.xMin[d] + sp.xStep[d] * (double)j) / sp.corrL[d];
        sincos(k * x, &s, &c);
      }
      E[t] = make_double2(c, s);
      return;
    }
    off += sz;
  }
}

// (Pr, Pi, Qr, Qi) of (rl, s2, i2, i1, i3), stored i3 fastest: C = a_k
// exp(i phi) with phi_{k,r} = 2 pi U(r K + k + 1) (K draws per realization in
// the reference's k order, randomFieldND.f90:278-279), the reference index
// k = q kn + i1 + n1 (i2 + n2 i3) of sign row q = s2 S3 + s3, a_k from S(k)
// (spectra_RF.f90:202-220).  One thread per (rl, s2, i2, i3) walks i1: the
// draws of a run of i1 are consecutive calls of the generator, so each of the
// two sign rows jumps ahead once and then steps.  Sign rows an axis does not
// have are zero.
__global__ void rf_sep_coeffs(const SepSpec sp, const JumpTable jt, double4* __restrict__ PQ) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t n1 = sp.kn[0], n2 = sp.kn[1], n3 = sp.kn[2];
  const int64_t total = (int64_t)sp.nr * 2 * n2 * n3;
  if (t >= total) return;
  const int32_t i3 = (int32_t)(t % n3);
  const int32_t i2 = (int32_t)((t / n3) % n2);
  const int32_t s2 = (int32_t)((t / ((int64_t)n3 * n2)) % 2);
  const int64_t rl = t / ((int64_t)n3 * n2 * 2);
  const int64_t rg = sp.r0 + rl;
  const int64_t kn = (int64_t)n1 * n2 * n3;
  double4* o = PQ + ((rl * 2 + s2) * n2 + i2) * (int64_t)n1 * n3 + i3;
  if (s2 >= sp.S2) {
    for (int32_t i1 = 0; i1 < n1; ++i1) o[(int64_t)i1 * n3] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  int64_t c1[2] = {0, 0}, c2[2] = {0, 0};
  // S(k) = prod_d exp(-k_d^2 / (4 pi)) multiplied from axis 1 up, as
  // spectra_RF.f90:202-208 does (corrL = 1); the sign of k_d does not enter
  auto factor = [&](int d, int32_t i) {
    const double k = 0.0 + sp.kDelta[d] * (double)i;
    return exp(-((k * k) * 1.0) / (4.0 * kRefPi));
  };
  const double f2 = sp.nDim >= 2 ? factor(1, i2) : 1.0, f3 = sp.nDim >= 3 ? factor(2, i3) : 1.0;
  for (int s3 = 0; s3 < sp.S3; ++s3) {
    const int64_t k0 = (int64_t)(s2 * sp.S3 + s3) * kn + (int64_t)n1 * (i2 + (int64_t)n2 * i3);
    uni_state_at(jt, sp.ig1, sp.ig2, (uint64_t)(rg * sp.K + k0 + 1), c1[s3], c2[s3]);
  }
  for (int32_t i1 = 0; i1 < n1; ++i1) {
    const double f1 = sp.corrMod == RF_CM_GAUSSIAN ? factor(0, i1) : 1.0;
    double cr[2] = {0.0, 0.0}, ci[2] = {0.0, 0.0};
    for (int s3 = 0; s3 < sp.S3; ++s3) {
      if (i1) uni_state_next(jt, c1[s3], c2[s3]);
      const int64_t kref = (int64_t)(s2 * sp.S3 + s3) * kn + i1 + (int64_t)n1 * (i2 + (int64_t)n2 * i3);
      double amp;
      if (sp.corrMod == RF_CM_GAUSSIAN) {
        double S = 1.0 * f1;
        if (sp.nDim >= 2) S = S * 1.0 * f2;
        if (sp.nDim >= 3) S = S * 1.0 * f3;
        amp = sqrt(S);
      } else {
        amp = (kref == 5) ? 1.0 : 0.0;  // cm_COS, spectra_RF.f90:210-220
      }
      const double phi = 2.0 * kRefPi * ((double)uni_value(c1[s3], c2[s3]) * kR8Scale);
      double sn, cs;
      sincos(phi, &sn, &cs);
      cr[s3] = amp * cs;
      ci[s3] = amp * sn;
    }
    o[(int64_t)i1 * n3] = make_double4(cr[0] + cr[1], ci[0] + ci[1], cr[0] - cr[1], ci[0] - ci[1]);
  }
}

// Axis 3.  Tile (rl, row block of 64 j3, block of 32 pairs m = i2 n1 + i1),
// an m8n8k4 FP64 tensor product G (64 x 128) = E3 (64 x 2 n3) B (2 n3 x 128)
// with k padded to a multiple of 4 by zero rows.  Column 8 q + c of B
// (c < 8) belongs to pair 2 q + (c >> 2), component (c >> 1) & 1 (real,
// imaginary) and sign row s2 = c & 1, from the k-rows 2 i3 (cos) and
// 2 i3 + 1 (sin):
//   Gr = sum Pr c3 - Qi s3,  Gi = sum Pi c3 + Qr s3,
// so that the lane holding D[g][2 t], D[g][2 t + 1] has both sign rows of
// one component and folds them into u = G+ + G-, v = G+ - G-.  The slab
// UV[rl][j3][m] is stored as (ur, vr, ui, vi).  Warps: 2 x 4 tiles of
// 32 rows x 32 columns.
__global__ void __launch_bounds__(kSepThreads) rf_sep_axis3(const SepSpec sp, const double2* __restrict__ E3,
                                                            const double4* __restrict__ PQ, double* __restrict__ UV) {
  constexpr int LDA = kRows + kPadLd, LDB = 128 + kPadLd;
  extern __shared__ __align__(16) double sm[];
  const int32_t n1 = sp.kn[0], n2 = sp.kn[1], n3 = sp.kn[2], N3 = sp.N[2];
  const int K = (2 * n3 + 3) & ~3;
  double* AT = sm;           // [K][LDA]
  double* B = sm + K * LDA;  // [K][LDB]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3, wr = warp & 1, wc = warp >> 1;
  const int64_t pairs = (int64_t)n1 * n2;
  const int64_t rowBlocks = (N3 + kRows - 1) / kRows, pairBlocks = (pairs + 31) / 32;
  const int64_t tiles = (int64_t)sp.nr * rowBlocks * pairBlocks;
  for (int e = threadIdx.x; e < (K - 2 * n3) * LDA; e += kSepThreads) AT[2 * n3 * LDA + e] = 0.0;
  for (int e = threadIdx.x; e < (K - 2 * n3) * LDB; e += kSepThreads) B[2 * n3 * LDB + e] = 0.0;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t pb = tile % pairBlocks;
    const int64_t rb = (tile / pairBlocks) % rowBlocks;
    const int64_t rl = tile / (pairBlocks * rowBlocks);
    __syncthreads();  // the previous tile's operands are consumed
    for (int e = threadIdx.x; e < n3 * kRows; e += kSepThreads) {
      const int i3 = e / kRows, row = e % kRows;
      const int64_t j3 = rb * kRows + row;
      const double2 v = j3 < N3 ? E3[(int64_t)i3 * N3 + j3] : make_double2(0.0, 0.0);
      AT[(2 * i3) * LDA + row] = v.x;
      AT[(2 * i3 + 1) * LDA + row] = v.y;
    }
    for (int e = threadIdx.x; e < 2 * n3 * 32; e += kSepThreads) {
      const int ml = e % 32, i3 = (e / 32) % n3, s2 = e / (32 * n3);
      const int64_t m = pb * 32 + ml;
      double4 pq = make_double4(0.0, 0.0, 0.0, 0.0);
      if (m < pairs) {
        const int64_t i2 = m / n1, i1 = m % n1;
        pq = PQ[(((rl * 2 + s2) * n2 + i2) * n1 + i1) * n3 + i3];
      }
      const int cr = 8 * (ml >> 1) + 4 * (ml & 1) + s2, ci = cr + 2;
      B[(2 * i3) * LDB + cr] = pq.x;       // Pr   -> Gr
      B[(2 * i3) * LDB + ci] = pq.y;       // Pi   -> Gi
      B[(2 * i3 + 1) * LDB + cr] = -pq.w;  // -Qi  -> Gr
      B[(2 * i3 + 1) * LDB + ci] = pq.z;   // Qr   -> Gi
    }
    __syncthreads();
    double acc[4][4][2];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[m][q][0] = acc[m][q][1] = 0.0;
#pragma unroll 2
    for (int k0 = 0; k0 < K; k0 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) a[m] = AT[(k0 + t) * LDA + 32 * wr + 8 * m + g];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = B[(k0 + t) * LDB + 32 * wc + 8 * q + g];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma(acc[m][q], a[m], b[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t mg = pb * 32 + 2 * (4 * wc + q) + (t >> 1);
      if (mg >= pairs) continue;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int64_t j3 = rb * kRows + 32 * wr + 8 * m + g;
        if (j3 < N3)
          *reinterpret_cast<double2*>(UV + ((rl * N3 + j3) * pairs + mg) * 4 + 2 * (t & 1)) =
              make_double2(acc[m][q][0] + acc[m][q][1], acc[m][q][0] - acc[m][q][1]);
      }
    }
  }
}

// 16-byte asynchronous copy global -> shared (sm_80 cp.async, L2 only), and
// the group fences around it.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Row stride (doubles) of a u, v slab in shared memory: 4 n1 rounded up to
// 8 mod 16, so that the two i2 rows one W fragment load touches sit 64 bytes
// apart in the banks.
__host__ __device__ inline int32_t uv_row_stride(int32_t n1) { return 4 * n1 + ((8 - 4 * n1) % 16 + 16) % 16; }

// Axes 2 and 1, persistent over items (column block, row block, rl, j3),
// the blocks outermost so that a CTA's consecutive items share E2T and E1.
// An item covers ROWS rows j2 (64 or 128) and 128 columns j1; both products
// run as m8n8k4 FP64 tensor products with the k dimension padded to a
// multiple of 4 by zero rows.  The u, v slab of item i + 1 streams into the
// other half of a double buffer (cp.async) while item i computes.
//   axis 2: H (ROWS x 2 n1) = E2 (ROWS x 2 n2) W (2 n2 x 2 n1), W read from
//           the slab: W[2 i2][2 i1 + {0,1}] = (ur, ui), W[2 i2 + 1][...] =
//           (-vi, vr); warp w takes ROWS/64 row tiles and every column tile;
//   axis 1: f (ROWS x 128) = H (ROWS x 2 n1) E1 (2 n1 x 128), E1 rows
//           ampMult (c1, -s1); warps in ROWS/32 x (256/ROWS) tiles of
//           32 x (ROWS/2) ... then the marginal map and the store.
template <int ROWS>
__global__ void __launch_bounds__(kAxesThreads, 1) rf_sep_axes21(const SepSpec sp, const double2* __restrict__ E1g,
                                                                const double2* __restrict__ E2g,
                                                                const double4* __restrict__ UV,
                                                                double* __restrict__ out) {
  constexpr int LD = ROWS + kPadLd;       // E2T, HT row stride
  constexpr int LDE = 128 + kPadLd;       // E1 row stride
  constexpr int WR = ROWS / 32;           // axis-1 warp rows (32 field rows each)
  constexpr int WC = kAxesWarps / WR;     // axis-1 warp columns
  constexpr int NTC = 128 / WC / 8;       // axis-1 column tiles per warp
  constexpr int MT = ROWS / 8;            // axis-2 row tiles, one per warp ...
  constexpr int WPM = kAxesWarps / MT;    // ... shared by WPM warps, which split the column tiles
  constexpr int NJ = 8 / WPM;             // axis-2 column tiles per warp (at most 8 in all)
  extern __shared__ __align__(16) double sm[];
  const int32_t n1 = sp.kn[0], n2 = sp.kn[1], N1 = sp.N[0], N2 = sp.N[1], N3 = sp.N[2];
  const int K1 = (2 * n1 + 3) & ~3, K2 = (2 * n2 + 3) & ~3;  // padded k extents
  const int NTB = (2 * n1 + 7) / 8;                          // axis-2 column tiles
  const int32_t pairs = n1 * n2;
  const int32_t uvLd = uv_row_stride(n1);                     // doubles per i2 row of a slab buffer
  double* E2T = sm;                                          // [K2][LD]: (c2, s2) rows of i2
  double* UVs = E2T + K2 * LD;                               // [2][n2][uvLd]: (ur, ui, vr, vi) per i1
  double* HT = UVs + 2 * n2 * uvLd;                          // [K1][LD]
  double* E1 = HT + K1 * LD;                                 // [K1][LDE]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int64_t rowBlocks = (N2 + ROWS - 1) / ROWS, colBlocks = (N1 + 127) / 128;
  const int64_t inner = (int64_t)sp.nr * N3;
  const int64_t items = colBlocks * rowBlocks * inner;
  const bool pairStore = (N1 % 2) == 0;  // 16-byte stores keep their alignment
  auto prefetch = [&](int64_t it, int buf) {
    if (it < items) {
      const int64_t rl = (it % inner) / N3, j3 = it % N3;
      const double2* src = reinterpret_cast<const double2*>(UV + (rl * N3 + j3) * pairs);
      double* dst = UVs + buf * n2 * uvLd;
      for (int e = threadIdx.x; e < 2 * pairs; e += kAxesThreads) {
        const int p = e >> 1, i2 = p / n1, i1 = p - i2 * n1;
        cp_async16(dst + i2 * uvLd + 4 * i1 + 2 * (e & 1), src + e);
      }
    }
    cp_async_commit();
  };
  // the padding rows of H (k >= 2 n1) are never written by the axis-2 stage
  for (int e = threadIdx.x; e < (K1 - 2 * n1) * LD; e += kAxesThreads) HT[2 * n1 * LD + e] = 0.0;
  // axis-2 operand from the slab: this lane's k row and column are fixed
  // modulo the tile steps, so are the component and sign it reads
  const int bc = t & 1, bre = g & 1;
  const int bcomp = bc ? (bre ? 1 : 3) : (bre ? 2 : 0);  // slab layout (ur, vr, ui, vi)
  const double bsign = (bc && !bre) ? -1.0 : 1.0;
  int64_t curBlock = -1;
  int buf = 0;
  prefetch(blockIdx.x, 0);
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x, buf ^= 1) {
    const int64_t blk = it / inner;
    const int64_t cb = blk / rowBlocks, rb = blk % rowBlocks;
    const int64_t rl = (it % inner) / N3, j3 = it % N3;
    __syncthreads();  // the previous item is done with HT (and E2T, E1, its slab buffer)
    prefetch(it + gridDim.x, buf ^ 1);
    if (blk != curBlock) {
      curBlock = blk;
      for (int e = threadIdx.x; e < K2 / 2 * ROWS; e += kAxesThreads) {
        const int i2 = e / ROWS, row = e % ROWS;
        const int64_t j2 = rb * ROWS + row;
        const double2 v = (i2 < n2 && j2 < N2) ? E2g[(int64_t)i2 * N2 + j2] : make_double2(0.0, 0.0);
        E2T[(2 * i2) * LD + row] = v.x;
        E2T[(2 * i2 + 1) * LD + row] = v.y;
      }
      for (int e = threadIdx.x; e < K1 / 2 * 128; e += kAxesThreads) {
        const int i1 = e / 128, col = e % 128;
        const int64_t j1 = cb * 128 + col;
        const double2 v = (i1 < n1 && j1 < N1) ? E1g[(int64_t)i1 * N1 + j1] : make_double2(0.0, 0.0);
        E1[(2 * i1) * LDE + col] = sp.ampMult * v.x;
        E1[(2 * i1 + 1) * LDE + col] = -(sp.ampMult * v.y);
      }
    }
    cp_async_wait_prev();  // this item's slab (the group before the one just issued)
    __syncthreads();
    {
      const double* uvd = UVs + buf * n2 * uvLd;
      double h[NJ][2];
#pragma unroll
      for (int j = 0; j < NJ; ++j) h[j][0] = h[j][1] = 0.0;
      const int r0 = 8 * (warp % MT), no = warp / MT;
      for (int k0 = 0; k0 < K2; k0 += 4) {
        const double a = E2T[(k0 + t) * LD + r0 + g];
        const int i2 = (k0 >> 1) + (t >> 1);
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const int nt = no + WPM * j;
          if (nt >= NTB) break;
          const int i1 = 4 * nt + (g >> 1);
          const double b = (i2 < n2 && i1 < n1) ? bsign * uvd[i2 * uvLd + 4 * i1 + bcomp] : 0.0;
          dmma(h[j], a, b);
        }
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int nt = no + WPM * j;
        if (nt >= NTB) break;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int col = 8 * nt + 2 * t + i;
          if (col < 2 * n1) HT[col * LD + r0 + g] = h[j][i];
        }
      }
    }
    __syncthreads();
    const int wr = warp % WR, wc = warp / WR;
    const int r0 = 32 * wr, c0 = wc * (128 / WC);
    double acc[4][NTC][2];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int nt = 0; nt < NTC; ++nt) acc[m][nt][0] = acc[m][nt][1] = 0.0;
#pragma unroll 2
    for (int k0 = 0; k0 < K1; k0 += 4) {
      double a[4], b[NTC];
#pragma unroll
      for (int m = 0; m < 4; ++m) a[m] = HT[(k0 + t) * LD + r0 + 8 * m + g];
#pragma unroll
      for (int nt = 0; nt < NTC; ++nt) b[nt] = E1[(k0 + t) * LDE + c0 + 8 * nt + g];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int nt = 0; nt < NTC; ++nt) dmma(acc[m][nt], a[m], b[nt]);
    }
    double* o = out + (int64_t)(sp.r0 + rl) * sp.n + j3 * (int64_t)N1 * N2;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int64_t j2 = rb * ROWS + r0 + 8 * m + g;
      if (j2 >= N2) continue;
#pragma unroll
      for (int nt = 0; nt < NTC; ++nt) {
        const int64_t j1 = cb * 128 + c0 + 8 * nt + 2 * t;
        double v0 = acc[m][nt][0], v1 = acc[m][nt][1];
        if (sp.applyMarginal) {  // multiVariateTransformation, randomFieldND.f90:139-178
          v0 = v0 * sp.margSd + sp.margAvg;
          v1 = v1 * sp.margSd + sp.margAvg;
          if (sp.lognormal) {
            v0 = exp(v0);
            v1 = exp(v1);
          }
        }
        double* d = o + j2 * N1 + j1;
        if (pairStore && j1 + 1 < N1) {
          *reinterpret_cast<double2*>(d) = make_double2(v0, v1);
        } else {
          if (j1 < N1) d[0] = v0;
          if (j1 + 1 < N1) d[1] = v1;
        }
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

size_t axis3_smem(const SepSpec& sp) {
  return (size_t)((2 * sp.kn[2] + 3) & ~3) * (kRows + kPadLd + 128 + kPadLd) * sizeof(double);
}
size_t axes21_smem(const SepSpec& sp, int rows) {
  const size_t K1 = (size_t)(2 * sp.kn[0] + 3) & ~(size_t)3, K2 = (size_t)(2 * sp.kn[1] + 3) & ~(size_t)3;
  const size_t slabs = (size_t)2 * sp.kn[1] * uv_row_stride(sp.kn[0]);
  return (K2 * (rows + kPadLd) + slabs + K1 * (rows + kPadLd) + K1 * (128 + kPadLd)) * sizeof(double);
}

template <int ROWS>
cudaError_t launch_axes21(const SepSpec& sp, const double2* E1, const double2* E2, const double4* UV, double* out,
                          int numSMs, cudaStream_t st) {
  const size_t smem = axes21_smem(sp, ROWS);
  cudaError_t e = cudaFuncSetAttribute(rf_sep_axes21<ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, rf_sep_axes21<ROWS>, kAxesThreads, smem);
  if (e != cudaSuccess) return e;
  if (occ < 1) return cudaErrorInvalidConfiguration;
  const int64_t items = ((sp.N[0] + 127) / 128) * ((sp.N[1] + ROWS - 1) / ROWS) * (int64_t)sp.nr * sp.N[2];
  const int grid = (int)std::min<int64_t>(items, (int64_t)occ * numSMs);
  rf_sep_axes21<ROWS><<<grid, kAxesThreads, smem, st>>>(sp, E1, E2, UV, out);
  return cudaGetLastError();
}

// Rows per item: 128 where the row axis is longer than 64 and the tiles fit
// shared memory (half the slab loads and syncs per field value), else 64.
constexpr size_t kMaxSmem = (size_t)227 * 1024;
cudaError_t launch_axes21_any(const SepSpec& sp, const double2* E1, const double2* E2, const double4* UV,
                              double* out, int numSMs, cudaStream_t st) {
  if (sp.N[1] > 64 && axes21_smem(sp, 128) <= kMaxSmem) return launch_axes21<128>(sp, E1, E2, UV, out, numSMs, st);
  return launch_axes21<64>(sp, E1, E2, UV, out, numSMs, st);
}

// Validation and the separable spec of a grid request (no device work).
int grid_spec(int nDim, const double* xMin, const double* xStep, const int64_t* xNStep, int corrMod, int margiFirst,
              const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method, const rf_options* opt,
              SepSpec& sp, Plan& P, int& device) {
  if (!xMin || !xStep || !xNStep || !corrL) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (nDim < 1 || nDim > 3) return fail(RF_EINVAL_NDIM, "nDim must be 1, 2 or 3 (got %d)", nDim);
  int64_t n = 1;
  for (int d = 0; d < nDim; ++d) {
    if (xNStep[d] < 1 || xNStep[d] > (1 << 24))
      return fail(RF_EINVAL_ARG, "xNStep(%d) = %lld outside 1..2^24", d + 1, (long long)xNStep[d]);
    if (xNStep[d] > 1 && !(xStep[d] > 0.0)) return fail(RF_EINVAL_ARG, "xStep(%d) must be > 0", d + 1);
    if (n > ((int64_t)1 << 40) / xNStep[d]) return fail(RF_EINVAL_ARG, "more than 2^40 grid points");
    n *= xNStep[d];
  }
  Request rq = make_request(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate(rq)) return rc;
  device = rq.opt.device;
  if (method != RF_SHINOZUKA)
    return fail(RF_ENOTSUP, "the grid path sums the Shinozuka tensor-grid spectrum (method 2); methods 1 and 3 "
                            "run through rf_generate_device");
  if (rq.opt.literal) return fail(RF_ENOTSUP, "literal mode (per-slab amplitudes) runs through rf_generate_device");
  // the extent the reference measures on the points: max - min of setGrid's coordinates
  double ext[3] = {0, 0, 0};
  for (int d = 0; d < nDim; ++d) ext[d] = (xMin[d] + xStep[d] * (double)(xNStep[d] - 1)) - xMin[d];
  rq.opt.precision = RF_PREC_FP32;  // the plan's operand layout is not used here
  if (int rc = build_plan(rq, ext, P)) return rc;
  memset(&sp, 0, sizeof(sp));
  sp.nDim = nDim;
  for (int d = 0; d < 3; ++d) {
    sp.N[d] = d < nDim ? (int32_t)xNStep[d] : 1;
    sp.kn[d] = d < nDim ? P.kNStep[d] : 1;
    sp.kDelta[d] = d < nDim ? P.kDelta[d] : 0.0;
    sp.xMin[d] = d < nDim ? xMin[d] : 0.0;
    sp.xStep[d] = d < nDim ? xStep[d] : 0.0;
    sp.corrL[d] = d < nDim ? corrL[d] : 1.0;
    if (sp.kn[d] > kMaxSepN)
      return fail(RF_ENOTSUP, "the grid path takes at most %d wavenumbers per axis (axis %d has %d); set "
                              "k_nstep or use rf_generate_device", kMaxSepN, d + 1, sp.kn[d]);
  }
  sp.S2 = nDim >= 2 ? 2 : 1;
  sp.S3 = nDim == 3 ? 2 : 1;
  sp.corrMod = corrMod;
  sp.ig1 = P.ig1;
  sp.ig2 = P.ig2;
  sp.K = P.K;
  sp.n = n;
  sp.ampMult = P.ampMult;
  sp.margSd = P.margSd;
  sp.margAvg = P.margAvg;
  sp.lognormal = P.lognormal;
  sp.applyMarginal = P.applyMarginal;
  return RF_OK;
}

// The kernels of a grid request on `st` (the caller holds the context's
// lock and has made its device current).
int grid_run(rf_context* ctx, SepSpec sp, const Plan& P, int Nmc, double* d_randField, cudaStream_t st) {
  ctx->launches = 0;
  ctx->evValid = false;
  const int64_t eCount = (int64_t)sp.kn[0] * sp.N[0] + (int64_t)sp.kn[1] * sp.N[1] + (int64_t)sp.kn[2] * sp.N[2];
  const int64_t pairs = (int64_t)sp.kn[0] * sp.kn[1];
  const int64_t perR = (2 * pairs * sp.kn[2] + (int64_t)sp.N[2] * pairs) * (int64_t)sizeof(double4);
  const int32_t rBlk = (int32_t)std::max<int64_t>(1, std::min<int64_t>(Nmc, (int64_t)kSepScratch / perR));
  const size_t eBytes = (size_t)((eCount * (int64_t)sizeof(double2) + 255) / 256 * 256);
  const size_t need = eBytes + (size_t)rBlk * (size_t)perR;
  if (int rc = ensure(ctx->dGrid, ctx->capGrid, need, "grid path scratch")) return rc;
  double2* E = reinterpret_cast<double2*>(ctx->dGrid);
  double4* PQ = reinterpret_cast<double4*>(reinterpret_cast<unsigned char*>(ctx->dGrid) + eBytes);
  double4* UV = PQ + (int64_t)rBlk * 2 * pairs * sp.kn[2];
  const double2* E1 = E;
  const double2* E2 = E1 + (int64_t)sp.kn[0] * sp.N[0];
  const double2* E3 = E2 + (int64_t)sp.kn[1] * sp.N[1];

  const size_t sm3 = axis3_smem(sp), sm21 = axes21_smem(sp, 64);
  RF_CUDA(cudaFuncSetAttribute(rf_sep_axis3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3), "smem attribute");
  int occ3 = 0;
  RF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, rf_sep_axis3, kSepThreads, sm3), "occupancy");
  if (occ3 < 1 || sm21 > kMaxSmem) return fail(RF_ENOTSUP, "grid path tiles do not fit shared memory");

  if (ctx->timing) {
    for (auto& e : ctx->ev)
      if (!e) RF_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    RF_CUDA(cudaEventRecord(ctx->ev[0], st), "cudaEventRecord");
  }
  rf_sep_phasors<<<(unsigned)((eCount + 255) / 256), 256, 0, st>>>(sp, E);
  RF_CUDA(cudaGetLastError(), "grid phasor kernel");
  ctx->launches = 1;
  bool first = true;
  for (int32_t r0 = 0; r0 < Nmc; r0 += rBlk) {
    sp.r0 = r0;
    sp.nr = std::min(rBlk, Nmc - r0);
    const int64_t nCoef = (int64_t)sp.nr * 2 * sp.kn[1] * sp.kn[2];
    rf_sep_coeffs<<<(unsigned)((nCoef + 255) / 256), 256, 0, st>>>(sp, jump_table(), PQ);
    RF_CUDA(cudaGetLastError(), "grid coefficient kernel");
    if (ctx->timing && first) RF_CUDA(cudaEventRecord(ctx->ev[1], st), "cudaEventRecord");
    first = false;
    const int64_t tiles3 = (int64_t)sp.nr * ((sp.N[2] + kRows - 1) / kRows) * ((pairs + 31) / 32);
    const int g3 = (int)std::min<int64_t>(tiles3, (int64_t)occ3 * ctx->numSMs);
    rf_sep_axis3<<<g3, kSepThreads, sm3, st>>>(sp, E3, PQ, reinterpret_cast<double*>(UV));
    RF_CUDA(cudaGetLastError(), "grid axis-3 kernel");
    RF_CUDA(launch_axes21_any(sp, E1, E2, UV, d_randField, ctx->numSMs, st), "grid axes-2/1 kernel");
    ctx->launches += 3;
  }
  if (ctx->timing) RF_CUDA(cudaEventRecord(ctx->ev[2], st), "cudaEventRecord");
  if (P.normalize) {
    if ((size_t)2 * Nmc * sizeof(double) > ctx->capWork)
      if (int rc = ensure(ctx->dWork, ctx->capWork, (size_t)2 * Nmc * sizeof(double), "moments")) return rc;
    RF_CUDA(launch_normalize_and_map(P, d_randField, Nmc, ctx->dWork, st), "normalisation kernels");
    ctx->launches += 3;
  }
  if (ctx->timing) {
    RF_CUDA(cudaEventRecord(ctx->ev[3], st), "cudaEventRecord");
    ctx->evValid = true;
  }
  return RF_OK;
}

// The separable spec of subdomain f of a blend (seed seedStart + f + 1, the
// reference's fieldNumber = f + 1, sample_RF.f90:311), its placement in the
// group grid in `bp`; the subdomain field leaves the marginal map to the group.
int blend_sub_spec(const rf_blend_grid* grid, const Request& base, const int32_t* L, const int32_t* O, int f,
                   int64_t seed0, SepSpec& sp, Plan& P, Plan& bp) {
  const int nd = grid->nDim;
  int32_t F[3] = {1, 1, 1}, G[3] = {1, 1, 1};
  for (int d = 0; d < nd; ++d) {
    F[d] = grid->nFields[d];
    G[d] = grid->xNStep[d];
  }
  const int32_t fi[3] = {f % F[0], (f / F[0]) % F[1], f / (F[0] * F[1])};
  double x0[3] = {0, 0, 0}, h[3] = {0, 0, 0};
  int64_t N[3] = {1, 1, 1};
  memset(&bp, 0, sizeof(bp));
  bp.nDim = nd;
  for (int d = 0; d < 3; ++d) {
    bp.bDims[d] = L[d];
    bp.bOrigin[d] = d < nd ? fi[d] * (L[d] - std::max(O[d], 0)) : 0;
    bp.gDims[d] = G[d];
    bp.bRamp[d] = d < nd ? O[d] : 0;
    if (d < nd) {
      h[d] = grid->xStep[d];
      x0[d] = grid->xMin[d] + (double)bp.bOrigin[d] * h[d];
      N[d] = L[d];
    }
  }
  bp.gTotal = (int64_t)G[0] * G[1] * G[2];
  rf_options o = base.opt;
  o.seed_start = seed0 + f + 1;
  o.normalize = 0;
  int device = 0;
  if (int rc = grid_spec(nd, x0, h, N, base.corrMod, base.margiFirst, base.corrL, base.fieldAvg, base.fieldVar,
                         base.Nmc, base.method, &o, sp, P, device))
    return rc;
  sp.applyMarginal = 0;
  return RF_OK;
}

}  // namespace

namespace rfh {

bool grid_blend_ok(const rf_blend_grid* grid, const Request& base) {
  if (base.method != RF_SHINOZUKA || base.opt.literal) return false;
  int32_t L[3], O[3];
  if (rf_blend_layout(grid, base.corrL, L, O) != RF_OK) return false;
  SepSpec sp;
  Plan P, bp;
  const int ok = blend_sub_spec(grid, base, L, O, 0, std::max<int64_t>(base.opt.seed_start, 0), sp, P, bp);
  g_err.clear();
  return ok == RF_OK;
}

int grid_blend_run(rf_context* c, const rf_blend_grid* grid, const Request& base, double* dOut, cudaStream_t st) {
  int32_t L[3], O[3];
  if (int rc = rf_blend_layout(grid, base.corrL, L, O)) return rc;
  int nSub = 1;
  int64_t gTotal = 1;
  for (int d = 0; d < grid->nDim; ++d) {
    nSub *= grid->nFields[d];
    gTotal *= grid->xNStep[d];
  }
  const int64_t sub = (int64_t)L[0] * L[1] * L[2];
  int64_t seed0 = base.opt.seed_start;
  if (seed0 < 0) {  // one stochastic seed, then + fieldNumber (sample_RF.f90:316-317)
    const auto t = std::chrono::steady_clock::now().time_since_epoch().count();
    seed0 = (int64_t)((uint64_t)t % 100000000ull);
  }
  if (int rc = ensure(c->dBlendSub, c->capBlendSub, sizeof(double) * (size_t)sub * base.Nmc, "blend subdomain field"))
    return rc;
  RF_CUDA(cudaMemsetAsync(dOut, 0, sizeof(double) * (size_t)gTotal * base.Nmc, st), "clear of randField");
  Plan Gp;
  for (int f = 0; f < nSub; ++f) {
    SepSpec sp;
    Plan P, bp;
    if (int rc = blend_sub_spec(grid, base, L, O, f, seed0, sp, P, bp)) return rc;
    if (int rc = grid_run(c, sp, P, base.Nmc, c->dBlendSub, st)) return rc;
    bp.dbgErr = c->dErr;
    RF_CUDA(launch_blend_add(bp, c->dBlendSub, dOut, sub, base.Nmc, st), "blend add kernel");
    if (f == nSub - 1) Gp = P;  // marginal parameters of the request
  }
  // the group plan of the border correction and the marginal map
  Gp.nDim = grid->nDim;
  Gp.Nmc = base.Nmc;
  Gp.n = gTotal;
  Gp.gTotal = gTotal;
  for (int d = 0; d < 3; ++d) {
    Gp.gDims[d] = d < grid->nDim ? grid->xNStep[d] : 1;
    Gp.bRamp[d] = d < grid->nDim ? O[d] : 0;
  }
  Gp.normalize = base.opt.normalize ? 1 : 0;
  return blend_finish(c, Gp, dOut, st);
}

}  // namespace rfh

extern "C" {

int rf_generate_grid(rf_context* ctx, int nDim, const double* xMin, const double* xStep, const int64_t* xNStep,
                     int corrMod, int margiFirst, const double* corrL, double fieldAvg, double fieldVar, int Nmc,
                     int method, double* d_randField, const rf_options* opt, void* stream) {
  rfh::NvtxRange nvtx_("rf_generate_grid");
  g_err.clear();
  if (!ctx || !d_randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  SepSpec sp;
  Plan P;
  int device = 0;
  if (int rc = grid_spec(nDim, xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt,
                         sp, P, device))
    return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  return grid_run(ctx, sp, P, Nmc, d_randField, stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream);
}

int rf_create_standard_gaussian_field_grid(int nDim, const double* xMin, const double* xStep, const int64_t* xNStep,
                                           int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                                           double fieldVar, int Nmc, int method, double* randField,
                                           const rf_options* opt) {
  rfh::NvtxRange nvtx_("rf_create_standard_gaussian_field_grid");
  g_err.clear();
  if (!randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  SepSpec sp;
  Plan P;
  int device = 0;
  if (int rc = grid_spec(nDim, xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt,
                         sp, P, device))
    return rc;
  rf_context* c = nullptr;
  if (int rc = default_context(device, &c)) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  RF_CUDA(cudaSetDevice(c->device), "cudaSetDevice");
  const size_t oBytes = sizeof(double) * (size_t)sp.n * (size_t)Nmc;
  if (int rc = ensure(c->dOut, c->capOut, oBytes, "field")) return rc;
  if (int rc = grid_run(c, sp, P, Nmc, c->dOut, c->stream)) return rc;
  RF_CUDA(cudaMemcpyAsync(randField, c->dOut, oBytes, cudaMemcpyDeviceToHost, c->stream), "copy of randField");
  RF_CUDA(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return check_device_error(c);
}

}  // extern "C"
