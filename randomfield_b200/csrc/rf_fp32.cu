// rf_fp32.cu -- the plain FP32 form of the spectral-sum contraction.
//
// Same generators and table layout as the tensor-core form, but the trig
// tile goes to shared memory as FP32 and the contraction runs on the FFMA
// pipes: each thread owns 4 points x RPT realizations.  Partial sums of one
// stage are formed in FP32 and added into FP64 accumulators, so the
// accumulation error does not grow with the number of wavevectors.
#include "rf_device.cuh"
#include "rf_gen.cuh"
#include "rf_launch.h"

namespace rfb {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxKel = 2 * kStageCols;  // FP32 elements per stage (cos and sin)

struct Fp32Args {
  Plan P;
  const double* x;
  const float* B;       // [nChunks][2*chunkK][nmcPad]
  const double* ktab;   // GEN_TABLE: [nChunks][3][kTableChunk]
  double* out;
  int64_t row0, rows;
  int nb;               // realizations per CTA (8 * RPT)
};

__device__ __forceinline__ double finish_value(const Plan& P, double acc) {
  double v = acc * P.outScale;
  if (P.applyMarginal) {
    v = v * P.margSd + P.margAvg;
    if (P.lognormal) v = exp(v);
  }
  return v;
}

template <int GEN, int RPT, int LPAD>
__global__ void __launch_bounds__(kThreads) rf_fp32_kernel(const __grid_constant__ Fp32Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Plan& P = a.P;
  constexpr int NB = 8 * RPT;
  float* As = reinterpret_cast<float*>(smem);                 // [kMaxKel][128]
  float* Bs = As + kMaxKel * kTileM;                          // [kMaxKel][NB]
  double* sK = reinterpret_cast<double*>(Bs + kMaxKel * NB);  // one wavevector chunk
  float2* e12 = reinterpret_cast<float2*>(sK + kKtabStageDoubles);

  const int tid = threadIdx.x;
  const int row = tid & (kTileM - 1), h = tid >> 7;
  const int pg = tid & 31, rg = tid >> 5;
  const int64_t tile = blockIdx.x;
  const int rBase = blockIdx.y * NB;
  const int64_t p = a.row0 + tile * kTileM + row;
  const bool valid = p < a.row0 + a.rows;

  double x[3] = {0.0, 0.0, 0.0};
  if (valid) {
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < P.nDim) x[d] = a.x[p * P.nDim + d] / P.corrL[d];
  }

  const bool fastPhase = table_fast_phase(x, P.kMax);
  Grid3Thread g3;
  if (GEN == GEN_GRID3) {
    grid3_thread_setup<LPAD>(g3, P, h, x);
    if (h == 0) {
      for (int i = 0; i < P.kNStep[0]; ++i) e12[i * kTileM + row] = axis_phasor(P.kDelta[0], i, x[0]);
    } else {
      for (int i = 0; i < P.kNStep[1]; ++i) e12[(P.kNStep[0] + i) * kTileM + row] = axis_phasor(P.kDelta[1], i, x[1]);
    }
  }

  double acc64[RPT][4];
#pragma unroll
  for (int i = 0; i < RPT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc64[i][j] = 0.0;

  const int kel = 2 * P.chunkK;
  Grid3Outer outer;
  for (int64_t ch = 0; ch < P.nChunks; ++ch) {
    __syncthreads();  // previous stage fully consumed (and e12 written)
    // B stage: rows kel, columns [rBase, rBase + NB)
    const float* bsrc = a.B + ch * (int64_t)kel * P.nmcPad + rBase;
    for (int i = tid; i < kel * NB; i += kThreads) {
      const int e = i / NB, c = i % NB;
      Bs[e * NB + c] = bsrc[(int64_t)e * P.nmcPad + c];
    }
    if (GEN == GEN_TABLE) {
      // the FP64 part of the chunk (the fixed-point arrays serve the tensor-core forms)
      for (int i = tid; i < 3 * kTableChunk; i += kThreads) sK[i] = a.ktab[ch * kKtabStageDoubles + i];
      __syncthreads();
    }
    // trig tile: element 2c = cos, 2c+1 = sin of stage column c
    if (GEN == GEN_GRID3) {
      const float2 Pq = grid3_outer(P, e12, row, outer);
      outer.next(P.kNStep[0], P.kNStep[1]);
      const int col0 = h * LPAD;
      grid3_pairs<LPAD>(g3, Pq, [&](int idx, float c, float sn) {
        As[(2 * (col0 + idx)) * kTileM + row] = c;
        As[(2 * (col0 + idx) + 1) * kTileM + row] = sn;
      });
    } else {
      const int col0 = h * (kTableChunk / 2);
      auto put = [&](int idx, float c, float sn) {
        As[(2 * (col0 + idx)) * kTileM + row] = c;
        As[(2 * (col0 + idx) + 1) * kTileM + row] = sn;
      };
      // FP64 phases: no tensor-core work here for FP64 to contend with, and
      // the fixed-point form costs more instructions per pair
      if (fastPhase) table_pairs<true, kTableChunk / 2>(sK, h, x, put);
      else table_pairs<false, kTableChunk / 2>(sK, h, x, put);
    }
    __syncthreads();

    float acc[RPT][4];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int e = 0; e < kel; ++e) {
      const float4 av = *reinterpret_cast<const float4*>(&As[e * kTileM + 4 * pg]);
      float bv[RPT];
#pragma unroll
      for (int i = 0; i < RPT; ++i) bv[i] = Bs[e * NB + rg * RPT + i];
#pragma unroll
      for (int i = 0; i < RPT; ++i) {
        acc[i][0] = fmaf(av.x, bv[i], acc[i][0]);
        acc[i][1] = fmaf(av.y, bv[i], acc[i][1]);
        acc[i][2] = fmaf(av.z, bv[i], acc[i][2]);
        acc[i][3] = fmaf(av.w, bv[i], acc[i][3]);
      }
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc64[i][j] += (double)acc[i][j];
  }

  // epilogue: ampMult, marginal map, FP64 stores (a warp covers 128
  // consecutive points of one realization)
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int r = rBase + rg * RPT + i;
    if (r >= P.nmcBlk) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t pp = a.row0 + tile * kTileM + 4 * pg + j;
      if (pp < a.row0 + a.rows) a.out[(int64_t)(P.rOff + r) * P.n + pp] = finish_value(P, acc64[i][j]);
    }
  }
}

template <int GEN, int RPT, int LPAD>
cudaError_t launch_one(const Fp32Args& args, size_t smem, dim3 grid, cudaStream_t st) {
  auto fn = rf_fp32_kernel<GEN, RPT, LPAD>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, kThreads, smem, st>>>(args);
  return cudaGetLastError();
}

template <int RPT>
cudaError_t launch_rpt(const Plan& P, const Fp32Args& args, size_t smem, dim3 grid, cudaStream_t st) {
  if (P.gen != GEN_GRID3) return launch_one<GEN_TABLE, RPT, 0>(args, smem, grid, st);
  switch (P.lPad) {
    case 8: return launch_one<GEN_GRID3, RPT, 8>(args, smem, grid, st);
    case 16: return launch_one<GEN_GRID3, RPT, 16>(args, smem, grid, st);
    case 24: return launch_one<GEN_GRID3, RPT, 24>(args, smem, grid, st);
    case 32: return launch_one<GEN_GRID3, RPT, 32>(args, smem, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

int rpt_of(const Plan& P) {
  const int nb = P.nmcPad < 64 ? P.nmcPad : 64;
  int rpt = nb / 8;
  if (rpt >= 8) return 8;
  if (rpt >= 4) return 4;
  if (rpt >= 2) return 2;
  return 1;
}

}  // namespace

size_t fp32_smem_bytes(const Plan& P) {
  const int nb = 8 * rpt_of(P);
  const size_t e12 = (P.gen == GEN_GRID3) ? (size_t)(P.kNStep[0] + P.kNStep[1]) * kTileM * sizeof(float2) : 0;
  return (size_t)kMaxKel * kTileM * 4 + (size_t)kMaxKel * nb * 4 + kKtabStageBytes + e12;
}

cudaError_t launch_fp32(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                        int64_t row0, int64_t rows, cudaStream_t st) {
  Fp32Args args;
  args.P = P;
  args.x = dX;
  args.B = reinterpret_cast<const float*>(dB);
  args.ktab = dKtab;
  args.out = dOut;
  args.row0 = row0;
  args.rows = rows;
  const int rpt = rpt_of(P);
  args.nb = 8 * rpt;
  const size_t smem = fp32_smem_bytes(P);
  const int64_t tiles = (rows + kTileM - 1) / kTileM;
  dim3 grid((unsigned)tiles, (unsigned)((P.nmcPad + args.nb - 1) / args.nb));
  switch (rpt) {
    case 1: return launch_rpt<1>(P, args, smem, grid, st);
    case 2: return launch_rpt<2>(P, args, smem, grid, st);
    case 4: return launch_rpt<4>(P, args, smem, grid, st);
    default: return launch_rpt<8>(P, args, smem, grid, st);
  }
}

}  // namespace rfb
