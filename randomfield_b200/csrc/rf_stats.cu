// rf_stats.cu -- statistics of a generated field on the device
// (statistics_RF.f90), with no copy of the field to the host.
//
//   moments      per realization r: S_r = sum_i f(i, r), Q_r = sum_i f(i, r)^2;
//                mean S_r / n, deviation sqrt(Q_r / n - mean^2), and the same
//                over all n * Nmc values (calculate_average_and_stdVar_MPI,
//                statistics_RF.f90:18-174);
//   correlation  for a structured grid, realization 1 normalised as
//                g = (f - globalAvg) / globalStdDev; per axis d the circular
//                autocorrelation R(l) = (1 / (N_d L_d)) sum over the L_d lines
//                along d of sum_z g(z) g(z + l mod N_d), l < N_d / 2.  The
//                reference gets it through FFTW (rebuild_Sk_FFT, :258-419:
//                forward FFT / N_d, times its conjugate, mean over the lines,
//                unnormalised backward FFT, real part), which is the same sum
//                by the correlation theorem; rebuild_Sk (:180-252) keeps lags
//                0 .. N_d / 2 - 1 and rebuild_corrL (:425-443) integrates
//                them: 2 (sum R - (R_0 + R_last) / 2) xStep_d.
//
// Every sum runs in FP64 in a fixed order (partials per block in a fixed
// partition, then summed in index order), so repeated calls agree bit for
// bit.  The direct correlation costs N_d / 2 multiply-adds per value and
// axis, a few milliseconds up to 256^3.
#include <algorithm>
#include <cmath>

#include "rf_internal.h"

using namespace rfb;
using namespace rfh;

namespace {

constexpr int kThreads = 256;
constexpr int kCorrThreads = 128;
constexpr int kCorrBlocks = 512;  // fixed partition of the lines: results independent of the device
constexpr int kMaxAxis = 4096;    // line + lags in 48 KB of shared memory

// Sum of a block's values in a fixed order: warp trees, then warp 0 over the
// warp sums.  Every thread gets the result.
__device__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[0] = v;
  }
  __syncthreads();
  return red[0];
}

// Partial sums of column r (blockIdx.y) over chunk blockIdx.x of its points.
__global__ void __launch_bounds__(kThreads) rf_moment_partials(const double* __restrict__ f, int64_t n, int nblk,
                                                               double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  const int64_t r = blockIdx.y;
  const double* col = f + r * n;
  const int64_t chunk = (n + nblk - 1) / nblk;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  double s = 0.0, q = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = col[i];
    s += v;
    q += v * v;
  }
  s = block_sum(s, red);
  q = block_sum(q, red);
  if (threadIdx.x == 0) {
    part[2 * (r * nblk + blockIdx.x)] = s;
    part[2 * (r * nblk + blockIdx.x) + 1] = q;
  }
}

// S_r, Q_r from the partials of column r, in block order.
__global__ void rf_moment_final(const double* __restrict__ part, int nblk, int Nmc, double* __restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Nmc) return;
  double s = 0.0, q = 0.0;
  for (int b = 0; b < nblk; ++b) {
    s += part[2 * ((int64_t)r * nblk + b)];
    q += part[2 * ((int64_t)r * nblk + b) + 1];
  }
  out[2 * r] = s;
  out[2 * r + 1] = q;
}

// Partial circular autocorrelation of g = (f - avg) / sd along axis d over
// the lines blockIdx.x, blockIdx.x + gridDim.x, ...; part[blockIdx.x][l].
__global__ void __launch_bounds__(kCorrThreads) rf_corr_partials(const double* __restrict__ f, int64_t N0, int64_t N1,
                                                                 int64_t N2, int d, int M, double avg, double sd,
                                                                 double* __restrict__ part) {
  extern __shared__ double sm[];
  const int64_t Nd = d == 0 ? N0 : (d == 1 ? N1 : N2);
  double* line = sm;     // [Nd]
  double* acc = sm + Nd;  // [M]
  const int64_t L = N0 * N1 * N2 / Nd;
  for (int l = threadIdx.x; l < M; l += blockDim.x) acc[l] = 0.0;
  for (int64_t ln = blockIdx.x; ln < L; ln += gridDim.x) {
    int64_t base, stride;
    if (d == 0) {
      base = ln * N0;
      stride = 1;
    } else if (d == 1) {
      base = (ln % N0) + (ln / N0) * N0 * N1;
      stride = N0;
    } else {
      base = ln;
      stride = N0 * N1;
    }
    __syncthreads();  // the previous line is consumed
    for (int64_t z = threadIdx.x; z < Nd; z += blockDim.x) line[z] = (f[base + z * stride] - avg) / sd;
    __syncthreads();
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
      double c = 0.0;
      int64_t zz = l;
      for (int64_t z = 0; z < Nd; ++z) {
        c += line[z] * line[zz];
        if (++zz == Nd) zz = 0;
      }
      acc[l] += c;
    }
  }
  __syncthreads();
  for (int l = threadIdx.x; l < M; l += blockDim.x) part[(int64_t)blockIdx.x * M + l] = acc[l];
}

// R(l) = sum of the block partials in block order / (N_d L_d).
__global__ void rf_corr_final(const double* __restrict__ part, int nb, int M, double scale, double* __restrict__ R) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= M) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[(int64_t)b * M + l];
  R[l] = s * scale;
}

}  // namespace

extern "C" {

int rf_field_statistics(rf_context* ctx, const double* d_randField, int64_t n, int Nmc, int nDim,
                        const int64_t* xNStep, const double* xStep, double* evnt_avg, double* evnt_std, double* sk,
                        double* corrL_out, rf_field_stats* out) {
  rfh::NvtxRange nvtx_("rf_field_statistics");
  g_err.clear();
  if (!ctx || !d_randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (n < 1) return fail(RF_EINVAL_ARG, "n must be >= 1 (got %lld)", (long long)n);
  if (Nmc < 1) return fail(RF_EINVAL_NMC, "Nmc must be >= 1 (got %d)", Nmc);
  if (Nmc > 65535) return fail(RF_ENOTSUP, "Nmc above 65535 (one grid row of the moment kernel per realization)");
  if (nDim < 1 || nDim > 3) return fail(RF_EINVAL_NDIM, "nDim must be 1, 2 or 3 (got %d)", nDim);
  int64_t N[3] = {1, 1, 1};
  int M[3] = {0, 0, 0};
  if (xNStep) {
    int64_t prod = 1;
    for (int d = 0; d < nDim; ++d) {
      if (xNStep[d] < 2) return fail(RF_EINVAL_ARG, "xNStep(%d) must be >= 2 (got %lld)", d + 1, (long long)xNStep[d]);
      if (xNStep[d] > kMaxAxis)
        return fail(RF_ENOTSUP, "xNStep(%d) = %lld is above the %d points per axis of the correlation kernel", d + 1,
                    (long long)xNStep[d], kMaxAxis);
      N[d] = xNStep[d];
      M[d] = (int)(xNStep[d] / 2);
      prod *= xNStep[d];
    }
    if (prod != n) return fail(RF_EINVAL_ARG, "the grid has %lld points, the field %lld", (long long)prod, (long long)n);
    if (corrL_out && !xStep) return fail(RF_EINVAL_ARG, "corrL_out needs xStep");
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = ctx->stream;

  // scratch: moment partials and finals, correlation partials and lags
  int64_t nblk = (n + 8191) / 8192;
  if (nblk > 256) nblk = 256;
  const size_t momPart = (size_t)Nmc * (size_t)nblk * 2;
  int mTot = M[0] + M[1] + M[2];
  size_t corrPart = 0;
  for (int d = 0; d < nDim; ++d) corrPart = std::max(corrPart, (size_t)kCorrBlocks * (size_t)M[d]);
  const size_t words = momPart + 2 * (size_t)Nmc + corrPart + (size_t)mTot;
  if (int rc = ensure(ctx->dStats, ctx->capStats, words * sizeof(double), "statistics scratch")) return rc;
  if (int rc = ensure_host(ctx->hStats, ctx->capHStats, (2 * (size_t)Nmc + mTot) * sizeof(double), "statistics"))
    return rc;
  double* dPart = ctx->dStats;
  double* dMom = dPart + momPart;
  double* dCorr = dMom + 2 * (size_t)Nmc;
  double* dR = dCorr + corrPart;

  rf_moment_partials<<<dim3((unsigned)nblk, (unsigned)Nmc), kThreads, 0, st>>>(d_randField, n, (int)nblk, dPart);
  RF_CUDA(cudaGetLastError(), "moment kernel");
  rf_moment_final<<<(Nmc + 127) / 128, 128, 0, st>>>(dPart, (int)nblk, Nmc, dMom);
  RF_CUDA(cudaGetLastError(), "moment kernel");
  RF_CUDA(cudaMemcpyAsync(ctx->hStats, dMom, 2 * (size_t)Nmc * sizeof(double), cudaMemcpyDeviceToHost, st),
          "moments to host");
  RF_CUDA(cudaStreamSynchronize(st), "moments");
  double S = 0.0, Q = 0.0;
  for (int r = 0; r < Nmc; ++r) {
    const double s = ctx->hStats[2 * r], q = ctx->hStats[2 * r + 1];
    const double avg = s / (double)n;
    if (evnt_avg) evnt_avg[r] = avg;
    if (evnt_std) evnt_std[r] = std::sqrt(q / (double)n - avg * avg);
    S += s;
    Q += q;
  }
  const double total = (double)n * (double)Nmc;
  const double gAvg = S / total;
  const double gStd = std::sqrt(Q / total - gAvg * gAvg);
  if (out) {
    out->global_avg = gAvg;
    out->global_std = gStd;
    out->n = n;
    out->Nmc = Nmc;
    out->nDim = nDim;
  }
  if (!xNStep) return RF_OK;

  int off = 0;
  for (int d = 0; d < nDim; ++d) {
    const int64_t L = n / N[d];
    const int nb = (int)std::min<int64_t>(L, kCorrBlocks);
    const size_t smem = (size_t)(N[d] + M[d]) * sizeof(double);
    rf_corr_partials<<<nb, kCorrThreads, smem, st>>>(d_randField, N[0], N[1], N[2], d, M[d], gAvg, gStd, dCorr);
    RF_CUDA(cudaGetLastError(), "correlation kernel");
    rf_corr_final<<<(M[d] + 127) / 128, 128, 0, st>>>(dCorr, nb, M[d], 1.0 / ((double)N[d] * (double)L), dR + off);
    RF_CUDA(cudaGetLastError(), "correlation kernel");
    off += M[d];
  }
  RF_CUDA(cudaMemcpyAsync(ctx->hStats, dR, (size_t)mTot * sizeof(double), cudaMemcpyDeviceToHost, st),
          "correlation to host");
  RF_CUDA(cudaStreamSynchronize(st), "correlation");
  off = 0;
  for (int d = 0; d < nDim; ++d) {
    const double* R = ctx->hStats + off;
    if (sk)
      for (int l = 0; l < M[d]; ++l) sk[off + l] = R[l];
    if (corrL_out) {
      double s = 0.0;
      for (int l = 0; l < M[d]; ++l) s += R[l];
      corrL_out[d] = 2.0 * (s - (R[0] + R[M[d] - 1]) / 2.0) * xStep[d];
    }
    off += M[d];
  }
  return RF_OK;
}

}  // extern "C"
