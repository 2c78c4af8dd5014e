// rf_fft.cu -- the FFT method (method 4) of randomFieldND on a structured
// grid (gen_Std_Gauss_FFT, randomFieldND.f90:520-763; k grid of
// set_kPoints's FFT branch, spectra_RF.f90:135-160).
//
// With coordinates and steps divided by corrL (gen_Std_Gauss,
// randomFieldND.f90:58-73) and n_d grid points per axis:
//   k grid   kNStep_d = 1 + nint(xRange_d / xStep_d) = n_d,
//            kDelta_d = 2 PI / (1.1 xRange_d), k = (i_1 kDelta_1, ...), axis 1
//            fastest (setGrid from 0); S(k) of set_SkVec (Gaussian:
//            prod_d exp(-k_d^2 / (4 PI)); cm_COS: the sixth k only);
//   draws    gamma_j = U_j (j = 1..K), then K - 1 draws skipped, then
//            phi_j = U_{2K-1+j} (the single-process case of :674-686);
//   X_j      (gamma_j - 1/2) sqrt(S(k_j)) cos(2 PI phi_j)            (:695-696);
//   field    the multi-dimensional FFTW REDFT01 (DCT-III, unnormalised:
//            Y_i = X_0 + 2 sum_{j>=1} X_j cos(pi j (2 i + 1) / (2 n))) of X
//            on the (n_1, n_2[, n_3]) grid, times sqrt(prod xStep) in 2-D and
//            2 sqrt(prod xStep) in 3-D (:702-736); 1-D stops in the reference.
// The transform is separable: one pass per axis, each a dense FP64
// n_d x n_d product applied to every line along the axis (n_d multiply-adds
// per value and pass; the cosine matrix is built on the device with cospi
// of exactly reduced arguments).  The last pass applies the scale and the
// marginal map (multiVariateTransformation, randomFieldND.f90:139-178).
// The reference fills realization 1 only; here realization r draws from the
// rnglib stream of seed_start + r (realization 1 is the reference's field).
#include <cmath>

#include "rf_internal.h"

using namespace rfb;
using namespace rfh;

namespace {

constexpr int kMaxFftAxis = 2048;
constexpr int kPassThreads = 256;

struct FftSpec {
  int32_t nDim;
  int32_t n[3];
  double kDelta[3];
  int32_t corrMod;
  int64_t K;
  int32_t ig1, ig2;
};

// X_j of the k grid point j (axis 1 fastest).
__global__ void rf_fft_amplitudes(const FftSpec sp, const JumpTable jt, double* __restrict__ X) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= sp.K) return;
  double S = 1.0;
  int64_t rem = j;
  for (int d = 0; d < sp.nDim; ++d) {
    const int64_t i = rem % sp.n[d];
    rem /= sp.n[d];
    const double k = 0.0 + sp.kDelta[d] * (double)i;
    S = S * 1.0 * exp(-((k * k) * 1.0) / (4.0 * kRefPi));  // spectra_RF.f90:202-208, corrL = 1
  }
  if (sp.corrMod == RF_CM_COS) S = (j == 5) ? 1.0 : 0.0;  // spectra_RF.f90:210-220
  const double gamma = r8_uni_at(jt, sp.ig1, sp.ig2, (uint64_t)(j + 1));
  const double phi = r8_uni_at(jt, sp.ig1, sp.ig2, (uint64_t)(2 * sp.K + j));
  X[j] = (gamma - 0.5) * sqrt(S) * cos(2.0 * kRefPi * phi);
}

// CT[j * n + i] = 1 (j = 0) or 2 cos(pi j (2 i + 1) / (2 n)).
__global__ void rf_dct3_matrix(int32_t n, double* __restrict__ CT) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * n) return;
  const int64_t j = t / n, i = t % n;
  if (j == 0) {
    CT[t] = 1.0;
    return;
  }
  const int64_t m = (j * (2 * i + 1)) % (4 * (int64_t)n);  // the argument modulo two periods, exactly
  CT[t] = 2.0 * cospi((double)m / (double)(2 * n));
}

// One DCT-III pass along the axis of length n with element stride `stride`:
// line l = (o, b), b < stride, starts at o * n * stride + b.  The last pass
// scales and applies the marginal map.
__global__ void __launch_bounds__(kPassThreads) rf_dct3_pass(const double* __restrict__ in, double* __restrict__ out,
                                                              const double* __restrict__ CT, int32_t n, int64_t stride,
                                                              int64_t lines, int32_t last, double scale, double sd,
                                                              double avg, int32_t lognormal) {
  extern __shared__ double line[];
  for (int64_t l = blockIdx.x; l < lines; l += gridDim.x) {
    const int64_t o = l / stride, b = l % stride;
    const int64_t base = o * (int64_t)n * stride + b;
    __syncthreads();  // the previous line is consumed
    for (int j = threadIdx.x; j < n; j += blockDim.x) line[j] = in[base + (int64_t)j * stride];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double acc = 0.0;
      for (int j = 0; j < n; ++j) acc += CT[(int64_t)j * n + i] * line[j];
      if (last) {
        acc = acc * scale * sd + avg;
        if (lognormal) acc = exp(acc);
      }
      out[base + (int64_t)i * stride] = acc;
    }
  }
}

}  // namespace

extern "C" {

int rf_generate_fft_grid(rf_context* ctx, int nDim, const int64_t* xNStep, const double* xStep, int corrMod,
                         int margiFirst, const double* corrL, double fieldAvg, double fieldVar, int Nmc,
                         double* d_randField, const rf_options* opt) {
  rfh::NvtxRange nvtx_("rf_generate_fft_grid");
  g_err.clear();
  if (!ctx || !xNStep || !xStep || !corrL || !d_randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (nDim != 2 && nDim != 3)
    return fail(RF_EINVAL_NDIM, "the FFT method is defined in 2-D and 3-D (got nDim = %d; randomFieldND.f90:591)",
                nDim);
  if (Nmc < 1) return fail(RF_EINVAL_NMC, "Nmc must be >= 1 (got %d)", Nmc);
  if (corrMod != RF_CM_GAUSSIAN && corrMod != RF_CM_COS) return fail(RF_EINVAL_CORRMOD, "corrMod must be 1 or 2");
  if (margiFirst != RF_FOM_GAUSSIAN && margiFirst != RF_FOM_LOGNORMAL)
    return fail(RF_EINVAL_MARGINAL, "margiFirst must be 1 or 2");
  if (margiFirst == RF_FOM_LOGNORMAL && !(fieldAvg > 0.0))
    return fail(RF_EINVAL_LOGNORMAL, "lognormal marginal needs fieldAvg > 0 (got %g)", fieldAvg);
  rf_options o;
  rf_options_init(&o);
  if (opt) o = *opt;
  FftSpec sp;
  sp.nDim = nDim;
  sp.corrMod = corrMod;
  sp.K = 1;
  double prodH = 1.0;
  for (int d = 0; d < 3; ++d) {
    sp.n[d] = 1;
    sp.kDelta[d] = 0.0;
  }
  for (int d = 0; d < nDim; ++d) {
    if (xNStep[d] < 2 || xNStep[d] > kMaxFftAxis)
      return fail(xNStep[d] < 2 ? RF_EINVAL_ARG : RF_ENOTSUP, "xNStep(%d) = %lld outside 2..%d", d + 1,
                  (long long)xNStep[d], kMaxFftAxis);
    if (!(corrL[d] > 0.0)) return fail(RF_EINVAL_CORRL, "corrL(%d) must be > 0", d + 1);
    if (!(xStep[d] > 0.0)) return fail(RF_EINVAL_ARG, "xStep(%d) must be > 0", d + 1);
    const double h = xStep[d] / corrL[d];
    const double xRange = (double)(xNStep[d] - 1) * h;
    sp.n[d] = (int32_t)xNStep[d];
    sp.kDelta[d] = 2.0 * kRefPi / (1.1 * xRange);
    sp.K *= xNStep[d];
    prodH *= h;
  }
  if (corrMod == RF_CM_COS && sp.K <= 6)
    return fail(RF_EINVAL_CORRMOD, "the cos correlation model needs more than 6 wavevectors");
  const double scale = (nDim == 3 ? 2.0 : 1.0) * std::sqrt(prodH);
  double sd = std::sqrt(fieldVar), avg = fieldAvg;
  if (margiFirst == RF_FOM_LOGNORMAL) {
    const double nv = std::log(1 + fieldVar / (fieldAvg * fieldAvg));
    sd = std::sqrt(nv);
    avg = std::log(fieldAvg) - nv / 2;
  }
  int64_t seed0 = o.seed_start;
  if (seed0 < 0) {
    Plan tmp;
    if (int rc = seeds(-1, tmp)) return rc;
    seed0 = (tmp.ig1 - 72) / 18;
  }

  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = ctx->stream;
  size_t ctWords = 0;
  for (int d = 0; d < nDim; ++d) ctWords += (size_t)sp.n[d] * (size_t)sp.n[d];
  if (int rc = ensure(ctx->dFft, ctx->capFft, (2 * (size_t)sp.K + ctWords) * sizeof(double), "FFT method buffers"))
    return rc;
  double* X = ctx->dFft;
  double* T = X + sp.K;
  double* CT[3] = {T + sp.K, nullptr, nullptr};
  for (int d = 1; d < nDim; ++d) CT[d] = CT[d - 1] + (size_t)sp.n[d - 1] * sp.n[d - 1];
  for (int d = 0; d < nDim; ++d) {
    const int64_t nn = (int64_t)sp.n[d] * sp.n[d];
    rf_dct3_matrix<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(sp.n[d], CT[d]);
    RF_CUDA(cudaGetLastError(), "DCT matrix kernel");
  }
  ctx->launches = nDim;
  for (int r = 0; r < Nmc; ++r) {
    Plan tmp;
    if (int rc = seeds(seed0 + r, tmp)) return rc;
    sp.ig1 = tmp.ig1;
    sp.ig2 = tmp.ig2;
    rf_fft_amplitudes<<<(unsigned)((sp.K + 255) / 256), 256, 0, st>>>(sp, jump_table(), X);
    RF_CUDA(cudaGetLastError(), "FFT amplitude kernel");
    // X -> T -> X (-> out), the last pass into column r
    double* src = X;
    double* dst = T;
    int64_t stride = 1;
    for (int d = 0; d < nDim; ++d) {
      const bool last = d + 1 == nDim;
      double* o2 = last ? d_randField + (int64_t)r * sp.K : dst;
      const int64_t lines = sp.K / sp.n[d];
      const int grid = (int)std::min<int64_t>(lines, 4 * (int64_t)ctx->numSMs);
      rf_dct3_pass<<<grid, kPassThreads, (size_t)sp.n[d] * sizeof(double), st>>>(
          src, o2, CT[d], sp.n[d], stride, lines, last ? 1 : 0, scale, sd, avg,
          margiFirst == RF_FOM_LOGNORMAL ? 1 : 0);
      RF_CUDA(cudaGetLastError(), "DCT pass kernel");
      stride *= sp.n[d];
      std::swap(src, dst);
    }
    ctx->launches += 1 + nDim;
  }
  RF_CUDA(cudaStreamSynchronize(st), "FFT method");
  return RF_OK;
}

}  // extern "C"
