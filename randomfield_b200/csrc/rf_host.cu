// rf_host.cu -- the C-ABI (include/randomfield_b200.h): validation with the
// reference's rules, problem geometry, device contexts, transfers and
// dispatch to the kernels.  No CPU fallback: without a usable CUDA device
// every generating entry point fails with RF_ENODEV / RF_ECUDA.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/randomfield_b200.h"
#include "rf_device.cuh"
#include "rf_internal.h"
#include "rf_launch.h"
#include "rf_plan.h"

using namespace rfb;

// ------------------------------------------------------------------ errors
namespace rfh {
thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  if (e == cudaErrorMemoryAllocation) return fail(RF_ENOMEM, "%s: %s", where, cudaGetErrorString(e));
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return fail(RF_ENODEV, "%s: %s", where, cudaGetErrorString(e));
  return fail(RF_ECUDA, "%s: %s", where, cudaGetErrorString(e));
}

// rnglib jump table: a^(2^j) mod m (rnglib.f90:548-659 multipliers).
const JumpTable& jump_table() {
  static JumpTable jt = [] {
    JumpTable t;
    int64_t b1 = kA1, b2 = kA2;
    for (int j = 0; j < 64; ++j) {
      t.p1[j] = b1;
      t.p2[j] = b2;
      b1 = (int64_t)(((unsigned __int128)b1 * (unsigned __int128)b1) % (unsigned __int128)kM1);
      b2 = (int64_t)(((unsigned __int128)b2 * (unsigned __int128)b2) % (unsigned __int128)kM2);
    }
    return t;
  }();
  return jt;
}

// spectra_RF.f90:15-44 (cm_GAUSSIAN values, also used for cm_COS whose
// reference kMax is left at init_RF's -1).
double kmax_nd(int nDim) { return nDim == 1 ? 6.457 : (nDim == 2 ? 7.035 : 7.355); }

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// type_inputRF.f90:1159-1206, randomFieldND.f90:162-166, constants_RF.f90:12-21
int validate(const Request& r) {
  if (r.opt.draws || r.opt.n_draws)
    return fail(RF_ENOTSUP, "caller-supplied draws are taken by rf_create_standard_gaussian_field_unstruct and "
                            "rf_generate_device only");
  if (r.n < 1) return fail(RF_EINVAL_ARG, "n must be >= 1 (got %lld)", (long long)r.n);
  if (r.nDim < 1 || r.nDim > 3) return fail(RF_EINVAL_NDIM, "nDim must be 1, 2 or 3 (got %d)", r.nDim);
  if (r.Nmc < 1) return fail(RF_EINVAL_NMC, "Nmc must be >= 1 (got %d)", r.Nmc);
  for (int d = 0; d < r.nDim; ++d)
    if (!(r.corrL[d] > 0.0)) return fail(RF_EINVAL_CORRL, "corrL(%d) must be > 0", d + 1);
  if (r.method != RF_ISOTROPIC && r.method != RF_SHINOZUKA && r.method != RF_RANDOMIZATION)
    return fail(RF_EINVAL_METHOD, "method must be 1 (isotropic), 2 (Shinozuka) or 3 (randomization), got %d",
                r.method);
  if (r.method == RF_ISOTROPIC && r.nDim < 2)
    return fail(RF_EINVAL_NDIM, "the isotropic method needs nDim 2 or 3");
  if (r.corrMod != RF_CM_GAUSSIAN && r.corrMod != RF_CM_COS)
    return fail(RF_EINVAL_CORRMOD, "corrMod must be 1 (gaussian) or 2 (cos), got %d", r.corrMod);
  if (r.margiFirst != RF_FOM_GAUSSIAN && r.margiFirst != RF_FOM_LOGNORMAL)
    return fail(RF_EINVAL_MARGINAL, "margiFirst must be 1 (gaussian) or 2 (lognormal), got %d", r.margiFirst);
  if (r.margiFirst == RF_FOM_LOGNORMAL && r.fieldAvg <= 0.0)
    return fail(RF_EINVAL_LOGNORMAL, "when using lognormal fieldAvg should be a positive number");
  const rf_options& o = r.opt;
  if (o.precision < RF_PREC_BF16 || o.precision > RF_PREC_FP8)
    return fail(RF_EINVAL_ARG, "unknown precision form %d", o.precision);
  if (o.literal && r.method == RF_ISOTROPIC)
    return fail(RF_EINVAL_ARG, "literal mode exists for the Shinozuka and randomization methods only");
  for (int d = 0; d < 3; ++d)
    if (o.k_nstep[d] < 0 || o.k_nstep[d] == 1) return fail(RF_EINVAL_ARG, "k_nstep must be 0 or >= 2");
  if (o.iso_n_radial < 0 || o.iso_n_radial == 1 || o.iso_n_dir < 0)
    return fail(RF_EINVAL_ARG, "iso_n_radial must be 0 or >= 2, iso_n_dir >= 0");
  return RF_OK;
}

// Geometry of spectra_RF.f90:50-133 (Shinozuka grid, isotropic radial rule),
// Whether axis d's extent enters the geometry: the Shinozuka/randomization
// step along d when its wavenumber count is not given, the isotropic radial
// step (from the diagonal) when the radial count is not given.
bool extent_needed(const Request& r, int d) {
  if (r.method == RF_ISOTROPIC) return !(r.opt.iso_n_radial > 0);
  return !(r.opt.k_nstep[d] > 0);
}

// ampMult of randomFieldND.f90:260-266.  ext[d] is the physical extent.
int geometry(const Request& r, const double* ext, Plan& P) {
  const rf_options& o = r.opt;
  memset(&P, 0, sizeof(P));
  P.nDim = r.nDim;
  P.n = r.n;
  P.Nmc = r.Nmc;
  P.method = r.method;
  P.corrMod = r.corrMod;
  P.margiFirst = r.margiFirst;
  P.literal = o.literal ? 1 : 0;
  P.normalize = o.normalize ? 1 : 0;
  P.prec = o.precision;
  for (int d = 0; d < 3; ++d) P.corrL[d] = d < r.nDim ? r.corrL[d] : 1.0;
  P.fieldAvg = r.fieldAvg;
  P.fieldVar = r.fieldVar;
  P.kMax = kmax_nd(r.nDim);
  double xr[3] = {0, 0, 0};
  for (int d = 0; d < r.nDim; ++d) {
    if (!extent_needed(r, d)) continue;  // an explicit wavenumber count leaves xRange unused
    const double e = o.x_range[d] > 0.0 ? o.x_range[d] : ext[d];
    if (!(e > 0.0) || !std::isfinite(e))
      return fail(RF_EINVAL_RANGE, "zero extent along axis %d: kDelta = 2 pi/(1.1 xRange) is infinite", d + 1);
    xr[d] = e / r.corrL[d];  // randomFieldND.f90:72
  }
  if (r.method != RF_ISOTROPIC) {  // Shinozuka grid; randomization shares its sizes (spectra_RF.f90:87-124)
    int64_t kn = 1;
    double prod = 1.0;
    for (int d = 0; d < r.nDim; ++d) {
      const double kd = 2.0 * kRefPi / (1.1 * xr[d]);
      const int ns = o.k_nstep[d] > 0 ? o.k_nstep[d] : 1 + (int)(1.0 * std::ceil(P.kMax / kd));
      if (ns < 2) return fail(RF_EINVAL_RANGE, "fewer than 2 wavenumbers along axis %d", d + 1);
      P.kNStep[d] = ns;
      P.kDelta[d] = P.kMax / (double)(ns - 1);
      kn *= ns;
      prod *= P.kDelta[d];
    }
    P.K = kn * ((int64_t)1 << (r.nDim - 1));
    P.ampMult = 2.0 * std::sqrt(prod / std::pow(2.0 * kRefPi, (double)r.nDim));
    if (r.method == RF_RANDOMIZATION) {
      // randomFieldND.f90:262 (literal); intended: a random wavevector of a
      // quadrant stands for kMax^nDim / kn of the spectral volume
      if (o.literal) P.ampMult = 2.0 * std::sqrt(1.0 / ((double)P.K * std::pow(2.0 * kRefPi, (double)r.nDim)));
      else
        P.ampMult = 2.0 * std::sqrt(std::pow(P.kMax, (double)r.nDim) / ((double)kn * std::pow(2.0 * kRefPi, (double)r.nDim)));
    }
  } else {
    double r2 = 0.0;
    for (int d = 0; d < r.nDim; ++d) r2 += xr[d] * xr[d];
    const double kd = 2.0 * kRefPi / (1.1 * std::sqrt(r2));
    const int nr = o.iso_n_radial > 0 ? o.iso_n_radial : 1 + (int)(5.0 * std::ceil(P.kMax / kd));
    const int nd = o.iso_n_dir > 0 ? o.iso_n_dir : 32;
    P.kNStep[0] = nr;
    P.kNStep[1] = nd;
    P.kDelta[0] = P.kMax / (double)(nr - 1);
    P.K = (int64_t)nr * nd;
    P.ampMult = 1.0;
  }
  if (r.corrMod == RF_CM_COS && P.K <= 6)
    return fail(RF_EINVAL_CORRMOD, "the cos correlation model needs more than 6 wavevectors");
  return RF_OK;
}

// Seed words after math_RF.f90:561: seed = 72 + 18*seedStart + 37*(i-1).
int seeds(int64_t seedStart, Plan& P) {
  if (seedStart < 0) {
    // stochastic seed from the clock, as calculate_random_seed does
    const auto t = std::chrono::steady_clock::now().time_since_epoch().count();
    seedStart = (int64_t)((uint64_t)t % 100000000ull);
  }
  const int64_t ig1 = 72 + 18 * seedStart, ig2 = ig1 + 37;
  if (ig2 >= kM2) return fail(RF_EINVAL_ARG, "seed_start too large for rnglib seeds");
  P.ig1 = (int32_t)ig1;
  P.ig2 = (int32_t)ig2;
  return RF_OK;
}

// Kernel layout of the plan.
int layout(Plan& P) {
  const bool tc = P.prec != PREC_FP32;
  P.gen = GEN_TABLE;
  if (P.method == RF_SHINOZUKA && P.nDim == 3 && !P.literal && !P.forceTable && P.kNStep[0] <= kMaxGridN &&
      P.kNStep[1] <= kMaxGridN && P.kNStep[2] <= kMaxGridN)
    P.gen = GEN_GRID3;
  if (P.gen == GEN_GRID3) {
    P.lPad = (int32_t)round_up(P.kNStep[2], 8);  // 8-aligned TMEM stores per half
    // Two outer groups per stage on the tensor-core path (up to 128 TMEM
    // columns): more MMAs per barrier wait of the issuing thread.  The number
    // of groups, n1*n2*2, is always even.
    P.gps = (tc && 4 * P.lPad <= kMaxStageCols) ? 2 : 1;
    P.chunkK = 2 * P.lPad * P.gps;
    P.nChunks = (int64_t)P.kNStep[0] * P.kNStep[1] * 2 / P.gps;
  } else {
    P.lPad = 0;
    P.gps = 1;
    P.chunkK = kTableChunk;
    P.nChunks = (P.K + kTableChunk - 1) / kTableChunk;
  }
  if (P.nmcBlk <= 0) {
    // the first realization block: one MMA holds at most 256 accumulator
    // columns and the hi/lo form uses two per realization
    const int32_t blk = P.prec == PREC_FP32 ? P.Nmc : (prec_hilo(P.prec) ? kMaxNmcPad / 2 : kMaxNmcPad);
    P.nmcBlk = std::min(P.Nmc, blk);
  }
  if (tc) {
    P.nmcPad = (int32_t)round_up(P.nmcBlk, 16);
    P.bRows = prec_hilo(P.prec) ? 2 * P.nmcPad : P.nmcPad;
    // one MMA covers all bRows (N <= 256); the accumulator uses bRows columns
    if (P.bRows > kMaxNmcPad) return fail(RF_ENOTSUP, "realization block too large for one MMA");
    P.stageBytes = (int64_t)2 * P.chunkK * P.bRows * (P.prec == PREC_FP8 ? 1 : 2);
  } else {
    int rpt = 1;
    while (rpt < 8 && 8 * rpt < P.nmcBlk) rpt *= 2;
    P.nmcPad = (int32_t)round_up(P.nmcBlk, 8 * rpt);
    P.bRows = P.nmcPad;
    P.stageBytes = (int64_t)2 * P.chunkK * P.nmcPad * 4;
  }
  // FP16 / FP8 operand side: scale B by 2^s so that the largest |B| sits near
  // 2^15 (FP16, max 65504) or 240 (e4m3, max 448).
  P.bScaleLog2 = 0;
  if (P.prec == PREC_FP16 || P.prec == PREC_FP8) {
    double bound = 1.0;  // Shinozuka: sqrt(S) <= 1
    if (P.method == RF_ISOTROPIC) {
      bound = 0.0;
      const int D = P.nDim;
      for (int j = 0; j < P.kNStep[0]; ++j) {
        const double rr = j * P.kDelta[0];
        const double S = P.corrMod == RF_CM_GAUSSIAN ? std::exp(-(rr * rr) / (4.0 * kRefPi)) : (j == 5 ? 1.0 : 0.0);
        const double shell = D == 3 ? 4.0 * kRefPi * rr * rr : 2.0 * kRefPi * rr;
        const double A = std::sqrt(2.0 * shell * S * P.kDelta[0] / (std::pow(2.0 * kRefPi, D) * P.kNStep[1]));
        bound = std::max(bound, A * std::sqrt(3.0));
      }
      if (bound <= 0.0) bound = 1.0;
    }
    P.bScaleLog2 = (int32_t)std::floor(std::log2((P.prec == PREC_FP8 ? 240.0 : 32768.0) / bound));
  }
  P.outScale = P.ampMult * std::ldexp(1.0, -P.bScaleLog2);
  // multiVariateTransformation (randomFieldND.f90:139-178)
  if (P.margiFirst == RF_FOM_GAUSSIAN) {
    P.margSd = std::sqrt(P.fieldVar);
    P.margAvg = P.fieldAvg;
    P.lognormal = 0;
  } else {
    const double nv = std::log(1 + P.fieldVar / (P.fieldAvg * P.fieldAvg));
    P.margSd = std::sqrt(nv);
    P.margAvg = std::log(P.fieldAvg) - nv / 2;
    P.lognormal = 1;
  }
  P.applyMarginal = P.normalize ? 0 : 1;
  return RF_OK;
}

// ----------------------------------------------------------------- extent
__global__ void rf_extent_kernel(const double* __restrict__ x, int64_t n, int nDim, double* __restrict__ part) {
  __shared__ double smin[3][256], smax[3][256];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < nDim; ++d) {
      const double v = x[i * nDim + d];
      lo[d] = fmin(lo[d], v);
      hi[d] = fmax(hi[d], v);
    }
  for (int d = 0; d < 3; ++d) {
    smin[d][threadIdx.x] = lo[d];
    smax[d][threadIdx.x] = hi[d];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int d = 0; d < 3; ++d) {
        smin[d][threadIdx.x] = fmin(smin[d][threadIdx.x], smin[d][threadIdx.x + s]);
        smax[d][threadIdx.x] = fmax(smax[d][threadIdx.x], smax[d][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      part[blockIdx.x * 6 + d] = smin[d][0];
      part[blockIdx.x * 6 + 3 + d] = smax[d][0];
    }
}

// ---------------------------------------------------------------- context

int context_init(rf_context* c, int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(RF_ENODEV, "no CUDA device available");
  }
  if (device < 0 || device >= count) return fail(RF_ENODEV, "device %d does not exist (%d present)", device, count);
  c->device = device;
  RF_CUDA(cudaSetDevice(device), "cudaSetDevice");
  cudaDeviceProp prop;
  RF_CUDA(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10) return fail(RF_ENODEV, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
  c->numSMs = prop.multiProcessorCount;
  RF_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  RF_CUDA(cudaMalloc(&c->dErr, sizeof(uint32_t)), "cudaMalloc(err)");
  RF_CUDA(cudaMemset(c->dErr, 0, sizeof(uint32_t)), "cudaMemset(err)");
  const size_t work = sizeof(double) * std::max<size_t>(6 * kExtentBlocks, 2 * 65536);
  if (int rc = ensure(c->dWork, c->capWork, work, "work")) return rc;
  RF_CUDA(cudaMallocHost(&c->hWork, work), "cudaMallocHost(work)");
  return RF_OK;
}

void context_free(rf_context* c) {
  if (c->device >= 0) cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->dB);
  cudaFree(c->dKtab);
  cudaFree(c->dWork);
  cudaFree(c->dStats);
  cudaFree(c->dFft);
  cudaFree(c->dGrid);
  cudaFree(c->dBlendSub);
  cudaFree(c->dDraws);
  if (c->hStats) cudaFreeHost(c->hStats);
  cudaFree(c->dErr);
  cudaFree(c->dX);
  cudaFree(c->dOut);
  if (c->hWork) cudaFreeHost(c->hWork);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->bev)
    if (e) cudaEventDestroy(e);
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  cudaFree(c->dArena);
  cudaFree(c->dDesc);
  cudaFree(c->dExt);
  if (c->hDesc) cudaFreeHost(c->hDesc);
  if (c->hExt) cudaFreeHost(c->hExt);
  for (auto& e : c->slabEv)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->h2dEv)
    if (e) cudaEventDestroy(e);
  if (c->copyStream) cudaStreamDestroy(c->copyStream);
  if (c->h2dStream) cudaStreamDestroy(c->h2dStream);
  if (c->stream) cudaStreamDestroy(c->stream);
}

void launch_extent(const double* dX, int64_t n, int nDim, double* part, cudaStream_t st) {
  rf_extent_kernel<<<kExtentBlocks, 256, 0, st>>>(dX, n, nDim, part);
}

// Extent of the device-resident points per axis (needed for xRange).
int device_extent(rf_context* c, const double* dX, int nDim, int64_t n, cudaStream_t st, double* ext) {
  launch_extent(dX, n, nDim, c->dWork, st);
  RF_CUDA(cudaGetLastError(), "extent kernel");
  ++c->launches;
  RF_CUDA(cudaMemcpyAsync(c->hWork, c->dWork, sizeof(double) * 6 * kExtentBlocks, cudaMemcpyDeviceToHost, st),
          "extent copy");
  RF_CUDA(cudaStreamSynchronize(st), "extent sync");
  for (int d = 0; d < nDim; ++d) {
    double lo = INFINITY, hi = -INFINITY;
    for (int b = 0; b < kExtentBlocks; ++b) {
      lo = std::min(lo, c->hWork[b * 6 + d]);
      hi = std::max(hi, c->hWork[b * 6 + 3 + d]);
    }
    ext[d] = hi - lo;
  }
  return RF_OK;
}

int build_plan(const Request& rq, const double* ext, Plan& P) {
  if (int rc = geometry(rq, ext, P)) return rc;
  if (int rc = seeds(rq.opt.seed_start, P)) return rc;
  if (rq.opt.draws && rq.opt.n_draws < draws_needed(P))
    return fail(RF_EINVAL_ARG, "the request makes %lld draws; draws holds %lld", (long long)draws_needed(P),
                (long long)rq.opt.n_draws);
  return layout(P);
}

// The caller's uniform draws (rf_options.draws) to the device, on `st`.
int upload_draws(rf_context* c, const Request& rq, Plan& P, cudaStream_t st) {
  P.dDraws = nullptr;
  P.nDraws = 0;
  if (!rq.opt.draws) return RF_OK;
  const int64_t need = draws_needed(P);
  if (int rc = ensure(c->dDraws, c->capDraws, sizeof(double) * (size_t)need, "caller draws")) return rc;
  RF_CUDA(cudaMemcpyAsync(c->dDraws, rq.opt.draws, sizeof(double) * (size_t)need, cudaMemcpyHostToDevice, st),
          "copy of the caller's draws");
  P.dDraws = c->dDraws;
  P.nDraws = need;
  return RF_OK;
}

// validate() for the entry points that take caller-supplied draws.
int validate_with_draws(const Request& rq) {
  Request r = rq;
  r.opt.draws = nullptr;
  r.opt.n_draws = 0;
  if (int rc = validate(r)) return rc;
  if (rq.opt.n_draws < 0 || (rq.opt.n_draws > 0 && !rq.opt.draws))
    return fail(RF_EINVAL_ARG, "draws must be non-null with n_draws > 0, or null");
  return RF_OK;
}

// The BF16 form splits each amplitude into hi and lo BF16 terms because one
// BF16 term leaves a relative rounding error of about 2^-9 per element, which
// with the trig tile's own rounding exceeds the 2e-3 bound.  The lo term of a
// wavevector matters in proportion to its share of the field's variance, so
// the stages whose wavevectors together carry at most kLoDropShare of it
// (sum of S(k) over the stage's wavevectors, the smallest stages first) keep
// the hi term only: their BF16 rounding adds a relative error of about
// 2^-9 sqrt(2 kLoDropShare / 3) = 5e-4 in quadrature to the trig tile's
// 1.1e-3.  For the 128^3 workload (24^3 x 4 wavevectors) that drops the lo
// rows of 347 of 576 stages: 30 % fewer MMAs and operand bytes.  GEN_GRID3
// requests of the Gaussian spectrum, alone or in a grouped launch (not the
// subdomains of a blend, nor the other generators, which keep both terms).
constexpr double kLoDropShare = 0.10;

void lo_layout(Plan& P) {
  P.loSkip = 0;
  if (P.prec != PREC_BF16 || P.gen != GEN_GRID3 || P.corrMod != RF_CM_GAUSSIAN || P.literal || P.blend) return;
  if (P.gps != 2 || P.nChunks > 32 * kLoMaskWords || P.nChunks < 2) return;
  const int32_t n1 = P.kNStep[0], n2 = P.kNStep[1];
  auto e = [&](int d, int32_t i) {
    const double k = P.kDelta[d] * (double)i;
    return std::exp(-(k * k) / (4.0 * kRefPi));
  };
  // a stage holds the groups 2s and 2s+1, g = i1 + n1 (i2 + n2 s2); the
  // axis-3 factor is common to all groups
  std::vector<std::pair<double, int64_t>> E((size_t)P.nChunks);
  double total = 0.0;
  for (int64_t s = 0; s < P.nChunks; ++s) {
    double w = 0.0;
    for (int64_t g = 2 * s; g < 2 * s + 2; ++g) {
      const int32_t i1 = (int32_t)(g % n1), i2 = (int32_t)((g / n1) % n2);
      w += e(0, i1) * e(1, i2);
    }
    E[(size_t)s] = {w, s};
    total += w;
  }
  std::sort(E.begin(), E.end());
  for (auto& m : P.loMask) m = ~0u;
  double dropped = 0.0;
  for (const auto& x : E) {
    if (x.second == 0) continue;  // the first stage initialises both accumulator halves
    if (dropped + x.first > kLoDropShare * total) break;
    dropped += x.first;
    P.loMask[x.second >> 5] &= ~(1u << (x.second & 31));
  }
  P.loSkip = 1;
}

// The table generator's trig tile in BF16 leaves a relative error of about
// 1.3e-3 in the field whatever the amplitude side does.  On a domain of a few
// correlation lengths the norm of one realization fluctuates a lot, and with
// it that realization's relative error (a 1-D field over 5 correlation
// lengths and 40 wavevectors: 2.4e-3 in one of 8).  Single BF16 requests of
// at most kTableALoPairs (point, wavevector) pairs therefore carry the trig
// tile's lo term too (its rounding residual: one more MMA per K-step), which
// removes that error; larger requests, whose cost it would double on the
// tensor side and whose realizations span many correlation lengths (the
// 200k-point isotropic config: 1.5e-3 worst realization without it), keep
// the hi term alone.
constexpr double kTableALoPairs = 67108864.0;  // 2^26

void table_alo_layout(Plan& P) {
  P.tableALo = 0;
  if (P.gen != GEN_TABLE || P.prec != PREC_BF16) return;
  if ((double)P.n * (double)P.K > kTableALoPairs) return;
  P.tableALo = 1;
}

// GEN_OUTER (rf_outer.cu) for single 3-D Shinozuka requests on the 16-bit
// tensor-core forms: the same sum as GEN_GRID3 with the outer phasors as the
// generated operand.  A 16-bit rounding of both operands leaves a relative
// error of about 2.1e-3 in the field (BF16), in proportion to the share of
// the field's variance the rounded terms carry.  The K-steps (8 outer groups
// each) are ranked by that share (sum of S1(k1) S2(k2) over the K-step's
// groups; the axis-3 factor is common), and in the BF16 form those carrying
// all but kOuterTf32Left of the variance take both operands as TF32 (oTf32):
// the two units of a K-step hold its 16 K values in 32-bit containers, and
// two kind::tf32 MMAs of K = 8 replace the one BF16 MMA.  A numpy emulation
// on the 128^3 workload (24^3 x 4 wavevectors, Nmc 64, 12,288 points) gives
// relative L2 1.08e-3, worst realization 1.17e-3, at 1.26x the MMA cycles of
// BF16 alone; 0.3 left: 1.19e-3 at 1.23x; 0.2: 9.8e-4 at 1.30x.  The BF16
// hi/lo split it replaced (the rounding residual of both operands as a
// second BF16 term, three MMAs per K-step) gave 1.16e-3 and 1.27e-3 at 1.46x
// with 0.3 of the variance left.
constexpr double kOuterTf32Left = 0.25;

// The K-steps that keep their lo terms: ranked by the field variance they
// carry (the Gaussian spectrum's axis-1 and axis-2 factors summed over the
// K-step's 8 groups), A keeps its lo term on the K-steps above the share
// leftA of the total, B on those above leftB (cm_COS: every K-step keeps
// both).
void outer_rank_masks(Plan& P, double leftA, double leftB) {
  const int32_t n1 = P.kNStep[0], nK = P.oNK;
  memset(P.loMask, 0, sizeof(P.loMask));
  memset(P.aLoMask, 0, sizeof(P.aLoMask));
  std::vector<std::pair<double, int32_t>> E((size_t)nK);
  double total = 0.0;
  for (int32_t j = 0; j < nK; ++j) {
    int32_t jj = 0, i2 = 0, s2 = 0;
    outer_kstep_groups(P, j, &jj, &i2, &s2);
    double w = 0.0;
    for (int32_t i1 = 8 * jj; i1 < std::min(n1, 8 * jj + 8); ++i1) {
      if (P.corrMod != RF_CM_GAUSSIAN) {
        w += 1.0;  // cm_COS: no ranking, every K-step keeps both lo terms
        continue;
      }
      const double k1 = P.kDelta[0] * i1, k2 = P.kDelta[1] * i2;
      w += std::exp(-(k1 * k1) / (4.0 * kRefPi)) * std::exp(-(k2 * k2) / (4.0 * kRefPi));
    }
    E[(size_t)j] = {w, j};
    total += w;
  }
  std::sort(E.begin(), E.end(), [](const std::pair<double, int32_t>& a, const std::pair<double, int32_t>& b) {
    return a.first > b.first || (a.first == b.first && a.second < b.second);
  });
  const bool all = P.corrMod != RF_CM_GAUSSIAN;
  double covered = 0.0;
  for (const auto& e : E) {
    const int32_t j = e.second;
    if (all || covered < (1.0 - leftA) * total) P.aLoMask[j >> 5] |= 1u << (j & 31);
    if (all || covered < (1.0 - leftB) * total) P.loMask[j >> 5] |= 1u << (j & 31);
    covered += e.first;
  }
}

// Ring stages of a GEN_OUTER chunk (kOuterStageUnits A and B units per
// stage, K-steps in order) and the chunk's B bytes.  CTA-pair plans also
// close a stage before every K-step that starts an i2 run (i2 = 0), so that
// a stage's K-steps share s2 and the axis-1 block (rf_outer_pair.cu's
// generators rely on it).
void outer_stage_layout(Plan& P) {
  const int32_t nK = P.oNK, n2 = P.kNStep[1];
  P.oChunkBytes = (int64_t)(nK + mask_rank(P.loMask, nK)) * P.oKstepBytes * (P.oPair ? 2 : 1);
  memset(P.oStageEnd, 0, sizeof(P.oStageEnd));
  int32_t ua = 0, ub = 0;
  for (int32_t j = 0; j < nK; ++j) {
    const int32_t a = outer_a_lo(P, j) ? 2 : 1, b = outer_b_lo(P, j) ? 2 : 1;
    const bool runStart = P.oPair && j > 0 && j % n2 == 0;
    if (runStart || ua + a > kOuterStageUnits || ub + b > kOuterStageUnits) {
      P.oStageEnd[(j - 1) >> 5] |= 1u << ((j - 1) & 31);
      ua = ub = 0;
    }
    ua += a;
    ub += b;
  }
  P.oStageEnd[(nK - 1) >> 5] |= 1u << ((nK - 1) & 31);
}

void outer_layout(Plan& P) {
  if (P.gen != GEN_GRID3 || P.literal) return;
  if (P.prec != PREC_BF16 && P.prec != PREC_FP16 && P.prec != PREC_BF16_FAST) return;
  if (P.kNStep[0] > kOuterMaxN1P || P.lPad > 32) return;
  const int32_t n1 = P.kNStep[0], n2 = P.kNStep[1];
  const int32_t n1p = (int32_t)round_up(n1, 8);
  const int32_t nK = (n1p / 8) * n2 * 2;
  if (nK > kOuterMaxKsteps) return;
  P.gen = GEN_OUTER;
  P.n1p = n1p;
  P.oNK = nK;
  P.oPair = 0;
  P.oTf32 = 0;
  P.oRc = std::min<int32_t>(P.nmcBlk, 256 / (2 * P.lPad));
  P.oNR = (P.nmcBlk + P.oRc - 1) / P.oRc;
  P.oKstepBytes = (int64_t)16 * (2 * P.lPad * P.oRc) * 2;
  memset(P.loMask, 0, sizeof(P.loMask));
  memset(P.aLoMask, 0, sizeof(P.aLoMask));
  P.loSkip = 1;  // B lo blocks only where loMask says
  if (P.prec == PREC_BF16) {  // TF32 K-steps (both masks) where the variance needs them
    P.oTf32 = 1;
    outer_rank_masks(P, kOuterTf32Left, kOuterTf32Left);
  }
  outer_stage_layout(P);
  // the draw of wavevector (s3 = -) lies n1 n2 n3 calls after that of (s3 = +)
  {
    const JumpTable& jt = jump_table();
    const uint64_t d = (uint64_t)n1 * (uint64_t)n2 * (uint64_t)P.kNStep[2];
    unsigned __int128 m1 = 1, m2 = 1;
    for (int j = 0; j < 64; ++j) {
      if ((d >> j) & 1u) {
        m1 = (m1 * (unsigned __int128)jt.p1[j]) % (unsigned __int128)kM1;
        m2 = (m2 * (unsigned __int128)jt.p2[j]) % (unsigned __int128)kM2;
      }
    }
    P.oStepM1 = (int64_t)m1;
    P.oStepM2 = (int64_t)m2;
  }
  // FP16: B holds sums of two amplitudes (|W| <= 2), scaled so that the
  // largest sits near 2^15
  if (P.prec == PREC_FP16) {
    P.bScaleLog2 = 14;
    P.outScale = P.ampMult * std::ldexp(1.0, -P.bScaleLog2);
  }
}

// The CTA-pair form of a GEN_OUTER plan (rf_outer_pair.cu) for single
// requests of at least two 256-point items and two realizations: an MMA of
// M = 256 (one 128-point tile per CTA) per N half, two halves of oRc
// realizations per chunk, so that a chunk covers twice the realizations and
// the generators build A for half as many chunks.  The last chunk's missing
// realizations are zero columns of B (their MMAs run, their values are not
// stored).  The TF32 K-steps (BF16) are outer_layout's.  `always`: every
// GEN_OUTER plan, whatever its size (the grouped kernel of a batch runs all
// its outer-group units on CTA pairs; a unit of one realization leaves a half
// of zero columns, one of fewer than 256 points the rows past its end).
void outer_pair_layout(Plan& P, bool always) {
  if (P.gen != GEN_OUTER) return;
  if (!always && (P.nmcBlk < 2 || P.n < 2 * 2 * kTileM)) return;
  P.oPair = 1;
  P.oRc = std::min<int32_t>((P.nmcBlk + 1) / 2, 256 / (2 * P.lPad));
  P.oNR = (P.nmcBlk + 2 * P.oRc - 1) / (2 * P.oRc);
  // per rank: the K-step block holds lPad oRc rows of each half
  P.oKstepBytes = (int64_t)16 * (2 * P.lPad * P.oRc) * 2;
  outer_stage_layout(P);
}

// Realizations per launch: one MMA holds at most 256 accumulator columns,
// and the hi/lo form uses two per realization.
int32_t realization_block(const Plan& P) {
  if (P.prec == PREC_FP32) return P.Nmc;
  return prec_hilo(P.prec) ? kMaxNmcPad / 2 : kMaxNmcPad;
}

int run_block(rf_context* c, const Plan& P, const double* dX, double* dOut, cudaStream_t st);

// Tables + contraction (+ normalisation) for a plan whose points sit in dX,
// one launch pair per realization block.
int run_plan(rf_context* c, const Plan& P0, const double* dX, double* dOut, cudaStream_t st) {
  const int32_t blk = realization_block(P0);
  if (c->timing) {
    for (auto& e : c->ev)
      if (!e) RF_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    RF_CUDA(cudaEventRecord(c->ev[0], st), "cudaEventRecord");
  }
  for (int32_t r0 = 0; r0 < P0.Nmc; r0 += blk) {
    Plan P = P0;
    P.rOff = r0;
    P.nmcBlk = std::min(blk, P0.Nmc - r0);
    if (int rc = layout(P)) return rc;
    lo_layout(P);
    outer_layout(P);
    outer_pair_layout(P);
    table_alo_layout(P);
    P.dbgErr = c->dErr;
    if (int rc = run_block(c, P, dX, dOut, st)) return rc;
  }
  if (c->timing) RF_CUDA(cudaEventRecord(c->ev[2], st), "cudaEventRecord");
  if (P0.normalize) {
    if ((size_t)2 * P0.Nmc * sizeof(double) > c->capWork)
      if (int rc = ensure(c->dWork, c->capWork, (size_t)2 * P0.Nmc * sizeof(double), "moments")) return rc;
    RF_CUDA(launch_normalize_and_map(P0, dOut, P0.literal ? 1 : P0.Nmc, c->dWork, st), "normalisation kernels");
    c->launches += 3;
  }
  if (c->timing) {
    RF_CUDA(cudaEventRecord(c->ev[3], st), "cudaEventRecord");
    c->evValid = true;
  }
  return RF_OK;
}

int run_block(rf_context* c, const Plan& P, const double* dX, double* dOut, cudaStream_t st) {
  const size_t bBytes = (size_t)operand_bytes(P);
  if (int rc = ensure(c->dB, c->capB, bBytes, "contraction operand")) return rc;
  double* ktab = nullptr;
  if (P.gen == GEN_TABLE) {
    if (int rc = ensure(c->dKtab, c->capK, (size_t)P.nChunks * kKtabStageBytes, "wavevector table"))
      return rc;
    ktab = c->dKtab;
  }
  if (P.prec != PREC_FP32 && tc_smem_bytes(P, nullptr) == 0)
    return fail(RF_ENOTSUP, "stage too large for shared memory (Nmc or wavenumbers per axis too large)");
  int64_t xSlab = P.n, nSlab = 1;
  if (P.literal) {
    // randomFieldND.f90:237-239
    xSlab = (int64_t)((double)P.nDim * 1e8 / (double)P.K);
    if (xSlab > P.n) xSlab = P.n;
    if (xSlab < 1) xSlab = 1;
    nSlab = (P.n + xSlab - 1) / xSlab;
  }
  for (int64_t m = 0; m < nSlab; ++m) {
    const int64_t row0 = m * xSlab;
    const int64_t rows = std::min(xSlab, P.n - row0);
    RF_CUDA(launch_tables(P, jump_table(), c->dB, ktab, P.literal ? m : -1, nSlab, st), "table kernel");
    if (c->timing && m == 0 && P.rOff == 0) RF_CUDA(cudaEventRecord(c->ev[1], st), "cudaEventRecord");
    if (P.prec == PREC_FP32) {
      RF_CUDA(launch_fp32(P, dX, c->dB, ktab, dOut, row0, rows, st), "FP32 contraction kernel");
    } else {
      RF_CUDA(launch_tc(P, dX, c->dB, ktab, dOut, row0, rows, c->dErr, c->numSMs, st), "tcgen05 contraction kernel");
    }
    c->launches += 2;
  }
  return RF_OK;
}

// The flat entry point's tail for large fields into page-locked host memory:
// the contraction runs in point slabs on the context's stream and each
// slab's n_slab x Nmc block goes to the host on a second stream while the
// next slab computes (one 2-D copy per slab: Nmc rows of the slab's points).
// Only the last slab's copy is left after the kernels.  With hX (the points
// still on the host) the slabs' points go up on a third stream, each ahead
// of its slab's kernel, behind the first slab's copy only.  Tensor-core forms,
// one realization block, no literal slabs, no normalisation pass (which needs
// the whole field first); returns RF_ENOTSUP otherwise so that the caller
// takes the plain path.
int run_plan_slabs(rf_context* c, const Plan& P0, double* dX, double* dOut, double* hOut, cudaStream_t st,
                   const double* hX) {
  if (P0.prec == PREC_FP32 || P0.literal || P0.normalize || P0.Nmc > realization_block(P0)) return RF_ENOTSUP;
  const int64_t tiles = (P0.n + kTileM - 1) / kTileM;
  int nSlabs = (int)std::min<int64_t>(16, tiles / (8 * (int64_t)c->numSMs));
  if (nSlabs < 2) return RF_ENOTSUP;
  Plan P = P0;
  P.rOff = 0;
  P.nmcBlk = P0.Nmc;
  if (int rc = layout(P)) return rc;
  lo_layout(P);
  outer_layout(P);
  outer_pair_layout(P);
  table_alo_layout(P);
  P.dbgErr = c->dErr;
  if (tc_smem_bytes(P, nullptr) == 0)
    return fail(RF_ENOTSUP, "stage too large for shared memory (Nmc or wavenumbers per axis too large)");
  if (!c->copyStream) RF_CUDA(cudaStreamCreateWithFlags(&c->copyStream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!c->h2dStream) RF_CUDA(cudaStreamCreateWithFlags(&c->h2dStream, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto& e : c->slabEv)
    if (!e) RF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  for (auto& e : c->h2dEv)
    if (!e) RF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  if (int rc = ensure(c->dB, c->capB, (size_t)operand_bytes(P), "contraction operand")) return rc;
  double* ktab = nullptr;
  if (P.gen == GEN_TABLE) {
    if (int rc = ensure(c->dKtab, c->capK, (size_t)P.nChunks * kKtabStageBytes, "wavevector table")) return rc;
    ktab = c->dKtab;
  }
  RF_CUDA(launch_tables(P, jump_table(), c->dB, ktab, -1, 1, st), "table kernel");
  const int64_t slabRows = round_up((P.n + nSlabs - 1) / nSlabs, kTileM);
  const size_t pitch = sizeof(double) * (size_t)P.n;
  if (hX) {
    int j = 0;
    for (int64_t row0 = 0; row0 < P.n; row0 += slabRows, ++j) {
      const int64_t rows = std::min(slabRows, P.n - row0);
      const size_t pb = sizeof(double) * (size_t)P.nDim;
      RF_CUDA(cudaMemcpyAsync(dX + row0 * P.nDim, hX + row0 * P.nDim, pb * (size_t)rows, cudaMemcpyHostToDevice,
                              c->h2dStream),
              "copy of a point slab");
      RF_CUDA(cudaEventRecord(c->h2dEv[j], c->h2dStream), "cudaEventRecord");
    }
  }
  int k = 0;
  for (int64_t row0 = 0; row0 < P.n; row0 += slabRows, ++k) {
    const int64_t rows = std::min(slabRows, P.n - row0);
    if (hX) RF_CUDA(cudaStreamWaitEvent(st, c->h2dEv[k], 0), "cudaStreamWaitEvent");
    RF_CUDA(launch_tc(P, dX, c->dB, ktab, dOut, row0, rows, c->dErr, c->numSMs, st), "tcgen05 contraction kernel");
    RF_CUDA(cudaEventRecord(c->slabEv[k], st), "cudaEventRecord");
    RF_CUDA(cudaStreamWaitEvent(c->copyStream, c->slabEv[k], 0), "cudaStreamWaitEvent");
    RF_CUDA(cudaMemcpy2DAsync(hOut + row0, pitch, dOut + row0, pitch, sizeof(double) * (size_t)rows, (size_t)P.Nmc,
                              cudaMemcpyDeviceToHost, c->copyStream),
            "copy of a field slab");
    c->launches += 1;
  }
  c->launches += 1;
  RF_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  RF_CUDA(cudaStreamSynchronize(c->copyStream), "cudaStreamSynchronize");
  if (hX) RF_CUDA(cudaStreamSynchronize(c->h2dStream), "cudaStreamSynchronize");
  return RF_OK;
}

int check_device_error(rf_context* c) {
  uint32_t err = 0;
  RF_CUDA(cudaMemcpy(&err, c->dErr, sizeof(err), cudaMemcpyDeviceToHost), "error word");
  if (err) {
    cudaMemset(c->dErr, 0, sizeof(uint32_t));
    if (err & kErrBounds)
      return fail(RF_EBOUNDS, "a device index check failed (error word 0x%x); results are invalid", err);
    return fail(RF_ETIMEDOUT, "a bounded device wait expired (error word 0x%x); results are invalid", err);
  }
  return RF_OK;
}

std::mutex g_default_mu;
rf_context* g_default[64] = {nullptr};

int default_context(int device, rf_context** out) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (device < 0 || device >= 64) return fail(RF_ENODEV, "bad device ordinal %d", device);
  if (!g_default[device]) {
    rf_context* c = new rf_context();
    if (int rc = context_init(c, device)) {
      context_free(c);
      delete c;
      return rc;
    }
    g_default[device] = c;
  }
  *out = g_default[device];
  return RF_OK;
}

Request make_request(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                     double fieldVar, int Nmc, int method, const rf_options* opt) {
  Request r;
  r.nDim = nDim;
  r.n = n;
  r.corrMod = corrMod;
  r.margiFirst = margiFirst;
  r.Nmc = Nmc;
  r.method = method;
  for (int d = 0; d < 3; ++d) r.corrL[d] = (corrL && d < nDim && d >= 0) ? corrL[d] : 1.0;
  r.fieldAvg = fieldAvg;
  r.fieldVar = fieldVar;
  rf_options_init(&r.opt);
  if (opt) {
    const size_t sz = (opt->size > 0 && (size_t)opt->size < sizeof(rf_options)) ? (size_t)opt->size : sizeof(rf_options);
    memcpy(&r.opt, opt, sz);
    r.opt.size = sizeof(rf_options);
  }
  return r;
}

}  // namespace rfh

using namespace rfh;

// ------------------------------------------------- planning for other units
// Thin wrappers over the validation and planning above for entry points
// implemented in other translation units (rf_noalloc.cu).
namespace rfb {

int host_fail(int code, const char* msg) { return fail(code, "%s", msg); }

void host_clear_error() { g_err.clear(); }

const JumpTable& host_jump_table() { return jump_table(); }

int host_validate(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                  double fieldVar, int Nmc, int method, const rf_options* opt, bool* needExtent) {
  Request rq = make_request(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate(rq)) return rc;
  bool need = false;
  for (int d = 0; d < nDim; ++d) need = need || (!(rq.opt.x_range[d] > 0.0) && extent_needed(rq, d));
  if (needExtent) *needExtent = need;
  return RF_OK;
}

int host_build_plan(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                    double fieldVar, int Nmc, int method, const rf_options* opt, const double* ext, Plan* P) {
  Request rq = make_request(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  return build_plan(rq, ext, *P);
}

// The same block layout as run_plan: stage layout, then the hi-only stages.
int host_block_layout(Plan* P, int32_t rOff, int32_t nmcBlk) {
  P->rOff = rOff;
  P->nmcBlk = nmcBlk;
  if (int rc = layout(*P)) return rc;
  lo_layout(*P);
  outer_layout(*P);
  outer_pair_layout(*P);
  table_alo_layout(*P);
  return RF_OK;
}

int32_t host_realization_block(const Plan& P) { return realization_block(P); }

}  // namespace rfb

// ================================================================== C-ABI
extern "C" {

void rf_options_init(rf_options* opt) {
  if (!opt) return;
  memset(opt, 0, sizeof(*opt));
  opt->size = sizeof(rf_options);
  opt->precision = RF_PREC_BF16;
}

const char* rf_last_error(void) { return g_err.c_str(); }

int rf_abi_version(void) { return RF_ABI_VERSION; }

int rf_query_geometry(const double* xPoints, int nDim, int64_t n, int corrMod, const double* corrL, int method,
                      const rf_options* opt, int64_t* K, int32_t* kNStep, double* kDelta, double* ampMult) {
  g_err.clear();
  if (!xPoints || !corrL) return fail(RF_EINVAL_ARG, "null pointer argument");
  Request rq = make_request(nDim, n, corrMod, RF_FOM_GAUSSIAN, corrL, 0.0, 1.0, 1, method, opt);
  if (int rc = validate(rq)) return rc;
  double ext[3] = {0, 0, 0};
  for (int d = 0; d < nDim; ++d) {
    double lo = xPoints[d], hi = xPoints[d];
    for (int64_t i = 1; i < n; ++i) {
      lo = std::min(lo, xPoints[i * nDim + d]);
      hi = std::max(hi, xPoints[i * nDim + d]);
    }
    ext[d] = hi - lo;
  }
  Plan P;
  if (int rc = geometry(rq, ext, P)) return rc;
  if (K) *K = P.K;
  for (int d = 0; d < 3; ++d) {
    if (kNStep) kNStep[d] = P.kNStep[d];
    if (kDelta) kDelta[d] = P.kDelta[d];
  }
  if (ampMult) *ampMult = P.ampMult;
  return RF_OK;
}

int rf_context_create(int device, rf_context** out) {
  g_err.clear();
  if (!out) return fail(RF_EINVAL_ARG, "null output pointer");
  *out = nullptr;
  rf_context* c = new rf_context();
  if (int rc = context_init(c, device)) {
    context_free(c);
    delete c;
    return rc;
  }
  *out = c;
  return RF_OK;
}

int rf_context_destroy(rf_context* ctx) {
  if (!ctx) return RF_OK;
  context_free(ctx);
  delete ctx;
  return RF_OK;
}

int rf_context_synchronize(rf_context* ctx) {
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  RF_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  return check_device_error(ctx);
}

int rf_context_set_timing(rf_context* ctx, int enable) {
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  ctx->timing = enable != 0;
  ctx->evValid = false;
  return RF_OK;
}

int rf_context_last_times(rf_context* ctx, double* tables_ms, double* contract_ms, double* post_ms,
                          int32_t* kernel_launches) {
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  if (kernel_launches) *kernel_launches = ctx->launches;
  if (!ctx->evValid) return fail(RF_EINVAL_ARG, "no timed generation on this context (enable timing first)");
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  RF_CUDA(cudaEventSynchronize(ctx->ev[3]), "cudaEventSynchronize");
  float a = 0, b = 0, p = 0;
  RF_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]), "cudaEventElapsedTime");
  RF_CUDA(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]), "cudaEventElapsedTime");
  RF_CUDA(cudaEventElapsedTime(&p, ctx->ev[2], ctx->ev[3]), "cudaEventElapsedTime");
  if (tables_ms) *tables_ms = a;
  if (contract_ms) *contract_ms = b;
  if (post_ms) *post_ms = p;
  return RF_OK;
}

int rf_generate_device(rf_context* ctx, const double* d_xPoints, int nDim, int64_t n, int corrMod, int margiFirst,
                       const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                       double* d_randField, const rf_options* opt, void* stream) {
  rfh::NvtxRange nvtx_("rf_generate_device");
  g_err.clear();
  if (!ctx || !d_xPoints || !corrL || !d_randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  Request rq = make_request(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate_with_draws(rq)) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
  ctx->launches = 0;
  ctx->evValid = false;
  double ext[3] = {0, 0, 0};
  bool need = false;  // the extent pass (and its host read-back) only where the geometry uses it
  for (int d = 0; d < nDim; ++d) need = need || (!(rq.opt.x_range[d] > 0.0) && extent_needed(rq, d));
  if (need)
    if (int rc = device_extent(ctx, d_xPoints, nDim, n, st, ext)) return rc;
  Plan P;
  if (int rc = build_plan(rq, ext, P)) return rc;
  if (int rc = upload_draws(ctx, rq, P, st)) return rc;
  return run_plan(ctx, P, d_xPoints, d_randField, st);
}

int rf_create_standard_gaussian_field_unstruct(const double* xPoints, int nDim, int64_t n, int corrMod,
                                               int margiFirst, const double* corrL, double fieldAvg,
                                               double fieldVar, int Nmc, int method, double* randField,
                                               const rf_options* opt) {
  rfh::NvtxRange nvtx_("rf_create_standard_gaussian_field_unstruct");
  g_err.clear();
  if (!xPoints || !corrL || !randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  Request rq = make_request(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate_with_draws(rq)) return rc;
  rf_context* c = nullptr;
  if (int rc = default_context(rq.opt.device, &c)) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  RF_CUDA(cudaSetDevice(c->device), "cudaSetDevice");
  c->launches = 0;
  c->evValid = false;
  const size_t xBytes = sizeof(double) * (size_t)nDim * (size_t)n;
  const size_t oBytes = sizeof(double) * (size_t)n * (size_t)Nmc;
  if (int rc = ensure(c->dX, c->capX, xBytes, "points")) return rc;
  if (int rc = ensure(c->dOut, c->capOut, oBytes, "field")) return rc;
  cudaStream_t st = c->stream;
  double ext[3] = {0, 0, 0};
  bool need = false;  // the extent pass (and its host read-back) only where the geometry uses it
  for (int d = 0; d < nDim; ++d) need = need || (!(rq.opt.x_range[d] > 0.0) && extent_needed(rq, d));
  bool onDevice = false;  // points copied up
  if (need) {
    RF_CUDA(cudaMemcpyAsync(c->dX, xPoints, xBytes, cudaMemcpyHostToDevice, st), "copy of xPoints");
    onDevice = true;
    if (int rc = device_extent(c, c->dX, nDim, n, st, ext)) return rc;
  }
  Plan P;
  if (int rc = build_plan(rq, ext, P)) return rc;
  if (int rc = upload_draws(c, rq, P, st)) return rc;
  // page-locked destination: copy slabs out while the next ones compute (and,
  // when the points are still on the host, copy them up slab by slab)
  cudaPointerAttributes pa;
  const bool pinned = cudaPointerGetAttributes(&pa, randField) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  if (!pinned) cudaGetLastError();
  if (pinned && !c->timing) {
    const int rc = run_plan_slabs(c, P, c->dX, c->dOut, randField, st, onDevice ? nullptr : xPoints);
    if (rc == RF_OK) return check_device_error(c);
    if (rc != RF_ENOTSUP) return rc;
    g_err.clear();
  }
  if (!onDevice) RF_CUDA(cudaMemcpyAsync(c->dX, xPoints, xBytes, cudaMemcpyHostToDevice, st), "copy of xPoints");
  if (int rc = run_plan(c, P, c->dX, c->dOut, st)) return rc;
  RF_CUDA(cudaMemcpyAsync(randField, c->dOut, oBytes, cudaMemcpyDeviceToHost, st), "copy of randField");
  RF_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return check_device_error(c);
}

}  // extern "C"
