// rf_post.cu -- optional empirical normalisation (normalize_randField,
// randomFieldND.f90:820-926) followed by the marginal map
// (multiVariateTransformation, :139-178).  Used only when the caller asks
// for normalisation; otherwise the map is fused into the contraction
// epilogue.  Sums are FP64: column mean, then the mean square of the
// centred column, exactly the two reductions of the reference.
#include <algorithm>

#include "rf_blend.cuh"
#include "rf_device.cuh"
#include "rf_launch.h"

namespace rfb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < kThreads / 32) t = red[threadIdx.x];
  if (w == 0)
    for (int o = 4; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

// pass 0: sum of the column; pass 1: sum of squares about `mean`.
__global__ void rf_colsum_kernel(const double* __restrict__ f, int64_t n, const double* __restrict__ mean,
                                 double* __restrict__ acc) {
  const int col = blockIdx.y;
  const double* c = f + (int64_t)col * n;
  const double m = mean ? mean[col] / (double)n : 0.0;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double v = c[i] - m;
    s += mean ? v * v : v;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) atomicAdd(&acc[col], s);
}

__global__ void rf_apply_kernel(double* __restrict__ f, int64_t n, int32_t ncols, const double* __restrict__ sum,
                                const double* __restrict__ sq, const Plan P) {
  const int col = blockIdx.y;
  double* c = f + (int64_t)col * n;
  const bool norm = col < ncols;
  const double m = norm ? sum[col] / (double)n : 0.0;
  const double sd = norm ? sqrt(sq[col] / (double)n) : 1.0;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    double v = c[i];
    if (norm) v = (v - m) / sd;
    v = v * P.margSd + P.margAvg;
    if (P.lognormal) v = exp(v);
    c[i] = v;
  }
}

// One subdomain's field (bDims points, axis 1 fastest, x Nmc, column-major)
// times its partition-of-unity weights, added into the group field
// (add_RF_to_Group, localization_RF.f90:199-263).  The subdomains of a group
// are added one launch after another on one stream, so plain read-modify-
// writes suffice and the sum is deterministic.
__global__ void rf_blend_add_kernel(const double* __restrict__ sub, double* __restrict__ group, const Plan P,
                                    int64_t subPoints, int32_t Nmc) {
  const int64_t total = subPoints * Nmc;
  for (int64_t t = (int64_t)blockIdx.x * kThreads + threadIdx.x; t < total; t += (int64_t)gridDim.x * kThreads) {
    const int64_t r = t / subPoints, p = t % subPoints;
    int64_t g = 0;
    const double w = blend_weight(P, p, &g);
    if (RF_IN_BOUNDS(g, P.gTotal, P.dbgErr)) group[r * P.gTotal + g] += w * sub[t];
  }
}

// Border correction of a blended group field (calls_RF.f90:324-369): a
// group without neighbours divides by its partition of unity built with
// `reverse`, i.e. the ramps of every outer face (the subdomains ramped their
// faces on the group border too); then the marginal map unless a
// normalisation pass follows.  P describes the group: gDims, bRamp, nDim.
__global__ void rf_blend_finish_kernel(double* __restrict__ f, const Plan P, int32_t applyMarginal) {
  const int col = blockIdx.y;
  double* c = f + (int64_t)col * P.gTotal;
  for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < P.gTotal; g += (int64_t)gridDim.x * kThreads) {
    const int32_t i1 = (int32_t)(g % P.gDims[0]);
    const int64_t t = g / P.gDims[0];
    const int32_t i2 = (int32_t)(t % P.gDims[1]), i3 = (int32_t)(t / P.gDims[1]);
    double w = blend_ramp(i1, P.gDims[0], P.bRamp[0]);
    if (P.nDim > 1) w = w * blend_ramp(i2, P.gDims[1], P.bRamp[1]);
    if (P.nDim > 2) w = w * blend_ramp(i3, P.gDims[2], P.bRamp[2]);
    double v = c[g] / w;
    if (applyMarginal) {
      v = v * P.margSd + P.margAvg;
      if (P.lognormal) v = exp(v);
    }
    c[g] = v;
  }
}

// Grid points of a box: x_d = x0_d + i_d * h_d, axis 1 fastest (setGrid,
// math_RF.f90:16-92), point-major (the coordinates of a point contiguous).
__global__ void rf_grid_points_kernel(double* __restrict__ x, int32_t nDim, int32_t L0, int32_t L1, int32_t L2,
                                      double x0, double x1, double x2, double h0, double h1, double h2) {
  const int64_t total = (int64_t)L0 * L1 * L2;
  for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < total; p += (int64_t)gridDim.x * kThreads) {
    const int32_t i0 = (int32_t)(p % L0);
    const int64_t t = p / L0;
    const int32_t i1 = (int32_t)(t % L1), i2 = (int32_t)(t / L1);
    x[p * nDim] = x0 + (double)i0 * h0;
    if (nDim > 1) x[p * nDim + 1] = x1 + (double)i1 * h1;
    if (nDim > 2) x[p * nDim + 2] = x2 + (double)i2 * h2;
  }
}

}  // namespace

cudaError_t launch_grid_points(double* dX, int32_t nDim, const int32_t* L, const double* x0, const double* h,
                               cudaStream_t st) {
  const int64_t total = (int64_t)L[0] * L[1] * L[2];
  const int64_t want = (total + kThreads - 1) / kThreads;
  const unsigned bx = (unsigned)(want < 1184 ? want : 1184);
  rf_grid_points_kernel<<<bx, kThreads, 0, st>>>(dX, nDim, L[0], L[1], L[2], x0[0], x0[1], x0[2], h[0], h[1], h[2]);
  return cudaGetLastError();
}

cudaError_t launch_blend_finish(const Plan& G, double* dOut, int32_t applyMarginal, cudaStream_t st) {
  const int64_t want = (G.gTotal + kThreads - 1) / kThreads;
  const unsigned bx = (unsigned)(want < 296 ? want : 296);
  rf_blend_finish_kernel<<<dim3(bx, G.Nmc), kThreads, 0, st>>>(dOut, G, applyMarginal);
  return cudaGetLastError();
}

cudaError_t launch_blend_add(const Plan& P, const double* dSub, double* dGroup, int64_t subPoints, int32_t Nmc,
                             cudaStream_t st) {
  const int64_t total = subPoints * Nmc;
  const int blocks = (int)std::min<int64_t>((total + kThreads - 1) / kThreads, 4096);
  rf_blend_add_kernel<<<blocks, kThreads, 0, st>>>(dSub, dGroup, P, subPoints, Nmc);
  return cudaGetLastError();
}

cudaError_t launch_normalize_and_map(const Plan& P, double* dOut, int32_t ncols, double* dWork, cudaStream_t st) {
  double* sum = dWork;
  double* sq = dWork + P.Nmc;
  cudaError_t e = cudaMemsetAsync(dWork, 0, sizeof(double) * 2 * P.Nmc, st);
  if (e != cudaSuccess) return e;
  const int64_t want = (P.n + kThreads - 1) / kThreads;
  const unsigned bx = (unsigned)(want < 296 ? want : 296);
  if (ncols > 0) {
    rf_colsum_kernel<<<dim3(bx, ncols), kThreads, 0, st>>>(dOut, P.n, nullptr, sum);
    rf_colsum_kernel<<<dim3(bx, ncols), kThreads, 0, st>>>(dOut, P.n, sum, sq);
  }
  rf_apply_kernel<<<dim3(bx, P.Nmc), kThreads, 0, st>>>(dOut, P.n, ncols, sum, sq, P);
  return cudaGetLastError();
}

}  // namespace rfb
