// rf_post.cu -- optional empirical normalisation (normalize_randField,
// randomFieldND.f90:820-926) followed by the marginal map
// (multiVariateTransformation, :139-178).  Used only when the caller asks
// for normalisation; otherwise the map is fused into the contraction
// epilogue.  Sums are FP64: column mean, then the mean square of the
// centred column, exactly the two reductions of the reference.
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

}  // namespace

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
