// rf_selftest.cu -- failure-detection self test of the bounded device waits,
// and the SFU (MUFU sin/cos) rate used by the roofline of GEN_TABLE.
//
// Every wait of the generation kernels is bounded (mbar_wait: globaltimer
// limit, abort flag); on expiry a kernel raises the context's error word,
// drains its own asynchronous work and returns, and the host reports
// RF_ETIMEDOUT.  This kernel exercises exactly that path without a fault:
// its warps wait, with the same bounded wait and a short limit, on an
// mbarrier phase that nothing completes, raise the error word when the limit
// passes and return.  The context stays usable afterwards.
#include <cuda_runtime.h>

#include <algorithm>

#include "rf_internal.h"
#include "rf_launch.h"

using namespace rfb;
using namespace rfh;

namespace {

__global__ void rf_wait_timeout_kernel(uint32_t* err, uint64_t limitNs) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival would complete phase 0; none comes
    abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();
  bool ok = true;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait_for(&bar, 0, &abort_flag, limitNs);
  ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
  if (!ok && (threadIdx.x & 31) == 0) atomicOr(err, kErrTimeout);
}

// MUFU sin/cos throughput: every thread runs 8 independent chains of
// __sincosf on arguments kept in [-pi, pi] (the reduced phases of GEN_TABLE),
// `iters` steps each; one step is one (sin, cos) pair.
__global__ void rf_sfu_rate_kernel(float* sink, int iters) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = 0.1f * (float)(threadIdx.x & 31) + 0.37f * (float)j - 1.5f;
  float acc = 0.f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float s, c;
      __sincosf(a[j], &s, &c);
      a[j] = s + c * 0.5f;  // stays in [-1.5, 1.5]
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) acc += a[j];
  if (acc == 12345.678f) sink[threadIdx.x] = acc;
}

#ifdef RF_DEBUG_BOUNDS
// One thread stores at index n of an n-element buffer through the checked
// form: the check records kErrBounds and skips the store.  Built only into
// the RF_DEBUG_BOUNDS library, where the check exists.
__global__ void rf_bounds_selftest_kernel(uint32_t* buf, int64_t n, uint32_t* err) {
  const int64_t i = n;
  if (RF_IN_BOUNDS(i, n, err)) buf[i] = 1u;
}
#endif

}  // namespace

extern "C" int rf_debug_bounds_build(void) {
#ifdef RF_DEBUG_BOUNDS
  return 1;
#else
  return 0;
#endif
}

extern "C" int rf_context_selftest_bounds(rf_context* ctx) {
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
#ifdef RF_DEBUG_BOUNDS
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  // the context's 4-byte error word doubles as the one-element buffer: the
  // kernel's index (1) is one past it
  rf_bounds_selftest_kernel<<<1, 1, 0, ctx->stream>>>(ctx->dErr, 1, ctx->dErr);
  RF_CUDA(cudaGetLastError(), "bounds self-test kernel");
  RF_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  return check_device_error(ctx);
#else
  return fail(RF_ENOTSUP, "index checks exist only in the RF_DEBUG_BOUNDS build (librf_b200_bounds.so)");
#endif
}

extern "C" int rf_measure_sfu_rate(int device, double* pairs_per_second) {
  g_err.clear();
  if (!pairs_per_second) return fail(RF_EINVAL_ARG, "null output pointer");
  RF_CUDA(cudaSetDevice(device), "cudaSetDevice");
  int sms = 0;
  RF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
  float* sink = nullptr;
  RF_CUDA(cudaMalloc(&sink, 1024 * sizeof(float)), "cudaMalloc");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4, threads = 512, iters = 4096;
  rf_sfu_rate_kernel<<<blocks, threads>>>(sink, 64);  // warm-up
  cudaEventRecord(e0);
  rf_sfu_rate_kernel<<<blocks, threads>>>(sink, iters);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_fail(e, "SFU rate kernel");
  *pairs_per_second = (double)blocks * threads * iters * 8.0 / ((double)ms * 1e-3);
  return RF_OK;
}

extern "C" int rf_context_selftest_timeout(rf_context* ctx, double limit_ms) {
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  if (!(limit_ms > 0.0) || limit_ms > 10000.0) return fail(RF_EINVAL_ARG, "limit_ms must be in (0, 10000]");
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  rf_wait_timeout_kernel<<<1, 64, 0, ctx->stream>>>(ctx->dErr, (uint64_t)(limit_ms * 1e6));
  RF_CUDA(cudaGetLastError(), "self-test kernel");
  RF_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  return check_device_error(ctx);
}

// The draws of the table builder, exported for a bit-exact check against a
// sequential rnglib run: the same runs, cursors and draw positions as the
// operand build (rf_tables.cu), realization block by realization block.
extern "C" int rf_debug_table_draws(int nDim, int method, int Nmc, const rf_options* opt, int64_t* K_out,
                                    int32_t* draws, int64_t draws_capacity, int32_t* k_draws,
                                    int64_t k_capacity) {
  g_err.clear();
  if (!K_out) return fail(RF_EINVAL_ARG, "null K_out");
  const double corrL[3] = {1.0, 1.0, 1.0};
  const Request rq = make_request(nDim, 1, RF_CM_GAUSSIAN, RF_FOM_GAUSSIAN, corrL, 0.0, 1.0, Nmc, method, opt);
  if (int rc = validate(rq)) return rc;
  const double ext[3] = {0.0, 0.0, 0.0};  // extents come from opt->x_range (or are unused with k_nstep)
  Plan P0;
  if (int rc = build_plan(rq, ext, P0)) return rc;
  *K_out = P0.K;
  if (!draws) return RF_OK;  // query of K only
  const int64_t D = method == RF_ISOTROPIC ? 2 : 1;
  const int64_t need = (int64_t)Nmc * P0.K * D;
  if (draws_capacity < need) return fail(RF_EINVAL_ARG, "draws needs Nmc * K * %d entries", (int)D);
  const bool wantK = k_draws && method == RF_ISOTROPIC;
  if (wantK && k_capacity < 2 * P0.K) return fail(RF_EINVAL_ARG, "k_draws needs 2 * K entries");
  RF_CUDA(cudaSetDevice(rq.opt.device), "cudaSetDevice");
  int32_t *dRk = nullptr, *dK = nullptr;
  RF_CUDA(cudaMalloc(&dRk, (size_t)need * sizeof(int32_t)), "cudaMalloc");
  if (wantK && cudaMalloc(&dK, (size_t)2 * P0.K * sizeof(int32_t)) != cudaSuccess) {
    cudaFree(dRk);
    return fail(RF_ENOMEM, "cudaMalloc of the direction draws failed");
  }
  cudaError_t e = cudaSuccess;
  const int32_t blk = realization_block(P0);
  for (int32_t r0 = 0; r0 < P0.Nmc && e == cudaSuccess; r0 += blk) {
    Plan P = P0;
    P.rOff = r0;
    P.nmcBlk = std::min(blk, P0.Nmc - r0);
    if (int rc = layout(P)) {
      cudaFree(dRk);
      cudaFree(dK);
      return rc;
    }
    lo_layout(P);
    outer_layout(P);  // the same plan as a generation of this request
    table_alo_layout(P);
    e = launch_table_draws(P, jump_table(), dRk, dK, 0);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(draws, dRk, (size_t)need * sizeof(int32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && wantK)
    e = cudaMemcpy(k_draws, dK, (size_t)2 * P0.K * sizeof(int32_t), cudaMemcpyDeviceToHost);
  cudaFree(dRk);
  cudaFree(dK);
  if (e != cudaSuccess) return cuda_fail(e, "table draws");
  return RF_OK;
}
