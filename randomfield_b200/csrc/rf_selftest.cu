// rf_selftest.cu -- failure-detection self test of the bounded device waits.
//
// Every wait of the generation kernels is bounded (mbar_wait: globaltimer
// limit, abort flag); on expiry a kernel raises the context's error word,
// drains its own asynchronous work and returns, and the host reports
// RF_ETIMEDOUT.  This kernel exercises exactly that path without a fault:
// its warps wait, with the same bounded wait and a short limit, on an
// mbarrier phase that nothing completes, raise the error word when the limit
// passes and return.  The context stays usable afterwards.
#include <cuda_runtime.h>

#include "rf_internal.h"

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

}  // namespace

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
