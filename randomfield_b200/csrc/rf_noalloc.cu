// rf_noalloc.cu -- generation into caller buffers with no device allocation.
//
// Who needs this: callers that must not allocate device memory at all while
// generating, e.g. an application whose allocator (a caching pool, or an
// OpenACC / CUDA Fortran runtime) owns and has reserved nearly all device
// memory, so a library cudaMalloc would fail or fragment the pool, or code on
// a latency-critical loop where cudaMalloc's implicit device synchronisation
// is unacceptable.  They pass device buffers for the points and the field;
// everything else the generation needs (the contraction operand, the
// wavevector table, the error word, extent and moment sums) lives in one
// file-scope device array of fixed size, kNoAllocScratchBytes, that the CUDA
// runtime places on every device where this library's module is loaded and
// keeps there until the process exits.
//
// Rules of use:
//   - the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (which may load the module on that device); make
//     that first call before any stream capture on the device;
//   - all calls share the one array per device: calls whose work overlaps on
//     the GPU (different streams or threads) race and corrupt each other's
//     tables; serialise them;
//   - requests whose tables exceed the array are rejected with RF_ESCRATCH;
//   - the call returns only after its work on `stream` has finished: it
//     synchronises the stream (after the extent pass when one is needed,
//     and at the end to read the device error word).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/randomfield_b200.h"
#include "rf_device.cuh"
#include "rf_launch.h"
#include "rf_plan.h"

namespace rfb {
int host_fail(int code, const char* msg);
void host_clear_error();
const JumpTable& host_jump_table();
int host_validate(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                  double fieldVar, int Nmc, int method, const rf_options* opt, bool* needExtent);
int host_build_plan(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                    double fieldVar, int Nmc, int method, const rf_options* opt, const double* ext, Plan* P);
int host_block_layout(Plan* P, int32_t rOff, int32_t nmcBlk);
int32_t host_realization_block(const Plan& P);
}  // namespace rfb

using namespace rfb;

namespace {

// Scratch layout (bytes): [0, 256) error word; [256, kExtentEnd) extent
// partials; [kExtentEnd, kMomentsEnd) normalisation sums (2 * Nmc doubles,
// Nmc <= 4096); [kMomentsEnd, kTableEnd) wavevector table; then the
// contraction operand up to the end.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
constexpr int kExtentBlocks = 128;
constexpr size_t kExtentOff = 256;
constexpr size_t kExtentEnd = kExtentOff + sizeof(double) * 6 * kExtentBlocks;
constexpr size_t kMomentsOff = (kExtentEnd + 255) / 256 * 256;
constexpr int kMaxNormNmc = 4096;
constexpr size_t kMomentsEnd = kMomentsOff + sizeof(double) * 2 * kMaxNormNmc;
constexpr size_t kTableOff = (kMomentsEnd + 255) / 256 * 256;
constexpr size_t kTableBytes = size_t(1) << 20;  // wavevector table: 3 doubles per k, up to 43690 k
constexpr size_t kOperandOff = kTableOff + kTableBytes;
constexpr size_t kOperandBytes = kNoAllocScratchBytes - kOperandOff;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char* g_scratch[64] = {nullptr};  // device address per device ordinal

// Once per device, with that device current: the device address of the
// array (the host-side name of a __device__ array is not a device address).
int scratch_for(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (device < 0 || device >= 64) return host_fail(RF_ENODEV, "device ordinal out of range");
  if (!g_scratch[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return host_fail(RF_ECUDA, "cudaGetSymbolAddress of the no-allocation scratch failed");
    }
    g_scratch[device] = reinterpret_cast<unsigned char*>(p);
  }
  *out = g_scratch[device];
  return RF_OK;
}

__global__ void rf_noalloc_extent_kernel(const double* __restrict__ x, int64_t n, int nDim,
                                         double* __restrict__ part) {
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

int cuda_err(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return RF_OK;
  cudaGetLastError();
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
  return host_fail(RF_ECUDA, buf);
}

}  // namespace

extern "C" int rf_generate_device_noalloc(const double* d_xPoints, int nDim, int64_t n, int corrMod,
                                          int margiFirst, const double* corrL, double fieldAvg, double fieldVar,
                                          int Nmc, int method, double* d_randField, const rf_options* opt,
                                          void* stream) {
  host_clear_error();
  if (!d_xPoints || !corrL || !d_randField) return host_fail(RF_EINVAL_ARG, "null pointer argument");
  bool needExtent = false;
  if (int rc = host_validate(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt,
                             &needExtent))
    return rc;
  int device = 0;
  if (int rc = cuda_err(cudaGetDevice(&device), "cudaGetDevice")) return rc;
  const int want = opt ? opt->device : 0;
  // the caller's current device is restored on every return
  struct DeviceGuard {
    int prev;
    ~DeviceGuard() { cudaSetDevice(prev); }
  } guard{device};
  if (want != device)
    if (int rc = cuda_err(cudaSetDevice(want), "cudaSetDevice")) return rc;
  device = want;
  unsigned char* scratch = nullptr;
  if (int rc = scratch_for(device, &scratch)) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int numSMs = 0;
  if (int rc = cuda_err(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device), "SM count"))
    return rc;

  uint32_t* dErr = reinterpret_cast<uint32_t*>(scratch);
  double* dExtent = reinterpret_cast<double*>(scratch + kExtentOff);
  double* dMoments = reinterpret_cast<double*>(scratch + kMomentsOff);
  double* dKtab = reinterpret_cast<double*>(scratch + kTableOff);
  void* dB = scratch + kOperandOff;

  // the error word starts at zero for every call (the array keeps the last
  // call's contents)
  if (int rc = cuda_err(cudaMemsetAsync(dErr, 0, sizeof(uint32_t), st), "clear error word")) return rc;

  double ext[3] = {0, 0, 0};
  if (needExtent) {
    double part[6 * kExtentBlocks];
    rf_noalloc_extent_kernel<<<kExtentBlocks, 256, 0, st>>>(d_xPoints, n, nDim, dExtent);
    if (int rc = cuda_err(cudaGetLastError(), "extent kernel")) return rc;
    if (int rc = cuda_err(cudaMemcpyAsync(part, dExtent, sizeof(part), cudaMemcpyDeviceToHost, st), "extent copy"))
      return rc;
    if (int rc = cuda_err(cudaStreamSynchronize(st), "extent sync")) return rc;
    for (int d = 0; d < nDim; ++d) {
      double lo = INFINITY, hi = -INFINITY;
      for (int b = 0; b < kExtentBlocks; ++b) {
        lo = std::min(lo, part[b * 6 + d]);
        hi = std::max(hi, part[b * 6 + 3 + d]);
      }
      ext[d] = hi - lo;
    }
  }
  Plan P0;
  if (int rc = host_build_plan(nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt, ext, &P0))
    return rc;
  if (P0.normalize && P0.Nmc > kMaxNormNmc)
    return host_fail(RF_ESCRATCH, "normalisation in the no-allocation path supports Nmc <= 4096");

  const int32_t blk = host_realization_block(P0);
  int64_t xSlab = P0.n, nSlab = 1;
  if (P0.literal) {
    // randomFieldND.f90:237-239
    xSlab = (int64_t)((double)P0.nDim * 1e8 / (double)P0.K);
    if (xSlab > P0.n) xSlab = P0.n;
    if (xSlab < 1) xSlab = 1;
    nSlab = (P0.n + xSlab - 1) / xSlab;
  }
  for (int32_t r0 = 0; r0 < P0.Nmc; r0 += blk) {
    Plan P = P0;
    if (int rc = host_block_layout(&P, r0, std::min(blk, P0.Nmc - r0))) return rc;
    P.dbgErr = dErr;
    const size_t opBytes = (size_t)operand_bytes(P);
    const size_t tabBytes = P.gen == GEN_TABLE ? (size_t)P.nChunks * kKtabStageBytes : 0;
    if (opBytes > kOperandBytes || tabBytes > kTableBytes) {
      char buf[256];
      snprintf(buf, sizeof(buf),
               "request needs %zu + %zu scratch bytes; the no-allocation scratch holds %zu + %zu (fewer "
               "wavevectors or realizations, or use rf_generate_device)",
               opBytes, tabBytes, kOperandBytes, kTableBytes);
      return host_fail(RF_ESCRATCH, buf);
    }
    if (P.prec != PREC_FP32 && tc_smem_bytes(P, nullptr) == 0)
      return host_fail(RF_ENOTSUP, "stage too large for shared memory");
    double* ktab = P.gen == GEN_TABLE ? dKtab : nullptr;
    for (int64_t m = 0; m < nSlab; ++m) {
      const int64_t row0 = m * xSlab;
      const int64_t rows = std::min(xSlab, P.n - row0);
      if (int rc = cuda_err(launch_tables(P, host_jump_table(), dB, ktab, P.literal ? m : -1, nSlab, st),
                            "table kernel"))
        return rc;
      cudaError_t e = P.prec == PREC_FP32 ? launch_fp32(P, d_xPoints, dB, ktab, d_randField, row0, rows, st)
                                          : launch_tc(P, d_xPoints, dB, ktab, d_randField, row0, rows, dErr,
                                                      numSMs, st);
      if (int rc = cuda_err(e, "contraction kernel")) return rc;
    }
  }
  if (P0.normalize)
    if (int rc = cuda_err(launch_normalize_and_map(P0, d_randField, P0.literal ? 1 : P0.Nmc, dMoments, st),
                          "normalisation kernels"))
      return rc;
  uint32_t err = 0;
  if (int rc = cuda_err(cudaMemcpyAsync(&err, dErr, sizeof(err), cudaMemcpyDeviceToHost, st), "error word"))
    return rc;
  if (int rc = cuda_err(cudaStreamSynchronize(st), "cudaStreamSynchronize")) return rc;
  if (err) return host_fail(RF_ETIMEDOUT, "a bounded device wait expired; results are invalid");
  return RF_OK;
}
