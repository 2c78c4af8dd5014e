// rf_internal.h -- host-side internals shared by the C-ABI translation units
// (rf_host.cu: single requests; rf_batch.cu: batches and the serving loop).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/randomfield_b200.h"
#include "rf_device.cuh"
#include "rf_launch.h"
#include "rf_plan.h"

// Device state of one context: streams, reusable buffers, timing events,
// and the grouped-launch state of the batch entry points.
struct rf_context {
  int device = 0;
  int numSMs = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copyStream = nullptr;  // flat API: slab copies to the host beside the contraction
  cudaStream_t h2dStream = nullptr;   // flat API: slab copies of the points ahead of the contraction
  cudaEvent_t slabEv[16] = {};
  cudaEvent_t h2dEv[16] = {};
  std::mutex mu;
  void* dB = nullptr;
  size_t capB = 0;
  double* dKtab = nullptr;
  size_t capK = 0;
  double* dWork = nullptr;  // extent partials and moments
  size_t capWork = 0;
  double* hWork = nullptr;  // pinned mirror of dWork
  double* dFft = nullptr;   // FFT method: amplitudes, pass buffer, cosine matrices (rf_fft.cu)
  size_t capFft = 0;
  void* dGrid = nullptr;    // grid path: phasor tables, coefficients, axis-3 partial sums (rf_grid.cu)
  size_t capGrid = 0;
  double* dBlendSub = nullptr;  // grid path blend: one subdomain's field
  size_t capBlendSub = 0;
  double* dDraws = nullptr;     // the caller's uniform draws (rf_options.draws)
  size_t capDraws = 0;
  double* dStats = nullptr; // field statistics scratch (rf_stats.cu)
  size_t capStats = 0;
  double* hStats = nullptr;
  size_t capHStats = 0;
  uint32_t* dErr = nullptr;
  double* dX = nullptr;     // flat API staging of the points
  size_t capX = 0;
  double* dOut = nullptr;   // flat API result buffer
  size_t capOut = 0;
  bool timing = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool evValid = false;
  int32_t launches = 0;     // kernels launched by the last generation

  // ---- grouped launches (rf_batch.cu)
  unsigned char* dArena = nullptr;  // operands, and points/fields of host batches
  size_t capArena = 0;
  unsigned char* dDesc = nullptr;   // units, prefix, CTA slices, work items
  size_t capDesc = 0;
  size_t descCapU = 0, descCapI = 0;  // unit and item capacities of its layout
  unsigned char* hDesc = nullptr;   // pinned staging of dDesc
  size_t capHDesc = 0;
  double* dExt = nullptr;           // extent partials of device batches
  size_t capExt = 0;
  double* hExt = nullptr;
  size_t capHExt = 0;
  cudaEvent_t bev[3] = {nullptr, nullptr, nullptr};
  struct GraphKey {
    int prec, S, aCol0;
    int64_t slotBytes;
    int oS, oSlotBytes, oABytes;  // the outer-group kernel's slot layout (oS = 0: not launched)
    int hasTc;                    // the grouped tcgen05 kernel is launched
    const void* desc;
    bool operator<(const GraphKey& o) const {
      if (prec != o.prec) return prec < o.prec;
      if (S != o.S) return S < o.S;
      if (aCol0 != o.aCol0) return aCol0 < o.aCol0;
      if (slotBytes != o.slotBytes) return slotBytes < o.slotBytes;
      if (oS != o.oS) return oS < o.oS;
      if (oSlotBytes != o.oSlotBytes) return oSlotBytes < o.oSlotBytes;
      if (oABytes != o.oABytes) return oABytes < o.oABytes;
      if (hasTc != o.hasTc) return hasTc < o.hasTc;
      return desc < o.desc;
    }
  };
  std::map<GraphKey, cudaGraphExec_t> graphs;
  // The grouped launch's tuner: per (precision form, batch class) the chosen
  // realization block and pipeline depths of both grouped kernels, with the
  // report of the search that chose them.
  struct TuneChoice {
    int blk = 0, sTc = 0, sOuter = 0;  // 0: the deepest pipeline that fits
    int candidates = 0;
    double defaultMs = 0.0, bestMs = 0.0;
  };
  std::map<int, TuneChoice> tuned;
  rf_batch_stats last{};
};

namespace rfh {

extern thread_local std::string g_err;
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* where);

// NVTX range over a host entry point or phase, visible in Nsight Systems
// timelines; without a tool attached the calls return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

#define RF_CUDA(call, where)                                     \
  do {                                                           \
    cudaError_t e_ = (call);                                     \
    if (e_ != cudaSuccess) return rfh::cuda_fail(e_, where);     \
  } while (0)

struct Request {
  int nDim;
  int64_t n;
  int corrMod, margiFirst, Nmc, method;
  double corrL[3];
  double fieldAvg, fieldVar;
  rf_options opt;
};

constexpr int kExtentBlocks = 128;

const rfb::JumpTable& jump_table();
int64_t round_up(int64_t v, int64_t m);
int validate(const Request& r);
// Whether axis d's extent enters the geometry (no explicit wavenumber count).
bool extent_needed(const Request& r, int d);
int layout(rfb::Plan& P);
int build_plan(const Request& rq, const double* ext, rfb::Plan& P);
int seeds(int64_t seedStart, rfb::Plan& P);
// BF16 GEN_GRID3 plans: the stages that keep only the hi term (rf_host.cu)
void lo_layout(rfb::Plan& P);
// Single-request 3-D Shinozuka plans on the 16-bit tensor-core forms: the
// outer-group contraction (rf_outer.cu) and its lo masks (rf_host.cu)
void outer_layout(rfb::Plan& P);
// Its CTA-pair form (rf_outer_pair.cu): single requests of at least two
// items and two realizations, or every GEN_OUTER plan when `always`
void outer_pair_layout(rfb::Plan& P, bool always = false);
// Small single BF16 table-generator requests: the trig tile's lo term (rf_host.cu)
void table_alo_layout(rfb::Plan& P);
int32_t realization_block(const rfb::Plan& P);
int device_extent(rf_context* c, const double* dX, int nDim, int64_t n, cudaStream_t st, double* ext);
int run_plan(rf_context* c, const rfb::Plan& P0, const double* dX, double* dOut, cudaStream_t st);
int check_device_error(rf_context* c);
int default_context(int device, rf_context** out);
Request make_request(int nDim, int64_t n, int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                     double fieldVar, int Nmc, int method, const rf_options* opt);
void launch_extent(const double* dX, int64_t n, int nDim, double* part, cudaStream_t st);

// A request that is a subdomain of a localization blend (rf_blend.cuh);
// gTotal == 0 marks a plain request in a batch that mixes both.
struct BlendSpec {
  int32_t bDims[3], bOrigin[3], gDims[3], bRamp[3];
  int64_t gTotal;
};

// rf_batch.cu: plan and run a batch whose points and fields are in device
// memory (queued on st; returns without waiting).  With `blend`, one spec per
// request.
int batch_run_device(rf_context* c, const std::vector<Request>& rq, const std::vector<const double*>& dx,
                     const std::vector<double*>& dout, const std::vector<double>& ext, cudaStream_t st,
                     const std::vector<BlendSpec>* blend = nullptr);
// Blend requests (rf_generate_blended): bytes of the subdomain points; the
// subdomain requests (appended, points generated into dPoints, dOut
// cleared) and the group plan; the border correction and marginal map.
int blend_points_bytes(const rf_blend_grid* grid, const double* corrL, size_t* bytes);
int blend_expand(const rf_blend_grid* grid, const Request& base, double* dOut, double* dPoints, cudaStream_t st,
                 std::vector<Request>& rq, std::vector<const double*>& dx, std::vector<double*>& dout,
                 std::vector<BlendSpec>& spec, rfb::Plan* groupPlan);
int blend_finish(rf_context* c, const rfb::Plan& Gp, double* dOut, cudaStream_t st);
// Whether the structured-grid path takes the blend of `grid` (Shinozuka, at
// most the grid path's wavenumbers per axis, not literal); no device work.
bool grid_blend_ok(const rf_blend_grid* grid, const Request& base);
// The blend through the structured-grid path (rf_grid.cu): each subdomain
// summed axis by axis in FP64, weighted and added into dOut, then the border
// correction and the marginal map.  Call only where grid_blend_ok holds.
int grid_blend_run(rf_context* c, const rf_blend_grid* grid, const Request& base, double* dOut, cudaStream_t st);
// Device bytes a request holds in a batch with realization block rblk:
// points, field, operands.
int request_footprint(const Request& rq, const double* ext, int rblk, size_t* bytes);
// Realization block of the grouped launch before the tuner has run.
int default_block(int prec);
// rf_host.cu: create / free a context.
int context_init(rf_context* c, int device);
void context_free(rf_context* c);

// Grows a device buffer to at least `bytes` (contents are not kept).
template <typename T>
int ensure(T*& p, size_t& cap, size_t bytes, const char* what) {
  if (bytes <= cap && p) return RF_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RF_ENOMEM, "cannot allocate %zu bytes of device memory for %s", bytes, what);
  }
  p = reinterpret_cast<T*>(q);
  cap = bytes;
  return RF_OK;
}

// Grows a pinned host buffer to at least `bytes` (contents are not kept).
template <typename T>
int ensure_host(T*& p, size_t& cap, size_t bytes, const char* what) {
  if (bytes <= cap && p) return RF_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  void* q = nullptr;
  cudaError_t e = cudaMallocHost(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RF_ENOMEM, "cannot allocate %zu bytes of pinned host memory for %s", bytes, what);
  }
  p = reinterpret_cast<T*>(q);
  cap = bytes;
  return RF_OK;
}

}  // namespace rfh
