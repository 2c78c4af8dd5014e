// rf_serve.cu -- the serving loop: continuous batching of generation
// requests over two grouped-launch slots with HBM-footprint admission.
//
// Submitting threads validate and plan a request (its device footprint:
// points, field, operands) and queue it.  One worker thread owns two slots,
// each an rf_context with its own stream, device buffers and pinned staging.
// While one slot's batch runs on the GPU the worker admits the queued
// requests into the other slot (FIFO, while the slot's share of the budget
// holds them) and queues that batch behind it, so arrivals wait at most for
// the batch in flight; when a slot's completion event fires the worker copies
// the fields out of staging into the callers' buffers and wakes the waiters.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rf_internal.h"

using namespace rfb;
using namespace rfh;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

struct Pending {
  int64_t ticket;
  rf_request req;  // the caller's request (its buffers stay valid until the wait returns)
  Request rq;      // validated copy
  double ext[3];
  size_t bytes;    // device footprint in a batch
  double tSubmit;
  bool blended = false;  // a localization blend on `grid` (rq.n unused; the field has gPoints points)
  rf_blend_grid grid;
  int64_t gPoints = 0;
  size_t pointBytes = 0;  // subdomain points of a blend
  // the number of field values and the input bytes the request moves
  int64_t fieldPoints() const { return blended ? gPoints : rq.n; }
};

struct Result {
  bool done = false;
  int status = RF_OK;
  double latency_ms = 0.0;
  std::string error;
};

struct Slot {
  rf_context* ctx = nullptr;
  cudaEvent_t evDone = nullptr;
  bool busy = false;
  std::vector<Pending> batch;
  unsigned char* hStage = nullptr;  // pinned: points then fields of the batch
  size_t capStage = 0;
  std::vector<size_t> outOff;       // field offsets inside hStage (SIZE_MAX: copied straight to the caller)
  int status = RF_OK;
  std::string error;
};

}  // namespace

struct rf_server {
  rf_server_config cfg{};
  size_t slotBudget = 0;
  std::mutex mu;
  std::condition_variable cvWork, cvDone;
  std::deque<Pending> queue;
  std::unordered_map<int64_t, Result> results;
  int64_t nextTicket = 1;
  bool stop = false;
  std::thread worker;
  Slot slots[2];
  int block = 64;  // realization block used for footprints
  // statistics (under mu)
  rf_server_stats st{};
  std::vector<double> latencies;
};

namespace {

// Launches the slot's batch: points into staging and onto the device, the
// grouped generation, fields back into staging, completion event.
bool pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int launch_slot(rf_server* s, Slot& sl) {
  rfh::NvtxRange nvtx_("serving batch launch");
  rf_context* c = sl.ctx;
  cudaStream_t st = c->stream;
  RF_CUDA(cudaSetDevice(c->device), "cudaSetDevice");
  const size_t n = sl.batch.size();
  size_t stage = 0, io = 0;
  // callers' page-locked buffers are copied to and from directly; pageable
  // ones go through the slot's pinned staging
  std::vector<char> pinX(n), pinO(n);
  for (size_t i = 0; i < n; ++i) {
    const Pending& p = sl.batch[i];
    const size_t ob = sizeof(double) * (size_t)p.fieldPoints() * p.rq.Nmc;
    const size_t xb = p.blended ? p.pointBytes : sizeof(double) * (size_t)p.rq.n * p.rq.nDim;
    pinX[i] = p.blended ? 1 : pinned(p.req.xPoints);
    pinO[i] = pinned(p.req.randField);
    stage += (pinX[i] ? 0 : align_up(xb)) + (pinO[i] ? 0 : align_up(ob));
    io += align_up(xb) + align_up(ob);
  }
  if (stage > 0)
    if (int rc = ensure_host(sl.hStage, sl.capStage, stage, "serving staging")) return rc;
  if (int rc = ensure(c->dX, c->capX, io, "serving points and fields")) return rc;
  std::vector<Request> rq;
  std::vector<const double*> dx;
  std::vector<double*> dout, fieldOut(n);
  std::vector<double> ext;
  std::vector<BlendSpec> spec;
  std::vector<std::pair<size_t, Plan>> groups;  // blended requests in the grouped launch: index, group plan
  std::vector<size_t> gridBlends;               // blended requests through the structured-grid path
  sl.outOff.assign(n, 0);
  unsigned char* dbase = reinterpret_cast<unsigned char*>(c->dX);
  size_t off = 0, soff = 0;
  for (size_t i = 0; i < n; ++i) {
    const Pending& p = sl.batch[i];
    const size_t ob = sizeof(double) * (size_t)p.fieldPoints() * p.rq.Nmc;
    double* pts = reinterpret_cast<double*>(dbase + off);
    off += align_up(p.blended ? p.pointBytes : sizeof(double) * (size_t)p.rq.n * p.rq.nDim);
    double* fld = reinterpret_cast<double*>(dbase + off);
    off += align_up(ob);
    fieldOut[i] = fld;
    if (pinO[i]) {
      sl.outOff[i] = SIZE_MAX;
    } else {
      sl.outOff[i] = soff;
      soff += align_up(ob);
    }
    if (p.blended && grid_blend_ok(&p.grid, p.rq)) {
      gridBlends.push_back(i);
      continue;
    }
    if (p.blended) {
      Plan Gp;
      if (int rc = blend_expand(&p.grid, p.rq, fld, pts, st, rq, dx, dout, spec, &Gp)) return rc;
      while (ext.size() < 3 * rq.size()) ext.push_back(0.0);
      groups.push_back({i, Gp});
      continue;
    }
    const size_t xb = sizeof(double) * (size_t)p.rq.n * p.rq.nDim;
    const void* src = p.req.xPoints;
    if (!pinX[i]) {
      memcpy(sl.hStage + soff, p.req.xPoints, xb);
      src = sl.hStage + soff;
      soff += align_up(xb);
    }
    RF_CUDA(cudaMemcpyAsync(pts, src, xb, cudaMemcpyHostToDevice, st), "copy of xPoints");
    rq.push_back(p.rq);
    dx.push_back(pts);
    dout.push_back(fld);
    for (int d = 0; d < 3; ++d) ext.push_back(p.ext[d]);
    BlendSpec none;
    memset(&none, 0, sizeof(none));
    spec.push_back(none);
  }
  if (!rq.empty())
    if (int rc = batch_run_device(c, rq, dx, dout, ext, st, groups.empty() ? nullptr : &spec)) return rc;
  for (auto& g : groups)
    if (int rc = blend_finish(c, g.second, fieldOut[g.first], st)) return rc;
  for (size_t i : gridBlends)
    if (int rc = grid_blend_run(c, &sl.batch[i].grid, sl.batch[i].rq, fieldOut[i], st)) return rc;
  for (size_t i = 0; i < n; ++i) {
    const Pending& p = sl.batch[i];
    const size_t ob = sizeof(double) * (size_t)p.fieldPoints() * p.rq.Nmc;
    void* dst = sl.outOff[i] == SIZE_MAX ? (void*)p.req.randField : (void*)(sl.hStage + sl.outOff[i]);
    RF_CUDA(cudaMemcpyAsync(dst, fieldOut[i], ob, cudaMemcpyDeviceToHost, st), "copy of randField");
  }
  RF_CUDA(cudaEventRecord(sl.evDone, st), "cudaEventRecord");
  (void)s;
  return RF_OK;
}

// The slot's batch is complete (or failed): fields to the callers, results.
void finish_slot(rf_server* s, Slot& sl) {
  int status = sl.status;
  double busy = 0.0;
  if (status == RF_OK) {
    cudaSetDevice(sl.ctx->device);
    if (cudaEventSynchronize(sl.evDone) != cudaSuccess) status = cuda_fail(cudaGetLastError(), "serving batch");
    if (status == RF_OK) status = check_device_error(sl.ctx);
    if (status == RF_OK) {
      float a = 0, b = 0;
      if (cudaEventElapsedTime(&a, sl.ctx->bev[0], sl.ctx->bev[1]) == cudaSuccess &&
          cudaEventElapsedTime(&b, sl.ctx->bev[1], sl.ctx->bev[2]) == cudaSuccess)
        busy = a + b;
      for (size_t i = 0; i < sl.batch.size(); ++i) {
        const Pending& p = sl.batch[i];
        if (sl.outOff[i] != SIZE_MAX)
          memcpy(p.req.randField, sl.hStage + sl.outOff[i], sizeof(double) * (size_t)p.fieldPoints() * p.rq.Nmc);
      }
    }
  }
  const double t = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (const Pending& p : sl.batch) {
      Result& r = s->results[p.ticket];
      r.done = true;
      r.status = status;
      r.latency_ms = (t - p.tSubmit) * 1e3;
      if (status != RF_OK) r.error = sl.error.empty() ? g_err : sl.error;
      if (status == RF_OK) {
        s->st.completed += 1;
        s->st.field_values += (double)p.fieldPoints() * (double)p.rq.Nmc;
        s->latencies.push_back(r.latency_ms);
      } else {
        s->st.failed += 1;
      }
    }
    s->st.busy_ms += busy;
  }
  sl.batch.clear();
  sl.busy = false;
  sl.status = RF_OK;
  sl.error.clear();
  s->cvDone.notify_all();
}

void worker_main(rf_server* s) {
  cudaSetDevice(s->cfg.device);
  int turn = 0;
  for (;;) {
    for (Slot& sl : s->slots)
      if (sl.busy && cudaEventQuery(sl.evDone) != cudaErrorNotReady) finish_slot(s, sl);
    Slot* freeSlot = nullptr;
    for (int k = 0; k < 2 && !freeSlot; ++k)
      if (!s->slots[(turn + k) & 1].busy) freeSlot = &s->slots[(turn + k) & 1];
    if (!freeSlot) {
      // both slots in flight: wait for the older one
      Slot& old = s->slots[turn];
      cudaEventSynchronize(old.evDone);
      finish_slot(s, old);
      continue;
    }
    std::vector<Pending> batch;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->queue.empty()) {
        const bool anyBusy = s->slots[0].busy || s->slots[1].busy;
        if (s->stop && !anyBusy) break;
        if (anyBusy) s->cvWork.wait_for(lk, std::chrono::microseconds(200));
        else s->cvWork.wait(lk, [&] { return s->stop || !s->queue.empty(); });
        continue;
      }
      size_t bytes = 0;
      while (!s->queue.empty() && (int)batch.size() < s->cfg.max_batch) {
        Pending& p = s->queue.front();
        if (p.bytes > s->slotBudget) {  // can never fit: reject
          Result& r = s->results[p.ticket];
          r.done = true;
          r.status = RF_ENOMEM_ADMISSION;
          r.error = "request footprint larger than a batch slot's share of the HBM budget";
          s->st.failed += 1;
          s->queue.pop_front();
          s->cvDone.notify_all();
          continue;
        }
        if (bytes + p.bytes > s->slotBudget) {
          s->st.admission_waits += 1;
          break;
        }
        bytes += p.bytes;
        batch.push_back(std::move(p));
        s->queue.pop_front();
      }
      if (batch.empty()) continue;
      s->st.batches += 1;
      s->st.peak_bytes = std::max<int64_t>(s->st.peak_bytes, (int64_t)bytes);
    }
    freeSlot->batch = std::move(batch);
    freeSlot->busy = true;
    if (int rc = launch_slot(s, *freeSlot)) {
      freeSlot->status = rc;
      freeSlot->error = g_err;
      cudaStreamSynchronize(freeSlot->ctx->stream);
      finish_slot(s, *freeSlot);
    }
    turn = (int)(freeSlot - s->slots) ^ 1;
  }
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

void free_server(rf_server* s) {
  for (Slot& sl : s->slots) {
    if (sl.ctx) {
      context_free(sl.ctx);
      delete sl.ctx;
    }
    if (sl.evDone) cudaEventDestroy(sl.evDone);
    if (sl.hStage) cudaFreeHost(sl.hStage);
  }
  delete s;
}

}  // namespace

extern "C" {

void rf_server_config_init(rf_server_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->size = sizeof(rf_server_config);
  cfg->precision = RF_PREC_BF16;
  cfg->max_batch = 512;
}

int rf_server_create(const rf_server_config* cfg, rf_server** out) {
  g_err.clear();
  if (!out) return fail(RF_EINVAL_ARG, "null output pointer");
  *out = nullptr;
  rf_server* s = new rf_server();
  rf_server_config_init(&s->cfg);
  if (cfg) {
    const size_t sz = (cfg->size > 0 && (size_t)cfg->size < sizeof(rf_server_config)) ? (size_t)cfg->size
                                                                                      : sizeof(rf_server_config);
    memcpy(&s->cfg, cfg, sz);
    s->cfg.size = sizeof(rf_server_config);
  }
  if (s->cfg.max_batch <= 0) s->cfg.max_batch = 512;
  if (s->cfg.precision == RF_PREC_FP32 || s->cfg.precision < RF_PREC_BF16 || s->cfg.precision > RF_PREC_FP8) {
    delete s;
    return fail(RF_EINVAL_ARG, "the serving loop runs the tensor-core forms (BF16, FP16, BF16 fast)");
  }
  for (Slot& sl : s->slots) {
    sl.ctx = new rf_context();
    if (int rc = context_init(sl.ctx, s->cfg.device)) {
      free_server(s);
      return rc;
    }
    if (cudaEventCreateWithFlags(&sl.evDone, cudaEventDisableTiming) != cudaSuccess) {
      free_server(s);
      return fail(RF_ECUDA, "cudaEventCreate");
    }
  }
  if (s->cfg.hbm_budget_bytes <= 0) {
    size_t freeB = 0, total = 0;
    cudaMemGetInfo(&freeB, &total);
    s->cfg.hbm_budget_bytes = (int64_t)(freeB / 2);
  }
  s->slotBudget = (size_t)s->cfg.hbm_budget_bytes / 2;
  s->block = default_block(s->cfg.precision);
  s->worker = std::thread(worker_main, s);
  *out = s;
  return RF_OK;
}

int rf_server_submit(rf_server* s, const rf_request* req, int64_t* ticket) {
  const double tEnter = now_s();  // latency counts the caller's whole wait, validation included
  g_err.clear();
  if (!s || !req || !ticket) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (!req->xPoints || !req->randField) return fail(RF_EINVAL_ARG, "null request buffer");
  Pending p;
  p.req = *req;
  p.rq = make_request(req->nDim, req->n, req->corrMod, req->margiFirst, req->corrL, req->fieldAvg, req->fieldVar,
                      req->Nmc, req->method, &req->opt);
  p.rq.opt.precision = s->cfg.precision;
  p.rq.opt.device = s->cfg.device;
  if (int rc = validate(p.rq)) return rc;
  if (p.rq.opt.literal) return fail(RF_ENOTSUP, "literal mode is not available in the serving loop");
  for (int d = 0; d < 3; ++d) p.ext[d] = 0.0;
  for (int d = 0; d < p.rq.nDim; ++d) {
    if (p.rq.opt.x_range[d] > 0.0 || !extent_needed(p.rq, d)) continue;  // no pass over the points
    double lo = req->xPoints[d], hi = req->xPoints[d];
    for (int64_t k = 1; k < req->n; ++k) {
      lo = std::min(lo, req->xPoints[k * req->nDim + d]);
      hi = std::max(hi, req->xPoints[k * req->nDim + d]);
    }
    p.ext[d] = hi - lo;
  }
  if (int rc = request_footprint(p.rq, p.ext, s->block, &p.bytes)) return rc;
  p.tSubmit = tEnter;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(RF_EINVAL_ARG, "the server is stopping");
    p.ticket = s->nextTicket++;
    *ticket = p.ticket;
    s->results[p.ticket] = Result{};
    s->st.submitted += 1;
    s->queue.push_back(std::move(p));
  }
  s->cvWork.notify_one();
  return RF_OK;
}

int rf_server_submit_blended(rf_server* s, const rf_blend_grid* grid, int corrMod, int margiFirst,
                             const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                             double* randField, const rf_options* opt, int64_t* ticket) {
  const double tEnter = now_s();
  g_err.clear();
  if (!s || !grid || !corrL || !randField || !ticket) return fail(RF_EINVAL_ARG, "null pointer argument");
  Pending p;
  memset(&p.req, 0, sizeof(p.req));
  p.req.randField = randField;
  p.rq = make_request(grid->nDim, 1, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  p.rq.opt.precision = s->cfg.precision;
  p.rq.opt.device = s->cfg.device;
  if (int rc = validate(p.rq)) return rc;
  if (p.rq.opt.literal) return fail(RF_ENOTSUP, "literal mode is not available in the serving loop");
  p.blended = true;
  p.grid = *grid;
  if (int rc = blend_points_bytes(grid, p.rq.corrL, &p.pointBytes)) return rc;
  p.gPoints = 1;
  for (int d = 0; d < grid->nDim; ++d) p.gPoints *= grid->xNStep[d];
  // footprint: points, group field, the operands of every subdomain
  int32_t L[3], O[3];
  if (int rc = rf_blend_layout(grid, p.rq.corrL, L, O)) return rc;
  Request sub = p.rq;
  sub.n = (int64_t)L[0] * L[1] * L[2];
  for (int d = 0; d < grid->nDim; ++d) sub.opt.x_range[d] = (double)(L[d] - 1) * grid->xStep[d];
  size_t subBytes = 0;
  const double zero[3] = {0, 0, 0};
  if (int rc = request_footprint(sub, zero, s->block, &subBytes)) return rc;
  int nSub = 1;
  for (int d = 0; d < grid->nDim; ++d) nSub *= grid->nFields[d];
  const size_t subIO = sizeof(double) * (size_t)sub.n * (sub.nDim + sub.Nmc);
  p.bytes = p.pointBytes + sizeof(double) * (size_t)p.gPoints * Nmc + (size_t)nSub * (subBytes > subIO ? subBytes - subIO : 0);
  for (int d = 0; d < 3; ++d) p.ext[d] = 0.0;
  p.tSubmit = tEnter;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(RF_EINVAL_ARG, "the server is stopping");
    p.ticket = s->nextTicket++;
    *ticket = p.ticket;
    s->results[p.ticket] = Result{};
    s->st.submitted += 1;
    s->queue.push_back(std::move(p));
  }
  s->cvWork.notify_one();
  return RF_OK;
}

int rf_server_wait(rf_server* s, int64_t ticket, double timeout_s, double* latency_ms) {
  g_err.clear();
  if (!s) return fail(RF_EINVAL_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->results.find(ticket);
  if (it == s->results.end()) return fail(RF_EINVAL_ARG, "unknown ticket %lld", (long long)ticket);
  auto ready = [&] { return s->results[ticket].done; };
  if (timeout_s < 0) {
    s->cvDone.wait(lk, ready);
  } else if (!s->cvDone.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return fail(RF_ETIMEDOUT, "request %lld not finished within %.3f s", (long long)ticket, timeout_s);
  }
  const Result r = s->results[ticket];
  s->results.erase(ticket);
  if (latency_ms) *latency_ms = r.latency_ms;
  if (r.status != RF_OK) return fail(r.status, "request %lld: %s", (long long)ticket, r.error.c_str());
  return RF_OK;
}

int rf_server_get_stats(rf_server* s, rf_server_stats* out) {
  g_err.clear();
  if (!s || !out) return fail(RF_EINVAL_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->p50_ms = percentile(s->latencies, 0.50);
  out->p99_ms = percentile(s->latencies, 0.99);
  out->max_ms = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
  double sum = 0.0;
  for (double v : s->latencies) sum += v;
  out->mean_ms = s->latencies.empty() ? 0.0 : sum / (double)s->latencies.size();
  return RF_OK;
}

int rf_server_destroy(rf_server* s) {
  if (!s) return RF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cvWork.notify_all();
  if (s->worker.joinable()) s->worker.join();
  free_server(s);
  return RF_OK;
}

}  // extern "C"
