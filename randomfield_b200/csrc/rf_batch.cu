// rf_batch.cu -- batches: many independent requests in one grouped launch.
//
// Each request (the arguments of createStandardGaussianFieldUnstruct,
// README.md:58-92) is planned exactly as a single call (validation, geometry,
// seeds: rf_host.cu) and split into realization blocks ("units").  Every
// unit's 128-point tiles become work items; a longest-processing-time-first
// assignment spreads the items over one persistent CTA per SM, and two
// kernels run the batch: the grouped table builder and the grouped tcgen05
// contraction (rf_tc.cu, rf_group_kernel), which picks the generator per tile
// (GEN_GRID3 for 3-D Shinozuka grids of 24 wavenumbers on the last axis after
// padding, GEN_TABLE otherwise).  Both kernels read every per-batch quantity
// from one descriptor buffer in device memory, so the pair is captured once
// as a CUDA graph per layout and replayed for every later batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <queue>
#include <utility>
#include <vector>

#include "rf_internal.h"

using namespace rfb;
using namespace rfh;

namespace {

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Relative device cost of one stage by generator (cycles per stage measured
// on the 128^3 Shinozuka workload and the 200k-point isotropic config); only
// the ratio matters, for the balance of the CTAs.
double stage_cost(const Plan& P) {
  const double n = (double)P.bRows / 128.0;
  return P.gen == GEN_GRID3 ? 1130.0 * std::max(0.6, n) : 600.0 * std::max(0.6, n);
}

// Relative device cost of one 256-point item of a GEN_OUTER unit on a CTA
// pair: its ring stages, one chunk after another.  The pair kernel's stage
// loop costs about the same per stage whatever the stage holds and however
// many realization columns a chunk carries (the generators write the same A
// and the bulk copy lands at the same pace), so a unit's width does not enter;
// one stage more per chunk stands for the epilogue between chunks.
double outer_pair_cost(const Plan& P) {
  const double stages = (double)mask_rank(P.oStageEnd, P.oNK) + (outer_stage_end(P, P.oNK - 1) ? 0.0 : 1.0);
  return (double)P.oNR * (stages + 1.0);
}

// Descriptor buffer: unit count, units, table prefix, then for each of the
// two grouped kernels (tcgen05 contraction; outer-group contraction) its CTA
// slices and work items.
struct DescLayout {
  size_t subs, prefix, stab, nst, cta, items, octa, oitems, total;
  size_t capUnits, capItems;
};

DescLayout desc_layout(size_t capUnits, size_t capItems, int numSMs) {
  DescLayout d;
  d.capUnits = capUnits;
  d.capItems = capItems;
  d.subs = kAlign;  // header: the unit count
  d.prefix = d.subs + align_up(capUnits * sizeof(GroupSub));
  d.stab = d.prefix + align_up((capUnits + 1) * sizeof(int64_t));  // outer-group units' stage tables
  d.nst = d.stab + align_up(capUnits * kOuterMaxKsteps * sizeof(uint32_t));
  d.cta = d.nst + align_up(capUnits * sizeof(int32_t));
  d.items = d.cta + align_up((size_t)(numSMs + 1) * sizeof(int32_t));
  d.octa = d.items + align_up(capItems * sizeof(GroupItem));
  d.oitems = d.octa + align_up((size_t)(numSMs + 1) * sizeof(int32_t));
  d.total = d.oitems + align_up(capItems * sizeof(GroupItem));
  return d;
}

// Longest-processing-time-first assignment of the work items of `units`
// (`count[u]` items of cost `cost[u]` each) to nCta CTAs.
std::vector<std::vector<GroupItem>> lpt_schedule(const std::vector<size_t>& units, const std::vector<int64_t>& count,
                                                 const std::vector<double>& cost, int nCta) {
  std::vector<size_t> order = units;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
  using Load = std::pair<double, int>;
  std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
  for (int b = 0; b < nCta; ++b) heap.push({0.0, b});
  std::vector<std::vector<GroupItem>> perCta(nCta);
  for (size_t u : order) {
    for (int64_t t = 0; t < count[u]; ++t) {
      Load l = heap.top();
      heap.pop();
      perCta[l.second].push_back(GroupItem{(int32_t)u, (int32_t)t});
      l.first += cost[u];
      heap.push(l);
    }
  }
  return perCta;
}

// Writes CTA slices and items of one kernel into the staging buffer; returns the item count.
int64_t put_schedule(const std::vector<std::vector<GroupItem>>& perCta, int32_t* cta, GroupItem* it) {
  int32_t pos = 0;
  for (size_t b = 0; b < perCta.size(); ++b) {
    cta[b] = pos;
    memcpy(it + pos, perCta[b].data(), perCta[b].size() * sizeof(GroupItem));
    pos += (int32_t)perCta[b].size();
  }
  cta[perCta.size()] = pos;
  return pos;
}

struct BatchState {
  std::vector<Plan> plans;         // per request, before the realization split
  std::vector<const double*> dx;   // device points per request
  std::vector<double*> dout;       // device fields per request (the group field for blend subdomains)
  std::vector<BlendSpec> blend;    // empty, or one per request
  bool accumulate = false;         // the launch adds into its outputs: run it once (no tuning runs)
};

void apply_blend(Plan& P, const BlendSpec& b) {
  P.blend = 1;
  for (int d = 0; d < 3; ++d) {
    P.bDims[d] = b.bDims[d];
    P.bOrigin[d] = b.bOrigin[d];
    P.gDims[d] = b.gDims[d];
    P.bRamp[d] = b.bRamp[d];
  }
  P.gTotal = b.gTotal;
  P.applyMarginal = 0;  // the marginal map follows the border correction
}

struct GroupRun {
  int prec = 0;
  int rblk = 0;
  SlotLayout L{};
  size_t smem = 0;
  OuterPairGroupArgs og{};  // slot layout of the outer-group kernel (CTA pairs)
  size_t osmem = 0;
  int64_t units = 0, items = 0;
  bool replayed = false;
};

// Realization-block candidates of the tuner: the MMA N of a unit is
// 2*block (BF16 hi/lo) or block; more columns amortise the trig tile over
// more realizations, fewer waste less on requests with small Nmc.
std::vector<int> block_candidates(int prec) {
  if (prec_hilo(prec)) return {64, 32};
  return {128, 64};
}

int destroy_graphs(rf_context* c) {
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  return RF_OK;
}

// Builds the units, operands, schedule and descriptors of one grouped run
// with realization block `rblk`, and launches it (graph replay when one is
// cached for the layout).  Timing events bev[0..2] bracket the two kernels.
int group_run(rf_context* c, const BatchState& B, int prec, int rblk, int sTc, int sOuter, cudaStream_t st,
              GroupRun& run) {
  run.prec = prec;
  run.rblk = rblk;
  // ---- units
  std::vector<GroupSub> subs;
  std::vector<int64_t> elems;
  std::vector<double> tileCost;
  std::vector<int64_t> tiles;
  int32_t maxBRows = 0;
  int64_t maxStage = 0;
  size_t arena = 0;
  for (size_t i = 0; i < B.plans.size(); ++i) {
    Plan P0 = B.plans[i];
    if (P0.gen == GEN_GRID3 && P0.lPad != kGroupLPad) P0.forceTable = 1;
    for (int32_t r0 = 0; r0 < P0.Nmc; r0 += rblk) {
      Plan P = P0;
      P.rOff = r0;
      P.nmcBlk = std::min(rblk, P0.Nmc - r0);
      if (int rc = layout(P)) return rc;
      if (!B.blend.empty() && B.blend[i].gTotal > 0) apply_blend(P, B.blend[i]);
      lo_layout(P);
      if (P.gen == GEN_GRID3 && P.lPad == kGroupLPad) {  // the outer-group kernel, on CTA pairs
        outer_layout(P);
        outer_pair_layout(P, true);
      }
      GroupSub g;
      memset(&g, 0, sizeof(g));
      P.dbgErr = c->dErr;
      g.P = P;
      g.x = B.dx[i];
      g.out = B.dout[i];
      subs.push_back(g);
      elems.push_back(table_threads(P));
      const int64_t nt = (P.n + kTileM - 1) / kTileM;
      if (P.gen == GEN_OUTER) {
        tiles.push_back((nt + 1) / 2);  // pairs of tiles
        tileCost.push_back(outer_pair_cost(P));
      } else {
        tiles.push_back(nt);
        tileCost.push_back((double)P.nChunks * stage_cost(P));
        maxBRows = std::max(maxBRows, P.bRows);
        maxStage = std::max(maxStage, P.stageBytes);
      }
      arena += align_up((size_t)operand_bytes(P));
      if (P.gen == GEN_TABLE) arena += align_up((size_t)P.nChunks * kKtabStageBytes);
    }
  }
  const size_t nU = subs.size();
  run.units = (int64_t)nU;
  std::vector<size_t> tcUnits, outerUnits;
  std::vector<const Plan*> outerPlans;
  for (size_t u = 0; u < nU; ++u) {
    if (subs[u].P.gen == GEN_OUTER) {
      outerUnits.push_back(u);
      outerPlans.push_back(&subs[u].P);
    } else {
      tcUnits.push_back(u);
    }
  }
  if (!tcUnits.empty()) {
    run.smem = group_layout(maxBRows, maxStage, sTc, &run.L);
    if (run.smem == 0) return fail(RF_ENOTSUP, "grouped launch: stages of %lld bytes do not fit", (long long)maxStage);
  }
  if (!outerUnits.empty()) {
    run.osmem = outer_pair_group_layout(outerPlans.data(), outerPlans.size(), sOuter, &run.og);
    if (run.osmem == 0) return fail(RF_ENOTSUP, "grouped launch: outer-group slots do not fit");
  }

  // ---- operands in the arena
  if (int rc = ensure(c->dArena, c->capArena, std::max<size_t>(arena, kAlign), "batch operands")) return rc;
  size_t off = 0;
  for (auto& g : subs) {
    g.B = c->dArena + off;
    off += align_up((size_t)operand_bytes(g.P));
    if (g.P.gen == GEN_TABLE) {
      g.ktab = reinterpret_cast<double*>(c->dArena + off);
      off += align_up((size_t)g.P.nChunks * kKtabStageBytes);
    }
  }

  // ---- schedules: LPT over each kernel's items (tiles; pairs of tiles for
  // the outer-group kernel), longest units first
  const int nCta = c->numSMs, nPairs = c->numSMs / 2;
  const auto perCta = lpt_schedule(tcUnits, tiles, tileCost, nCta);
  const auto perCtaO = lpt_schedule(outerUnits, tiles, tileCost, nPairs);
  int64_t nItems = 0, nItemsO = 0;
  for (size_t u : tcUnits) nItems += tiles[u];
  for (size_t u : outerUnits) nItemsO += tiles[u];
  run.items = nItems + nItemsO;

  // ---- descriptors (pinned staging -> device).  Their capacities only
  // grow, so the offsets inside the buffer stay those of the cached graphs.
  size_t capU = std::max<size_t>(c->descCapU, 1024), capI = std::max<size_t>(c->descCapI, (size_t)1 << 16);
  while (capU < nU) capU *= 2;
  while (capI < (size_t)std::max(nItems, nItemsO)) capI *= 2;
  const DescLayout D = desc_layout(capU, capI, nCta);
  if (capU != c->descCapU || capI != c->descCapI || !c->dDesc) {
    RF_CUDA(cudaStreamSynchronize(st), "batch sync");
    destroy_graphs(c);  // the graphs point into the old layout
    if (c->dDesc) cudaFree(c->dDesc);
    c->dDesc = nullptr;
    c->capDesc = 0;
    if (int rc = ensure(c->dDesc, c->capDesc, D.total, "batch descriptors")) return rc;
    c->descCapU = capU;
    c->descCapI = capI;
  }
  if (int rc = ensure_host(c->hDesc, c->capHDesc, D.total, "batch descriptor staging")) return rc;
  RF_CUDA(cudaStreamSynchronize(st), "batch staging sync");  // the staging buffer may still feed a copy
  unsigned char* h = c->hDesc;
  *reinterpret_cast<int32_t*>(h) = (int32_t)nU;
  memcpy(h + D.subs, subs.data(), nU * sizeof(GroupSub));
  int64_t* pre = reinterpret_cast<int64_t*>(h + D.prefix);
  pre[0] = 0;
  for (size_t u = 0; u < nU; ++u) pre[u + 1] = pre[u] + elems[u];
  uint32_t* stabs = reinterpret_cast<uint32_t*>(h + D.stab);
  int32_t* nst = reinterpret_cast<int32_t*>(h + D.nst);
  for (size_t u : outerUnits)
    if (!pair_group_stage_table(subs[u].P, stabs + u * kOuterMaxKsteps, nst + u))
      return fail(RF_ENOTSUP, "grouped launch: unit %d has no CTA-pair stage table", (int)u);
  put_schedule(perCta, reinterpret_cast<int32_t*>(h + D.cta), reinterpret_cast<GroupItem*>(h + D.items));
  put_schedule(perCtaO, reinterpret_cast<int32_t*>(h + D.octa), reinterpret_cast<GroupItem*>(h + D.oitems));
  RF_CUDA(cudaMemcpyAsync(c->dDesc, h, D.oitems + (size_t)nItemsO * sizeof(GroupItem), cudaMemcpyHostToDevice, st),
          "batch descriptor copy");

  // ---- launch: tables, contraction (graph per layout)
  GroupArgs g;
  g.subs = reinterpret_cast<const GroupSub*>(c->dDesc + D.subs);
  g.items = reinterpret_cast<const GroupItem*>(c->dDesc + D.items);
  g.ctaStart = reinterpret_cast<const int32_t*>(c->dDesc + D.cta);
  g.err = c->dErr;
  g.L = run.L;
  OuterPairGroupArgs og = run.og;
  og.subs = g.subs;
  og.items = reinterpret_cast<const GroupItem*>(c->dDesc + D.oitems);
  og.ctaStart = reinterpret_cast<const int32_t*>(c->dDesc + D.octa);
  og.stabs = reinterpret_cast<const uint32_t*>(c->dDesc + D.stab);
  og.nStages = reinterpret_cast<const int32_t*>(c->dDesc + D.nst);
  og.err = c->dErr;
  const bool hasTc = !tcUnits.empty(), hasOuter = !outerUnits.empty();
  const GroupSub* dSubs = g.subs;
  const int64_t* dPrefix = reinterpret_cast<const int64_t*>(c->dDesc + D.prefix);
  const int32_t* dCount = reinterpret_cast<const int32_t*>(c->dDesc);
  for (auto& e : c->bev)
    if (!e) RF_CUDA(cudaEventCreate(&e), "cudaEventCreate");
  if (hasTc) RF_CUDA(group_set_smem(prec, run.smem), "grouped kernel attributes");
  if (hasOuter) RF_CUDA(outer_pair_group_set_smem(prec, run.osmem), "outer-group kernel attributes");
  rf_context::GraphKey key{prec,          hasTc ? run.L.S : 0, hasTc ? run.L.aCol0 : 0, hasTc ? run.L.slotBytes : 0,
                           hasOuter ? og.S : 0, hasOuter ? og.slotBytes : 0, 0,
                           hasTc ? 1 : 0, c->dDesc};
  auto found = c->graphs.find(key);
  cudaGraphExec_t exec = nullptr;
  if (found != c->graphs.end()) {
    exec = found->second;
    run.replayed = true;
  } else {
    cudaGraph_t graph = nullptr;
    RF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t e1 = cudaEventRecordWithFlags(c->bev[0], st, cudaEventRecordExternal);
    cudaError_t e2 = launch_group_tables(dSubs, dPrefix, dCount, jump_table(), nCta * 8, st);
    cudaError_t e3 = cudaEventRecordWithFlags(c->bev[1], st, cudaEventRecordExternal);
    cudaError_t e4 = hasTc ? launch_group(prec, g, run.smem, nCta, st) : cudaSuccess;
    cudaError_t e4o = hasOuter ? launch_outer_pair_group(prec, og, run.osmem, 2 * nPairs, st) : cudaSuccess;
    cudaError_t e5 = cudaEventRecordWithFlags(c->bev[2], st, cudaEventRecordExternal);
    cudaError_t ee = cudaStreamEndCapture(st, &graph);
    for (cudaError_t e : {e1, e2, e3, e4, e4o, e5, ee})
      if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return cuda_fail(e, "capture of the grouped launch");
      }
    cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    c->graphs[key] = exec;
  }
  RF_CUDA(cudaGraphLaunch(exec, st), "cudaGraphLaunch");
  c->launches += 1 + (hasTc ? 1 : 0) + (hasOuter ? 1 : 0);
  return RF_OK;
}

// The batch class of the tuner's key: whether the batch holds units of the
// grouped tcgen05 kernel (bit 0) and of the outer-group kernel (bit 1).
int batch_class(const BatchState& B) {
  int cls = 0;
  for (const Plan& P : B.plans) {
    const bool outer = P.gen == GEN_GRID3 && P.lPad == kGroupLPad && P.kNStep[0] <= kOuterMaxN1P &&
                       (P.prec == PREC_BF16 || P.prec == PREC_FP16 || P.prec == PREC_BF16_FAST);
    cls |= outer ? 2 : 1;
  }
  return cls;
}

int batch_times(rf_context* c, double* tables, double* contract) {
  RF_CUDA(cudaEventSynchronize(c->bev[2]), "cudaEventSynchronize");
  float a = 0, b = 0;
  RF_CUDA(cudaEventElapsedTime(&a, c->bev[0], c->bev[1]), "cudaEventElapsedTime");
  RF_CUDA(cudaEventElapsedTime(&b, c->bev[1], c->bev[2]), "cudaEventElapsedTime");
  *tables = a;
  *contract = b;
  return RF_OK;
}

// Plans every request (extents from `ext`), then runs the grouped launch,
// tuning the realization block on the first batch of a precision form.
int run_batch(rf_context* c, const rf_request* reqs, int32_t count, const std::vector<Request>& rq,
              const std::vector<double>& ext, BatchState& B, cudaStream_t st) {
  const int prec = rq[0].opt.precision;
  B.plans.resize(count);
  for (int32_t i = 0; i < count; ++i)
    if (int rc = build_plan(rq[i], &ext[3 * i], B.plans[i])) return rc;
  (void)reqs;
  GroupRun run;
  rf_batch_stats stats{};
  const int key = prec * 4 + batch_class(B);
  auto tuned = c->tuned.find(key);
  if (tuned == c->tuned.end() && !B.accumulate) {
    // Coordinate search from the default (first realization block, deepest
    // pipelines): the realization block, then one slot fewer in the grouped
    // tcgen05 kernel, then a shallower outer-group pipeline; a candidate is
    // kept when the whole batch (tables + contractions) runs faster.  Every
    // candidate computes the same field.
    rf_context::TuneChoice best;
    best.blk = block_candidates(prec)[0];
    auto time_of = [&](const rf_context::TuneChoice& t, double* ms, GroupRun* r) -> int {
      if (int rc = group_run(c, B, prec, t.blk, t.sTc, t.sOuter, st, *r)) return rc;
      double a = 0, b = 0;
      if (int rc = batch_times(c, &a, &b)) return rc;
      *ms = a + b;
      return RF_OK;
    };
    GroupRun r0;
    if (int rc = time_of(best, &best.bestMs, &r0)) return rc;
    best.defaultMs = best.bestMs;
    best.candidates = 1;
    std::vector<rf_context::TuneChoice> tries;
    for (int blk : block_candidates(prec))
      if (blk != best.blk) {
        rf_context::TuneChoice t = best;
        t.blk = blk;
        tries.push_back(t);
      }
    for (const rf_context::TuneChoice& t0 : tries) {
      double ms = 0;
      GroupRun r;
      if (int rc = time_of(t0, &ms, &r)) return rc;
      ++best.candidates;
      if (ms < best.bestMs) {
        const int n = best.candidates;
        const double d = best.defaultMs;
        best = t0;
        best.bestMs = ms;
        best.defaultMs = d;
        best.candidates = n;
      }
    }
    // pipeline depths, one coordinate at a time (only the kernels the batch launches)
    if (r0.L.S > 2) {
      rf_context::TuneChoice t = best;
      t.sTc = r0.L.S - 1;
      double ms = 0;
      GroupRun r;
      if (int rc = time_of(t, &ms, &r)) return rc;
      ++best.candidates;
      if (ms < best.bestMs) {
        best.sTc = t.sTc;
        best.bestMs = ms;
      }
    }
    if (r0.og.S > 4) {
      rf_context::TuneChoice t = best;
      t.sOuter = 4;
      double ms = 0;
      GroupRun r;
      if (int rc = time_of(t, &ms, &r)) return rc;
      ++best.candidates;
      if (ms < best.bestMs) {
        best.sOuter = t.sOuter;
        best.bestMs = ms;
      }
    }
    tuned = c->tuned.emplace(key, best).first;
    stats.tuned = 1;
  }
  const rf_context::TuneChoice choice =
      tuned != c->tuned.end() ? tuned->second : rf_context::TuneChoice{block_candidates(prec)[0], 0, 0, 0, 0.0, 0.0};
  if (int rc = group_run(c, B, prec, choice.blk, choice.sTc, choice.sOuter, st, run)) return rc;
  stats.units = run.units;
  stats.work_items = run.items;
  stats.realization_block = run.rblk;
  stats.stages = run.L.S;
  stats.outer_stages = run.og.S;
  stats.graph_replayed = run.replayed ? 1 : 0;
  stats.tune_candidates = choice.candidates;
  stats.tune_default_ms = choice.defaultMs;
  stats.tune_best_ms = choice.bestMs;
  // normalisation passes (per request, after the contraction)
  for (int32_t i = 0; i < count; ++i) {
    const Plan& P = B.plans[i];
    if (!P.normalize) continue;
    if ((size_t)2 * P.Nmc * sizeof(double) > c->capWork)
      if (int rc = ensure(c->dWork, c->capWork, (size_t)2 * P.Nmc * sizeof(double), "moments")) return rc;
    RF_CUDA(launch_normalize_and_map(P, B.dout[i], P.Nmc, c->dWork, st), "normalisation kernels");
    c->launches += 3;
  }
  c->last = stats;
  return RF_OK;
}

}  // namespace

namespace rfh {

int batch_run_device(rf_context* c, const std::vector<Request>& rq, const std::vector<const double*>& dx,
                     const std::vector<double*>& dout, const std::vector<double>& ext, cudaStream_t st,
                     const std::vector<BlendSpec>* blend) {
  BatchState B;
  B.dx = dx;
  B.dout = dout;
  if (blend && !blend->empty()) {
    B.blend = *blend;
    B.accumulate = true;
  }
  return run_batch(c, nullptr, (int32_t)rq.size(), rq, ext, B, st);
}

int request_footprint(const Request& rq, const double* ext, int rblk, size_t* bytes) {
  Plan P0;
  if (int rc = build_plan(rq, ext, P0)) return rc;
  if (P0.gen == GEN_GRID3 && P0.lPad != kGroupLPad) P0.forceTable = 1;
  size_t b = align_up(sizeof(double) * (size_t)rq.n * rq.nDim) + align_up(sizeof(double) * (size_t)rq.n * rq.Nmc);
  for (int32_t r0 = 0; r0 < P0.Nmc; r0 += rblk) {
    Plan P = P0;
    P.rOff = r0;
    P.nmcBlk = std::min(rblk, P0.Nmc - r0);
    if (int rc = layout(P)) return rc;
    lo_layout(P);
    if (P.gen == GEN_GRID3 && P.lPad == kGroupLPad) {  // as group_run plans it
      outer_layout(P);
      outer_pair_layout(P, true);
    }
    b += align_up((size_t)operand_bytes(P));
    if (P.gen == GEN_TABLE) b += align_up((size_t)P.nChunks * kKtabStageBytes);
  }
  *bytes = b;
  return RF_OK;
}

int default_block(int prec) { return block_candidates(prec)[0]; }

}  // namespace rfh

namespace {

int check_batch(const rf_request* reqs, int32_t count, std::vector<Request>& rq) {
  if (!reqs || count < 1) return fail(RF_EINVAL_ARG, "empty batch");
  rq.resize(count);
  for (int32_t i = 0; i < count; ++i) {
    const rf_request& r = reqs[i];
    if (!r.xPoints || !r.randField) return fail(RF_EINVAL_ARG, "request %d: null pointer", i);
    rq[i] = make_request(r.nDim, r.n, r.corrMod, r.margiFirst, r.corrL, r.fieldAvg, r.fieldVar, r.Nmc, r.method,
                         &r.opt);
    if (int rc = validate(rq[i])) return fail(rc, "request %d: %s", i, g_err.c_str());
    if (rq[i].opt.precision != rq[0].opt.precision)
      return fail(RF_EINVAL_ARG, "request %d: all requests of a batch need the same precision form", i);
    if (rq[i].opt.device != rq[0].opt.device)
      return fail(RF_EINVAL_ARG, "request %d: all requests of a batch need the same device", i);
    if (rq[i].opt.literal) return fail(RF_ENOTSUP, "request %d: literal mode is not available in a batch", i);
  }
  return RF_OK;
}

bool needs_extent(const Request& r) {
  for (int d = 0; d < r.nDim; ++d)
    if (!(r.opt.x_range[d] > 0.0)) return true;
  return false;
}

// topography_RF.f90:49-52 (overlap rounded to the grid, at least two steps
// where the axis is split) and localization_RF.f90:746 (overlapNPoints);
// subdomains of L points start every L - overlapNPoints points.
int blend_geometry(const rf_blend_grid* g, const double* corrL, int32_t* L, int32_t* O) {
  if (!g || !corrL) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (g->nDim < 1 || g->nDim > 3) return fail(RF_EINVAL_NDIM, "nDim must be 1, 2 or 3 (got %d)", g->nDim);
  for (int d = 0; d < 3; ++d) {
    L[d] = 1;
    O[d] = 0;
    if (d >= g->nDim) continue;
    const int32_t N = g->xNStep[d], F = g->nFields[d];
    const double h = g->xStep[d];
    if (N < 2 || F < 1 || !(h > 0.0) || !(corrL[d] > 0.0))
      return fail(RF_EINVAL_ARG, "blend axis %d: xNStep >= 2, nFields >= 1, xStep > 0, corrL > 0 needed", d + 1);
    double ov = F == 1 ? 0.0 : g->overlap;
    ov = std::nearbyint(ov * corrL[d] / h) * h / corrL[d];
    if (F != 1 && ov < 2.0 * h / corrL[d]) ov = 2.0 * h / corrL[d];
    O[d] = (int32_t)std::lround((ov * corrL[d] - 2.0 * h) / h) + 1;
    const int32_t shared = (F - 1) * std::max(O[d], 0);
    if ((N + shared) % F != 0)
      return fail(RF_EINVAL_RANGE,
                  "blend axis %d: %d points do not split into %d subdomains sharing %d points (N + (F-1)*O "
                  "must be a multiple of F)",
                  d + 1, N, F, O[d]);
    L[d] = (N + shared) / F;
    if (F > 1 && L[d] <= O[d]) return fail(RF_EINVAL_RANGE, "blend axis %d: overlap wider than a subdomain", d + 1);
  }
  return RF_OK;
}

}  // namespace

namespace rfh {

int blend_points_bytes(const rf_blend_grid* grid, const double* corrL, size_t* bytes) {
  int32_t L[3], O[3];
  if (int rc = blend_geometry(grid, corrL, L, O)) return rc;
  int nSub = 1;
  for (int d = 0; d < grid->nDim; ++d) nSub *= grid->nFields[d];
  *bytes = sizeof(double) * (size_t)L[0] * L[1] * L[2] * grid->nDim * nSub;
  return RF_OK;
}

int blend_expand(const rf_blend_grid* grid, const Request& base, double* dOut, double* dPoints, cudaStream_t st,
                 std::vector<Request>& rq, std::vector<const double*>& dx, std::vector<double*>& dout,
                 std::vector<BlendSpec>& spec, Plan* groupPlan) {
  int32_t L[3], O[3];
  if (int rc = blend_geometry(grid, base.corrL, L, O)) return rc;
  if (base.opt.precision == RF_PREC_FP32) return fail(RF_ENOTSUP, "the blend runs the tensor-core forms");
  if (base.opt.literal) return fail(RF_ENOTSUP, "literal mode is not available for the blend");
  const int nd = grid->nDim;
  int32_t F[3] = {1, 1, 1}, G[3] = {1, 1, 1};
  for (int d = 0; d < nd; ++d) {
    F[d] = grid->nFields[d];
    G[d] = grid->xNStep[d];
  }
  const int64_t gTotal = (int64_t)G[0] * G[1] * G[2];
  const int64_t sub = (int64_t)L[0] * L[1] * L[2];
  const int nSub = F[0] * F[1] * F[2];
  int64_t seed0 = base.opt.seed_start;
  if (seed0 < 0) {  // one stochastic seed, then + fieldNumber (sample_RF.f90:316-317)
    const auto t = std::chrono::steady_clock::now().time_since_epoch().count();
    seed0 = (int64_t)((uint64_t)t % 100000000ull);
  }
  RF_CUDA(cudaMemsetAsync(dOut, 0, sizeof(double) * (size_t)gTotal * base.Nmc, st), "clear of randField");
  for (int f = 0; f < nSub; ++f) {
    const int32_t fi[3] = {f % F[0], (f / F[0]) % F[1], f / (F[0] * F[1])};
    BlendSpec b;
    double x0[3] = {0, 0, 0}, h[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) {
      b.bDims[d] = L[d];
      b.bOrigin[d] = d < nd ? fi[d] * (L[d] - std::max(O[d], 0)) : 0;
      b.gDims[d] = G[d];
      b.bRamp[d] = d < nd ? O[d] : 0;
      if (d < nd) {
        h[d] = grid->xStep[d];
        x0[d] = grid->xMin[d] + (double)b.bOrigin[d] * h[d];
      }
    }
    b.gTotal = gTotal;
    double* px = dPoints + (size_t)f * sub * nd;
    RF_CUDA(launch_grid_points(px, nd, L, x0, h, st), "subdomain points kernel");
    Request r = base;
    r.n = sub;
    r.opt.seed_start = seed0 + f + 1;  // fieldNumber = f + 1
    r.opt.normalize = 0;
    for (int d = 0; d < nd; ++d) r.opt.x_range[d] = (double)(L[d] - 1) * grid->xStep[d];
    rq.push_back(r);
    dx.push_back(px);
    dout.push_back(dOut);
    spec.push_back(b);
  }
  // the group plan: marginal parameters of the request, group geometry
  const double zero[3] = {0, 0, 0};
  if (int rc = build_plan(rq.back(), zero, *groupPlan)) return rc;
  Plan& Gp = *groupPlan;
  Gp.nDim = nd;
  Gp.n = gTotal;
  Gp.gTotal = gTotal;
  for (int d = 0; d < 3; ++d) {
    Gp.gDims[d] = G[d];
    Gp.bRamp[d] = d < nd ? O[d] : 0;
  }
  Gp.normalize = base.opt.normalize ? 1 : 0;
  return RF_OK;
}

int blend_finish(rf_context* c, const Plan& Gp, double* dOut, cudaStream_t st) {
  RF_CUDA(launch_blend_finish(Gp, dOut, Gp.normalize ? 0 : 1, st), "border correction kernel");
  c->launches += 1;
  if (Gp.normalize) {
    if ((size_t)2 * Gp.Nmc * sizeof(double) > c->capWork)
      if (int rc = ensure(c->dWork, c->capWork, (size_t)2 * Gp.Nmc * sizeof(double), "moments")) return rc;
    RF_CUDA(launch_normalize_and_map(Gp, dOut, Gp.Nmc, c->dWork, st), "normalisation kernels");
    c->launches += 3;
  }
  return RF_OK;
}

}  // namespace rfh

namespace {

// The blended field of `grid` into the device array dOut (group points x Nmc):
// through the structured-grid path where it applies (its subdomains are
// grids), else as grouped-launch units whose epilogue adds the weighted field.
int run_blended(rf_context* c, const rf_blend_grid* grid, const Request& base, double* dOut, cudaStream_t st) {
  if (grid_blend_ok(grid, base)) return grid_blend_run(c, grid, base, dOut, st);
  size_t pb = 0;
  if (int rc = blend_points_bytes(grid, base.corrL, &pb)) return rc;
  if (int rc = ensure(c->dX, c->capX, pb, "subdomain points")) return rc;
  std::vector<Request> rq;
  std::vector<const double*> dx;
  std::vector<double*> dout;
  std::vector<BlendSpec> spec;
  Plan Gp;
  if (int rc = blend_expand(grid, base, dOut, c->dX, st, rq, dx, dout, spec, &Gp)) return rc;
  c->launches += (int32_t)rq.size();
  const std::vector<double> ext(3 * rq.size(), 0.0);
  if (int rc = batch_run_device(c, rq, dx, dout, ext, st, &spec)) return rc;
  return blend_finish(c, Gp, dOut, st);
}

}  // namespace

extern "C" {

int rf_blend_layout(const rf_blend_grid* grid, const double* corrL, int32_t* subNStep, int32_t* overlapNPoints) {
  g_err.clear();
  int32_t L[3], O[3];
  if (int rc = blend_geometry(grid, corrL, L, O)) return rc;
  for (int d = 0; d < 3; ++d) {
    if (subNStep) subNStep[d] = L[d];
    if (overlapNPoints) overlapNPoints[d] = O[d];
  }
  return RF_OK;
}

int rf_generate_blended_device(rf_context* ctx, const rf_blend_grid* grid, int corrMod, int margiFirst,
                               const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                               double* d_randField, const rf_options* opt, void* stream) {
  rfh::NvtxRange nvtx_("rf_generate_blended_device");
  g_err.clear();
  if (!ctx || !grid || !corrL || !d_randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  Request rq = make_request(grid->nDim, 1, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate(rq)) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
  ctx->launches = 0;
  return run_blended(ctx, grid, rq, d_randField, st);
}

int rf_generate_blended(rf_context* ctx, const rf_blend_grid* grid, int corrMod, int margiFirst, const double* corrL,
                        double fieldAvg, double fieldVar, int Nmc, int method, double* randField,
                        const rf_options* opt) {
  rfh::NvtxRange nvtx_("rf_generate_blended");
  g_err.clear();
  if (!ctx || !grid || !corrL || !randField) return fail(RF_EINVAL_ARG, "null pointer argument");
  Request rq = make_request(grid->nDim, 1, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, opt);
  if (int rc = validate(rq)) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = ctx->stream;
  ctx->launches = 0;
  int64_t gTotal = 1;
  for (int d = 0; d < grid->nDim && d < 3; ++d) gTotal *= std::max(grid->xNStep[d], 1);
  const size_t bytes = sizeof(double) * (size_t)gTotal * Nmc;
  if (int rc = ensure(ctx->dOut, ctx->capOut, bytes, "blended field")) return rc;
  if (int rc = run_blended(ctx, grid, rq, ctx->dOut, st)) return rc;
  RF_CUDA(cudaMemcpyAsync(randField, ctx->dOut, bytes, cudaMemcpyDeviceToHost, st), "copy of randField");
  RF_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return check_device_error(ctx);
}

int rf_generate_batch(rf_context* ctx, const rf_request* reqs, int32_t count) {
  rfh::NvtxRange nvtx_("rf_generate_batch");
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  std::vector<Request> rq;
  if (int rc = check_batch(reqs, count, rq)) return rc;
  if (rq[0].opt.precision == RF_PREC_FP32) {
    // the plain form has no grouped kernel: request by request
    for (int32_t i = 0; i < count; ++i) {
      const rf_request& r = reqs[i];
      rf_options o = rq[i].opt;
      if (int rc = rf_create_standard_gaussian_field_unstruct(r.xPoints, r.nDim, r.n, r.corrMod, r.margiFirst, r.corrL,
                                                              r.fieldAvg, r.fieldVar, r.Nmc, r.method, r.randField,
                                                              &o))
        return rc;
    }
    return RF_OK;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = ctx->stream;
  ctx->launches = 0;
  // host extents, arena for points and fields after the operands
  std::vector<double> ext(3 * count, 0.0);
  size_t io = 0;
  for (int32_t i = 0; i < count; ++i) {
    const rf_request& r = reqs[i];
    if (needs_extent(rq[i]))
      for (int d = 0; d < r.nDim; ++d) {
        double lo = r.xPoints[d], hi = r.xPoints[d];
        for (int64_t k = 1; k < r.n; ++k) {
          lo = std::min(lo, r.xPoints[k * r.nDim + d]);
          hi = std::max(hi, r.xPoints[k * r.nDim + d]);
        }
        ext[3 * i + d] = hi - lo;
      }
    io += align_up(sizeof(double) * (size_t)r.n * r.nDim) + align_up(sizeof(double) * (size_t)r.n * r.Nmc);
  }
  if (int rc = ensure(ctx->dX, ctx->capX, io, "batch points and fields")) return rc;
  BatchState B;
  B.dx.resize(count);
  B.dout.resize(count);
  unsigned char* base = reinterpret_cast<unsigned char*>(ctx->dX);
  size_t off = 0;
  for (int32_t i = 0; i < count; ++i) {
    const rf_request& r = reqs[i];
    const size_t xb = sizeof(double) * (size_t)r.n * r.nDim, ob = sizeof(double) * (size_t)r.n * r.Nmc;
    B.dx[i] = reinterpret_cast<double*>(base + off);
    off += align_up(xb);
    B.dout[i] = reinterpret_cast<double*>(base + off);
    off += align_up(ob);
    RF_CUDA(cudaMemcpyAsync(const_cast<double*>(B.dx[i]), r.xPoints, xb, cudaMemcpyHostToDevice, st),
            "copy of xPoints");
  }
  if (int rc = run_batch(ctx, reqs, count, rq, ext, B, st)) return rc;
  for (int32_t i = 0; i < count; ++i) {
    const rf_request& r = reqs[i];
    RF_CUDA(cudaMemcpyAsync(r.randField, B.dout[i], sizeof(double) * (size_t)r.n * r.Nmc, cudaMemcpyDeviceToHost,
                            st),
            "copy of randField");
  }
  RF_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return check_device_error(ctx);
}

int rf_generate_batch_device(rf_context* ctx, const rf_request* reqs, int32_t count, void* stream) {
  rfh::NvtxRange nvtx_("rf_generate_batch_device");
  g_err.clear();
  if (!ctx) return fail(RF_EINVAL_ARG, "null context");
  std::vector<Request> rq;
  if (int rc = check_batch(reqs, count, rq)) return rc;
  if (rq[0].opt.precision == RF_PREC_FP32) {
    for (int32_t i = 0; i < count; ++i) {
      const rf_request& r = reqs[i];
      rf_options o = rq[i].opt;
      if (int rc = rf_generate_device(ctx, r.xPoints, r.nDim, r.n, r.corrMod, r.margiFirst, r.corrL, r.fieldAvg,
                                      r.fieldVar, r.Nmc, r.method, r.randField, &o, stream))
        return rc;
    }
    return RF_OK;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
  ctx->launches = 0;
  // device extents: one reduction per request that needs it, one copy back
  std::vector<double> ext(3 * count, 0.0);
  int32_t nx = 0;
  for (int32_t i = 0; i < count; ++i) nx += needs_extent(rq[i]) ? 1 : 0;
  if (nx > 0) {
    const size_t per = (size_t)6 * kExtentBlocks;
    if (int rc = ensure(ctx->dExt, ctx->capExt, sizeof(double) * per * nx, "batch extents")) return rc;
    if (int rc = ensure_host(ctx->hExt, ctx->capHExt, sizeof(double) * per * nx, "batch extents")) return rc;
    int32_t k = 0;
    for (int32_t i = 0; i < count; ++i)
      if (needs_extent(rq[i])) launch_extent(reqs[i].xPoints, reqs[i].n, reqs[i].nDim, ctx->dExt + per * k++, st);
    RF_CUDA(cudaGetLastError(), "extent kernels");
    ctx->launches += nx;
    RF_CUDA(cudaMemcpyAsync(ctx->hExt, ctx->dExt, sizeof(double) * per * nx, cudaMemcpyDeviceToHost, st),
            "extent copy");
    RF_CUDA(cudaStreamSynchronize(st), "extent sync");
    k = 0;
    for (int32_t i = 0; i < count; ++i) {
      if (!needs_extent(rq[i])) continue;
      const double* part = ctx->hExt + per * k++;
      for (int d = 0; d < reqs[i].nDim; ++d) {
        double lo = INFINITY, hi = -INFINITY;
        for (int b = 0; b < kExtentBlocks; ++b) {
          lo = std::min(lo, part[b * 6 + d]);
          hi = std::max(hi, part[b * 6 + 3 + d]);
        }
        ext[3 * i + d] = hi - lo;
      }
    }
  }
  BatchState B;
  B.dx.resize(count);
  B.dout.resize(count);
  for (int32_t i = 0; i < count; ++i) {
    B.dx[i] = reqs[i].xPoints;
    B.dout[i] = reqs[i].randField;
  }
  return run_batch(ctx, reqs, count, rq, ext, B, st);
}

int rf_batch_last_stats(rf_context* ctx, rf_batch_stats* out) {
  g_err.clear();
  if (!ctx || !out) return fail(RF_EINVAL_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  RF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  *out = ctx->last;
  if (ctx->bev[2]) {
    if (int rc = batch_times(ctx, &out->tables_ms, &out->contract_ms)) return rc;
  }
  return RF_OK;
}

}  // extern "C"
