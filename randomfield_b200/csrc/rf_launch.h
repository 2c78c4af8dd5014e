// rf_launch.h -- host-side launchers of the device kernels (one per .cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rf_plan.h"

namespace rfb {

struct JumpTable;

// Builds the contraction operand B (and, for GEN_TABLE, the wavevector
// table) on the device from the rnglib stream: see rf_tables.cu.
// literalSlab >= 0 selects the literal-mode amplitude of that point slab.
cudaError_t launch_tables(const Plan& P, const JumpTable& jt, void* dB, double* dKtab, int64_t literalSlab,
                          int64_t nSlab, cudaStream_t st);

// The i4_uni draws the table builder consumes for this plan's realization
// block, in reference order: dRk[(r * K + k) * D + j] (D = 2 isotropic:
// gamma, psi; else 1: the phase), dK[2 k + j] the isotropic direction draws
// (theta, phi); dK may be null.
cudaError_t launch_table_draws(const Plan& P, const JumpTable& jt, int32_t* dRk, int32_t* dK, cudaStream_t st);

// tcgen05 contraction + fused epilogue over points [row0, row0 + rows).
cudaError_t launch_tc(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                      int64_t row0, int64_t rows, uint32_t* dErr, int numSMs, cudaStream_t st);

// Outer-group contraction of GEN_OUTER plans (rf_outer.cu) over points
// [row0, row0 + rows); outer_smem_bytes is its shared-memory size (0: the
// slot does not fit), *stages its slot count.
cudaError_t launch_outer(const Plan& P, const double* dX, const void* dB, double* dOut, int64_t row0, int64_t rows,
                         uint32_t* dErr, int numSMs, cudaStream_t st);
size_t outer_smem_bytes(const Plan& P, int* stages);
// The CTA-pair form (P.oPair, rf_outer_pair.cu): clusters of two CTAs, one
// 256-point item per pair.
cudaError_t launch_outer_pair(const Plan& P, const double* dX, const void* dB, double* dOut, int64_t row0,
                              int64_t rows, uint32_t* dErr, int numSMs, cudaStream_t st);
size_t outer_pair_smem_bytes(const Plan& P, int* stages);

// Plain FP32 contraction (FFMA) + the same epilogue.
cudaError_t launch_fp32(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                        int64_t row0, int64_t rows, cudaStream_t st);

// Empirical normalisation (randomFieldND.f90:820-926) over `ncols` columns,
// then the marginal map over all Nmc columns.  dWork holds 2*Nmc doubles.
cudaError_t launch_normalize_and_map(const Plan& P, double* dOut, int32_t ncols, double* dWork,
                                     cudaStream_t st);

// Grid points x0 + i*h of an L[0] x L[1] x L[2] box (axis 1 fastest).
cudaError_t launch_grid_points(double* dX, int32_t nDim, const int32_t* L, const double* x0, const double* h,
                               cudaStream_t st);

// One subdomain's field (subPoints x Nmc) times its partition-of-unity
// weights added into the group field; P carries nDim, bDims, bOrigin, gDims,
// bRamp and gTotal.
cudaError_t launch_blend_add(const Plan& P, const double* dSub, double* dGroup, int64_t subPoints, int32_t Nmc,
                             cudaStream_t st);

// Border correction of a blended group field, then (applyMarginal) the
// marginal map; G carries nDim, Nmc, gDims, gTotal, bRamp and the marginal.
cudaError_t launch_blend_finish(const Plan& G, double* dOut, int32_t applyMarginal, cudaStream_t st);

// Shared-memory bytes the tcgen05 kernel needs for this plan (0 if it
// cannot fit).
size_t tc_smem_bytes(const Plan& P, int* stages);

// Grouped launch (rf_tc.cu): every CTA b runs the work items
// items[ctaStart[b] .. ctaStart[b+1]) of the units `subs`, all with the
// shared slot layout L.  GEN_GRID3 units must have lPad == kGroupLPad; the
// others run GEN_TABLE.
constexpr int kGroupLPad = 24;
struct GroupArgs {
  const GroupSub* subs;
  const GroupItem* items;
  const int32_t* ctaStart;
  uint32_t* err;
  SlotLayout L;
};
// Slot layout for units with at most maxBRows B rows and maxStageBytes per
// stage, at most maxStages deep; returns the shared-memory bytes (0: none fits).
size_t group_layout(int32_t maxBRows, int64_t maxStageBytes, int32_t maxStages, SlotLayout* L);
// Sets the grouped kernel's shared-memory size (outside any stream capture),
// then launch_group queues it.
cudaError_t group_set_smem(int prec, size_t smem);
cudaError_t launch_group(int prec, const GroupArgs& g, size_t smem, int grid, cudaStream_t st);

// Grouped outer-group contraction on CTA pairs (rf_outer_pair.cu): every
// pair b (CTAs 2b, 2b + 1) runs the items items[ctaStart[b] ..
// ctaStart[b+1]) of the GEN_OUTER units `subs` in the CTA-pair layout
// (outer_pair_layout; an item's `tile` is its 256-point item; lPad ==
// kGroupLPad); unit u's stage table is stabs[u * kOuterMaxKsteps ..], its
// length nStages[u] (pair_group_stage_table).  One slot layout for all: S
// slots of slotBytes.
struct OuterPairGroupArgs {
  const GroupSub* subs;
  const GroupItem* items;
  const int32_t* ctaStart;
  const uint32_t* stabs;
  const int32_t* nStages;
  uint32_t* err;
  int32_t S, slotBytes;
};
// The stage table of a CTA-pair plan as the grouped kernel reads it (false
// when the plan's stage marks break the kernel's rule).
bool pair_group_stage_table(const Plan& P, uint32_t* stab, int32_t* nStages);
// Slot layout covering every plan, at most maxStages slots (0: as many as
// fit); returns the shared-memory bytes (0: none fits) and fills S and
// slotBytes.
size_t outer_pair_group_layout(const Plan* const* plans, size_t count, int maxStages, OuterPairGroupArgs* g);
cudaError_t outer_pair_group_set_smem(int prec, size_t smem);
// grid: two CTAs per pair of the schedule
cudaError_t launch_outer_pair_group(int prec, const OuterPairGroupArgs& g, size_t smem, int grid, cudaStream_t st);

// Grouped table builder: B (and the wavevector chunks) of every unit; the
// element range of unit u is [prefix[u], prefix[u+1]) of prefix[*nsubs]
// (all three in device memory, read when the kernel runs).
cudaError_t launch_group_tables(const GroupSub* subs, const int64_t* prefix, const int32_t* nsubs,
                                const JumpTable& jt, int blocks, cudaStream_t st);
size_t fp32_smem_bytes(const Plan& P);

}  // namespace rfb
