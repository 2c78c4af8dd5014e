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

// tcgen05 contraction + fused epilogue over points [row0, row0 + rows).
cudaError_t launch_tc(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                      int64_t row0, int64_t rows, uint32_t* dErr, int numSMs, cudaStream_t st);

// Plain FP32 contraction (FFMA) + the same epilogue.
cudaError_t launch_fp32(const Plan& P, const double* dX, const void* dB, const double* dKtab, double* dOut,
                        int64_t row0, int64_t rows, cudaStream_t st);

// Empirical normalisation (randomFieldND.f90:820-926) over `ncols` columns,
// then the marginal map over all Nmc columns.  dWork holds 2*Nmc doubles.
cudaError_t launch_normalize_and_map(const Plan& P, double* dOut, int32_t ncols, double* dWork,
                                     cudaStream_t st);

// Shared-memory bytes the tcgen05 kernel needs for this plan (0 if it
// cannot fit).
size_t tc_smem_bytes(const Plan& P, int* stages);
size_t fp32_smem_bytes(const Plan& P);

}  // namespace rfb
