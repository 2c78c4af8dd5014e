// rf_tables.cu -- device builder of the contraction operand.
//
// The Shinozuka sum f(x, r) = ampMult * sum_k a_k cos(k.x + phi_{k,r})
// (randomFieldND.f90:276-330) is evaluated as the contraction
//   f = ampMult * [cos(Kx) | sin(Kx)] (points x 2K)  *  B (2K x Nmc),
//   B[2k, r] = a_k cos(phi_{k,r}),  B[2k+1, r] = -a_k sin(phi_{k,r}).
// One thread per (wavevector in kernel order, realization).  The phases come
// from the rnglib stream (rnglib.f90:548-659) by jump-ahead: the p-th draw of
// generator 1 is (a1^p s1 mod m1) - (a2^p s2 mod m2) folded, so every
// element is computed independently and the table matches a sequential run
// draw for draw.  Draw order follows the reference: Shinozuka K phases per
// realization in k order (:278-279); isotropic direction blocks then, per
// realization, a gamma block and a psi block (:460-468 restated).
#include <cuda_fp8.h>

#include "rf_device.cuh"
#include "rf_gen.cuh"
#include "rf_launch.h"

namespace rfb {

struct KVal {
  int64_t ref;   // reference index, -1 for padding
  double k[3];
  double amp;    // a_k before the per-realization factor
};

// Quadrant sign of axis d (d >= 1) for sign row q (spectra_RF.f90:267-286).
__device__ __forceinline__ double quad_sign(int q, int d, int nDim) {
  return ((q >> (nDim - 1 - d)) & 1) ? -1.0 : 1.0;
}

__device__ __forceinline__ double gauss_spectrum(const double* k, int nDim) {
  // spectra_RF.f90:202-208 with corrL = 1 after normalisation
  double s = 1.0;
  for (int d = 0; d < nDim; ++d) s = s * 1.0 * exp(-((k[d] * k[d]) * 1.0) / (4.0 * kRefPi));
  return s;
}

__device__ KVal kvalue(const Plan& P, const JumpTable& jt, int64_t kk) {
  KVal v;
  v.ref = -1;
  v.k[0] = v.k[1] = v.k[2] = 0.0;
  v.amp = 0.0;
  const int64_t stage = kk / P.chunkK;
  const int32_t c = (int32_t)(kk % P.chunkK);
  if (P.gen == GEN_GRID3) {
    int32_t idx[3], sg[3];
    const int32_t gw = 2 * P.lPad;  // columns per group
    v.ref = grid3_ref_index(P.kNStep, P.lPad, stage * P.gps + c / gw, c % gw, idx, sg);
    if (v.ref < 0) return v;
    for (int d = 0; d < 3; ++d) {
      const double base = 0.0 + P.kDelta[d] * (double)idx[d];
      v.k[d] = sg[d] ? base * -1.0 : base * 1.0;
    }
  } else if (P.method != 1) {  // Shinozuka through the table, or randomization
    if (kk >= P.K) return v;
    v.ref = kk;
    int64_t kn = 1;
    for (int d = 0; d < P.nDim; ++d) kn *= P.kNStep[d];
    const int q = (int)(kk / kn);
    const int64_t b = kk % kn;
    int64_t rem = b;
    for (int d = 0; d < P.nDim; ++d) {
      const int64_t i = rem % P.kNStep[d];
      rem /= P.kNStep[d];
      // randomization: kPoints_base = random_number * kMax, axis fastest,
      // the first nDim*kn draws of the stream (spectra_RF.f90:119-124)
      const double base =
          (P.method == 3) ? r8_uni_at(jt, P.ig1, P.ig2, (uint64_t)(b * P.nDim + d + 1)) * P.kMax
                          : 0.0 + P.kDelta[d] * (double)i;
      // B2 in literal mode: the first quadrant is never written.
      v.k[d] = (P.literal && q == 0) ? 0.0 : base * (d == 0 ? 1.0 : quad_sign(q, d, P.nDim));
    }
  } else {  // isotropic, intended maths
    if (kk >= P.K) return v;
    v.ref = kk;
    const int64_t K = P.K;
    const int nd = P.kNStep[1];
    const int j = (int)(kk / nd);
    const double r = (double)j * P.kDelta[0];
    const double s1 = P.ig1, s2 = P.ig2;
    const double uth = r8_uni_at(jt, (int64_t)s1, (int64_t)s2, (uint64_t)((P.nDim == 3 ? K : 0) + kk + 1));
    const double th = 2.0 * kRefPi * uth;
    double S;
    if (P.corrMod == 1) S = exp(-((r * r) * 1.0) / (4.0 * kRefPi));
    else S = (j == 5) ? 1.0 : 0.0;
    double shell;
    if (P.nDim == 3) {
      const double uphi = r8_uni_at(jt, (int64_t)s1, (int64_t)s2, (uint64_t)(kk + 1));
      const double cph = 1.0 - 2.0 * uphi;
      const double sph = sqrt(fmax(0.0, 1.0 - cph * cph));
      v.k[0] = r * (sph * cos(th));
      v.k[1] = r * (sph * sin(th));
      v.k[2] = r * cph;
      shell = 4.0 * kRefPi * r * r;
    } else {
      v.k[0] = r * cos(th);
      v.k[1] = r * sin(th);
      shell = 2.0 * kRefPi * r;
    }
    v.amp = sqrt(2.0 * shell * S * P.kDelta[0] / (pow(2.0 * kRefPi, (double)P.nDim) * (double)nd));
    return v;
  }
  if (P.corrMod == 1) {
    v.amp = sqrt(gauss_spectrum(v.k, P.nDim));
  } else {
    v.amp = (v.ref == 5) ? 1.0 : 0.0;  // cm_COS, spectra_RF.f90:210-220
  }
  return v;
}

// Byte offset of B element (row, kel) inside one stage of the tcgen05
// layout: K-major core matrices of 8 rows x 8 elements (128 contiguous
// bytes); K groups of 8 elements are bRows*16 bytes apart (the descriptor's
// leading byte offset), 8-row groups 128 bytes apart (stride byte offset).
__device__ __forceinline__ int64_t tc_b_offset(int32_t bRows, int32_t row, int32_t kel) {
  return (int64_t)(kel >> 3) * (bRows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (kel & 7) * 2;
}
// The same core-matrix layout for 8-bit elements (16 elements per 16-byte row).
__device__ __forceinline__ int64_t tc_b_offset8(int32_t bRows, int32_t row, int32_t kel) {
  return (int64_t)(kel >> 4) * (bRows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (kel & 15);
}

__device__ __forceinline__ unsigned char to_e4m3(double v) {
  return (unsigned char)__nv_cvt_double_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
}
__device__ __forceinline__ double from_e4m3(unsigned char b) {
  return (double)__half2float(__half(__nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)b, __NV_E4M3)));
}

// Element tid = kk * nmcPad + r of the operand: B rows of wavevector kk (in
// kernel order) for realization column r, and the wavevector itself (r = 0).
__device__ __forceinline__ void table_element(const Plan& P, const JumpTable& jt, void* __restrict__ B,
                                              double* __restrict__ ktab, int64_t literalSlab, int64_t nSlab,
                                              int64_t tid) {
  const int64_t total = P.nChunks * P.chunkK;
  const int r = (int)(tid % P.nmcPad);
  const int64_t kk = tid / P.nmcPad;
  if (kk >= total) return;
  const KVal v = kvalue(P, jt, kk);
  const int64_t stage = kk / P.chunkK;
  const int32_t c = (int32_t)(kk % P.chunkK);

  if (ktab && r == 0) {
    // k / 2 pi in FP64 and as fixed point with 30 fraction bits (range
    // |k / 2 pi| < 2; every table has |k_d| <= kMax <= 7.36 < 4 pi), and k in
    // FP32 (radians).  GEN_TABLE plans have chunkK == kTableChunk.
    double* kt = ktab + stage * kKtabStageDoubles;
    int32_t* kc = reinterpret_cast<int32_t*>(kt + 3 * kTableChunk);
    float* kf = reinterpret_cast<float*>(kc + 3 * kTableChunk);
    for (int d = 0; d < 3; ++d) {
      const double t = v.k[d] / 6.283185307179586;
      kt[d * kTableChunk + c] = t;
      kc[d * kTableChunk + c] = (fabs(t) < 2.0) ? (int32_t)llrint(t * 0x1p30) : 0;
      kf[d * kTableChunk + c] = (float)v.k[d];
    }
  }

  double bc = 0.0, bs = 0.0;
  if (v.ref >= 0 && r < P.nmcBlk) {
    const int64_t rg = (int64_t)P.rOff + r;  // realization index in the request
    double phi, gam = 1.0, amp = v.amp;
    const int64_t s1 = P.ig1, s2 = P.ig2;
    if (P.method != 1) {
      // randomization: the phases follow the nDim*kn wavevector draws
      const int64_t skip = (P.method == 3) ? (P.K >> (P.nDim - 1)) * P.nDim : 0;
      phi = 2.0 * kRefPi * r8_uni_at(jt, s1, s2, (uint64_t)(skip + rg * P.K + v.ref + 1));
      if (P.literal && literalSlab >= 0) {
        // B1: slab m of realization n uses S^(1/2^t), t = (n-1)*nSlab + m
        // (randomFieldND.f90:312 inside the loops :276 and :284).
        const double S = (P.corrMod == 1) ? gauss_spectrum(v.k, P.nDim) : ((v.ref == 5) ? 1.0 : 0.0);
        int64_t t = rg * nSlab + literalSlab + 1;
        if (t > 200) t = 200;  // the iterate is exactly 1.0 (or 0.0) long before
        amp = S;
        for (int64_t i = 0; i < t; ++i) amp = sqrt(amp);
      }
    } else {
      const int64_t base = (P.nDim == 3 ? 2 : 1) * P.K + rg * 2 * P.K;
      const double ug = r8_uni_at(jt, s1, s2, (uint64_t)(base + v.ref + 1));
      const double up = r8_uni_at(jt, s1, s2, (uint64_t)(base + P.K + v.ref + 1));
      gam = (double)sqrtf(12.0f) * (ug - 0.5);  // randomFieldND.f90:468 (single-precision sqrt(12.0))
      phi = 2.0 * kRefPi * up;
    }
    const double a = amp * gam;
    bc = a * cos(phi);
    bs = -a * sin(phi);
  }

  if (P.prec == PREC_FP32) {
    float* b = reinterpret_cast<float*>(B) + stage * (int64_t)(2 * P.chunkK) * P.nmcPad;
    b[(int64_t)(2 * c) * P.nmcPad + r] = (float)bc;
    b[(int64_t)(2 * c + 1) * P.nmcPad + r] = (float)bs;
    return;
  }
  unsigned char* b = reinterpret_cast<unsigned char*>(B) + stage_offset(P, stage);
  if (P.prec == PREC_FP8) {  // scaled e4m3, hi and lo rows
    const double sc = ldexp(1.0, P.bScaleLog2);
    const unsigned char hc = to_e4m3(bc * sc), hs = to_e4m3(bs * sc);
    b[tc_b_offset8(P.bRows, r, 2 * c)] = hc;
    b[tc_b_offset8(P.bRows, r, 2 * c + 1)] = hs;
    b[tc_b_offset8(P.bRows, P.nmcPad + r, 2 * c)] = to_e4m3(bc * sc - from_e4m3(hc));
    b[tc_b_offset8(P.bRows, P.nmcPad + r, 2 * c + 1)] = to_e4m3(bs * sc - from_e4m3(hs));
    return;
  }
  if (P.prec == PREC_FP16) {
    const double sc = ldexp(1.0, P.bScaleLog2);
    *reinterpret_cast<__half*>(b + tc_b_offset(P.bRows, r, 2 * c)) = __double2half(bc * sc);
    *reinterpret_cast<__half*>(b + tc_b_offset(P.bRows, r, 2 * c + 1)) = __double2half(bs * sc);
    return;
  }
  // a stage without the lo rows is laid out for nmcPad rows
  const bool lo = stage_has_lo(P, stage);
  const int32_t rowsS = lo ? P.bRows : P.nmcPad;
  const __nv_bfloat16 hc = __double2bfloat16(bc), hs = __double2bfloat16(bs);
  *reinterpret_cast<__nv_bfloat16*>(b + tc_b_offset(rowsS, r, 2 * c)) = hc;
  *reinterpret_cast<__nv_bfloat16*>(b + tc_b_offset(rowsS, r, 2 * c + 1)) = hs;
  if (P.prec == PREC_BF16 && lo) {  // hi/lo split of the amplitude side
    const __nv_bfloat16 lc = __double2bfloat16(bc - (double)__bfloat162float(hc));
    const __nv_bfloat16 ls = __double2bfloat16(bs - (double)__bfloat162float(hs));
    *reinterpret_cast<__nv_bfloat16*>(b + tc_b_offset(P.bRows, P.nmcPad + r, 2 * c)) = lc;
    *reinterpret_cast<__nv_bfloat16*>(b + tc_b_offset(P.bRows, P.nmcPad + r, 2 * c + 1)) = ls;
  }
}

__global__ void rf_tables_kernel(const Plan P, const JumpTable jt, void* __restrict__ B, double* __restrict__ ktab,
                                 int64_t literalSlab, int64_t nSlab) {
  table_element(P, jt, B, ktab, literalSlab, nSlab, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// Grouped builder: a grid-stride loop over the concatenated elements of all
// units (a fixed grid, so that the launch can sit in a captured graph).
__global__ void rf_group_tables_kernel(const GroupSub* __restrict__ subs, const int64_t* __restrict__ prefix,
                                       const int32_t* __restrict__ nsubsPtr, const JumpTable jt) {
  const int32_t nsubs = *nsubsPtr;
  const int64_t total = prefix[nsubs];
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int32_t lo = 0, hi = nsubs - 1;  // last unit whose prefix <= t
    while (lo < hi) {
      const int32_t mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const GroupSub& u = subs[lo];
    table_element(u.P, jt, u.B, u.ktab, -1, 1, t - prefix[lo]);
  }
}

cudaError_t launch_group_tables(const GroupSub* subs, const int64_t* prefix, const int32_t* nsubs,
                                const JumpTable& jt, int blocks, cudaStream_t st) {
  rf_group_tables_kernel<<<blocks, 256, 0, st>>>(subs, prefix, nsubs, jt);
  return cudaGetLastError();
}

cudaError_t launch_tables(const Plan& P, const JumpTable& jt, void* dB, double* dKtab, int64_t literalSlab,
                          int64_t nSlab, cudaStream_t st) {
  const int64_t total = P.nChunks * P.chunkK * P.nmcPad;
  const int threads = 256;
  const int64_t blocks = (total + threads - 1) / threads;
  rf_tables_kernel<<<(unsigned)blocks, threads, 0, st>>>(P, jt, dB, dKtab, literalSlab, nSlab);
  return cudaGetLastError();
}

}  // namespace rfb
