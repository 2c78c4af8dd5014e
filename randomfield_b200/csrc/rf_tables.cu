// rf_tables.cu -- device builder of the contraction operand.
//
// The Shinozuka sum f(x, r) = ampMult * sum_k a_k cos(k.x + phi_{k,r})
// (randomFieldND.f90:276-330) is evaluated as the contraction
//   f = ampMult * [cos(Kx) | sin(Kx)] (points x 2K)  *  B (2K x Nmc),
//   B[2k, r] = a_k cos(phi_{k,r}),  B[2k+1, r] = -a_k sin(phi_{k,r}).
// One thread per (run, realization): a run is a set of wavevectors whose
// reference indices are consecutive (GEN_GRID3: the n1 values of i1 at fixed
// (i2, s2, column); the other generators: kRun consecutive wavevectors), so
// the draws a thread needs are consecutive calls of the generator.  The
// phases come from the rnglib stream (rnglib.f90:548-659): the p-th draw of
// generator 1 is (a1^p s1 mod m1) - (a2^p s2 mod m2) folded; a thread jumps
// ahead once per stream (square-and-multiply) and then steps one call at a
// time (DrawCursor), and the table matches a sequential run draw for draw.
// Draw order follows the reference: Shinozuka K phases per realization in k
// order (:278-279); isotropic direction blocks then, per realization, a gamma
// block and a psi block (:460-468 restated).
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

// Position in one rnglib stream: the state after `pos` calls (pos = 0: not
// set).  A draw at pos + 1 costs one step (two modular products); any other
// position a jump-ahead.
struct DrawCursor {
  int64_t c1, c2;
  uint64_t pos;
  int32_t last;  // i4_uni value of call `pos`
};

// r8_uni_01 of the p-th call (p >= 1), through the cursor; the caller's
// draw p - 1 where the request supplies its own stream.
__device__ __forceinline__ double draw_r8(const Plan& P, const JumpTable& jt, int64_t s1, int64_t s2, DrawCursor& cur,
                                          uint64_t p) {
  if (P.dDraws) {
    cur.pos = p;
    cur.last = 0;
    return P.dDraws[p - 1];
  }
  if (cur.pos != 0 && p == cur.pos + 1) uni_state_next(jt, cur.c1, cur.c2);
  else if (p != cur.pos) uni_state_at(jt, s1, s2, p, cur.c1, cur.c2);
  cur.pos = p;
  cur.last = uni_value(cur.c1, cur.c2);
  return (double)cur.last * kR8Scale;
}

// Where the draw export (rf_debug_table_draws) writes the i4_uni values the
// builder consumed, in reference order: per (realization, wavevector) the
// phase draw (isotropic: gamma, then psi), and per wavevector the isotropic
// direction draws (theta, then phi in 3-D).  Null in the operand builds.
struct DrawSink {
  int32_t* rk;
  int32_t* k;
};

// The streams a run draws from: wavevector draws (randomization bases,
// isotropic directions phi and theta) and per-realization draws (phase, or
// isotropic gamma and psi).
struct RunCursors {
  DrawCursor kA, kB, rA, rB;
};

__device__ KVal kvalue(const Plan& P, const JumpTable& jt, int64_t kk, RunCursors& cu) {
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
          (P.method == 3) ? draw_r8(P, jt, P.ig1, P.ig2, cu.kA, (uint64_t)(b * P.nDim + d + 1)) * P.kMax
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
    const double uth = draw_r8(P, jt, (int64_t)s1, (int64_t)s2, cu.kA, (uint64_t)((P.nDim == 3 ? K : 0) + kk + 1));
    const double th = 2.0 * kRefPi * uth;
    double S;
    if (P.corrMod == 1) S = exp(-((r * r) * 1.0) / (4.0 * kRefPi));
    else S = (j == 5) ? 1.0 : 0.0;
    double shell;
    if (P.nDim == 3) {
      const double uphi = draw_r8(P, jt, (int64_t)s1, (int64_t)s2, cu.kB, (uint64_t)(kk + 1));
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

// Element (kk, r) of the operand: B rows of wavevector kk (in kernel order)
// for realization column r, and the wavevector itself (r = 0).
// SINK: write the consumed draws to `sink` instead of the operand.
template <bool SINK>
__device__ __forceinline__ void table_element(const Plan& P, const JumpTable& jt, void* __restrict__ B,
                                              double* __restrict__ ktab, int64_t literalSlab, int64_t nSlab,
                                              int64_t kk, int r, RunCursors& cu, const DrawSink& sink) {
  const KVal v = kvalue(P, jt, kk, cu);
  const int64_t stage = kk / P.chunkK;
  const int32_t c = (int32_t)(kk % P.chunkK);

  if (!SINK && ktab && r == 0) {
    // k / 2 pi in FP64 and as fixed point with 30 fraction bits (range
    // |k / 2 pi| < 2; every table has |k_d| <= kMax <= 7.36 < 4 pi), and k in
    // FP32 (radians).  GEN_TABLE plans have chunkK == kTableChunk.
    double* kt = ktab + stage * kKtabStageDoubles;
    int32_t* kc = reinterpret_cast<int32_t*>(kt + 3 * kTableChunk);
    float* kf = reinterpret_cast<float*>(kc + 3 * kTableChunk);
    if (!RF_IN_BOUNDS(stage, P.nChunks, P.dbgErr)) return;
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
      phi = 2.0 * kRefPi * draw_r8(P, jt, s1, s2, cu.rA, (uint64_t)(skip + rg * P.K + v.ref + 1));
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
      const double ug = draw_r8(P, jt, s1, s2, cu.rA, (uint64_t)(base + v.ref + 1));
      const double up = draw_r8(P, jt, s1, s2, cu.rB, (uint64_t)(base + P.K + v.ref + 1));
      gam = (double)sqrtf(12.0f) * (ug - 0.5);  // randomFieldND.f90:468 (single-precision sqrt(12.0))
      phi = 2.0 * kRefPi * up;
    }
    const double a = amp * gam;
    bc = a * cos(phi);
    bs = -a * sin(phi);
  }
  if (SINK) {
    if (v.ref < 0) return;
    if (P.method == 1 && r == 0 && sink.k) {
      sink.k[v.ref * 2] = cu.kA.last;
      sink.k[v.ref * 2 + 1] = P.nDim == 3 ? cu.kB.last : 0;
    }
    if (r < P.nmcBlk) {
      const int64_t rg = (int64_t)P.rOff + r;
      if (P.method == 1) {
        sink.rk[(rg * P.K + v.ref) * 2] = cu.rA.last;
        sink.rk[(rg * P.K + v.ref) * 2 + 1] = cu.rB.last;
      } else {
        sink.rk[rg * P.K + v.ref] = cu.rA.last;
      }
    }
    return;
  }

  // every operand write of this element lies in stage `stage` of B
  if (!RF_IN_BOUNDS(stage_offset(P, stage), operand_bytes(P), P.dbgErr)) return;
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

// Run j's element i (i < table_run_length) in kernel order.  GEN_GRID3: run
// j = cc + gw (i2 + n2 s2) holds column cc of the groups g = i + n1 (i2 +
// n2 s2), whose reference indices are consecutive in i = i1
// (grid3_ref_index); the other generators keep the reference order.
__device__ __forceinline__ int64_t table_run_kk(const Plan& P, int64_t j, int32_t i) {
  if (P.gen == GEN_GRID3) {
    const int32_t gw = 2 * P.lPad;
    const int64_t cc = j % gw, g = (int64_t)i + (int64_t)P.kNStep[0] * (j / gw);
    return (g / P.gps) * P.chunkK + (g % P.gps) * gw + cc;
  }
  return j * kRun + i;
}
__device__ __forceinline__ int32_t table_run_length(const Plan& P, int64_t j) {
  if (P.gen == GEN_GRID3) return P.kNStep[0];
  const int64_t left = P.nChunks * P.chunkK - j * kRun;
  return (int32_t)(left < kRun ? left : kRun);
}

// GEN_OUTER operand.  For the outer group g = (i1, i2, s2), axis-3 index i3
// and realization r, the two wavevectors s3 = +/- give C+- = a+- e^{i phi+-};
// with P = C+ + C-, Q = C+ - C- the field's term is
//   Re[E1 E2^{s2} (P cos(k3 x3) + i Q sin(k3 x3))]
//     = pr c3 Re P - pi c3 Im P - pr s3 Im Q - pi s3 Re Q
// (pr, pi: the outer phasor, the A operand; c3, s3: the epilogue's factors),
// so B row (g, re) holds (Re P, -Im Q) and row (g, im) holds (-Im P, -Re Q)
// in the (i3, cos) and (i3, sin) columns of realization r.  In terms of the
// plain operand's pair (a cos phi, -a sin phi) = (bc, bs):
//   W(re, cos) = bc+ + bc-,  W(im, cos) = bs+ + bs-,
//   W(re, sin) = bs+ - bs-,  W(im, sin) = bc- - bc+.
// W of group (i1, i2, s2), axis-3 index i3 and realization column rc (zero
// in the padding); with SINK the draws are recorded instead.  The amplitude
// sqrt(S(k)) is the FP64 product of the per-axis factors exp(-k_d^2 / 8 pi)
// (a23: axes 2 and 3, fixed per run), the draws are rnglib's to the bit (the
// s3 = - draw from the s3 = + one by the plan's multiplier, one modular
// product per stream), and cos, sin of the phase 2 pi U are FP32 (sincospi
// of 2U; the operand is stored as 16-bit hi/lo pairs, about 16 bits).
template <bool SINK>
__device__ __forceinline__ void outer_w(const Plan& P, const JumpTable& jt, int32_t i1, int32_t i2, int32_t s2,
                                        int32_t i3, int32_t rc, double a23, RunCursors& cu, const DrawSink& sink,
                                        float W[4]) {
  const int32_t n1 = P.kNStep[0], n2 = P.kNStep[1], n3 = P.kNStep[2];
  W[0] = W[1] = W[2] = W[3] = 0.f;  // (re, cos), (im, cos), (re, sin), (im, sin)
  if (i1 < n1 && i3 < n3 && rc < P.nmcBlk) {
    const int64_t n123 = (int64_t)n1 * n2 * n3;
    const int64_t refP = (int64_t)(2 * s2) * n123 + i1 + (int64_t)n1 * (i2 + (int64_t)n2 * i3);
    const int64_t refM = refP + n123;
    const int64_t rg = (int64_t)P.rOff + rc;
    double aP, aM;
    if (P.corrMod == 1) {
      const double k1 = 0.0 + P.kDelta[0] * (double)i1;
      aP = aM = a23 * exp(-(k1 * k1) / (8.0 * kRefPi));  // S(k) is even in k3
    } else {
      aP = (refP == 5) ? 1.0 : 0.0;  // cm_COS, spectra_RF.f90:210-220
      aM = (refM == 5) ? 1.0 : 0.0;
    }
    double uP, uM;
    if (P.dDraws) {
      uP = draw_r8(P, jt, P.ig1, P.ig2, cu.rA, (uint64_t)(rg * P.K + refP + 1));
      uM = draw_r8(P, jt, P.ig1, P.ig2, cu.rB, (uint64_t)(rg * P.K + refM + 1));
    } else {
      uP = draw_r8(P, jt, P.ig1, P.ig2, cu.rA, (uint64_t)(rg * P.K + refP + 1));
      cu.rB.c1 = mulmod(P.oStepM1, cu.rA.c1, kM1);
      cu.rB.c2 = mulmod(P.oStepM2, cu.rA.c2, kM2);
      cu.rB.pos = cu.rA.pos + (uint64_t)n123;
      cu.rB.last = uni_value(cu.rB.c1, cu.rB.c2);
      uM = (double)cu.rB.last * kR8Scale;
    }
    if (SINK) {
      sink.rk[rg * P.K + refP] = cu.rA.last;
      sink.rk[rg * P.K + refM] = cu.rB.last;
      return;
    }
    float sP, cP, sM, cM;
    sincospif((float)(2.0 * uP), &sP, &cP);
    sincospif((float)(2.0 * uM), &sM, &cM);
    const float fP = (float)aP, fM = (float)aM;
    // bc = a cos phi, bs = -a sin phi
    W[0] = fP * cP + fM * cM;
    W[1] = -(fP * sP + fM * sM);
    W[2] = fM * sM - fP * sP;
    W[3] = fM * cM - fP * cP;
  }
}

// Two 16-bit values of the operand in one word (a: low half): BF16, or
// FP16 scaled by 2^bScaleLog2; *res gets the BF16 rounding residuals.
__device__ __forceinline__ uint32_t outer_pack(const Plan& P, float a, float b, uint32_t* res) {
  if (P.prec == PREC_FP16) {
    const float sc = ldexpf(1.f, P.bScaleLog2);
    *res = 0u;
    return pack_f16x2(a * sc, b * sc);
  }
  const uint32_t h = pack_bf16x2(a, b);
  *res = pack_bf16x2(a - __uint_as_float(h << 16), b - __uint_as_float(h & 0xffff0000u));
  return h;
}

// One run of the GEN_OUTER operand: group (i2, s2), axis-3 index i3 and
// realization column rc over i1 = 0 .. n1p-1.  For the outer group g = (i1,
// i2, s2) the two wavevectors s3 = +/- give C+- = a+- e^{i phi+-}; with P =
// C+ + C-, Q = C+ - C- the field's term is
//   Re[E1 E2^{s2} (P cos(k3 x3) + i Q sin(k3 x3))]
//     = pr c3 Re P - pi c3 Im P - pr s3 Im Q - pi s3 Re Q
// (pr, pi: the outer phasor, the A operand; c3, s3: the epilogue's factors),
// so B row (g, re) holds (Re P, -Im Q) and row (g, im) holds (-Im P, -Re Q)
// in the (i3, cos) and (i3, sin) columns of realization r.  In terms of the
// plain operand's pair (a cos phi, -a sin phi) = (bc, bs):
//   W(re, cos) = bc+ + bc-,  W(im, cos) = bs+ + bs-,
//   W(re, sin) = bs+ - bs-,  W(im, sin) = bc- - bc+.
// K-step j = outer_kstep(i1 / 8, i2, s2) holds element k = 2 (i1 % 8) + e
// of rows n = rl 2 lPad + 2 i3 + cs (cs = 0 cos, 1 sin): the run owns two
// rows of every K-step block, and each four consecutive i1 fill one 16-byte
// core-matrix row of each, stored whole (neighbouring threads hold the
// neighbouring rows, so a warp's stores fill whole lines).
template <bool SINK>
__device__ __forceinline__ void outer_run(const Plan& P, const JumpTable& jt, unsigned char* __restrict__ B,
                                          int32_t i2, int32_t s2, int32_t i3, int32_t rc, RunCursors& cu,
                                          const DrawSink& sink) {
  // realization column rc -> chunk c, block rows nRows, row0 of (cs = 0)
  // (cs = 1 is the next row) and the byte offset of that block in the chunk
  int32_t c, nRows, row0;
  int64_t part = 0, inblk = 0;  // CTA-pair form: the rank's part of the chunk; the half inside a K-step block
  if (P.oPair) {
    const int32_t per = 2 * P.oRc;  // realizations per chunk
    c = rc / per;
    const int32_t hh = (rc % per) / P.oRc, rl = rc % P.oRc;
    const int32_t half = P.lPad * P.oRc;  // rows of a half per rank
    const int32_t nh = rl * 2 * P.lPad + 2 * i3;  // column of the half
    const int32_t rank = nh / half;
    nRows = half;
    row0 = nh % half;
    part = (int64_t)rank * (P.oChunkBytes / 2);
    inblk = (int64_t)hh * (half * 32);
  } else {
    c = rc / P.oRc;
    const int32_t rl = rc % P.oRc;
    nRows = 2 * P.lPad * P.oRc;
    row0 = rl * 2 * P.lPad + 2 * i3;
  }
  const double k2 = 0.0 + P.kDelta[1] * (double)i2, k3 = 0.0 + P.kDelta[2] * (double)i3;
  const double a23 = exp(-(k2 * k2) / (8.0 * kRefPi)) * exp(-(k3 * k3) / (8.0 * kRefPi));
  for (int32_t i0 = 0; i0 < P.n1p; i0 += 4) {  // n1p is a multiple of 8
    float W[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) outer_w<SINK>(P, jt, i0 + u, i2, s2, i3, rc, a23, cu, sink, W[u]);
    if (SINK) continue;
    const int32_t i1 = i0 + 3;
    const int64_t j = outer_kstep(P, i1 >> 3, i2, s2);
    const int64_t base = (int64_t)c * P.oChunkBytes + part + outer_kstep_offset(P, j);
    const bool blo = outer_b_lo(P, j);
    if (!RF_IN_BOUNDS(base + (blo ? 2 : 1) * P.oKstepBytes - 1, operand_bytes(P), P.dbgErr)) continue;
    const int64_t kh = (i1 >> 2) & 1;  // which K half of the K-step these four groups fill
    if (blo && P.oTf32) {
      // TF32 K-step: the block of MMA kh (K = 8: groups 4 kh .. 4 kh + 3),
      // its first core-matrix column groups 4 kh, 4 kh + 1 and its second
      // 4 kh + 2, 4 kh + 3, each group (re, im)
#pragma unroll
      for (int cs = 0; cs < 2; ++cs) {
        const int32_t row = row0 + cs;
        unsigned char* dst = B + base + kh * P.oKstepBytes + inblk + (row >> 3) * 128 + (row & 7) * 16;
        *reinterpret_cast<uint4*>(dst) = make_uint4(tf32_bits(W[0][2 * cs]), tf32_bits(W[0][2 * cs + 1]),
                                                    tf32_bits(W[1][2 * cs]), tf32_bits(W[1][2 * cs + 1]));
        *reinterpret_cast<uint4*>(dst + nRows * 16) = make_uint4(tf32_bits(W[2][2 * cs]), tf32_bits(W[2][2 * cs + 1]),
                                                                 tf32_bits(W[3][2 * cs]), tf32_bits(W[3][2 * cs + 1]));
      }
      continue;
    }
    uint32_t hi[2][4], lo[2][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int cs = 0; cs < 2; ++cs) hi[cs][u] = outer_pack(P, W[u][2 * cs], W[u][2 * cs + 1], &lo[cs][u]);
    }
    const int64_t half = kh * (nRows * 16);  // K half of the block
#pragma unroll
    for (int cs = 0; cs < 2; ++cs) {
      const int32_t row = row0 + cs;
      unsigned char* dst = B + base + inblk + half + (row >> 3) * 128 + (row & 7) * 16;
      *reinterpret_cast<uint4*>(dst) = make_uint4(hi[cs][0], hi[cs][1], hi[cs][2], hi[cs][3]);
      if (blo) *reinterpret_cast<uint4*>(dst + P.oKstepBytes) = make_uint4(lo[cs][0], lo[cs][1], lo[cs][2], lo[cs][3]);
    }
  }
}

// Thread t = j * cols + r: run j for realization column r (GEN_OUTER:
// t = r * runs + j, so that neighbouring threads fill neighbouring rows).
template <bool SINK = false>
__device__ __forceinline__ void table_run(const Plan& P, const JumpTable& jt, void* __restrict__ B,
                                         double* __restrict__ ktab, int64_t literalSlab, int64_t nSlab, int64_t t,
                                         const DrawSink& sink = DrawSink{nullptr, nullptr}) {
  const int32_t cols = table_cols(P);
  const int64_t runs = table_runs(P);
  const bool outer = P.gen == GEN_OUTER;
  const int64_t j = outer ? t % runs : t / cols;
  const int r = (int)(outer ? t / runs : t % cols);
  if (j >= runs || r >= cols) return;
  RunCursors cu;
  cu.kA.pos = cu.kB.pos = cu.rA.pos = cu.rB.pos = 0;
  cu.kA.last = cu.kB.last = cu.rA.last = cu.rB.last = 0;
  if (outer) {
    // run j = i3 + lPad (i2 + n2 s2): i1 = 0 .. n1p-1, consecutive draws per sign s3
    const int32_t i3 = (int32_t)(j % P.lPad);
    const int64_t t2 = j / P.lPad;
    const int32_t i2 = (int32_t)(t2 % P.kNStep[1]), s2 = (int32_t)(t2 / P.kNStep[1]);
    outer_run<SINK>(P, jt, reinterpret_cast<unsigned char*>(B), i2, s2, i3, r, cu, sink);
    return;
  }
  const int32_t len = table_run_length(P, j);
  for (int32_t i = 0; i < len; ++i)
    table_element<SINK>(P, jt, B, ktab, literalSlab, nSlab, table_run_kk(P, j, i), r, cu, sink);
}

__global__ void rf_tables_kernel(const Plan P, const JumpTable jt, void* __restrict__ B, double* __restrict__ ktab,
                                 int64_t literalSlab, int64_t nSlab) {
  table_run(P, jt, B, ktab, literalSlab, nSlab, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// The same runs, cursors and draw positions as rf_tables_kernel, writing the
// draws it consumes to `sink` (the bit-exact check of the device rnglib).
__global__ void rf_table_draws_kernel(const Plan P, const JumpTable jt, DrawSink sink) {
  table_run<true>(P, jt, nullptr, nullptr, -1, 1, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, sink);
}

// Grouped builder: a grid-stride loop over the concatenated run threads
// (table_threads) of all units (a fixed grid, so that the launch can sit in
// a captured graph).
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
    table_run(u.P, jt, u.B, u.ktab, -1, 1, t - prefix[lo]);
  }
}

cudaError_t launch_group_tables(const GroupSub* subs, const int64_t* prefix, const int32_t* nsubs,
                                const JumpTable& jt, int blocks, cudaStream_t st) {
  rf_group_tables_kernel<<<blocks, 256, 0, st>>>(subs, prefix, nsubs, jt);
  return cudaGetLastError();
}

cudaError_t launch_table_draws(const Plan& P, const JumpTable& jt, int32_t* dRk, int32_t* dK, cudaStream_t st) {
  const int64_t total = table_threads(P);
  const int threads = 128;
  const int64_t blocks = (total + threads - 1) / threads;
  rf_table_draws_kernel<<<(unsigned)blocks, threads, 0, st>>>(P, jt, DrawSink{dRk, dK});
  return cudaGetLastError();
}

cudaError_t launch_tables(const Plan& P, const JumpTable& jt, void* dB, double* dKtab, int64_t literalSlab,
                          int64_t nSlab, cudaStream_t st) {
  const int64_t total = table_threads(P);
  const int threads = 128;
  const int64_t blocks = (total + threads - 1) / threads;
  rf_tables_kernel<<<(unsigned)blocks, threads, 0, st>>>(P, jt, dB, dKtab, literalSlab, nSlab);
  return cudaGetLastError();
}

}  // namespace rfb
