// rf_gen.cuh -- trig-tile generators shared by the tcgen05 and FP32 kernels.
//
// A trig tile holds, for 128 points and a stage of wavevectors, the pair
// (cos(k.x), sin(k.x)) of every (point, k).  Two generators:
//   GEN_TABLE  explicit wavevector table: FP64 phase k.x in turns, reduced
//              modulo one turn, SFU sincos (one MUFU sin + cos per pair);
//   GEN_GRID3  3-D tensor-grid wavevectors k = (i1 d1, s2 i2 d2, s3 i3 d3)
//              (spectra_RF.f90:87-133): per-axis FP64-reduced tables
//              E_d(i) = exp(i k_d(i) x_d) per point and angle addition
//              exp(i k.x) = E1 E2^{s2} E3^{s3}; P = E1 E2^{s2} is fixed for a
//              stage and each E3 entry yields both signs s3 from four
//              products.  lPad (axis-3 length padded) is a multiple of 8.
#pragma once
#include "rf_device.cuh"

namespace rfb {

// Kernel order of GEN_GRID3: a stage holds gps consecutive outer groups
// (i1, i2, s2), group g = i1 + n1*(i2 + n2*s2); inside a group, column
// c in [0, 2*lPad): half h = c / lPad, cc = c % lPad, i3 = h*(lPad/2) + cc/2,
// s3 = cc & 1.  Returns the reference index k = q*n1*n2*n3 +
// i1 + n1*(i2 + n2*i3) with the quadrant q = 2*s2 + s3 of set_kSign
// (spectra_RF.f90:267-286), or -1 for a padding column (i3 >= n3).
__host__ __device__ inline int64_t grid3_ref_index(const int32_t* kn, int32_t lPad, int64_t group, int32_t c,
                                                   int32_t* i_out, int32_t* s_out) {
  const int64_t n1 = kn[0], n2 = kn[1], n3 = kn[2];
  const int32_t i1 = (int32_t)(group % n1);
  const int64_t t = group / n1;
  const int32_t i2 = (int32_t)(t % n2);
  const int32_t s2 = (int32_t)(t / n2);
  const int32_t h = c / lPad, cc = c % lPad;
  const int32_t i3 = h * (lPad / 2) + cc / 2;
  const int32_t s3 = cc & 1;
  if (i_out) { i_out[0] = i1; i_out[1] = i2; i_out[2] = i3; }
  if (s_out) { s_out[0] = 0; s_out[1] = s2; s_out[2] = s3; }
  if (i3 >= n3) return -1;
  return (int64_t)(2 * s2 + s3) * n1 * n2 * n3 + i1 + n1 * ((int64_t)i2 + n2 * i3);
}

// exp(i * k_d(i) * x_d) with k_d(i) = 0 + kDelta_d * i (setGrid from 0,
// spectra_RF.f90:118): FP64 phase, Cody-Waite reduction, accurate FP32 sincos.
__device__ __forceinline__ float2 axis_phasor(double kDelta, int32_t i, double x) {
  const double k = 0.0 + kDelta * (double)i;
  const float r = (float)reduce_2pi(k * x);
  float s, c;
  sincosf(r, &s, &c);
  return make_float2(c, s);
}

// Per-thread GEN_GRID3 state: this thread's half of the axis-3 phasors as
// pairs of entries, c2[u] = (cos_2u, cos_2u+1), d2[u] = (sin_2u, sin_2u+1),
// the layout the packed FP32x2 arithmetic of grid3_pairs consumes.
struct Grid3Thread {
  float2 c2[kMaxGridN / 4];
  float2 d2[kMaxGridN / 4];
};

// Fill the entries i3 = h*LH + t, t < LH (LH = LPAD/2, a multiple of 4).
// LPAD is a compile-time constant so that every loop over the stage is
// straight-line code: guarded unrolled loops cost the warp a branch
// resolution per iteration.
template <int LPAD>
__device__ __forceinline__ void grid3_thread_setup(Grid3Thread& g, const Plan& P, int h, const double* x) {
  constexpr int LH = LPAD / 2;
#pragma unroll
  for (int u = 0; u < LH / 2; ++u) {
    const float2 e0 = axis_phasor(P.kDelta[2], h * LH + 2 * u, x[2]);
    const float2 e1 = axis_phasor(P.kDelta[2], h * LH + 2 * u + 1, x[2]);
    g.c2[u] = make_float2(e0.x, e1.x);
    g.d2[u] = make_float2(e0.y, e1.y);
  }
}

// Outer index (i1, i2, s2) of group g = i1 + n1*(i2 + n2*s2), advanced by
// one group at a time without integer division.
struct Grid3Outer {
  int i1 = 0, i2 = 0, s2 = 0;
  __device__ __forceinline__ void next(int n1, int n2) {
    if (++i1 == n1) {
      i1 = 0;
      if (++i2 == n2) {
        i2 = 0;
        ++s2;
      }
    }
  }
};

// Outer phasor P = E1(i1) * E2(i2)^{s2} from the shared table
// e12[(i)*128 + row] (i < n1: axis 1; n1 <= i < n1+n2: axis 2).
__device__ __forceinline__ float2 grid3_outer(const Plan& P, const float2* e12, int row, const Grid3Outer& o) {
  const float2 e1 = e12[o.i1 * kTileM + row];
  float2 e2 = e12[(P.kNStep[0] + o.i2) * kTileM + row];
  if (o.s2) e2.y = -e2.y;
  return make_float2(e1.x * e2.x - e1.y * e2.y, e1.x * e2.y + e1.y * e2.x);
}

// Outer phasor P = E1(i1) * E2(i2)^{s2} walked group by group in registers,
// for the tensor-core forms: E1 by the recurrence E1(i1+1) = E1(i1) * E1(1),
// restarted at E1(0) = 1 on every wrap of i1 (at most n1 - 1 <= 31 FP32
// complex products, relative error below 4e-6, far under the BF16/FP16
// rounding of the tile); E2(i2) from an FP64-reduced phase at each wrap.
// The FP32 plain form keeps the accurate per-axis tables (grid3_outer).
struct Grid3Walk {
  float2 e1, e1step, e2;
  int i1, i2, s2;
  __device__ __forceinline__ void init(const Plan& P, const double* x) {
    i1 = i2 = s2 = 0;
    e1 = make_float2(1.f, 0.f);
    e2 = e1;
    e1step = axis_phasor(P.kDelta[0], 1, x[0]);
  }
  __device__ __forceinline__ float2 outer() const {
    const float e2y = s2 ? -e2.y : e2.y;
    return make_float2(e1.x * e2.x - e1.y * e2y, e1.x * e2y + e1.y * e2.x);
  }
  // Advance one group; the wrap test is uniform across the warp.
  __device__ __forceinline__ void next(const Plan& P, const double* x) {
    if (++i1 == P.kNStep[0]) {
      i1 = 0;
      e1 = make_float2(1.f, 0.f);
      if (++i2 == P.kNStep[1]) {
        i2 = 0;
        ++s2;
      }
      e2 = axis_phasor(P.kDelta[1], i2, x[1]);
    } else {
      e1 = make_float2(e1.x * e1step.x - e1.y * e1step.y, e1.x * e1step.y + e1.y * e1step.x);
    }
  }
};

// The 2*LH (cos, sin) pairs of one half-stage: for t < LH, pair 2t is
// P*E3(t) (s3 = +) and pair 2t+1 is P*conj(E3(t)) (s3 = -).  With P = a+ib
// and E3 = c+id, both signs share a*c and b*c:
//   P E3 = (ac - bd) + i(bc + ad),  P conj(E3) = (ac + bd) + i(bc - ad);
// two E3 entries go through one packed FP32x2 instruction (sm_100), so four
// pairs cost two multiplies and four fused multiply-adds.
template <int LPAD, typename Emit>
__device__ __forceinline__ void grid3_pairs(const Grid3Thread& g, float2 Pq, Emit&& emit) {
  constexpr int LH = LPAD / 2;
  const float2 a2 = make_float2(Pq.x, Pq.x), b2 = make_float2(Pq.y, Pq.y);
  const float2 na2 = make_float2(-Pq.x, -Pq.x), nb2 = make_float2(-Pq.y, -Pq.y);
#pragma unroll
  for (int u = 0; u < LH / 2; ++u) {
    const float2 ac = __fmul2_rn(a2, g.c2[u]);
    const float2 bc = __fmul2_rn(b2, g.c2[u]);
    const float2 rp = __ffma2_rn(nb2, g.d2[u], ac);
    const float2 rm = __ffma2_rn(b2, g.d2[u], ac);
    const float2 ip = __ffma2_rn(a2, g.d2[u], bc);
    const float2 im = __ffma2_rn(na2, g.d2[u], bc);
    emit(4 * u + 0, rp.x, ip.x);
    emit(4 * u + 1, rm.x, im.x);
    emit(4 * u + 2, rp.y, ip.y);
    emit(4 * u + 3, rm.y, im.y);
  }
}

// GEN_TABLE: (cos, sin) of k_j . x for the T wavevectors j = h * T + t,
// t < T, of a stage (column part h); kt = [3][kTableChunk] FP64
// wavevector components in turns (k / 2 pi).  The phase accumulates x.k in
// FP64 from the first axis, as DGEMM 'T' does (BLAS/dgemm.f90:246-249).
//
// Reduction modulo one turn.  FAST (the caller's bound |x.k| < 2^18 turns):
// adding 1.5 * 2^20 puts the phase on the FP64 grid of 2^-32 turns, so the
// low word of the sum is the phase modulo one turn as a signed 32-bit
// fixed-point number; an arithmetic shift keeps 2^-23 turns (the shift
// constant carries the half unit that rounds), and the integer becomes a
// float exactly through the exponent of 1.5 * 2^23.  One FP64 add and no
// conversion instruction: the conversion unit is the one the SFU sincos
// also needs.  Otherwise the integer part is removed with rint (exact).
// Both keep the angle within 2^-24 turns of the FP64 phase, inside
// [-pi, pi], where __sincosf is accurate to 2^-21.4.
template <bool FAST, int T, typename Emit>
__device__ __forceinline__ void table_pairs(const double* kt, int h, const double* x, Emit&& emit) {
  static_assert(T % 2 == 0 && T <= kTableChunk, "pairs of wavevectors per thread");
  constexpr double kShift = 1572864.0 + 0x1p-24;         // 1.5 * 2^20 + half a unit of 2^-23
  constexpr float kUnit = 6.283185307179586f * 0x1p-23f;  // radians per 2^-23 turn
  float r[T];
#pragma unroll
  for (int t = 0; t < T; t += 2) {
    const int j = h * T + t;
    const double2 k0 = *reinterpret_cast<const double2*>(kt + j);
    const double2 k1 = *reinterpret_cast<const double2*>(kt + kTableChunk + j);
    const double2 k2 = *reinterpret_cast<const double2*>(kt + 2 * kTableChunk + j);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      double th = 0.0;
      th = th + x[0] * (e ? k0.y : k0.x);
      th = th + x[1] * (e ? k1.y : k1.x);
      th = th + x[2] * (e ? k2.y : k2.x);
      if (FAST) {
        const int32_t q = __double2loint(th + kShift) >> 9;
        r[t + e] = (__int_as_float(0x4B400000 + q) - 12582912.0f) * kUnit;
      } else {
        r[t + e] = (float)(th - rint(th)) * 6.283185307179586f;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < T; ++t) {
    float s, c;
    __sincosf(r[t], &s, &c);
    emit(t, c, s);
  }
}

// GEN_TABLE for the tensor-core forms, without FP64 in the per-pair work.
// FP64 instructions issue to the sub-partition pipe the tcgen05 MMAs also
// occupy, so an FP64 phase per (point, wavevector) stalls behind the
// contraction.  Fixed point instead: with x = a + b, a = A / 4 (A integer)
// and |b| <= 1/8, and k / 2 pi = C 2^-30 + e (C integer, |e| <= 2^-31),
//   x.k = 2 pi (sum_d A_d C_d) 2^-32 + sum_d b_d k_d + 2 pi sum_d a_d e_d.
// The first term modulo 2 pi is the wrapped 32-bit integer sum (exact for
// any magnitude), kept to 2^-23 turns; the second, below 1.6 rad
// (|b| <= 1/8, |k_1| <= sqrt(3) kMax), is formed in FP32; the third is below
// 2 pi |x|_1 2^-31 and is dropped: the point takes this path when
// |x|_1 <= 128 (2^-24 turns).  The angle lies in [-1.51 pi, 1.51 pi] and
// carries at most 9e-7 rad of error (rms 2.4e-7); __sincosf measured on this
// range stays within 7.1e-7 of sin and cos (4.0e-7 on [-pi, pi]).  All of
// it is far below the 16-bit rounding of the trig tile.  Other points take
// the FP64 table_pairs, as does the plain FP32 form.
struct FxpPoint {
  int32_t A[3];
  float b[3];
  bool ok;
};

__device__ __forceinline__ FxpPoint fxp_point(const double* x, double kMax) {
  FxpPoint f;
  // |k / 2 pi| <= kMax / 2 pi < 2 keeps C within int32
  f.ok = (fabs(x[0]) + fabs(x[1]) + fabs(x[2])) <= 128.0 && kMax < 4.0 * 3.141592653589793;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double a = f.ok ? rint(x[d] * 4.0) : 0.0;
    f.A[d] = (int32_t)a;
    f.b[d] = (float)(x[d] - 0.25 * a);
  }
  return f;
}

// The T pairs j = h * T + t of a stage (T a multiple of 4) from the fixed
// point and FP32 arrays of the stage's wavevector chunk kt.
template <int T, typename Emit>
__device__ __forceinline__ void table_pairs_fxp(const double* kt, int h, const FxpPoint& f, Emit&& emit) {
  static_assert(T % 4 == 0 && T <= kTableChunk, "pairs of wavevectors per thread");
  const int32_t* kc = reinterpret_cast<const int32_t*>(kt + 3 * kTableChunk);
  const float* kf = reinterpret_cast<const float*>(kc + 3 * kTableChunk);
  constexpr float kUnit = 6.283185307179586f * 0x1p-23f;  // radians per 2^-23 turn
  float r[T];
#pragma unroll
  for (int t = 0; t < T; t += 4) {
    const int j = h * T + t;
    const int4 c0 = *reinterpret_cast<const int4*>(kc + j);
    const int4 c1 = *reinterpret_cast<const int4*>(kc + kTableChunk + j);
    const int4 c2 = *reinterpret_cast<const int4*>(kc + 2 * kTableChunk + j);
    const float4 f0 = *reinterpret_cast<const float4*>(kf + j);  // k in radians, FP32
    const float4 f1 = *reinterpret_cast<const float4*>(kf + kTableChunk + j);
    const float4 f2 = *reinterpret_cast<const float4*>(kf + 2 * kTableChunk + j);
    const int32_t cc[3][4] = {{c0.x, c0.y, c0.z, c0.w}, {c1.x, c1.y, c1.z, c1.w}, {c2.x, c2.y, c2.z, c2.w}};
    const float ff[3][4] = {{f0.x, f0.y, f0.z, f0.w}, {f1.x, f1.y, f1.z, f1.w}, {f2.x, f2.y, f2.z, f2.w}};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      // coarse term in units of 2^-32 turns, wrapping (unsigned arithmetic)
      const uint32_t P = (uint32_t)f.A[0] * (uint32_t)cc[0][e] + (uint32_t)f.A[1] * (uint32_t)cc[1][e] +
                         (uint32_t)f.A[2] * (uint32_t)cc[2][e];
      // fine term in radians, plus half a unit of 2^-23 turn: the shift
      // below truncates, so the sum rounds
      const float s = fmaf(f.b[2], ff[2][e], fmaf(f.b[1], ff[1][e], fmaf(f.b[0], ff[0][e], 0.5f * kUnit)));
      // to units of 2^-23 turns, as a float through the exponent of 1.5 * 2^23
      const int32_t q = (int32_t)P >> 9;
      const float qf = __int_as_float(0x4B400000 + q) - 12582912.0f;
      r[t + e] = fmaf(qf, kUnit, s);
    }
  }
#pragma unroll
  for (int t = 0; t < T; ++t) {
    float s, c;
    __sincosf(r[t], &s, &c);
    emit(t, c, s);
  }
}

// GEN_TABLE for the tensor-core forms near the origin: the phase k.x in FP32
// (three fused multiply-adds of the FP32 wavevector and point) and
// __sincosf on it.  Rounding k and x to FP32 and the three operations leave
// at most about |k|_2 |x|_1 2^-22 rad of error, and __sincosf's argument
// reduction of an angle of n turns keeps 24 - log2(n) bits of its fraction;
// for |x|_1 kMax <= 256 (table_f32_phase) both stay below 1e-4 rad, about
// 1/20 of the 16-bit rounding of the trig tile that follows.  Five
// instructions per pair besides the two MUFU operations, against about
// twelve for the fixed-point phase.
template <int T, typename Emit>
__device__ __forceinline__ void table_pairs_f32(const double* kt, int h, const float* xf, Emit&& emit) {
  static_assert(T % 4 == 0 && T <= kTableChunk, "pairs of wavevectors per thread");
  const float* kf = reinterpret_cast<const float*>(reinterpret_cast<const int32_t*>(kt + 3 * kTableChunk) +
                                                   3 * kTableChunk);
  float r[T];
#pragma unroll
  for (int t = 0; t < T; t += 4) {
    const int j = h * T + t;
    const float4 f0 = *reinterpret_cast<const float4*>(kf + j);
    const float4 f1 = *reinterpret_cast<const float4*>(kf + kTableChunk + j);
    const float4 f2 = *reinterpret_cast<const float4*>(kf + 2 * kTableChunk + j);
    r[t + 0] = fmaf(xf[2], f2.x, fmaf(xf[1], f1.x, xf[0] * f0.x));
    r[t + 1] = fmaf(xf[2], f2.y, fmaf(xf[1], f1.y, xf[0] * f0.y));
    r[t + 2] = fmaf(xf[2], f2.z, fmaf(xf[1], f1.z, xf[0] * f0.z));
    r[t + 3] = fmaf(xf[2], f2.w, fmaf(xf[1], f1.w, xf[0] * f0.w));
  }
#pragma unroll
  for (int t = 0; t < T; ++t) {
    float s, c;
    __sincosf(r[t], &s, &c);
    emit(t, c, s);
  }
}
__device__ __forceinline__ bool table_f32_phase(const double* x, double kMax) {
  return (fabs(x[0]) + fabs(x[1]) + fabs(x[2])) * kMax <= 256.0;
}

// Whether a point may take the FAST reduction of table_pairs: |x.k| / 2 pi is
// below 2^18 turns for every |k_d| <= kMax (every table's bound).
__device__ __forceinline__ bool table_fast_phase(const double* x, double kMax) {
  return (fabs(x[0]) + fabs(x[1]) + fabs(x[2])) * kMax < 0x1p18 * 6.283185307179586;
}

}  // namespace rfb
