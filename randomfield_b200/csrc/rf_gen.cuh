// rf_gen.cuh -- trig-tile generators shared by the tcgen05 and FP32 kernels.
//
// A trig tile holds, for 128 points and a stage of wavevectors, the pair
// (cos(k.x), sin(k.x)) of every (point, k).  Two generators:
//   GEN_TABLE  explicit wavevector table: FP64 phase k.x, Cody-Waite reduction
//              to [-pi, pi], SFU sincos (one MUFU sin + cos per pair);
//   GEN_GRID3  3-D tensor-grid wavevectors k = (i1 d1, s2 i2 d2, s3 i3 d3)
//              (spectra_RF.f90:87-133): per-axis FP64-reduced tables
//              E_d(i) = exp(i k_d(i) x_d) per point and angle addition
//              exp(i k.x) = E1 E2^{s2} E3^{s3}; P = E1 E2^{s2} is fixed for a
//              stage and each E3 entry yields both signs s3 from four
//              products.  lPad (axis-3 length padded) is a multiple of 8.
#pragma once
#include "rf_device.cuh"

namespace rfb {

// Kernel order of GEN_GRID3: stage g holds outer index (i1, i2, s2) with
// g = i1 + n1*(i2 + n2*s2); inside a stage, column c in [0, 2*lPad):
// half h = c / lPad, cc = c % lPad, i3 = h*(lPad/2) + cc/2, s3 = cc & 1.
// Returns the reference index k = q*n1*n2*n3 + i1 + n1*(i2 + n2*i3) with the
// quadrant q = 2*s2 + s3 of set_kSign (spectra_RF.f90:267-286), or -1 for a
// padding column (i3 >= n3).
__host__ __device__ inline int64_t grid3_ref_index(const int32_t* kn, int32_t lPad, int64_t stage, int32_t c,
                                                   int32_t* i_out, int32_t* s_out) {
  const int64_t n1 = kn[0], n2 = kn[1], n3 = kn[2];
  const int32_t i1 = (int32_t)(stage % n1);
  const int64_t t = stage / n1;
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

// Per-thread GEN_GRID3 state: this thread's half of the axis-3 phasors.
struct Grid3Thread {
  float2 e3[kMaxGridN / 2];
};

// Fill e3 for i3 = h*LH + t, t < LH.
__device__ __forceinline__ void grid3_thread_setup(Grid3Thread& g, const Plan& P, int h, const double* x) {
  const int LH = P.lPad / 2;
#pragma unroll
  for (int t = 0; t < kMaxGridN / 2; ++t) {
    if (t < LH) {
      const int i3 = h * LH + t;
      g.e3[t] = axis_phasor(P.kDelta[2], i3, x[2]);
    } else {
      g.e3[t] = make_float2(0.f, 0.f);
    }
  }
}

// Outer index (i1, i2, s2) of stage g = i1 + n1*(i2 + n2*s2), advanced by
// one stage at a time without integer division.
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

// The 2*LH (cos, sin) pairs of one half-stage: for t < LH, pair 2t is
// P*E3(t) (s3 = +) and pair 2t+1 is P*conj(E3(t)) (s3 = -).
template <typename Emit>
__device__ __forceinline__ void grid3_pairs(const Grid3Thread& g, float2 Pq, int LH, Emit&& emit) {
  const float a = Pq.x, b = Pq.y;
#pragma unroll
  for (int t = 0; t < kMaxGridN / 2; ++t) {
    if (t < LH) {
      const float c = g.e3[t].x, d = g.e3[t].y;
      const float bd = b * d, ad = a * d;
      emit(2 * t, fmaf(a, c, -bd), fmaf(b, c, ad));
      emit(2 * t + 1, fmaf(a, c, bd), fmaf(b, c, -ad));
    }
  }
}

// GEN_TABLE: (cos, sin) of k_j . x for the 16 wavevectors j = h*16 + t of a
// stage; kt = [3][kTableChunk] FP64.  The phase accumulates x.k from zero in
// axis order as DGEMM 'T' does (BLAS/dgemm.f90:246-249).
template <typename Emit>
__device__ __forceinline__ void table_pairs(const double* kt, int h, const double* x, Emit&& emit) {
#pragma unroll
  for (int t = 0; t < kTableChunk / 2; ++t) {
    const int j = h * (kTableChunk / 2) + t;
    double th = 0.0;
    th = th + x[0] * kt[j];
    th = th + x[1] * kt[kTableChunk + j];
    th = th + x[2] * kt[2 * kTableChunk + j];
    const float r = (float)reduce_2pi(th);
    float s, c;
    __sincosf(r, &s, &c);
    emit(t, c, s);
  }
}

}  // namespace rfb
