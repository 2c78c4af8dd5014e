// rf_blend.cuh -- the localization blend in the contraction epilogues.
//
// generateUnityPartition_Matrix (localization_RF.f90:705-857) with
// partitionType 1 builds, per axis with overlapNPoints = O >= 1, the cosine
// ramp w(s) = (1 + cos(PI * s / (O + 2))) / 2, s = 1..O, applied to the last
// O points of the axis and, reversed, to the first O; the axes multiply.
// add_RF_to_Group (:199-263) multiplies a subdomain field by that partition
// and adds it into the group field at the subdomain's offset.  The epilogue
// does both per point: weight from the point's subdomain grid index, FP64
// atomic add into the group field (subdomains overlap and their tiles run on
// different CTAs).  The marginal map runs after the group's border
// correction (rf_post.cu), on the blended Gaussian field.
#pragma once
#include "rf_plan.h"

namespace rfb {

// Product of the low- and high-face ramps at index i of an axis of L points.
__device__ __forceinline__ double blend_ramp(int32_t i, int32_t L, int32_t O) {
  double w = 1.0;
  if (O < 1) return w;
  if (i < O) {  // low face: pattern reversed, s = i + 1
    const double pat = (double)(O - i) / (double)(O + 2);
    w = w * ((1.0 + cos(kRefPi * pat)) / 2.0);
  }
  if (i >= L - O) {  // high face: s = i - (L - O) + 1
    const double pat = (double)(i - (L - O) + 1) / (double)(O + 2);
    w = w * ((1.0 + cos(kRefPi * pat)) / 2.0);
  }
  return w;
}

// Partition-of-unity weight and group index of subdomain point p.
__device__ __forceinline__ double blend_weight(const Plan& P, int64_t p, int64_t* g) {
  const int32_t L1 = P.bDims[0], L2 = P.bDims[1];
  const int32_t i1 = (int32_t)(p % L1);
  const int64_t t = p / L1;
  const int32_t i2 = (int32_t)(t % L2), i3 = (int32_t)(t / L2);
  double w = blend_ramp(i1, L1, P.bRamp[0]);
  if (P.nDim > 1) w = w * blend_ramp(i2, L2, P.bRamp[1]);
  if (P.nDim > 2) w = w * blend_ramp(i3, P.bDims[2], P.bRamp[2]);
  *g = (int64_t)(P.bOrigin[0] + i1) +
       (int64_t)P.gDims[0] * ((int64_t)(P.bOrigin[1] + i2) + (int64_t)P.gDims[1] * (int64_t)(P.bOrigin[2] + i3));
  return w;
}

}  // namespace rfb
