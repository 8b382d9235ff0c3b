// Detector-ray rotation, square Lambert map and bilinear master-pattern
// sampling shared by the projector (K1) and the grid refinement (K9):
// qu_apply quaternions.py:186-213, rosca_lambert_side_by_side
// sphere.py:145-185, grid_sample master_pattern.py:197-206.
#pragma once

#include "common.cuh"

namespace ebsd {

__device__ __forceinline__ float2 lambert_side_by_side(float x, float y, float z) {
  const float fac = sqrtf(fmaxf(2.0f * (1.0f - fabsf(z)), 0.0f));
  const bool cond = fabsf(y) <= fabsf(x);
  const float big = cond ? x : y;
  const float sml = cond ? y : x;
  const float sgn = big < 0.0f ? -1.0f : 1.0f;
  const float simple = sgn * fac * 0.70710678118654752f;  // 2 / sqrt(8)
  const float arct = sgn * fac * atan2f(sml * sgn, fabsf(big)) * 0.90031631615710607f;  // 2 sqrt2/pi
  float u = cond ? simple : arct;
  const float v = cond ? arct : simple;
  u = u / 2.0f - 0.5f + (z < 0.0f ? 1.0f : 0.0f);
  return make_float2(u, v);
}

// grid_sample(bilinear, padding_mode="border") of one point (u, v) in
// [-1, 1]^2 on an (h, w) image; AC = align_corners (False for dictionary
// indexing, master_pattern.py:197-206; True for grid refinement,
// refining.py:206).
template <bool AC = false>
__device__ __forceinline__ float sample_border(const float* __restrict__ img, int h, int w, float u,
                                               float v) {
  float ix, iy;
  if constexpr (AC) {
    ix = (u + 1.0f) / 2.0f * (float)(w - 1);
    iy = (v + 1.0f) / 2.0f * (float)(h - 1);
  } else {
    ix = ((u + 1.0f) * (float)w - 1.0f) / 2.0f;
    iy = ((v + 1.0f) * (float)h - 1.0f) / 2.0f;
  }
  ix = fminf(fmaxf(ix, 0.0f), (float)(w - 1));
  iy = fminf(fmaxf(iy, 0.0f), (float)(h - 1));
  const float fx0 = floorf(ix), fy0 = floorf(iy);
  const int x0 = (int)fx0, y0 = (int)fy0;
  const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
  const float wnw = (fx0 + 1.0f - ix) * (fy0 + 1.0f - iy);
  const float wne = (ix - fx0) * (fy0 + 1.0f - iy);
  const float wsw = (fx0 + 1.0f - ix) * (iy - fy0);
  const float wse = (ix - fx0) * (iy - fy0);
  const float* r0 = img + (int64_t)y0 * w;
  const float* r1 = img + (int64_t)y1 * w;
  return __ldg(r0 + x0) * wnw + __ldg(r0 + x1) * wne + __ldg(r1 + x0) * wsw + __ldg(r1 + x1) * wse;
}

// The four taps of sample_border<AC> (same arithmetic), split from their
// loads so that a caller can issue the gathers of several samples together.
struct BorderTaps {
  int i00, i01, i10, i11;
  float w00, w01, w10, w11;
};

template <bool AC = false>
__device__ __forceinline__ BorderTaps border_taps(int h, int w, float u, float v) {
  float ix, iy;
  if constexpr (AC) {
    ix = (u + 1.0f) / 2.0f * (float)(w - 1);
    iy = (v + 1.0f) / 2.0f * (float)(h - 1);
  } else {
    ix = ((u + 1.0f) * (float)w - 1.0f) / 2.0f;
    iy = ((v + 1.0f) * (float)h - 1.0f) / 2.0f;
  }
  ix = fminf(fmaxf(ix, 0.0f), (float)(w - 1));
  iy = fminf(fmaxf(iy, 0.0f), (float)(h - 1));
  const float fx0 = floorf(ix), fy0 = floorf(iy);
  const int x0 = (int)fx0, y0 = (int)fy0;
  const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
  BorderTaps t;
  t.w00 = (fx0 + 1.0f - ix) * (fy0 + 1.0f - iy);
  t.w01 = (ix - fx0) * (fy0 + 1.0f - iy);
  t.w10 = (fx0 + 1.0f - ix) * (iy - fy0);
  t.w11 = (ix - fx0) * (iy - fy0);
  t.i00 = y0 * w + x0;
  t.i01 = y0 * w + x1;
  t.i10 = y1 * w + x0;
  t.i11 = y1 * w + x1;
  return t;
}

// Rotate v by unit quaternion q = (w, x, y, z): v + w t + q_vec x t,
// t = 2 q_vec x v (equal to q (0, v) q* for unit q).
__device__ __forceinline__ float3 rotate(float4 q, float vx, float vy, float vz) {
  const float tx = 2.0f * (q.z * vz - q.w * vy);
  const float ty = 2.0f * (q.w * vx - q.y * vz);
  const float tz = 2.0f * (q.y * vy - q.z * vx);
  return make_float3(vx + q.x * tx + (q.z * tz - q.w * ty), vy + q.x * ty + (q.w * tx - q.y * tz),
                     vz + q.x * tz + (q.y * ty - q.z * tx));
}

}  // namespace ebsd
