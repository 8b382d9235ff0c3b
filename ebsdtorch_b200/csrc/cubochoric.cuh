// Cubochoric -> homochoric -> quaternion in FP64 (Rosca et al. 2014; the
// rotation angle from |h|^3 = 3/4 (w - sin w) by Newton's method), shared by
// the grid generator (K0) and the grid refinement (K9).
#pragma once

#include "common.cuh"

namespace ebsd {

__device__ __forceinline__ double omega_from_ho_norm(double t) {
  const double kPi = 3.14159265358979323846;
  const double g = (4.0 / 3.0) * t * t * t;  // = w - sin(w)
  double w = fmin(cbrt(6.0 * g), kPi);
#pragma unroll 1
  for (int it = 0; it < 40; ++it) {
    const double w2 = w * w;
    double wms;
    if (w < 0.25) {
      wms = w * w2 / 6.0 *
            (1.0 - w2 / 20.0 * (1.0 - w2 / 42.0 * (1.0 - w2 / 72.0 * (1.0 - w2 / 110.0))));
    } else {
      wms = w - sin(w);
    }
    const double sh = sin(0.5 * w);
    const double omc = 2.0 * sh * sh;
    if (!(omc > 0.0)) break;
    double wn = w - (wms - g) / omc;
    wn = fmin(fmax(wn, 0.0), kPi);
    const double dw = fabs(wn - w);
    w = wn;
    if (dw <= 1e-16 * fmax(1.0, w)) break;
  }
  return w;
}

// Cubochoric (x, y, z) -> unit quaternion (w, x, y, z) with w >= 0.
__device__ __forceinline__ void cu_to_qu(const double c[3], double q[4]) {
  const double kPi = 3.14159265358979323846;
  const double kR2 = 1.41421356237309504880;
  double a[3] = {fabs(c[0]), fabs(c[1]), fabs(c[2])};
  int o[3] = {0, 1, 2};
  // ascending order of magnitudes: o[0] smallest, o[2] largest
  if (a[o[0]] > a[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  if (a[o[1]] > a[o[2]]) { int t = o[1]; o[1] = o[2]; o[2] = t; }
  if (a[o[0]] > a[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  const double s = a[o[0]], m = a[o[1]], b = a[o[2]];
  double h[3] = {0.0, 0.0, 0.0};
  if (b > 0.0) {
    const double t = (m > 0.0) ? s * kPi / (12.0 * m) : 0.0;
    const double ct = cos(t), st = sin(t);
    const double num = 4.0 * b * b * (ct - kR2) + kR2 * m * m * (-2.0 * kR2 * ct + 3.0);
    const double fac = 1.0594630943592953 /* 2^(1/12) */ * 1.4422495703074083 /* 3^(1/3) */ * m *
                       sqrt(num / (ct - kR2)) /
                       (1.4645918875615231 /* pi^(1/3) */ * b * sqrt(kR2 - ct));
    const double hs = fac * st;
    const double hm = fac * 0.70710678118654752440 * (kR2 * ct - 1.0);
    const double hb = (2.0 * 1.8171205928321397 /* 6^(1/3) */ * b * b * (ct - kR2) +
                       1.7817974362806785 /* 2^(5/6) */ * 1.4422495703074083 * m * m *
                           (-2.0 * kR2 * ct + 3.0)) /
                      (2.0 * 1.4645918875615231 * b * (ct - kR2));
    h[o[0]] = hs;
    h[o[1]] = hm;
    h[o[2]] = hb;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (isnan(h[i])) h[i] = 0.0;
      h[i] = copysign(fabs(h[i]), c[i]);
    }
  }
  const double n2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  if (n2 < 1e-6) {  // the reference maps tiny rotations to the identity
    q[0] = 1.0; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0;
    return;
  }
  const double tn = sqrt(n2);
  const double w = omega_from_ho_norm(tn);
  const double cw = cos(0.5 * w), sw = sin(0.5 * w) / tn;
  q[0] = cw; q[1] = h[0] * sw; q[2] = h[1] * sw; q[3] = h[2] * sw;
  if (q[0] < 0.0) { q[0] = -q[0]; q[1] = -q[1]; q[2] = -q[2]; q[3] = -q[3]; }
}

}  // namespace ebsd
