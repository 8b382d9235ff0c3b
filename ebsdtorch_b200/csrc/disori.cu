// A14: disorientation angle under one Laue group (measurement only).
//
// Follows disori_angle_laue (ebsdtorch/s2_and_so3/laue_fz_misori.py:148-203):
// for the misorientation m = q1 q2^-1, the disorientation angle is
// 2 acos(max over Laue operators g, h of |w(g m h)|). The operator tables are
// the rotation groups listed in laue_generators.py:54-249, built on the host
// by closing each group's generators and passed as a kernel parameter.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"

namespace ebsd {

struct LaueOps {
  float q[24 * 4];
};

struct Q4 {
  double w, x, y, z;
};

static Q4 qmul_h(Q4 a, Q4 b) {
  return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
          a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}

static Q4 axis_angle(double ax, double ay, double az, double deg) {
  const double n = std::sqrt(ax * ax + ay * ay + az * az);
  const double h = deg * M_PI / 360.0;
  return {std::cos(h), std::sin(h) * ax / n, std::sin(h) * ay / n, std::sin(h) * az / n};
}

// Closure of the group generated by `gens`, as unit quaternions with w >= 0.
static int close_group(const Q4* gens, int n_gens, Q4* out) {
  int n = 1;
  out[0] = {1, 0, 0, 0};
  auto known = [&](Q4 q) {
    for (int i = 0; i < n; ++i)
      if (std::fabs(std::fabs(q.w * out[i].w + q.x * out[i].x + q.y * out[i].y + q.z * out[i].z) - 1.0) <
          1e-9)
        return true;
    return false;
  };
  bool grew = true;
  while (grew) {
    grew = false;
    const int cur = n;
    for (int i = 0; i < cur; ++i)
      for (int g = 0; g < n_gens; ++g) {
        Q4 c = qmul_h(out[i], gens[g]);
        if (c.w < 0) c = {-c.w, -c.x, -c.y, -c.z};
        if (!known(c) && n < 24) {
          out[n++] = c;
          grew = true;
        }
      }
  }
  return n;
}

static int laue_ops(int laue, Q4* ops) {
  const Q4 z4 = axis_angle(0, 0, 1, 90), z2 = axis_angle(0, 0, 1, 180), z3 = axis_angle(0, 0, 1, 120),
           z6 = axis_angle(0, 0, 1, 60), x2 = axis_angle(1, 0, 0, 180),
           d3 = axis_angle(1, 1, 1, 120);
  Q4 g[3];
  int ng = 0;
  switch (laue) {
    case 1: break;
    case 2: g[ng++] = z2; break;
    case 3: g[ng++] = z2; g[ng++] = x2; break;
    case 4: g[ng++] = z4; break;
    case 5: g[ng++] = z4; g[ng++] = x2; break;
    case 6: g[ng++] = z3; break;
    case 7: g[ng++] = z3; g[ng++] = x2; break;
    case 8: g[ng++] = z6; break;
    case 9: g[ng++] = z6; g[ng++] = x2; break;
    case 10: g[ng++] = z2; g[ng++] = x2; g[ng++] = d3; break;
    case 11: g[ng++] = z4; g[ng++] = x2; g[ng++] = d3; break;
    default: return 0;
  }
  return close_group(g, ng, ops);
}

__global__ void k_disori(const float4* __restrict__ q1, const float4* __restrict__ q2, int64_t n,
                         int n_ops, const LaueOps ops, float* __restrict__ out) {
  const float* c_laue_ops = ops.q;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 a = q1[i], b = q2[i];
    // m = a * conj(b), (w, x, y, z) = (.x, .y, .z, .w)
    const float mw = a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    const float mx = -a.x * b.y + a.y * b.x - a.z * b.w + a.w * b.z;
    const float my = -a.x * b.z + a.y * b.w + a.z * b.x - a.w * b.y;
    const float mz = -a.x * b.w - a.y * b.z + a.z * b.y + a.w * b.x;
    float best = 0.0f;
    for (int g = 0; g < n_ops; ++g) {
      const float gw = c_laue_ops[4 * g], gx = c_laue_ops[4 * g + 1], gy = c_laue_ops[4 * g + 2],
                  gz = c_laue_ops[4 * g + 3];
      // t = g * m
      const float tw = gw * mw - gx * mx - gy * my - gz * mz;
      const float tx = gw * mx + gx * mw + gy * mz - gz * my;
      const float ty = gw * my - gx * mz + gy * mw + gz * mx;
      const float tz = gw * mz + gx * my - gy * mx + gz * mw;
      for (int h = 0; h < n_ops; ++h) {
        // real part of t * h
        const float w = tw * c_laue_ops[4 * h] - tx * c_laue_ops[4 * h + 1] -
                        ty * c_laue_ops[4 * h + 2] - tz * c_laue_ops[4 * h + 3];
        best = fmaxf(best, fabsf(w));
      }
    }
    out[i] = 2.0f * acosf(fminf(best, 1.0f));
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_disori_angle(const float* q1, const float* q2, int64_t n, int laue_id, float* out,
                                 void* stream) {
  EBSD_ARG_CHECK(q1 && q2 && out, "ebsd_disori_angle: null pointer");
  EBSD_ARG_CHECK(laue_id >= 1 && laue_id <= 11, "Laue group %d is not supported", laue_id);
  EBSD_ARG_CHECK(((uintptr_t)q1 & 15) == 0 && ((uintptr_t)q2 & 15) == 0,
                 "quaternion arrays must be 16-byte aligned");
  if (n <= 0) return 0;
  Q4 ops[24];
  const int n_ops = laue_ops(laue_id, ops);
  LaueOps h{};
  for (int i = 0; i < n_ops; ++i) {
    h.q[4 * i] = (float)ops[i].w;
    h.q[4 * i + 1] = (float)ops[i].x;
    h.q[4 * i + 2] = (float)ops[i].y;
    h.q[4 * i + 3] = (float)ops[i].z;
  }
  cudaStream_t s = as_stream(stream);
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_disori<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(q1),
                                  reinterpret_cast<const float4*>(q2), n, n_ops, h, out);
  EBSD_LAUNCH_CHECK();
  return 0;
}
