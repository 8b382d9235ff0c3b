// A15: 6-D rotation representation (Zhou et al. 2019) <-> quaternion, and the
// symmetry-aware rotation loss used to train the orientation-proposal CNN.
//
// zh2om follows ebsdtorch/s2_and_so3/orientations.py:940-963 (Gram-Schmidt;
// the matrix rows are b1, b2, b3 = b1 x b2), om2qu follows :52-132 (largest
// diagonal branch, then w >= 0 and the axis signs from the antisymmetric
// part), qu2om :913-937, qu2zh :1008-1020 (first two rows).
// The loss has no counterpart in the reference (it has no learned indexer):
//   L_i = min over Laue operators g of || zh2om(z_i) - om(g q_i) ||_F^2,
// with the exact gradient through the Gram-Schmidt map.
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace ebsd {

__device__ __forceinline__ void zh_to_om(const float* z, float b[3][3], float& n1, float& n2, float& nc,
                                         float u[3]) {
  n1 = sqrtf(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
  for (int i = 0; i < 3; ++i) b[0][i] = z[i] / n1;
  const float d = b[0][0] * z[3] + b[0][1] * z[4] + b[0][2] * z[5];
  for (int i = 0; i < 3; ++i) u[i] = z[3 + i] - d * b[0][i];
  n2 = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  for (int i = 0; i < 3; ++i) b[1][i] = u[i] / n2;
  float c[3] = {b[0][1] * b[1][2] - b[0][2] * b[1][1], b[0][2] * b[1][0] - b[0][0] * b[1][2],
                b[0][0] * b[1][1] - b[0][1] * b[1][0]};
  nc = sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int i = 0; i < 3; ++i) b[2][i] = c[i] / nc;
}

__device__ __forceinline__ void qu_to_om(const float* q, float m[3][3]) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  const float qb = w * w - (x * x + y * y + z * z);
  m[0][0] = qb + 2 * x * x;
  m[0][1] = 2 * (x * y - w * z);
  m[0][2] = 2 * (x * z + w * y);
  m[1][0] = 2 * (y * x + w * z);
  m[1][1] = qb + 2 * y * y;
  m[1][2] = 2 * (y * z - w * x);
  m[2][0] = 2 * (z * x - w * y);
  m[2][1] = 2 * (z * y + w * x);
  m[2][2] = qb + 2 * z * z;
}

__device__ __forceinline__ void om_to_qu(const float m[3][3], float* q) {
  const float m00 = m[0][0], m11 = m[1][1], m22 = m[2][2];
  float t;
  if (m22 < 0.f) {
    if (m00 > m11) {
      t = 1 + m00 - m11 - m22;
      const float r = 0.5f * rsqrtf(t);
      q[1] = t * r; q[2] = (m[0][1] + m[1][0]) * r; q[3] = (m[2][0] + m[0][2]) * r; q[0] = (m[1][2] - m[2][1]) * r;
    } else {
      t = 1 - m00 + m11 - m22;
      const float r = 0.5f * rsqrtf(t);
      q[1] = (m[0][1] + m[1][0]) * r; q[2] = t * r; q[3] = (m[1][2] + m[2][1]) * r; q[0] = (m[2][0] - m[0][2]) * r;
    }
  } else {
    if (m00 < -m11) {
      t = 1 - m00 - m11 + m22;
      const float r = 0.5f * rsqrtf(t);
      q[1] = (m[2][0] + m[0][2]) * r; q[2] = (m[1][2] + m[2][1]) * r; q[3] = t * r; q[0] = (m[0][1] - m[1][0]) * r;
    } else {
      t = 1 + m00 + m11 + m22;
      const float r = 0.5f * rsqrtf(t);
      q[1] = (m[1][2] - m[2][1]) * r; q[2] = (m[2][0] - m[0][2]) * r; q[3] = (m[0][1] - m[1][0]) * r; q[0] = t * r;
    }
  }
  q[0] = fabsf(q[0]);
  q[1] = copysignf(q[1], m[2][1] - m[1][2]);
  q[2] = copysignf(q[2], m[0][2] - m[2][0]);
  q[3] = copysignf(q[3], m[1][0] - m[0][1]);
}

__global__ void k_zh_to_qu(const float* __restrict__ zh, int64_t n, float* __restrict__ qu,
                           float* __restrict__ om) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float z[6], b[3][3], n1, n2, nc, u[3];
    for (int j = 0; j < 6; ++j) z[j] = zh[6 * i + j];
    zh_to_om(z, b, n1, n2, nc, u);
    if (om)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) om[9 * i + 3 * r + c] = b[r][c];
    float q[4];
    om_to_qu(b, q);
    for (int j = 0; j < 4; ++j) qu[4 * i + j] = q[j];
  }
}

__global__ void k_qu_to_zh(const float* __restrict__ qu, int64_t n, float* __restrict__ zh) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float m[3][3];
    qu_to_om(qu + 4 * i, m);
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c) zh[6 * i + 3 * r + c] = m[r][c];
  }
}

__global__ void k_rot6d_loss(const float* __restrict__ zh, const float* __restrict__ q_true, int64_t n,
                             const LaueTable ops, float grad_scale, float* __restrict__ loss,
                             float* __restrict__ grad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float z[6], b[3][3], n1, n2, nc, u[3];
    for (int j = 0; j < 6; ++j) z[j] = zh[6 * i + j];
    zh_to_om(z, b, n1, n2, nc, u);
    const float* qt = q_true + 4 * i;
    float best = INFINITY, tgt[3][3] = {};
    for (int g = 0; g < ops.n; ++g) {
      const float* o = ops.q + 4 * g;
      // g q: crystal symmetry acts on the left (pattern(g q) == pattern(q)
      // for the projector's q v q* ray rotation)
      const float qg[4] = {o[0] * qt[0] - o[1] * qt[1] - o[2] * qt[2] - o[3] * qt[3],
                           o[0] * qt[1] + o[1] * qt[0] + o[2] * qt[3] - o[3] * qt[2],
                           o[0] * qt[2] - o[1] * qt[3] + o[2] * qt[0] + o[3] * qt[1],
                           o[0] * qt[3] + o[1] * qt[2] - o[2] * qt[1] + o[3] * qt[0]};
      float m[3][3];
      qu_to_om(qg, m);
      float d = 0.f;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) d += (b[r][c] - m[r][c]) * (b[r][c] - m[r][c]);
      if (d < best) {
        best = d;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) tgt[r][c] = m[r][c];
      }
    }
    if (loss) loss[i] = best;
    if (!grad) continue;
    float g1[3], g2[3], g3[3];
    for (int c = 0; c < 3; ++c) {
      g1[c] = 2.f * (b[0][c] - tgt[0][c]);
      g2[c] = 2.f * (b[1][c] - tgt[1][c]);
      g3[c] = 2.f * (b[2][c] - tgt[2][c]);
    }
    // b3 = c / |c|, c = b1 x b2
    const float d3 = g3[0] * b[2][0] + g3[1] * b[2][1] + g3[2] * b[2][2];
    float gc[3];
    for (int c = 0; c < 3; ++c) gc[c] = (g3[c] - d3 * b[2][c]) / nc;
    g1[0] += b[1][1] * gc[2] - b[1][2] * gc[1];
    g1[1] += b[1][2] * gc[0] - b[1][0] * gc[2];
    g1[2] += b[1][0] * gc[1] - b[1][1] * gc[0];
    g2[0] += gc[1] * b[0][2] - gc[2] * b[0][1];
    g2[1] += gc[2] * b[0][0] - gc[0] * b[0][2];
    g2[2] += gc[0] * b[0][1] - gc[1] * b[0][0];
    // b2 = u / |u|, u = a2 - (b1 . a2) b1
    const float d2 = g2[0] * b[1][0] + g2[1] * b[1][1] + g2[2] * b[1][2];
    float gu[3];
    for (int c = 0; c < 3; ++c) gu[c] = (g2[c] - d2 * b[1][c]) / n2;
    const float gub1 = gu[0] * b[0][0] + gu[1] * b[0][1] + gu[2] * b[0][2];
    const float b1a2 = b[0][0] * z[3] + b[0][1] * z[4] + b[0][2] * z[5];
    float ga2[3];
    for (int c = 0; c < 3; ++c) {
      ga2[c] = gu[c] - gub1 * b[0][c];
      g1[c] = g1[c] - gub1 * z[3 + c] - b1a2 * gu[c];
    }
    // b1 = a1 / |a1|
    const float d1 = g1[0] * b[0][0] + g1[1] * b[0][1] + g1[2] * b[0][2];
    for (int c = 0; c < 3; ++c) {
      grad[6 * i + c] = grad_scale * (g1[c] - d1 * b[0][c]) / n1;
      grad[6 * i + 3 + c] = grad_scale * ga2[c];
    }
  }
}

static int blocks_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 8); }

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_zh_to_qu(const float* zh, int64_t n, float* out_qu, float* out_om, void* stream) {
  EBSD_ARG_CHECK(zh && out_qu && n >= 0, "ebsd_zh_to_qu: bad arguments");
  if (n == 0) return 0;
  k_zh_to_qu<<<blocks_for(n), 256, 0, as_stream(stream)>>>(zh, n, out_qu, out_om);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_qu_to_zh(const float* qu, int64_t n, float* out_zh, void* stream) {
  EBSD_ARG_CHECK(qu && out_zh && n >= 0, "ebsd_qu_to_zh: bad arguments");
  if (n == 0) return 0;
  k_qu_to_zh<<<blocks_for(n), 256, 0, as_stream(stream)>>>(qu, n, out_zh);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_rot6d_sym_loss(const float* zh, const float* q_true, int64_t n, int laue_id, float grad_scale,
                                   float* out_loss, float* out_grad, void* stream) {
  EBSD_ARG_CHECK(zh && q_true && n >= 0, "ebsd_rot6d_sym_loss: bad arguments");
  EBSD_ARG_CHECK(laue_id >= 1 && laue_id <= 11, "Laue group %d is not supported", laue_id);
  if (n == 0) return 0;
  LaueTable t{};
  build_laue_table(laue_id, &t);
  k_rot6d_loss<<<blocks_for(n), 256, 0, as_stream(stream)>>>(zh, q_true, n, t, grad_scale, out_loss, out_grad);
  EBSD_LAUNCH_CHECK();
  return 0;
}
