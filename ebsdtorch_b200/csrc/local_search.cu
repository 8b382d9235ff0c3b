// Local dictionary search around per-pattern orientation proposals.
//
// For each pattern: every symmetry-equivalent copy g q of its proposal q
// (Laue operators g) is mapped to cubochoric coordinates (quaternion ->
// homochoric -> cubochoric; the inverse of the map in grid.cu, Rosca et al.
// 2014, as qu2cu orientations.py:1024-1035 and ho2cu :352-416), the grid cells
// within `radius_cells` of it are looked up in the cell -> dictionary-row map,
// and the dictionary orientations within `max_angle` of the copy become
// candidates. Their exact FP32 scores (dot of the zero-mean pattern row with
// the zero-mean dictionary row, the reference metric) decide the best match.
// No counterpart in the reference: it is the search step of the learned
// proposal path; candidates come from the same global dictionary as plain DI,
// so a proposal within max_angle of the plain-DI answer reproduces it.
#include <algorithm>

#include "common.cuh"

namespace ebsd {

constexpr int kLocalThreads = 256;
constexpr int kMaxLocalCand = 1024;

// FZ test of laue_fz_ori.py:144-239 loosened by `s`: true for any
// orientation whose neighbourhood of the search radius may reach the FZ.
__device__ bool near_fz(const float4 q, int laue, float s) {
  const float w = q.x, x = fabsf(q.y), y = fabsf(q.z), z = fabsf(q.w);
  const float r2m1 = 0.41421356f, r3 = 1.7320508f;
  switch (laue) {
    case 11: return fmaxf(fmaxf(x, y), z) <= w * r2m1 + s && x + y + z <= w + s;
    case 10: return x + y + z <= w + s;
    case 9: {
      const float m = fmaxf(x, y), n = fminf(x, y);
      const float rot = (m > (2.f + r3) * n) ? m : 0.5f * r3 * m + 0.5f * n;
      return z <= (2.f - r3) * w + s && rot <= w + s;
    }
    case 8: return z <= (2.f - r3) * w + s;
    case 7: {
      const float rot = (x >= y * r3) ? x : 0.5f * r3 * y + 0.5f * x;
      return z <= w / r3 + s && rot <= w + s;
    }
    case 6: return z <= w / r3 + s;
    case 5: {
      const float m = fmaxf(x, y), n = fminf(x, y);
      const float rot = (m > (r2m1 + 2.f) * n) ? m : 0.70710678f * (m + n);
      return z <= r2m1 * w + s && rot <= w + s;
    }
    case 4: return z <= r2m1 * w + s;
    case 3: return fmaxf(fmaxf(x, y), z) <= w + s;
    case 2: return z <= w + s;
    default: return true;
  }
}

// Quaternion (w >= 0) -> cubochoric coordinates, FP64.
__device__ void qu_to_cu(const double q[4], double cu[3]) {
  const double kPi = 3.14159265358979323846;
  const double w = 2.0 * acos(fmin(fmax(q[0], -1.0), 1.0));
  const double n = sqrt(q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const double w2 = w * w;
  const double wms = (w < 0.25) ? w * w2 / 6.0 * (1 - w2 / 20.0 * (1 - w2 / 42.0 * (1 - w2 / 72.0))) : w - sin(w);
  const double s = (n > 0.0) ? cbrt(0.75 * wms) / n : 0.0;
  const double h[3] = {q[1] * s, q[2] * s, q[3] * s};
  double a[3] = {fabs(h[0]), fabs(h[1]), fabs(h[2])};
  int o[3] = {0, 1, 2};
  if (a[o[0]] > a[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  if (a[o[1]] > a[o[2]]) { int t = o[1]; o[1] = o[2]; o[2] = t; }
  if (a[o[0]] > a[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  const double x3 = a[o[0]], y3 = a[o[1]], z3 = a[o[2]];
  const double r = sqrt(x3 * x3 + y3 * y3 + z3 * z3);
  double c[3] = {0.0, 0.0, 0.0};
  if (r > 0.0) {
    const double pf = sqrt(2.0 * r / (r + z3));
    const double x2 = x3 * pf, y2 = y3 * pf;
    const double z2 = sqrt(kPi / 6.0) * r;
    const double qq = sqrt(x2 * x2 + 2.0 * y2 * y2);
    const double pf2 = sqrt(kPi / 6.0) * sqrt(x2 * x2 + y2 * (qq + 2.0 * y2)) / sqrt(2.0);
    const double den = sqrt(2.0) * (x2 * x2 + y2 * y2);
    double x1 = 0.0;
    if (den > 0.0) x1 = pf2 * 12.0 / kPi * acos(fmin(fmax((x2 * x2 + y2 * qq) / den, -1.0), 1.0));
    const double inv = 1.0 / 0.89777278696128607;  // (pi/6)^(1/6)
    c[o[0]] = x1 * inv;
    c[o[1]] = pf2 * inv;
    c[o[2]] = z2 * inv;
  }
  for (int i = 0; i < 3; ++i) cu[i] = copysign(isnan(c[i]) ? 0.0 : c[i], h[i]);
}

__global__ void __launch_bounds__(kLocalThreads) k_local_search(
    const float* __restrict__ q_f32, int64_t ld_q, const float4* __restrict__ proposals, const LaueTable ops,
    int edge, const int32_t* __restrict__ cell_to_row, const float4* __restrict__ dict_quats,
    const float* __restrict__ d_f32, int64_t ld_d, int64_t n_dict, int n_pix, int laue, int radius,
    float cos_half_max, float fz_slack, int max_cand, int64_t* __restrict__ out_idx, float* __restrict__ out_score,
    int32_t* __restrict__ out_ncand) {
  extern __shared__ float qrow[];
  __shared__ int cand[kMaxLocalCand];
  __shared__ int base_cell[24][3];
  __shared__ float4 copy_q[24];
  __shared__ int n_cand;
  __shared__ int copy_ok[24];
  __shared__ float best_v[kLocalThreads / 32];
  __shared__ int64_t best_i[kLocalThreads / 32];
  const int64_t q = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int p = tid; p < n_pix; p += blockDim.x) qrow[p] = q_f32[q * ld_q + p];
  if (tid == 0) n_cand = 0;
  const double kHalf = 1.0725146985555127, step = 2.0 * kHalf / edge;
  if (tid < ops.n) {
    const float4 pr = proposals[q];
    const float* o = ops.q + 4 * tid;
    // copy g q: crystal symmetry acts on the left (pattern(g q) == pattern(q))
    double g[4] = {o[0] * (double)pr.x - o[1] * (double)pr.y - o[2] * (double)pr.z - o[3] * (double)pr.w,
                   o[0] * (double)pr.y + o[1] * (double)pr.x + o[2] * (double)pr.w - o[3] * (double)pr.z,
                   o[0] * (double)pr.z - o[1] * (double)pr.w + o[2] * (double)pr.x + o[3] * (double)pr.y,
                   o[0] * (double)pr.w + o[1] * (double)pr.z - o[2] * (double)pr.y + o[3] * (double)pr.x};
    const double nrm = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + g[3] * g[3]);
    for (double& v : g) v /= nrm;
    if (g[0] < 0.0)
      for (double& v : g) v = -v;
    double cu[3];
    qu_to_cu(g, cu);
    for (int i = 0; i < 3; ++i) base_cell[tid][i] = (int)llround((cu[i] + kHalf) / step);
    copy_q[tid] = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
    copy_ok[tid] = near_fz(copy_q[tid], laue, fz_slack) ? 1 : 0;
  }
  __syncthreads();
  const int side = 2 * radius + 1, cube = side * side * side;
  const int total = ops.n * cube;
  for (int t = tid; t < total; t += blockDim.x) {
    const int gi = t / cube, off = t - gi * cube;
    if (!copy_ok[gi]) continue;
    const int di = off / (side * side) - radius, dj = (off / side) % side - radius, dk = off % side - radius;
    const int ci = base_cell[gi][0] + di, cj = base_cell[gi][1] + dj, ck = base_cell[gi][2] + dk;
    if (ci < 0 || cj < 0 || ck < 0 || ci >= edge || cj >= edge || ck >= edge) continue;
    const int32_t row = __ldg(cell_to_row + ((int64_t)ci * edge + cj) * edge + ck);
    if (row < 0 || row >= n_dict) continue;
    const float4 d = __ldg(dict_quats + row), c = copy_q[gi];
    const float dot = fabsf(d.x * c.x + d.y * c.y + d.z * c.z + d.w * c.w);
    if (!(dot >= cos_half_max)) continue;
    const int slot = atomicAdd(&n_cand, 1);
    if (slot < max_cand) cand[slot] = row;
  }
  __syncthreads();
  const int nc = min(n_cand, max_cand);
  float bv = -INFINITY;
  int64_t bi = -1;
  for (int c = wid; c < nc; c += blockDim.x / 32) {
    const int64_t row = cand[c];
    const float* drow = d_f32 + row * ld_d;
    float acc = 0.f;
    for (int p = lane; p < n_pix; p += 32) acc = fmaf(__ldg(drow + p), qrow[p], acc);
    acc = warp_sum(acc);
    if (acc > bv || (acc == bv && row < bi)) {
      bv = acc;
      bi = row;
    }
  }
  if (lane == 0) {
    best_v[wid] = bv;
    best_i[wid] = bi;
  }
  __syncthreads();
  if (tid == 0) {
    float v = -INFINITY;
    int64_t i = -1;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w)
      if (best_i[w] >= 0 && (best_v[w] > v || (best_v[w] == v && best_i[w] < i))) {
        v = best_v[w];
        i = best_i[w];
      }
    out_idx[q] = i;
    out_score[q] = v;
    if (out_ncand) out_ncand[q] = n_cand;
  }
}

__global__ void k_cell_map_fill(int32_t* __restrict__ cell_to_row, int64_t n_cells) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_cells; t += (int64_t)gridDim.x * blockDim.x)
    cell_to_row[t] = -1;
}

__global__ void k_cell_map_scatter(const int32_t* __restrict__ cells, const int64_t* __restrict__ perm, int64_t n,
                                   int64_t n_cells, int32_t* __restrict__ cell_to_row) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = perm ? perm[j] : j;
    if (r < 0 || r >= n) continue;
    const int32_t c = cells[r];
    if (c >= 0 && c < n_cells) cell_to_row[c] = (int32_t)j;
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_cell_to_row(const int32_t* cells, const int64_t* perm, int64_t n, int64_t n_cells,
                                int32_t* cell_to_row, void* stream) {
  EBSD_ARG_CHECK(cells && cell_to_row && n >= 0 && n_cells > 0 && n <= INT32_MAX, "ebsd_cell_to_row: bad arguments");
  cudaStream_t s = as_stream(stream);
  const int b1 = (int)std::min<int64_t>((n_cells + 255) / 256, 148 * 16);
  k_cell_map_fill<<<b1, 256, 0, s>>>(cell_to_row, n_cells);
  EBSD_LAUNCH_CHECK();
  if (n > 0) {
    const int b2 = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_cell_map_scatter<<<b2, 256, 0, s>>>(cells, perm, n, n_cells, cell_to_row);
    EBSD_LAUNCH_CHECK();
  }
  return 0;
}

extern "C" int ebsd_local_search(const float* q_f32, int64_t ld_q, int64_t n_queries, const float* proposals,
                                 int laue_id, int edge_length, const int32_t* cell_to_row, const float* dict_quats,
                                 const float* d_f32, int64_t ld_d, int64_t n_dict, int n_pix, int radius_cells,
                                 float max_angle_rad, int max_candidates, int64_t* out_idx, float* out_score,
                                 int32_t* out_ncand, void* stream) {
  EBSD_ARG_CHECK(q_f32 && proposals && cell_to_row && dict_quats && d_f32 && out_idx && out_score,
                 "ebsd_local_search: null pointer");
  EBSD_ARG_CHECK(laue_id >= 1 && laue_id <= 11, "Laue group %d is not supported", laue_id);
  EBSD_ARG_CHECK(edge_length >= 1 && edge_length <= 2048, "bad grid edge length");
  EBSD_ARG_CHECK(radius_cells >= 0 && radius_cells <= 8, "radius_cells must be in [0, 8]");
  EBSD_ARG_CHECK(n_dict >= 1 && n_dict <= INT32_MAX, "bad dictionary size");
  EBSD_ARG_CHECK(max_candidates >= 1 && max_candidates <= kMaxLocalCand, "max_candidates must be in [1, %d]",
                 kMaxLocalCand);
  EBSD_ARG_CHECK(n_pix >= 1 && n_pix <= 40960 && ld_q >= n_pix && ld_d >= n_pix, "bad row length");
  EBSD_ARG_CHECK(((uintptr_t)proposals & 15) == 0 && ((uintptr_t)dict_quats & 15) == 0,
                 "quaternion arrays must be 16-byte aligned");
  if (n_queries == 0) return 0;
  EBSD_ARG_CHECK(n_queries < INT32_MAX, "too many queries");
  LaueTable t{};
  build_laue_table(laue_id, &t);
  const size_t smem = (size_t)n_pix * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_local_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_local_search<<<(int)n_queries, kLocalThreads, smem, as_stream(stream)>>>(
      q_f32, ld_q, reinterpret_cast<const float4*>(proposals), t, edge_length, cell_to_row,
      reinterpret_cast<const float4*>(dict_quats), d_f32, ld_d, n_dict, n_pix, laue_id, radius_cells,
      cosf(0.5f * max_angle_rad), 2.25f * max_angle_rad + 1e-3f, max_candidates, out_idx, out_score, out_ncand);
  EBSD_LAUNCH_CHECK();
  return 0;
}
