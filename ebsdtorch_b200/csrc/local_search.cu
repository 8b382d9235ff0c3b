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

struct LocalRows {
  const float* f32;    // zero-mean FP32 rows (the reference metric)
  int64_t ld_f32;
  const void* lp;      // unit-norm low-precision rows (null: score in FP32)
  int64_t ld_lp;
  const float* norm;   // |row| (lp scoring: raw dot = norm * lp_scale * q . lp)
  const float* lp_scale;
  int n_rescore;       // lp scoring: FP32 re-score of the best n (0: none)
};

constexpr int kLocalWarps = kLocalThreads / 32;
constexpr int kRescoreMax = kLocalWarps;

// Keeps (v, i) lists sorted best-first (higher v, then lower i); identical in
// all lanes of a warp.
template <int R>
__device__ __forceinline__ void keep_best(float (&bv)[R], int64_t (&bi)[R], float v, int64_t i) {
  if (!(v > bv[R - 1] || (v == bv[R - 1] && i >= 0 && (bi[R - 1] < 0 || i < bi[R - 1])))) return;
  bv[R - 1] = v;
  bi[R - 1] = i;
#pragma unroll
  for (int j = R - 1; j > 0; --j) {
    const bool sw = bv[j] > bv[j - 1] || (bv[j] == bv[j - 1] && bi[j] >= 0 && (bi[j - 1] < 0 || bi[j] < bi[j - 1]));
    if (sw) {
      const float tv = bv[j];
      bv[j] = bv[j - 1];
      bv[j - 1] = tv;
      const int64_t ti = bi[j];
      bi[j] = bi[j - 1];
      bi[j - 1] = ti;
    }
  }
}

__device__ __forceinline__ bool better(float v, int64_t i, float bv, int64_t bi) {
  return i >= 0 && (bi < 0 || v > bv || (v == bv && i < bi));
}

// Dot of the shared-memory bf16 query row with one low-precision row covering
// n_vec 16-byte chunks (zero padded; the query is padded with zeros). One
// candidate row per warp measured fastest on B200 (two or four rows per warp
// interleaved, or deeper unrolling, were 5-30 % slower).
template <int LP>
__device__ __forceinline__ float lp_dot(const __nv_bfloat16* qh, const uint4* __restrict__ d, int n_vec, int lane) {
  // qh: the query row in bf16 (shared memory): 16 bytes of query per 16 bytes
  // of bf16 row instead of 32, which halves the shared-memory side of the
  // L1/shared pipe these stages are bound by; products and sums stay FP32
  float acc = 0.f;
  const uint4* q16 = reinterpret_cast<const uint4*>(qh);
  for (int v = lane; v < n_vec; v += 32) {
    const uint4 u = __ldg(d + v);
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
    if constexpr (LP == EBSD_DT_BF16) {
      const uint4 qv = q16[v];
      const uint32_t qw[4] = {qv.x, qv.y, qv.z, qv.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[e]));
        const float2 g = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&qw[e]));
        acc = fmaf(f.x, g.x, acc);
        acc = fmaf(f.y, g.y, acc);
      }
    } else {
      const uint4 qa = q16[2 * v], qb = q16[2 * v + 1];
      const uint32_t qw[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[e] & 0xffffu), __NV_E4M3);
        const __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[e] >> 16), __NV_E4M3);
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&lo));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&hi));
        const float2 g0 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&qw[2 * e]));
        const float2 g1 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&qw[2 * e + 1]));
        acc = fmaf(a.x, g0.x, acc);
        acc = fmaf(a.y, g0.y, acc);
        acc = fmaf(b.x, g1.x, acc);
        acc = fmaf(b.y, g1.y, acc);
      }
    }
  }
  return warp_sum(acc);
}

// FP32 dot of the query row (shared or global memory) with one FP32 row;
// 16-byte loads, four in flight per lane, when both rows are 16-byte aligned
// and n_pix % 4 == 0.
__device__ __forceinline__ float f32_dot(const float* qrow, const float* __restrict__ drow, int n_pix, int lane) {
  float acc = 0.f;
  if ((n_pix & 3) == 0 && ((reinterpret_cast<uintptr_t>(drow) | reinterpret_cast<uintptr_t>(qrow)) & 15) == 0) {
    const float4* d4 = reinterpret_cast<const float4*>(drow);
    const float4* q4 = reinterpret_cast<const float4*>(qrow);
    const int n4 = n_pix >> 2;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    int v = lane;
    for (; v + 96 < n4; v += 128) {
      const float4 x0 = __ldg(d4 + v), x1 = __ldg(d4 + v + 32), x2 = __ldg(d4 + v + 64), x3 = __ldg(d4 + v + 96);
      const float4 y0 = q4[v], y1 = q4[v + 32], y2 = q4[v + 64], y3 = q4[v + 96];
      a0 += x0.x * y0.x + x0.y * y0.y + x0.z * y0.z + x0.w * y0.w;
      a1 += x1.x * y1.x + x1.y * y1.y + x1.z * y1.z + x1.w * y1.w;
      a2 += x2.x * y2.x + x2.y * y2.y + x2.z * y2.z + x2.w * y2.w;
      a3 += x3.x * y3.x + x3.y * y3.y + x3.z * y3.z + x3.w * y3.w;
    }
    for (; v < n4; v += 32) {
      const float4 x = __ldg(d4 + v), y = q4[v];
      a0 += x.x * y.x + x.y * y.y + x.z * y.z + x.w * y.w;
    }
    acc = (a0 + a1) + (a2 + a3);
  } else {
    for (int p = lane; p < n_pix; p += 32) acc = fmaf(__ldg(drow + p), qrow[p], acc);
  }
  return warp_sum(acc);
}

// LP 0: every candidate scored in FP32. LP = EBSD_DT_BF16 / EBSD_DT_E4M3:
// candidates ranked by their low-precision rows (half or a quarter of the
// bytes), then the best n_rescore re-scored in FP32 (or, with n_rescore 0,
// the low-precision estimate of the best one returned).
template <int LP>
__global__ void __launch_bounds__(kLocalThreads) k_local_search(
    const float* __restrict__ q_f32, int64_t ld_q, const float4* __restrict__ proposals, const LaueTable ops,
    int edge, const int32_t* __restrict__ cell_to_row, const float4* __restrict__ dict_quats, const LocalRows rows,
    int64_t n_dict, int n_pix, int n_pix_pad, int laue, int radius, float cos_half_max, float fz_slack, int max_cand,
    int64_t* __restrict__ out_idx, float* __restrict__ out_score, int32_t* __restrict__ out_ncand) {
  extern __shared__ __align__(16) uint8_t qsm[];
  float* qrow = reinterpret_cast<float*>(qsm);                  // LP 0: FP32 query row
  __nv_bfloat16* qh = reinterpret_cast<__nv_bfloat16*>(qsm);    // LP rows: bf16 query row
  __shared__ int cand[kMaxLocalCand];
  __shared__ int base_cell[24][3];
  __shared__ float4 copy_q[24];
  __shared__ int n_cand;
  __shared__ int ok_list[24];
  __shared__ int n_ok;
  __shared__ float best_v[kLocalWarps][kRescoreMax];
  __shared__ int64_t best_i[kLocalWarps][kRescoreMax];
  __shared__ int64_t sel[kRescoreMax];
  const int64_t q = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int p = tid; p < n_pix_pad; p += blockDim.x) {
    const float v = p < n_pix ? q_f32[q * ld_q + p] : 0.f;
    if constexpr (LP == 0)
      qrow[p] = v;
    else
      qh[p] = __float2bfloat16_rn(v);
  }
  if (tid == 0) n_cand = 0;
  const double kHalf = 1.0725146985555127, step = 2.0 * kHalf / edge;
  bool my_ok = false;
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
    my_ok = near_fz(copy_q[tid], laue, fz_slack);
  }
  if (wid == 0) {
    // compact list of the copies whose neighbourhood may reach the FZ (ops.n <= 24 < 32)
    const unsigned m = __ballot_sync(0xffffffffu, my_ok);
    if (my_ok) ok_list[__popc(m & ((1u << lane) - 1u))] = lane;
    if (lane == 0) n_ok = __popc(m);
  }
  __syncthreads();
  // one thread per (copy, i, j) column of the (2 radius + 1)^3 neighbourhood;
  // the k cells of a column are consecutive in the cell map
  const int side = 2 * radius + 1, n_col = side * side;
  const int total = n_ok * n_col;
  for (int t = tid; t < total; t += blockDim.x) {
    const int gk = t / n_col, off = t - gk * n_col;
    const int gi = ok_list[gk];
    const int oi = off / side;
    const int ci = base_cell[gi][0] + oi - radius, cj = base_cell[gi][1] + (off - oi * side) - radius;
    if (ci < 0 || cj < 0 || ci >= edge || cj >= edge) continue;
    const int k0 = max(0, base_cell[gi][2] - radius), k1 = min(edge - 1, base_cell[gi][2] + radius);
    const int32_t* col = cell_to_row + ((int64_t)ci * edge + cj) * edge;
    const float4 c = copy_q[gi];
    for (int ck = k0; ck <= k1; ++ck) {
      const int32_t row = __ldg(col + ck);
      if (row < 0 || row >= n_dict) continue;
      const float4 d = __ldg(dict_quats + row);
      const float dot = fabsf(d.x * c.x + d.y * c.y + d.z * c.z + d.w * c.w);
      if (!(dot >= cos_half_max)) continue;
      const int slot = atomicAdd(&n_cand, 1);
      if (slot < max_cand) cand[slot] = row;
    }
  }
  __syncthreads();
  const int nc = min(n_cand, max_cand);
  float v_out = -INFINITY;
  int64_t i_out = -1;
  if constexpr (LP == 0) {
    float bv = -INFINITY;
    int64_t bi = -1;
    for (int c = wid; c < nc; c += kLocalWarps) {
      const int64_t row = cand[c];
      const float acc = f32_dot(qrow, rows.f32 + row * rows.ld_f32, n_pix, lane);
      if (better(acc, row, bv, bi)) {
        bv = acc;
        bi = row;
      }
    }
    if (lane == 0) {
      best_v[wid][0] = bv;
      best_i[wid][0] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 0; w < kLocalWarps; ++w)
        if (better(best_v[w][0], best_i[w][0], v_out, i_out)) {
          v_out = best_v[w][0];
          i_out = best_i[w][0];
        }
    }
  } else {
    constexpr int kChunk = 16;  // bytes per vector load
    const int n_vec = n_pix_pad / (LP == EBSD_DT_BF16 ? kChunk / 2 : kChunk);
    float bv[kRescoreMax];
    int64_t bi[kRescoreMax];
#pragma unroll
    for (int j = 0; j < kRescoreMax; ++j) {
      bv[j] = -INFINITY;
      bi[j] = -1;
    }
    const int esz = LP == EBSD_DT_BF16 ? 2 : 1;
    const uint8_t* lp_base = static_cast<const uint8_t*>(rows.lp);
    for (int c = wid; c < nc; c += kLocalWarps) {
      const int64_t row = cand[c];
      const uint4* d = reinterpret_cast<const uint4*>(lp_base + row * rows.ld_lp * esz);
      const float v = lp_dot<LP>(qh, d, n_vec, lane) * __ldg(rows.norm + row) *
                      (rows.lp_scale ? __ldg(rows.lp_scale + row) : 1.f);
      keep_best<kRescoreMax>(bv, bi, v, row);
    }
    if (lane == 0) {
#pragma unroll
      for (int j = 0; j < kRescoreMax; ++j) {
        best_v[wid][j] = bv[j];
        best_i[wid][j] = bi[j];
      }
    }
    __syncthreads();
    const int n_sel = max(1, min(rows.n_rescore, kRescoreMax));
    if (wid == 0) {
      // merge the warps' lists: n_sel rounds of a warp-wide arg-max over the
      // kLocalWarps x kRescoreMax entries (two per lane)
      float* fv = &best_v[0][0];
      int64_t* fi = &best_i[0][0];
      for (int r = 0; r < n_sel; ++r) {
        float v = -INFINITY;
        int64_t i = -1;
        int at = -1;
        for (int e = lane; e < kLocalWarps * kRescoreMax; e += 32)
          if (better(fv[e], fi[e], v, i)) {
            v = fv[e];
            i = fi[e];
            at = e;
          }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, v, o);
          const int64_t oi = __shfl_xor_sync(0xffffffffu, i, o);
          const int oat = __shfl_xor_sync(0xffffffffu, at, o);
          if (better(ov, oi, v, i)) {
            v = ov;
            i = oi;
            at = oat;
          }
        }
        if (lane == 0) {
          sel[r] = i;
          if (r == 0) {
            v_out = v;
            i_out = i;
          }
          if (at >= 0) fi[at] = -1;
        }
        __syncwarp();
      }
    }
    if (rows.n_rescore > 0) {
      __syncthreads();
      // FP32 re-score: warp w takes the w-th selected row
      if (wid < n_sel) {
        const int64_t row = sel[wid];
        // the FP32 query row from global memory (L2-resident after the fill)
        const float acc = row >= 0 ? f32_dot(q_f32 + q * ld_q, rows.f32 + row * rows.ld_f32, n_pix, lane)
                                   : -INFINITY;
        if (lane == 0) {
          best_v[wid][0] = acc;
          best_i[wid][0] = row;
        }
      }
      __syncthreads();
      if (tid == 0) {
        v_out = -INFINITY;
        i_out = -1;
        for (int w = 0; w < n_sel; ++w)
          if (better(best_v[w][0], best_i[w][0], v_out, i_out)) {
            v_out = best_v[w][0];
            i_out = best_i[w][0];
          }
      }
    }
  }
  if (tid == 0) {
    out_idx[q] = i_out;
    out_score[q] = v_out;
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
                                 const float* d_f32, int64_t ld_d, const void* d_lp, int lp_dtype, int64_t ld_lp,
                                 const float* d_norm, const float* d_lp_scale, int n_rescore, int64_t n_dict,
                                 int n_pix, int radius_cells, float max_angle_rad, int max_candidates,
                                 int64_t* out_idx, float* out_score, int32_t* out_ncand, void* stream) {
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
  int n_pix_pad = n_pix;
  if (d_lp) {
    EBSD_ARG_CHECK(lp_dtype == EBSD_DT_BF16 || lp_dtype == EBSD_DT_E4M3, "bad lp_dtype");
    EBSD_ARG_CHECK(d_norm != nullptr && (lp_dtype == EBSD_DT_BF16 || d_lp_scale != nullptr),
                   "low-precision scoring needs the row norms (and e4m3 scales)");
    EBSD_ARG_CHECK(n_rescore >= 0 && n_rescore <= kRescoreMax, "n_rescore must be in [0, %d]", kRescoreMax);
    const int per = lp_dtype == EBSD_DT_BF16 ? 8 : 16;
    n_pix_pad = (n_pix + per - 1) / per * per;
    const int esz = lp_dtype == EBSD_DT_BF16 ? 2 : 1;
    // the vector loads read n_pix_pad elements: the row padding must cover
    // them (and be zero, as the projector writes it)
    EBSD_ARG_CHECK(ld_lp >= n_pix_pad && (ld_lp * esz) % 16 == 0 && ((uintptr_t)d_lp & 15) == 0,
                   "low-precision rows must be 16-byte aligned with ld_lp >= %d", n_pix_pad);
  }
  if (n_queries == 0) return 0;
  EBSD_ARG_CHECK(n_queries < INT32_MAX, "too many queries");
  LaueTable t{};
  build_laue_table(laue_id, &t);
  LocalRows rows{d_f32, ld_d, d_lp, ld_lp, d_norm, d_lp_scale, n_rescore};
  const size_t smem = (size_t)n_pix_pad * (d_lp ? sizeof(__nv_bfloat16) : sizeof(float));
  auto run = [&](auto kern) -> int {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(int)n_queries, kLocalThreads, smem, as_stream(stream)>>>(
        q_f32, ld_q, reinterpret_cast<const float4*>(proposals), t, edge_length, cell_to_row,
        reinterpret_cast<const float4*>(dict_quats), rows, n_dict, n_pix, n_pix_pad, laue_id, radius_cells,
        cosf(0.5f * max_angle_rad), 2.25f * max_angle_rad + 1e-3f, max_candidates, out_idx, out_score, out_ncand);
    EBSD_LAUNCH_CHECK();
    return 0;
  };
  if (!d_lp) return run(k_local_search<0>);
  return lp_dtype == EBSD_DT_BF16 ? run(k_local_search<EBSD_DT_BF16>) : run(k_local_search<EBSD_DT_E4M3>);
}
