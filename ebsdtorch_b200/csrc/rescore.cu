// K4/K6: merge of the per-range candidate lists, FP32 re-score of the best
// candidates, and the final sorted top-k per query.
//
// Replaces ChunkedKNN.retrieve_topk (ebsdtorch/utils/knn.py:268-287; the
// reference sorts its running top-k with torch.topk(sorted=True)). The exact
// scores are the reference's metric: the FP32 dot product of the zero-mean
// query row with the zero-mean dictionary row (knn.py:96-97).
// One CTA per query; candidates are ordered by (score desc, index asc).
//
// Margin gate (gate_rel > 0): a candidate's low-precision score s' and its
// exact score s (both per unit query norm) satisfy |s' - s| <= gate_rel * w,
// w = |d| for the dot metric and 1 for cosine, when gate_rel bounds the
// rounding of the unit rows and the FP32 accumulation (the caller derives it
// from the element type and the row length). Let tau be the k_out-th largest
// lower bound s' - gate_rel * w among the n_rescore best candidates. A
// candidate whose upper bound s' + gate_rel * w is below tau cannot be among
// the exact top k_out, so only the others are re-scored; the result equals
// re-scoring all n_rescore.
#include "common.cuh"

namespace ebsd {

constexpr int kMergeThreads = 256;
constexpr int kMaxCand = 4096;    // part_slots * n_cand per query
constexpr int kMaxRescore = 128;  // candidates re-scored per query
constexpr int kMaxKOut = 128;
static_assert(kMaxRescore + kMaxKOut <= kMergeThreads, "one finalist per thread");

// (v1, i1) ranks before (v2, i2)?
__device__ __forceinline__ bool ranks_before(float v1, int64_t i1, float v2, int64_t i2) {
  if (i1 < 0) return false;
  if (i2 < 0) return true;
  if (v1 != v2) return v1 > v2;
  return i1 < i2;
}

// In-place bitonic sort of n (power of two) entries in shared memory.
__device__ void bitonic_sort(float* v, int64_t* idx, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool up = ((lo & size) == 0);
        const bool before = ranks_before(v[lo], idx[lo], v[hi], idx[hi]);
        // ascending "rank order" in up-segments: element that ranks first goes low
        if (up != before) {
          const float tv = v[lo];
          v[lo] = v[hi];
          v[hi] = tv;
          const int64_t ti = idx[lo];
          idx[lo] = idx[hi];
          idx[hi] = ti;
        }
      }
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kMergeThreads) k_merge_rescore(
    const float* __restrict__ part_val, const int32_t* __restrict__ part_idx, int n_list,
    const float* __restrict__ q_f32, int64_t ld_q, const float* __restrict__ d_f32, int64_t ld_d,
    int64_t d_base, int64_t d_rows, int n_pix, const float* __restrict__ q_norm, const float* __restrict__ d_norm,
    const float* __restrict__ q_lp_scale, int similarity, int n_rescore, int k_out,
    const float* __restrict__ run_val, const int64_t* __restrict__ run_idx, int sort_n,
    float* __restrict__ out_val, int64_t* __restrict__ out_idx, float gate_rel,
    unsigned long long* __restrict__ n_rescored) {
  extern __shared__ float dyn[];
  // the query row is read from global memory (L1/L2-resident after its
  // first pass): staging it in shared memory would cap the CTAs per SM
  float* cv = dyn;                                                     // sort_n
  int64_t* ci = reinterpret_cast<int64_t*>(cv + ((sort_n + 1) & ~1));  // sort_n
  __shared__ float fin_v[kMaxRescore + kMaxKOut];
  __shared__ int64_t fin_i[kMaxRescore + kMaxKOut];
  __shared__ float lb[kMaxRescore];
  __shared__ int sel[kMaxRescore];
  __shared__ float tau_s;
  __shared__ int n_sel;
  __shared__ float part[(kMergeThreads / 32) * kMaxRescore];  // per-warp partial dots

  const int64_t q = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;

  // 1. gather all candidates of this query
  for (int t = tid; t < sort_n; t += blockDim.x) {
    if (t < n_list) {
      const int32_t i = part_idx[q * n_list + t];
      cv[t] = part_val[q * n_list + t];
      ci[t] = i;
    } else {
      cv[t] = -INFINITY;
      ci[t] = -1;
    }
  }
  const float* qrow = d_f32 ? q_f32 + q * ld_q : nullptr;
  bitonic_sort(cv, ci, sort_n);

  // 2. exact FP32 scores of the best n_rescore (or approximate * |q|).
  // Euclidean scores are kept internally as the negated squared distance, so
  // that "larger ranks first" holds for every metric.
  const int nr = n_rescore;
  const bool euclid = similarity == EBSD_SIM_EUCLIDEAN;
  // distances (euclidean, manhattan) are reported positive, smallest first
  const bool dist = euclid || similarity == EBSD_SIM_MANHATTAN;
  if (d_f32) {
    // 2a. which of them can reach the exact top k_out (margin gate)
    const bool gate = gate_rel > 0.0f && nr > k_out && !euclid;
    if (gate) {
      float w = 0.0f;
      if (tid < nr) {
        const int64_t i = ci[tid];
        const bool ok = i >= d_base && i < d_base + d_rows;
        w = gate_rel * ((similarity == EBSD_SIM_DOT && ok) ? d_norm[i - d_base] : 1.0f);
        lb[tid] = ok ? cv[tid] - w : -INFINITY;
      }
      if (tid == 0) n_sel = 0;
      __syncthreads();
      if (tid < nr) {
        // tau: the k_out-th largest lower bound (rank selection, index order on ties)
        const float v = lb[tid];
        int rank = 0;
        for (int o = 0; o < nr; ++o) rank += (lb[o] > v || (lb[o] == v && o < tid)) ? 1 : 0;
        if (rank == k_out - 1) tau_s = v;
      }
      __syncthreads();
      if (tid < nr) {
        const bool keep = ci[tid] >= 0 && cv[tid] + w >= tau_s;
        if (keep) sel[atomicAdd(&n_sel, 1)] = tid;
        fin_v[tid] = -INFINITY;  // candidates left out stay out of the final selection
        fin_i[tid] = -1;
      }
      __syncthreads();
    } else {
      for (int c = tid; c < nr; c += blockDim.x) sel[c] = c;
      if (tid == 0) n_sel = nr;
      __syncthreads();
    }
    const int ns = n_sel;
    if (n_rescored && tid == 0) atomicAdd(n_rescored, (unsigned long long)ns);
    // Every warp takes a slice of the pixels of every selected row, R rows at
    // a time (R 16-byte loads in flight per lane), so all warps stream even
    // when few rows are selected; the per-warp partial dots are summed in a
    // fixed order (deterministic).
    constexpr int R = 8;
    const bool vec = (n_pix & 3) == 0 && (ld_d & 3) == 0 && ((uintptr_t)d_f32 & 15) == 0 && (ld_q & 3) == 0 &&
                     ((uintptr_t)q_f32 & 15) == 0;
    const int n4 = n_pix >> 2;
    for (int s0 = 0; s0 < ns; s0 += R) {
      const float* d[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int c = s0 + j < ns ? sel[s0 + j] : -1;
        const int64_t i = (c >= 0 && ci[c] >= d_base && ci[c] < d_base + d_rows) ? ci[c] : -1;
        d[j] = d_f32 + (i >= 0 ? i - d_base : 0) * ld_d;  // a missing row re-reads row 0
      }
      float acc[R];
#pragma unroll
      for (int j = 0; j < R; ++j) acc[j] = 0.0f;
      if (vec) {
        const float4* q4 = reinterpret_cast<const float4*>(qrow);
        for (int v = tid; v < n4; v += blockDim.x) {
          float4 x[R];
#pragma unroll
          for (int j = 0; j < R; ++j)  // rows past ns are skipped (uniform over the CTA)
            x[j] = s0 + j < ns ? __ldg(reinterpret_cast<const float4*>(d[j]) + v) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float4 y = __ldg(q4 + v);
#pragma unroll
          for (int j = 0; j < R; ++j) {
            acc[j] = fmaf(x[j].x, y.x, acc[j]);
            acc[j] = fmaf(x[j].y, y.y, acc[j]);
            acc[j] = fmaf(x[j].z, y.z, acc[j]);
            acc[j] = fmaf(x[j].w, y.w, acc[j]);
          }
        }
      } else {
        for (int p = tid; p < n_pix; p += blockDim.x) {
          const float y = __ldg(qrow + p);
#pragma unroll
          for (int j = 0; j < R; ++j)
            if (s0 + j < ns) acc[j] = fmaf(__ldg(d[j] + p), y, acc[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const float w = warp_sum(acc[j]);
        if (lane == 0 && s0 + j < ns) part[wid * kMaxRescore + s0 + j] = w;
      }
    }
    __syncthreads();
    if (tid < ns) {
      const int c = sel[tid];
      const int64_t i = (ci[c] >= d_base && ci[c] < d_base + d_rows) ? ci[c] : -1;
      float v = 0.0f;
      for (int w = 0; w < nw; ++w) v += part[w * kMaxRescore + tid];
      if (similarity == EBSD_SIM_COSINE && i >= 0) {
        const float den = q_norm[q] * d_norm[i - d_base];
        v = den > 0.0f ? v / den : 0.0f;
      } else if (euclid && i >= 0) {
        // |q|^2 + |d|^2 - 2 q.d with FP32 norms of the zero-mean rows (knn.py:85-91)
        const float qn = q_norm[q], dn = d_norm[i - d_base];
        v = -(fmaf(qn, qn, dn * dn) - 2.0f * v);
      }
      fin_v[c] = i >= 0 ? v : -INFINITY;
      fin_i[c] = i;
    }
  } else {
    float qn = q_lp_scale ? q_lp_scale[q] : 1.0f;
    if ((similarity == EBSD_SIM_DOT || euclid) && q_norm) qn *= q_norm[q];
    // euclidean: cv * qn = 2 q.d - |d|^2 (see ebsd_match_topk_tiled), so the
    // negated squared distance is cv * qn - |q|^2
    const float qq = (euclid && q_norm) ? q_norm[q] * q_norm[q] : 0.0f;
    for (int c = tid; c < nr; c += blockDim.x) {
      fin_v[c] = ci[c] >= 0 ? cv[c] * qn - qq : -INFINITY;
      fin_i[c] = ci[c];
    }
  }
  // 3. running results
  int nf = nr;
  if (run_val) {
    for (int c = tid; c < k_out; c += blockDim.x) {
      const float rv = run_val[q * k_out + c];
      fin_v[nr + c] = dist ? -rv : rv;
      fin_i[nr + c] = run_idx[q * k_out + c];
    }
    nf += k_out;
  }
  __syncthreads();
  // 4. top k_out of the nf finalists by rank selection (nf <= blockDim.x).
  // Running results and new candidates come from disjoint dictionary ranges.
  const int valid = (tid < nf && fin_i[tid] >= 0) ? 1 : 0;
  const int n_valid = __syncthreads_count(valid);
  if (valid) {
    const float v = fin_v[tid];
    const int64_t i = fin_i[tid];
    int rank = 0;
    for (int o = 0; o < nf; ++o)
      if (o != tid && ranks_before(fin_v[o], fin_i[o], v, i)) ++rank;
    if (rank < k_out) {
      out_val[q * k_out + rank] = dist ? -v : v;
      out_idx[q * k_out + rank] = i;
    }
  }
  for (int r = n_valid + tid; r < k_out; r += blockDim.x) {
    out_val[q * k_out + r] = dist ? INFINITY : -INFINITY;
    out_idx[q * k_out + r] = -1;
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_merge_rescore_gated(const float* part_val, const int32_t* part_idx, int64_t n_queries,
                                        int part_slots, int n_cand, const float* q_f32, int64_t ld_q,
                                        const float* d_f32, int64_t ld_d, int64_t d_index_base,
                                        int64_t d_rows, int n_pix,
                                        const float* q_norm, const float* d_norm, const float* q_lp_scale,
                                        int similarity,
                                        int n_rescore, int k_out, const float* run_val,
                                        const int64_t* run_idx, float* out_val, int64_t* out_idx,
                                        float gate_rel, unsigned long long* n_rescored, void* stream) {
  EBSD_ARG_CHECK(part_val && part_idx && out_val && out_idx, "ebsd_merge_rescore: null pointer");
  EBSD_ARG_CHECK(n_queries >= 0 && part_slots >= 1 && n_cand >= 1, "bad candidate-list sizes");
  const int n_list = part_slots * n_cand;
  EBSD_ARG_CHECK(n_list <= kMaxCand, "part_slots * n_cand = %d exceeds %d", n_list, kMaxCand);
  EBSD_ARG_CHECK(k_out >= 1 && k_out <= kMaxKOut, "k_out %d outside [1, %d]", k_out, kMaxKOut);
  EBSD_ARG_CHECK(n_rescore >= 1 && n_rescore <= kMaxRescore && n_rescore <= n_list,
                 "n_rescore %d outside [1, min(%d, %d)]", n_rescore, kMaxRescore, n_list);
  EBSD_ARG_CHECK(!(run_val == nullptr) == !(run_idx == nullptr), "run_val/run_idx must be given together");
  EBSD_ARG_CHECK(similarity == EBSD_SIM_DOT || similarity == EBSD_SIM_COSINE || similarity == EBSD_SIM_EUCLIDEAN ||
                     similarity == EBSD_SIM_MANHATTAN,
                 "similarity must be EBSD_SIM_DOT, EBSD_SIM_COSINE, EBSD_SIM_EUCLIDEAN or EBSD_SIM_MANHATTAN");
  EBSD_ARG_CHECK(similarity != EBSD_SIM_MANHATTAN || !d_f32, "manhattan candidates are exact: no re-score");
  EBSD_ARG_CHECK(similarity != EBSD_SIM_EUCLIDEAN || q_norm, "euclidean scores need q_norm");
  if (d_f32) {
    EBSD_ARG_CHECK(q_f32 != nullptr, "q_f32 is required for re-scoring");
    EBSD_ARG_CHECK(similarity == EBSD_SIM_DOT || (q_norm && d_norm),
                   "cosine and euclidean re-scoring need q_norm and d_norm");
    EBSD_ARG_CHECK(n_pix >= 1 && ld_q >= n_pix && ld_d >= n_pix, "bad re-score row length");
    EBSD_ARG_CHECK(d_rows >= 1 && d_index_base >= 0, "bad dictionary row range");
    EBSD_ARG_CHECK(!(gate_rel > 0.0f) || similarity == EBSD_SIM_COSINE || d_norm,
                   "the margin gate of the dot metric needs d_norm");
  }
  EBSD_ARG_CHECK(!(gate_rel < 0.0f) && gate_rel < 1.0f, "gate_rel %g outside [0, 1)", (double)gate_rel);
  if (n_queries == 0) return 0;
  int sort_n = 1;
  while (sort_n < n_list) sort_n <<= 1;
  const size_t smem = (size_t)((sort_n + 1) & ~1) * 4 + (size_t)sort_n * 8 + 16;
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_merge_rescore, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
  EBSD_ARG_CHECK(n_queries < INT32_MAX, "too many queries");
  k_merge_rescore<<<(int)n_queries, kMergeThreads, smem, as_stream(stream)>>>(
      part_val, part_idx, n_list, q_f32, ld_q, d_f32, ld_d, d_index_base, d_rows, n_pix, q_norm, d_norm, q_lp_scale,
      similarity, n_rescore, k_out, run_val, run_idx, sort_n, out_val, out_idx, gate_rel, n_rescored);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_merge_rescore(const float* part_val, const int32_t* part_idx, int64_t n_queries,
                                  int part_slots, int n_cand, const float* q_f32, int64_t ld_q,
                                  const float* d_f32, int64_t ld_d, int64_t d_index_base,
                                  int64_t d_rows, int n_pix,
                                  const float* q_norm, const float* d_norm, const float* q_lp_scale,
                                  int similarity,
                                  int n_rescore, int k_out, const float* run_val,
                                  const int64_t* run_idx, float* out_val, int64_t* out_idx,
                                  void* stream) {
  return ebsd_merge_rescore_gated(part_val, part_idx, n_queries, part_slots, n_cand, q_f32, ld_q, d_f32, ld_d,
                                  d_index_base, d_rows, n_pix, q_norm, d_norm, q_lp_scale, similarity, n_rescore,
                                  k_out, run_val, run_idx, out_val, out_idx, 0.0f, nullptr, stream);
}
