// Manhattan (L1) distance top-k: the reference's distance_metric="manhattan"
// (ebsdtorch/utils/knn.py:92-93: (query[:, None, :] - data[None, :, :])
// .abs().sum(dim=2), smallest first). Not a contraction, so it runs on the
// CUDA cores: FP32 rows, exact FP32 sums.
//
// One CTA (256 threads) per (64-query tile, dictionary range): for each
// 64-row dictionary tile, the 64 x 64 block of distances is accumulated over
// 32-pixel chunks staged in shared memory (each thread owns a 4 x 4 block),
// then written negated to shared memory, and the thread that owns each
// query row folds the 64 new scores into its sorted top-n_cand in registers.
// The candidate lists have the layout of ebsd_match_topk's (score = -L1,
// best first), so ebsd_merge_rescore (EBSD_SIM_MANHATTAN, no re-score)
// merges them.
#include "common.cuh"

namespace ebsd {

constexpr int L1_TQ = 64, L1_TD = 64, L1_TP = 32, L1_THREADS = 256;

template <int KC>
__device__ __forceinline__ void l1_insert(float (&bv)[KC], int (&bi)[KC], float v, int idx) {
  bv[KC - 1] = v;
  bi[KC - 1] = idx;
#pragma unroll
  for (int j = KC - 1; j > 0; --j) {
    const bool sw = bv[j] > bv[j - 1];
    const float a = bv[j], b = bv[j - 1];
    const int ia = bi[j], ib = bi[j - 1];
    bv[j - 1] = sw ? a : b;
    bv[j] = sw ? b : a;
    bi[j - 1] = sw ? ia : ib;
    bi[j] = sw ? ib : ia;
  }
}

template <int KC>
__global__ void __launch_bounds__(L1_THREADS) k_manhattan_topk(
    const float* __restrict__ q, int64_t ld_q, int64_t n_q, const float* __restrict__ d, int64_t ld_d,
    int64_t n_d, int n_pix, int splits, float* __restrict__ part_val, int32_t* __restrict__ part_idx,
    int part_slots, int slot_base, int32_t index_base) {
  __shared__ float sq[L1_TP][L1_TQ + 1];
  __shared__ float sd[L1_TP][L1_TD + 1];
  __shared__ float sc[L1_TQ][L1_TD + 1];
  const int tid = threadIdx.x;
  const int tile = blockIdx.x / splits, split = blockIdx.x - tile * splits;
  const int64_t q0 = (int64_t)tile * L1_TQ;
  const int64_t n_dtiles = (n_d + L1_TD - 1) / L1_TD;
  const int64_t t_begin = split * n_dtiles / splits, t_end = (split + 1) * n_dtiles / splits;
  const int ty = tid / 16, tx = tid % 16;  // 4 x 4 outputs at rows ty*4.., cols tx*4..
  float bv[KC];
  int bi[KC];
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    bv[j] = -INFINITY;
    bi[j] = -1;
  }
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int64_t d0 = t * L1_TD;
    float acc[4][4] = {};
    for (int p0 = 0; p0 < n_pix; p0 += L1_TP) {
      // stage 64 x 32 of each side (row-major in global, pixel-major in shared)
      for (int e = tid; e < L1_TQ * L1_TP; e += L1_THREADS) {
        const int r = e / L1_TP, c = e % L1_TP;
        const int64_t gq = q0 + r;
        const int gp = p0 + c;
        sq[c][r] = (gq < n_q && gp < n_pix) ? q[gq * ld_q + gp] : 0.0f;
        const int64_t gd = d0 + r;
        sd[c][r] = (gd < n_d && gp < n_pix) ? d[gd * ld_d + gp] : 0.0f;
      }
      __syncthreads();
#pragma unroll 4
      for (int c = 0; c < L1_TP; ++c) {
        float a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          a[i] = sq[c][ty * 4 + i];
          b[i] = sd[c][tx * 4 + i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] += fabsf(a[i] - b[j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool valid = d0 + tx * 4 + j < n_d;
        sc[ty * 4 + i][tx * 4 + j] = valid ? -acc[i][j] : -INFINITY;
      }
    __syncthreads();
    if (tid < L1_TQ) {
      for (int j = 0; j < L1_TD; ++j) {
        const float v = sc[tid][j];
        if (v > bv[KC - 1]) l1_insert<KC>(bv, bi, v, (int)(d0 + j) + index_base);
      }
    }
    __syncthreads();
  }
  if (tid < L1_TQ) {
    const int64_t gq = q0 + tid;
    const int64_t base = (gq * part_slots + slot_base + split) * KC;
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      part_val[base + j] = bv[j];
      part_idx[base + j] = bi[j];
    }
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_manhattan_topk(const float* q_f32, int64_t ld_q, int64_t n_queries, int64_t n_queries_pad,
                                   const float* d_f32, int64_t ld_d, int64_t n_dict, int n_pix, int n_cand,
                                   int splits, float* part_val, int32_t* part_idx, int part_slots, int slot_base,
                                   int32_t index_base, void* stream) {
  EBSD_ARG_CHECK(q_f32 && d_f32 && part_val && part_idx, "ebsd_manhattan_topk: null pointer");
  EBSD_ARG_CHECK(n_queries >= 1 && n_queries <= n_queries_pad && n_queries_pad % L1_TQ == 0,
                 "n_queries_pad %lld must be a multiple of %d and hold n_queries %lld", (long long)n_queries_pad,
                 L1_TQ, (long long)n_queries);
  EBSD_ARG_CHECK(n_dict >= 1 && n_pix >= 1 && ld_q >= n_pix && ld_d >= n_pix, "bad row sizes");
  EBSD_ARG_CHECK((int64_t)index_base + n_dict <= INT32_MAX, "dictionary index overflow");
  const int64_t n_dtiles = (n_dict + L1_TD - 1) / L1_TD;
  EBSD_ARG_CHECK(splits >= 1 && splits <= n_dtiles, "splits %d outside [1, %lld dictionary tiles of %d]", splits,
                 (long long)n_dtiles, L1_TD);
  EBSD_ARG_CHECK(slot_base >= 0 && slot_base + splits <= part_slots, "part_slots (%d) < slot_base (%d) + splits (%d)",
                 part_slots, slot_base, splits);
  const int64_t grid = n_queries_pad / L1_TQ * splits;
  EBSD_ARG_CHECK(grid < INT32_MAX, "too many work units");
  cudaStream_t s = as_stream(stream);
  // queries beyond n_queries read zero rows and write candidates nobody reads
  // (the part lists cover n_queries_pad rows)
  switch (n_cand) {
#define EBSD_L1_CASE(KC)                                                                                    \
  case KC:                                                                                                  \
    k_manhattan_topk<KC><<<(int)grid, L1_THREADS, 0, s>>>(q_f32, ld_q, n_queries, d_f32, ld_d, n_dict, n_pix, \
                                                         splits, part_val, part_idx, part_slots, slot_base,  \
                                                         index_base);                                        \
    break;
    EBSD_L1_CASE(1)
    EBSD_L1_CASE(2)
    EBSD_L1_CASE(4)
    EBSD_L1_CASE(8)
    EBSD_L1_CASE(16)
    EBSD_L1_CASE(32)
    EBSD_L1_CASE(64)
#undef EBSD_L1_CASE
    default:
      set_error("n_cand %d not in {1,2,4,8,16,32,64}", n_cand);
      return EBSD_ERR_ARG;
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}
