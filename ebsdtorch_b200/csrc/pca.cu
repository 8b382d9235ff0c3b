// PCA support kernels (A11/A12).
//
// The reference builds the covariance with Chan/Welford batch updates in
// FP32 (ebsdtorch/utils/pca_covmat.py:53-91) and projects with FP32
// torch.matmul (indexing.py:401, 421, 452). Here both products run on the
// bf16 tensor-core GEMM (ebsd_gemm_nt) over a tripled K: each FP32 operand is
// split as x = hi + lo (hi = bf16(x), lo = bf16(x - hi)) and
//   [hi | hi | lo] . [hi' | lo' | hi'] = hi hi' + hi lo' + lo hi',
// which keeps the product accurate to ~2^-17 relative (FP32-class); the
// covariance is formed from column-centred data (two-pass, no Welford update
// needed once the mean is known).
#include "common.cuh"

namespace ebsd {

// Column sums via per-block partial sums in double, one thread per column.
__global__ void k_col_mean(const float* __restrict__ X, int64_t n_rows, int n_cols, int64_t ld,
                           float* __restrict__ mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cols) return;
  double s = 0.0;
  for (int64_t r = 0; r < n_rows; ++r) s += X[r * ld + c];
  mean[c] = (float)(s / (double)n_rows);
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Non-transposed: one output row per input row.
__global__ void k_split3_rows(const float* __restrict__ X, int64_t n_rows, int n_cols, int64_t ld,
                              const float* __restrict__ shift, int pattern,
                              __nv_bfloat16* __restrict__ out, int64_t ld_out, int64_t seg) {
  const int64_t r = blockIdx.y * (int64_t)gridDim.z + blockIdx.z;  // one row per (y, z)
  if (r >= n_rows) return;
  const float* src = X + r * ld;
  __nv_bfloat16* dst = out + r * ld_out;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < seg;
       c += (int64_t)gridDim.x * blockDim.x) {
    __nv_bfloat16 hi = __float2bfloat16_rn(0.0f), lo = hi;
    if (c < n_cols) split_bf16(src[c] - (shift ? shift[c] : 0.0f), hi, lo);
    dst[c] = hi;
    dst[seg + c] = pattern == 0 ? hi : lo;
    dst[2 * seg + c] = pattern == 0 ? lo : hi;
  }
  // zero the tail beyond the three segments
  for (int64_t c = 3 * seg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ld_out;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = __float2bfloat16_rn(0.0f);
}

// Transposed: column c of X becomes output row c. 32x32 tiles through smem.
__global__ void k_split3_cols(const float* __restrict__ X, int64_t n_rows, int n_cols, int64_t ld,
                              const float* __restrict__ shift, int pattern,
                              __nv_bfloat16* __restrict__ out, int64_t ld_out, int64_t seg) {
  __shared__ float tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;  // input row block (-> output column)
  const int c0 = blockIdx.y * 32;               // input column block (-> output row)
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    const int64_t r = r0 + i;
    const int c = c0 + tx;
    float v = 0.0f;
    if (r < n_rows && c < n_cols) v = X[r * ld + c] - (shift ? shift[c] : 0.0f);
    tile[i][tx] = v;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int c = c0 + i;  // output row
    const int64_t r = r0 + tx;  // output column within segment
    if (c < n_cols && r < seg) {
      __nv_bfloat16 hi, lo;
      split_bf16(tile[tx][i], hi, lo);
      __nv_bfloat16* dst = out + (int64_t)c * ld_out;
      dst[r] = hi;
      dst[seg + r] = pattern == 0 ? hi : lo;
      dst[2 * seg + r] = pattern == 0 ? lo : hi;
    }
  }
}

__global__ void k_zero_tail_rows(__nv_bfloat16* __restrict__ out, int n_rows, int64_t ld_out,
                                 int64_t from) {
  const int r = blockIdx.y;
  if (r >= n_rows) return;
  for (int64_t c = from + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ld_out;
       c += (int64_t)gridDim.x * blockDim.x)
    out[(int64_t)r * ld_out + c] = __float2bfloat16_rn(0.0f);
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_col_mean(const float* X, int64_t n_rows, int n_cols, int64_t ld, float* mean,
                             void* stream) {
  EBSD_ARG_CHECK(X && mean, "ebsd_col_mean: null pointer");
  EBSD_ARG_CHECK(n_rows >= 1 && n_cols >= 1 && ld >= n_cols, "ebsd_col_mean: bad sizes");
  k_col_mean<<<ceil_div(n_cols, 128), 128, 0, as_stream(stream)>>>(X, n_rows, n_cols, ld, mean);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_split3_bf16(const float* X, int64_t n_rows, int n_cols, int64_t ld,
                                const float* shift, int transpose, int pattern, void* out,
                                int64_t ld_out, int64_t seg_len, void* stream) {
  EBSD_ARG_CHECK(X && out, "ebsd_split3_bf16: null pointer");
  EBSD_ARG_CHECK(n_rows >= 1 && n_cols >= 1 && ld >= n_cols, "ebsd_split3_bf16: bad sizes");
  EBSD_ARG_CHECK(pattern == 0 || pattern == 1, "pattern must be 0 or 1");
  EBSD_ARG_CHECK(ld_out >= 3 * seg_len, "ld_out < 3 * seg_len");
  __nv_bfloat16* o = reinterpret_cast<__nv_bfloat16*>(out);
  cudaStream_t s = as_stream(stream);
  if (!transpose) {
    EBSD_ARG_CHECK(seg_len >= n_cols, "seg_len < n_cols");
    const int gz = (int)std::min<int64_t>(n_rows, 65535);
    const int gy = ceil_div(n_rows, gz);
    EBSD_ARG_CHECK(gy <= 65535, "too many rows");
    dim3 grid(ceil_div(std::min<int64_t>(seg_len, 4096), 256), gy, gz);
    k_split3_rows<<<grid, 256, 0, s>>>(X, n_rows, n_cols, ld, shift, pattern, o, ld_out, seg_len);
  } else {
    EBSD_ARG_CHECK(seg_len >= n_rows, "seg_len < n_rows");
    EBSD_ARG_CHECK(ceil_div(n_cols, 32) <= 65535, "too many columns");
    // zero-pad segment tails [n_rows, seg_len) via the tile kernel covering seg_len rows
    dim3 grid(ceil_div(seg_len, 32), ceil_div(n_cols, 32));
    k_split3_cols<<<grid, dim3(32, 8), 0, s>>>(X, n_rows, n_cols, ld, shift, pattern, o, ld_out,
                                               seg_len);
    EBSD_LAUNCH_CHECK();
    if (ld_out > 3 * seg_len) {
      dim3 g2(ceil_div(ld_out - 3 * seg_len, 256), n_cols);
      EBSD_ARG_CHECK(n_cols <= 65535, "too many columns");
      k_zero_tail_rows<<<g2, 256, 0, s>>>(o, n_cols, ld_out, 3 * seg_len);
    }
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}
