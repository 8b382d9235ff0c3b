// K1: dictionary projector and K2: pattern preparation.
//
// K1 follows ebsdtorch/ebsd/indexing.py:117-143: rotate each unit detector
// ray by the orientation (qu_apply, quaternions.py:186-213), map it to the
// side-by-side square Lambert projection (rosca_lambert_side_by_side,
// sphere.py:145-185), sample the (H, 2W) master pattern bilinearly with
// grid_sample semantics (align_corners=False, padding_mode="border";
// master_pattern.py:197-206), then subtract the row mean.
// K2 follows experiment_pats.py:318-346 (avg-pool binning) and
// indexing.py:175-187 (mask select, row mean subtraction).
//
// Both end in the same row finaliser: the zero-mean FP32 row, its L2 norm, and
// a unit-norm copy in the low-precision matching type (bf16, or e4m3 with a
// per-row absmax scale), zero padded to the GEMM row length.
#include <algorithm>

#include "common.cuh"
#include "sampling.cuh"

namespace ebsd {

constexpr int kRowThreads = 512;
constexpr int kProjIlp = 2;  // independent pixels per projector thread and step
constexpr int kMaxRowPix = 57344;  // 224 KiB of fp32 in shared memory

struct RowOut {
  float* f32;
  int64_t ld_f32;
  void* lp;
  int lp_dtype;
  int64_t ld_lp;
  float* norm;
  float* lp_scale;
};

// Row values are in row[0..n); part_sum is this thread's sum of the values it
// wrote. Finalise and write the outputs of row `r` (the shared row itself is
// left as it was): mean (FP64 block sum), then the norm and absmax of the
// zero-mean row, then the FP32 and low-precision rows in one pass (16-byte
// stores when the row length and strides allow).
__device__ void finalize_row(const float* row, int n, int subtract_mean, float part_sum, int64_t r,
                             const RowOut& o, float* fred, double* dred) {
  const int tid = threadIdx.x;
  double mean = 0.0;
  if (subtract_mean) mean = block_sum<double>((double)part_sum, dred) / (double)n;
  const float meanf = (float)mean;
  float ss = 0.0f, amax = 0.0f;
  for (int p = tid; p < n; p += blockDim.x) {
    const float v = row[p] - meanf;
    ss += v * v;
    amax = fmaxf(amax, fabsf(v));
  }
  const double nrm2 = block_sum<double>((double)ss, dred);
  const float nrm = (float)sqrt(nrm2);
  const float inv = nrm > 0.0f ? 1.0f / nrm : 0.0f;
  float qscale = 1.0f;
  if (o.lp && o.lp_dtype == EBSD_DT_E4M3) {
    const float m = block_max(amax, fred) * inv;  // absmax of the unit row
    qscale = m > 0.0f ? m / 448.0f : 1.0f;
  }
  if (tid == 0) {
    if (o.norm) o.norm[r] = nrm;
    if (o.lp_scale) o.lp_scale[r] = qscale;
  }
  float* f32 = o.f32 ? o.f32 + r * o.ld_f32 : nullptr;
  const bool bf16 = o.lp && o.lp_dtype == EBSD_DT_BF16;
  __nv_bfloat16* lp16 = bf16 ? reinterpret_cast<__nv_bfloat16*>(o.lp) + r * o.ld_lp : nullptr;
  const bool vec = (n & 7) == 0 && (!f32 || ((reinterpret_cast<uintptr_t>(f32) & 15) == 0)) &&
                   (!lp16 || ((reinterpret_cast<uintptr_t>(lp16) & 15) == 0)) && (o.lp == nullptr || bf16);
  if (vec) {
    // eight values per thread and step: two float4 loads and stores, one
    // 16-byte bf16 store
    for (int c = tid; c < n / 8; c += blockDim.x) {
      const float4 a = reinterpret_cast<const float4*>(row)[2 * c];
      const float4 b = reinterpret_cast<const float4*>(row)[2 * c + 1];
      const float v[8] = {a.x - meanf, a.y - meanf, a.z - meanf, a.w - meanf,
                          b.x - meanf, b.y - meanf, b.z - meanf, b.w - meanf};
      if (f32) {
        reinterpret_cast<float4*>(f32)[2 * c] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4*>(f32)[2 * c + 1] = make_float4(v[4], v[5], v[6], v[7]);
      }
      if (lp16) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) h[e] = __float2bfloat16_rn(v[e] * inv);
        reinterpret_cast<uint4*>(lp16)[c] = *reinterpret_cast<const uint4*>(h);
      }
    }
    if (lp16)
      for (int p = n + tid; p < o.ld_lp; p += blockDim.x) lp16[p] = __float2bfloat16_rn(0.0f);
    return;
  }
  if (f32)
    for (int p = tid; p < n; p += blockDim.x) f32[p] = row[p] - meanf;
  if (lp16) {
    for (int p = tid; p < o.ld_lp; p += blockDim.x) lp16[p] = __float2bfloat16_rn(p < n ? (row[p] - meanf) * inv : 0.0f);
  } else if (o.lp) {
    __nv_fp8_e4m3* dst = reinterpret_cast<__nv_fp8_e4m3*>(o.lp) + r * o.ld_lp;
    const float sc = inv / qscale;
    for (int p = tid; p < o.ld_lp; p += blockDim.x) dst[p] = __nv_fp8_e4m3(p < n ? (row[p] - meanf) * sc : 0.0f);
  }
}

__global__ void __launch_bounds__(kRowThreads, 2) k_project(
    const float* __restrict__ mp, int mp_h, int mp_w2, const float* __restrict__ rays, int n_pix,
    const float4* __restrict__ quats, int64_t n_rows, int subtract_mean, RowOut o) {
  extern __shared__ float row[];
  __shared__ float fred[32];
  __shared__ double dred[32];
  const float* rx = rays;
  const float* ry = rays + n_pix;
  const float* rz = rays + 2 * (int64_t)n_pix;
  for (int64_t r = blockIdx.x; r < n_rows; r += gridDim.x) {
    const float4 q = quats[r];
    float part = 0.0f;
    // kProjIlp pixels per thread and step, their master-pattern gathers
    // issued together: the projector is bound by the gather latency through
    // L2, and independent gathers in flight hide it
    for (int p0 = threadIdx.x; p0 < n_pix; p0 += kProjIlp * blockDim.x) {
      BorderTaps t[kProjIlp];
#pragma unroll
      for (int k = 0; k < kProjIlp; ++k) {
        const int p = min(p0 + k * (int)blockDim.x, n_pix - 1);
        const float3 v = rotate(q, __ldg(rx + p), __ldg(ry + p), __ldg(rz + p));
        const float2 uv = lambert_side_by_side(v.x, v.y, v.z);
        t[k] = border_taps(mp_h, mp_w2, uv.x, uv.y);
      }
      float g[kProjIlp][4];
#pragma unroll
      for (int k = 0; k < kProjIlp; ++k) {
        g[k][0] = __ldg(mp + t[k].i00);
        g[k][1] = __ldg(mp + t[k].i01);
        g[k][2] = __ldg(mp + t[k].i10);
        g[k][3] = __ldg(mp + t[k].i11);
      }
#pragma unroll
      for (int k = 0; k < kProjIlp; ++k) {
        const int p = p0 + k * (int)blockDim.x;
        if (p < n_pix) {
          const float val = g[k][0] * t[k].w00 + g[k][1] * t[k].w01 + g[k][2] * t[k].w10 + g[k][3] * t[k].w11;
          row[p] = val;
          part += val;
        }
      }
    }
    __syncthreads();
    finalize_row(row, n_pix, subtract_mean, part, r, o, fred, dred);
    __syncthreads();
  }
}

__device__ __forceinline__ float load_pixel(const float* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ float load_pixel(const uint16_t* p, int64_t i) { return (float)__ldg(p + i); }
__device__ __forceinline__ float load_pixel(const uint8_t* p, int64_t i) { return (float)__ldg(p + i); }
__device__ __forceinline__ float load_pixel(const __half* p, int64_t i) { return __half2float(__ldg(p + i)); }

// Patterns of type T (fp32, uint16 or uint8 detector counts, fp16) -> rows.
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_prep(const T* __restrict__ pats, int64_t n_rows,
                                                      int h, int w, int64_t stride, int b,
                                                      const int32_t* __restrict__ pix, int n_pix,
                                                      int subtract_mean, RowOut o) {
  extern __shared__ float row[];
  __shared__ float fred[32];
  __shared__ double dred[32];
  const int wb = w / b;
  const float cnt = (float)(b * b);
  for (int64_t r = blockIdx.x; r < n_rows; r += gridDim.x) {
    const T* img = pats + r * stride;
    float part = 0.0f;
    for (int p = threadIdx.x; p < n_pix; p += blockDim.x) {
      const int idx = pix ? __ldg(pix + p) : p;
      float v;
      if (b == 1) {
        v = load_pixel(img, idx);
      } else {
        const int i = idx / wb, j = idx - i * wb;
        const int64_t src = (int64_t)(i * b) * w + j * b;
        float s = 0.0f;
        for (int a = 0; a < b; ++a)
          for (int c = 0; c < b; ++c) s += load_pixel(img, src + (int64_t)a * w + c);
        v = s / cnt;
      }
      row[p] = v;
      part += v;
    }
    __syncthreads();
    finalize_row(row, n_pix, subtract_mean, part, r, o, fred, dred);
    __syncthreads();
  }
}

__global__ void k_sample_points(const float* __restrict__ mp, int mp_h, int mp_w2,
                                const float* __restrict__ xyz, int64_t n, int normalize,
                                float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (normalize) {
      const float nrm = sqrtf(x * x + y * y + z * z);
      x /= nrm;
      y /= nrm;
      z /= nrm;
    }
    const float2 uv = lambert_side_by_side(x, y, z);
    out[i] = sample_border(mp, mp_h, mp_w2, uv.x, uv.y);
  }
}

static int check_row_out(const RowOut& o, int n_pix) {
  EBSD_ARG_CHECK(!o.f32 || o.ld_f32 >= n_pix, "ld_f32 (%lld) < row length (%d)", (long long)o.ld_f32,
                 n_pix);
  if (o.lp) {
    EBSD_ARG_CHECK(o.lp_dtype == EBSD_DT_BF16 || o.lp_dtype == EBSD_DT_E4M3,
                   "lp_dtype must be EBSD_DT_BF16 or EBSD_DT_E4M3");
    EBSD_ARG_CHECK(o.ld_lp >= n_pix, "ld_lp (%lld) < row length (%d)", (long long)o.ld_lp, n_pix);
  }
  return 0;
}

static int row_grid(int64_t n_rows, size_t smem, const void* fn) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kRowThreads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int64_t cap = (int64_t)device_sm_count() * per_sm * 8;
  return (int)std::min<int64_t>(n_rows, cap);
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_project_dictionary(const float* master_pattern, int mp_h, int mp_w2,
                                       const float* rays_soa, int n_pix, const float* quats,
                                       int64_t n_rows, int subtract_mean, float* out_f32,
                                       int64_t ld_f32, void* out_lp, int lp_dtype, int64_t ld_lp,
                                       float* out_norm, float* out_lp_scale, void* stream) {
  EBSD_ARG_CHECK(master_pattern && rays_soa && quats, "ebsd_project_dictionary: null input");
  EBSD_ARG_CHECK(mp_h >= 1 && mp_w2 >= 1, "master pattern shape (%d, %d) invalid", mp_h, mp_w2);
  EBSD_ARG_CHECK(n_pix >= 1 && n_pix <= kMaxRowPix, "row length %d outside [1, %d]", n_pix,
                 kMaxRowPix);
  EBSD_ARG_CHECK(n_rows >= 0, "n_rows < 0");
  EBSD_ARG_CHECK((reinterpret_cast<uintptr_t>(quats) & 15) == 0, "quats must be 16-byte aligned");
  RowOut o{out_f32, ld_f32, out_lp, lp_dtype, ld_lp, out_norm, out_lp_scale};
  if (int rc = check_row_out(o, n_pix)) return rc;
  if (n_rows == 0) return 0;
  const size_t smem = (size_t)n_pix * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_project, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
  const int grid = row_grid(n_rows, smem, (const void*)k_project);
  k_project<<<grid, kRowThreads, smem, as_stream(stream)>>>(
      master_pattern, mp_h, mp_w2, rays_soa, n_pix, reinterpret_cast<const float4*>(quats), n_rows,
      subtract_mean, o);
  EBSD_LAUNCH_CHECK();
  return 0;
}

template <typename T>
static int launch_prep(const T* patterns, int64_t n_rows, int height, int width, int64_t pattern_stride,
                       int binning, const int32_t* pix_index, int n_pix, int subtract_mean, const RowOut& o,
                       void* stream) {
  const size_t smem = (size_t)n_pix * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_prep<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = row_grid(n_rows, smem, (const void*)k_prep<T>);
  k_prep<T><<<grid, kRowThreads, smem, as_stream(stream)>>>(patterns, n_rows, height, width, pattern_stride,
                                                           binning, pix_index, n_pix, subtract_mean, o);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_prep_patterns_typed(const void* patterns, int pattern_dtype, int64_t n_rows, int height,
                                        int width, int64_t pattern_stride, int binning, const int32_t* pix_index,
                                        int n_pix, int subtract_mean, float* out_f32, int64_t ld_f32, void* out_lp,
                                        int lp_dtype, int64_t ld_lp, float* out_norm, float* out_lp_scale,
                                        void* stream) {
  EBSD_ARG_CHECK(patterns != nullptr, "ebsd_prep_patterns: null patterns");
  EBSD_ARG_CHECK(pattern_dtype >= EBSD_PAT_F32 && pattern_dtype <= EBSD_PAT_F16, "unknown pattern_dtype %d",
                 pattern_dtype);
  EBSD_ARG_CHECK(binning >= 1 && height % binning == 0 && width % binning == 0,
                 "binning %d must divide the pattern shape (%d, %d)", binning, height, width);
  const int n_binned = (height / binning) * (width / binning);
  EBSD_ARG_CHECK(n_pix >= 1 && n_pix <= kMaxRowPix, "row length %d outside [1, %d]", n_pix,
                 kMaxRowPix);
  EBSD_ARG_CHECK(pix_index || n_pix == n_binned,
                 "without a pixel index the row length must equal the binned pixel count");
  EBSD_ARG_CHECK(pattern_stride >= (int64_t)height * width, "pattern_stride too small");
  RowOut o{out_f32, ld_f32, out_lp, lp_dtype, ld_lp, out_norm, out_lp_scale};
  if (int rc = check_row_out(o, n_pix)) return rc;
  if (n_rows == 0) return 0;
  switch (pattern_dtype) {
    case EBSD_PAT_U16:
      return launch_prep(static_cast<const uint16_t*>(patterns), n_rows, height, width, pattern_stride, binning,
                         pix_index, n_pix, subtract_mean, o, stream);
    case EBSD_PAT_U8:
      return launch_prep(static_cast<const uint8_t*>(patterns), n_rows, height, width, pattern_stride, binning,
                         pix_index, n_pix, subtract_mean, o, stream);
    case EBSD_PAT_F16:
      return launch_prep(static_cast<const __half*>(patterns), n_rows, height, width, pattern_stride, binning,
                         pix_index, n_pix, subtract_mean, o, stream);
    default:
      return launch_prep(static_cast<const float*>(patterns), n_rows, height, width, pattern_stride, binning,
                         pix_index, n_pix, subtract_mean, o, stream);
  }
}

extern "C" int ebsd_prep_patterns(const float* patterns, int64_t n_rows, int height, int width,
                                  int64_t pattern_stride, int binning, const int32_t* pix_index,
                                  int n_pix, int subtract_mean, float* out_f32, int64_t ld_f32,
                                  void* out_lp, int lp_dtype, int64_t ld_lp, float* out_norm,
                                  float* out_lp_scale, void* stream) {
  return ebsd_prep_patterns_typed(patterns, EBSD_PAT_F32, n_rows, height, width, pattern_stride, binning,
                                  pix_index, n_pix, subtract_mean, out_f32, ld_f32, out_lp, lp_dtype, ld_lp,
                                  out_norm, out_lp_scale, stream);
}

extern "C" int ebsd_sample_master_pattern(const float* master_pattern, int mp_h, int mp_w2,
                                          const float* xyz, int64_t n, int normalize, float* out,
                                          void* stream) {
  EBSD_ARG_CHECK(master_pattern && xyz && out, "ebsd_sample_master_pattern: null pointer");
  EBSD_ARG_CHECK(mp_h >= 1 && mp_w2 >= 1 && n >= 0, "ebsd_sample_master_pattern: bad sizes");
  if (n == 0) return 0;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)device_sm_count() * 16);
  k_sample_points<<<blocks, 256, 0, as_stream(stream)>>>(master_pattern, mp_h, mp_w2, xyz, n,
                                                         normalize, out);
  EBSD_LAUNCH_CHECK();
  return 0;
}
