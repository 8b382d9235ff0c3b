// Support kernels of the orientation-proposal CNN (no counterpart in the
// reference, which has no learned indexer). Convolutions are 3x3, stride 2,
// padding 1, NHWC activations; a convolution runs as im2col + the bf16
// tensor-core GEMM (ebsd_gemm_nt) forward, and as two GEMMs (weight gradient
// and column gradient) + col2im backward. The fully connected head uses the
// FP32 SIMT kernels below. Optimiser: Adam on FP32 master weights, which also
// refreshes the bf16 copies the GEMMs read.
#include <algorithm>

#include "common.cuh"

namespace ebsd {

static int nblocks(int64_t n, int per = 256) {
  return (int)std::min<int64_t>((n + per - 1) / per, (int64_t)device_sm_count() * 16);
}

// cols[(b, oy, ox), (ky, kx, c)] = x[b, 2 oy - 1 + ky, 2 ox - 1 + kx, c] (0 outside);
// rows >= M and columns >= K of the padded output (row stride ld, ld % 8 == 0)
// are zero. One thread per 8-column chunk of a row, consecutive threads on
// consecutive chunks, so each warp's 16-byte stores are contiguous; with
// C % 8 == 0 (vec) a chunk lies in one tap and is one 16-byte load. Rows
// [r0, r0 + n_rows) per launch, with 32-bit chunk indices.
__global__ void k_im2col(const __nv_bfloat16* __restrict__ x, int H, int W, int C, int Ho, int Wo, int M, int r0,
                         int n_rows, int ld, int vec, __nv_bfloat16* __restrict__ cols) {
  const int nj = ld >> 3;
  const unsigned total = (unsigned)n_rows * (unsigned)nj;
  const int K = 9 * C, hw = Ho * Wo;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int rl = (int)(t / (unsigned)nj);
    const int j = (int)(t - (unsigned)rl * (unsigned)nj);
    const int r = r0 + rl, k0 = 8 * j;
    uint4 chunk = make_uint4(0u, 0u, 0u, 0u);
    if (r < M && k0 < K) {
      const int b = r / hw, rem = r - b * hw;
      const int oy = rem / Wo, ox = rem - oy * Wo;
      if (vec) {
        const int tap = k0 / C, c0 = k0 - tap * C;
        const int iy = 2 * oy - 1 + tap / 3, ix = 2 * ox - 1 + tap % 3;
        if (iy >= 0 && iy < H && ix >= 0 && ix < W)
          chunk = __ldg(reinterpret_cast<const uint4*>(x + (((int64_t)b * H + iy) * W + ix) * C + c0));
      } else {
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = k0 + e;
          __nv_bfloat16 val = __float2bfloat16_rn(0.f);
          if (k < K) {
            const int tap = k / C, c = k - tap * C;
            const int iy = 2 * oy - 1 + tap / 3, ix = 2 * ox - 1 + tap % 3;
            if (iy >= 0 && iy < H && ix >= 0 && ix < W) val = x[(((int64_t)b * H + iy) * W + ix) * C + c];
          }
          v[e] = val;
        }
        chunk = *reinterpret_cast<const uint4*>(v);
      }
    }
    *reinterpret_cast<uint4*>(cols + (int64_t)r * ld + k0) = chunk;
  }
}

// The same for C % 8 == 0 (C <= 32) with 16-byte aligned input: one thread
// per (output pixel, tap) pair copies the tap's C channels in 16-byte chunks
// (the pixel's coordinates decoded once per pair instead of once per chunk);
// tap 9 writes the zero padding of K from 9 C to ld. Measured at 128 x 128,
// batch 4,096: 0.90 ms against 0.97 ms for C = 32; for C = 64-256 one thread
// per chunk was up to 2x faster (more loads in flight), so it keeps that.
__global__ void k_im2col_taps(const __nv_bfloat16* __restrict__ x, int H, int W, int C, int Ho, int Wo, int M,
                              int r0, int n_rows, int ld, int ntap, __nv_bfloat16* __restrict__ cols) {
  const unsigned total = (unsigned)n_rows * (unsigned)ntap;
  const int hw = Ho * Wo, nc = C >> 3;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int rl = (int)(t / (unsigned)ntap);
    const int tap = (int)(t - (unsigned)rl * (unsigned)ntap);
    const int r = r0 + rl;
    uint4* dst = reinterpret_cast<uint4*>(cols + (int64_t)r * ld);
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    if (tap == 9) {  // K padding
      for (int j = (9 * C) >> 3; j < (ld >> 3); ++j) dst[j] = zero;
      continue;
    }
    const uint4* src = nullptr;
    if (r < M) {
      const int b = r / hw, rem = r - b * hw;
      const int oy = rem / Wo, ox = rem - oy * Wo;
      const int iy = 2 * oy - 1 + tap / 3, ix = 2 * ox - 1 + tap % 3;
      if (iy >= 0 && iy < H && ix >= 0 && ix < W)
        src = reinterpret_cast<const uint4*>(x + (((int64_t)b * H + iy) * W + ix) * C);
    }
    uint4* d = dst + tap * nc;
    if (src) {
      for (int j = 0; j < nc; ++j) d[j] = __ldg(src + j);
    } else {
      for (int j = 0; j < nc; ++j) d[j] = zero;
    }
  }
}

// Direct convolution of a single-channel input (the first layer):
// out[(b, oy, ox), c] = act(sum_{ky,kx} x[b, 2 oy - 1 + ky, 2 ox - 1 + kx] w[c, 3 ky + kx] + bias[c]),
// one thread per output pixel and all COUT channels, weights (bf16, as the
// GEMM path reads them) broadcast from shared memory, 16-byte stores.
template <int COUT>
__global__ void k_conv_c1(const __nv_bfloat16* __restrict__ x, int H, int W, int Ho, int Wo, int M,
                          const __nv_bfloat16* __restrict__ w16, int ldw, const float* __restrict__ bias, int relu,
                          __nv_bfloat16* __restrict__ out, float* __restrict__ out32) {
  __shared__ float ws[COUT][9];
  __shared__ float bs[COUT];
  for (int i = threadIdx.x; i < COUT * 9; i += blockDim.x) ws[i / 9][i % 9] = __bfloat162float(w16[(i / 9) * ldw + i % 9]);
  for (int i = threadIdx.x; i < COUT; i += blockDim.x) bs[i] = bias ? bias[i] : 0.f;
  __syncthreads();
  const int hw = Ho * Wo;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
    const int b = r / hw, rem = r - b * hw;
    const int oy = rem / Wo, ox = rem - oy * Wo;
    float xv[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int iy = 2 * oy - 1 + t / 3, ix = 2 * ox - 1 + t % 3;
      xv[t] = (iy >= 0 && iy < H && ix >= 0 && ix < W) ? __bfloat162float(x[((int64_t)b * H + iy) * W + ix]) : 0.f;
    }
    // one 8-channel group at a time: fully unrolled over all COUT channels
    // the kernel needed 186 registers (one CTA per SM)
#pragma unroll 1
    for (int c = 0; c < COUT; c += 8) {
      float o[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        float acc = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) acc = fmaf(xv[t], ws[c + e][t], acc);
        acc += bs[c + e];
        o[e] = relu ? fmaxf(acc, 0.f) : acc;
      }
      __align__(16) __nv_bfloat16 v[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16_rn(o[e]);
      *reinterpret_cast<uint4*>(out + (int64_t)r * COUT + c) = *reinterpret_cast<const uint4*>(v);
      if (out32) {
        float4* d = reinterpret_cast<float4*>(out32 + (int64_t)r * COUT + c);
        d[0] = make_float4(o[0], o[1], o[2], o[3]);
        d[1] = make_float4(o[4], o[5], o[6], o[7]);
      }
    }
  }
}

// dx[b, iy, ix, c] = sum over the (output, tap) pairs that read it of dcols.
__global__ void k_col2im(const float* __restrict__ dcols, int64_t ld, int B, int H, int W, int C, int Ho, int Wo,
                         float* __restrict__ dx) {
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const int64_t p = t / C;
    const int ix = (int)(p % W), iy = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
    float s = 0.f;
    for (int ky = 0; ky < 3; ++ky) {
      const int ny = iy + 1 - ky;  // = 2 oy
      if (ny < 0 || (ny & 1)) continue;
      const int oy = ny >> 1;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int nx = ix + 1 - kx;
        if (nx < 0 || (nx & 1)) continue;
        const int ox = nx >> 1;
        if (ox >= Wo) continue;
        const int64_t r = ((int64_t)b * Ho + oy) * Wo + ox;
        s += dcols[r * ld + (ky * 3 + kx) * C + c];
      }
    }
    dx[t] = s;
  }
}

// out = act(y + bias) as bf16 (M x C, row stride ld_out); act: 0 none, 1 ReLU
__global__ void k_bias_act(const float* __restrict__ y, int64_t ldy, const float* __restrict__ bias, int64_t M, int C,
                           int relu, __nv_bfloat16* __restrict__ out, int64_t ld_out, float* __restrict__ out32) {
  const int64_t total = M * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / C;
    const int c = (int)(t - r * C);
    float v = y[r * ldy + c] + (bias ? bias[c] : 0.f);
    if (relu) v = fmaxf(v, 0.f);
    out[r * ld_out + c] = __float2bfloat16_rn(v);
    if (out32) out32[r * C + c] = v;
  }
}

// g = dy * (act > 0) for a ReLU layer whose bf16 output was act; written as
// fp32 (optional) and bf16 (optional, row stride ld_out, zero-padded columns).
__global__ void k_relu_grad(const float* __restrict__ dy, int64_t ldy, const __nv_bfloat16* __restrict__ act,
                            int64_t lda, int64_t M, int C, float* __restrict__ g32, __nv_bfloat16* __restrict__ g16,
                            int64_t ld_out) {
  const int64_t total = M * ld_out;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / ld_out;
    const int c = (int)(t - r * ld_out);
    float v = 0.f;
    if (c < C) v = __bfloat162float(act[r * lda + c]) > 0.f ? dy[r * ldy + c] : 0.f;
    if (g32 && c < C) g32[r * C + c] = v;
    if (g16) g16[t] = __float2bfloat16_rn(v);
  }
}

// Column sums of an (M x C) fp32 matrix into db (one thread per column,
// grid-stride partial sums combined with atomics).
__global__ void k_col_sum(const float* __restrict__ g, int64_t M, int C, float* __restrict__ db) {
  for (int col = threadIdx.x; col < C; col += blockDim.x) {
    float s = 0.f;
    for (int64_t r = blockIdx.x; r < M; r += gridDim.x) s += g[r * C + col];
    atomicAdd(db + col, s);
  }
}

// out (cols_pad x rows_pad, bf16) = in^T for an (rows x cols) matrix of
// bf16 or fp32 (row stride ld_in); padding zero-filled.
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, int64_t rows, int64_t cols, int64_t ld_in,
                            __nv_bfloat16* __restrict__ out, int64_t ld_out) {
  __shared__ float tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32, c0 = (int64_t)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t r = r0 + i, c = c0 + threadIdx.x;
    float v = 0.f;
    if (r < rows && c < cols) v = (float)in[r * ld_in + c];
    tile[i][threadIdx.x] = v;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t c = c0 + i, r = r0 + threadIdx.x;
    out[c * ld_out + r] = __float2bfloat16_rn(tile[threadIdx.x][i]);
  }
}

__global__ void k_scale_cast(const float* __restrict__ x, int64_t n, float scale, __nv_bfloat16* __restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = __float2bfloat16_rn(x[t] * scale);
}

// y (M x N) = x (M x K) W^T (N x K) + b, FP32, 16x16 tiles through smem.
__global__ void k_dense_fwd(const float* __restrict__ x, int64_t ldx, const float* __restrict__ w,
                            const float* __restrict__ b, int M, int N, int K, int relu, float* __restrict__ y,
                            __nv_bfloat16* __restrict__ y16) {
  __shared__ float xs[16][17], ws[16][17];
  const int row = blockIdx.y * 16 + threadIdx.y, col = blockIdx.x * 16 + threadIdx.x;
  float acc = 0.f;
  for (int k0 = 0; k0 < K; k0 += 16) {
    const int kx = k0 + threadIdx.x, ky = k0 + threadIdx.y;
    xs[threadIdx.y][threadIdx.x] = (row < M && kx < K) ? x[(int64_t)row * ldx + kx] : 0.f;
    ws[threadIdx.y][threadIdx.x] = (blockIdx.x * 16 + threadIdx.y < N && kx < K)
                                       ? w[(int64_t)(blockIdx.x * 16 + threadIdx.y) * K + kx] : 0.f;
    (void)ky;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 16; ++j) acc += xs[threadIdx.y][j] * ws[threadIdx.x][j];
    __syncthreads();
  }
  if (row < M && col < N) {
    float v = acc + (b ? b[col] : 0.f);
    if (relu) v = fmaxf(v, 0.f);
    y[(int64_t)row * N + col] = v;
    if (y16) y16[(int64_t)row * N + col] = __float2bfloat16_rn(v);
  }
}

// dW (N x K) = dy^T (N x M) x (M x K), FP32.
__global__ void k_dense_wgrad(const float* __restrict__ dy, const float* __restrict__ x, int64_t ldx, int M, int N,
                              int K, float* __restrict__ dw) {
  __shared__ float ds[16][17], xs[16][17];
  const int n = blockIdx.y * 16 + threadIdx.y, k = blockIdx.x * 16 + threadIdx.x;
  float acc = 0.f;
  for (int m0 = 0; m0 < M; m0 += 16) {
    const int mm = m0 + threadIdx.x;
    ds[threadIdx.y][threadIdx.x] = (n < N && mm < M) ? dy[(int64_t)mm * N + n] : 0.f;
    const int mr = m0 + threadIdx.y;
    xs[threadIdx.y][threadIdx.x] = (mr < M && k < K) ? x[(int64_t)mr * ldx + k] : 0.f;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 16; ++j) acc += ds[threadIdx.y][j] * xs[j][threadIdx.x];
    __syncthreads();
  }
  if (n < N && k < K) dw[(int64_t)n * K + k] = acc;
}

// dx (M x K) = dy (M x N) W (N x K), FP32.
__global__ void k_dense_dgrad(const float* __restrict__ dy, const float* __restrict__ w, int M, int N, int K,
                              float* __restrict__ dx) {
  __shared__ float ds[16][17], ws[16][17];
  const int m = blockIdx.y * 16 + threadIdx.y, k = blockIdx.x * 16 + threadIdx.x;
  float acc = 0.f;
  for (int n0 = 0; n0 < N; n0 += 16) {
    const int nn = n0 + threadIdx.x;
    ds[threadIdx.y][threadIdx.x] = (m < M && nn < N) ? dy[(int64_t)m * N + nn] : 0.f;
    const int nr = n0 + threadIdx.y;
    ws[threadIdx.y][threadIdx.x] = (nr < N && k < K) ? w[(int64_t)nr * K + k] : 0.f;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 16; ++j) acc += ds[threadIdx.y][j] * ws[j][threadIdx.x];
    __syncthreads();
  }
  if (m < M && k < K) dx[(int64_t)m * K + k] = acc;
}

// Adam on FP32 master weights (rows x cols); also writes the bf16 copy
// (row stride ld16, padding untouched) and its transpose (row stride ld16t).
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int64_t rows, int cols, float lr, float b1, float b2, float eps,
                       float c1, float c2, float wd, __nv_bfloat16* __restrict__ w16, int64_t ld16,
                       __nv_bfloat16* __restrict__ w16t, int64_t ld16t) {
  const int64_t n = rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const float gr = g[t] + wd * w[t];
    const float mm = b1 * m[t] + (1.f - b1) * gr;
    const float vv = b2 * v[t] + (1.f - b2) * gr * gr;
    m[t] = mm;
    v[t] = vv;
    const float wn = w[t] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    w[t] = wn;
    const int64_t r = t / cols;
    const int c = (int)(t - r * cols);
    if (w16) w16[r * ld16 + c] = __float2bfloat16_rn(wn);
    if (w16t) w16t[(int64_t)c * ld16t + r] = __float2bfloat16_rn(wn);
  }
}

}  // namespace ebsd

using namespace ebsd;

#define CNN_STREAM as_stream(stream)

extern "C" int ebsd_cnn_im2col(const void* x, int B, int H, int W, int C, int64_t m_pad, int ld, void* cols,
                               void* stream) {
  EBSD_ARG_CHECK(x && cols && B > 0 && H > 0 && W > 0 && C > 0, "ebsd_cnn_im2col: bad arguments");
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
  const int64_t M = (int64_t)B * Ho * Wo;
  EBSD_ARG_CHECK(ld >= 9 * C && ld % 8 == 0 && m_pad >= M, "ebsd_cnn_im2col: output too small or ld % 8 != 0");
  EBSD_ARG_CHECK(m_pad < INT32_MAX && (int64_t)B * H * W * C < ((int64_t)1 << 40), "ebsd_cnn_im2col: too large");
  EBSD_ARG_CHECK(((uintptr_t)cols & 15) == 0, "ebsd_cnn_im2col: cols must be 16-byte aligned");
  const int vec = (C % 8 == 0) && (((uintptr_t)x & 15) == 0);
  const int64_t nj = ld / 8;
  const int64_t rows_per = std::max<int64_t>(1, (INT32_MAX / 2) / nj);
  const int ntap = ld > 9 * C ? 10 : 9;
  for (int64_t r0 = 0; r0 < m_pad; r0 += rows_per) {
    const int n_rows = (int)std::min(rows_per, m_pad - r0);
    if (vec && C <= 32) {  // wider taps: one thread per 16-byte chunk keeps more loads in flight
      k_im2col_taps<<<nblocks((int64_t)n_rows * ntap), 256, 0, CNN_STREAM>>>(
          reinterpret_cast<const __nv_bfloat16*>(x), H, W, C, Ho, Wo, (int)M, (int)r0, n_rows, ld, ntap,
          reinterpret_cast<__nv_bfloat16*>(cols));
    } else {
      k_im2col<<<nblocks((int64_t)n_rows * nj), 256, 0, CNN_STREAM>>>(
          reinterpret_cast<const __nv_bfloat16*>(x), H, W, C, Ho, Wo, (int)M, (int)r0, n_rows, ld, vec,
          reinterpret_cast<__nv_bfloat16*>(cols));
    }
    EBSD_LAUNCH_CHECK();
  }
  return 0;
}

extern "C" int ebsd_cnn_conv_c1(const void* x, int B, int H, int W, const void* w16, int ldw, const float* bias,
                                int cout, int relu, void* out16, float* out32, void* stream) {
  EBSD_ARG_CHECK(x && w16 && out16 && B > 0 && H > 0 && W > 0 && ldw >= 9, "ebsd_cnn_conv_c1: bad arguments");
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
  const int64_t M = (int64_t)B * Ho * Wo;
  EBSD_ARG_CHECK(M < INT32_MAX, "ebsd_cnn_conv_c1: too many output pixels");
  EBSD_ARG_CHECK(((uintptr_t)out16 & 15) == 0 && ((uintptr_t)out32 & 15) == 0,
                 "ebsd_cnn_conv_c1: outputs must be 16-byte aligned");
  const int blocks = nblocks(M);
  auto args = [&](auto kern) {
    kern<<<blocks, 256, 0, CNN_STREAM>>>(reinterpret_cast<const __nv_bfloat16*>(x), H, W, Ho, Wo, (int)M,
                                         reinterpret_cast<const __nv_bfloat16*>(w16), ldw, bias, relu,
                                         reinterpret_cast<__nv_bfloat16*>(out16), out32);
  };
  switch (cout) {
    case 16: args(k_conv_c1<16>); break;
    case 32: args(k_conv_c1<32>); break;
    case 64: args(k_conv_c1<64>); break;
    default: EBSD_ARG_CHECK(false, "ebsd_cnn_conv_c1: cout %d not in {16, 32, 64}", cout);
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_col2im(const float* dcols, int64_t ld, int B, int H, int W, int C, float* dx,
                               void* stream) {
  EBSD_ARG_CHECK(dcols && dx && ld >= 9 * C, "ebsd_cnn_col2im: bad arguments");
  const int Ho = (H + 1) / 2, Wo = (W + 1) / 2;
  k_col2im<<<nblocks((int64_t)B * H * W * C), 256, 0, CNN_STREAM>>>(dcols, ld, B, H, W, C, Ho, Wo, dx);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_bias_act(const float* y, int64_t ldy, const float* bias, int64_t M, int C, int relu,
                                 void* out, int64_t ld_out, float* out32, void* stream) {
  EBSD_ARG_CHECK(y && out && ldy >= C && ld_out >= C, "ebsd_cnn_bias_act: bad arguments");
  k_bias_act<<<nblocks(M * C), 256, 0, CNN_STREAM>>>(y, ldy, bias, M, C, relu,
                                                     reinterpret_cast<__nv_bfloat16*>(out), ld_out, out32);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_relu_grad(const float* dy, int64_t ldy, const void* act, int64_t lda, int64_t M, int C,
                                  float* g32, void* g16, int64_t ld_out, void* stream) {
  EBSD_ARG_CHECK(dy && act && ld_out >= C, "ebsd_cnn_relu_grad: bad arguments");
  k_relu_grad<<<nblocks(M * ld_out), 256, 0, CNN_STREAM>>>(dy, ldy, reinterpret_cast<const __nv_bfloat16*>(act), lda,
                                                          M, C, g32, reinterpret_cast<__nv_bfloat16*>(g16), ld_out);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_col_sum(const float* g, int64_t M, int C, float* db, void* stream) {
  EBSD_ARG_CHECK(g && db && C > 0 && C <= 1024, "ebsd_cnn_col_sum: bad arguments");
  EBSD_CUDA_CHECK(cudaMemsetAsync(db, 0, sizeof(float) * C, CNN_STREAM));
  const int blocks = (int)std::min<int64_t>(M, 1024);
  k_col_sum<<<blocks, std::min(C, 256), 0, CNN_STREAM>>>(g, M, C, db);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_transpose(const void* in, int in_is_f32, int64_t rows, int64_t cols, int64_t ld_in,
                                  void* out, int64_t out_rows, int64_t ld_out, void* stream) {
  EBSD_ARG_CHECK(in && out && out_rows >= cols && ld_out >= rows, "ebsd_cnn_transpose: bad arguments");
  EBSD_ARG_CHECK(ld_out % 32 == 0 && out_rows % 32 == 0, "transpose output dimensions must be multiples of 32");
  dim3 grid((unsigned)((ld_out + 31) / 32), (unsigned)((out_rows + 31) / 32));
  EBSD_ARG_CHECK(grid.y <= 65535, "transpose too tall");
  if (in_is_f32)
    k_transpose<float><<<grid, dim3(32, 8), 0, CNN_STREAM>>>(reinterpret_cast<const float*>(in), rows, cols, ld_in,
                                                              reinterpret_cast<__nv_bfloat16*>(out), ld_out);
  else
    k_transpose<__nv_bfloat16><<<grid, dim3(32, 8), 0, CNN_STREAM>>>(
        reinterpret_cast<const __nv_bfloat16*>(in), rows, cols, ld_in, reinterpret_cast<__nv_bfloat16*>(out), ld_out);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_scale_cast(const float* x, int64_t n, float scale, void* out, void* stream) {
  EBSD_ARG_CHECK(x && out, "ebsd_cnn_scale_cast: bad arguments");
  k_scale_cast<<<nblocks(n), 256, 0, CNN_STREAM>>>(x, n, scale, reinterpret_cast<__nv_bfloat16*>(out));
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_dense_fwd(const float* x, int64_t ldx, const float* w, const float* b, int M, int N, int K,
                                  int relu, float* y, void* y16, void* stream) {
  EBSD_ARG_CHECK(x && w && y && M > 0 && N > 0 && K > 0, "ebsd_cnn_dense_fwd: bad arguments");
  dim3 grid((N + 15) / 16, (M + 15) / 16);
  k_dense_fwd<<<grid, dim3(16, 16), 0, CNN_STREAM>>>(x, ldx, w, b, M, N, K, relu, y,
                                                      reinterpret_cast<__nv_bfloat16*>(y16));
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_cnn_dense_bwd(const float* dy, const float* x, int64_t ldx, const float* w, int M, int N, int K,
                                  float* dw, float* db, float* dx, void* stream) {
  EBSD_ARG_CHECK(dy && x && w && dw, "ebsd_cnn_dense_bwd: bad arguments");
  cudaStream_t s = CNN_STREAM;
  k_dense_wgrad<<<dim3((K + 15) / 16, (N + 15) / 16), dim3(16, 16), 0, s>>>(dy, x, ldx, M, N, K, dw);
  EBSD_LAUNCH_CHECK();
  if (db) {
    EBSD_CUDA_CHECK(cudaMemsetAsync(db, 0, sizeof(float) * N, s));
    k_col_sum<<<(int)std::min<int64_t>(M, 1024), std::min(N, 256), 0, s>>>(dy, M, N, db);
    EBSD_LAUNCH_CHECK();
  }
  if (dx) {
    k_dense_dgrad<<<dim3((K + 15) / 16, (M + 15) / 16), dim3(16, 16), 0, s>>>(dy, w, M, N, K, dx);
    EBSD_LAUNCH_CHECK();
  }
  return 0;
}

extern "C" int ebsd_cnn_adam(float* w, float* m, float* v, const float* g, int64_t rows, int cols, float lr, float b1,
                             float b2, float eps, int step, float weight_decay, void* w16, int64_t ld16, void* w16t,
                             int64_t ld16t, void* stream) {
  EBSD_ARG_CHECK(w && m && v && g && step >= 1, "ebsd_cnn_adam: bad arguments");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<nblocks(rows * cols), 256, 0, CNN_STREAM>>>(w, m, v, g, rows, cols, lr, b1, b2, eps, c1, c2, weight_decay,
                                                      reinterpret_cast<__nv_bfloat16*>(w16), ld16,
                                                      reinterpret_cast<__nv_bfloat16*>(w16t), ld16t);
  EBSD_LAUNCH_CHECK();
  return 0;
}
