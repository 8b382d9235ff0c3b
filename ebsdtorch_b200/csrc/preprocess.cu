// Experimental-pattern preprocessing: overall background subtraction,
// per-pattern normalisation, CLAHE (optionally fused with the background
// subtraction and the two min-max passes of standard_clean) and the two
// scan-neighbourhood passes of NLPAR.
//
// Follows ebsdtorch/ebsd/experiment_pats.py:223-316 (subtract_overall_
// background, contrast_enhance_clahe, normalize_per_pattern, standard_clean,
// do_nlpar), ebsdtorch/preprocessing/clahe.py:17-130 and
// ebsdtorch/preprocessing/nlpar.py:19-192 (Brewick et al. 2019). Every pass
// here is an image pass over FP32 patterns: HBM-bound (mean, subtract,
// normalise, CLAHE) or shared-memory-bound (the NLPAR window passes, whose
// scan tile and halo are staged in shared memory once per pixel chunk).
#include <algorithm>
#include <climits>

#include "common.cuh"

namespace ebsd {

// ---------------------------------------------------------------- background

// partial[s][c] = sum of X[r, c] over the rows r of split s (FP64)
__global__ void k_colsum_partial(const float* __restrict__ X, int64_t n, int n_cols, int64_t ld, int n_splits,
                                 double* __restrict__ partial) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (c >= n_cols) return;
  const int64_t r0 = (int64_t)s * n / n_splits, r1 = (int64_t)(s + 1) * n / n_splits;
  double acc = 0.0;
#pragma unroll 8
  for (int64_t r = r0; r < r1; ++r) acc += __ldg(X + r * ld + c);
  partial[(int64_t)s * n_cols + c] = acc;
}

__global__ void k_colsum_final(const double* __restrict__ partial, int n_splits, int n_cols, int64_t n,
                               float* __restrict__ mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cols) return;
  double s = 0.0;
  for (int k = 0; k < n_splits; ++k) s += partial[(int64_t)k * n_cols + c];
  mean[c] = (float)(s / (double)n);
}

__global__ void k_sub_vector(float* __restrict__ X, int64_t n, int n_cols, int64_t ld, const float* __restrict__ v) {
  const int64_t total = n * n_cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / n_cols;
    const int c = (int)(t - r * n_cols);
    X[r * ld + c] -= __ldg(v + c);
  }
}

// ------------------------------------------------------------- normalisation

constexpr int kNormThreads = 256;

// mode 0 min-max: (x - min) / ((1e-4 + max) - min); 1 zero mean; 2 zero mean
// and unit unbiased standard deviation (torch.std). One CTA per pattern.
__global__ void __launch_bounds__(kNormThreads) k_normalize(float* __restrict__ X, int64_t n, int n_cols,
                                                           int64_t ld, int mode) {
  __shared__ float fred[32];
  __shared__ double dred[32];
  for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
    float* row = X + r * ld;
    if (mode == 0) {
      float mn = INFINITY, mx = -INFINITY;
      for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
        mn = fminf(mn, row[c]);
        mx = fmaxf(mx, row[c]);
      }
      mx = block_max(mx, fred);
      mn = -block_max(-mn, fred);
      const float den = (1e-4f + mx) - mn;
      for (int c = threadIdx.x; c < n_cols; c += blockDim.x) row[c] = (row[c] - mn) / den;
    } else {
      double s = 0.0;
      for (int c = threadIdx.x; c < n_cols; c += blockDim.x) s += row[c];
      const float mean = (float)(block_sum(s, dred) / n_cols);
      float sd = 1.0f;
      if (mode == 2) {
        double ss = 0.0;
        for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
          const double d = (double)(row[c] - mean);
          ss += d * d;
        }
        sd = (float)sqrt(block_sum(ss, dred) / (double)(n_cols - 1));
      }
      for (int c = threadIdx.x; c < n_cols; c += blockDim.x) {
        const float v = row[c] - mean;
        row[c] = mode == 2 ? v / sd : v;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------- CLAHE

constexpr int kClaheThreads = 256;
// dynamic shared memory of one CTA: the CDF and histogram tables, plus the
// image when it fits (then global memory is read once and written once)
constexpr size_t kClaheSmemCap = 220 * 1024;

__device__ __forceinline__ int reflect_index(int i, int n) { return i < n ? i : 2 * (n - 1) - i; }

// Block-wide min and max (all threads get both).
__device__ __forceinline__ float2 block_minmax(float mn, float mx, float* red) {
  mx = block_max(mx, red);
  mn = -block_max(-mn, red);
  return make_float2(mn, mx);
}

struct ClaheArgs {
  const float* X;
  int64_t n, ld;
  int H, W;
  const float* sub;  // optional pattern subtracted first (background)
  int minmax_in, minmax_out;
  float limit;
  int clip, nb, gh, gw;
  float* out;
  int64_t ld_out;
};

// One CTA per image. Optional pre-pass (x - sub, then min-max); tile
// histograms of floor(x (n_bins - 1)) over the bottom/right reflect-padded
// image; per tile (one warp) clip at `limit`, spread the excess evenly and
// the remainder one count to each of the first bins, cumulate into a CDF;
// then each pixel reads the (tile-y, tile-x, bin) CDF volume by trilinear
// interpolation with grid_sample's align_corners=False / border rules;
// optional post min-max. STAGED keeps the image in shared memory so global
// memory is read once and written once.
template <bool STAGED>
__global__ void __launch_bounds__(kClaheThreads) k_clahe(const ClaheArgs a) {
  extern __shared__ __align__(16) float sm[];
  __shared__ float red[32];
  const int n_tiles = a.gh * a.gw, nb = a.nb, H = a.H, W = a.W, P = H * W;
  float* cdf = sm;                                               // n_tiles * nb
  int* hist = reinterpret_cast<int*>(cdf + n_tiles * nb);        // n_tiles * nb
  float* img_s = reinterpret_cast<float*>(hist + n_tiles * nb);  // P (STAGED)
  const int th = (H + a.gh - 1) / a.gh, tw = (W + a.gw - 1) / a.gw;
  const int vpt = th * tw;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  for (int64_t r = blockIdx.x; r < a.n; r += gridDim.x) {
    const float* img = a.X + r * a.ld;
    float* dst = a.out + r * a.ld_out;
    // pre-pass: x - sub, min / max
    float mn = INFINITY, mx = -INFINITY;
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
      float v = img[t];
      if (a.sub) v -= __ldg(a.sub + t);
      if constexpr (STAGED) img_s[t] = v;
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
    }
    float in_mn = 0.f, in_den = 1.f;
    if (a.minmax_in) {
      const float2 m = block_minmax(mn, mx, red);
      in_mn = m.x;
      in_den = (1e-4f + m.y) - m.x;
    }
    // the value CLAHE sees at pixel t
    auto value = [&](int t) -> float {
      float v;
      if constexpr (STAGED) {
        v = img_s[t];
      } else {
        v = img[t];
        if (a.sub) v -= __ldg(a.sub + t);
      }
      return a.minmax_in ? (v - in_mn) / in_den : v;
    };
    for (int t = threadIdx.x; t < n_tiles * nb; t += blockDim.x) hist[t] = 0;
    __syncthreads();
    const int hp = a.gh * th, wp = a.gw * tw;
    for (int t = threadIdx.x; t < hp * wp; t += blockDim.x) {
      const int y = t / wp, x = t - y * wp;
      const float v = value(reflect_index(y, H) * W + reflect_index(x, W));
      const int b = min(max((int)(v * (float)(nb - 1)), 0), nb - 1);
      atomicAdd(&hist[((y / th) * a.gw + x / tw) * nb + b], 1);
    }
    __syncthreads();
    for (int tile = wid; tile < n_tiles; tile += n_warps) {
      const int* h = hist + tile * nb;
      float* c = cdf + tile * nb;
      // pixel counts as the reference forms them (count / total * voxels)
      float part = 0.f;
      for (int b = lane; b < nb; b += 32) {
        float v = (float)h[b] / (float)vpt * (float)vpt;
        if (a.clip) v = fminf(v, a.limit);
        c[b] = v;
        part += v;
      }
      const float sum = warp_sum(part);
      float residual = 0.f, redist = 0.f;
      if (a.clip) {
        const float clipped = (float)vpt - sum;
        residual = clipped - (float)nb * floorf(clipped / (float)nb);  // torch.remainder
        redist = (clipped - residual) / (float)nb;
      }
      __syncwarp();
      float carry = 0.f;
      for (int b0 = 0; b0 < nb; b0 += 32) {
        const int b = b0 + lane;
        float v = 0.f;
        if (b < nb) {
          v = c[b];
          if (a.clip) v = v + redist + ((float)b < residual ? 1.f : 0.f);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const float u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        v += carry;
        if (b < nb) c[b] = fminf(fmaxf(v / (float)vpt, 0.f), 1.f);
        carry = __shfl_sync(0xffffffffu, v, 31);
      }
    }
    __syncthreads();
    mn = INFINITY;
    mx = -INFINITY;
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
      const int y = t / W, x = t - y * W;
      const float v = value(t);
      // grid_sample coordinates: value -> bins, image x -> tile columns,
      // image y -> tile rows (torch.linspace(-1, 1, n) grids)
      const float cx = -1.0f + 2.0f * (float)x / (float)(W - 1);
      const float cy = -1.0f + 2.0f * (float)y / (float)(H - 1);
      float fb = ((v * 2.0f - 1.0f + 1.0f) * nb - 1.0f) / 2.0f;
      float fx = ((cx + 1.0f) * a.gw - 1.0f) / 2.0f;
      float fy = ((cy + 1.0f) * a.gh - 1.0f) / 2.0f;
      fb = fminf(fmaxf(fb, 0.0f), (float)(nb - 1));
      fx = fminf(fmaxf(fx, 0.0f), (float)(a.gw - 1));
      fy = fminf(fmaxf(fy, 0.0f), (float)(a.gh - 1));
      const int b0 = (int)fb, x0 = (int)fx, y0 = (int)fy;
      const int b1 = min(b0 + 1, nb - 1), x1 = min(x0 + 1, a.gw - 1), y1 = min(y0 + 1, a.gh - 1);
      const float wb = fb - b0, wx = fx - x0, wy = fy - y0;
      const float* c00 = cdf + (y0 * a.gw + x0) * nb;
      const float* c01 = cdf + (y0 * a.gw + x1) * nb;
      const float* c10 = cdf + (y1 * a.gw + x0) * nb;
      const float* c11 = cdf + (y1 * a.gw + x1) * nb;
      const float v00 = c00[b0] * (1.f - wb) + c00[b1] * wb;
      const float v01 = c01[b0] * (1.f - wb) + c01[b1] * wb;
      const float v10 = c10[b0] * (1.f - wb) + c10[b1] * wb;
      const float v11 = c11[b0] * (1.f - wb) + c11[b1] * wb;
      const float o = (v00 * (1.f - wx) + v01 * wx) * (1.f - wy) + (v10 * (1.f - wx) + v11 * wx) * wy;
      mn = fminf(mn, o);
      mx = fmaxf(mx, o);
      if constexpr (STAGED) {
        if (a.minmax_out) {
          img_s[t] = o;  // pixel t is read and written by this thread only
          continue;
        }
      }
      dst[t] = o;
    }
    if (a.minmax_out) {
      const float2 m = block_minmax(mn, mx, red);  // synchronises the block
      const float den = (1e-4f + m.y) - m.x;
      for (int t = threadIdx.x; t < P; t += blockDim.x) {
        float o;
        if constexpr (STAGED) {
          o = img_s[t];
        } else {
          o = dst[t];
        }
        dst[t] = (o - m.x) / den;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------- NLPAR

constexpr int kNlTile = 8;          // 8 x 8 scan points per CTA
constexpr int kNlChunk = 32;        // pattern pixels per shared-memory chunk
constexpr int kNlPitch = 24;        // row pitch of the staged tile + halo (side <= 22)
constexpr int kNlMaxRad = 7;
constexpr int kNlThreads = 256;
constexpr int kNlMaxOffsets = 128;  // offsets per launch
constexpr int kNlPairs = kNlMaxOffsets / (kNlThreads / (kNlTile * kNlTile));  // 32 per thread

// Words per staged pixel plane: odd, so the 32 pixels a warp stores land in
// distinct banks; with the pitch of 24 the 4 x 8 scan points a warp reads at
// one offset land in distinct banks as well.
__host__ __device__ __forceinline__ int nl_plane(int halo) { return (kNlTile + 2 * halo) * kNlPitch + 1; }

// T[q * plane + yy * pitch + xx] = data[point (y0 - halo + yy, x0 - halo + xx), p0 + q];
// zero outside the scan (the reference zero-pads the data, nlpar.py:56-61)
__device__ __forceinline__ void nl_load_chunk(float* T, const float* __restrict__ data, int hs, int ws, int64_t ld,
                                              int y0, int x0, int halo, int p0, int np) {
  const int side = kNlTile + 2 * halo, plane = nl_plane(halo);
  for (int t = threadIdx.x; t < side * side * kNlChunk; t += blockDim.x) {
    const int row = t / kNlChunk, q = t - row * kNlChunk;
    const int yy = row / side, xx = row - yy * side;
    const int y = y0 - halo + yy, x = x0 - halo + xx;
    float v = 0.f;
    if (q < np && y >= 0 && y < hs && x >= 0 && x < ws) v = __ldg(data + ((int64_t)y * ws + x) * ld + p0 + q);
    T[q * plane + yy * kNlPitch + xx] = v;
  }
}

// Offsets of one launch as shared-memory displacements; an offset outside
// [-halo, halo]^2 is marked INT_MIN and yields NaN.
__device__ __forceinline__ void nl_load_offsets(int* off_s, const int* __restrict__ offsets, int o0, int n_off,
                                                int halo) {
  for (int o = threadIdx.x; o < n_off; o += blockDim.x) {
    const int di = offsets[2 * (o0 + o)], dj = offsets[2 * (o0 + o) + 1];
    const bool ok = di >= -halo && di <= halo && dj >= -halo && dj <= halo;
    off_s[o] = ok ? di * kNlPitch + dj : INT_MIN;
  }
}

// dists[pt, o0 + o] = sum_p (x[pt + off[o]] - x[pt])^2. Thread: one scan
// point (tid % 64) and the offsets o = tid / 64 + 4 j; a warp shares o.
__global__ void __launch_bounds__(kNlThreads) k_nlpar_dists(const float* __restrict__ data, int hs, int ws,
                                                           int n_pix, int64_t ld, int halo,
                                                           const int* __restrict__ offsets, int o0, int n_off,
                                                           int n_off_total, float* __restrict__ dists) {
  extern __shared__ __align__(16) float T[];
  __shared__ int off_s[kNlMaxOffsets];
  const int plane = nl_plane(halo);
  const int tiles_x = (ws + kNlTile - 1) / kNlTile;
  const int y0 = (blockIdx.x / tiles_x) * kNlTile, x0 = (blockIdx.x % tiles_x) * kNlTile;
  const int pt = threadIdx.x % (kNlTile * kNlTile), ob = threadIdx.x / (kNlTile * kNlTile);
  const int self = (pt / kNlTile + halo) * kNlPitch + pt % kNlTile + halo;
  nl_load_offsets(off_s, offsets, o0, n_off, halo);
  float acc[kNlPairs];
#pragma unroll
  for (int j = 0; j < kNlPairs; ++j) acc[j] = 0.f;
  for (int p0 = 0; p0 < n_pix; p0 += kNlChunk) {
    const int np = min(kNlChunk, n_pix - p0);
    __syncthreads();
    nl_load_chunk(T, data, hs, ws, ld, y0, x0, halo, p0, np);
    __syncthreads();
    for (int q = 0; q < np; ++q) {
      const float* Tq = T + q * plane + self;
      const float s = Tq[0];
#pragma unroll
      for (int j = 0; j < kNlPairs; ++j) {
        const int o = ob + 4 * j;
        if (o < n_off) {
          const int d = off_s[o];
          if (d != INT_MIN) {
            const float e = Tq[d] - s;
            acc[j] = fmaf(e, e, acc[j]);
          }
        }
      }
    }
  }
  const int y = y0 + pt / kNlTile, x = x0 + pt % kNlTile;
  if (y >= hs || x >= ws) return;
#pragma unroll
  for (int j = 0; j < kNlPairs; ++j) {
    const int o = ob + 4 * j;
    if (o < n_off) dists[((int64_t)y * ws + x) * n_off_total + o0 + o] = off_s[o] == INT_MIN ? NAN : acc[j];
  }
}

// out[pt] (+)= sum_o w[pt, o0 + o] x[pt + off[o]]. Warp: 8 scan points,
// lane = pattern pixel of the chunk; weights staged per tile.
__global__ void __launch_bounds__(kNlThreads) k_nlpar_average(const float* __restrict__ data, int hs, int ws,
                                                             int n_pix, int64_t ld, int halo,
                                                             const int* __restrict__ offsets, int o0, int n_off,
                                                             int n_off_total, const float* __restrict__ weights,
                                                             int accumulate, float* __restrict__ out,
                                                             int64_t ld_out) {
  extern __shared__ __align__(16) float T[];
  __shared__ int off_s[kNlMaxOffsets];
  const int plane = nl_plane(halo);
  float* w_s = T + kNlChunk * plane;  // [64][n_off]
  const int tiles_x = (ws + kNlTile - 1) / kNlTile;
  const int y0 = (blockIdx.x / tiles_x) * kNlTile, x0 = (blockIdx.x % tiles_x) * kNlTile;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  nl_load_offsets(off_s, offsets, o0, n_off, halo);
  for (int t = threadIdx.x; t < kNlTile * kNlTile * n_off; t += blockDim.x) {
    const int pt = t / n_off, o = t - pt * n_off;
    const int y = y0 + pt / kNlTile, x = x0 + pt % kNlTile;
    w_s[t] = (y < hs && x < ws) ? weights[((int64_t)y * ws + x) * n_off_total + o0 + o] : 0.f;
  }
  constexpr int kPtsPerWarp = kNlTile * kNlTile / (kNlThreads / 32);  // 8
  for (int p0 = 0; p0 < n_pix; p0 += kNlChunk) {
    const int np = min(kNlChunk, n_pix - p0);
    __syncthreads();
    nl_load_chunk(T, data, hs, ws, ld, y0, x0, halo, p0, np);
    __syncthreads();
    if (lane >= np) continue;
    for (int k = 0; k < kPtsPerWarp; ++k) {
      const int pt = wid * kPtsPerWarp + k;
      const int y = y0 + pt / kNlTile, x = x0 + pt % kNlTile;
      if (y >= hs || x >= ws) continue;
      const float* Tq = T + lane * plane + (pt / kNlTile + halo) * kNlPitch + pt % kNlTile + halo;
      const float* w = w_s + pt * n_off;
      float s = 0.f;
      for (int o = 0; o < n_off; ++o) {
        const int d = off_s[o];
        s = fmaf(w[o], d == INT_MIN ? NAN : Tq[d], s);
      }
      float* dp = out + ((int64_t)y * ws + x) * ld_out + p0 + lane;
      *dp = accumulate ? *dp + s : s;
    }
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_pattern_mean(const float* patterns, int64_t n, int n_pix, int64_t ld, double* partial,
                                 int n_splits, float* mean, void* stream) {
  EBSD_ARG_CHECK(patterns && partial && mean, "ebsd_pattern_mean: null pointer");
  EBSD_ARG_CHECK(n >= 1 && n_pix >= 1 && ld >= n_pix, "ebsd_pattern_mean: bad sizes");
  EBSD_ARG_CHECK(n_splits >= 1 && n_splits <= 65535, "n_splits must be in [1, 65535]");
  cudaStream_t s = as_stream(stream);
  k_colsum_partial<<<dim3(ceil_div(n_pix, 256), n_splits), 256, 0, s>>>(patterns, n, n_pix, ld, n_splits, partial);
  EBSD_LAUNCH_CHECK();
  k_colsum_final<<<ceil_div(n_pix, 256), 256, 0, s>>>(partial, n_splits, n_pix, n, mean);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_subtract_pattern(float* patterns, int64_t n, int n_pix, int64_t ld, const float* v,
                                     void* stream) {
  EBSD_ARG_CHECK(patterns && v && n >= 0 && n_pix >= 1 && ld >= n_pix, "ebsd_subtract_pattern: bad arguments");
  if (n == 0) return 0;
  const int blocks = (int)std::min<int64_t>((n * n_pix + 255) / 256, (int64_t)device_sm_count() * 32);
  k_sub_vector<<<blocks, 256, 0, as_stream(stream)>>>(patterns, n, n_pix, ld, v);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_normalize_patterns(float* patterns, int64_t n, int n_pix, int64_t ld, int mode, void* stream) {
  EBSD_ARG_CHECK(patterns && n >= 0 && n_pix >= 2 && ld >= n_pix, "ebsd_normalize_patterns: bad arguments");
  EBSD_ARG_CHECK(mode >= 0 && mode <= 2, "mode must be 0 (minmax), 1 (zeromean) or 2 (standard)");
  if (n == 0) return 0;
  const int blocks = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * 8);
  k_normalize<<<blocks, kNormThreads, 0, as_stream(stream)>>>(patterns, n, n_pix, ld, mode);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_clahe(const float* images, int64_t n, int height, int width, int64_t ld, const float* subtract,
                          int minmax_in, float clip_limit, int n_bins, int grid_h, int grid_w, int minmax_out,
                          float* out, int64_t ld_out, void* stream) {
  EBSD_ARG_CHECK(images && out && n >= 0, "ebsd_clahe: bad arguments");
  EBSD_ARG_CHECK(height >= 2 && width >= 2 && ld >= (int64_t)height * width && ld_out >= (int64_t)height * width,
                 "ebsd_clahe: bad image shape");
  EBSD_ARG_CHECK(grid_h >= 1 && grid_w >= 1 && grid_h <= height && grid_w <= width, "ebsd_clahe: bad grid");
  EBSD_ARG_CHECK(n_bins >= 2 && n_bins <= 2048, "n_bins must be in [2, 2048]");
  const int th = (height + grid_h - 1) / grid_h, tw = (width + grid_w - 1) / grid_w;
  // reflect padding needs the pad to be smaller than the image
  EBSD_ARG_CHECK(grid_h * th - height < height && grid_w * tw - width < width, "ebsd_clahe: padding too large");
  const size_t tables = (size_t)grid_h * grid_w * n_bins * (sizeof(float) + sizeof(int));
  EBSD_ARG_CHECK(tables <= kClaheSmemCap, "ebsd_clahe: grid x bins too large for shared memory");
  EBSD_ARG_CHECK(images != out || ld == ld_out, "ebsd_clahe: in place needs ld == ld_out");
  if (n == 0) return 0;
  ClaheArgs a;
  a.X = images;
  a.n = n;
  a.ld = ld;
  a.H = height;
  a.W = width;
  a.sub = subtract;
  a.minmax_in = minmax_in ? 1 : 0;
  a.minmax_out = minmax_out ? 1 : 0;
  // clip limit as the reference computes it: max(clip * voxels // bins, 1)
  a.limit = (float)std::max(std::floor((double)clip_limit * th * tw / n_bins), 1.0);
  a.clip = clip_limit > 0.0f ? 1 : 0;
  a.nb = n_bins;
  a.gh = grid_h;
  a.gw = grid_w;
  a.out = out;
  a.ld_out = ld_out;
  const int n_pix = height * width;
  const bool staged = tables + (size_t)n_pix * sizeof(float) <= kClaheSmemCap;
  const size_t smem = tables + (staged ? (size_t)n_pix * sizeof(float) : 0);
  cudaStream_t s = as_stream(stream);
  if (staged) {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_clahe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EBSD_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clahe<true>, kClaheThreads, smem));
    const int blocks = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * std::max(per_sm, 1));
    k_clahe<true><<<blocks, kClaheThreads, smem, s>>>(a);
  } else {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_clahe<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * 4);
    k_clahe<false><<<blocks, kClaheThreads, smem, s>>>(a);
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}

static int nl_check(const float* data, int hs, int ws, int n_pix, int64_t ld, int halo, const int* offsets, int o0,
                    int n_off, int n_off_total) {
  EBSD_ARG_CHECK(data && offsets, "NLPAR: null pointer");
  EBSD_ARG_CHECK(hs >= 1 && ws >= 1 && n_pix >= 1 && ld >= n_pix, "NLPAR: bad sizes");
  EBSD_ARG_CHECK(halo >= 0 && halo <= kNlMaxRad, "NLPAR: kernel radius must be in [0, %d]", kNlMaxRad);
  EBSD_ARG_CHECK(n_off >= 1 && n_off <= kNlMaxOffsets && o0 >= 0 && o0 + n_off <= n_off_total,
                 "NLPAR: an offset block holds 1..%d offsets", kNlMaxOffsets);
  EBSD_ARG_CHECK((int64_t)ceil_div(hs, kNlTile) * ceil_div(ws, kNlTile) <= INT_MAX, "NLPAR: scan too large");
  return 0;
}

extern "C" int ebsd_nlpar_dists(const float* data, int scan_h, int scan_w, int n_pix, int64_t ld, int k_rad,
                                const int* offsets, int o0, int n_off, int n_off_total, float* dists, void* stream) {
  if (int rc = nl_check(data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0, n_off, n_off_total)) return rc;
  EBSD_ARG_CHECK(dists != nullptr, "NLPAR: null output");
  const size_t smem = (size_t)kNlChunk * nl_plane(k_rad) * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_nlpar_dists, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = ceil_div(scan_h, kNlTile) * ceil_div(scan_w, kNlTile);
  k_nlpar_dists<<<tiles, kNlThreads, smem, as_stream(stream)>>>(data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0,
                                                              n_off, n_off_total, dists);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_nlpar_average(const float* data, int scan_h, int scan_w, int n_pix, int64_t ld, int k_rad,
                                  const int* offsets, int o0, int n_off, int n_off_total, const float* weights,
                                  int accumulate, float* out, int64_t ld_out, void* stream) {
  if (int rc = nl_check(data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0, n_off, n_off_total)) return rc;
  EBSD_ARG_CHECK(weights && out && ld_out >= n_pix, "NLPAR: bad output");
  EBSD_ARG_CHECK(out != data, "NLPAR: the average cannot be written in place");
  const size_t smem = ((size_t)kNlChunk * nl_plane(k_rad) + (size_t)kNlTile * kNlTile * n_off) * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_nlpar_average, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = ceil_div(scan_h, kNlTile) * ceil_div(scan_w, kNlTile);
  k_nlpar_average<<<tiles, kNlThreads, smem, as_stream(stream)>>>(data, scan_h, scan_w, n_pix, ld, k_rad, offsets,
                                                                o0, n_off, n_off_total, weights, accumulate, out,
                                                                ld_out);
  EBSD_LAUNCH_CHECK();
  return 0;
}
