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

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// mode 0 min-max: (x - min) / ((1e-4 + max) - min); 1 zero mean; 2 zero mean
// and unit unbiased standard deviation (torch.std). One CTA per pattern; with
// PER > 0 a row of up to PER * 256 values is held in registers (one read, one
// write), otherwise it is re-read from global memory (L2) per pass.
template <int PER>
__global__ void __launch_bounds__(kNormThreads) k_normalize(float* __restrict__ X, int64_t n, int n_cols,
                                                           int64_t ld, int mode) {
  __shared__ float fred[32];
  __shared__ double dred[32];
  constexpr int R = PER > 0 ? PER : 1;
  float v[R];
  for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
    float* row = X + r * ld;
    auto at = [&](int k, int c) -> float {
      if constexpr (PER > 0) {
        return v[k];
      } else {
        return row[c];
      }
    };
    if constexpr (PER > 0) {
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int c = threadIdx.x + k * kNormThreads;
        v[k] = c < n_cols ? row[c] : 0.f;
      }
    }
    if (mode == 0) {
      float mn = INFINITY, mx = -INFINITY;
#pragma unroll
      for (int k = 0; k < R; ++k)
        for (int c = threadIdx.x + k * kNormThreads; c < n_cols; c += R * kNormThreads) {
          const float x = at(k, c);
          mn = fminf(mn, x);
          mx = fmaxf(mx, x);
          if constexpr (PER > 0) break;
        }
      mx = block_max(mx, fred);
      mn = -block_max(-mn, fred);
      const float den = (1e-4f + mx) - mn;
#pragma unroll
      for (int k = 0; k < R; ++k)
        for (int c = threadIdx.x + k * kNormThreads; c < n_cols; c += R * kNormThreads) {
          row[c] = (at(k, c) - mn) / den;
          if constexpr (PER > 0) break;
        }
    } else {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < R; ++k)
        for (int c = threadIdx.x + k * kNormThreads; c < n_cols; c += R * kNormThreads) {
          s += at(k, c);
          if constexpr (PER > 0) break;
        }
      const float mean = (float)(block_sum(s, dred) / n_cols);
      float sd = 1.0f;
      if (mode == 2) {
        double ss = 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k)
          for (int c = threadIdx.x + k * kNormThreads; c < n_cols; c += R * kNormThreads) {
            const double d = (double)(at(k, c) - mean);
            ss += d * d;
            if constexpr (PER > 0) break;
          }
        sd = (float)sqrt(block_sum(ss, dred) / (double)(n_cols - 1));
      }
#pragma unroll
      for (int k = 0; k < R; ++k)
        for (int c = threadIdx.x + k * kNormThreads; c < n_cols; c += R * kNormThreads) {
          const float x = at(k, c) - mean;
          row[c] = mode == 2 ? x / sd : x;
          if constexpr (PER > 0) break;
        }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------- CLAHE

constexpr int kClaheThreads = 256;
// dynamic shared memory of one CTA: the CDF and histogram tables, the
// coordinate tables, plus two image buffers when they fit (then each image
// is read once, prefetched while the previous one is equalised, and written
// once)
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
  int vec16;  // rows 16-byte aligned with H * W % 4 == 0: 16-byte async copies
  float* out;
  int64_t ld_out;
};

// Shared-memory layout of k_clahe (bytes), shared with the host.
struct ClaheLayout {
  size_t cdf, hist, colsrc, coltile, rowsrc, rowtile, colx, colw, rowy, roww, img, total_tables;
  __host__ __device__ ClaheLayout(int H, int W, int gh, int gw, int nb) {
    const int th = (H + gh - 1) / gh, tw = (W + gw - 1) / gw;
    const int hp = gh * th, wp = gw * tw;
    size_t o = 0;
    cdf = o;
    o += (size_t)gh * gw * nb * 4;
    hist = o;
    o += (size_t)gh * gw * nb * 4;
    colsrc = o;
    o += (size_t)wp * 4;
    coltile = o;
    o += (size_t)wp * 4;
    rowsrc = o;
    o += (size_t)hp * 4;
    rowtile = o;
    o += (size_t)hp * 4;
    colx = o;
    o += (size_t)W * 4;
    colw = o;
    o += (size_t)W * 4;
    rowy = o;
    o += (size_t)H * 4;
    roww = o;
    o += (size_t)H * 4;
    img = (o + 15) / 16 * 16;
    total_tables = img;
  }
};

// One CTA per image. Optional pre-pass (x - sub, then min-max); tile
// histograms of floor(x (n_bins - 1)) over the bottom/right reflect-padded
// image; per tile (one warp) clip at `limit`, spread the excess evenly and
// the remainder one count to each of the first bins, cumulate into a CDF;
// then each pixel reads the (tile-y, tile-x, bin) CDF volume by trilinear
// interpolation with grid_sample's align_corners=False / border rules;
// optional post min-max. STAGED keeps the image in shared memory, the next
// image arriving by cp.async while this one is processed; otherwise every
// pass reads global memory (L2).
template <bool STAGED>
__global__ void __launch_bounds__(kClaheThreads) k_clahe(const ClaheArgs a) {
  extern __shared__ __align__(16) uint8_t smraw[];
  __shared__ float red[32];
  const int n_tiles = a.gh * a.gw, nb = a.nb, H = a.H, W = a.W, P = H * W;
  const ClaheLayout L(H, W, a.gh, a.gw, nb);
  float* cdf = reinterpret_cast<float*>(smraw + L.cdf);
  int* hist = reinterpret_cast<int*>(smraw + L.hist);
  int* colsrc = reinterpret_cast<int*>(smraw + L.colsrc);
  int* coltile = reinterpret_cast<int*>(smraw + L.coltile);
  int* rowsrc = reinterpret_cast<int*>(smraw + L.rowsrc);
  int* rowtile = reinterpret_cast<int*>(smraw + L.rowtile);
  int* colx = reinterpret_cast<int*>(smraw + L.colx);
  float* colw = reinterpret_cast<float*>(smraw + L.colw);
  int* rowy = reinterpret_cast<int*>(smraw + L.rowy);
  float* roww = reinterpret_cast<float*>(smraw + L.roww);
  float* img_s = reinterpret_cast<float*>(smraw + L.img);  // 2 x P (STAGED)
  const int th = (H + a.gh - 1) / a.gh, tw = (W + a.gw - 1) / a.gw;
  const int hp = a.gh * th, wp = a.gw * tw, vpt = th * tw;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, n_warps = blockDim.x >> 5;

  // coordinate tables: padded pixel -> source pixel and tile; output pixel
  // -> lower CDF cell and weight (torch.linspace(-1, 1, n) grids unnormalised
  // with align_corners=False, clamped at the border)
  for (int x = threadIdx.x; x < wp; x += blockDim.x) {
    colsrc[x] = reflect_index(x, W);
    coltile[x] = x / tw;
  }
  for (int y = threadIdx.x; y < hp; y += blockDim.x) {
    rowsrc[y] = reflect_index(y, H) * W;
    rowtile[y] = (y / th) * a.gw;
  }
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    const float c = -1.0f + 2.0f * (float)x / (float)(W - 1);
    const float f = fminf(fmaxf(((c + 1.0f) * a.gw - 1.0f) / 2.0f, 0.0f), (float)(a.gw - 1));
    colx[x] = (int)f;
    colw[x] = f - (int)f;
  }
  for (int y = threadIdx.x; y < H; y += blockDim.x) {
    const float c = -1.0f + 2.0f * (float)y / (float)(H - 1);
    const float f = fminf(fmaxf(((c + 1.0f) * a.gh - 1.0f) / 2.0f, 0.0f), (float)(a.gh - 1));
    rowy[y] = (int)f;
    roww[y] = f - (int)f;
  }

  auto prefetch = [&](int64_t r, float* buf) {
    const float* src = a.X + r * a.ld;
    if (a.vec16) {
      for (int t = threadIdx.x; t < P / 4; t += blockDim.x) cp_async16(buf + 4 * t, src + 4 * t);
    } else {
      for (int t = threadIdx.x; t < P; t += blockDim.x) cp_async4(buf + t, src + t);
    }
  };
  if constexpr (STAGED) {
    if (blockIdx.x < a.n) prefetch(blockIdx.x, img_s);
    cp_async_commit();
  }
  int it = 0;
  for (int64_t r = blockIdx.x; r < a.n; r += gridDim.x, ++it) {
    const float* img = a.X + r * a.ld;
    float* dst = a.out + r * a.ld_out;
    float* buf = img_s + (it & 1) * P;
    if constexpr (STAGED) {
      if (r + gridDim.x < a.n) prefetch(r + gridDim.x, img_s + ((it + 1) & 1) * P);
      cp_async_commit();
      cp_async_wait<1>();
    }
    for (int t = threadIdx.x; t < n_tiles * nb; t += blockDim.x) hist[t] = 0;
    __syncthreads();
    // pre-pass: x - sub, min / max (in place in shared memory when staged)
    float mn = INFINITY, mx = -INFINITY;
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
      float v = STAGED ? buf[t] : img[t];
      if (a.sub) v -= __ldg(a.sub + t);
      if constexpr (STAGED) buf[t] = v;
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
    }
    float in_mn = 0.f, in_den = 1.f;
    if (a.minmax_in) {
      const float2 m = block_minmax(mn, mx, red);
      in_mn = m.x;
      in_den = (1e-4f + m.y) - m.x;
      if constexpr (STAGED)
        for (int t = threadIdx.x; t < P; t += blockDim.x) buf[t] = (buf[t] - in_mn) / in_den;
    }
    __syncthreads();
    // the value CLAHE sees at pixel t
    auto value = [&](int t) -> float {
      if constexpr (STAGED) {
        return buf[t];
      } else {
        float v = img[t];
        if (a.sub) v -= __ldg(a.sub + t);
        return a.minmax_in ? (v - in_mn) / in_den : v;
      }
    };
    for (int y = wid; y < hp; y += n_warps) {
      const int src = rowsrc[y], tile_row = rowtile[y];
      for (int x = lane; x < wp; x += 32) {
        const float v = value(src + colsrc[x]);
        const int b = min(max((int)(v * (float)(nb - 1)), 0), nb - 1);
        atomicAdd(&hist[(tile_row + coltile[x]) * nb + b], 1);
      }
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
    for (int y = wid; y < H; y += n_warps) {
      const int y0 = rowy[y], y1 = min(y0 + 1, a.gh - 1);
      const float wy = roww[y];
      for (int x = lane; x < W; x += 32) {
        const int t = y * W + x;
        const float v = value(t);
        // value coordinate: ((2 v - 1) + 1) n_bins - 1) / 2, as grid_sample
        // unnormalises the reference's v * 2 - 1
        const float fb = fminf(fmaxf(((v * 2.0f - 1.0f + 1.0f) * nb - 1.0f) / 2.0f, 0.0f), (float)(nb - 1));
        const int b0 = (int)fb, b1 = min(b0 + 1, nb - 1);
        const int x0 = colx[x], x1 = min(x0 + 1, a.gw - 1);
        const float wb = fb - b0, wx = colw[x];
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
        if (STAGED && a.minmax_out) {
          buf[t] = o;  // pixel t is read and written by this thread only
        } else {
          dst[t] = o;
        }
      }
    }
    if (a.minmax_out) {
      const float2 m = block_minmax(mn, mx, red);  // synchronises the block
      const float den = (1e-4f + m.y) - m.x;
      for (int t = threadIdx.x; t < P; t += blockDim.x) dst[t] = ((STAGED ? buf[t] : dst[t]) - m.x) / den;
    }
    __syncthreads();
  }
  if constexpr (STAGED) cp_async_wait<0>();
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
__host__ __device__ constexpr int nl_plane(int halo) { return (kNlTile + 2 * halo) * kNlPitch + 1; }

constexpr int kNlMaxRows = (kNlTile + 2 * kNlMaxRad) * (kNlTile + 2 * kNlMaxRad);

// Per CTA, once: for each row (yy, xx) of the staged tile + halo, the scan
// point it holds (-1 outside the scan) and its shared-memory offset.
template <int HALO>
__device__ __forceinline__ void nl_rows(int* src_s, int* dst_s, int hs, int ws, int y0, int x0) {
  constexpr int side = kNlTile + 2 * HALO;
  for (int r = threadIdx.x; r < side * side; r += blockDim.x) {
    const int yy = r / side, xx = r - (r / side) * side;
    const int y = y0 - HALO + yy, x = x0 - HALO + xx;
    src_s[r] = (y >= 0 && y < hs && x >= 0 && x < ws) ? y * ws + x : -1;
    dst_s[r] = yy * kNlPitch + xx;
  }
}

// T[q * plane + yy * pitch + xx] = data[point (y0 - halo + yy, x0 - halo + xx), p0 + q]
// by 4-byte cp.async (lane = pixel q, one row per warp and step); zero
// outside the scan (the reference zero-pads the data, nlpar.py:56-61) and
// beyond the last pixel. Completes before return.
template <int HALO>
__device__ __forceinline__ void nl_load_chunk(float* T, const float* __restrict__ data, int64_t ld,
                                              const int* src_s, const int* dst_s, int p0, int np) {
  constexpr int side = kNlTile + 2 * HALO, plane = nl_plane(HALO);
  static_assert(kNlChunk == 32, "one warp lane per pixel of the chunk");
  const int q = threadIdx.x & 31;
  for (int row = threadIdx.x >> 5; row < side * side; row += blockDim.x >> 5) {
    const int src = src_s[row];
    float* dst = T + q * plane + dst_s[row];
    if (src >= 0 && q < np)
      cp_async4(dst, data + (int64_t)src * ld + p0 + q);
    else
      *dst = 0.f;
  }
  cp_async_commit();
  cp_async_wait<0>();
}

// Offsets of one launch as shared-memory displacements; an offset outside
// [-halo, halo]^2 reads the point itself and is flagged (its results are NaN).
__device__ __forceinline__ void nl_load_offsets(int* off_s, unsigned char* bad_s, const int* __restrict__ offsets,
                                                int o0, int n_off, int halo) {
  for (int o = threadIdx.x; o < n_off; o += blockDim.x) {
    const int di = offsets[2 * (o0 + o)], dj = offsets[2 * (o0 + o) + 1];
    const bool ok = di >= -halo && di <= halo && dj >= -halo && dj <= halo;
    off_s[o] = ok ? di * kNlPitch + dj : 0;
    bad_s[o] = ok ? 0 : 1;
  }
}

// dists[pt, o0 + o] = sum_p (x[pt + off[o]] - x[pt])^2. Thread: one scan
// point (tid % 64) and the offsets o = tid / 64 + 4 j (a warp shares o); per
// chunk the point's own 32 values sit in registers and each offset costs one
// shared-memory load (immediate offset) per pixel.
template <int HALO>
__global__ void __launch_bounds__(kNlThreads, 3) k_nlpar_dists(const float* __restrict__ data, int hs, int ws,
                                                           int n_pix, int64_t ld, const int* __restrict__ offsets,
                                                           int o0, int n_off, int per_group, int n_off_total,
                                                           float* __restrict__ dists) {
  constexpr int plane = nl_plane(HALO);
  extern __shared__ __align__(16) float T[];
  __shared__ int off_s[kNlMaxOffsets];
  __shared__ unsigned char bad_s[kNlMaxOffsets];
  __shared__ int src_s[kNlMaxRows], dst_s[kNlMaxRows];
  // this CTA's group of offsets (blockIdx.y) within the launch's block
  o0 += blockIdx.y * per_group;
  n_off = min(per_group, n_off - (int)blockIdx.y * per_group);
  const int tiles_x = (ws + kNlTile - 1) / kNlTile;
  const int y0 = (blockIdx.x / tiles_x) * kNlTile, x0 = (blockIdx.x % tiles_x) * kNlTile;
  const int pt = threadIdx.x % (kNlTile * kNlTile), ob = threadIdx.x / (kNlTile * kNlTile);
  const int self = (pt / kNlTile + HALO) * kNlPitch + pt % kNlTile + HALO;
  const int nj = (n_off - ob + 3) / 4;  // offsets of this thread
  nl_load_offsets(off_s, bad_s, offsets, o0, n_off, HALO);
  nl_rows<HALO>(src_s, dst_s, hs, ws, y0, x0);
  float acc[kNlPairs];
#pragma unroll
  for (int j = 0; j < kNlPairs; ++j) acc[j] = 0.f;
  for (int p0 = 0; p0 < n_pix; p0 += kNlChunk) {
    __syncthreads();
    nl_load_chunk<HALO>(T, data, ld, src_s, dst_s, p0, min(kNlChunk, n_pix - p0));
    __syncthreads();
    // two halves of 16 pixels keep 16 own values in registers (3 CTAs per SM)
#pragma unroll 1
    for (int h = 0; h < kNlChunk; h += kNlChunk / 2) {
      const float* Th = T + h * plane;
      float sv[kNlChunk / 2];
#pragma unroll
      for (int q = 0; q < kNlChunk / 2; ++q) sv[q] = Th[q * plane + self];
#pragma unroll
      for (int j = 0; j < kNlPairs; ++j) {
        if (j < nj) {
          const float* b = Th + self + off_s[ob + 4 * j];
          float a = acc[j];
#pragma unroll
          for (int q = 0; q < kNlChunk / 2; ++q) {
            const float e = b[q * plane] - sv[q];
            a = fmaf(e, e, a);
          }
          acc[j] = a;
        }
      }
    }
  }
  const int y = y0 + pt / kNlTile, x = x0 + pt % kNlTile;
  if (y >= hs || x >= ws) return;
#pragma unroll
  for (int j = 0; j < kNlPairs; ++j) {
    const int o = ob + 4 * j;
    if (o < n_off) dists[((int64_t)y * ws + x) * n_off_total + o0 + o] = bad_s[o] ? NAN : acc[j];
  }
}

// out[pt] (+)= sum_o w[pt, o0 + o] x[pt + off[o]]. Warp w: the 8 scan
// points of tile row w, lane = pattern pixel of the chunk. The offsets are
// walked by window row (di) and column (dj): for each di the warp loads the
// 8 + 2 halo values of that row of the staged tile once, and every dj of the
// row reuses them (8 FMAs per offset, two float4 weight loads). Each (di, dj)
// may appear at most once per call; an offset outside the window makes the
// outputs NaN.
template <int HALO>
__global__ void __launch_bounds__(kNlThreads) k_nlpar_average(const float* __restrict__ data, int hs, int ws,
                                                             int n_pix, int pix_per_split, int64_t ld,
                                                             const int* __restrict__ offsets, int o0, int n_off,
                                                             int n_off_total, const float* __restrict__ weights,
                                                             int accumulate, float* __restrict__ out,
                                                             int64_t ld_out) {
  constexpr int plane = nl_plane(HALO);
  constexpr int side = kNlTile + 2 * HALO, w2 = 2 * HALO + 1;
  extern __shared__ __align__(16) float T[];
  __shared__ int orow_s[(2 * kNlMaxRad + 1) * (2 * kNlMaxRad + 1)];  // (di, dj) -> offset of this call, or -1
  __shared__ int any_bad;
  __shared__ int src_s[kNlMaxRows], dst_s[kNlMaxRows];
  float* w_s = T + ((kNlChunk * plane + 3) & ~3);  // [o][64 points], 16-byte aligned
  const int tiles_x = (ws + kNlTile - 1) / kNlTile;
  const int y0 = (blockIdx.x / tiles_x) * kNlTile, x0 = (blockIdx.x % tiles_x) * kNlTile;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // this CTA's range of pattern pixels (blockIdx.y); outputs are disjoint
  const int pix_begin = blockIdx.y * pix_per_split, pix_end = min(n_pix, pix_begin + pix_per_split);
  for (int r = threadIdx.x; r < w2 * w2; r += blockDim.x) orow_s[r] = -1;
  if (threadIdx.x == 0) any_bad = 0;
  nl_rows<HALO>(src_s, dst_s, hs, ws, y0, x0);
  __syncthreads();
  for (int o = threadIdx.x; o < n_off; o += blockDim.x) {
    const int di = offsets[2 * (o0 + o)], dj = offsets[2 * (o0 + o) + 1];
    if (di >= -HALO && di <= HALO && dj >= -HALO && dj <= HALO)
      orow_s[(di + HALO) * w2 + dj + HALO] = o;
    else
      any_bad = 1;
  }
  for (int t = threadIdx.x; t < kNlTile * kNlTile * n_off; t += blockDim.x) {
    const int pt = t % (kNlTile * kNlTile), o = t / (kNlTile * kNlTile);
    const int y = y0 + pt / kNlTile, x = x0 + pt % kNlTile;
    w_s[t] = (y < hs && x < ws) ? weights[((int64_t)y * ws + x) * n_off_total + o0 + o] : 0.f;
  }
  const int y = y0 + wid;
  const float4* w4 = reinterpret_cast<const float4*>(w_s) + wid * 2;
  for (int p0 = pix_begin; p0 < pix_end; p0 += kNlChunk) {
    const int np = min(kNlChunk, pix_end - p0);
    __syncthreads();
    nl_load_chunk<HALO>(T, data, ld, src_s, dst_s, p0, np);
    __syncthreads();
    if (y >= hs) continue;
    const float* rows = T + lane * plane + wid * kNlPitch;  // window row wid + (di + HALO)
    float s[kNlTile];
#pragma unroll
    for (int k = 0; k < kNlTile; ++k) s[k] = 0.f;
#pragma unroll 1
    for (int a = 0; a < w2; ++a) {
      const float* r = rows + a * kNlPitch;
      float v[side];
#pragma unroll
      for (int x = 0; x < side; ++x) v[x] = r[x];
#pragma unroll
      for (int c = 0; c < w2; ++c) {
        const int o = orow_s[a * w2 + c];
        if (o < 0) continue;
        const float4 wa = w4[o * (kNlTile * kNlTile / 4)], wb = w4[o * (kNlTile * kNlTile / 4) + 1];
        s[0] = fmaf(wa.x, v[0 + c], s[0]);
        s[1] = fmaf(wa.y, v[1 + c], s[1]);
        s[2] = fmaf(wa.z, v[2 + c], s[2]);
        s[3] = fmaf(wa.w, v[3 + c], s[3]);
        s[4] = fmaf(wb.x, v[4 + c], s[4]);
        s[5] = fmaf(wb.y, v[5 + c], s[5]);
        s[6] = fmaf(wb.z, v[6 + c], s[6]);
        s[7] = fmaf(wb.w, v[7 + c], s[7]);
      }
    }
    if (lane < np) {
#pragma unroll
      for (int k = 0; k < kNlTile; ++k) {
        if (x0 + k < ws) {
          float* dp = out + ((int64_t)y * ws + x0 + k) * ld_out + p0 + lane;
          const float val = any_bad ? NAN : s[k];
          *dp = accumulate ? *dp + val : val;
        }
      }
    }
  }
}

// ---- NLPAR weights (nlpar.py:122-183): noise estimate, normalised
// distances, Newton fit of the global coefficient, masked softmax

constexpr int kNlWThreads = 256;
constexpr int kNlFitBlocks = 592;  // partial sums of one fit iteration

struct NlFitState {
  double g;       // the coefficient (the reference's guess_coeff)
  int done;       // |obj| fell below the tolerance in an earlier iteration
  unsigned ticket;
};

__global__ void k_nlpar_fit_init(NlFitState* st) {
  st->g = 1.0;
  st->done = 0;
  st->ticket = 0u;
}

// sigma[pt] = sqrt(min(d[pt, 1..8]) / (2 P))
__global__ void k_nlpar_sigma(const float* __restrict__ d, int64_t n_pts, int K, int n_pix,
                              float* __restrict__ sigma) {
  const int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= n_pts) return;
  float m = INFINITY;
  for (int o = 1; o < 9; ++o) m = fminf(m, d[pt * K + o]);
  sigma[pt] = sqrtf(m / (float)(2 * n_pix));
}

// w[pt, o] = -max((d - P s2) / (sqrt(2) sqrt(P) s2), 0), s2 = sigma^2 +
// sigma_other^2 (sigma_other = 1 outside the scan), in place over d
__global__ void k_nlpar_logits(float* __restrict__ d, int hs, int ws, int K, int n_pix,
                               const int* __restrict__ offsets, const float* __restrict__ sigma) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)hs * ws * K) return;
  const int64_t pt = t / K;
  const int o = (int)(t - pt * K);
  const int y = (int)(pt / ws) + offsets[2 * o], x = (int)(pt % ws) + offsets[2 * o + 1];
  const float so = (y >= 0 && y < hs && x >= 0 && x < ws) ? sigma[(int64_t)y * ws + x] : 1.0f;
  const float sp = sigma[pt];
  const float s2 = sp * sp + so * so;
  const float scale = (float)(1.4142135623730951 * sqrt((double)n_pix));  // 2**0.5 * n_pix**0.5
  const float v = (d[t] - (float)n_pix * s2) / (scale * s2);
  d[t] = -fmaxf(v, 0.0f);
}

// One Newton iteration: per point e_o = exp(w_o / g^2) over offsets 0..8,
// S = sum e_o; obj = mean(e_0 / S) - coeff, grad = mean(-2 e_0 (w_0 S -
// sum w_o e_o) / (g^3 S^2)); the last block to finish updates g (FP64 sums).
__global__ void __launch_bounds__(kNlWThreads) k_nlpar_fit(const float* __restrict__ w, int64_t n_pts, int K,
                                                          double coeff, double tol, NlFitState* st,
                                                          double2* __restrict__ partial) {
  __shared__ double red[32];
  __shared__ bool last;
  if (st->done) return;  // uniform: the state is written only by the previous launch
  const double g = st->g;
  const float g2 = (float)(g * g), g3 = (float)(g * g * g);
  double so = 0.0, sg = 0.0;
  for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < n_pts;
       pt += (int64_t)gridDim.x * blockDim.x) {
    const float* r = w + pt * K;
    const float w0 = r[0];
    const float e0 = expf(w0 / g2);
    float S = e0, Swe = w0 * e0;
    for (int o = 1; o < 9; ++o) {
      const float wo = r[o];
      const float e = expf(wo / g2);
      S += e;
      Swe += wo * e;
    }
    so += e0 / S;
    sg += -2.0f * e0 * (w0 * S - Swe) / (g3 * S * S);
  }
  so = block_sum(so, red);
  sg = block_sum(sg, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = make_double2(so, sg);
    __threadfence();
    last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
    const double2 v = __ldcg(partial + i);
    a += v.x;
    b += v.y;
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) {
    const double obj = a / (double)n_pts - coeff, grad = b / (double)n_pts;
    st->g = g - obj / grad;
    st->done = fabs(obj) < tol ? 1 : 0;
    st->ticket = 0;
  }
}

// weights[pt, :] = softmax over o of (w / g^2, + bias at o = 0; -inf for
// neighbours outside the scan), in place. One warp per point.
__global__ void k_nlpar_softmax(float* __restrict__ w, int hs, int ws, int K, const int* __restrict__ offsets,
                                const NlFitState* st, float bias) {
  const int64_t pt = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (pt >= (int64_t)hs * ws) return;
  const float g2 = (float)(st->g * st->g);
  const int py = (int)(pt / ws), px = (int)(pt % ws);
  float* r = w + pt * K;
  float mx = -INFINITY;
  for (int o = lane; o < K; o += 32) {
    const int y = py + offsets[2 * o], x = px + offsets[2 * o + 1];
    float v = r[o] / g2;
    if (o == 0 && bias > 0.0f) v += bias;
    if (y < 0 || y >= hs || x < 0 || x >= ws) v = -INFINITY;
    r[o] = v;
    mx = fmaxf(mx, v);
  }
  mx = warp_max(mx);
  float sum = 0.f;
  for (int o = lane; o < K; o += 32) sum += expf(r[o] - mx);
  sum = warp_sum(sum);
  for (int o = lane; o < K; o += 32) r[o] = expf(r[o] - mx) / sum;
}

// Second grid dimension, so that small scans still fill the GPU: offset
// groups (distances) or pixel ranges (average), each CTA writing disjoint
// outputs. Aim for `waves` waves at the kernel's occupancy. A distance CTA
// reloads the whole tile for fewer offsets, so distances split only to fill
// one wave; the average splits its pixel range, which costs nothing extra.
static int nl_splits(const void* func, size_t smem, int tiles, int max_splits, int waves) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kNlThreads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int64_t want = (int64_t)waves * device_sm_count() * per_sm;
  return (int)std::max<int64_t>(1, std::min<int64_t>(max_splits, (want + tiles - 1) / tiles));
}

template <int HALO>
static int nl_launch(bool average, const float* data, int hs, int ws, int n_pix, int64_t ld, const int* offsets,
                     int o0, int n_off, int n_off_total, float* dists, const float* weights, int accumulate,
                     float* out, int64_t ld_out, cudaStream_t s) {
  const int tiles = ceil_div(hs, kNlTile) * ceil_div(ws, kNlTile);
  const size_t chunk_bytes = (size_t)kNlChunk * nl_plane(HALO) * sizeof(float);
  if (!average) {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_nlpar_dists<HALO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)chunk_bytes));
    // groups of at least 16 offsets
    const int groups = nl_splits((const void*)k_nlpar_dists<HALO>, chunk_bytes, tiles, std::max(1, n_off / 16), 1);
    const int per_group = ceil_div(n_off, groups);
    const int n_groups = ceil_div(n_off, per_group);
    k_nlpar_dists<HALO><<<dim3(tiles, n_groups), kNlThreads, chunk_bytes, s>>>(data, hs, ws, n_pix, ld, offsets, o0,
                                                                              n_off, per_group, n_off_total, dists);
  } else {
    const size_t smem = ((chunk_bytes + 15) & ~(size_t)15) + (size_t)kNlTile * kNlTile * n_off * sizeof(float);
    EBSD_CUDA_CHECK(
        cudaFuncSetAttribute(k_nlpar_average<HALO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // ranges of whole chunks, at least 4 chunks each
    const int n_chunks = ceil_div(n_pix, kNlChunk);
    const int splits = nl_splits((const void*)k_nlpar_average<HALO>, smem, tiles, std::max(1, n_chunks / 4), 3);
    const int pix_per_split = ceil_div(n_chunks, splits) * kNlChunk;
    const int n_splits = ceil_div(n_pix, pix_per_split);
    k_nlpar_average<HALO><<<dim3(tiles, n_splits), kNlThreads, smem, s>>>(data, hs, ws, n_pix, pix_per_split, ld,
                                                                         offsets, o0, n_off, n_off_total, weights,
                                                                         accumulate, out, ld_out);
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}

static int nl_dispatch(bool average, const float* data, int hs, int ws, int n_pix, int64_t ld, int k_rad,
                       const int* offsets, int o0, int n_off, int n_off_total, float* dists, const float* weights,
                       int accumulate, float* out, int64_t ld_out, cudaStream_t s) {
  switch (k_rad) {
#define EBSD_NL_CASE(R)                                                                                          \
  case R:                                                                                                        \
    return nl_launch<R>(average, data, hs, ws, n_pix, ld, offsets, o0, n_off, n_off_total, dists, weights,      \
                        accumulate, out, ld_out, s);
    EBSD_NL_CASE(0)
    EBSD_NL_CASE(1)
    EBSD_NL_CASE(2)
    EBSD_NL_CASE(3)
    EBSD_NL_CASE(4)
    EBSD_NL_CASE(5)
    EBSD_NL_CASE(6)
    EBSD_NL_CASE(7)
#undef EBSD_NL_CASE
    default:
      EBSD_ARG_CHECK(false, "NLPAR: kernel radius must be in [0, %d]", kNlMaxRad);
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
  cudaStream_t s = as_stream(stream);
  if (n_pix <= 4 * kNormThreads)
    k_normalize<4><<<blocks, kNormThreads, 0, s>>>(patterns, n, n_pix, ld, mode);
  else if (n_pix <= 8 * kNormThreads)
    k_normalize<8><<<blocks, kNormThreads, 0, s>>>(patterns, n, n_pix, ld, mode);
  else if (n_pix <= 16 * kNormThreads)
    k_normalize<16><<<blocks, kNormThreads, 0, s>>>(patterns, n, n_pix, ld, mode);
  else
    k_normalize<0><<<blocks, kNormThreads, 0, s>>>(patterns, n, n_pix, ld, mode);
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
  const ClaheLayout lay(height, width, grid_h, grid_w, n_bins);
  EBSD_ARG_CHECK(lay.total_tables <= kClaheSmemCap, "ebsd_clahe: grid x bins too large for shared memory");
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
  const int n_pix = height * width;
  a.vec16 = (reinterpret_cast<uintptr_t>(images) % 16 == 0 && ld % 4 == 0 && n_pix % 4 == 0) ? 1 : 0;
  a.out = out;
  a.ld_out = ld_out;
  const size_t staged_smem = lay.total_tables + 2 * (size_t)n_pix * sizeof(float);
  const bool staged = staged_smem <= kClaheSmemCap;
  const size_t smem = staged ? staged_smem : lay.total_tables;
  cudaStream_t s = as_stream(stream);
  if (staged) {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_clahe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EBSD_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clahe<true>, kClaheThreads, smem));
    const int blocks = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * std::max(per_sm, 1));
    k_clahe<true><<<blocks, kClaheThreads, smem, s>>>(a);
  } else {
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_clahe<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EBSD_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clahe<false>, kClaheThreads, smem));
    const int blocks = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * std::max(per_sm, 1));
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
  return nl_dispatch(false, data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0, n_off, n_off_total, dists, nullptr,
                     0, nullptr, 0, as_stream(stream));
}

extern "C" int ebsd_nlpar_average(const float* data, int scan_h, int scan_w, int n_pix, int64_t ld, int k_rad,
                                  const int* offsets, int o0, int n_off, int n_off_total, const float* weights,
                                  int accumulate, float* out, int64_t ld_out, void* stream) {
  if (int rc = nl_check(data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0, n_off, n_off_total)) return rc;
  EBSD_ARG_CHECK(weights && out && ld_out >= n_pix, "NLPAR: bad output");
  EBSD_ARG_CHECK(out != data, "NLPAR: the average cannot be written in place");
  return nl_dispatch(true, data, scan_h, scan_w, n_pix, ld, k_rad, offsets, o0, n_off, n_off_total, nullptr, weights,
                     accumulate, out, ld_out, as_stream(stream));
}

extern "C" size_t ebsd_nlpar_workspace_bytes(int scan_h, int scan_w) {
  return 64 + (size_t)kNlFitBlocks * sizeof(double2) + (size_t)scan_h * scan_w * sizeof(float);
}

extern "C" int ebsd_nlpar_weights(float* dists, int scan_h, int scan_w, int n_pix, const int* offsets, int n_off,
                                  float coeff, float coeff_fit_tol, float center_logit_bias, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  EBSD_ARG_CHECK(dists && offsets && workspace, "ebsd_nlpar_weights: null pointer");
  EBSD_ARG_CHECK(scan_h >= 1 && scan_w >= 1 && n_pix >= 1, "ebsd_nlpar_weights: bad sizes");
  EBSD_ARG_CHECK(n_off >= 9, "ebsd_nlpar_weights: the window needs at least 9 offsets (k_rad >= 1)");
  EBSD_ARG_CHECK(workspace_bytes >= ebsd_nlpar_workspace_bytes(scan_h, scan_w),
                 "ebsd_nlpar_weights: workspace too small");
  EBSD_ARG_CHECK(reinterpret_cast<uintptr_t>(workspace) % 16 == 0, "ebsd_nlpar_weights: workspace not 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  auto* st = reinterpret_cast<NlFitState*>(workspace);
  auto* partial = reinterpret_cast<double2*>(static_cast<uint8_t*>(workspace) + 64);
  float* sigma = reinterpret_cast<float*>(partial + kNlFitBlocks);
  const int64_t n_pts = (int64_t)scan_h * scan_w;
  k_nlpar_fit_init<<<1, 1, 0, s>>>(st);
  EBSD_LAUNCH_CHECK();
  k_nlpar_sigma<<<ceil_div(n_pts, 256), 256, 0, s>>>(dists, n_pts, n_off, n_pix, sigma);
  EBSD_LAUNCH_CHECK();
  k_nlpar_logits<<<ceil_div(n_pts * n_off, 256), 256, 0, s>>>(dists, scan_h, scan_w, n_off, n_pix, offsets, sigma);
  EBSD_LAUNCH_CHECK();
  const int fit_blocks = (int)std::min<int64_t>(kNlFitBlocks, ceil_div(n_pts, kNlWThreads));
  for (int i = 0; i < 10; ++i) {
    k_nlpar_fit<<<fit_blocks, kNlWThreads, 0, s>>>(dists, n_pts, n_off, (double)coeff, (double)coeff_fit_tol, st,
                                                   partial);
    EBSD_LAUNCH_CHECK();
  }
  k_nlpar_softmax<<<ceil_div(n_pts * 32, 256), 256, 0, s>>>(dists, scan_h, scan_w, n_off, offsets, st,
                                                            center_logit_bias);
  EBSD_LAUNCH_CHECK();
  return 0;
}
