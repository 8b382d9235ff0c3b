// Pattern-centre fitting by the spatial FFT search (ebsdtorch/ebsd/fitting.py:
// 359-540): the two kernels around the FFT cross-correlation.
//
// k_pcfit_prep: per pattern, x - min, divided by the max of that, minus the
// mean (the "dot" metric), written into the zero-padded enlarged detector
// (fitting.py:387-412).
// k_pcfit_reduce: for every (pattern, shift) of the enlarged detector, the
// maximum over one dictionary chunk of the circular cross-correlations (the
// irfft2 output, read through fftshift) and its index, folded into the
// running best of the current pc_z: best = max(best, chunk max), index
// replaced where the chunk's maximum equals the new best (fitting.py:498-507).
// The correlation tensor is read once, coalesced along the detector rows,
// each output's dictionary chunk split over 4 threads.
#include <algorithm>
#include <climits>

#include "common.cuh"

namespace ebsd {

constexpr int kFitThreads = 256;

__global__ void __launch_bounds__(kFitThreads) k_pcfit_prep(const float* __restrict__ pats, int hb, int wb,
                                                           int hp, int wp, int pad_top, int pad_left, int zero_mean,
                                                           float* __restrict__ out) {
  __shared__ float fred[32];
  __shared__ double dred[32];
  const int n_pix = hb * wb;
  const float* x = pats + (int64_t)blockIdx.x * n_pix;
  float* o = out + (int64_t)blockIdx.x * hp * wp;
  for (int t = threadIdx.x; t < hp * wp; t += blockDim.x) o[t] = 0.0f;
  float mn = INFINITY;
  for (int t = threadIdx.x; t < n_pix; t += blockDim.x) mn = fminf(mn, x[t]);
  mn = -block_max(-mn, fred);
  float mx = -INFINITY;
  for (int t = threadIdx.x; t < n_pix; t += blockDim.x) mx = fmaxf(mx, x[t] - mn);
  mx = block_max(mx, fred);
  float mean = 0.0f;
  if (zero_mean) {
    double s = 0.0;
    for (int t = threadIdx.x; t < n_pix; t += blockDim.x) s += (x[t] - mn) / mx;
    mean = (float)(block_sum(s, dred) / n_pix);
  }
  __syncthreads();  // the zero fill is complete before the interior is written
  for (int t = threadIdx.x; t < n_pix; t += blockDim.x) {
    const int r = t / wb, c = t - r * wb;
    o[(r + pad_top) * wp + c + pad_left] = (x[t] - mn) / mx - mean;
  }
}

constexpr int kRedPos = 64;     // (pattern, shift) outputs per CTA
constexpr int kRedSplits = 4;   // dictionary slices per output, one per 64 threads

// Thread (slice, position): the maximum over its slice of the chunk, 8 loads
// in flight; the 4 slices combine in shared memory (the larger value wins,
// the smaller dictionary index on ties, so the first maximum wins).
__global__ void __launch_bounds__(kRedPos * kRedSplits) k_pcfit_reduce(const float* __restrict__ corr, int n,
                                                                       int n_pat, int hp, int wp,
                                                                       int64_t index_base, float* __restrict__ best,
                                                                       int64_t* __restrict__ best_index) {
  __shared__ float sv[kRedSplits][kRedPos];
  __shared__ int sa[kRedSplits][kRedPos];
  const int64_t plane = (int64_t)hp * wp;
  const int64_t total = (int64_t)n_pat * plane;
  const int pos = threadIdx.x % kRedPos, slice = threadIdx.x / kRedPos;
  const int64_t t = blockIdx.x * (int64_t)kRedPos + pos;
  float vmax = -INFINITY;
  int arg = INT_MAX;
  if (t < total) {
    const int b = (int)(t / plane);
    const int rem = (int)(t - (int64_t)b * plane);
    const int y = rem / wp, x = rem - y * wp;
    // fftshift: output (y, x) holds input ((y - hp / 2) mod hp, (x - wp / 2) mod wp)
    const int sy = (y - hp / 2 + hp) % hp, sx = (x - wp / 2 + wp) % wp;
    const float* src = corr + (int64_t)b * plane + (int64_t)sy * wp + sx;
    const int d0 = (int)((int64_t)n * slice / kRedSplits), d1 = (int)((int64_t)n * (slice + 1) / kRedSplits);
    int d = d0;
    for (; d + 8 <= d1; d += 8) {
      float v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = __ldg(src + (int64_t)(d + k) * total);
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (v[k] > vmax) {
          vmax = v[k];
          arg = d + k;
        }
    }
    for (; d < d1; ++d) {
      const float v = __ldg(src + (int64_t)d * total);
      if (v > vmax) {
        vmax = v;
        arg = d;
      }
    }
  }
  sv[slice][pos] = vmax;
  sa[slice][pos] = arg;
  __syncthreads();
  if (slice != 0 || t >= total) return;
  for (int s = 1; s < kRedSplits; ++s) {
    const float v = sv[s][pos];
    if (v > vmax || (v == vmax && sa[s][pos] < arg)) {
      vmax = v;
      arg = sa[s][pos];
    }
  }
  const float nb = fmaxf(best[t], vmax);
  best[t] = nb;
  if (nb == vmax) best_index[t] = index_base + arg;
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_pcfit_prep(const float* patterns, int n, int height, int width, int padded_h, int padded_w,
                               int pad_top, int pad_left, int zero_mean, float* out, void* stream) {
  EBSD_ARG_CHECK(patterns && out, "ebsd_pcfit_prep: null pointer");
  EBSD_ARG_CHECK(n >= 0 && height >= 1 && width >= 1, "ebsd_pcfit_prep: bad sizes");
  EBSD_ARG_CHECK(pad_top >= 0 && pad_left >= 0 && pad_top + height <= padded_h && pad_left + width <= padded_w,
                 "ebsd_pcfit_prep: the pattern does not fit the padded detector");
  if (n == 0) return 0;
  k_pcfit_prep<<<n, kFitThreads, 0, as_stream(stream)>>>(patterns, height, width, padded_h, padded_w, pad_top,
                                                         pad_left, zero_mean ? 1 : 0, out);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_pcfit_reduce(const float* corr, int n, int n_patterns, int padded_h, int padded_w,
                                 int64_t index_base, float* best, int64_t* best_index, void* stream) {
  EBSD_ARG_CHECK(corr && best && best_index, "ebsd_pcfit_reduce: null pointer");
  EBSD_ARG_CHECK(n >= 1 && n_patterns >= 1 && padded_h >= 1 && padded_w >= 1, "ebsd_pcfit_reduce: bad sizes");
  const int64_t total = (int64_t)n_patterns * padded_h * padded_w;
  EBSD_ARG_CHECK(total * n < ((int64_t)1 << 62), "ebsd_pcfit_reduce: too large");
  k_pcfit_reduce<<<ceil_div(total, kRedPos), kRedPos * kRedSplits, 0, as_stream(stream)>>>(
      corr, n, n_patterns, padded_h, padded_w, index_base, best, best_index);
  EBSD_LAUNCH_CHECK();
  return 0;
}
