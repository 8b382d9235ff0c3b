// K9: orientation grid refinement, the step after dictionary indexing.
//
// Follows ebsdtorch/ebsd/refining.py:71-244 (orientation_grid_refinement):
// per pattern and iteration, every point of a local cubochoric grid
// (get_local_orientation_grid, refining.py:13-68) is turned into a rotation
// (cu2qu) and composed with the current orientation (qu_prod(grid, current)),
// moved to the fundamental zone, simulated with grid_sample(align_corners=True)
// (refining.py:200-207), mean-subtracted and dotted with the mean-subtracted
// experimental pattern; the best candidate becomes the current orientation,
// and a pattern whose grid centre stayed best has its grid scaled by
// shrink_factor.
//
// B200 design: one CTA (512 threads) per pattern runs all iterations; the
// experimental row stays in shared memory, the candidate rotations are built
// in FP64 by the first threads, and the candidates are simulated on the fly (no dictionary)
// and scored 16 at a time per pass over the pixels, each thread carrying 16
// (dot, sum) accumulators; the simulation mean is folded in as
// dot - sum(sim) / P * sum(exp). Scores are FP32 (the reference uses
// match_dtype, FP16 by default).
//
// FZ reduction: fz_left 0 reproduces the reference (ori_to_fz_laue,
// laue_fz_ori.py:36-81: the operator g maximising |(q g).w|, applied on the
// right, q g); fz_left 1 applies it on the left, g q, which keeps the
// simulated pattern (pattern(g q) == pattern(q) for the projector's q v q*).
#include <algorithm>

#include "common.cuh"
#include "cubochoric.cuh"
#include "sampling.cuh"

namespace ebsd {

constexpr int kRefThreads = 512;
constexpr int kRefGroup = 16;      // candidates scored per pass over the pixels
constexpr int kRefIlp = 4;         // candidates whose gathers are issued together
constexpr int kMaxRefGrid = 343;   // (2 * 3 + 1)^3
constexpr int kMaxRefPix = 40960;  // FP32 pattern row in shared memory (160 KiB)

__device__ __forceinline__ void qmul_d(const double a[4], const double b[4], double o[4]) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

__device__ __forceinline__ void qstd_d(double q[4]) {
  if (q[0] < 0.0)
    for (int k = 0; k < 4; ++k) q[k] = -q[k];
}

__global__ void __launch_bounds__(kRefThreads) k_refine(
    const float* __restrict__ mp, int mp_h, int mp_w2, const float* __restrict__ coords, int n_pix,
    const float* __restrict__ offsets, const float* __restrict__ exp_rows, int64_t ld_e,
    const float* __restrict__ q_in, int64_t n, const float* __restrict__ grid, int n_grid, int centre,
    const LaueTable ops, int fz_left, int n_iter, float shrink, float* __restrict__ q_out,
    float* __restrict__ dots) {
  extern __shared__ float erow[];
  __shared__ float4 cand[kMaxRefGrid];
  __shared__ float score[kMaxRefGrid];
  __shared__ float part_d[kRefThreads / 32][kRefGroup];
  __shared__ float part_s[kRefThreads / 32][kRefGroup];
  __shared__ double qcur[4];
  __shared__ float scale_s;
  __shared__ float red[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const float* rx = coords;
  const float* ry = coords + n_pix;
  const float* rz = coords + 2 * (int64_t)n_pix;
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    float es = 0.f;
    for (int p = tid; p < n_pix; p += blockDim.x) {
      const float e = exp_rows[i * ld_e + p];
      erow[p] = e;
      es += e;
    }
    const float esum = block_sum(es, red);  // synchronises the block
    if (tid == 0) {
      for (int k = 0; k < 4; ++k) qcur[k] = (double)q_in[4 * i + k];
      scale_s = 1.0f;
    }
    const float ox = offsets ? offsets[2 * i] : 0.f, oy = offsets ? offsets[2 * i + 1] : 0.f;
    __syncthreads();
    for (int it = 0; it < n_iter; ++it) {
      const float scale = scale_s;
      // candidate rotations: FZ(cu2qu(scale * grid[t]) * current)
      for (int t = tid; t < n_grid; t += blockDim.x) {
        double c[3], qg[4], qa[4];
        for (int k = 0; k < 3; ++k) c[k] = (double)(grid[3 * t + k] * scale);
        cu_to_qu(c, qg);
        double qc[4] = {qcur[0], qcur[1], qcur[2], qcur[3]};
        qmul_d(qg, qc, qa);
        qstd_d(qa);
        double best[4] = {qa[0], qa[1], qa[2], qa[3]}, bw = -1.0;
        for (int g = 0; g < ops.n; ++g) {
          const double o[4] = {ops.q[4 * g], ops.q[4 * g + 1], ops.q[4 * g + 2], ops.q[4 * g + 3]};
          double pr[4];
          if (fz_left)
            qmul_d(o, qa, pr);
          else
            qmul_d(qa, o, pr);
          if (fabs(pr[0]) > bw) {
            bw = fabs(pr[0]);
            for (int k = 0; k < 4; ++k) best[k] = pr[k];
          }
        }
        qstd_d(best);
        cand[t] = make_float4((float)best[0], (float)best[1], (float)best[2], (float)best[3]);
      }
      __syncthreads();
      for (int g0 = 0; g0 < n_grid; g0 += kRefGroup) {
        const int ng = min(kRefGroup, n_grid - g0);
        float ad[kRefGroup], as[kRefGroup];
#pragma unroll
        for (int c = 0; c < kRefGroup; ++c) {
          ad[c] = 0.f;
          as[c] = 0.f;
        }
        for (int p = tid; p < n_pix; p += blockDim.x) {
          float vx = __ldg(rx + p), vy = __ldg(ry + p), vz = __ldg(rz + p);
          if (offsets) {
            // per-pattern source point (refining.py:117-128), then unit rays
            vx += ox;
            vy += oy;
            const float nr = sqrtf(vx * vx + vy * vy + vz * vz);
            vx /= nr;
            vy /= nr;
            vz /= nr;
          }
          const float e = erow[p];
          // kRefIlp candidates at a time: taps first, then their gathers
          // together (the loop is bound by the gather latency through L2)
#pragma unroll
          for (int c0 = 0; c0 < kRefGroup; c0 += kRefIlp) {
            BorderTaps t[kRefIlp];
#pragma unroll
            for (int k = 0; k < kRefIlp; ++k) {
              const float3 r = rotate(cand[g0 + min(c0 + k, ng - 1)], vx, vy, vz);
              const float2 uv = lambert_side_by_side(r.x, r.y, r.z);
              t[k] = border_taps<true>(mp_h, mp_w2, uv.x, uv.y);
            }
            float gv[kRefIlp][4];
#pragma unroll
            for (int k = 0; k < kRefIlp; ++k) {
              gv[k][0] = __ldg(mp + t[k].i00);
              gv[k][1] = __ldg(mp + t[k].i01);
              gv[k][2] = __ldg(mp + t[k].i10);
              gv[k][3] = __ldg(mp + t[k].i11);
            }
#pragma unroll
            for (int k = 0; k < kRefIlp; ++k) {
              const int c = c0 + k;
              if (c < ng) {
                const float val = gv[k][0] * t[k].w00 + gv[k][1] * t[k].w01 + gv[k][2] * t[k].w10 +
                                  gv[k][3] * t[k].w11;
                ad[c] = fmaf(val, e, ad[c]);
                as[c] += val;
              }
            }
          }
        }
#pragma unroll
        for (int c = 0; c < kRefGroup; ++c) {
          const float d = warp_sum(ad[c]), s = warp_sum(as[c]);
          if (lane == 0) {
            part_d[wid][c] = d;
            part_s[wid][c] = s;
          }
        }
        __syncthreads();
        if (tid < ng) {
          double d = 0.0, s = 0.0;
          for (int w = 0; w < kRefThreads / 32; ++w) {
            d += part_d[w][tid];
            s += part_s[w][tid];
          }
          score[g0 + tid] = (float)(d - s / n_pix * (double)esum);
        }
        __syncthreads();
      }
      if (tid == 0) {
        int b = 0;
        float bv = score[0];
        for (int t = 1; t < n_grid; ++t)
          if (score[t] > bv) {
            bv = score[t];
            b = t;
          }
        dots[i * n_iter + it] = bv;
        const float4 qb = cand[b];
        qcur[0] = qb.x;
        qcur[1] = qb.y;
        qcur[2] = qb.z;
        qcur[3] = qb.w;
        if (b == centre) scale_s = scale * shrink;
      }
      __syncthreads();
    }
    if (tid == 0)
      for (int k = 0; k < 4; ++k) q_out[4 * i + k] = (float)qcur[k];
    __syncthreads();
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_refine_grid(const float* master_pattern, int mp_h, int mp_w2, const float* coords_soa,
                                int n_pix, const float* offsets, const float* exp_rows, int64_t ld_e,
                                const float* q_in, int64_t n, const float* grid_cu, int n_grid, int laue_id,
                                int fz_left, int n_iter, float shrink, float* q_out, float* dots,
                                void* stream) {
  EBSD_ARG_CHECK(master_pattern && coords_soa && exp_rows && q_in && grid_cu && q_out && dots,
                 "ebsd_refine_grid: null pointer");
  EBSD_ARG_CHECK(mp_h >= 2 && mp_w2 >= 2, "master pattern shape (%d, %d) invalid", mp_h, mp_w2);
  EBSD_ARG_CHECK(n_pix >= 1 && n_pix <= kMaxRefPix && ld_e >= n_pix, "row length %d outside [1, %d]", n_pix,
                 kMaxRefPix);
  EBSD_ARG_CHECK(n_grid >= 1 && n_grid <= kMaxRefGrid && (n_grid & 1), "grid of %d points: odd, at most %d",
                 n_grid, kMaxRefGrid);
  EBSD_ARG_CHECK(laue_id >= 1 && laue_id <= 11, "Laue group %d is not supported", laue_id);
  EBSD_ARG_CHECK(n_iter >= 1 && n_iter <= 64, "n_iter must be in [1, 64]");
  EBSD_ARG_CHECK(n >= 0, "n < 0");
  if (n == 0) return 0;
  LaueTable t{};
  build_laue_table(laue_id, &t);
  const size_t smem = (size_t)n_pix * sizeof(float);
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * 16);
  k_refine<<<grid, kRefThreads, smem, as_stream(stream)>>>(master_pattern, mp_h, mp_w2, coords_soa, n_pix, offsets,
                                                           exp_rows, ld_e, q_in, n, grid_cu, n_grid,
                                                           (n_grid - 1) / 2, t, fz_left, n_iter, shrink, q_out,
                                                           dots);
  EBSD_LAUNCH_CHECK();
  return 0;
}
