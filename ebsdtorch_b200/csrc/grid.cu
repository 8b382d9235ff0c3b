// K0: FP64 cubochoric SO(3) grid -> quaternions -> Laue fundamental-zone
// filter -> order-preserving compaction.
//
// Follows ebsdtorch/s2_and_so3/laue_fz_ori.py:516-557 (grid size rule and
// filter), sampling.py:179-205 (grid coordinates, 'ij' order), cu2ho
// orientations.py:293-349, ho2ax :419-517, ax2qu :730-746, qu_std
// quaternions.py:27-38, ori_in_fz_laue laue_fz_ori.py:144-239.
//
// Differences from the reference, by design: everything is FP64 (the
// reference works in FP32 and fits cos(w/2) with a polynomial); the rotation
// angle is obtained by solving |h|^3 = 3/4 (w - sin w) with Newton's method.
// The output set and order equal the reference's for every grid checked.
#include "common.cuh"
#include "cubochoric.cuh"

namespace ebsd {

constexpr int kGridBlock = 1024;

__device__ __forceinline__ bool in_fz(const double q[4], int laue) {
  const double w = q[0], x = fabs(q[1]), y = fabs(q[2]), z = fabs(q[3]);
  const double kR2M1 = 0.41421356237309504880, kR3 = 1.73205080756887729353;
  switch (laue) {
    case 11: return (fmax(fmax(x, y), z) <= w * kR2M1) && (x + y + z <= w);
    case 10: return x + y + z <= w;
    case 9: {
      const double mm = fmax(x, y), nn = fmin(x, y);
      const double rot = (mm > (2.0 + kR3) * nn) ? mm : (kR3 / 2.0) * mm + 0.5 * nn;
      return (z <= (2.0 - kR3) * w) && (rot <= w);
    }
    case 8: return z <= (2.0 - kR3) * w;
    case 7: {
      const double rot = (x >= y * kR3) ? x : (kR3 / 2.0) * y + 0.5 * x;
      return (z <= (1.0 / kR3) * w) && (rot <= w);
    }
    case 6: return z <= (1.0 / kR3) * w;
    case 5: {
      const double mm = fmax(x, y), nn = fmin(x, y);
      const double rot = (mm > (kR2M1 + 2.0) * nn) ? mm : 0.70710678118654752440 * (mm + nn);
      return (z <= kR2M1 * w) && (rot <= w);
    }
    case 4: return z <= kR2M1 * w;
    case 3: return fmax(fmax(x, y), z) <= w;
    case 2: return z <= w;
    default: return true;
  }
}

// Grid coordinate i of `edge` along each axis: the edge + 1 points spanning
// [-a/2, a/2] with the last dropped, i.e. a/2 * (2i - edge) / edge. This form
// is exactly 0 at i = edge / 2 and exactly antisymmetric, as the reference's
// symmetric linspace is; the FZ test of 180-degree rotations about in-plane
// axes (z exactly 0) depends on that. grid.cu is compiled without FMA
// contraction so the FP64 arithmetic rounds like the CPU oracle.
__device__ __forceinline__ void grid_point(int64_t i, int edge, double c[3]) {
  const double kHalf = 1.0725146985555127;  // 0.5 * pi^(2/3)
  const int64_t e2 = (int64_t)edge * edge;
  const int ia = (int)(i / e2), ib = (int)((i / edge) % edge), ic = (int)(i % edge);
  c[0] = kHalf * (double)(2 * ia - edge) / (double)edge;
  c[1] = kHalf * (double)(2 * ib - edge) / (double)edge;
  c[2] = kHalf * (double)(2 * ic - edge) / (double)edge;
}

__global__ void __launch_bounds__(kGridBlock) k_grid_count(int laue, int edge, int64_t n_total,
                                                           int32_t* __restrict__ block_counts) {
  const int64_t i = blockIdx.x * (int64_t)kGridBlock + threadIdx.x;
  int flag = 0;
  if (i < n_total) {
    double c[3], q[4];
    grid_point(i, edge, c);
    cu_to_qu(c, q);
    flag = in_fz(q, laue) ? 1 : 0;
  }
  const int cnt = __syncthreads_count(flag);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(1024) k_grid_scan(const int32_t* __restrict__ block_counts,
                                                    int n_blocks, int64_t* __restrict__ offsets,
                                                    int64_t* __restrict__ d_count) {
  __shared__ int64_t red[32];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n_blocks; base += 1024) {
    const int j = base + threadIdx.x;
    const int64_t v = (j < n_blocks) ? block_counts[j] : 0;
    // inclusive warp scan
    int64_t x = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) red[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int64_t w = red[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      red[lane] = w;
    }
    __syncthreads();
    const int64_t incl = x + (wid > 0 ? red[wid - 1] : 0);
    if (j < n_blocks) offsets[j] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *d_count = carry;
}

__global__ void __launch_bounds__(kGridBlock) k_grid_write(int laue, int edge, int64_t n_total,
                                                           const int64_t* __restrict__ offsets,
                                                           float* __restrict__ out_f32,
                                                           double* __restrict__ out_f64,
                                                           int32_t* __restrict__ out_cells) {
  __shared__ int warp_cnt[kGridBlock / 32];
  const int64_t i = blockIdx.x * (int64_t)kGridBlock + threadIdx.x;
  double q[4] = {0, 0, 0, 0};
  bool flag = false;
  if (i < n_total) {
    double c[3];
    grid_point(i, edge, c);
    cu_to_qu(c, q);
    flag = in_fz(q, laue);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) warp_cnt[wid] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int w = 0; w < wid; ++w) before += warp_cnt[w];
  if (flag) {
    const int64_t r = offsets[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u));
    reinterpret_cast<float4*>(out_f32)[r] =
        make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    if (out_cells) out_cells[r] = (int32_t)i;
    if (out_f64) {
      out_f64[4 * r + 0] = q[0];
      out_f64[4 * r + 1] = q[1];
      out_f64[4 * r + 2] = q[2];
      out_f64[4 * r + 3] = q[3];
    }
  }
}

static int64_t grid_points(int edge) { return (int64_t)edge * edge * edge; }
static int grid_blocks(int edge) { return (int)((grid_points(edge) + kGridBlock - 1) / kGridBlock); }

}  // namespace ebsd

using namespace ebsd;

extern "C" size_t ebsd_grid_workspace_bytes(int edge_length) {
  if (edge_length <= 0) return 0;
  const size_t nb = (size_t)grid_blocks(edge_length);
  return nb * sizeof(int64_t) + nb * sizeof(int32_t) + 256;
}

static int grid_check(int laue_id, int edge, const void* ws, size_t ws_bytes) {
  EBSD_ARG_CHECK(laue_id >= 1 && laue_id <= 11, "Laue group %d is not supported", laue_id);
  EBSD_ARG_CHECK(edge >= 1 && edge <= 2048, "grid edge length %d out of range [1, 2048]", edge);
  EBSD_ARG_CHECK(ws != nullptr, "grid workspace is null");
  EBSD_ARG_CHECK(ws_bytes >= ebsd_grid_workspace_bytes(edge),
                 "grid workspace too small: %zu < %zu bytes", ws_bytes,
                 ebsd_grid_workspace_bytes(edge));
  return 0;
}

extern "C" int ebsd_grid_fz_count(int laue_id, int edge_length, void* workspace,
                                  size_t workspace_bytes, int64_t* d_count, void* stream) {
  if (int rc = grid_check(laue_id, edge_length, workspace, workspace_bytes)) return rc;
  EBSD_ARG_CHECK(d_count != nullptr, "d_count is null");
  const int nb = grid_blocks(edge_length);
  int64_t* offsets = reinterpret_cast<int64_t*>(workspace);
  int32_t* counts = reinterpret_cast<int32_t*>(offsets + nb);
  cudaStream_t s = as_stream(stream);
  k_grid_count<<<nb, kGridBlock, 0, s>>>(laue_id, edge_length, grid_points(edge_length), counts);
  EBSD_LAUNCH_CHECK();
  k_grid_scan<<<1, 1024, 0, s>>>(counts, nb, offsets, d_count);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_grid_fz_write(int laue_id, int edge_length, const void* workspace,
                                  size_t workspace_bytes, float* out_f32, double* out_f64,
                                  int32_t* out_cells, void* stream) {
  if (int rc = grid_check(laue_id, edge_length, workspace, workspace_bytes)) return rc;
  EBSD_ARG_CHECK(out_f32 != nullptr, "out_f32 is null");
  EBSD_ARG_CHECK((reinterpret_cast<uintptr_t>(out_f32) & 15) == 0, "out_f32 must be 16-byte aligned");
  const int nb = grid_blocks(edge_length);
  const int64_t* offsets = reinterpret_cast<const int64_t*>(workspace);
  k_grid_write<<<nb, kGridBlock, 0, as_stream(stream)>>>(laue_id, edge_length,
                                                         grid_points(edge_length), offsets, out_f32,
                                                         out_f64, out_cells);
  EBSD_LAUNCH_CHECK();
  return 0;
}
