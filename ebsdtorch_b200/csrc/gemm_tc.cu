// K3: pattern x dictionary contraction on the 5th-generation tensor cores
// (tcgen05) with a fused streaming top-k epilogue, and the same main loop
// with a plain FP32 store epilogue (PCA covariance and projections).
//
// Replaces knn_batch (ebsdtorch/utils/knn.py:80-103: `query @ data.t()` then
// torch.topk) and the ChunkedKNN running merge (knn.py:219-266); the store
// variant replaces the einsum in update_covmat (pca_covmat.py:53-91) and the
// PCA projections (indexing.py:401, 421, 452).
//
// Structure (one CTA per SM, 192 threads):
//   warp 0      TMA producer: A tile (128 rows x 128 B) and B tile
//               (256 rows x 128 B) per stage, 128-byte swizzle, 4 stages.
//   warp 1      allocates 512 TMEM columns (two 128x256 FP32 accumulators)
//               and issues tcgen05.mma (M=128, N=256, 32 B of K each).
//   warps 2-5   epilogue: tcgen05.ld of the accumulator rows; each thread
//               owns one query row and keeps its best candidates sorted in
//               registers across all dictionary tiles of its range.
// A unit of work is (query tile, dictionary range); the epilogue of tile t
// overlaps the MMAs of tile t+1 through the second accumulator.
// Every wait is bounded (p.wait_ns); a timeout is reported in *status. When
// any role gives up, the CTA still lets every TMA copy and MMA it issued
// complete (bounded by the default limit) before it releases TMEM and exits.
#include <algorithm>
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace ebsd {

constexpr int BM = 128;
constexpr int BKB = 128;  // bytes of K per stage and row (one 128-byte swizzle atom)
constexpr int A_BYTES = BM * BKB;
constexpr int EPI_THREADS = 128;
constexpr int THREADS = 64 + EPI_THREADS;
constexpr int SCRATCH_BYTES = 32 * EPI_THREADS * 4;

// Shape of one CTA tile: 128 query rows x BN dictionary rows (N of the MMA).
template <int BN_>
struct Tile {
  static constexpr int BN = BN_;
  static constexpr int STAGES = BN_ == 256 ? 4 : 6;
  static constexpr int B_BYTES = BN_ * BKB;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int BAR_BYTES = 8 * (2 * STAGES + 4 + 1) + 16;
  static constexpr int SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + SCRATCH_BYTES + BAR_BYTES;
  static constexpr uint32_t TMEM_COLS = 2 * BN_;  // two accumulators
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

struct GemmParams {
  int m_tiles;  // query tiles with rows (the pair kernel's odd CTA may have none)
  int n_tiles;
  int splits;
  int units;  // m_tiles * splits; a CTA takes units blockIdx.x, + gridDim.x, ...
  int k_iters;
  int64_t n_valid;
  const float* col_scale;
  // MODE 0, optional: score = acc * col_scale[d] + col_bias[d] * row_scale[q]
  // (the euclidean ranking 2 |d| cos - |d|^2 / |q|)
  const float* col_bias;
  const float* row_scale;
  float* part_val;
  int32_t* part_idx;
  int part_slots;
  int slot_base;
  int32_t index_base;
  float* C;
  int64_t ldc;
  int64_t m_valid;
  float alpha;
  int accumulate;
  const float* bias;     // MODE 2: per-row (output channel) bias
  __nv_bfloat16* out16;  // MODE 2: bf16 activations, (n_valid x ld_out)
  float* out32;          // MODE 2: optional FP32 copy, same layout
  int64_t ld_out;
  int relu;
  int* status;
  uint64_t wait_ns;  // limit of every role's waits (kWaitLimitNs by default)
};

// Operand kinds: 0 kind::f16 with BF16, 1 kind::f8f6f4 with E4M3, 2 kind::tf32.
template <int KIND>
__host__ __device__ constexpr int kind_elem_bytes() {
  return KIND == 0 ? 2 : KIND == 1 ? 1 : 4;
}

template <int KIND, int BN>
__host__ __device__ constexpr uint32_t make_idesc() {
  // c_format F32 (bit 4); a/b format bits 7-9 / 10-12 (kind::f16: 1 = BF16;
  // kind::tf32: 2 = TF32; kind::f8f6f4: 0 = E4M3); K-major A and B; N >> 3 at
  // bit 17; M >> 4 at bit 24.
  return (1u << 4) | (KIND == 0 ? ((1u << 7) | (1u << 10)) : KIND == 2 ? ((2u << 7) | (2u << 10)) : 0u) |
         ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int KC>
__device__ __forceinline__ void topk_insert(float (&bv)[KC], int (&bi)[KC], float v, int idx) {
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

__device__ __forceinline__ void report_timeout(const GemmParams& p, volatile int* abort_flag) {
  *abort_flag = 1;
  atomicExch(p.status, EBSD_DEVICE_TIMEOUT);
}

// MODE 0: top-k epilogue (BIAS: plus col_bias[col] * row_scale[row], the
// euclidean ranking; a separate instantiation so that the angular kernel's
// epilogue carries none of it). MODE 1: store epilogue. MODE 2: convolution
// epilogue, out[col, row] = act(acc[row, col] + bias[row]) stored transposed
// in bf16 (and FP32 when asked).
template <int KIND, int MODE, int KC, int BN, bool PERSIST, bool BIAS = false>
__global__ void __launch_bounds__(THREADS, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const GemmParams p) {
  using T = Tile<BN>;
  constexpr int STAGES = T::STAGES;
  constexpr int STAGE_BYTES = T::STAGE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const uint32_t sbase = smem_u32(smem);
  float* scratch = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES + SCRATCH_BYTES);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
  auto accf_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + a); };
  auto acce_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + 2 + a); };
  const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // work unit -> (query tile, dictionary tile range); the lambdas capture
  // copies of the two fields rather than the kernel parameter itself
  const int n_splits = p.splits, n_tiles = p.n_tiles;
  auto unit_tile = [=](int u) { return u / n_splits; };
  auto unit_range = [=](int u, int& n_begin, int& n_end) {
    const int split = u - (u / n_splits) * n_splits;
    n_begin = (int)((int64_t)split * n_tiles / n_splits);
    n_end = (int)((int64_t)(split + 1) * n_tiles / n_splits);
  };
  // units of this CTA: blockIdx.x, + gridDim.x, ... when persistent; else
  // only blockIdx.x
  const int u_step = PERSIST ? (int)gridDim.x : 1;
  const int u_end = PERSIST ? p.units : (int)blockIdx.x + 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(accf_bar(a), 1);
      mbar_init(acce_bar(a), EPI_THREADS);
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) tmem_alloc(smem_u32(tmem_slot), T::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

  const uint64_t wait_ns = p.wait_ns;
  // producer progress (warp 0, lane 0) and whether any MMA was issued (warp 1,
  // lane 0): read by the drain after the roles when a role gave up
  uint32_t prod_stage = 0, prod_phase = 0;
  int64_t issued = 0;
  bool any_mma = false;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      bool ok = true;
      const int k_iters = p.k_iters;
      auto produce_unit = [&](int u) {
        const int a_row = unit_tile(u) * BM;
        int n_begin, n_end;
        unit_range(u, n_begin, n_end);
        for (int n = n_begin; n < n_end && ok; ++n) {
          for (int k = 0; k < k_iters; ++k) {
            if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag, wait_ns)) {
              ok = false;
              break;
            }
            const uint32_t a_dst = sbase + stage * STAGE_BYTES;
            mbar_arrive_expect_tx(full_bar(stage), STAGE_BYTES);
            const int kx = k * (BKB / kind_elem_bytes<KIND>());  // element coordinate
            tma_load_2d(a_dst, &tmA, kx, a_row, full_bar(stage));
            tma_load_2d(a_dst + A_BYTES, &tmB, kx, n * BN, full_bar(stage));
            ++issued;
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
      };
      // one unit: straight-line code (a unit loop in the producer or MMA
      // thread measured 15 % slower on one-wave launches)
      if constexpr (PERSIST) {
        for (int u = blockIdx.x; u < u_end && ok; u += u_step) produce_unit(u);
      } else {
        produce_unit(blockIdx.x);
      }
      if (!ok) report_timeout(p, abort_flag);
      prod_stage = stage;
      prod_phase = phase;
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      constexpr uint32_t idesc = make_idesc<KIND, BN>();
      const int k_iters = p.k_iters;
      auto mma_unit = [&](int u) {
        int n_begin, n_end;
        unit_range(u, n_begin, n_end);
        for (int n = n_begin; n < n_end && ok; ++n) {
          if (!mbar_wait(acce_bar(acc), acc_phase ^ 1u, abort_flag, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
          for (int k = 0; k < k_iters; ++k) {
            if (!mbar_wait(full_bar(stage), phase, abort_flag, wait_ns)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_addr = sbase + stage * STAGE_BYTES;
            const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BKB / 32; ++kk) {
              tc_mma<KIND>(d_tmem, smem_desc_sw128(a_addr + kk * 32), smem_desc_sw128(b_addr + kk * 32),
                           idesc, (k | kk) != 0 ? 1u : 0u);
            }
            any_mma = true;
            tc_commit(empty_bar(stage));
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          tc_commit(accf_bar(acc));
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1u;
          }
        }
      };
      if constexpr (PERSIST) {
        for (int u = blockIdx.x; u < u_end && ok; u += u_step) mma_unit(u);
      } else {
        mma_unit(blockIdx.x);
      }
      if (!ok) report_timeout(p, abort_flag);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue ----------------
    const int wq = warp & 3;              // TMEM lane quarter this warp may access
    const int etid = threadIdx.x - 64;    // 0..127, scratch column
    const int row = wq * 32 + lane;       // row of the 128-row tile
    const uint32_t lane_addr = (uint32_t)(wq * 32) << 16;
    float bv[KC];
    int bi[KC];
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < u_end && ok; u += u_step) {
      const int m_tile = unit_tile(u);
      const int split = u - m_tile * n_splits;
      int n_begin, n_end;
      unit_range(u, n_begin, n_end);
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        bv[j] = -INFINITY;
        bi[j] = -1;
      }
      float rs = 0.0f;
      if constexpr (MODE == 0 && BIAS) rs = __ldg(p.row_scale + (int64_t)m_tile * BM + row);
      for (int n = n_begin; n < n_end; ++n) {
        bool got = mbar_wait_sleep(accf_bar(acc), acc_phase, abort_flag, wait_ns);
        got = __all_sync(0xffffffffu, got);
        if (!got) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int64_t tile_col = (int64_t)n * BN;
#pragma unroll 1
        for (int c = 0; c < BN / 32; ++c) {
          __syncwarp();
          float v[32];
          tmem_ld32(tmem_base + lane_addr + (uint32_t)(acc * BN + c * 32), v);
          const int64_t col0 = tile_col + c * 32;
          if constexpr (MODE == 0) {
            uint32_t mask = 0;
            const float thr = bv[KC - 1];
            if (col0 + 32 <= p.n_valid) {
              if (p.col_scale) {
                const float4* cs = reinterpret_cast<const float4*>(p.col_scale + col0);
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4) {
                  const float4 s4 = __ldg(cs + j4);
                  v[4 * j4 + 0] *= s4.x;
                  v[4 * j4 + 1] *= s4.y;
                  v[4 * j4 + 2] *= s4.z;
                  v[4 * j4 + 3] *= s4.w;
                }
              }
              if constexpr (BIAS) {
                const float4* cb = reinterpret_cast<const float4*>(p.col_bias + col0);
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4) {
                  const float4 b4 = __ldg(cb + j4);
                  v[4 * j4 + 0] = fmaf(b4.x, rs, v[4 * j4 + 0]);
                  v[4 * j4 + 1] = fmaf(b4.y, rs, v[4 * j4 + 1]);
                  v[4 * j4 + 2] = fmaf(b4.z, rs, v[4 * j4 + 2]);
                  v[4 * j4 + 3] = fmaf(b4.w, rs, v[4 * j4 + 3]);
                }
              }
            } else {
#pragma unroll
              for (int j = 0; j < 32; ++j) {
                const bool valid = col0 + j < p.n_valid;
                const float sc = (valid && p.col_scale) ? __ldg(p.col_scale + col0 + j) : 1.0f;
                if constexpr (BIAS) {
                  const float cb = valid ? __ldg(p.col_bias + col0 + j) : 0.0f;
                  v[j] = valid ? fmaf(cb, rs, v[j] * sc) : -INFINITY;
                } else {
                  v[j] = valid ? v[j] * sc : -INFINITY;
                }
              }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) mask |= (v[j] > thr) ? (1u << j) : 0u;
            if (mask) {
#pragma unroll
              for (int j = 0; j < 32; ++j) scratch[j * EPI_THREADS + etid] = v[j];
              while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1u;
                const float sc = scratch[j * EPI_THREADS + etid];
                if (sc > bv[KC - 1]) topk_insert<KC>(bv, bi, sc, (int)(col0 + j) + p.index_base);
              }
            }
          } else if constexpr (MODE == 2) {
            const int64_t grow = (int64_t)m_tile * BM + row;
            if (grow < p.m_valid) {
              const float b = p.bias ? __ldg(p.bias + grow) : 0.f;
              // the warp's 32 threads own 32 consecutive channels: each store
              // instruction writes 32 consecutive values of one pixel
#pragma unroll
              for (int j = 0; j < 32; ++j) {
                const int64_t col = col0 + j;
                if (col < p.n_valid) {
                  float r = v[j] + b;
                  if (p.relu) r = fmaxf(r, 0.f);
                  p.out16[col * p.ld_out + grow] = __float2bfloat16_rn(r);
                  if (p.out32) p.out32[col * p.ld_out + grow] = r;
                }
              }
            }
          } else {
            const int64_t grow = (int64_t)m_tile * BM + row;
            if (grow < p.m_valid) {
              float* dst = p.C + grow * p.ldc;
#pragma unroll
              for (int j = 0; j < 32; ++j) {
                const int64_t col = col0 + j;
                if (col < p.n_valid) {
                  const float r = p.alpha * v[j];
                  dst[col] = p.accumulate ? dst[col] + r : r;
                }
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(acce_bar(acc));
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1u;
        }
      }
      if constexpr (MODE == 0) {
        if (ok) {
          const int64_t q = (int64_t)m_tile * BM + row;
          const int64_t base = (q * p.part_slots + p.slot_base + split) * KC;
#pragma unroll
          for (int j = 0; j < KC; ++j) {
            p.part_val[base + j] = bv[j];
            p.part_idx[base + j] = bi[j];
          }
        }
      }
    }
    if (!ok && lane == 0) report_timeout(p, abort_flag);
  }

  // Every role has finished. If one gave up, the others may have stopped
  // with work in flight: the producer's last copies (up to STAGES of them;
  // earlier ones were consumed by the MMA thread) and the MMA thread's last
  // MMAs. Wait for both, with the default limit and no abort, before shared
  // memory and TMEM are released.
  __syncthreads();
  if (*abort_flag) {
    volatile int never = 0;
    if (warp == 0 && lane == 0) {
      const int64_t inflight = issued < STAGES ? issued : (int64_t)STAGES;
      uint32_t s = prod_stage, ph = prod_phase;
      for (int64_t i = 0; i < inflight; ++i) {
        if (s == 0) {
          s = STAGES - 1;
          ph ^= 1u;
        } else {
          --s;
        }
        mbar_wait(full_bar(s), ph, &never);
      }
    } else if (warp == 1 && lane == 0 && any_mma) {
      tc_commit(drain_bar);
      mbar_wait(drain_bar, 0, &never);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, T::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// Pair variant of the top-k match (angular ranking, 256-row dictionary
// tiles, non-persistent). The two CTAs of a cluster take two consecutive
// query tiles and the same dictionary range; the even CTA issues
// tcgen05.mma.cta_group::2 with M = 256 (the two query tiles) and N = 256.
// Each CTA stages its own 128 query rows and HALF of each 256-row dictionary
// tile (rows rank * 128 ...), so a CTA moves 32 KB per K step instead of
// 48 KB (the dictionary tile is read once per pair, not once per CTA), and
// each CTA's TMEM receives its 128 query rows x 256 dictionary columns for
// the same top-k epilogue as k_tc_gemm.
//
// Barriers (every wait bounded; per CTA unless noted):
//   full[s]       even CTA: stage s of BOTH CTAs landed. The even CTA's
//                 producer expects both CTAs' bytes; both CTAs' copies
//                 (cp.async.bulk.tensor .cta_group::2) signal this barrier.
//   empty[s]      the even CTA's MMA commit, multicast to both CTAs
//   accf[a]       accumulator a complete: commit multicast to both CTAs
//   acce[a]       even CTA: accumulator a drained, 8 arrivals (4 epilogue
//                 warps x 2 CTAs)
// The MMA thread's waits are CTA-scoped waits on its own barriers. The pair
// ends with a cluster barrier so that neither CTA exits (and frees its
// shared memory or TMEM) while the other may still reach it.
// ---------------------------------------------------------------------------
constexpr int PAIR_STAGES = 6;
constexpr int PAIR_B_BYTES = 128 * BKB;
constexpr int PAIR_STAGE_BYTES = A_BYTES + PAIR_B_BYTES;
constexpr int PAIR_BAR_BYTES = 8 * (2 * PAIR_STAGES + 4 + 1) + 16;
constexpr int PAIR_SMEM_BYTES = 1024 + PAIR_STAGES * PAIR_STAGE_BYTES + SCRATCH_BYTES + PAIR_BAR_BYTES;
constexpr uint32_t PAIR_TMEM_COLS = 512;  // two 128 x 256 FP32 accumulators per CTA
static_assert(PAIR_SMEM_BYTES <= 232448, "shared memory budget");

template <int KIND>
__host__ __device__ constexpr uint32_t make_idesc_pair() {
  // as make_idesc, with M = 256 (both CTAs' query tiles) and N = 256
  return (1u << 4) | (KIND == 0 ? ((1u << 7) | (1u << 10)) : 0u) | ((uint32_t)(256 >> 3) << 17) |
         ((uint32_t)(256 >> 4) << 24);
}

template <int KIND, int KC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    k_tc_gemm_pair(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GemmParams p) {
  constexpr int STAGES = PAIR_STAGES;
  constexpr int STAGE_BYTES = PAIR_STAGE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const uint32_t sbase = smem_u32(smem);
  float* scratch = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES + SCRATCH_BYTES);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
  auto accf_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + a); };
  auto acce_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + 2 + a); };
  const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  // unit of this pair -> (pair of query tiles, dictionary tile range)
  const int u = (int)(blockIdx.x >> 1);
  const int n_splits = p.splits;
  const int pair_tile = u / n_splits;
  const int split = u - pair_tile * n_splits;
  const int m_tile = 2 * pair_tile + (int)rank;
  const int n_begin = (int)((int64_t)split * p.n_tiles / n_splits);
  const int n_end = (int)((int64_t)(split + 1) * p.n_tiles / n_splits);
  const int k_iters = p.k_iters;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(accf_bar(a), 1);
      mbar_init(acce_bar(a), 8);
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) tmem_alloc_pair(smem_u32(tmem_slot), PAIR_TMEM_COLS);
  __syncwarp();
  tc_fence_before();
  // both CTAs' barriers are initialised before any arrival from the peer
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

  const uint64_t wait_ns = p.wait_ns;
  uint32_t prod_stage = 0, prod_phase = 0;
  int64_t issued = 0;
  bool prod_ok = true, any_mma = false;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      const int a_row = m_tile * BM;
      const uint32_t full0 = mapa_shared(full_bar(0), 0);  // the even CTA's full[0]
      for (int n = n_begin; n < n_end && prod_ok; ++n) {
        const int b_row = n * 256 + (int)rank * 128;
        for (int k = 0; k < k_iters; ++k) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag, wait_ns)) {
            prod_ok = false;
            break;
          }
          const uint32_t a_dst = sbase + stage * STAGE_BYTES;
          if (leader) mbar_arrive_expect_tx(full_bar(stage), 2 * STAGE_BYTES);
          const int kx = k * (BKB / kind_elem_bytes<KIND>());
          tma_load_2d_pair(a_dst, &tmA, kx, a_row, full0 + 8u * stage);
          tma_load_2d_pair(a_dst + A_BYTES, &tmB, kx, b_row, full0 + 8u * stage);
          ++issued;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!prod_ok) report_timeout(p, abort_flag);
      prod_stage = stage;
      prod_phase = phase;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      // ---------------- MMA issuer (even CTA) ----------------
      uint32_t stage = 0, phase = 0;
      bool ok = true;
      {
        int acc = 0;
        uint32_t acc_phase = 0;
        constexpr uint32_t idesc = make_idesc_pair<KIND>();
        for (int n = n_begin; n < n_end && ok; ++n) {
          if (!mbar_wait_cluster(acce_bar(acc), acc_phase ^ 1u, abort_flag, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(acc * 256);
          for (int k = 0; k < k_iters; ++k) {
            if (!mbar_wait(full_bar(stage), phase, abort_flag, wait_ns)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_addr = sbase + stage * STAGE_BYTES;
            const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BKB / 32; ++kk) {
              tc_mma_pair<KIND>(d_tmem, smem_desc_sw128(a_addr + kk * 32), smem_desc_sw128(b_addr + kk * 32), idesc,
                                (k | kk) != 0 ? 1u : 0u);
            }
            any_mma = true;
            tc_commit_pair_mc(empty_bar(stage), 0x3);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          tc_commit_pair_mc(accf_bar(acc), 0x3);
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1u;
          }
        }
      }
      if (!ok) report_timeout(p, abort_flag);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (both CTAs) ----------------
    const int wq = warp & 3;
    const int etid = threadIdx.x - 64;
    const int row = wq * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(wq * 32) << 16;
    const uint32_t acce0 = mapa_shared(acce_bar(0), 0);
    float bv[KC];
    int bi[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      bv[j] = -INFINITY;
      bi[j] = -1;
    }
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int n = n_begin; n < n_end; ++n) {
      bool got = mbar_wait_sleep(accf_bar(acc), acc_phase, abort_flag, wait_ns);
      got = __all_sync(0xffffffffu, got);
      if (!got) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int64_t tile_col = (int64_t)n * 256;
#pragma unroll 1
      for (int c = 0; c < 256 / 32; ++c) {
        __syncwarp();
        float v[32];
        tmem_ld32(tmem_base + lane_addr + (uint32_t)(acc * 256 + c * 32), v);
        const int64_t col0 = tile_col + c * 32;
        uint32_t mask = 0;
        const float thr = bv[KC - 1];
        if (col0 + 32 <= p.n_valid) {
          if (p.col_scale) {
            const float4* cs = reinterpret_cast<const float4*>(p.col_scale + col0);
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4) {
              const float4 s4 = __ldg(cs + j4);
              v[4 * j4 + 0] *= s4.x;
              v[4 * j4 + 1] *= s4.y;
              v[4 * j4 + 2] *= s4.z;
              v[4 * j4 + 3] *= s4.w;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const bool valid = col0 + j < p.n_valid;
            const float sc = (valid && p.col_scale) ? __ldg(p.col_scale + col0 + j) : 1.0f;
            v[j] = valid ? v[j] * sc : -INFINITY;
          }
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) mask |= (v[j] > thr) ? (1u << j) : 0u;
        if (mask) {
#pragma unroll
          for (int j = 0; j < 32; ++j) scratch[j * EPI_THREADS + etid] = v[j];
          while (mask) {
            const int j = __ffs(mask) - 1;
            mask &= mask - 1u;
            const float sc = scratch[j * EPI_THREADS + etid];
            if (sc > bv[KC - 1]) topk_insert<KC>(bv, bi, sc, (int)(col0 + j) + p.index_base);
          }
        }
      }
      // this warp's TMEM reads are complete: one arrival per warp on the
      // even CTA's acce[acc]
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(acce0 + 8u * acc);
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1u;
      }
    }
    if (ok && m_tile < p.m_tiles) {
      const int64_t q = (int64_t)m_tile * BM + row;
      const int64_t base = (q * p.part_slots + p.slot_base + split) * KC;
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        p.part_val[base + j] = bv[j];
        p.part_idx[base + j] = bi[j];
      }
    }
    if (!ok && lane == 0) report_timeout(p, abort_flag);
  }

  __syncthreads();
  if (warp == 0 && lane == 0) {
    // On the normal path: wait for the even CTA's last commits to this CTA's
    // empty barriers, so that no arrival reaches this CTA's shared memory
    // after the cluster barrier below. After a give-up: the even CTA waits
    // for the pair's copies still in flight (they all signal its full
    // barriers; a phase whose copies were never all issued ends the drain at
    // the default limit), and the odd CTA, which cannot observe its copies,
    // is held at the cluster barrier until then.
    volatile int never = 0;
    const bool aborted = *abort_flag != 0;
    const int64_t last = issued < STAGES ? issued : (int64_t)STAGES;
    uint32_t s = prod_stage, ph = prod_phase;
    for (int64_t i = 0; i < last && (leader || !aborted); ++i) {
      if (s == 0) {
        s = STAGES - 1;
        ph ^= 1u;
      } else {
        --s;
      }
      if (!mbar_wait(aborted ? full_bar(s) : empty_bar(s), ph, &never)) break;
    }
  } else if (warp == 1 && lane == 0 && leader && any_mma && *abort_flag) {
    tc_commit_pair(drain_bar);
    volatile int never = 0;
    mbar_wait(drain_bar, 0, &never);
  }
  __syncwarp();
  tc_fence_before();
  cluster_sync_all();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, PAIR_TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// Dual variant of the top-k match (angular ranking, 256-row dictionary
// tiles, non-persistent): one CTA takes TWO consecutive query tiles and one
// dictionary range, and every K step issues two M = 128, N = 256 MMAs (one
// per query tile) against the same staged dictionary tile. Per K step a CTA
// stages 64 KB for twice the MMA work of k_tc_gemm's 48 KB, i.e. a third
// less L2 -> SM operand traffic per FLOP, with no operand exchange between
// SMs (which the CTA-pair variant pays for in power).
//   warp 0      TMA producer (A0, A1: 128 rows x 128 B; B: 256 rows x 128 B
//               per stage; 3 stages of 64 KB)
//   warp 1      TMEM (512 columns: query tile h accumulates in columns
//               h * 256 ...) and the MMAs
//   warps 2-9   epilogue: warps 2-5 read query tile 0's accumulator, 6-9
//               tile 1's; each thread owns one query row's top-k
// The two accumulators fill TMEM, so they are single-buffered: the MMAs of
// dictionary tile n + 1 wait until the epilogue has read tile n (the
// epilogue takes about 1 % of a tile's MMA time at 128^2 px).
// ---------------------------------------------------------------------------
constexpr int DUAL_EPI = 256;
constexpr int DUAL_THREADS = 64 + DUAL_EPI;
constexpr int DUAL_STAGES = 3;
constexpr int DUAL_STAGE_BYTES = 2 * A_BYTES + 256 * BKB;
constexpr int DUAL_SCRATCH_BYTES = 32 * DUAL_EPI * 4;
constexpr int DUAL_BAR_BYTES = 8 * (2 * DUAL_STAGES + 2 + 1) + 16;
constexpr int DUAL_SMEM_BYTES = 1024 + DUAL_STAGES * DUAL_STAGE_BYTES + DUAL_SCRATCH_BYTES + DUAL_BAR_BYTES;
static_assert(DUAL_SMEM_BYTES <= 232448, "shared memory budget");

template <int KIND, int KC>
__global__ void __launch_bounds__(DUAL_THREADS, 1)
    k_tc_gemm_dual(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GemmParams p) {
  constexpr int STAGES = DUAL_STAGES;
  constexpr int STAGE_BYTES = DUAL_STAGE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const uint32_t sbase = smem_u32(smem);
  float* scratch = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES + DUAL_SCRATCH_BYTES);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
  const uint32_t accf_bar = bar0 + 8u * (2 * STAGES);
  const uint32_t acce_bar = bar0 + 8u * (2 * STAGES + 1);
  const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 2);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 3);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // unit -> (pair of query tiles, dictionary tile range)
  const int u = (int)blockIdx.x;
  const int n_splits = p.splits;
  const int pair_tile = u / n_splits;
  const int split = u - pair_tile * n_splits;
  const int n_begin = (int)((int64_t)split * p.n_tiles / n_splits);
  const int n_end = (int)((int64_t)(split + 1) * p.n_tiles / n_splits);
  const int k_iters = p.k_iters;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(accf_bar, 1);
    mbar_init(acce_bar, DUAL_EPI);
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) tmem_alloc(smem_u32(tmem_slot), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

  const uint64_t wait_ns = p.wait_ns;
  uint32_t prod_stage = 0, prod_phase = 0;
  int64_t issued = 0;
  bool any_mma = false;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      bool ok = true;
      const int a_row = 2 * pair_tile * BM;
      for (int n = n_begin; n < n_end && ok; ++n) {
        for (int k = 0; k < k_iters; ++k) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag, wait_ns)) {
            ok = false;
            break;
          }
          const uint32_t dst = sbase + stage * STAGE_BYTES;
          mbar_arrive_expect_tx(full_bar(stage), STAGE_BYTES);
          const int kx = k * (BKB / kind_elem_bytes<KIND>());
          tma_load_2d(dst, &tmA, kx, a_row, full_bar(stage));
          tma_load_2d(dst + A_BYTES, &tmA, kx, a_row + BM, full_bar(stage));
          tma_load_2d(dst + 2 * A_BYTES, &tmB, kx, n * 256, full_bar(stage));
          ++issued;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) report_timeout(p, abort_flag);
      prod_stage = stage;
      prod_phase = phase;
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0, acc_phase = 0;
      bool ok = true;
      constexpr uint32_t idesc = make_idesc<KIND, 256>();
      for (int n = n_begin; n < n_end && ok; ++n) {
        if (!mbar_wait(acce_bar, acc_phase ^ 1u, abort_flag, wait_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int k = 0; k < k_iters; ++k) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = sbase + stage * STAGE_BYTES;
          const uint32_t b_addr = a_addr + 2 * A_BYTES;
#pragma unroll
          for (int kk = 0; kk < BKB / 32; ++kk) {
            const uint64_t bdesc = smem_desc_sw128(b_addr + kk * 32);
            const uint32_t accum = (k | kk) != 0 ? 1u : 0u;
            tc_mma<KIND>(tmem_base, smem_desc_sw128(a_addr + kk * 32), bdesc, idesc, accum);
            tc_mma<KIND>(tmem_base + 256u, smem_desc_sw128(a_addr + A_BYTES + kk * 32), bdesc, idesc, accum);
          }
          any_mma = true;
          tc_commit(empty_bar(stage));
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        tc_commit(accf_bar);
        acc_phase ^= 1u;
      }
      if (!ok) report_timeout(p, abort_flag);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue ----------------
    const int h = (warp - 2) >> 2;        // query tile of the pair
    const int wq = warp & 3;              // TMEM lane quarter this warp may access
    const int etid = threadIdx.x - 64;    // 0..255, scratch column
    const int row = wq * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(wq * 32) << 16;
    const int m_tile = 2 * pair_tile + h;
    float bv[KC];
    int bi[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      bv[j] = -INFINITY;
      bi[j] = -1;
    }
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int n = n_begin; n < n_end; ++n) {
      bool got = mbar_wait_sleep(accf_bar, acc_phase, abort_flag, wait_ns);
      got = __all_sync(0xffffffffu, got);
      if (!got) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int64_t tile_col = (int64_t)n * 256;
#pragma unroll 1
      for (int c = 0; c < 256 / 32; ++c) {
        __syncwarp();
        float v[32];
        tmem_ld32(tmem_base + lane_addr + (uint32_t)(h * 256 + c * 32), v);
        const int64_t col0 = tile_col + c * 32;
        uint32_t mask = 0;
        const float thr = bv[KC - 1];
        if (col0 + 32 <= p.n_valid) {
          if (p.col_scale) {
            const float4* cs = reinterpret_cast<const float4*>(p.col_scale + col0);
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4) {
              const float4 s4 = __ldg(cs + j4);
              v[4 * j4 + 0] *= s4.x;
              v[4 * j4 + 1] *= s4.y;
              v[4 * j4 + 2] *= s4.z;
              v[4 * j4 + 3] *= s4.w;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const bool valid = col0 + j < p.n_valid;
            const float sc = (valid && p.col_scale) ? __ldg(p.col_scale + col0 + j) : 1.0f;
            v[j] = valid ? v[j] * sc : -INFINITY;
          }
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) mask |= (v[j] > thr) ? (1u << j) : 0u;
        if (mask) {
#pragma unroll
          for (int j = 0; j < 32; ++j) scratch[j * DUAL_EPI + etid] = v[j];
          while (mask) {
            const int j = __ffs(mask) - 1;
            mask &= mask - 1u;
            const float sc = scratch[j * DUAL_EPI + etid];
            if (sc > bv[KC - 1]) topk_insert<KC>(bv, bi, sc, (int)(col0 + j) + p.index_base);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acce_bar);
      acc_phase ^= 1u;
    }
    if (ok && m_tile < p.m_tiles) {
      const int64_t q = (int64_t)m_tile * BM + row;
      const int64_t base = (q * p.part_slots + p.slot_base + split) * KC;
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        p.part_val[base + j] = bv[j];
        p.part_idx[base + j] = bi[j];
      }
    }
    if (!ok && lane == 0) report_timeout(p, abort_flag);
  }

  // As in k_tc_gemm: after a give-up, let this CTA's copies and MMAs finish
  // before shared memory and TMEM are released.
  __syncthreads();
  if (*abort_flag) {
    volatile int never = 0;
    if (warp == 0 && lane == 0) {
      const int64_t inflight = issued < STAGES ? issued : (int64_t)STAGES;
      uint32_t s = prod_stage, ph = prod_phase;
      for (int64_t i = 0; i < inflight; ++i) {
        if (s == 0) {
          s = STAGES - 1;
          ph ^= 1u;
        } else {
          --s;
        }
        mbar_wait(full_bar(s), ph, &never);
      }
    } else if (warp == 1 && lane == 0 && any_mma) {
      tc_commit(drain_bar);
      mbar_wait(drain_bar, 0, &never);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Wait limit handed to every tensor-core kernel launch (0 = kWaitLimitNs).
static std::atomic<uint64_t> g_wait_limit_ns{0};

uint64_t wait_limit_ns() {
  const uint64_t v = g_wait_limit_ns.load(std::memory_order_relaxed);
  return v ? v : kWaitLimitNs;
}

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  });
  return fn;
}

static int make_tmap(CUtensorMap* map, const void* ptr, int lp_dtype, int64_t rows, int64_t k_pad,
                     int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is unavailable from the CUDA driver");
    return EBSD_ERR_UNSUPPORTED;
  }
  const int esz = lp_dtype == EBSD_DT_BF16 ? 2 : 1;
  cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(k_pad * esz)};
  cuuint32_t box[2] = {(cuuint32_t)(BKB / esz), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map,
                   lp_dtype == EBSD_DT_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                            : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                   2, const_cast<void*>(ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (CUresult %d) for rows=%lld k=%lld", (int)r,
              (long long)rows, (long long)k_pad);
    return EBSD_ERR_ARG;
  }
  return 0;
}

// FP32 rows (ld floats apart) of `rows` x `k` valid elements, read as TF32
// (the copy rounds each element to TF32); reads past either extent return
// zeros, so the operands need no padding.
static int make_tmap_f32(CUtensorMap* map, const float* ptr, int64_t ld, int64_t rows, int64_t k, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is unavailable from the CUDA driver");
    return EBSD_ERR_UNSUPPORTED;
  }
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 4)};
  cuuint32_t box[2] = {(cuuint32_t)(BKB / 4), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32, 2, const_cast<float*>(ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (CUresult %d) for FP32 rows=%lld k=%lld ld=%lld", (int)r,
              (long long)rows, (long long)k, (long long)ld);
    return EBSD_ERR_ARG;
  }
  return 0;
}

template <int KIND, int MODE, int KC, int BN, bool PERSIST = false, bool BIAS = false>
static int launch(const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p_in, int grid,
                  cudaStream_t s) {
  auto kern = k_tc_gemm<KIND, MODE, KC, BN, PERSIST, BIAS>;
  constexpr int smem = Tile<BN>::SMEM_BYTES;
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  GemmParams p = p_in;
  p.wait_ns = wait_limit_ns();
  kern<<<grid, THREADS, smem, s>>>(a, b, p);
  EBSD_LAUNCH_CHECK();
  return 0;
}

template <int KIND, int KC>
static int launch_pair_kc(const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p_in, int grid,
                          cudaStream_t s) {
  auto kern = k_tc_gemm_pair<KIND, KC>;
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM_BYTES));
  GemmParams p = p_in;
  p.wait_ns = wait_limit_ns();
  kern<<<grid, THREADS, PAIR_SMEM_BYTES, s>>>(a, b, p);
  EBSD_LAUNCH_CHECK();
  return 0;
}

template <int KIND>
static int launch_pair(int kc, const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p, int grid,
                       cudaStream_t s) {
  switch (kc) {
    case 1: return launch_pair_kc<KIND, 1>(a, b, p, grid, s);
    case 2: return launch_pair_kc<KIND, 2>(a, b, p, grid, s);
    case 4: return launch_pair_kc<KIND, 4>(a, b, p, grid, s);
    case 8: return launch_pair_kc<KIND, 8>(a, b, p, grid, s);
    case 16: return launch_pair_kc<KIND, 16>(a, b, p, grid, s);
    case 32: return launch_pair_kc<KIND, 32>(a, b, p, grid, s);
    case 64: return launch_pair_kc<KIND, 64>(a, b, p, grid, s);
  }
  set_error("n_cand %d not in {1,2,4,8,16,32,64}", kc);
  return EBSD_ERR_ARG;
}

// Whether eligible top-k matches run as CTA pairs (ebsd_set_match_pairs).
static std::atomic<int> g_match_pairs{0};

template <int KIND, int KC>
static int launch_dual_kc(const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p_in, int grid,
                          cudaStream_t s) {
  auto kern = k_tc_gemm_dual<KIND, KC>;
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, DUAL_SMEM_BYTES));
  GemmParams p = p_in;
  p.wait_ns = wait_limit_ns();
  kern<<<grid, DUAL_THREADS, DUAL_SMEM_BYTES, s>>>(a, b, p);
  EBSD_LAUNCH_CHECK();
  return 0;
}

template <int KIND>
static int launch_dual(int kc, const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p, int grid,
                       cudaStream_t s) {
  switch (kc) {
    case 1: return launch_dual_kc<KIND, 1>(a, b, p, grid, s);
    case 2: return launch_dual_kc<KIND, 2>(a, b, p, grid, s);
    case 4: return launch_dual_kc<KIND, 4>(a, b, p, grid, s);
    case 8: return launch_dual_kc<KIND, 8>(a, b, p, grid, s);
    case 16: return launch_dual_kc<KIND, 16>(a, b, p, grid, s);
    case 32: return launch_dual_kc<KIND, 32>(a, b, p, grid, s);
    case 64: return launch_dual_kc<KIND, 64>(a, b, p, grid, s);
  }
  set_error("n_cand %d not in {1,2,4,8,16,32,64}", kc);
  return EBSD_ERR_ARG;
}

// Which eligible top-k matches take two query tiles per CTA
// (ebsd_set_match_dual): 0 none, 1 all, 2 those of e4m3 rows (default).
// Measured on a B200 under the 1 kW power cap (full bench, two alternating
// pairs of runs): e4m3 190,500 vs 182,000 patterns/s; bf16 within the noise
// (about 8 % more work per clock, about 8 % less clock).
static std::atomic<int> g_match_dual{2};

// The variant an eligible launch (256-row tiles, angular ranking, not
// persistent) of m_tiles query tiles of lp_dtype rows runs: 1 CTA pairs, 2
// two query tiles per CTA, 0 the one-tile kernel (always for an odd tile
// count).
static int match_variant(int64_t m_tiles, int lp_dtype) {
  if (m_tiles % 2) return 0;
  if (g_match_pairs.load(std::memory_order_relaxed)) return 1;
  const int dual = g_match_dual.load(std::memory_order_relaxed);
  if (dual == 1 || (dual == 2 && lp_dtype == EBSD_DT_E4M3)) return 2;
  return 0;
}

template <int KIND, int BN, bool PERSIST, bool BIAS = false>
static int launch_topk(int kc, const CUtensorMap& a, const CUtensorMap& b, const GemmParams& p,
                       int grid, cudaStream_t s) {
  switch (kc) {
    case 1: return launch<KIND, 0, 1, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 2: return launch<KIND, 0, 2, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 4: return launch<KIND, 0, 4, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 8: return launch<KIND, 0, 8, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 16: return launch<KIND, 0, 16, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 32: return launch<KIND, 0, 32, BN, PERSIST, BIAS>(a, b, p, grid, s);
    case 64: return launch<KIND, 0, 64, BN, PERSIST, BIAS>(a, b, p, grid, s);
  }
  set_error("n_cand %d not in {1,2,4,8,16,32,64}", kc);
  return EBSD_ERR_ARG;
}

template <int KIND>
static int launch_topk_shape(int kc, int tile_n, bool persist, const CUtensorMap& a, const CUtensorMap& b,
                             const GemmParams& p, int grid, cudaStream_t s) {
  if (p.col_bias) {
    // the euclidean variant exists for the default launch shape only
    EBSD_ARG_CHECK(tile_n == 256 && !persist, "col_bias needs 256-row tiles and a non-persistent launch");
    return launch_topk<KIND, 256, false, true>(kc, a, b, p, grid, s);
  }
  if (tile_n == 128)
    return persist ? launch_topk<KIND, 128, true>(kc, a, b, p, grid, s)
                   : launch_topk<KIND, 128, false>(kc, a, b, p, grid, s);
  return persist ? launch_topk<KIND, 256, true>(kc, a, b, p, grid, s)
                 : launch_topk<KIND, 256, false>(kc, a, b, p, grid, s);
}

static int check_operands(const void* A, int64_t m_pad, const void* B, int64_t n_pad, int64_t k_pad,
                          int lp_dtype, int* status, int BN = 256) {
  EBSD_ARG_CHECK(A && B && status, "null operand or status pointer");
  EBSD_ARG_CHECK(lp_dtype == EBSD_DT_BF16 || lp_dtype == EBSD_DT_E4M3,
                 "lp_dtype must be EBSD_DT_BF16 or EBSD_DT_E4M3");
  const int kmul = lp_dtype == EBSD_DT_BF16 ? 64 : 128;
  EBSD_ARG_CHECK(k_pad > 0 && k_pad % kmul == 0, "k_pad %lld must be a positive multiple of %d",
                 (long long)k_pad, kmul);
  EBSD_ARG_CHECK(m_pad > 0 && m_pad % BM == 0, "row count %lld must be a positive multiple of %d",
                 (long long)m_pad, BM);
  EBSD_ARG_CHECK(n_pad > 0 && n_pad % BN == 0, "row count %lld must be a positive multiple of %d",
                 (long long)n_pad, BN);
  EBSD_ARG_CHECK(((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0,
                 "operands must be 16-byte aligned");
  EBSD_ARG_CHECK(m_pad / BM < (1 << 20) && n_pad / BN < (1 << 22), "operand too large");
  return 0;
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int64_t ebsd_set_wait_limit_ns(int64_t ns) {
  const uint64_t prev = g_wait_limit_ns.exchange(ns > 0 ? (uint64_t)ns : 0u);
  return prev ? (int64_t)prev : (int64_t)kWaitLimitNs;
}

extern "C" int ebsd_set_match_pairs(int on) {
  if (on < 0) return g_match_pairs.load();
  return g_match_pairs.exchange(on ? 1 : 0);
}

extern "C" int ebsd_set_match_dual(int mode) {
  if (mode < 0) return g_match_dual.load();
  return g_match_dual.exchange(mode == 0 ? 0 : mode == 2 ? 2 : 1);
}

extern "C" int ebsd_match_pair_max_clusters(void) {
  // every instantiation has the same block, cluster and shared-memory size
  auto kern = k_tc_gemm_pair<0, 32>;
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM_BYTES));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * 1024);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = PAIR_SMEM_BYTES;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = 2;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  EBSD_CUDA_CHECK(cudaOccupancyMaxActiveClusters(&n, kern, &cfg));
  return n;
}

extern "C" int ebsd_match_auto_splits_typed(int64_t n_queries_pad, int64_t n_dict_pad, int lp_dtype) {
  // One wave: query tiles x dictionary ranges ~= number of SMs, so all units
  // start and finish together. Measured on B200 at 128^2 px x 328,720 rows:
  // one-wave shapes with 16-37 query tiles x 4-9 ranges run at ~1.26 PFLOP/s
  // and ~1.3 GHz under the power cap (18 x 8 fastest: its query tiles stay
  // in L2); multi-wave or 1-range shapes that keep many more operand tiles in
  // flight settle at 0.68-1.1 PFLOP/s.
  // (with two query tiles per CTA, the CTAs of a range are half as many)
  const int64_t m_tiles = std::max<int64_t>(1, n_queries_pad / BM);
  const int64_t n_tiles = std::max<int64_t>(1, n_dict_pad / 256);
  const int64_t sms = device_sm_count();
  const int64_t ctas_per_range = match_variant(m_tiles, lp_dtype) == 2 ? m_tiles / 2 : m_tiles;
  int64_t splits = std::max<int64_t>(1, sms / ctas_per_range);
  splits = std::min(splits, n_tiles);
  return (int)splits;
}

extern "C" int ebsd_match_auto_splits(int64_t n_queries_pad, int64_t n_dict_pad) {
  return ebsd_match_auto_splits_typed(n_queries_pad, n_dict_pad, EBSD_DT_BF16);
}

extern "C" int ebsd_match_topk_tiled(const void* queries_lp, int64_t n_queries_pad, const void* dict_lp,
                                     int64_t n_dict_pad, int64_t n_dict_valid, int64_t k_pad, int lp_dtype,
                                     const float* col_scale, const float* col_bias, const float* row_scale,
                                     int n_cand, int splits, float* part_val,
                                     int32_t* part_idx, int part_slots, int slot_base, int32_t index_base,
                                     int tile_n, int max_ctas, int* d_status, void* stream) {
  if (tile_n == 0) tile_n = 256;
  EBSD_ARG_CHECK(tile_n == 128 || tile_n == 256, "tile_n must be 128 or 256");
  if (int rc = check_operands(queries_lp, n_queries_pad, dict_lp, n_dict_pad, k_pad, lp_dtype, d_status, tile_n))
    return rc;
  EBSD_ARG_CHECK(part_val && part_idx, "null partial-result buffers");
  EBSD_ARG_CHECK(n_dict_valid > 0 && n_dict_valid <= n_dict_pad, "n_dict_valid out of range");
  EBSD_ARG_CHECK((int64_t)index_base + n_dict_valid <= INT32_MAX, "dictionary index overflow");
  EBSD_ARG_CHECK(!col_scale || ((uintptr_t)col_scale & 15) == 0, "col_scale must be 16-byte aligned");
  EBSD_ARG_CHECK(!col_bias || ((uintptr_t)col_bias & 15) == 0, "col_bias must be 16-byte aligned");
  EBSD_ARG_CHECK(!col_bias == !row_scale, "col_bias and row_scale must be given together");
  const int n_tiles = (int)(n_dict_pad / tile_n);
  if (splits <= 0) splits = ebsd_match_auto_splits_typed(n_queries_pad, n_dict_pad, lp_dtype);
  splits = std::min(splits, n_tiles);
  EBSD_ARG_CHECK(slot_base >= 0 && slot_base + splits <= part_slots,
                 "part_slots (%d) < slot_base (%d) + splits (%d)", part_slots, slot_base, splits);
  const int64_t m_tiles = n_queries_pad / BM;
  EBSD_ARG_CHECK(m_tiles * splits < INT32_MAX, "too many work units");
  // max_ctas > 0 and fewer CTAs than units: persistent launch, each CTA
  // loops over its units. Otherwise, with pairs switched on, 256-row tiles,
  // the angular ranking and an even number of query tiles, one cluster of
  // two CTAs takes two query tiles and a dictionary range.
  const bool persist = max_ctas > 0 && max_ctas < m_tiles * splits;
  const int variant = (!persist && tile_n == 256 && !col_bias) ? match_variant(m_tiles, lp_dtype) : 0;
  const bool pair = variant == 1;
  CUtensorMap ta, tb;
  if (int rc = make_tmap(&ta, queries_lp, lp_dtype, n_queries_pad, k_pad, BM)) return rc;
  if (int rc = make_tmap(&tb, dict_lp, lp_dtype, n_dict_pad, k_pad, pair ? tile_n / 2 : tile_n)) return rc;
  GemmParams p{};
  p.m_tiles = (int)m_tiles;
  p.n_tiles = n_tiles;
  p.splits = splits;
  p.units = (int)(m_tiles * splits);
  p.k_iters = (int)(k_pad * (lp_dtype == EBSD_DT_BF16 ? 2 : 1) / BKB);
  p.n_valid = n_dict_valid;
  p.col_scale = col_scale;
  p.col_bias = col_bias;
  p.row_scale = row_scale;
  p.part_val = part_val;
  p.part_idx = part_idx;
  p.part_slots = part_slots;
  p.slot_base = slot_base;
  p.index_base = index_base;
  p.status = d_status;
  cudaStream_t s = as_stream(stream);
  if (pair) {
    p.units = (int)(m_tiles / 2 * splits);
    return lp_dtype == EBSD_DT_BF16 ? launch_pair<0>(n_cand, ta, tb, p, 2 * p.units, s)
                                    : launch_pair<1>(n_cand, ta, tb, p, 2 * p.units, s);
  }
  if (variant == 2) {
    p.units = (int)(m_tiles / 2 * splits);
    return lp_dtype == EBSD_DT_BF16 ? launch_dual<0>(n_cand, ta, tb, p, p.units, s)
                                    : launch_dual<1>(n_cand, ta, tb, p, p.units, s);
  }
  const int grid = persist ? max_ctas : p.units;
  return lp_dtype == EBSD_DT_BF16 ? launch_topk_shape<0>(n_cand, tile_n, persist, ta, tb, p, grid, s)
                                  : launch_topk_shape<1>(n_cand, tile_n, persist, ta, tb, p, grid, s);
}

extern "C" int ebsd_match_topk(const void* queries_lp, int64_t n_queries_pad, const void* dict_lp,
                               int64_t n_dict_pad, int64_t n_dict_valid, int64_t k_pad,
                               int lp_dtype, const float* col_scale, int n_cand, int splits,
                               float* part_val, int32_t* part_idx, int part_slots, int slot_base,
                               int32_t index_base, int* d_status, void* stream) {
  if (splits > 0 && n_dict_pad >= 256)
    EBSD_ARG_CHECK(splits <= n_dict_pad / 256, "splits (%d) > dictionary tiles (%lld)", splits,
                   (long long)(n_dict_pad / 256));
  return ebsd_match_topk_tiled(queries_lp, n_queries_pad, dict_lp, n_dict_pad, n_dict_valid, k_pad, lp_dtype,
                               col_scale, nullptr, nullptr, n_cand, splits, part_val, part_idx, part_slots, slot_base,
                               index_base, 256, 0, d_status, stream);
}

extern "C" int ebsd_gemm_nt(const void* A, int64_t m_pad, const void* B, int64_t n_pad, int64_t k_pad,
                            int lp_dtype, float alpha, int accumulate, float* C, int64_t ldc, int64_t m_valid,
                            int64_t n_valid, int splits, int* d_status, void* stream) {
  if (int rc = check_operands(A, m_pad, B, n_pad, k_pad, lp_dtype, d_status)) return rc;
  EBSD_ARG_CHECK(C != nullptr, "null output");
  EBSD_ARG_CHECK(m_valid > 0 && m_valid <= m_pad && n_valid > 0 && n_valid <= n_pad,
                 "valid extents out of range");
  EBSD_ARG_CHECK(ldc >= n_valid, "ldc < n_valid");
  CUtensorMap ta, tb;
  if (int rc = make_tmap(&ta, A, lp_dtype, m_pad, k_pad, BM)) return rc;
  if (int rc = make_tmap(&tb, B, lp_dtype, n_pad, k_pad, 256)) return rc;
  GemmParams p{};
  p.n_tiles = (int)(n_pad / 256);
  // splits <= 0: one B tile per unit; otherwise each unit streams a range of
  // n_tiles / splits B tiles (amortises CTA set-up when K is short)
  p.splits = splits <= 0 ? p.n_tiles : std::min(splits, p.n_tiles);
  p.k_iters = (int)(k_pad * (lp_dtype == EBSD_DT_BF16 ? 2 : 1) / BKB);
  p.n_valid = n_valid;
  p.C = C;
  p.ldc = ldc;
  p.m_valid = m_valid;
  p.alpha = alpha;
  p.accumulate = accumulate;
  p.status = d_status;
  const int64_t m_tiles = m_pad / BM;
  EBSD_ARG_CHECK(m_tiles * p.splits < INT32_MAX, "too many work units");
  p.units = (int)(m_tiles * p.splits);
  cudaStream_t s = as_stream(stream);
  return lp_dtype == EBSD_DT_BF16 ? launch<0, 1, 1, 256>(ta, tb, p, p.units, s)
                                  : launch<1, 1, 1, 256>(ta, tb, p, p.units, s);
}

extern "C" int ebsd_gemm_f32(const float* A, int64_t lda, int64_t m, const float* B, int64_t ldb, int64_t n,
                             int64_t k, float alpha, int accumulate, float* C, int64_t ldc, int splits, int* d_status,
                             void* stream) {
  EBSD_ARG_CHECK(A && B && C && d_status, "ebsd_gemm_f32: null pointer");
  EBSD_ARG_CHECK(m > 0 && n > 0 && k > 0, "empty product");
  EBSD_ARG_CHECK(lda >= k && ldb >= k && ldc >= n, "leading dimensions smaller than the extents");
  EBSD_ARG_CHECK(lda % 4 == 0 && ldb % 4 == 0, "lda and ldb must be multiples of 4 floats (16-byte rows)");
  EBSD_ARG_CHECK(((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0, "operands must be 16-byte aligned");
  const int64_t m_tiles = (m + BM - 1) / BM, n_tiles = (n + 255) / 256;
  EBSD_ARG_CHECK(m_tiles < (1 << 20) && n_tiles < (1 << 22), "operand too large");
  CUtensorMap ta, tb;
  if (int rc = make_tmap_f32(&ta, A, lda, m, k, BM)) return rc;
  if (int rc = make_tmap_f32(&tb, B, ldb, n, k, 256)) return rc;
  GemmParams p{};
  p.n_tiles = (int)n_tiles;
  p.splits = splits <= 0 ? p.n_tiles : std::min<int>(splits, p.n_tiles);
  p.k_iters = (int)((k + BKB / 4 - 1) / (BKB / 4));
  p.n_valid = n;
  p.C = C;
  p.ldc = ldc;
  p.m_valid = m;
  p.alpha = alpha;
  p.accumulate = accumulate;
  p.status = d_status;
  EBSD_ARG_CHECK(m_tiles * p.splits < INT32_MAX, "too many work units");
  p.units = (int)(m_tiles * p.splits);
  return launch<2, 1, 1, 256>(ta, tb, p, p.units, as_stream(stream));
}

extern "C" int ebsd_cnn_conv_fwd(const void* w16, int64_t cout_pad, const void* cols, int64_t rows_pad,
                                 int64_t k_pad, const float* bias, int cout, int64_t n_rows, int relu, void* out16,
                                 int64_t ld_out, float* out32, int splits, int* d_status, void* stream) {
  if (int rc = check_operands(w16, cout_pad, cols, rows_pad, k_pad, EBSD_DT_BF16, d_status)) return rc;
  EBSD_ARG_CHECK(out16 != nullptr, "null output");
  EBSD_ARG_CHECK(cout > 0 && cout <= cout_pad && n_rows > 0 && n_rows <= rows_pad, "valid extents out of range");
  EBSD_ARG_CHECK(ld_out >= cout, "ld_out < cout");
  CUtensorMap ta, tb;
  if (int rc = make_tmap(&ta, w16, EBSD_DT_BF16, cout_pad, k_pad, BM)) return rc;
  if (int rc = make_tmap(&tb, cols, EBSD_DT_BF16, rows_pad, k_pad, 256)) return rc;
  GemmParams p{};
  p.n_tiles = (int)(rows_pad / 256);
  p.splits = splits <= 0 ? p.n_tiles : std::min(splits, p.n_tiles);
  p.k_iters = (int)(k_pad * 2 / BKB);
  p.n_valid = n_rows;
  p.m_valid = cout;
  p.bias = bias;
  p.out16 = reinterpret_cast<__nv_bfloat16*>(out16);
  p.out32 = out32;
  p.ld_out = ld_out;
  p.relu = relu;
  p.status = d_status;
  const int64_t m_tiles = cout_pad / BM;
  EBSD_ARG_CHECK(m_tiles * p.splits < INT32_MAX, "too many work units");
  p.units = (int)(m_tiles * p.splits);
  return launch<0, 2, 1, 256>(ta, tb, p, p.units, as_stream(stream));
}
