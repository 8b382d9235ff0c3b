// Shared definitions for the ebsd_b200 C-ABI library (sm_100a only).
//
// Status convention of every exported entry point:
//   0   success
//   >0  argument error (EBSD_ERR_*), nothing was launched
//   <0  CUDA error: -(cudaError_t) of the failing call
// The human-readable message of the last failure on the calling host thread
// is available through ebsd_last_error().
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "../../include/ebsd_b200.h"

namespace ebsd {

void set_error(const char* fmt, ...);
// Limit of the bounded waits of the next tensor-core kernel launches
// (ebsd_set_wait_limit_ns; kWaitLimitNs by default).
uint64_t wait_limit_ns();

// Debug checks. In the checking build (-DEBSD_CHECK: `python -m
// ebsdtorch_b200.build --check`, loaded when EBSD_CHECK_BUILD=1) a failed
// EBSD_DCHECK(cond) records its source line in this translation unit's
// device word (the first failure wins) and evaluates to false, so the caller
// skips the access; ebsd_debug_check_line() reads and clears the words of
// every translation unit. In the normal build the checks compile away.
int register_check_word(const void* symbol, const char* file);
#ifdef EBSD_CHECK
static __device__ int g_check_line;
static const int g_check_registered = register_check_word(&g_check_line, __FILE__);
#define EBSD_DCHECK(cond) ((cond) ? true : (atomicCAS(&::ebsd::g_check_line, 0, __LINE__), false))
#else
#define EBSD_DCHECK(cond) true
#endif

#define EBSD_ARG_CHECK(cond, ...)              \
  do {                                         \
    if (!(cond)) {                             \
      ::ebsd::set_error(__VA_ARGS__);          \
      return EBSD_ERR_ARG;                     \
    }                                          \
  } while (0)

#define EBSD_CUDA_CHECK(call)                                                      \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      ::ebsd::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                        __FILE__, __LINE__);                                       \
      return -(int)e_;                                                             \
    }                                                                              \
  } while (0)

#define EBSD_LAUNCH_CHECK() EBSD_CUDA_CHECK(cudaGetLastError())

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

int device_sm_count();

// ---------------------------------------------------------------------------
// Laue groups (host): rotation operators as unit quaternions, w >= 0
// ---------------------------------------------------------------------------

struct LaueTable {
  float q[24 * 4];
  int n;
};

// Rotation operators of each Laue group as closed sets of unit quaternions
// (the groups of laue_generators.py:54-249), generated on the host.
static inline void laue_qmul_d(const double* a, const double* b, double* o) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

static inline int build_laue_table(int laue, LaueTable* t) {
  auto rot = [](double x, double y, double z, double deg, double* q) {
    const double n = std::sqrt(x * x + y * y + z * z), h = deg * M_PI / 360.0;
    q[0] = std::cos(h);
    q[1] = std::sin(h) * x / n;
    q[2] = std::sin(h) * y / n;
    q[3] = std::sin(h) * z / n;
  };
  double g[3][4];
  int ng = 0;
  const int ax[11][3] = {{0, 0, 0}, {1, 0, 0}, {1, 4, 0}, {2, 0, 0}, {2, 4, 0}, {3, 0, 0},
                         {3, 4, 0}, {5, 0, 0}, {5, 4, 0}, {1, 4, 6}, {2, 4, 6}};
  // generator codes: 1 z2, 2 z4, 3 z3, 5 z6, 4 x2, 6 <111> 3-fold
  for (int j = 0; j < 3; ++j) {
    const int c = ax[laue - 1][j];
    if (c == 0) continue;
    switch (c) {
      case 1: rot(0, 0, 1, 180, g[ng]); break;
      case 2: rot(0, 0, 1, 90, g[ng]); break;
      case 3: rot(0, 0, 1, 120, g[ng]); break;
      case 5: rot(0, 0, 1, 60, g[ng]); break;
      case 4: rot(1, 0, 0, 180, g[ng]); break;
      case 6: rot(1, 1, 1, 120, g[ng]); break;
    }
    ++ng;
  }
  double el[24][4] = {{1, 0, 0, 0}};
  int n = 1;
  bool grew = true;
  while (grew) {
    grew = false;
    const int cur = n;
    for (int i = 0; i < cur; ++i)
      for (int k = 0; k < ng; ++k) {
        double c[4];
        laue_qmul_d(el[i], g[k], c);
        if (c[0] < 0)
          for (double& v : c) v = -v;
        bool known = false;
        for (int e = 0; e < n && !known; ++e)
          known = std::fabs(std::fabs(c[0] * el[e][0] + c[1] * el[e][1] + c[2] * el[e][2] + c[3] * el[e][3]) -
                            1.0) < 1e-9;
        if (!known && n < 24) {
          for (int d = 0; d < 4; ++d) el[n][d] = c[d];
          ++n;
          grew = true;
        }
      }
  }
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 4; ++d) t->q[4 * i + d] = (float)el[i][d];
  t->n = n;
  return n;
}



// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Default upper bound on any spin-wait inside a kernel (kernels take the
// limit as a parameter; ebsd_set_wait_limit_ns changes it). A wait that
// exceeds it sets the caller's status word to EBSD_DEVICE_TIMEOUT and the
// kernel unwinds. Waits for a CTA's own copies and MMAs before it exits
// always use this default.
constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Dots of a shared-memory FP32 row with R FP32 rows of n4 float4 chunks
// (16-byte aligned); every lane keeps R independent 16-byte loads in flight.
// All lanes get the sums.
template <int R>
__device__ __forceinline__ void f32_dot_rows(const float* qrow, const float* const (&d)[R], int n4, int lane,
                                             float (&acc)[R]) {
#pragma unroll
  for (int j = 0; j < R; ++j) acc[j] = 0.f;
  const float4* q4 = reinterpret_cast<const float4*>(qrow);
  for (int v = lane; v < n4; v += 32) {
    float4 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = __ldg(reinterpret_cast<const float4*>(d[j]) + v);
    const float4 y = q4[v];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      acc[j] = fmaf(x[j].x, y.x, acc[j]);
      acc[j] = fmaf(x[j].y, y.y, acc[j]);
      acc[j] = fmaf(x[j].z, y.z, acc[j]);
      acc[j] = fmaf(x[j].w, y.w, acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < R; ++j) acc[j] = warp_sum(acc[j]);
}

// Block-wide sum; `red` must hold one slot per warp. All threads get the sum.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  T t = (lane < nw) ? red[lane] : T(0);
  if (wid == 0) {
    t = warp_sum(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  T r = red[0];
  return r;
}

__device__ __forceinline__ float block_max(float v, float* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  float t = (lane < nw) ? red[lane] : -INFINITY;
  if (wid == 0) {
    t = warp_max(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

// ---------------------------------------------------------------------------
// mbarrier / TMA / tcgen05 wrappers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait that suspends the thread for at most about hint_ns (the
// instruction's suspend-time hint) before it reports "not yet".
__device__ __forceinline__ bool mbar_try_wait_hint(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Wait under a limit shorter than the default (a caller-set watchdog): no
// spin phase, and every try_wait suspends for at most 200 ns, so the limit
// is checked at least every 200 ns whatever the hardware's own suspend time.
// Only the epilogue's waits (mbar_wait_sleep) take this path: it gives up
// first, and the producer and MMA threads then stop on the abort flag, so
// their latency-critical waits keep the plain form below.
static __device__ __noinline__ bool mbar_wait_short(uint32_t bar, uint32_t parity, volatile int* abort,
                                             uint64_t limit_ns) {
  const uint64_t t0 = globaltimer_ns();
#pragma unroll 1
  while (true) {
    if (mbar_try_wait_hint(bar, parity, 200u)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// Bounded wait on an mbarrier phase. Returns false when the wait limit
// (limit_ns, counted after a short spin) expired or when *abort became
// non-zero (another role gave up).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort,
                                          uint64_t limit_ns = kWaitLimitNs) {
#pragma unroll 1
  for (int i = 0; i < 256; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
#pragma unroll 1
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// As mbar_wait, for waits expected to last many microseconds (the epilogue
// waiting for a whole accumulator): after a short spin the thread sleeps
// between polls instead of issuing back-to-back try_waits.
__device__ __forceinline__ bool mbar_wait_sleep(uint32_t bar, uint32_t parity, volatile int* abort,
                                                uint64_t limit_ns = kWaitLimitNs) {
  if (limit_ns < kWaitLimitNs) return mbar_wait_short(bar, parity, abort, limit_ns);
#pragma unroll 1
  for (int i = 0; i < 32; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
#pragma unroll 1
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limit_ns) return false;
    __nanosleep(500);
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// 2-D tiled TMA load global -> shared, completion signalled on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Whole warp: allocate `ncols` TMEM columns, base address written to smem.
__device__ __forceinline__ void tmem_alloc(uint32_t smem_slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_slot),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one instruction, issued by one thread.
template <int KIND>  // 0: kind::f16 (bf16/f16 inputs), 1: kind::f8f6f4, 2: kind::tf32
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (KIND == 2) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}

// Arrive once on `bar` when all previously issued tcgen05 ops of this thread
// have completed.
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

// ---- CTA pairs (clusters of two CTAs sharing one tcgen05.mma.cta_group::2)
// Rank of this CTA in its cluster.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Shared::cluster address of the same shared-memory offset in CTA `rank`.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
// Arrive (release at cluster scope) on an mbarrier of any CTA in the cluster.
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// try_wait with acquire at cluster scope (for phases completed by arrivals
// from the peer CTA).
__device__ __forceinline__ bool mbar_try_wait_cluster(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// As mbar_wait, with cluster-scope acquire.
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity, volatile int* abort,
                                                  uint64_t limit_ns = kWaitLimitNs) {
#pragma unroll 1
  for (int i = 0; i < 256; ++i)
    if (mbar_try_wait_cluster(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
#pragma unroll 1
  while (true) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}
// 2-D tiled TMA load into this CTA's shared memory (dst) whose completion
// (complete_tx) is signalled on an mbarrier of either CTA of the pair
// (bar_cluster: a shared::cluster address, e.g. from mapa_shared).
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
      : "memory");
}
// Every thread of both CTAs: cluster-wide barrier (release / acquire).
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Whole warp, the same warp in both CTAs of the pair: allocate `ncols` TMEM
// columns at the same address in both CTAs.
__device__ __forceinline__ void tmem_alloc_pair(uint32_t smem_slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_slot), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (M = 256 over the pair) (+)= A * B^T: issued by one thread of the even
// CTA; A rows 0-127 and B rows 0..N/2-1 come from the even CTA's shared
// memory, the rest from the odd CTA's at the same offsets; each CTA's TMEM
// receives its 128 rows x N columns.
template <int KIND>  // 0: kind::f16 (bf16), 1: kind::f8f6f4 (e4m3)
__device__ __forceinline__ void tc_mma_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  if constexpr (KIND == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}
// Arrive once on the mbarrier at offset `bar` of every CTA in `cta_mask` when
// the pair's previously issued tcgen05 ops have completed.
__device__ __forceinline__ void tc_commit_pair_mc(uint32_t bar, uint16_t cta_mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"(cta_mask)
      : "memory");
}
// As tc_commit_pair_mc, arriving on this CTA's barrier only.
__device__ __forceinline__ void tc_commit_pair(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// 32 lanes x 32 consecutive fp32 columns from TMEM; lane i of the warp gets
// row (taddr.lane + i).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor for a K-major operand tile written by TMA
// with 128-byte swizzling: 8-row groups 1024 bytes apart (SBO), leading
// offset unused for swizzled K-major layouts, descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;            // LBO (ignored for SW128 K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // SBO
  d |= (uint64_t)1 << 46;            // version
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

}  // namespace ebsd
