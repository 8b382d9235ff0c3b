// Pattern-centre fitting (ebsdtorch/ebsd/fitting.py:413, 479-507): the
// circular cross-correlation of every simulated pattern with every
// experimental pattern over all shifts of the enlarged detector, and the
// maximum over the dictionary batch per (pattern, shift), without an FFT
// library and without materialising the correlation maps.
//
// The reference computes fftshift(irfft2(rfft2(sim) * conj(rfft2(pat)))) and
// max-reduces it over the batch. Here both 2-D transforms are products with
// DFT matrices on the tensor cores (tcgen05.mma kind::f16, bf16 operands in
// a 3-term split x = hi + lo: hi*hi + hi*lo + lo*hi, FP32 accumulation in
// TMEM, about 1e-5 relative error per product), and the max / argmax is
// taken in the same kernel:
//
//   forward (k_xc_forward, one image per 128-row tile):
//     F1  T[y, kx]      = sum_x img[y, x] e^(-2 pi i kx x / W)    kx < WF = W/2+1
//     F2  Cc[ky, kx]    = sum_y T[y, kx] cos(2 pi ky y / H)       ky < H2 = H/2+1
//         Ss[ky, kx]    = sum_y T[y, kx] sin(2 pi ky y / H)
//     so that S[ky] = Cc - i Ss and S[H - ky] = Cc + i Ss.
//   inverse (k_xc_max, per (pattern, simulated pattern) pair), with
//     Pe = conj(P[ky]) + conj(P[H-ky]), Po = conj(P[ky]) - conj(P[H-ky])
//     (one term only at ky = 0 and ky = H/2):
//     E = Cc Pe - i Ss Po,  O = Cc Po - i Ss Pe     (the even / odd parts of
//                                                    M = S conj(P) in ky)
//     A   U[y, kx] = sum_ky E cos(2 pi ky y'/H) + i O sin(2 pi ky y'/H)
//     B   c[y, x]  = sum_kx a_kx Re(U[y, kx] e^(2 pi i kx x'/W)) / (H W)
//     with y' = y - H/2, x' = x - W/2 (the fftshift) and a_kx = 1 for the
//     DC and Nyquist columns, 2 otherwise (the c2r Hermitian fold).
//
// Each stage is D[128 lanes, N] = A[128 rows, K] B[N rows, K]^T. The
// constant DFT matrices are built once per detector size and copied by each
// CTA into shared memory; data operands are written by the CTA's threads in
// the 128-byte-swizzled K-major layout the MMA descriptors read.
//
// The inverse kernels: a CTA owns one experimental pattern and a slice of
// the batch and correlates PP simulated patterns with it per pass; the max
// over pairs and passes is kept per shift in registers (the first maximum
// wins on ties, i.e. the smaller index), and at the end each (shift, max,
// index) is merged into a 64-bit key (ordered float bits, inverted index)
// with atomicMax; ebsd_pcfit_fold applies the reference's running-best rule
// (fitting.py:498-507) per batch and clears the keys.
//   k_xc_max_tm (used when its operands fit shared memory, up to about
//     96 x 96): stage A leaves its output in TMEM laid out as stage B's A
//     operand (lanes y, K along the columns); passes are software-pipelined.
//   k_xc_max (larger detectors): stage A's output is written transposed
//     through shared memory and the pass's maps are staged there.
//
// Supported: enlarged detectors up to 127 x 127 (one 128-row tile per
// image, K <= 128). Every wait is bounded; a timeout is reported in *status.
#include <algorithm>
#include <climits>
#include <cstdint>

#include "common.cuh"

namespace ebsd {
namespace xc {

constexpr int THREADS = 512;
constexpr int MAX_HW = 127;
constexpr int SMEM_LIMIT = 232448;
constexpr int SMEM_ONE_CTA = 120 * 1024;  // more than half of an SM's 228 KB

__host__ __device__ constexpr int round_up_i(int a, int b) { return (a + b - 1) / b * b; }
__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Derived sizes of one enlarged detector (H rows, W columns).
struct Geo {
  int H, W;
  int H2, WF;     // ky < H2 = H/2 + 1, kx < WF = W/2 + 1
  int KOA, KOB;   // H2, WF rounded up to 8 (the second half of a K row starts there)
  int RW;         // rows per image in the (part, kx) layout: 2 KOB
  int NA, NB;     // inverse: N of stage A (y) and stage B (x)
  int N1, N2;     // forward: N of F1 ((part, kx)) and F2 ((trig, ky))
  int KSA, KSB;   // inverse: 16-element K steps of stage A (2 KOA) and B (2 KOB)
  int KS1, KS2;   // forward: K steps of F1 (W) and F2 (H)
  int KPA, KPB, KP1, KP2;  // 64-element K planes of the constant matrices
  int spec;       // floats per spectrum: [trig or eo][part][H2][WF]
};

__host__ __device__ inline Geo make_geo(int H, int W) {
  Geo g{};
  g.H = H;
  g.W = W;
  g.H2 = H / 2 + 1;
  g.WF = W / 2 + 1;
  g.KOA = round_up_i(g.H2, 8);
  g.KOB = round_up_i(g.WF, 8);
  g.RW = 2 * g.KOB;
  g.NA = round_up_i(H, 16);
  g.NB = round_up_i(W, 16);
  g.N1 = round_up_i(2 * g.KOB, 16);
  g.N2 = round_up_i(2 * g.KOA, 16);
  g.KSA = cdiv(2 * g.KOA, 16);
  g.KSB = cdiv(2 * g.KOB, 16);
  g.KS1 = cdiv(W, 16);
  g.KS2 = cdiv(H, 16);
  g.KPA = cdiv(2 * g.KOA, 64);
  g.KPB = cdiv(2 * g.KOB, 64);
  g.KP1 = cdiv(W, 64);
  g.KP2 = cdiv(H, 64);
  g.spec = 4 * g.H2 * g.WF;
  return g;
}

// Byte offset of element (row, k) in a K-major bf16 operand of `rows` rows
// stored as 64-element K planes, each plane 128-byte swizzled in 8-row
// groups (the layout TMA writes with CU_TENSOR_MAP_SWIZZLE_128B).
__host__ __device__ inline uint32_t op_offset(int rows, int row, int k) {
  const uint32_t kb = (uint32_t)(k & 63) * 2u;
  return (uint32_t)(k >> 6) * (uint32_t)rows * 128u + (uint32_t)(row >> 3) * 1024u + (uint32_t)(row & 7) * 128u +
         ((((kb >> 4) ^ (uint32_t)(row & 7)) << 4) | (kb & 15u));
}

// Bytes of one constant matrix image (hi or lo) of `rows` rows, `planes` planes.
__host__ __device__ constexpr int mat_bytes(int rows, int planes) { return rows * 128 * planes; }

// The constant matrices, each stored as two images (hi and lo halves of the
// bf16 split, or for the mixed stage-B matrix of the TMEM kernel the
// [hi | hi] and [lo | 0] images described at k_xc_max_tm):
//   0 inverse stage A        rows y (NA), K [cos | sin] over ky
//   1 inverse stage B        rows x (NB), K [a cos | -a sin] / (H W) over kx
//   2 forward F1             rows (re/im, kx) (N1), K x
//   3 forward F2             rows (cos/sin, ky) (N2), K y
//   4 inverse stage A (TMEM) matrix 0 with 128 rows (the MMA's A operand)
//   5 inverse stage B (TMEM) rows x (NB), K' = 2 * RW: per 8 K elements of
//     matrix 1, 16 K' elements
// Matrices are stored one after the other; kernels copy a contiguous run.
constexpr int N_MATS = 6;
struct Tables {
  int rows[N_MATS], planes[N_MATS];
  int img[N_MATS];  // bytes of one image
  int off[N_MATS];  // byte offset of the matrix's first image
  int total;
  // contiguous runs per kernel: inverse (0, 1), forward (2, 3), TMEM inverse (4, 5)
  int inv_bytes, fwd_bytes, tm_bytes;
  int inv_a, inv_b, fwd_1, fwd_2, tm_a, tm_b;  // image bytes, for the kernels' layouts
};

__host__ __device__ inline Tables table_sizes(const Geo& g) {
  Tables t{};
  const int rows[N_MATS] = {g.NA, g.NB, g.N1, g.N2, 128, g.NB};
  const int planes[N_MATS] = {g.KPA, g.KPB, g.KP1, g.KP2, g.KPA, cdiv(2 * g.RW, 64)};
  int off = 0;
  for (int m = 0; m < N_MATS; ++m) {
    t.rows[m] = rows[m];
    t.planes[m] = planes[m];
    t.img[m] = mat_bytes(rows[m], planes[m]);
    t.off[m] = off;
    off += 2 * t.img[m];
  }
  t.total = off;
  t.inv_bytes = 2 * (t.img[0] + t.img[1]);
  t.fwd_bytes = 2 * (t.img[2] + t.img[3]);
  t.tm_bytes = 2 * (t.img[4] + t.img[5]);
  t.inv_a = t.img[0];
  t.inv_b = t.img[1];
  t.fwd_1 = t.img[2];
  t.fwd_2 = t.img[3];
  t.tm_a = t.img[4];
  t.tm_b = t.img[5];
  return t;
}

// cos and sin of 2 pi m / n for an integer m (reduced mod n), exact on the
// quarter turns.
__device__ inline void cos_sin_turn(int64_t m, int n, double& c, double& s) {
  int64_t r = m % n;
  if (r < 0) r += n;
  if (r == 0) {
    c = 1.0;
    s = 0.0;
  } else if (2 * r == n) {
    c = -1.0;
    s = 0.0;
  } else if (4 * r == n) {
    c = 0.0;
    s = 1.0;
  } else if (4 * r == 3 * (int64_t)n) {
    c = 0.0;
    s = -1.0;
  } else {
    sincospi(2.0 * (double)r / (double)n, &s, &c);
  }
}

__device__ inline void split_bf16(double v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn((float)v);
  lo = __float2bfloat16_rn((float)(v - (double)__bfloat162float(hi)));
}

// Entry (row, k) of the inverse transforms: stage A (y, [cos | sin] over ky)
// and stage B (x, [a cos | -a sin] / (H W) over kx).
__device__ inline double inv_a_value(const Geo& g, int y, int k) {
  const int part = k >= g.KOA, ky = k - part * g.KOA;
  if (y >= g.H || ky >= g.H2) return 0.0;
  double c, s;
  cos_sin_turn((int64_t)ky * (y - g.H / 2), g.H, c, s);
  return part ? s : c;
}

__device__ inline double inv_b_value(const Geo& g, int x, int k) {
  const int part = k >= g.KOB, kx = k - part * g.KOB;
  if (x >= g.W || kx >= g.WF || part > 1) return 0.0;
  double c, s;
  cos_sin_turn((int64_t)kx * (x - g.W / 2), g.W, c, s);
  const double a = (kx == 0 || 2 * kx == g.W) ? 1.0 : 2.0;
  return a * (part ? -s : c) / ((double)g.H * (double)g.W);
}

// One thread per (matrix, row, k) element; writes both images.
__global__ void k_xc_tables(Geo g, Tables t, uint8_t* __restrict__ out) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int m = 0;
  for (; m < N_MATS; ++m) {
    const int64_t n = (int64_t)t.rows[m] * 64 * t.planes[m];
    if (r < n) break;
    r -= n;
  }
  if (m == N_MATS) return;
  const int width = 64 * t.planes[m];
  const int row = (int)(r / width), k = (int)(r % width);
  __nv_bfloat16 v0, v1;
  if (m == 5) {
    // K' = 16 q + 8 half + j holds K = 8 q + j: image 0 [hi | hi], image 1 [lo | 0]
    const int q = k / 16, half = (k / 8) & 1, j = k & 7, kk = 8 * q + j;
    __nv_bfloat16 hi, lo;
    split_bf16(kk < g.RW ? inv_b_value(g, row, kk) : 0.0, hi, lo);
    v0 = hi;
    v1 = half ? __float2bfloat16_rn(0.0f) : lo;
  } else {
    double v = 0.0, c, s;
    if (m == 0 || m == 4) {
      v = inv_a_value(g, row, k);
    } else if (m == 1) {
      v = inv_b_value(g, row, k);
    } else if (m == 2) {  // forward F1: rows (part, kx), K = x: cos / -sin
      const int part = row >= g.KOB, kx = row - part * g.KOB, x = k;
      if (kx < g.WF && x < g.W) {
        cos_sin_turn((int64_t)kx * x, g.W, c, s);
        v = part ? -s : c;
      }
    } else {  // forward F2: rows (trig, ky), K = y: cos / sin
      const int trig = row >= g.KOA, ky = row - trig * g.KOA, y = k;
      if (ky < g.H2 && y < g.H) {
        cos_sin_turn((int64_t)ky * y, g.H, c, s);
        v = trig ? s : c;
      }
    }
    split_bf16(v, v0, v1);
  }
  const uint32_t o = op_offset(t.rows[m], row, k);
  *reinterpret_cast<__nv_bfloat16*>(out + t.off[m] + o) = v0;
  *reinterpret_cast<__nv_bfloat16*>(out + t.off[m] + t.img[m] + o) = v1;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 lanes x 8 consecutive fp32 columns; lane i of the warp gets row (lane base + i).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// Eight consecutive K elements (k8 a multiple of 8) of one row, split into
// the hi and lo operands: one 16-byte store each.
__device__ __forceinline__ void put8(uint8_t* hi, uint8_t* lo, int rows, int row, int k8, const float (&v)[8]) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * j]), h1 = __float2bfloat16_rn(v[2 * j + 1]);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * j] - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * j + 1] - __bfloat162float(h1));
    h[j] = pack_bf16(h0, h1);
    l[j] = pack_bf16(l0, l1);
  }
  const uint32_t off = op_offset(rows, row, k8);
  *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// One element, split into hi and lo.
__device__ __forceinline__ void put1(uint8_t* hi, uint8_t* lo, int rows, int row, int k, float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
  const uint32_t off = op_offset(rows, row, k);
  *reinterpret_cast<__nv_bfloat16*>(hi + off) = h;
  *reinterpret_cast<__nv_bfloat16*>(lo + off) = l;
}

__device__ __forceinline__ uint32_t xc_idesc(int n) {
  // F32 accumulator, BF16 A and B, both K-major, N >> 3 at bit 17, M = 128.
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// One stage of split products: for each of n_tiles 128-row tiles of A,
// D[tile] = (A_hi B_hi + A_hi B_lo + A_lo B_hi)^T over ksteps 16-element K
// steps. A has a_rows rows per plane, B b_rows. Issued by one thread.
__device__ __forceinline__ void issue_stage(uint32_t d_tmem, int n, int n_tiles, uint32_t a_hi, uint32_t a_lo,
                                            int a_rows, uint32_t b_hi, uint32_t b_lo, int b_rows, int ksteps) {
  const uint32_t idesc = xc_idesc(n);
  for (int t = 0; t < n_tiles; ++t) {
    const uint32_t d = d_tmem + (uint32_t)(t * n);
    for (int ks = 0; ks < ksteps; ++ks) {
      const uint32_t aoff = (uint32_t)(ks >> 2) * (uint32_t)a_rows * 128u + (uint32_t)t * 16384u + (uint32_t)(ks & 3) * 32u;
      const uint32_t boff = (uint32_t)(ks >> 2) * (uint32_t)b_rows * 128u + (uint32_t)(ks & 3) * 32u;
      tc_mma<0>(d, smem_desc_sw128(a_hi + aoff), smem_desc_sw128(b_hi + boff), idesc, ks > 0 ? 1u : 0u);
      tc_mma<0>(d, smem_desc_sw128(a_hi + aoff), smem_desc_sw128(b_lo + boff), idesc, 1u);
      tc_mma<0>(d, smem_desc_sw128(a_lo + aoff), smem_desc_sw128(b_hi + boff), idesc, 1u);
    }
  }
}

// D[tmem] (+)= A[tmem] * B[smem]^T (kind::f16, BF16 A packed two per TMEM
// column, the even K element in the low half), issued by one thread.
__device__ __forceinline__ void tc_mma_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns into TMEM (lane i of the warp
// writes row lane base + i).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
      "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
      : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

struct XcParams {
  Geo g;
  int mt;          // 128-row tiles per pass (1 or 2)
  int pp;          // inverse: pairs per pass
  int buf_rows;    // rows of the A operand buffers (mt * 128)
  int buf_planes;  // K planes of the A operand buffers
  int buf_bytes;   // bytes of one A operand buffer (hi or lo)
  Tables tb;
  const uint8_t* tables;
  // forward
  const float* img;
  int64_t ld_img;
  int64_t n_img;
  float* spec_out;
  // inverse
  const float* sim_spec;
  int64_t n_sims;
  const float* pat_terms;
  int n_pats;
  int slices;
  int pp_tm;  // TMEM kernel: pairs per pass
  int64_t index_base;
  unsigned long long* keys;
  int* status;
  uint64_t wait_ns;
};

// Shared-memory layout (1024-aligned base): A hi | A lo | C0 hi | C0 lo |
// C1 hi | C1 lo | mbarrier | TMEM slot | flags.
struct Smem {
  uint8_t* a_hi;
  uint8_t* a_lo;
  uint8_t* c0;
  uint8_t* c1;
  uint64_t* bar;
  uint32_t* tmem_slot;
  volatile int* flag;
};

__device__ __forceinline__ Smem carve(uint8_t* base, const XcParams& p, int c0_bytes, int c1_bytes) {
  Smem s;
  s.a_hi = base;
  s.a_lo = base + p.buf_bytes;
  s.c0 = base + 2 * p.buf_bytes;
  s.c1 = s.c0 + 2 * c0_bytes;
  uint8_t* tail = s.c1 + 2 * c1_bytes;
  s.bar = reinterpret_cast<uint64_t*>(tail);
  s.tmem_slot = reinterpret_cast<uint32_t*>(tail + 8);
  s.flag = reinterpret_cast<volatile int*>(tail + 12);
  return s;
}

__host__ __device__ inline int smem_bytes(int buf_bytes, int c0_bytes, int c1_bytes) {
  return 1024 + 2 * buf_bytes + 2 * c0_bytes + 2 * c1_bytes + 64;
}

// Copy the mode's constant images into shared memory (16-byte loads) and
// zero the A buffers (their K padding and unused rows must hold finite
// values: they multiply the zero padding of the constant matrices).
__device__ __forceinline__ void load_constants(const Smem& s, const uint8_t* src, int bytes, const XcParams& p) {
  const uint4* g4 = reinterpret_cast<const uint4*>(src);
  uint4* d4 = reinterpret_cast<uint4*>(s.c0);
  for (int i = threadIdx.x; i < bytes / 16; i += THREADS) d4[i] = __ldg(g4 + i);
  uint4* a4 = reinterpret_cast<uint4*>(s.a_hi);
  for (int i = threadIdx.x; i < 2 * p.buf_bytes / 16; i += THREADS) a4[i] = make_uint4(0, 0, 0, 0);
}

// Issue-and-wait step shared by both kernels: the operand writes of all
// threads are made visible to the tensor core, thread 0 issues the stage and
// waits (bounded) for its completion, everyone learns the outcome.
// Returns false when the wait gave up (the status word is set).
template <typename Issue>
__device__ __forceinline__ bool run_stage(const Smem& s, const XcParams& p, uint32_t& phase, Issue issue) {
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    issue();
    tc_commit(smem_u32(s.bar));
    const bool ok = mbar_wait(smem_u32(s.bar), phase, s.flag, p.wait_ns);
    if (!ok) {
      *s.flag = 1;
      atomicExch(p.status, EBSD_DEVICE_TIMEOUT);
    }
  }
  phase ^= 1u;
  __syncthreads();
  tc_fence_after();
  return *s.flag == 0;
}

// Before TMEM is released after a timeout: the stage that timed out may
// still be running; wait for it under the default limit.
__device__ __forceinline__ void drain(const Smem& s, uint32_t phase_of_last) {
  if (threadIdx.x == 0 && *s.flag) {
    volatile int never = 0;
    mbar_wait(smem_u32(s.bar), phase_of_last, &never, kWaitLimitNs);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// forward: spectra (Cc, Ss) of images, mt images per pass
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(THREADS, 1) k_xc_forward(const XcParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* base = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const Geo& g = p.g;
  const Smem s = carve(base, p, p.tb.fwd_1, p.tb.fwd_2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int lg = warp & 3, t_of_warp = (warp >> 2) % p.mt, cg = (warp >> 2) / p.mt, n_cg = 4 / p.mt;

  load_constants(s, p.tables + p.tb.inv_bytes, p.tb.fwd_bytes, p);
  if (tid == 0) {
    mbar_init(smem_u32(s.bar), 1);
    *s.flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(smem_u32(s.tmem_slot), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem_slot;
  const uint32_t d1 = tmem, d2 = tmem + (uint32_t)(p.mt * g.N1);
  const uint32_t a_hi = smem_u32(s.a_hi), a_lo = smem_u32(s.a_lo);
  const uint32_t f1_hi = smem_u32(s.c0), f1_lo = f1_hi + p.tb.fwd_1;
  const uint32_t f2_hi = smem_u32(s.c1), f2_lo = f2_hi + p.tb.fwd_2;
  uint32_t phase = 0;
  const int64_t n_groups = (p.n_img + p.mt - 1) / p.mt;
  const int xg = cdiv(g.W, 8);

  for (int64_t grp = blockIdx.x; grp < n_groups; grp += gridDim.x) {
    const int64_t i0 = grp * p.mt;
    const int ni = (int)(p.n_img - i0 < p.mt ? p.n_img - i0 : p.mt);
    // F1 operand: image t's rows y in tile t, K = x
    for (int it = tid; it < ni * g.H * xg; it += THREADS) {
      const int t = it / (g.H * xg), rem = it - t * g.H * xg, y = rem / xg, x0 = (rem - y * xg) * 8;
      const float* row = p.img + (i0 + t) * p.ld_img + (int64_t)y * g.W;
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = x0 + j < g.W ? __ldg(row + x0 + j) : 0.0f;
      if (EBSD_DCHECK(t * 128 + y < p.buf_rows && x0 + 8 <= 64 * p.buf_planes))
        put8(s.a_hi, s.a_lo, p.buf_rows, t * 128 + y, x0, v);
    }
    if (!run_stage(s, p, phase, [&] {
          issue_stage(d1, g.N1, ni, a_hi, a_lo, p.buf_rows, f1_hi, f1_lo, g.N1, g.KS1);
        }))
      break;
    // F2 operand: rows (image, part, kx), K = y, from T (lanes y, columns (part, kx))
    {
      const int y = lg * 32 + lane;
      const bool valid = t_of_warp < ni && y < g.H;
      for (int c8 = cg; c8 < g.N1 / 8; c8 += n_cg) {
        float v[8];
        tmem_ld8(d1 + ((uint32_t)(lg * 32) << 16) + (uint32_t)(t_of_warp * g.N1 + c8 * 8), v);
        if (valid) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int c = c8 * 8 + j;
            if (c < g.RW && EBSD_DCHECK(t_of_warp * g.RW + c < p.buf_rows && y < 64 * p.buf_planes))
              put1(s.a_hi, s.a_lo, p.buf_rows, t_of_warp * g.RW + c, y, v[j]);
          }
        }
      }
    }
    if (!run_stage(s, p, phase, [&] {
          issue_stage(d2, g.N2, cdiv(ni * g.RW, 128), a_hi, a_lo, p.buf_rows, f2_hi, f2_lo, g.N2, g.KS2);
        }))
      break;
    // epilogue: lanes (image, part, kx), columns (trig, ky) -> spec[img][trig][part][ky][kx]
    {
      const int r = t_of_warp * 128 + lg * 32 + lane;
      const int im = r / g.RW, c = r - im * g.RW;
      const int part = c >= g.KOB, kx = c - part * g.KOB;
      const bool valid = r < ni * g.RW && kx < g.WF;
      float* out = p.spec_out + (i0 + im) * (int64_t)g.spec + (int64_t)part * g.H2 * g.WF + kx;
      if (t_of_warp * 128 < ni * g.RW) {
        for (int c8 = cg; c8 < g.N2 / 8; c8 += n_cg) {
          float v[8];
          tmem_ld8(d2 + ((uint32_t)(lg * 32) << 16) + (uint32_t)(t_of_warp * g.N2 + c8 * 8), v);
          if (valid) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int n2 = c8 * 8 + j;
              const int trig = n2 >= g.KOA, ky = n2 - trig * g.KOA;
              if (ky < g.H2 && trig < 2) out[((int64_t)trig * 2 * g.H2 + ky) * g.WF] = v[j];
            }
          }
        }
      }
    }
  }
  drain(s, phase ^ 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------
// inverse: correlation maps of (pattern, simulated pattern) pairs, max over
// the slice of simulated patterns, merged into 64-bit keys
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long max_key(float v, uint32_t idx) {
  const uint32_t u = __float_as_uint(v);
  const uint32_t ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  return ((unsigned long long)ord << 32) | (unsigned long long)(0xFFFFFFFFu - idx);
}

template <int POS>  // shifts per thread: H * W <= POS * THREADS
__global__ void __launch_bounds__(THREADS, 1) k_xc_max(const XcParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* base = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const Geo& g = p.g;
  const Smem s = carve(base, p, p.tb.inv_a, p.tb.inv_b);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int lg = warp & 3, t_of_warp = (warp >> 2) % p.mt, cg = (warp >> 2) / p.mt, n_cg = 4 / p.mt;
  const int b = blockIdx.x / p.slices, sl = blockIdx.x - b * p.slices;
  const int64_t s_begin = p.n_sims * sl / p.slices, s_end = p.n_sims * (sl + 1) / p.slices;

  load_constants(s, p.tables, p.tb.inv_bytes, p);
  if (tid == 0) {
    mbar_init(smem_u32(s.bar), 1);
    *s.flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(smem_u32(s.tmem_slot), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem_slot;
  const uint32_t da = tmem, db = tmem + (uint32_t)(p.mt * g.NA);
  const uint32_t a_hi = smem_u32(s.a_hi), a_lo = smem_u32(s.a_lo);
  const uint32_t ca_hi = smem_u32(s.c0), ca_lo = ca_hi + p.tb.inv_a;
  const uint32_t cb_hi = smem_u32(s.c1), cb_lo = cb_hi + p.tb.inv_b;
  float* scratch = reinterpret_cast<float*>(s.a_hi);  // the pass's maps, [pair][y][x]
  const int hw = g.H * g.W, ng = g.KOA / 8, hwf = g.H2 * g.WF;
  const float* pt = p.pat_terms + (int64_t)b * g.spec;

  float best_v[POS];
  int best_i[POS];  // index inside the launch's batch (n_sims < 2^31)
#pragma unroll
  for (int j = 0; j < POS; ++j) {
    best_v[j] = -INFINITY;
    best_i[j] = -1;
  }
  uint32_t phase = 0;

  for (int64_t s0 = s_begin; s0 < s_end; s0 += p.pp) {
    const int np = (int)(s_end - s0 < p.pp ? s_end - s0 : p.pp);
    // stage A operand: rows (pair, part, kx), K = [E part | O part] over ky
    for (int it = tid; it < np * g.WF * ng; it += THREADS) {
      const int pr = it / (g.WF * ng), rem = it - pr * g.WF * ng, grp = rem / g.WF, kx = rem - grp * g.WF;
      const float* cs = p.sim_spec + (s0 + pr) * (int64_t)g.spec + kx;
      float er[8], ei[8], orr[8], oi[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int ky = grp * 8 + j;
        er[j] = ei[j] = orr[j] = oi[j] = 0.0f;
        if (ky < g.H2) {
          const int o = ky * g.WF;
          const float a = __ldg(cs + o), bi = __ldg(cs + hwf + o);                // Cc
          const float c = __ldg(cs + 2 * hwf + o), d = __ldg(cs + 3 * hwf + o);   // Ss
          const float e = __ldg(pt + o + kx), f = __ldg(pt + hwf + o + kx);       // Pe
          const float gg = __ldg(pt + 2 * hwf + o + kx), h = __ldg(pt + 3 * hwf + o + kx);  // Po
          er[j] = a * e - bi * f + c * h + d * gg;
          ei[j] = a * f + bi * e - c * gg + d * h;
          orr[j] = a * gg - bi * h + c * f + d * e;
          oi[j] = a * h + bi * gg - c * e + d * f;
        }
      }
      float neg_oi[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) neg_oi[j] = -oi[j];
      const int row_re = pr * g.RW + kx, row_im = row_re + g.KOB;
      put8(s.a_hi, s.a_lo, p.buf_rows, row_re, grp * 8, er);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_re, g.KOA + grp * 8, neg_oi);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_im, grp * 8, ei);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_im, g.KOA + grp * 8, orr);
    }
    if (!run_stage(s, p, phase, [&] {
          issue_stage(da, g.NA, cdiv(np * g.RW, 128), a_hi, a_lo, p.buf_rows, ca_hi, ca_lo, g.NA, g.KSA);
        }))
      break;
    // stage B operand: rows (pair, y), K = [Ur | Ui] over kx, from U (lanes
    // (pair, part, kx), columns y)
    {
      const int r = t_of_warp * 128 + lg * 32 + lane;
      const int pr = r / g.RW, c = r - pr * g.RW;
      const int part = c >= g.KOB, kx = c - part * g.KOB;
      const bool valid = r < np * g.RW && kx < g.WF;
      if (t_of_warp * 128 < np * g.RW) {
        for (int c8 = cg; c8 < g.NA / 8; c8 += n_cg) {
          float v[8];
          tmem_ld8(da + ((uint32_t)(lg * 32) << 16) + (uint32_t)(t_of_warp * g.NA + c8 * 8), v);
          if (valid) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int y = c8 * 8 + j;
              if (y < g.H) put1(s.a_hi, s.a_lo, p.buf_rows, pr * g.H + y, part * g.KOB + kx, v[j]);
            }
          }
        }
      }
    }
    if (!run_stage(s, p, phase, [&] {
          issue_stage(db, g.NB, cdiv(np * g.H, 128), a_hi, a_lo, p.buf_rows, cb_hi, cb_lo, g.NB, g.KSB);
        }))
      break;
    // maps (lanes (pair, y), columns x) into scratch, then the max over the pass
    {
      const int r = t_of_warp * 128 + lg * 32 + lane;
      const bool valid = r < np * g.H;
      if (t_of_warp * 128 < np * g.H) {
        for (int c8 = cg; c8 < g.NB / 8; c8 += n_cg) {
          float v[8];
          tmem_ld8(db + ((uint32_t)(lg * 32) << 16) + (uint32_t)(t_of_warp * g.NB + c8 * 8), v);
          if (valid) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int x = c8 * 8 + j;
              if (x < g.W) scratch[r * g.W + x] = v[j];
            }
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
#pragma unroll
    for (int j = 0; j < POS; ++j) {
      const int pos = tid + j * THREADS;
      if (pos < hw) {
        for (int pr = 0; pr < np; ++pr) {
          const float v = scratch[pr * hw + pos];
          if (v > best_v[j]) {
            best_v[j] = v;
            best_i[j] = (int)(s0 + pr);
          }
        }
      }
    }
    __syncthreads();  // scratch (the A buffers) is rewritten by the next pass
  }
  if (*s.flag == 0) {
    unsigned long long* keys = p.keys + (int64_t)b * hw;
#pragma unroll
    for (int j = 0; j < POS; ++j) {
      const int pos = tid + j * THREADS;
      if (pos < hw && best_i[j] >= 0) atomicMax(keys + pos, max_key(best_v[j], (uint32_t)(p.index_base + best_i[j])));
    }
  }
  drain(s, phase ^ 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// k_xc_max_tm: the inverse transforms with stage A's output kept in TMEM as
// stage B's A operand (no shared-memory transpose, no staged maps):
//   stage A  D_A[y, (pair, part, kx)] = CA[y, K] . Data[(pair, part, kx), K]^T
//            with the constant (128 rows y) as the A operand and the pass's
//            [E | O] rows as B (N = pairs * RW);
//   convert  each thread rewrites its own 8-column chunks of D_A in place as
//            [hi x 8 | lo x 8] bf16, 8 columns = 16 K' elements;
//   stage B  D_B[y, (pair, x)] = sum over chunks q of A'(q) . P(q)^T +
//            A'(q) . Q(q)^T, with P = [Bhi | Bhi] and Q = [Blo | 0] over the
//            chunk's 8 K elements: hi Bhi + lo Bhi + hi Blo, the 3-term split;
//   epilogue each thread owns lane y and CPT x chunks; the max over the
//            pass's pairs and over passes stays in its registers.
template <int CPT>  // x chunks of 8 per thread: NB / 8 <= 4 CPT
__global__ void __launch_bounds__(THREADS, 1) k_xc_max_tm(const XcParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_s = smem_u32(smem_raw);
  uint8_t* base = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
  const Geo& g = p.g;
  const Smem s = carve(base, p, p.tb.tm_a, p.tb.tm_b);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int lg = warp & 3, cg = warp >> 2;
  const int b = blockIdx.x / p.slices, sl = blockIdx.x - b * p.slices;
  const int64_t s_begin = p.n_sims * sl / p.slices, s_end = p.n_sims * (sl + 1) / p.slices;

  load_constants(s, p.tables + p.tb.off[4], p.tb.tm_bytes, p);
  if (tid == 0) {
    mbar_init(smem_u32(s.bar), 1);
    *s.flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(smem_u32(s.tmem_slot), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s.tmem_slot;
  const uint32_t da = tmem, db = tmem + 256u;
  const uint32_t lane_off = (uint32_t)(lg * 32) << 16;
  const uint32_t d_hi = smem_u32(s.a_hi), d_lo = smem_u32(s.a_lo);
  const uint32_t ca_hi = smem_u32(s.c0), ca_lo = ca_hi + p.tb.tm_a;
  const uint32_t cp = smem_u32(s.c1), cq = cp + p.tb.tm_b;
  const int ng = g.KOA / 8, hwf = g.H2 * g.WF, nb8 = g.NB / 8, rw8 = g.RW / 8;
  const float* pt = p.pat_terms + (int64_t)b * g.spec;
  const int y = lg * 32 + lane;

  float best_v[CPT][8];
  int best_i[CPT][8];
#pragma unroll
  for (int j = 0; j < CPT; ++j)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      best_v[j][i] = -INFINITY;
      best_i[j][i] = -1;
    }
  uint32_t phase = 0;
  const int64_t n_pass = (s_end - s_begin + p.pp_tm - 1) / p.pp_tm;
  auto pass_np = [&](int64_t i) {
    const int64_t left = s_end - (s_begin + i * p.pp_tm);
    return (int)(left < p.pp_tm ? left : p.pp_tm);
  };

  // this thread's operand-formation items, the same in every pass (at most
  // two: pp * WF * KOA / 8 <= 1024): (pair, ky group of 8, kx), decoded once
  int it_pr[2], it_grp[2], it_kx[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int it = tid + k * THREADS;
    it_pr[k] = INT_MAX;  // inactive
    it_grp[k] = it_kx[k] = 0;
    if (it < p.pp_tm * g.WF * ng) {
      const int pr = it / (g.WF * ng), rem = it - pr * g.WF * ng;
      it_pr[k] = pr;
      it_grp[k] = rem / g.WF;
      it_kx[k] = rem - it_grp[k] * g.WF;
    }
  }
  // stage A's B operand of pass i: rows (pair, part, kx), K = [E | O] over ky
  auto form = [&](int64_t i) {
    const int64_t s0 = s_begin + i * p.pp_tm;
    const int np = pass_np(i);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (it_pr[k] >= np) continue;
      const int pr = it_pr[k], grp = it_grp[k], kx = it_kx[k];
      const float* cs = p.sim_spec + (s0 + pr) * (int64_t)g.spec + kx;
      float er[8], ei[8], orr[8], noi[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int ky = grp * 8 + j;
        er[j] = ei[j] = orr[j] = noi[j] = 0.0f;
        if (ky < g.H2) {
          const int o = ky * g.WF;
          const float a = __ldg(cs + o), bi = __ldg(cs + hwf + o);                // Cc
          const float c = __ldg(cs + 2 * hwf + o), d = __ldg(cs + 3 * hwf + o);   // Ss
          const float e = __ldg(pt + o + kx), f = __ldg(pt + hwf + o + kx);       // Pe
          const float gg = __ldg(pt + 2 * hwf + o + kx), h = __ldg(pt + 3 * hwf + o + kx);  // Po
          er[j] = a * e - bi * f + c * h + d * gg;
          ei[j] = a * f + bi * e - c * gg + d * h;
          orr[j] = a * gg - bi * h + c * f + d * e;
          noi[j] = -(a * h + bi * gg - c * e + d * f);
        }
      }
      const int row_re = pr * g.RW + kx, row_im = row_re + g.KOB;
      if (!EBSD_DCHECK(row_im < p.buf_rows && g.KOA + grp * 8 + 8 <= 64 * p.buf_planes)) continue;
      put8(s.a_hi, s.a_lo, p.buf_rows, row_re, grp * 8, er);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_re, g.KOA + grp * 8, noi);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_im, grp * 8, ei);
      put8(s.a_hi, s.a_lo, p.buf_rows, row_im, g.KOA + grp * 8, orr);
    }
  };
  auto issue_a = [&](int np) {
    const int n = np * g.RW;
    const uint32_t idesc = xc_idesc(n);
    for (int ks = 0; ks < g.KSA; ++ks) {
      const uint32_t aoff = (uint32_t)(ks >> 2) * 128u * 128u + (uint32_t)(ks & 3) * 32u;
      const uint32_t boff = (uint32_t)(ks >> 2) * (uint32_t)p.buf_rows * 128u + (uint32_t)(ks & 3) * 32u;
      tc_mma<0>(da, smem_desc_sw128(ca_hi + aoff), smem_desc_sw128(d_hi + boff), idesc, ks > 0 ? 1u : 0u);
      tc_mma<0>(da, smem_desc_sw128(ca_hi + aoff), smem_desc_sw128(d_lo + boff), idesc, 1u);
      tc_mma<0>(da, smem_desc_sw128(ca_lo + aoff), smem_desc_sw128(d_hi + boff), idesc, 1u);
    }
  };
  auto issue_b = [&](int np) {
    const uint32_t idesc = xc_idesc(g.NB);
    for (int pr = 0; pr < np; ++pr) {
      for (int q = 0; q < rw8; ++q) {
        const uint32_t boff = (uint32_t)((16 * q) >> 6) * (uint32_t)g.NB * 128u + (uint32_t)(q & 3) * 32u;
        const uint32_t a = da + (uint32_t)(pr * g.RW + 8 * q);
        tc_mma_ta(db + (uint32_t)(pr * g.NB), a, smem_desc_sw128(cp + boff), idesc, q > 0 ? 1u : 0u);
        tc_mma_ta(db + (uint32_t)(pr * g.NB), a, smem_desc_sw128(cq + boff), idesc, 1u);
      }
    }
  };
  // D_A chunks -> [hi | lo] bf16 in place (this thread's lanes and columns only)
  auto convert = [&](int np) {
    for (int c8 = cg; c8 < np * rw8; c8 += 4) {
      if (!EBSD_DCHECK(c8 * 8 + 8 <= 256)) break;  // warp-uniform
      float v[8];
      tmem_ld8(da + lane_off + (uint32_t)(c8 * 8), v);
      uint32_t w[8];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * j]), h1 = __float2bfloat16_rn(v[2 * j + 1]);
        w[j] = pack_bf16(h0, h1);
        w[4 + j] = pack_bf16(__float2bfloat16_rn(v[2 * j] - __bfloat162float(h0)),
                             __float2bfloat16_rn(v[2 * j + 1] - __bfloat162float(h1)));
      }
      tmem_st8(da + lane_off + (uint32_t)(c8 * 8), w);
    }
    tmem_wait_st();
  };
  // maps of pass i: lane y, columns (pair, x); max over the pairs, then the running max
  auto epilogue = [&](int64_t i) {
    const int64_t s0 = s_begin + i * p.pp_tm;
    const int np = pass_np(i);
    for (int pr = 0; pr < np; ++pr) {
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int c8 = cg + 4 * j;
        if (c8 < nb8 && EBSD_DCHECK(pr * g.NB + c8 * 8 + 8 <= 256)) {  // warp-uniform
          float v[8];
          tmem_ld8(db + lane_off + (uint32_t)(pr * g.NB + c8 * 8), v);
#pragma unroll
          for (int i8 = 0; i8 < 8; ++i8) {
            if (v[i8] > best_v[j][i8]) {
              best_v[j][i8] = v[i8];
              best_i[j][i8] = (int)(s0 + pr);
            }
          }
        }
      }
    }
  };
  // Software pipeline, one MMA batch in flight at a time: stage B of pass i
  // runs under the operand formation of pass i + 1, stage A of pass i + 1
  // under the epilogue of pass i. issue(): writes made visible to the
  // tensor core, thread 0 issues and commits; wait(): thread 0 waits
  // (bounded), everyone learns the outcome.
  auto issue = [&](auto&& mmas) {
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      mmas();
      tc_commit(smem_u32(s.bar));
    }
  };
  auto wait = [&]() {
    if (tid == 0 && !mbar_wait(smem_u32(s.bar), phase, s.flag, p.wait_ns)) {
      *s.flag = 1;
      atomicExch(p.status, EBSD_DEVICE_TIMEOUT);
    }
    phase ^= 1u;
    __syncthreads();
    tc_fence_after();
    return *s.flag == 0;
  };
  bool ok = true;
  if (n_pass > 0) {
    form(0);
    issue([&] { issue_a(pass_np(0)); });
    ok = wait();
    if (ok) {
      convert(pass_np(0));
      issue([&] { issue_b(pass_np(0)); });
    }
  }
  for (int64_t i = 0; ok && i < n_pass; ++i) {
    const bool more = i + 1 < n_pass;
    if (more) form(i + 1);  // the data operand is free: stage A of pass i is done
    if (!(ok = wait())) break;  // stage B of pass i
    if (more) issue([&] { issue_a(pass_np(i + 1)); });  // stage B of pass i has read D_A
    epilogue(i);
    if (more) {
      if (!(ok = wait())) break;  // stage A of pass i + 1
      convert(pass_np(i + 1));
      issue([&] { issue_b(pass_np(i + 1)); });
    }
  }
  if (*s.flag == 0 && y < g.H) {
    unsigned long long* keys = p.keys + ((int64_t)b * g.H + y) * g.W;
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int x = (cg + 4 * j) * 8 + i;
        if (x < g.W && best_i[j][i] >= 0)
          atomicMax(keys + x, max_key(best_v[j][i], (uint32_t)(p.index_base + best_i[j][i])));
      }
    }
  }
  drain(s, phase ^ 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// Running best of one pc_z (fitting.py:498-507) from a batch's keys:
// best = max(best, batch max); index replaced where best == batch max; the
// keys are cleared for the next batch.
__global__ void k_xc_fold(unsigned long long* __restrict__ keys, int64_t n, float* __restrict__ best,
                          int64_t* __restrict__ best_idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = keys[i];
  if (k == 0ull) return;
  keys[i] = 0ull;
  const uint32_t ord = (uint32_t)(k >> 32);
  const float v = __uint_as_float((ord & 0x80000000u) ? (ord & 0x7FFFFFFFu) : ~ord);
  const int64_t idx = (int64_t)(0xFFFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull));
  const float nb = fmaxf(best[i], v);
  if (nb == v) best_idx[i] = idx;
  best[i] = nb;
}

// Pattern terms from pattern spectra: Pe = 2 conj(Cc), Po = 2 i conj(Ss),
// with weight 1 instead of 2 at ky = 0 and at ky = H/2 (H even), where the
// pair (ky, H - ky) is a single frequency.
__global__ void k_xc_pattern_terms(const float* __restrict__ spec, int64_t n, Geo g, float* __restrict__ out) {
  const int64_t hwf = (int64_t)g.H2 * g.WF;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * hwf) return;
  const int64_t im = i / hwf, e = i - im * hwf;
  const int ky = (int)(e / g.WF);
  const float w = (ky == 0 || 2 * ky == g.H) ? 1.0f : 2.0f;
  const float* sp = spec + im * g.spec;
  float* o = out + im * g.spec;
  const float ccr = sp[e], cci = sp[hwf + e], ssr = sp[2 * hwf + e], ssi = sp[3 * hwf + e];
  o[e] = w * ccr;
  o[hwf + e] = -w * cci;
  o[2 * hwf + e] = w * ssi;
  o[3 * hwf + e] = w * ssr;
}

}  // namespace xc
}  // namespace ebsd

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

using namespace ebsd;
using namespace ebsd::xc;

namespace {

struct Plan {
  Geo g;
  Tables tb;
  int mt, pp, buf_rows, buf_planes, buf_bytes, smem_fwd, smem_inv, pos;
  int pp_tm, smem_tm, cpt;  // TMEM kernel (pp_tm 0: the detector does not fit it)
};

bool make_plan(int hp, int wp, Plan& pl) {
  if (hp < 2 || wp < 2 || hp > MAX_HW || wp > MAX_HW) return false;
  pl.g = make_geo(hp, wp);
  pl.tb = table_sizes(pl.g);
  const Geo& g = pl.g;
  pl.buf_planes = std::max(std::max(g.KPA, g.KPB), std::max(g.KP1, g.KP2));
  for (int mt = 2; mt >= 1; --mt) {
    pl.mt = mt;
    pl.buf_rows = mt * 128;
    pl.buf_bytes = pl.buf_rows * 128 * pl.buf_planes;
    pl.smem_inv = smem_bytes(pl.buf_bytes, pl.tb.inv_a, pl.tb.inv_b);
    pl.smem_fwd = smem_bytes(pl.buf_bytes, pl.tb.fwd_1, pl.tb.fwd_2);
    pl.pp = std::min(pl.buf_rows / g.RW, pl.buf_rows / g.H);
    // the pass's maps are staged in the A buffers
    while (pl.pp > 1 && (int64_t)pl.pp * g.H * g.W * 4 > 2 * (int64_t)pl.buf_bytes) --pl.pp;
    if (pl.smem_inv <= SMEM_LIMIT && pl.smem_fwd <= SMEM_LIMIT && pl.pp >= 1 &&
        (int64_t)pl.pp * g.H * g.W * 4 <= 2 * (int64_t)pl.buf_bytes)
      break;
    pl.mt = 0;
  }
  if (pl.mt == 0) return false;
  const int pos = cdiv(hp * wp, THREADS);
  pl.pos = pos <= 8 ? 8 : pos <= 16 ? 16 : 32;
  // TMEM kernel: pairs per pass limited by N <= 256 for both stages, the
  // 256 + 256 TMEM columns and shared memory
  pl.pp_tm = 0;
  for (int pp = std::min(256 / g.RW, 256 / g.NB); pp >= 1; --pp) {
    const int bytes = smem_bytes(pp * g.RW * 128 * g.KPA, pl.tb.tm_a, pl.tb.tm_b);
    if (bytes <= SMEM_LIMIT) {
      pl.pp_tm = pp;
      pl.smem_tm = std::max(bytes, SMEM_ONE_CTA);
      break;
    }
  }
  pl.cpt = cdiv(g.NB / 8, 4);
  // every CTA allocates all 512 TMEM columns: ask for enough shared memory
  // that no second CTA fits on the SM
  pl.smem_inv = std::max(pl.smem_inv, SMEM_ONE_CTA);
  pl.smem_fwd = std::max(pl.smem_fwd, SMEM_ONE_CTA);
  return true;
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
  return n;
}

XcParams base_params(const Plan& pl, const void* tables, int* status) {
  XcParams p{};
  p.g = pl.g;
  p.mt = pl.mt;
  p.pp = pl.pp;
  p.buf_rows = pl.buf_rows;
  p.buf_planes = pl.buf_planes;
  p.buf_bytes = pl.buf_bytes;
  p.tb = pl.tb;
  p.tables = static_cast<const uint8_t*>(tables);
  p.status = status;
  p.wait_ns = wait_limit_ns();
  return p;
}

}  // namespace

extern "C" int64_t ebsd_pcfit_xcorr_table_bytes(int hp, int wp) {
  Plan pl;
  if (!make_plan(hp, wp, pl)) return 0;
  return pl.tb.total;
}

extern "C" int ebsd_pcfit_xcorr_tables(int hp, int wp, void* tables, int64_t bytes, void* stream) {
  Plan pl;
  EBSD_ARG_CHECK(make_plan(hp, wp, pl), "enlarged detector %d x %d not supported (2..%d each)", hp, wp, MAX_HW);
  EBSD_ARG_CHECK(tables != nullptr, "ebsd_pcfit_xcorr_tables: null pointer");
  EBSD_ARG_CHECK(((uintptr_t)tables & 15) == 0, "tables must be 16-byte aligned");
  const int64_t need = pl.tb.total;
  EBSD_ARG_CHECK(bytes >= need, "tables hold %lld bytes, %lld needed", (long long)bytes, (long long)need);
  const Geo& g = pl.g;
  int64_t n = 0;
  for (int m = 0; m < N_MATS; ++m) n += (int64_t)pl.tb.rows[m] * 64 * pl.tb.planes[m];
  k_xc_tables<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(g, pl.tb, static_cast<uint8_t*>(tables));
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_pcfit_spectra(const float* images, int64_t ld, int64_t n, int hp, int wp, const void* tables,
                                  float* spectra, int* status, void* stream) {
  Plan pl;
  EBSD_ARG_CHECK(make_plan(hp, wp, pl), "enlarged detector %d x %d not supported (2..%d each)", hp, wp, MAX_HW);
  EBSD_ARG_CHECK(images && tables && spectra && status, "ebsd_pcfit_spectra: null pointer");
  EBSD_ARG_CHECK(n >= 0 && ld >= (int64_t)hp * wp, "bad image count or leading dimension");
  EBSD_ARG_CHECK(((uintptr_t)tables & 15) == 0, "tables must be 16-byte aligned");
  if (n == 0) return 0;
  XcParams p = base_params(pl, tables, status);
  p.img = images;
  p.ld_img = ld;
  p.n_img = n;
  p.spec_out = spectra;
  const int64_t groups = (n + pl.mt - 1) / pl.mt;
  const int grid = (int)std::min<int64_t>(groups, sm_count());
  EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_xc_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, pl.smem_fwd));
  k_xc_forward<<<grid, THREADS, pl.smem_fwd, as_stream(stream)>>>(p);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_pcfit_pattern_terms(const float* spectra, int64_t n, int hp, int wp, float* terms,
                                        void* stream) {
  Plan pl;
  EBSD_ARG_CHECK(make_plan(hp, wp, pl), "enlarged detector %d x %d not supported (2..%d each)", hp, wp, MAX_HW);
  EBSD_ARG_CHECK(spectra && terms, "ebsd_pcfit_pattern_terms: null pointer");
  EBSD_ARG_CHECK(n >= 0, "bad pattern count");
  const int64_t e = n * pl.g.H2 * pl.g.WF;
  if (e == 0) return 0;
  k_xc_pattern_terms<<<(unsigned)((e + 255) / 256), 256, 0, as_stream(stream)>>>(spectra, n, pl.g, terms);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_pcfit_xcorr_max(const float* sim_spectra, int64_t n_sims, const float* pat_terms, int n_pats,
                                    int hp, int wp, const void* tables, unsigned long long* keys,
                                    int64_t index_base, int* status, void* stream) {
  Plan pl;
  EBSD_ARG_CHECK(make_plan(hp, wp, pl), "enlarged detector %d x %d not supported (2..%d each)", hp, wp, MAX_HW);
  EBSD_ARG_CHECK(sim_spectra && pat_terms && tables && keys && status, "ebsd_pcfit_xcorr_max: null pointer");
  EBSD_ARG_CHECK(n_sims >= 0 && n_sims < INT32_MAX && n_pats >= 0, "bad counts");
  EBSD_ARG_CHECK(index_base >= 0 && index_base + n_sims < (int64_t)UINT32_MAX, "index range exceeds 32 bits");
  EBSD_ARG_CHECK(((uintptr_t)tables & 15) == 0, "tables must be 16-byte aligned");
  if (n_sims == 0 || n_pats == 0) return 0;
  XcParams p = base_params(pl, tables, status);
  p.sim_spec = sim_spectra;
  p.n_sims = n_sims;
  p.pat_terms = pat_terms;
  p.n_pats = n_pats;
  p.index_base = index_base;
  p.keys = keys;
  const int pp = pl.pp_tm > 0 ? pl.pp_tm : pl.pp;
  const int64_t passes = (n_sims + pp - 1) / pp;
  p.slices = (int)std::max<int64_t>(1, std::min<int64_t>(passes, sm_count() / std::max(1, n_pats)));
  const int64_t grid = (int64_t)n_pats * p.slices;
  EBSD_ARG_CHECK(grid < INT32_MAX, "too many patterns");
  cudaStream_t s = as_stream(stream);
  if (pl.pp_tm > 0) {
    p.pp_tm = pl.pp_tm;
    p.buf_rows = pl.pp_tm * pl.g.RW;
    p.buf_planes = pl.g.KPA;
    p.buf_bytes = p.buf_rows * 128 * p.buf_planes;
    switch (pl.cpt) {
#define EBSD_XC_TM_CASE(CPT)                                                                                       \
  case CPT:                                                                                                         \
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_xc_max_tm<CPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, pl.smem_tm)); \
    k_xc_max_tm<CPT><<<(int)grid, THREADS, pl.smem_tm, s>>>(p);                                                     \
    break;
      EBSD_XC_TM_CASE(1)
      EBSD_XC_TM_CASE(2)
      EBSD_XC_TM_CASE(3)
      EBSD_XC_TM_CASE(4)
#undef EBSD_XC_TM_CASE
      default:
        set_error("internal: no kernel for %d column chunks per thread", pl.cpt);
        return EBSD_ERR_ARG;
    }
    EBSD_LAUNCH_CHECK();
    return 0;
  }
  switch (pl.pos) {
#define EBSD_XC_CASE(POS)                                                                                         \
  case POS:                                                                                                        \
    EBSD_CUDA_CHECK(cudaFuncSetAttribute(k_xc_max<POS>, cudaFuncAttributeMaxDynamicSharedMemorySize, pl.smem_inv)); \
    k_xc_max<POS><<<(int)grid, THREADS, pl.smem_inv, s>>>(p);                                                      \
    break;
    EBSD_XC_CASE(8)
    EBSD_XC_CASE(16)
    EBSD_XC_CASE(32)
#undef EBSD_XC_CASE
    default:
      set_error("internal: no kernel for %d shifts per thread", pl.pos);
      return EBSD_ERR_ARG;
  }
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_pcfit_fold(unsigned long long* keys, int64_t n, float* best, int64_t* best_idx, void* stream) {
  EBSD_ARG_CHECK(keys && best && best_idx, "ebsd_pcfit_fold: null pointer");
  EBSD_ARG_CHECK(n >= 0, "bad count");
  if (n == 0) return 0;
  k_xc_fold<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(keys, n, best, best_idx);
  EBSD_LAUNCH_CHECK();
  return 0;
}
