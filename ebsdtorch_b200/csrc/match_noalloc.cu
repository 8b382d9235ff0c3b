// Allocation-free variant of the dictionary match (ebsd_match_topk followed by
// ebsd_merge_rescore without re-scoring).
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// index patterns, for example a detector-acquisition callback that must never
// block (cudaMalloc and cudaFree can synchronise the device), or a host
// application that owns all device memory and does not let its plugins
// allocate. They still pass their own inputs and outputs; the only scratch the
// match needs, the per-range candidate lists and a status word, lives in the
// file-scope device array below.
//
// The array is kNoAllocScratchBytes (32 MiB) on every GPU that loads this
// library and stays allocated until the process exits. Every call on a device
// uses the same array and leaves its last contents there; the status word is
// cleared at the start of each call and the candidate lists are overwritten
// completely. Calls that overlap on the GPU (different streams, or different
// host threads on the same device) race on the array and must be serialised
// by the caller.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace ebsd {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr size_t kNoAllocStatusBytes = 256;  // status word, padded for alignment
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device. In host code the symbol is
// only a host-side stand-in, so the address is looked up once per device,
// with that device current, and cached. The cache is keyed by device ordinal
// and is valid for the runtime's primary context only: a cudaDeviceReset, or
// a caller running on another driver context, would leave a stale address.
// The first lookup may load the module (lazy loading), which allocates the
// array; callers make one warm-up call at set-up time.
static void* g_scratch_addr[kMaxDevices] = {nullptr};
static std::mutex g_scratch_mu;

static int scratch_address(void** out) {
  int dev = 0;
  EBSD_CUDA_CHECK(cudaGetDevice(&dev));
  EBSD_ARG_CHECK(dev >= 0 && dev < kMaxDevices, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    EBSD_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_match_topk_noalloc(const void* queries_lp, int64_t n_queries, int64_t n_queries_pad,
                                       const void* dict_lp, int64_t n_dict_pad, int64_t n_dict_valid,
                                       int64_t k_pad, int lp_dtype, const float* col_scale,
                                       const float* q_scale, int k_out, float* out_val, int64_t* out_idx,
                                       int* out_status, void* stream) {
  EBSD_ARG_CHECK(k_out >= 1 && k_out <= 64, "k_out %d outside [1, 64]", k_out);
  EBSD_ARG_CHECK(n_queries >= 1 && n_queries <= n_queries_pad, "n_queries out of range");
  EBSD_ARG_CHECK(out_val && out_idx, "null output");
  int n_cand = 1;
  while (n_cand < k_out) n_cand <<= 1;
  const size_t per_query_slot = (size_t)n_cand * (sizeof(float) + sizeof(int32_t));
  const size_t cap = kNoAllocScratchBytes - kNoAllocStatusBytes;
  EBSD_ARG_CHECK(n_queries_pad > 0 && (size_t)n_queries_pad * per_query_slot <= cap,
                 "ebsd_match_topk_noalloc: %lld padded queries x %d candidates need %zu bytes of scratch; "
                 "the fixed scratch holds %zu (at most %zu padded queries for this k)",
                 (long long)n_queries_pad, n_cand, (size_t)n_queries_pad * per_query_slot, cap,
                 cap / per_query_slot);
  int splits = std::min(ebsd_match_auto_splits_typed(n_queries_pad, n_dict_pad, lp_dtype), 4096 / n_cand);
  while (splits > 1 && (size_t)n_queries_pad * splits * per_query_slot > cap) --splits;

  void* base = nullptr;
  if (int rc = scratch_address(&base)) return rc;
  int* status = reinterpret_cast<int*>(base);
  float* part_val = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + kNoAllocStatusBytes);
  int32_t* part_idx = reinterpret_cast<int32_t*>(part_val + (size_t)n_queries_pad * splits * n_cand);
  cudaStream_t s = as_stream(stream);
  EBSD_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int), s));
  if (int rc = ebsd_match_topk(queries_lp, n_queries_pad, dict_lp, n_dict_pad, n_dict_valid, k_pad, lp_dtype,
                               col_scale, n_cand, splits, part_val, part_idx, splits, 0, 0, status, stream))
    return rc;
  if (int rc = ebsd_merge_rescore(part_val, part_idx, n_queries, splits, n_cand, nullptr, 0, nullptr, 0, 0, 1, 0,
                                  nullptr, nullptr, q_scale, EBSD_SIM_DOT, std::min(n_cand * splits, 128), k_out,
                                  nullptr, nullptr, out_val, out_idx, stream))
    return rc;
  if (out_status) EBSD_CUDA_CHECK(cudaMemcpyAsync(out_status, status, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return 0;
}
