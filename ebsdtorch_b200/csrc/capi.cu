// Library-level entry points: version, error reporting, device check,
// row gather and b x b average pooling.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace ebsd {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

struct CheckWord {
  const void* symbol;
  const char* file;
};

static std::vector<CheckWord>& check_words() {
  static std::vector<CheckWord> words;
  return words;
}

int register_check_word(const void* symbol, const char* file) {
  check_words().push_back({symbol, file});
  return 0;
}

int device_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
  return n > 0 ? n : 148;
}

__global__ void k_gather_rows(const float* __restrict__ in, int64_t n_in, int width,
                              const int64_t* __restrict__ index, int64_t n_out,
                              float* __restrict__ out) {
  const int64_t total = n_out * width;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / width, c = t - r * width;
    const int64_t src = index[r];
    out[t] = (src >= 0 && src < n_in) ? in[src * width + c] : nanf("");
  }
}

__global__ void k_avg_pool(const float* __restrict__ in, int64_t n, int h, int w, int b,
                           float* __restrict__ out) {
  const int hb = h / b, wb = w / b;
  const int64_t total = n * hb * wb;
  const float cnt = (float)(b * b);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t img = t / (hb * wb);
    const int rem = (int)(t - img * hb * wb);
    const int i = rem / wb, j = rem - i * wb;
    const float* src = in + img * (int64_t)h * w + (int64_t)(i * b) * w + j * b;
    float s = 0.f;
    for (int a = 0; a < b; ++a)
      for (int c = 0; c < b; ++c) s += src[(int64_t)a * w + c];
    out[t] = s / cnt;
  }
}

}  // namespace ebsd

using namespace ebsd;

extern "C" int ebsd_version(void) { return 100; }

extern "C" int ebsd_debug_check_line(char* file, size_t n) {
#ifdef EBSD_CHECK
  int found = 0;
  for (const CheckWord& w : check_words()) {
    int line = 0;
    EBSD_CUDA_CHECK(cudaMemcpyFromSymbol(&line, w.symbol, sizeof(int)));
    if (line != 0) {
      const int zero = 0;
      EBSD_CUDA_CHECK(cudaMemcpyToSymbol(w.symbol, &zero, sizeof(int)));
      if (found == 0) {
        found = line;
        if (file && n) {
          strncpy(file, w.file, n - 1);
          file[n - 1] = 0;
        }
      }
    }
  }
  return found;
#else
  (void)file;
  (void)n;
  return -1;  // built without checks
#endif
}

extern "C" int ebsd_last_error(char* buf, size_t n) {
  if (buf && n) {
    strncpy(buf, g_last_error.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return (int)g_last_error.size();
}

extern "C" int ebsd_device_check(int device) {
  cudaDeviceProp p;
  EBSD_CUDA_CHECK(cudaGetDeviceProperties(&p, device));
  if (p.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a only", device, p.major,
              p.minor);
    return EBSD_ERR_UNSUPPORTED;
  }
  return 0;
}

extern "C" int ebsd_gather_rows(const float* in, int64_t n_in, int width, const int64_t* index,
                                int64_t n_out, float* out, void* stream) {
  EBSD_ARG_CHECK(in && index && out, "ebsd_gather_rows: null pointer");
  EBSD_ARG_CHECK(width > 0 && n_in >= 0 && n_out >= 0, "ebsd_gather_rows: bad sizes");
  if (n_out == 0) return 0;
  const int64_t total = n_out * width;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  k_gather_rows<<<blocks, 256, 0, as_stream(stream)>>>(in, n_in, width, index, n_out, out);
  EBSD_LAUNCH_CHECK();
  return 0;
}

extern "C" int ebsd_avg_pool(const float* in, int64_t n, int height, int width, int binning,
                             float* out, void* stream) {
  EBSD_ARG_CHECK(in && out, "ebsd_avg_pool: null pointer");
  EBSD_ARG_CHECK(binning >= 1 && height >= binning && width >= binning && n >= 0,
                 "ebsd_avg_pool: bad sizes (h=%d w=%d b=%d)", height, width, binning);
  if (n == 0) return 0;
  const int64_t total = n * (height / binning) * (width / binning);
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  k_avg_pool<<<blocks, 256, 0, as_stream(stream)>>>(in, n, height, width, binning, out);
  EBSD_LAUNCH_CHECK();
  return 0;
}
