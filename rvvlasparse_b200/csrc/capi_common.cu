// capi_common.cu — status strings, per-thread error text, launch counter and
// device queries shared by every entry point.
#include <cstdio>
#include <mutex>
#include <vector>

#include "rvvla_internal.cuh"

namespace rvvla {

static thread_local std::string t_last_error;
static std::atomic<uint64_t> g_launches{0};

void set_error(const std::string& msg) { t_last_error = msg; }

int fail(int status, const std::string& msg) {
  t_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* where) {
  t_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return RVVLA_ERR_CUDA;
}

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// One int per device that kernels with bounded waits set when a wait expires.
int* device_status_word() {
  static std::mutex mu;
  static std::vector<int*> words;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)words.size() <= dev) words.resize((size_t)dev + 1, nullptr);
  if (!words[(size_t)dev]) {
    int* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) return nullptr;
    words[(size_t)dev] = p;
  }
  return words[(size_t)dev];
}

int sm_count() {
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize((size_t)dev + 1, 0);
  if (cache[(size_t)dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[(size_t)dev] = n;
  }
  return cache[(size_t)dev];
}

}  // namespace rvvla

extern "C" {

const char* rvvla_version(void) { return "rvvlasparse-b200 0.1 (sm_100a)"; }

const char* rvvla_status_string(int s) {
  switch (s) {
    case RVVLA_OK: return "ok";
    case RVVLA_ERR_INVALID_ARG: return "invalid argument";
    case RVVLA_ERR_CUDA: return "CUDA error";
    case RVVLA_ERR_FORMAT: return "malformed format";
    case RVVLA_ERR_UNSUPPORTED: return "unsupported";
    case RVVLA_ERR_TOO_LARGE: return "too large";
    case RVVLA_ERR_TIMEOUT: return "device wait timed out";
    case RVVLA_ERR_NO_DEVICE: return "no CUDA device";
    case RVVLA_ERR_IO: return "file input/output error";
    default: return "unknown status";
  }
}

const char* rvvla_last_error(void) { return rvvla::t_last_error.c_str(); }

int rvvla_device_info(int* cc_major, int* cc_minor, int* sms) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return rvvla::fail(RVVLA_ERR_NO_DEVICE, "no CUDA device visible");
  }
  int dev = 0;
  RVVLA_CUDA(cudaGetDevice(&dev));
  int a = 0, b = 0, c = 0;
  RVVLA_CUDA(cudaDeviceGetAttribute(&a, cudaDevAttrComputeCapabilityMajor, dev));
  RVVLA_CUDA(cudaDeviceGetAttribute(&b, cudaDevAttrComputeCapabilityMinor, dev));
  RVVLA_CUDA(cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev));
  if (cc_major) *cc_major = a;
  if (cc_minor) *cc_minor = b;
  if (sms) *sms = c;
  return RVVLA_OK;
}

uint64_t rvvla_kernel_launch_count(void) { return rvvla::g_launches.load(); }

int rvvla_device_status(int* code, void* stream) {
  if (!code) return rvvla::fail(RVVLA_ERR_INVALID_ARG, "rvvla_device_status: null code");
  *code = 0;
  int* w = rvvla::device_status_word();
  if (!w) return rvvla::fail(RVVLA_ERR_CUDA, "rvvla_device_status: no status word");
  cudaStream_t st = rvvla::as_stream(stream);
  RVVLA_CUDA(cudaStreamSynchronize(st));
  RVVLA_CUDA(cudaMemcpy(code, w, sizeof(int), cudaMemcpyDeviceToHost));
  RVVLA_CUDA(cudaMemset(w, 0, sizeof(int)));
  return *code ? RVVLA_ERR_TIMEOUT : RVVLA_OK;
}

int rvvla_malloc(void** ptr, size_t bytes) {
  if (!ptr) return rvvla::fail(RVVLA_ERR_INVALID_ARG, "rvvla_malloc: null pointer");
  *ptr = nullptr;
  if (bytes == 0) return RVVLA_OK;
  RVVLA_CUDA(cudaMalloc(ptr, bytes));
  return RVVLA_OK;
}

int rvvla_free(void* ptr) {
  if (ptr) RVVLA_CUDA(cudaFree(ptr));
  return RVVLA_OK;
}

int rvvla_memcpy(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return RVVLA_OK;
  if (!dst || !src) return rvvla::fail(RVVLA_ERR_INVALID_ARG, "rvvla_memcpy: null pointer");
  cudaStream_t st = rvvla::as_stream(stream);
  RVVLA_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // extern "C"
