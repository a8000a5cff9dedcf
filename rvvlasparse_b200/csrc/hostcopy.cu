// hostcopy.cu — copies between pageable host memory (a caller's
// std::vector, a numpy array) and the device through the library's pinned
// staging buffers.
//
// A DMA can only read or write page-locked memory, so a pageable copy is
// always staged.  Here it is staged in chunks of kStageBytes through
// kStageBufs page-locked buffers per device: the host side of chunk i (a
// memcpy split across up to kCopyThreads OpenMP threads) overlaps the DMA of
// chunk i-1, so a copy runs at the slower of the host memcpy and the PCIe
// link instead of their sum.  The staging buffers are allocated on the first
// large copy on each device and kept until exit; calls on one device are
// serialised by a mutex (the buffers are shared).
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

constexpr size_t kStageBytes = (size_t)4 << 20;
constexpr int kStageBufs = 3;
constexpr int kCopyThreads = 8;
constexpr size_t kSmallCopy = (size_t)256 << 10;  // below this, one plain copy
constexpr int kMaxDevices = 64;

struct Staging {
  std::mutex mu;
  char* buf[kStageBufs] = {};
  cudaEvent_t done[kStageBufs] = {};  // the DMA that last used buf[i] has finished
  bool ready = false;
};

Staging g_staging[kMaxDevices];

int staging_for_current_device(Staging** out) {
  int dev = 0;
  RVVLA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(RVVLA_ERR_UNSUPPORTED, "host copy: device ordinal beyond 63");
  *out = &g_staging[dev];
  return RVVLA_OK;
}

// caller holds s.mu
int staging_init(Staging& s) {
  if (s.ready) return RVVLA_OK;
  for (int i = 0; i < kStageBufs; ++i) {
    RVVLA_CUDA(cudaHostAlloc((void**)&s.buf[i], kStageBytes, cudaHostAllocDefault));
    RVVLA_CUDA(cudaEventCreateWithFlags(&s.done[i], cudaEventDisableTiming));
  }
  s.ready = true;
  return RVVLA_OK;
}

// memcpy of one chunk, split across threads when it is large enough to pay
void chunk_copy(char* dst, const char* src, size_t n) {
  const int nt = (int)std::min<size_t>(kCopyThreads, std::max<size_t>(1, n >> 19));  // >= 512 KB a thread
  if (nt <= 1) {
    std::memcpy(dst, src, n);
    return;
  }
  const size_t per = (n + nt - 1) / nt;
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t) {
    const size_t a = (size_t)t * per, b = std::min(n, a + per);
    if (a < b) std::memcpy(dst + a, src + a, b - a);
  }
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_copy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return RVVLA_OK;
  if (!dst || !src) return fail(RVVLA_ERR_INVALID_ARG, "rvvla_copy_h2d: null pointer");
  cudaStream_t st = as_stream(stream);
  if (bytes <= kSmallCopy) {
    RVVLA_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return RVVLA_OK;
  }
  Staging* s = nullptr;
  int rc = staging_for_current_device(&s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(s->mu);
  rc = staging_init(*s);
  if (rc) return rc;
  const char* h = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  int i = 0;
  for (size_t off = 0; off < bytes; off += kStageBytes, ++i) {
    const int b = i % kStageBufs;
    const size_t n = std::min(kStageBytes, bytes - off);
    RVVLA_CUDA(cudaEventSynchronize(s->done[b]));  // the buffer's previous DMA has read it
    chunk_copy(s->buf[b], h + off, n);
    RVVLA_CUDA(cudaMemcpyAsync(d + off, s->buf[b], n, cudaMemcpyHostToDevice, st));
    RVVLA_CUDA(cudaEventRecord(s->done[b], st));
  }
  return RVVLA_OK;
}

int rvvla_copy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return RVVLA_OK;
  if (!dst || !src) return fail(RVVLA_ERR_INVALID_ARG, "rvvla_copy_d2h: null pointer");
  cudaStream_t st = as_stream(stream);
  if (bytes <= kSmallCopy) {
    RVVLA_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    return RVVLA_OK;
  }
  Staging* s = nullptr;
  int rc = staging_for_current_device(&s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(s->mu);
  rc = staging_init(*s);
  if (rc) return rc;
  char* h = static_cast<char*>(dst);
  const char* d = static_cast<const char*>(src);
  const size_t nch = (bytes + kStageBytes - 1) / kStageBytes;
  auto issue = [&](size_t c) -> int {
    const int b = (int)(c % kStageBufs);
    const size_t off = c * kStageBytes, n = std::min(kStageBytes, bytes - off);
    RVVLA_CUDA(cudaEventSynchronize(s->done[b]));  // an earlier DMA (either direction) may still use it
    RVVLA_CUDA(cudaMemcpyAsync(s->buf[b], d + off, n, cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaEventRecord(s->done[b], st));
    return RVVLA_OK;
  };
  for (size_t c = 0; c < std::min<size_t>(nch, kStageBufs); ++c)
    if ((rc = issue(c))) return rc;
  for (size_t c = 0; c < nch; ++c) {
    const int b = (int)(c % kStageBufs);
    const size_t off = c * kStageBytes, n = std::min(kStageBytes, bytes - off);
    RVVLA_CUDA(cudaEventSynchronize(s->done[b]));
    chunk_copy(h + off, s->buf[b], n);
    if (c + kStageBufs < nch && (rc = issue(c + kStageBufs))) return rc;
  }
  return RVVLA_OK;
}

}  // extern "C"
