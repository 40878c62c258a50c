// Staged host <-> device copies (see hostcopy.hpp).
#include "hostcopy.hpp"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "devutil.hpp"

namespace gnufft
{
namespace
{
constexpr size_t kChunk = 8u << 20;   // bytes per staging buffer
constexpr size_t kSmall = 16u << 20;  // below: one plain copy
constexpr int kCopyThreads = 4;       // host threads per chunk
constexpr int kMaxDevices = 64;

struct Ring
{
  std::mutex m;  // one staged copy at a time per device
  bool tried = false, ok = false;
  char *buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

std::mutex g_init;  // guards the rings' allocation
Ring g_rings[kMaxDevices];

// The current device's ring, allocated on first use and kept for the
// process (pinned allocations are slow, ~15 ms).  Null if it cannot be
// had: the caller copies without staging.
Ring *ring()
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return nullptr;
  Ring &r = g_rings[dev];
  std::lock_guard<std::mutex> lock(g_init);
  if (!r.tried)
  {
    r.tried = true;
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b)
      ok = cudaHostAlloc(reinterpret_cast<void **>(&r.buf[b]), kChunk,
                         cudaHostAllocDefault) == cudaSuccess &&
           cudaEventCreateWithFlags(&r.ev[b], cudaEventDisableTiming) ==
               cudaSuccess;
    if (!ok)
    {
      cudaGetLastError();  // clear the failed allocation's status
      for (int b = 0; b < 2; ++b)
      {
        if (r.buf[b])
          cudaFreeHost(r.buf[b]);
        if (r.ev[b])
          cudaEventDestroy(r.ev[b]);
        r.buf[b] = nullptr;
        r.ev[b] = nullptr;
      }
    }
    r.ok = ok;
  }
  return r.ok ? &r : nullptr;
}

// memcpy of len bytes split over kCopyThreads threads (the caller's one
// of them; parts whose thread cannot be started are copied by the caller).
void parallel_copy(char *dst, const char *src, size_t len)
{
  const size_t part = (len + kCopyThreads - 1) / kCopyThreads;
  auto copy_part = [=](int k) {
    const size_t o = (size_t)k * part;
    if (o < len)
      std::memcpy(dst + o, src + o, std::min(part, len - o));
  };
  std::vector<std::thread> th;
  int k = 1;
  for (; k < kCopyThreads && (size_t)k * part < len; ++k)
  {
    try
    {
      th.emplace_back(copy_part, k);
    }
    catch (...)
    {
      break;  // no more threads: the rest below, on this one
    }
  }
  for (int q = k; q < kCopyThreads; ++q)
    copy_part(q);
  copy_part(0);
  for (auto &t : th)
    t.join();
}
}  // namespace

void copy_host_to_device(void *dst, const void *src, size_t bytes,
                         cudaStream_t s)
{
  if (!bytes)
    return;
  Ring *r = bytes >= kSmall ? ring() : nullptr;
  if (!r)
  {
    GN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  std::lock_guard<std::mutex> lock(r->m);
  char *d = static_cast<char *>(dst);
  const char *h = static_cast<const char *>(src);
  for (size_t off = 0, i = 0; off < bytes; off += kChunk, ++i)
  {
    const int b = (int)(i & 1);
    const size_t len = std::min(kChunk, bytes - off);
    GN_CUDA(cudaEventSynchronize(r->ev[b]));  // its previous copy is done
    parallel_copy(r->buf[b], h + off, len);
    GN_CUDA(cudaMemcpyAsync(d + off, r->buf[b], len, cudaMemcpyHostToDevice,
                            s));
    GN_CUDA(cudaEventRecord(r->ev[b], s));
  }
}

void copy_device_to_host(void *dst, const void *src, size_t bytes,
                         cudaStream_t s)
{
  if (!bytes)
    return;
  Ring *r = bytes >= kSmall ? ring() : nullptr;
  if (!r)
  {
    GN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    GN_CUDA(cudaStreamSynchronize(s));
    return;
  }
  std::lock_guard<std::mutex> lock(r->m);
  char *h = static_cast<char *>(dst);
  const char *d = static_cast<const char *>(src);
  size_t prev_off = 0, prev_len = 0;
  int prev_b = -1;
  for (size_t off = 0, i = 0; off < bytes; off += kChunk, ++i)
  {
    const int b = (int)(i & 1);
    const size_t len = std::min(kChunk, bytes - off);
    // buffer b: its earlier chunk was copied out below (this thread), and
    // any copy of another call into it has finished
    GN_CUDA(cudaEventSynchronize(r->ev[b]));
    GN_CUDA(cudaMemcpyAsync(r->buf[b], d + off, len, cudaMemcpyDeviceToHost,
                            s));
    GN_CUDA(cudaEventRecord(r->ev[b], s));
    if (prev_b >= 0)
    {  // the previous chunk out of its buffer while this one is copied
      GN_CUDA(cudaEventSynchronize(r->ev[prev_b]));
      parallel_copy(h + prev_off, r->buf[prev_b], prev_len);
    }
    prev_off = off;
    prev_len = len;
    prev_b = b;
  }
  GN_CUDA(cudaEventSynchronize(r->ev[prev_b]));
  parallel_copy(h + prev_off, r->buf[prev_b], prev_len);
}

}  // namespace gnufft
