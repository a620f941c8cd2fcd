// host_stager.cpp -- see host_stager.h.
#include "host_stager.h"

#include <algorithm>
#include <cstring>

namespace eb2 {

// ------------------------------------------------------------------ CopyPool
CopyPool::CopyPool(int workers) {
  for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { work(); });
  for (auto& t : threads_) t.detach();  // the pool lives until the process exits
}

// A worker joins a generation under the lock (active_) and leaves it under the lock, so run()
// returns only when no worker can still be running that generation's job: a late worker sees
// either the finished job's null pointer or the next generation, never a stale job.
void CopyPool::work() {
  uint64_t seen = 0;
  for (;;) {
    const std::function<void(int)>* job;
    int n;
    {
      std::unique_lock<std::mutex> lock(mu_);
      start_cv_.wait(lock, [&] { return generation_ != seen; });
      seen = generation_;
      job = job_;
      n = n_;
      if (!job) continue;
      ++active_;
    }
    int done = 0;
    for (int i; (i = next_.fetch_add(1)) < n;) {
      (*job)(i);
      ++done;
    }
    {
      std::lock_guard<std::mutex> lock(mu_);
      remaining_ -= done;
      --active_;
      if (remaining_ == 0 && active_ == 0) done_cv_.notify_all();
    }
  }
}

void CopyPool::run(int n, const std::function<void(int)>& fn) {
  if (n <= 0) return;
  if (threads_.empty() || n == 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  {
    std::lock_guard<std::mutex> lock(mu_);
    job_ = &fn;
    n_ = n;
    remaining_ = n;
    next_ = 0;
    ++generation_;
  }
  start_cv_.notify_all();
  int done = 0;
  for (int i; (i = next_.fetch_add(1)) < n;) {
    fn(i);
    ++done;
  }
  std::unique_lock<std::mutex> lock(mu_);
  remaining_ -= done;
  done_cv_.wait(lock, [&] { return remaining_ == 0 && active_ == 0; });
  job_ = nullptr;
}

// ------------------------------------------------------------------ HostStager
bool HostStager::pinned(const void* p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

cudaError_t HostStager::init() {
  if (ready_) return cudaSuccess;
  for (Buffer* ring : {in_, out_}) {
    const int count = ring == in_ ? kInBuffers : kOutBuffers;
    for (int i = 0; i < count; ++i) {
      if (!ring[i].ptr) {
        cudaError_t e = cudaHostAlloc(&ring[i].ptr, kChunkBytes, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
      }
      if (!ring[i].done) {
        cudaError_t e = cudaEventCreateWithFlags(&ring[i].done, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
      }
    }
  }
  const unsigned hc = std::thread::hardware_concurrency();
  // a few memcpy threads: host memory bandwidth, not core count, bounds the copies
  pool_ = new CopyPool(int(std::clamp(hc / 2, 1u, 8u)) - 1);
  ready_ = true;
  return cudaSuccess;
}

// `height` rows of `width` bytes, split over the pool by rows
void HostStager::copy_rows(char* dst, size_t dpitch, const char* src, size_t spitch, size_t width, size_t height) {
  const int parts = int(std::min<size_t>(height, size_t(pool_->threads()) * 2));
  pool_->run(parts, [&](int p) {
    const size_t r0 = height * size_t(p) / size_t(parts), r1 = height * size_t(p + 1) / size_t(parts);
    if (dpitch == width && spitch == width) {
      std::memcpy(dst + r0 * width, src + r0 * width, (r1 - r0) * width);
    } else {
      for (size_t r = r0; r < r1; ++r) std::memcpy(dst + r * dpitch, src + r * spitch, width);
    }
  });
}

cudaError_t HostStager::to_device(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                                  size_t height, cudaStream_t st) {
  if (width == 0 || height == 0) return cudaSuccess;
  if (pinned(src)) return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyHostToDevice, st);
  if (cudaError_t e = init(); e != cudaSuccess) return e;
  if (width > kChunkBytes)  // one row larger than a bounce buffer: the runtime's own staging
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyHostToDevice, st);
  const size_t rows_per_chunk = kChunkBytes / width;
  for (size_t r0 = 0; r0 < height; r0 += rows_per_chunk) {
    const size_t h = std::min(rows_per_chunk, height - r0);
    Buffer& b = in_[next_in_];
    next_in_ = (next_in_ + 1) % kInBuffers;
    if (b.busy) {  // its previous chunk must have reached the device
      if (cudaError_t e = cudaEventSynchronize(b.done); e != cudaSuccess) return e;
      b.busy = false;
    }
    copy_rows(static_cast<char*>(b.ptr), width, static_cast<const char*>(src) + r0 * spitch, spitch, width, h);
    cudaError_t e = cudaMemcpy2DAsync(static_cast<char*>(dst) + r0 * dpitch, dpitch, b.ptr, width, width, h,
                                      cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(b.done, st);
    if (e != cudaSuccess) return e;
    b.busy = true;
  }
  return cudaSuccess;
}

cudaError_t HostStager::finish_out(const OutChunk& c) {
  Buffer& b = out_[c.buf];
  if (cudaError_t e = cudaEventSynchronize(b.done); e != cudaSuccess) return e;
  copy_rows(c.dst, c.dpitch, static_cast<const char*>(b.ptr), c.width, c.width, c.height);
  b.busy = false;
  return cudaSuccess;
}

cudaError_t HostStager::to_host(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                                size_t height, cudaStream_t st) {
  if (width == 0 || height == 0) return cudaSuccess;
  if (pinned(dst)) return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = init(); e != cudaSuccess) return e;
  if (width > kChunkBytes) {
    if (cudaError_t e = drain(); e != cudaSuccess) return e;
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost, st);
  }
  const size_t rows_per_chunk = kChunkBytes / width;
  for (size_t r0 = 0; r0 < height; r0 += rows_per_chunk) {
    const size_t h = std::min(rows_per_chunk, height - r0);
    Buffer& b = out_[next_out_];
    if (b.busy) {  // the oldest pending chunk is in this buffer (FIFO over the ring)
      const OutChunk c = pending_.front();
      pending_.pop_front();
      if (cudaError_t e = finish_out(c); e != cudaSuccess) return e;
    }
    cudaError_t e = cudaMemcpy2DAsync(b.ptr, width, static_cast<const char*>(src) + r0 * spitch, spitch, width, h,
                                      cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(b.done, st);
    if (e != cudaSuccess) return e;
    b.busy = true;
    pending_.push_back(OutChunk{next_out_, static_cast<char*>(dst) + r0 * dpitch, dpitch, width, h});
    next_out_ = (next_out_ + 1) % kOutBuffers;
  }
  return cudaSuccess;
}

cudaError_t HostStager::progress() {
  while (!pending_.empty()) {
    const cudaError_t q = cudaEventQuery(out_[pending_.front().buf].done);
    if (q == cudaErrorNotReady) {
      (void)cudaGetLastError();
      return cudaSuccess;
    }
    if (q != cudaSuccess) return q;
    const OutChunk c = pending_.front();
    pending_.pop_front();
    if (cudaError_t e = finish_out(c); e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t HostStager::drain() {
  while (!pending_.empty()) {
    const OutChunk c = pending_.front();
    pending_.pop_front();
    if (cudaError_t e = finish_out(c); e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace eb2
