// host_stager.h -- copies between host memory and the device for the BLAS entry points.
//
// Pinned (page-locked) host buffers go straight to the copy engine with cudaMemcpy2DAsync.
// Ordinary pageable buffers -- what an Eigen MatrixXd, a malloc'd Fortran array or a numpy
// array is -- would make the runtime stage every copy through its own small pinned buffer,
// synchronously with the calling thread.  Here they go through a ring of pinned bounce
// buffers instead: host threads copy a chunk of whole columns into a free bounce buffer
// while the copy engine moves the chunks before it, one cudaMemcpy2DAsync per chunk.  The
// device -> host direction is the mirror image: chunks land in bounce buffers and host
// threads copy them out once their event has completed, while later chunks are in flight.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace eb2 {

// fn(i) for i in [0, n) on a few persistent worker threads plus the calling thread.
class CopyPool {
 public:
  explicit CopyPool(int workers);
  CopyPool(const CopyPool&) = delete;
  CopyPool& operator=(const CopyPool&) = delete;
  // Returns when every fn(i) has returned.  Not reentrant (one caller at a time).
  void run(int n, const std::function<void(int)>& fn);
  int threads() const { return int(threads_.size()) + 1; }

 private:
  void work();
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable start_cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0, remaining_ = 0, active_ = 0;
  uint64_t generation_ = 0;
  std::atomic<int> next_{0};
};

class HostStager {
 public:
  static constexpr size_t kChunkBytes = size_t(16) << 20;
  static constexpr int kInBuffers = 6, kOutBuffers = 4;

  // True if p is host memory the copy engine can read directly (pinned or registered).
  static bool pinned(const void* p);

  // dst (device, pitch dpitch) <- src (host, pitch spitch): `height` rows of `width` bytes,
  // enqueued on `st`.  Pageable sources are copied into bounce buffers first; the call
  // returns once every chunk is enqueued (the host side of the copy is done).
  cudaError_t to_device(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                        cudaStream_t st);
  // dst (host) <- src (device) after the work already on `st`.  Pageable destinations go
  // through bounce buffers: the copies are enqueued now and land in dst by progress() /
  // drain(); dst must stay untouched until drain() returns.
  cudaError_t to_host(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                      cudaStream_t st);
  // Copies out the device -> host chunks whose transfers have completed (non-blocking).
  cudaError_t progress();
  // Waits for and copies out every pending device -> host chunk.
  cudaError_t drain();

 private:
  struct Buffer {
    void* ptr = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
  };
  struct OutChunk {
    int buf;
    char* dst;
    size_t dpitch, width, height;
  };
  cudaError_t init();
  cudaError_t finish_out(const OutChunk& c);
  void copy_rows(char* dst, size_t dpitch, const char* src, size_t spitch, size_t width, size_t height);

  bool ready_ = false;
  CopyPool* pool_ = nullptr;
  Buffer in_[kInBuffers], out_[kOutBuffers];
  int next_in_ = 0, next_out_ = 0;
  std::deque<OutChunk> pending_;
};

}  // namespace eb2
