// context.h -- per-device state of the library: the stream BLAS calls run on,
// grow-only device workspaces, the small device/pinned flag block the kernels
// report through, and the thread-local error / call-info records.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

#include "eigen_b200/blas.h"
#include "host_stager.h"

namespace eb2 {

// Grow-only device allocation (never shrinks; freed at process exit).
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t cap = 0;
  // A CUDA graph captured a call that used `ptr`: its replays read and write that address,
  // so a later growth keeps the old allocation alive (in `retired`) instead of freeing it.
  bool held_by_graph = false;
  std::vector<void*> retired;
  // Returns false (and leaves the old buffer) if the allocation fails.
  bool ensure(size_t bytes);
};

// Sizes `buf` to at least `bytes` for a call on stream `st`.  Outside a capture it grows the
// buffer as needed (EB2_ERR_ALLOC if that fails).  In a stream capture an allocation would
// invalidate the caller's graph, so a buffer that is too small gives EB2_ERR_ARG ("make a
// direct call of this size first") before anything is enqueued, and a buffer that is large
// enough becomes held by the graph.  Sets the thread's error on failure; `what` names the
// buffer in the message.
int reserve_buffer(DeviceBuffer& buf, size_t bytes, cudaStream_t st, const char* what);

// Flags the kernels write; mirrored into pinned host memory after a call.
struct DeviceFlags {
  int nonfinite;
  uint32_t status;
  double err_sq[2];
  double spread[2];  // exponent-spread statistic of the scans: sum, count
};

struct Context {
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  cudaStream_t stream = nullptr;  // stream of the synchronous BLAS entry points
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;  // around all product kernels
  cudaEvent_t ev_gemm0 = nullptr, ev_gemm1 = nullptr;  // around the main GEMM kernel
  std::mutex mu;                  // one product at a time per device
  DeviceBuffer ws;                // emulation workspace (digits, exponents, scan results)
  DeviceBuffer stage_a, stage_b, stage_c;  // device copies of host operands
  DeviceBuffer tmp;               // level-3 routines: expanded operands, diagonal-block products
  DeviceBuffer cplx;              // complex products: packed real operands and the two real results
  DeviceFlags* dflags = nullptr;  // device
  DeviceFlags* hflags = nullptr;  // pinned host mirror
  // Host-buffer pipeline of the BLAS entry (copies overlapped with the product by column
  // blocks): one stream per copy direction, events without timing, pinned estimate slots.
  static constexpr int kPipeChunks = 16;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_a = nullptr;
  cudaEvent_t ev_scan = nullptr;  // the scans' statistics have reached the host (picker stage 2)
  cudaEvent_t ev_in[kPipeChunks] = {};
  cudaEvent_t ev_done[kPipeChunks] = {};
  double* hchunk = nullptr;  // pinned [kPipeChunks][2]: per-block error-estimate energies
  // End of the last call's work on its stream (fence_armed: recorded since the last call);
  // see StreamFence.
  cudaEvent_t ev_fence = nullptr;
  bool fence_armed = false;
  // host <-> device copies of the BLAS entry points (bounce buffers for pageable memory)
  HostStager stager;
};

// The workspaces and the flag block of a context pass from one call to the next in stream
// order.  A stream-ordered call (eb2_dgemm_device without the check, eb2_sgemm_device) may
// return with its kernels still running, and the next call may come on another stream or from
// another host thread: so every call's stream first waits for the previous call's end event,
// and records its own when it is done.  Construct it with the context's mutex held.  Nothing
// is waited for or recorded on a stream that is being captured into a graph.
class StreamFence {
 public:
  StreamFence(Context& cx, cudaStream_t st);
  ~StreamFence();
  StreamFence(const StreamFence&) = delete;
  StreamFence& operator=(const StreamFence&) = delete;

 private:
  Context& cx_;
  cudaStream_t st_;
  bool active_;
};

// Context of the calling thread's current device, created on first use.
// Returns nullptr (and sets the thread's error) when no usable device exists.
Context* current_context();
// current_context() for a call enqueued on `st`: creating a device's context allocates, which
// would invalidate a stream capture, so a capture on a device that has no context yet gets
// nullptr with EB2_ERR_ARG ("make a direct call first") and nothing enqueued.
Context* context_for_stream(cudaStream_t st);

struct Settings {
  std::atomic<int> dgemm_method{EB2_METHOD_AUTO};
  std::atomic<int> sgemm_method{EB2_METHOD_AUTO};
  std::atomic<int> dgemm_slices{0};
  std::atomic<int> dgemm_moduli{0};
  std::atomic<int> sgemm_pieces{3};
  std::atomic<int> tile_n{0};
  std::atomic<double> dgemm_tol{1.1102230246251565e-16};  // 2^-53
  std::atomic<int> timing{0};
};
Settings& settings();

// Thread-local sticky error.
void set_error(int code, const char* fmt, ...);
int last_error();
const char* last_error_string();
eb2_call_info& call_info();
// The configuration class and K splits of the thread's last product (eb2_last_call_config).
struct CallConfig {
  int config = -1;
  int splits = 1;
};
CallConfig& call_config();
// The context whose events hold the calling thread's last timed call (or null);
// `gemm_timed` tells whether ev_gemm0/ev_gemm1 bracket a kernel in that call.
void set_pending_timing(Context* cx, bool gemm_timed);
// Resolves pending event times into call_info() (waits for the events).
void resolve_timing();

}  // namespace eb2
