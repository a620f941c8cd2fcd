// context.cpp -- see context.h.
#include "context.h"
#include "kernels.h"
#include "mlp.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace eb2 {

namespace {
thread_local int t_error = EB2_OK;
thread_local char t_message[512] = "";
thread_local eb2_call_info t_info = {0, 0, 0, 0, 0, 0, 0, -1.0, -1.0, -1.0, 0, 0.0};
thread_local CallConfig t_config;
thread_local Context* t_pending = nullptr;
thread_local bool t_pending_gemm = false;

constexpr int kMaxDevices = 64;
std::mutex g_ctx_mu;
Context* g_ctx[kMaxDevices] = {};
}  // namespace

SliceTuning& tuning() {
  static SliceTuning t;
  return t;
}

Settings& settings() {
  static Settings s;
  return s;
}

void set_error(int code, const char* fmt, ...) {
  t_error = code;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(t_message, sizeof(t_message), fmt, ap);
  va_end(ap);
}

int last_error() { return t_error; }
const char* last_error_string() { return t_message; }
eb2_call_info& call_info() { return t_info; }
CallConfig& call_config() { return t_config; }

void set_pending_timing(Context* cx, bool gemm_timed) {
  t_pending = cx;
  t_pending_gemm = gemm_timed;
}

void resolve_timing() {
  Context* cx = t_pending;
  if (!cx) return;
  t_pending = nullptr;
  float ms = 0.f;
  if (cudaEventSynchronize(cx->ev_stop) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  if (cudaEventElapsedTime(&ms, cx->ev_start, cx->ev_stop) == cudaSuccess) t_info.kernel_ms = ms;
  if (t_pending_gemm && cudaEventElapsedTime(&ms, cx->ev_gemm0, cx->ev_gemm1) == cudaSuccess) t_info.gemm_kernel_ms = ms;
  (void)cudaGetLastError();
}

bool DeviceBuffer::ensure(size_t bytes) {
  if (bytes <= cap) return true;
  const size_t gran = size_t(2) << 20;
  size_t want = bytes + bytes / 8;
  want = (want + gran - 1) / gran * gran;
  void* p = nullptr;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    (void)cudaGetLastError();
    want = (bytes + gran - 1) / gran * gran;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      (void)cudaGetLastError();
      return false;
    }
  }
  if (ptr) {
    if (held_by_graph)
      retired.push_back(ptr);  // a captured graph still replays into it
    else
      cudaFree(ptr);  // implicitly waits for work still using the old buffer
  }
  ptr = p;
  cap = want;
  held_by_graph = false;
  return true;
}

int reserve_buffer(DeviceBuffer& buf, size_t bytes, cudaStream_t st, const char* what) {
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &status) != cudaSuccess) {
    (void)cudaGetLastError();
    status = cudaStreamCaptureStatusNone;
  }
  if (status != cudaStreamCaptureStatusNone) {
    if (bytes > buf.cap) {
      set_error(EB2_ERR_ARG,
                "a captured call needs %zu bytes of %s, more than the %zu sized so far; make a direct call of this "
                "size first",
                bytes, what, buf.cap);
      return EB2_ERR_ARG;
    }
    buf.held_by_graph = true;
    return EB2_OK;
  }
  if (!buf.ensure(bytes)) {
    set_error(EB2_ERR_ALLOC, "could not allocate %zu bytes of %s", bytes, what);
    return EB2_ERR_ALLOC;
  }
  return EB2_OK;
}

StreamFence::StreamFence(Context& cx, cudaStream_t st) : cx_(cx), st_(st), active_(false) {
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &status) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  active_ = status == cudaStreamCaptureStatusNone;
  if (active_ && cx_.fence_armed) (void)cudaStreamWaitEvent(st_, cx_.ev_fence, 0);
}

StreamFence::~StreamFence() {
  if (!active_) return;
  if (cudaEventRecord(cx_.ev_fence, st_) == cudaSuccess)
    cx_.fence_armed = true;
  else
    (void)cudaGetLastError();
}

Context* current_context() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_NO_DEVICE, "no CUDA device is available");
    return nullptr;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_NO_DEVICE, "cudaGetDevice failed");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_ctx_mu);
  if (g_ctx[dev]) return g_ctx[dev];
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_NO_DEVICE, "cudaGetDeviceProperties failed for device %d", dev);
    return nullptr;
  }
  if (prop.major != 10 || prop.minor != 0) {
    set_error(EB2_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a (B200) only", dev,
              prop.major, prop.minor);
    return nullptr;
  }
  Context* c = new Context();
  c->device = dev;
  c->num_sms = prop.multiProcessorCount;
  c->cc_major = prop.major;
  c->cc_minor = prop.minor;
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaEventCreate(&c->ev_start) == cudaSuccess;
  ok = ok && cudaEventCreate(&c->ev_stop) == cudaSuccess;
  ok = ok && cudaEventCreate(&c->ev_gemm0) == cudaSuccess;
  ok = ok && cudaEventCreate(&c->ev_gemm1) == cudaSuccess;
  ok = ok && cudaMalloc(&c->dflags, sizeof(DeviceFlags)) == cudaSuccess;
  ok = ok && cudaHostAlloc(&c->hflags, sizeof(DeviceFlags), cudaHostAllocDefault) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&c->ev_a, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&c->ev_fence, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&c->ev_scan, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < Context::kPipeChunks && ok; ++i) {
    ok = cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming) == cudaSuccess;
  }
  ok = ok && cudaHostAlloc(&c->hchunk, sizeof(double) * 2 * Context::kPipeChunks, cudaHostAllocDefault) ==
                 cudaSuccess;
  if (!ok) {
    set_error(EB2_ERR_CUDA, "creating the device context failed: %s", cudaGetErrorString(cudaGetLastError()));
    delete c;  // the few handles that were created are reclaimed at process exit
    return nullptr;
  }
  std::memset(c->hflags, 0, sizeof(DeviceFlags));
  g_ctx[dev] = c;
  static std::once_flag picker_once;
  std::call_once(picker_once, [&] { picker_autoload(c->num_sms); });
  return c;
}

Context* context_for_stream(cudaStream_t st) {
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &status) != cudaSuccess) {
    (void)cudaGetLastError();
    status = cudaStreamCaptureStatusNone;
  }
  if (status != cudaStreamCaptureStatusNone) {
    int dev = -1;
    bool exists = false;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices) {
      std::lock_guard<std::mutex> lock(g_ctx_mu);
      exists = g_ctx[dev] != nullptr;
    } else {
      (void)cudaGetLastError();
    }
    if (!exists) {
      set_error(EB2_ERR_ARG,
                "the first call on a device creates its context (allocations) and cannot be captured; make a "
                "direct call first");
      return nullptr;
    }
  }
  return current_context();
}

}  // namespace eb2

extern "C" const char* eb2_last_error_string(void) { return eb2::last_error_string(); }

extern "C" int eb2_last_call_config(int* config, int* splits) {
  if (!config || !splits) return EB2_ERR_ARG;
  *config = eb2::call_config().config;
  *splits = eb2::call_config().splits;
  return EB2_OK;
}
