// picker.cpp -- host side of the learned configuration picker: the feature vector, a
// host forward pass of the MLP (the same operations as mlp_forward_kernel, in FP32 with
// fused multiply-adds), and the process-wide installed weights.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <string>

#include "context.h"
#include "eigen_b200/blas.h"
#include "mlp.h"

namespace eb2 {

namespace {
std::mutex g_mu;
std::vector<float> g_weights;  // empty: no picker installed
}  // namespace

void picker_features(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                     float* out) {
  const double lm = std::log2(double(m > 0 ? m : 1)), ln = std::log2(double(n > 0 ? n : 1)),
               lk = std::log2(double(k > 0 ? k : 1));
  const double t = tol > 0.0 && tol < 1.0 ? tol : 1.0;
  out[0] = float(lm / 14.0);
  out[1] = float(ln / 14.0);
  out[2] = float(lk / 14.0);
  out[3] = dtype == 'd' ? 1.f : 0.f;
  out[4] = float(spread / 32.0);
  out[5] = float(std::log2(double(batch > 0 ? batch : 1)) / 14.0);
  out[6] = float((lm + ln + lk) / 42.0);
  out[7] = float(-std::log2(t) / 64.0);
}

void picker_config_range(char dtype, int64_t batch, int* lo, int* hi) {
  if (batch > 1) {
    *lo = kCfgBatchClasses;
    *hi = kCfgBatchTiles + 1;
  } else if (dtype == 's') {
    *lo = kCfgSgemmFfma;
    *hi = kCfgSgemmBf16Pair + 1;
  } else {
    *lo = kCfgNative;
    *hi = kCfgCrtSplitK + 1;
  }
}

namespace {
std::atomic<int> g_forced_config{-1};
}
int forced_config() { return g_forced_config.load(); }

void picker_forward(const float* w, const float* x, float* logits) {
  constexpr int H = kMlpHidden;
  const float* W1 = w;
  const float* b1 = W1 + H * kMlpIn;
  const float* W2 = b1 + H;
  const float* b2 = W2 + H * H;
  const float* W3 = b2 + H;
  const float* b3 = W3 + kMlpOut * H;
  float h1[H], h2[H];
  for (int j = 0; j < H; ++j) {
    float s = b1[j];
    for (int i = 0; i < kMlpIn; ++i) s = std::fma(W1[j * kMlpIn + i], x[i], s);
    h1[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < H; ++j) {
    float s = b2[j];
    for (int i = 0; i < H; ++i) s = std::fma(W2[j * H + i], h1[i], s);
    h2[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kMlpOut; ++j) {
    float s = b3[j];
    for (int i = 0; i < H; ++i) s = std::fma(W3[j * H + i], h2[i], s);
    logits[j] = s;
  }
}

const float* picker_weights() {
  std::lock_guard<std::mutex> lock(g_mu);
  return g_weights.empty() ? nullptr : g_weights.data();
}

bool picker_predict(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                    int* config, int* slices) {
  std::vector<float> w;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_weights.empty()) return false;
    w = g_weights;
  }
  float x[kMlpIn], lg[kMlpOut];
  picker_features(m, n, k, dtype, spread, batch, tol, x);
  picker_forward(w.data(), x, lg);
  int lo = 0, hi = 0;
  picker_config_range(dtype, batch, &lo, &hi);
  int c = lo;
  for (int j = lo + 1; j < hi; ++j)
    if (lg[j] > lg[c]) c = j;
  int s = 0;
  for (int j = 1; j < kMlpSlices; ++j)
    if (lg[kMlpConfigs + j] > lg[kMlpConfigs + s]) s = j;
  *config = c;
  *slices = kMlpSliceBase + s;
  return true;
}

// Reads picker weights written by the tuner: "EB2PICK1", uint32 count, uint32 SM count,
// then count float32.  Accepted only for this network size and the device's SM count.
bool picker_load_file(const char* path, int num_sms) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  char magic[8];
  uint32_t hdr[2];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "EB2PICK1", 8) == 0 &&
            std::fread(hdr, 4, 2, f) == 2 && hdr[0] == uint32_t(kMlpParams) && int(hdr[1]) == num_sms;
  std::vector<float> w;
  if (ok) {
    w.resize(kMlpParams);
    ok = std::fread(w.data(), 4, w.size(), f) == w.size();
  }
  std::fclose(f);
  if (!ok) return false;
  std::lock_guard<std::mutex> lock(g_mu);
  g_weights = std::move(w);
  return true;
}

// Default location: <directory of libeigen_b200.so>/../data/picker_weights.bin, or the
// path in EB2_PICKER_WEIGHTS ("off" disables the picker).
void picker_autoload(int num_sms) {
  const char* env = std::getenv("EB2_PICKER_WEIGHTS");
  if (env && std::strcmp(env, "off") == 0) return;
  if (env && *env) {
    picker_load_file(env, num_sms);
    return;
  }
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&picker_autoload), &info) == 0 || !info.dli_fname) return;
  std::string lib(info.dli_fname);
  const size_t slash = lib.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string(".") : lib.substr(0, slash);
  picker_load_file((dir + "/../data/picker_weights.bin").c_str(), num_sms);
}

}  // namespace eb2

extern "C" {

int eb2_mlp_param_count(void) { return eb2::kMlpParams; }

int eb2_picker_set_weights(const float* weights, int count) {
  std::lock_guard<std::mutex> lock(eb2::g_mu);
  if (!weights || count == 0) {
    eb2::g_weights.clear();
    return EB2_OK;
  }
  if (count != eb2::kMlpParams) {
    eb2::set_error(EB2_ERR_ARG, "picker weights: expected %d floats, got %d", eb2::kMlpParams, count);
    return EB2_ERR_ARG;
  }
  eb2::g_weights.assign(weights, weights + count);
  return EB2_OK;
}

int eb2_picker_features(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                        float* out) {
  if (!out) return EB2_ERR_ARG;
  eb2::picker_features(m, n, k, dtype, spread, batch, tol, out);
  return EB2_OK;
}

int eb2_set_config(int config) {
  if (config < -1 || config >= eb2::kMlpConfigs) {
    eb2::set_error(EB2_ERR_ARG, "eb2_set_config: %d is not a configuration class (-1 .. %d)", config,
                   eb2::kMlpConfigs - 1);
    return EB2_ERR_ARG;
  }
  eb2::g_forced_config = config;
  return EB2_OK;
}

int eb2_config_count(void) { return eb2::kMlpConfigs; }

int eb2_picker_forward_host(const float* weights, const float* features, float* logits) {
  if (!weights || !features || !logits) return EB2_ERR_ARG;
  eb2::picker_forward(weights, features, logits);
  return EB2_OK;
}

int eb2_picker_predict(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                       int* config, int* slices) {
  if (!config || !slices) return EB2_ERR_ARG;
  return eb2::picker_predict(m, n, k, dtype, spread, batch, tol, config, slices) ? EB2_OK : EB2_ERR_ARG;
}

int eb2_mlp_forward(const float* w, const float* X, int batch, float* logits, void* stream) {
  cudaError_t e = eb2::launch_mlp_forward(w, X, batch, logits, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    eb2::set_error(EB2_ERR_CUDA, "mlp forward: %s", cudaGetErrorString(e));
    return EB2_ERR_CUDA;
  }
  return EB2_OK;
}

int eb2_mlp_backward(const float* w, const float* X, const int* cfg_label, const int* slice_label, int batch,
                     float* grads, float* loss, void* stream) {
  cudaError_t e = eb2::launch_mlp_backward(w, X, cfg_label, slice_label, batch, grads, loss,
                                           static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    eb2::set_error(EB2_ERR_CUDA, "mlp backward: %s", cudaGetErrorString(e));
    return EB2_ERR_CUDA;
  }
  return EB2_OK;
}

int eb2_mlp_adam(float* w, const float* grads, float* m, float* v, int step, float lr, void* stream) {
  if (step < 1) return EB2_ERR_ARG;
  cudaError_t e = eb2::launch_mlp_adam(w, grads, m, v, step, lr, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    eb2::set_error(EB2_ERR_CUDA, "mlp adam: %s", cudaGetErrorString(e));
    return EB2_ERR_CUDA;
  }
  return EB2_OK;
}

}  // extern "C"
