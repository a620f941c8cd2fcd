// mlp.h -- the configuration picker's network (see mlp.cu) and its host-side use.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace eb2 {

constexpr int kMlpIn = 8;       // feature vector length
constexpr int kMlpHidden = 64;
constexpr int kMlpConfigs = 4;  // 0 native, 1 emulated 128x128, 2 emulated 128x256, 3 emulated CTA pair 256x256
constexpr int kMlpSlices = 7;   // digit slices 6..12 of the emulated DGEMM
constexpr int kMlpSliceBase = 6;
constexpr int kMlpOut = kMlpConfigs + kMlpSlices;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpOut * kMlpHidden + kMlpOut;

cudaError_t launch_mlp_forward(const float* w, const float* X, int batch, float* logits, cudaStream_t st);
cudaError_t launch_mlp_backward(const float* w, const float* X, const int* cfg_label, const int* slice_label,
                                int batch, float* grads, float* loss, cudaStream_t st);
cudaError_t launch_mlp_adam(float* w, const float* g, float* m, float* v, int step, float lr, cudaStream_t st);

// Feature vector of one call: log2 sizes, dtype, exponent spread, batch size.
void picker_features(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, float* out);
// Host forward (same arithmetic as the device kernel); logits[kMlpOut].
void picker_forward(const float* w, const float* x, float* logits);
// Installed picker weights (null when none).
const float* picker_weights();
bool picker_load_file(const char* path, int num_sms);
void picker_autoload(int num_sms);
bool picker_predict(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, int* config,
                    int* slices);

}  // namespace eb2
