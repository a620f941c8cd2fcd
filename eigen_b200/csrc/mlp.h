// mlp.h -- the configuration picker's network (see mlp.cu) and its host-side use.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace eb2 {

constexpr int kMlpIn = 8;       // feature vector length
constexpr int kMlpHidden = 64;
// Configuration classes of the first head (one softmax; a prediction takes the argmax over
// the classes of its kind: DGEMM [0, 6), SGEMM [6, 10), grouped batch [10, 12)).
enum MlpConfig : int {
  kCfgNative = 0,          // FP64 DMMA kernel
  kCfgCrtCta = 1,          // CRT emulation, one CTA per 128 x 256 tile, column-major tile order
  kCfgCrtPair = 2,         // CRT emulation, a CTA pair per 256 x 256 tile, column-major tile order
  kCfgCrtCtaGroup = 3,     // CRT emulation, one CTA, raster groups of kCfgGroupM row tiles
  kCfgCrtPairGroup = 4,    // CRT emulation, CTA pair, raster groups of kCfgGroupM row tiles
  kCfgCrtSplitK = 5,       // CRT emulation, one CTA, K split so that the work items fill the SMs
  kCfgSgemmFfma = 6,       // FP32 FFMA kernel
  kCfgSgemmBf16_128 = 7,   // split-BF16, one CTA per 128 x 128 tile
  kCfgSgemmBf16_256 = 8,   // split-BF16, one CTA per 128 x 256 tile
  kCfgSgemmBf16Pair = 9,   // split-BF16, a CTA pair per 256 x 256 tile
  kCfgBatchClasses = 10,   // grouped batch: small products share a warp (classes 8 and 16)
  kCfgBatchTiles = 11,     // grouped batch: every product as 32 x 32 tiles
  kMlpConfigs = 12
};
constexpr int kCfgGroupM = 16;
constexpr int kMlpSlices = 7;   // precision classes c: CRT moduli 8 + 2c (DGEMM only)
constexpr int kMlpSliceBase = 6;
constexpr int kMlpOut = kMlpConfigs + kMlpSlices;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpOut * kMlpHidden + kMlpOut;

cudaError_t launch_mlp_forward(const float* w, const float* X, int batch, float* logits, cudaStream_t st);
cudaError_t launch_mlp_backward(const float* w, const float* X, const int* cfg_label, const int* slice_label,
                                int batch, float* grads, float* loss, cudaStream_t st);
cudaError_t launch_mlp_adam(float* w, const float* g, float* m, float* v, int step, float lr, cudaStream_t st);

// Feature vector of one call: log2 sizes, dtype, exponent spread, batch size, log2 of the
// accuracy target.
void picker_features(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                     float* out);
// Host forward (same arithmetic as the device kernel); logits[kMlpOut].
void picker_forward(const float* w, const float* x, float* logits);
// Installed picker weights (null when none).
const float* picker_weights();
bool picker_load_file(const char* path, int num_sms);
void picker_autoload(int num_sms);
// The class of kind dtype ('d' or 's'; a grouped batch when batch > 1) with the largest
// score, and the precision class (kMlpSliceBase + c).  False without weights.
bool picker_predict(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                    int* config, int* slices);
// First and one-past-last configuration class of a kind.
void picker_config_range(char dtype, int64_t batch, int* lo, int* hi);
// The configuration class forced by eb2_set_config (-1: none).
int forced_config();

}  // namespace eb2
