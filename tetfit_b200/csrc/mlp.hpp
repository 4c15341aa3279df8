// Host-side interface of the learned CG warm-start network (kernels and
// device helpers in mlp.cuh / mlp.cu): parameter layout, weight image layout,
// training buffers and launches.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace tf {

constexpr int kMlpIn = 6, kMlpInP = 16, kMlpH = 64;
constexpr int kOffW1 = 0, kOffB1 = kMlpH * kMlpInP, kOffW2 = kOffB1 + kMlpH, kOffB2 = kOffW2 + kMlpH * kMlpH,
              kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH, kNParam = kOffB3 + 1;
constexpr int kLd1 = 24, kLd2 = 72;
constexpr int kImgW1 = 0, kImgW2T = kImgW1 + 64 * kLd1, kImgW2K = kImgW2T + 64 * kLd2, kImgW3 = kImgW2K + 64 * kLd2,
              kImgBf16 = kImgW3 + 8 * kLd2;                  // BF16 elements
constexpr int kImgBytes = kImgBf16 * 2 + (64 + 64 + 4) * 4;  // + FP32 biases

void mlp_init_params(float* params, uint64_t seed);
cudaError_t mlp_launch_pack(const float* params, unsigned char* image, cudaStream_t st);
// One training pass over n samples (inputs [n][6], targets [n], weights [n]):
// gradients of the loss sum_i w_i (y_i - t_i)^2 / n, reduced in a fixed order
// into grad[kNParam] (and the loss into *loss), then an Adam step on params
// (when adam_step > 0) and a fresh weight image.
struct MlpTrain {
  float* params = nullptr;      // [kNParam]
  float* adam_m = nullptr;      // [kNParam]
  float* adam_v = nullptr;      // [kNParam]
  unsigned char* image = nullptr;
  float* grad_part = nullptr;   // [blocks][kNParam]
  float* loss_part = nullptr;   // [blocks]
  float* grad = nullptr;        // [kNParam]
  float* loss = nullptr;        // [1]
  int max_blocks = 0;
};
cudaError_t mlp_launch_train(const MlpTrain& m, const float* inputs, const float* targets, const float* weights, int n,
                             int adam_step, float lr, cudaStream_t st);
int mlp_train_rows_per_block();
cudaError_t mlp_launch_eval(const unsigned char* image, const float* in, int64_t n, float* out, cudaStream_t st);

}  // namespace tf
