// bcc_mlp.h -- shapes and launchers of the collision-likelihood MLP (internal).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bcc {

constexpr int kMlpIn = 48;       // 7 joints + 32 environment code + 9 zero padding
constexpr int kMlpJoints = 7;
constexpr int kEnvCode = 32;
constexpr int kMlpHidden = 128;
constexpr int kMlpParams = kMlpIn * kMlpHidden + kMlpHidden + 2 * (kMlpHidden * kMlpHidden + kMlpHidden) +
                           kMlpHidden + 1;

cudaError_t mlp_pack(const float* d_params, uint8_t* d_images, cudaStream_t st);
// d_rows (optional): device row count computed by earlier kernels, capped by rows.
cudaError_t mlp_forward(const uint16_t* d_x, int rows, const uint8_t* d_images, const float* d_params,
                        float* d_logits, int* d_err, int num_sms, cudaStream_t st, const int* d_rows = nullptr);

cudaError_t mlp_train_grads(const uint16_t* d_x, const uint8_t* d_y, int rows, const uint8_t* d_images,
                            const float* d_params, float* d_grads, float* d_loss, int* d_err, int num_sms,
                            cudaStream_t st);
cudaError_t mlp_adam(float* d_params, const float* d_grads, float* d_m, float* d_v, long long step, float lr,
                     cudaStream_t st);

}  // namespace bcc
