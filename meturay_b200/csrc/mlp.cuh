// Learned guiding proposal: a small MLP that maps a path vertex (position
// encoding, normal, outgoing direction) to a mixture of 8 von Mises-Fisher
// lobes over incident directions, trained online from the tracer's own path
// samples.  Forward and backward passes run on the 5th-generation tensor
// cores (tcgen05.mma, BF16 operands in shared memory, FP32 accumulators in
// tensor memory); see mlp.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace mrb {

// Network shape: 78 input features (12-frequency sin/cos encoding of the
// position, 3 x 2 x 12 = 72, + normal 3 + outgoing direction 3), padded to
// 80; three hidden layers of 64 (ReLU); 40 outputs (8 lobes x (direction 3,
// log concentration 1, weight logit 1)), padded to 64.
constexpr int kMlpIn = 80;
constexpr int kMlpFeatures = 78;
constexpr int kMlpWidth = 64;
constexpr int kMlpOut = 40;
constexpr int kMlpLobes = 8;
constexpr int kMlpLayers = 4;
constexpr int kMlpTile = 128;  // samples per tensor-core tile
// Flat parameters: per layer its weights W[in][out] (out contiguous, 64
// outputs; the output layer's columns 40..63 stay zero) then its 64 biases.
constexpr int kMlpLayerIn[kMlpLayers] = {kMlpIn, kMlpWidth, kMlpWidth, kMlpWidth};
constexpr int kMlpParams = (kMlpIn * 64 + 64) + 3 * (64 * 64 + 64);  // 17,664
__host__ __device__ constexpr int mlp_layer_offset(int l) {
    return l == 0 ? 0 : (kMlpIn * 64 + 64) + (l - 1) * (64 * 64 + 64);
}
// log concentration clamp: kappa = exp(min(raw, kMlpLogKappaMax))
constexpr float kMlpLogKappaMax = 8.0f;

struct MlpDev {
    const float* params;          // kMlpParams fp32 (master copy)
    const uint16_t* wImage;       // bf16 weights in the shared-memory image layout
    uint32_t* errorFlag;          // set when a bounded wait gives up
};

// Bytes of the bf16 weight image (all layers).
constexpr size_t kMlpImageBytes = size_t(kMlpIn + 3 * 64) / 8 * 1024;  // 34,816

// Forward pass: inputs n x kMlpIn fp32 (features, the padding zero), outputs
// n x kMlpOut fp32 (raw lobe parameters).
int mlp_forward(const MlpDev& m, const float* in, uint32_t n, float* out, cudaStream_t st);
// Loss and gradients: targets n x 4 (incident direction xyz, weight); the
// loss is sum_s w_s * -log q(dir_s | x_s) / sum_s w_s.  grad (kMlpParams)
// and loss (2 floats: weighted loss sum, weight sum) are accumulated into.
int mlp_gradients(const MlpDev& m, const float* in, const float* targets, uint32_t n,
                  float* grad, float* loss, cudaStream_t st);
// Adam (lr, 0.9, 0.999, 1e-8) on params with state m1/m2 and step count on
// the device; grad is divided by loss[1] (the weight sum) first, then
// cleared; the bf16 image is rewritten.
int mlp_adam(float* params, float* m1, float* m2, uint32_t* step, float* grad, const float* loss,
             float lr, uint16_t* wImage, cudaStream_t st);
// Rebuild the bf16 image from fp32 params.
int mlp_build_image(const float* params, uint16_t* wImage, cudaStream_t st);
// Encoding of n vertices: pos normalised to [0,1]^3, normal, outgoing
// direction -> n x kMlpIn features.
int mlp_encode(const float* pos, const float* nrm, const float* wo, uint32_t n, float* out,
               cudaStream_t st);

}  // namespace mrb
struct mrb_mlp;
namespace mrb {
// The device view of a C-ABI network handle, and its fp32 parameters.
MlpDev mlp_dev(const mrb_mlp* m);
float* mlp_params(mrb_mlp* m);

// Mixture evaluation shared by the sampler and the loss.
struct VmfMixture {
    float mu[kMlpLobes][3];
    float kappa[kMlpLobes];
    float logNorm[kMlpLobes];  // log(kappa / (2 pi (1 - exp(-2 kappa))))
    float logPi[kMlpLobes];
};

}  // namespace mrb
