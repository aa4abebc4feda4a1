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

#include "common.cuh"

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
int mlp_forward(const MlpDev& m, const float* in, uint32_t n, float* out, cudaStream_t st,
                const uint32_t* dCount = nullptr);
// Loss and gradients: targets n x 4 (incident direction xyz, weight); the
// loss is sum_s w_s * -log q(dir_s | x_s) / sum_s w_s.  grad (kMlpParams)
// and loss (2 floats: weighted loss sum, weight sum) are accumulated into.
int mlp_gradients(const MlpDev& m, const float* in, const float* targets, uint32_t n,
                  float* grad, float* loss, cudaStream_t st, const uint32_t* dCount = nullptr,
                  uint32_t maxCtas = 0);
// (dCount, when given, holds the sample count on the device; n bounds it.
// maxCtas > 0 caps the grid, each CTA then taking more tiles.)
// Adam (lr, 0.9, 0.999, 1e-8) on params with state m1/m2 and step count on
// the device; grad is divided by loss[1] (the weight sum) first, then
// cleared; the bf16 image is rewritten.  A batch of weight sum 0 takes no
// step.
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
// One Adam step of a network handle on a batch whose count is on the device.
int mlp_train_step_dev(mrb_mlp* m, const float* in, const float* targets, uint32_t maxN,
                       const uint32_t* dCount, float lr, cudaStream_t st, uint32_t maxCtas = 0);
uint32_t* mlp_error_flag(mrb_mlp* m);
// (weighted loss sum, weight sum) of the last training step's batch.
float* mlp_loss(mrb_mlp* m);
size_t mlp_state_bytes();
int mlp_state_copy(mrb_mlp* m, void* buf, bool save, cudaStream_t st);

// Mixture evaluation shared by the sampler and the loss.
struct VmfMixture {
    float mu[kMlpLobes][3];
    float kappa[kMlpLobes];
    float logNorm[kMlpLobes];  // log(kappa / (2 pi (1 - exp(-2 kappa))))
    float logPi[kMlpLobes];
};

// ---- the von Mises-Fisher mixture ---------------------------------------------
// Lobe k of the raw outputs r: direction r[5k..5k+2] (normalised), log
// concentration r[5k+3] clamped to [-10, kMlpLogKappaMax], weight logit
// r[5k+4] (softmax over the lobes).  vMF(w; mu, kappa) =
// kappa / (2 pi (1 - exp(-2 kappa))) * exp(kappa (mu.w - 1)).
__device__ __forceinline__ void mixture_from_raw(const float* r, VmfMixture& mx, float* rawLen) {
    float lse = -INFINITY;
    float logit[kMlpLobes];
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) {
        const float x = r[5 * k], y = r[5 * k + 1], z = r[5 * k + 2];
        const float nn = sqrtf(x * x + y * y + z * z + 1e-12f);
        rawLen[k] = nn;
        mx.mu[k][0] = x / nn;
        mx.mu[k][1] = y / nn;
        mx.mu[k][2] = z / nn;
        const float lk = fminf(fmaxf(r[5 * k + 3], -10.0f), kMlpLogKappaMax);
        const float kap = expf(lk);
        mx.kappa[k] = kap;
        mx.logNorm[k] = lk - logf(2.0f * kPiF) - logf(-expm1f(-2.0f * kap));
        logit[k] = r[5 * k + 4];
        lse = fmaxf(lse, logit[k]);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) s += expf(logit[k] - lse);
    lse += logf(s);
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) mx.logPi[k] = logit[k] - lse;
}

// log q(w) and each lobe's log(pi_k vMF_k(w)).
__device__ __forceinline__ float mixture_logpdf(const VmfMixture& mx, float wx, float wy, float wz,
                                                float* lobeLog) {
    float m = -INFINITY;
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) {
        const float c = mx.mu[k][0] * wx + mx.mu[k][1] * wy + mx.mu[k][2] * wz;
        lobeLog[k] = mx.logPi[k] + mx.logNorm[k] + mx.kappa[k] * (c - 1.0f);
        m = fmaxf(m, lobeLog[k]);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) s += expf(lobeLog[k] - m);
    return m + logf(s);
}

// Features of a vertex: per axis c and frequency j, sin and cos of
// 2^j pi p_c at 24c + 2j and 24c + 2j + 1; then the normal and the
// outgoing direction; then two zeros.
__device__ __forceinline__ void encode_vertex(float px, float py, float pz, float nx, float ny,
                                              float nz, float ox, float oy, float oz, float* f) {
    const float p[3] = {px, py, pz};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float x = p[c];
#pragma unroll
        for (int j = 0; j < 12; j++) {
            float sv, cv;
            sincospif(x, &sv, &cv);
            f[24 * c + 2 * j] = sv;
            f[24 * c + 2 * j + 1] = cv;
            x *= 2.0f;
        }
    }
    f[72] = nx;
    f[73] = ny;
    f[74] = nz;
    f[75] = ox;
    f[76] = oy;
    f[77] = oz;
    f[78] = 0.0f;
    f[79] = 0.0f;
}


}  // namespace mrb
