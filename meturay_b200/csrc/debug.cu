// Exposes the device copy of the portable sin/cos/acos so the CPU check can
// confirm both copies round identically.
#include "../../include/mrb200.h"
#include "common.cuh"

namespace mrb {
namespace {
__global__ void k_debug_math(const float* __restrict__ x, uint32_t n, float* __restrict__ sc,
                             const float* __restrict__ y, float* __restrict__ ac) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s, c;
        pm_sincos(x[i], s, c);
        sc[2 * i] = s;
        sc[2 * i + 1] = c;
        ac[i] = pm_acos(y[i]);
    }
}
}  // namespace
}  // namespace mrb

extern "C" int mrb_debug_math(const float* x, uint32_t n, float* sc, const float* y, float* ac,
                              void* stream) {
    if (n == 0) return 0;
    mrb::k_debug_math<<<(n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184, 256, 0,
                        static_cast<cudaStream_t>(stream)>>>(x, n, sc, y, ac);
    MRB_CUDA(cudaGetLastError());
    return 0;
}
