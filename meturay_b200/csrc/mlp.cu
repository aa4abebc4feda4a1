// Learned guiding MLP on the tcgen05 tensor cores.
//
// Shared-memory operand layout (no swizzle, "interleaved" core matrices):
// a core matrix is 8 rows x 16 bytes (8 bf16), its rows 16 bytes apart.
//   activations  X / H / G  (128 samples x F features): core matrix
//                (sample group sg, feature group fg) at sg*(F/8)*128 + fg*128
//   weights      W (in x 64 out): core matrix (input group ig, output group
//                og) at ig*1024 + og*128, each of its rows one input's 8
//                outputs
// One copy of each serves every product it enters:
//   forward      D[s][o] = sum_i X[s][i] W[i][o]      A = X  K-major,
//                                                     B = W  MN-major
//   input grad   dX[s][i] = sum_o G[s][o] W[i][o]     A = G  K-major,
//                                                     B = W  K-major
//   weight grad  dW^T[o][i] = sum_s G[s][o] X[s][i]   A = G  MN-major,
//                                                     B = X  MN-major
// Forward and input gradients use M = 128 (one sample per TMEM lane);
// weight gradients use M = 64 (output features; TMEM lanes 0-15, 32-47,
// 64-79, 96-111) and accumulate in TMEM over all tiles a CTA processes.
// One elected thread issues the MMAs; completion is signalled through an
// mbarrier whose waits are bounded (on expiry the kernel flags an error,
// frees its tensor memory and returns).
#include "../../include/mrb200.h"
#include "mlp_tile.cuh"

namespace mrb {

namespace {

// d(-w log q(dir))/d raw into g[0..39]; returns -log q.
__device__ __forceinline__ float mixture_grad(const float* r, float wx, float wy, float wz,
                                              float weight, float* g) {
    VmfMixture mx;
    float rawLen[kMlpLobes], lobeLog[kMlpLobes];
    mixture_from_raw(r, mx, rawLen);
    const float lq = mixture_logpdf(mx, wx, wy, wz, lobeLog);
#pragma unroll
    for (int k = 0; k < kMlpLobes; k++) {
        const float gamma = expf(lobeLog[k] - lq);
        const float pi = expf(mx.logPi[k]);
        const float kap = mx.kappa[k];
        const float c = mx.mu[k][0] * wx + mx.mu[k][1] * wy + mx.mu[k][2] * wz;
        // direction: (I - mu mu^T) (w kappa) / |r|
        const float sd = -weight * gamma * kap / rawLen[k];
        g[5 * k + 0] = sd * (wx - c * mx.mu[k][0]);
        g[5 * k + 1] = sd * (wy - c * mx.mu[k][1]);
        g[5 * k + 2] = sd * (wz - c * mx.mu[k][2]);
        // concentration through kappa = exp(r3) inside the clamp
        const float r3 = r[5 * k + 3];
        const float dlog = 1.0f / kap - 2.0f / expm1f(2.0f * kap) + (c - 1.0f);
        g[5 * k + 3] = (r3 > -10.0f && r3 < kMlpLogKappaMax) ? -weight * gamma * dlog * kap : 0.0f;
        // weight logit (softmax)
        g[5 * k + 4] = -weight * (gamma - pi);
    }
    return -lq;
}

// ---- shared memory ------------------------------------------------------------
struct alignas(1024) MlpSmem {
    unsigned char w[kMlpImageBytes];       // weight images, all layers
    unsigned char x[kMlpTile * kMlpIn * 2];
    unsigned char h[3][kMlpTile * 64 * 2];  // post-ReLU activations of the hidden layers
    unsigned char g[2][kMlpTile * 64 * 2];  // output gradients (ping-pong)
    float bias[kMlpLayers][64];
    float dbias[kMlpLayers][64];
    uint64_t mbar;
    uint32_t tmem;
    uint32_t fail;
    __device__ unsigned char* hidden(int l) { return h[l]; }
};
// TMEM columns: the 128 x 64 accumulator (kColD), then dW^T of each layer
// (64 rows x the layer's inputs), all starting at multiples of 16.
__host__ __device__ constexpr uint32_t col_dw(int l) {
    return l == 0 ? 64u : 64u + 80u + 64u * uint32_t(l - 1);
}

// Plain inference: features from and outputs to row-major fp32 buffers.
struct BufferIO {
    const float* in;
    float* out;
    uint32_t maxN;
    const uint32_t* dCount;
    __device__ uint32_t rows() const { return dCount ? min(*dCount, maxN) : maxN; }
    __device__ void input(uint32_t s, uint32_t n, float* v) const {
        if (s < n) {
            const float4* p = reinterpret_cast<const float4*>(in + size_t(s) * kMlpIn);
#pragma unroll
            for (int c = 0; c < kMlpIn / 4; c++) {
                const float4 q = p[c];
                v[4 * c] = q.x;
                v[4 * c + 1] = q.y;
                v[4 * c + 2] = q.z;
                v[4 * c + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int c = 0; c < kMlpIn; c++) v[c] = 0.0f;
        }
    }
    __device__ void output(uint32_t s, const float* o) const {
        float4* dst = reinterpret_cast<float4*>(out + size_t(s) * kMlpOut);
#pragma unroll
        for (int c = 0; c < kMlpOut / 4; c++)
            dst[c] = make_float4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
    }
};

// Column sums of a per-thread row (one sample per thread) into dst[64],
// one shared-memory atomic per warp and column.
__device__ __forceinline__ void add_column_sums(const float* v, float* dst) {
#pragma unroll
    for (int o = 0; o < 64; o++) {
        float x = v[o];
        for (int sh = 16; sh > 0; sh >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, sh);
        if ((threadIdx.x & 31u) == 0) atomicAdd(dst + o, x);
    }
}

// Values of a row after bf16 rounding (what the tensor cores read back).
__device__ __forceinline__ void round_bf16(float* v, int n) {
    for (int i = 0; i < n; i++) v[i] = bf16_float(bf16_bits(v[i]));
}

__global__ void __launch_bounds__(kMlpTile, 1) k_mlp_train(MlpDev m, const float* __restrict__ in,
                                                          const float* __restrict__ targets,
                                                          uint32_t maxN,
                                                          const uint32_t* __restrict__ dCount,
                                                          float* __restrict__ grad,
                                                          float* __restrict__ loss) {
    extern __shared__ __align__(1024) unsigned char smemRaw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smemRaw);
    const uint32_t n = dCount ? min(*dCount, maxN) : maxN;
    const uint32_t tmem = mlp_prologue(S, m, 512);
    const uint32_t row = threadIdx.x;
    const uint32_t lane = (threadIdx.x & ~31u) << 16;
    uint32_t phase = 0;
    bool first = true, ok = true;
    float lossSum = 0.0f, weightSum = 0.0f;
    const uint32_t tiles = (n + kMlpTile - 1) / kMlpTile;
    for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const uint32_t s = t * kMlpTile + row;
        load_input(S, in, n, s, row);
        fence_async_smem();
        __syncthreads();
        float o[64];
        if (!forward_tile(S, tmem, phase, m.errorFlag, o)) {
            ok = false;
            break;
        }
        // output gradient of -w log q(dir)
        float g[64];
#pragma unroll
        for (int k = 0; k < 64; k++) g[k] = 0.0f;
        if (s < n) {
            const float4 tg = reinterpret_cast<const float4*>(targets)[s];
            if (tg.w > 0.0f) {
                lossSum += tg.w * mixture_grad(o, tg.x, tg.y, tg.z, tg.w, g);
                weightSum += tg.w;
            }
        }
        store_row<64>(S.g[0], row, g);
        round_bf16(g, 64);
        add_column_sums(g, S.dbias[kMlpLayers - 1]);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // backward, output layer first
        int cur = 0;
#pragma unroll 1
        for (int l = kMlpLayers - 1; l >= 0; l--) {
            const unsigned char* X = (l == 0) ? S.x : S.h[l - 1];
            const uint32_t F = (l == 0) ? kMlpIn : 64;
            if (threadIdx.x == 0) {
                const uint32_t gA = smem_u32(S.g[cur]), xB = smem_u32(X);
                // dW^T[o][i] += sum_s G[s][o] X[s][i]: M = 64 outputs, N = F inputs,
                // K = 128 samples; both operands MN-major (sample groups are the K
                // chunks, 8 * row stride apart)
                for (uint32_t k0 = 0; k0 < kMlpTile; k0 += 16) {
                    const uint64_t ad = smem_desc(gA + (k0 / 8) * 1024u, 1024u, 128u);
                    const uint64_t bd = smem_desc(xB + (k0 / 8) * (F / 8) * 128u, (F / 8) * 128u, 128u);
                    mma_bf16(tmem + col_dw(l), ad, bd, idesc_bf16(64, int(F), true, true),
                             (first && k0 == 0) ? 0u : 1u);
                }
                if (l > 0) {
                    // dX[s][i] = sum_o G[s][o] W[i][o]: A = G K-major, B = W K-major
                    const uint32_t w0 = smem_u32(S.w + image_layer_offset(l));
                    for (uint32_t k0 = 0; k0 < 64; k0 += 16) {
                        const uint64_t ad = smem_desc(gA + (k0 / 8) * 128u, 128u, 1024u);
                        const uint64_t bd = smem_desc(w0 + (k0 / 8) * 128u, 128u, 1024u);
                        mma_bf16(tmem + kColD, ad, bd, idesc_bf16(128, 64, false, false),
                                 k0 > 0 ? 1u : 0u);
                    }
                }
                mma_commit(&S.mbar);
            }
            if (!mlp_wait(S, phase, m.errorFlag)) {
                ok = false;
                break;
            }
            if (l > 0) {
                float dx[64], h[64];
                read_acc(tmem, dx);
                load_row<64>(S.h[l - 1], row, h);
#pragma unroll
                for (int i = 0; i < 64; i++) dx[i] = (h[i] > 0.0f) ? dx[i] : 0.0f;
                store_row<64>(S.g[cur ^ 1], row, dx);
                round_bf16(dx, 64);
                add_column_sums(dx, S.dbias[l - 1]);
                cur ^= 1;
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
        }
        first = false;
    }
    // weight gradients out of TMEM: warp w, lanes 32w..32w+15 hold rows (outputs)
    // 16w..16w+15 of every dW^T
    if (ok && !first) {
        const uint32_t warp = threadIdx.x >> 5, t = threadIdx.x & 31u;
        const uint32_t o = 16 * warp + t;
#pragma unroll 1
        for (int l = 0; l < kMlpLayers; l++) {
            const uint32_t F = (l == 0) ? kMlpIn : 64;
            float* gw = grad + mlp_layer_offset(l);
#pragma unroll 1
            for (uint32_t c = 0; c < F; c += 16) {
                float v[16];
                tmem_ld16(tmem + lane + col_dw(l) + c, v);
                tmem_wait_ld();
                if (t < 16) {
#pragma unroll
                    for (int k = 0; k < 16; k++) atomicAdd(gw + (c + k) * 64 + o, v[k]);
                }
            }
        }
    }
    __syncthreads();
    if (ok) {
        for (uint32_t i = threadIdx.x; i < kMlpLayers * 64; i += blockDim.x) {
            const int l = int(i / 64), oo = int(i % 64);
            atomicAdd(grad + mlp_layer_offset(l) + (l == 0 ? kMlpIn : 64) * 64 + oo, S.dbias[l][oo]);
        }
        for (int sh = 16; sh > 0; sh >>= 1) {
            lossSum += __shfl_xor_sync(0xFFFFFFFFu, lossSum, sh);
            weightSum += __shfl_xor_sync(0xFFFFFFFFu, weightSum, sh);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(loss + 0, lossSum);
            atomicAdd(loss + 1, weightSum);
        }
    }
    mlp_epilogue(S, tmem, 512);
}

// Parameter i: its layer, and for weights (i, o) and the image offset.
__device__ __forceinline__ bool param_weight(uint32_t i, int& l, uint32_t& in, uint32_t& out) {
    l = 0;
    while (l + 1 < kMlpLayers && i >= uint32_t(mlp_layer_offset(l + 1))) l++;
    const uint32_t local = i - uint32_t(mlp_layer_offset(l));
    const uint32_t K = (l == 0) ? kMlpIn : 64;
    if (local >= K * 64) return false;  // a bias
    in = local / 64;
    out = local % 64;
    return true;
}

// The output layer's columns past the 40 outputs (weights and biases) and
// the input rows past the 78 features stay zero.
__device__ __forceinline__ bool param_frozen(uint32_t i) {
    int l;
    uint32_t in, out;
    if (param_weight(i, l, in, out))
        return (l == kMlpLayers - 1 && out >= kMlpOut) || (l == 0 && in >= kMlpFeatures);
    const uint32_t o = (i - uint32_t(mlp_layer_offset(l))) % 64;
    return l == kMlpLayers - 1 && o >= kMlpOut;
}

__global__ void __launch_bounds__(256) k_mlp_adam(float* __restrict__ params, float* __restrict__ m1,
                                                  float* __restrict__ m2, const uint32_t* step,
                                                  float* __restrict__ grad,
                                                  const float* __restrict__ loss, float lr,
                                                  uint16_t* __restrict__ image) {
    const bool empty = !(loss[1] > 0.0f);  // a batch without weight: no step
    const uint32_t t = *step + 1u;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, float(t)), c2 = 1.0f - powf(b2, float(t));
    const float inv = 1.0f / fmaxf(loss[1], 1e-20f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < uint32_t(kMlpParams);
         i += gridDim.x * blockDim.x) {
        float p = params[i];
        if (!empty && !param_frozen(i)) {
            const float g = grad[i] * inv;
            const float a = b1 * m1[i] + (1.0f - b1) * g;
            const float b = b2 * m2[i] + (1.0f - b2) * g * g;
            m1[i] = a;
            m2[i] = b;
            p -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
            params[i] = p;
        }
        grad[i] = 0.0f;
        int l;
        uint32_t in, out;
        if (param_weight(i, l, in, out))
            image[(image_layer_offset(l) + w_offset(in, out)) / 2] = bf16_bits(p);
    }
}

__global__ void k_mlp_step(uint32_t* step, const float* loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && loss[1] > 0.0f) *step += 1u;
}

__global__ void __launch_bounds__(256) k_mlp_image(const float* __restrict__ params,
                                                   uint16_t* __restrict__ image) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < uint32_t(kMlpParams);
         i += gridDim.x * blockDim.x) {
        int l;
        uint32_t in, out;
        if (param_weight(i, l, in, out))
            image[(image_layer_offset(l) + w_offset(in, out)) / 2] = bf16_bits(params[i]);
    }
}

__global__ void __launch_bounds__(256) k_mlp_encode(const float* __restrict__ pos,
                                                    const float* __restrict__ nrm,
                                                    const float* __restrict__ wo, uint32_t n,
                                                    float* __restrict__ out) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float f[kMlpIn];
        encode_vertex(pos[3 * s], pos[3 * s + 1], pos[3 * s + 2], nrm[3 * s], nrm[3 * s + 1],
                      nrm[3 * s + 2], wo[3 * s], wo[3 * s + 1], wo[3 * s + 2], f);
        float4* d = reinterpret_cast<float4*>(out + size_t(s) * kMlpIn);
#pragma unroll
        for (int c = 0; c < kMlpIn / 4; c++)
            d[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
    }
}

int mlp_smem_setup() {
    static bool done[64] = {};
    int dev = 0;
    MRB_CUDA(cudaGetDevice(&dev));
    if (!done[dev & 63]) {
        MRB_CUDA(cudaFuncSetAttribute(k_mlp_forward_io<BufferIO>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(sizeof(MlpFwdSmem))));
        MRB_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(sizeof(MlpSmem))));
        done[dev & 63] = true;
    }
    return 0;
}

uint32_t mlp_grid(uint32_t n, uint32_t perSm = 1) {
    const uint32_t tiles = (n + kMlpTile - 1) / kMlpTile;
    const uint32_t cap = 148u * perSm;
    return tiles < cap ? (tiles ? tiles : 1u) : cap;
}

}  // namespace

int mlp_forward(const MlpDev& m, const float* in, uint32_t n, float* out, cudaStream_t st,
                const uint32_t* dCount) {
    if (n == 0) return 0;
    if (mlp_smem_setup()) return MRB_E_CUDA;
    k_mlp_forward_io<<<mlp_grid(n, kMlpFwdCtasPerSm), kMlpTile, sizeof(MlpFwdSmem), st>>>(
        m, BufferIO{in, out, n, dCount});
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mlp_gradients(const MlpDev& m, const float* in, const float* targets, uint32_t n, float* grad,
                  float* loss, cudaStream_t st, const uint32_t* dCount, uint32_t maxCtas) {
    if (n == 0) return 0;
    if (mlp_smem_setup()) return MRB_E_CUDA;
    uint32_t grid = mlp_grid(n);
    if (maxCtas && grid > maxCtas) grid = maxCtas;
    k_mlp_train<<<grid, kMlpTile, sizeof(MlpSmem), st>>>(m, in, targets, n, dCount, grad, loss);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mlp_adam(float* params, float* m1, float* m2, uint32_t* step, float* grad, const float* loss,
             float lr, uint16_t* wImage, cudaStream_t st) {
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, m1, m2, step, grad, loss, lr,
                                                        wImage);
    k_mlp_step<<<1, 32, 0, st>>>(step, loss);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mlp_build_image(const float* params, uint16_t* wImage, cudaStream_t st) {
    k_mlp_image<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, wImage);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mlp_encode(const float* pos, const float* nrm, const float* wo, uint32_t n, float* out,
               cudaStream_t st) {
    if (n == 0) return 0;
    k_mlp_encode<<<(n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8, 256, 0, st>>>(pos, nrm,
                                                                                     wo, n, out);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#include "objects.cuh"

struct mrb_mlp {
    mrb_system* sys = nullptr;
    DBuf params, m1, m2, grad, loss, step, image, err;
    mrb::MlpDev dev() const {
        return mrb::MlpDev{params.as<float>(), image.as<uint16_t>(), err.as<uint32_t>()};
    }
};

namespace {
int mlp_check(mrb_mlp* m, cudaStream_t st) {
    uint32_t e = 0;
    MRB_CUDA(cudaMemcpyAsync(&e, m->err.p, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    if (e) {
        mrb::set_error("MLP: a tensor-core wait gave up");
        return MRB_E_DEVICE;
    }
    return 0;
}
}  // namespace

namespace mrb {
MlpDev mlp_dev(const mrb_mlp* m) { return m->dev(); }
float* mlp_params(mrb_mlp* m) { return m->params.as<float>(); }
int mlp_train_step_dev(mrb_mlp* m, const float* in, const float* targets, uint32_t maxN,
                       const uint32_t* dCount, float lr, cudaStream_t st, uint32_t maxCtas) {
    MRB_CUDA(cudaMemsetAsync(m->loss.p, 0, 8, st));
    int r = mlp_gradients(m->dev(), in, targets, maxN, m->grad.as<float>(), m->loss.as<float>(),
                          st, dCount, maxCtas);
    if (r) return r;
    return mlp_adam(m->params.as<float>(), m->m1.as<float>(), m->m2.as<float>(),
                    m->step.as<uint32_t>(), m->grad.as<float>(), m->loss.as<float>(), lr,
                    m->image.as<uint16_t>(), st);
}
uint32_t* mlp_error_flag(mrb_mlp* m) { return m->err.as<uint32_t>(); }
float* mlp_loss(mrb_mlp* m) { return m->loss.as<float>(); }
size_t mlp_state_bytes() { return size_t(kMlpParams) * 4 * 3 + 16 + kMlpImageBytes; }
// Parameters, optimiser state and weight image to / from a device buffer.
int mlp_state_copy(mrb_mlp* m, void* buf, bool save, cudaStream_t st) {
    const size_t P = size_t(kMlpParams) * 4;
    unsigned char* b = static_cast<unsigned char*>(buf);
    DBuf* parts[5] = {&m->params, &m->m1, &m->m2, &m->step, &m->image};
    const size_t sizes[5] = {P, P, P, 16, kMlpImageBytes};
    for (int i = 0; i < 5; i++) {
        if (save) MRB_CUDA(cudaMemcpyAsync(b, parts[i]->p, sizes[i], cudaMemcpyDeviceToDevice, st));
        else MRB_CUDA(cudaMemcpyAsync(parts[i]->p, b, sizes[i], cudaMemcpyDeviceToDevice, st));
        b += sizes[i];
    }
    return 0;
}
}  // namespace mrb

extern "C" {

uint32_t mrb_mlp_param_count(void) { return uint32_t(mrb::kMlpParams); }

int mrb_mlp_create(mrb_system* sys, mrb_mlp** out) {
    if (!sys || !out) return MRB_E_ARG;
    *out = nullptr;
    MRB_CUDA(cudaSetDevice(sys->device));
    mrb_mlp* m = new mrb_mlp();
    m->sys = sys;
    const size_t P = size_t(mrb::kMlpParams) * 4;
    int r;
    if ((r = m->params.alloc(P)) || (r = m->m1.alloc(P)) || (r = m->m2.alloc(P)) ||
        (r = m->grad.alloc(P)) || (r = m->loss.alloc(16)) || (r = m->step.alloc(16)) ||
        (r = m->image.alloc(mrb::kMlpImageBytes)) || (r = m->err.alloc(16))) {
        delete m;
        return r;
    }
    cudaError_t e = cudaSuccess;
    for (DBuf* b : {&m->params, &m->m1, &m->m2, &m->grad, &m->loss, &m->step, &m->image, &m->err})
        if (e == cudaSuccess) e = cudaMemset(b->p, 0, b->bytes);
    if (e != cudaSuccess) {
        delete m;
        MRB_CUDA(e);
    }
    *out = m;
    return 0;
}

void mrb_mlp_destroy(mrb_mlp* m) { delete m; }

int mrb_mlp_set_params(mrb_mlp* m, const float* host) {
    if (!m || !host) return MRB_E_ARG;
    const size_t P = size_t(mrb::kMlpParams) * 4;
    MRB_CUDA(cudaMemcpy(m->params.p, host, P, cudaMemcpyHostToDevice));
    MRB_CUDA(cudaMemset(m->m1.p, 0, P));
    MRB_CUDA(cudaMemset(m->m2.p, 0, P));
    MRB_CUDA(cudaMemset(m->grad.p, 0, P));
    MRB_CUDA(cudaMemset(m->step.p, 0, 16));
    if (mrb::mlp_build_image(m->params.as<float>(), m->image.as<uint16_t>(), nullptr))
        return MRB_E_CUDA;
    MRB_CUDA(cudaDeviceSynchronize());
    return 0;
}

int mrb_mlp_get_params(const mrb_mlp* m, float* host) {
    if (!m || !host) return MRB_E_ARG;
    MRB_CUDA(cudaMemcpy(host, m->params.p, size_t(mrb::kMlpParams) * 4, cudaMemcpyDeviceToHost));
    return 0;
}

int mrb_mlp_encode(const float* d_pos, const float* d_nrm, const float* d_wo, uint32_t n,
                   float* d_features, void* stream) {
    if (n && (!d_pos || !d_nrm || !d_wo || !d_features)) return MRB_E_ARG;
    return mrb::mlp_encode(d_pos, d_nrm, d_wo, n, d_features, static_cast<cudaStream_t>(stream));
}

int mrb_mlp_forward(mrb_mlp* m, const float* d_features, uint32_t n, float* d_out, void* stream) {
    if (!m || (n && (!d_features || !d_out))) return MRB_E_ARG;
    if ((reinterpret_cast<uintptr_t>(d_features) | reinterpret_cast<uintptr_t>(d_out)) & 15) {
        mrb::set_error("MLP: features and outputs need 16-byte alignment");
        return MRB_E_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int r = mrb::mlp_forward(m->dev(), d_features, n, d_out, st);
    return r ? r : mlp_check(m, st);
}

int mrb_mlp_gradients(mrb_mlp* m, const float* d_features, const float* d_targets, uint32_t n,
                      float* d_grad, float* d_loss, void* stream) {
    if (!m || !d_grad || !d_loss || (n && (!d_features || !d_targets))) return MRB_E_ARG;
    if ((reinterpret_cast<uintptr_t>(d_features) | reinterpret_cast<uintptr_t>(d_targets)) & 15) {
        mrb::set_error("MLP: features and targets need 16-byte alignment");
        return MRB_E_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int r = mrb::mlp_gradients(m->dev(), d_features, d_targets, n, d_grad, d_loss, st);
    return r ? r : mlp_check(m, st);
}

int mrb_mlp_train_step(mrb_mlp* m, const float* d_features, const float* d_targets, uint32_t n,
                       float lr, float* host_loss2, void* stream) {
    if (!m || (n && (!d_features || !d_targets))) return MRB_E_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MRB_CUDA(cudaMemsetAsync(m->loss.p, 0, 8, st));
    int r = mrb::mlp_gradients(m->dev(), d_features, d_targets, n, m->grad.as<float>(),
                               m->loss.as<float>(), st);
    if (r) return r;
    if (host_loss2)
        MRB_CUDA(cudaMemcpyAsync(host_loss2, m->loss.p, 8, cudaMemcpyDeviceToHost, st));
    r = mrb::mlp_adam(m->params.as<float>(), m->m1.as<float>(), m->m2.as<float>(),
                      m->step.as<uint32_t>(), m->grad.as<float>(), m->loss.as<float>(), lr,
                      m->image.as<uint16_t>(), st);
    if (r) return r;
    return mlp_check(m, st);
}

}  // extern "C"
