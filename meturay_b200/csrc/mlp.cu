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
#include <cuda_bf16.h>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "mlp.cuh"

namespace mrb {

namespace {

constexpr uint32_t kSpinLimit = 1u << 26;

// ---- PTX wrappers ----------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dstSmem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dstSmem)),
                 "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
                 : "memory");
}

// Shared-memory matrix descriptor, SWIZZLE_NONE: start, leading and stride
// byte offsets in 16-byte units; bits 46-47 = 1 (Blackwell descriptor).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// Instruction descriptor, kind::f16: BF16 A and B, FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool aMN, bool bMN) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(aMN) << 15) | (uint32_t(bMN) << 16) |
           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(mbar))
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count)
                 : "memory");
}

// Bounded wait for the phase `parity` of the barrier to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < kSpinLimit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive fp32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- shared-memory layout helpers -----------------------------------------
// Byte offset of element (row, col) of a row-major-by-core-matrix operand
// with `cols` columns: core matrix (row/8, col/8), 16-byte rows.
__host__ __device__ __forceinline__ uint32_t act_offset(uint32_t row, uint32_t col,
                                                        uint32_t cols) {
    return (row >> 3) * (cols >> 3) * 128u + (col >> 3) * 128u + (row & 7u) * 16u +
           (col & 7u) * 2u;
}
// Weight image of one layer: (input i, output o), 64 outputs.
__host__ __device__ __forceinline__ uint32_t w_offset(uint32_t i, uint32_t o) {
    return (i >> 3) * 1024u + (o >> 3) * 128u + (i & 7u) * 16u + (o & 7u) * 2u;
}
__host__ __device__ constexpr uint32_t image_layer_offset(int l) {
    return l == 0 ? 0u : uint32_t(kMlpIn / 8 * 1024 + (l - 1) * 8 * 1024);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf16_float(uint16_t b) {
    return __uint_as_float(uint32_t(b) << 16);
}

// Write one sample row (F values) into an activation buffer, 8 at a time.
template <int F>
__device__ __forceinline__ void store_row(unsigned char* buf, uint32_t row, const float* v) {
#pragma unroll
    for (int c = 0; c < F / 8; c++) {
        uint4 q;
        q.x = uint32_t(bf16_bits(v[8 * c + 0])) | (uint32_t(bf16_bits(v[8 * c + 1])) << 16);
        q.y = uint32_t(bf16_bits(v[8 * c + 2])) | (uint32_t(bf16_bits(v[8 * c + 3])) << 16);
        q.z = uint32_t(bf16_bits(v[8 * c + 4])) | (uint32_t(bf16_bits(v[8 * c + 5])) << 16);
        q.w = uint32_t(bf16_bits(v[8 * c + 6])) | (uint32_t(bf16_bits(v[8 * c + 7])) << 16);
        *reinterpret_cast<uint4*>(buf + act_offset(row, 8 * c, F)) = q;
    }
}
// Read one sample row (F values) of an activation buffer.
template <int F>
__device__ __forceinline__ void load_row(const unsigned char* buf, uint32_t row, float* v) {
#pragma unroll
    for (int c = 0; c < F / 8; c++) {
        const uint4 q = *reinterpret_cast<const uint4*>(buf + act_offset(row, 8 * c, F));
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[8 * c + 2 * k] = bf16_float(uint16_t(w[k] & 0xFFFFu));
            v[8 * c + 2 * k + 1] = bf16_float(uint16_t(w[k] >> 16));
        }
    }
}

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
// Inference keeps no activations for a backward pass: two hidden buffers in
// turn (about 89 KB, two CTAs per SM).
struct alignas(1024) MlpFwdSmem {
    unsigned char w[kMlpImageBytes];
    unsigned char x[kMlpTile * kMlpIn * 2];
    unsigned char h[2][kMlpTile * 64 * 2];
    float bias[kMlpLayers][64];
    float dbias[kMlpLayers][64];
    uint64_t mbar;
    uint32_t tmem;
    uint32_t fail;
    __device__ unsigned char* hidden(int l) { return h[l & 1]; }
};

// TMEM columns: the 128 x 64 accumulator, then dW^T of each layer (64 rows
// x the layer's inputs), all starting at multiples of 16.
constexpr uint32_t kColD = 0;
__host__ __device__ constexpr uint32_t col_dw(int l) {
    return l == 0 ? 64u : 64u + 80u + 64u * uint32_t(l - 1);
}

// Weights (bf16 image) and biases into shared memory, barrier init, TMEM
// allocation by warp 0.  Returns the TMEM base address.
template <class SM>
__device__ __forceinline__ uint32_t mlp_prologue(SM& S, const MlpDev& m, uint32_t cols) {
    const uint4* src = reinterpret_cast<const uint4*>(m.wImage);
    uint4* dst = reinterpret_cast<uint4*>(S.w);
    for (uint32_t i = threadIdx.x; i < kMlpImageBytes / 16; i += blockDim.x) dst[i] = src[i];
    for (uint32_t i = threadIdx.x; i < kMlpLayers * 64; i += blockDim.x) {
        const int l = int(i / 64), o = int(i % 64);
        S.bias[l][o] = m.params[mlp_layer_offset(l) + (l == 0 ? kMlpIn : 64) * 64 + o];
        S.dbias[l][o] = 0.0f;
    }
    if (threadIdx.x == 0) {
        mbar_init(&S.mbar, 1);
        S.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        tmem_alloc(&S.tmem, cols);
        tmem_relinquish();
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return S.tmem;
}

template <class SM>
__device__ __forceinline__ void mlp_epilogue(SM& S, uint32_t tmem, uint32_t cols) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, cols);
    }
}

// One sample row of the input features into the X buffer (zeros past n).
template <class SM>
__device__ __forceinline__ void load_input(SM& S, const float* in, uint32_t n, uint32_t s,
                                           uint32_t row) {
    float v[kMlpIn];
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
    store_row<kMlpIn>(S.x, row, v);
}

// Wait for the MMAs committed to S.mbar; on expiry mark the CTA failed.
// Every thread of the CTA calls it at the same point; the outcome is made
// common with a block-wide vote so that no thread leaves a barrier behind.
template <class SM>
__device__ __forceinline__ bool mlp_wait(SM& S, uint32_t& phase, uint32_t* errorFlag) {
    bool ok = mbar_wait(&S.mbar, phase);
    phase ^= 1u;
    ok = __syncthreads_and(ok) != 0;
    if (!ok && threadIdx.x == 0) {
        S.fail = 1;
        atomicExch(errorFlag, 1u);
    }
    tc_fence_after();
    return ok;
}

// This thread's row (TMEM lane = threadIdx.x) of the 128 x 64 accumulator.
__device__ __forceinline__ void read_acc(uint32_t tmem, float* v) {
    const uint32_t lane = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int c = 0; c < 4; c++) tmem_ld16(tmem + lane + kColD + 16 * c, v + 16 * c);
    tmem_wait_ld();
}

// Forward pass of the tile in S.x: hidden activations into S.h[0..2], the
// output layer (bias added) into out[64].  Returns false after a failed wait.
template <class SM>
__device__ __forceinline__ bool forward_tile(SM& S, uint32_t tmem, uint32_t& phase,
                                             uint32_t* errorFlag, float* out) {
    const uint32_t row = threadIdx.x;
#pragma unroll 1
    for (int l = 0; l < kMlpLayers; l++) {
        const unsigned char* A = (l == 0) ? S.x : S.hidden(l - 1);
        const uint32_t K = (l == 0) ? kMlpIn : 64;
        if (threadIdx.x == 0) {
            const uint32_t a0 = smem_u32(A), b0 = smem_u32(S.w + image_layer_offset(l));
            for (uint32_t k0 = 0; k0 < K; k0 += 16) {
                // A = activations, K-major: K chunks 128 B apart, 8-row groups K/8*128 apart
                const uint64_t ad = smem_desc(a0 + (k0 / 8) * 128u, 128u, (K / 8) * 128u);
                // B = weights, MN-major: input chunks 1024 B apart, output groups 128 B apart
                const uint64_t bd = smem_desc(b0 + (k0 / 8) * 1024u, 1024u, 128u);
                mma_bf16(tmem + kColD, ad, bd, idesc_bf16(128, 64, false, true), k0 > 0 ? 1u : 0u);
            }
            mma_commit(&S.mbar);
        }
        if (!mlp_wait(S, phase, errorFlag)) return false;
        float v[64];
        read_acc(tmem, v);
#pragma unroll
        for (int o = 0; o < 64; o++) v[o] += S.bias[l][o];
        if (l < kMlpLayers - 1) {
#pragma unroll
            for (int o = 0; o < 64; o++) v[o] = fmaxf(v[o], 0.0f);
            store_row<64>(S.hidden(l), row, v);
        } else {
#pragma unroll
            for (int o = 0; o < 64; o++) out[o] = v[o];
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    return true;
}

__global__ void __launch_bounds__(kMlpTile, 2) k_mlp_forward(MlpDev m, const float* __restrict__ in,
                                                            uint32_t maxN,
                                                            const uint32_t* __restrict__ dCount,
                                                            float* __restrict__ out) {
    extern __shared__ __align__(1024) unsigned char smemRaw[];
    MlpFwdSmem& S = *reinterpret_cast<MlpFwdSmem*>(smemRaw);
    const uint32_t n = dCount ? min(*dCount, maxN) : maxN;
    const uint32_t tmem = mlp_prologue(S, m, 64);
    uint32_t phase = 0;
    const uint32_t tiles = (n + kMlpTile - 1) / kMlpTile;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t s = t * kMlpTile + threadIdx.x;
        load_input(S, in, n, s, threadIdx.x);
        fence_async_smem();
        __syncthreads();
        float o[64];
        if (!forward_tile(S, tmem, phase, m.errorFlag, o)) break;
        if (s < n) {
            float4* dst = reinterpret_cast<float4*>(out + size_t(s) * kMlpOut);
#pragma unroll
            for (int c = 0; c < kMlpOut / 4; c++)
                dst[c] = make_float4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
        }
    }
    mlp_epilogue(S, tmem, 64);
}

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
        MRB_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
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
    k_mlp_forward<<<mlp_grid(n, 2), kMlpTile, sizeof(MlpFwdSmem), st>>>(m, in, n, dCount, out);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mlp_gradients(const MlpDev& m, const float* in, const float* targets, uint32_t n, float* grad,
                  float* loss, cudaStream_t st, const uint32_t* dCount) {
    if (n == 0) return 0;
    if (mlp_smem_setup()) return MRB_E_CUDA;
    k_mlp_train<<<mlp_grid(n), kMlpTile, sizeof(MlpSmem), st>>>(m, in, targets, n, dCount, grad,
                                                               loss);
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
                       const uint32_t* dCount, float lr, cudaStream_t st) {
    MRB_CUDA(cudaMemsetAsync(m->loss.p, 0, 8, st));
    int r = mlp_gradients(m->dev(), in, targets, maxN, m->grad.as<float>(), m->loss.as<float>(),
                          st, dCount);
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
