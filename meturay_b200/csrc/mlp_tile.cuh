// Learned guiding MLP: the tensor-core forward pass shared by the plain
// inference kernel (mlp.cu) and the fused guide kernel (learned.cu).
//
// Shared-memory operand layout (no swizzle, "interleaved" core matrices):
// a core matrix is 8 rows x 16 bytes (8 bf16), its rows 16 bytes apart.
// Activations (128 samples x F features): core matrix (sample group sg,
// feature group fg) at sg*(F/8)*128 + fg*128.  Weights (in x 64 out): core
// matrix (input group ig, output group og) at ig*1024 + og*128.  The
// forward product D[s][o] = sum_i X[s][i] W[i][o] takes A = X K-major and
// B = W MN-major, M = 128 (one sample per TMEM lane), N = 64.  One elected
// thread issues the MMAs; completion is signalled through an mbarrier whose
// waits are bounded (on expiry the kernel flags an error, frees its tensor
// memory and returns).
#pragma once
#include <cuda_bf16.h>

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

// Inference keeps no activations for a backward pass: one activation
// buffer holds the input tile and then each hidden layer in turn (a
// layer's epilogue overwrites its own operand only after the product has
// completed).  About 56 KB: four CTAs per SM.
struct alignas(1024) MlpFwdSmem {
    unsigned char w[kMlpImageBytes];
    unsigned char x[kMlpTile * kMlpIn * 2];
    float bias[kMlpLayers][64];
    uint64_t mbar;
    uint32_t tmem;
    uint32_t fail;
    __device__ unsigned char* hidden(int) { return x; }
};
constexpr uint32_t kMlpFwdCtasPerSm = 4;
static_assert(kMlpTile * kMlpIn * 2 >= kMlpTile * 64 * 2, "x holds a hidden tile");

// TMEM column of the 128 x 64 forward accumulator.
constexpr uint32_t kColD = 0;

// Bias-gradient accumulators exist only in the training layout.
template <class SM>
__device__ __forceinline__ auto clear_dbias(SM& S, int l, int o) -> decltype(S.dbias, void()) {
    S.dbias[l][o] = 0.0f;
}
__device__ __forceinline__ void clear_dbias(MlpFwdSmem&, int, int) {}

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
        clear_dbias(S, l, o);
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

// Forward passes over tiles of 128 rows whose inputs and outputs IO
// supplies: io.rows() rows; io.input(s, v) writes the kMlpIn features of row
// s into v (called for every lane of a tile; rows past the end give zeros);
// io.output(s, o) takes the outputs of row s < rows (o[0..kMlpOut), bias
// added).  Four CTAs per SM (MlpFwdSmem, dynamic shared memory).
template <class IO>
__global__ void __launch_bounds__(kMlpTile, kMlpFwdCtasPerSm) k_mlp_forward_io(MlpDev m, IO io) {
    extern __shared__ __align__(1024) unsigned char smemRaw[];
    MlpFwdSmem& S = *reinterpret_cast<MlpFwdSmem*>(smemRaw);
    const uint32_t n = io.rows();
    const uint32_t tmem = mlp_prologue(S, m, 64);
    uint32_t phase = 0;
    const uint32_t tiles = (n + kMlpTile - 1) / kMlpTile;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t s = t * kMlpTile + threadIdx.x;
        {
            float v[kMlpIn];
            io.input(s, n, v);
            store_row<kMlpIn>(S.x, threadIdx.x, v);
        }
        fence_async_smem();
        __syncthreads();
        float o[64];
        if (!forward_tile(S, tmem, phase, m.errorFlag, o)) break;
        if (s < n) io.output(s, o);
    }
    mlp_epilogue(S, tmem, 64);
}

}  // namespace
}  // namespace mrb
