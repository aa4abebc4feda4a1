// Traversal tree by parallel locally-ordered clustering (PLOC; Meister and
// Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction", IEEE TVCG 2018), from the LBVH's Morton-sorted
// leaves.
//
// The LBVH splits where the Morton codes split, so over a sparse scene its
// upper nodes are loose boxes around far-apart geometry and rays open many
// of them to find nothing.  PLOC builds bottom-up instead: every cluster
// (first the leaves, in Morton order) looks for the neighbour within a
// window of kRadius clusters on either side whose merged box has the least
// surface area; mutually nearest pairs merge into a new inner node; the
// survivors are compacted, keeping their Morton order, and the step repeats
// until one cluster is left.  Every step is deterministic: ties go to the
// lower index and new nodes are numbered by a prefix sum over the merging
// pairs.
//
// The result uses the LBVH's numbering (leaf g < n is sorted slot g, inner
// node j is global n + j), so the 8-wide collapse (wide.cu) takes it as it
// takes the LBVH.  The LBVH itself, in the reference's numbering, is kept
// unchanged for its parity checks and the binary traversal.
#include <algorithm>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "ploc.cuh"
#include "scan.cuh"

namespace mrb {
namespace {

constexpr int kRadius = 16;
constexpr int kBlock = 256;

__device__ __forceinline__ void node_box(uint32_t g, const PlocIn& in, const float* inner,
                                         float b[6]) {
    const float* s = (g < in.n) ? in.triAabb + 6 * size_t(in.sortedIdx[g])
                                : inner + 6 * size_t(g - in.n);
    for (int c = 0; c < 6; c++) b[c] = s[c];
}

__device__ __forceinline__ float merged_area(const float* a, const float* b) {
    const float dx = fmaxf(a[3], b[3]) - fminf(a[0], b[0]);
    const float dy = fmaxf(a[4], b[4]) - fminf(a[1], b[1]);
    const float dz = fmaxf(a[5], b[5]) - fminf(a[2], b[2]);
    return dx * dy + dy * dz + dz * dx;
}

// Nearest neighbour of every cluster in [i - kRadius, i + kRadius].
__global__ void __launch_bounds__(kBlock) k_ploc_nn(const uint32_t* __restrict__ C, uint32_t m,
                                                    PlocIn in, const float* __restrict__ inner,
                                                    uint32_t* __restrict__ nn) {
    __shared__ float sb[(kBlock + 2 * kRadius) * 6];
    const int b0 = int(blockIdx.x) * kBlock;
    for (int k = threadIdx.x; k < kBlock + 2 * kRadius; k += kBlock) {
        const int j = b0 - kRadius + k;
        if (j >= 0 && j < int(m)) node_box(C[j], in, inner, sb + 6 * k);
    }
    __syncthreads();
    const int i = b0 + int(threadIdx.x);
    if (i >= int(m)) return;
    const float* bi = sb + 6 * (threadIdx.x + kRadius);
    float best = INFINITY;
    int bj = (i == 0) ? 1 : i - 1;
    for (int d = -kRadius; d <= kRadius; d++) {
        const int j = i + d;
        if (d == 0 || j < 0 || j >= int(m)) continue;
        const float a = merged_area(bi, sb + 6 * (int(threadIdx.x) + kRadius + d));
        if (a < best) {  // ascending j: equal areas keep the lower index
            best = a;
            bj = j;
        }
    }
    nn[i] = uint32_t(bj);
}

// merge[i]: i is the lower index of a mutually nearest pair; keep[i]: i is
// not the upper index of one.
__global__ void k_ploc_flags(const uint32_t* __restrict__ nn, uint32_t m, uint32_t* merge,
                             uint32_t* keep) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t j = nn[i];
        const bool mutual = nn[j] == i;
        merge[i] = (mutual && i < j) ? 1u : 0u;
        keep[i] = (mutual && i > j) ? 0u : 1u;
    }
}

__global__ void k_ploc_merge(uint32_t* C, const uint32_t* __restrict__ nn, uint32_t m,
                             const uint32_t* __restrict__ merge, const uint32_t* __restrict__ slot,
                             uint32_t base, PlocIn in, PlocOut out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (!merge[i]) continue;
        const uint32_t j = nn[i];
        const uint32_t node = base + slot[i];
        const uint32_t a = C[i], b = C[j];
        float ba[6], bb[6];
        node_box(a, in, out.inner, ba);
        node_box(b, in, out.inner, bb);
        float* o = out.inner + 6 * size_t(node);
        for (int c = 0; c < 3; c++) {
            o[c] = fminf(ba[c], bb[c]);
            o[3 + c] = fmaxf(ba[3 + c], bb[3 + c]);
        }
        out.left[node] = a;
        out.right[node] = b;
        C[i] = in.n + node;
    }
}

__global__ void k_ploc_compact(const uint32_t* __restrict__ C, uint32_t m,
                               const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos,
                               uint32_t* Cout) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        if (keep[i]) Cout[pos[i]] = C[i];
}

__global__ void k_ploc_iota(uint32_t* C, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        C[i] = i;
}

__global__ void k_ploc_root(const uint32_t* C, uint32_t* root) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *root = C[0];
}

// Sum of the inner boxes' half surface areas (the SAH's node term) in
// double; blocks reduce in shared memory and add their sums atomically.
__global__ void __launch_bounds__(256) k_area_sum(const float* __restrict__ inner, uint32_t count,
                                                  double* out) {
    __shared__ double red[256];
    double a = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += gridDim.x * blockDim.x) {
        const float* b = inner + 6 * size_t(i);
        const double dx = double(b[3]) - b[0], dy = double(b[4]) - b[1], dz = double(b[5]) - b[2];
        a += dx * dy + dy * dz + dz * dx;
    }
    red[threadIdx.x] = a;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

inline uint32_t grid_of(uint32_t n, uint32_t block) {
    const uint32_t b = (n + block - 1) / block;
    return std::max(1u, std::min(b, 148u * 16u));
}

}  // namespace

int inner_area_sum(const float* inner, uint32_t count, double* scratch8, double* out,
                   cudaStream_t st) {
    MRB_CUDA(cudaMemsetAsync(scratch8, 0, 8, st));
    if (count) k_area_sum<<<grid_of(count, 256), 256, 0, st>>>(inner, count, scratch8);
    MRB_CUDA(cudaGetLastError());
    MRB_CUDA(cudaMemcpyAsync(out, scratch8, 8, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

size_t ploc_scratch_bytes(uint32_t n) {
    // C x2, nn, merge, keep, slot (n + 1), pos (n + 1), scan temp
    const size_t w = (size_t(n) + 1) * 4;
    return 7 * w + exclusive_scan_temp_bytes(n) + 256;
}

int ploc_build(const PlocIn& in, const PlocOut& out, void* scratch, uint32_t* iterations,
               cudaStream_t st) {
    const uint32_t n = in.n;
    if (n < 2) {
        set_error("PLOC: needs at least two leaves");
        return MRB_E_ARG;
    }
    const size_t w = (size_t(n) + 1) * 4;
    char* p = static_cast<char*>(scratch);
    uint32_t* C[2] = {reinterpret_cast<uint32_t*>(p), reinterpret_cast<uint32_t*>(p + w)};
    uint32_t* nn = reinterpret_cast<uint32_t*>(p + 2 * w);
    uint32_t* merge = reinterpret_cast<uint32_t*>(p + 3 * w);
    uint32_t* keep = reinterpret_cast<uint32_t*>(p + 4 * w);
    uint32_t* slot = reinterpret_cast<uint32_t*>(p + 5 * w);
    uint32_t* pos = reinterpret_cast<uint32_t*>(p + 6 * w);
    void* scanTemp = p + 7 * w;
    k_ploc_iota<<<grid_of(n, 256), 256, 0, st>>>(C[0], n);
    MRB_CUDA(cudaGetLastError());
    uint32_t m = n, base = 0;
    int cur = 0, it = 0;
    // every step merges at least the pair with the globally least merged
    // area, so n - 1 steps bound the loop
    while (m > 1 && it < int(n)) {
        k_ploc_nn<<<(m + kBlock - 1) / kBlock, kBlock, 0, st>>>(C[cur], m, in, out.inner, nn);
        k_ploc_flags<<<grid_of(m, 256), 256, 0, st>>>(nn, m, merge, keep);
        MRB_CUDA(cudaGetLastError());
        int r;
        if ((r = exclusive_scan_u32(merge, slot, m, scanTemp, st))) return r;
        k_ploc_merge<<<grid_of(m, 256), 256, 0, st>>>(C[cur], nn, m, merge, slot, base, in, out);
        MRB_CUDA(cudaGetLastError());
        if ((r = exclusive_scan_u32(keep, pos, m, scanTemp, st))) return r;
        k_ploc_compact<<<grid_of(m, 256), 256, 0, st>>>(C[cur], m, keep, pos, C[cur ^ 1]);
        MRB_CUDA(cudaGetLastError());
        uint32_t h[2] = {0, 0};
        MRB_CUDA(cudaMemcpyAsync(&h[0], slot + m, 4, cudaMemcpyDeviceToHost, st));
        MRB_CUDA(cudaMemcpyAsync(&h[1], pos + m, 4, cudaMemcpyDeviceToHost, st));
        MRB_CUDA(cudaStreamSynchronize(st));
        if (h[0] == 0 || h[1] + h[0] != m) {
            set_error("PLOC: step %d merged %u of %u clusters", it, h[0], m);
            return MRB_E_DEVICE;
        }
        base += h[0];
        m = h[1];
        cur ^= 1;
        it++;
    }
    if (m != 1 || base != n - 1) {
        set_error("PLOC: %u clusters and %u inner nodes left after %d steps", m, base, it);
        return MRB_E_DEVICE;
    }
    k_ploc_root<<<1, 32, 0, st>>>(C[cur], out.root);
    MRB_CUDA(cudaGetLastError());
    if (iterations) *iterations = uint32_t(it);
    return 0;
}

}  // namespace mrb
