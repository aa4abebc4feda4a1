// Exclusive prefix sum of 32-bit counts (three phases: per-block sums, a
// scan of the block sums, and a per-block scan that adds the block's base).
// Used by the sparse-voxel-octree build for voxel offsets and level ranks.
#include "common.cuh"
#include "scan.cuh"

namespace mrb {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warpSums[kScanBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = (lane < kScanBlock / 32) ? warpSums[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanBlock / 32) warpSums[lane] = s;
    }
    __syncthreads();
    const uint32_t warpBase = warp ? warpSums[warp - 1] : 0u;
    *total = warpSums[kScanBlock / 32 - 1];
    __syncthreads();
    return warpBase + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_tile_sums(const uint32_t* __restrict__ in, uint32_t n,
                                                          uint32_t* __restrict__ sums) {
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
    for (int i = 0; i < kScanItems; i++)
        if (base + i < n) s += in[base + i];
    uint32_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_sums(uint32_t* sums, uint32_t count) {
    // one block walks the tile sums in chunks of kScanBlock
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t b = 0; b < count; b += kScanBlock) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < count ? sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive(v, &total);
        if (i < count) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanBlock) k_tile_scan(const uint32_t* __restrict__ in, uint32_t n,
                                                          const uint32_t* __restrict__ sums,
                                                          uint32_t* __restrict__ out) {
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
    for (int i = 0; i < kScanItems; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t total;
    uint32_t run = sums[blockIdx.x] + block_exclusive(s, &total);
    for (int i = 0; i < kScanItems; i++) {
        if (base + i < n) out[base + i] = run;
        else if (base + i == n) out[n] = run;  // the grand total
        run += v[i];
    }
}

}  // namespace

size_t exclusive_scan_temp_bytes(uint32_t n) {
    return (size_t(n) / kScanTile + 2) * 4;
}

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, void* temp,
                       cudaStream_t stream) {
    if (n == 0) {
        MRB_CUDA(cudaMemsetAsync(out, 0, 4, stream));
        return 0;
    }
    // tiles cover n + 1 outputs so the grand total lands in out[n]
    const uint32_t tiles = n / kScanTile + 1;
    uint32_t* sums = static_cast<uint32_t*>(temp);
    k_tile_sums<<<tiles, kScanBlock, 0, stream>>>(in, n, sums);
    k_scan_sums<<<1, kScanBlock, 0, stream>>>(sums, tiles);
    k_tile_scan<<<tiles, kScanBlock, 0, stream>>>(in, n, sums, out);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
