// Onesweep LSD radix sort of (key, value) pairs, 8-bit digits.
//
// Semantics follow cub::DeviceRadixSort::SortPairs / SortPairsDescending as
// the reference calls them (ParallelRadixSort.cuh:60-100, RayMemory.cu:187-228,
// LinearBVH.hpp:489-492): stable, on bits [beginBit, endBit), ascending or
// descending.  Structure (Adinets & Merrill, "Onesweep", 2022):
//   1. one read of the keys builds the digit histograms of every pass;
//   2. one exclusive scan per pass turns them into global digit offsets;
//   3. per pass, one kernel: each CTA takes a tile by atomic ticket, ranks
//      its keys with warp-level match/ballot multisplit, resolves its global
//      digit offsets with decoupled look-back, reorders the tile through
//      shared memory and writes coalesced runs.
// The element count may live on the device (rays whose count a previous
// kernel produced); tiles past the count exit at once, so the sort needs no
// host synchronisation and can be captured in a CUDA graph.
#include <mutex>

#include "common.cuh"
#include "sort.cuh"

namespace mrb {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 24;

template <class K>
__device__ __forceinline__ uint32_t digit_of(K k, int bit, uint32_t mask, bool desc) {
    uint32_t d = static_cast<uint32_t>(k >> bit) & mask;
    return desc ? (mask - d) : d;
}

// Pass histograms: hist[p * 256 + d] for pass p (digit bits beginBit + 8p).
template <class K>
__global__ void __launch_bounds__(kThreads) k_histogram(const K* __restrict__ keys,
                                                        const uint32_t* __restrict__ dCount,
                                                        uint32_t hCount, int beginBit, int endBit,
                                                        int desc, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[8][256];
    const int passes = (endBit - beginBit + 7) / 8;
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) (&sh[0][0])[i] = 0;
    __syncthreads();
    const uint32_t n = dCount ? *dCount : hCount;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        K k = keys[i];
        for (int p = 0; p < passes; p++) {
            int bit = beginBit + 8 * p;
            int nb = min(8, endBit - bit);
            uint32_t mask = (1u << nb) - 1u;
            atomicAdd(&sh[p][digit_of(k, bit, mask, desc != 0)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) {
        uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Exclusive scan of each pass histogram (one CTA per pass).
__global__ void __launch_bounds__(256) k_hist_scan(uint32_t* hist) {
    __shared__ uint32_t s[256];
    uint32_t* h = hist + blockIdx.x * 256;
    uint32_t v = h[threadIdx.x];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t t = (threadIdx.x >= off) ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    h[threadIdx.x] = s[threadIdx.x] - v;
}

template <class K>
struct SortSmem {
    K keys[kTile];
    uint32_t vals[kTile];
    uint32_t warpHist[kWarps][256];
    uint32_t digitStart[256];
    uint32_t globalBase[256];
    uint32_t tile;
    uint32_t validCount;
};

template <class K>
__global__ void __launch_bounds__(kThreads) k_onesweep(
    const K* __restrict__ keysIn, K* __restrict__ keysOut, const uint32_t* __restrict__ valsIn,
    uint32_t* __restrict__ valsOut, const uint32_t* __restrict__ dCount, uint32_t hCount,
    const uint32_t* __restrict__ passOffsets, uint32_t* tileStatus, uint32_t* tileTicket, int bit,
    int nbits, int desc, uint32_t* errorFlag) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    SortSmem<K>& sm = *reinterpret_cast<SortSmem<K>*>(smemRaw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t mask = (1u << nbits) - 1u;
    const uint32_t n = dCount ? *dCount : hCount;

    if (tid == 0) sm.tile = atomicAdd(tileTicket, 1u);
    for (int i = tid; i < kWarps * 256; i += kThreads) (&sm.warpHist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = sm.tile;
    const uint32_t base = tile * kTile;
    if (base >= n) return;

    // ---- load: warp w owns [base + w*512, base + (w+1)*512), item-major ----
    K key[kItems];
    uint32_t val[kItems], dig[kItems], rank[kItems];
    const uint32_t wbase = base + warp * (32 * kItems);
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        uint32_t idx = wbase + i * 32 + lane;
        bool ok = idx < n;
        key[i] = ok ? keysIn[idx] : K(0);
        val[i] = ok ? (valsIn ? valsIn[idx] : idx) : 0u;
        dig[i] = digit_of(key[i], bit, mask, desc != 0);
    }
    // ---- warp-level multisplit ranking (stable: item-major, lane order) ----
    const uint32_t ltMask = (1u << lane) - 1u;
    uint32_t* wh = sm.warpHist[warp];
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        uint32_t idx = wbase + i * 32 + lane;
        bool ok = idx < n;
        uint32_t vmask = __ballot_sync(0xFFFFFFFFu, ok);
        if (ok) {
            uint32_t peers = __match_any_sync(vmask, dig[i]);
            uint32_t prior = wh[dig[i]];
            __syncwarp(vmask);
            if (lane == (__ffs(peers) - 1)) wh[dig[i]] = prior + __popc(peers);
            rank[i] = prior + __popc(peers & ltMask);
        }
        __syncwarp();
    }
    __syncthreads();

    // ---- per digit: warp prefix, tile count, look-back ----
    {
        const uint32_t d = tid;  // kThreads == 256 digits
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            uint32_t c = sm.warpHist[w][d];
            sm.warpHist[w][d] = run;
            run += c;
        }
        const uint32_t total = run;
        // tile-local exclusive scan over digits (digitStart)
        sm.digitStart[d] = total;
        __syncthreads();
        for (int off = 1; off < 256; off <<= 1) {
            uint32_t t = (d >= (uint32_t)off) ? sm.digitStart[d - off] : 0u;
            __syncthreads();
            sm.digitStart[d] += t;
            __syncthreads();
        }
        sm.digitStart[d] -= total;
        if (d == 255) sm.validCount = sm.digitStart[255] + total;

        // decoupled look-back over earlier tiles for digit d
        volatile uint32_t* st = tileStatus;
        uint32_t excl = 0;
        if (tile == 0) {
            st[d] = kFlagPrefix | total;
        } else {
            st[tile * 256 + d] = kFlagAgg | total;
            int32_t k = static_cast<int32_t>(tile) - 1;
            uint32_t spins = 0;
            while (k >= 0) {
                uint32_t s = st[k * 256 + d];
                uint32_t flag = s & ~kValueMask;
                if (flag == 0) {
                    if (++spins > kSpinLimit) {
                        atomicExch(errorFlag, 1u);
                        break;
                    }
                    continue;
                }
                excl += s & kValueMask;
                if (flag == kFlagPrefix) break;
                k--;
            }
            __threadfence();
            st[tile * 256 + d] = kFlagPrefix | (excl + total);
        }
        sm.globalBase[d] = passOffsets[d] + excl;
    }
    __syncthreads();

    // ---- reorder the tile through shared memory ----
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            uint32_t p = sm.digitStart[dig[i]] + sm.warpHist[warp][dig[i]] + rank[i];
            sm.keys[p] = key[i];
            sm.vals[p] = val[i];
        }
    }
    __syncthreads();
    const uint32_t cnt = sm.validCount;
    for (uint32_t j = tid; j < cnt; j += kThreads) {
        K k = sm.keys[j];
        uint32_t d = digit_of(k, bit, mask, desc != 0);
        uint32_t g = sm.globalBase[d] + (j - sm.digitStart[d]);
        keysOut[g] = k;
        valsOut[g] = sm.vals[j];
    }
}

template <class K>
__global__ void k_copy_back(const K* __restrict__ ks, K* __restrict__ kd,
                            const uint32_t* __restrict__ vs, uint32_t* __restrict__ vd,
                            const uint32_t* __restrict__ dCount, uint32_t hCount) {
    const uint32_t n = dCount ? *dCount : hCount;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        kd[i] = ks[i];
        vd[i] = vs[i];
    }
}

inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

// Head of the scratch, cleared by one memset per sort: eight 256-bin
// histograms, eight pass tickets, the give-up flag.
constexpr size_t kHistBytes = size_t(8) * 256 * 4;
constexpr size_t kHeadBytes = kHistBytes + size_t(8) * 4 + 4;

}  // namespace

size_t radix_sort_temp_bytes(uint32_t maxCount, int keyBytes, int beginBit, int endBit) {
    const int passes = (endBit - beginBit + 7) / 8;
    const size_t tiles = (size_t(maxCount) + kTile - 1) / kTile;
    size_t bytes = 0;
    bytes += align_up(kHeadBytes);                          // histograms, tickets, error flag
    bytes += align_up((tiles + 1) * 256 * 4);               // tile status
    bytes += align_up(size_t(maxCount) * keyBytes);         // key ping-pong
    bytes += align_up(size_t(maxCount) * 4);                // value ping-pong
    (void)passes;
    return bytes;
}

template <class K>
int radix_sort_pairs(K* keys, uint32_t* vals, const uint32_t* dCount, uint32_t maxCount,
                     int beginBit, int endBit, bool desc, void* temp, size_t tempBytes,
                     cudaStream_t stream, bool valsAreIota) {
    if (endBit <= beginBit || maxCount == 0) return 0;
    if (tempBytes < radix_sort_temp_bytes(maxCount, sizeof(K), beginBit, endBit)) {
        set_error("radix sort: scratch of %zu bytes is below the %zu required", tempBytes,
                  radix_sort_temp_bytes(maxCount, sizeof(K), beginBit, endBit));
        return -1;
    }
    const int passes = (endBit - beginBit + 7) / 8;
    const uint32_t tiles = (maxCount + kTile - 1) / kTile;
    unsigned char* p = static_cast<unsigned char*>(temp);
    uint32_t* hist = reinterpret_cast<uint32_t*>(p);
    uint32_t* tickets = hist + 8 * 256;
    uint32_t* err = tickets + 8;
    p += align_up(kHeadBytes);
    uint32_t* status = reinterpret_cast<uint32_t*>(p);
    p += align_up((size_t(tiles) + 1) * 256 * 4);
    K* keysAlt = reinterpret_cast<K*>(p);
    p += align_up(size_t(maxCount) * sizeof(K));
    uint32_t* valsAlt = reinterpret_cast<uint32_t*>(p);

    const size_t smem = sizeof(SortSmem<K>);
    // the attribute is set once per device, before any stream capture; the
    // lock keeps two host threads' first sorts on a device from racing
    constexpr int kMaxDevices = 64;
    static bool configured[2][kMaxDevices] = {};
    static std::mutex configuredMutex;
    int dev = 0;
    MRB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("radix sort: device %d out of the supported range [0, %d)", dev, kMaxDevices);
        return -1;
    }
    {
        std::lock_guard<std::mutex> lock(configuredMutex);
        bool& done = configured[sizeof(K) == 8 ? 1 : 0][dev];
        if (!done) {
            MRB_CUDA(cudaFuncSetAttribute(k_onesweep<K>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
            done = true;
        }
    }
    MRB_CUDA(cudaMemsetAsync(hist, 0, kHeadBytes, stream));  // histograms, tickets, flag
    k_histogram<K><<<148 * 4, kThreads, 0, stream>>>(keys, dCount, maxCount, beginBit, endBit,
                                                    desc ? 1 : 0, hist);
    k_hist_scan<<<passes, 256, 0, stream>>>(hist);
    K* kbuf[2] = {keys, keysAlt};
    uint32_t* vbuf[2] = {vals, valsAlt};
    for (int pass = 0; pass < passes; pass++) {
        const int src = pass & 1, dst = src ^ 1;
        const int bit = beginBit + 8 * pass;
        const int nb = (endBit - bit) < 8 ? (endBit - bit) : 8;
        const uint32_t* vin = (pass == 0 && valsAreIota) ? nullptr : vbuf[src];
        MRB_CUDA(cudaMemsetAsync(status, 0, size_t(tiles) * 256 * 4, stream));
        k_onesweep<K><<<tiles, kThreads, smem, stream>>>(kbuf[src], kbuf[dst], vin, vbuf[dst],
                                                        dCount, maxCount, hist + pass * 256,
                                                        status, tickets + pass, bit, nb,
                                                        desc ? 1 : 0, err);
    }
    if (passes & 1) {
        // odd pass count: the result sits in the scratch copy
        k_copy_back<K><<<148 * 4, 256, 0, stream>>>(keysAlt, keys, valsAlt, vals, dCount,
                                                   maxCount);
    }
    MRB_CUDA(cudaGetLastError());
    return 0;
}

uint32_t* radix_sort_error_flag(void* temp, uint32_t) {
    return reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(temp) + kHistBytes) + 8;
}

template int radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, const uint32_t*, uint32_t, int, int,
                                        bool, void*, size_t, cudaStream_t, bool);
template int radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, const uint32_t*, uint32_t, int, int,
                                        bool, void*, size_t, cudaStream_t, bool);

}  // namespace mrb
