// Reconstruction filters: splat camera samples onto the image.
//
// The reference (GPUReconFilter.h:59-260, GPUReconFilterKC.cuh:34-377)
// expands every sample to the pixels its filter reaches (one (pixel,
// sample) pair per pixel), radix-sorts the pairs by pixel and reduces each
// pixel's run with a block or warp reduction.  Here:
//   - the general entry point (any image coordinates) keeps that structure,
//     but compacts the valid pairs first (count, scan, write in sample
//     order), sorts only those with the onesweep sort on the pixel bits,
//     keeps the element count on the device (no host round trip, so the
//     splat can sit inside a captured graph) and sums each pixel's run in
//     one thread in ascending sample order;
//   - the tracer's own samples lie on the camera's stratified grid, so each
//     pixel finds its candidates by index arithmetic in a small
//     neighbourhood and sums them in the same ascending sample order: the
//     same bits as the general path, with no pairs, no sort and no atomics.
// Per pixel, ascending sample order is also the order of the reference's
// own CPU expectation (Test_TracerCUDA/T_ReconFilter.cu:96-140).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mrb200.h"
#include "recon.cuh"
#include "scan.cuh"
#include "sort.cuh"

namespace mrb {

namespace {

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Where a sample lands: modf of its image coordinates and the window of
// pixel offsets KCExpandSamplesToPixels walks (GPUReconFilterKC.cuh:44-91).
struct SamplePix {
    float fx, fy;        // integer parts (as floats)
    int32_t ix, iy;      // integer parts (as ints)
    int32_t x0, x1, y0, y1;  // offset window [x0, x1) x [y0, y1)
    bool ok;
};

__host__ __device__ inline SamplePix sample_pix(float cx, float cy, uint32_t wh) {
    SamplePix s{};
    // coordinates beyond +-1e9 (or NaN) reach no pixel of any image this
    // library accepts; they are dropped instead of overflowing the ints
    s.ok = fabsf(cx) < 1.0e9f && fabsf(cy) < 1.0e9f;
    if (!s.ok) return s;
    s.fx = truncf(cx);
    s.fy = truncf(cy);
    const float relX = cx - s.fx, relY = cy - s.fy;
    s.ix = static_cast<int32_t>(s.fx);
    s.iy = static_cast<int32_t>(s.fy);
    const int32_t range = static_cast<int32_t>(wh);
    const int32_t lo = -(range - 1) / 2, hi = (range + 2) / 2;
    s.x0 = lo; s.x1 = hi; s.y0 = lo; s.y1 = hi;
    // even windows lean towards the half of the pixel the sample is in
    if (range % 2 == 0) {
        if (relX < 0.5f) { s.x0 -= 1; s.x1 -= 1; }
        if (relY < 0.5f) { s.y0 -= 1; s.y1 -= 1; }
    }
    return s;
}

// The distance test for offset (x, y) (radius 0: the sample's own pixel).
__host__ __device__ inline bool sample_reaches(const SamplePix& s, float cx, float cy, int32_t x,
                                               int32_t y, uint32_t wh, float r2) {
    if (wh == 1u) return true;
    const float pcx = (s.fx + static_cast<float>(x)) + 0.5f;
    const float pcy = (s.fy + static_cast<float>(y)) + 0.5f;
    const float dx = cx - pcx, dy = cy - pcy;
    return (dx * dx + dy * dy) <= r2;
}

__host__ __device__ inline bool in_segment(const ImageSeg& g, int32_t px, int32_t py) {
    return px >= 0 && px < g.resW && py >= 0 && py < g.resH && px >= g.offX &&
           px < g.offX + g.w && py >= g.offY && py < g.offY + g.h;
}

// Pass 1: number of (pixel, sample) pairs per sample.
__global__ void __launch_bounds__(256) k_expand_count(const float2* __restrict__ coords, uint32_t n,
                                                      ReconFilterDev f, ImageSeg g,
                                                      uint32_t* __restrict__ count) {
    const float r2 = f.radius * f.radius;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 c = coords[i];
        const SamplePix s = sample_pix(c.x, c.y, f.wh);
        uint32_t k = 0;
        if (s.ok) {
            for (int32_t y = s.y0; y < s.y1; y++)
                for (int32_t x = s.x0; x < s.x1; x++)
                    if (sample_reaches(s, c.x, c.y, x, y, f.wh, r2) &&
                        in_segment(g, s.ix + x, s.iy + y))
                        k++;
        }
        count[i] = k;
    }
}

// Pass 2: the pairs themselves, at the sample's scanned offset, in the
// reference's (y, x) window order.  Keys are segment-local pixel indices.
__global__ void __launch_bounds__(256) k_expand_write(const float2* __restrict__ coords, uint32_t n,
                                                      ReconFilterDev f, ImageSeg g,
                                                      const uint32_t* __restrict__ offset,
                                                      uint32_t* __restrict__ keys,
                                                      uint32_t* __restrict__ vals) {
    const float r2 = f.radius * f.radius;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 c = coords[i];
        const SamplePix s = sample_pix(c.x, c.y, f.wh);
        if (!s.ok) continue;
        uint32_t o = offset[i];
        for (int32_t y = s.y0; y < s.y1; y++)
            for (int32_t x = s.x0; x < s.x1; x++) {
                const int32_t px = s.ix + x, py = s.iy + y;
                if (!sample_reaches(s, c.x, c.y, x, y, f.wh, r2) || !in_segment(g, px, py))
                    continue;
                keys[o] = static_cast<uint32_t>((py - g.offY) * g.w + (px - g.offX));
                vals[o] = i;
                o++;
            }
    }
}

// Run boundaries of the sorted keys: [begin[p], end[p]) for every pixel
// that received a pair (both stay 0 for the others).
__global__ void __launch_bounds__(256) k_pixel_bounds(const uint32_t* __restrict__ keys,
                                                      const uint32_t* __restrict__ dCount,
                                                      uint32_t* __restrict__ begin,
                                                      uint32_t* __restrict__ end) {
    const uint32_t n = *dCount;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        if (i == 0 || keys[i - 1] != k) begin[k] = i;
        if (i + 1 == n || keys[i + 1] != k) end[k] = i + 1;
    }
}

// KCFilterToImgBlock / KCFilterToImgWarp (GPUReconFilterKC.cuh:146-377):
// one thread per segment pixel sums its run in sample order, then adds the
// sums into the image and the weight into the sample counts.
template <int C>
__global__ void __launch_bounds__(256) k_filter_pixels(
    const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
    const uint32_t* __restrict__ vals, const float* __restrict__ values,
    const float2* __restrict__ coords, ReconFilterDev f, ImageSeg g, float multiplier,
    float* __restrict__ pixels, float* __restrict__ counts) {
    const uint32_t total = static_cast<uint32_t>(g.w) * static_cast<uint32_t>(g.h);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += gridDim.x * blockDim.x) {
        const uint32_t b = begin[q], e = end[q];
        if (b == e) continue;
        const int32_t gx = static_cast<int32_t>(q % static_cast<uint32_t>(g.w)) + g.offX;
        const int32_t gy = static_cast<int32_t>(q / static_cast<uint32_t>(g.w)) + g.offY;
        const float pcx = static_cast<float>(gx) + 0.5f, pcy = static_cast<float>(gy) + 0.5f;
        float acc[C];
        for (int k = 0; k < C; k++) acc[k] = 0.0f;
        float wsum = 0.0f;
        for (uint32_t i = b; i < e; i++) {
            const uint32_t sid = vals[i];
            const float2 c = coords[sid];
            const float w = recon_weight(f, pcx, pcy, c.x, c.y) * multiplier;
            wsum += w;
            if constexpr (C == 4) {
                const float4 v = reinterpret_cast<const float4*>(values)[sid];
                acc[0] += w * v.x;
                acc[1] += w * v.y;
                acc[2] += w * v.z;
                acc[3] += w * v.w;
            } else {
                acc[0] += w * values[sid];
            }
        }
        if constexpr (C == 4) {
            float4* p4 = reinterpret_cast<float4*>(pixels) + q;
            float4 p = *p4;
            p.x += acc[0];
            p.y += acc[1];
            p.z += acc[2];
            p.w += acc[3];
            *p4 = p;
        } else {
            pixels[q] += acc[0];
        }
        counts[q] += wsum;
    }
}

// Tracer splat over the camera's sample grid.  Sample sid = sy * (W*sp) + sx
// belongs to pixel (sx / sp, sy / sp) and its image coordinates lie within
// one pixel of it, so pixel p can only receive samples of the pixels q with
// q in [p - hi, p - loMin + 1] per axis (the window offsets being
// [loMin, hi)).  Rows then columns ascending = ascending sample order.
__global__ void __launch_bounds__(256) k_filter_grid(const float4* __restrict__ samples,
                                                     const float2* __restrict__ coords,
                                                     uint32_t width, uint32_t height, uint32_t sp,
                                                     ReconFilterDev f, float multiplier,
                                                     float4* __restrict__ image) {
    const int32_t range = static_cast<int32_t>(f.wh);
    const int32_t hi = (range + 2) / 2;
    const int32_t loMin = -(range - 1) / 2 - ((range % 2 == 0) ? 1 : 0);
    const float r2 = f.radius * f.radius;
    const int32_t S = static_cast<int32_t>(sp);
    const int32_t SW = static_cast<int32_t>(width) * S, SH = static_cast<int32_t>(height) * S;
    const uint32_t total = width * height;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total;
         p += gridDim.x * blockDim.x) {
        const int32_t px = static_cast<int32_t>(p % width), py = static_cast<int32_t>(p / width);
        const float pcx = static_cast<float>(px) + 0.5f, pcy = static_cast<float>(py) + 0.5f;
        const int32_t sy0 = max(0, (py - hi) * S), sy1 = min(SH, (py - loMin + 2) * S);
        const int32_t sx0 = max(0, (px - hi) * S), sx1 = min(SW, (px - loMin + 2) * S);
        float ax = 0.0f, ay = 0.0f, az = 0.0f, wsum = 0.0f;
        for (int32_t sy = sy0; sy < sy1; sy++)
            for (int32_t sx = sx0; sx < sx1; sx++) {
                const uint32_t sid = static_cast<uint32_t>(sy) * static_cast<uint32_t>(SW) +
                                     static_cast<uint32_t>(sx);
                const float2 c = coords[sid];
                const SamplePix s = sample_pix(c.x, c.y, f.wh);
                if (!s.ok) continue;
                const int32_t x = px - s.ix, y = py - s.iy;
                if (x < s.x0 || x >= s.x1 || y < s.y0 || y >= s.y1) continue;
                if (!sample_reaches(s, c.x, c.y, x, y, f.wh, r2)) continue;
                const float w = recon_weight(f, pcx, pcy, c.x, c.y) * multiplier;
                const float4 v = samples[sid];
                wsum += w;
                ax += w * v.x;
                ay += w * v.y;
                az += w * v.z;
            }
        float4 acc = image[p];
        image[p] = make_float4(acc.x + ax, acc.y + ay, acc.z + az, acc.w + wsum);
    }
}

// The same splat for a 16x16 pixel tile per block: the tile's samples with
// their halo (coordinates and values) are staged once in shared memory by
// coalesced row loads, then each thread sums its pixel's window from there in
// the order of k_filter_grid (rows, then columns, ascending), so the image is
// the same bit for bit; only the reads change (each sample was read by up to
// win^2 pixels through L1/L2).
constexpr int32_t kFilterTile = 16;
__global__ void __launch_bounds__(256) k_filter_grid_tiled(const float4* __restrict__ samples,
                                                           const float2* __restrict__ coords,
                                                           uint32_t width, uint32_t height,
                                                           uint32_t sp, ReconFilterDev f,
                                                           float multiplier,
                                                           float4* __restrict__ image) {
    extern __shared__ float4 smem[];
    const int32_t range = static_cast<int32_t>(f.wh);
    const int32_t hi = (range + 2) / 2;
    const int32_t loMin = -(range - 1) / 2 - ((range % 2 == 0) ? 1 : 0);
    const float r2 = f.radius * f.radius;
    const int32_t S = static_cast<int32_t>(sp);
    const int32_t SW = static_cast<int32_t>(width) * S, SH = static_cast<int32_t>(height) * S;
    // staged sample rectangle: pixels [t0 - hi, t0 + tile - 1 - loMin + 1], times S
    const int32_t span = (kFilterTile + hi - loMin + 1) * S;
    float4* sv = smem;                                           // span * span values
    float2* sc = reinterpret_cast<float2*>(smem + span * span);  // span * span coordinates
    const int32_t tilesX = (static_cast<int32_t>(width) + kFilterTile - 1) / kFilterTile;
    const int32_t tx0 = (static_cast<int32_t>(blockIdx.x) % tilesX) * kFilterTile;
    const int32_t ty0 = (static_cast<int32_t>(blockIdx.x) / tilesX) * kFilterTile;
    const int32_t ox = (tx0 - hi) * S, oy = (ty0 - hi) * S;      // staged origin (samples)
    for (int32_t i = threadIdx.x; i < span * span; i += blockDim.x) {
        const int32_t ly = i / span, lx = i - ly * span;
        const int32_t sy = oy + ly, sx = ox + lx;
        if (sy >= 0 && sy < SH && sx >= 0 && sx < SW) {
            const size_t sid = size_t(sy) * size_t(SW) + size_t(sx);
            sc[i] = coords[sid];
            sv[i] = samples[sid];
        }
    }
    __syncthreads();
    const int32_t px = tx0 + static_cast<int32_t>(threadIdx.x) % kFilterTile;
    const int32_t py = ty0 + static_cast<int32_t>(threadIdx.x) / kFilterTile;
    if (px >= static_cast<int32_t>(width) || py >= static_cast<int32_t>(height)) return;
    const float pcx = static_cast<float>(px) + 0.5f, pcy = static_cast<float>(py) + 0.5f;
    const int32_t sy0 = max(0, (py - hi) * S), sy1 = min(SH, (py - loMin + 2) * S);
    const int32_t sx0 = max(0, (px - hi) * S), sx1 = min(SW, (px - loMin + 2) * S);
    float ax = 0.0f, ay = 0.0f, az = 0.0f, wsum = 0.0f;
    for (int32_t sy = sy0; sy < sy1; sy++)
        for (int32_t sx = sx0; sx < sx1; sx++) {
            const int32_t li = (sy - oy) * span + (sx - ox);
            const float2 c = sc[li];
            const SamplePix s = sample_pix(c.x, c.y, f.wh);
            if (!s.ok) continue;
            const int32_t x = px - s.ix, y = py - s.iy;
            if (x < s.x0 || x >= s.x1 || y < s.y0 || y >= s.y1) continue;
            if (!sample_reaches(s, c.x, c.y, x, y, f.wh, r2)) continue;
            const float w = recon_weight(f, pcx, pcy, c.x, c.y) * multiplier;
            const float4 v = sv[li];
            wsum += w;
            ax += w * v.x;
            ay += w * v.y;
            az += w * v.z;
        }
    const size_t p = size_t(py) * width + size_t(px);
    float4 acc = image[p];
    image[p] = make_float4(acc.x + ax, acc.y + ay, acc.z + az, acc.w + wsum);
}

// KCCheckPixels (ImageMemory.cu:34-60)
__global__ void __launch_bounds__(256) k_check_pixels(float* __restrict__ pixels, uint32_t channels,
                                                      size_t count) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count;
         i += size_t(gridDim.x) * blockDim.x) {
        if (channels == 4) {
            float4* p4 = reinterpret_cast<float4*>(pixels) + i;
            const float4 v = *p4;
            if (isnan(v.x) || isnan(v.y) || isnan(v.z) || isnan(v.w))
                *p4 = make_float4(1.0e30f, 0.0f, 1.0e30f, 1.0f);
        } else if (isnan(pixels[i])) {
            pixels[i] = 1.0e30f;
        }
    }
}

inline uint32_t grid_of(size_t n, uint32_t cap) {
    size_t g = (n + 255) / 256;
    if (g == 0) g = 1;
    return static_cast<uint32_t>(g < cap ? g : cap);
}

inline int key_bits(uint32_t pixels) {
    int b = 1;
    while (b < 32 && (uint64_t(1) << b) < pixels) b++;
    return b;
}

}  // namespace

int recon_filter_make(const char* type, float radius, uint32_t optCount, const char* const* names,
                      const float* values, ReconFilterDev* out) {
    if (!type || !out || (optCount && (!names || !values))) {
        set_error("recon filter: null argument");
        return MRB_E_ARG;
    }
    // the window grows with the radius (wh^2 pairs per sample); 64 pixels
    // is far beyond any filter the tracer configurations use
    if (!(radius >= 0.0f) || !(radius <= 64.0f)) {
        set_error("recon filter: radius %g outside [0, 64]", double(radius));
        return MRB_E_ARG;
    }
    auto option = [&](const char* key, float* v) {
        for (uint32_t i = 0; i < optCount; i++)
            if (names[i] && std::strcmp(names[i], key) == 0) {
                *v = values[i];
                return true;
            }
        return false;
    };
    ReconFilterDev f{};
    f.radius = radius;
    f.wh = filter_pixel_wh(radius);
    if (std::strcmp(type, "Box") == 0) {
        f.type = kReconBox;
    } else {
        if (radius == 0.0f) {
            set_error("recon filter: radius 0 is only defined for the Box filter");
            return MRB_E_ARG;
        }
        if (std::strcmp(type, "Tent") == 0) {
            f.type = kReconTent;
            f.recipRadius = 1.0f / radius;
        } else if (std::strcmp(type, "Gaussian") == 0) {
            float alpha;
            if (!option("alpha", &alpha)) {
                set_error("Gauss Filter parameter \"alpha\" not found");
                return MRB_E_ARG;
            }
            f.type = kReconGaussian;
            f.negAlpha = -alpha;
            f.gaussEdge = recon_gauss(f, radius);
        } else if (std::strcmp(type, "Mitchell") == 0) {
            float b, c;
            if (!option("b", &b)) {
                set_error("Mitchell Filter parameter \"b\" not found");
                return MRB_E_ARG;
            }
            if (!option("c", &c)) {
                set_error("Mitchell Filter parameter \"c\" not found");
                return MRB_E_ARG;
            }
            // GPUMitchellFilterFunctor (GPUReconFilterMitchell.h:78-95)
            const float t = 1.0f / 6.0f;
            f.type = kReconMitchell;
            f.recipRadius = 1.0f / radius;
            f.c01[0] = t * (12 - 9 * b - 6 * c);
            f.c01[1] = t * (-18 + 12 * b + 6 * c);
            f.c01[2] = 0.0f;
            f.c01[3] = t * (6 + 2 * b + 0 * c);
            f.c12[0] = t * (-1 * b - 6 * c);
            f.c12[1] = t * (6 * b + 30 * c);
            f.c12[2] = t * (-12 * b - 48 * c);
            f.c12[3] = t * (8 * b + 24 * c);
        } else {
            set_error("recon filter: unknown type \"%s\" (Box, Tent, Gaussian, Mitchell)", type);
            return MRB_E_ARG;
        }
    }
    *out = f;
    return 0;
}

static size_t pair_capacity(const ReconFilterDev& f, uint32_t n) {
    return size_t(n) * f.wh * f.wh;
}

size_t recon_scratch_bytes(const ReconFilterDev& f, uint32_t n, const ImageSeg& seg) {
    const size_t pairs = pair_capacity(f, n);
    const size_t pix = size_t(seg.w) * size_t(seg.h);
    const int bits = key_bits(static_cast<uint32_t>(pix));
    size_t b = 0;
    b += align256((size_t(n) + 1) * 4) * 2;
    b += align256(exclusive_scan_temp_bytes(n));
    b += align256(pairs * 4) * 2;
    b += align256(radix_sort_temp_bytes(static_cast<uint32_t>(pairs), 4, 0, bits));
    b += align256(pix * 4) * 2;
    return b;
}

ReconScratch recon_scratch_carve(void* base, const ReconFilterDev& f, uint32_t n,
                                 const ImageSeg& seg) {
    const size_t pairs = pair_capacity(f, n);
    const size_t pix = size_t(seg.w) * size_t(seg.h);
    const int bits = key_bits(static_cast<uint32_t>(pix));
    unsigned char* p = static_cast<unsigned char*>(base);
    ReconScratch s{};
    s.count = reinterpret_cast<uint32_t*>(p);
    p += align256((size_t(n) + 1) * 4);
    s.offset = reinterpret_cast<uint32_t*>(p);
    p += align256((size_t(n) + 1) * 4);
    s.scanTemp = p;
    p += align256(exclusive_scan_temp_bytes(n));
    s.keys = reinterpret_cast<uint32_t*>(p);
    p += align256(pairs * 4);
    s.vals = reinterpret_cast<uint32_t*>(p);
    p += align256(pairs * 4);
    s.sortTemp = p;
    s.sortTempBytes = radix_sort_temp_bytes(static_cast<uint32_t>(pairs), 4, 0, bits);
    p += align256(s.sortTempBytes);
    s.begin = reinterpret_cast<uint32_t*>(p);
    p += align256(pix * 4);
    s.end = reinterpret_cast<uint32_t*>(p);
    return s;
}

int recon_filter_to_img(const ReconFilterDev& f, const ImageSeg& seg, const float* values,
                        uint32_t channels, const float2* coords, uint32_t n, float multiplier,
                        float* pixels, float* counts, const ReconScratch& s, cudaStream_t stream) {
    if (n == 0 || seg.w <= 0 || seg.h <= 0) return 0;
    const size_t pairs = pair_capacity(f, n);
    const size_t pix = size_t(seg.w) * size_t(seg.h);
    const int bits = key_bits(static_cast<uint32_t>(pix));
    const uint32_t g = grid_of(n, 148 * 8);
    k_expand_count<<<g, 256, 0, stream>>>(coords, n, f, seg, s.count);
    if (exclusive_scan_u32(s.count, s.offset, n, s.scanTemp, stream)) return MRB_E_CUDA;
    k_expand_write<<<g, 256, 0, stream>>>(coords, n, f, seg, s.offset, s.keys, s.vals);
    const uint32_t* dTotal = s.offset + n;
    if (radix_sort_pairs<uint32_t>(s.keys, s.vals, dTotal, static_cast<uint32_t>(pairs), 0, bits,
                                   false, s.sortTemp, s.sortTempBytes, stream, false))
        return MRB_E_CUDA;
    MRB_CUDA(cudaMemsetAsync(s.begin, 0, pix * 4, stream));
    MRB_CUDA(cudaMemsetAsync(s.end, 0, pix * 4, stream));
    k_pixel_bounds<<<grid_of(pairs, 148 * 8), 256, 0, stream>>>(s.keys, dTotal, s.begin, s.end);
    const uint32_t gp = grid_of(pix, 148 * 16);
    if (channels == 4)
        k_filter_pixels<4><<<gp, 256, 0, stream>>>(s.begin, s.end, s.vals, values, coords, f, seg,
                                                   multiplier, pixels, counts);
    else
        k_filter_pixels<1><<<gp, 256, 0, stream>>>(s.begin, s.end, s.vals, values, coords, f, seg,
                                                   multiplier, pixels, counts);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int recon_filter_grid(const ReconFilterDev& f, const float4* samples, const float2* coords,
                      uint32_t width, uint32_t height, uint32_t sp, float multiplier,
                      float4* image, cudaStream_t stream) {
    const size_t pix = size_t(width) * height;
    // the tiled form where its staged rectangle fits the default 48 KB of
    // shared memory (1 and 2 samples per pixel axis with small filters)
    const int32_t range = static_cast<int32_t>(f.wh);
    const int32_t hi = (range + 2) / 2;
    const int32_t loMin = -(range - 1) / 2 - ((range % 2 == 0) ? 1 : 0);
    const size_t span = size_t(kFilterTile + hi - loMin + 1) * sp;
    const size_t smemBytes = span * span * (sizeof(float4) + sizeof(float2));
    if (smemBytes <= 48 * 1024) {
        const size_t tiles = size_t((width + kFilterTile - 1) / kFilterTile) *
                             ((height + kFilterTile - 1) / kFilterTile);
        k_filter_grid_tiled<<<static_cast<uint32_t>(tiles), 256, smemBytes, stream>>>(
            samples, coords, width, height, sp, f, multiplier, image);
    } else {
        k_filter_grid<<<grid_of(pix, 148 * 16), 256, 0, stream>>>(samples, coords, width, height,
                                                                 sp, f, multiplier, image);
    }
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int image_check_pixels(float* pixels, uint32_t channels, size_t count, cudaStream_t stream) {
    if (count == 0) return 0;
    k_check_pixels<<<grid_of(count, 148 * 8), 256, 0, stream>>>(pixels, channels, count);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb

// ---------------------------------------------------------------------------
// C ABI: GPUReconFilterI (GPUReconFilterI.h:6-33) and ImageMemory
// (ImageMemory.h:14-78)
// ---------------------------------------------------------------------------
struct mrb_recon_filter {
    mrb::ReconFilterDev f{};
    char type[16] = {};
    void* scratch = nullptr;
    size_t scratchBytes = 0;
    ~mrb_recon_filter() {
        if (scratch) cudaFree(scratch);
    }
};

struct mrb_image {
    int32_t resW = 0, resH = 0, offX = 0, offY = 0, w = 0, h = 0;
    uint32_t channels = 4;
    float* pixels = nullptr;
    float* counts = nullptr;
    void* mem = nullptr;
    ~mrb_image() {
        if (mem) cudaFree(mem);
    }
    size_t pixel_count() const { return size_t(w) * size_t(h); }
    mrb::ImageSeg seg() const { return mrb::ImageSeg{offX, offY, w, h, resW, resH}; }
};

namespace mrb {
const ReconFilterDev* recon_filter_dev(const mrb_recon_filter* f) { return f ? &f->f : nullptr; }
}  // namespace mrb

namespace {
int image_alloc(mrb_image* im) {
    if (im->mem) cudaFree(im->mem);
    im->mem = nullptr;
    im->pixels = im->counts = nullptr;
    const size_t pix = im->pixel_count();
    if (pix == 0) return 0;
    const size_t pbytes = (pix * im->channels * 4 + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&im->mem, pbytes + pix * 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        im->mem = nullptr;
        mrb::set_error("image: cudaMalloc of %zu bytes failed: %s", pbytes + pix * 4,
                       cudaGetErrorString(e));
        return MRB_E_OOM;
    }
    im->pixels = static_cast<float*>(im->mem);
    im->counts = reinterpret_cast<float*>(static_cast<unsigned char*>(im->mem) + pbytes);
    MRB_CUDA(cudaMemset(im->mem, 0, pbytes + pix * 4));
    return 0;
}
}  // namespace

extern "C" {

int mrb_recon_filter_create(const char* type, float radius, uint32_t option_count,
                            const char* const* option_names, const float* option_values,
                            mrb_recon_filter** out) {
    if (!out) {
        mrb::set_error("recon filter: null output");
        return MRB_E_ARG;
    }
    *out = nullptr;
    mrb::ReconFilterDev f;
    int r = mrb::recon_filter_make(type, radius, option_count, option_names, option_values, &f);
    if (r) return r;
    mrb_recon_filter* h = new mrb_recon_filter();
    h->f = f;
    std::strncpy(h->type, type, sizeof(h->type) - 1);
    *out = h;
    return 0;
}

void mrb_recon_filter_destroy(mrb_recon_filter* f) { delete f; }

const char* mrb_recon_filter_type(const mrb_recon_filter* f) { return f ? f->type : nullptr; }

size_t mrb_recon_filter_used_bytes(const mrb_recon_filter* f) { return f ? f->scratchBytes : 0; }

uint32_t mrb_recon_filter_pixel_wh(float radius) { return mrb::filter_pixel_wh(radius); }

float mrb_recon_filter_weight(const mrb_recon_filter* f, float pixel_x, float pixel_y,
                              float sample_x, float sample_y) {
    if (!f) return 0.0f;
    return mrb::recon_weight(f->f, pixel_x, pixel_y, sample_x, sample_y);
}

int mrb_recon_filter_to_img(mrb_recon_filter* f, mrb_image* img, const float* d_values,
                            uint32_t channels, const float* d_img_coords, uint32_t sample_count,
                            float scalar_multiplier, void* stream) {
    if (!f || !img || (sample_count && (!d_values || !d_img_coords))) {
        mrb::set_error("recon filter: null argument");
        return MRB_E_ARG;
    }
    if (channels != img->channels) {
        mrb::set_error("recon filter: %u-channel values into a %u-channel image", channels,
                       img->channels);
        return MRB_E_ARG;
    }
    if ((channels == 4 && (reinterpret_cast<uintptr_t>(d_values) & 15)) ||
        (reinterpret_cast<uintptr_t>(d_img_coords) & 7)) {
        mrb::set_error("recon filter: values need 16-byte (RGBA) and coordinates 8-byte alignment");
        return MRB_E_ARG;
    }
    if (sample_count == 0 || img->pixel_count() == 0) return 0;
    if (size_t(sample_count) * f->f.wh * f->f.wh >= (size_t(1) << 32)) {
        mrb::set_error("recon filter: %u samples x %u pixels each exceed 2^32 pairs", sample_count,
                       f->f.wh * f->f.wh);
        return MRB_E_ARG;
    }
    const mrb::ImageSeg seg = img->seg();
    const size_t need = mrb::recon_scratch_bytes(f->f, sample_count, seg);
    if (need > f->scratchBytes) {
        if (f->scratch) {
            cudaFree(f->scratch);
            f->scratch = nullptr;
            f->scratchBytes = 0;
        }
        cudaError_t e = cudaMalloc(&f->scratch, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            f->scratch = nullptr;
            mrb::set_error("recon filter: cudaMalloc of %zu bytes failed: %s", need,
                           cudaGetErrorString(e));
            return MRB_E_OOM;
        }
        f->scratchBytes = need;
    }
    const mrb::ReconScratch s = mrb::recon_scratch_carve(f->scratch, f->f, sample_count, seg);
    return mrb::recon_filter_to_img(f->f, seg, d_values, channels,
                                    reinterpret_cast<const float2*>(d_img_coords), sample_count,
                                    scalar_multiplier, img->pixels, img->counts, s,
                                    static_cast<cudaStream_t>(stream));
}

int mrb_image_create(int32_t width, int32_t height, uint32_t channels, mrb_image** out) {
    if (!out || width <= 0 || height <= 0 || (channels != 1 && channels != 4) ||
        int64_t(width) * height > (int64_t(1) << 31)) {
        mrb::set_error("image: bad size %dx%d or channel count %u (1 or 4)", width, height,
                       channels);
        return MRB_E_ARG;
    }
    mrb_image* im = new mrb_image();
    im->resW = im->w = width;
    im->resH = im->h = height;
    im->channels = channels;
    int r = image_alloc(im);
    if (r) {
        delete im;
        return r;
    }
    *out = im;
    return 0;
}

void mrb_image_destroy(mrb_image* img) { delete img; }

int mrb_image_reportion(mrb_image* img, int32_t start_x, int32_t start_y, int32_t end_x,
                        int32_t end_y) {
    if (!img) return MRB_E_ARG;
    // ImageMemory::Reportion (ImageMemory.cu:111-137): end clamped to the resolution
    end_x = end_x < img->resW ? end_x : img->resW;
    end_y = end_y < img->resH ? end_y : img->resH;
    if (start_x < 0 || start_y < 0 || end_x < start_x || end_y < start_y) {
        mrb::set_error("image: portion [%d,%d)-[%d,%d) outside the image", start_x, start_y,
                       end_x, end_y);
        return MRB_E_ARG;
    }
    img->offX = start_x;
    img->offY = start_y;
    img->w = end_x - start_x;
    img->h = end_y - start_y;
    return image_alloc(img);
}

int mrb_image_resize(mrb_image* img, int32_t width, int32_t height) {
    if (!img) return MRB_E_ARG;
    // ImageMemory::Resize: the segment must still fit
    if (width <= 0 || height <= 0 || img->offX + img->w > width || img->offY + img->h > height) {
        mrb::set_error("image: resolution %dx%d does not hold the current portion", width, height);
        return MRB_E_ARG;
    }
    img->resW = width;
    img->resH = height;
    return 0;
}

int mrb_image_reset(mrb_image* img, void* stream) {
    if (!img) return MRB_E_ARG;
    if (!img->mem) return 0;
    const size_t pix = img->pixel_count();
    const size_t pbytes = (pix * img->channels * 4 + 255) & ~size_t(255);
    MRB_CUDA(cudaMemsetAsync(img->mem, 0, pbytes + pix * 4, static_cast<cudaStream_t>(stream)));
    return 0;
}

int mrb_image_info(const mrb_image* img, int32_t* info7) {
    if (!img || !info7) return MRB_E_ARG;
    const int32_t v[7] = {img->offX, img->offY, img->w, img->h, img->resW, img->resH,
                          static_cast<int32_t>(img->channels)};
    std::memcpy(info7, v, sizeof(v));
    return 0;
}

int mrb_image_device(const mrb_image* img, float** d_pixels, float** d_sample_counts) {
    if (!img) return MRB_E_ARG;
    if (d_pixels) *d_pixels = img->pixels;
    if (d_sample_counts) *d_sample_counts = img->counts;
    return 0;
}

int mrb_image_get(mrb_image* img, float* host_pixels, float* host_counts, void* stream) {
    if (!img || !host_pixels || !host_counts) return MRB_E_ARG;
    const size_t pix = img->pixel_count();
    if (pix == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // ImageMemory::GetImageToCPU (ImageMemory.cu:150-190): NaN check, copy, reset
    if (mrb::image_check_pixels(img->pixels, img->channels, pix, st)) return MRB_E_CUDA;
    MRB_CUDA(cudaMemcpyAsync(host_pixels, img->pixels, pix * img->channels * 4,
                             cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaMemcpyAsync(host_counts, img->counts, pix * 4, cudaMemcpyDeviceToHost, st));
    if (mrb_image_reset(img, stream)) return MRB_E_CUDA;
    MRB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

}  // extern "C"

#include "io.cuh"

extern "C" int mrb_image_write(mrb_image* img, const char* path) {
    if (!img || !path) return MRB_E_ARG;
    const size_t pix = img->pixel_count();
    if (pix == 0) return MRB_E_ARG;
    std::vector<float> px(pix * img->channels), cnt(pix);
    MRB_CUDA(cudaMemcpy(px.data(), img->pixels, px.size() * 4, cudaMemcpyDeviceToHost));
    MRB_CUDA(cudaMemcpy(cnt.data(), img->counts, cnt.size() * 4, cudaMemcpyDeviceToHost));
    return mrb::write_averaged(path, px.data(), cnt.data(), 1, static_cast<uint32_t>(img->w),
                               static_cast<uint32_t>(img->h), img->channels, img->channels);
}
