// CPU oracle of the reconstruction filters -- TEST INFRASTRUCTURE ONLY.
//
// Restates MRay's filter functors (GPUReconFilterBox.h:47-60,
// GPUReconFilterTent.h:51-66, GPUReconFilterGaussian.h:68-95,
// GPUReconFilterMitchell.h:78-121), FilterRadiusToPixelWH
// (GPUReconFilterKC.cuh:10-31), KCExpandSamplesToPixels
// (GPUReconFilterKC.cuh:33-141) and the sort-then-reduce of
// GPUReconFilter::FilterToImgInternal (GPUReconFilter.h:59-260), summing
// each pixel's samples in ascending sample order, plus the reference test's
// own CPU expectation (Test_TracerCUDA/T_ReconFilter.cu:96-140) and its
// input generator (std::mt19937 + std::uniform_real_distribution<float>,
// T_ReconFilter.cu:38-62).  Compiled with -ffp-contract=off so every
// product and sum rounds as written.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

// exp by Cody-Waite reduction with a 16-bit head of ln 2 and the Taylor
// series of e^r through r^8 / 8!, scaled by 2^k in two exact steps.  The
// device library computes exp with these same steps, so Gaussian weights
// agree bit for bit.
float bits_float(int b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
float rexp(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return bits_float(0x7F800000);
    if (x < -103.97208f) return 0.0f;
    const float kf = std::rint(x * 0x1.715476p+0f);
    const int k = static_cast<int>(kf);
    float r = x - kf * 0x1.62e4p-1f;
    r = r - kf * 0x1.7f7d1cp-20f;
    float p = 0x1.a01a02p-16f;
    p = p * r + 0x1.a01a02p-13f;
    p = p * r + 0x1.6c16c2p-10f;
    p = p * r + 0x1.111112p-7f;
    p = p * r + 0x1.555556p-5f;
    p = p * r + 0x1.555556p-3f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    const int k1 = k / 2, k2 = k - k1;
    p = p * bits_float((k1 + 127) << 23);
    return p * bits_float((k2 + 127) << 23);
}

struct Functor {
    int type = 0;
    float radius = 0.0f;
    float recip = 0.0f;
    float negAlpha = 0.0f, edge = 0.0f;
    float c01[4] = {}, c12[4] = {};

    float gauss(float x) const { return rexp(negAlpha * x * x); }
    float mitchell(float x) const {
        x = std::fabs(x);
        float x2 = x * x;
        float x3 = x2 * x;
        const float* c = nullptr;
        static const float zero[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (x < 1.0f) c = c01;
        else if (x < 2.0f) c = c12;
        else c = zero;
        return c[0] * x3 + c[1] * x2 + c[2] * x + c[3];
    }
    float operator()(float px, float py, float sx, float sy) const {
        const float dx = std::fabs(px - sx), dy = std::fabs(py - sy);
        if (type == 0) {  // Box
            if (radius == 0.0f) return 1.0f;
            return (dx < radius && dy < radius) ? 1.0f : 0.0f;
        }
        if (type == 1) {  // Tent
            float lx = std::max(0.0f, radius - dx), ly = std::max(0.0f, radius - dy);
            lx *= recip;
            ly *= recip;
            return lx * ly;
        }
        if (type == 2) {  // Gaussian
            return std::max(0.0f, gauss(dx) - edge) * std::max(0.0f, gauss(dy) - edge);
        }
        return mitchell(2.0f * dx * recip) * mitchell(2.0f * dy * recip);
    }
};

Functor make_functor(const oracle_filter* f) {
    Functor F;
    F.type = static_cast<int>(f->type);
    F.radius = f->radius;
    if (F.type == 1) F.recip = 1.0f / f->radius;
    if (F.type == 2) {
        F.negAlpha = -f->alpha;
        F.edge = F.gauss(f->radius);
    }
    if (F.type == 3) {
        const float b = f->b, c = f->c;
        const float t = 1.0f / 6.0f;
        F.recip = 1.0f / f->radius;
        F.c01[0] = t * (12 - 9 * b - 6 * c);
        F.c01[1] = t * (-18 + 12 * b + 6 * c);
        F.c01[2] = 0.0f;
        F.c01[3] = t * (6 + 2 * b + 0 * c);
        F.c12[0] = t * (-1 * b - 6 * c);
        F.c12[1] = t * (6 * b + 30 * c);
        F.c12[2] = t * (-12 * b - 48 * c);
        F.c12[3] = t * (8 * b + 24 * c);
    }
    return F;
}

uint32_t pixel_wh(float radius) {
    uint32_t result = 1;
    if (radius == 0.0f) return result;
    uint32_t quot = static_cast<uint32_t>(radius / 0.5f);
    float remainder = std::fmod(radius, 0.5f);
    if (remainder == 0.0f) quot -= 1;
    result += (quot + 1);
    return result;
}

}  // namespace

extern "C" {

uint32_t oracle_filter_pixel_wh(float radius) { return pixel_wh(radius); }

// The portable exp the Gaussian functor uses, for its accuracy check.
void oracle_exp(const float* x, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; i++) out[i] = rexp(x[i]);
}

float oracle_filter_weight(const oracle_filter* f, float px, float py, float sx, float sy) {
    return make_functor(f)(px, py, sx, sy);
}

// GPUReconFilter::FilterToImgInternal (GPUReconFilter.h:59-260) with
// KCExpandSamplesToPixels (GPUReconFilterKC.cuh:33-141): every sample is
// expanded to the pixels of its window whose centre lies within the radius
// (radius 0: its own pixel), the (pixel, sample) pairs are stably sorted by
// pixel, and each pixel sums weight * value and weight over its run in
// ascending sample order before adding them to the image.  Pixels outside
// the image portion [off, off + size) are dropped, and so are samples with
// a NaN coordinate or one beyond +-1e9.
void oracle_filter_to_img(const oracle_filter* f, const float* values, uint32_t channels,
                          const float* coords, uint32_t n, int32_t resW, int32_t resH,
                          int32_t offX, int32_t offY, int32_t segW, int32_t segH,
                          float multiplier, float* pixels, float* counts) {
    const Functor F = make_functor(f);
    const int32_t rangeInt = static_cast<int32_t>(pixel_wh(f->radius));
    const int32_t lo = -(rangeInt - 1) / 2, hi = (rangeInt + 2) / 2;
    const float r2 = f->radius * f->radius;
    std::vector<std::pair<uint32_t, uint32_t>> pairs;  // (pixel id, sample)
    for (uint32_t i = 0; i < n; i++) {
        const float cx = coords[2 * i], cy = coords[2 * i + 1];
        if (!(std::fabs(cx) < 1.0e9f && std::fabs(cy) < 1.0e9f)) continue;
        float ipx, ipy;
        const float relX = std::modf(cx, &ipx), relY = std::modf(cy, &ipy);
        const int32_t ix = static_cast<int32_t>(ipx), iy = static_cast<int32_t>(ipy);
        int32_t x0 = lo, x1 = hi, y0 = lo, y1 = hi;
        if (rangeInt % 2 == 0) {
            if (relX < 0.5f) { x0 -= 1; x1 -= 1; }
            if (relY < 0.5f) { y0 -= 1; y1 -= 1; }
        }
        for (int32_t y = y0; y < y1; y++)
            for (int32_t x = x0; x < x1; x++) {
                const float pcx = (ipx + static_cast<float>(x)) + 0.5f;
                const float pcy = (ipy + static_cast<float>(y)) + 0.5f;
                const float dx = cx - pcx, dy = cy - pcy;
                if (!(rangeInt == 1 || (dx * dx + dy * dy) <= r2)) continue;
                const int32_t px = ix + x, py = iy + y;
                if (px < 0 || px >= resW || py < 0 || py >= resH) continue;
                if (px < offX || px >= offX + segW || py < offY || py >= offY + segH) continue;
                pairs.emplace_back(static_cast<uint32_t>(py * resW + px), i);
            }
    }
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const std::pair<uint32_t, uint32_t>& a,
                        const std::pair<uint32_t, uint32_t>& b) { return a.first < b.first; });
    size_t k = 0;
    while (k < pairs.size()) {
        const uint32_t pix = pairs[k].first;
        const int32_t gx = static_cast<int32_t>(pix % static_cast<uint32_t>(resW));
        const int32_t gy = static_cast<int32_t>(pix / static_cast<uint32_t>(resW));
        const float pcx = static_cast<float>(gx) + 0.5f, pcy = static_cast<float>(gy) + 0.5f;
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float wsum = 0.0f;
        for (; k < pairs.size() && pairs[k].first == pix; k++) {
            const uint32_t s = pairs[k].second;
            const float w = F(pcx, pcy, coords[2 * s], coords[2 * s + 1]) * multiplier;
            wsum += w;
            for (uint32_t c = 0; c < channels; c++) acc[c] += w * values[size_t(s) * channels + c];
        }
        const size_t q = size_t(gy - offY) * size_t(segW) + size_t(gx - offX);
        for (uint32_t c = 0; c < channels; c++) pixels[q * channels + c] += acc[c];
        counts[q] += wsum;
    }
}

// The reference test's CPU expectation (T_ReconFilter.cu:96-140): every
// sample in order, a [-wh, wh] window, pixels whose centre lies within the
// radius get weight * value and weight added directly.
void oracle_filter_direct(const oracle_filter* f, const float* values, const float* coords,
                          uint32_t n, int32_t resW, int32_t resH, float* pixels, float* counts) {
    const Functor F = make_functor(f);
    const int32_t wh = static_cast<int32_t>(pixel_wh(f->radius));
    const float R = f->radius;
    for (uint32_t i = 0; i < n; i++) {
        const float cx = coords[2 * i], cy = coords[2 * i + 1];
        float spx, spy;
        std::modf(cx, &spx);
        std::modf(cy, &spy);
        const int32_t ix = static_cast<int32_t>(spx), iy = static_cast<int32_t>(spy);
        for (int32_t y = -wh; y <= wh; y++)
            for (int32_t x = -wh; x <= wh; x++) {
                const float pcx = (spx + static_cast<float>(x)) + 0.5f;
                const float pcy = (spy + static_cast<float>(y)) + 0.5f;
                const float dx = cx - pcx, dy = cy - pcy;
                if (!((dx * dx + dy * dy) <= R * R)) continue;
                const int32_t px = ix + x, py = iy + y;
                if (px < 0 || px >= resW || py < 0 || py >= resH) continue;
                const size_t q = size_t(py) * size_t(resW) + size_t(px);
                const float w = F(pcx, pcy, cx, cy);
                for (int c = 0; c < 4; c++) pixels[q * 4 + c] += w * values[size_t(i) * 4 + c];
                counts[q] += w;
            }
    }
}

// The reference test's inputs (T_ReconFilter.cu:38-62): std::mt19937 seeded
// with `seed`, x then y per sample from uniform_real_distribution<float>
// over [0, width) and [0, height).
void oracle_mt19937_coords(uint32_t n, int32_t width, int32_t height, uint32_t seed,
                           float* out) {
    std::mt19937 rng;
    rng.seed(seed);
    std::uniform_real_distribution<float> dx(0.0f, static_cast<float>(width));
    std::uniform_real_distribution<float> dy(0.0f, static_cast<float>(height));
    for (uint32_t i = 0; i < n; i++) {
        out[2 * i] = dx(rng);
        out[2 * i + 1] = dy(rng);
    }
}

}  // extern "C"
