// Wavefront path guiding (WFPG) over the sparse voxel octree radiance
// cache, the hot path of yalcinerbora/meturay's WFPGTracer:
//
//   k_bin_init        KCInitializeSVOBins (WFPGTracerKC.cuh:965-1020): each
//                     surface hit finds its leaf (8-neighbour search) and
//                     counts itself into the leaf's bin word
//   k_collapse_*      KCCollapseRayCounts(Leaf) (AnisoSVO.cu:265-350): bins
//                     with fewer than BinRayCount rays hand their count to
//                     the parent, down to MinRayBinLevel
//   k_bin_resolve     KCCheckReducedSVOBins / FindMarkedBin
//   radix sort, k_bin_heads/k_bin_ranges
//                     PartitionRaysWRTCustomData: rays grouped by bin
//   k_guide<X, kProduct>  KCGenAndSampleDistributionProduct (kProduct) or
//                     KCGenAndSampleDistribution (2D PWC over the field)
//                     (WFPGTracerKC.cuh:1560-1766), one block per bin:
//                     representative surface -> X*X cone traces through
//                     the octree -> radiance read -> 11-tap Gaussian filter
//                     (BlockTextureFilter.cuh) -> 8x8 outer field ->
//                     per ray (one warp each) BxDF x field product, CDF
//                     scans, row/column search, rejection sampling of the
//                     inner cell, one-sample MIS with the BxDF
//                     (ProductSampler.cuh:16-725)
//   k_path_deposit    KCAccumulateRadianceToLeaf (AnisoSVO.cu:224-263)
//   k_leaf_normalize, k_bottom_up, k_top_down
//                     NormalizeAndFilterRadiance (AnisoSVO.cu:352-428,
//                     1415-1484)
//   k_average_normals KCAverageNormals (AnisoSVO.cu:428-528)
//
// Determinism: bin ray counts are integer atomics; radiance sums are 2^24
// fixed-point integer atomics; every random number comes from Philox keyed
// by (path, frame, depth, purpose); the bin's representative ray is the
// one with the smallest hash of its path index (the reference picks a
// uniformly random ray of the bin, here independent of the ray order in
// the wavefront).  So the octree state and every guided direction are
// reproducible bit for bit; only the image sums use float atomics.
#include "../../include/mrb200.h"
#include "bxdf.cuh"
#include "guide.cuh"
#include "scan.cuh"
#include "sort.cuh"

namespace mrb {
namespace {

constexpr uint32_t kGuideValid = 1u << 17;
constexpr uint32_t kGuideBxdf = 1u << 16;
constexpr uint32_t kTagGuide = 0x20000u;     // per-ray guide draws
constexpr uint32_t kTagGuideBin = 0x30000u;  // per-bin jitter
constexpr float kInv4Pi = 0.25f * kInvPiF;
constexpr float kLargeEpsilon = 1.0e-4f;
constexpr float kVeryLargeEpsilon = 1.0e-3f;

__device__ __forceinline__ float lum3(V3 c) { return 0.2120f * c.x + 0.7150f * c.y + 0.0722f * c.z; }

inline uint32_t grid_for(uint32_t n, uint32_t block, uint32_t cap) {
    uint32_t g = (n + block - 1) / block;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

__device__ __forceinline__ unsigned long long to_fixed(float x) {
    return (x > 0.0f) ? __double2ull_rn(static_cast<double>(x) * kFixScale) : 0ull;
}

// ---------------------------------------------------------------------------
// binning
// ---------------------------------------------------------------------------
struct BinArgs {
    GuideDev g;
    GuideWave w;
    uint32_t* binKey;
    uint2* guide;
};

__global__ void __launch_bounds__(256) k_bin_init(BinArgs A) {
    const uint32_t n = *A.w.count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.w.maxRays;
         i += gridDim.x * blockDim.x) {
        if (i >= n) {
            A.binKey[i] = kBinInvalid;
            continue;
        }
        A.guide[i] = make_uint2(0u, 0x7E00u);
        const uint32_t key = A.w.hit.key[i];
        const uint8_t type = A.w.aux[i].type;
        if (type == kNeeRay || (key >> kIdBits) == kBatchNull) {
            A.binKey[i] = kBinInvalid;
            continue;
        }
        const float4 o = A.w.rayO[i], d = A.w.rayD[i];
        const float t = A.w.hit.t[i];
        const V3 p = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        uint32_t leaf;
        if (svo_nearest(A.g, leaf, p, A.g.leafDepth)) {
            A.binKey[i] = leaf | kBinLeaf;
            atomicAdd(A.g.leafBin + leaf, 1u);
        } else {
            A.binKey[i] = kBinInvalid;
        }
    }
}

__global__ void __launch_bounds__(256) k_collapse_leaf(GuideDev g, uint32_t minLevel,
                                                       uint32_t minRayCount) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < g.leafCount;
         l += gridDim.x * blockDim.x) {
        if (g.leafDepth == minLevel) {
            g.leafBin[l] |= kBinMark;
            continue;
        }
        const uint32_t c = g.leafBin[l] & ~kBinMark;
        if (c == 0) continue;
        if (c < minRayCount) atomicAdd(g.nodeBin + g.leafParents[l], c);
        else g.leafBin[l] |= kBinMark;
    }
}

__global__ void __launch_bounds__(256) k_collapse_nodes(GuideDev g, uint32_t begin, uint32_t end,
                                                        uint32_t level, uint32_t minLevel,
                                                        uint32_t minRayCount) {
    for (uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += gridDim.x * blockDim.x) {
        if (level == minLevel) {
            g.nodeBin[k] |= kBinMark;
            continue;
        }
        const uint32_t c = g.nodeBin[k] & ~kBinMark;
        if (c < minRayCount) atomicAdd(g.nodeBin + svo_parent(g.nodes[k]), c);
        else g.nodeBin[k] |= kBinMark;
    }
}

__global__ void __launch_bounds__(256) k_bin_resolve(GuideDev g, const uint32_t* __restrict__ count,
                                                     uint32_t* binKey) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = binKey[i];
        if (k == kBinInvalid) continue;
        bool isLeaf;
        const uint32_t node = svo_marked_bin(g, k & ~kBinLeaf, isLeaf);
        if (!isLeaf) binKey[i] = node;
    }
}

// bin segments of the sorted keys: heads -> exclusive scan -> ranges
__global__ void __launch_bounds__(256) k_bin_heads(const uint32_t* __restrict__ key,
                                                   const uint32_t* __restrict__ count,
                                                   uint32_t maxRays, uint32_t* heads) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < maxRays;
         i += gridDim.x * blockDim.x) {
        const uint32_t k = (i < n) ? key[i] : kBinInvalid;
        heads[i] = (k != kBinInvalid && (i == 0 || key[i - 1] != k)) ? 1u : 0u;
    }
}
__global__ void __launch_bounds__(256) k_bin_ranges(const uint32_t* __restrict__ key,
                                                    const uint32_t* __restrict__ count,
                                                    const uint32_t* __restrict__ heads,
                                                    const uint32_t* __restrict__ scan,
                                                    uint32_t* binBegin, uint32_t* binEnd) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = key[i];
        if (k == kBinInvalid) continue;
        if (heads[i]) binBegin[scan[i]] = i;
        if (i + 1 == n || key[i + 1] != k) binEnd[scan[i + 1] - 1u] = i + 1;
    }
}

// ---------------------------------------------------------------------------
// per-bin radiance field and product sampling
// ---------------------------------------------------------------------------
struct GuideArgs {
    SceneDev sc;
    GuideDev g;
    GuideWave w;
    const uint32_t* binKey;   // sorted
    const uint32_t* binRid;   // ray index per sorted slot
    const uint32_t* binBegin;
    const uint32_t* binEnd;
    const uint32_t* binCount; // headScan[maxRays]
    uint32_t* binNext;        // bins are taken in turn from this counter (zeroed)
    uint2* guide;
    GuideOptions go;
    PathOptions opt;
    uint32_t depthTag;
};

constexpr int kGuideTPB = 256;
constexpr int kGuideWarps = kGuideTPB / 32;

template <int X>
struct GuideSmem {
    float field[X * X];
    float tmp[X * X];
    float small[64];
    float norm[64];
    float pdfX[kGuideWarps][64];
    float cdfX[kGuideWarps][64];
    float pdfY[kGuideWarps][8];
    float cdfY[kGuideWarps][8];
    float rowTot[kGuideWarps][8];
    unsigned long long repKey[kGuideWarps];
    uint32_t repRid[kGuideWarps];
    float origin[4];
    float jitter[2];
    float marg[X];      // non-product sampler: row marginal prefix sums
    float span[12];     // cone loop constants per level (ConeTables)
    float vs2[11];
    ConePrefix prefix;  // the descent every cone of the bin shares
    uint32_t begin, end, key, bin;
    int nextTile;
};

// BxDFProjFunc of KCGenAndSampleDistributionProduct: cell centre of the
// 8x8 map, tilted toward the normal by one cell's solid angle
__device__ __forceinline__ V3 bxdf_proj(int cx, int cy, V3 nrm) {
    const float rc = 1.0f / 8.0f;
    const float s = (static_cast<float>(cx) + 0.5f) * rc, t = (static_cast<float>(cy) + 0.5f) * rc;
    V3 dir = octa_to_dir_yup(s, t);
    const V3 right = normalize(cross(dir, nrm));
    float angle = 4.0f * kPiF / 64.0f;
    angle *= 0.5f;
    float sn, cs;
    pm_sincos(angle, sn, cs);
    const Q4 q = {cs, right.x * sn, right.y * sn, right.z * sn};
    return qrotate(q, dir);
}

// inclusive Kogge-Stone scan over aligned groups of 8 lanes
__device__ __forceinline__ float scan8(float x, uint32_t lane) {
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
        const float y = __shfl_up_sync(0xFFFFFFFFu, x, off, 8);
        if ((lane & 7u) >= static_cast<uint32_t>(off)) x = y + x;
    }
    return x;
}

// ProductSampler::Pdf (ProductSampler.cuh:508-540) for the warp's fields
template <int X>
__device__ __forceinline__ float product_pdf(const GuideSmem<X>& S, int warp, float s, float t) {
    constexpr int DPP = X / 8;
    const float dppF = static_cast<float>(DPP);
    const float ex = s * 8.0f, ey = t * 8.0f;
    const float ox = floorf(ex), oy = floorf(ey);
    const float ix = (ex - ox) * dppF, iy = (ey - oy) * dppF;
    int ocx = f2i_sat(ox), ocy = f2i_sat(oy);
    ocx = ocx < 0 ? 0 : (ocx > 7 ? 7 : ocx);
    ocy = ocy < 0 ? 0 : (ocy > 7 ? 7 : ocy);
    int gx = ocx * DPP + f2i_sat(floorf(ix)), gy = ocy * DPP + f2i_sat(floorf(iy));
    gx = gx < 0 ? 0 : (gx > X - 1 ? X - 1 : gx);
    gy = gy < 0 ? 0 : (gy > X - 1 ? X - 1 : gy);
    const int cell = ocy * 8 + ocx;
    const float inner = S.field[gy * X + gx] / S.small[cell];
    return S.pdfX[warp][cell] * S.pdfY[warp][ocy] * inner;
}

// KCGenAndSampleDistribution (WFPGTracerKC.cuh:1356-1559), the non-product
// sampler of one bin: a 2D piecewise-constant distribution over the
// filtered X x X field (S.field).  Row prefix sums run left to right, one
// thread per row, into S.tmp; the marginal over rows bottom to top, by one
// thread, into S.marg (both in float, in this order on both sides of the
// oracle comparison).  Then one thread per ray: a draw from the
// distribution (probability misRatio) or from the BxDF.  A draw takes the
// first row whose prefix exceeds xi0 * total and the first cell of that row
// whose prefix exceeds xi1 * rowTotal, with the offset inside the cell from
// the remainder.  The density over the unit square is f * X^2 / total, over
// the sphere (equal-area map) that / (4 pi).  The guide word carries the
// one-sample MIS pdf as the product sampler's does.
template <int X>
__device__ __forceinline__ void pwc_sample_bin(const GuideArgs& A, GuideSmem<X>& S, uint32_t begin,
                                               uint32_t end, uint32_t frame) {
    const uint32_t tid = threadIdx.x;
    const SceneDev& sc = A.sc;
    if (tid < static_cast<uint32_t>(X)) {
        float acc = 0.0f;
        for (int x = 0; x < X; x++) {
            acc += S.field[tid * X + x];
            S.tmp[tid * X + x] = acc;
        }
    }
    __syncthreads();
    if (tid == 0) {
        float acc = 0.0f;
        for (int y = 0; y < X; y++) {
            acc += S.tmp[y * X + X - 1];
            S.marg[y] = acc;
        }
    }
    __syncthreads();
    const float total = S.marg[X - 1];
    const float scale = static_cast<float>(X * X) / total;
    const float below1 = 0x1.fffffep-1f;
    auto pdf_at = [&](float u, float v) {
        int ix = f2i_sat(floorf(u * static_cast<float>(X)));
        int iy = f2i_sat(floorf(v * static_cast<float>(X)));
        ix = ix < 0 ? 0 : (ix > X - 1 ? X - 1 : ix);
        iy = iy < 0 ? 0 : (iy > X - 1 ? X - 1 : iy);
        return S.field[iy * X + ix] * scale * kInv4Pi;
    };
    for (uint32_t r = tid; begin + r < end; r += kGuideTPB) {
        const uint32_t rid = A.binRid[begin + r];
        const uint32_t key = A.w.hit.key[rid];
        const uint32_t batch = key >> kIdBits, id = key & kIdMask;
        const float4 rd = A.w.rayD[rid];
        const V3 d = v3(rd.x, rd.y, rd.z);
        const RayAux aux = A.w.aux[rid];
        const bool isLight = batch == kBatchLight;
        const bool spec = !isLight && mat_specular(sc, batch, id);
        const float2 hb = A.w.hit.bary[rid];
        const Surface sf = gen_surface(sc, A.w.hit.prim[rid], hb.x, hb.y, d);
        const V3 wi = -d;
        const Rand4 r0 = philox_uniform4(aux.sample, frame, kTagGuide | A.depthTag, 0u,
                                         A.opt.seedLo, A.opt.seedHi);
        const bool purePG = A.go.purePG != 0;
        float s = 0.0f, t = 0.0f, pdf = 1.0f;
        bool bxdfSel = true;
        if (!purePG && (isLight || spec)) {
            // SampleMIS early out: light or specular surface
        } else if (!purePG && r0.u[0] >= A.go.misRatio) {
            const Rand4 r1 = philox_uniform4(aux.sample, frame, kTagGuide | A.depthTag, 1u,
                                             A.opt.seedLo, A.opt.seedHi);
            const BSample bs = mat_sample(sc, batch, id, wi, sf, aux.medium, r1.u[0], r1.u[1],
                                          r1.u[2]);
            dir_yup_to_octa(bs.dir, s, t);
            const float pdfSampled = bs.pdf;
            const float pdfOther = pdf_at(s, t);
            const float ratio = 1.0f - A.go.misRatio;
            const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
            pdf = pdfSampled * ratio / (w0 / (w0 + w1));
            pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
            bxdfSel = true;
        } else {
            const float tY = r0.u[1] * total;
            int lo = 0, hi = X - 1;  // first row whose prefix exceeds tY, else the last
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (S.marg[mid] > tY) hi = mid;
                else lo = mid + 1;
            }
            const int y = lo;
            const float rowTot = S.tmp[y * X + X - 1];
            const float prevY = (y > 0) ? S.marg[y - 1] : 0.0f;
            const float dv = fminf(fmaxf((tY - prevY) / rowTot, 0.0f), below1);
            const float tX = r0.u[2] * rowTot;
            lo = 0;
            hi = X - 1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (S.tmp[y * X + mid] > tX) hi = mid;
                else lo = mid + 1;
            }
            const int x = lo;
            const float prevX = (x > 0) ? S.tmp[y * X + x - 1] : 0.0f;
            const float du = fminf(fmaxf((tX - prevX) / S.field[y * X + x], 0.0f), below1);
            const float rcpX = 1.0f / static_cast<float>(X);
            s = (static_cast<float>(x) + du) * rcpX;
            t = (static_cast<float>(y) + dv) * rcpX;
            const float pdfSampled = S.field[y * X + x] * scale * kInv4Pi;
            if (purePG) {
                pdf = pdfSampled;
            } else {
                const V3 wo = octa_to_dir_yup(s, t);
                const float pdfOther = mat_pdf(sc, batch, id, wo, wi, sf);
                const float ratio = A.go.misRatio;
                const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
                pdf = pdfSampled * ratio / (w0 / (w0 + w1));
                pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
            }
            bxdfSel = false;
        }
        if (pdf != pdf || s != s || t != t) {
            s = 0.5f;
            t = 0.5f;
            pdf = 1.0f;
        }
        A.guide[rid] = make_uint2(uint32_t(f2h(s)) | (uint32_t(f2h(t)) << 16),
                                  uint32_t(f2h(pdf)) | (bxdfSel ? kGuideBxdf : 0u) | kGuideValid);
    }
}

template <int X, bool kProduct>
__global__ void __launch_bounds__(kGuideTPB, 4) k_guide(GuideArgs A) {
    __shared__ GuideSmem<X> S;
    constexpr int DPP = X / 8;
    const float dppF = static_cast<float>(DPP);
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const int warp = static_cast<int>(tid >> 5);
    const uint32_t nBins = *A.binCount;
    const uint32_t frame = *A.opt.frame;
    const SceneDev& sc = A.sc;
    const float aperture = (4.0f * kPiF) / (static_cast<float>(X) * static_cast<float>(X));
    const uint32_t mix = hash32(frame ^ hash32(A.depthTag ^ 0xA511E9B3u ^ A.opt.seedLo));
    if (tid < 12) S.span[tid] = neg_exp2i(tid);
    if (tid < 11) S.vs2[tid] = level_voxel_size_sqr(A.g, tid);
    const ConeTables tables{S.span, S.vs2};  // read after the first bin's barrier
    // bins differ widely in cost (rays, cone lengths): blocks take them in
    // turn from a counter rather than in a fixed stride
    for (;;) {
        if (tid == 0) {
            const uint32_t b = atomicAdd(A.binNext, 1u);
            S.bin = b;
            if (b < nBins) {
                S.begin = A.binBegin[b];
                S.end = A.binEnd[b];
                S.key = A.binKey[S.begin];
            }
        }
        __syncthreads();
        if (S.bin >= nBins) break;
        const uint32_t begin = S.begin, end = S.end;
        // representative ray: smallest (hash(path), path) of the bin
        unsigned long long best = ~0ull;
        uint32_t bestRid = 0;
        for (uint32_t i = begin + tid; i < end; i += kGuideTPB) {
            const uint32_t rid = A.binRid[i];
            const uint32_t smp = A.w.aux[rid].sample;
            const unsigned long long k = (static_cast<unsigned long long>(hash32(smp ^ mix)) << 32) | smp;
            if (k < best) {
                best = k;
                bestRid = rid;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long ob = __shfl_down_sync(0xFFFFFFFFu, best, off);
            const uint32_t orid = __shfl_down_sync(0xFFFFFFFFu, bestRid, off);
            if (ob < best) {
                best = ob;
                bestRid = orid;
            }
        }
        if (lane == 0) {
            S.repKey[warp] = best;
            S.repRid[warp] = bestRid;
        }
        __syncthreads();
        if (tid == 0) {
            unsigned long long b = S.repKey[0];
            uint32_t rid = S.repRid[0];
            for (int k = 1; k < kGuideWarps; k++)
                if (S.repKey[k] < b) {
                    b = S.repKey[k];
                    rid = S.repRid[k];
                }
            // CalculateJitterAndBinRayOrigin (WFPGTracerKC.cuh:1130-1188)
            const float4 rd = A.w.rayD[rid];
            const float2 hb = A.w.hit.bary[rid];
            const Surface sf = gen_surface(sc, A.w.hit.prim[rid], hb.x, hb.y, v3(rd.x, rd.y, rd.z));
            V3 pos = nudge(sf.pos, sf.geo);
            pos = pos + sf.geo * (A.g.leafVoxelSize * 0.01f);
            float tMin = A.g.leafVoxelSize * 0.15f;
            tMin += 1.0e-5f;
            S.origin[0] = pos.x;
            S.origin[1] = pos.y;
            S.origin[2] = pos.z;
            S.origin[3] = tMin;
            S.prefix = cone_prefix(A.g, pos, tMin, aperture, 0u);
            const Rand4 rj = philox_uniform4(S.key, frame, kTagGuideBin | A.depthTag, 0u,
                                             A.opt.seedLo, A.opt.seedHi);
            S.jitter[0] = rj.u[0];
            S.jitter[1] = rj.u[1];
            S.nextTile = 0;
        }
        __syncthreads();
        // GenerateRadianceField: one cone per texel of the X*X map.  Warps
        // take 8x4 texel tiles from a shared counter (neighbouring cones
        // traverse similar nodes; fast warps take more tiles); every cone
        // starts below the bin's shared descent.
        {
            const V3 org = v3(S.origin[0], S.origin[1], S.origin[2]);
            const float tMin = S.origin[3];
            const float jx = S.jitter[0], jy = S.jitter[1];
            constexpr int kTiles = (X / 8) * (X / 4);
            for (;;) {
                int tile = 0;
                if (lane == 0) tile = atomicAdd(&S.nextTile, 1);
                tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
                if (tile >= kTiles) break;
                const int x = (tile % (X / 8)) * 8 + static_cast<int>(lane & 7u);
                const int y = (tile / (X / 8)) * 4 + static_cast<int>(lane >> 3);
                const int p = y * X + x;
                float s = (static_cast<float>(x) + jx) / static_cast<float>(X);
                float t = (static_cast<float>(y) + jy) / static_cast<float>(X);
                octa_wrap(s, t);
                const V3 dir = octa_to_dir_yup(s, t);
                bool isLeaf;
                uint32_t id;
                cone_trace(A.g, org, dir, tMin, aperture, 0u, isLeaf, id, &S.prefix, &tables);
                float r = read_radiance(A.g, dir, id, isLeaf);
                if (r == 0.0f) r = kLargeEpsilon;
                S.field[p] = r;
            }
        }
        __syncthreads();
        // separable Gaussian, rows then columns, octahedral wrap at the edges
        for (int p = static_cast<int>(tid); p < X * X; p += kGuideTPB) {
            const int x = p % X, y = p / X;
            float acc = 0.0f;
#pragma unroll
            for (int j = -5; j <= 5; j++) {
                int nx = x + j, ny = y;
                if (nx >= X || nx < 0) octa_wrap_int(nx, ny, X, X);
                acc += S.field[ny * X + nx] * A.go.filter[j + 5];
            }
            S.tmp[p] = acc;
        }
        __syncthreads();
        for (int p = static_cast<int>(tid); p < X * X; p += kGuideTPB) {
            const int x = p % X, y = p / X;
            float acc = 0.0f;
#pragma unroll
            for (int j = -5; j <= 5; j++) {
                int nx = x, ny = y + j;
                if (ny >= X || ny < 0) octa_wrap_int(nx, ny, X, X);
                acc += S.tmp[ny * X + nx] * A.go.filter[j + 5];
            }
            S.field[p] = acc;
        }
        __syncthreads();
        if constexpr (!kProduct) {
            pwc_sample_bin<X>(A, S, begin, end, frame);
        } else {
            // 8x8 outer field: mean and max of each DPP x DPP block
            // (ProductSampler.cuh:160-215).  The mean adds the block's texels
            // as the reference's cub warp reduction does: row-major, in chunks
            // of at most 32 (a logical warp of min(32, max(2, DPP^2)) lanes,
            // lanes past DPP^2 holding 0), each chunk as a pairwise tree
            // (pairs at distance 1, 2, 4, ...), the chunk sums added in order
            if (tid < 64) {
                constexpr int N = DPP * DPP;
                constexpr int W = N >= 32 ? 32 : (N < 2 ? 2 : N);
                constexpr int IT = N >= 32 ? N / 32 : 1;
                const int cx = static_cast<int>(tid) & 7, cy = static_cast<int>(tid) >> 3;
                float total = 0.0f, mx = 0.0f;
                for (int it = 0; it < IT; it++) {
                    float v[W];
#pragma unroll
                    for (int l = 0; l < W; l++) {
                        const int li = l + it * 32;
                        v[l] = (li < N) ? S.field[(cy * DPP + li / DPP) * X + cx * DPP + li % DPP]
                                        : 0.0f;
                        mx = fmaxf(mx, v[l]);
                    }
#pragma unroll
                    for (int off = 1; off < W; off <<= 1)
#pragma unroll
                        for (int l = 0; l + off < W; l += 2 * off) v[l] = v[l] + v[l + off];
                    total += v[0];
                }
                S.small[tid] = total / static_cast<float>(N);
                S.norm[tid] = mx;
            }
            __syncthreads();
            // one warp per ray of the bin
            for (uint32_t r = static_cast<uint32_t>(warp); begin + r < end; r += kGuideWarps) {
                const uint32_t rid = A.binRid[begin + r];
                const uint32_t key = A.w.hit.key[rid];
                const uint32_t batch = key >> kIdBits, id = key & kIdMask;
                const float4 rd = A.w.rayD[rid];
                const V3 d = v3(rd.x, rd.y, rd.z);
                const RayAux aux = A.w.aux[rid];
                const bool isLight = batch == kBatchLight;
                const bool spec = !isLight && mat_specular(sc, batch, id);
                const float2 hb = A.w.hit.bary[rid];
                const Surface sf = gen_surface(sc, A.w.hit.prim[rid], hb.x, hb.y, d);
                const V3 wi = -d;
                const V3 nrm = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
                // MultiplyWithBXDF + GeneratePDFAndCDF
    #pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int c = static_cast<int>(lane) + 32 * j;
                    const int cx = c & 7, cy = c >> 3;
                    float gray = 1.0f;
                    if (!isLight && !spec) {
                        const V3 wo = bxdf_proj(cx, cy, nrm);
                        gray = lum3(mat_eval(sc, batch, id, wo, wi, sf));
                    }
                    const float prod = fmaxf(kVeryLargeEpsilon, gray * S.small[c]);
                    const float incl = scan8(prod, lane);
                    const float rowTotal = __shfl_sync(0xFFFFFFFFu, incl, 7, 8);
                    const float rcp = 1.0f / rowTotal;
                    S.cdfX[warp][c] = incl * rcp;
                    S.pdfX[warp][c] = prod * 8.0f * rcp;
                    if ((lane & 7u) == 0) S.rowTot[warp][cy] = rowTotal;
                }
                __syncwarp();
                {
                    const float py = (lane < 8) ? S.rowTot[warp][lane] : 0.0f;
                    const float incl = scan8(py, lane);
                    const float colTotal = __shfl_sync(0xFFFFFFFFu, incl, 7, 8);
                    const float rcp = 1.0f / colTotal;
                    if (lane < 8) {
                        S.cdfY[warp][lane] = incl * rcp;
                        S.pdfY[warp][lane] = py * (8.0f * rcp);
                    }
                }
                __syncwarp();
                const Rand4 r0 = philox_uniform4(aux.sample, frame, kTagGuide | A.depthTag, 0u,
                                                 A.opt.seedLo, A.opt.seedHi);
                const bool purePG = A.go.purePG != 0;
                float s = 0.0f, t = 0.0f, pdf = 1.0f;
                bool bxdfSel = true;
                if (!purePG && (isLight || spec)) {
                    // SampleMIS early out: light or specular surface
                } else if (!purePG && r0.u[0] >= A.go.misRatio) {
                    // BxDF sample, guide pdf of its direction
                    const Rand4 r1 = philox_uniform4(aux.sample, frame, kTagGuide | A.depthTag, 1u,
                                                     A.opt.seedLo, A.opt.seedHi);
                    const BSample bs = mat_sample(sc, batch, id, wi, sf, aux.medium, r1.u[0], r1.u[1],
                                                  r1.u[2]);
                    dir_yup_to_octa(bs.dir, s, t);
                    const float pdfSampled = bs.pdf;
                    const float pdfOther = product_pdf<X>(S, warp, s, t) * kInv4Pi;
                    const float ratio = 1.0f - A.go.misRatio;
                    const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
                    pdf = pdfSampled * ratio / (w0 / (w0 + w1));
                    pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
                    bxdfSel = true;
                } else {
                    // ProductSampler::Sample (ProductSampler.cuh:337-470)
                    const float xi0 = r0.u[1], xi1 = r0.u[2];
                    const float cY = (lane < 8) ? S.cdfY[warp][lane] : 0.0f;
                    uint32_t mask = __ballot_sync(0xFFFFFFFFu, lane < 8 && xi0 > cY);
                    int rowId = __ffs(~mask) - 1;
                    rowId = rowId > 7 ? 7 : rowId;
                    const float cX = (lane < 8) ? S.cdfX[warp][rowId * 8 + static_cast<int>(lane)] : 0.0f;
                    mask = __ballot_sync(0xFFFFFFFFu, lane < 8 && xi1 > cX);
                    int colId = __ffs(~mask) - 1;
                    colId = colId > 7 ? 7 : colId;
                    const int cell = rowId * 8 + colId;
                    const float normC = S.norm[cell];
                    float u = 0.0f, v = 0.0f, tex = 0.0f;
                    int lucky = -1;
                    for (int round = 0; round < 24; round++) {
                        const Rand4 rl = philox_uniform4(aux.sample, frame, kTagGuide | A.depthTag,
                                                         2u + static_cast<uint32_t>(round) * 32u + lane,
                                                         A.opt.seedLo, A.opt.seedHi);
                        u = rl.u[0];
                        v = rl.u[1];
                        const int ix = f2i_sat(u * dppF), iy = f2i_sat(v * dppF);
                        tex = S.field[(rowId * DPP + iy) * X + colId * DPP + ix];
                        const float nv = tex / normC;
                        const uint32_t acc = __ballot_sync(0xFFFFFFFFu, rl.u[2] <= nv);
                        lucky = __ffs(acc) - 1;
                        if (lucky >= 0) {
                            u = __shfl_sync(0xFFFFFFFFu, u, lucky);
                            v = __shfl_sync(0xFFFFFFFFu, v, lucky);
                            tex = __shfl_sync(0xFFFFFFFFu, tex, lucky);
                            break;
                        }
                    }
                    u = __shfl_sync(0xFFFFFFFFu, u, 0);
                    v = __shfl_sync(0xFFFFFFFFu, v, 0);
                    tex = __shfl_sync(0xFFFFFFFFu, tex, 0);
                    const float pdfInner = (lucky >= 0) ? tex / S.small[cell] : 1.0f;
                    const float pdfS = S.pdfY[warp][rowId] * S.pdfX[warp][cell] * pdfInner;
                    const float rcpX = 1.0f / static_cast<float>(X);
                    s = (static_cast<float>(colId) * dppF + u * dppF) * rcpX;
                    t = (static_cast<float>(rowId) * dppF + v * dppF) * rcpX;
                    if (purePG) {
                        pdf = pdfS * kInv4Pi;
                    } else {
                        const float pdfSampled = pdfS * kInv4Pi;
                        const V3 wo = octa_to_dir_yup(s, t);
                        const float pdfOther = mat_pdf(sc, batch, id, wo, wi, sf);
                        const float ratio = A.go.misRatio;
                        const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
                        pdf = pdfSampled * ratio / (w0 / (w0 + w1));
                        pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
                    }
                    bxdfSel = false;
                }
                if (lane == 0) {
                    if (pdf != pdf || s != s || t != t) {
                        s = 0.5f;
                        t = 0.5f;
                        pdf = 1.0f;
                    }
                    A.guide[rid] = make_uint2(uint32_t(f2h(s)) | (uint32_t(f2h(t)) << 16),
                                              uint32_t(f2h(pdf)) | (bxdfSel ? kGuideBxdf : 0u) |
                                                  kGuideValid);
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// radiance deposit, averages and level filters
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_path_deposit(GuideDev g, PathChain pc,
                                                      const uint32_t* __restrict__ framePtr) {
    const uint32_t frame = *framePtr;
    const size_t P = pc.paths;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pc.paths;
         p += gridDim.x * blockDim.x) {
        uint32_t L = 0;
        while (L + 1 < pc.levels && fbits(pc.nodeA[size_t(L + 1) * P + p].w) == frame) L++;
        const uint32_t lastD = (L + 1 < pc.levels) ? L + 1 : pc.levels - 1;
        for (uint32_t d = 1; d <= L; d++) {
            const float4 a = pc.nodeA[size_t(d) * P + p];
            const float4 b = pc.nodeB[size_t(d) * P + p];
            V3 tot = v3(0.0f, 0.0f, 0.0f);
            for (uint32_t D = d + 1; D <= lastD; D++) {
                const float4 cn = pc.contribNee[size_t(D) * P + p];
                const float4 cp = pc.contribPath[size_t(D) * P + p];
                tot.x += (b.x == 0.0f) ? 0.0f : cn.x / b.x;
                tot.y += (b.y == 0.0f) ? 0.0f : cn.y / b.y;
                tot.z += (b.z == 0.0f) ? 0.0f : cn.z / b.z;
                tot.x += (b.x == 0.0f) ? 0.0f : cp.x / b.x;
                tot.y += (b.y == 0.0f) ? 0.0f : cp.y / b.y;
                tot.z += (b.z == 0.0f) ? 0.0f : cp.z / b.z;
            }
            const V3 pos = v3(a.x, a.y, a.z);
            const float4 pa = pc.nodeA[size_t(d - 1) * P + p];
            const V3 wo = normalize(v3(pa.x, pa.y, pa.z) - pos);
            uint32_t leaf;
            if (!svo_nearest(g, leaf, pos, g.leafDepth)) continue;
            if (d + 1 <= lastD) {
                // DepositNEEHitMiss (AnisoSVO.cuh:1101-1115) of the rays this
                // vertex launched, at its own leaf
                const float en = pc.contribNee[size_t(d + 1) * P + p].w;
                const float ep = pc.contribPath[size_t(d + 1) * P + p].w;
                const uint32_t hits = (en == kChainHit ? 1u : 0u) + (ep == kChainHit ? 1u : 0u);
                if (hits) atomicAdd(g.leafShadow + 2 * leaf, hits);
                if (en == kChainMiss) atomicAdd(g.leafShadow + 2 * leaf + 1, 1u);
            }
            float sd, sp;
            const V3 n = read_normal_spec(g.leafNormSpec[leaf], sd, sp);
            const float NdL = dot(n, wo);
            int side;
            if (NdL >= 0.0f) side = 0;
            else if (NdL < 0.0f) side = 1;
            else continue;
            atomicAdd(g.leafIrr + 2 * leaf + side, to_fixed(lum3(tot)));
            atomicAdd(g.leafCnt + 2 * leaf + side, 1u);
        }
    }
}

// KCCCopyRadianceToHalfBufferLeaf: average (computed in double from the
// fixed-point sum), clamped to the half range
__global__ void __launch_bounds__(256) k_leaf_normalize(GuideDev g) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < g.leafCount;
         l += gridDim.x * blockDim.x) {
        uint32_t w = 0;
        for (int s = 0; s < 2; s++) {
            const uint32_t c = g.leafCnt[2 * l + s];
            float avg = 0.0f;
            if (c) avg = static_cast<float>(static_cast<double>(g.leafIrr[2 * l + s]) / kFixScale /
                                            static_cast<double>(c));
            avg = fminf(avg, 65504.0f);
            w |= uint32_t(f2h(avg)) << (16 * s);
        }
        g.leafAvg[l] = w;
    }
}

// KCBottomUpFilterIrradiance: per node, the children's averages on the
// side that matches the node normal (swapped where the child's normal
// faces away); children at HALF_MAX carry no data.  The sum runs in FP32
// and is rounded to FP16 once.  The guiding factor is the FP32 mean of the
// children's factors that are not NaN, rounded to FP16 (AnisoSVO.cu:
// 586-613); a leaf's factor is misses / (hits + misses) of its shadow rays
// (VoxelPayload::ReadGuidingFactor, AnisoSVO.cuh:477-488), NaN without any.
// A node whose children are all NaN gets the binary16 NaN 0x7FFF (0 / 0).
__global__ void __launch_bounds__(256) k_bottom_up(GuideDev g, uint32_t begin, uint32_t end,
                                                   int childrenAreLeaf) {
    for (uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += gridDim.x * blockDim.x) {
        const uint64_t node = g.nodes[k];
        const uint32_t cnt = __popc(svo_mask(node)), ci = svo_child_index(node);
        float sd, sp;
        const V3 n = read_normal_spec(g.nodeNormSpec[k], sd, sp);
        float sum[2] = {0.0f, 0.0f};
        uint32_t valid[2] = {0u, 0u};
        float factorSum = 0.0f;
        uint32_t factorValid = 0;
        for (uint32_t i = 0; i < cnt; i++) {
            const uint32_t c = ci + i;
            float factor;
            if (childrenAreLeaf) {
                const uint2 hm = reinterpret_cast<const uint2*>(g.leafShadow)[c];
                const float hit = static_cast<float>(hm.x), miss = static_cast<float>(hm.y);
                factor = miss / (hit + miss);
            } else {
                factor = h2f(g.nodeFactor[c]);
            }
            if (!isnan(factor)) {
                factorValid++;
                factorSum += factor;
            }
            const uint32_t irr = childrenAreLeaf ? g.leafAvg[c] : g.nodeAvg[c];
            const V3 cn = read_normal_spec(childrenAreLeaf ? g.leafNormSpec[c] : g.nodeNormSpec[c],
                                           sd, sp);
            const bool swap = dot(cn, n) < 0.0f;
            for (int j = 0; j < 2; j++) {
                const int rdx = swap ? ((j + 1) % 2) : j;
                const uint16_t h = static_cast<uint16_t>(irr >> (16 * rdx));
                if (h != kHalfMax) {
                    valid[j]++;
                    sum[j] += h2f(h);
                }
            }
        }
        uint32_t w = 0;
        for (int j = 0; j < 2; j++) {
            const uint16_t h = valid[j] ? f2h(fminf(sum[j] / static_cast<float>(valid[j]), 65504.0f))
                                        : kHalfMax;
            w |= uint32_t(h) << (16 * j);
        }
        g.nodeAvg[k] = w;
        g.nodeFactor[k] =
            factorValid ? f2h(factorSum / static_cast<float>(factorValid)) : kFactorNone;
    }
}

// KCTopDownFilterIrradiance: a side without data takes the parent's value
__global__ void __launch_bounds__(256) k_top_down(GuideDev g, uint32_t begin, uint32_t end,
                                                  int isLeaf) {
    for (uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += gridDim.x * blockDim.x) {
        const uint32_t parent = isLeaf ? g.leafParents[k] : svo_parent(g.nodes[k]);
        uint32_t* arr = isLeaf ? g.leafAvg : g.nodeAvg;
        const uint32_t w = arr[k], pw = g.nodeAvg[parent];
        uint32_t lo = w & 0xFFFFu, hi = w >> 16;
        if (lo == kHalfMax) lo = pw & 0xFFFFu;
        if (hi == kHalfMax) hi = pw >> 16;
        arr[k] = lo | (hi << 16);
    }
}

// KCAverageNormals: 2-means of the children's normals scaled by
// 1 / (1 + std dev); the larger cluster's mean keeps its length, which
// encodes the spread (Toksvig).  The reference's accumulation buffer of
// the first pass is uninitialised; here it starts at zero.
__global__ void __launch_bounds__(256) k_average_normals(GuideDev g, uint32_t begin, uint32_t end,
                                                         int childrenAreLeaf) {
    for (uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += gridDim.x * blockDim.x) {
        const uint64_t node = g.nodes[k];
        const uint32_t cnt = __popc(svo_mask(node)), ci = svo_child_index(node);
        V3 nb[8];
        float avgSpec = 0.0f;
        for (uint32_t i = 0; i < cnt; i++) {
            float sd, sp;
            const V3 n = read_normal_spec(childrenAreLeaf ? g.leafNormSpec[ci + i] : g.nodeNormSpec[ci + i],
                                          sd, sp);
            const float len = 1.0f / (1.0f + sd);
            nb[i] = n * len;
            avgSpec += sp;
        }
        avgSpec *= 1.0f / static_cast<float>(cnt);
        V3 mean[2][2];
        uint32_t counts[2][2];
        mean[0][0] = nb[0];
        mean[0][1] = -nb[0];
        mean[1][0] = mean[1][1] = v3(0.0f, 0.0f, 0.0f);
        counts[0][0] = counts[0][1] = 0;
        counts[1][0] = counts[1][1] = 0;
        for (int pass = 0; pass < 4; pass++) {
            const int rd = pass % 2, wr = rd ? 0 : 1;
            for (uint32_t i = 0; i < cnt; i++) {
                const V3 n = nb[i];
                if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) continue;
                const float d0 = 1.0f - dot(mean[rd][0], n), d1 = 1.0f - dot(mean[rd][1], n);
                const int up = (d0 >= d1) ? 0 : 1;
                mean[wr][up] = mean[wr][up] + n;
                counts[wr][up] += 1;
            }
            mean[rd][0] = mean[rd][1] = v3(0.0f, 0.0f, 0.0f);
            counts[rd][0] = counts[rd][1] = 0;
        }
        const int idx = (counts[0][0] >= counts[0][1]) ? 0 : 1;
        const V3 m = mean[0][idx] * (1.0f / static_cast<float>(counts[0][idx]));
        g.nodeNormSpec[k] = write_normal_spec(m, avgSpec);
    }
}

}  // namespace

GuideDev guide_dev(const SvoResult& v, const SvoParams& p) {
    GuideDev g{};
    g.nodes = v.nodes;
    g.leafParents = v.leafParents;
    g.levelOffsets = v.dLevelOffsets;
    g.nodeCount = v.nodeCount;
    g.leafCount = v.leafCount;
    g.leafDepth = p.depth;
    g.res = p.res;
    for (int c = 0; c < 3; c++) {
        g.lo[c] = p.lo[c];
        g.hi[c] = p.hi[c];
    }
    g.leafVoxelSize = p.leafVoxelSize;
    g.leafNormSpec = v.leafNormSpec;
    g.nodeNormSpec = v.nodeNormSpec;
    g.leafIrr = v.leafIrr;
    g.leafCnt = v.leafCnt;
    g.leafAvg = v.leafAvg;
    g.nodeAvg = v.nodeAvg;
    g.leafShadow = v.leafShadow;
    g.nodeFactor = v.nodeFactor;
    g.leafBin = v.leafBin;
    g.nodeBin = v.nodeBin;
    return g;
}

int svo_normalize_filter(const GuideDev& g, const SvoResult& v, cudaStream_t st) {
    const uint32_t D = g.leafDepth;
    k_leaf_normalize<<<grid_for(g.leafCount, 256, 148 * 8), 256, 0, st>>>(g);
    for (int L = int(D) - 1; L >= 0; L--) {
        const uint32_t b = v.levelOffsets[L], e = v.levelOffsets[L + 1];
        k_bottom_up<<<grid_for(e - b, 256, 148 * 8), 256, 0, st>>>(g, b, e, L == int(D) - 1 ? 1 : 0);
    }
    for (uint32_t L = 1; L <= D; L++) {
        const bool leaf = (L == D);
        const uint32_t b = leaf ? 0u : v.levelOffsets[L];
        const uint32_t e = leaf ? v.leafCount : v.levelOffsets[L + 1];
        k_top_down<<<grid_for(e - b, 256, 148 * 8), 256, 0, st>>>(g, b, e, leaf ? 1 : 0);
    }
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int svo_payload_finish(const GuideDev& g, const SvoResult& v, cudaStream_t st) {
    const uint32_t D = g.leafDepth;
    for (int L = int(D) - 1; L >= 0; L--) {
        const uint32_t b = v.levelOffsets[L], e = v.levelOffsets[L + 1];
        k_average_normals<<<grid_for(e - b, 256, 148 * 8), 256, 0, st>>>(g, b, e,
                                                                          L == int(D) - 1 ? 1 : 0);
    }
    MRB_CUDA(cudaGetLastError());
    return svo_normalize_filter(g, v, st);
}

size_t guide_sort_temp_bytes(uint32_t maxRays) { return radix_sort_temp_bytes(maxRays, 4, 0, 32); }
size_t guide_scan_temp_bytes(uint32_t maxRays) { return exclusive_scan_temp_bytes(maxRays); }

uint32_t guide_launches(const SvoResult& v, const GuideOptions& go, uint32_t maxRays) {
    (void)v;
    (void)maxRays;
    const uint32_t D = static_cast<uint32_t>(v.levelOffsets.size()) - 2;
    const uint32_t collapse = 1 + (D > go.minBinLevel ? D - go.minBinLevel : 0);
    // memsets are not kernels; init, collapse, resolve, sort (histogram,
    // scan, 4 onesweep passes), heads, scan (3), ranges, guide
    return 1 + collapse + 1 + 6 + 1 + 3 + 1 + 1;
}

int guide_wavefront(const SceneDev& sc, const GuideDev& g, const SvoResult& v, const GuideWave& w,
                    const GuideScratch& s, const GuideOptions& go, const PathOptions& opt,
                    uint32_t iteration, uint32_t depthTag, cudaStream_t st, cudaEvent_t* marks) {
    auto mark = [&](int i) -> cudaError_t {
        return marks ? cudaEventRecord(marks[i], st) : cudaSuccess;
    };
    const uint32_t grid = grid_for(w.maxRays, 256, 148 * 8);
    MRB_CUDA(mark(0));
    MRB_CUDA(cudaMemsetAsync(g.leafBin, 0, size_t(g.leafCount) * 4, st));
    MRB_CUDA(cudaMemsetAsync(g.nodeBin, 0, size_t(g.nodeCount) * 4, st));
    MRB_CUDA(mark(1));
    BinArgs ba{g, w, s.binKey, s.guide};
    k_bin_init<<<grid, 256, 0, st>>>(ba);
    k_collapse_leaf<<<grid_for(g.leafCount, 256, 148 * 8), 256, 0, st>>>(g, go.minBinLevel,
                                                                         go.binRayCount);
    for (int L = int(g.leafDepth) - 1; L >= int(go.minBinLevel); L--) {
        const uint32_t b = v.levelOffsets[L], e = v.levelOffsets[L + 1];
        k_collapse_nodes<<<grid_for(e - b, 256, 148 * 8), 256, 0, st>>>(g, b, e, uint32_t(L),
                                                                       go.minBinLevel,
                                                                       go.binRayCount);
    }
    k_bin_resolve<<<grid, 256, 0, st>>>(g, w.count, s.binKey);
    MRB_CUDA(mark(2));
    int r = radix_sort_pairs<uint32_t>(s.binKey, s.binRid, w.count, w.maxRays, 0, 32, false,
                                       s.sortTemp, s.sortTempBytes, st, true);
    if (r) return r;
    k_bin_heads<<<grid, 256, 0, st>>>(s.binKey, w.count, w.maxRays, s.heads);
    if ((r = exclusive_scan_u32(s.heads, s.headScan, w.maxRays, s.scanTemp, st))) return r;
    k_bin_ranges<<<grid, 256, 0, st>>>(s.binKey, w.count, s.heads, s.headScan, s.binBegin,
                                       s.binEnd);
    MRB_CUDA(cudaMemsetAsync(s.binNext, 0, 4, st));
    MRB_CUDA(mark(3));
    GuideArgs ga{sc, g, w, s.binKey, s.binRid, s.binBegin, s.binEnd, s.headScan + w.maxRays,
                 s.binNext, s.guide, go, opt, depthTag};
    const uint32_t kernelIndex = iteration < 4 ? iteration : 4;
    switch (kernelIndex) {
        case 0:
        case 1:
            if (go.product) k_guide<64, true><<<148 * 4, kGuideTPB, 0, st>>>(ga);
            else k_guide<64, false><<<148 * 4, kGuideTPB, 0, st>>>(ga);
            break;
        case 2:
            if (go.product) k_guide<32, true><<<148 * 4, kGuideTPB, 0, st>>>(ga);
            else k_guide<32, false><<<148 * 4, kGuideTPB, 0, st>>>(ga);
            break;
        case 3:
            if (go.product) k_guide<16, true><<<148 * 6, kGuideTPB, 0, st>>>(ga);
            else k_guide<16, false><<<148 * 6, kGuideTPB, 0, st>>>(ga);
            break;
        default:
            if (go.product) k_guide<8, true><<<148 * 6, kGuideTPB, 0, st>>>(ga);
            else k_guide<8, false><<<148 * 6, kGuideTPB, 0, st>>>(ga);
            break;
    }
    MRB_CUDA(cudaGetLastError());
    MRB_CUDA(mark(4));
    return 0;
}

int path_deposit(const GuideDev& g, const PathChain& pc, const uint32_t* frame, cudaStream_t st) {
    k_path_deposit<<<grid_for(pc.paths, 256, 148 * 16), 256, 0, st>>>(g, pc, frame);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
