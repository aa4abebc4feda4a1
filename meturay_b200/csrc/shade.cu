// Camera ray generation, ray partitioning helpers, shading and image resolve
// for the plain wavefront path tracer.
//
//   k_camera       KCGenCameraRaysFromArrayGPU + GPUCameraPinhole::GenerateRay
//                  (GenerationKernels.cuh:26-108, GPUCameraPinhole.cuh:209-243)
//   k_dense_keys   HitKey -> dense (batch, id) key for the partition sort
//                  (FillMatIdsForSortKC, RayMemory.cu:17-30)
//   k_portions     batch boundaries of the sorted keys -> device portion
//                  table (FindSplitsSparseKC/FindSplitBatchesKC,
//                  RayMemory.cu:64-104,230-312), found with warp ballots
//   k_shade        one launch over all non-null rays in partition order:
//                  PathTracerPathWork / PathTracerBoundaryWork
//                  (PathTracerKC.cuh:335-649) with Lambert, Metal (GGX) and
//                  Refract BxDFs; outputs are compacted with warp-aggregated
//                  atomics into the next wavefront
//   k_resolve      per-pixel mean of its s*s samples, accumulated per frame
//                  (with no reconstruction filter attached; recon.cu splats
//                  through the filter otherwise)
#include "common.cuh"
#include "bxdf.cuh"
#include "shade.cuh"
#include "svo_dev.cuh"
#include "pool.cuh"

namespace mrb {

namespace {

// GPUCameraPinhole::GenerateRay for sample (sx, sy) of an SW x SH sample grid
// (GPUCameraPinhole.cuh:209-243); the tracer and the pool share it.
__device__ __forceinline__ void camera_ray(const CameraDev& cam, uint32_t sx, uint32_t sy,
                                           uint32_t SW, uint32_t SH, const Rand4& rc,
                                           float4& o, float4& d) {
    float dx = cam.planeSize[0] / static_cast<float>(SW);
    float dy = cam.planeSize[1] / static_cast<float>(SH);
    float sdx = static_cast<float>(sx) * dx;
    float sdy = static_cast<float>(sy) * dy;
    sdx += rc.u[0] * dx;
    sdy += rc.u[1] * dy;
    V3 sp = {cam.bottomLeft[0] + ((sdx * cam.right[0]) + (sdy * cam.up[0])),
             cam.bottomLeft[1] + ((sdx * cam.right[1]) + (sdy * cam.up[1])),
             cam.bottomLeft[2] + ((sdx * cam.right[2]) + (sdy * cam.up[2]))};
    V3 dir = normalize(sp - ld3(cam.position));
    o = make_float4(cam.position[0], cam.position[1], cam.position[2], cam.nearFar[0]);
    d = make_float4(dir.x, dir.y, dir.z, cam.nearFar[1]);
}

__global__ void __launch_bounds__(256) k_camera(const CameraDev* __restrict__ camPtr,
                                                PathOptions opt, uint32_t baseMedium,
                                                float4* __restrict__ rayO,
                                                float4* __restrict__ rayD,
                                                RayAux* __restrict__ aux,
                                                float4* __restrict__ samples,
                                                uint32_t* __restrict__ count, uint32_t total,
                                                PathChain chain,
                                                float2* __restrict__ imgCoords) {
    const uint32_t SW = opt.width * opt.samples, SH = opt.height * opt.samples;
    const uint32_t frame = *opt.frame;
    const CameraDev cam = *camPtr;
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = total;
    // wavefront slot i -> sample: 4 x 8 sample tiles (4 wide, 8 tall), so
    // that the 32 camera rays of a warp cover a compact patch of the image
    // (more shared node visits in the first traversal; on clusters-1M
    // 4 x 8 beat 8 x 4, 16 x 2, 2 x 16 and rows).  Every ray carries its sample id,
    // which keys its random numbers and its outputs, so the order of the
    // wavefront changes no result.
    const bool tiled = (SW % 4u == 0u) && (SH % 8u == 0u);
    const uint32_t tilesX = SW / 4u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += gridDim.x * blockDim.x) {
        uint32_t sx, sy;
        if (tiled) {
            const uint32_t tile = i >> 5, w = i & 31u;
            sx = (tile % tilesX) * 4u + (w & 3u);
            sy = (tile / tilesX) * 8u + (w >> 2);
        } else {
            sx = i % SW;
            sy = i / SW;
        }
        const uint32_t sid = sy * SW + sx;
        Rand4 rc = philox_uniform4(sid, frame, kTagCamera, 0u, opt.seedLo, opt.seedHi);
        camera_ray(cam, sx, sy, SW, SH, rc, rayO[i], rayD[i]);
        RayAux a;
        a.rf[0] = a.rf[1] = a.rf[2] = 1.0f;
        a.sample = sid;
        a.endpoint = kInvalid;
        a.medium = static_cast<uint16_t>(baseMedium);
        // WFPG numbers the camera ray depth 1 (RayAuxInitWFPG,
        // RayAuxStruct.cuh:322-350); its path chain starts at the camera
        a.depth = opt.wfpg ? 1 : 0;
        a.type = kCameraRay;
        a.prevPDF = __int_as_float(0x7fc00000);
        a.pad = 0;
        aux[i] = a;
        samples[sid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        // image-space coordinates for the reconstruction filter
        // (GPUCameraPinhole::GenerateRay localCoords * resolution,
        // GenerationKernels.cuh:62-88)
        if (imgCoords) {
            const float lx = (static_cast<float>(sx) + rc.u[0]) / static_cast<float>(SW);
            const float ly = (static_cast<float>(sy) + rc.u[1]) / static_cast<float>(SH);
            imgCoords[sid] = make_float2(lx * static_cast<float>(opt.width),
                                         ly * static_cast<float>(opt.height));
        }
        if (opt.wfpg) {
            chain.nodeA[sid] = make_float4(cam.position[0], cam.position[1], cam.position[2],
                                           __uint_as_float(frame));
            chain.nodeB[sid] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        }
    }
}

// Block 0 also adds the wavefront's ray count to the traced-ray total and
// clears the next wavefront's counter (where given): two tiny launches less
// per depth.
__global__ void __launch_bounds__(256) k_dense_keys(const uint32_t* __restrict__ hitKey,
                                                    const uint32_t* __restrict__ dCount,
                                                    uint32_t idBits, uint32_t* __restrict__ dense,
                                                    PortionTable table,
                                                    unsigned long long* rayTotal,
                                                    uint32_t* nextCount) {
    const uint32_t n = *dCount;
    if (blockIdx.x == 0 && threadIdx.x < 8) {
        table.offset[threadIdx.x] = 0;
        table.end[threadIdx.x] = 0;
        if (threadIdx.x == 0) {
            *table.nonNull = n;
            if (rayTotal) *rayTotal += n;
            if (nextCount) *nextCount = 0u;
        }
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = hitKey[i];
        dense[i] = ((k >> kIdBits) << idBits) | (k & ((1u << idBits) - 1u));
    }
}

// Batch boundaries of the sorted dense keys.  Each warp compares every key
// with its predecessor (shuffle, one global read at the warp edge), and the
// lanes where the batch changes write the portion bounds.
__global__ void __launch_bounds__(256) k_portions(const uint32_t* __restrict__ sortedDense,
                                                  const uint32_t* __restrict__ dCount,
                                                  uint32_t idBits, PortionTable table) {
    const uint32_t n = *dCount;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool ok = i < n;
        const uint32_t b = ok ? (sortedDense[i] >> idBits) : 0xFFFFFFFFu;
        uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, b, 1);
        uint32_t next = __shfl_down_sync(0xFFFFFFFFu, b, 1);
        if (lane == 0) prev = (i > 0 && ok) ? (sortedDense[i - 1] >> idBits) : 0xFFFFFFFEu;
        if (lane == 31) next = (i + 1 < n) ? (sortedDense[i + 1] >> idBits) : 0xFFFFFFFEu;
        if (!ok) continue;
        if (i + 1 == n) next = 0xFFFFFFFEu;
        if (b != prev) {
            table.offset[b] = i;
            if (b == kBatchNull) *table.nonNull = i;
        }
        if (b != next) table.end[b] = i + 1;
    }
}

struct ShadeArgs {
    SceneDev sc;
    const float4* rayO;
    const float4* rayD;
    const RayAux* aux;
    HitIn hit;
    const uint32_t* sortedIds;
    const uint32_t* nonNull;
    const uint32_t* count;  // all rays of the wavefront
    float4* samples;
    PathOptions opt;
    int gen;
    float4* outO;
    float4* outD;
    RayAux* outAux;
    uint32_t* outCount;
    PathChain chain;     // WFPG only
    const uint2* guide;  // WFPG guided directions of this wavefront, or null
    const JobDev* jobs;  // wavefront pool: the job table (null for one tracer)
};

__device__ __forceinline__ void accumulate(float4* samples, uint32_t s, V3 v) {
    float* p = reinterpret_cast<float*>(samples + s);
    atomicAdd(p + 0, v.x);
    atomicAdd(p + 1, v.y);
    atomicAdd(p + 2, v.z);
}

// kMulti: rays of a wavefront pool; scene, options, frame and the RNG
// sample index come from each ray's job (pool.cuh).
template <bool kMulti>
// Six 128-thread blocks per SM (80 registers, a little spilled): the
// kernel's gathers want resident warps (closed Cornell 1080p frame: 11.9 ->
// 11.2 ms of shading at 112 -> 80 registers).
__global__ void __launch_bounds__(128, 6) k_shade(ShadeArgs A) {
    // the WFPG tracer also visits the rays that left the scene (sorted
    // last), for the shadow-ray events of the boundary work
    const uint32_t n = (!kMulti && A.opt.wfpg) ? *A.count : *A.nonNull;
    const uint32_t tracerFrame = kMulti ? 0u : *A.opt.frame;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ltMask = (1u << lane) - 1u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        bool emitNee = false, emitPath = false;
        float4 neeO, neeD, pathO, pathD;
        RayAux neeAux, pathAux;
        if (j < n) {
            const uint32_t rid = A.sortedIds[j];
            const uint32_t key = A.hit.key[rid];
            const uint32_t batch = key >> kIdBits, id = key & kIdMask;
            const float4 rd = A.rayD[rid];
            const RayAux aux = A.aux[rid];
            const JobDev* job = kMulti ? A.jobs + aux.pad : nullptr;
            const SceneDev& s = kMulti ? job->sc : A.sc;
            const uint32_t frame = kMulti ? job->frame : tracerFrame;
            const uint32_t oNee = kMulti ? job->nee : A.opt.nee;
            const uint32_t oMis = kMulti ? job->mis : A.opt.mis;
            const uint32_t oRr = kMulti ? job->rrStart : A.opt.rrStart;
            const uint32_t oSeedLo = kMulti ? job->seedLo : A.opt.seedLo;
            const uint32_t oSeedHi = kMulti ? job->seedHi : A.opt.seedHi;
            const uint32_t rngSample = kMulti ? aux.sample - job->sampleBase : aux.sample;
            const bool gen = kMulti ? (uint32_t(aux.depth) + 1u < job->maxDepth) : (A.gen != 0);
            if (batch == kBatchLight) {
                // PathTracerBoundaryWork (PathTracerKC.cuh:335-426)
                const bool pathAsMis = oMis && aux.type == kPathRay;
                const bool camera = aux.type == kCameraRay;
                const bool specPath = aux.type == kSpecPathRay;
                const bool neeOn = oNee && aux.type == kNeeRay;
                const bool pathNeeOff =
                    (!oNee) && (aux.type == kPathRay || aux.type == kSpecPathRay);
                const bool correct = neeOn && (aux.endpoint == id);
                float misWeight = 1.0f;
                if (pathAsMis) {
                    // light pdf of this hit: GPULightSamplerUniform::Pdf and
                    // GPULight::Pdf(distance, position, direction, tbn)
                    const uint32_t prim = A.hit.prim[rid];
                    const float2 hb = A.hit.bary[rid];
                    const V3 d = {rd.x, rd.y, rd.z};
                    const Surface sf = gen_surface(s, prim, hb.x, hb.y, d);
                    const V3 dir = normalize(d);
                    float pdfM = 0.0f, pdfC = 0.0f;
                    if (id < s.lightCount) {
                        pdfM = 1.0f / static_cast<float>(s.lightCount);
                        const uint32_t i0 = s.idx[3 * prim], i1 = s.idx[3 * prim + 1],
                                       i2 = s.idx[3 * prim + 2];
                        const V3 p0 = ld3(s.pos + 3 * size_t(i0)), p1 = ld3(s.pos + 3 * size_t(i1)),
                                 p2 = ld3(s.pos + 3 * size_t(i2));
                        const V3 cr = cross(p1 - p0, p2 - p0);
                        const float area = sqrtf(dot(cr, cr)) * 0.5f;
                        const V3 ln = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
                        const float nDotL = fabsf(dot(ln, -dir));
                        const float dist = A.hit.t[rid];
                        pdfC = (1.0f / area) * dist * dist / nDotL;
                    }
                    misWeight = power_heuristic(aux.prevPDF, pdfC * pdfM);
                }
                if (pathNeeOff || pathAsMis || correct || camera || specPath) {
                    V3 total = ld3(s.lightRadiance + 3 * id) * v3(aux.rf[0], aux.rf[1], aux.rf[2]);
                    total = total * misWeight;
                    accumulate(A.samples, aux.sample, total);
                    // WFPGTracerBoundaryWork: the chain below this ray takes the
                    // endpoint radiance (AccumRadianceDownChain, WFPGTracerKC.cuh:300-310)
                    if (A.opt.wfpg && !camera) {
                        float4* c = (aux.type == kNeeRay) ? A.chain.contribNee : A.chain.contribPath;
                        c[size_t(aux.depth) * A.chain.paths + aux.sample] =
                            make_float4(total.x, total.y, total.z, kChainHit);
                    }
                }
            } else if (batch == kBatchNull) {
                // WFPGTracerBoundaryWork of the Null boundary light (emits
                // zero): the rays it accepts still count as reaching a light
                // for the vertex that launched them (WFPGTracerKC.cuh:163-195)
                const bool accepted = aux.type == kSpecPathRay ||
                                      (aux.type == kPathRay && (oMis || !oNee));
                if (accepted)
                    A.chain.contribPath[size_t(aux.depth) * A.chain.paths + aux.sample].w = kChainHit;
            } else if (aux.type == kNeeRay) {
                // a NEE ray stopped by a surface (WFPGTracerPathWork,
                // WFPGTracerKC.cuh:250-260)
                if (A.opt.wfpg)
                    A.chain.contribNee[size_t(aux.depth) * A.chain.paths + aux.sample].w = kChainMiss;
            } else if (gen || A.opt.wfpg) {
                // PathTracerPathWork (PathTracerKC.cuh:428-649)
                const uint32_t prim = A.hit.prim[rid];
                const float2 hb = A.hit.bary[rid];
                const V3 d = {rd.x, rd.y, rd.z};
                const Surface sf = gen_surface(s, prim, hb.x, hb.y, d);
                const V3 wi = -normalize(d);
                const V3 rf = {aux.rf[0], aux.rf[1], aux.rf[2]};
                bool specular;
                if (batch == kBatchLambert || batch == kBatchLambertC) specular = false;
                else if (batch == kBatchMetal) specular = (1.0f - s.metalParams[10 * id + 9]) >= 0.99f;
                else if (batch == kBatchUnreal) specular = (1.0f - s.unrealParams[6 * id + 3]) >= 0.99f;
                else specular = true;
                if (A.opt.wfpg) {
                    // WFPGPathNode of this vertex; the slots for the rays it
                    // launches are cleared for this frame
                    const size_t P = A.chain.paths;
                    const size_t at = size_t(aux.depth) * P + aux.sample;
                    A.chain.nodeA[at] = make_float4(sf.pos.x, sf.pos.y, sf.pos.z, __uint_as_float(frame));
                    A.chain.nodeB[at] = make_float4(rf.x, rf.y, rf.z, 0.0f);
                    if (A.chain.nodeN) {
                        const V3 nrm = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
                        A.chain.nodeN[at] = make_float4(nrm.x, nrm.y, nrm.z, specular ? 1.0f : 0.0f);
                        A.chain.nodeT[at] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0xFFFFFFFFu));
                    }
                    if (uint32_t(aux.depth) + 1 < A.chain.levels) {
                        const size_t nx = at + P;
                        A.chain.contribNee[nx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        A.chain.contribPath[nx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    }
                }
                // the last step's outputs are never traced; WFPG still keeps its
                // chain vertex (WorkRays runs at every depth, WFPGTracer.cu:1590-1697)
                if (gen) {
                const Rand4 ra = philox_uniform4(rngSample, frame, aux.depth, 0u,
                                                 oSeedLo, oSeedHi);
                const Rand4 rb = philox_uniform4(rngSample, frame, aux.depth, 1u,
                                                 oSeedLo, oSeedHi);
                // ---- NEE: GPULightSamplerUniform::SampleLight + primitive light
                if (oNee && !specular && s.lightCount > 0) {
                    const uint32_t lc = s.lightCount;
                    float r1 = ra.u[0] * static_cast<float>(lc);
                    uint32_t li = static_cast<uint32_t>(r1);
                    if (li == lc) li--;
                    const uint32_t lp = s.lightPrim[li];
                    // TriangleSurfaceGenerator SamplePosition (GPUPrimitiveTriangle.h:65-115)
                    const float sx = sqrtf(ra.u[1]);
                    const float r2 = ra.u[2];
                    const float la = 1.0f - sx;
                    const float lb = (1.0f - r2) * sx;
                    const float lcw = sx * r2;
                    const uint32_t i0 = s.idx[3 * lp], i1 = s.idx[3 * lp + 1], i2 = s.idx[3 * lp + 2];
                    const V3 p0 = ld3(s.pos + 3 * size_t(i0)), p1 = ld3(s.pos + 3 * size_t(i1)),
                             p2 = ld3(s.pos + 3 * size_t(i2));
                    const V3 cr = cross(p1 - p0, p2 - p0);
                    const float area = sqrtf(dot(cr, cr)) * 0.5f;
                    float lpdf = 1.0f / area;
                    Q4 q = bary_slerp(qnormalize(q_from(__ldg(s.tbn + i0))),
                                      qnormalize(q_from(__ldg(s.tbn + i1))),
                                      qnormalize(q_from(__ldg(s.tbn + i2))), la, lb);
                    V3 ln = to_space(v3(0.0f, 0.0f, 1.0f), q);
                    const V3 lpos = (p0 * la + p1 * lb) + p2 * lcw;
                    ln = normalize(ln);
                    V3 ldir = lpos - sf.pos;
                    const float d2 = dot(ldir, ldir);
                    const float dist = sqrtf(d2);
                    ldir = ldir * (1.0f / dist);
                    const float nDotL = fabsf(dot(ln, -ldir));
                    lpdf *= d2 / nDotL;
                    lpdf *= (1.0f / static_cast<float>(lc));
                    V3 refl;
                    float pdfBxdf;
                    if (batch == kBatchLambert) {
                        refl = lambert_eval(ld3(s.lambertAlbedo + 3 * id), ldir, sf);
                        pdfBxdf = oMis ? lambert_pdf(ldir, sf) : 0.0f;
                    } else if (batch == kBatchLambertC) {
                        refl = lambertc_eval(ld3(s.lambertCAlbedo + 3 * id), ldir, sf);
                        pdfBxdf = oMis ? lambert_pdf(ldir, sf) : 0.0f;
                    } else if (batch == kBatchUnreal) {
                        const UnrealP up = unreal_params(s.unrealParams + 6 * id);
                        refl = unreal_eval(up, ldir, wi, sf);
                        pdfBxdf = oMis ? unreal_pdf(up, ldir, wi, sf) : 0.0f;
                    } else {
                        const MetalP mp = metal_params(s.metalParams + 10 * id);
                        refl = metal_eval(mp, ldir, wi, sf);
                        pdfBxdf = oMis ? metal_pdf(mp, ldir, wi, sf) : 0.0f;
                    }
                    float pdfNee = lpdf;
                    if (oMis) {
                        pdfNee /= power_heuristic(lpdf, pdfBxdf);
                        if (isnan(pdfNee)) pdfNee = 0.0f;
                    }
                    V3 nrf = rf * refl;
                    nrf = (pdfNee == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : (nrf / pdfNee);
                    if (nonzero(nrf)) {
                        const V3 o = nudge(sf.pos, sf.geo);
                        emitNee = true;
                        neeO = make_float4(o.x, o.y, o.z, 0.0f);
                        neeD = make_float4(ldir.x, ldir.y, ldir.z, kFltMax);
                        neeAux = aux;
                        neeAux.rf[0] = nrf.x;
                        neeAux.rf[1] = nrf.y;
                        neeAux.rf[2] = nrf.z;
                        neeAux.endpoint = li;
                        neeAux.type = kNeeRay;
                        neeAux.prevPDF = __int_as_float(0x7fc00000);
                    }
                }
                // ---- BxDF sample, or the guided direction of this ray
                // (WFPGTracerPathWork, WFPGTracerKC.cuh:430-470)
                BSample bs;
                bool guided = false;
                if (A.guide && !specular) {
                    const uint2 gw = A.guide[rid];
                    const float gp = h2f(static_cast<uint16_t>(gw.y & 0xFFFFu));
                    if ((gw.y & (1u << 17)) && gp == gp) {
                        const V3 dir = octa_to_dir_yup(h2f(static_cast<uint16_t>(gw.x & 0xFFFFu)),
                                                       h2f(static_cast<uint16_t>(gw.x >> 16)));
                        bs.dir = dir;
                        bs.pdf = gp;
                        bs.refl = mat_eval(s, batch, id, dir, wi, sf);
                        bs.pos = nudge(sf.pos, sf.geo);
                        bs.medium = aux.medium;
                        guided = true;
                    }
                }
                if (guided) {
                } else if (batch == kBatchLambert) {
                    bs = lambert_sample(ld3(s.lambertAlbedo + 3 * id), sf, rb.u[0], rb.u[1],
                                        aux.medium);
                } else if (batch == kBatchLambertC) {
                    bs = lambertc_sample(ld3(s.lambertCAlbedo + 3 * id), sf, rb.u[0], rb.u[1],
                                         aux.medium);
                } else if (batch == kBatchUnreal) {
                    bs = unreal_sample(unreal_params(s.unrealParams + 6 * id), wi, sf, rb.u[2],
                                       rb.u[0], rb.u[1], aux.medium);
                } else if (batch == kBatchMetal) {
                    bs = metal_sample(metal_params(s.metalParams + 10 * id), wi, sf, rb.u[0],
                                      rb.u[1], aux.medium);
                } else {
                    bs = refract_sample(ld3(s.refractAlbedo + 3 * id), s.refractMedium[id], s, wi,
                                        sf, aux.medium, rb.u[0]);
                }
                V3 prf = rf * bs.refl;
                prf = (bs.pdf == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : (prf / bs.pdf);
                const float avg = dot(prf, v3(0.333f, 0.333f, 0.333f));
                bool term = false;
                if (!specular && aux.depth > oRr) {
                    // TracerFunctions::RussianRoulette (TracerFunctions.cuh:320-331)
                    const float prob = fminf(fmaxf(avg, 0.005f), 1.0f);
                    if (ra.u[3] >= prob) term = true;
                    else prf = prf * (1.0f / prob);
                }
                if ((!term || specular) && nonzero(prf)) {
                    emitPath = true;
                    pathO = make_float4(bs.pos.x, bs.pos.y, bs.pos.z, 0.0f);
                    pathD = make_float4(bs.dir.x, bs.dir.y, bs.dir.z, kFltMax);
                    pathAux = aux;
                    pathAux.medium = static_cast<uint16_t>(bs.medium);
                    pathAux.rf[0] = prf.x;
                    pathAux.rf[1] = prf.y;
                    pathAux.rf[2] = prf.z;
                    pathAux.type = specular ? kSpecPathRay : kPathRay;
                    pathAux.prevPDF = bs.pdf;
                    pathAux.depth = static_cast<uint8_t>(aux.depth + 1);
                    if (A.opt.wfpg && A.chain.nodeN) {
                        const size_t at = size_t(aux.depth) * A.chain.paths + aux.sample;
                        A.chain.nodeD[at] = make_float4(bs.dir.x, bs.dir.y, bs.dir.z, bs.pdf);
                        A.chain.nodeT[at] = make_float4(prf.x, prf.y, prf.z, __uint_as_float(frame));
                    }
                }
                }  // gen
            }
        }
        // warp-aggregated compaction of the outputs into the next wavefront
        const uint32_t bN = __ballot_sync(0xFFFFFFFFu, emitNee);
        const uint32_t bP = __ballot_sync(0xFFFFFFFFu, emitPath);
        const uint32_t tot = __popc(bN) + __popc(bP);
        if (tot == 0) continue;
        uint32_t wbase = 0;
        if (lane == 0) wbase = atomicAdd(A.outCount, tot);
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (emitNee) {
            const uint32_t o = wbase + __popc(bN & ltMask);
            A.outO[o] = neeO;
            A.outD[o] = neeD;
            A.outAux[o] = neeAux;
        }
        if (emitPath) {
            const uint32_t o = wbase + __popc(bN) + __popc(bP & ltMask);
            A.outO[o] = pathO;
            A.outD[o] = pathD;
            A.outAux[o] = pathAux;
        }
    }
}

__global__ void __launch_bounds__(256) k_resolve(const float4* __restrict__ samples,
                                                 uint32_t width, uint32_t height, uint32_t sp,
                                                 float4* __restrict__ image) {
    const uint32_t SW = width * sp;
    const float inv = 1.0f / static_cast<float>(sp * sp);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < width * height;
         p += gridDim.x * blockDim.x) {
        const uint32_t px = p % width, py = p / width;
        float r = 0.0f, g = 0.0f, b = 0.0f;
        for (uint32_t j = 0; j < sp; j++)
            for (uint32_t i = 0; i < sp; i++) {
                float4 v = samples[(py * sp + j) * SW + (px * sp + i)];
                r += v.x;
                g += v.y;
                b += v.z;
            }
        float4 acc = image[p];
        image[p] = make_float4(acc.x + r * inv, acc.y + g * inv, acc.z + b * inv, acc.w + 1.0f);
    }
}

__global__ void k_frame_advance(uint32_t* frame) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *frame += 1u;
}

inline uint32_t grid_for(uint32_t n, uint32_t block, uint32_t cap) {
    uint32_t g = (n + block - 1) / block;
    return g < cap ? (g ? g : 1) : cap;
}


// Largest j < n with base[j] <= g (base ascending, base[0] = 0).
__device__ __forceinline__ uint32_t job_of(const uint32_t* base, uint32_t n, uint32_t g) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (base[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Camera rays of every job of a pool iteration: slot g belongs to the job
// whose sample range holds it, and is that job's sample g - sampleBase.
__global__ void __launch_bounds__(256) k_pool_camera(const PoolHeader* __restrict__ hdr,
                                                     const JobDev* __restrict__ jobs,
                                                     float4* __restrict__ rayO,
                                                     float4* __restrict__ rayD,
                                                     RayAux* __restrict__ aux,
                                                     float4* __restrict__ samples,
                                                     uint32_t* __restrict__ count) {
    __shared__ uint32_t sBase[kPoolMaxJobs];
    const uint32_t nj = hdr->jobs, total = hdr->samples;
    for (uint32_t j = threadIdx.x; j < nj; j += blockDim.x) sBase[j] = jobs[j].sampleBase;
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = total;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += gridDim.x * blockDim.x) {
        const uint32_t j = job_of(sBase, nj, g);
        const JobDev& J = jobs[j];
        const uint32_t li = g - J.sampleBase;
        const uint32_t SW = J.width * J.samples, SH = J.height * J.samples;
        // slot -> sample of the job in 4 x 8 tiles, as k_camera lays them out
        uint32_t sx, sy;
        if ((SW % 4u == 0u) && (SH % 8u == 0u)) {
            const uint32_t tile = li >> 5, w = li & 31u, tilesX = SW / 4u;
            sx = (tile % tilesX) * 4u + (w & 3u);
            sy = (tile / tilesX) * 8u + (w >> 2);
        } else {
            sx = li % SW;
            sy = li / SW;
        }
        const uint32_t sid = sy * SW + sx;
        const uint32_t gs = J.sampleBase + sid;  // the sample this slot renders
        const Rand4 rc = philox_uniform4(sid, J.frame, kTagCamera, 0u, J.seedLo, J.seedHi);
        camera_ray(J.cam, sx, sy, SW, SH, rc, rayO[g], rayD[g]);
        RayAux a;
        a.rf[0] = a.rf[1] = a.rf[2] = 1.0f;
        a.sample = gs;
        a.endpoint = kInvalid;
        a.medium = static_cast<uint16_t>(J.sc.baseMedium);
        a.depth = 0;
        a.type = kCameraRay;
        a.prevPDF = __int_as_float(0x7fc00000);
        a.pad = j;
        aux[g] = a;
        samples[gs] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// k_resolve over every job's image: per pixel the mean of its s*s samples
// is added to the job's image, the frame counted in .w.
__global__ void __launch_bounds__(256) k_pool_resolve(const PoolHeader* __restrict__ hdr,
                                                      const JobDev* __restrict__ jobs,
                                                      const float4* __restrict__ samples) {
    __shared__ uint32_t sBase[kPoolMaxJobs];
    const uint32_t nj = hdr->jobs, total = hdr->pixels;
    for (uint32_t j = threadIdx.x; j < nj; j += blockDim.x) sBase[j] = jobs[j].pixelBase;
    __syncthreads();
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += gridDim.x * blockDim.x) {
        const JobDev& J = jobs[job_of(sBase, nj, g)];
        const uint32_t p = g - J.pixelBase;
        const uint32_t sp = J.samples, SW = J.width * sp;
        const uint32_t px = p % J.width, py = p / J.width;
        const float inv = 1.0f / static_cast<float>(sp * sp);
        const float4* base = samples + J.sampleBase;
        float r = 0.0f, gg = 0.0f, b = 0.0f;
        for (uint32_t j = 0; j < sp; j++)
            for (uint32_t i = 0; i < sp; i++) {
                const float4 v = base[(py * sp + j) * SW + (px * sp + i)];
                r += v.x;
                gg += v.y;
                b += v.z;
            }
        const float4 acc = J.image[p];
        J.image[p] = make_float4(acc.x + r * inv, acc.y + gg * inv, acc.z + b * inv, acc.w + 1.0f);
    }
}

}  // namespace

int camera_generate(const CameraDev* cam, const PathOptions& opt, uint32_t baseMedium,
                    float4* rayO, float4* rayD, RayAux* aux, float4* samples, uint32_t* count,
                    const PathChain& chain, float2* imgCoords, cudaStream_t stream) {
    const uint32_t total = opt.width * opt.samples * opt.height * opt.samples;
    k_camera<<<grid_for(total, 256, 148 * 16), 256, 0, stream>>>(cam, opt, baseMedium, rayO, rayD,
                                                                aux, samples, count, total, chain,
                                                                imgCoords);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int dense_keys(const uint32_t* hitKey, const uint32_t* dCount, uint32_t maxCount, uint32_t idBits,
               uint32_t* dense, const PortionTable& table, cudaStream_t stream,
               unsigned long long* rayTotal, uint32_t* nextCount) {
    k_dense_keys<<<grid_for(maxCount, 256, 148 * 8), 256, 0, stream>>>(hitKey, dCount, idBits, dense,
                                                                      table, rayTotal, nextCount);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int find_portions(const uint32_t* sortedDense, const uint32_t* dCount, uint32_t maxCount,
                  uint32_t idBits, const PortionTable& table, cudaStream_t stream) {
    k_portions<<<grid_for(maxCount, 256, 148 * 8), 256, 0, stream>>>(sortedDense, dCount, idBits,
                                                                    table);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int shade(const SceneDev& sc, const float4* rayO, const float4* rayD, const RayAux* aux,
          const HitIn& hit, const uint32_t* sortedIds, const uint32_t* nonNull,
          const uint32_t* count, uint32_t maxCount, float4* samples, const PathOptions& opt,
          bool gen, float4* outO, float4* outD, RayAux* outAux, uint32_t* outCount,
          const PathChain& chain, const uint2* guide, cudaStream_t stream) {
    ShadeArgs a{sc,   rayO,    rayD, aux,  hit,  sortedIds, nonNull, count, samples,
                opt,  gen ? 1 : 0, outO, outD, outAux, outCount, chain, guide, nullptr};
    k_shade<false><<<grid_for(maxCount, 128, 148 * 16), 128, 0, stream>>>(a);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int resolve(const float4* samples, uint32_t width, uint32_t height, uint32_t sp, float4* image,
            cudaStream_t stream) {
    k_resolve<<<grid_for(width * height, 256, 148 * 8), 256, 0, stream>>>(samples, width, height,
                                                                         sp, image);
    MRB_CUDA(cudaGetLastError());
    return 0;
}


int frame_advance(uint32_t* frame, cudaStream_t stream) {
    k_frame_advance<<<1, 32, 0, stream>>>(frame);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int pool_camera(const PoolHeader* hdr, const JobDev* jobs, uint32_t maxSamples, float4* rayO,
                float4* rayD, RayAux* aux, float4* samples, uint32_t* count, cudaStream_t stream) {
    k_pool_camera<<<grid_for(maxSamples, 256, 148 * 16), 256, 0, stream>>>(hdr, jobs, rayO, rayD,
                                                                          aux, samples, count);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int pool_resolve(const PoolHeader* hdr, const JobDev* jobs, uint32_t maxPixels,
                 const float4* samples, cudaStream_t stream) {
    k_pool_resolve<<<grid_for(maxPixels, 256, 148 * 8), 256, 0, stream>>>(hdr, jobs, samples);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int shade_jobs(const JobDev* jobs, const float4* rayO, const float4* rayD, const RayAux* aux,
               const HitIn& hit, const uint32_t* sortedIds, const uint32_t* nonNull,
               uint32_t maxCount, float4* samples, float4* outO, float4* outD, RayAux* outAux,
               uint32_t* outCount, cudaStream_t stream) {
    PathOptions opt{};
    ShadeArgs a{SceneDev{}, rayO, rayD, aux, hit, sortedIds, nonNull, nonNull, samples, opt, 1,
                outO, outD, outAux, outCount, PathChain{}, nullptr, jobs};
    k_shade<true><<<grid_for(maxCount, 128, 148 * 16), 128, 0, stream>>>(a);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
