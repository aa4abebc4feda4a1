// Host runtime and C ABI of the meturay_b200 core.
//
// Objects mirror the MRay plugin surfaces on the hot path:
//   mrb_system  <- TracerSystemI / TracerSystemCUDA (TracerSystemCUDA.cpp:19-100)
//   mrb_scene   <- GPUSceneI with one triangle primitive group, its material
//                  groups, primitive lights and the "LBVH" accelerator group
//   mrb_tracer  <- GPUTracerI "PathTracer" (PathTracer.cu:144-326) and
//                  "WFPGTracer" (WFPGTracer.cu:435-1833): the same wavefront
//                  with a per-depth guiding step and a per-frame radiance
//                  deposit into the tracer's own voxel octree
// The wavefront loop keeps every count on the device: trace -> partition ->
// shade per depth with no host synchronisation, and a whole frame can be
// captured once as a CUDA graph and replayed.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <array>
#include <vector>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "lbvh.cuh"
#include "shade.cuh"
#include "sort.cuh"
#include "trace.cuh"
#include "wide.cuh"
#include "svo.cuh"
#include "guide.cuh"
#include "recon.cuh"
#include "io.cuh"
#include "learned.cuh"
#include "objects.cuh"
#include "ploc.cuh"

namespace mrb {

static thread_local std::string g_error;
void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

namespace {


// ---------------------------------------------------------------------------
// Host-side tangent space, as the triangle loader does it
// (GPUPrimitiveTriangle.cpp:160-320, Triangle.h:73-111, Quaternion.hpp:372-480)
// ---------------------------------------------------------------------------
struct H3 {
    float v[3];
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
inline H3 h3(float a, float b, float c) { return H3{{a, b, c}}; }
inline H3 hsub(H3 a, H3 b) { return h3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline H3 hadd(H3 a, H3 b) { return h3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline H3 hmul(H3 a, float s) { return h3(a[0] * s, a[1] * s, a[2] * s); }
inline float hdot(H3 a, H3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline H3 hcross(H3 a, H3 b) {
    return h3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline H3 hnorm(H3 a) {
    float inv = 1.0f / std::sqrt(hdot(a, a));
    return hmul(a, inv);
}
inline bool hnan(H3 a) { return std::isnan(a[0]) || std::isnan(a[1]) || std::isnan(a[2]); }
inline H3 orthogonal(H3 v) {  // OrthogonalVector (Vector.hpp:877-886)
    if (std::fabs(v[0]) > std::fabs(v[1])) {
        float s = std::sqrt(v[0] * v[0] + v[2] * v[2]);
        return h3(-v[2] / s, 0.0f / s, v[0] / s);
    }
    float s = std::sqrt(v[1] * v[1] + v[2] * v[2]);
    return h3(0.0f / s, v[2] / s, -v[1] / s);
}
inline H3 calc_tangent(H3 p0, H3 p1, H3 p2, const float* uv0, const float* uv1,
                       const float* uv2) {
    H3 vec0 = hsub(p1, p0), vec1 = hsub(p2, p0);
    float du0x = uv1[0] - uv0[0], du0y = uv1[1] - uv0[1];
    float du1x = uv2[0] - uv0[0], du1y = uv2[1] - uv0[1];
    float t = (du0x * du1y - du1x * du0y);
    if (t == 0.0f) return h3(NAN, NAN, NAN);
    float r = 1.0f / t;
    H3 a = hmul(vec0, du1y), b = hmul(vec1, du0y);
    H3 tan = hmul(hsub(a, b), r);
    if (t < 0) tan = h3(-tan[0], -tan[1], -tan[2]);
    return tan;
}
inline void space_quat(H3 xIn, H3 y, H3 z, float q[4]) {
    H3 x = xIn;
    H3 c = hsub(hcross(x, y), z);
    if (std::fabs(c[0]) > 0.1f && std::fabs(c[1]) > 0.1f && std::fabs(c[2]) > 0.1f)
        x = h3(-x[0], -x[1], -x[2]);
    float t;
    float w, qx, qy, qz;
    if (z[2] < 0) {
        if (x[0] > y[1]) {
            t = 1 + x[0] - y[1] - z[2];
            w = y[2] - z[1]; qx = t; qy = x[1] + y[0]; qz = z[0] + x[2];
        } else {
            t = 1 - x[0] + y[1] - z[2];
            w = z[0] - x[2]; qx = x[1] + y[0]; qy = t; qz = y[2] + z[1];
        }
    } else {
        if (x[0] < -y[1]) {
            t = 1 - x[0] - y[1] + z[2];
            w = x[1] - y[0]; qx = z[0] + x[2]; qy = y[2] + z[1]; qz = t;
        } else {
            t = 1 + x[0] + y[1] + z[2];
            w = t; qx = y[2] - z[1]; qy = z[0] - x[2]; qz = x[1] - y[0];
        }
    }
    float s = 0.5f / std::sqrt(t);
    w *= s; qx *= s; qy *= s; qz *= s;
    float inv = 1.0f / std::sqrt(w * w + qx * qx + qy * qy + qz * qz);
    q[0] = w * inv;
    q[1] = -(qx * inv);
    q[2] = -(qy * inv);
    q[3] = -(qz * inv);
}

void build_tbn(const mrb_scene_desc& d, std::vector<float>& tbn) {
    const uint32_t V = d.vertex_count, T = d.triangle_count;
    std::vector<H3> tangents(V, h3(0, 0, 0));
    static const float kDefUv[3][2] = {{0.f, 0.f}, {1.f, 0.f}, {0.f, 1.f}};
    auto P = [&](uint32_t v) { return h3(d.positions[3 * v], d.positions[3 * v + 1], d.positions[3 * v + 2]); };
    auto N = [&](uint32_t v) { return h3(d.normals[3 * v], d.normals[3 * v + 1], d.normals[3 * v + 2]); };
    for (uint32_t t = 0; t < T; t++) {
        uint32_t ix[3] = {d.indices[3 * t], d.indices[3 * t + 1], d.indices[3 * t + 2]};
        const float* uv[3];
        for (int k = 0; k < 3; k++) uv[k] = d.uvs ? d.uvs + 2 * ix[k] : kDefUv[k];
        for (int k = 0; k < 3; k++) {
            int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
            H3 tk = calc_tangent(P(ix[k]), P(ix[k1]), P(ix[k2]), uv[k], uv[k1], uv[k2]);
            if (hnan(tk)) tk = orthogonal(N(ix[k]));
            tangents[ix[k]] = hadd(tangents[ix[k]], tk);
        }
    }
    tbn.resize(size_t(V) * 4);
    for (uint32_t v = 0; v < V; v++) {
        H3 n = N(v), t = tangents[v];
        if (hdot(t, t) < 1.0e-5f) t = orthogonal(n);
        t = hnorm(t);
        H3 tn = hnorm(hsub(t, hmul(n, hdot(n, t))));
        H3 b = hcross(n, tn);
        space_quat(tn, b, n, &tbn[4 * size_t(v)]);
    }
}

inline uint32_t bits_for(uint32_t maxId) {
    uint32_t b = 1;
    while (b < 24 && (1u << b) <= maxId) b++;
    return b;
}

}  // namespace
}  // namespace mrb

using namespace mrb;


struct mrb_tracer {
    mrb_system* sys = nullptr;
    mrb_scene* scene = nullptr;
    cudaStream_t stream = nullptr;
    // options (PathTracer.h:17-33 defaults)
    uint32_t samples = 1, maxDepth = 5, nee = 1, rrStart = 3, mis = 0;
    uint64_t seed = 1;
    uint32_t width = 0, height = 0;
    // pinned staging copies of the camera frame, used in turn; camEv[i] marks
    // the upload that last read slot i
    static constexpr int kCamSlots = 4;
    CameraDev* hostCam = nullptr;
    cudaEvent_t camEv[kCamSlots] = {};
    bool camEvUsed[kCamSlots] = {};
    int camSlot = 0;
    DBuf devCam;                   // the frame the camera kernel reads
    bool camSet = false;
    uint32_t launchesPerFrame = 0;
    // wavefront memory
    uint32_t maxRays = 0;
    DBuf rayO[2], rayD[2], aux[2], count, hitKey, hitPrim, hitT, hitBary, dense, sortedIds,
        portion, samplesBuf, image, counters, frameWord, errorFlags, sortTemp;
    size_t sortTempBytes = 0;
    // stepwise GPUTracerI state
    uint32_t depth = 0;
    bool working = false;
    uint32_t frames = 0;
    uint32_t frameStart = 0;  // "Frame": RNG iteration of the next frame
    // WFPG tracer (WFPGTracer.h:58-96 defaults)
    bool wfpg = false;
    uint32_t octreeLevel = 10, minRayBinLevel = 5, binRayCount = 512, productPG = 1, purePG = 0,
             skipPG = 0, guideBounce = 512, omitDirect = 0;
    float misRatio = 0.5f, filterAlpha = 1.0f;
    // octree files: "InitialSVO" replaces the build with a dump; with
    // "PGDumpDataStruct" the octree is dumped after the frames numbered
    // interval^0, interval^1, ... ("PGDataStructDumpIntervalExp") to
    // "<frame>_<PGDataStructDumpName>" (WFPGTracer.cu:1289-1309,1733-1745)
    std::string initialSvo, dumpName = "wfpg_svo";
    // learned guiding: the network's mixture replaces the octree sampler
    // after learnedWarmup frames; it trains every frame from the path chains
    uint32_t learned = 0, learnedWarmup = 16, learnedSteps = 4, learnedSamples = 1u << 16;
    uint32_t learnedProduct = 1;
    uint32_t learnedWarmupOctree = 1;  // 0: the BxDF alone samples the warm-up frames
    uint64_t learnedSeed = 1;
    float learnedRate = 1.0e-2f, learnedWeightMax = 0.0f;
    // inference weights: an exponential moving average of the trained ones
    // with this decay per frame (0: the trained weights themselves)
    float learnedEma = 0.0f;
    DBuf lEma, lEmaBackup;
    mrb_mlp* net = nullptr;
    DBuf chainN, chainD, chainT, lTrainX, lTrainT, lCount, lOffset, lScan, lSteps,
        lLoss, netBackup;
    // The network trains on a side stream while the frame renders: frame f
    // trains on frame f-1's samples and renders with the weights as they
    // were at the start of frame f (lFwd: fp32 parameters, then the bf16
    // weight image; refreshed after the join).
    DBuf lFwd;
    cudaStream_t trainStream = nullptr;
    cudaEvent_t trainFork = nullptr, trainJoin = nullptr;
    bool trainPending = false;  // forked in the current frame, not yet joined
    bool learnedReset = true;   // step counts and forward image to (re)initialise
    uint32_t dumpEnabled = 0, dumpInterval = 2, iterationCount = 0, treeDumpCount = 0;
    bool svoReady = false;
    SvoParams svoP{};
    SvoResult svo;
    DBuf chainA, chainB, chainNee, chainPath, binKey, binRid, heads, headScan, binBegin, binEnd,
        guideSort, guideScan, guideBuf, payloadBackup;
    DBuf imageBackup;  // image and ray counters around the eager frame of a capture
    // asynchronous image read-back: device snapshot, copied on copyStream
    DBuf imageStage;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t snapDone = nullptr, copyDone = nullptr;
    bool copyPending = false;
    size_t guideSortBytes = 0;
    uint32_t chainPaths = 0, chainLevels = 0;
    // reconstruction filter (AttachReconFilter); image coordinates per sample
    bool hasFilter = false;
    ReconFilterDev filter{};
    DBuf imgCoords;
    // graph
    cudaGraphExec_t graph = nullptr;
    bool graphDirty = true;
    uint32_t graphEpoch = 0;  // scene traceEpoch the graph was captured for
    // 8-wide traversal kernel per depth, chosen on this tracer's own rays:
    // the eager frame before a capture times every kernel at every depth
    bool orderTune = false;
    uint32_t orderEpoch = ~0u;  // scene traceEpoch depthOrder was tuned for
    std::vector<int> depthOrder;
    std::vector<std::array<float, kTunedOrders>> depthMs;
    ~mrb_tracer() {
        if (trainStream) cudaStreamSynchronize(trainStream);
        if (copyStream) cudaStreamSynchronize(copyStream);
        if (net) mrb_mlp_destroy(net);
        if (svoReady) svo_free(svo);
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamSynchronize(stream);
        if (hostCam) cudaFreeHost(hostCam);
        for (cudaEvent_t ev : camEv)
            if (ev) cudaEventDestroy(ev);
        if (trainFork) cudaEventDestroy(trainFork);
        if (trainJoin) cudaEventDestroy(trainJoin);
        if (trainStream) cudaStreamDestroy(trainStream);
        if (snapDone) cudaEventDestroy(snapDone);
        if (copyDone) cudaEventDestroy(copyDone);
        if (copyStream) cudaStreamDestroy(copyStream);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int ensure_buffers(mrb_tracer* t) {
    if (!t->width || !t->height) {
        set_error("tracer: resolution not set");
        return MRB_E_STATE;
    }
    const uint64_t paths = uint64_t(t->width) * t->samples * t->height * t->samples;
    if (paths == 0 || paths > (1ull << 29)) {
        set_error("tracer: %llu samples per iteration is out of range",
                  (unsigned long long)paths);
        return MRB_E_ARG;
    }
    const uint32_t maxRays = static_cast<uint32_t>(2 * paths);
    if (maxRays == t->maxRays && t->rayO[0].p) return 0;
    t->maxRays = maxRays;
    int r = 0;
    for (int i = 0; i < 2; i++) {
        if ((r = t->rayO[i].alloc(size_t(maxRays) * 16))) return r;
        if ((r = t->rayD[i].alloc(size_t(maxRays) * 16))) return r;
        if ((r = t->aux[i].alloc(size_t(maxRays) * sizeof(RayAux)))) return r;
    }
    if ((r = t->count.alloc(2 * 4))) return r;
    if ((r = t->hitKey.alloc(size_t(maxRays) * 4))) return r;
    if ((r = t->hitPrim.alloc(size_t(maxRays) * 4))) return r;
    if ((r = t->hitT.alloc(size_t(maxRays) * 4))) return r;
    if ((r = t->hitBary.alloc(size_t(maxRays) * 8))) return r;
    if ((r = t->dense.alloc(size_t(maxRays) * 4))) return r;
    if ((r = t->sortedIds.alloc(size_t(maxRays) * 4))) return r;
    if ((r = t->portion.alloc(32 * 4))) return r;
    if ((r = t->samplesBuf.alloc(size_t(paths) * 16))) return r;
    if (t->hasFilter && (r = t->imgCoords.alloc(size_t(paths) * 8))) return r;
    if ((r = t->image.alloc(size_t(t->width) * t->height * 16))) return r;
    if ((r = t->counters.alloc(16))) return r;
    if ((r = t->frameWord.alloc(4))) return r;
    if ((r = t->errorFlags.alloc(16))) return r;
    t->sortTempBytes = radix_sort_temp_bytes(maxRays, 4, 0, 3 + 24);
    if ((r = t->sortTemp.alloc(t->sortTempBytes))) return r;
    if (t->wfpg) {
        const size_t levels = size_t(t->maxDepth) + 1;
        const size_t chain = levels * paths * 16;
        if ((r = t->chainA.alloc(chain)) || (r = t->chainB.alloc(chain)) ||
            (r = t->chainNee.alloc(chain)) || (r = t->chainPath.alloc(chain)) ||
            (r = t->binKey.alloc(size_t(maxRays) * 4)) || (r = t->binRid.alloc(size_t(maxRays) * 4)) ||
            (r = t->heads.alloc((size_t(maxRays) + 1) * 4)) ||
            (r = t->headScan.alloc((size_t(maxRays) + 1) * 4)) ||
            (r = t->binBegin.alloc(size_t(maxRays) * 4)) || (r = t->binEnd.alloc((size_t(maxRays) + 1) * 4)) ||
            (r = t->guideScan.alloc(guide_scan_temp_bytes(maxRays))) ||
            (r = t->guideBuf.alloc(size_t(maxRays) * 8)))
            return r;
        t->guideSortBytes = guide_sort_temp_bytes(maxRays);
        if ((r = t->guideSort.alloc(t->guideSortBytes))) return r;
        // frame stamps start out matching no frame
        MRB_CUDA(cudaMemsetAsync(t->chainA.p, 0xFF, chain, t->stream));
        t->chainPaths = static_cast<uint32_t>(paths);
        t->chainLevels = static_cast<uint32_t>(levels);
    }
    MRB_CUDA(cudaMemsetAsync(t->image.p, 0, t->image.bytes, t->stream));
    MRB_CUDA(cudaMemsetAsync(t->counters.p, 0, 16, t->stream));
    MRB_CUDA(cudaMemsetAsync(t->errorFlags.p, 0, 16, t->stream));
    // the sorts' give-up flags are read after every frame, also where a sort
    // has not run yet (the guide sort under SkipPG)
    MRB_CUDA(cudaMemsetAsync(radix_sort_error_flag(t->sortTemp.p, t->maxRays), 0, 4, t->stream));
    if (t->wfpg)
        MRB_CUDA(cudaMemsetAsync(radix_sort_error_flag(t->guideSort.p, t->maxRays), 0, 4,
                                 t->stream));
    MRB_CUDA(cudaMemcpyAsync(t->frameWord.p, &t->frameStart, 4, cudaMemcpyHostToDevice,
                             t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    t->graphDirty = true;
    return 0;
}

PathOptions path_options(const mrb_tracer* t) {
    PathOptions o{};
    o.width = t->width;
    o.height = t->height;
    o.samples = t->samples;
    o.maxDepth = t->maxDepth;
    o.rrStart = t->rrStart;
    o.nee = t->nee;
    o.mis = t->mis;
    o.seedLo = static_cast<uint32_t>(t->seed);
    o.seedHi = static_cast<uint32_t>(t->seed >> 32);
    o.frame = t->frameWord.as<uint32_t>();
    o.wfpg = t->wfpg ? 1 : 0;
    return o;
}

PathChain path_chain(const mrb_tracer* t) {
    PathChain c{};
    if (!t->wfpg) return c;
    c.nodeA = t->chainA.as<float4>();
    c.nodeB = t->chainB.as<float4>();
    c.contribNee = t->chainNee.as<float4>();
    c.contribPath = t->chainPath.as<float4>();
    c.paths = t->chainPaths;
    c.levels = t->chainLevels;
    if (t->learned) {
        c.nodeN = t->chainN.as<float4>();
        c.nodeD = t->chainD.as<float4>();
        c.nodeT = t->chainT.as<float4>();
    }
    return c;
}

// He-uniform initial weights from a seed (splitmix64 stream), zero biases;
// the padded entries stay zero.
std::vector<float> learned_init(uint64_t seed) {
    std::vector<float> p(kMlpParams, 0.0f);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    auto next = [&x]() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return static_cast<float>(z >> 40) * 0x1p-24f;
    };
    for (int l = 0; l < kMlpLayers; l++) {
        const int K = l == 0 ? kMlpIn : 64;
        const float lim = std::sqrt((l < kMlpLayers - 1 ? 6.0f : 3.0f) / float(K));
        float* w = p.data() + mlp_layer_offset(l);
        for (int i = 0; i < K; i++)
            for (int o = 0; o < 64; o++) {
                const float u = next();
                const bool frozen = (l == 0 && i >= kMlpFeatures) ||
                                    (l == kMlpLayers - 1 && o >= kMlpOut);
                w[i * 64 + o] = frozen ? 0.0f : (2.0f * u - 1.0f) * lim;
            }
    }
    return p;
}

LearnedScratch learned_scratch(const mrb_tracer* t) {
    LearnedScratch s{};
    s.trainX = t->lTrainX.as<float>();
    s.trainT = t->lTrainT.as<float>();
    s.pathCount = t->lCount.as<uint32_t>();
    s.pathOffset = t->lOffset.as<uint32_t>();
    s.scanTemp = t->lScan.p;
    s.stepCount = t->lSteps.as<uint32_t>();
    s.frameLoss = t->lLoss.as<float>();
    s.weightMax = t->learnedWeightMax;
    s.product = t->learnedProduct;
    s.steps = t->learnedSteps;
    s.capacity = t->learnedSamples / t->learnedSteps * t->learnedSteps;
    return s;
}

// The forward passes' copy of the network (parameters and weight image):
// the trained weights, or their moving average (advanced by one step when
// `step`, else taken as it stands).
int learned_refresh_forward(mrb_tracer* t, bool step = true) {
    const MlpDev m = mlp_dev(t->net);
    char* f = t->lFwd.as<char>();
    uint16_t* image = reinterpret_cast<uint16_t*>(f + size_t(kMlpParams) * 4);
    if (t->learnedEma > 0.0f) {
        if (step) {
            if (learned_ema(m.params, t->lEma.as<float>(), t->learnedEma,
                            reinterpret_cast<float*>(f), t->stream))
                return MRB_E_CUDA;
        } else {
            MRB_CUDA(cudaMemcpyAsync(f, t->lEma.p, size_t(kMlpParams) * 4,
                                     cudaMemcpyDeviceToDevice, t->stream));
        }
        return mlp_build_image(reinterpret_cast<const float*>(f), image, t->stream);
    }
    MRB_CUDA(cudaMemcpyAsync(f, m.params, size_t(kMlpParams) * 4, cudaMemcpyDeviceToDevice,
                             t->stream));
    MRB_CUDA(cudaMemcpyAsync(image, m.wImage, kMlpImageBytes, cudaMemcpyDeviceToDevice,
                             t->stream));
    return 0;
}

// Buffers and network of learned guiding (after ensure_buffers).
int ensure_learned(mrb_tracer* t) {
    if (!t->wfpg || !t->learned) return 0;
    const size_t chain = size_t(t->chainLevels) * t->chainPaths * 16;
    const uint32_t cap = t->learnedSamples / t->learnedSteps * t->learnedSteps;
    int r;
    if ((r = t->chainN.alloc(chain)) || (r = t->chainD.alloc(chain)) ||
        (r = t->chainT.alloc(chain)) ||
        (r = t->lTrainX.alloc(size_t(cap) * kMlpIn * 4)) ||
        (r = t->lTrainT.alloc(size_t(cap) * 16)) ||
        (r = t->lCount.alloc((size_t(t->chainPaths) + 1) * 4)) ||
        (r = t->lOffset.alloc((size_t(t->chainPaths) + 1) * 4)) ||
        (r = t->lScan.alloc(learned_scan_temp_bytes(t->chainPaths))) ||
        (r = t->lSteps.alloc(size_t(t->learnedSteps) * 4)) || (r = t->lLoss.alloc(16)) ||
        (r = t->netBackup.alloc(mlp_state_bytes())) || (r = t->lFwd.alloc(size_t(kMlpParams) * 4 + kMlpImageBytes)) ||
        (r = t->lEma.alloc(size_t(kMlpParams) * 4)) ||
        (r = t->lEmaBackup.alloc(size_t(kMlpParams) * 4)))
        return r;
    if (!t->trainStream) {
        MRB_CUDA(cudaStreamCreateWithFlags(&t->trainStream, cudaStreamNonBlocking));
        MRB_CUDA(cudaEventCreateWithFlags(&t->trainFork, cudaEventDisableTiming));
        MRB_CUDA(cudaEventCreateWithFlags(&t->trainJoin, cudaEventDisableTiming));
    }
    if (!t->net) {
        if ((r = mrb_mlp_create(t->sys, &t->net))) return r;
        const std::vector<float> p = learned_init(t->learnedSeed);
        if ((r = mrb_mlp_set_params(t->net, p.data()))) return r;
        t->learnedReset = true;
    }
    if (t->learnedReset) {
        // no samples collected yet: the first frame's steps train on nothing
        MRB_CUDA(cudaMemsetAsync(t->lSteps.p, 0, t->lSteps.bytes, t->stream));
        MRB_CUDA(cudaMemsetAsync(t->lLoss.p, 0, t->lLoss.bytes, t->stream));
        MRB_CUDA(cudaMemcpyAsync(t->lEma.p, mlp_dev(t->net).params, size_t(kMlpParams) * 4,
                                 cudaMemcpyDeviceToDevice, t->stream));
        if ((r = learned_refresh_forward(t, false))) return r;
        t->learnedReset = false;
    }
    return 0;
}

// The network's weights as the frame's forward passes read them.
MlpDev learned_forward_net(const mrb_tracer* t) {
    MlpDev m = mlp_dev(t->net);
    m.params = t->lFwd.as<float>();
    m.wImage = reinterpret_cast<const uint16_t*>(t->lFwd.as<char>() + size_t(kMlpParams) * 4);
    return m;
}

// Fork the frame's training onto the side stream (once per frame).
int learned_fork(mrb_tracer* t) {
    if (!t->wfpg || !t->learned || !t->net || t->trainPending) return 0;
    MRB_CUDA(cudaEventRecord(t->trainFork, t->stream));
    MRB_CUDA(cudaStreamWaitEvent(t->trainStream, t->trainFork, 0));
    int r = learned_train(t->net, learned_scratch(t), t->learnedRate, t->trainStream);
    if (r) return r;
    MRB_CUDA(cudaEventRecord(t->trainJoin, t->trainStream));
    t->trainPending = true;
    return 0;
}

// Join the training branch; the forward image takes the trained weights.
int learned_join(mrb_tracer* t) {
    if (!t->trainPending) return 0;
    MRB_CUDA(cudaStreamWaitEvent(t->stream, t->trainJoin, 0));
    t->trainPending = false;
    return learned_refresh_forward(t);
}

bool learned_active(const mrb_tracer* t) {
    return t->wfpg && t->learned && t->net && t->frames >= t->learnedWarmup;
}

// The octree guides (and learns) this frame: always without learned
// guiding; with it, during the warm-up if LearnedWarmupOctree is set.
bool octree_guides(const mrb_tracer* t) {
    if (!t->wfpg) return false;
    if (!t->learned || !t->net) return true;
    return !learned_active(t) && t->learnedWarmupOctree;
}

GuideOptions guide_options(const mrb_tracer* t) {
    GuideOptions g{};
    g.minBinLevel = std::min(t->octreeLevel, t->minRayBinLevel);
    g.binRayCount = t->binRayCount;
    g.purePG = t->purePG;
    g.product = t->productPG;
    g.misRatio = t->misRatio;
    // StaticGaussianFilter1D<11> (BlockTextureFilter.cuh:72-110): taps
    // exp(-t^2 / (2 alpha)) normalised to sum 1, evaluated in double
    double w[11], tot = 0.0;
    for (int i = 0; i < 11; i++) {
        const double x = double(i - 5);
        w[i] = std::exp(-(x * x) * 0.5 / double(t->filterAlpha));
        tot += w[i];
    }
    for (int i = 0; i < 11; i++) g.filter[i] = static_cast<float>(w[i] / tot);
    return g;
}

// The tracer's own octree: AnisoSVOctreeCPU::Constrcut at
// WFPGTracer::Initialize, resolution 2^OctreeLevel.
int ensure_svo(mrb_tracer* t) {
    if (!t->wfpg || t->svoReady) return 0;
    mrb_scene* sc = t->scene;
    float ext[8];
    MRB_CUDA(cudaMemcpyAsync(ext, sc->aExtent.p, 24, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    if (!t->initialSvo.empty()) {
        // Constrcut(data) (AnisoSVO.cu:1190-1413): the dump replaces the build
        FILE* f = std::fopen(t->initialSvo.c_str(), "rb");
        if (!f) {
            set_error("InitialSVO: cannot open %s", t->initialSvo.c_str());
            return MRB_E_ARG;
        }
        std::vector<uint8_t> data;
        uint8_t buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + got);
        std::fclose(f);
        int r = svo_load(data.data(), data.size(), t->svoP, t->svo, t->stream);
        if (r) return r;
        t->svoReady = true;
        t->graphDirty = true;
        return 0;
    }
    t->svoP = svo_params(ext, 1u << t->octreeLevel);
    SvoBuildIn in{sc->T, sc->dPos.as<float>(), sc->dIdx.as<uint32_t>(), sc->dKey.as<uint32_t>(),
                  sc->dLightRad.as<float>(), t->omitDirect};
    int r = svo_build(in, t->svoP, t->svo, t->stream);
    if (!r) r = svo_payload_finish(guide_dev(t->svo, t->svoP), t->svo, t->stream);
    if (r) {
        svo_free(t->svo);
        return r;
    }
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    t->svoReady = true;
    t->graphDirty = true;
    return 0;
}

PortionTable portion_table(const mrb_tracer* t) {
    uint32_t* p = t->portion.as<uint32_t>();
    return PortionTable{p, p + 8, p + 16};
}

// order: the 8-wide kernel, or -1 for the scene's.
int trace_dispatch(const mrb_scene* sc, const float4* rayO, const float4* rayD,
                   const uint32_t* dCount, uint32_t maxCount, const HitOut& ho, uint32_t* err,
                   cudaStream_t st, unsigned long long* counters = nullptr, int order = -1) {
    if (sc->traversal == 1 && sc->T > 1) {
        // orders kWideOrders.. run the same kernels over the alternate layout
        if (order >= kWideOrders && sc->wAltNodeCount)
            return trace_closest_wide(sc->wideAlt(), rayO, rayD, dCount, maxCount, ho, err, st,
                                      counters, order - kWideOrders);
        return trace_closest_wide(sc->wide(), rayO, rayD, dCount, maxCount, ho, err, st, counters,
                                  order >= 0 ? order % kWideOrders : sc->wideOrder);
    }
    return trace_closest(sc->accel(), rayO, rayD, dCount, maxCount, ho, err, st, counters);
}

int step_camera(mrb_tracer* t) {
    uint32_t* cnt = t->count.as<uint32_t>();
    int r = learned_fork(t);
    if (r) return r;
    return camera_generate(t->devCam.as<CameraDev>(), path_options(t), t->scene->baseMedium,
                           t->rayO[0].as<float4>(),
                           t->rayD[0].as<float4>(), t->aux[0].as<RayAux>(),
                           t->samplesBuf.as<float4>(), cnt, path_chain(t),
                           t->hasFilter ? t->imgCoords.as<float2>() : nullptr, t->stream);
}

// Stage slots of a profiled frame (stage_ms of mrb_tracer_profile_stages).
enum Stage : int {
    kStCamera = 0, kStTrace, kStPartition, kStShade, kStResolve,
    kStGuideClear, kStGuideBin, kStGuideSort, kStGuideKernel,
    kStDeposit, kStNormalize, kStLearned, kStageCount
};

struct StageTimer {
    cudaEvent_t ev[24] = {};
    float ms[kStageCount] = {};
};

// Every 8-wide traversal kernel run over the rays of buffer `cur` of depth
// d, over the scene's layout and, where the scene keeps one, its alternate
// layout (twice each, the faster pass kept: the first launch of a kernel may
// load its module), into t->depthMs[d] (entries kWideOrders.. for the
// alternate; 1e30 where there is none).  Every pass writes the same closest hits
// but for ties; the frame's own trace follows and overwrites them.
int time_wide_orders(mrb_tracer* t, int cur, const HitOut& ho, uint32_t d) {
    const mrb_scene* sc = t->scene;
    if (d >= t->depthMs.size()) return 0;
    cudaEvent_t e[2];
    MRB_CUDA(cudaEventCreate(&e[0]));
    MRB_CUDA(cudaEventCreate(&e[1]));
    std::array<float, kTunedOrders> best;
    best.fill(1e30f);
    const int orders = sc->wAltNodeCount ? kTunedOrders : kWideOrders;
    int r = 0;
    for (int rep = 0; rep < 2 && !r; rep++)
        for (int o = 0; o < orders && !r; o++) {
            cudaEventRecord(e[0], t->stream);
            r = trace_closest_wide(o < kWideOrders ? sc->wide() : sc->wideAlt(),
                                   t->rayO[cur].as<float4>(), t->rayD[cur].as<float4>(),
                                   t->count.as<uint32_t>() + cur, t->maxRays, ho,
                                   t->errorFlags.as<uint32_t>(), t->stream, nullptr,
                                   o % kWideOrders);
            cudaEventRecord(e[1], t->stream);
            if (!r && cudaEventSynchronize(e[1]) == cudaSuccess) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e[0], e[1]);
                best[o] = std::min(best[o], ms);
            }
        }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    if (r) return r;
    MRB_CUDA(cudaGetLastError());
    t->depthMs[d] = best;
    return 0;
}

// The traversal kernel of depth d: the tracer's own choice where it tuned
// one for the scene's current traversal, else the scene's.
int depth_order(const mrb_tracer* t, uint32_t d) {
    if (!t->orderTune && t->orderEpoch == t->scene->traceEpoch && d < t->depthOrder.size())
        return t->depthOrder[d];
    return -1;
}

// One Render() step: HitRays -> PartitionRaysWRTWork -> WorkRays
// (PathTracer.cu:144-291) for the rays of buffer `cur`.  With a timer the
// stages are bracketed by events and the traversal is repeated once in its
// counting form (outside the timed interval) for the work figures.
int step_depth(mrb_tracer* t, uint32_t d, StageTimer* tm = nullptr,
               unsigned long long* workCounters = nullptr) {
    mrb_scene* sc = t->scene;
    const int cur = d & 1, nxt = cur ^ 1;
    uint32_t* cnt = t->count.as<uint32_t>();
    HitOut ho{t->hitKey.as<uint32_t>(), t->hitPrim.as<uint32_t>(), t->hitT.as<float>(),
              t->hitBary.as<float2>()};
    int r;
    auto mark = [&](int i) -> int {
        if (tm) MRB_CUDA(cudaEventRecord(tm->ev[i], t->stream));
        return 0;
    };
    auto lap = [&](int stage, int i0) -> int {
        if (!tm) return 0;
        MRB_CUDA(cudaEventSynchronize(tm->ev[i0 + 1]));
        float ms = 0.f;
        MRB_CUDA(cudaEventElapsedTime(&ms, tm->ev[i0], tm->ev[i0 + 1]));
        tm->ms[stage] += ms;
        return 0;
    };
    if (t->orderTune && (r = time_wide_orders(t, cur, ho, d))) return r;
    const int order = depth_order(t, d);
    if (mark(0)) return MRB_E_CUDA;
    if ((r = trace_dispatch(sc, t->rayO[cur].as<float4>(), t->rayD[cur].as<float4>(), cnt + cur,
                            t->maxRays, ho, t->errorFlags.as<uint32_t>(), t->stream, nullptr,
                            order)))
        return r;
    if (mark(1) || lap(1, 0)) return MRB_E_CUDA;
    if (workCounters) {
        if ((r = trace_dispatch(sc, t->rayO[cur].as<float4>(), t->rayD[cur].as<float4>(),
                                cnt + cur, t->maxRays, ho, t->errorFlags.as<uint32_t>(), t->stream,
                                workCounters, order)))
            return r;
    }
    // the learned sampler skips the last depth, whose guide words no ray
    // reads (the octree guider keeps the reference's schedule)
    const bool guideNow = t->wfpg && !t->skipPG && d < t->guideBounce &&
                          (learned_active(t) ? d + 1 < t->maxDepth : octree_guides(t));
    if (guideNow) {
        GuideWave gw{t->rayO[cur].as<float4>(), t->rayD[cur].as<float4>(), t->aux[cur].as<RayAux>(),
                     HitIn{ho.key, ho.prim, ho.t, ho.bary}, cnt + cur, t->maxRays};
        GuideScratch gs{t->binKey.as<uint32_t>(), t->binRid.as<uint32_t>(), t->heads.as<uint32_t>(),
                        t->headScan.as<uint32_t>(), t->binBegin.as<uint32_t>(),
                        t->binEnd.as<uint32_t>(), t->guideSort.p, t->guideSortBytes,
                        t->guideScan.p, t->guideBuf.as<uint2>(), t->binEnd.as<uint32_t>() + t->maxRays};
        cudaEvent_t* gm = tm ? &tm->ev[16] : nullptr;
        if (learned_active(t)) {
            if (mark(16)) return MRB_E_CUDA;
            r = learned_guide_wavefront(sc->dev(), guide_dev(t->svo, t->svoP), gw,
                                        learned_forward_net(t),
                                        learned_scratch(t), t->misRatio, path_options(t), d,
                                        t->guideBuf.as<uint2>(), t->stream);
            if (r || mark(17) || lap(kStGuideKernel, 16)) return r ? r : MRB_E_CUDA;
        } else {
            r = guide_wavefront(sc->dev(), guide_dev(t->svo, t->svoP), t->svo, gw, gs,
                                guide_options(t), path_options(t), d, d, t->stream, gm);
            if (r) return r;
            if (tm) {
                const int st[4] = {kStGuideClear, kStGuideBin, kStGuideSort, kStGuideKernel};
                MRB_CUDA(cudaEventSynchronize(gm[4]));
                for (int i = 0; i < 4; i++) {
                    float ms = 0.f;
                    MRB_CUDA(cudaEventElapsedTime(&ms, gm[i], gm[i + 1]));
                    tm->ms[st[i]] += ms;
                }
            }
        }
    }
    if (mark(2)) return MRB_E_CUDA;
    PortionTable pt = portion_table(t);
    // also adds this wavefront to the traced-ray total and clears the next
    // wavefront's counter
    if ((r = dense_keys(ho.key, cnt + cur, t->maxRays, sc->idBits, t->dense.as<uint32_t>(), pt,
                        t->stream, t->counters.as<unsigned long long>(), cnt + nxt)))
        return r;
    if ((r = radix_sort_pairs<uint32_t>(t->dense.as<uint32_t>(), t->sortedIds.as<uint32_t>(),
                                        cnt + cur, t->maxRays, 0, 3 + int(sc->idBits), true,
                                        t->sortTemp.p, t->sortTempBytes, t->stream, true)))
        return r;
    if ((r = find_portions(t->dense.as<uint32_t>(), cnt + cur, t->maxRays, sc->idBits, pt,
                           t->stream)))
        return r;
    if (mark(3) || lap(2, 2)) return MRB_E_CUDA;
    HitIn hi{ho.key, ho.prim, ho.t, ho.bary};
    const bool gen = (d + 1) < t->maxDepth;
    if (mark(4)) return MRB_E_CUDA;
    r = shade(sc->dev(), t->rayO[cur].as<float4>(), t->rayD[cur].as<float4>(),
              t->aux[cur].as<RayAux>(), hi, t->sortedIds.as<uint32_t>(), pt.nonNull, cnt + cur,
              t->maxRays,
              t->samplesBuf.as<float4>(), path_options(t), gen, t->rayO[nxt].as<float4>(),
              t->rayD[nxt].as<float4>(), t->aux[nxt].as<RayAux>(), cnt + nxt, path_chain(t),
              guideNow ? t->guideBuf.as<uint2>() : nullptr, t->stream);
    if (r) return r;
    if (mark(5) || lap(3, 4)) return MRB_E_CUDA;
    return 0;
}

int step_finalize(mrb_tracer* t, StageTimer* tm = nullptr) {
    int r;
    // with a timer: deposit | normalize and filter | learned join and
    // collect | reconstruction, bracketed by events 8..12
    auto mark = [&](int i) -> int {
        if (tm) MRB_CUDA(cudaEventRecord(tm->ev[8 + i], t->stream));
        return 0;
    };
    if (mark(0)) return MRB_E_CUDA;
    if (t->wfpg) {
        // WFPGTracer::Finalize: AccumulateRaidances + NormalizeAndFilterRadiance
        const GuideDev g = guide_dev(t->svo, t->svoP);
        // the octree learns while it guides; once the network guides, the
        // octree keeps its state as the fallback and skips the update
        if (octree_guides(t)) {
            if ((r = path_deposit(g, path_chain(t), t->frameWord.as<uint32_t>(), t->stream)))
                return r;
            if (mark(1)) return MRB_E_CUDA;
            if ((r = svo_normalize_filter(g, t->svo, t->stream))) return r;
        } else if (mark(1)) {
            return MRB_E_CUDA;
        }
        if (mark(2)) return MRB_E_CUDA;
        if ((r = learned_join(t))) return r;
        if (t->learned && t->net &&
            (r = learned_collect(g, path_chain(t), t->frameWord.as<uint32_t>(),
                                 learned_scratch(t), t->stream)))
            return r;
    } else if (mark(1) || mark(2)) {
        return MRB_E_CUDA;
    }
    if (mark(3)) return MRB_E_CUDA;
    if (t->hasFilter)
        r = recon_filter_grid(t->filter, t->samplesBuf.as<float4>(), t->imgCoords.as<float2>(),
                              t->width, t->height, t->samples, 1.0f, t->image.as<float4>(),
                              t->stream);
    else
        r = resolve(t->samplesBuf.as<float4>(), t->width, t->height, t->samples,
                    t->image.as<float4>(), t->stream);
    if (r) return r;
    if ((r = frame_advance(t->frameWord.as<uint32_t>(), t->stream))) return r;
    if (tm) {
        if (mark(4)) return MRB_E_CUDA;
        MRB_CUDA(cudaEventSynchronize(tm->ev[12]));
        const int st[4] = {kStDeposit, kStNormalize, kStLearned, kStResolve};
        for (int i = 0; i < 4; i++) {
            float ms = 0.f;
            MRB_CUDA(cudaEventElapsedTime(&ms, tm->ev[8 + i], tm->ev[9 + i]));
            tm->ms[st[i]] += ms;
        }
    }
    return 0;
}

int record_frame(mrb_tracer* t) {
    int r;
    if ((r = step_camera(t))) return r;
    for (uint32_t d = 0; d < t->maxDepth; d++)
        if ((r = step_depth(t, d))) return r;
    return step_finalize(t);
}

// Kernel launches recorded per frame (camera, per depth: trace, dense keys
// (with the ray count), histogram, histogram scan, onesweep passes
// (+copy-back), portions, shade; then resolve and frame advance).
uint32_t launches_per_frame(const mrb_tracer* t) {
    const uint32_t bits = 3 + t->scene->idBits;
    const uint32_t passes = (bits + 7) / 8;
    const uint32_t sort = 2 + passes + (passes & 1);
    uint32_t n = 1 + t->maxDepth * (2 + sort + 2) + 2;
    if (t->wfpg && t->svoReady) {
        // guiding per guided depth; deposit, leaf averages and the two
        // level filters per frame
        uint32_t guided = t->skipPG ? 0u : std::min(t->maxDepth, t->guideBounce);
        if (learned_active(t) && guided == t->maxDepth) guided--;
        if (!learned_active(t) && !octree_guides(t)) guided = 0;
        // learned guiding: one fused encode / forward / sample kernel per
        // guided depth, and the frame's training
        const uint32_t perDepth = learned_active(t) ? 1u
                                                    : guide_launches(t->svo, guide_options(t), t->maxRays);
        n += guided * perDepth + (octree_guides(t) ? 2 + 2 * t->svoP.depth : 0u);
        if (t->learned && t->net)
            n += learned_launches(t->learnedSteps) + (t->learnedEma > 0.0f ? 2u : 0u);
    }
    return n;
}

// WFPGTracer::Finalize's frame count and periodic octree dump
// (WFPGTracer.cu:1703,1733-1745): dumps after frames interval^k, k = 0, 1, ...
int wfpg_after_frame(mrb_tracer* t) {
    if (!t->wfpg) return 0;
    t->iterationCount++;
    if (!t->dumpEnabled) return 0;
    uint64_t due = 1;
    for (uint32_t k = 0; k < t->treeDumpCount && due <= 0xFFFFFFFFull; k++) due *= t->dumpInterval;
    if (due != t->iterationCount) return 0;
    std::vector<uint8_t> data;
    int r = svo_dump(t->svo, t->svoP, data, t->stream);
    if (r) return r;
    // "<frame>_<name>", the frame number in front of the file name itself
    const size_t slash = t->dumpName.find_last_of('/');
    const std::string dir = slash == std::string::npos ? "" : t->dumpName.substr(0, slash + 1);
    const std::string base = slash == std::string::npos ? t->dumpName : t->dumpName.substr(slash + 1);
    const std::string path = dir + std::to_string(t->iterationCount) + "_" + base;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(data.data(), 1, data.size(), f) != data.size()) {
        if (f) std::fclose(f);
        set_error("octree dump: cannot write %s", path.c_str());
        return MRB_E_ARG;
    }
    std::fclose(f);
    t->treeDumpCount++;
    return 0;
}

int check_device_errors(mrb_tracer* t) {
    uint32_t e[3] = {0, 0, 0};
    MRB_CUDA(cudaMemcpyAsync(e, t->errorFlags.p, 4, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaMemcpyAsync(e + 1, radix_sort_error_flag(t->sortTemp.p, t->maxRays), 4,
                             cudaMemcpyDeviceToHost, t->stream));
    if (t->wfpg && t->guideSort.p)
        MRB_CUDA(cudaMemcpyAsync(e + 2, radix_sort_error_flag(t->guideSort.p, t->maxRays), 4,
                                 cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    if (e[0] || e[1] || e[2]) {
        set_error("device-side limit hit (trace flag %u, sort flags %u %u)", e[0], e[1], e[2]);
        return MRB_E_DEVICE;
    }
    return 0;
}

int svo_copy(void* dst, const void* src, size_t bytes) {
    if (!dst || !bytes) return 0;
    if (!src) {  // arrays a loaded dump does not carry (leaf codes, light keys)
        std::memset(dst, 0, bytes);
        return 0;
    }
    MRB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return 0;
}

int export_svo(const SvoResult& v, uint64_t* nodes, uint32_t* leafParents, uint64_t* leafCodes,
               uint32_t* leafNormSpec, uint32_t* leafLight, uint32_t* levelOffsets) {
    if (svo_copy(nodes, v.nodes, size_t(v.nodeCount) * 8) ||
        svo_copy(leafParents, v.leafParents, size_t(v.leafCount) * 4) ||
        svo_copy(leafCodes, v.leafCodes, size_t(v.leafCount) * 8) ||
        svo_copy(leafNormSpec, v.leafNormSpec, size_t(v.leafCount) * 4) ||
        svo_copy(leafLight, v.leafLight, size_t(v.leafCount) * 4))
        return MRB_E_CUDA;
    if (levelOffsets)
        std::memcpy(levelOffsets, v.levelOffsets.data(), v.levelOffsets.size() * 4);
    return 0;
}

int export_payload(const SvoResult& v, uint32_t* nodeNormSpec, uint64_t* leafIrr,
                   uint32_t* leafCnt, uint32_t* leafAvg, uint32_t* nodeAvg) {
    const size_t U = v.leafCount, N = v.nodeCount;
    if (svo_copy(nodeNormSpec, v.nodeNormSpec, N * 4) || svo_copy(leafIrr, v.leafIrr, U * 16) ||
        svo_copy(leafCnt, v.leafCnt, U * 8) || svo_copy(leafAvg, v.leafAvg, U * 4) ||
        svo_copy(nodeAvg, v.nodeAvg, N * 4))
        return MRB_E_CUDA;
    return 0;
}

void svo_info(const SvoResult& v, const SvoParams& p, uint32_t* info, float* params) {
    if (info) {
        info[0] = v.voxelCount;
        info[1] = v.leafCount;
        info[2] = v.nodeCount;
        info[3] = p.depth;
        info[4] = p.res;
        info[5] = static_cast<uint32_t>(v.levelOffsets.size());
    }
    if (params) {
        for (int c = 0; c < 3; c++) {
            params[c] = p.lo[c];
            params[3 + c] = p.hi[c];
        }
        params[6] = p.leafVoxelSize;
    }
}

int set_device(mrb_system* s) {
    MRB_CUDA(cudaSetDevice(s->device));
    return 0;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* mrb_last_error(void) { return g_error.c_str(); }

int mrb_system_create(int device, mrb_system** out) {
    if (!out) {
        set_error("mrb_system_create: out is NULL");
        return MRB_E_ARG;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no CUDA device available (%s)", cudaGetErrorString(e));
        return MRB_E_CUDA;
    }
    if (device < 0 || device >= n) {
        set_error("device %d out of range (%d devices)", device, n);
        return MRB_E_ARG;
    }
    mrb_system* s = new mrb_system();
    s->device = device;
    MRB_CUDA(cudaSetDevice(device));
    *out = s;
    return 0;
}

void mrb_system_destroy(mrb_system* s) { delete s; }

int mrb_scene_create(mrb_system* sys, const mrb_scene_desc* d, mrb_scene** out) {
    if (!sys || !d || !out || !d->positions || !d->normals || !d->indices || !d->tri_material ||
        (d->material_count && !d->materials)) {
        set_error("mrb_scene_create: missing argument");
        return MRB_E_ARG;
    }
    if (set_device(sys)) return MRB_E_CUDA;
    const uint32_t T = d->triangle_count, V = d->vertex_count;
    for (uint64_t i = 0; i < uint64_t(T) * 3; i++)
        if (d->indices[i] >= V) {
            set_error("triangle %llu references vertex %u >= %u",
                      (unsigned long long)(i / 3), d->indices[i], V);
            return MRB_E_ARG;
        }
    if (d->base_medium >= d->medium_count || !d->medium_ior) {
        set_error("base medium %u not among %u media", d->base_medium, d->medium_count);
        return MRB_E_ARG;
    }
    mrb_scene* s = new mrb_scene();
    s->sys = sys;
    s->V = V;
    s->T = T;
    s->baseMedium = d->base_medium;
    s->mediumIor.assign(d->medium_ior, d->medium_ior + d->medium_count);
    // Material groups -> batch ids and per-group ids (HitKey batch/id)
    std::vector<uint32_t> matKey(d->material_count, 0);
    std::vector<uint32_t> matType(d->material_count, 0);
    for (uint32_t m = 0; m < d->material_count; m++) {
        const mrb_material& mt = d->materials[m];
        matType[m] = mt.type;
        switch (mt.type) {
            case MRB_MAT_LAMBERT:
                matKey[m] = (kBatchLambert << kIdBits) | uint32_t(s->lambert.size() / 3);
                s->lambert.insert(s->lambert.end(), mt.albedo, mt.albedo + 3);
                break;
            case MRB_MAT_METAL:
                matKey[m] = (kBatchMetal << kIdBits) | uint32_t(s->metal.size() / 10);
                s->metal.insert(s->metal.end(), mt.eta, mt.eta + 3);
                s->metal.insert(s->metal.end(), mt.k, mt.k + 3);
                s->metal.insert(s->metal.end(), mt.specular, mt.specular + 3);
                s->metal.push_back(mt.roughness);
                break;
            case MRB_MAT_REFRACT:
                if (mt.medium >= d->medium_count) {
                    delete s;
                    set_error("material %u: medium %u out of range", m, mt.medium);
                    return MRB_E_ARG;
                }
                matKey[m] = (kBatchRefract << kIdBits) | uint32_t(s->refract.size() / 3);
                s->refract.insert(s->refract.end(), mt.albedo, mt.albedo + 3);
                s->refractMed.push_back(mt.medium);
                break;
            case MRB_MAT_LAMBERTC:
                matKey[m] = (kBatchLambertC << kIdBits) | uint32_t(s->lambertC.size() / 3);
                s->lambertC.insert(s->lambertC.end(), mt.albedo, mt.albedo + 3);
                break;
            case MRB_MAT_UNREAL:
                matKey[m] = (kBatchUnreal << kIdBits) | uint32_t(s->unreal.size() / 6);
                s->unreal.insert(s->unreal.end(), mt.albedo, mt.albedo + 3);
                s->unreal.push_back(mt.roughness);
                s->unreal.push_back(mt.metallic);
                s->unreal.push_back(mt.specular[0]);
                break;
            case MRB_MAT_LIGHT:
                break;
            default:
                delete s;
                set_error("material %u: unsupported type %u", m, mt.type);
                return MRB_E_UNSUPPORTED;
        }
    }
    s->triKey.resize(T);
    uint32_t maxId = 0;
    for (uint32_t t = 0; t < T; t++) {
        uint32_t m = d->tri_material[t];
        if (m >= d->material_count) {
            delete s;
            set_error("triangle %u: material %u out of range", t, m);
            return MRB_E_ARG;
        }
        if (matType[m] == MRB_MAT_LIGHT) {
            // every triangle of a light surface is one primitive light
            uint32_t li = static_cast<uint32_t>(s->lightPrim.size());
            s->lightPrim.push_back(t);
            s->lightRad.insert(s->lightRad.end(), d->materials[m].radiance,
                               d->materials[m].radiance + 3);
            s->triKey[t] = (kBatchLight << kIdBits) | li;
        } else {
            s->triKey[t] = matKey[m];
        }
        maxId = std::max(maxId, s->triKey[t] & kIdMask);
    }
    if (s->lightPrim.size() > kIdMask || s->lambert.size() / 3 > kIdMask) {
        delete s;
        set_error("more than 2^24 entries in one batch");
        return MRB_E_ARG;
    }
    s->idBits = bits_for(maxId);
    build_tbn(*d, s->tbn);
    std::vector<float> pos(d->positions, d->positions + size_t(V) * 3);
    std::vector<uint32_t> idx(d->indices, d->indices + size_t(T) * 3);
    int r = 0;
    if ((r = upload(s->dPos, pos)) || (r = upload(s->dTbn, s->tbn)) || (r = upload(s->dIdx, idx)) ||
        (r = upload(s->dKey, s->triKey)) || (r = upload(s->dLambert, s->lambert)) ||
        (r = upload(s->dMetal, s->metal)) || (r = upload(s->dRefract, s->refract)) ||
        (r = upload(s->dRefractMed, s->refractMed)) || (r = upload(s->dLightRad, s->lightRad)) ||
        (r = upload(s->dLightPrim, s->lightPrim)) || (r = upload(s->dMediumIor, s->mediumIor)) ||
        (r = upload(s->dLambertC, s->lambertC)) || (r = upload(s->dUnreal, s->unreal))) {
        delete s;
        return r;
    }
    if (d->tri_cull) {
        std::vector<uint8_t> cull(d->tri_cull, d->tri_cull + T);
        if ((r = upload(s->dCull, cull))) {
            delete s;
            return r;
        }
    }
    *out = s;
    return 0;
}

void mrb_scene_destroy(mrb_scene* s) { delete s; }

int mrb_scene_counts(const mrb_scene* s, uint32_t* c) {
    if (!s || !c) return MRB_E_ARG;
    c[0] = s->T;
    c[1] = s->V;
    c[2] = static_cast<uint32_t>(s->lightPrim.size());
    c[3] = static_cast<uint32_t>(s->lambert.size() / 3);
    c[4] = static_cast<uint32_t>(s->metal.size() / 10);
    c[5] = static_cast<uint32_t>(s->refract.size() / 3);
    c[6] = static_cast<uint32_t>(s->mediumIor.size());
    c[7] = s->idBits;
    return 0;
}

int mrb_scene_export(const mrb_scene* s, float* tbn, uint32_t* key, float* lambert, float* metal,
                     float* refract, uint32_t* refractMed, float* lightRad, uint32_t* lightPrim) {
    if (!s) return MRB_E_ARG;
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(tbn, s->tbn);
    cp(key, s->triKey);
    cp(lambert, s->lambert);
    cp(metal, s->metal);
    cp(refract, s->refract);
    cp(refractMed, s->refractMed);
    cp(lightRad, s->lightRad);
    cp(lightPrim, s->lightPrim);
    return 0;
}

int mrb_scene_export_ext(const mrb_scene* s, float* lambertC, float* unreal, uint32_t* counts2) {
    if (!s) return MRB_E_ARG;
    if (counts2) {
        counts2[0] = static_cast<uint32_t>(s->lambertC.size() / 3);
        counts2[1] = static_cast<uint32_t>(s->unreal.size() / 6);
    }
    if (lambertC && !s->lambertC.empty())
        std::memcpy(lambertC, s->lambertC.data(), s->lambertC.size() * 4);
    if (unreal && !s->unreal.empty()) std::memcpy(unreal, s->unreal.data(), s->unreal.size() * 4);
    return 0;
}

int mrb_accel_construct(mrb_scene* s, void* stream) {
    if (!s) return MRB_E_ARG;
    if (set_device(s->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t n = s->T;
    if (n == 0) {
        set_error("LBVH: scene has no triangles");
        return MRB_E_ARG;
    }
    int r = 0;
    const size_t ni = n > 1 ? n - 1 : 1;
    if ((r = s->aTriAabb.alloc(size_t(n) * 24)) || (r = s->aExtent.alloc(32)) ||
        (r = s->aCodes.alloc(size_t(n) * 8)) || (r = s->aSorted.alloc(size_t(n) * 4)) ||
        (r = s->aLeft.alloc(ni * 4)) || (r = s->aRight.alloc(ni * 4)) ||
        (r = s->aParent.alloc((2 * size_t(n) - 1) * 4)) || (r = s->aInner.alloc(ni * 24)) ||
        (r = s->aScratch.alloc(ni * 12)) || (r = s->aRoot.alloc(4)) ||
        (r = s->aNodes.alloc(ni * sizeof(BvhNode))) || (r = s->aTv0.alloc(size_t(n) * 16)) ||
        (r = s->aTe0.alloc(size_t(n) * 16)) || (r = s->aTe1.alloc(size_t(n) * 16)))
        return r;
    const size_t tb = radix_sort_temp_bytes(n, 8, 0, 63);
    if ((r = s->aSortTemp.alloc(tb))) return r;
    if ((r = lbvh_morton(s->dPos.as<float>(), s->dIdx.as<uint32_t>(), n, s->aTriAabb.as<float>(),
                         s->aExtent.as<float>(), s->aCodes.as<uint64_t>(), nullptr,
                         s->aExtent.as<float>() + 6, st)))
        return r;
    if ((r = radix_sort_pairs<uint64_t>(s->aCodes.as<uint64_t>(), s->aSorted.as<uint32_t>(),
                                        nullptr, n, 0, 63, false, s->aSortTemp.p, tb, st, true)))
        return r;
    uint32_t* scr = s->aScratch.as<uint32_t>();
    LbvhArrays a{s->aLeft.as<uint32_t>(), s->aRight.as<uint32_t>(), s->aParent.as<uint32_t>(),
                 s->aInner.as<float>(), scr, scr + ni, scr + 2 * ni, s->aRoot.as<uint32_t>(),
                 s->aNodes.as<BvhNode>()};
    if ((r = lbvh_hierarchy(s->aCodes.as<uint64_t>(), s->aSorted.as<uint32_t>(),
                            s->aTriAabb.as<float>(), n, a, st)))
        return r;
    if ((r = lbvh_gather(s->dPos.as<float>(), s->dIdx.as<uint32_t>(), s->dKey.as<uint32_t>(),
                         s->dCull.as<uint8_t>(), s->aSorted.as<uint32_t>(), n, s->aTv0.as<float4>(),
                         s->aTe0.as<float4>(), s->aTe1.as<float4>(), st)))
        return r;
    if (n >= 2) {
        if ((r = s->wNodes.alloc((n - 1) * sizeof(WideNode))) || (r = s->wTv0.alloc(size_t(n) * 16)) ||
            (r = s->wTe0.alloc(size_t(n) * 16)) || (r = s->wTe1.alloc(size_t(n) * 16)) ||
            (r = s->wScratch.alloc(wide_scratch_bytes(n))))
            return r;
        WideBuildIn wi{n, s->aRoot.as<uint32_t>(), s->aLeft.as<uint32_t>(), s->aRight.as<uint32_t>(),
                       s->aInner.as<float>(), s->aTriAabb.as<float>(), s->aSorted.as<uint32_t>(),
                       s->dPos.as<float>(), s->dIdx.as<uint32_t>(), s->dKey.as<uint32_t>(),
                       s->dCull.as<uint8_t>(), s->wideCollapse};
        // the PLOC tree over the same sorted leaves: tighter upper boxes than
        // the Morton splits give the collapse better nodes to start from
        DBuf pLeft, pRight, pInner, pRoot, pScratch;
        s->wideTreeUsed = 0;
        if (s->wideTree != 0) {
            if ((r = pLeft.alloc((n - 1) * 4)) || (r = pRight.alloc((n - 1) * 4)) ||
                (r = pInner.alloc((n - 1) * 24)) || (r = pRoot.alloc(4)) ||
                (r = pScratch.alloc(ploc_scratch_bytes(n))))
                return r;
            PlocIn pi{n, s->aTriAabb.as<float>(), s->aSorted.as<uint32_t>()};
            PlocOut po{pLeft.as<uint32_t>(), pRight.as<uint32_t>(), pInner.as<float>(),
                       pRoot.as<uint32_t>()};
            if ((r = ploc_build(pi, po, pScratch.p, &s->plocSteps, st))) return r;
            double* d8 = static_cast<double*>(pScratch.p);
            if ((r = inner_area_sum(s->aInner.as<float>(), n - 1, d8, &s->areaLbvh, st)) ||
                (r = inner_area_sum(pInner.as<float>(), n - 1, d8, &s->areaPloc, st)))
                return r;
            pScratch.release();
            if (s->wideTree == 1 || s->areaPloc < s->areaLbvh) {
                s->wideTreeUsed = 1;
                wi.root = pRoot.as<uint32_t>();
                wi.left = pLeft.as<uint32_t>();
                wi.right = pRight.as<uint32_t>();
                wi.inner = pInner.as<float>();
            }
        }
        wi.collapse = (s->wideCollapse == kWideCollapseGreedy) ? kWideCollapseGreedy : kWideCollapseSah;
        if ((r = wide_build(wi, s->wNodes.as<WideNode>(), s->wTv0.as<float4>(), s->wTe0.as<float4>(),
                            s->wTe1.as<float4>(), s->wScratch.p, &s->wNodeCount, st)))
            return r;
        s->wideCollapseUsed = wi.collapse;
        s->collapseProbeBytes[0] = s->collapseProbeBytes[1] = 0.0;
        s->aNodes2.release();
        s->aTv02.release();
        s->aTe02.release();
        s->aTe12.release();
        s->wAltNodeCount = 0;
        if (s->wideCollapse == 2) {
            // both collapses: the layout the probe rays read fewer bytes of is
            // the scene's; the other stays as the alternate that tracers time
            // per depth on their own rays
            if ((r = s->aNodes2.alloc((n - 1) * sizeof(WideNode))) ||
                (r = s->aTv02.alloc(size_t(n) * 16)) || (r = s->aTe02.alloc(size_t(n) * 16)) ||
                (r = s->aTe12.alloc(size_t(n) * 16)))
                return r;
            wi.collapse = kWideCollapseGreedy;
            if ((r = wide_build(wi, s->aNodes2.as<WideNode>(), s->aTv02.as<float4>(),
                                s->aTe02.as<float4>(), s->aTe12.as<float4>(), s->wScratch.p,
                                &s->wAltNodeCount, st)))
                return r;
            double pb[2];
            if ((r = wide_probe_compare(s->wide(), s->wideAlt(), s->aExtent.as<float>(), st, pb)))
                return r;
            s->collapseProbeBytes[kWideCollapseSah] = pb[0];
            s->collapseProbeBytes[kWideCollapseGreedy] = pb[1];
            if (pb[1] < pb[0]) {
                s->wNodes.swap(s->aNodes2);
                s->wTv0.swap(s->aTv02);
                s->wTe0.swap(s->aTe02);
                s->wTe1.swap(s->aTe12);
                std::swap(s->wNodeCount, s->wAltNodeCount);
                s->wideCollapseUsed = kWideCollapseGreedy;
            }
        }
        s->wScratch.release();
        for (float& m : s->wideOrderMs) m = 0.0f;
        if (s->wideOrderMode == MRB_WIDE_AUTO) {
            if ((r = wide_order_autotune(s->wide(), s->aExtent.as<float>(), st, &s->wideOrder,
                                         s->wideOrderMs)))
                return r;
        } else {
            s->wideOrder = s->wideOrderMode;
        }
    }
    uint32_t root = 0, err = 0;
    MRB_CUDA(cudaMemcpyAsync(&root, s->aRoot.p, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaMemcpyAsync(&err, radix_sort_error_flag(s->aSortTemp.p, n), 4,
                             cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    if (err) {
        set_error("LBVH: radix sort look-back gave up");
        return MRB_E_DEVICE;
    }
    s->rootInner = (n == 1) ? ~0 : static_cast<int>(root - n);
    s->built = true;
    s->traceEpoch++;
    return 0;
}

int mrb_accel_export(const mrb_scene* s, uint64_t* codes, uint32_t* sorted, uint32_t* left,
                     uint32_t* right, uint32_t* parent, float* inner, uint32_t* root,
                     float* triAabbs, float* extent) {
    if (!s || !s->built) {
        set_error("accelerator not constructed");
        return MRB_E_STATE;
    }
    const size_t n = s->T, ni = n > 1 ? n - 1 : 0;
    auto cp = [](void* dst, const DBuf& b, size_t bytes) -> int {
        if (!dst || !bytes) return 0;
        MRB_CUDA(cudaMemcpy(dst, b.p, bytes, cudaMemcpyDeviceToHost));
        return 0;
    };
    if (cp(codes, s->aCodes, n * 8) || cp(sorted, s->aSorted, n * 4) || cp(left, s->aLeft, ni * 4) ||
        cp(right, s->aRight, ni * 4) || cp(parent, s->aParent, (2 * n - 1) * 4) ||
        cp(inner, s->aInner, ni * 24) || cp(root, s->aRoot, 4) || cp(triAabbs, s->aTriAabb, n * 24) ||
        cp(extent, s->aExtent, 28))
        return MRB_E_CUDA;
    return 0;
}

int mrb_accel_hit(const mrb_scene* s, const float* rayO, const float* rayD, uint32_t n,
                  uint32_t* key, uint32_t* prim, float* t, float* bary, void* stream) {
    if (!s || !s->built) {
        set_error("accelerator not constructed");
        return MRB_E_STATE;
    }
    if (n == 0) return 0;
    HitOut ho{key, prim, t, reinterpret_cast<float2*>(bary)};
    static DBuf flag;
    if (!flag.p) {
        if (flag.alloc(16)) return MRB_E_OOM;
        MRB_CUDA(cudaMemset(flag.p, 0, 16));
    }
    return trace_dispatch(s, reinterpret_cast<const float4*>(rayO),
                          reinterpret_cast<const float4*>(rayD), nullptr, n, ho,
                          flag.as<uint32_t>(), static_cast<cudaStream_t>(stream));
}

int mrb_svo_build(mrb_scene* s, uint32_t resolution, void* stream) {
    if (!s || !s->built) {
        set_error("SVO: construct the accelerator first (the scene extent comes from it)");
        return MRB_E_STATE;
    }
    if (resolution < 2 || resolution > 1024 || (resolution & (resolution - 1))) {
        set_error("SVO: resolution %u must be a power of two in [2, 1024]", resolution);
        return MRB_E_ARG;
    }
    if (set_device(s->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float ext[8];
    MRB_CUDA(cudaMemcpyAsync(ext, s->aExtent.p, 24, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    if (s->svoBuilt) {
        svo_free(s->svo);
        s->svoBuilt = false;
    }
    s->svoP = svo_params(ext, resolution);
    SvoBuildIn in{s->T, s->dPos.as<float>(), s->dIdx.as<uint32_t>(), s->dKey.as<uint32_t>(),
                  s->dLightRad.as<float>(), 0u};
    int r = svo_build(in, s->svoP, s->svo, st);
    if (!r) r = svo_payload_finish(guide_dev(s->svo, s->svoP), s->svo, st);
    if (!r) MRB_CUDA(cudaStreamSynchronize(st));
    if (r) {
        svo_free(s->svo);
        return r;
    }
    s->svoBuilt = true;
    return 0;
}

int mrb_svo_info(const mrb_scene* s, uint32_t* info, float* params) {
    if (!s || !s->svoBuilt) {
        set_error("SVO not built");
        return MRB_E_STATE;
    }
    svo_info(s->svo, s->svoP, info, params);
    return 0;
}

int mrb_svo_export(const mrb_scene* s, uint64_t* nodes, uint32_t* leafParents,
                   uint64_t* leafCodes, uint32_t* leafNormal, uint32_t* leafLight,
                   uint32_t* levelOffsets) {
    if (!s || !s->svoBuilt) {
        set_error("SVO not built");
        return MRB_E_STATE;
    }
    return export_svo(s->svo, nodes, leafParents, leafCodes, leafNormal, leafLight, levelOffsets);
}

int mrb_svo_export_payload(const mrb_scene* s, uint32_t* nodeNormSpec, uint64_t* leafIrr,
                           uint32_t* leafCnt, uint32_t* leafAvg, uint32_t* nodeAvg) {
    if (!s || !s->svoBuilt) {
        set_error("SVO not built");
        return MRB_E_STATE;
    }
    return export_payload(s->svo, nodeNormSpec, leafIrr, leafCnt, leafAvg, nodeAvg);
}

int mrb_accel_set_traversal(mrb_scene* s, int mode) {
    if (!s || (mode != 0 && mode != 1)) {
        set_error("traversal mode must be 0 (binary) or 1 (8-wide)");
        return MRB_E_ARG;
    }
    s->traversal = mode;
    s->traceEpoch++;
    return 0;
}

int mrb_accel_set_wide_order(mrb_scene* s, int order) {
    if (!s || order < 0 || order > MRB_WIDE_AUTO) {
        set_error("wide order must be 0 (sorted), 1 (octant), 2 (sorted, refilled lanes), "
                  "3 (octant, refilled lanes) or 4 (the fastest as timed)");
        return MRB_E_ARG;
    }
    s->wideOrderMode = order;
    s->traceEpoch++;
    for (float& m : s->wideOrderMs) m = 0.0f;
    if (order != MRB_WIDE_AUTO) {
        s->wideOrder = order;
        return 0;
    }
    if (!s->built || s->T < 2) return 0;
    if (set_device(s->sys)) return MRB_E_CUDA;
    return wide_order_autotune(s->wide(), s->aExtent.as<float>(), nullptr, &s->wideOrder,
                               s->wideOrderMs);
}

int mrb_accel_wide_order(const mrb_scene* s, int* order, float* ms4) {
    if (!s || !order) return MRB_E_ARG;
    *order = s->wideOrder;
    if (ms4)
        for (int o = 0; o < kWideOrders; o++) ms4[o] = s->wideOrderMs[o];
    return 0;
}

int mrb_tracer_wide_orders(const mrb_tracer* t, int* orders, uint32_t n) {
    if (!t || (n && !orders)) return MRB_E_ARG;
    uint32_t k = 0;
    for (; k < n && k < t->maxDepth; k++) {
        const int o = depth_order(t, k);
        orders[k] = o >= kWideOrders ? (o - kWideOrders) | MRB_WIDE_ALT_LAYOUT
                  : o >= 0           ? o
                  : (t->scene->traversal == 1 ? t->scene->wideOrder : -1);
    }
    return int(k);
}

int mrb_accel_set_wide_tree(mrb_scene* s, int tree) {
    if (!s || tree < 0 || tree > 2) {
        set_error("wide tree must be 0 (LBVH), 1 (PLOC) or 2 (the one with less box area)");
        return MRB_E_ARG;
    }
    if (s->built) {
        set_error("wide tree: set it before mrb_accel_construct");
        return MRB_E_STATE;
    }
    s->wideTree = tree;
    return 0;
}

int mrb_accel_set_wide_collapse(mrb_scene* s, int collapse) {
    if (!s || collapse < 0 || collapse > 2) {
        set_error("wide collapse must be 0 (largest area first), 1 (surface-area plan) or 2 "
                  "(the one the probe rays read less of)");
        return MRB_E_ARG;
    }
    if (s->built) {
        set_error("wide collapse: set it before mrb_accel_construct");
        return MRB_E_STATE;
    }
    s->wideCollapse = collapse;
    return 0;
}

int mrb_accel_wide_collapse(const mrb_scene* s, int* used, double* probeBytes2) {
    if (!s || !used) return MRB_E_ARG;
    *used = s->wideCollapseUsed;
    if (probeBytes2) {
        probeBytes2[0] = s->collapseProbeBytes[0];
        probeBytes2[1] = s->collapseProbeBytes[1];
    }
    return 0;
}

int mrb_accel_info(const mrb_scene* s, uint32_t* info) {
    if (!s || !info) return MRB_E_ARG;
    info[0] = s->T;
    info[1] = s->T > 1 ? s->T - 1 : 0;
    info[2] = s->wNodeCount;
    info[3] = static_cast<uint32_t>(s->traversal);
    return 0;
}

int mrb_accel_info_ext(const mrb_scene* s, uint32_t* info, double* areas) {
    if (!s || !info) return MRB_E_ARG;
    info[0] = static_cast<uint32_t>(s->wideTreeUsed);
    info[1] = s->plocSteps;
    if (areas) {
        areas[0] = s->areaLbvh;
        areas[1] = s->areaPloc;
    }
    return 0;
}

int mrb_tracer_create(mrb_system* sys, mrb_scene* scene, const char* type, mrb_tracer** out) {
    if (!sys || !scene || !out) return MRB_E_ARG;
    const bool wfpg = type && std::strcmp(type, "WFPGTracer") == 0;
    if (!type || (!wfpg && std::strcmp(type, "PathTracer") != 0)) {
        set_error("tracer type '%s' is not supported (PathTracer, WFPGTracer)",
                  type ? type : "(null)");
        return MRB_E_UNSUPPORTED;
    }
    if (!scene->built) {
        set_error("tracer: construct the accelerator first");
        return MRB_E_STATE;
    }
    if (set_device(sys)) return MRB_E_CUDA;
    mrb_tracer* t = new mrb_tracer();
    t->sys = sys;
    t->scene = scene;
    t->wfpg = wfpg;
    if (wfpg) t->maxDepth = 10;  // WFPGTracer::Options::maximumDepth
    cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMallocHost(reinterpret_cast<void**>(&t->hostCam),
                           sizeof(CameraDev) * mrb_tracer::kCamSlots);
    for (int i = 0; i < mrb_tracer::kCamSlots && e == cudaSuccess; i++)
        e = cudaEventCreateWithFlags(&t->camEv[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete t;
        set_error("tracer setup: %s", cudaGetErrorString(e));
        return MRB_E_CUDA;
    }
    if (t->devCam.alloc(sizeof(CameraDev))) {
        delete t;
        return MRB_E_OOM;
    }
    *out = t;
    return 0;
}

void mrb_tracer_destroy(mrb_tracer* t) { delete t; }

int mrb_tracer_set_option_float(mrb_tracer* t, const char* name, double v) {
    if (!t || !name) return MRB_E_ARG;
    std::string k(name);
    if (t->wfpg && k == "BXDF-GuideMISRatio") {
        if (!(v >= 0.0 && v <= 1.0)) {
            set_error("BXDF-GuideMISRatio must be in [0, 1]");
            return MRB_E_ARG;
        }
        t->misRatio = static_cast<float>(v);
    } else if (t->wfpg && k == "RFieldFilterAlpha") {
        if (!(v > 0.0)) {
            set_error("RFieldFilterAlpha must be > 0");
            return MRB_E_ARG;
        }
        t->filterAlpha = static_cast<float>(v);
    } else if (t->wfpg && k == "LearnedRate") {
        if (!(v > 0.0 && v < 1.0)) {
            set_error("LearnedRate must be in (0, 1)");
            return MRB_E_ARG;
        }
        t->learnedRate = static_cast<float>(v);
    } else if (t->wfpg && k == "LearnedEMA") {
        if (!(v >= 0.0 && v < 1.0)) {
            set_error("LearnedEMA must be in [0, 1)");
            return MRB_E_ARG;
        }
        t->learnedEma = static_cast<float>(v);
    } else if (t->wfpg && k == "LearnedWeightMax") {
        if (!(v >= 0.0)) {
            set_error("LearnedWeightMax must be >= 0");
            return MRB_E_ARG;
        }
        t->learnedWeightMax = static_cast<float>(v);
    } else {
        set_error("unknown float option '%s'", name);
        return MRB_E_ARG;
    }
    t->graphDirty = true;
    return 0;
}

int mrb_tracer_set_option(mrb_tracer* t, const char* name, uint64_t v) {
    if (!t || !name) return MRB_E_ARG;
    std::string k(name);
    if (k == "Samples") {
        if (v == 0 || v > 64) {
            set_error("Samples must be in [1, 64]");
            return MRB_E_ARG;
        }
        t->samples = uint32_t(v);
    } else if (k == "MaxDepth") {
        if (v == 0 || v > 255) {
            set_error("MaxDepth must be in [1, 255]");
            return MRB_E_ARG;
        }
        t->maxDepth = uint32_t(v);
    } else if (k == "NextEventEstimation") {
        t->nee = v ? 1 : 0;
    } else if (k == "RussianRouletteStart") {
        t->rrStart = uint32_t(v);
    } else if (k == "DirectLightMIS") {
        t->mis = v ? 1 : 0;
    } else if (k == "Seed") {
        t->seed = v;
    } else if (t->wfpg && (k == "OctreeLevel" || k == "OmitDirectRadiance")) {
        if (k == "OctreeLevel" && (v < 1 || v > 10)) {
            set_error("OctreeLevel must be in [1, 10]");
            return MRB_E_ARG;
        }
        if (k == "OctreeLevel") t->octreeLevel = uint32_t(v);
        else t->omitDirect = v ? 1 : 0;
        if (t->svoReady) {
            MRB_CUDA(cudaStreamSynchronize(t->stream));
            svo_free(t->svo);
            t->svoReady = false;
        }
    } else if (t->wfpg && k == "MinRayBinLevel") {
        t->minRayBinLevel = uint32_t(v);
    } else if (t->wfpg && k == "BinRayCount") {
        if (v == 0 || v > 0x7FFFFFFF) {
            set_error("BinRayCount must be in [1, 2^31)");
            return MRB_E_ARG;
        }
        t->binRayCount = uint32_t(v);
    } else if (t->wfpg && k == "DoProductPathGuiding") {
        t->productPG = v ? 1 : 0;
    } else if (t->wfpg && k == "PurePG") {
        t->purePG = v ? 1 : 0;
    } else if (t->wfpg && k == "SkipPG") {
        t->skipPG = v ? 1 : 0;
    } else if (t->wfpg && k == "GuideBounceAmount") {
        t->guideBounce = uint32_t(v);
    } else if (t->wfpg && k == "LearnedGuiding") {
        t->learned = v ? 1 : 0;
    } else if (t->wfpg && k == "LearnedWarmupFrames") {
        t->learnedWarmup = uint32_t(v);
    } else if (t->wfpg && (k == "LearnedTrainSteps" || k == "LearnedSamples")) {
        if (k == "LearnedTrainSteps" && (v == 0 || v > 32)) {
            set_error("LearnedTrainSteps must be in [1, 32]");
            return MRB_E_ARG;
        }
        if (k == "LearnedSamples" && (v < 128 || v > (1u << 24))) {
            set_error("LearnedSamples must be in [128, 2^24]");
            return MRB_E_ARG;
        }
        if (k == "LearnedTrainSteps") t->learnedSteps = uint32_t(v);
        else t->learnedSamples = uint32_t(v);
        t->learnedReset = true;
    } else if (t->wfpg && k == "LearnedWarmupOctree") {
        t->learnedWarmupOctree = v ? 1 : 0;
    } else if (t->wfpg && k == "LearnedProductTarget") {
        t->learnedProduct = v ? 1 : 0;
    } else if (t->wfpg && k == "LearnedSeed") {
        t->learnedSeed = v;
        if (t->net) {
            const std::vector<float> p = learned_init(v);
            if (mrb_mlp_set_params(t->net, p.data())) return MRB_E_CUDA;
            t->learnedReset = true;
        }
    } else if (t->wfpg && k == "PGDumpDataStruct") {
        t->dumpEnabled = v ? 1 : 0;
        return 0;
    } else if (t->wfpg && k == "PGDataStructDumpIntervalExp") {
        t->dumpInterval = uint32_t(v);
        return 0;
    } else if (k == "Frame") {
        // applied now, or when the buffers are first allocated
        t->frameStart = uint32_t(v);
        if (t->frameWord.p) {
            MRB_CUDA(cudaMemcpyAsync(t->frameWord.p, &t->frameStart, 4, cudaMemcpyHostToDevice,
                                     t->stream));
            MRB_CUDA(cudaStreamSynchronize(t->stream));
        }
        return 0;
    } else {
        set_error("unknown option '%s'", name);
        return MRB_E_ARG;
    }
    t->graphDirty = true;
    return 0;
}

int mrb_tracer_set_resolution(mrb_tracer* t, uint32_t w, uint32_t h) {
    if (!t || !w || !h) return MRB_E_ARG;
    t->width = w;
    t->height = h;
    t->graphDirty = true;
    return 0;
}

int mrb_camera_frame(const mrb_camera* c, float* o) {
    if (!c || !o) return MRB_E_ARG;
    // GPUCameraPinhole constructor (GPUCameraPinhole.cuh:135-162)
    H3 pos = h3(c->position[0], c->position[1], c->position[2]);
    H3 gz = h3(c->gaze[0], c->gaze[1], c->gaze[2]);
    H3 up = h3(c->up[0], c->up[1], c->up[2]);
    float nearP = c->near_far[0];
    float wh = std::tan(c->fov[0] * 0.5f) * nearP;
    float hh = std::tan(c->fov[1] * 0.5f) * nearP;
    H3 gd = hsub(gz, pos);
    H3 right = hnorm(hcross(gd, up));
    up = hnorm(hcross(right, gd));
    gd = hnorm(hcross(up, right));
    H3 bl = hadd(hsub(hsub(pos, hmul(right, wh)), hmul(up, hh)), hmul(gd, nearP));
    for (int i = 0; i < 3; i++) {
        o[i] = pos[i];
        o[3 + i] = bl[i];
        o[6 + i] = right[i];
        o[9 + i] = up[i];
    }
    o[12] = wh * 2.0f;
    o[13] = hh * 2.0f;
    return 0;
}

int mrb_tracer_set_camera(mrb_tracer* t, const mrb_camera* c) {
    if (!t || !c) return MRB_E_ARG;
    float f[14];
    mrb_camera_frame(c, f);
    // the next staging slot; the upload that last read it may still be queued
    // (no wait on the frames in flight: the stream orders each upload after
    // the frames before it)
    const int slot = (t->camSlot + 1) % mrb_tracer::kCamSlots;
    if (t->camEvUsed[slot]) MRB_CUDA(cudaEventSynchronize(t->camEv[slot]));
    CameraDev& cam = t->hostCam[slot];
    for (int i = 0; i < 3; i++) {
        cam.position[i] = f[i];
        cam.bottomLeft[i] = f[3 + i];
        cam.right[i] = f[6 + i];
        cam.up[i] = f[9 + i];
    }
    cam.planeSize[0] = f[12];
    cam.planeSize[1] = f[13];
    cam.nearFar[0] = c->near_far[0];
    cam.nearFar[1] = c->near_far[1];
    // host -> device copy of the frame; graphs read it from device memory
    MRB_CUDA(cudaMemcpyAsync(t->devCam.p, &cam, sizeof(CameraDev), cudaMemcpyHostToDevice,
                             t->stream));
    MRB_CUDA(cudaEventRecord(t->camEv[slot], t->stream));
    t->camEvUsed[slot] = true;
    t->camSlot = slot;
    t->camSet = true;
    return 0;
}

int mrb_tracer_generate_work(mrb_tracer* t, uint32_t) {
    if (!t) return MRB_E_ARG;
    if (!t->camSet) {
        set_error("tracer: camera not set");
        return MRB_E_STATE;
    }
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_buffers(t);
    if (r) return r;
    if ((r = ensure_svo(t))) return r;
    if ((r = ensure_learned(t))) return r;
    if ((r = step_camera(t))) return r;
    t->depth = 0;
    t->working = true;
    return 0;
}

int mrb_tracer_render(mrb_tracer* t) {
    if (!t) return MRB_E_ARG;
    if (!t->working) {
        set_error("Render() before GenerateWork()");
        return MRB_E_STATE;
    }
    if (t->depth >= t->maxDepth) return 0;
    int r = step_depth(t, t->depth);
    if (r) return r;
    t->depth++;
    return t->depth < t->maxDepth ? 1 : 0;
}

int mrb_tracer_finalize(mrb_tracer* t) {
    if (!t || !t->working) return MRB_E_STATE;
    int r = step_finalize(t);
    if (r) return r;
    t->working = false;
    t->frames++;
    if ((r = check_device_errors(t))) return r;
    return wfpg_after_frame(t);
}

int mrb_tracer_render_frame(mrb_tracer* t) {
    if (!t) return MRB_E_ARG;
    if (!t->camSet) {
        set_error("tracer: camera not set");
        return MRB_E_STATE;
    }
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_buffers(t);
    if (r) return r;
    if ((r = ensure_svo(t))) return r;
    if ((r = ensure_learned(t))) return r;
    // a training branch left open by the step-wise calls ends first
    if ((r = learned_join(t))) return r;
    // the captured frame bakes in which sampler guides: capture again when
    // the network takes over
    if (t->wfpg && t->learned && t->frames == t->learnedWarmup) t->graphDirty = true;
    // the scene's traversal changed since the capture
    if (t->graphEpoch != t->scene->traceEpoch) t->graphDirty = true;
    if (t->graphDirty || !t->graph) {
        if (t->graph) {
            cudaGraphExecDestroy(t->graph);
            t->graph = nullptr;
        }
        // run one frame eagerly first so that one-time setup (kernel
        // attributes) happens outside the capture, then rewind the frame:
        // frame word, octree radiance, network state, the accumulated image
        // and the ray counters are put back
        uint32_t f0 = 0;
        if ((r = t->imageBackup.alloc(t->image.bytes + 16))) return r;
        MRB_CUDA(cudaMemcpyAsync(t->imageBackup.p, t->image.p, t->image.bytes,
                                 cudaMemcpyDeviceToDevice, t->stream));
        MRB_CUDA(cudaMemcpyAsync(t->imageBackup.as<char>() + t->image.bytes, t->counters.p, 16,
                                 cudaMemcpyDeviceToDevice, t->stream));
        MRB_CUDA(cudaMemcpyAsync(&f0, t->frameWord.p, 4, cudaMemcpyDeviceToHost, t->stream));
        MRB_CUDA(cudaStreamSynchronize(t->stream));
        // with the automatic traversal kernel, each depth's kernel is settled
        // on this frame's rays (once per tracer and scene traversal; the
        // captured frame bakes the choice in)
        mrb_scene* sc = t->scene;
        t->orderTune = sc->traversal == 1 && sc->T > 1 && sc->wideOrderMode == MRB_WIDE_AUTO &&
                       t->orderEpoch != sc->traceEpoch;
        if (t->orderTune) {
            std::array<float, kTunedOrders> z;
            z.fill(0.0f);
            t->depthMs.assign(t->maxDepth, z);
            t->depthOrder.assign(t->maxDepth, 0);
        }
        // the octree's radiance state of a WFPG tracer is put back too
        const size_t U = t->svo.leafCount, N = t->svo.nodeCount;
        const size_t pb = t->wfpg ? U * 16 + U * 8 + U * 4 + N * 4 + U * 8 + N * 2 : 0;
        if (pb) {
            if ((r = t->payloadBackup.alloc(pb))) return r;
            char* b = t->payloadBackup.as<char>();
            MRB_CUDA(cudaMemcpyAsync(b, t->svo.leafIrr, U * 16, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(b + U * 16, t->svo.leafCnt, U * 8, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(b + U * 24, t->svo.leafAvg, U * 4, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(b + U * 28, t->svo.nodeAvg, N * 4, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(b + U * 28 + N * 4, t->svo.leafShadow, U * 8,
                                     cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(b + U * 36 + N * 4, t->svo.nodeFactor, N * 2,
                                     cudaMemcpyDeviceToDevice, t->stream));
        }
        if (t->net && mlp_state_copy(t->net, t->netBackup.p, true, t->stream)) return MRB_E_CUDA;
        if (t->net)
            MRB_CUDA(cudaMemcpyAsync(t->lEmaBackup.p, t->lEma.p, size_t(kMlpParams) * 4,
                                     cudaMemcpyDeviceToDevice, t->stream));
        r = record_frame(t);
        if (t->orderTune) {
            t->orderTune = false;
            if (!r) {
                // one layout for the whole frame (mixing them per depth would
                // keep both trees in L2 and slow the next frame's first depth):
                // the one whose fastest kernels sum to less; then per depth the
                // fastest kernel on it.  For the scene's other callers the
                // fastest kernel over the whole frame on the scene's layout.
                std::array<float, kWideOrders> sum;
                sum.fill(0.0f);
                float layoutMs[2] = {0.0f, 0.0f};
                for (size_t d = 0; d < t->depthMs.size(); d++) {
                    for (int L = 0; L < 2; L++) {
                        float m = t->depthMs[d][L * kWideOrders];
                        for (int o = 1; o < kWideOrders; o++)
                            m = std::min(m, t->depthMs[d][L * kWideOrders + o]);
                        layoutMs[L] += m;
                    }
                    for (int o = 0; o < kWideOrders; o++) sum[o] += t->depthMs[d][o];
                }
                const int L = layoutMs[1] < layoutMs[0] ? 1 : 0;
                for (size_t d = 0; d < t->depthMs.size(); d++) {
                    int best = 0;
                    for (int o = 1; o < kWideOrders; o++)
                        if (t->depthMs[d][L * kWideOrders + o] < t->depthMs[d][L * kWideOrders + best])
                            best = o;
                    t->depthOrder[d] = L * kWideOrders + best;
                }
                int best = 0;
                for (int o = 0; o < kWideOrders; o++) {
                    sc->wideOrderMs[o] = sum[o];
                    if (sum[o] < sum[best]) best = o;
                }
                sc->wideOrder = best;
                t->orderEpoch = sc->traceEpoch;
            }
        }
        if (r) return r;
        if (t->net && mlp_state_copy(t->net, t->netBackup.p, false, t->stream)) return MRB_E_CUDA;
        if (t->net) {
            MRB_CUDA(cudaMemcpyAsync(t->lEma.p, t->lEmaBackup.p, size_t(kMlpParams) * 4,
                                     cudaMemcpyDeviceToDevice, t->stream));
            // the forward copy as it was: the restored state, without a new
            // average step
            if ((r = learned_refresh_forward(t, false))) return r;
        }
        MRB_CUDA(cudaMemcpyAsync(t->frameWord.p, &f0, 4, cudaMemcpyHostToDevice, t->stream));
        if (pb) {
            const char* b = t->payloadBackup.as<char>();
            MRB_CUDA(cudaMemcpyAsync(t->svo.leafIrr, b, U * 16, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(t->svo.leafCnt, b + U * 16, U * 8, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(t->svo.leafAvg, b + U * 24, U * 4, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(t->svo.nodeAvg, b + U * 28, N * 4, cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(t->svo.leafShadow, b + U * 28 + N * 4, U * 8,
                                     cudaMemcpyDeviceToDevice, t->stream));
            MRB_CUDA(cudaMemcpyAsync(t->svo.nodeFactor, b + U * 36 + N * 4, N * 2,
                                     cudaMemcpyDeviceToDevice, t->stream));
        }
        MRB_CUDA(cudaMemcpyAsync(t->image.p, t->imageBackup.p, t->image.bytes,
                                 cudaMemcpyDeviceToDevice, t->stream));
        MRB_CUDA(cudaMemcpyAsync(t->counters.p, t->imageBackup.as<char>() + t->image.bytes, 16,
                                 cudaMemcpyDeviceToDevice, t->stream));
        MRB_CUDA(cudaStreamSynchronize(t->stream));
        cudaGraph_t g = nullptr;
        MRB_CUDA(cudaStreamBeginCapture(t->stream, cudaStreamCaptureModeThreadLocal));
        r = record_frame(t);
        cudaError_t e = cudaStreamEndCapture(t->stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) {
            set_error("graph capture failed: %s", cudaGetErrorString(e));
            return MRB_E_CUDA;
        }
        e = cudaGraphInstantiate(&t->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error("graph instantiate failed: %s", cudaGetErrorString(e));
            return MRB_E_CUDA;
        }
        t->graphDirty = false;
        t->graphEpoch = t->scene->traceEpoch;
    }
    MRB_CUDA(cudaGraphLaunch(t->graph, t->stream));
    t->frames++;
    return wfpg_after_frame(t);
}

int mrb_tracer_get_image(mrb_tracer* t, float* host) {
    if (!t || !host || !t->image.p) return MRB_E_ARG;
    MRB_CUDA(cudaMemcpyAsync(host, t->image.p, size_t(t->width) * t->height * 16,
                             cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    return check_device_errors(t);
}

int mrb_tracer_get_image_async(mrb_tracer* t, float* host) {
    if (!t || !host || !t->image.p) return MRB_E_ARG;
    const size_t bytes = size_t(t->width) * t->height * 16;
    if (!t->copyStream) {
        MRB_CUDA(cudaStreamCreateWithFlags(&t->copyStream, cudaStreamNonBlocking));
        MRB_CUDA(cudaEventCreateWithFlags(&t->snapDone, cudaEventDisableTiming));
        MRB_CUDA(cudaEventCreateWithFlags(&t->copyDone, cudaEventDisableTiming));
    }
    if (int r = t->imageStage.alloc(bytes)) return r;
    // the previous copy must have left the snapshot buffer
    if (t->copyPending) MRB_CUDA(cudaStreamWaitEvent(t->stream, t->copyDone, 0));
    MRB_CUDA(cudaMemcpyAsync(t->imageStage.p, t->image.p, bytes, cudaMemcpyDeviceToDevice,
                             t->stream));
    MRB_CUDA(cudaEventRecord(t->snapDone, t->stream));
    MRB_CUDA(cudaStreamWaitEvent(t->copyStream, t->snapDone, 0));
    MRB_CUDA(cudaMemcpyAsync(host, t->imageStage.p, bytes, cudaMemcpyDeviceToHost,
                             t->copyStream));
    MRB_CUDA(cudaEventRecord(t->copyDone, t->copyStream));
    t->copyPending = true;
    return 0;
}

int mrb_tracer_wait_image(mrb_tracer* t) {
    if (!t) return MRB_E_ARG;
    if (t->copyPending) {
        MRB_CUDA(cudaEventSynchronize(t->copyDone));
        t->copyPending = false;
    }
    return check_device_errors(t);
}

int mrb_tracer_get_samples(mrb_tracer* t, float* host) {
    if (!t || !host || !t->samplesBuf.p) return MRB_E_ARG;
    const size_t n = size_t(t->width) * t->samples * t->height * t->samples;
    MRB_CUDA(cudaMemcpyAsync(host, t->samplesBuf.p, n * 16, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    return check_device_errors(t);
}

int mrb_tracer_reset_image(mrb_tracer* t) {
    if (!t) return MRB_E_ARG;
    if (t->image.p) MRB_CUDA(cudaMemsetAsync(t->image.p, 0, t->image.bytes, t->stream));
    return 0;
}

int mrb_tracer_learned_loss(mrb_tracer* t, float* host_loss2) {
    if (!t || !host_loss2 || !t->net) {
        set_error("tracer: no learned guiding network (option LearnedGuiding, then a frame)");
        return MRB_E_STATE;
    }
    if (set_device(t->sys)) return MRB_E_CUDA;
    MRB_CUDA(cudaMemcpyAsync(host_loss2, t->lLoss.p, 8, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    return 0;
}

int mrb_tracer_learned_params(mrb_tracer* t, float* host_params) {
    if (!t || !host_params || !t->net) {
        set_error("tracer: no learned guiding network (option LearnedGuiding, then a frame)");
        return MRB_E_STATE;
    }
    if (set_device(t->sys)) return MRB_E_CUDA;
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    return mrb_mlp_get_params(t->net, host_params);
}

int mrb_tracer_set_option_string(mrb_tracer* t, const char* name, const char* value) {
    if (!t || !name || !value) return MRB_E_ARG;
    const std::string k(name);
    if (t->wfpg && k == "InitialSVO") {
        t->initialSvo = value;
        // the next GenerateWork builds (empty path) or loads the octree
        if (t->svoReady) {
            if (set_device(t->sys)) return MRB_E_CUDA;
            MRB_CUDA(cudaStreamSynchronize(t->stream));
            svo_free(t->svo);
            t->svoReady = false;
        }
        t->graphDirty = true;
        return 0;
    }
    if (t->wfpg && k == "PGDataStructDumpName") {
        if (!*value) {
            set_error("PGDataStructDumpName must not be empty");
            return MRB_E_ARG;
        }
        t->dumpName = value;
        return 0;
    }
    set_error("unknown string option '%s'", name);
    return MRB_E_ARG;
}

int mrb_tracer_svo_dump(mrb_tracer* t, void* out, size_t capacity, size_t* size) {
    if (!t || !t->wfpg || !size) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_svo(t);
    if (r) return r;
    *size = svo_dump_size(t->svo.nodeCount, t->svo.leafCount,
                          static_cast<uint32_t>(t->svo.levelOffsets.size()));
    if (!out) return 0;
    if (capacity < *size) {
        set_error("octree dump: %zu bytes needed, %zu given", *size, capacity);
        return MRB_E_ARG;
    }
    std::vector<uint8_t> data;
    if ((r = svo_dump(t->svo, t->svoP, data, t->stream))) return r;
    std::memcpy(out, data.data(), data.size());
    return 0;
}

int mrb_tracer_svo_load(mrb_tracer* t, const void* data, size_t size) {
    if (!t || !t->wfpg || !data) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    SvoParams P{};
    SvoResult v{};
    int r = svo_load(static_cast<const uint8_t*>(data), size, P, v, t->stream);
    if (r) return r;
    if (t->svoReady) svo_free(t->svo);
    t->svo = v;
    t->svoP = P;
    t->svoReady = true;
    t->graphDirty = true;
    return 0;
}

int mrb_tracer_write_image(mrb_tracer* t, const char* path) {
    if (!t || !path || !t->image.p) return MRB_E_ARG;
    std::vector<float> img(size_t(t->width) * t->height * 4);
    int r = mrb_tracer_get_image(t, img.data());
    if (r) return r;
    // rgb / w: the per-pixel estimate whether w counts frames or weights
    return write_averaged(path, img.data(), img.data() + 3, 4, t->width, t->height, 4, 3);
}

int mrb_tracer_set_filter(mrb_tracer* t, const mrb_recon_filter* f) {
    if (!t) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    t->hasFilter = f != nullptr;
    if (f) t->filter = *recon_filter_dev(f);
    // the camera kernel writes one coordinate pair per sample from now on
    if (t->hasFilter && t->maxRays) {
        int r = t->imgCoords.alloc(size_t(t->maxRays / 2) * 8);
        if (r) return r;
    }
    // the image's .w changes meaning (weight sum vs frame count): start over
    if (t->image.p) MRB_CUDA(cudaMemsetAsync(t->image.p, 0, t->image.bytes, t->stream));
    t->graphDirty = true;
    return 0;
}

int mrb_tracer_svo_info(mrb_tracer* t, uint32_t* info, float* params) {
    if (!t || !t->wfpg) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_svo(t);
    if (r) return r;
    svo_info(t->svo, t->svoP, info, params);
    return 0;
}

int mrb_tracer_svo_export(mrb_tracer* t, uint64_t* nodes, uint32_t* leafParents,
                          uint64_t* leafCodes, uint32_t* leafNormSpec, uint32_t* leafLight,
                          uint32_t* levelOffsets, uint32_t* nodeNormSpec, uint64_t* leafIrr,
                          uint32_t* leafCnt, uint32_t* leafAvg, uint32_t* nodeAvg) {
    if (!t || !t->wfpg) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_svo(t);
    if (r) return r;
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    if ((r = export_svo(t->svo, nodes, leafParents, leafCodes, leafNormSpec, leafLight,
                        levelOffsets)))
        return r;
    return export_payload(t->svo, nodeNormSpec, leafIrr, leafCnt, leafAvg, nodeAvg);
}

int mrb_tracer_svo_guiding(mrb_tracer* t, uint32_t* leafShadow, uint16_t* nodeFactor) {
    if (!t || !t->wfpg) return MRB_E_ARG;
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_svo(t);
    if (r) return r;
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    if (svo_copy(leafShadow, t->svo.leafShadow, size_t(t->svo.leafCount) * 8) ||
        svo_copy(nodeFactor, t->svo.nodeFactor, size_t(t->svo.nodeCount) * 2))
        return MRB_E_CUDA;
    return 0;
}

int mrb_tracer_guide_export(mrb_tracer* t, uint32_t* count, uint32_t* samples, uint32_t* guide2,
                            uint32_t* sortedBinKey, uint32_t* sortedRid) {
    if (!t || !t->wfpg || !t->working || t->depth == 0) {
        set_error("guide export: render at least one step of a WFPG frame first");
        return MRB_E_STATE;
    }
    const int cur = (t->depth - 1) & 1;
    uint32_t n = 0;
    MRB_CUDA(cudaMemcpyAsync(&n, t->count.as<uint32_t>() + cur, 4, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    if (count) *count = n;
    if (samples && n) {
        std::vector<RayAux> aux(n);
        MRB_CUDA(cudaMemcpy(aux.data(), t->aux[cur].p, size_t(n) * sizeof(RayAux),
                            cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++) samples[i] = aux[i].sample;
    }
    if (svo_copy(guide2, t->guideBuf.p, size_t(n) * 8) ||
        svo_copy(sortedBinKey, t->binKey.p, size_t(n) * 4) ||
        svo_copy(sortedRid, t->binRid.p, size_t(n) * 4))
        return MRB_E_CUDA;
    return 0;
}

int mrb_tracer_stats(mrb_tracer* t, uint64_t* rays, uint32_t* frames) {
    if (!t) return MRB_E_ARG;
    unsigned long long c = 0;
    if (t->counters.p) {
        MRB_CUDA(cudaMemcpyAsync(&c, t->counters.p, 8, cudaMemcpyDeviceToHost, t->stream));
        MRB_CUDA(cudaStreamSynchronize(t->stream));
    }
    if (rays) *rays = c;
    if (frames) *frames = t->frames;
    return 0;
}

void* mrb_tracer_stream(mrb_tracer* t) { return t ? static_cast<void*>(t->stream) : nullptr; }

int mrb_tracer_launches_per_frame(mrb_tracer* t) {
    if (!t) return MRB_E_ARG;
    return static_cast<int>(launches_per_frame(t));
}

int mrb_tracer_profile_frame(mrb_tracer* t, float* stageMs, uint64_t* work) {
    float all[kStageCount] = {};
    int r = mrb_tracer_profile_stages(t, all, kStageCount, work);
    if (r) return r;
    // the five-stage form folds the finalize stages into "resolve"
    for (int i = 0; i < 4; i++) stageMs[i] = all[i];
    stageMs[kStResolve] = all[kStResolve] + all[kStDeposit] + all[kStNormalize] + all[kStLearned];
    return 0;
}

int mrb_tracer_profile_stages(mrb_tracer* t, float* stageMs, uint32_t nStages, uint64_t* work) {
    if (!t || !stageMs || !work) return MRB_E_ARG;
    if (!t->camSet) {
        set_error("tracer: camera not set");
        return MRB_E_STATE;
    }
    if (set_device(t->sys)) return MRB_E_CUDA;
    int r = ensure_buffers(t);
    if (r) return r;
    StageTimer tm;
    for (auto& e : tm.ev) MRB_CUDA(cudaEventCreate(&e));
    DBuf wc;
    if ((r = wc.alloc(16))) return r;
    MRB_CUDA(cudaMemsetAsync(wc.p, 0, 16, t->stream));
    unsigned long long rays0 = 0, rays1 = 0;
    MRB_CUDA(cudaMemcpyAsync(&rays0, t->counters.p, 8, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    MRB_CUDA(cudaEventRecord(tm.ev[6], t->stream));
    if ((r = step_camera(t))) return r;
    MRB_CUDA(cudaEventRecord(tm.ev[7], t->stream));
    MRB_CUDA(cudaEventSynchronize(tm.ev[7]));
    MRB_CUDA(cudaEventElapsedTime(&tm.ms[kStCamera], tm.ev[6], tm.ev[7]));
    for (uint32_t d = 0; d < t->maxDepth; d++)
        if ((r = step_depth(t, d, &tm, wc.as<unsigned long long>()))) return r;
    if ((r = step_finalize(t, &tm))) return r;
    unsigned long long w[2] = {0, 0};
    MRB_CUDA(cudaMemcpyAsync(w, wc.p, 16, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaMemcpyAsync(&rays1, t->counters.p, 8, cudaMemcpyDeviceToHost, t->stream));
    MRB_CUDA(cudaStreamSynchronize(t->stream));
    for (auto& e : tm.ev) cudaEventDestroy(e);
    for (uint32_t i = 0; i < nStages && i < uint32_t(kStageCount); i++) stageMs[i] = tm.ms[i];
    work[0] = rays1 - rays0;
    work[1] = w[0];
    work[2] = w[1];
    work[3] = t->maxDepth;
    t->frames++;
    return check_device_errors(t);
}

// ---- kernel-level ----------------------------------------------------------
int mrb_morton_codes(const float* pos, const uint32_t* idx, uint32_t n, float* triAabb,
                     float* extent, uint64_t* codes, void* stream) {
    return lbvh_morton(pos, idx, n, triAabb, extent, codes, nullptr, extent + 6,
                       static_cast<cudaStream_t>(stream));
}

size_t mrb_radix_sort_temp_bytes(uint32_t n, int keyBytes, int b, int e) {
    return radix_sort_temp_bytes(n, keyBytes, b, e);
}

int mrb_radix_sort_pairs_u64(uint64_t* k, uint32_t* v, uint32_t n, int b, int e, int desc,
                             void* tmp, size_t tb, void* stream) {
    if (b < 0 || e > 64 || b > e) {
        set_error("bit range [%d, %d) invalid for 64-bit keys", b, e);
        return MRB_E_ARG;
    }
    return radix_sort_pairs<uint64_t>(k, v, nullptr, n, b, e, desc != 0, tmp, tb,
                                      static_cast<cudaStream_t>(stream), false);
}

int mrb_radix_sort_pairs_u32(uint32_t* k, uint32_t* v, uint32_t n, int b, int e, int desc,
                             void* tmp, size_t tb, void* stream) {
    if (b < 0 || e > 32 || b > e) {
        set_error("bit range [%d, %d) invalid for 32-bit keys", b, e);
        return MRB_E_ARG;
    }
    return radix_sort_pairs<uint32_t>(k, v, nullptr, n, b, e, desc != 0, tmp, tb,
                                      static_cast<cudaStream_t>(stream), false);
}

int mrb_lbvh_hierarchy(const uint64_t* codes, const uint32_t* sorted, const float* triAabb,
                       uint32_t n, uint32_t* left, uint32_t* right, uint32_t* parent, float* inner,
                       uint32_t* root, uint32_t* scratch, void* nodes, void* stream) {
    const size_t ni = n > 1 ? n - 1 : 1;
    LbvhArrays a{left, right, parent, inner, scratch, scratch + ni, scratch + 2 * ni, root,
                 static_cast<BvhNode*>(nodes)};
    return lbvh_hierarchy(codes, sorted, triAabb, n, a, static_cast<cudaStream_t>(stream));
}

size_t mrb_partition_temp_bytes(uint32_t n, uint32_t idBits) {
    return radix_sort_temp_bytes(n, 4, 0, 3 + int(idBits)) + 256 + 16;
}

int mrb_partition(const uint32_t* keys, uint32_t n, uint32_t idBits, uint32_t* sortedIds,
                  uint32_t* sortedDense, uint32_t* pOff, uint32_t* pEnd, uint32_t* nonNull,
                  void* tmp, size_t tb, void* stream) {
    if (idBits == 0 || idBits > 24) {
        set_error("id bits %u out of [1, 24]", idBits);
        return MRB_E_ARG;
    }
    if (tb < mrb_partition_temp_bytes(n, idBits)) {
        set_error("partition scratch too small");
        return MRB_E_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the element count is staged in the first word of the scratch
    uint32_t* dCount = static_cast<uint32_t*>(tmp);
    void* sortTmp = static_cast<unsigned char*>(tmp) + 256;
    size_t sortBytes = tb - 256;
    MRB_CUDA(cudaMemcpyAsync(dCount, &n, 4, cudaMemcpyHostToDevice, st));
    PortionTable pt{pOff, pEnd, nonNull};
    int r;
    if ((r = dense_keys(keys, dCount, n, idBits, sortedDense, pt, st))) return r;
    if ((r = radix_sort_pairs<uint32_t>(sortedDense, sortedIds, dCount, n, 0, 3 + int(idBits), true,
                                        sortTmp, sortBytes, st, true)))
        return r;
    if ((r = find_portions(sortedDense, dCount, n, idBits, pt, st))) return r;
    MRB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

}  // extern "C"
