// Host objects shared by the runtime's translation units: device buffers,
// the tracer system and the scene (triangle group, materials, lights and
// their accelerators).  Internal to the library; the C ABI exposes them as
// opaque handles.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "svo.cuh"
#include "wide.cuh"

namespace mrb {

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    int alloc(size_t b) {
        if (b <= bytes && p) return 0;
        release();
        if (b == 0) return 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
            p = nullptr;
            return MRB_E_OOM;
        }
        bytes = b;
        return 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
    void swap(DBuf& o) {
        std::swap(p, o.p);
        std::swap(bytes, o.bytes);
    }
};

template <class T>
inline int upload(DBuf& b, const std::vector<T>& v) {
    if (v.empty()) {
        b.release();
        return 0;
    }
    int r = b.alloc(v.size() * sizeof(T));
    if (r) return r;
    MRB_CUDA(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

}  // namespace mrb

// The objects are the C ABI's opaque handle types, so they live at global
// scope; their members use the library's types.
using namespace mrb;

// ===========================================================================
// Objects
// ===========================================================================
struct mrb_system {
    int device = 0;
    cudaStream_t stream = nullptr;
};

struct mrb_scene {
    mrb_system* sys = nullptr;
    uint32_t V = 0, T = 0;
    std::vector<float> tbn;
    std::vector<uint32_t> triKey;
    std::vector<float> lambert, metal, refract, lightRad, lambertC, unreal;
    std::vector<uint32_t> refractMed, lightPrim;
    std::vector<float> mediumIor;
    uint32_t baseMedium = 0;
    uint32_t idBits = 1;
    DBuf dPos, dTbn, dIdx, dKey, dCull, dLambert, dMetal, dRefract, dRefractMed, dLightRad,
        dLightPrim, dMediumIor, dLambertC, dUnreal;
    // LBVH
    bool built = false;
    DBuf aTriAabb, aExtent, aCodes, aSorted, aLeft, aRight, aParent, aInner, aScratch, aRoot,
        aNodes, aTv0, aTe0, aTe1, aSortTemp;
    int rootInner = 0;
    // sparse voxel octree (path-guiding radiance cache)
    bool svoBuilt = false;
    SvoParams svoP{};
    SvoResult svo;
    ~mrb_scene() {
        if (svoBuilt) svo_free(svo);
    }
    // 8-wide quantised traversal layout, collapsed from the PLOC tree built
    // over the LBVH's sorted leaves (wideTree 1) or from the LBVH itself (0)
    DBuf wNodes, wTv0, wTe0, wTe1, wScratch;
    uint32_t wNodeCount = 0;
    int traversal = 1;  // 0: binary LBVH nodes, 1: 8-wide nodes
    int wideTree = 2;        // 0 LBVH, 1 PLOC, 2 the one with less inner-box area
    int wideCollapse = 2;    // kWideCollapseGreedy / kWideCollapseSah / 2: the one the probe reads less of
    int wideCollapseUsed = 1;
    double collapseProbeBytes[2] = {0.0, 0.0};  // per collapse (automatic choice only)
    // traversal kernel (WideOrder), or MRB_WIDE_AUTO: the fastest as timed
    int wideOrderMode = MRB_WIDE_AUTO;
    int wideOrder = 0;  // in use where no tracer has tuned its own
    float wideOrderMs[kWideOrders] = {};
    // bumped whenever the traversal choice changes, so that captured frames
    // and tuned per-depth kernels are redone
    uint32_t traceEpoch = 0;
    int wideTreeUsed = 0;
    uint32_t plocSteps = 0;
    double areaLbvh = 0.0, areaPloc = 0.0;  // sums of inner half areas
    // the alternate 8-wide layout (the other collapse; automatic choice only)
    DBuf aNodes2, aTv02, aTe02, aTe12;
    uint32_t wAltNodeCount = 0;
    WideAccelDev wideAlt() const {
        WideAccelDev a{};
        a.nodes = aNodes2.as<WideNode>();
        a.tv0 = aTv02.as<float4>();
        a.te0 = aTe02.as<float4>();
        a.te1 = aTe12.as<float4>();
        a.nodeCount = wAltNodeCount;
        a.triCount = T;
        return a;
    }
    WideAccelDev wide() const {
        WideAccelDev a{};
        a.nodes = wNodes.as<WideNode>();
        a.tv0 = wTv0.as<float4>();
        a.te0 = wTe0.as<float4>();
        a.te1 = wTe1.as<float4>();
        a.nodeCount = wNodeCount;
        a.triCount = T;
        return a;
    }
    SceneDev dev() const {
        SceneDev s{};
        s.vertexCount = V;
        s.triCount = T;
        s.pos = dPos.as<float>();
        s.tbn = dTbn.as<float4>();
        s.idx = dIdx.as<uint32_t>();
        s.triKey = dKey.as<uint32_t>();
        s.triCull = dCull.as<uint8_t>();
        s.lambertAlbedo = dLambert.as<float>();
        s.metalParams = dMetal.as<float>();
        s.refractAlbedo = dRefract.as<float>();
        s.refractMedium = dRefractMed.as<uint32_t>();
        s.lambertCAlbedo = dLambertC.as<float>();
        s.unrealParams = dUnreal.as<float>();
        s.lightRadiance = dLightRad.as<float>();
        s.lightPrim = dLightPrim.as<uint32_t>();
        s.lightCount = static_cast<uint32_t>(lightPrim.size());
        s.mediumIor = dMediumIor.as<float>();
        s.baseMedium = baseMedium;
        return s;
    }
    AccelDev accel() const {
        AccelDev a{};
        a.nodes = aNodes.as<BvhNode>();
        a.tv0 = aTv0.as<float4>();
        a.te0 = aTe0.as<float4>();
        a.te1 = aTe1.as<float4>();
        a.root = rootInner;
        a.triCount = T;
        return a;
    }
};
