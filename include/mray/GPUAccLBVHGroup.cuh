// MRay-side binding of the meturay_b200 accelerator group and base
// accelerator: GPUAcceleratorGroupI and GPUBaseAcceleratorI
// (TracerCUDA/GPUAcceleratorI.h:46-173) implemented over the C ABI of
// include/mrb200.h.  A maintainer adds this header to MRay's TracerCUDA
// build (nvcc) and registers the two classes under the accelerator name
// "LBVH" next to "BasicBVH" (TracerLogicGenerator.cu:108-140); scene files
// then select it with "Accelerators": [{"type": "LBVH"}].
//
// The group reads the triangle primitive group's device arrays (positions,
// tangent rotations, 64-bit indices) once at InitializeGroup and packs each
// surface's primitive batches into one contiguous triangle range, keeping
// the primitive group's own primitive ids (reported by Hit) and applying
// key expansion (material key id + index in the batch, as
// GPUAcceleratorCommonKC.cuh:140-152 does).  Transforms are read from the
// device objects through GPUTransformI::GetLocalToWorldAsMatrix.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <vector>

#include "RayLib/SceneError.h"
#include "RayLib/SceneNodeI.h"
#include "RayLib/TracerError.h"
#include "TracerCUDA/CudaSystem.h"
#include "TracerCUDA/GPUAcceleratorI.h"
#include "TracerCUDA/GPUPrimitiveTriangle.h"
#include "TracerCUDA/GPUTransformI.h"
#include "TracerCUDA/RayStructs.h"

#include "mrb200.h"

namespace mrb_mray {

static_assert(sizeof(Vector3f) == 12, "sample outputs are packed float triples");
static_assert(sizeof(RayGMem) == 32, "RayGMem is position, tMin, direction, tMax");
static_assert(sizeof(HitKey) == 4 && sizeof(TransformId) == 4 && sizeof(PrimitiveId) == 8,
              "the C ABI's key and id widths");
static_assert(sizeof(QuatF) == 16, "tangent rotations are w, x, y, z floats");

// Rows of every transform's local-to-world Matrix4x4 (column-major,
// operator()(row, column)), as the row-major 3x4 of the C ABI.
static __global__ void KCLocalToWorldRows(float* out, const GPUTransformI** transforms,
                                          uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const Matrix4x4 m = transforms[i]->GetLocalToWorldAsMatrix();
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) out[12 * i + 4 * r + c] = m(r, c);
}

inline AABB3f ToAABB(const float* b) {
    return AABB3f(Vector3f(b[0], b[1], b[2]), Vector3f(b[3], b[4], b[5]));
}

class GPUAccLBVHGroup final : public GPUAcceleratorGroupI {
    const GPUPrimitiveTriangle& prims;
    mrb_system* system = nullptr;
    mrb_accel_group* group = nullptr;
    std::map<uint32_t, uint32_t> innerIds;     // surface id -> accelerator index
    std::vector<uint32_t> surfaceIds;          // accelerator index -> surface id
    std::vector<mrb_surface> ranges;           // packed triangle range per surface
    std::vector<uint32_t> surfaceTransforms;   // global transform index per surface
    size_t triCount = 0;
    SurfaceAABBList aabbs;
    const GPUTransformI** dTransforms = nullptr;
    uint32_t identityIndex = 0;
    uint64_t sampleSeed = 0;

    static cudaStream_t Stream() { return static_cast<cudaStream_t>(0); }

   public:
    static const char* TypeName() { return "LBVH"; }

    explicit GPUAccLBVHGroup(const GPUPrimitiveGroupI& p)
        : prims(static_cast<const GPUPrimitiveTriangle&>(p)) {}
    ~GPUAccLBVHGroup() override {
        if (group) mrb_accel_group_destroy(group);
        if (system) mrb_system_destroy(system);
    }
    const char* Type() const override { return TypeName(); }

    SceneError InitializeGroup(const SceneNodePtr&,
                               const std::map<uint32_t, SurfaceDefinition>& surfaceList,
                               double) override {
        const TriData d = PrimDataAccessor::Data(prims);
        const uint64_t vertexCount = prims.TotalDataCount();
        const uint64_t primCount = prims.TotalPrimitiveCount();
        std::vector<float> pos(3 * vertexCount), tbn(4 * vertexCount);
        std::vector<uint64_t> idx64(3 * primCount);
        if (cudaMemcpy(pos.data(), d.positions, pos.size() * 4, cudaMemcpyDeviceToHost) ||
            cudaMemcpy(tbn.data(), d.tbnRotations, tbn.size() * 4, cudaMemcpyDeviceToHost) ||
            cudaMemcpy(idx64.data(), d.indexList, idx64.size() * 8, cudaMemcpyDeviceToHost))
            return SceneError::PRIMITIVE_TYPE_INTERNAL_ERROR;
        std::vector<uint32_t> idx, keys;
        std::vector<uint8_t> cull;
        std::vector<uint64_t> primIds;
        for (const auto& [surfaceId, def] : surfaceList) {
            const uint32_t begin = static_cast<uint32_t>(keys.size());
            for (const IdKeyPair& pair : def.primIdWorkKeyPairs) {
                if (pair.first == std::numeric_limits<uint32_t>::max()) break;
                const Vector2ul range = prims.PrimitiveBatchRange(pair.first);
                const uint8_t culled = prims.PrimitiveBatchBackFaceCulled(pair.first) ? 1 : 0;
                for (uint64_t t = range[0]; t < range[1]; t++) {
                    for (int k = 0; k < 3; k++) idx.push_back(static_cast<uint32_t>(idx64[3 * t + k]));
                    HitKey key = pair.second;
                    if (def.doKeyExpansion)
                        key = HitKey::CombinedKey(
                            HitKey::FetchBatchPortion(key),
                            static_cast<HitKey::Type>(HitKey::FetchIdPortion(key) + (t - range[0])));
                    keys.push_back(static_cast<HitKey::Type>(key));
                    cull.push_back(culled);
                    primIds.push_back(t);
                }
            }
            const uint32_t end = static_cast<uint32_t>(keys.size());
            if (end == begin) return SceneError::PRIMITIVE_TYPE_INTERNAL_ERROR;
            innerIds.emplace(surfaceId, static_cast<uint32_t>(ranges.size()));
            surfaceIds.push_back(surfaceId);
            ranges.push_back(mrb_surface{begin, end, def.globalTransformIndex});
            surfaceTransforms.push_back(def.globalTransformIndex);
        }
        triCount = keys.size();
        int device = 0;
        cudaGetDevice(&device);
        if (mrb_system_create(device, &system) ||
            mrb_accel_group_create(system, pos.data(), static_cast<uint32_t>(vertexCount),
                                   tbn.data(), idx.data(), keys.data(), cull.data(), primIds.data(),
                                   static_cast<uint32_t>(triCount), ranges.data(),
                                   static_cast<uint32_t>(ranges.size()), &group))
            return SceneError::PRIMITIVE_TYPE_INTERNAL_ERROR;
        return SceneError::OK;
    }

    uint32_t InnerId(uint32_t surfaceId) const override { return innerIds.at(surfaceId); }

    TracerError ConstructAccelerators(const CudaSystem&) override {
        if (!group) return TracerError::UNABLE_TO_CONSTRUCT_ACCELERATOR;
        // the global array's length is not passed along; every index read here
        // (the surfaces' transforms and the identity) is one of its entries
        uint32_t count = identityIndex + 1;
        for (uint32_t t : surfaceTransforms) count = std::max(count, t + 1);
        if (dTransforms) {
            float* dRows = nullptr;
            std::vector<float> rows(12 * size_t(count));
            if (cudaMalloc(&dRows, rows.size() * 4)) return TracerError::UNABLE_TO_CONSTRUCT_ACCELERATOR;
            KCLocalToWorldRows<<<(count + 127) / 128, 128>>>(dRows, dTransforms, count);
            const bool ok = cudaMemcpy(rows.data(), dRows, rows.size() * 4,
                                       cudaMemcpyDeviceToHost) == cudaSuccess;
            cudaFree(dRows);
            if (!ok || mrb_accel_group_attach_transforms(group, rows.data(), count, identityIndex))
                return TracerError::UNABLE_TO_CONSTRUCT_ACCELERATOR;
        }
        if (mrb_accel_group_construct(group, Stream()))
            return TracerError::UNABLE_TO_CONSTRUCT_ACCELERATOR;
        std::vector<float> boxes(6 * ranges.size());
        mrb_accel_group_aabbs(group, boxes.data(), static_cast<uint32_t>(ranges.size()));
        aabbs.clear();
        for (size_t i = 0; i < ranges.size(); i++) aabbs.emplace(surfaceIds[i], ToAABB(&boxes[6 * i]));
        return TracerError::OK;
    }
    // The C ABI builds every surface of the group together.
    TracerError ConstructAccelerator(uint32_t, const CudaSystem& s) override {
        return ConstructAccelerators(s);
    }
    TracerError ConstructAccelerators(const std::vector<uint32_t>&, const CudaSystem& s) override {
        return ConstructAccelerators(s);
    }
    TracerError DestroyAccelerators(const CudaSystem&) override { return TracerError::OK; }
    TracerError DestroyAccelerator(uint32_t, const CudaSystem&) override { return TracerError::OK; }
    TracerError DestroyAccelerators(const std::vector<uint32_t>&, const CudaSystem&) override {
        return TracerError::OK;
    }

    // nodes (64 B) + sorted triangles (48 B) + Morton code / index (12 B)
    size_t UsedGPUMemory() const override { return triCount * 124; }
    size_t UsedCPUMemory() const override { return ranges.size() * sizeof(mrb_surface); }

    void Hit(const CudaGPU&, HitKey* dMaterialKeys, TransformId* dTransformIds,
             PrimitiveId* dPrimitiveIds, HitStructPtr dHitStructs, RayGMem* dRays,
             const RayId* dRayIds, const HitKey* dAcceleratorKeys,
             const uint32_t rayCount) const override {
        mrb_accel_group_hit(group, reinterpret_cast<uint32_t*>(dMaterialKeys), dTransformIds,
                            dPrimitiveIds, &dHitStructs.Ref<Byte>(0), dHitStructs.CombinedSize(),
                            dRays, dRayIds, reinterpret_cast<const uint32_t*>(dAcceleratorKeys),
                            rayCount, Stream());
    }

    const SurfaceAABBList& AcceleratorAABBs() const override { return aabbs; }
    const GPUPrimitiveGroupI& PrimitiveGroup() const override { return prims; }
    void AttachGlobalTransformArray(const GPUTransformI** deviceTransforms,
                                    uint32_t identityTransformIndex) override {
        dTransforms = deviceTransforms;
        identityIndex = identityTransformIndex;
    }
    size_t AcceleratorCount() const override { return ranges.size(); }
    size_t TotalPrimitiveCount() const override { return triCount; }
    float TotalApproximateArea(const CudaSystem&) const override {
        float area = 0.0f;
        mrb_accel_group_total_area(group, &area, Stream());
        return area;
    }
    // The Sobol generator is not used: the samples come from Philox keyed by
    // a per-group call counter.
    void SampleAreaWeightedPoints(Vector3f* dPositions, Vector3f* dNormals, RNGSobolCPU&,
                                  uint32_t surfacePatchCount, const CudaSystem&) const override {
        mrb_accel_group_sample_points(group, reinterpret_cast<float*>(dPositions),
                                      reinterpret_cast<float*>(dNormals), surfacePatchCount,
                                      const_cast<GPUAccLBVHGroup*>(this)->sampleSeed++, Stream());
    }
    void EachPrimVoxelCount(uint64_t* dVoxCounts, uint32_t resolutionXYZ,
                            const AABB3f& sceneAABB, const CudaSystem&) const override {
        const float box[6] = {sceneAABB.Min()[0], sceneAABB.Min()[1], sceneAABB.Min()[2],
                              sceneAABB.Max()[0], sceneAABB.Max()[1], sceneAABB.Max()[2]};
        mrb_accel_group_voxel_counts(group, dVoxCounts, resolutionXYZ, box, Stream());
    }
    void VoxelizeSurfaces(uint64_t* dVoxels, Vector2us* dVoxelNormals, HitKey* gVoxelLightKeys,
                          const uint64_t* dVoxelOffsets, const HitKey* dLightKeys,
                          uint32_t totalLightCount, uint32_t resolutionXYZ,
                          const AABB3f& sceneAABB, const CudaSystem&) const override {
        const float box[6] = {sceneAABB.Min()[0], sceneAABB.Min()[1], sceneAABB.Min()[2],
                              sceneAABB.Max()[0], sceneAABB.Max()[1], sceneAABB.Max()[2]};
        mrb_accel_group_voxelize(group, dVoxels, reinterpret_cast<uint32_t*>(dVoxelNormals),
                                 reinterpret_cast<uint32_t*>(gVoxelLightKeys), dVoxelOffsets,
                                 reinterpret_cast<const uint32_t*>(dLightKeys), totalLightCount,
                                 resolutionXYZ, box, Stream());
    }
};

class GPUBaseAccLBVH final : public GPUBaseAcceleratorI {
    mrb_system* system = nullptr;
    mrb_base_accel* base = nullptr;
    std::map<uint32_t, HitKey> keys;  // surface id -> accelerator key
    AABB3f extents;

   public:
    static const char* TypeName() { return "LBVH"; }

    GPUBaseAccLBVH() = default;
    ~GPUBaseAccLBVH() override {
        if (base) mrb_base_accel_destroy(base);
        if (system) mrb_system_destroy(system);
    }

    const char* Type() const override { return TypeName(); }
    void GetReady(const CudaSystem&, uint32_t rayCount) override {
        mrb_base_accel_get_ready(base, rayCount, nullptr);
    }
    void Hit(const CudaSystem&, HitKey* dMaterialKeys, const RayGMem* dRays, const RayId* dRayIds,
             const uint32_t rayCount) const override {
        mrb_base_accel_hit(base, reinterpret_cast<uint32_t*>(dMaterialKeys), dRays, dRayIds,
                           rayCount, nullptr);
    }
    SceneError Initialize(const SceneNodePtr&, const std::map<uint32_t, HitKey>& surfaceKeys) override {
        keys = surfaceKeys;
        int device = 0;
        cudaGetDevice(&device);
        if (mrb_system_create(device, &system) || mrb_base_accel_create(system, &base))
            return SceneError::PRIMITIVE_TYPE_INTERNAL_ERROR;
        return SceneError::OK;
    }
    TracerError Construct(const CudaSystem&, const SurfaceAABBList& surfaceAabbs) override {
        std::vector<float> boxes;
        std::vector<uint32_t> accKeys;
        for (const auto& [surfaceId, box] : surfaceAabbs) {
            const auto k = keys.find(surfaceId);
            if (k == keys.end()) return TracerError::UNABLE_TO_CONSTRUCT_BASE_ACCELERATOR;
            for (int c = 0; c < 3; c++) boxes.push_back(box.Min()[c]);
            for (int c = 0; c < 3; c++) boxes.push_back(box.Max()[c]);
            accKeys.push_back(static_cast<HitKey::Type>(k->second));
        }
        if (accKeys.empty() ||
            mrb_base_accel_construct(base, boxes.data(), accKeys.data(),
                                     static_cast<uint32_t>(accKeys.size())))
            return TracerError::UNABLE_TO_CONSTRUCT_BASE_ACCELERATOR;
        float e[6];
        mrb_base_accel_extents(base, e);
        extents = ToAABB(e);
        return TracerError::OK;
    }
    TracerError Destruct(const CudaSystem&) override { return TracerError::OK; }
    const AABB3f& SceneExtents() const override { return extents; }
    size_t UsedGPUMemory() const override { return keys.size() * 40; }
    size_t UsedCPUMemory() const override { return keys.size() * 40; }
};

}  // namespace mrb_mray
