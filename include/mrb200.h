/*
 * meturay_b200 -- C ABI of the B200 wavefront path-tracing core.
 *
 * The library (meturay_b200/libmrb200.so) replaces the MRay
 * (yalcinerbora/meturay) TracerCUDA plugin on its hot path: the "LBVH"
 * triangle accelerator group and the plain wavefront PathTracer.  Every
 * object entry point names the reference interface it stands in for.
 * Signatures use plain pointers and sizes only.
 *
 * Conventions
 *   - Return value: 0 (MRB_OK) on success, a negative MRB_E* code on
 *     failure; mrb_last_error() then describes the failure (per thread).
 *     Nothing aborts the process (reference: TracerError values,
 *     RayLib/TracerError.h, and TracerException on GPU OOM,
 *     RayLib/CudaCheck.h:31-38, become status codes here).
 *   - "d_" pointers are device pointers on the current CUDA device; "stream"
 *     is a cudaStream_t passed as void* (NULL = legacy default stream).
 *   - HitKey layout: batch << 24 | id (RayLib/HitStructs.h:154); batches:
 *     0 null, 1 Lambert, 2 Metal, 3 Refract, 4 primitive light, 5 LambertC,
 *     6 Unreal.
 */
#ifndef MRB200_H
#define MRB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MRB_OK 0
#define MRB_E_ARG (-1)
#define MRB_E_CUDA (-2)
#define MRB_E_OOM (-3)
#define MRB_E_STATE (-4)
#define MRB_E_UNSUPPORTED (-5)
#define MRB_E_DEVICE (-6) /* a device-side bounded wait or stack limit gave up */

typedef struct mrb_system mrb_system;
typedef struct mrb_scene mrb_scene;
typedef struct mrb_tracer mrb_tracer;

/* Material types of a scene description (JSON names of the reference). */
#define MRB_MAT_LAMBERT 1 /* "Lambert"  LambertMaterialKC.cuh:12-111 */
#define MRB_MAT_METAL 2   /* "Metal"    MetalGlassMaterialsKC.cuh:11-222 */
#define MRB_MAT_REFRACT 3 /* "Refract"  SimpleMaterialsKC.cuh:172-302 */
#define MRB_MAT_LIGHT 4   /* primitive-backed light, GPULightPrimitive.cuh */
#define MRB_MAT_LAMBERTC 5 /* "LambertC" SimpleMaterialsKC.cuh:16-103 */
#define MRB_MAT_UNREAL 6  /* "Unreal"   UnrealMaterialKC.cuh:19-359 */

typedef struct mrb_material {
    uint32_t type;
    float albedo[3];   /* Lambert / Refract */
    float eta[3];      /* Metal */
    float k[3];        /* Metal */
    float specular[3]; /* Metal (Unreal uses specular[0]) */
    float roughness;   /* Metal, Unreal */
    float metallic;    /* Unreal */
    uint32_t medium;   /* Refract: medium index inside the surface */
    float radiance[3]; /* Light */
} mrb_material;

typedef struct mrb_scene_desc {
    uint32_t vertex_count;
    uint32_t triangle_count;
    const float* positions;      /* vertex_count * 3 */
    const float* normals;        /* vertex_count * 3 */
    const float* uvs;            /* vertex_count * 2, may be NULL */
    const uint32_t* indices;     /* triangle_count * 3 */
    const uint32_t* tri_material;/* triangle_count, index into materials */
    const uint8_t* tri_cull;     /* triangle_count, may be NULL (two-sided) */
    uint32_t material_count;
    const mrb_material* materials;
    uint32_t medium_count;       /* homogeneous media without absorption */
    const float* medium_ior;     /* medium_count */
    uint32_t base_medium;
} mrb_scene_desc;

/* Pinhole camera node ("Pinhole": position, gaze, up, planes, fov in
 * radians; GPUCameraPinhole.cuh:83-106). */
typedef struct mrb_camera {
    float position[3];
    float gaze[3];
    float up[3];
    float near_far[2];
    float fov[2];
} mrb_camera;

/* ---- errors ---------------------------------------------------------- */
const char* mrb_last_error(void);

/* ---- tracer system: TracerSystemI (RayLib/TracerSystemI.h:34-50) ------
 * replaces GenerateTracerSystem / DeleteTracerSystem
 * (TracerCUDA/EntryPoint.h:12-16) plus TracerSystemI::Initialize. */
int mrb_system_create(int device, mrb_system** out);
void mrb_system_destroy(mrb_system* sys);

/* ---- scene: TracerSystemI::GenerateScene (GPUSceneJson.cpp:163-360).
 * Builds per-vertex tangent-space rotations as GPUPrimitiveTriangle.cpp:
 * 160-320 does and uploads the scene to the device. */
int mrb_scene_create(mrb_system* sys, const mrb_scene_desc* desc, mrb_scene** out);
void mrb_scene_destroy(mrb_scene* scene);
/* counts[0..7]: triangles, vertices, lights, lambert, metal, refract,
 * media, id bits of the partition key. */
int mrb_scene_counts(const mrb_scene* scene, uint32_t* counts8);
/* Host copies of the device-side scene arrays: tbn (vertex_count*4,
 * w,x,y,z), tri_key (triangle_count), lambert (3 each), metal (10 each:
 * eta3 k3 spec3 roughness), refract albedo (3 each), refract medium,
 * light radiance (3 each), light primitive.  Any pointer may be NULL. */
int mrb_scene_export(const mrb_scene* scene, float* tbn, uint32_t* tri_key, float* lambert,
                     float* metal, float* refract, uint32_t* refract_medium,
                     float* light_radiance, uint32_t* light_prim);

/* LambertC albedo (3 each) and Unreal parameters (6 each: albedo3,
 * roughness, metallic, specular); counts2 = their counts.  NULL skips. */
int mrb_scene_export_ext(const mrb_scene* scene, float* lambertc, float* unreal,
                         uint32_t* counts2);

/* ---- accelerator group "LBVH": GPUAcceleratorGroupI
 * (GPUAcceleratorI.h:46-134), drop-in for GPUAccBVHGroup
 * (GPUAcceleratorBVH.cuh:63-203). */
/* ConstructAccelerators: Morton codes, onesweep sort, hierarchy + AABBs. */
int mrb_accel_construct(mrb_scene* scene, void* stream);
/* Host copies of the build in reference numbering (LinearBVH.cuh:22-43):
 * codes/sorted_idx (n), left/right (n-1), parent (2n-1), inner AABBs
 * ((n-1)*6), root, triangle AABBs (n*6), extent (6).  NULL skips. */
int mrb_accel_export(const mrb_scene* scene, uint64_t* codes, uint32_t* sorted_idx,
                     uint32_t* left, uint32_t* right, uint32_t* parent, float* inner,
                     uint32_t* root, float* tri_aabbs, float* extent);
/* Hit (GPUAcceleratorI.h:95-108): closest hit of n rays.
 * d_ray_o[i] = (origin, tMin), d_ray_d[i] = (direction, tMax) as float4.
 * Outputs: HitKey (0 on miss), triangle index (0xFFFFFFFF on miss), t,
 * barycentrics (1-u-v, u) as TriangleHit. */
int mrb_accel_hit(const mrb_scene* scene, const float* d_ray_o, const float* d_ray_d, uint32_t n,
                  uint32_t* d_key, uint32_t* d_prim, float* d_t, float* d_bary, void* stream);

/* Traversal layout used by Hit and by tracers of this scene: 1 (default) =
 * 8-wide nodes with 8-bit quantised child boxes collapsed from the LBVH,
 * 0 = the binary LBVH nodes.  Both give the same closest distance; the
 * primitive can differ only where two triangles report the same distance. */
int mrb_accel_set_traversal(mrb_scene* scene, int mode);
/* info[4]: triangles, binary inner nodes, wide nodes, traversal mode. */
int mrb_accel_info(const mrb_scene* scene, uint32_t* info4);
/* Traversal kernel of the 8-wide layout.  Child order: sorted (exact
 * front to back: entry distances sorted, one stack entry per pushed child)
 * or octant (the collapse places children by the octant of their centroid,
 * visited in the order slot ^ ray octant; one stack entry per node group).
 * Either tests the triangles of a node's hit leaves after its eight box
 * tests.  Refill: a warp's idle
 * lanes take its next rays once eight of them are idle (a gain where path
 * lengths differ, a loss for coherent camera rays).  MRB_WIDE_AUTO
 * (default): the fastest kernel, timed first on 65,536 seeded rays over the
 * scene box at mrb_accel_construct (or at once when the accelerator is
 * built), then per depth on a tracer's own rays: the frame that
 * mrb_tracer_render_frame runs before it captures its graph traces every
 * depth's rays with every kernel and keeps the fastest per depth (once per
 * tracer and traversal setting).  Closest hits are the same with every
 * kernel, up to the choice among triangles at the same distance. */
#define MRB_WIDE_SORTED 0
#define MRB_WIDE_OCTANT 1
#define MRB_WIDE_SORTED_REFILL 2
#define MRB_WIDE_OCTANT_REFILL 3
#define MRB_WIDE_AUTO 4
/* Flag in mrb_tracer_wide_orders: the kernel runs over the scene's
 * alternate 8-wide layout (mrb_accel_wide_collapse). */
#define MRB_WIDE_ALT_LAYOUT 16
int mrb_accel_set_wide_order(mrb_scene* s, int order);
/* The kernel in use where no tracer tuned its own (MRB_WIDE_SORTED ..
 * MRB_WIDE_OCTANT_REFILL) and, in ms4 (may be NULL), the last measured
 * times per kernel (the probe's, or the per-depth sums of a tracer's
 * frame; 0 when the kernel was set rather than measured). */
int mrb_accel_wide_order(const mrb_scene* s, int* order, float* ms4);
/* The tree the 8-wide traversal layout is collapsed from (before
 * mrb_accel_construct): 0 the LBVH, 1 a PLOC tree (parallel locally-ordered
 * clustering by merged-box area) over the LBVH's Morton-sorted leaves, 2
 * (default) whichever of the two has the smaller sum of inner-box surface
 * areas.  The LBVH arrays and the binary traversal are the same either way. */
int mrb_accel_set_wide_tree(mrb_scene* s, int tree);
/* How each 8-wide node picks its children among the binary tree's
 * descendants (before mrb_accel_construct): 0 opens the internal child with
 * the largest surface area until eight children; 1 follows a bottom-up
 * dynamic program that minimises the sum of the wide nodes' surface areas
 * (Ylitie, Karras and Laine, HPG 2017, one triangle per leaf); 2 (default)
 * builds both and keeps the layout of which 65,536 seeded probe rays (origins
 * uniform in the scene box, directions uniform) read fewer bytes (node
 * visits x 80 B + triangle tests x 48 B, counted on the device, so the
 * choice is deterministic).  The traversal layout only; the LBVH arrays do
 * not change. */
int mrb_accel_set_wide_collapse(mrb_scene* s, int collapse);
/* The collapse of the scene's layout (0 or 1) and, after an automatic
 * choice, the probe bytes of each (probe_bytes2[0] largest-area-first, [1]
 * surface-area plan; zeros otherwise; may be NULL).  The automatic choice
 * keeps the other layout as the scene's alternate: a tracer whose traversal
 * kernel is automatic times every kernel over both layouts on the rays of
 * each depth of its first frame, keeps for the whole frame the layout whose
 * fastest kernels sum to less (one tree in L2 at a time) and per depth the
 * fastest kernel on it (the probe rays, spread through the scene box, need
 * not look like a camera's); every other caller traces the scene's layout. */
int mrb_accel_wide_collapse(const mrb_scene* s, int* used, double* probe_bytes2);
/* info[2]: the source used (0 LBVH, 1 PLOC), PLOC clustering steps;
 * areas[2] (may be NULL): inner half-area sums of the LBVH and PLOC trees. */
int mrb_accel_info_ext(const mrb_scene* s, uint32_t* info, double* areas);

/* ---- sparse voxel octree of the scene (the WFPG radiance cache):
 * AnisoSVOctreeCPU::Constrcut (AnisoSVO.cu:657-1188) with the accelerator
 * group's EachPrimVoxelCount / VoxelizeSurfaces (GPUAcceleratorI.h:118-134,
 * TriFunctions::Voxelize, GPUPrimitiveTriangle.h:385-620).  resolution: leaf
 * voxels per axis, a power of two in [2, 1024] (leaf depth = log2).
 * Needs mrb_accel_construct first (its extent bounds the octree). */
int mrb_svo_build(mrb_scene* scene, uint32_t resolution, void* stream);
/* info[6]: voxels before de-duplication, leaves, nodes, leaf depth,
 * resolution, level-offset count; params[7]: cube min xyz, max xyz, leaf
 * voxel size.  Either pointer may be NULL. */
int mrb_svo_info(const mrb_scene* scene, uint32_t* info6, float* params7);
/* Host copies: packed nodes (child 0-26 | parent 27-54 | child mask 55-62
 * | children-are-leaves 63; AnisoSVO.cuh:125-151), leaf parents, sorted
 * unique leaf Morton codes, leaf normal words (VoxelPayload packing, see
 * mrb_svo_export_payload), leaf light HitKeys, level offsets (depth + 2).
 * NULL skips. */
int mrb_svo_export(const mrb_scene* scene, uint64_t* nodes, uint32_t* leaf_parents,
                   uint64_t* leaf_codes, uint32_t* leaf_normals, uint32_t* leaf_lights,
                   uint32_t* level_offsets);

/* Radiance-cache payload of the scene-level octree (VoxelPayload,
 * AnisoSVO.cuh:22-114): node normal words (normal x,y 9+9 bits | length 7 |
 * specular 6 | z sign 1; the leaf words come from mrb_svo_export), leaf
 * radiance sums (2 per leaf, 2^24 fixed point), leaf sample counts (2 per
 * leaf), leaf and node averages (half2, front | back << 16).  NULL skips. */
int mrb_svo_export_payload(const mrb_scene* scene, uint32_t* node_norm_spec, uint64_t* leaf_irr,
                           uint32_t* leaf_cnt, uint32_t* leaf_avg, uint32_t* node_avg);

/* ---- scene JSON: TracerSystemI::GenerateScene's parse of an MRay scene
 * file (GPUSceneJson.cpp:150-560, RayLib/SceneIO.cpp:78-226) for the hot
 * path's subset: Pinhole cameras; Null and Primitive lights; Vacuum and
 * IOR-only Homogeneous media; Identity and Single (matrix4x4 / trs)
 * transforms, applied at load; Lambert, LambertC, Metal, Unreal, Refract
 * materials with constant parameters; in-node triangles (".nodeTriangle",
 * ".nodeTriangleIndexed") with "cullFace"; Surfaces, LightSurfaces,
 * CameraSurfaces, BaseMedium, a Null BaseBoundaryLight.  // and block
 * comments and trailing commas are accepted.  Anything else returns
 * MRB_E_UNSUPPORTED naming it.  The description's arrays stay valid until
 * mrb_json_scene_destroy; pass it to mrb_scene_create. */
typedef struct mrb_json_scene mrb_json_scene;
int mrb_json_scene_load(const char* json_text, size_t length, mrb_json_scene** out);
int mrb_json_scene_load_file(const char* path, mrb_json_scene** out);
void mrb_json_scene_destroy(mrb_json_scene* js);
int mrb_json_scene_get(const mrb_json_scene* js, mrb_scene_desc* desc, uint32_t* camera_count);
/* CameraSurfaces entry `index` as a pinhole camera (fov in radians). */
int mrb_json_scene_camera(const mrb_json_scene* js, uint32_t index, mrb_camera* cam);

/* ---- reconstruction filters: GPUReconFilterI (GPUReconFilterI.h:6-33) --
 * replaces TracerSystemI::GenerateReconFilter (TracerSystemCUDA.cpp:109-137)
 * and the "Box" / "Tent" / "Gaussian" / "Mitchell" filters
 * (GPUReconFilterBox.h, ...Tent.h, ...Gaussian.h, ...Mitchell.h).
 * Options as name/value pairs: Gaussian needs "alpha", Mitchell "b" and "c";
 * a missing one returns MRB_E_ARG naming it.  radius in [0, 64] pixels;
 * radius 0 is the Box filter's no-filter mode (one pixel, weight 1) and is
 * rejected for the other types. */
typedef struct mrb_recon_filter mrb_recon_filter;
typedef struct mrb_image mrb_image;
int mrb_recon_filter_create(const char* type, float radius, uint32_t option_count,
                            const char* const* option_names, const float* option_values,
                            mrb_recon_filter** out);
void mrb_recon_filter_destroy(mrb_recon_filter* f);
const char* mrb_recon_filter_type(const mrb_recon_filter* f);
/* Device scratch the filter holds (GPUReconFilter::UsedGPUMemory). */
size_t mrb_recon_filter_used_bytes(const mrb_recon_filter* f);
/* FilterRadiusToPixelWH (GPUReconFilterKC.cuh:10-31). */
uint32_t mrb_recon_filter_pixel_wh(float radius);
/* The filter functor evaluated on the host (pixel centre, sample). */
float mrb_recon_filter_weight(const mrb_recon_filter* f, float pixel_x, float pixel_y,
                              float sample_x, float sample_y);
/* FilterToImg (GPUReconFilter.h:59-260): splat sample_count samples
 * (d_values: channels floats each, channels = the image's 1 or 4; d_img_coords:
 * 2 floats each, image-space pixel units) into the image's pixels and sample
 * counts, every weight times scalar_multiplier.  Each pixel adds its samples
 * in ascending sample order.  Pixels outside the image's portion are not
 * written.  Allocates scratch on first use or growth. */
int mrb_recon_filter_to_img(mrb_recon_filter* f, mrb_image* img, const float* d_values,
                            uint32_t channels, const float* d_img_coords, uint32_t sample_count,
                            float scalar_multiplier, void* stream);

/* ---- image memory: ImageMemory (ImageMemory.h:14-78) ----------------------
 * Pixels (channels floats each, 1 = R_FLOAT, 4 = RGBA_FLOAT) and per-pixel
 * sample counts (weight sums) of the image portion, zeroed at creation. */
int mrb_image_create(int32_t width, int32_t height, uint32_t channels, mrb_image** out);
void mrb_image_destroy(mrb_image* img);
/* Reportion(start, end): end clamped to the resolution; reallocates, zeroed. */
int mrb_image_reportion(mrb_image* img, int32_t start_x, int32_t start_y, int32_t end_x,
                        int32_t end_y);
/* Resize(resolution): the portion must still fit. */
int mrb_image_resize(mrb_image* img, int32_t width, int32_t height);
int mrb_image_reset(mrb_image* img, void* stream);
/* info7: portion offset x, y, portion size w, h, resolution w, h, channels. */
int mrb_image_info(const mrb_image* img, int32_t* info7);
int mrb_image_device(const mrb_image* img, float** d_pixels, float** d_sample_counts);
/* GetImageToCPU (ImageMemory.cu:150-190): NaN pixels set to 1e30 magenta,
 * pixels and counts copied out, then the image reset.  Synchronises. */
int mrb_image_get(mrb_image* img, float* host_pixels, float* host_counts, void* stream);
/* Pixels divided by their sample counts, to a .exr (FLOAT) or .pfm file. */
int mrb_image_write(mrb_image* img, const char* path);

/* ---- image files (the headless stand-in for ImageIO's EXR writer,
 * ImageIO/ImageIO.cpp:290-360) ----------------------------------------------
 * pixels: width*height*channels floats, rows bottom to top as the tracers
 * produce them (EXR files store the top row first, so rows are flipped on
 * write and read).  channels 1, 3 or 4.  OpenEXR: single-part scanline,
 * uncompressed, FLOAT or HALF (half != 0) channels R,G,B(,A) or Y.  PFM:
 * "PF" RGB (the alpha of 4-channel input dropped) or "Pf" grey, little
 * endian. */
int mrb_write_exr(const char* path, const float* pixels, uint32_t width, uint32_t height,
                  uint32_t channels, int half);
int mrb_write_pfm(const char* path, const float* pixels, uint32_t width, uint32_t height,
                  uint32_t channels);
/* Read a .exr (uncompressed scanline) or .pfm file.  pixels == NULL returns
 * the size only; otherwise capacity must hold width*height*channels floats. */
int mrb_read_image(const char* path, float* pixels, size_t capacity, uint32_t* width,
                   uint32_t* height, uint32_t* channels);

/* ---- tracers: GPUTracerI (RayLib/GPUTracerI.h:24-71) ----
 * type "PathTracer" (PathTracer.cu) or "WFPGTracer" (WFPGTracer.cu, product
 * path guiding over the tracer's own voxel octree). */
int mrb_tracer_create(mrb_system* sys, mrb_scene* scene, const char* type, mrb_tracer** out);
void mrb_tracer_destroy(mrb_tracer* t);
/* SetOptions keys (PathTracer.h:17-33): "Samples", "MaxDepth",
 * "NextEventEstimation", "RussianRouletteStart", "DirectLightMIS",
 * plus "Seed" (RNG key) and "Frame" (RNG iteration counter).  WFPGTracer
 * also takes (WFPGTracer.h:25-56) "OctreeLevel", "MinRayBinLevel",
 * "BinRayCount", "DoProductPathGuiding" (true: product sampler; false: 2D
 * piecewise-constant sampler over the field), "PurePG", "SkipPG",
 * "GuideBounceAmount", "OmitDirectRadiance". */
int mrb_tracer_set_option(mrb_tracer* t, const char* name, uint64_t value);
/* Floating-point WFPG options: "BXDF-GuideMISRatio", "RFieldFilterAlpha",
 * "LearnedRate" (Adam step size of the learned guide, default 1e-2),
 * "LearnedWeightMax" (cap on a training sample's weight, 0 = none),
 * "LearnedEMA" (inference weights = moving average of the trained ones with
 * this decay per frame, [0, 1), default 0 = the trained weights).
 * Learned guiding (no counterpart in the reference), integer options of the
 * WFPG tracer: "LearnedGuiding" (0/1): a guiding network (mrb_mlp_*) trains
 * every frame from the path chains (on a side stream, overlapped with the
 * next frame) and, after "LearnedWarmupFrames" frames (default 16), its vMF
 * mixture replaces the octree product sampler (one-sample MIS with the BxDF,
 * ratio BXDF-GuideMISRatio; the last depth is not guided);
 * "LearnedWarmupOctree" (1, default: the octree guides the warm-up frames;
 * 0: the BxDF alone samples them), "LearnedTrainSteps" (Adam steps per
 * frame, default 4), "LearnedSamples" (training samples per frame, default
 * 65,536), "LearnedProductTarget" (1, default: training weights carry the
 * |cos| at the vertex, so the mixture learns L_in |cos|; 0: L_in),
 * "LearnedSeed" (weights' initial draw). */
int mrb_tracer_set_option_float(mrb_tracer* t, const char* name, double value);
/* The learned guiding network's parameters (mrb_mlp_param_count floats). */
int mrb_tracer_learned_params(mrb_tracer* t, float* host_params);
/* The last frame's training: (sum of w * -log q over its batches, sum of w),
 * each batch scored before the step that learns from it. */
int mrb_tracer_learned_loss(mrb_tracer* t, float* host_loss2);
/* String WFPG options (WFPGTracer.h:39,54): "InitialSVO" -- path of an
 * octree dump that the next GenerateWork loads instead of building the
 * octree (empty: build); "PGDataStructDumpName" -- file name of the periodic
 * dumps (default "wfpg_svo").  The integer options "PGDumpDataStruct" (0/1)
 * and "PGDataStructDumpIntervalExp" (default 2) switch the dumps on: after
 * the frames numbered interval^0, interval^1, ... the octree is written to
 * "<frame>_<name>" (WFPGTracer.cu:1733-1745). */
int mrb_tracer_set_option_string(mrb_tracer* t, const char* name, const char* value);
/* The WFPG octree in DumpSVOAsBinary's byte layout (AnisoSVO.cu:1555-1697).
 * out == NULL returns the size only.  Builds the octree if it does not
 * exist yet. */
int mrb_tracer_svo_dump(mrb_tracer* t, void* out, size_t capacity, size_t* size);
/* Replace the WFPG octree with a dump (Constrcut(data), AnisoSVO.cu:
 * 1190-1413).  Structure indices are range-checked before upload; a dump
 * that fails a check returns MRB_E_ARG naming it. */
int mrb_tracer_svo_load(mrb_tracer* t, const void* data, size_t size);
/* The WFPG tracer's octree (built at first use): info/params as
 * mrb_svo_info, and its structure plus payload as mrb_svo_export and
 * mrb_svo_export_payload.  NULL skips. */
int mrb_tracer_svo_info(mrb_tracer* t, uint32_t* info6, float* params7);
int mrb_tracer_svo_export(mrb_tracer* t, uint64_t* nodes, uint32_t* leaf_parents,
                          uint64_t* leaf_codes, uint32_t* leaf_norm_spec, uint32_t* leaf_lights,
                          uint32_t* level_offsets, uint32_t* node_norm_spec, uint64_t* leaf_irr,
                          uint32_t* leaf_cnt, uint32_t* leaf_avg, uint32_t* node_avg);
/* The octree's shadow-ray statistics (VoxelPayload dShadowRayHitLeaf /
 * dShadowRayMissLeaf and dGuidingFactorNode, AnisoSVO.cuh:75-85):
 * leaf_shadow[2 * leaf] counts the rays launched from a path vertex in the
 * leaf whose light contribution was taken (a NEE ray reaching its light, or
 * a path ray reaching a light or the boundary where the boundary work
 * accepts it), leaf_shadow[2 * leaf + 1] the NEE rays stopped by a surface
 * (DepositNEEHitMiss, WFPGTracerKC.cuh:194, 258), summed since the octree
 * was built or loaded; node_factor[node] is the binary16 guiding factor, the
 * mean of the children's miss ratios (NaN: none of the leaves below has a
 * shadow ray), as of the last NormalizeAndFilterRadiance.  NULL skips. */
int mrb_tracer_svo_guiding(mrb_tracer* t, uint32_t* leaf_shadow, uint16_t* node_factor);
/* Guide state of the wavefront shaded by the last Render() step of a WFPG
 * frame: ray count, per ray its path (sample) index and guide words (uv
 * half2 | pdf half + flags bit16 BxDF-selected, bit17 valid), and the
 * bin-sorted keys with their ray indices.  NULL skips. */
int mrb_tracer_guide_export(mrb_tracer* t, uint32_t* count, uint32_t* samples, uint32_t* guide2,
                            uint32_t* sorted_bin_key, uint32_t* sorted_rid);
int mrb_tracer_set_resolution(mrb_tracer* t, uint32_t width, uint32_t height);
/* The camera of the next frames.  The frame is copied to the device in
 * stream order (after the frames already enqueued) from one of four pinned
 * staging slots; the call waits only when the upload that last used its
 * slot, four calls back, is still queued. */
int mrb_tracer_set_camera(mrb_tracer* t, const mrb_camera* cam);
/* The camera frame as the device sees it (14 floats: position, bottom-left,
 * right, up, plane size, near/far); GPUCameraPinhole.cuh:135-162. */
int mrb_camera_frame(const mrb_camera* cam, float* out14);
/* GenerateWork / Render (1 while work remains, 0 when done) / Finalize. */
int mrb_tracer_generate_work(mrb_tracer* t, uint32_t camera_index);
int mrb_tracer_render(mrb_tracer* t);
int mrb_tracer_finalize(mrb_tracer* t);
/* GenerateWork + all Render steps + Finalize as one captured CUDA graph. */
int mrb_tracer_render_frame(mrb_tracer* t);
/* AttachReconFilter (RayTracer.cu:71-74): Finalize splats each frame's
 * samples through a copy of the filter's functor (NULL detaches). */
int mrb_tracer_set_filter(mrb_tracer* t, const mrb_recon_filter* f);
/* Per-pixel image (width*height*4) and the last frame's per-sample radiance
 * ((w*s)*(h*s)*4).  With a filter attached the image holds the filtered sums
 * (rgb = sum of weight * radiance, .w = sum of weights); without one, the
 * sum of per-frame per-pixel means with the frame count in .w.  Either way
 * rgb / w is the pixel's estimate. */
int mrb_tracer_get_image(mrb_tracer* t, float* host_rgba);
/* Asynchronous read-back for pipelined hosts: the image as it stands after
 * the work queued so far is snapshotted on the device, and copied into
 * `host_rgba` (pinned memory; width x height x 4 floats) on a separate copy
 * stream while later frames render.  The host buffer is valid after
 * mrb_tracer_wait_image.  A new call first waits for the previous copy to
 * leave the snapshot buffer. */
int mrb_tracer_get_image_async(mrb_tracer* t, float* host_rgba);
int mrb_tracer_wait_image(mrb_tracer* t);
int mrb_tracer_get_samples(mrb_tracer* t, float* host_rgba);
int mrb_tracer_reset_image(mrb_tracer* t);
/* The image's per-pixel estimate (rgb / w) as a .exr (FLOAT RGB) or .pfm file. */
int mrb_tracer_write_image(mrb_tracer* t, const char* path);
/* Rays traced (camera + path + NEE, summed over depths) since creation. */
int mrb_tracer_stats(mrb_tracer* t, uint64_t* rays_traced, uint32_t* frames);
/* Stream the tracer launches on (cudaStream_t as void*). */
void* mrb_tracer_stream(mrb_tracer* t);
/* Number of kernels one frame launches (>= 0), or a negative status. */
int mrb_tracer_launches_per_frame(mrb_tracer* t);
/* The 8-wide traversal kernel of each depth (MRB_WIDE_SORTED ..
 * MRB_WIDE_OCTANT_REFILL, with MRB_WIDE_ALT_LAYOUT set where it runs over
 * the scene's alternate layout, the other collapse, which the automatic
 * collapse keeps for tracers to time; -1 with the binary traversal) for the
 * first n depths; returns how many were written. */
int mrb_tracer_wide_orders(const mrb_tracer* t, int* orders, uint32_t n);
/* Render one frame stage by stage with CUDA events around each stage.
 * stage_ms[5]: camera, traversal, partition, shading, resolve (summed over
 * depths).  work[4]: rays traced, inner nodes visited, triangles tested,
 * depths.  The frame counts like any other. */
int mrb_tracer_profile_frame(mrb_tracer* t, float* stage_ms, uint64_t* work);
/* The same with the guided stages apart.  stage_ms[n_stages] (up to 12):
 * camera, traversal, partition, shading, reconstruction, then the octree
 * guider's clear of the bin words, binning and collapse, bin sort and
 * ranges, guide kernel (the learned guider's fused kernel counts here too),
 * and per frame the radiance deposit, the normalize-and-filter passes and
 * the learned guider's join and sample collection. */
int mrb_tracer_profile_stages(mrb_tracer* t, float* stage_ms, uint32_t n_stages, uint64_t* work);

/* ---- accelerator group and base accelerator (the ray caster's interface)
 * GPUAcceleratorGroupI / GPUBaseAcceleratorI (GPUAcceleratorI.h:46-173) as
 * RayCasterCUDA::HitRays drives them (RayCasterCUDA.cu:35-166): the base
 * accelerator hands each ray the key of the next surface whose box it
 * crosses, the group's Hit traverses that surface's local-space LBVH.
 * Transforms are row-major 3x4 local-to-world matrices (the fourth row of
 * the reference's Matrix4x4 is 0 0 0 1).  Rays are RayGMem (32 B:
 * position, tMin, direction, tMax) in device memory. */
typedef struct mrb_accel_group mrb_accel_group;
typedef struct mrb_base_accel mrb_base_accel;
/* One surface of a group: triangles [tri_begin, tri_end) of the group's
 * primitives under global transform transform_id (SurfaceDefinition,
 * GPUAcceleratorI.h:34-39).  Ranges ascend and do not overlap. */
typedef struct mrb_surface {
    uint32_t tri_begin, tri_end;
    uint32_t transform_id;
} mrb_surface;
/* InitializeGroup: host arrays of the group's triangles; tbn (w,x,y,z per
 * vertex, as the triangle loader builds them), tri_cull and primitive_ids
 * may be NULL.  Keys are the triangles' material HitKeys; primitive_ids are
 * the ids Hit reports for each triangle (the primitive group's own indices
 * when the caller packed several batches into one surface range; NULL: the
 * triangle's index here).  Transform 0 is the identity until transforms are
 * attached. */
int mrb_accel_group_create(mrb_system* sys, const float* positions, uint32_t vertex_count,
                           const float* tbn, const uint32_t* indices, const uint32_t* tri_keys,
                           const uint8_t* tri_cull, const uint64_t* primitive_ids,
                           uint32_t tri_count, const mrb_surface* surfaces,
                           uint32_t surface_count, mrb_accel_group** out);
void mrb_accel_group_destroy(mrb_accel_group* g);
/* AttachGlobalTransformArray: count local-to-world matrices (12 floats
 * each, host); their inverses are computed in double and rounded once. */
int mrb_accel_group_attach_transforms(mrb_accel_group* g, const float* local_to_world,
                                      uint32_t count, uint32_t identity_index);
/* ConstructAccelerators: one LBVH per surface in its local space. */
int mrb_accel_group_construct(mrb_accel_group* g, void* stream);
/* Hit (GPUAcceleratorI.h:83-94; KCIntersectBVH, GPUAcceleratorBVHKC.cuh:
 * 229-346): for i < ray_count, ray d_ray_ids[i] against surface
 * (d_accel_keys[i] & 0xFFFFFF); a hit closer than the ray's tMax writes tMax
 * back into d_rays and material key, transform id, 64-bit primitive id and
 * the barycentrics (2 floats, TriangleHit) at index d_ray_ids[i]; hit
 * structs are hit_stride bytes apart (HitStructPtr's combined size, a
 * multiple of 4, at least 8).  Keys of surfaces the group does not have
 * leave the ray untouched. */
int mrb_accel_group_hit(const mrb_accel_group* g, uint32_t* d_material_keys,
                        uint32_t* d_transform_ids, uint64_t* d_primitive_ids, void* d_hit_structs,
                        uint32_t hit_stride, void* d_rays, const uint32_t* d_ray_ids,
                        const uint32_t* d_accel_keys, uint32_t ray_count, void* stream);
/* AcceleratorAABBs: world AABB of each surface (6 floats, min then max),
 * up to capacity; returns the surface count. */
int mrb_accel_group_aabbs(const mrb_accel_group* g, float* aabbs, uint32_t capacity);
/* TotalPrimitiveCount, AcceleratorCount. */
uint64_t mrb_accel_group_primitive_count(const mrb_accel_group* g);
uint32_t mrb_accel_group_accelerator_count(const mrb_accel_group* g);
/* TotalApproximateArea: sum of the triangles' world-space areas. */
int mrb_accel_group_total_area(const mrb_accel_group* g, float* area, void* stream);
/* SampleAreaWeightedPoints: count world positions and normals (3 floats
 * each, device) on the surfaces, triangles drawn by area.  Philox with the
 * seed replaces the reference's Sobol generator. */
int mrb_accel_group_sample_points(const mrb_accel_group* g, float* d_positions, float* d_normals,
                                  uint32_t count, uint64_t seed, void* stream);
/* EachPrimVoxelCount / VoxelizeSurfaces (GPUAcceleratorI.h:113-133) over
 * the octree box (6 floats, host) at resolution^3: per-primitive voxel
 * counts, then codes, packed spherical normals (u16 | u16 << 16, the
 * reference's Vector2us) and light keys at d_voxel_offsets[t] (exclusive
 * scan of the counts, tri_count + 1 entries). */
int mrb_accel_group_voxel_counts(const mrb_accel_group* g, uint64_t* d_counts, uint32_t resolution,
                                 const float* octree_aabb, void* stream);
int mrb_accel_group_voxelize(const mrb_accel_group* g, uint64_t* d_voxels,
                             uint32_t* d_voxel_normals, uint32_t* d_voxel_light_keys,
                             const uint64_t* d_voxel_offsets, const uint32_t* d_sorted_light_keys,
                             uint32_t light_count, uint32_t resolution, const float* octree_aabb,
                             void* stream);
/* Base accelerator (GPUBaseAcceleratorBVH, GPUAcceleratorBVH.cu:35-260):
 * Construct from the surfaces' world AABBs and accelerator keys (host);
 * GetReady puts every ray id below ray_count at the root; Hit writes the
 * next surface's key for each d_ray_ids[i] at d_accel_keys[i], 0 once the
 * ray has no surface left (KCIntersectBaseBVH, GPUAcceleratorBVHKC.cuh:
 * 513-652). */
int mrb_base_accel_create(mrb_system* sys, mrb_base_accel** out);
void mrb_base_accel_destroy(mrb_base_accel* b);
int mrb_base_accel_construct(mrb_base_accel* b, const float* aabbs, const uint32_t* accel_keys,
                             uint32_t count);
int mrb_base_accel_get_ready(mrb_base_accel* b, uint32_t ray_count, void* stream);
int mrb_base_accel_hit(const mrb_base_accel* b, uint32_t* d_accel_keys, const void* d_rays,
                       const uint32_t* d_ray_ids, uint32_t ray_count, void* stream);
/* SceneExtents. */
int mrb_base_accel_extents(const mrb_base_accel* b, float* aabb);

/* ---- wavefront pool: continuous batching of render jobs ----------------
 * (no counterpart in the reference: MRay renders one scene per tracer.)
 * Jobs of different scenes, resolutions and sample counts share one
 * device-resident wavefront: every iteration generates one frame of each
 * admitted job (as many as `capacity` camera samples hold, round robin),
 * traces all their rays in one traversal launch per depth, shades them in
 * one launch and resolves each job's frame into its own image.  Jobs are
 * admitted first come first served while their images fit the HBM budget
 * (hbm_budget 0: the free memory at creation minus the pool's buffers and a
 * 10 % reserve).  A job renders the same samples alone and in any mix: its
 * random numbers are keyed by its own sample index, frame and seed.  The
 * pool's iteration is one captured CUDA graph. */
typedef struct mrb_pool mrb_pool;
typedef struct mrb_pool_job {
    mrb_camera camera;
    uint32_t width, height;
    uint32_t samples;        /* "Samples": s -> s*s per pixel per frame */
    uint32_t frames;         /* frames to render (spp = frames * s*s) */
    uint32_t max_depth, rr_start, nee, mis;
    uint64_t seed;
} mrb_pool_job;
#define MRB_JOB_QUEUED 0
#define MRB_JOB_ACTIVE 1
#define MRB_JOB_DONE 2
/* capacity: camera samples per iteration (the wavefront holds 2 rays per
 * sample); max_depth: depths per iteration, the bound of every job's. */
int mrb_pool_create(mrb_system* sys, uint32_t capacity, uint32_t max_depth, size_t hbm_budget,
                    mrb_pool** out);
void mrb_pool_destroy(mrb_pool* pool);
/* Traversal launch shape: block 64/128/256 threads, stack 64/128 entries. */
int mrb_pool_set_launch(mrb_pool* pool, int trace_block, int trace_stack);
/* trace_stack 0 selects the 8-wide traversal's octant child order (node
 * groups on the stack) instead of the sorted order's 64 or 128 entries. */
/* Queue a job (the scene's accelerator must be built; the scene must stay
 * alive until the job is done).  One frame must fit the capacity. */
int mrb_pool_submit(mrb_pool* pool, mrb_scene* scene, const mrb_pool_job* job, uint64_t* job_id);
/* Admit what fits, run one iteration (synchronous).  Outputs: jobs that
 * finished in this iteration, jobs active and queued afterwards. */
int mrb_pool_step(mrb_pool* pool, uint32_t* finished, uint32_t* active, uint32_t* queued);
int mrb_pool_job_status(mrb_pool* pool, uint64_t job_id, uint32_t* state, uint32_t* frames_done);
/* A done job's image (width*height*4: sum of per-frame means, frame count
 * in .w); release != 0 frees it and forgets the job. */
int mrb_pool_job_image(mrb_pool* pool, uint64_t job_id, float* host_rgba, int release);
/* Rays traced, iterations run, HBM held by admitted jobs and the budget. */
int mrb_pool_stats(mrb_pool* pool, uint64_t* rays, uint64_t* iterations, size_t* hbm_used,
                   size_t* hbm_budget);
void* mrb_pool_stream(mrb_pool* pool);

/* ---- learned guiding network (no counterpart in the reference) ---------
 * An MLP from a path vertex to a mixture of 8 von Mises-Fisher lobes over
 * incident directions: 80 input features (sin/cos of 2^j pi p for j < 12 on
 * each axis of the position normalised to the scene box, the normal, the
 * outgoing direction, two zeros) -> 64 -> 64 -> 64 (ReLU) -> 40 raw lobe
 * parameters (per lobe: direction xyz, log concentration, weight logit).
 * BF16 weights and activations, FP32 accumulation, on the tcgen05 tensor
 * cores; Adam (0.9, 0.999, 1e-8) on FP32 master parameters.  Parameters:
 * per layer W[in][64] (out contiguous) then 64 biases; the output layer's
 * columns 40..63 and the first layer's inputs 78..79 are held at zero. */
typedef struct mrb_mlp mrb_mlp;
uint32_t mrb_mlp_param_count(void);
int mrb_mlp_create(mrb_system* sys, mrb_mlp** out);
void mrb_mlp_destroy(mrb_mlp* mlp);
/* Host parameters in; resets the optimiser state. */
int mrb_mlp_set_params(mrb_mlp* mlp, const float* host_params);
int mrb_mlp_get_params(const mrb_mlp* mlp, float* host_params);
/* Device arrays: pos (normalised to [0,1]^3), normal, outgoing direction,
 * 3 floats each -> n x 80 features. */
int mrb_mlp_encode(const float* d_pos, const float* d_nrm, const float* d_wo, uint32_t n,
                   float* d_features, void* stream);
/* n x 80 features -> n x 40 raw outputs (16-byte aligned arrays). */
int mrb_mlp_forward(mrb_mlp* mlp, const float* d_features, uint32_t n, float* d_out,
                    void* stream);
/* Adds the gradient of sum_s w_s * -log q(dir_s | x_s) into d_grad
 * (param_count floats) and (sum w_s * -log q, sum w_s) into d_loss[2];
 * targets n x 4: incident direction xyz (unit), weight w_s >= 0. */
int mrb_mlp_gradients(mrb_mlp* mlp, const float* d_features, const float* d_targets, uint32_t n,
                      float* d_grad, float* d_loss, void* stream);
/* One optimiser step on the loss normalised by sum w_s; host_loss2 (may be
 * NULL) receives (weighted loss sum, weight sum) of the batch. */
int mrb_mlp_train_step(mrb_mlp* mlp, const float* d_features, const float* d_targets, uint32_t n,
                       float lr, float* host_loss2, void* stream);

/* ---- kernel-level entry points (device pointers) ---------------------- */
/* KCGenerateAABBs + extent reduce + KCGenMortonCodes
 * (LinearBVH.hpp:102-166,444-482). */
int mrb_morton_codes(const float* d_pos, const uint32_t* d_idx, uint32_t n, float* d_tri_aabb,
                     float* d_extent, uint64_t* d_codes, void* stream);
/* Stable radix sort of pairs on bits [begin_bit, end_bit), as
 * cub::DeviceRadixSort::SortPairs(Descending) (ParallelRadixSort.cuh:60-100). */
size_t mrb_radix_sort_temp_bytes(uint32_t n, int key_bytes, int begin_bit, int end_bit);
int mrb_radix_sort_pairs_u64(uint64_t* d_keys, uint32_t* d_vals, uint32_t n, int begin_bit,
                             int end_bit, int descending, void* d_temp, size_t temp_bytes,
                             void* stream);
int mrb_radix_sort_pairs_u32(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, int begin_bit,
                             int end_bit, int descending, void* d_temp, size_t temp_bytes,
                             void* stream);
/* Allocation-free variant of mrb_radix_sort_pairs_u32 (no counterpart in
 * the reference).  For callers that cannot call cudaMalloc -- a host that
 * manages all device memory itself and forbids libraries to allocate, or a
 * latency-critical path that cannot afford cudaMalloc's implicit device
 * synchronisation.  Scratch is a file-scope device array of 8.5 MiB
 * (8,912,896 bytes), resident on every device that loads the library until
 * exit; n is limited to 1,048,576 pairs (larger n returns MRB_E_ARG).  All
 * calls share the array: calls that overlap on the GPU race, so serialise
 * them on one stream.  The first call on a device looks up the array's
 * address with that device current; make it before any stream capture, and
 * do not call this entry point on a device after cudaDeviceReset (the
 * cached address is then stale).  A look-back wait of the sort that gives up
 * (bounded; not expected in practice) leaves the output unordered and is not
 * reported by this entry point.  Allocates nothing. */
int mrb_radix_sort_pairs_u32_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint32_t n,
                                     int begin_bit, int end_bit, int descending, void* stream);
/* LBVH hierarchy + AABBs from sorted codes (LinearBVH.hpp:30-100,181-396).
 * d_scratch: 3*(n-1) u32.  Outputs in reference numbering. */
int mrb_lbvh_hierarchy(const uint64_t* d_sorted_codes, const uint32_t* d_sorted_idx,
                       const float* d_tri_aabb, uint32_t n, uint32_t* d_left, uint32_t* d_right,
                       uint32_t* d_parent, float* d_inner, uint32_t* d_root, uint32_t* d_scratch,
                       void* d_nodes64, void* stream);
/* RayMemory::SortKeys + Partition (RayMemory.cu:187-312): stable descending
 * sort of the rays by (batch, id) key bits and per-batch [offset, end).
 * d_portion_offset / d_portion_end: 8 entries each; d_non_null: 1. */
size_t mrb_partition_temp_bytes(uint32_t n, uint32_t id_bits);
int mrb_partition(const uint32_t* d_keys, uint32_t n, uint32_t id_bits, uint32_t* d_sorted_ids,
                  uint32_t* d_sorted_dense, uint32_t* d_portion_offset, uint32_t* d_portion_end,
                  uint32_t* d_non_null, void* d_temp, size_t temp_bytes, void* stream);

/* Portable math of the device path, for the CPU/GPU bit-parity check:
 * out[i*2+0..1] = sin, cos of x[i]; out2[i] = acos(y[i]). */
int mrb_debug_math(const float* d_x, uint32_t n, float* d_sincos, const float* d_y,
                   float* d_acos, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MRB200_H */
