/*
 * CPU oracle for the meturay_b200 wavefront path-tracing path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * library: it is loaded by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline / reference leg of bench.py, always as the checker.
 *
 * Every function restates the algorithm of the MRay reference
 * (yalcinerbora/meturay, Source/...) at the cited file:line.  FP32 entry
 * points use the same operation order as the CUDA kernels (no contraction,
 * explicit fmaf where the kernels use one, the same portable sin/cos/acos),
 * so that integer stages are bit-exact and radiance is bit-exact up to the
 * order of float atomic additions.  FP64 entry points run the same
 * algorithm in double precision and state the error of the FP32 image.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- portable math (same algorithm as the device copy) ---- */
void  oracle_sincosf(float x, float* s, float* c);
float oracle_acosf(float x);

/* ---- counter-based RNG: Philox4x32-10 (Salmon et al., SC'11) ---- */
void oracle_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- a1..a5: Morton codes and sort (LinearBVH.hpp:102-179,398-414) ---- */
uint64_t oracle_morton3d(uint32_t x, uint32_t y, uint32_t z);
/* tri_pos: tri_count*9 floats (p0,p1,p2).  Writes per-triangle AABB
 * (tri_count*6: min xyz, max xyz), the extent (6), the Morton delta and the
 * codes. */
void oracle_morton_codes(const float* pos, const uint32_t* idx, uint32_t tri_count,
                         float* aabbs, float* extent, float* delta, uint64_t* codes);
/* Stable LSD radix sort of (key, value) pairs on bits [begin_bit, end_bit)
 * (cub::DeviceRadixSort semantics, ascending or descending). */
void oracle_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint32_t n,
                           int begin_bit, int end_bit, int descending);
void oracle_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t n,
                           int begin_bit, int end_bit, int descending);

/* ---- a6/a7: Karras/Apetrei hierarchy and bottom-up AABBs
 *      (LinearBVH.hpp:30-100,181-396).  Node numbering as the reference:
 *      leaves 0..n-1, internal nodes n..2n-2.  Returns 0 on success,
 *      1 on duplicate codes (LinearBVH.hpp:505-521). ---- */
int oracle_lbvh_build(const uint64_t* sorted_codes, const uint32_t* sorted_idx,
                      const float* leaf_aabbs, uint32_t n,
                      uint32_t* left, uint32_t* right, uint32_t* parent,
                      float* inner_aabbs, uint32_t* root);

/* ---- a13/a14: key sort + partition (RayMemory.cu:187-312) ---- */
/* Sorts (key, id=0..n-1) descending on the dense key bits and returns the
 * portions: (batch, offset, count) for each batch present, in ascending
 * batch order like std::set<ArrayPortion>.  Returns the portion count. */
uint32_t oracle_partition(const uint32_t* keys, uint32_t n, uint32_t batch_bits,
                          uint32_t id_bits, uint32_t* sorted_keys, uint32_t* sorted_ids,
                          uint32_t* portion_batch, uint32_t* portion_offset,
                          uint32_t* portion_count);

/* ---- scene, as consumed by the hot path ---- */
typedef struct oracle_scene {
    uint32_t vertex_count;
    uint32_t tri_count;
    const float*    pos;        /* vertex_count*3 */
    const float*    tbn;        /* vertex_count*4 (w,x,y,z) */
    const uint32_t* idx;        /* tri_count*3 */
    const uint32_t* tri_key;    /* tri_count HitKey (batch<<24 | id) */
    const uint8_t*  tri_cull;   /* tri_count, may be NULL (two-sided) */
    uint32_t lambert_count;  const float* lambert_albedo;   /* 3 each */
    uint32_t metal_count;    const float* metal_params;     /* eta3 k3 spec3 rough */
    uint32_t refract_count;  const float* refract_albedo;   /* 3 each */
    const uint32_t* refract_medium;
    uint32_t light_count;    const float* light_radiance;   /* 3 each */
    const uint32_t* light_prim;
    uint32_t medium_count;   const float* medium_ior;
    uint32_t base_medium;
    uint32_t lambertc_count; const float* lambertc_albedo;  /* 3 each */
    uint32_t unreal_count;   const float* unreal_params;    /* albedo3 rough metal spec */
} oracle_scene;

typedef struct oracle_camera {
    float position[3];
    float bottom_left[3];
    float right[3];
    float up[3];
    float plane_size[2];
    float near_far[2];
} oracle_camera;

typedef struct oracle_options {
    uint32_t width, height;
    uint32_t samples;        /* "Samples": s -> s*s spp per iteration */
    uint32_t max_depth;
    uint32_t rr_start;
    uint32_t nee;
    uint32_t mis;
    uint32_t seed_lo, seed_hi;
    uint32_t frame;
    uint32_t threads;        /* 0 = all hardware threads */
    uint32_t row_begin, row_end;  /* sample rows to render (0,0 = all) */
    uint32_t row_step;       /* render every row_step-th row from row_begin (0 = 1) */
} oracle_options;

/* Build the LBVH of the scene (a1..a7) and keep it inside a handle. */
typedef struct oracle_bvh oracle_bvh;
oracle_bvh* oracle_bvh_create(const oracle_scene* scene, int* status);
void        oracle_bvh_destroy(oracle_bvh*);
uint32_t    oracle_bvh_root(const oracle_bvh*);

/* a8..a11: closest hit of rays (origin3, tmin, dir3, tmax) per ray.
 * out: key, prim (original triangle index or 0xFFFFFFFF), t, bary2. */
void oracle_trace(const oracle_scene* scene, const oracle_bvh* bvh,
                  const float* rays, uint32_t n,
                  uint32_t* out_key, uint32_t* out_prim, float* out_t, float* out_bary,
                  uint32_t threads);
/* Inner nodes entered and triangles tested by oracle_trace / oracle_render
 * since the last reset (out[2]). */
void oracle_trace_counters(uint64_t* out, int reset);
/* The reference "Linear" accelerator: brute force, triangle order, strict <. */
void oracle_trace_linear(const oracle_scene* scene, const float* rays, uint32_t n,
                         uint32_t* out_key, uint32_t* out_prim, float* out_t, float* out_bary,
                         uint32_t threads);

/* a16..a24: one iteration of the plain path tracer (GenerateWork, Render
 * until done, sample radiance).  sample_rgb: (W*s)*(H*s)*3 per-sample
 * radiance.  Returns the number of rays traced (camera+path+NEE). */
uint64_t oracle_render(const oracle_scene* scene, const oracle_bvh* bvh,
                       const oracle_camera* cam, const oracle_options* opt,
                       float* sample_rgb);
uint64_t oracle_render_f64(const oracle_scene* scene, const oracle_bvh* bvh,
                           const oracle_camera* cam, const oracle_options* opt,
                           double* sample_rgb);

/* Per-vertex tangent-space rotations (w,x,y,z) of a triangle mesh, as the
 * triangle loader builds them (GPUPrimitiveTriangle.cpp:160-320).  uvs may
 * be NULL: each triangle then uses (0,0),(1,0),(0,1). */
void oracle_build_tbn(const float* pos, const float* nrm, const float* uvs, const uint32_t* idx,
                      uint32_t vertex_count, uint32_t tri_count, float* tbn_out);

/* Sparse voxel octree (AnisoSVO.cu:657-1188 with TriFunctions::Voxelize,
 * GPUPrimitiveTriangle.h:385-620), built in the reference's own order:
 * voxelise, sort + RLE, then per level mark children from the root, scan
 * child counts, set child and parent pointers. */
typedef struct oracle_svo oracle_svo;
oracle_svo* oracle_svo_build(const float* pos, const uint32_t* idx, const uint32_t* key,
                             uint32_t tri_count, const float* extent6, uint32_t resolution,
                             int* status);
void oracle_svo_destroy(oracle_svo*);
/* sizes[6]: voxels, leaves, nodes, depth, level-offset count, triangles */
void oracle_svo_sizes(const oracle_svo*, uint32_t* sizes);
void oracle_svo_get(const oracle_svo*, uint64_t* nodes, uint32_t* leaf_parents,
                    uint64_t* leaf_codes, uint32_t* leaf_lights, uint32_t* level_offsets,
                    uint32_t* tri_voxel_counts, float* params7);

/* Radiance-cache payload of the octree (KCReduceVoxelPayload,
 * KCAverageNormals, NormalizeAndFilterRadiance): light radiance per light
 * (3 floats), omit = OmitDirectRadiance.  Get: leaf / node normal words,
 * leaf radiance sums (2 per leaf, 2^24 fixed point), leaf counts (2 per
 * leaf), leaf / node half2 averages. */
void oracle_svo_payload_init(oracle_svo*, const float* light_rad, uint32_t omit);
void oracle_svo_payload_get(const oracle_svo*, uint32_t* leaf_norm_spec, uint32_t* node_norm_spec,
                            uint64_t* leaf_irr, uint32_t* leaf_cnt, uint32_t* leaf_avg,
                            uint32_t* node_avg);
/* Shadow-ray counters (hits, misses per leaf: DepositNEEHitMiss) and the
 * binary16 node guiding factors of the last NormalizeAndFilterRadiance.
 * Set replaces the counters (the factors follow at the next normalise). */
void oracle_svo_set_shadow(oracle_svo*, const uint32_t* leaf_shadow);
/* DepositNEEHitMiss of n vertices over zeroed counters (is_hit: 1 hit, 0 miss). */
void oracle_svo_deposit_nee(oracle_svo*, const float* pos, const uint8_t* is_hit, uint32_t n);
void oracle_svo_guiding_get(const oracle_svo*, uint32_t* leaf_shadow, uint16_t* node_factor);

/* TriFunctions::Voxelize over every triangle (counting pass, then codes and
 * packed spherical normals u16 | u16 << 16 in triangle order, at most
 * capacity); codes == NULL counts only.  Returns the voxel count, -1 when
 * capacity is too small. */
int64_t oracle_voxelize(const float* pos, const uint32_t* idx, uint32_t tri_count,
                        const float* extent6, uint32_t resolution, uint64_t* counts,
                        uint64_t* codes, uint32_t* normals, uint64_t capacity);
/* Ray bins of one wavefront over the octree: rays i with valid[i] hit at
 * org + t * dir; bin_out: 0xFFFFFFFF, leaf | 1 << 31, or a node index. */
void oracle_svo_bin_rays(oracle_svo*, const float* org, const float* dir, const float* t,
                         const uint8_t* valid, uint32_t n, uint32_t min_level,
                         uint32_t bin_ray_count, uint32_t* bin_out);
/* Leaf radiance sums (2 per leaf, 2^-24 fixed point) and sample counts (2
 * per leaf) set directly; NormalizeAndFilterRadiance over them. */
void oracle_svo_set_radiance(oracle_svo*, const uint64_t* leaf_irr, const uint32_t* leaf_cnt);
void oracle_svo_normalize(oracle_svo*);
/* DepositRadiance of n vertices (position, wo, luminance) over zeroed sums. */
void oracle_svo_deposit(oracle_svo*, const float* pos, const float* wo, const float* lum,
                        uint32_t n);
/* ConeTraceRay + ReadRadiance for n cones. */
void oracle_svo_cone_trace(const oracle_svo*, const float* org, const float* dir,
                           const float* tmin, const float* aperture, uint32_t max_query_offset,
                           uint32_t n, float* t_out, uint32_t* id_out, uint8_t* leaf_out,
                           float* rad_out);

/* One WFPG frame (WFPGTracer.cu:1480-1833) over the octree, which it
 * updates (deposit + normalise/filter).  Per-sample radiance to out (3 per
 * sample); guide words and bin ids of step dump_iteration per path to
 * dump_guide (2 per path) / dump_bin (1 per path), either may be NULL.
 * Returns the rays traced. */
typedef struct oracle_wfpg_options {
    uint32_t min_bin_level;
    uint32_t bin_ray_count;
    uint32_t pure_pg;
    uint32_t skip_pg;
    uint32_t guide_bounce;
    float mis_ratio;
    float filter[11];
    uint32_t dump_iteration;
    uint32_t product;  /* 1: KCGenAndSampleDistributionProduct, 0: KCGenAndSampleDistribution */
} oracle_wfpg_options;
/* The product sampler on table inputs, for its pin against the reference's
 * own sampler (test infrastructure; see oracle.cpp). */
void oracle_product_pin(const float* fields, uint32_t bins, uint32_t rays_per_bin,
                        const float* surfaces, const float* streams, uint32_t stream_len,
                        float mis_ratio, float mult, float* uv, float* pdf, uint32_t* sel,
                        float* small, float* norm);
uint64_t oracle_render_wfpg(const oracle_scene* scene, const oracle_bvh* bvh,
                            const oracle_camera* cam, const oracle_options* opt,
                            const oracle_wfpg_options* wopt, oracle_svo* svo, float* out_rgb,
                            uint32_t* dump_guide, uint32_t* dump_bin);

/* Single-vertex BxDF probes used by the golden-vector tests. */
void oracle_bxdf_sample(uint32_t type, const float* params, const float* wi,
                        const float* w2t, const float* geo_normal, const float* pos,
                        uint32_t backside, float from_ior, float to_ior,
                        const float* xi, float* out_dir, float* out_pos,
                        float* out_refl, float* out_pdf);
/* Named single-function probes (hemi_cosine, reflect, refract, quat_rotate,
 * quat_mul, dggx, gsmith_corr, gsmith_single, fresnel_conductor,
 * fresnel_dielectric, vndf_sample, vndf_pdf, power_heuristic); argument
 * layouts are listed next to each case in oracle.cpp.  0 ok, -1 unknown. */
int oracle_probe(const char* name, const float* in, float* out);
void oracle_bary_slerp(const float* q0, const float* q1, const float* q2,
                       float a, float b, float* out);
void oracle_nudge(const float* p, const float* dir, float* out);
int  oracle_intersect_tri(const float* ro, const float* rd, const float* p0,
                          const float* p1, const float* p2, int cull,
                          float* t, float* bary3);

/* ---- reconstruction filters (oracle/recon.cpp) ----
 * type 0 Box, 1 Tent, 2 Gaussian (alpha), 3 Mitchell (b, c). */
typedef struct oracle_filter {
    uint32_t type;
    float radius, alpha, b, c;
} oracle_filter;
uint32_t oracle_filter_pixel_wh(float radius);
void oracle_exp(const float* x, uint32_t n, float* out);
float oracle_filter_weight(const oracle_filter* f, float px, float py, float sx, float sy);
/* FilterToImg: values (channels 1 or 4 per sample), coords (2 per sample);
 * pixels (segW*segH*channels) and counts (segW*segH) are added to. */
void oracle_filter_to_img(const oracle_filter* f, const float* values, uint32_t channels,
                          const float* coords, uint32_t n, int32_t resW, int32_t resH,
                          int32_t offX, int32_t offY, int32_t segW, int32_t segH,
                          float multiplier, float* pixels, float* counts);
/* The reference test's direct CPU expectation (RGBA, whole image). */
void oracle_filter_direct(const oracle_filter* f, const float* values, const float* coords,
                          uint32_t n, int32_t resW, int32_t resH, float* pixels, float* counts);
/* The reference test's mt19937 sample coordinates (2 floats per sample). */
void oracle_mt19937_coords(uint32_t n, int32_t width, int32_t height, uint32_t seed, float* out);
/* Image coordinates of the camera samples of one iteration (2 per sample):
 * ((s + jitter) / samples across) * resolution per axis. */
void oracle_camera_img_coords(const oracle_options* opt, float* out);

#ifdef __cplusplus
}
#endif
