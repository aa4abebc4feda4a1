// Learned guiding: the network's vMF mixture as the guide of each wavefront,
// and its online training from the frame's path chains.
#include "../../include/mrb200.h"
#include "bxdf.cuh"
#include "learned.cuh"
#include "mlp_tile.cuh"
#include "scan.cuh"

namespace mrb {

namespace {

constexpr uint32_t kTagLearned = 0x40000u;  // per-ray draws of the learned sampler
constexpr uint32_t kGuideValid = 1u << 17;
constexpr uint32_t kGuideBxdf = 1u << 16;

__device__ __forceinline__ float lum3(V3 c) { return 0.2120f * c.x + 0.7150f * c.y + 0.0722f * c.z; }

inline uint32_t grid_for(uint32_t n, uint32_t block, uint32_t cap) {
    uint32_t g = (n + block - 1) / block;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

__device__ __forceinline__ float unit01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// Position in the octree's box, normalised to [0, 1]^3.
__device__ __forceinline__ V3 box_coords(const GuideDev& g, V3 p) {
    return v3(unit01((p.x - g.lo[0]) / (g.hi[0] - g.lo[0])),
              unit01((p.y - g.lo[1]) / (g.hi[1] - g.lo[1])),
              unit01((p.z - g.lo[2]) / (g.hi[2] - g.lo[2])));
}

// A ray the network guides: a non-NEE ray that hit a non-specular surface.
__device__ __forceinline__ bool guided_hit(const SceneDev& sc, const GuideWave& w, uint32_t i,
                                           uint32_t& batch, uint32_t& id) {
    const uint32_t key = w.hit.key[i];
    batch = key >> kIdBits;
    id = key & kIdMask;
    if (w.aux[i].type == kNeeRay || batch == kBatchNull || batch == kBatchLight) return false;
    return !mat_specular(sc, batch, id);
}

// Orthonormal basis around a unit vector (Duff et al., "Building an
// Orthonormal Basis, Revisited", JCGT 2017).
__device__ __forceinline__ void onb(V3 n, V3& t1, V3& t2) {
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    t1 = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    t2 = v3(b, sign + n.y * n.y * a, -n.y);
}

// vMF sample around mu (Wenzel Jakob, "Numerically stable sampling of the
// von Mises-Fisher distribution on S^2"): cos = 1 + log(x + (1-x) e^-2k) / k.
__device__ __forceinline__ V3 vmf_sample(V3 mu, float kappa, float u0, float u1) {
    float c = 1.0f + logf(u0 + (1.0f - u0) * expf(-2.0f * kappa)) / kappa;
    c = fminf(fmaxf(c, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float sp, cp;
    sincospif(2.0f * u1, &sp, &cp);
    V3 t1, t2;
    onb(mu, t1, t2);
    return normalize(t1 * (s * cp) + t2 * (s * sp) + mu * c);
}

// The guide of one wavefront in one kernel: each thread of a 128-row tile
// encodes its ray's hit as the network's input, the tile goes through the
// tensor-core forward pass, and each thread draws its ray's direction from
// the vMF mixture (probability misRatio) or the BxDF, with the one-sample
// MIS pdf of the drawn direction at its half-precision octahedral
// coordinates (the form the shading kernel decodes).  Rays at specular
// surfaces, lights or none get no guide word.
struct GuideIO {
    SceneDev sc;
    GuideDev g;
    GuideWave w;
    float misRatio;
    PathOptions opt;
    uint32_t depthTag;
    uint2* guide;

    __device__ uint32_t rows() const {
        const uint32_t n = *w.count;
        return n < w.maxRays ? n : w.maxRays;
    }
    __device__ void input(uint32_t i, uint32_t n, float* f) const {
        uint32_t batch, id;
        if (i < n && guided_hit(sc, w, i, batch, id)) {
            const float4 rd = w.rayD[i];
            const float2 hb = w.hit.bary[i];
            const V3 d = v3(rd.x, rd.y, rd.z);
            const Surface sf = gen_surface(sc, w.hit.prim[i], hb.x, hb.y, d);
            const V3 nrm = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
            const V3 wo = -normalize(d);
            const V3 p = box_coords(g, sf.pos);
            encode_vertex(p.x, p.y, p.z, nrm.x, nrm.y, nrm.z, wo.x, wo.y, wo.z, f);
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; k++) f[k] = 0.0f;
        }
    }
    __device__ void output(uint32_t i, const float* r) const {
        uint32_t batch, id;
        uint2 word = make_uint2(0u, 0x7E00u);  // no guide: the BxDF samples the ray
        if (guided_hit(sc, w, i, batch, id)) {
            const uint32_t frame = *opt.frame;
            VmfMixture mx;
            float rawLen[kMlpLobes], lobeLog[kMlpLobes];
            mixture_from_raw(r, mx, rawLen);
            const RayAux aux = w.aux[i];
            const float4 rd = w.rayD[i];
            const float2 hb = w.hit.bary[i];
            const V3 d = v3(rd.x, rd.y, rd.z);
            const Surface sf = gen_surface(sc, w.hit.prim[i], hb.x, hb.y, d);
            const V3 wi = -normalize(d);
            const Rand4 r0 = philox_uniform4(aux.sample, frame, kTagLearned | depthTag, 0u,
                                             opt.seedLo, opt.seedHi);
            V3 dir;
            const bool fromGuide = r0.u[0] < misRatio;
            if (fromGuide) {
                // the lobe by its weight, then a direction from it
                int k = 0;
                float acc = 0.0f;
                for (; k < kMlpLobes - 1; k++) {
                    acc += expf(mx.logPi[k]);
                    if (r0.u[1] < acc) break;
                }
                dir = vmf_sample(v3(mx.mu[k][0], mx.mu[k][1], mx.mu[k][2]), mx.kappa[k], r0.u[2],
                                 r0.u[3]);
            } else {
                const Rand4 r1 = philox_uniform4(aux.sample, frame, kTagLearned | depthTag, 1u,
                                                 opt.seedLo, opt.seedHi);
                dir = mat_sample(sc, batch, id, wi, sf, aux.medium, r1.u[0], r1.u[1], r1.u[2]).dir;
            }
            float s, t;
            dir_yup_to_octa(dir, s, t);
            const uint16_t sh = f2h(s), th = f2h(t);
            const V3 dq = octa_to_dir_yup(h2f(sh), h2f(th));
            const float q = expf(mixture_logpdf(mx, dq.x, dq.y, dq.z, lobeLog));
            const float pb = mat_pdf(sc, batch, id, dq, wi, sf);
            const float pdf = misRatio * q + (1.0f - misRatio) * pb;
            if (pdf > 0.0f && pdf < 65504.0f && dq.x == dq.x)
                word = make_uint2(uint32_t(sh) | (uint32_t(th) << 16),
                                  uint32_t(f2h(pdf)) | (fromGuide ? 0u : kGuideBxdf) | kGuideValid);
        }
        guide[i] = word;
    }
};

// ---- training samples ---------------------------------------------------------
struct ChainView {
    GuideDev g;
    PathChain pc;
    const uint32_t* frame;
    float weightMax;
    uint32_t product;
};

__device__ __forceinline__ uint32_t chain_length(const PathChain& pc, uint32_t p, uint32_t frame) {
    const size_t P = pc.paths;
    uint32_t L = 0;
    while (L + 1 < pc.levels && __float_as_uint(pc.nodeA[size_t(L + 1) * P + p].w) == frame) L++;
    return L;
}

// Vertex d of path p as a training sample: false if it is not one.  With
// feat == nullptr only the validity is decided.
__device__ __forceinline__ bool chain_sample(const ChainView& v, uint32_t p, uint32_t d,
                                             uint32_t lastD, uint32_t frame, float* feat,
                                             float4& target) {
    const PathChain& pc = v.pc;
    const size_t P = pc.paths, at = size_t(d) * P + p;
    const float4 nn = pc.nodeN[at], tt = pc.nodeT[at];
    if (nn.w != 0.0f || __float_as_uint(tt.w) != frame) return false;  // specular / no path ray
    const float4 dd = pc.nodeD[at];
    if (!(dd.w > 0.0f) || !(dd.w < 3.0e38f)) return false;
    V3 sum = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t D = d + 1; D <= lastD; D++) {
        const float4 cn = pc.contribNee[size_t(D) * P + p];
        const float4 cp = pc.contribPath[size_t(D) * P + p];
        sum = sum + v3(cn.x + cp.x, cn.y + cp.y, cn.z + cp.z);
    }
    const V3 li = v3(tt.x > 0.0f ? sum.x / tt.x : 0.0f, tt.y > 0.0f ? sum.y / tt.y : 0.0f,
                     tt.z > 0.0f ? sum.z / tt.z : 0.0f);
    float wgt = lum3(li) / dd.w;
    // the integrand's cosine: the mixture then learns L_in |cos| (for a
    // diffuse vertex the ideal sampling density up to a constant)
    if (v.product) wgt *= fabsf(nn.x * dd.x + nn.y * dd.y + nn.z * dd.z);
    if (!(wgt > 0.0f) || !(wgt < 3.0e38f)) return false;
    if (v.weightMax > 0.0f) wgt = fminf(wgt, v.weightMax);
    if (!feat) return true;  // counting pass: validity only
    const float4 a = pc.nodeA[at], pa = pc.nodeA[at - P];
    const V3 pos = v3(a.x, a.y, a.z);
    const V3 wo = normalize(v3(pa.x, pa.y, pa.z) - pos);
    const V3 bc = box_coords(v.g, pos);
    encode_vertex(bc.x, bc.y, bc.z, nn.x, nn.y, nn.z, wo.x, wo.y, wo.z, feat);
    target = make_float4(dd.x, dd.y, dd.z, wgt);
    return true;
}

__global__ void __launch_bounds__(256) k_learned_count(ChainView v, uint32_t* __restrict__ count) {
    const uint32_t frame = *v.frame;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < v.pc.paths;
         p += gridDim.x * blockDim.x) {
        const uint32_t L = chain_length(v.pc, p, frame);
        const uint32_t lastD = (L + 1 < v.pc.levels) ? L + 1 : v.pc.levels - 1;
        uint32_t c = 0;
        for (uint32_t d = 1; d <= L; d++) {
            float4 t;
            if (chain_sample(v, p, d, lastD, frame, nullptr, t)) c++;
        }
        count[p] = c;
    }
}

// Sample j goes to slot (j mod steps) * perStep + j / steps, so that step k
// trains on every steps-th sample of the frame.
__global__ void __launch_bounds__(256) k_learned_write(ChainView v, const uint32_t* __restrict__ offset,
                                                       LearnedScratch s) {
    const uint32_t frame = *v.frame;
    const uint32_t perStep = s.capacity / s.steps;
    float f[kMlpIn];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < v.pc.paths;
         p += gridDim.x * blockDim.x) {
        const uint32_t L = chain_length(v.pc, p, frame);
        const uint32_t lastD = (L + 1 < v.pc.levels) ? L + 1 : v.pc.levels - 1;
        uint32_t j = offset[p];
        for (uint32_t d = 1; d <= L; d++) {
            float4 t;
            if (!chain_sample(v, p, d, lastD, frame, f, t)) continue;
            const uint32_t slot = j / s.steps;
            if (slot < perStep) {
                const size_t o = size_t(j % s.steps) * perStep + slot;
                float4* dst = reinterpret_cast<float4*>(s.trainX + o * kMlpIn);
#pragma unroll
                for (int c = 0; c < kMlpIn / 4; c++)
                    dst[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
                reinterpret_cast<float4*>(s.trainT)[o] = t;
            }
            j++;
        }
    }
}

__global__ void k_learned_loss(const float* __restrict__ stepLoss, float* __restrict__ frameLoss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        frameLoss[0] += stepLoss[0];
        frameLoss[1] += stepLoss[1];
    }
}

__global__ void k_learned_steps(const uint32_t* __restrict__ total, LearnedScratch s) {
    const uint32_t k = threadIdx.x;
    if (k >= s.steps) return;
    const uint32_t n = *total, perStep = s.capacity / s.steps;
    const uint32_t c = n > k ? (n - k + s.steps - 1) / s.steps : 0u;
    s.stepCount[k] = c < perStep ? c : perStep;
}

__global__ void __launch_bounds__(256) k_learned_ema(const float* __restrict__ params,
                                                     float* __restrict__ ema, float beta,
                                                     float* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < uint32_t(kMlpParams);
         i += gridDim.x * blockDim.x) {
        const float e = beta * ema[i] + (1.0f - beta) * params[i];
        ema[i] = e;
        out[i] = e;
    }
}

}  // namespace

int learned_ema(const float* params, float* ema, float beta, float* out, cudaStream_t st) {
    k_learned_ema<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, ema, beta, out);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int learned_guide_wavefront(const SceneDev& sc, const GuideDev& g, const GuideWave& w,
                            const MlpDev& net, const LearnedScratch& s, float misRatio,
                            const PathOptions& opt, uint32_t depthTag, uint2* guide,
                            cudaStream_t st) {
    (void)s;
    static bool attr[64] = {};
    int dev = 0;
    MRB_CUDA(cudaGetDevice(&dev));
    if (!attr[dev & 63]) {
        MRB_CUDA(cudaFuncSetAttribute(k_mlp_forward_io<GuideIO>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(sizeof(MlpFwdSmem))));
        attr[dev & 63] = true;
    }
    const uint32_t tiles = (w.maxRays + kMlpTile - 1) / kMlpTile;
    const uint32_t cap = 148u * kMlpFwdCtasPerSm;
    const uint32_t grid = tiles < cap ? (tiles ? tiles : 1u) : cap;
    k_mlp_forward_io<<<grid, kMlpTile, sizeof(MlpFwdSmem), st>>>(
        net, GuideIO{sc, g, w, misRatio, opt, depthTag, guide});
    MRB_CUDA(cudaGetLastError());
    return 0;
}

size_t learned_scan_temp_bytes(uint32_t paths) { return exclusive_scan_temp_bytes(paths); }

uint32_t learned_launches(uint32_t steps) {
    // count, scan (3), write, steps; per step: train, Adam, step counter, loss
    return 6 + 4 * steps;
}

int learned_collect(const GuideDev& g, const PathChain& pc, const uint32_t* frame,
                    const LearnedScratch& s, cudaStream_t st) {
    const ChainView v{g, pc, frame, s.weightMax, s.product};
    const uint32_t grid = grid_for(pc.paths, 256, 148 * 8);
    k_learned_count<<<grid, 256, 0, st>>>(v, s.pathCount);
    MRB_CUDA(cudaGetLastError());
    if (exclusive_scan_u32(s.pathCount, s.pathOffset, pc.paths, s.scanTemp, st)) return MRB_E_CUDA;
    k_learned_write<<<grid, 256, 0, st>>>(v, s.pathOffset, s);
    k_learned_steps<<<1, 32, 0, st>>>(s.pathOffset + pc.paths, s);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int learned_train(mrb_mlp* net, const LearnedScratch& s, float lr, cudaStream_t st) {
    MRB_CUDA(cudaMemsetAsync(s.frameLoss, 0, 8, st));
    const uint32_t perStep = s.capacity / s.steps;
    for (uint32_t k = 0; k < s.steps; k++) {
        // at most half the SMs: the training overlaps the frame, whose
        // kernels need the rest (a training CTA holds 140 KB of shared memory)
        int r = mlp_train_step_dev(net, s.trainX + size_t(k) * perStep * kMlpIn,
                                   s.trainT + size_t(k) * perStep * 4, perStep, s.stepCount + k, lr,
                                   st, 74);
        if (r) return r;
        k_learned_loss<<<1, 32, 0, st>>>(mlp_loss(net), s.frameLoss);
    }
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
