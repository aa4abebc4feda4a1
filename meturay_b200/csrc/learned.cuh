// Learned guiding in the wavefront tracer: the MLP's mixture replaces the
// octree product sampler once it has trained (learned.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "guide.cuh"
#include "mlp.cuh"
#include "shade.cuh"
#include "svo_dev.cuh"

namespace mrb {

struct LearnedScratch {
    float* trainX;        // capacity x 80
    float* trainT;        // capacity x 4
    uint32_t* pathCount;  // paths + 1
    uint32_t* pathOffset; // paths + 1
    void* scanTemp;
    uint32_t* stepCount;  // steps
    uint32_t capacity;    // training samples per frame
    uint32_t steps;       // optimiser steps per frame
    float* frameLoss;     // 2: weighted loss and weight sums of the frame's batches
    float weightMax;      // training weights capped at this (0: no cap)
    uint32_t product;     // 1: weights carry |cos| at the vertex (target L_in |cos|)
};

// Guide words for one wavefront from the network, in one kernel: features
// of every ray's hit, the forward pass, then per ray a draw from the vMF
// mixture (with probability misRatio) or from the BxDF, the one-sample MIS
// pdf of the drawn direction, and its octahedral coordinates (half
// precision, as the octree sampler writes them).  Rays at specular
// surfaces, lights or none get no guide word.
int learned_guide_wavefront(const SceneDev& sc, const GuideDev& g, const GuideWave& w,
                            const MlpDev& net, const LearnedScratch& s, float misRatio,
                            const PathOptions& opt, uint32_t depthTag, uint2* guide,
                            cudaStream_t st);

// Training samples of the frame from the path chain: every non-specular
// vertex whose path ray carried radiance gives its features, the ray's
// direction and the weight lum(L_in) / pdf (times |cos| at the vertex with
// s.product), L_in the radiance that arrived along it.  Sample j goes to
// step j mod steps; the per-step counts are written for learned_train.
int learned_collect(const GuideDev& g, const PathChain& pc, const uint32_t* frame,
                    const LearnedScratch& s, cudaStream_t st);
// `steps` Adam steps on the collected samples, step k on its share; the
// frame loss sums the batches' losses, each scored before its step.
int learned_train(mrb_mlp* net, const LearnedScratch& s, float lr, cudaStream_t st);
// Exponential moving average of the parameters for inference:
// ema = beta ema + (1 - beta) params, then out = ema (fp32).
int learned_ema(const float* params, float* ema, float beta, float* out, cudaStream_t st);
size_t learned_scan_temp_bytes(uint32_t paths);
uint32_t learned_launches(uint32_t steps);

}  // namespace mrb
