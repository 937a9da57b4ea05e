// The learned stop predictor: a 3-layer MLP (16 -> 32 -> 32 -> 1, ReLU)
// with BF16 inputs and weights and FP32 accumulation (sm_100a CUDA cores;
// 1,633 parameters, so the work is latency-bound, not tensor-bound).
//
// Arithmetic contract (restated exactly by the CPU oracle):
//  * a layer input is rounded to bf16 (round to nearest even); weights and
//    biases are bf16 values;
//  * every neuron starts from its bias and adds w * x for x in input order,
//    one float addition per term (the product of two bf16 values is exact
//    in float, so fused and unfused forms agree);
//  * hidden activations are ReLU, then rounded to bf16 for the next layer;
//  * in the backward pass the gradient operands (dL/dy and the
//    pre-activation gradients) are rounded to bf16 before they multiply,
//    sums are float in sample order within a block of kMlpBlockSamples
//    samples, block partials are summed in block order, then divided by n.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace pxr {

constexpr int kMlpIn = 16;
constexpr int kMlpHidden = 32;
constexpr int kOffW1 = 0;                                   // [hidden][in]
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;        // 512
constexpr int kOffW2 = kOffB1 + kMlpHidden;                 // 544, [hidden][hidden]
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;    // 1568
constexpr int kOffW3 = kOffB2 + kMlpHidden;                 // 1600
constexpr int kOffB3 = kOffW3 + kMlpHidden;                 // 1632
constexpr int kMlpParams = kOffB3 + 1;                      // 1633
// float image in shared memory: parameters, then input mean[16] and scale[16]
constexpr int kMlpImage = kMlpParams + 2 * kMlpIn;
constexpr int kMlpBlockSamples = 64;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Widen the bf16 parameters and copy the input normalisation into shared memory.
__device__ __forceinline__ void mlp_load_image(float* img, const uint16_t* w, const float* norm) {
    for (int p = threadIdx.x; p < kMlpImage; p += blockDim.x)
        img[p] = p < kMlpParams ? bf16_bits_to_float(w[p]) : norm[p - kMlpParams];
}

// Forward pass of one sample.  f: raw features; outputs the layer inputs and
// pre-activations the backward pass needs (any of them may be discarded).
__device__ __forceinline__ float mlp_forward(const float* img, const float* f, float* z, float* a1, float* h1,
                                             float* a2, float* h2) {
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i)
        z[i] = bf16_round(__fmul_rn(__fsub_rn(f[i], img[kMlpParams + i]), img[kMlpParams + kMlpIn + i]));
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) a1[o] = img[kOffB1 + o];
#pragma unroll 1
    for (int i = 0; i < kMlpIn; ++i) {
        const float zi = z[i];
#pragma unroll
        for (int o = 0; o < kMlpHidden; ++o) a1[o] = __fadd_rn(a1[o], __fmul_rn(img[kOffW1 + o * kMlpIn + i], zi));
    }
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) h1[o] = bf16_round(fmaxf(a1[o], 0.0f));
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) a2[o] = img[kOffB2 + o];
#pragma unroll 1
    for (int i = 0; i < kMlpHidden; ++i) {
        const float hi = h1[i];
#pragma unroll
        for (int o = 0; o < kMlpHidden; ++o) a2[o] = __fadd_rn(a2[o], __fmul_rn(img[kOffW2 + o * kMlpHidden + i], hi));
    }
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) h2[o] = bf16_round(fmaxf(a2[o], 0.0f));
    float y = img[kOffB3];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) y = __fadd_rn(y, __fmul_rn(img[kOffW3 + i], h2[i]));
    return y;
}

// The output of mlp_forward without its intermediates, for inference: the
// same float operations in the same order (layer-1 neurons summed over the
// inputs in order; each layer-2 neuron summed over layer 1 in order, then
// added to the output in neuron order), so the result is bit-identical,
// with 32 live accumulators instead of 144 stored values.
__device__ __forceinline__ float mlp_infer(const float* img, const float* f) {
    float h1[kMlpHidden];
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) h1[o] = img[kOffB1 + o];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) {
        const float zi = bf16_round(__fmul_rn(__fsub_rn(f[i], img[kMlpParams + i]), img[kMlpParams + kMlpIn + i]));
#pragma unroll
        for (int o = 0; o < kMlpHidden; ++o) h1[o] = __fadd_rn(h1[o], __fmul_rn(img[kOffW1 + o * kMlpIn + i], zi));
    }
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) h1[o] = bf16_round(fmaxf(h1[o], 0.0f));
    float y = img[kOffB3];
#pragma unroll 1
    for (int o = 0; o < kMlpHidden; ++o) {
        float a = img[kOffB2 + o];
#pragma unroll
        for (int i = 0; i < kMlpHidden; ++i) a = __fadd_rn(a, __fmul_rn(img[kOffW2 + o * kMlpHidden + i], h1[i]));
        y = __fadd_rn(y, __fmul_rn(img[kOffW3 + o], bf16_round(fmaxf(a, 0.0f))));
    }
    return y;
}

// Per-cluster features of the schedule (pxr_cluster_record::features).
// s, vol: size and internal volume; pot: potential spread (max - min); sp:
// best sweep sparsity this round (2 when none); prev_*: the same at the
// cluster's previous sweep, dr rounds ago (has_prev false for a new
// cluster); age: sweeps since the cluster was created; round: rounds done.
__device__ __forceinline__ void cluster_features(float* f, uint32_t s, uint32_t vol, float pot, float sp,
                                                 bool has_prev, float prev_pot, float prev_sp, uint32_t dr,
                                                 uint32_t age, uint32_t round, float rw, float sc) {
    const float lp = log10f(fmaxf(pot, 1e-12f) / rw);
    const float spc = fminf(sp, 2.0f);
    const float fdr = (float)(dr > 0 ? dr : 1u);
    const float decay = has_prev ? (lp - log10f(fmaxf(prev_pot, 1e-12f) / rw)) / fdr : 0.0f;
    const float slope = has_prev ? (spc - fminf(prev_sp, 2.0f)) / fdr : 0.0f;
    f[0] = log2f((float)s);
    f[1] = log2f((float)vol + 1.0f);
    f[2] = (float)vol / (float)s / 8.0f;
    f[3] = lp;
    f[4] = decay;
    f[5] = spc;
    f[6] = slope;
    f[7] = spc - sc;
    f[8] = log2f(1.0f + (float)age);
    f[9] = has_prev ? 1.0f : 0.0f;
    f[10] = has_prev ? fminf(fdr, 64.0f) / 8.0f : 0.0f;
    f[11] = log2f(1.0f + (float)round) / 8.0f;
    f[12] = (has_prev && decay < -1e-3f) ? fminf(fmaxf(lp, 0.0f) / -decay, 64.0f) / 16.0f : 4.0f;
    f[13] = (has_prev && slope < -1e-3f) ? fminf(fmaxf(spc - sc, 0.0f) / -slope, 64.0f) / 16.0f : 4.0f;
    f[14] = 0.0f;
    f[15] = 0.0f;
}

// Skipped rounds from the prediction y = log2(1 + safe skips).
__device__ __forceinline__ uint32_t skip_from_prediction(float y, float safety, uint32_t max_skip) {
    if (!(y > 0.0f)) return 0u;
    const float r = floorf(safety * (exp2f(fminf(y, 16.0f)) - 1.0f));
    if (!(r > 0.0f)) return 0u;
    return r >= (float)max_skip ? max_skip : (uint32_t)r;
}

}  // namespace pxr
