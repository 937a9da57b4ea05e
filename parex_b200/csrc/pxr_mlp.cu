// Training and batch inference of the learned stop predictor (sm_100a):
// forward, loss gradient and Adam step as hand-written kernels with bf16
// operands and float accumulation.  The arithmetic contract is stated in
// pxr_mlp.cuh; every sum runs in a fixed order, so a training run is
// deterministic and the CPU oracle reproduces it bit for bit.
#include <algorithm>
#include <cmath>

#include "pxr_mlp.cuh"
#include "../../include/parex_b200.h"

namespace pxr {
namespace {

constexpr int kMlpThreads = 256;

__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_forward(const float* X, uint32_t n, const uint16_t* w,
                                                              const float* norm, float* Y) {
    __shared__ float img[kMlpImage];
    mlp_load_image(img, w, norm);
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float f[kMlpIn], z[kMlpIn], a1[kMlpHidden], h1[kMlpHidden], a2[kMlpHidden], h2[kMlpHidden];
#pragma unroll
        for (int q = 0; q < kMlpIn; ++q) f[q] = X[(size_t)i * kMlpIn + q];
        Y[i] = mlp_forward(img, f, z, a1, h1, a2, h2);
    }
}

// One block of kMlpBlockSamples samples: forward, loss, backward per sample
// (threads 0..63), then every parameter's gradient summed over the block's
// samples in sample order.  partial: [blocks][kMlpParams + 1], the last entry
// the block's summed loss.
__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_grad_partial(const float* X, const float* T, uint32_t n,
                                                                   const uint16_t* w, const float* norm, float delta,
                                                                   float over, float* partial) {
    __shared__ float img[kMlpImage];
    __shared__ float sZ[kMlpBlockSamples][kMlpIn];
    __shared__ float sH1[kMlpBlockSamples][kMlpHidden];
    __shared__ float sH2[kMlpBlockSamples][kMlpHidden];
    __shared__ float sD1[kMlpBlockSamples][kMlpHidden];
    __shared__ float sD2[kMlpBlockSamples][kMlpHidden];
    __shared__ float sG[kMlpBlockSamples];
    __shared__ float sL[kMlpBlockSamples];
    mlp_load_image(img, w, norm);
    __syncthreads();
    if (threadIdx.x < kMlpBlockSamples) {
        const uint32_t t = threadIdx.x;
        const uint32_t i = blockIdx.x * kMlpBlockSamples + t;
        float z[kMlpIn], a1[kMlpHidden], h1[kMlpHidden], a2[kMlpHidden], h2[kMlpHidden];
        if (i < n) {
            float f[kMlpIn];
#pragma unroll
            for (int q = 0; q < kMlpIn; ++q) f[q] = X[(size_t)i * kMlpIn + q];
            const float y = mlp_forward(img, f, z, a1, h1, a2, h2);
            const float e = __fsub_rn(y, T[i]);
            const float ae = fabsf(e);
            const float wt = e > 0.0f ? over : 1.0f;
            const float loss = __fmul_rn(wt, ae <= delta ? __fmul_rn(__fmul_rn(0.5f, e), e)
                                                         : __fmul_rn(delta, __fsub_rn(ae, __fmul_rn(0.5f, delta))));
            const float g = __fmul_rn(wt, ae <= delta ? e : copysignf(delta, e));
            const float gb = bf16_round(g);
            float d2[kMlpHidden];
#pragma unroll
            for (int o = 0; o < kMlpHidden; ++o)
                d2[o] = bf16_round(a2[o] > 0.0f ? __fmul_rn(img[kOffW3 + o], gb) : 0.0f);
#pragma unroll
            for (int q = 0; q < kMlpHidden; ++q) {
                float dh = 0.0f;
#pragma unroll
                for (int o = 0; o < kMlpHidden; ++o) dh = __fadd_rn(dh, __fmul_rn(img[kOffW2 + o * kMlpHidden + q], d2[o]));
                sD1[t][q] = bf16_round(a1[q] > 0.0f ? dh : 0.0f);
                sD2[t][q] = d2[q];
                sH1[t][q] = h1[q];
                sH2[t][q] = h2[q];
            }
#pragma unroll
            for (int q = 0; q < kMlpIn; ++q) sZ[t][q] = z[q];
            sG[t] = gb;
            sL[t] = loss;
        } else {
            for (int q = 0; q < kMlpHidden; ++q) sD1[t][q] = sD2[t][q] = sH1[t][q] = sH2[t][q] = 0.0f;
            for (int q = 0; q < kMlpIn; ++q) sZ[t][q] = 0.0f;
            sG[t] = 0.0f;
            sL[t] = 0.0f;
        }
    }
    __syncthreads();
    float* out = partial + (size_t)blockIdx.x * (kMlpParams + 1);
    for (int p = threadIdx.x; p < kMlpParams + 1; p += blockDim.x) {
        float acc = 0.0f;
        if (p < kOffB1) {
            const int o = p / kMlpIn, q = p % kMlpIn;
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, __fmul_rn(sD1[s][o], sZ[s][q]));
        } else if (p < kOffW2) {
            const int o = p - kOffB1;
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, sD1[s][o]);
        } else if (p < kOffB2) {
            const int o = (p - kOffW2) / kMlpHidden, q = (p - kOffW2) % kMlpHidden;
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, __fmul_rn(sD2[s][o], sH1[s][q]));
        } else if (p < kOffW3) {
            const int o = p - kOffB2;
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, sD2[s][o]);
        } else if (p < kOffB3) {
            const int q = p - kOffW3;
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, __fmul_rn(sG[s], sH2[s][q]));
        } else if (p == kOffB3) {
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, sG[s]);
        } else {
            for (int s = 0; s < kMlpBlockSamples; ++s) acc = __fadd_rn(acc, sL[s]);
        }
        out[p] = acc;
    }
}

// block partials summed in block order, divided by n
__global__ void k_mlp_reduce(const float* partial, uint32_t blocks, uint32_t n, float* grad, float* loss) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kMlpParams + 1; p += gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (uint32_t b = 0; b < blocks; ++b) acc = __fadd_rn(acc, partial[(size_t)b * (kMlpParams + 1) + p]);
        const float mean = __fdiv_rn(acc, (float)n);
        if (p < kMlpParams) grad[p] = mean;
        else if (loss) *loss = mean;
    }
}

// Adam with the bias corrections c1 = 1 - beta1^t, c2 = 1 - beta2^t given
__global__ void k_mlp_adam(float* master, float* m, float* v, const float* grad, uint16_t* w, float lr, float b1,
                           float b2, float eps, float c1, float c2) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kMlpParams; p += gridDim.x * blockDim.x) {
        const float g = grad[p];
        const float mp = __fadd_rn(__fmul_rn(b1, m[p]), __fmul_rn(__fsub_rn(1.0f, b1), g));
        const float vp = __fadd_rn(__fmul_rn(b2, v[p]), __fmul_rn(__fsub_rn(1.0f, b2), __fmul_rn(g, g)));
        m[p] = mp;
        v[p] = vp;
        const float mh = __fdiv_rn(mp, c1);
        const float vh = __fdiv_rn(vp, c2);
        const float step = __fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(__fsqrt_rn(vh), eps));
        const float x = __fsub_rn(master[p], step);
        master[p] = x;
        w[p] = __bfloat16_as_ushort(__float2bfloat16_rn(x));
    }
}

inline uint32_t mlp_blocks(uint32_t n) { return (n + kMlpBlockSamples - 1) / kMlpBlockSamples; }

}  // namespace
}  // namespace pxr

using namespace pxr;

extern "C" {

pxr_status pxr_mlp_forward(const float* features, uint32_t n, const uint16_t* weights, const float* norm, float* out,
                           void* stream) {
    if (!weights || !norm || (n && (!features || !out))) return PXR_INVALID_ARG;
    if (!n) return PXR_OK;
    const uint32_t grid = std::min<uint32_t>((n + kMlpThreads - 1) / kMlpThreads, 148u * 8u);
    k_mlp_forward<<<grid, kMlpThreads, 0, static_cast<cudaStream_t>(stream)>>>(features, n, weights, norm, out);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}

size_t pxr_mlp_scratch_floats(uint32_t n) { return (size_t)std::max<uint32_t>(mlp_blocks(n), 1u) * (kMlpParams + 1); }

pxr_status pxr_mlp_gradient(const float* features, const float* targets, uint32_t n, const uint16_t* weights,
                            const float* norm, const pxr_mlp_loss* loss, float* scratch, float* grad, float* loss_out,
                            void* stream) {
    if (!features || !targets || !weights || !norm || !loss || !scratch || !grad || n == 0) return PXR_INVALID_ARG;
    if (!(loss->delta > 0.0f) || !(loss->over_weight > 0.0f)) return PXR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t blocks = mlp_blocks(n);
    k_mlp_grad_partial<<<blocks, kMlpThreads, 0, s>>>(features, targets, n, weights, norm, loss->delta,
                                                      loss->over_weight, scratch);
    k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256, 0, s>>>(scratch, blocks, n, grad, loss_out);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}

pxr_status pxr_mlp_adam_step(float* master, float* m, float* v, const float* grad, uint16_t* weights, uint32_t step,
                             const pxr_mlp_adam* opt, void* stream) {
    if (!master || !m || !v || !grad || !weights || !opt || step == 0) return PXR_INVALID_ARG;
    const float c1 = (float)(1.0 - std::pow((double)opt->beta1, (double)step));
    const float c2 = (float)(1.0 - std::pow((double)opt->beta2, (double)step));
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        master, m, v, grad, weights, opt->lr, opt->beta1, opt->beta2, opt->eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}

}  // extern "C"
