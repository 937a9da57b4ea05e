// Initial potentials x0[v] ~ N(0, sqrt(deg v)) (RandomWalkManager::initRandomWalk,
// cuda/devRandomWalk.h:22-48 and 509-519).
//
// Per vertex: seed = hash(seed ^ v) with the reference's 3-round
// xorshift-multiply hash; one step of the minimal-standard LCG
// (x <- 48271 x mod 2^31-1, the engine thrust::default_random_engine names);
// the inverse-CDF normal sample z = -sqrt(2) erfcinv(2p) with p the LCG
// output mapped to [0, 1/2) and the sign folded into the factor, as thrust's
// normal_distribution does for device code; scaled by float(sqrt(deg)).
//
// This translation unit is compiled with --use_fast_math, the reference's
// flag, so that erfcinvf is evaluated in the same compilation mode.
#include <cstdint>
#include <cuda_runtime.h>

namespace pxr {

__device__ __forceinline__ uint32_t hash_idx(uint32_t x) {
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = (x >> 16) ^ x;
    return x;
}

template <typename OffT>
__global__ void k_initial_potentials(const OffT* off, uint32_t n, uint32_t seed, float* x, uint32_t* xmax_bits) {
    constexpr uint32_t kModulus = 2147483647u, kMult = 48271u;
    constexpr uint32_t kRange = 2147483646u - 1u;  // engine max - min
    const float s1 = (float)(1.0 / (double)kRange);
    const float s2 = s1 / 2.0f;
    uint32_t vmax = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t state = hash_idx(seed ^ v) % kModulus;
        if (state == 0) state = 1;
        state = (uint32_t)(((uint64_t)kMult * state) % kModulus);
        uint32_t u = state - 1u;
        float s3 = -1.41421356237309504880f;
        if (u > kRange / 2u) {
            u = kRange - u;
            s3 = -s3;
        }
        const float p = __fmaf_rn((float)u, s1, s2);
        const float stddev = (float)sqrt((double)(off[v + 1] - off[v]));
        const float z = erfcinvf(2.0f * p);
        const float xv = __fmul_rn(__fmul_rn(stddev, s3), z);
        x[v] = xv;
        const uint32_t b = __float_as_uint(fabsf(xv));
        vmax = b > vmax ? b : vmax;
    }
    for (int o = 16; o > 0; o >>= 1) vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
    if ((threadIdx.x & 31u) == 0 && vmax) atomicMax(xmax_bits, vmax);
}

void launch_initial_potentials(const void* off, bool off64, uint32_t n, uint32_t seed, float* x,
                               uint32_t* xmax_bits, cudaStream_t stream) {
    if (n == 0) return;
    const uint32_t grid = (n + 255u) / 256u < 148u * 16u ? (n + 255u) / 256u : 148u * 16u;
    if (off64)
        k_initial_potentials<uint64_t><<<grid, 256, 0, stream>>>((const uint64_t*)off, n, seed, x, xmax_bits);
    else
        k_initial_potentials<uint32_t><<<grid, 256, 0, stream>>>((const uint32_t*)off, n, seed, x, xmax_bits);
}

}  // namespace pxr
