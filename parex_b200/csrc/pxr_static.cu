// Final partition without any device allocation.
//
// Who needs this: callers that must not call cudaMalloc / cudaFree at the
// point where they want the cluster ids - for example a service whose device
// memory is owned by a pooling allocator that has to account for every byte,
// or a latency-bound pipeline that cannot afford the implicit device
// synchronisation cudaMalloc and cudaFree may perform.  Every other entry
// point allocates its working memory when a graph is initialised; this one
// works on arrays the caller already owns and keeps its scratch in a
// fixed-size array that lives in this file, allocated once when the library
// is loaded.
//
// The scratch array (g_scratch) is a file-scope __device__ array: every GPU
// that loads the library holds it (about 1.1 MB) until the process exits.
// Host code cannot use g_scratch's name as an address - in host code that
// name is only a stand-in - so every call resolves the real device address
// with cudaGetSymbolAddress while the caller's device is current (nothing is
// cached, so a cudaDeviceReset between calls is harmless).  The first call
// on a device also loads the library's kernels there and should therefore be
// made before any stream capture begins.
//
// All calls share the one array and it keeps the previous call's contents,
// so every call first clears the parts that must start at zero.  Calls whose
// work overlaps on the GPU (different streams, no ordering between them)
// race on the array and must be avoided.
#include "pxr_kernels.cuh"

namespace pxr {
namespace noalloc {

constexpr uint32_t kMaxLabels = PXR_STATIC_SCRATCH_MAX_LABELS;
constexpr uint32_t kSortTiles = kMaxLabels / kSortTile + 1;
constexpr uint32_t kRankTiles = kMaxLabels / kScanTile + 1;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// byte offsets of the pieces inside the scratch array
constexpr size_t kKeys0 = 0;
constexpr size_t kKeys1 = align256(kKeys0 + 4ull * kMaxLabels);
constexpr size_t kVals0 = align256(kKeys1 + 4ull * kMaxLabels);
constexpr size_t kVals1 = align256(kVals0 + 4ull * kMaxLabels);
constexpr size_t kCtrl = align256(kVals1 + 4ull * kMaxLabels);   // start of the region cleared per call
constexpr size_t kHist = kCtrl;
constexpr size_t kBases = align256(kHist + 4ull * kMaxPasses * kRadix);
constexpr size_t kPassInfo = align256(kBases + 4ull * kMaxPasses * kRadix);
constexpr size_t kTileCtr = align256(kPassInfo + 4ull * (kMaxPasses + 1));
constexpr size_t kEpoch = align256(kTileCtr + 4ull * kMaxPasses);
constexpr size_t kStatus = align256(kEpoch + 4);
constexpr size_t kLbFlags = align256(kStatus + 8ull * kSortTiles * kRadix);
constexpr size_t kLbAgg = align256(kLbFlags + 4ull * kRankTiles);
constexpr size_t kLbInc = align256(kLbAgg + 8ull * kRankTiles);
constexpr size_t kCtr = align256(kLbInc + 8ull * kRankTiles);
constexpr size_t kCount = align256(kCtr + sizeof(RoundCtr));
constexpr size_t kEndBit = kCount + 4;
constexpr size_t kBytes = align256(kEndBit + 4);
// words cleared per call: the control region up to the item count and end
// bit, which block 0 writes while the other blocks clear (so never cleared)
constexpr size_t kCtrlWords = (kCount - kCtrl) / 4;

static __device__ __align__(256) unsigned char g_scratch[kBytes];

// Clear the control region, then load (label ^ sign bit, vertex) pairs and
// set the item count and end bit (outside the cleared words).
__global__ void k_static_setup(unsigned char* base, const int32_t* labels, uint32_t n) {
    uint32_t* ctrl = reinterpret_cast<uint32_t*>(base + kCtrl);
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + kKeys0);
    uint32_t* vals = reinterpret_cast<uint32_t*>(base + kVals0);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kCtrlWords; i += stride) ctrl[i] = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        keys[i] = (uint32_t)labels[i] ^ 0x80000000u;
        vals[i] = i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *reinterpret_cast<uint32_t*>(base + kCount) = n;
        *reinterpret_cast<uint32_t*>(base + kEndBit) = 32u;
    }
}

// Rank the distinct labels of the sorted pairs (decoupled look-back over
// head flags) and scatter each vertex's rank.  The variant of the rank step
// of pxr_final_partition with its look-back state in the scratch array.
__global__ void __launch_bounds__(kBlock) k_static_rank(unsigned char* base, int32_t* ids, int32_t* num_out) {
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t* pass_info = reinterpret_cast<const uint32_t*>(base + kPassInfo);
    const uint32_t sel = pass_info[kMaxPasses];
    const uint32_t* keys = reinterpret_cast<const uint32_t*>(base + (sel ? kKeys1 : kKeys0));
    const uint32_t* vals = reinterpret_cast<const uint32_t*>(base + (sel ? kVals1 : kVals0));
    RoundCtr* ctr = reinterpret_cast<RoundCtr*>(base + kCtr);
    LookbackState lb{reinterpret_cast<uint32_t*>(base + kLbFlags), reinterpret_cast<uint64_t*>(base + kLbAgg),
                     reinterpret_cast<uint64_t*>(base + kLbInc)};
    const uint32_t count = *reinterpret_cast<const uint32_t*>(base + kCount);
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(ctr, 0);
    if (tile >= ntiles) return;
    const uint32_t epoch = 1u;  // the flags were cleared by k_static_setup
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t heads = 0, run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        if (i < count && (i == 0 || keys[i] != keys[i - 1])) { heads |= 1u << k; ++run; }
    }
    uint64_t total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(lb, tile, epoch, total, &ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
        // a device-side wait that ran out (sort or look-back) is reported as -1
        if (threadIdx.x == 0 && tile == ntiles - 1) *num_out = ctr->err ? -1 : (int32_t)(ex + total);
    }
    __syncthreads();
    uint32_t r = (uint32_t)(s_excl + incl - run);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        if (i >= count) break;
        if (heads & (1u << k)) ++r;
        ids[vals[i]] = (int32_t)r - 1;
    }
}

__global__ void k_static_zero(int32_t* num_out) { *num_out = 0; }

// Device address of g_scratch on the current device, looked up on every call
// with that device current, and the sort kernels' shared-memory attribute
// set again: both are cheap, and nothing cached can outlive a
// cudaDeviceReset in the caller's process.
cudaError_t scratch_for_current_device(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    e = radix_sort_prepare<uint32_t>();
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

}  // namespace noalloc
}  // namespace pxr

extern "C" pxr_status pxr_final_partition_static(const int32_t* labels, uint32_t n, int32_t* ids,
                                                 int32_t* num_clusters, void* stream) {
    using namespace pxr;
    using namespace pxr::noalloc;
    if (n > kMaxLabels) return PXR_INVALID_ARG;  // beyond the fixed scratch: use pxr_final_partition
    if (!num_clusters || (n > 0 && (!labels || !ids))) return PXR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    if (scratch_for_current_device(&base) != cudaSuccess) return PXR_CUDA_ERROR;
    if (n == 0) {
        k_static_zero<<<1, 1, 0, s>>>(num_clusters);
        return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
    }
    k_static_setup<<<64, kBlock, 0, s>>>(base, labels, n);
    SortBuffers<uint32_t> b{};
    b.keys[0] = reinterpret_cast<uint32_t*>(base + kKeys0);
    b.keys[1] = reinterpret_cast<uint32_t*>(base + kKeys1);
    b.vals[0] = reinterpret_cast<uint32_t*>(base + kVals0);
    b.vals[1] = reinterpret_cast<uint32_t*>(base + kVals1);
    b.count = reinterpret_cast<const uint32_t*>(base + kCount);
    b.end_bit = reinterpret_cast<const uint32_t*>(base + kEndBit);
    b.capacity = n;
    SortState st{};
    st.hist = reinterpret_cast<uint32_t*>(base + kHist);
    st.bases = reinterpret_cast<uint32_t*>(base + kBases);
    st.pass_info = reinterpret_cast<uint32_t*>(base + kPassInfo);
    st.tile_ctr = reinterpret_cast<uint32_t*>(base + kTileCtr);
    st.epoch = reinterpret_cast<uint32_t*>(base + kEpoch);
    st.status = reinterpret_cast<uint64_t*>(base + kStatus);
    st.max_tiles = kSortTiles;
    st.items_moved = nullptr;
    RoundCtr* ctr = reinterpret_cast<RoundCtr*>(base + kCtr);
    if (radix_sort<uint32_t>(b, st, &ctr->err, s, 32) != cudaSuccess) return PXR_CUDA_ERROR;
    const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    k_static_rank<<<tiles, kBlock, 0, s>>>(base, ids, num_clusters);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}
