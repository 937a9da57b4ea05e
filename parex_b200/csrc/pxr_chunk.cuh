// Chunked sweep sort (sm_100a): the sort of a round done CTA by CTA in
// shared memory, when every cluster of the previous round is small.
//
// The active list is in the previous round's sort order with deactivated
// vertices removed, so the vertices of each previous-round cluster (a
// "parent") form one contiguous run of it, and every cluster of this round
// lies inside one parent's run.  When every parent holds at most kChunkCap
// vertices, CTA k takes the parents whose run starts in
// [k * kChunk, (k + 1) * kChunk) - at most kChunk + kChunkCap - 1 items -
// sorts them stably by (label, potential) with an LSD radix sort in shared
// memory, and writes every cluster to its start position from the cluster
// tables.  The result is the global stable sort's, item for item: the same
// key, the same tie order (the active list's order), the same positions.
// Rounds with larger parents use the global onesweep sort.
#pragma once

#include "pxr_kernels.cuh"

namespace pxr {

constexpr uint32_t kChunk = 4096;
constexpr uint32_t kChunkCap = kChunkCapRows;
constexpr uint32_t kChunkItems = kChunk + kChunkCap;
constexpr int kChunkThreads = 512;
constexpr int kChunkIPT = kChunkItems / kChunkThreads;   // 16 items per thread
constexpr int kChunkWarps = kChunkThreads / 32;
constexpr uint32_t kChunkSlots = 16384;                  // label hash table (in the second key buffer)
// Direct ranking (comparisons within a parent run) is used when no parent
// run of the chunk is longer than this.
constexpr uint32_t kCountRun = 512;

constexpr size_t chunk_sort_smem() {
    return 2 * kChunkItems * sizeof(uint64_t) + 2 * kChunkItems * sizeof(uint32_t) +
           kChunkWarps * 256 * sizeof(uint32_t);
}

// first p >= p0 where a parent run starts (p == 0, or the parent changes), else n
__device__ __forceinline__ uint32_t chunk_boundary(const uint32_t* par, uint32_t p0, uint32_t n, uint32_t* s_min) {
    if (p0 == 0) return 0;
    if (p0 >= n) return n;
    for (uint32_t base = p0; base < n; base += kChunkThreads) {
        if (threadIdx.x == 0) *s_min = n;
        __syncthreads();
        const uint32_t p = base + threadIdx.x;
        if (p < n && par[p] != par[p - 1]) atomicMin(s_min, p);
        __syncthreads();
        const uint32_t found = *s_min;
        __syncthreads();
        if (found < n) return found;
    }
    return n;
}

// block sum over kChunkThreads threads (valid in every thread)
__device__ __forceinline__ uint32_t chunk_block_sum(uint32_t v, uint32_t* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < kChunkWarps; ++w) t += sh[w];
    __syncthreads();
    return t;
}

// One stable LSD pass over cnt items (8-bit digit at `shift`), src -> dst.
__device__ __forceinline__ void chunk_pass(const uint64_t* sk, const uint32_t* sv, uint64_t* dk, uint32_t* dv,
                                           uint32_t cnt, int shift, uint32_t (*whist)[256], uint32_t* tpre,
                                           uint32_t* sh) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt = lanemask_lt();
    for (int i = lane; i < 256; i += 32) whist[warp][i] = 0;
    __syncwarp();
    const uint32_t base = warp * (32 * kChunkIPT);
    uint32_t dg[kChunkIPT], rank[kChunkIPT];
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t j = base + k * 32 + lane;
        dg[k] = j < cnt ? ((uint32_t)(sk[j] >> shift) & 0xFFu) : 0x100u;
    }
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const bool valid = dg[k] < 0x100u;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, dg[k]);
        // the lowest lane of each digit reads and advances the warp's count
        const uint32_t leader = (uint32_t)__ffs(peers) - 1u;
        uint32_t before = 0;
        if (valid && lane == leader) {
            before = whist[warp][dg[k]];
            whist[warp][dg[k]] = before + __popc(peers);
        }
        before = __shfl_sync(0xFFFFFFFFu, before, leader);
        rank[k] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // digit d: offsets of the warps, then the block's exclusive digit prefix
    if (threadIdx.x < 256) {
        const uint32_t d = threadIdx.x;
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kChunkWarps; ++w) {
            const uint32_t c = whist[w][d];
            whist[w][d] = tot;
            tot += c;
        }
        tpre[d] = tot;
    }
    __syncthreads();
    if (threadIdx.x < 32) {   // exclusive scan of 256 digit totals by one warp (8 per lane)
        uint32_t v[8], sum = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) { v[q] = tpre[threadIdx.x * 8 + q]; sum += v[q]; }
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (threadIdx.x >= (uint32_t)o) inc += u;
        }
        uint32_t run = inc - sum;
#pragma unroll
        for (int q = 0; q < 8; ++q) { tpre[threadIdx.x * 8 + q] = run; run += v[q]; }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t j = base + k * 32 + lane;
        if (dg[k] < 0x100u) {
            const uint32_t pos = tpre[dg[k]] + whist[warp][dg[k]] + rank[k];
            dk[pos] = sk[j];
            dv[pos] = sv[j];
        }
    }
    __syncthreads();
    (void)sh;
}

template <typename OffT>
__device__ __forceinline__ void chunk_one(const Dev<OffT>& d, const ClusterTables& t, const uint32_t* act,
                                          const uint32_t* par, uint64_t* keys_out, uint32_t* vals_out, uint32_t lo,
                                          uint32_t n, uint64_t* ka, uint64_t* kb, uint32_t* va, uint32_t* vb,
                                          uint32_t (*whist)[256], uint32_t* tpre, uint32_t* sh, uint32_t* s_min_p,
                                          uint32_t* s_and_p, uint32_t* s_or_p) {
    uint32_t& s_min = *s_min_p;
    uint32_t& s_and = *s_and_p;
    uint32_t& s_or = *s_or_p;
    uint32_t* table = reinterpret_cast<uint32_t*>(kb);   // label hash table until the first pass
    const uint32_t begin = chunk_boundary(par, lo, n, &s_min);
    const uint32_t end = chunk_boundary(par, lo + kChunk, n, &s_min);
    if (begin >= end) return;
    const uint32_t cnt = end - begin;
    if (cnt > kChunkItems) {   // a parent longer than kChunkCap: the path was chosen wrongly
        if (threadIdx.x == 0) atomicOr(&d.ctr->err, kErrLabelRange);
        return;
    }
    for (uint32_t q = threadIdx.x; q < kChunkSlots; q += kChunkThreads) table[q] = 0xFFFFFFFFu;
    if (threadIdx.x == 0) { s_and = 0xFFFFFFFFu; s_or = 0u; }
    // gathers: every load of a thread in flight together
    uint32_t v[kChunkIPT], L[kChunkIPT], xo[kChunkIPT];
#pragma unroll
    for (int r = 0; r < kChunkIPT; ++r) {
        const uint32_t j = threadIdx.x + r * kChunkThreads;
        v[r] = j < cnt ? act[begin + j] : 0u;
    }
#pragma unroll
    for (int r = 0; r < kChunkIPT; ++r) {
        const uint32_t j = threadIdx.x + r * kChunkThreads;
        L[r] = j < cnt ? (uint32_t)d.lab[v[r]] : 0u;
        xo[r] = j < cnt ? ordered_bits(d.x[v[r]]) : 0u;
    }
    // Short parent runs: rank every vertex directly among the vertices of its
    // run with the same label (earlier by potential, ties by list position),
    // which is its place in the stable sort.  Work: sum of squared run lengths.
#pragma unroll
    for (int r = 0; r < kChunkIPT; ++r) {
        const uint32_t j = threadIdx.x + r * kChunkThreads;
        if (j < cnt) {
            ka[j] = ((uint64_t)L[r] << 32) | xo[r];
            va[j] = v[r];
            vb[j] = par[begin + j];
        }
    }
    __syncthreads();
    // parent runs by block scans over a contiguous layout (16 items per thread):
    // run start = last head at or before i, run end = first head after i
    const uint32_t c0 = threadIdx.x * kChunkIPT;
    uint32_t rs[kChunkIPT], re[kChunkIPT];
    uint32_t last = 0;
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t i = c0 + k;
        if (i < cnt && (i == 0 || vb[i] != vb[i - 1])) last = i;
        rs[k] = last;
    }
    uint32_t first = cnt;   // first head after this thread's items, from the right
#pragma unroll
    for (int k = kChunkIPT - 1; k >= 0; --k) {
        const uint32_t i = c0 + k;
        re[k] = first;
        if (i < cnt && (i == 0 || vb[i] != vb[i - 1])) first = i;
    }
    // carries: max of earlier threads' last heads, min of later threads' first heads
    uint32_t mx = last, mn = first;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, mx, o);
        const uint32_t w = __shfl_down_sync(0xFFFFFFFFu, mn, o);
        if ((threadIdx.x & 31u) >= (uint32_t)o) mx = max(mx, u);
        if ((threadIdx.x & 31u) + o < 32u) mn = min(mn, w);
    }
    __syncthreads();
    if ((threadIdx.x & 31u) == 31u) tpre[threadIdx.x >> 5] = mx;           // warp's max head
    if ((threadIdx.x & 31u) == 0u) tpre[32 + (threadIdx.x >> 5)] = mn;      // warp's min first head
    __syncthreads();
    uint32_t before_max = __shfl_up_sync(0xFFFFFFFFu, mx, 1);
    if ((threadIdx.x & 31u) == 0) before_max = 0;
    uint32_t after_min = __shfl_down_sync(0xFFFFFFFFu, mn, 1);
    if ((threadIdx.x & 31u) == 31u) after_min = cnt;
    for (uint32_t w = 0; w < (threadIdx.x >> 5); ++w) before_max = max(before_max, tpre[w]);
    for (uint32_t w = (threadIdx.x >> 5) + 1; w < (uint32_t)kChunkWarps; ++w) after_min = min(after_min, tpre[32 + w]);
    uint32_t longest = 0;
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t i = c0 + k;
        rs[k] = max(rs[k], before_max);
        if (i >= cnt) continue;
        re[k] = min(re[k], after_min);
        longest = max(longest, re[k] - rs[k]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xFFFFFFFFu, longest, o));
    __syncthreads();
    if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = longest;
    __syncthreads();
    uint32_t run_max = 0;
    for (int w = 0; w < kChunkWarps; ++w) run_max = max(run_max, sh[w]);
    __syncthreads();
    if (run_max <= kCountRun) {
        // run bounds to shared memory (the second key buffer is free on this
        // path), then neighbouring lanes rank neighbouring items: the lanes
        // of a warp read the same run, so the reads are broadcasts
        uint32_t* srs = reinterpret_cast<uint32_t*>(kb);
        uint32_t* sre = srs + kChunkItems;
#pragma unroll
        for (int k = 0; k < kChunkIPT; ++k)
            if (c0 + k < cnt) { srs[c0 + k] = rs[k]; sre[c0 + k] = re[k]; }
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < kChunkIPT; ++k) {
            const uint32_t i = threadIdx.x + k * kChunkThreads;
            if (i >= cnt) break;
            const uint64_t ki = ka[i];
            const uint32_t li = (uint32_t)(ki >> 32), xi = (uint32_t)ki;
            const uint32_t jb = srs[i], je = sre[i];
            uint32_t rank = 0;
            for (uint32_t j = jb; j < je; ++j) {
                const uint64_t kj = ka[j];
                const uint32_t xj = (uint32_t)kj;
                rank += ((uint32_t)(kj >> 32) == li && (xj < xi || (xj == xi && j < i))) ? 1u : 0u;
            }
            const uint32_t pos = t.start[li] + rank;
            keys_out[pos] = ki;
            vals_out[pos] = va[i];
        }
        return;
    }
    __syncthreads();
    // local cluster slot: the label's place in a hash table (injective; the
    // order of clusters inside a chunk is irrelevant, positions come from
    // the cluster starts)
    uint32_t slot[kChunkIPT];
    uint32_t a = 0xFFFFFFFFu, o = 0u;
#pragma unroll
    for (int r = 0; r < kChunkIPT; ++r) {
        const uint32_t j = threadIdx.x + r * kChunkThreads;
        const bool valid = j < cnt;
        if (valid) {
            a &= xo[r];
            o |= xo[r];
        }
        // one insertion per distinct label of the warp (the lanes of a
        // cluster would otherwise serialise on one slot)
        const uint32_t key = valid ? L[r] : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
        const int leader = __ffs(peers) - 1;
        uint32_t h = (key * 2654435761u) >> 18;   // 14 bits
        if (valid && (int)(threadIdx.x & 31u) == leader) {
            for (uint32_t probe = 0; probe < kChunkSlots; ++probe) {
                const uint32_t prev = atomicCAS(&table[h], 0xFFFFFFFFu, key);
                if (prev == 0xFFFFFFFFu || prev == key) break;
                h = (h + 1) & (kChunkSlots - 1);
            }
        }
        slot[r] = __shfl_sync(0xFFFFFFFFu, h, leader);
    }
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) {
        a &= __shfl_xor_sync(0xFFFFFFFFu, a, q);
        o |= __shfl_xor_sync(0xFFFFFFFFu, o, q);
    }
    if ((threadIdx.x & 31u) == 0) { atomicAnd(&s_and, a); atomicOr(&s_or, o); }
    __syncthreads();
    // dense local ids: rank of the occupied slots (32 slots per thread)
    uint32_t occ = 0, mine[kChunkSlots / kChunkThreads];
#pragma unroll
    for (int q = 0; q < (int)(kChunkSlots / kChunkThreads); ++q) {
        mine[q] = table[threadIdx.x * (kChunkSlots / kChunkThreads) + q] != 0xFFFFFFFFu ? 1u : 0u;
        occ += mine[q];
    }
    uint32_t inc = occ;
#pragma unroll
    for (int q = 1; q < 32; q <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, inc, q);
        if ((threadIdx.x & 31u) >= (uint32_t)q) inc += u;
    }
    if ((threadIdx.x & 31u) == 31u) sh[threadIdx.x >> 5] = inc;
    __syncthreads();
    uint32_t wbase = 0, distinct = 0;
    for (int w = 0; w < kChunkWarps; ++w) {
        if (w < (int)(threadIdx.x >> 5)) wbase += sh[w];
        distinct += sh[w];
    }
    __syncthreads();
    uint32_t rk = wbase + inc - occ;
#pragma unroll
    for (int q = 0; q < (int)(kChunkSlots / kChunkThreads); ++q) {
        // the slot's dense id replaces its label (each thread rewrites only its own slots)
        const uint32_t idx = threadIdx.x * (kChunkSlots / kChunkThreads) + q;
        table[idx] = mine[q] ? rk : 0u;
        rk += mine[q];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kChunkIPT; ++r) {
        const uint32_t j = threadIdx.x + r * kChunkThreads;
        if (j < cnt) {
            ka[j] = ((uint64_t)table[slot[r]] << 32) | xo[r];
            va[j] = v[r];
        }
    }
    __syncthreads();
    // passes: the potential digits that vary inside the chunk, then the local id's
    const uint32_t varying = s_and ^ s_or;
    const int id_bits = (int)bitlen(distinct > 0 ? distinct - 1 : 0);
    uint64_t *sk = ka, *dk = kb;
    uint32_t *sv = va, *dv = vb;
    for (int shift = 0; shift < 32 + id_bits; shift += 8) {
        if (shift < 32 && ((varying >> shift) & 0xFFu) == 0u) continue;
        chunk_pass(sk, sv, dk, dv, cnt, shift, whist, tpre, sh);
        uint64_t* tk = sk; sk = dk; dk = tk;
        uint32_t* tv = sv; sv = dv; dv = tv;
    }
    // write out: position = cluster start + index inside the cluster's run
    const uint32_t q0 = threadIdx.x * kChunkIPT;
    uint32_t head = 0;   // last run start at or before this thread's items
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t q = q0 + k;
        if (q < cnt && (q == 0 || (sk[q] >> 32) != (sk[q - 1] >> 32))) head = q;
    }
    uint32_t hinc = head;
#pragma unroll
    for (int q = 1; q < 32; q <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, hinc, q);
        if ((threadIdx.x & 31u) >= (uint32_t)q) hinc = max(hinc, u);
    }
    if ((threadIdx.x & 31u) == 31u) sh[threadIdx.x >> 5] = hinc;
    __syncthreads();
    uint32_t carry = 0;
    for (uint32_t w = 0; w < (threadIdx.x >> 5); ++w) carry = max(carry, sh[w]);
    uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, hinc, 1);
    if ((threadIdx.x & 31u) == 0) prev = 0;
    uint32_t run = max(carry, prev);
    uint32_t vv[kChunkIPT], LL[kChunkIPT];
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t q = q0 + k;
        vv[k] = q < cnt ? sv[q] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) LL[k] = q0 + k < cnt ? (uint32_t)d.lab[vv[k]] : 0u;
#pragma unroll
    for (int k = 0; k < kChunkIPT; ++k) {
        const uint32_t q = q0 + k;
        if (q >= cnt) break;
        const uint64_t key = sk[q];
        if (q == 0 || (key >> 32) != (sk[q - 1] >> 32)) run = q;
        const uint32_t pos = t.start[LL[k]] + (q - run);
        keys_out[pos] = ((uint64_t)LL[k] << 32) | (uint32_t)key;
        vals_out[pos] = vv[k];
    }
}

template <typename OffT>
__global__ void __launch_bounds__(kChunkThreads, 1) k_chunk_sort(Dev<OffT> d, ClusterTables t, const uint32_t* act,
                                                                 const uint32_t* par, uint64_t* keys_out,
                                                                 uint32_t* vals_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* ka = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* kb = ka + kChunkItems;
    uint32_t* va = reinterpret_cast<uint32_t*>(kb + kChunkItems);
    uint32_t* vb = va + kChunkItems;
    uint32_t (*whist)[256] = reinterpret_cast<uint32_t (*)[256]>(vb + kChunkItems);
    __shared__ uint32_t tpre[256];
    __shared__ uint32_t sh[kChunkWarps];
    __shared__ uint32_t s_min, s_and, s_or;

    if (!d.ctr->chunk_path) return;
    const uint32_t n = d.ctr->n_active;
    for (uint32_t chunk = blockIdx.x; chunk * kChunk < n; chunk += gridDim.x) {
        chunk_one(d, t, act, par, keys_out, vals_out, chunk * kChunk, n, ka, kb, va, vb, whist, tpre, sh, &s_min,
                  &s_and, &s_or);
        __syncthreads();
    }
}

}  // namespace pxr
