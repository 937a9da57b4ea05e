/* Host-side R-MAT CSR builder (test infrastructure, part of liboracle.so).
 *
 * Builds the same graph as parex_b200/graphs.py rmat() and the library's
 * device generator (pxr_rmat_edges + pxr_build_csr): edge_factor * 2^scale
 * samples, one quadrant per bit level chosen by a 16-bit uniform from a
 * counter-based splitmix64 hash of (seed, sample, level); self-loops dropped,
 * duplicates merged, both directions stored, rows sorted.  It exists so that
 * the reference's CPU decomposition can be timed on the benchmark's graph
 * without loading the product library (bench.py --impl reference), and so a
 * CPU test can pin the three generators against each other.
 *
 * The sorts are LSD radix sorts on 16-bit digits; memory peaks at about
 * 24 bytes per sample. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static uint64_t hash_at(uint64_t seed, uint64_t stream, uint64_t idx) {
    const uint64_t base = seed * 0x100000001B3ull + stream * 0x9E3779B1ull;
    return splitmix64(splitmix64(idx ^ base) + base);
}

/* sort keys[0..count) in place on bits [0, bits) with a scratch array */
static int radix_sort_u64(uint64_t* keys, uint64_t count, unsigned bits) {
    uint64_t* tmp = (uint64_t*)malloc((count ? count : 1) * sizeof(uint64_t));
    uint64_t* hist = (uint64_t*)malloc(65536 * sizeof(uint64_t));
    if (!tmp || !hist) { free(tmp); free(hist); return -1; }
    uint64_t* src = keys;
    uint64_t* dst = tmp;
    for (unsigned shift = 0; shift < bits; shift += 16) {
        memset(hist, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < count; ++i) hist[(src[i] >> shift) & 0xFFFF]++;
        uint64_t sum = 0;
        for (unsigned d = 0; d < 65536; ++d) { const uint64_t h = hist[d]; hist[d] = sum; sum += h; }
        for (uint64_t i = 0; i < count; ++i) dst[hist[(src[i] >> shift) & 0xFFFF]++] = src[i];
        uint64_t* t = src; src = dst; dst = t;
    }
    if (src != keys) memcpy(keys, src, count * sizeof(uint64_t));
    free(tmp);
    free(hist);
    return 0;
}

/* thresholds: ta = a * 65536, tab = (a + b) * 65536, tabc = (a + b + c) * 65536,
 * each rounded to an integer by the caller.  offsets: n + 1 entries (n =
 * 2^scale); *cols_out is malloc'ed (2m entries), freed with orc_free.
 * Returns 0, or -1 when memory ran out. */
int orc_rmat_csr(uint32_t scale, uint64_t samples, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t seed,
                 uint64_t* offsets, uint32_t** cols_out, uint64_t* m_out) {
    const uint64_t n = 1ull << scale;
    uint64_t* key = (uint64_t*)malloc((samples ? samples : 1) * sizeof(uint64_t));
    if (!key) return -1;
    uint64_t kept = 0;
    for (uint64_t i = 0; i < samples; ++i) {
        uint32_t u = 0, v = 0;
        uint64_t h = 0;
        for (uint32_t lvl = 0; lvl < scale; ++lvl) {
            if (lvl % 4 == 0) h = hash_at(seed, 1000 + lvl / 4, i);
            const uint32_t r = (uint32_t)((h >> (16 * (lvl % 4))) & 0xFFFF);
            const uint32_t bit = 1u << (scale - 1 - lvl);
            if (r >= tab) u |= bit;
            if ((r >= ta && r < tab) || r >= tabc) v |= bit;
        }
        if (u == v) continue;
        const uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
        key[kept++] = (lo << 32) | hi;
    }
    if (radix_sort_u64(key, kept, 64) != 0) { free(key); return -1; }
    uint64_t m = 0;
    for (uint64_t i = 0; i < kept; ++i)
        if (i == 0 || key[i] != key[i - 1]) key[m++] = key[i];
    uint64_t* full = (uint64_t*)malloc((m ? 2 * m : 1) * sizeof(uint64_t));
    if (!full) { free(key); return -1; }
    for (uint64_t i = 0; i < m; ++i) {
        const uint64_t lo = key[i] >> 32, hi = key[i] & 0xFFFFFFFFull;
        full[2 * i] = (lo << 32) | hi;
        full[2 * i + 1] = (hi << 32) | lo;
    }
    free(key);
    if (radix_sort_u64(full, 2 * m, 64) != 0) { free(full); return -1; }
    uint32_t* cols = (uint32_t*)malloc((m ? 2 * m : 1) * sizeof(uint32_t));
    if (!cols) { free(full); return -1; }
    memset(offsets, 0, (n + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < 2 * m; ++i) {
        offsets[(full[i] >> 32) + 1]++;
        cols[i] = (uint32_t)(full[i] & 0xFFFFFFFFull);
    }
    free(full);
    for (uint64_t v = 0; v < n; ++v) offsets[v + 1] += offsets[v];
    *cols_out = cols;
    *m_out = m;
    return 0;
}

void orc_free(void* p) { free(p); }
