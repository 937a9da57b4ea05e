/* CPU oracle for the random-walk expander decomposition round (test infrastructure;
 * see pxr_oracle.h).  Each function names the reference code it restates.
 * Build with -ffp-contract=off: every floating-point operation here is one
 * IEEE operation, the same sequence the CUDA product issues with _rn
 * intrinsics. */
#include "pxr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_state {
    int mode;
    uint32_t n;
    uint64_t m, slots;
    uint64_t* off;
    uint32_t* cols;
    float sc_threshold, rw_threshold;
    uint32_t nb_bits;        /* bit length of max(n, max row length): fixed-point headroom */

    int32_t* labels;
    uint32_t* ideg;
    /* potentials: REF mode uses xd[2] (double buffers, swapped per walk);
     * PXR mode uses xf (float, updated in place) and xt (x / internal degree). */
    double* xd[2];
    int cur;
    float* xf;
    float* xt;
    float xmax;              /* PXR: max |x| over the vertices last updated */

    orc_lnode* act;
    uint32_t n_act;
    uint32_t n_clusters;     /* numActiveClusters */
    int32_t smallest;        /* *d_smallestLabel */

    uint64_t* keys;          /* per act position */
    orc_node_data* nd;       /* per act position, nodeDiff output */
    orc_node_data* sorted;   /* post-scan NodeData in sweep order */
    int32_t* ulabels;
    uint32_t* vols;
    int32_t* lookup;         /* labelLookup, size n */
    orc_sweep_cut* allcuts;
    orc_sweep_cut* cuts;
    uint32_t k_sweep, n_cut;
    int32_t* clabels;
    orc_cluster_data* cdata;
    double* csum_fixed_avg;  /* PXR: per data cluster, the exact average */
    uint32_t k_data;
    uint32_t* parent;
    uint32_t* tmp_u32;
    /* certificate record (no reference counterpart): per vertex, the round in
     * which its cluster was certified (+1) with bit 31 set when the certified
     * set is not the whole set swept that round (cut, or split into
     * components); 0 while active.  sweep_of / sweep_cnt / sweep_cut hold the
     * last sweep's cluster of each vertex, its size and its cut decision. */
    uint32_t* cert;
    int32_t* sweep_of;
    uint32_t* sweep_cnt;
    uint8_t* sweep_cut;
    uint32_t round;
};

static void* xcalloc(size_t count, size_t size) {
    void* p = calloc(count ? count : 1, size ? size : 1);
    if (!p) abort();
    return p;
}

/* ------------------------------------------------------------------------ */
/* key packing: cuda/devRandomWalk.h:50-67                                   */

static uint32_t ordered_float_bits(float v) {
    uint32_t i;
    memcpy(&i, &v, 4);
    const uint32_t mask = (i & 0x80000000u) ? 0xFFFFFFFFu : 0x80000000u;
    return i ^ mask;
}

static uint64_t pack_key(int32_t label, float v) {
    const uint32_t ol = (uint32_t)label ^ 0x80000000u;
    return ((uint64_t)ol << 32) | ordered_float_bits(v);
}

static int32_t key_label(uint64_t key) {  /* extractLabel, cuda/devSweepCut.h:295-299 */
    return (int32_t)((uint32_t)(key >> 32) ^ 0x80000000u);
}

static float potential_f(const orc_state* s, uint32_t v) {
    return s->mode == ORC_MODE_REF ? (float)s->xd[s->cur][v] : s->xf[v];
}

/* ------------------------------------------------------------------------ */
/* fixed-point helpers for ORC_MODE_PXR                                      */

static int fixed_exponent(float xmax, uint32_t nb_bits) {
    if (!(xmax > 0.0f) || isinf(xmax)) return 0;
    int ex;
    frexpf(xmax, &ex);                 /* xmax < 2^ex */
    int e = 62 - ex - (int)nb_bits;
    if (e > 900) e = 900;
    if (e < -900) e = -900;
    return e;
}

static int64_t to_fixed(float v, double scale) {
    return (int64_t)llrint((double)v * scale);
}

/* ------------------------------------------------------------------------ */
/* x0: cuda/devRandomWalk.h:22-48 with thrust's minstd engine and its
 * inverse-CDF normal sampler; erfcinv is this file's own (Newton on erfc). */

static uint32_t hash_idx(uint32_t x) {
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = (x >> 16) ^ x;
    return x;
}

static double erfcinv_newton(double y) {
    /* solve erfc(z) = y for y in (0, 2) */
    if (y <= 0.0) return INFINITY;
    if (y >= 2.0) return -INFINITY;
    double t = y < 1.0 ? y : 2.0 - y;
    /* initial guess from the tail asymptotics */
    double z = sqrt(-log(t / 2.0)) * 0.9;
    if (t > 0.5) z = (1.0 - t) * 0.886226925452758;   /* near the centre: erfinv ~ sqrt(pi)/2 x */
    for (int it = 0; it < 60; ++it) {
        double f = erfc(z) - t;
        double d = -2.0 / sqrt(3.14159265358979323846) * exp(-z * z);
        double step = f / d;
        z -= step;
        if (fabs(step) < 1e-17 * (1.0 + fabs(z))) break;
    }
    return y < 1.0 ? z : -z;
}

void orc_initial_potentials(uint32_t n, const uint64_t* off, uint32_t seed, float* out) {
    const uint32_t modulus = 2147483647u, mult = 48271u;
    const uint32_t range = 2147483646u - 1u;         /* max - min of minstd_rand */
    const float s1 = (float)(1.0 / (double)range);
    const float s2 = s1 / 2.0f;
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t tseed = hash_idx(seed ^ v);
        uint32_t state = tseed % modulus;
        if (state == 0) state = 1;
        state = (uint32_t)(((uint64_t)mult * state) % modulus);
        uint32_t u = state - 1u;
        float s3 = -1.41421356237309504880f;
        if (u > range / 2u) { u = range - u; s3 = -s3; }
        const float p = fmaf((float)u, s1, s2);
        const float stddev = (float)sqrt((double)(off[v + 1] - off[v]));
        const float z = (float)erfcinv_newton((double)(2.0f * p));
        out[v] = (stddev * s3) * z;
    }
}

/* ------------------------------------------------------------------------ */
/* construction: GraphManager / PartitionManager / RandomWalkManager ctors    */

orc_state* orc_create(uint32_t n, uint64_t m, const uint64_t* offsets, const uint32_t* cols,
                      int mode, float sc_threshold, float rw_threshold) {
    orc_state* s = (orc_state*)xcalloc(1, sizeof(orc_state));
    s->mode = mode;
    s->n = n;
    s->m = m;
    s->slots = 2 * m;
    s->sc_threshold = sc_threshold;
    s->rw_threshold = rw_threshold;
    s->off = (uint64_t*)xcalloc(n + 1, 8);
    memcpy(s->off, offsets, (size_t)(n + 1) * 8);
    s->cols = (uint32_t*)xcalloc(s->slots, 4);
    if (s->slots) memcpy(s->cols, cols, s->slots * 4);
    s->labels = (int32_t*)xcalloc(n, 4);
    s->ideg = (uint32_t*)xcalloc(n, 4);
    s->xd[0] = (double*)xcalloc(n, 8);
    s->xd[1] = (double*)xcalloc(n, 8);
    s->xf = (float*)xcalloc(n, 4);
    s->xt = (float*)xcalloc(n, 4);
    s->act = (orc_lnode*)xcalloc(n, sizeof(orc_lnode));
    s->keys = (uint64_t*)xcalloc(n, 8);
    s->nd = (orc_node_data*)xcalloc(n, sizeof(orc_node_data));
    s->sorted = (orc_node_data*)xcalloc(n, sizeof(orc_node_data));
    s->ulabels = (int32_t*)xcalloc(n, 4);
    s->vols = (uint32_t*)xcalloc(n, 4);
    s->lookup = (int32_t*)xcalloc(n, 4);
    s->allcuts = (orc_sweep_cut*)xcalloc(n, sizeof(orc_sweep_cut));
    s->cuts = (orc_sweep_cut*)xcalloc(n, sizeof(orc_sweep_cut));
    s->clabels = (int32_t*)xcalloc(n, 4);
    s->cdata = (orc_cluster_data*)xcalloc(n, sizeof(orc_cluster_data));
    s->csum_fixed_avg = (double*)xcalloc(n, 8);
    s->parent = (uint32_t*)xcalloc(n, 4);
    s->tmp_u32 = (uint32_t*)xcalloc(n, 4);
    s->cert = (uint32_t*)xcalloc(n, 4);
    s->sweep_of = (int32_t*)xcalloc(n, 4);
    s->sweep_cnt = (uint32_t*)xcalloc(n, 4);
    s->sweep_cut = (uint8_t*)xcalloc(n, 1);
    uint64_t maxdeg = 0;
    for (uint32_t v = 0; v < n; ++v) {
        const uint64_t d = offsets[v + 1] - offsets[v];
        s->ideg[v] = (uint32_t)d;                    /* devPartition.h:295-296 */
        if (d > maxdeg) maxdeg = d;
        s->act[v].nix = v;                           /* MakeLabeledNodeOp */
        s->act[v].label = 0;
        s->lookup[v] = -1;
        s->sweep_of[v] = -1;
    }
    uint64_t big = maxdeg > n ? maxdeg : n;
    uint32_t bits = 0;
    while (big) { ++bits; big >>= 1; }
    s->nb_bits = bits;
    s->n_act = n;
    s->n_clusters = 1;
    s->smallest = 0x7FFFFFFF;                        /* devSweepCut.h:244-246 */
    s->cur = 0;
    return s;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    void* ptrs[] = {s->off, s->cols, s->labels, s->ideg, s->xd[0], s->xd[1], s->xf, s->xt,
                    s->act, s->keys, s->nd, s->sorted, s->ulabels, s->vols, s->lookup,
                    s->allcuts, s->cuts, s->clabels, s->cdata, s->csum_fixed_avg, s->parent,
                    s->tmp_u32, s->cert, s->sweep_of, s->sweep_cnt, s->sweep_cut};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
    free(s);
}

static void pxr_refresh_scaled(orc_state* s) {
    /* x~ = x / internal degree, and the max |x| that sets the fixed-point scale */
    float mx = 0.0f;
    for (uint32_t v = 0; v < s->n; ++v) {
        const uint32_t d = s->ideg[v];
        s->xt[v] = d ? (float)((double)s->xf[v] / (double)d) : 0.0f;
        const float a = fabsf(s->xf[v]);
        if (a > mx) mx = a;
    }
    s->xmax = mx;
}

void orc_set_potentials(orc_state* s, const double* x) {
    for (uint32_t v = 0; v < s->n; ++v) {
        s->xd[s->cur][v] = x[v];
        s->xf[v] = (float)x[v];
    }
    if (s->mode == ORC_MODE_PXR) pxr_refresh_scaled(s);
}

void orc_get_potentials(const orc_state* s, double* out) {
    for (uint32_t v = 0; v < s->n; ++v)
        out[v] = s->mode == ORC_MODE_REF ? s->xd[s->cur][v] : (double)s->xf[v];
}

void orc_set_state(orc_state* s, const int32_t* labels, const orc_lnode* act, uint32_t n_act,
                   const double* x, const uint32_t* ideg, const uint32_t* cols,
                   uint32_t n_clusters, int32_t smallest) {
    memcpy(s->labels, labels, (size_t)s->n * 4);
    memcpy(s->act, act, (size_t)n_act * sizeof(orc_lnode));
    s->n_act = n_act;
    memcpy(s->ideg, ideg, (size_t)s->n * 4);
    if (s->slots) memcpy(s->cols, cols, s->slots * 4);
    s->n_clusters = n_clusters;
    s->smallest = smallest;
    orc_set_potentials(s, x);
}

/* ------------------------------------------------------------------------ */
/* walk: fusedRandomWalk_WarpParallel, cuda/devRandomWalk.h:117-203          */

static void walk_ref(orc_state* s) {
    const double* x = s->xd[s->cur];
    double* y = s->xd[s->cur ^ 1];
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const uint32_t v = s->act[i].nix;
        const int32_t lab = s->act[i].label;
        if (lab < 0) { s->keys[i] = pack_key(lab, 0.0f); continue; }
        double lane[32];
        for (int l = 0; l < 32; ++l) {
            double acc = 0.0;
            for (uint64_t j = s->off[v] + (uint64_t)l; j < s->off[v + 1]; j += 32) {
                const uint32_t nb = s->cols[j];
                if (nb == ORC_INVALID_EDGE) continue;
                const uint32_t d = s->ideg[nb];
                if (d == 0) continue;
                acc += x[nb] / (double)d;
            }
            lane[l] = acc;
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int l = 0; l < o; ++l) lane[l] = lane[l] + lane[l + o];
        const double val = lane[0] * (1.0 - 0.1) + x[v] * 0.1;
        y[v] = val;
        s->keys[i] = pack_key(lab, (float)val);
    }
    s->cur ^= 1;
}

static void walk_pxr(orc_state* s) {
    const int e = fixed_exponent(s->xmax, s->nb_bits);
    const double scale = ldexp(1.0, e), inv = ldexp(1.0, -e);
    float* xt_new = (float*)xcalloc(s->n, 4);
    memcpy(xt_new, s->xt, (size_t)s->n * 4);
    float mx = 0.0f;
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const uint32_t v = s->act[i].nix;
        const int32_t lab = s->act[i].label;
        if (lab < 0) { s->keys[i] = pack_key(lab, 0.0f); continue; }
        int64_t acc = 0;
        for (uint64_t j = s->off[v]; j < s->off[v + 1]; ++j) {
            const uint32_t nb = s->cols[j];
            if (nb == ORC_INVALID_EDGE) continue;
            acc = (int64_t)((uint64_t)acc + (uint64_t)to_fixed(s->xt[nb], scale));
        }
        const double sum = (double)acc * inv;
        const double val = sum * 0.9 + (double)s->xf[v] * 0.1;
        const float xv = (float)val;
        s->xf[v] = xv;
        const uint32_t d = s->ideg[v];
        xt_new[v] = d ? (float)((double)xv / (double)d) : 0.0f;
        const float a = fabsf(xv);
        if (a > mx) mx = a;
        s->keys[i] = pack_key(lab, xv);
    }
    memcpy(s->xt, xt_new, (size_t)s->n * 4);
    free(xt_new);
    s->xmax = mx;
}

/* Recompute the sort keys of the active list from the current potentials, as
 * the walk emits them (used to feed recorded potentials to the sweep). */
void orc_rekey(orc_state* s) {
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const int32_t lab = s->act[i].label;
        s->keys[i] = lab < 0 ? pack_key(lab, 0.0f) : pack_key(lab, potential_f(s, s->act[i].nix));
    }
}

void orc_walk(orc_state* s) {
    if (s->mode == ORC_MODE_REF) walk_ref(s); else walk_pxr(s);
}

/* ------------------------------------------------------------------------ */
/* sweep: SweepCutManager::prepare_nodes + compute_sweep_cuts,
 * cuda/devSweepCut.h:20-112, 469-730                                        */

/* perm = the stable ascending order of keys[0..n): an LSD radix sort of
 * (key, index) on 16-bit digits, skipping digits that are equal in every key
 * (the result is that of a stable comparison sort, as CUB's radix sort and
 * thrust::stable_sort give). */
static void stable_order_u64(const uint64_t* keys, uint32_t n, uint32_t* perm) {
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    if (n < 2) return;
    uint64_t all_or = 0, all_and = ~0ull;
    for (uint32_t i = 0; i < n; ++i) { all_or |= keys[i]; all_and &= keys[i]; }
    const uint64_t varying = all_or ^ all_and;
    uint32_t* tmp = (uint32_t*)xcalloc(n, 4);
    uint32_t* cnt = (uint32_t*)xcalloc(65536, 4);
    uint32_t* src = perm;
    uint32_t* dst = tmp;
    for (unsigned shift = 0; shift < 64; shift += 16) {
        if (((varying >> shift) & 0xFFFFull) == 0) continue;
        memset(cnt, 0, 65536 * 4);
        for (uint32_t i = 0; i < n; ++i) cnt[(keys[src[i]] >> shift) & 0xFFFF]++;
        uint32_t sum = 0;
        for (uint32_t d = 0; d < 65536; ++d) { const uint32_t c = cnt[d]; cnt[d] = sum; sum += c; }
        for (uint32_t i = 0; i < n; ++i) dst[cnt[(keys[src[i]] >> shift) & 0xFFFF]++] = src[i];
        uint32_t* t = src; src = dst; dst = t;
    }
    if (src != perm) memcpy(perm, src, (size_t)n * 4);
    free(tmp);
    free(cnt);
}

void orc_sweep(orc_state* s) {
    const uint32_t nA = s->n_act;
    /* nodeDiffKernel_Sparse_WarpParallel */
    for (uint32_t i = 0; i < nA; ++i) {
        const uint32_t v = s->act[i].nix;
        const int32_t lab = s->act[i].label;
        if (lab < 0) { s->nd[i].nix = v; continue; }  /* the reference leaves this slot unwritten */
        const uint64_t mykey = s->keys[i];
        int32_t contrib = 0;
        for (uint64_t j = s->off[v]; j < s->off[v + 1]; ++j) {
            const uint32_t nb = s->cols[j];
            if (nb == ORC_INVALID_EDGE) continue;
            const uint64_t nbkey = pack_key(s->labels[nb], potential_f(s, nb));
            const int before = nbkey != mykey ? nbkey < mykey : nb < v;
            contrib += before ? -1 : 1;
        }
        s->nd[i].nix = v;
        s->nd[i].prefix_edge_diff = contrib;
        s->nd[i].prefix_volume = s->ideg[v];
        s->nd[i].offset = 1;
    }
    /* cub::DeviceRadixSort::SortPairs: stable by the 64-bit key */
    uint32_t* perm = (uint32_t*)xcalloc(nA, 4);
    stable_order_u64(s->keys, nA, perm);
    uint64_t* skeys = (uint64_t*)xcalloc(nA, 8);
    orc_node_data* snd = (orc_node_data*)xcalloc(nA, sizeof(orc_node_data));
    for (uint32_t i = 0; i < nA; ++i) { skeys[i] = s->keys[perm[i]]; snd[i] = s->nd[perm[i]]; }
    free(perm);
    /* StoreSmallestLabelOp + lower_bound: drop the just-deactivated prefix */
    if (nA > 0) s->smallest = key_label(skeys[0]);
    uint32_t first = 0;
    while (first < nA && key_label(skeys[first]) < 0) ++first;
    const uint32_t na = nA - first;
    s->n_act = na;
    for (uint32_t i = 0; i < na; ++i) {          /* ExtractLabeledNodeOp */
        s->act[i].nix = snd[first + i].nix;
        s->act[i].label = key_label(skeys[first + i]);
    }
    /* inclusive_scan_by_key with NodeDataScanOp; reduce_by_key for volumes */
    uint32_t k = 0;
    for (uint32_t i = 0; i < na; ++i) {
        orc_node_data d = snd[first + i];
        const int32_t lab = s->act[i].label;
        if (i > 0 && s->act[i - 1].label == lab) {
            const orc_node_data p = s->sorted[i - 1];
            d.prefix_edge_diff += p.prefix_edge_diff;
            d.prefix_volume += p.prefix_volume;
            d.offset += p.offset;
        } else {
            s->ulabels[k] = lab;
            s->vols[k] = 0;
            ++k;
        }
        s->vols[k - 1] += s->ideg[s->act[i].nix];
        s->sorted[i] = d;
    }
    s->k_sweep = k;
    s->n_clusters = k;
    for (uint32_t c = 0; c < k; ++c)             /* updateLabelLookup */
        if (s->ulabels[c] >= 0 && (uint32_t)s->ulabels[c] < s->n) s->lookup[s->ulabels[c]] = (int32_t)c;
    /* SweepCutTransform + ArgMinOp: the last position holding the minimum */
    uint32_t c = 0;
    for (uint32_t i = 0; i < na; ++i) {
        const int32_t lab = s->act[i].label;
        if (i > 0 && s->act[i - 1].label != lab) ++c;
        const orc_node_data d = s->sorted[i];
        const uint32_t tot = s->vols[c];
        const uint32_t edge_diff = (uint32_t)d.prefix_edge_diff;
        const uint32_t pv = d.prefix_volume;
        const uint32_t denom = pv >= tot ? 0u : (pv < tot - pv ? pv : tot - pv);
        const float sp = denom > 0 ? (float)edge_diff / (float)denom : 2.0f;
        const orc_sweep_cut cand = {lab, sp, d.offset};
        if (i == 0 || s->act[i - 1].label != lab) s->allcuts[c] = cand;
        else if (!(s->allcuts[c].sparsity < sp)) s->allcuts[c] = cand;
    }
    /* copy_if(CheckThreshold) */
    uint32_t nc = 0;
    for (uint32_t j = 0; j < k; ++j) {
        const int cut = (double)s->allcuts[j].sparsity < (double)s->sc_threshold;
        if (cut) s->cuts[nc++] = s->allcuts[j];
        s->sweep_cut[j] = (uint8_t)cut;
        s->sweep_cnt[j] = 0;
    }
    s->n_cut = nc;
    /* certificate record: the swept cluster of every vertex and its size */
    c = 0;
    for (uint32_t i = 0; i < na; ++i) {
        if (i > 0 && s->act[i - 1].label != s->act[i].label) ++c;
        s->sweep_of[s->act[i].nix] = (int32_t)c;
        s->sweep_cnt[c] += 1;
    }
    free(skeys);
    free(snd);
}

/* ------------------------------------------------------------------------ */
/* PartitionManager::cutClusters, cuda/devPartition.h:545-622                */

void orc_cut_stage(orc_state* s) {
    if (s->n_cut == 0) return;                   /* cuda/device.h:168 */
    const int64_t max_label = s->ulabels[s->n_clusters - 1];
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const int32_t lab = s->act[i].label;
        if (lab < 0) continue;
        /* lower_bound over the filtered cuts (ascending labels) */
        uint32_t lo = 0, hi = s->n_cut;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (s->cuts[mid].label < lab) lo = mid + 1; else hi = mid;
        }
        if (lo == s->n_cut || s->cuts[lo].label != lab) continue;
        if (s->sorted[i].offset > s->cuts[lo].offset) {
            const int32_t nl = (int32_t)((int64_t)lo + max_label + 1);
            s->act[i].label = nl;
            s->labels[s->act[i].nix] = nl;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* ConsolidationManager::consolidate, cuda/devConsolidate.h:168-204:
 * components over same-label valid edges; every active vertex takes the
 * minimum vertex id of its component as label.                             */

static uint32_t uf_find(uint32_t* p, uint32_t v) {
    while (p[v] != v) { p[v] = p[p[v]]; v = p[v]; }
    return v;
}

void orc_components_stage(orc_state* s) {
    for (uint32_t v = 0; v < s->n; ++v) s->parent[v] = v;
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const uint32_t v = s->act[i].nix;
        const int32_t lab = s->act[i].label;
        if (lab < 0) continue;
        for (uint64_t j = s->off[v]; j < s->off[v + 1]; ++j) {
            const uint32_t nb = s->cols[j];
            if (nb == ORC_INVALID_EDGE || s->labels[nb] != lab) continue;
            uint32_t a = uf_find(s->parent, v), b = uf_find(s->parent, nb);
            if (a == b) continue;
            if (a < b) s->parent[b] = a; else s->parent[a] = b;
        }
    }
    for (uint32_t i = 0; i < s->n_act; ++i) {
        if (s->act[i].label < 0) continue;
        const int32_t root = (int32_t)uf_find(s->parent, s->act[i].nix);
        s->act[i].label = root;
        s->labels[s->act[i].nix] = root;
    }
}

/* ------------------------------------------------------------------------ */
/* PartitionManager::computeClusterData, cuda/devPartition.h:380-411          */

void orc_cluster_data_stage(orc_state* s) {
    const uint32_t nA = s->n_act;
    /* stable_sort(LabeledNodeLabelLess) */
    uint32_t* perm = (uint32_t*)xcalloc(nA, 4);
    uint64_t* lkey = (uint64_t*)xcalloc(nA, 8);
    for (uint32_t i = 0; i < nA; ++i) lkey[i] = (uint64_t)((uint32_t)s->act[i].label ^ 0x80000000u);
    stable_order_u64(lkey, nA, perm);
    free(lkey);
    orc_lnode* sorted = (orc_lnode*)xcalloc(nA, sizeof(orc_lnode));
    for (uint32_t i = 0; i < nA; ++i) sorted[i] = s->act[perm[i]];
    memcpy(s->act, sorted, (size_t)nA * sizeof(orc_lnode));
    free(sorted);
    free(perm);
    /* reduce_by_key(ClusterDataFromLabeledNodeOp, ClusterDataReduceOp) */
    uint32_t k = 0;
    int64_t fixed = 0;
    const int e = fixed_exponent(s->xmax, s->nb_bits);
    const double scale = ldexp(1.0, e), inv = ldexp(1.0, -e);
    for (uint32_t i = 0; i < nA; ++i) {
        const float xv = potential_f(s, s->act[i].nix);
        const int32_t lab = s->act[i].label;
        if (i == 0 || s->act[i - 1].label != lab) {
            if (k > 0 && s->mode == ORC_MODE_PXR)
                s->csum_fixed_avg[k - 1] = ((double)fixed * inv) / (double)s->cdata[k - 1].count;
            s->clabels[k] = lab;
            s->cdata[k].sum = xv;
            s->cdata[k].max = xv;
            s->cdata[k].min = xv;
            s->cdata[k].count = 1;
            fixed = to_fixed(xv, scale);
            ++k;
        } else {
            orc_cluster_data* c = &s->cdata[k - 1];
            c->sum = c->sum + xv;
            c->max = c->max > xv ? c->max : xv;
            c->min = c->min < xv ? c->min : xv;
            c->count += 1;
            fixed = (int64_t)((uint64_t)fixed + (uint64_t)to_fixed(xv, scale));
        }
    }
    if (k > 0 && s->mode == ORC_MODE_PXR)
        s->csum_fixed_avg[k - 1] = ((double)fixed * inv) / (double)s->cdata[k - 1].count;
    s->k_data = k;
    s->n_clusters = k;
    for (uint32_t c = 0; c < k; ++c)             /* updateLabelLookup */
        if (s->clabels[c] >= 0 && (uint32_t)s->clabels[c] < s->n) s->lookup[s->clabels[c]] = (int32_t)c;
}

/* ------------------------------------------------------------------------ */
/* Certificate record of a vertex whose cluster is certified (deactivated) now:
 * the round, and whether the certified set (count vertices) is exactly the
 * set swept this round - only then does that sweep's "no cut below sc" speak
 * for it.  No reference counterpart: the reference keeps no such record.    */

static void certify_vertex(orc_state* s, uint32_t v, uint32_t count) {
    const int32_t c = s->sweep_of[v];
    const int whole = c >= 0 && !s->sweep_cut[c] && s->sweep_cnt[c] == count;
    s->cert[v] = (s->round + 1u) | (whole ? 0u : 0x80000000u);
}

/* ------------------------------------------------------------------------ */
/* PartitionManager::recenterAndDeactivateClusters, cuda/devPartition.h:624-711 */

void orc_recenter_stage(orc_state* s) {
    const uint32_t k = s->k_data;
    int32_t* newlab = (int32_t*)xcalloc(k, 4);
    int32_t survivors = 0;
    for (uint32_t c = 0; c < k; ++c) {           /* KeepClusterFlagOp + exclusive_scan */
        const float pot = s->cdata[c].max - s->cdata[c].min;
        const int keep = pot >= s->rw_threshold && s->cdata[c].count >= 2;
        newlab[c] = survivors;
        survivors += keep;
    }
    float mx = 0.0f;
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const int32_t lab = s->act[i].label;
        const uint32_t v = s->act[i].nix;
        if (lab < 0 || (uint32_t)lab >= s->n) continue;
        const int32_t c = s->lookup[lab];
        const orc_cluster_data cd = s->cdata[c];
        const float pot = cd.max - cd.min;
        if (pot < s->rw_threshold || cd.count < 2) {
            const int32_t nl = s->smallest - c - 1;
            s->act[i].label = nl;
            s->labels[v] = nl;
            certify_vertex(s, v, cd.count);
        } else {
            s->act[i].label = newlab[c];
            s->labels[v] = newlab[c];
            if (s->mode == ORC_MODE_REF) {
                const double avg = (double)cd.sum / (double)cd.count;
                s->xd[s->cur][v] -= avg;
            } else {
                const float xv = (float)((double)s->xf[v] - s->csum_fixed_avg[c]);
                s->xf[v] = xv;
                const float a = fabsf(xv);
                if (a > mx) mx = a;
            }
        }
    }
    if (s->mode == ORC_MODE_PXR) s->xmax = mx;
    s->n_clusters = (uint32_t)survivors;
    free(newlab);
}

/* ------------------------------------------------------------------------ */
/* PartitionManager::disableEdges, cuda/devPartition.h:80-146, 503-522        */

void orc_disable_stage(orc_state* s) {
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const uint32_t v = s->act[i].nix;
        const int32_t lab = s->act[i].label;
        if (lab < 0) continue;
        uint32_t deg = 0;
        for (uint64_t j = s->off[v]; j < s->off[v + 1]; ++j) {
            const uint32_t nb = s->cols[j];
            if (nb == ORC_INVALID_EDGE) continue;
            if (s->labels[nb] != lab) s->cols[j] = ORC_INVALID_EDGE;
            else ++deg;
        }
        s->ideg[v] = deg;
    }
    if (s->mode == ORC_MODE_PXR) {
        for (uint32_t i = 0; i < s->n_act; ++i) {
            const uint32_t v = s->act[i].nix;
            if (s->act[i].label < 0) continue;
            const uint32_t d = s->ideg[v];
            s->xt[v] = d ? (float)((double)s->xf[v] / (double)d) : 0.0f;
        }
    }
}

void orc_cut_clusters(orc_state* s) {
    orc_cut_stage(s);
    orc_components_stage(s);
    orc_cluster_data_stage(s);
    orc_recenter_stage(s);
    orc_disable_stage(s);
    s->round += 1;
}

/* ------------------------------------------------------------------------ */
/* Scheduled round (no reference counterpart: the sweep schedule of the
 * learned stop predictor).  Every active vertex walks; only the clusters with
 * due[c] != 0 go through the sweep, the cut, components, cluster data,
 * recentering and edge disabling, exactly as in the plain round.  The other
 * ("carried") clusters keep their vertices, potentials and rows; they are
 * relabelled with the rest: dense labels in the order of the clusters' root
 * vertices (minimum vertex id) over swept and carried clusters together, and
 * a swept cluster that is certified takes smallest - j - 1 with j its position
 * in that merged root order.  smallest is the least label of the sweep (0 when
 * it holds no negative label).  With every cluster due this is the plain
 * round. */

static const uint32_t* g_root_of;
static int cmp_root_entry(const void* a, const void* b) {
    const uint32_t ra = g_root_of[*(const uint32_t*)a], rb = g_root_of[*(const uint32_t*)b];
    return ra < rb ? -1 : (ra > rb);
}

void orc_scheduled_round(orc_state* s, const uint8_t* due) {
    const uint32_t K = s->n_clusters;
    orc_walk(s);
    const uint32_t nA = s->n_act;
    orc_lnode* carried = (orc_lnode*)xcalloc(nA ? nA : 1, sizeof(orc_lnode));
    uint32_t* croot = (uint32_t*)xcalloc(K ? K : 1, 4);
    for (uint32_t c = 0; c < K; ++c) croot[c] = 0xFFFFFFFFu;
    uint32_t nd = 0, nc = 0;
    for (uint32_t i = 0; i < nA; ++i) {
        const orc_lnode a = s->act[i];
        if (a.label < 0 || due[a.label]) {
            s->act[nd] = a;
            s->keys[nd] = s->keys[i];
            ++nd;
        } else {
            carried[nc++] = a;
            if (a.nix < croot[a.label]) croot[a.label] = a.nix;
        }
    }
    s->n_act = nd;
    if (nd > 0) {
        orc_sweep(s);
        if (s->smallest > 0) s->smallest = 0;
    } else {
        s->smallest = 0;
        s->k_sweep = 0;
        s->n_cut = 0;
        s->n_clusters = 0;
    }
    orc_cut_stage(s);
    orc_components_stage(s);
    orc_cluster_data_stage(s);

    /* merged root order: swept clusters (cluster data) and carried clusters */
    const uint32_t kd = s->k_data;
    uint32_t* root_of = (uint32_t*)xcalloc(kd + K + 1, 4);
    uint32_t* order = (uint32_t*)xcalloc(kd + K + 1, 4);
    uint32_t ne = 0;
    for (uint32_t c = 0; c < kd; ++c) { root_of[ne] = (uint32_t)s->clabels[c]; order[ne] = ne; ++ne; }
    for (uint32_t c = 0; c < K; ++c)
        if (croot[c] != 0xFFFFFFFFu) { root_of[ne] = croot[c]; order[ne] = ne; ++ne; }
    g_root_of = root_of;
    qsort(order, ne, 4, cmp_root_entry);
    int32_t* data_nl = (int32_t*)xcalloc(kd ? kd : 1, 4);
    int32_t* carried_nl = (int32_t*)xcalloc(K ? K : 1, 4);
    /* entry e < kd is data cluster e; entry kd + q is the q-th carried cluster in label order */
    uint32_t* carried_label = (uint32_t*)xcalloc(K ? K : 1, 4);
    {
        uint32_t q = 0;
        for (uint32_t c = 0; c < K; ++c)
            if (croot[c] != 0xFFFFFFFFu) carried_label[q++] = c;
    }
    int32_t survivors = 0;
    for (uint32_t j = 0; j < ne; ++j) {
        const uint32_t e = order[j];
        if (e < kd) {
            const orc_cluster_data cd = s->cdata[e];
            const float pot = cd.max - cd.min;
            const int keep = pot >= s->rw_threshold && cd.count >= 2;
            data_nl[e] = keep ? survivors++ : (int32_t)((uint32_t)s->smallest - j - 1u);
        } else {
            carried_nl[carried_label[e - kd]] = survivors++;
        }
    }
    float mx = 0.0f;
    for (uint32_t i = 0; i < s->n_act; ++i) {
        const int32_t lab = s->act[i].label;
        const uint32_t v = s->act[i].nix;
        if (lab < 0 || (uint32_t)lab >= s->n) continue;
        const int32_t c = s->lookup[lab];
        const int32_t nl = data_nl[c];
        s->act[i].label = nl;
        s->labels[v] = nl;
        if (nl < 0) {
            certify_vertex(s, v, s->cdata[c].count);
            continue;
        }
        if (s->mode == ORC_MODE_REF) {
            const double avg = (double)s->cdata[c].sum / (double)s->cdata[c].count;
            s->xd[s->cur][v] -= avg;
        } else {
            const float xv = (float)((double)s->xf[v] - s->csum_fixed_avg[c]);
            s->xf[v] = xv;
            const float a = fabsf(xv);
            if (a > mx) mx = a;
        }
    }
    for (uint32_t j = 0; j < nc; ++j) {
        const uint32_t v = carried[j].nix;
        const int32_t nl = carried_nl[carried[j].label];
        carried[j].label = nl;
        s->labels[v] = nl;
        if (s->mode == ORC_MODE_PXR) {
            const float a = fabsf(s->xf[v]);
            if (a > mx) mx = a;
        }
    }
    if (s->mode == ORC_MODE_PXR) s->xmax = mx;
    orc_disable_stage(s);   /* rows of the swept, kept vertices */
    memcpy(s->act + s->n_act, carried, (size_t)nc * sizeof(orc_lnode));
    s->n_act += nc;
    s->n_clusters = (uint32_t)survivors;
    s->round += 1;
    free(carried); free(croot); free(root_of); free(order); free(data_nl); free(carried_nl); free(carried_label);
}

uint32_t orc_decompose(orc_state* s, uint32_t max_rounds) {
    uint32_t rounds = 0;
    while (rounds < max_rounds && s->n_clusters > 0 && s->n_act > 0) {
        ++rounds;
        orc_walk(s);
        orc_sweep(s);
        if (s->n_act == 0) break;
        orc_cut_clusters(s);
    }
    return rounds;
}

/* ------------------------------------------------------------------------ */

static int cmp_i32(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return x < y ? -1 : (x > y);
}

int32_t orc_final_partition(const orc_state* s, int32_t* ids) {
    int32_t* u = (int32_t*)xcalloc(s->n, 4);
    memcpy(u, s->labels, (size_t)s->n * 4);
    qsort(u, s->n, 4, cmp_i32);
    uint32_t k = 0;
    for (uint32_t i = 0; i < s->n; ++i)
        if (i == 0 || u[i] != u[i - 1]) u[k++] = u[i];
    for (uint32_t v = 0; v < s->n; ++v) {
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (u[mid] < s->labels[v]) lo = mid + 1; else hi = mid;
        }
        ids[v] = (int32_t)lo;
    }
    free(u);
    return (int32_t)k;
}

uint64_t orc_num_cut_edges(const orc_state* s) {
    uint64_t valid = 0;
    for (uint64_t j = 0; j < s->slots; ++j) valid += s->cols[j] != ORC_INVALID_EDGE;
    return s->m - valid / 2;
}

uint32_t orc_n_active(const orc_state* s) { return s->n_act; }
uint32_t orc_n_clusters(const orc_state* s) { return s->n_clusters; }
uint32_t orc_n_sweep_clusters(const orc_state* s) { return s->k_sweep; }
uint32_t orc_n_cuts(const orc_state* s) { return s->n_cut; }
uint32_t orc_n_data_clusters(const orc_state* s) { return s->k_data; }
int32_t orc_smallest_label(const orc_state* s) { return s->smallest; }
const int32_t* orc_labels(const orc_state* s) { return s->labels; }
const orc_lnode* orc_active(const orc_state* s) { return s->act; }
const uint32_t* orc_internal_degrees(const orc_state* s) { return s->ideg; }
const uint32_t* orc_cols(const orc_state* s) { return s->cols; }
const uint64_t* orc_keys(const orc_state* s) { return s->keys; }
const orc_node_data* orc_sorted(const orc_state* s) { return s->sorted; }
const int32_t* orc_sweep_labels(const orc_state* s) { return s->ulabels; }
const uint32_t* orc_sweep_volumes(const orc_state* s) { return s->vols; }
const orc_sweep_cut* orc_all_cuts(const orc_state* s) { return s->allcuts; }
const orc_sweep_cut* orc_cuts(const orc_state* s) { return s->cuts; }
const int32_t* orc_data_labels(const orc_state* s) { return s->clabels; }
const orc_cluster_data* orc_cluster_values(const orc_state* s) { return s->cdata; }
const uint32_t* orc_certificates(const orc_state* s) { return s->cert; }
