/* Test infrastructure only (see coresg_oracle.h): a plain-C restatement of the
 * reference algorithms, used as the checker.  Built with -ffp-contract=off so every
 * float operation below is exactly the one written. */
#include "coresg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define INVALID 0xFFFFFFFFu

static uint32_t fbits(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b;
}

/* l2sqr_avx2 (include/coresg/distance.hpp:191-211): lane l of acc0 accumulates
 * element i+l of every 16-wide block and of the trailing 8-wide block, lane l of
 * acc1 element i+8+l of every 16-wide block, each with one fused multiply-add;
 * hsum256(acc0 + acc1) (:180-189) reduces v = acc0+acc1 as
 * ((v0+v4)+(v1+v5)) + ((v2+v6)+(v3+v7)); a scalar tail follows. */
float orc_l2sqr(const float* a, const float* b, uint32_t d) {
    float acc0[8] = {0}, acc1[8] = {0};
    uint32_t i = 0;
    for (; i + 16 <= d; i += 16) {
        for (int l = 0; l < 8; ++l) {
            const float d0 = a[i + l] - b[i + l];
            const float d1 = a[i + 8 + l] - b[i + 8 + l];
            acc0[l] = fmaf(d0, d0, acc0[l]);
            acc1[l] = fmaf(d1, d1, acc1[l]);
        }
    }
    for (; i + 8 <= d; i += 8) {
        for (int l = 0; l < 8; ++l) {
            const float d0 = a[i + l] - b[i + l];
            acc0[l] = fmaf(d0, d0, acc0[l]);
        }
    }
    float v[8];
    for (int l = 0; l < 8; ++l) v[l] = acc0[l] + acc1[l];
    const float lo0 = v[0] + v[4], lo1 = v[1] + v[5], lo2 = v[2] + v[6], lo3 = v[3] + v[7];
    float s = (lo0 + lo1) + (lo2 + lo3);
    for (; i < d; ++i) {
        const float t = a[i] - b[i];
        s += t * t;
    }
    return s;
}

float orc_dist(const float* a, const float* b, uint32_t stride) {
    return sqrtf(orc_l2sqr(a, b, stride));
}

void orc_core(const float* dists, const uint32_t* counts, uint32_t n, uint32_t k, uint32_t mpts,
              float* out) {
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t c = counts[v];
        if (c == 0) {
            out[v] = INFINITY;
            continue;
        }
        uint32_t pos = mpts == 0 ? 0 : mpts - 1;
        if (pos >= c) pos = c - 1;
        out[v] = dists[(uint64_t)v * k + pos];
    }
}

uint64_t orc_undirected(const uint32_t* ids, const float* dists, const uint32_t* counts,
                        uint32_t n, uint32_t k, orc_edge* out) {
    uint64_t m = 0;
    for (uint32_t p = 0; p < n; ++p) {
        const uint32_t* I = ids + (uint64_t)p * k;
        const float* D = dists + (uint64_t)p * k;
        const uint32_t c = counts[p];
        for (uint32_t j = 0; j < c; ++j) {
            const uint32_t q = I[j];
            if (q == INVALID || q == p) continue;
            if (q < p) {
                const uint32_t cq = counts[q];
                /* !(D[j] > last) also admits NaN; distances are never NaN here. */
                if (cq > 0 && !(D[j] > dists[(uint64_t)q * k + cq - 1])) {
                    const uint32_t* J = ids + (uint64_t)q * k;
                    int mutual = 0;
                    for (uint32_t t = 0; t < cq; ++t) {
                        if (J[t] == p) {
                            mutual = 1;
                            break;
                        }
                    }
                    if (mutual) continue;
                }
            }
            if (out) {
                out[m].u = p < q ? p : q;
                out[m].v = p < q ? q : p;
                out[m].w = D[j];
            }
            ++m;
        }
    }
    return m;
}

static float fmax_ref(float a, float b) { return (a < b) ? b : a; } /* std::max(a, b) */

uint64_t orc_edges(uint32_t mpts, const uint32_t* ids, const float* dists, const uint32_t* counts,
                   uint32_t n, uint32_t k, const orc_edge* bridges, uint64_t n_bridges,
                   orc_edge* out) {
    if (mpts == 0) mpts = 1;
    float* core = (float*)malloc(sizeof(float) * (n ? n : 1));
    orc_core(dists, counts, n, k, mpts, core);
    const uint64_t m = orc_undirected(ids, dists, counts, n, k, out);
    if (out) {
        for (uint64_t i = 0; i < m; ++i) {
            const float c = fmax_ref(core[out[i].u], core[out[i].v]);
            out[i].w = fmax_ref(out[i].w, c);
        }
        for (uint64_t b = 0; b < n_bridges; ++b) {
            orc_edge e = bridges[b];
            const float c = fmax_ref(core[e.u], core[e.v]);
            out[m + b].u = e.u < e.v ? e.u : e.v;
            out[m + b].v = e.u < e.v ? e.v : e.u;
            out[m + b].w = fmax_ref(e.w, c);
        }
    }
    free(core);
    return m + n_bridges;
}

/* ---- union-find ---------------------------------------------------------- */

static uint32_t uf_find(uint32_t* parent, uint32_t x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

/* Links the larger root under the smaller, so a root is always its set's minimum. */
static int uf_unite(uint32_t* parent, uint32_t a, uint32_t b) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return 0;
    if (a > b) {
        uint32_t t = a;
        a = b;
        b = t;
    }
    parent[b] = a;
    return 1;
}

/* Dense labels numbered by each set's first node (UnionFind::labels, mst.cpp:48-59). */
static uint32_t uf_labels(uint32_t* parent, uint32_t n, uint32_t* labels) {
    uint32_t* remap = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) remap[i] = INVALID;
    uint32_t next = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t r = uf_find(parent, i);
        if (remap[r] == INVALID) remap[r] = next++;
        if (labels) labels[i] = remap[r];
    }
    free(remap);
    return next;
}

/* ---- MST ------------------------------------------------------------------ */

static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

/* pack_edge (src/mst.cpp:19-24): float bits (complemented when negative) << 32 | index. */
static uint64_t pack_key(float w, uint32_t idx) {
    uint32_t b = fbits(w);
    if (w < 0.0f) b = ~b;
    return ((uint64_t)b << 32) | idx;
}

int orc_mst(const orc_edge* e, uint64_t m, uint32_t n, uint8_t* in_tree, uint32_t* labels,
            uint32_t* ncomp, uint64_t* nedges, double* exact_weight) {
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
    uint32_t* parent = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    float* w = (float*)malloc(sizeof(float) * (n ? n : 1));
    if (!keys || !parent || !w) return 1;
    for (uint64_t i = 0; i < m; ++i) keys[i] = pack_key(e[i].w, (uint32_t)i);
    qsort(keys, m, sizeof(uint64_t), cmp_u64);
    for (uint32_t i = 0; i < n; ++i) parent[i] = i;
    if (in_tree) memset(in_tree, 0, m);
    uint64_t cnt = 0;
    for (uint64_t t = 0; t < m; ++t) {
        const uint32_t idx = (uint32_t)(keys[t] & 0xFFFFFFFFu);
        const orc_edge* x = &e[idx];
        if (x->u >= n || x->v >= n) continue;
        if (uf_unite(parent, x->u, x->v)) {
            if (in_tree) in_tree[idx] = 1;
            w[cnt++] = x->w;
        }
    }
    const uint32_t nc = uf_labels(parent, n, labels);
    if (ncomp) *ncomp = nc;
    if (nedges) *nedges = cnt;
    if (exact_weight) *exact_weight = orc_exact_sum(w, cnt);
    free(keys);
    free(parent);
    free(w);
    return 0;
}

typedef struct {
    float w;
    uint32_t u, v, idx;
} kedge;

static int cmp_kedge(const void* a, const void* b) {
    const kedge* x = (const kedge*)a;
    const kedge* y = (const kedge*)b;
    if (x->w != y->w) return x->w < y->w ? -1 : 1;
    if (x->u != y->u) return x->u < y->u ? -1 : 1;
    if (x->v != y->v) return x->v < y->v ? -1 : 1;
    return (x->idx > y->idx) - (x->idx < y->idx); /* std::sort is unstable; any order is valid */
}

int orc_mst_kruskal(const orc_edge* e, uint64_t m, uint32_t n, uint8_t* in_tree,
                    uint32_t* ncomp, uint64_t* nedges) {
    kedge* ks = (kedge*)malloc(sizeof(kedge) * (m ? m : 1));
    uint32_t* parent = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint64_t i = 0; i < m; ++i) {
        ks[i].w = e[i].w;
        ks[i].u = e[i].u;
        ks[i].v = e[i].v;
        ks[i].idx = (uint32_t)i;
    }
    qsort(ks, m, sizeof(kedge), cmp_kedge);
    for (uint32_t i = 0; i < n; ++i) parent[i] = i;
    if (in_tree) memset(in_tree, 0, m);
    uint64_t cnt = 0;
    for (uint64_t t = 0; t < m; ++t) {
        if (ks[t].u >= n || ks[t].v >= n) continue;
        if (uf_unite(parent, ks[t].u, ks[t].v)) {
            if (in_tree) in_tree[ks[t].idx] = 1;
            ++cnt;
            if (cnt + 1 == n) break;
        }
    }
    if (ncomp) *ncomp = uf_labels(parent, n, NULL);
    if (nedges) *nedges = cnt;
    free(ks);
    free(parent);
    return 0;
}

/* Exact sum: float = mant * 2^(E-150) with E = max(biased exponent, 1); mantissas are
 * accumulated per exponent, then summed as a big integer in units of 2^-149 and
 * rounded once (to nearest, ties to even) into a double. */
double orc_exact_sum(const float* w, uint64_t count) {
    uint64_t bins[256];
    memset(bins, 0, sizeof(bins));
    int has_inf = 0, has_nan = 0;
    for (uint64_t i = 0; i < count; ++i) {
        const uint32_t b = fbits(w[i]) & 0x7FFFFFFFu; /* weights are >= 0 */
        const uint32_t e = b >> 23;
        if (e == 255) {
            if (b & 0x7FFFFFu) has_nan = 1; else has_inf = 1;
            continue;
        }
        const uint32_t mant = (b & 0x7FFFFFu) | (e ? 0x800000u : 0u);
        bins[e ? e : 1] += mant;
    }
    if (has_nan) return NAN;
    if (has_inf) return INFINITY;
    /* 32-bit limbs; bins[e] (< 2^64) lands at bit e-1. */
    enum { L = 12 };
    uint64_t limb[L];
    memset(limb, 0, sizeof(limb));
    for (int e = 1; e < 255; ++e) {
        uint64_t v = bins[e];
        if (!v) continue;
        const int sh = e - 1;
        int li = sh / 32, off = sh % 32;
        /* add v << off at limb li (v < 2^64, so spans up to 3 limbs) */
        unsigned __int128 x = (unsigned __int128)v << off;
        while (x && li < L) {
            unsigned __int128 s = (unsigned __int128)limb[li] + (uint64_t)(x & 0xFFFFFFFFu);
            limb[li] = (uint64_t)(s & 0xFFFFFFFFu);
            x = (x >> 32) + (s >> 32);
            ++li;
        }
    }
    int top = -1;
    for (int li = L - 1; li >= 0 && top < 0; --li) {
        if (limb[li]) {
            for (int bit = 31; bit >= 0; --bit) {
                if (limb[li] >> bit & 1u) {
                    top = li * 32 + bit;
                    break;
                }
            }
        }
    }
    if (top < 0) return 0.0;
#define BIT(p) ((p) < 0 ? 0u : (unsigned)((limb[(p) / 32] >> ((p) % 32)) & 1u))
    uint64_t mant = 0;
    const int lowbit = top - 52;
    for (int p = top; p >= lowbit && p >= 0; --p) mant = (mant << 1) | BIT(p);
    if (lowbit <= 0) return ldexp((double)mant, -149); /* at most 53 significant bits: exact */
    const int exp2 = lowbit; /* value = mant * 2^(exp2 - 149) */
    const unsigned round_bit = BIT(lowbit - 1);
    unsigned sticky = 0;
    for (int p = lowbit - 2; p >= 0 && !sticky; --p) sticky |= BIT(p);
#undef BIT
    if (round_bit && (sticky || (mant & 1u))) ++mant;
    return ldexp((double)mant, exp2 - 149);
}

/* ---- hubness --------------------------------------------------------------- */

void orc_rdeg(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k, int32_t* rdeg) {
    memset(rdeg, 0, sizeof(int32_t) * n);
    for (uint32_t p = 0; p < n; ++p) {
        for (uint32_t j = 0; j < counts[p]; ++j) {
            const uint32_t q = ids[(uint64_t)p * k + j];
            if (q < n) ++rdeg[q];
        }
    }
}

void orc_scores(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k,
                uint32_t k_for_score, const int32_t* rdeg, double* score) {
    const uint32_t ks = k_for_score ? k_for_score : k;
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t deg = counts[v];
        const int32_t rd = rdeg[v];
        int64_t sum = 0;
        for (uint32_t j = 0; j < deg; ++j) {
            const uint32_t q = ids[(uint64_t)v * k + j];
            if (q >= n) continue;
            sum += rdeg[q];
        }
        double s;
        if (rd > 0 && sum <= 0) s = (double)ks;
        else if (rd <= 0 && sum > 0) s = 0.0;
        else if (rd <= 0 && sum <= 0) s = 1.0;
        else if (deg == 0) s = 1.0;
        else {
            const double denom = (double)sum / (double)deg;
            s = (denom > 0.0) ? (double)rd / denom : (double)ks;
        }
        score[v] = s;
    }
}

uint64_t orc_budget(uint32_t dim, uint64_t num_edges, uint32_t n, double multiplier,
                    double max_pair_ops, uint64_t min_selected, uint64_t max_selected) {
    if (n == 0) return 0;
    const double logs = (num_edges > 1) ? log((double)num_edges) : 0.0;
    double raw = multiplier * (double)dim * logs;
    if (!(raw > 0.0)) raw = 0.0;
    uint64_t count = (uint64_t)llround(raw);
    if (max_pair_ops > 0.0 && dim > 0) {
        const double m_max = sqrt(2.0 * max_pair_ops / (double)dim);
        if (m_max >= 1.0 && (double)count > m_max) count = (uint64_t)m_max;
    }
    if (max_selected && count > max_selected) count = max_selected;
    if (count < min_selected) count = min_selected;
    if (count > n) count = n;
    return count;
}

static const double* g_score;
static const int32_t* g_rdeg;

static int sel_less(uint32_t a, uint32_t b) {
    if (g_score[a] != g_score[b]) return g_score[a] < g_score[b];
    if (g_rdeg[a] != g_rdeg[b]) return g_rdeg[a] < g_rdeg[b];
    return a < b;
}

static int cmp_sel(const void* x, const void* y) {
    const uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
    if (a == b) return 0;
    return sel_less(a, b) ? -1 : 1;
}

uint64_t orc_select(const double* score, const int32_t* rdeg, uint32_t n, uint64_t budget,
                    const uint32_t* comp, uint32_t ncomp, uint32_t per, uint32_t* out) {
    g_score = score;
    g_rdeg = rdeg;
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    qsort(order, n, sizeof(uint32_t), cmp_sel); /* the budget lowest under a strict order */
    uint64_t cnt = budget < n ? budget : n;
    uint8_t* chosen = (uint8_t*)calloc(n ? n : 1, 1);
    for (uint64_t i = 0; i < cnt; ++i) {
        out[i] = order[i];
        chosen[order[i]] = 1;
    }
    if (per && comp && ncomp > 0) {
        uint32_t* buckets = (uint32_t*)malloc(sizeof(uint32_t) * (uint64_t)ncomp * per);
        uint32_t* bsize = (uint32_t*)calloc(ncomp, sizeof(uint32_t));
        for (uint32_t v = 0; v < n; ++v) {
            const uint32_t c = comp[v];
            if (c >= ncomp) continue;
            uint32_t* b = buckets + (uint64_t)c * per;
            if (bsize[c] < per) {
                b[bsize[c]++] = v;
            } else {
                uint32_t worst = 0;
                for (uint32_t t = 1; t < bsize[c]; ++t) {
                    if (sel_less(b[worst], b[t])) worst = t;
                }
                if (sel_less(v, b[worst])) b[worst] = v;
            }
        }
        for (uint32_t c = 0; c < ncomp; ++c) {
            for (uint32_t t = 0; t < bsize[c]; ++t) {
                const uint32_t v = buckets[(uint64_t)c * per + t];
                if (!chosen[v]) {
                    chosen[v] = 1;
                    out[cnt++] = v;
                }
            }
        }
        qsort(out, cnt, sizeof(uint32_t), cmp_sel);
        free(buckets);
        free(bsize);
    }
    free(order);
    free(chosen);
    return cnt;
}

uint32_t orc_conn(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k,
                  uint32_t* labels) {
    uint32_t* parent = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) parent[i] = i;
    for (uint32_t p = 0; p < n; ++p) {
        for (uint32_t j = 0; j < counts[p]; ++j) {
            const uint32_t q = ids[(uint64_t)p * k + j];
            if (q < n && q != p) uf_unite(parent, p, q);
        }
    }
    const uint32_t nc = uf_labels(parent, n, labels);
    free(parent);
    return nc;
}

/* ---- bridges ---------------------------------------------------------------- */

void orc_mrd_block(const float* pts, uint32_t m, uint32_t stride, const float* core, uint32_t r0,
                   uint32_t r1, float* out) {
    for (uint32_t i = r0; i < r1; ++i) {
        const float* a = pts + (uint64_t)i * stride;
        float* row = out + (uint64_t)(i - r0) * m;
        for (uint32_t j = 0; j < m; ++j) {
            if (i == j) {
                row[j] = 0.0f;
                continue;
            }
            const float d = orc_dist(a, pts + (uint64_t)j * stride, stride);
            row[j] = fmax_ref(d, fmax_ref(core[i], core[j]));
        }
    }
}

uint64_t orc_prim_dense(const float* mat, uint32_t m, orc_edge* out) {
    if (m < 2) return 0;
    float* best = (float*)malloc(sizeof(float) * m);
    uint32_t* from = (uint32_t*)malloc(sizeof(uint32_t) * m);
    uint8_t* in_tree = (uint8_t*)calloc(m, 1);
    for (uint32_t j = 0; j < m; ++j) {
        best[j] = INFINITY;
        from[j] = INVALID;
    }
    uint64_t cnt = 0;
    uint32_t current = 0;
    in_tree[0] = 1;
    best[0] = 0.0f;
    for (uint32_t step = 1; step < m; ++step) {
        const float* row = mat + (uint64_t)current * m;
        for (uint32_t j = 0; j < m; ++j) {
            if (in_tree[j]) continue;
            if (row[j] < best[j]) {
                best[j] = row[j];
                from[j] = current;
            }
        }
        uint32_t pick = INVALID;
        float pick_w = INFINITY;
        for (uint32_t j = 0; j < m; ++j) {
            if (in_tree[j]) continue;
            if (best[j] < pick_w || (best[j] == pick_w && pick == INVALID)) {
                pick_w = best[j];
                pick = j;
            }
        }
        if (pick == INVALID) break;
        in_tree[pick] = 1;
        if (from[pick] != INVALID && pick_w < INFINITY) {
            const uint32_t a = from[pick];
            out[cnt].u = a < pick ? a : pick;
            out[cnt].v = a < pick ? pick : a;
            out[cnt].w = pick_w;
            ++cnt;
        }
        current = pick;
    }
    free(best);
    free(from);
    free(in_tree);
    return cnt;
}

/* mst_over_subset (src/coresg.cpp:97-141) for the dense branch (m <= 8192). */
static uint64_t mst_over_subset(const float* padded, uint32_t stride, const float* dists,
                                const uint32_t* counts, uint32_t k, const uint32_t* sel,
                                uint32_t m, orc_edge* out) {
    if (m < 2) return 0;
    float* pts = (float*)malloc(sizeof(float) * (uint64_t)m * stride);
    float* core = (float*)malloc(sizeof(float) * m);
    float* mat = (float*)malloc(sizeof(float) * (uint64_t)m * m);
    orc_edge* local = (orc_edge*)malloc(sizeof(orc_edge) * m);
    for (uint32_t i = 0; i < m; ++i) {
        memcpy(pts + (uint64_t)i * stride, padded + (uint64_t)sel[i] * stride, sizeof(float) * stride);
        const uint32_t c = counts[sel[i]];
        if (c == 0) core[i] = INFINITY;
        else core[i] = dists[(uint64_t)sel[i] * k + (k - 1 < c ? k - 1 : c - 1)];
    }
    orc_mrd_block(pts, m, stride, core, 0, m, mat);
    const uint64_t ne = orc_prim_dense(mat, m, local);
    for (uint64_t t = 0; t < ne; ++t) {
        const float base = orc_dist(pts + (uint64_t)local[t].u * stride,
                                    pts + (uint64_t)local[t].v * stride, stride);
        const uint32_t a = sel[local[t].u], b = sel[local[t].v];
        out[t].u = a < b ? a : b;
        out[t].v = a < b ? b : a;
        out[t].w = base;
    }
    free(pts);
    free(core);
    free(mat);
    free(local);
    return ne;
}

uint64_t orc_bridges(const float* padded, uint32_t n, uint32_t dim, uint32_t stride,
                     const uint32_t* ids, const float* dists, const uint32_t* counts, uint32_t k,
                     orc_edge* out, uint64_t cap, uint64_t* n_selected, uint64_t* n_repair) {
    uint32_t* comp = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    const uint32_t ncomp = orc_conn(ids, counts, n, k, comp);
    int32_t* rdeg = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    double* score = (double*)malloc(sizeof(double) * (n ? n : 1));
    orc_rdeg(ids, counts, n, k, rdeg);
    orc_scores(ids, counts, n, k, k, rdeg, score);
    const uint64_t edges = orc_undirected(ids, dists, counts, n, k, NULL);
    const uint64_t budget = orc_budget(dim, edges, n, 1.0, 2e9, 2, 0);
    uint32_t* sel = (uint32_t*)malloc(sizeof(uint32_t) * ((uint64_t)budget + 2ull * ncomp + 1));
    const uint64_t m = orc_select(score, rdeg, n, budget, comp, ncomp, 2, sel);
    if (n_selected) *n_selected = m;

    orc_edge* missing = (orc_edge*)malloc(sizeof(orc_edge) * (m + 4097 + n));
    uint64_t nm = mst_over_subset(padded, stride, dists, counts, k, sel, (uint32_t)m, missing);

    /* repair_connectivity (src/coresg.cpp:171-258) with reps_per_component 4,
     * max_reps 4096.  labels_with: k-NN components contracted and united over the
     * bridges; dense labels by first node. */
    uint64_t added = 0;
    uint32_t* cparent = (uint32_t*)malloc(sizeof(uint32_t) * (ncomp ? ncomp : 1));
    for (uint32_t c = 0; c < ncomp; ++c) cparent[c] = c;
    for (uint64_t t = 0; t < nm; ++t) uf_unite(cparent, comp[missing[t].u], comp[missing[t].v]);
    uint32_t* merged = (uint32_t*)malloc(sizeof(uint32_t) * (ncomp ? ncomp : 1));
    const uint32_t nc2 = uf_labels(cparent, ncomp, merged);
    if (nc2 > 1) {
        uint32_t per = 4;
        if ((uint64_t)nc2 * per > 4096) per = 4096 / nc2 > 1 ? 4096 / nc2 : 1;
        uint32_t* buckets = (uint32_t*)malloc(sizeof(uint32_t) * (uint64_t)nc2 * per);
        uint32_t* bsize = (uint32_t*)calloc(nc2, sizeof(uint32_t));
        for (uint32_t v = 0; v < n; ++v) {
            const uint32_t c = merged[comp[v]];
            uint32_t* b = buckets + (uint64_t)c * per;
            if (bsize[c] < per) {
                b[bsize[c]++] = v;
            } else {
                uint32_t worst = 0;
                for (uint32_t t = 1; t < bsize[c]; ++t) {
                    if (score[b[t]] > score[b[worst]]) worst = t;
                }
                if (score[v] < score[b[worst]]) b[worst] = v;
            }
        }
        uint64_t nreps = 0;
        for (uint32_t c = 0; c < nc2; ++c) nreps += bsize[c];
        uint32_t* reps = (uint32_t*)malloc(sizeof(uint32_t) * (nreps ? nreps : 1));
        uint64_t r = 0;
        for (uint32_t c = 0; c < nc2; ++c)
            for (uint32_t t = 0; t < bsize[c]; ++t) reps[r++] = buckets[(uint64_t)c * per + t];
        /* reps.size() > max_reps only with more than 4096 components; that branch
         * (partial_sort by score) is not restated here. */
        if (nreps >= 2 && nreps <= 4096) {
            orc_edge* rep_mst = (orc_edge*)malloc(sizeof(orc_edge) * nreps);
            const uint64_t nr = mst_over_subset(padded, stride, dists, counts, k, reps,
                                                (uint32_t)nreps, rep_mst);
            uint32_t* rp = (uint32_t*)malloc(sizeof(uint32_t) * nc2);
            for (uint32_t c = 0; c < nc2; ++c) rp[c] = c;
            for (uint64_t t = 0; t < nr; ++t) {
                if (uf_unite(rp, merged[comp[rep_mst[t].u]], merged[comp[rep_mst[t].v]])) {
                    missing[nm++] = rep_mst[t];
                    ++added;
                }
            }
            free(rp);
            free(rep_mst);
        }
        free(reps);
        free(buckets);
        free(bsize);
    }
    if (n_repair) *n_repair = added;
    const uint64_t w = nm < cap ? nm : cap;
    if (out) memcpy(out, missing, sizeof(orc_edge) * w);
    free(cparent);
    free(merged);
    free(missing);
    free(sel);
    free(comp);
    free(rdeg);
    free(score);
    return nm;
}

/* ---- brute force ------------------------------------------------------------- */

void orc_brute_knn(const float* padded, uint32_t n, uint32_t stride, uint32_t k,
                   const uint32_t* queries, uint32_t nq, uint32_t* out_ids, float* out_dists) {
    uint64_t* best = (uint64_t*)malloc(sizeof(uint64_t) * (k + 1));
    for (uint32_t t = 0; t < nq; ++t) {
        const uint32_t q = queries[t];
        uint32_t cnt = 0;
        for (uint32_t u = 0; u < n; ++u) {
            if (u == q) continue;
            const float r = orc_l2sqr(padded + (uint64_t)q * stride, padded + (uint64_t)u * stride, stride);
            const uint64_t key = ((uint64_t)fbits(r) << 32) | u;
            if (cnt == k && key >= best[k - 1]) continue;
            uint32_t pos = cnt < k ? cnt++ : k - 1;
            while (pos > 0 && best[pos - 1] > key) {
                best[pos] = best[pos - 1];
                --pos;
            }
            best[pos] = key;
        }
        for (uint32_t j = 0; j < k; ++j) {
            out_ids[(uint64_t)t * k + j] = j < cnt ? (uint32_t)(best[j] & 0xFFFFFFFFu) : INVALID;
            if (out_dists) {
                float r;
                uint32_t b = (uint32_t)(best[j] >> 32);
                memcpy(&r, &b, 4);
                out_dists[(uint64_t)t * k + j] = j < cnt ? sqrtf(r) : INFINITY;
            }
        }
    }
    free(best);
}
