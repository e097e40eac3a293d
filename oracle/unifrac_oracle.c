/*
 * ORACLE - test infrastructure only.  Never linked into, called by or shipped
 * with the product; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, as the checker.
 *
 * A plain-C restatement of the reference's Strided State UniFrac CPU path
 * (biocore/unifrac-binaries), written from its algorithm:
 *
 *   tree from BP arrays, open/close pairing  src/tree.cpp:72-99, 370-385
 *   postorder = matching open of the k-th ')'  src/tree.cpp:248-250
 *   shear(obs ids)                           src/tree.cpp:145-163
 *   collapse (single-child chains)           src/tree.cpp:165-191
 *   per-sample totals                        src/biom_inmem.cpp:513-526
 *   leaf proportions data/total (fp64 then T) src/biom_inmem.cpp:473-497
 *   internal = sum of children, left first   src/unifrac_internal.cpp:231-258
 *   postorder traversal, bypass_tips         src/unifrac_cmp.cpp:97-136
 *   method tables                            src/unifrac_task_impl.hpp:35-1932
 *   stripes -> full matrix                   src/unifrac.cpp:229-328
 *   Faith PD (+ zero-count sample filter)    src/unifrac.cpp:362-387,
 *                                            src/api.cpp:569-603, src/biom_inmem.cpp:284-338
 *
 * T is double for the *_fp64 methods and float for the fp32 ones (bare method
 * names are fp32, src/api.cpp:55-88).  The summation structure follows the
 * reference CPU tasks where it shapes fp32 rounding: weighted terms are summed
 * per batch of 496 embedded nodes and the batch sum is added to the stripe
 * (src/unifrac_task.hpp:376, src/unifrac_task_impl.hpp:107-193); unweighted
 * sums go through 8-node look-up tables in batches of 2048
 * (src/unifrac_task_impl.hpp:1281-1361, 1448-1514); generalized and VAW terms
 * run straight into the stripe (src/unifrac_task_impl.hpp:435-502, 924-1119,
 * 1755-1932).
 */
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { ST_OK = 0, ST_TABLE_EMPTY = 3, ST_UNKNOWN_METHOD = 4, ST_NO_OVERLAP = 5, ST_OUTPUT = 6 };
enum { M_UNWEIGHTED, M_UNWEIGHTED_UNNORM, M_WEIGHTED_NORM, M_WEIGHTED_UNNORM, M_GENERALIZED };

#define BATCH_WEIGHTED 496u
#define BATCH_UNWEIGHTED 2048u

/* ------------------------------------------------------------------ BP tree */

typedef struct {
    uint32_t n;          /* number of parentheses */
    bool *open;          /* structure */
    double *len;
    const char **name;
    uint32_t *match;     /* open <-> close */
} bp_t;

static void bp_free(bp_t *t) {
    free(t->open); free(t->len); free(t->name); free(t->match);
}

static void bp_pair(bp_t *t) {
    uint32_t *stack = malloc(sizeof(uint32_t) * (t->n / 2 + 1));
    uint32_t top = 0;
    for (uint32_t i = 0; i < t->n; i++) {
        if (t->open[i]) stack[top++] = i;
        else { uint32_t o = stack[--top]; t->match[o] = i; t->match[i] = o; }
    }
    free(stack);
}

static bp_t bp_copy_in(const bool *s, const double *len, const char *const *names, uint32_t n) {
    bp_t t;
    t.n = n;
    t.open = malloc(n ? n : 1); t.len = malloc(sizeof(double) * (n ? n : 1));
    t.name = malloc(sizeof(char *) * (n ? n : 1)); t.match = malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; i++) { t.open[i] = s[i]; t.len[i] = len[i]; t.name[i] = names[i]; }
    bp_pair(&t);
    return t;
}

static bool bp_leaf(const bp_t *t, uint32_t i) { return t->open[i] && !t->open[i + 1]; }

static bp_t bp_mask(const bp_t *t, const bool *keep, const double *len) {
    uint32_t m = 0;
    for (uint32_t i = 0; i < t->n; i++) m += keep[i];
    bp_t r;
    r.n = m;
    r.open = malloc(m ? m : 1); r.len = malloc(sizeof(double) * (m ? m : 1));
    r.name = malloc(sizeof(char *) * (m ? m : 1)); r.match = malloc(sizeof(uint32_t) * (m ? m : 1));
    uint32_t j = 0;
    for (uint32_t i = 0; i < t->n; i++)
        if (keep[i]) { r.open[j] = t->open[i]; r.len[j] = len[i]; r.name[j] = t->name[i]; j++; }
    bp_pair(&r);
    return r;
}

static int cmp_str(const void *a, const void *b) { return strcmp(*(const char *const *)a, *(const char *const *)b); }

static bool name_in(const char *const *sorted, uint32_t n, const char *key) {
    return bsearch(&key, sorted, n, sizeof(char *), cmp_str) != NULL;
}

/* shear: keep every tip named in `keep` plus all its ancestors (src/tree.cpp:145-163) */
static bp_t bp_shear(const bp_t *t, const char *const *keep_sorted, uint32_t n_keep) {
    bool *mask = calloc(t->n ? t->n : 1, 1);
    uint32_t *parent = malloc(sizeof(uint32_t) * (t->n ? t->n : 1));
    uint32_t *stack = malloc(sizeof(uint32_t) * (t->n / 2 + 1));
    uint32_t top = 0;
    for (uint32_t i = 0; i < t->n; i++) {
        if (t->open[i]) { parent[i] = top ? stack[top - 1] : UINT32_MAX; stack[top++] = i; }
        else top--;
    }
    for (uint32_t i = 0; i + 1 < t->n; i++) {
        if (bp_leaf(t, i) && name_in(keep_sorted, n_keep, t->name[i])) {
            mask[i] = mask[i + 1] = true;
            uint32_t p = parent[i];
            while (p != UINT32_MAX && !mask[p]) { mask[p] = mask[t->match[p]] = true; p = parent[p]; }
        }
    }
    bp_t r = bp_mask(t, mask, t->len);
    free(mask); free(parent); free(stack);
    return r;
}

/* collapse: a non-root node with one child is removed and its length added to
 * the child, visiting nodes in preorder (src/tree.cpp:165-191) */
static bp_t bp_collapse(const bp_t *t) {
    bool *mask = calloc(t->n ? t->n : 1, 1);
    double *len = malloc(sizeof(double) * (t->n ? t->n : 1));
    memcpy(len, t->len, sizeof(double) * t->n);
    for (uint32_t cur = 0; cur < t->n; cur++) {
        if (!t->open[cur]) continue;
        if (bp_leaf(t, cur) || cur == 0) { mask[cur] = mask[t->match[cur]] = true; continue; }
        uint32_t first = cur + 1;
        uint32_t last = t->match[t->match[cur] - 1];
        if (first == last) len[first] = len[first] + len[cur];
        else mask[cur] = mask[t->match[cur]] = true;
    }
    bp_t r = bp_mask(t, mask, len);
    free(mask); free(len);
    return r;
}

/* ----------------------------------------------------------------- table */

typedef struct {
    const uint32_t *indptr, *indices;
    const double *data;
    uint32_t n_obs, n_samples;
    const char *const *obs_ids;
    double *totals;     /* per sample, summed in observation order */
} table_t;

static void table_totals(table_t *tb) {
    tb->totals = calloc(tb->n_samples ? tb->n_samples : 1, sizeof(double));
    for (uint32_t i = 0; i < tb->n_obs; i++)
        for (uint32_t p = tb->indptr[i]; p < tb->indptr[i + 1]; p++) tb->totals[tb->indices[p]] += tb->data[p];
}

typedef struct { const char *name; uint32_t idx; } name_idx_t;
static int cmp_name_idx(const void *a, const void *b) {
    return strcmp(((const name_idx_t *)a)->name, ((const name_idx_t *)b)->name);
}

/* ------------------------------------------------------------- embedding */

typedef struct {
    uint32_t n_nodes;     /* non-root postorder nodes */
    uint32_t *node;       /* postorder k -> open index */
    int64_t *obs;         /* per postorder node: table row for leaves, -1 otherwise */
    bool *leaf;
} post_t;

static post_t postorder(const bp_t *t, const table_t *tb) {
    post_t p;
    uint32_t total = t->n / 2;
    p.n_nodes = total ? total - 1 : 0;
    p.node = malloc(sizeof(uint32_t) * (total ? total : 1));
    p.obs = malloc(sizeof(int64_t) * (total ? total : 1));
    p.leaf = malloc(total ? total : 1);
    name_idx_t *ix = malloc(sizeof(name_idx_t) * (tb->n_obs ? tb->n_obs : 1));
    for (uint32_t i = 0; i < tb->n_obs; i++) { ix[i].name = tb->obs_ids[i]; ix[i].idx = i; }
    qsort(ix, tb->n_obs, sizeof(name_idx_t), cmp_name_idx);
    uint32_t k = 0;
    for (uint32_t i = 0; i < t->n; i++) {
        if (t->open[i]) continue;
        uint32_t o = t->match[i];
        p.node[k] = o;
        p.leaf[k] = bp_leaf(t, o);
        p.obs[k] = -1;
        if (p.leaf[k]) {
            name_idx_t key = {t->name[o], 0};
            name_idx_t *hit = bsearch(&key, ix, tb->n_obs, sizeof(name_idx_t), cmp_name_idx);
            if (hit) p.obs[k] = hit->idx;
        }
        k++;
    }
    free(ix);
    return p;
}

static void post_free(post_t *p) { free(p->node); free(p->obs); free(p->leaf); }

/* u_n per node (rows in postorder), T = double or float.  Children are added
 * left to right onto a zeroed vector (src/unifrac_internal.cpp:240-257). */
#define DEFINE_EMBED(T)                                                                          \
    static T *embed_##T(const bp_t *t, const post_t *p, const table_t *tb, bool normalize) {     \
        uint32_t n = tb->n_samples;                                                              \
        T *u = calloc((size_t)p->n_nodes * n + 1, sizeof(T));                                    \
        uint32_t *row_of = malloc(sizeof(uint32_t) * (t->n ? t->n : 1));                          \
        for (uint32_t k = 0; k < p->n_nodes; k++) {                                              \
            uint32_t o = p->node[k];                                                             \
            row_of[o] = k;                                                                       \
            T *dst = u + (size_t)k * n;                                                          \
            if (p->leaf[k]) {                                                                    \
                if (p->obs[k] < 0) continue;                                                     \
                uint32_t r = (uint32_t)p->obs[k];                                                \
                for (uint32_t q = tb->indptr[r]; q < tb->indptr[r + 1]; q++) {                   \
                    uint32_t j = tb->indices[q];                                                 \
                    dst[j] = normalize ? (T)(tb->data[q] / tb->totals[j]) : (T)tb->data[q];      \
                }                                                                                \
            } else {                                                                             \
                uint32_t c = o + 1;                                                              \
                while (c < t->n && t->open[c]) {                                                 \
                    const T *src = u + (size_t)row_of[c] * n;                                    \
                    for (uint32_t j = 0; j < n; j++) dst[j] = dst[j] + src[j];                   \
                    c = t->match[c] + 1;                                                         \
                }                                                                                \
            }                                                                                    \
        }                                                                                        \
        free(row_of);                                                                            \
        return u;                                                                                \
    }
DEFINE_EMBED(double)
DEFINE_EMBED(float)

/* -------------------------------------------------------------- stripes */

typedef struct {
    int method;
    bool vaw, bypass, normalize;
    double alpha;
} params_t;

/* Embedded node list: postorder nodes minus tips when bypass_tips. */
static uint32_t embedded_nodes(const post_t *p, bool bypass, uint32_t *out) {
    uint32_t e = 0;
    for (uint32_t k = 0; k < p->n_nodes; k++)
        if (!(bypass && p->leaf[k])) out[e++] = k;
    return e;
}

/* One stripe element dm[s][k] (and its total), pair (k, l = (k+s+1) mod n).
 * Returns num/den for normalized methods, num otherwise. */
#define DEFINE_PAIR(T, SQRT, POW, FABS)                                                               \
    static double pair_##T(const params_t *pr, const T *u, const T *cnt, const T *tot, const T *len,  \
                           const uint32_t *emb, uint32_t n_emb, uint32_t n, uint32_t k, uint32_t l) {   \
        T num = 0, den = 0;                                                                           \
        if (pr->vaw) {                                                                                \
            const T m = tot[k] + tot[l];                                                              \
            for (uint32_t e = 0; e < n_emb; e++) {                                                    \
                const T *ur = u + (size_t)emb[e] * n, *cr = cnt + (size_t)emb[e] * n;                 \
                T mi = cr[k] + cr[l];                                                                 \
                T vaw = SQRT(mi * (m - mi));                                                          \
                if (!(vaw > 0)) continue;                                                             \
                T a = ur[k], b = ur[l], L = len[e];                                                   \
                switch (pr->method) {                                                                 \
                case M_UNWEIGHTED:                                                                    \
                case M_UNWEIGHTED_UNNORM: {                                                           \
                    T lv = L / vaw;                                                                   \
                    num += (T)((a > 0) != (b > 0)) * lv;                                              \
                    den += (T)((a > 0) || (b > 0)) * lv;                                              \
                } break;                                                                              \
                case M_WEIGHTED_NORM:                                                                 \
                case M_WEIGHTED_UNNORM:                                                               \
                    num += (FABS(a - b) * L) / vaw;                                                   \
                    den += ((a + b) * L) / vaw;                                                       \
                    break;                                                                            \
                default: {                                                                            \
                    T s1 = (a + b) / vaw, d1 = FABS(a - b) / vaw;                                     \
                    T sp = POW(s1, (T)pr->alpha) * L;                                                 \
                    num += sp * (d1 / s1);                                                            \
                    den += sp;                                                                        \
                }                                                                                     \
                }                                                                                     \
            }                                                                                         \
        } else if (pr->method == M_GENERALIZED) {                                                     \
            for (uint32_t e = 0; e < n_emb; e++) {                                                    \
                const T *ur = u + (size_t)emb[e] * n;                                                 \
                T a = ur[k], b = ur[l], s1 = a + b;                                                   \
                if (s1 != 0) {                                                                        \
                    T sp = POW(s1, (T)pr->alpha) * len[e];                                            \
                    num += sp * (FABS(a - b) / s1);                                                   \
                    den += sp;                                                                        \
                }                                                                                     \
            }                                                                                         \
        } else if (pr->method == M_WEIGHTED_NORM || pr->method == M_WEIGHTED_UNNORM) {                \
            for (uint32_t e0 = 0; e0 < n_emb; e0 += BATCH_WEIGHTED) {                                 \
                uint32_t e1 = e0 + BATCH_WEIGHTED < n_emb ? e0 + BATCH_WEIGHTED : n_emb;              \
                T part = 0, sk = 0, sl = 0;                                                           \
                for (uint32_t e = e0; e < e1; e++) {                                                  \
                    const T *ur = u + (size_t)emb[e] * n;                                             \
                    part += FABS(ur[k] - ur[l]) * len[e];                                             \
                    sk += ur[k] * len[e];                                                             \
                    sl += ur[l] * len[e];                                                             \
                }                                                                                     \
                num += part;                                                                          \
                den += sk + sl;                                                                       \
            }                                                                                         \
        } else { /* unweighted, 8-node length tables */                                               \
            for (uint32_t e0 = 0; e0 < n_emb; e0 += BATCH_UNWEIGHTED) {                               \
                uint32_t e1 = e0 + BATCH_UNWEIGHTED < n_emb ? e0 + BATCH_UNWEIGHTED : n_emb;          \
                T part = 0, part_tot = 0;                                                             \
                for (uint32_t g = e0; g < e1; g += 8) {                                               \
                    T x8 = 0, o8 = 0;                                                                 \
                    bool any_x = false, any_o = false;                                                \
                    for (uint32_t e = g; e < g + 8 && e < e1; e++) {                                  \
                        const T *ur = u + (size_t)emb[e] * n;                                         \
                        bool pa = ur[k] > 0, pb = ur[l] > 0;                                          \
                        if (pa != pb) { x8 += len[e]; any_x = true; }                                 \
                        if (pa || pb) { o8 += len[e]; any_o = true; }                                 \
                    }                                                                                 \
                    if (any_o) { part_tot += o8; if (any_x) part += x8; }                             \
                }                                                                                     \
                num += part;                                                                          \
                den += part_tot;                                                                      \
            }                                                                                         \
        }                                                                                             \
        if (pr->method == M_WEIGHTED_UNNORM || pr->method == M_UNWEIGHTED_UNNORM) return (double)num;  \
        return (double)(num / den);                                                                   \
    }
DEFINE_PAIR(double, sqrt, pow, fabs)
DEFINE_PAIR(float, sqrtf, powf, fabsf)

static int parse_method(const char *m, int *method, bool *fp64) {
    static const struct { const char *name; int method; bool fp64; } tab[] = {
        {"unweighted", M_UNWEIGHTED, false}, {"weighted_normalized", M_WEIGHTED_NORM, false},
        {"weighted_unnormalized", M_WEIGHTED_UNNORM, false}, {"unweighted_unnormalized", M_UNWEIGHTED_UNNORM, false},
        {"generalized", M_GENERALIZED, false},
        {"unweighted_fp64", M_UNWEIGHTED, true}, {"weighted_normalized_fp64", M_WEIGHTED_NORM, true},
        {"weighted_unnormalized_fp64", M_WEIGHTED_UNNORM, true},
        {"unweighted_unnormalized_fp64", M_UNWEIGHTED_UNNORM, true}, {"generalized_fp64", M_GENERALIZED, true},
        {"unweighted_fp32", M_UNWEIGHTED, false}, {"weighted_normalized_fp32", M_WEIGHTED_NORM, false},
        {"weighted_unnormalized_fp32", M_WEIGHTED_UNNORM, false},
        {"unweighted_unnormalized_fp32", M_UNWEIGHTED_UNNORM, false}, {"generalized_fp32", M_GENERALIZED, false},
    };
    for (size_t i = 0; i < sizeof(tab) / sizeof(tab[0]); i++)
        if (strcmp(m, tab[i].name) == 0) { *method = tab[i].method; *fp64 = tab[i].fp64; return 0; }
    return -1;
}

/* Validation + shear/collapse shared by both entry points. */
static int prepare(const uint32_t *indptr, const uint32_t *indices, const double *data, int n_obs, int n_samples,
                   const char *const *obs_ids, const bool *structure, const double *lengths,
                   const char *const *names, int n_parens, table_t *tb, bp_t *sheared) {
    if (n_samples <= 0 || n_obs <= 0) return ST_TABLE_EMPTY;
    tb->indptr = indptr; tb->indices = indices; tb->data = data;
    tb->n_obs = (uint32_t)n_obs; tb->n_samples = (uint32_t)n_samples; tb->obs_ids = obs_ids;
    bp_t full = bp_copy_in(structure, lengths, names, (uint32_t)n_parens);
    /* every table id must be a tip name (src/unifrac.cpp:46-60) */
    uint32_t n_tips = 0;
    const char **tips = malloc(sizeof(char *) * (full.n ? full.n : 1));
    for (uint32_t i = 0; i + 1 < full.n; i++)
        if (bp_leaf(&full, i)) tips[n_tips++] = full.name[i];
    qsort(tips, n_tips, sizeof(char *), cmp_str);
    for (uint32_t i = 0; i < tb->n_obs; i++)
        if (!name_in(tips, n_tips, obs_ids[i])) { free(tips); bp_free(&full); return ST_NO_OVERLAP; }
    free(tips);
    const char **keep = malloc(sizeof(char *) * tb->n_obs);
    for (uint32_t i = 0; i < tb->n_obs; i++) keep[i] = obs_ids[i];
    qsort(keep, tb->n_obs, sizeof(char *), cmp_str);
    bp_t sh = bp_shear(&full, keep, tb->n_obs);
    *sheared = bp_collapse(&sh);
    bp_free(&sh); bp_free(&full); free(keep);
    table_totals(tb);
    return ST_OK;
}

/* Full matrix from stripes, as stripes_to_matrix (src/unifrac.cpp:229-328). */
static void stripes_to_matrix(const double *stripes, uint32_t n, double *out) {
    uint32_t n_stripes = (n + 1) / 2;
    for (uint32_t i = 0; i < n; i++) out[(size_t)i * n + i] = 0.0;
    for (uint32_t s = 0; s < n_stripes; s++)
        for (uint32_t k = 0; k < n; k++) {
            uint32_t l = (k + s + 1) % n;
            double v = stripes[(size_t)s * n + k];
            out[(size_t)k * n + l] = v;
            out[(size_t)l * n + k] = v;
        }
}

int oracle_one_off(const uint32_t *indptr, const uint32_t *indices, const double *data, int n_obs, int n_samples,
                   const char *const *obs_ids, const char *const *sample_ids, const bool *structure,
                   const double *lengths, const char *const *names, int n_parens, const char *method,
                   bool variance_adjust, double alpha, bool bypass_tips, bool normalize, unsigned stripe_start,
                   unsigned stripe_stop, double *out_stripes, double *out_matrix, uint64_t *out_n_embedded) {
    (void)sample_ids;
    params_t pr = {0};
    bool fp64;
    if (parse_method(method, &pr.method, &fp64) != 0) return ST_UNKNOWN_METHOD;
    pr.vaw = variance_adjust; pr.bypass = bypass_tips; pr.normalize = normalize; pr.alpha = alpha;
    table_t tb; bp_t t;
    int rc = prepare(indptr, indices, data, n_obs, n_samples, obs_ids, structure, lengths, names, n_parens, &tb, &t);
    if (rc != ST_OK) return rc;
    const uint32_t n = tb.n_samples, n_stripes = (n + 1) / 2;
    if (stripe_stop == 0 || stripe_stop <= stripe_start) { stripe_start = 0; stripe_stop = n_stripes; }
    if (stripe_stop > n_stripes) { bp_free(&t); free(tb.totals); return ST_OUTPUT; }
    post_t p = postorder(&t, &tb);
    uint32_t *emb = malloc(sizeof(uint32_t) * (p.n_nodes + 1));
    uint32_t n_emb = embedded_nodes(&p, bypass_tips, emb);
    if (out_n_embedded) *out_n_embedded = n_emb;
    double *full = out_matrix ? calloc((size_t)n_stripes * n, sizeof(double)) : NULL;

    if (fp64) {
        double *u = embed_double(&t, &p, &tb, normalize);
        double *cnt = variance_adjust ? embed_double(&t, &p, &tb, false) : NULL;
        double *len = malloc(sizeof(double) * (n_emb + 1));
        for (uint32_t e = 0; e < n_emb; e++) len[e] = t.len[p.node[emb[e]]];
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t s = stripe_start; s < (int64_t)stripe_stop; s++)
            for (uint32_t k = 0; k < n; k++) {
                double v = pair_double(&pr, u, cnt, tb.totals, len, emb, n_emb, n, k, (uint32_t)((k + s + 1) % n));
                out_stripes[(size_t)(s - stripe_start) * n + k] = v;
                if (full) full[(size_t)s * n + k] = v;
            }
        free(u); free(cnt); free(len);
    } else {
        float *u = embed_float(&t, &p, &tb, normalize);
        float *cnt = variance_adjust ? embed_float(&t, &p, &tb, false) : NULL;
        float *len = malloc(sizeof(float) * (n_emb + 1));
        float *tot = malloc(sizeof(float) * n);
        for (uint32_t e = 0; e < n_emb; e++) len[e] = (float)t.len[p.node[emb[e]]];
        for (uint32_t j = 0; j < n; j++) tot[j] = (float)tb.totals[j];
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t s = stripe_start; s < (int64_t)stripe_stop; s++)
            for (uint32_t k = 0; k < n; k++) {
                double v = pair_float(&pr, u, cnt, tot, len, emb, n_emb, n, k, (uint32_t)((k + s + 1) % n));
                out_stripes[(size_t)(s - stripe_start) * n + k] = v;
                if (full) full[(size_t)s * n + k] = v;
            }
        free(u); free(cnt); free(len); free(tot);
    }
    if (full) { stripes_to_matrix(full, n, out_matrix); free(full); }
    free(emb); post_free(&p); bp_free(&t); free(tb.totals);
    return ST_OK;
}

/* Faith PD over the zero-count-filtered table (src/api.cpp:569-603,
 * src/biom_inmem.cpp:284-338, src/unifrac.cpp:362-387). */
int oracle_faith_pd(const uint32_t *indptr, const uint32_t *indices, const double *data, int n_obs, int n_samples,
                    const char *const *obs_ids, const char *const *sample_ids, const bool *structure,
                    const double *lengths, const char *const *names, int n_parens, double *out_values,
                    uint32_t *out_kept, uint32_t *out_n_kept) {
    (void)sample_ids;
    if (n_samples <= 0 || n_obs <= 0) return ST_TABLE_EMPTY;
    table_t full_tb = {indptr, indices, data, (uint32_t)n_obs, (uint32_t)n_samples, obs_ids, NULL};
    table_totals(&full_tb);
    /* keep samples with total >= 1, renumbered; keep observations left with entries */
    uint32_t *new_idx = malloc(sizeof(uint32_t) * n_samples);
    uint32_t n_keep = 0;
    for (uint32_t j = 0; j < (uint32_t)n_samples; j++) {
        new_idx[j] = full_tb.totals[j] >= 1.0 ? n_keep : UINT32_MAX;
        if (full_tb.totals[j] >= 1.0) out_kept[n_keep++] = j;
    }
    uint32_t *f_indptr = calloc(n_obs + 1, sizeof(uint32_t));
    uint32_t *f_indices = malloc(sizeof(uint32_t) * (indptr[n_obs] + 1));
    double *f_data = malloc(sizeof(double) * (indptr[n_obs] + 1));
    const char **f_ids = malloc(sizeof(char *) * n_obs);
    uint32_t rows = 0, nnz = 0;
    for (uint32_t i = 0; i < (uint32_t)n_obs; i++) {
        uint32_t start = nnz;
        for (uint32_t q = indptr[i]; q < indptr[i + 1]; q++)
            if (new_idx[indices[q]] != UINT32_MAX) { f_indices[nnz] = new_idx[indices[q]]; f_data[nnz] = data[q]; nnz++; }
        if (nnz > start) { f_ids[rows] = obs_ids[i]; rows++; f_indptr[rows] = nnz; }
    }
    int rc = ST_OK;
    if (n_keep == 0 || rows == 0) {
        /* all samples empty: zero result for every sample (src/api.cpp:580-586) */
        *out_n_kept = (uint32_t)n_samples;
        for (uint32_t j = 0; j < (uint32_t)n_samples; j++) { out_values[j] = 0.0; out_kept[j] = j; }
    } else {
        table_t tb; bp_t t;
        rc = prepare(f_indptr, f_indices, f_data, (int)rows, (int)n_keep, f_ids, structure, lengths, names, n_parens,
                     &tb, &t);
        if (rc == ST_OK) {
            post_t p = postorder(&t, &tb);
            double *u = embed_double(&t, &p, &tb, true);
            for (uint32_t j = 0; j < n_keep; j++) out_values[j] = 0.0;
            for (uint32_t k = 0; k < p.n_nodes; k++) {
                double L = t.len[p.node[k]];
                const double *ur = u + (size_t)k * n_keep;
                for (uint32_t j = 0; j < n_keep; j++) out_values[j] += (double)(ur[j] > 0) * L;
            }
            *out_n_kept = n_keep;
            free(u); post_free(&p); bp_free(&t); free(tb.totals);
        }
    }
    free(new_idx); free(f_indptr); free(f_indices); free(f_data); free(f_ids); free(full_tb.totals);
    return rc;
}
