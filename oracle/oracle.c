/*
 * oracle.c -- CPU restatement of tensor-episdet's contingency-table and
 * scoring path (see oracle.h for the data format and the parity status).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, and the timed CPU
 * baseline ("port").  Scalar 64-bit popcount, one pthread per core.
 *
 * Deliberate differences from the reference, each a fix of a reference
 * defect rather than a change of the intended result:
 *  - K2 table covers every index the scorer reads (0..N+1); the reference
 *    allocates max(nc,nctrl)+1 entries and reads past them
 *    (src/search-pairs.cu:98-102 vs include/scoring.hpp:6).
 *  - MI table covers index N (a cell holding every sample).
 *  - Ties between equal scores go to the lowest set key; the reference keeps
 *    whichever block wins a racy CAS (include/reduction.hpp:96-108).
 *  - Pair counts are exact for every class size; the reference 3-way count
 *    kernels overrun when a padded class is not a multiple of 4096 samples
 *    (src/helper.cu:237-277, :414-421).
 *
 * Floating point: this file must be compiled with -ffp-contract=off so that
 * every fused multiply-add is the explicit fma()/fmaf() written below, which
 * the CUDA scorers issue in the same order.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

int32_t od_class_words(int32_t n) { return ((n + 1023) / 1024) * 32; }

static inline const uint32_t* od_row(const uint32_t* planes, int32_t W, int32_t snp, int32_t g) {
    return planes + ((size_t)snp * 2 + (size_t)g) * (size_t)W;
}

/* Valid-sample mask of word w of an n-sample row (MSB-first), helper.cu:72-73. */
static inline uint32_t od_word_mask(int32_t n, int32_t w) {
    int32_t lo = w * 32;
    if (lo + 32 <= n) return 0xFFFFFFFFu;
    if (lo >= n) return 0u;
    return 0xFFFFFFFFu << (32 - (n - lo));
}

static inline int od_popc(uint32_t v) { return __builtin_popcount(v); }
static inline int od_popc64(uint64_t v) { return __builtin_popcountll(v); }

uint64_t od_set_key(int order, uint32_t a, uint32_t b, uint32_t c) {
    if (order == 2) return ((uint64_t)a << 32) | (uint64_t)b;
    return ((uint64_t)a << 42) | ((uint64_t)b << 21) | (uint64_t)c;
}

void od_set_unkey(int order, uint64_t key, uint32_t out[3]) {
    if (order == 2) {
        out[0] = (uint32_t)(key >> 32);
        out[1] = (uint32_t)(key & 0xFFFFFFFFu);
        out[2] = 0;
    } else {
        out[0] = (uint32_t)((key >> 42) & 0x1FFFFF);
        out[1] = (uint32_t)((key >> 21) & 0x1FFFFF);
        out[2] = (uint32_t)(key & 0x1FFFFF);
    }
}

/* helper.cu:13-52 */
void od_marginals(const uint32_t* planes, int32_t M, int32_t n, uint32_t* out) {
    int32_t W = od_class_words(n);
    int32_t nw = (n + 31) / 32;
    for (int32_t s = 0; s < M; ++s) {
        uint32_t c0 = 0, c1 = 0;
        const uint32_t* r0 = od_row(planes, W, s, 0);
        const uint32_t* r1 = od_row(planes, W, s, 1);
        for (int32_t w = 0; w < nw; ++w) {
            c0 += (uint32_t)od_popc(r0[w]);
            c1 += (uint32_t)od_popc(r1[w]);
        }
        out[0 * (size_t)M + s] = c0;
        out[1 * (size_t)M + s] = c1;
        out[2 * (size_t)M + s] = (uint32_t)n - (c0 + c1);
    }
}

int od_validate(const uint32_t* planes, int32_t M, int32_t n) {
    int32_t W = od_class_words(n);
    for (int32_t s = 0; s < M; ++s) {
        const uint32_t* r0 = od_row(planes, W, s, 0);
        const uint32_t* r1 = od_row(planes, W, s, 1);
        for (int32_t w = 0; w < W; ++w) {
            uint32_t m = od_word_mask(n, w);
            if ((r0[w] & ~m) || (r1[w] & ~m) || (r0[w] & r1[w])) return 1;
        }
    }
    return 0;
}

/* helper.cu:58-194: direct 9-cell pair count; genotype-2 plane is ~(g0|g1)
 * restricted to the n valid samples. */
void od_pair9(const uint32_t* planes, int32_t n, int32_t a, int32_t b, uint32_t out[9]) {
    int32_t W = od_class_words(n);
    int32_t nw = (n + 31) / 32;
    const uint32_t* a0 = od_row(planes, W, a, 0);
    const uint32_t* a1 = od_row(planes, W, a, 1);
    const uint32_t* b0 = od_row(planes, W, b, 0);
    const uint32_t* b1 = od_row(planes, W, b, 1);
    uint32_t acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int32_t w = 0; w < nw; ++w) {
        uint32_t m = od_word_mask(n, w);
        uint32_t A[3] = {a0[w], a1[w], ~(a0[w] | a1[w]) & m};
        uint32_t B[3] = {b0[w], b1[w], ~(b0[w] | b1[w]) & m};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) acc[i * 3 + j] += (uint32_t)od_popc(A[i] & B[j]);
    }
    memcpy(out, acc, sizeof(acc));
}

static uint32_t od_and2(const uint32_t* p, int32_t W, int32_t a, int32_t ga, int32_t b, int32_t gb) {
    const uint64_t* x = (const uint64_t*)od_row(p, W, a, ga);
    const uint64_t* y = (const uint64_t*)od_row(p, W, b, gb);
    uint32_t c = 0;
    for (int32_t w = 0; w < W / 2; ++w) c += (uint32_t)od_popc64(x[w] & y[w]);
    return c;
}

static uint32_t od_and3(const uint32_t* p, int32_t W, int32_t x, int32_t gx, int32_t y, int32_t gy, int32_t z,
                        int32_t gz) {
    const uint64_t* X = (const uint64_t*)od_row(p, W, x, gx);
    const uint64_t* Y = (const uint64_t*)od_row(p, W, y, gy);
    const uint64_t* Z = (const uint64_t*)od_row(p, W, z, gz);
    uint32_t c = 0;
    for (int32_t w = 0; w < W / 2; ++w) c += (uint32_t)od_popc64(X[w] & Y[w] & Z[w]);
    return c;
}

/* helper.cu:634-662 for one class.  AND cells are counted directly; for
 * zero-padded rows they equal (popcA+popcB-popc(A^B))/2 of helper.cu:636. */
static void od_table2_class(const uint32_t* p, int32_t n, int32_t a, int32_t b, int32_t t[9]) {
    int32_t W = od_class_words(n);
    int32_t nw = (n + 31) / 32;
    int32_t pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
    for (int32_t w = 0; w < nw; ++w) {
        pa[0] += od_popc(od_row(p, W, a, 0)[w]);
        pa[1] += od_popc(od_row(p, W, a, 1)[w]);
        pb[0] += od_popc(od_row(p, W, b, 0)[w]);
        pb[1] += od_popc(od_row(p, W, b, 1)[w]);
    }
    pa[2] = n - (pa[0] + pa[1]);
    pb[2] = n - (pb[0] + pb[1]);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) t[i * 3 + j] = (int32_t)od_and2(p, W, a, i, b, j);
    t[0 * 3 + 2] = pa[0] - (t[0 * 3 + 0] + t[0 * 3 + 1]);
    t[1 * 3 + 2] = pa[1] - (t[1 * 3 + 0] + t[1 * 3 + 1]);
    t[2 * 3 + 0] = pb[0] - (t[0 * 3 + 0] + t[1 * 3 + 0]);
    t[2 * 3 + 1] = pb[1] - (t[0 * 3 + 1] + t[1 * 3 + 1]);
    t[2 * 3 + 2] = pa[2] - (t[2 * 3 + 0] + t[2 * 3 + 1]);
}

void od_table2(const od_dataset* ds, int32_t a, int32_t b, int32_t cases[9], int32_t controls[9]) {
    od_table2_class(ds->cases, ds->num_cases, a, b, cases);
    od_table2_class(ds->controls, ds->num_controls, a, b, controls);
}

#define C3(i, j, k) ((i) * 9 + (j) * 3 + (k))

/* The 19 derived cells of helper.cu:494-548 (macros include/helper.hpp:34-51).
 * xy[a*3+b] = count(X=a,Y=b), xz[a*3+b] = count(X=a,Z=b),
 * yz[a*3+b] = count(Y=a,Z=b); t holds the 8 AND cells on entry. */
static void od_derive27(int32_t t[27], const uint32_t xy[9], const uint32_t xz[9], const uint32_t yz[9]) {
    t[C3(0, 0, 2)] = (int32_t)xy[0 * 3 + 0] - (t[C3(0, 0, 0)] + t[C3(0, 0, 1)]);
    t[C3(0, 1, 2)] = (int32_t)xy[0 * 3 + 1] - (t[C3(0, 1, 0)] + t[C3(0, 1, 1)]);
    t[C3(0, 2, 0)] = (int32_t)xz[0 * 3 + 0] - (t[C3(0, 0, 0)] + t[C3(0, 1, 0)]);
    t[C3(0, 2, 1)] = (int32_t)xz[0 * 3 + 1] - (t[C3(0, 0, 1)] + t[C3(0, 1, 1)]);
    t[C3(0, 2, 2)] = (int32_t)xz[0 * 3 + 2] - (t[C3(0, 0, 2)] + t[C3(0, 1, 2)]);
    t[C3(1, 0, 2)] = (int32_t)xy[1 * 3 + 0] - (t[C3(1, 0, 0)] + t[C3(1, 0, 1)]);
    t[C3(1, 1, 2)] = (int32_t)xy[1 * 3 + 1] - (t[C3(1, 1, 0)] + t[C3(1, 1, 1)]);
    t[C3(1, 2, 0)] = (int32_t)xz[1 * 3 + 0] - (t[C3(1, 0, 0)] + t[C3(1, 1, 0)]);
    t[C3(1, 2, 1)] = (int32_t)xz[1 * 3 + 1] - (t[C3(1, 0, 1)] + t[C3(1, 1, 1)]);
    t[C3(1, 2, 2)] = (int32_t)xz[1 * 3 + 2] - (t[C3(1, 0, 2)] + t[C3(1, 1, 2)]);
    t[C3(2, 0, 0)] = (int32_t)yz[0 * 3 + 0] - (t[C3(0, 0, 0)] + t[C3(1, 0, 0)]);
    t[C3(2, 0, 1)] = (int32_t)yz[0 * 3 + 1] - (t[C3(0, 0, 1)] + t[C3(1, 0, 1)]);
    t[C3(2, 0, 2)] = (int32_t)xy[2 * 3 + 0] - (t[C3(2, 0, 0)] + t[C3(2, 0, 1)]);
    t[C3(2, 1, 0)] = (int32_t)yz[1 * 3 + 0] - (t[C3(0, 1, 0)] + t[C3(1, 1, 0)]);
    t[C3(2, 1, 1)] = (int32_t)yz[1 * 3 + 1] - (t[C3(0, 1, 1)] + t[C3(1, 1, 1)]);
    t[C3(2, 1, 2)] = (int32_t)xy[2 * 3 + 1] - (t[C3(2, 1, 0)] + t[C3(2, 1, 1)]);
    t[C3(2, 2, 0)] = (int32_t)xz[2 * 3 + 0] - (t[C3(2, 0, 0)] + t[C3(2, 1, 0)]);
    t[C3(2, 2, 1)] = (int32_t)xz[2 * 3 + 1] - (t[C3(2, 0, 1)] + t[C3(2, 1, 1)]);
    t[C3(2, 2, 2)] = (int32_t)xz[2 * 3 + 2] - (t[C3(2, 0, 2)] + t[C3(2, 1, 2)]);
}

static void od_table3_class(const uint32_t* p, int32_t n, int32_t x, int32_t y, int32_t z, int32_t t[27]) {
    int32_t W = od_class_words(n);
    uint32_t xy[9], xz[9], yz[9];
    od_pair9(p, n, x, y, xy);
    od_pair9(p, n, x, z, xz);
    od_pair9(p, n, y, z, yz);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) t[C3(i, j, k)] = (int32_t)od_and3(p, W, x, i, y, j, z, k);
    od_derive27(t, xy, xz, yz);
}

void od_table3(const od_dataset* ds, int32_t x, int32_t y, int32_t z, int32_t cases[27], int32_t controls[27]) {
    od_table3_class(ds->cases, ds->num_cases, x, y, z, cases);
    od_table3_class(ds->controls, ds->num_controls, x, y, z, controls);
}

/* Tables: K2 follows src/search-pairs.cu:97-102 (lnG(v+1) at index v, built
 * in double with glibc lgamma); MI follows src/search-pairs.cu:88-95
 * (log2(v * invN), index 0 -> 0). */
int od_tables_build(int32_t score, int32_t num_cases, int32_t num_controls, od_tables* t) {
    memset(t, 0, sizeof(*t));
    int32_t N = num_cases + num_controls;
    t->score = score;
    t->num_cases = num_cases;
    t->num_controls = num_controls;
    t->size = (score == OD_K2) ? N + 2 : N + 1;
    t->t32 = (float*)malloc(sizeof(float) * (size_t)t->size);
    t->t64 = (double*)malloc(sizeof(double) * (size_t)t->size);
    if (!t->t32 || !t->t64) return 1;
    if (score == OD_K2) {
        for (int32_t v = 0; v < t->size; ++v) {
            double g = lgamma((double)v + 1.0);
            t->t64[v] = g;
            t->t32[v] = (float)g;
        }
    } else {
        t->inv_n32 = (float)(1.0 / (double)N);
        t->inv_n64 = 1.0 / (double)N;
        t->t32[0] = 0.0f;
        t->t64[0] = 0.0;
        for (int32_t v = 1; v < t->size; ++v) {
            t->t32[v] = (float)log2((double)v * (double)t->inv_n32);
            t->t64[v] = log2((double)v / (double)N);
        }
        /* H(Y), scoring.hpp:29-30.  FP64 score: in double throughout.  FP32
         * score: as the reference's device code evaluates those two lines --
         * p = n * invN as a float product, the first term a double product
         * rounded to float, the second a double fused multiply-add (nvcc
         * contracts `entropyY += (-1.0) * p * t`) rounded to float. */
        double p1 = (double)num_cases * t->inv_n64;
        double p2 = (double)num_controls * t->inv_n64;
        t->hy64 = -(p1 * t->t64[num_cases]) - (p2 * t->t64[num_controls]);
        float q1 = (float)num_cases * t->inv_n32;
        float hy = (float)(-((double)q1 * (double)t->t32[num_cases]));
        float q2 = (float)num_controls * t->inv_n32;
        t->hy32 = (float)fma(-(double)q2, (double)t->t32[num_controls], (double)hy);
    }
    return 0;
}

void od_tables_free(od_tables* t) {
    free(t->t32);
    free(t->t64);
    t->t32 = NULL;
    t->t64 = NULL;
}

/* include/scoring.hpp:5-16 (CALC_K2 / CALC_MI), :18-51, :53-90: cells are
 * visited in index order (i outer, then j, then k). */
float od_score32(const od_tables* t, const int32_t* cs, const int32_t* cn, int32_t ncells) {
    if (t->score == OD_K2) {
        float s = 0.0f;
        for (int32_t c = 0; c < ncells; ++c) {
            float term = (t->t32[cn[c]] + t->t32[cs[c]]) - t->t32[cn[c] + cs[c] + 1];
            s = s + term;
        }
        return fabsf(s);
    }
    float ha = 0.0f, hx = 0.0f;
    for (int32_t c = 0; c < ncells; ++c) {
        float pc = (float)cs[c] * t->inv_n32;
        ha = fmaf(-pc, t->t32[cs[c]], ha);
        float pn = (float)cn[c] * t->inv_n32;
        ha = fmaf(-pn, t->t32[cn[c]], ha);
        hx = fmaf(-(pc + pn), t->t32[cs[c] + cn[c]], hx);
    }
    return (hx + t->hy32) - ha;
}

double od_score64(const od_tables* t, const int32_t* cs, const int32_t* cn, int32_t ncells) {
    if (t->score == OD_K2) {
        double s = 0.0;
        for (int32_t c = 0; c < ncells; ++c) {
            double term = (t->t64[cn[c]] + t->t64[cs[c]]) - t->t64[cn[c] + cs[c] + 1];
            s = s + term;
        }
        return fabs(s);
    }
    double ha = 0.0, hx = 0.0;
    for (int32_t c = 0; c < ncells; ++c) {
        double pc = (double)cs[c] * t->inv_n64;
        ha = fma(-pc, t->t64[cs[c]], ha);
        double pn = (double)cn[c] * t->inv_n64;
        ha = fma(-pn, t->t64[cn[c]], ha);
        hx = fma(-(pc + pn), t->t64[cs[c] + cn[c]], hx);
    }
    return (hx + t->hy64) - ha;
}

uint32_t od_score_key(int32_t score, float s) {
    if (score == OD_MI) s = -s;
    uint32_t u;
    memcpy(&u, &s, sizeof(u));
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* ---------------------------------------------------------------- search */

typedef struct od_cand {
    uint32_t key;
    uint64_t set;
    float s32;
} od_cand;

/* a is strictly better than b */
static inline int od_better(const od_cand* a, const od_cand* b) {
    return a->key < b->key || (a->key == b->key && a->set < b->set);
}

typedef struct od_heap {  /* max-heap on "worse" = root is the worst kept */
    od_cand* v;
    int32_t n, cap;
} od_heap;

static void od_heap_push(od_heap* h, od_cand c) {
    if (h->cap <= 0) return;
    if (h->n < h->cap) {
        int32_t i = h->n++;
        h->v[i] = c;
        while (i > 0) {
            int32_t p = (i - 1) / 2;
            if (od_better(&h->v[p], &h->v[i])) {
                od_cand tmp = h->v[p];
                h->v[p] = h->v[i];
                h->v[i] = tmp;
                i = p;
            } else
                break;
        }
        return;
    }
    if (!od_better(&c, &h->v[0])) return;
    h->v[0] = c;
    int32_t i = 0;
    for (;;) {
        int32_t l = 2 * i + 1, r = l + 1, w = i;
        if (l < h->n && od_better(&h->v[w], &h->v[l])) w = l;
        if (r < h->n && od_better(&h->v[w], &h->v[r])) w = r;
        if (w == i) break;
        od_cand tmp = h->v[w];
        h->v[w] = h->v[i];
        h->v[i] = tmp;
        i = w;
    }
}

typedef struct od_worker {
    const od_dataset* ds;
    const od_options* opt;
    const od_tables* tab;
    atomic_long* next;
    long total_items;
    od_heap heap;
    uint64_t best_set;
    double best64;
    float best32;
    int has_best;
    uint64_t sets;
    int failed;
} od_worker;

static inline void od_consider(od_worker* w, int32_t order, uint32_t a, uint32_t b, uint32_t c, const int32_t* cs,
                               const int32_t* cn, int32_t ncells) {
    float s32 = od_score32(w->tab, cs, cn, ncells);
    double s64 = od_score64(w->tab, cs, cn, ncells);
    uint64_t set = od_set_key(order, a, b, c);
    od_cand cand = {od_score_key(w->opt->score, s32), set, s32};
    od_heap_push(&w->heap, cand);
    int better;
    if (!w->has_best)
        better = 1;
    else if (w->opt->score == OD_K2)
        better = s64 < w->best64 || (s64 == w->best64 && set < w->best_set);
    else
        better = s64 > w->best64 || (s64 == w->best64 && set < w->best_set);
    if (better) {
        w->has_best = 1;
        w->best64 = s64;
        w->best32 = s32;
        w->best_set = set;
    }
    w->sets++;
}

static void* od_worker2(void* arg) {
    od_worker* w = (od_worker*)arg;
    const od_dataset* ds = w->ds;
    int32_t M = ds->num_snps;
    int32_t cases[9], ctrls[9];
    for (;;) {
        long item = atomic_fetch_add(w->next, 1);
        if (item >= w->total_items) break;
        int32_t a = w->opt->first_begin + (int32_t)item;
        for (int32_t b = a + 1; b < M; ++b) {
            od_table2(ds, a, b, cases, ctrls);
            od_consider(w, 2, (uint32_t)a, (uint32_t)b, 0, cases, ctrls, 9);
        }
    }
    return NULL;
}

/* Per-class scratch of the 3-way worker. */
typedef struct od_cls3 {
    const uint32_t* p;
    int32_t n, W;
    uint32_t* xy4;   /* [4][W]: X_i & Y_j */
    uint32_t* xz9;   /* [M][9] pair counts of X against every Z */
} od_cls3;

static void od_cls3_prepare_x(od_cls3* c, int32_t M, int32_t x) {
    for (int32_t z = x + 1; z < M; ++z) od_pair9(c->p, c->n, x, z, c->xz9 + (size_t)z * 9);
}

/* 8 AND cells X_i&Y_j&Z_k and 4 AND cells Y_j&Z_k for one (X,Y) against Z. */
static void od_cls3_counts(const od_cls3* c, int32_t y, int32_t z, int32_t t8[8], uint32_t yz4[4]) {
    const uint64_t* q = (const uint64_t*)c->xy4;
    int32_t W2 = c->W / 2;
    const uint64_t* y0 = (const uint64_t*)od_row(c->p, c->W, y, 0);
    const uint64_t* y1 = (const uint64_t*)od_row(c->p, c->W, y, 1);
    const uint64_t* z0 = (const uint64_t*)od_row(c->p, c->W, z, 0);
    const uint64_t* z1 = (const uint64_t*)od_row(c->p, c->W, z, 1);
    uint32_t a[8] = {0, 0, 0, 0, 0, 0, 0, 0}, p[4] = {0, 0, 0, 0};
    for (int32_t w = 0; w < W2; ++w) {
        uint64_t Z0 = z0[w], Z1 = z1[w];
        for (int ij = 0; ij < 4; ++ij) {
            uint64_t v = q[(size_t)ij * W2 + w];
            a[ij * 2 + 0] += (uint32_t)od_popc64(v & Z0);
            a[ij * 2 + 1] += (uint32_t)od_popc64(v & Z1);
        }
        p[0] += (uint32_t)od_popc64(y0[w] & Z0);
        p[1] += (uint32_t)od_popc64(y0[w] & Z1);
        p[2] += (uint32_t)od_popc64(y1[w] & Z0);
        p[3] += (uint32_t)od_popc64(y1[w] & Z1);
    }
    for (int i = 0; i < 8; ++i) t8[i] = (int32_t)a[i];
    memcpy(yz4, p, sizeof(p));
}

static void od_cls3_table(const od_cls3* c, int32_t x, int32_t y, int32_t z, const uint32_t xy9[9], int32_t t[27]) {
    int32_t t8[8];
    uint32_t yz4[4];
    (void)x;
    od_cls3_counts(c, y, z, t8, yz4);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) t[C3(i, j, k)] = t8[(i * 2 + j) * 2 + k];
    uint32_t yz9[9] = {yz4[0], yz4[1], 0, yz4[2], yz4[3], 0, 0, 0, 0};
    od_derive27(t, xy9, c->xz9 + (size_t)z * 9, yz9);
}

static void* od_worker3(void* arg) {
    od_worker* w = (od_worker*)arg;
    const od_dataset* ds = w->ds;
    const od_options* o = w->opt;
    int32_t M = ds->num_snps;
    od_cls3 cl[2];
    const uint32_t* planes[2] = {ds->cases, ds->controls};
    int32_t ns[2] = {ds->num_cases, ds->num_controls};
    for (int k = 0; k < 2; ++k) {
        cl[k].p = planes[k];
        cl[k].n = ns[k];
        cl[k].W = od_class_words(ns[k]);
        cl[k].xy4 = (uint32_t*)malloc(sizeof(uint32_t) * 4 * (size_t)cl[k].W);
        cl[k].xz9 = (uint32_t*)malloc(sizeof(uint32_t) * 9 * (size_t)M);
        if (!cl[k].xy4 || !cl[k].xz9) w->failed = 1;
    }
    int32_t cur_x = -1;
    int32_t ylo = o->second_begin, yhi = o->second_end;
    if (yhi <= 0) {
        ylo = 0;
        yhi = M;
    }
    int32_t cases[27], ctrls[27];
    while (!w->failed) {
        long item = atomic_fetch_add(w->next, 1);
        if (item >= w->total_items) break;
        int32_t x = o->first_begin + (int32_t)(item / M);
        int32_t y = (int32_t)(item % M);
        if (y <= x || y < ylo || y >= yhi) continue;
        if (x != cur_x) {
            for (int k = 0; k < 2; ++k) od_cls3_prepare_x(&cl[k], M, x);
            cur_x = x;
        }
        uint32_t xy9[2][9];
        for (int k = 0; k < 2; ++k) {
            od_pair9(cl[k].p, cl[k].n, x, y, xy9[k]);
            int32_t W = cl[k].W;
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j) {
                    const uint32_t* xr = od_row(cl[k].p, W, x, i);
                    const uint32_t* yr = od_row(cl[k].p, W, y, j);
                    uint32_t* d = cl[k].xy4 + (size_t)(i * 2 + j) * W;
                    for (int32_t q = 0; q < W; ++q) d[q] = xr[q] & yr[q];
                }
        }
        for (int32_t z = y + 1; z < M; ++z) {
            od_cls3_table(&cl[0], x, y, z, xy9[0], cases);
            od_cls3_table(&cl[1], x, y, z, xy9[1], ctrls);
            od_consider(w, 3, (uint32_t)x, (uint32_t)y, (uint32_t)z, cases, ctrls, 27);
        }
    }
    for (int k = 0; k < 2; ++k) {
        free(cl[k].xy4);
        free(cl[k].xz9);
    }
    return NULL;
}

static int od_cand_cmp(const void* pa, const void* pb) {
    const od_cand* a = (const od_cand*)pa;
    const od_cand* b = (const od_cand*)pb;
    if (od_better(a, b)) return -1;
    if (od_better(b, a)) return 1;
    return 0;
}

int od_search(const od_dataset* ds, const od_options* opt_in, od_result* res) {
    od_options o = *opt_in;
    int32_t M = ds->num_snps;
    if (M < o.order || ds->num_cases < 1 || ds->num_controls < 1) return 1;
    if (o.first_end <= 0 || o.first_end > M) o.first_end = M;
    if (o.first_begin < 0) o.first_begin = 0;
    if (o.first_begin >= o.first_end) return 1;
    int32_t nthreads = o.threads > 0 ? o.threads : (int32_t)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    od_tables tab;
    if (od_tables_build(o.score, ds->num_cases, ds->num_controls, &tab)) return 2;

    atomic_long next;
    atomic_init(&next, 0);
    long total = (o.order == 2) ? (long)(o.first_end - o.first_begin) : (long)(o.first_end - o.first_begin) * M;
    od_worker* ws = (od_worker*)calloc((size_t)nthreads, sizeof(od_worker));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    int rc = 0;
    for (int32_t i = 0; i < nthreads; ++i) {
        ws[i].ds = ds;
        ws[i].opt = &o;
        ws[i].tab = &tab;
        ws[i].next = &next;
        ws[i].total_items = total;
        ws[i].heap.cap = o.top_k;
        ws[i].heap.v = (od_cand*)malloc(sizeof(od_cand) * (size_t)(o.top_k > 0 ? o.top_k : 1));
        pthread_create(&th[i], NULL, o.order == 2 ? od_worker2 : od_worker3, &ws[i]);
    }
    for (int32_t i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);

    /* merge */
    long allc = 0;
    for (int32_t i = 0; i < nthreads; ++i) allc += ws[i].heap.n;
    od_cand* all = (od_cand*)malloc(sizeof(od_cand) * (size_t)(allc > 0 ? allc : 1));
    long at = 0;
    res->sets = 0;
    res->best_set = 0;
    res->best_fp64 = 0.0;
    res->best_fp32 = 0.0f;
    res->top_count = 0;
    int has = 0;
    for (int32_t i = 0; i < nthreads; ++i) {
        if (ws[i].failed) rc = 2;
        memcpy(all + at, ws[i].heap.v, sizeof(od_cand) * (size_t)ws[i].heap.n);
        at += ws[i].heap.n;
        res->sets += ws[i].sets;
        if (ws[i].has_best) {
            int better;
            if (!has)
                better = 1;
            else if (o.score == OD_K2)
                better = ws[i].best64 < res->best_fp64 ||
                         (ws[i].best64 == res->best_fp64 && ws[i].best_set < res->best_set);
            else
                better = ws[i].best64 > res->best_fp64 ||
                         (ws[i].best64 == res->best_fp64 && ws[i].best_set < res->best_set);
            if (better) {
                has = 1;
                res->best_fp64 = ws[i].best64;
                res->best_fp32 = ws[i].best32;
                res->best_set = ws[i].best_set;
            }
        }
        free(ws[i].heap.v);
    }
    qsort(all, (size_t)allc, sizeof(od_cand), od_cand_cmp);
    int32_t k = (int32_t)(allc < o.top_k ? allc : o.top_k);
    for (int32_t i = 0; i < k; ++i) {
        if (res->top_sets) res->top_sets[i] = all[i].set;
        if (res->top_fp32) res->top_fp32[i] = all[i].s32;
        if (res->top_fp64) {
            uint32_t idx[3];
            od_set_unkey(o.order, all[i].set, idx);
            if (o.order == 2) {
                int32_t cs[9], cn[9];
                od_table2(ds, (int32_t)idx[0], (int32_t)idx[1], cs, cn);
                res->top_fp64[i] = od_score64(&tab, cs, cn, 9);
            } else {
                int32_t cs[27], cn[27];
                od_table3(ds, (int32_t)idx[0], (int32_t)idx[1], (int32_t)idx[2], cs, cn);
                res->top_fp64[i] = od_score64(&tab, cs, cn, 27);
            }
        }
    }
    res->top_count = k;
    free(all);
    free(ws);
    free(th);
    od_tables_free(&tab);
    return rc;
}

int32_t od_split_by_label(const uint32_t* planes, int32_t M, int32_t n, const uint32_t* label, uint32_t* cases_out,
                          uint32_t* controls_out, int32_t* num_controls) {
    int32_t W = od_class_words(n);
    int32_t nc = 0;
    for (int32_t s = 0; s < n; ++s) nc += (label[s / 32] >> (31 - s % 32)) & 1u;
    int32_t nn = n - nc;
    int32_t Wc = od_class_words(nc > 0 ? nc : 1), Wn = od_class_words(nn > 0 ? nn : 1);
    memset(cases_out, 0, sizeof(uint32_t) * (size_t)M * 2 * (size_t)Wc);
    memset(controls_out, 0, sizeof(uint32_t) * (size_t)M * 2 * (size_t)Wn);
    for (int32_t snp = 0; snp < M; ++snp)
        for (int32_t g = 0; g < 2; ++g) {
            const uint32_t* r = od_row(planes, W, snp, g);
            uint32_t* rc = cases_out + ((size_t)snp * 2 + (size_t)g) * (size_t)Wc;
            uint32_t* rn = controls_out + ((size_t)snp * 2 + (size_t)g) * (size_t)Wn;
            int32_t ic = 0, in = 0;
            for (int32_t s = 0; s < n; ++s) {
                uint32_t bit = (r[s / 32] >> (31 - s % 32)) & 1u;
                if ((label[s / 32] >> (31 - s % 32)) & 1u) {
                    rc[ic / 32] |= bit << (31 - ic % 32);
                    ++ic;
                } else {
                    rn[in / 32] |= bit << (31 - in % 32);
                    ++in;
                }
            }
        }
    if (num_controls) *num_controls = nn;
    return nc;
}

/* ------------------------------------------------------------------------
 * Synthetic datasets, generated here so that a process timing the oracle
 * (the CPU baseline, the reference arm of bench.py) never loads the product
 * library.  Bit-identical to episdet_generate by construction: the same
 * counter-based draws (the SplitMix64 finaliser of Steele, Lea & Flood 2014
 * applied to (seed, stream, index)), the same Hardy-Weinberg thresholds and
 * the same penetrance model, so tests can check the two against each other.
 * ---------------------------------------------------------------------- */
static uint64_t od_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t od_draw(uint64_t seed, uint64_t stream, uint64_t idx) {
    return od_mix64(od_mix64(seed ^ od_mix64(stream)) ^ idx);
}
static double od_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

#define OD_TAG_MAF 0x4D4146ull
#define OD_TAG_GENO (0x47454E4Full << 24)
#define OD_TAG_LABEL 0x4C4142ull

static int od_genotype(uint64_t seed, int32_t snp, uint64_t ind, double p) {
    double u = od_u01(od_draw(seed, OD_TAG_GENO + (uint64_t)snp, ind));
    double q0 = (1.0 - p) * (1.0 - p);
    if (u < q0) return 0;
    if (u < 1.0 - p * p) return 1;
    return 2;
}

typedef struct od_fill_arg {
    uint64_t seed;
    int32_t M, n, t, nt;
    const double* maf;
    const uint64_t* ids;
    uint32_t* planes;
} od_fill_arg;

static void* od_fill_worker(void* p) {
    od_fill_arg* a = (od_fill_arg*)p;
    size_t W = (size_t)od_class_words(a->n);
    for (int32_t snp = a->t; snp < a->M; snp += a->nt) {
        uint32_t* r0 = a->planes + ((size_t)snp * 2) * W;
        uint32_t* r1 = r0 + W;
        memset(r0, 0, sizeof(uint32_t) * 2 * W);
        for (int32_t s = 0; s < a->n; ++s) {
            int g = od_genotype(a->seed, snp, a->ids[s], a->maf[snp]);
            if (g < 2) (g == 0 ? r0 : r1)[s / 32] |= 1u << (31 - s % 32);
        }
    }
    return NULL;
}

static int od_fill(uint64_t seed, int32_t M, const double* maf, const uint64_t* ids, int32_t n, uint32_t* planes,
                   int threads) {
    int nt = threads > 0 ? threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > 256) nt = 256;
    pthread_t th[256];
    od_fill_arg args[256];
    for (int i = 0; i < nt; ++i) {
        args[i] = (od_fill_arg){seed, M, n, i, nt, maf, ids, planes};
        if (pthread_create(&th[i], NULL, od_fill_worker, &args[i]) != 0) {
            for (int j = 0; j < i; ++j) pthread_join(th[j], NULL);
            return -1;
        }
    }
    for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
    return 0;
}

int od_generate(const od_synth* sp, uint32_t* cases, uint32_t* controls, int threads) {
    if (!sp || !cases || !controls || sp->num_snps < 1 || sp->num_cases < 1 || sp->num_controls < 1 ||
        sp->num_planted < 0 || sp->num_planted > 2 || !(sp->maf_min >= 0.0f) || !(sp->maf_max <= 0.5f) ||
        sp->maf_min > sp->maf_max)
        return -1;
    const int32_t M = sp->num_snps;
    const int ord = sp->planted_order == 2 ? 2 : 3;
    double* maf = (double*)malloc(sizeof(double) * (size_t)M);
    uint64_t* cid = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)sp->num_cases);
    uint64_t* nid = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)sp->num_controls);
    int rc = 0;
    if (!maf || !cid || !nid) {
        rc = -2;
        goto out;
    }
    for (int32_t s = 0; s < M; ++s)
        maf[s] = (double)sp->maf_min + ((double)sp->maf_max - (double)sp->maf_min) * od_u01(od_draw(sp->seed, OD_TAG_MAF, (uint64_t)s));
    for (int q = 0; q < sp->num_planted; ++q)
        for (int e = 0; e < ord; ++e) {
            int32_t s = sp->planted[q][e];
            if (s < 0 || s >= M) {
                rc = -1;
                goto out;
            }
            if (sp->planted_maf > 0.0f) maf[s] = (double)sp->planted_maf;
        }
    int32_t nc = 0, nn = 0;
    if (sp->num_planted == 0) {
        for (int32_t i = 0; i < sp->num_cases; ++i) cid[nc++] = (uint64_t)i;
        for (int32_t i = 0; i < sp->num_controls; ++i) nid[nn++] = (uint64_t)(sp->num_cases + i);
    } else {
        uint64_t ind = 0;
        const uint64_t limit = 64ull * (uint64_t)(sp->num_cases + sp->num_controls) + 1000000ull;
        while (nc < sp->num_cases || nn < sp->num_controls) {
            if (ind > limit) {
                rc = -1;
                goto out;
            }
            double risk = (double)sp->base_risk;
            for (int q = 0; q < sp->num_planted; ++q) {
                int carried = 1;
                for (int e = 0; e < ord; ++e) {
                    int32_t s = sp->planted[q][e];
                    carried = carried && od_genotype(sp->seed, s, ind, maf[s]) >= 1;
                }
                if (carried) risk += (double)sp->effect;
            }
            int is_case = od_u01(od_draw(sp->seed, OD_TAG_LABEL, ind)) < risk;
            if (is_case && nc < sp->num_cases) cid[nc++] = ind;
            if (!is_case && nn < sp->num_controls) nid[nn++] = ind;
            ++ind;
        }
    }
    if (od_fill(sp->seed, M, maf, cid, sp->num_cases, cases, threads) != 0 ||
        od_fill(sp->seed, M, maf, nid, sp->num_controls, controls, threads) != 0)
        rc = -3;
out:
    free(maf);
    free(cid);
    free(nid);
    return rc;
}
