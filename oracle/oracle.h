/*
 * oracle.h -- CPU restatement of tensor-episdet's contingency-table and
 * scoring path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product (libepisdet.so and the four CLIs) never links or calls it.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors and
 * its GEMM lives in an absent third-party library (CUTLASS 1.3.x), so this
 * oracle is pinned only by the project's own known-answer tests (hand-built
 * tables, planted sets, algebraic invariants).  Parity unpinned against the
 * reference binary itself.
 *
 * Data format (reference include/helper.hpp:10-25, src/tensor-episdet.cu:111-148):
 * one array per class, [SNP][genotype g in {0,1}][W] uint32 words, W =
 * ceil(n/1024)*32.  Sample s sits in word s/32 at bit 31 - s%32 (MSB first:
 * the padding mask in src/helper.cu:72-73 clears the low bits of the last
 * word).  Genotype 2 is not stored.
 */
#ifndef EPISDET_ORACLE_H_
#define EPISDET_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OD_K2 = 0, OD_MI = 1 };

typedef struct od_dataset {
    const uint32_t* cases;     /* [M][2][Wc] */
    const uint32_t* controls;  /* [M][2][Wn] */
    int32_t num_snps;          /* M */
    int32_t num_cases;
    int32_t num_controls;
} od_dataset;

/* Score tables shared by the FP32 and FP64 scorers. */
typedef struct od_tables {
    int32_t score;        /* OD_K2 or OD_MI */
    int32_t num_cases, num_controls;
    int32_t size;         /* entries in t32 / t64 */
    float* t32;           /* K2: lnG(v+1); MI: log2(v/N) (index 0 -> 0) */
    double* t64;
    float inv_n32;        /* MI: (float)(1.0/N) */
    double inv_n64;       /* MI: 1.0/N */
    float hy32;           /* MI: class entropy H(Y) in the FP32 score's own evaluation order */
    double hy64;
} od_tables;

typedef struct od_options {
    int32_t order;        /* 2 or 3 */
    int32_t score;        /* OD_K2 / OD_MI */
    int32_t top_k;        /* size of the FP32 candidate list kept */
    int32_t threads;      /* worker threads (<=0: all online cores) */
    int32_t first_begin;  /* restrict the first SNP index of a set to [begin,end) */
    int32_t first_end;    /* 0 -> num_snps */
    int32_t second_begin; /* 3-way only: restrict Y to [begin,end) (0,0 -> all) */
    int32_t second_end;
} od_options;

typedef struct od_result {
    /* FP32 candidate list in rank order (best first); caller-owned, capacity top_k */
    uint64_t* top_sets;   /* lexicographic key, see od_set_key */
    float* top_fp32;
    double* top_fp64;
    int32_t top_count;
    /* FP64 optimum over every evaluated set; ties go to the lowest key */
    uint64_t best_set;
    double best_fp64;
    float best_fp32;
    uint64_t sets;        /* sets evaluated */
} od_result;

/* Lexicographic set key: pairs (a<<32)|b, triplets (x<<42)|(y<<21)|z. */
uint64_t od_set_key(int order, uint32_t a, uint32_t b, uint32_t c);
void od_set_unkey(int order, uint64_t key, uint32_t out[3]);

/* helper.cu:13-52: per-SNP genotype counts, out[g*M + snp], g2 = n - g0 - g1. */
void od_marginals(const uint32_t* planes, int32_t M, int32_t n, uint32_t* out);

/* Returns 0 when every row has zero padding bits and disjoint genotype planes. */
int od_validate(const uint32_t* planes, int32_t M, int32_t n);

/* helper.cu:58-194 (genotype-2 plane ~(g0|g1) masked to n samples): 9 pair
 * counts, out[ga*3+gb]. */
void od_pair9(const uint32_t* planes, int32_t n, int32_t a, int32_t b, uint32_t out[9]);

/* helper.cu:634-662: 2-way table, 4 AND cells + 5 derived from marginals. */
void od_table2(const od_dataset* ds, int32_t a, int32_t b, int32_t cases[9], int32_t controls[9]);

/* helper.cu:480-548 + include/helper.hpp:34-51: 3-way table, 8 AND cells +
 * 19 cells derived from pair tables. */
void od_table3(const od_dataset* ds, int32_t x, int32_t y, int32_t z, int32_t cases[27], int32_t controls[27]);

int od_tables_build(int32_t score, int32_t num_cases, int32_t num_controls, od_tables* t);
void od_tables_free(od_tables* t);

/* include/scoring.hpp:5-90 with the intended table range (see .c). */
float od_score32(const od_tables* t, const int32_t* cases, const int32_t* controls, int32_t ncells);
double od_score64(const od_tables* t, const int32_t* cases, const int32_t* controls, int32_t ncells);

/* Orderable 32-bit key of an FP32 score (smaller = better for both scores). */
uint32_t od_score_key(int32_t score, float s);

/* Exhaustive search (src/search-pairs.cu:137-215, src/search-triplets.cu:162-273). */
int od_search(const od_dataset* ds, const od_options* opt, od_result* res);

/* Splits one single-class plane set [M][2][Wall] by a label bit vector
 * (bit = 1 -> case) into reference-format case/control arrays (caller-owned,
 * sized with od_class_words). Returns the number of cases. */
int32_t od_split_by_label(const uint32_t* planes, int32_t M, int32_t n, const uint32_t* label,
                          uint32_t* cases_out, uint32_t* controls_out, int32_t* num_controls);
int32_t od_class_words(int32_t n);

/* Seeded synthetic dataset in the reference format (the generator of the
 * product library, restated here so that oracle-only processes need no other
 * library): Hardy-Weinberg genotypes with MAF ~ U[maf_min, maf_max] per SNP,
 * optional planted sets with penetrance base_risk + effect per set carried
 * (all SNPs of the set with >= 1 minor allele), individuals drawn in order and
 * kept while their class has room.  threads <= 0: all online cores. */
typedef struct od_synth {
    uint64_t seed;
    int32_t num_snps, num_cases, num_controls;
    float maf_min, maf_max;
    int32_t num_planted, planted_order;
    int32_t planted[2][3];
    float planted_maf, base_risk, effect;
} od_synth;
int od_generate(const od_synth* spec, uint32_t* cases, uint32_t* controls, int threads);

#ifdef __cplusplus
}
#endif
#endif
