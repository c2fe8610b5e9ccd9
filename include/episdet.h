/*
 * episdet.h -- C-ABI of the B200 epistasis-search library (libepisdet.so).
 *
 * Exhaustive 2-way / 3-way epistasis detection over binarized genotype bit
 * planes, K2 or mutual-information scoring, best set by an FP64 re-score.
 *
 * Every entry point replaces one role of hiperbio/tensor-episdet:
 *   episdet_search          <- EpistasisDetectionSearch(), src/search-pairs.cu:9
 *                              and src/search-triplets.cu:8 (declared in
 *                              include/search-pairs.hpp:4, search-triplets.hpp:4);
 *                              the order (pairs/triplets) and score (K2/MI),
 *                              fixed at build time there by -DTRIPLETS and
 *                              -DMI_SCORE (Makefile:8-22), are options here.
 *   episdet_search_batched  <- no counterpart (one dataset per process there,
 *                              src/tensor-episdet.cu:159-172); many cohorts,
 *                              run concurrently, in one call.
 *   episdet_search_perm     <- no counterpart (one label vector there); many
 *                              phenotype permutations of one cohort.
 *   episdet_read_dataset    <- the descriptor/.bin loader of
 *                              src/tensor-episdet.cu:58-148.
 *   episdet_n_choose_k      <- n_choose_k(), src/helper.cu:758-768.
 *
 * Data format (unchanged from the reference, src/tensor-episdet.cu:111-148,
 * include/helper.hpp:10-25): one uint32 array per class laid out
 * [SNP][genotype g in {0,1}][W] with W = ceil(n/1024)*32 words; sample s of a
 * row sits in word s/32 at bit 31 - s%32.  Genotype 2 is implied (neither
 * plane set).  Padding bits must be zero and the two planes of a row must be
 * disjoint; inputs that break this are rejected with EPISDET_ERR_INVALID_INPUT
 * (the reference silently produced undefined counts for them).
 *
 * Errors: every call returns an episdet_status; episdet_last_error() gives a
 * thread-local message for the last failure.  No call exits or traps.
 */
#ifndef EPISDET_H_
#define EPISDET_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPISDET_ABI_VERSION 1

typedef enum episdet_status {
    EPISDET_OK = 0,
    EPISDET_ERR_INVALID_ARGUMENT = 1, /* bad sizes, null pointers, unknown option */
    EPISDET_ERR_INVALID_INPUT = 2,    /* padding bits set or genotype planes overlap */
    EPISDET_ERR_NO_DEVICE = 3,        /* no usable sm_100 device */
    EPISDET_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    EPISDET_ERR_OUT_OF_MEMORY = 5,
    EPISDET_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
    EPISDET_ERR_IO = 7,               /* descriptor or .bin file problem */
    EPISDET_ERR_UNSUPPORTED = 8,
    EPISDET_ERR_INTERNAL = 9
} episdet_status;

enum { EPISDET_SCORE_K2 = 0, EPISDET_SCORE_MI = 1 };
enum { EPISDET_HOST = 0, EPISDET_DEVICE = 1 };

/* Counting engine.  AUTO picks the tcgen05 tensor-core path. */
enum { EPISDET_ENGINE_AUTO = 0, EPISDET_ENGINE_TENSOR = 1, EPISDET_ENGINE_SIMT = 2 };

/* options.flags */
#define EPISDET_FLAG_PROGRESS 0x1u     /* print the reference's "Outer loop iteration" lines */
#define EPISDET_FLAG_NO_VALIDATE 0x2u  /* skip the padding / plane-overlap check */
#define EPISDET_FLAG_TIMING 0x4u       /* time every counting-kernel launch (result.count_kernel_ms) */
/* Pick the triplet kernel instance for this shape by measurement: the first
 * search of a shape (order, score, log2 of the smaller class) times the plain
 * and the segment-staging instance on the first 8 first SNPs of its own data
 * and keeps the faster; the choice is cached for the process and, when the
 * environment variable EPISDET_TUNE_CACHE names a file, read from and appended
 * to it.  Without the flag the instance follows a fixed rule (staging from
 * classes of 32,768 samples).  Results are the same either way. */
#define EPISDET_FLAG_AUTOTUNE 0x8u
/* Testing aid for failure detection: the tensor engine's scoring warps first
 * wait for a device word that nothing ever sets, so every counting launch
 * gives up after wait_limit_ms, drains its copies and MMAs, frees its tensor
 * memory and returns; the call then fails with EPISDET_ERR_TIMEOUT and the
 * device stays usable for the next call. */
#define EPISDET_FLAG_INJECT_STALL 0x10u
/* K2 triplet searches on the tensor engine bound each set's score without
 * table reads and score exactly only the sets that can still enter the top-k
 * list (same results either way).  By default this runs when every CTA scores
 * far more sets than its candidate list holds (about 1.5e9 sets in the
 * search); these flags force it on or off. */
#define EPISDET_FLAG_FILTER_ON 0x20u
#define EPISDET_FLAG_FILTER_OFF 0x40u
/* episdet_search_perm with order 2 on the tensor engine counts, per label,
 * only the cases' AND cells (the label as a third AND operand, by regrouping
 * the case samples) and derives the controls' cells from the label-free
 * pair counts, computed once per call.  This flag runs each label as a plain
 * two-class search instead (same results). */
#define EPISDET_FLAG_PERM_SPLIT 0x80u

/* One cohort split into cases and controls (the reference's two .bin files). */
typedef struct episdet_dataset {
    const uint32_t* cases;    /* [num_snps][2][episdet_class_words(num_cases)] */
    const uint32_t* controls; /* [num_snps][2][episdet_class_words(num_controls)] */
    int32_t num_snps;         /* M >= order, M <= 2^21 - 1 */
    int32_t num_cases;        /* >= 1 */
    int32_t num_controls;     /* >= 1 */
    int32_t memory;           /* EPISDET_HOST or EPISDET_DEVICE (current device) */
} episdet_dataset;

/* One cohort without a class split (all samples as one plane set). */
typedef struct episdet_cohort {
    const uint32_t* planes;   /* [num_snps][2][episdet_class_words(num_samples)] */
    int32_t num_snps;
    int32_t num_samples;
    int32_t memory;
} episdet_cohort;

typedef struct episdet_options {
    int32_t order;        /* 2 (pairs) or 3 (triplets) */
    int32_t score;        /* EPISDET_SCORE_K2 (minimised) or EPISDET_SCORE_MI (maximised) */
    int32_t top_k;        /* FP32 candidates re-scored in FP64; 1..1536, default 1024 */
    int32_t device;       /* CUDA device ordinal, default 0 */
    int32_t engine;       /* EPISDET_ENGINE_* */
    int32_t first_begin;  /* evaluate only sets whose first SNP is in [first_begin, first_end) */
    int32_t first_end;    /* 0 -> num_snps */
    uint32_t flags;       /* EPISDET_FLAG_* */
    uint64_t stream;      /* cudaStream_t to run on; 0 = the library's own stream */
    /* Longest time one in-kernel wait of the tensor engine (for an operand
     * copy, an MMA commit, the scoring warps) may take before the launch gives
     * up and the call returns EPISDET_ERR_TIMEOUT; 0 = 4000 ms. */
    int32_t wait_limit_ms;
    /* 3-way tensor engine: SNP rows of the Y-Z pair table held in device
     * memory at once (rounded up to a multiple of 128).  0 = automatic: the
     * whole table (32 x num_snps^2 bytes) when it fits beside the engine's
     * other buffers, else the largest block that fits; the search then runs
     * one pass per block of second SNPs Y (as the reference keeps its pair
     * counts per 256-SNP Y block, src/search-triplets.cu:173-176), with the
     * same results. */
    int32_t pair_block_snps;
    int32_t reserved[4];
} episdet_options;

typedef struct episdet_result {
    uint32_t snps[3];         /* best set (FP64 re-score, lowest index on ties); snps[2] = 0 for pairs */
    uint64_t packed_indices;  /* reference packing: pairs a|b<<32 (src/helper.cu:690),
                                 triplets x|y<<21|z<<42 (src/helper.cu:576) */
    double score;             /* FP64 score of the best set */
    float score_fp32;         /* FP32 epilogue score of the same set */
    int32_t top_count;        /* entries written to top_* */
    int64_t sets_evaluated;   /* C(M,k) restricted to the first_begin/end slab */
    int64_t rounds;           /* reference block-round count (BLOCK_SIZE 256) */
    double seconds;           /* wall time of the call (the reference's searchTime) */
    double device_ms;         /* device time of the counting+scoring launches */
    uint64_t kernel_launches; /* kernels this call launched */
    double count_kernel_ms;   /* EPISDET_FLAG_TIMING: summed device time of the counting launches */
    int64_t count_kernel_launches; /* launches of the counting kernel */
    double executed_macs;     /* EPISDET_FLAG_TIMING: MACs the tensor engine issued (u8 for pairs and the
                                 pair table, e2m1 for triplets; 0 for SIMT) */
    int64_t h2d_bytes;        /* host->device bytes this call copied */
    int64_t d2h_bytes;        /* device->host bytes this call copied */
    /* Optional caller-owned outputs of capacity top_capacity (may be NULL). */
    int32_t top_capacity;
    uint32_t* top_snps;       /* [top_capacity][3] in FP32 rank order */
    float* top_fp32;
    double* top_fp64;
} episdet_result;

/* Words per genotype plane row for a class of n samples: ceil(n/1024)*32. */
int32_t episdet_class_words(int32_t num_samples);

void episdet_default_options(episdet_options* opts);

/* Replaces EpistasisDetectionSearch (src/search-pairs.cu:9, src/search-triplets.cu:8). */
episdet_status episdet_search(const episdet_dataset* data, const episdet_options* opts, episdet_result* result);

/* Many independent cohorts (uneven SNP and sample counts) in one call: up to
 * four run at a time, largest first, each on its own library stream and
 * buffers, so one cohort's small launches share the GPU with the others'.
 * opts[i] gives cohort i's order/score (leave options.stream 0: cohorts on one
 * caller stream cannot overlap); results[i] receives exactly the answer
 * episdet_search would give.  The first failing cohort's error is returned,
 * naming the cohort. */
episdet_status episdet_search_batched(const episdet_dataset* cohorts, const episdet_options* opts, int32_t count,
                                      episdet_result* results);

/* Phenotype permutations of one cohort: labels is [num_labels][class_words(num_samples)],
 * bit = 1 marks a case.  results[i] is the best pair/triplet under label i. */
episdet_status episdet_search_perm(const episdet_cohort* cohort, const uint32_t* labels, int32_t num_labels,
                                   const episdet_options* opts, episdet_result* results);

/* Permutation significance -- no counterpart in the reference, which prints
 * one best set (src/tensor-episdet.cu:181-185).  results[0] is the search
 * under the observed labels, results[1..num_labels-1] under permuted ones (as
 * episdet_search_perm returns them).  Single-step max-statistic adjusted
 * p-values (Westfall-Young): for a set with FP64 score s,
 *   p = (1 + #{i >= 1 : results[i].score at least as extreme as s}) / num_labels,
 * "at least as extreme" meaning <= s for K2 (minimised) and >= s for MI.
 * pvalues[j] is the p-value of entry j of results[0]'s top list when it has
 * one (top_count > 0, top_fp64 set), else pvalues[0] is the best set's;
 * *count receives the number written (at most capacity). */
episdet_status episdet_perm_pvalues(const episdet_result* results, int32_t num_labels, int32_t score,
                                    double* pvalues, int32_t capacity, int32_t* count);

/* Resumable search -- a checkpoint cursor for long runs; no counterpart in
 * the reference.  The first-SNP range of opts is searched in num_slabs slabs
 * of about equal work (episdet_search with first_begin/first_end); after each
 * slab the merged top_k candidate list (sets, FP32 and FP64 scores) and the
 * cursor (next first SNP) are written to `path` (a temporary file renamed
 * over it, so an interrupted call leaves the previous checkpoint).  A call
 * that finds a checkpoint of the same search (same sizes, options and plane
 * contents, by a 64-bit fingerprint) continues from its cursor; one of another
 * search is refused with EPISDET_ERR_INVALID_ARGUMENT.  Merging the slabs'
 * top_k lists by (FP32 score, set) gives exactly the list of one uninterrupted
 * search, so the final result is the same. */
typedef struct episdet_resume {
    const char* path;       /* checkpoint file */
    int32_t num_slabs;      /* slabs over the whole first-SNP range; 0 -> 16 */
    int32_t max_slabs;      /* > 0: return after this many slabs (done = 0 if work remains) */
    int32_t done;           /* out: 1 when the search is complete and `result` holds its answer */
    int32_t next_first;     /* out: the cursor, first SNP of the next slab */
    int32_t slabs_run;      /* out: slabs searched by this call */
    int32_t reserved[3];
} episdet_resume;
episdet_status episdet_search_resumable(const episdet_dataset* data, const episdet_options* opts,
                                        episdet_resume* resume, episdet_result* result);

/* Reads the reference's 5-line dataset descriptor and its two .bin files
 * (src/tensor-episdet.cu:58-148) into malloc'd arrays; free with episdet_free_dataset. */
episdet_status episdet_read_dataset(const char* descriptor_path, episdet_dataset* out);
void episdet_free_dataset(episdet_dataset* data);

/* Writes a dataset in the reference's format: descriptor + <stem>.cases.bin + <stem>.controls.bin. */
episdet_status episdet_write_dataset(const char* descriptor_path, const episdet_dataset* data);

/* Genotype matrix -> the reference's per-class bit planes, on the GPU.  No
 * counterpart in the reference, which reads pre-binarized .bin files
 * (README.md:48-50).  genotypes: [num_snps][num_samples] bytes, each 0, 1 or 2;
 * is_case: [num_samples] bytes, non-zero marks a case.  cases / controls:
 * [num_snps][2][episdet_class_words(n)] words for the n cases / controls in
 * sample order (planes of genotypes 0 and 1, MSB first, zero padding).  All
 * four arrays live in `memory` (EPISDET_HOST arrays pass through the device).
 * A genotype above 2 returns EPISDET_ERR_INVALID_INPUT; a class left empty
 * returns EPISDET_ERR_INVALID_ARGUMENT. */
episdet_status episdet_binarize(const uint8_t* genotypes, int32_t num_snps, int32_t num_samples,
                                const uint8_t* is_case, uint32_t* cases, uint32_t* controls, int32_t memory,
                                int32_t device);

/* Seeded synthetic data (Hardy-Weinberg genotypes, optional planted sets).
 * planted: up to 2 sets of `order` SNP indices (flat array, -1 terminated or
 * num_planted sets); penetrance: P(case) = base, or base + effect for each
 * planted set whose SNPs all carry a minor allele. */
typedef struct episdet_synth {
    uint64_t seed;
    int32_t num_snps;
    int32_t num_cases;
    int32_t num_controls;
    float maf_min, maf_max;     /* minor-allele frequency ~ U[maf_min, maf_max] */
    int32_t num_planted;        /* 0, 1 or 2 planted sets */
    int32_t planted_order;      /* 2 or 3 */
    int32_t planted[2][3];
    float planted_maf;          /* > 0: fixed MAF for planted SNPs */
    float base_risk;            /* P(case) baseline, e.g. 0.5 */
    float effect;               /* added per planted set carried, e.g. 0.25 */
} episdet_synth;

/* Fills caller-allocated host arrays sized for the reference format. */
episdet_status episdet_generate(const episdet_synth* spec, uint32_t* cases, uint32_t* controls);
/* One plane set over num_samples individuals with independent labels. */
episdet_status episdet_generate_cohort(uint64_t seed, int32_t num_snps, int32_t num_samples, float maf_min,
                                       float maf_max, uint32_t* planes);
/* num_labels label vectors; vector 0 has exactly num_cases cases (the first
 * num_cases individuals), the others are seeded random permutations of it. */
episdet_status episdet_generate_labels(uint64_t seed, int32_t num_samples, int32_t num_cases, int32_t num_labels,
                                       uint32_t* labels);

/* The cached EPISDET_FLAG_AUTOTUNE choice for a shape: 1 = segment-staging
 * triplet instance, 0 = plain instance, -1 = not tuned yet. */
int32_t episdet_tuned_stage(int32_t order, int32_t score, int32_t num_cases, int32_t num_controls);

uint64_t episdet_n_choose_k(uint32_t n, uint32_t k);
const char* episdet_status_string(episdet_status s);
const char* episdet_last_error(void);
int32_t episdet_abi_version(void);

/* Frees the per-device workspace the library keeps between calls. */
episdet_status episdet_release_workspace(int32_t device);

/* Profiling aid -- no counterpart in the reference: after an episdet_search
 * with EPISDET_FLAG_TIMING on `device`, the device time (ms, CUDA events on
 * the launching stream) and the tensor MACs issued of each counting launch, in
 * launch order (at most cap entries each; either pointer may be NULL).
 * Returns the number of counting launches of that search (0 without the flag). */
int64_t episdet_last_launch_profile(int32_t device, double* ms, double* macs, int64_t cap);

/* Testing aid for failure detection -- no counterpart in the reference: the
 * after-th device allocation the library makes from now on (in any thread)
 * fails as if the device were out of memory, once; the call that needed it
 * returns EPISDET_ERR_OUT_OF_MEMORY and later calls allocate normally.
 * after <= 0 disarms it. */
void episdet_test_fail_allocation(int32_t after);

/* Pairs search that allocates nothing -- no counterpart in the reference.
 * For callers that cannot let a library allocate device memory: a process
 * whose memory pool or caching allocator already holds the GPU's memory, or a
 * pipeline that cannot take the device-wide synchronisation of cudaFree.
 * Same results as episdet_search with order 2 (the same best pair, candidate
 * list and FP32 / FP64 scores), computed by the integer-pipe (LOP3 + POPC)
 * pairs kernel rather than the tensor-core one, with every intermediate
 * buffer in one fixed 8 MiB device array that the library holds on each GPU
 * that loads it until the process exits.  Limits (beyond them the call
 * returns EPISDET_ERR_INVALID_ARGUMENT): data->memory must be EPISDET_DEVICE,
 * at most 4096 SNPs, 131072 samples (cases + controls) and top_k 1024.  The
 * first call on a device looks up the array's address and should come before
 * any stream capture; after a cudaDeviceReset of that device the entry point
 * must not be called again in the process.  Calls share the array: they are
 * serialised by a host lock and each waits for its GPU work before returning,
 * failed calls included, since GPU work of two calls that overlapped would
 * race on it. */
episdet_status episdet_search_pairs_noalloc(const episdet_dataset* data, const episdet_options* opts,
                                            episdet_result* result);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
/* Reference-compatible entry point (C++ linkage, cudaError_t return), one
 * variant per link: libepisdet_compat_{pairs,triplets}_{k2,mi}.a defines
 *   cudaError_t EpistasisDetectionSearch(unsigned int* cases, unsigned int* controls,
 *       int numSNPs, int numCases, int numControls, uint numSNPsWithPadding,
 *       int numCasesWithPadding, int numControlsWithPadding, int* roundsCounter,
 *       double* searchTime, float* outputFromGpu, unsigned long long* packedIndices);
 * with the semantics of src/search-pairs.cu:9 / src/search-triplets.cu:8. */
#endif

#endif /* EPISDET_H_ */
