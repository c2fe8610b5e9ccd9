// compat.cpp -- the reference's EpistasisDetectionSearch() on top of the C-ABI.
//
// Built four times (EPISDET_COMPAT_ORDER = 2|3, EPISDET_COMPAT_SCORE = 0|1)
// into libepisdet_compat_{pairs,triplets}_{k2,mi}.a, exactly as the reference
// links one of src/search-pairs.cu / src/search-triplets.cu per binary and
// picks K2 or MI with -DMI_SCORE (Makefile:8-22).  Signature and output
// semantics: include/search-pairs.hpp:4, src/search-pairs.cu:9-246.
#include <cuda_runtime.h>

#include <cstdio>

#include "episdet.h"

#ifndef EPISDET_COMPAT_ORDER
#define EPISDET_COMPAT_ORDER 3
#endif
#ifndef EPISDET_COMPAT_SCORE
#define EPISDET_COMPAT_SCORE EPISDET_SCORE_K2
#endif

// The reference's main prints C(numSNPs, k) through n_choose_k (declared at
// include/helper.hpp:76, defined with its kernels at src/helper.cu:758-768).
// A main linked against this shim without src/helper.cu finds it here; weak,
// so a build that keeps src/helper.cu uses that one.
__attribute__((weak)) unsigned long long n_choose_k(unsigned int n, unsigned int k) {
    return (unsigned long long)episdet_n_choose_k(n, k);
}

cudaError_t EpistasisDetectionSearch(unsigned int* datasetCases, unsigned int* datasetControls, int numSNPs,
                                     int numCases, int numControls, unsigned int numSNPsWithPadding,
                                     int numCasesWithPadding, int numControlsWithPadding, int* roundsCounter,
                                     double* searchTime, float* outputFromGpu, unsigned long long* packedIndices) {
    // The padded sizes are implied by the format; reject inconsistent ones.
    if (numCases < 1 || numControls < 1 || numCasesWithPadding != episdet_class_words(numCases) * 32 ||
        numControlsWithPadding != episdet_class_words(numControls) * 32 || numSNPsWithPadding < (unsigned)numSNPs) {
        fprintf(stderr, "EpistasisDetectionSearch: inconsistent padded sizes\n");
        return cudaErrorInvalidValue;
    }
    episdet_dataset d;
    d.cases = datasetCases;
    d.controls = datasetControls;
    d.num_snps = numSNPs;
    d.num_cases = numCases;
    d.num_controls = numControls;
    d.memory = EPISDET_HOST;
    episdet_options o;
    episdet_default_options(&o);
    o.order = EPISDET_COMPAT_ORDER;
    o.score = EPISDET_COMPAT_SCORE;
    o.flags = EPISDET_FLAG_PROGRESS;
    episdet_result r = {};
    episdet_status s = episdet_search(&d, &o, &r);
    if (s != EPISDET_OK) {
        fprintf(stderr, "%s: %s\n", episdet_status_string(s), episdet_last_error());
        switch (s) {
            case EPISDET_ERR_OUT_OF_MEMORY: return cudaErrorMemoryAllocation;
            case EPISDET_ERR_NO_DEVICE: return cudaErrorNoDevice;
            case EPISDET_ERR_INVALID_ARGUMENT:
            case EPISDET_ERR_INVALID_INPUT: return cudaErrorInvalidValue;
            default: return cudaErrorUnknown;
        }
    }
    *roundsCounter = (int)r.rounds;
    *searchTime = r.seconds;
    *outputFromGpu = (float)r.score;
    *packedIndices = (unsigned long long)r.packed_indices;
    return cudaSuccess;
}
