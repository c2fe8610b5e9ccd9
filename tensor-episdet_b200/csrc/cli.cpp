// cli.cpp -- the four executables tensor-episdet.{pairs,triplets}.{k2,mi}.bin.
//
// Same command line (one argument: the dataset descriptor) and the same
// stdout lines as src/tensor-episdet.cu:32-206 of hiperbio/tensor-episdet;
// the search itself goes through the reference-compatible
// EpistasisDetectionSearch() of compat.cpp.
//
// Optional, after the descriptor: `--checkpoint FILE [--slabs N]` runs the
// search in N slabs (default 16) through episdet_search_resumable, saving
// the progress to FILE after each slab; rerunning the same command after an
// interruption continues from FILE.  The output lines are the same.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <iomanip>
#include <iostream>

#include "episdet.h"

#include <cstdlib>
#include <cstring>

#ifndef EPISDET_COMPAT_ORDER
#define EPISDET_COMPAT_ORDER 3
#endif
#ifndef EPISDET_COMPAT_SCORE
#define EPISDET_COMPAT_SCORE EPISDET_SCORE_K2
#endif

cudaError_t EpistasisDetectionSearch(unsigned int* datasetCases, unsigned int* datasetControls, int numSNPs,
                                     int numCases, int numControls, unsigned int numSNPsWithPadding,
                                     int numCasesWithPadding, int numControlsWithPadding, int* roundsCounter,
                                     double* searchTime, float* outputFromGpu, unsigned long long* packedIndices);

static const int kBlockSize = 256;  // the reference's BLOCK_SIZE (Makefile:2)

int main(int argc, const char* argv[]) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, 0);
    if (e != cudaSuccess) {
        std::cerr << "Could not get device properties: " << cudaGetErrorString(e) << std::endl;
        return 1;
    }
    if (prop.major != 10) {
        std::cerr << "Compute capability 10.0 (sm_100a) is required." << std::endl;
        return 1;
    }
    const char* checkpoint = nullptr;
    int slabs = 0;
    for (int i = 2; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--checkpoint") && i + 1 < argc)
            checkpoint = argv[++i];
        else if (!std::strcmp(argv[i], "--slabs") && i + 1 < argc)
            slabs = std::atoi(argv[++i]);
        else
            argc = 0;  // unknown option: print the usage
    }
    if (argc < 2) {
        std::cerr << "Usage: tensor-episdet dataset.txt [--checkpoint FILE [--slabs N]]" << std::endl;
        return 1;
    }
    episdet_dataset d;
    episdet_status s = episdet_read_dataset(argv[1], &d);
    if (s != EPISDET_OK) {
        std::cerr << episdet_last_error() << std::endl;
        return 1;
    }
    unsigned numSNPs = (unsigned)d.num_snps;
    unsigned numBlocks = (numSNPs + kBlockSize - 1) / kBlockSize;
    unsigned numSNPsWithPadding = numBlocks * kBlockSize;
    int casesPad = episdet_class_words(d.num_cases) * 32;
    int controlsPad = episdet_class_words(d.num_controls) * 32;

    std::cout << "Num. SNPs: " << numSNPs << std::endl;
    std::cout << "Num. Blocks of SNPs: " << numBlocks << std::endl;
    std::cout << "Num. Cases: " << d.num_cases << std::endl;
    std::cout << "Num. Controls: " << d.num_controls << std::endl;
    std::cout << "-------------------------------" << std::endl;

    int rounds = 0;
    double seconds = 0.0;
    float best = 0.0f;
    unsigned long long packed = 0;
    if (checkpoint) {
        episdet_options o;
        episdet_default_options(&o);
        o.order = EPISDET_COMPAT_ORDER;
        o.score = EPISDET_COMPAT_SCORE;
        episdet_resume rs;
        std::memset(&rs, 0, sizeof(rs));
        rs.path = checkpoint;
        rs.num_slabs = slabs;
        episdet_result r;
        std::memset(&r, 0, sizeof(r));
        if (episdet_search_resumable(&d, &o, &rs, &r) != EPISDET_OK || !rs.done) {
            std::cerr << "Epistasis detection search failed: " << episdet_last_error() << std::endl;
            e = cudaErrorUnknown;
        } else {
            e = cudaSuccess;
            rounds = (int)r.rounds;
            seconds = r.seconds;
            best = (float)r.score;
            packed = (unsigned long long)r.packed_indices;
        }
    } else {
        e = EpistasisDetectionSearch((unsigned int*)d.cases, (unsigned int*)d.controls, d.num_snps, d.num_cases,
                                     d.num_controls, numSNPsWithPadding, casesPad, controlsPad, &rounds, &seconds,
                                     &best, &packed);
        if (e != cudaSuccess) std::cerr << "Epistasis detection search failed." << std::endl;
    }

#if EPISDET_COMPAT_ORDER == 3
    std::cout << "-------------------------------" << std::endl
              << "{SNP_X_i, SNP_Y_i, SNP_Z_i}: SCORE\t->\t{" << ((packed >> 0) & 0x1FFFFF) << ", "
              << ((packed >> 21) & 0x1FFFFF) << ", " << ((packed >> 42) & 0x1FFFFF) << "}: " << std::fixed
              << std::setprecision(6) << best << std::endl;
    const int k = 3, cells_calc = 8;
#else
    std::cout << "-------------------------------" << std::endl
              << "{SNP_X_i, SNP_Y_i}: SCORE\t->\t{" << ((packed >> 0) & 0xFFFFFFFF) << ", " << ((packed >> 32) & 0xFFFFFFFF)
              << "}: " << std::fixed << std::setprecision(6) << best << std::endl;
    const int k = 2, cells_calc = 4;
#endif
    unsigned long long combos = episdet_n_choose_k(numSNPs, k);
    std::cout << "Num. of rounds processed: " << rounds << std::endl;
    std::cout << "Wall-clock time:\t" << std::fixed << std::setprecision(3) << seconds << " seconds" << std::endl;
    std::cout << "Tensor TOPS: " << std::fixed << std::setprecision(3)
              << (((double)kBlockSize * (double)kBlockSize * (double)(casesPad + controlsPad) * 2 * cells_calc *
                   (double)rounds) /
                  seconds) /
                     1e12
              << std::endl;
    std::cout << "Num. unique sets per sec. (scaled to sample size): " << std::fixed << std::setprecision(3)
              << (((double)combos * (double)(d.num_cases + d.num_controls) / seconds) / 1e12) << " × 10^12"
              << std::endl;
    std::cout << "Unique sets of SNPs evaluated (k=" << k << "): " << combos << std::endl;
    std::cout << "Ratio of unique sets of SNPs: "
              << (((double)combos) / (((double)rounds) * (kBlockSize * kBlockSize))) << std::endl;
    episdet_free_dataset(&d);
    return e == cudaSuccess ? 0 : 1;
}
