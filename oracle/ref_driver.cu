// Test infrastructure: runs hiperbio/tensor-episdet's own search on one
// dataset and prints its answer with the score's exact bits.
//
// The oracle/Makefile `ref` target compiles this file together with the
// reference's unmodified src/helper.cu and src/search-{pairs,triplets}.cu
// (against the CUTLASS stand-in under oracle/refgemm) into oracle/_ref/.  The
// reference's main (src/tensor-episdet.cu:58-148) reads the same dataset
// files but prints the score to six decimals only, so this driver reads the
// descriptor the same way, calls EpistasisDetectionSearch
// (include/search-triplets.hpp, include/search-pairs.hpp) with the same
// padded sizes (src/tensor-episdet.cu:85-96), and prints one line:
//
//   reference_result order=3 score_bits=0x... score=... packed=... rounds=... status=0
//
// `packed` is the reference's set encoding (src/helper.cu:574 for triplets,
// :690 for pairs).  Kernel launches are serialised (CUDA_LAUNCH_BLOCKING=1,
// set before the first CUDA call): the reference's drivers let the GEMMs of a
// first SNP on other streams start before the operand kernel on the first
// stream has written their operand (src/search-triplets.cu:196-224), and read
// one block's planes on streams other than the one that copied them
// (src/search-pairs.cu:70-80, :150-165); serialising keeps every read after
// its write, which is the order the host code issues them in.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

cudaError_t EpistasisDetectionSearch(unsigned int* datasetCases_host_matrixA, unsigned int* datasetControls_host_matrixA,
                                     int numSNPs, int numCases, int numControls, unsigned int numSNPsWithPadding,
                                     int numCasesWithPadding, int numControlsWithPadding, int* roundsCounter,
                                     double* searchTime, float* outputFromGpu,
                                     unsigned long long int* output_indexFromGpu_packedIndices);

#ifndef BLOCK_SIZE
#error "build with the reference's -DBLOCK_SIZE"
#endif
#if defined(TRIPLETS)
static const int kOrder = 3;
#else
static const int kOrder = 2;
#endif

static bool read_line(FILE* f, std::string* out) {
    char buf[4096];
    if (!fgets(buf, sizeof(buf), f)) return false;
    buf[strcspn(buf, "\r\n")] = 0;
    *out = buf;
    return true;
}

static unsigned int* read_class(const std::string& path, size_t words_read, size_t words_alloc) {
    unsigned int* p = nullptr;
    if (cudaHostAlloc((void**)&p, words_alloc * sizeof(unsigned int), cudaHostAllocDefault) != cudaSuccess) return nullptr;
    memset(p, 0, words_alloc * sizeof(unsigned int));
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return nullptr;
    size_t got = fread(p, sizeof(unsigned int), words_read, f);
    fclose(f);
    return got == words_read ? p : nullptr;
}

int main(int argc, char** argv) {
    if (argc != 2) {
        fprintf(stderr, "usage: %s dataset.txt\n", argv[0]);
        return 2;
    }
    setenv("CUDA_LAUNCH_BLOCKING", "1", 1);

    FILE* f = fopen(argv[1], "r");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    std::string dir(argv[1]);
    size_t slash = dir.find_last_of('/');
    dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
    std::string l_snps, l_ctrl_file, l_ctrl, l_case_file, l_case;
    bool ok = read_line(f, &l_snps) && read_line(f, &l_ctrl_file) && read_line(f, &l_ctrl) &&
              read_line(f, &l_case_file) && read_line(f, &l_case);
    fclose(f);
    if (!ok) {
        fprintf(stderr, "short descriptor\n");
        return 2;
    }
    const int num_snps = atoi(l_snps.c_str());
    const int num_controls = atoi(l_ctrl.c_str());
    const int num_cases = atoi(l_case.c_str());
    if (num_snps <= 0 || num_cases <= 0 || num_controls <= 0) {
        fprintf(stderr, "bad descriptor\n");
        return 2;
    }
    const unsigned int snps_padded = (unsigned int)((num_snps + BLOCK_SIZE - 1) / BLOCK_SIZE) * BLOCK_SIZE;
    const int cases_padded = (num_cases + 1023) / 1024 * 1024;
    const int controls_padded = (num_controls + 1023) / 1024 * 1024;
    const size_t wc = (size_t)cases_padded / 32, wn = (size_t)controls_padded / 32;

    unsigned int* cases = read_class(dir + "/" + l_case_file, wc * 2 * num_snps, wc * 2 * snps_padded);
    unsigned int* controls = read_class(dir + "/" + l_ctrl_file, wn * 2 * num_snps, wn * 2 * snps_padded);
    if (!cases || !controls) {
        fprintf(stderr, "cannot read the class files\n");
        return 2;
    }

    int rounds = 0;
    double seconds = 0.0;
    float score = 0.0f;
    unsigned long long packed = 0;
    cudaError_t st = EpistasisDetectionSearch(cases, controls, num_snps, num_cases, num_controls, snps_padded,
                                              cases_padded, controls_padded, &rounds, &seconds, &score, &packed);
    cudaError_t after = cudaDeviceSynchronize();
    if (st == cudaSuccess) st = after;
    if (st == cudaSuccess) st = cudaGetLastError();
    uint32_t bits;
    memcpy(&bits, &score, sizeof(bits));
    printf("reference_result order=%d score_bits=0x%08x score=%.9g packed=%llu rounds=%d status=%d\n", kOrder, bits,
           (double)score, packed, rounds, (int)st);
    cudaFreeHost(cases);
    cudaFreeHost(controls);
    return st == cudaSuccess ? 0 : 1;
}
