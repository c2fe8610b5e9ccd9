// binarize.cu -- genotype matrix -> the reference's per-class bit planes.
//
// hiperbio/tensor-episdet reads datasets that are already binarized: per class,
// [SNP][genotype 0/1][W] 32-bit words, MSB first, each row zero-padded to a
// multiple of 1024 bits (src/tensor-episdet.cu:58-148, README.md:48-50).  This
// builds that layout on the GPU from a dense [SNP][sample] matrix of 0/1/2
// genotype bytes and a case flag per sample: one thread per output word of a
// (SNP, class) row packs the 32 samples of that word, taken in sample order
// within the class through a per-class sample index list.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "episdet.h"
#include "host_util.h"
#include "search_internal.h"

namespace episdet {

__global__ void __launch_bounds__(256) binarize_kernel(const uint8_t* __restrict__ geno, int M, int n,
                                                       const int* __restrict__ idx, int n_class, int W,
                                                       uint32_t* __restrict__ out, int* __restrict__ bad) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)M * W) return;
    const int snp = (int)(t / W), w = (int)(t % W);
    const uint8_t* row = geno + (size_t)snp * n;
    uint32_t p0 = 0, p1 = 0;
    int over = 0;
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
        const int s = w * 32 + b;
        if (s < n_class) {
            const uint32_t g = __ldg(row + __ldg(idx + s));
            p0 |= (uint32_t)(g == 0) << (31 - b);
            p1 |= (uint32_t)(g == 1) << (31 - b);
            over |= g > 2;
        }
    }
    out[((size_t)snp * 2 + 0) * W + w] = p0;
    out[((size_t)snp * 2 + 1) * W + w] = p1;
    if (over) atomicExch(bad, 1);
}

}  // namespace episdet

using namespace episdet;

extern "C" episdet_status episdet_binarize(const uint8_t* genotypes, int32_t num_snps, int32_t num_samples,
                                           const uint8_t* is_case, uint32_t* cases, uint32_t* controls,
                                           int32_t memory, int32_t device) {
    clear_error();
    if (!genotypes || !is_case || !cases || !controls)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "binarize needs genotypes, case flags and two outputs");
    if (memory != EPISDET_HOST && memory != EPISDET_DEVICE)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown memory kind");
    const int M = num_snps, n = num_samples;
    if (M < 1 || n < 2 || (int64_t)M * n > ((int64_t)1 << 40))
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad matrix size %d x %d", M, n);
    Workspace* w = nullptr;
    episdet_status st = get_workspace(device, &w);
    if (st != EPISDET_OK) return st;
    std::lock_guard<std::mutex> lock(w->mu);
    CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = w->own_st;
    // Sample index lists, cases first, in sample order.
    std::vector<uint8_t> flag((size_t)n);
    if (memory == EPISDET_HOST)
        memcpy(flag.data(), is_case, (size_t)n);
    else {
        CUDA_TRY(cudaMemcpyAsync(flag.data(), is_case, (size_t)n, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    std::vector<int> idx((size_t)n);
    int nc = 0;
    for (int i = 0; i < n; ++i)
        if (flag[(size_t)i]) idx[(size_t)nc++] = i;
    int pos = nc;
    for (int i = 0; i < n; ++i)
        if (!flag[(size_t)i]) idx[(size_t)pos++] = i;
    const int nn = n - nc;
    if (nc < 1 || nn < 1) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "the case flags leave a class empty");
    const int Wc = episdet_class_words(nc), Wn = episdet_class_words(nn);
    const size_t geno_bytes = (size_t)M * n;
    const size_t out_words[2] = {(size_t)M * 2 * Wc, (size_t)M * 2 * Wn};
    const uint8_t* d_geno = genotypes;
    uint32_t* d_out[2] = {cases, controls};
    if (memory == EPISDET_HOST) {
        CUDA_TRY(w->bin_geno.ensure(geno_bytes));
        CUDA_TRY(cudaMemcpyAsync(w->bin_geno.p, genotypes, geno_bytes, cudaMemcpyHostToDevice, s));
        d_geno = (const uint8_t*)w->bin_geno.p;
        for (int c = 0; c < 2; ++c) {
            CUDA_TRY(w->bin_out[c].ensure(sizeof(uint32_t) * out_words[c]));
            d_out[c] = (uint32_t*)w->bin_out[c].p;
        }
    }
    CUDA_TRY(w->bin_idx.ensure(sizeof(int) * (size_t)n));
    CUDA_TRY(w->flag.ensure(sizeof(int) * 4));
    CUDA_TRY(cudaMemcpyAsync(w->bin_idx.p, idx.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(w->flag.p, 0, sizeof(int), s));
    const int ncls[2] = {nc, nn}, Ws[2] = {Wc, Wn};
    for (int c = 0; c < 2; ++c) {
        const long threads = (long)M * Ws[c];
        binarize_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
            d_geno, M, n, (const int*)w->bin_idx.p + (c ? nc : 0), ncls[c], Ws[c], d_out[c], (int*)w->flag.p);
        CHECK_LAUNCH();
    }
    int bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&bad, w->flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (memory == EPISDET_HOST) {
        CUDA_TRY(cudaMemcpyAsync(cases, d_out[0], sizeof(uint32_t) * out_words[0], cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(controls, d_out[1], sizeof(uint32_t) * out_words[1], cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    if (bad) return set_error(EPISDET_ERR_INVALID_INPUT, "a genotype value is above 2");
    return EPISDET_OK;
}
