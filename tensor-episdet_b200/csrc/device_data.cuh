// device_data.cuh -- the resident per-search device state shared by all engines.
#pragma once
#include <cstdint>
#include "common.cuh"

namespace episdet {

// Class 0 = cases, class 1 = controls (the reference's two .bin arrays).
struct DevData {
    const uint32_t* bits[2];  // [M][2][W[c]] packed planes, reference layout
    int W[2];                 // words per plane row
    int n[2];                 // samples per class
    int M;                    // SNPs
    const int* marg[2];       // [3][M] genotype counts (g2 = n - g0 - g1)
    const uint4* pair4[2];    // [M][M] AND cells (00,01,10,11) of SNP pair (a<b); 3-way only
};

// Search slot lists: one persistent top-K list per CTA, kept in global memory
// between launches of the same search.
struct Slots {
    Cand* lists;     // [nslots][k]
    int* counts;     // [nslots]
    int nslots;
    int k;
    // The smallest k-th best key any CTA has held in this search (0xFFFFFFFF
    // until one held k candidates): a set whose key is larger has k better
    // sets and cannot be in the search's top k.
    uint32_t* gkey;
};

__device__ __forceinline__ void load_marg3(const int* m, int M, int snp, int out[3]) {
    out[0] = __ldg(m + snp);
    out[1] = __ldg(m + M + snp);
    out[2] = __ldg(m + 2 * M + snp);
}

}  // namespace episdet
