// kernels.h -- kernel declarations shared by the host orchestration.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"
#include "device_data.cuh"

namespace episdet {

constexpr int kSimtTileSnps = 32;
constexpr int kSimtBlockThreads = 256;
constexpr size_t kSimtSmem2 = 16 * 4096 + 2 * 64 * 33 * 4 + 32;
constexpr size_t kSimtSmem3 = kSimtSmem2 + 2 * 32 * 4;
constexpr int kMergeBlockThreads = 1024;
constexpr size_t kMergeSmem = 16 * 8192;

__global__ void marginals_kernel(DevData D, int* marg0, int* marg1, int* bad_flag);

extern "C" __global__ void search2_simt_kernel(DevData D, ScoreTables T, const int2* tiles, int ntiles,
                                               int first_begin, int first_end, Slots S, int store_pairs,
                                               uint4* pair_out0, uint4* pair_out1);
extern "C" __global__ void search3_simt_kernel(DevData D, ScoreTables T, int xsnp, const int2* tiles, int ntiles,
                                               Slots S);
extern "C" __global__ void merge_topk_kernel(Slots S, Cand* out, int* out_count);
extern "C" __global__ void rescore_kernel(DevData D, ScoreTables T, int order, const Cand* cands, const int* count,
                                          double* fp64_out, int* cells_out);

}  // namespace episdet
