// search_internal.h -- host-side workspace and helpers shared by the engines.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "device_data.cuh"
#include "episdet.h"

namespace episdet {

episdet_status cuda_fail(cudaError_t e, const char* what);

#define CUDA_TRY(x)                                     \
    do {                                                \
        cudaError_t e_ = (x);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #x); \
    } while (0)

// Launch-error check naming the launch site.
#define CHECK_LAUNCH()                                                         \
    do {                                                                       \
        cudaError_t e_ = cudaGetLastError();                                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, "launch at " __FILE__ ":" EPI_STR(__LINE__)); \
    } while (0)
#define EPI_STR2(x) #x
#define EPI_STR(x) EPI_STR2(x)

// Grow-only device allocation kept between calls.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

// Sets of regrouped operand buffers of the triplet engine: the regrouping of
// group g + kXSets - 1 (second stream) overlaps the counting launch of group g.
constexpr int kXSets = 2;
constexpr int kXGroup = 4;  // first SNPs per triplet launch (tc::kMaxGroup)

struct Workspace {
    int device = 0;
    int sms = 0;
    cudaStream_t st = nullptr;      // stream of the current call (own_st or the caller's)
    cudaStream_t own_st = nullptr;  // the library's own stream
    cudaStream_t aux_st = nullptr;  // operand regrouping, overlapped with the counting launches
    cudaEvent_t ev_ready = nullptr, ev_cmp[kXSets] = {}, ev_tc[kXSets] = {};  // ordering between st and aux_st
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::mutex mu;
    DevBuf bits[2], marg[2], pair4[2], t32, t64, slots, counts, tiles, merged, mcount, fp64, flag;
    DevBuf pairx[2];      // 3-way tensor engine, Y-blocked pair table: pair rows of the current first SNPs
    DevBuf planes8;       // unpacked 0/1 byte operand rows (tensor engine)
    DevBuf planes_t[2];   // sample-major transposed planes per class (3-way tensor engine's regrouping)
    DevBuf xsub[kXSets * kXGroup];  // per-X sample-regrouped operand rows (tensor engine)
    DevBuf xinfo;         // per-X segment tables (tensor engine)
    DevBuf tensor_flag;   // device error / progress words of the tensor engine
    DevBuf cbuf;          // per-CTA candidate buffers of the filtered triplet kernel
    DevBuf perm_tot;      // label-free pair totals of a permutation batch's cohort
    const uint4* label_tot = nullptr;  // set during a label-mode 2-way search (episdet_search_perm)
    DevBuf perm_planes, perm_cls[2], perm_idx;  // phenotype-permutation staging
    DevBuf bin_geno, bin_idx, bin_out[2];       // genotype-matrix binarizer staging
    // Per-call accounting.
    int64_t h2d = 0, d2h = 0;
    bool timing = false;
    std::vector<cudaEvent_t> tev;  // event pool: (start, end) around each counting launch
    int tev_used = 0;
    int64_t count_launches = 0;
    double executed_macs = 0.0;
    std::vector<double> launch_ms, launch_macs;  // EPISDET_FLAG_TIMING: per counting launch of the last call
    int tab_score = -1, tab_nc = -1, tab_nn = -1;
    int stage_override = -1;  // triplet instance: -1 by the class-size rule, 0 plain, 1 staged
    float inv32 = 0.0f, hy32 = 0.0f, k2_margin = 0.0f;
    double inv64 = 0.0, hy64 = 0.0;

    void release_all() {
        for (DevBuf& b : xsub) b.release();
        DevBuf* all[] = {&bits[0], &bits[1], &marg[0], &marg[1], &pair4[0], &pair4[1], &pairx[0], &pairx[1], &t32,
                         &t64, &slots,
                         &counts, &tiles, &merged, &mcount, &fp64, &flag, &planes8, &planes_t[0], &planes_t[1],
                         &xinfo,
                         &tensor_flag, &cbuf, &perm_tot, &perm_planes, &perm_cls[0], &perm_cls[1], &perm_idx,
                         &bin_geno, &bin_idx, &bin_out[0], &bin_out[1]};
        for (DevBuf* b : all) b->release();
        tab_score = tab_nc = tab_nn = -1;
    }
};

constexpr int kMaxLanes = 4;  // concurrent cohorts of one batched call
// Samples of count segment 0 from which the staged triplet instance copies it
// out of TMEM early (below, that instance runs like the plain one).
constexpr int kStageMinSamples = 8192;
episdet_status get_workspace(int device, Workspace** out);
episdet_status get_workspace_lane(int device, int lane, Workspace** out);
episdet_status build_tables(Workspace* w, int score, int nc, int nn, ScoreTables* T);
episdet_status stage_dataset(Workspace* w, const episdet_dataset* d, bool validate, DevData* D, uint64_t* launches);
episdet_status prepare_slots(Workspace* w, int nslots, int k, Slots* S);
episdet_status check_options(const episdet_options* in, int M, episdet_options* o);
episdet_status check_dataset(const episdet_dataset* d, int order);
// Largest class the tensor engine counts exactly (FP32 accumulators: 2^24).
constexpr int kTensorMaxClass = 1 << 24;
// Largest label-free pair table (M x M x 16 bytes) a permutation batch builds
// for its label mode; beyond it every label runs as a two-class search.
constexpr long long kLabelTotalsMaxBytes = 32ll << 30;
// H(Y) of the FP32 MI score as include/scoring.hpp:29-30 evaluates it on the
// device: each class's p = n * (1/N) is a float product; the first term is a
// double product rounded to float, the second a double multiply-add (nvcc
// contracts `entropyY += (-1.0) * p * t` into one fused operation) rounded to
// float.  t32 is the FP32 log2 table, indexed by count.
inline float mi_hy32(int nc, int nn, float inv32, const float* t32) {
    float p1 = (float)nc * inv32;
    float hy = (float)(-((double)p1 * (double)t32[nc]));
    float p2 = (float)nn * inv32;
    return (float)std::fma(-(double)p2, (double)t32[nn], (double)hy);
}

bool tensor_exact_for(const episdet_dataset* d);
episdet_status check_engine(const episdet_dataset* d, const episdet_options& o);

// Brackets one counting-kernel launch with events when timing is on.
cudaError_t timer_begin(Workspace* w);
cudaError_t timer_end(Workspace* w);

// Selects the stream of this call and resets the per-call accounting.
void begin_call(Workspace* w, const episdet_options& o);

// One search; the caller holds w->mu and has validated the options.
episdet_status search_locked(Workspace* w, const episdet_dataset* data, const episdet_options& o,
                             episdet_result* result);

// Bound of the K2 scoring filter for a sample count (tensor.cu): measures the
// filter's largest distance to the FP32 table d_t32 on the device.
episdet_status k2_filter_margin(Workspace* w, int nc, int nn, const float* d_t32, float* margin);

// Label-free AND cells of every pair of one plane set (tensor.cu), for the
// label-mode 2-way permutation search.
episdet_status tensor_pair_totals(Workspace* w, const uint32_t* d_planes, int M, int n, uint4* out);

// Sets the tensor engine's kernel attributes on the current device.
episdet_status tensor_init_attributes();

// Tensor-core engine (tensor.cu).  Fills S with the per-CTA candidate lists.
episdet_status run_tensor(Workspace* w, DevData& D, const ScoreTables& T, const episdet_options& o, int fb, int fe,
                          Slots* S, uint64_t* launches, bool progress);

}  // namespace episdet
