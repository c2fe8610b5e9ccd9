// batch.cu -- many cohorts and many phenotype permutations per call.
//
// Neither has a counterpart in hiperbio/tensor-episdet, which searches one
// dataset with one label vector per process (src/tensor-episdet.cu:159-172).
//
// Cohorts of a batch run concurrently: kMaxLanes host workers, each with its
// own workspace (buffers and stream) on the device, take cohorts in order of
// decreasing work (C(M, k) x N) from a shared counter and run the ordinary
// search on them.  Kernels are sized to their work, so the small launches of
// one cohort (tails of the triplet launch sequence, the single-block
// candidate merge, small tile sets) leave SMs to the launches of the others.
// Every cohort's result is computed exactly as by a plain call.
// A permutation is applied on the GPU: a label vector splits the cohort's
// sample columns into case and control plane sets in the reference layout,
// which then go through the ordinary search with device-resident inputs.
// For 2-way searches on the tensor engine the label acts as a third AND
// operand: the AND cells of every pair over all samples are counted once per
// call, and per label only the cases' cells are counted (over the regrouped
// case samples, half the MACs of counting both classes at a balanced split);
// the controls' cells are the totals minus the cases'.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "episdet.h"
#include "host_util.h"
#include "search_internal.h"

namespace episdet {

// Gathers sample columns idx[0..n_out) of every plane row into a fresh
// reference-layout row of W_out words (MSB-first, zero padding).
__global__ void __launch_bounds__(256) gather_columns_kernel(const uint32_t* __restrict__ planes, int rows, int W_in,
                                                             const int* __restrict__ idx, int n_out, int W_out,
                                                             uint32_t* __restrict__ out) {
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)rows * W_out) return;
    int r = (int)(t / W_out), ow = (int)(t % W_out);
    const uint32_t* src = planes + (size_t)r * W_in;
    uint32_t v = 0;
    int base = ow * 32;
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
        int s = base + b;
        if (s < n_out) {
            int j = __ldg(idx + s);
            v |= ((__ldg(src + (j >> 5)) >> (31 - (j & 31))) & 1u) << (31 - b);
        }
    }
    out[(size_t)r * W_out + ow] = v;
}

}  // namespace episdet

using namespace episdet;

// Prefixes the current error message (copied first: it is the output buffer too).
static episdet_status with_prefix(episdet_status st, const char* what, int i) {
    char msg[900];
    snprintf(msg, sizeof(msg), "%s", episdet_last_error());
    return set_error(st, "%s %d: %s", what, i, msg);
}

extern "C" episdet_status episdet_search_batched(const episdet_dataset* cohorts, const episdet_options* opts,
                                                 int32_t count, episdet_result* results) {
    clear_error();
    if (!cohorts || !opts || !results || count < 1)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "batched search needs cohorts, options and results");
    std::vector<episdet_options> os((size_t)count);
    for (int32_t i = 0; i < count; ++i) {
        episdet_status st = check_options(&opts[i], cohorts[i].num_snps, &os[i]);
        if (st == EPISDET_OK) st = check_dataset(&cohorts[i], os[i].order);
        if (st == EPISDET_OK) st = check_engine(&cohorts[i], os[i]);
        if (st != EPISDET_OK) return with_prefix(st, "cohort", i);
        if (os[i].device != os[0].device)
            return set_error(EPISDET_ERR_INVALID_ARGUMENT, "all cohorts of a batch run on one device");
    }
    const int device = os[0].device;
    const int lanes = std::min<int>(count, kMaxLanes);
    std::vector<Workspace*> ws((size_t)lanes, nullptr);
    for (int l = 0; l < lanes; ++l) {
        episdet_status st = get_workspace_lane(device, l, &ws[(size_t)l]);
        if (st != EPISDET_OK) return st;
    }
    // Largest first, so the long cohorts start early and the short ones fill in.
    std::vector<double> work((size_t)count);
    for (int32_t i = 0; i < count; ++i) {
        double m = cohorts[i].num_snps, sets = os[i].order == 2 ? m * (m - 1) / 2 : m * (m - 1) * (m - 2) / 6;
        work[(size_t)i] = sets * ((double)cohorts[i].num_cases + cohorts[i].num_controls);
    }
    std::vector<int32_t> order((size_t)count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return work[(size_t)a] > work[(size_t)b]; });
    std::atomic<int32_t> next{0};
    std::atomic<bool> stop{false};
    std::mutex fail_mu;
    episdet_status fail_st = EPISDET_OK;
    int32_t fail_i = -1;
    std::string fail_msg;
    auto worker = [&](int lane) {
        Workspace* w = ws[(size_t)lane];
        std::lock_guard<std::mutex> lock(w->mu);
        if (cudaSetDevice(device) != cudaSuccess) {
            cudaGetLastError();
            std::lock_guard<std::mutex> g(fail_mu);
            if (fail_i < 0) fail_st = EPISDET_ERR_CUDA, fail_i = 0, fail_msg = "cudaSetDevice failed in a batch worker";
            stop = true;
            return;
        }
        for (;;) {
            if (stop.load()) return;
            const int32_t j = next.fetch_add(1);
            if (j >= count) return;
            const int32_t i = order[(size_t)j];
            clear_error();
            episdet_status st = search_locked(w, &cohorts[i], os[(size_t)i], &results[i]);
            if (st != EPISDET_OK) {
                std::lock_guard<std::mutex> g(fail_mu);
                if (fail_i < 0 || i < fail_i) fail_st = st, fail_i = i, fail_msg = episdet_last_error();
                stop = true;
                return;
            }
        }
    };
    std::vector<std::thread> threads;
    for (int l = 1; l < lanes; ++l) threads.emplace_back(worker, l);
    worker(0);
    for (auto& t : threads) t.join();
    if (fail_i >= 0) return set_error(fail_st, "cohort %d: %s", fail_i, fail_msg.c_str());
    return EPISDET_OK;
}

// One label vector of a permutation batch: split the cohort's sample columns
// into case and control plane sets on the GPU, then search them.
static episdet_status perm_one(Workspace* w, const uint32_t* d_planes, int M, int n, int W, const uint32_t* label,
                               bool label_on_device, bool first_label, const episdet_options& o,
                               episdet_result* result) {
    std::vector<uint32_t> lab((size_t)W);
    std::vector<int> idx((size_t)n);
    if (!label_on_device)
        memcpy(lab.data(), label, sizeof(uint32_t) * W);
    else {
        CUDA_TRY(cudaMemcpyAsync(lab.data(), label, sizeof(uint32_t) * W, cudaMemcpyDeviceToHost, w->st));
        CUDA_TRY(cudaStreamSynchronize(w->st));
    }
    int nc = 0;
    for (int s = 0; s < n; ++s)
        if ((lab[s / 32] >> (31 - s % 32)) & 1u) idx[nc++] = s;
    int nn = nc;
    for (int s = 0; s < n; ++s)
        if (!((lab[s / 32] >> (31 - s % 32)) & 1u)) idx[nn++] = s;
    nn -= nc;
    if (nc < 1 || nn < 1) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "the label leaves a class empty");
    const int Wc = episdet_class_words(nc), Wn = episdet_class_words(nn);
    CUDA_TRY(w->perm_idx.ensure(sizeof(int) * (size_t)n));
    CUDA_TRY(w->perm_cls[0].ensure(sizeof(uint32_t) * (size_t)M * 2 * Wc));
    CUDA_TRY(w->perm_cls[1].ensure(sizeof(uint32_t) * (size_t)M * 2 * Wn));
    CUDA_TRY(cudaMemcpyAsync(w->perm_idx.p, idx.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, w->st));
    // The host vector must outlive the copy.
    CUDA_TRY(cudaStreamSynchronize(w->st));
    long t0 = (long)2 * M * Wc, t1 = (long)2 * M * Wn;
    gather_columns_kernel<<<(unsigned)((t0 + 255) / 256), 256, 0, w->st>>>(d_planes, 2 * M, W, (const int*)w->perm_idx.p,
                                                                            nc, Wc, (uint32_t*)w->perm_cls[0].p);
    CHECK_LAUNCH();
    gather_columns_kernel<<<(unsigned)((t1 + 255) / 256), 256, 0, w->st>>>(
        d_planes, 2 * M, W, (const int*)w->perm_idx.p + nc, nn, Wn, (uint32_t*)w->perm_cls[1].p);
    CHECK_LAUNCH();
    episdet_dataset d;
    d.cases = (const uint32_t*)w->perm_cls[0].p;
    d.controls = (const uint32_t*)w->perm_cls[1].p;
    d.num_snps = M;
    d.num_cases = nc;
    d.num_controls = nn;
    d.memory = EPISDET_DEVICE;
    episdet_status st = check_dataset(&d, o.order);
    // The planes of every label are columns of the cohort's, validated (when
    // asked) with its first label; re-checking them per label would add a
    // synchronising read-back each time.
    episdet_options ol = o;
    if (!first_label) ol.flags |= EPISDET_FLAG_NO_VALIDATE;
    if (st == EPISDET_OK) st = search_locked(w, &d, ol, result);
    if (st == EPISDET_OK) result->kernel_launches += 2;
    return st;
}

// Label vectors run concurrently on the workspace lanes, like the cohorts of a
// batch; the cohort's planes are read by every lane from one device copy.
extern "C" episdet_status episdet_search_perm(const episdet_cohort* cohort, const uint32_t* labels,
                                              int32_t num_labels, const episdet_options* opts,
                                              episdet_result* results) {
    clear_error();
    if (!cohort || !cohort->planes || !labels || num_labels < 1 || !results)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "permutation search needs a cohort, labels and results");
    if (cohort->memory != EPISDET_HOST && cohort->memory != EPISDET_DEVICE)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown memory kind");
    const int M = cohort->num_snps, n = cohort->num_samples;
    if (M < 2 || n < 2 || M > (1 << 21) - 1) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad cohort sizes");
    episdet_options o;
    episdet_status st = check_options(opts, M, &o);
    if (st != EPISDET_OK) return st;
    const int lanes = std::min<int>(num_labels, kMaxLanes);
    std::vector<Workspace*> ws((size_t)lanes, nullptr);
    for (int l = 0; l < lanes; ++l) {
        st = get_workspace_lane(o.device, l, &ws[(size_t)l]);
        if (st != EPISDET_OK) return st;
    }
    const int W = episdet_class_words(n);
    const size_t plane_words = (size_t)M * 2 * W;
    const uint32_t* d_planes = cohort->planes;
    Workspace* w0 = ws[0];
    std::unique_lock<std::mutex> lock0(w0->mu);
    CUDA_TRY(cudaSetDevice(o.device));
    if (cohort->memory == EPISDET_HOST) {
        CUDA_TRY(w0->perm_planes.ensure(sizeof(uint32_t) * plane_words));
        CUDA_TRY(cudaMemcpyAsync(w0->perm_planes.p, cohort->planes, sizeof(uint32_t) * plane_words,
                                 cudaMemcpyHostToDevice, w0->own_st));
        CUDA_TRY(cudaStreamSynchronize(w0->own_st));
        d_planes = (const uint32_t*)w0->perm_planes.p;
    }
    const bool on_device = cohort->memory == EPISDET_DEVICE;
    // Label mode: the pair totals of the whole cohort, once, shared read-only
    // by every lane (the computation ends with a synchronise of lane 0's stream).
    const uint4* tot = nullptr;
    const size_t tot_bytes = sizeof(uint4) * (size_t)M * (size_t)M;
    if (o.order == 2 && o.engine != EPISDET_ENGINE_SIMT && !(o.flags & EPISDET_FLAG_PERM_SPLIT) &&
        n <= kTensorMaxClass && tot_bytes <= (size_t)kLabelTotalsMaxBytes) {
        begin_call(w0, o);
        CUDA_TRY(w0->perm_tot.ensure(tot_bytes));
        st = tensor_pair_totals(w0, d_planes, M, n, (uint4*)w0->perm_tot.p);
        if (st != EPISDET_OK) return st;
        tot = (const uint4*)w0->perm_tot.p;
    }
    std::atomic<int32_t> next{0};
    std::atomic<bool> stop{false};
    std::mutex fail_mu;
    episdet_status fail_st = EPISDET_OK;
    int32_t fail_p = -1;
    std::string fail_msg;
    auto worker = [&](int lane) {
        Workspace* w = ws[(size_t)lane];
        std::unique_lock<std::mutex> lock;
        if (lane != 0) lock = std::unique_lock<std::mutex>(w->mu);
        if (cudaSetDevice(o.device) != cudaSuccess) {
            cudaGetLastError();
            std::lock_guard<std::mutex> g(fail_mu);
            if (fail_p < 0) fail_st = EPISDET_ERR_CUDA, fail_p = 0, fail_msg = "cudaSetDevice failed in a worker";
            stop = true;
            return;
        }
        for (;;) {
            if (stop.load()) return;
            const int32_t p = next.fetch_add(1);
            if (p >= num_labels) return;
            clear_error();
            begin_call(w, o);
            w->label_tot = tot;
            episdet_status s2 =
                perm_one(w, d_planes, M, n, W, labels + (size_t)p * W, on_device, p == 0, o, &results[p]);
            w->label_tot = nullptr;
            if (s2 != EPISDET_OK) {
                std::lock_guard<std::mutex> g(fail_mu);
                if (fail_p < 0 || p < fail_p) fail_st = s2, fail_p = p, fail_msg = episdet_last_error();
                stop = true;
                return;
            }
        }
    };
    std::vector<std::thread> threads;
    for (int l = 1; l < lanes; ++l) threads.emplace_back(worker, l);
    worker(0);
    for (auto& t : threads) t.join();
    if (fail_p >= 0) return set_error(fail_st, "label %d: %s", fail_p, fail_msg.c_str());
    return EPISDET_OK;
}
