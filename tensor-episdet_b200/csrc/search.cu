// search.cu -- host orchestration behind the C-ABI: device workspace,
// upload and validation, score tables, engine dispatch, top-K merge, FP64
// re-score and result assembly.
//
// Replaces the host drivers src/search-pairs.cu:9-246 and
// src/search-triplets.cu:8-305 of hiperbio/tensor-episdet.  Where those issue
// ~700k launches and ~280k stream syncs for a 4096-SNP 3-way search, this
// driver issues one persistent counting launch per first SNP (3-way) or one in
// total (2-way), and synchronises once at the end.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "episdet.h"
#include "host_util.h"
#include "kernels.h"
#include "search_internal.h"

namespace episdet {

static thread_local char g_err[1024] = "";

episdet_status set_error(episdet_status s, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return s;
}
void clear_error() { g_err[0] = 0; }

episdet_status cuda_fail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) return set_error(EPISDET_ERR_OUT_OF_MEMORY, "%s: out of device memory", what);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(EPISDET_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return set_error(EPISDET_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Allocation-failure injection (episdet_test_fail_allocation): the number of
// allocations still to make before one fails; 0 = disarmed.
static std::atomic<int> g_fail_alloc{0};

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    int left = g_fail_alloc.load();
    while (left > 0 && !g_fail_alloc.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 1) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

static std::mutex g_ws_mu;
static Workspace* g_ws[64][kMaxLanes] = {};

// Lane 0 serves every single-dataset call; lanes 1.. let the batched entry
// point run several cohorts at once, each with its own buffers and stream.
episdet_status get_workspace(int device, Workspace** out) { return get_workspace_lane(device, 0, out); }

episdet_status get_workspace_lane(int device, int lane, Workspace** out) {
    if (lane < 0 || lane >= kMaxLanes) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "workspace lane %d out of range", lane);
    if (device < 0 || device >= 64) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(EPISDET_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    }
    if (device >= ndev) return set_error(EPISDET_ERR_NO_DEVICE, "device %d not present (%d devices)", device, ndev);
    std::lock_guard<std::mutex> g(g_ws_mu);
    if (!g_ws[device][lane]) {
        CUDA_TRY(cudaSetDevice(device));
        cudaDeviceProp prop;
        CUDA_TRY(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10)
            return set_error(EPISDET_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a only",
                             device, prop.major, prop.minor);
        Workspace* w = new Workspace();
        w->device = device;
        w->sms = prop.multiProcessorCount;
        CUDA_TRY(cudaStreamCreateWithFlags(&w->own_st, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&w->aux_st, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&w->ev_ready, cudaEventDisableTiming));
        for (int i = 0; i < kXSets; ++i) {
            CUDA_TRY(cudaEventCreateWithFlags(&w->ev_cmp[i], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&w->ev_tc[i], cudaEventDisableTiming));
        }
        w->st = w->own_st;
        CUDA_TRY(cudaEventCreate(&w->e0));
        CUDA_TRY(cudaEventCreate(&w->e1));
        // Every kernel with more than 48 KB of dynamic shared memory, once per device.
        CUDA_TRY(cudaFuncSetAttribute(search2_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSimtSmem2));
        CUDA_TRY(cudaFuncSetAttribute(search3_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSimtSmem3));
        CUDA_TRY(cudaFuncSetAttribute(merge_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMergeSmem));
        episdet_status st = tensor_init_attributes();
        if (st != EPISDET_OK) return st;
        g_ws[device][lane] = w;
    }
    *out = g_ws[device][lane];
    return EPISDET_OK;
}

void begin_call(Workspace* w, const episdet_options& o) {
    w->st = o.stream ? (cudaStream_t)(uintptr_t)o.stream : w->own_st;
    w->h2d = w->d2h = 0;
    w->timing = (o.flags & EPISDET_FLAG_TIMING) != 0;
    w->tev_used = 0;
    w->count_launches = 0;
    w->executed_macs = 0.0;
    w->launch_ms.clear();
    w->launch_macs.clear();
}

cudaError_t timer_begin(Workspace* w) {
    ++w->count_launches;
    if (!w->timing) return cudaSuccess;
    while ((int)w->tev.size() < w->tev_used + 2) {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        w->tev.push_back(e);
    }
    return cudaEventRecord(w->tev[w->tev_used++], w->st);
}

cudaError_t timer_end(Workspace* w) {
    if (!w->timing) return cudaSuccess;
    return cudaEventRecord(w->tev[w->tev_used++], w->st);
}

// Score tables, built on the host in double with glibc (src/search-pairs.cu:83-106):
// K2 holds lnGamma(v+1) for v in [0, N+1]; MI holds log2(v * invN) for v in [1, N].
episdet_status build_tables(Workspace* w, int score, int nc, int nn, ScoreTables* T) {
    if (w->tab_score != score || w->tab_nc != nc || w->tab_nn != nn) {
        int N = nc + nn;
        int size = score == EPISDET_SCORE_K2 ? N + 2 : N + 1;
        std::vector<float> t32((size_t)size);
        std::vector<double> t64((size_t)size);
        if (score == EPISDET_SCORE_K2) {
            for (int v = 0; v < size; ++v) {
                double g = lgamma((double)v + 1.0);
                t64[v] = g;
                t32[v] = (float)g;
            }
            w->inv32 = 0.0f;
            w->inv64 = 0.0;
            w->hy32 = 0.0f;
            w->hy64 = 0.0;
        } else {
            w->inv32 = (float)(1.0 / (double)N);
            w->inv64 = 1.0 / (double)N;
            t32[0] = 0.0f;
            t64[0] = 0.0;
            for (int v = 1; v < size; ++v) {
                t32[v] = (float)log2((double)v * (double)w->inv32);
                t64[v] = log2((double)v / (double)N);
            }
            double p1 = (double)nc * w->inv64, p2 = (double)nn * w->inv64;
            w->hy64 = -(p1 * t64[nc]) - (p2 * t64[nn]);
            w->hy32 = mi_hy32(nc, nn, w->inv32, t32.data());
        }
        CUDA_TRY(w->t32.ensure(sizeof(float) * size));
        CUDA_TRY(w->t64.ensure(sizeof(double) * size));
        CUDA_TRY(cudaMemcpyAsync(w->t32.p, t32.data(), sizeof(float) * size, cudaMemcpyHostToDevice, w->st));
        CUDA_TRY(cudaMemcpyAsync(w->t64.p, t64.data(), sizeof(double) * size, cudaMemcpyHostToDevice, w->st));
        CUDA_TRY(cudaStreamSynchronize(w->st));
        w->h2d += (int64_t)size * (sizeof(float) + sizeof(double));
        w->k2_margin = 0.0f;
        if (score == EPISDET_SCORE_K2) {
            episdet_status st = k2_filter_margin(w, nc, nn, (const float*)w->t32.p, &w->k2_margin);
            if (st != EPISDET_OK) return st;
        }
        w->tab_score = score;
        w->tab_nc = nc;
        w->tab_nn = nn;
    }
    T->t32 = (const float*)w->t32.p;
    T->t64 = (const double*)w->t64.p;
    T->inv_n32 = w->inv32;
    T->inv_n64 = w->inv64;
    T->hy32 = w->hy32;
    T->hy64 = w->hy64;
    T->score = score;
    T->k2_margin = w->k2_margin;
    return EPISDET_OK;
}

static int64_t sets_in_slab(int order, int64_t M, int64_t fb, int64_t fe) {
    int64_t s = 0;
    for (int64_t a = fb; a < fe; ++a) {
        int64_t r = M - 1 - a;
        s += order == 2 ? r : (r * (r - 1)) / 2;
    }
    return s;
}

static int64_t reference_rounds(int order, int64_t M) {
    const int64_t bs = 256;
    int64_t nb = (M + bs - 1) / bs;
    if (order == 2) return nb * (nb + 1) / 2;
    int64_t r = 0;
    for (int64_t yb = 0; yb < nb; ++yb) r += std::min((yb + 1) * bs, M) * (nb - yb);
    return r;
}

// Uploads (or adopts) the planes, computes marginals and checks the input contract.
episdet_status stage_dataset(Workspace* w, const episdet_dataset* d, bool validate, DevData* D, uint64_t* launches) {
    const uint32_t* src[2] = {d->cases, d->controls};
    int ns[2] = {d->num_cases, d->num_controls};
    D->M = d->num_snps;
    for (int c = 0; c < 2; ++c) {
        D->n[c] = ns[c];
        D->W[c] = episdet_class_words(ns[c]);
        size_t bytes = sizeof(uint32_t) * (size_t)d->num_snps * 2 * D->W[c];
        if (d->memory == EPISDET_DEVICE) {
            if (((uintptr_t)src[c]) & 15)
                return set_error(EPISDET_ERR_INVALID_ARGUMENT, "device planes must be 16-byte aligned");
            D->bits[c] = src[c];
        } else {
            CUDA_TRY(w->bits[c].ensure(bytes));
            CUDA_TRY(cudaMemcpyAsync(w->bits[c].p, src[c], bytes, cudaMemcpyHostToDevice, w->st));
            w->h2d += (int64_t)bytes;
            D->bits[c] = (const uint32_t*)w->bits[c].p;
        }
        CUDA_TRY(w->marg[c].ensure(sizeof(int) * 3 * (size_t)d->num_snps));
        D->marg[c] = (const int*)w->marg[c].p;
        D->pair4[c] = nullptr;
    }
    CUDA_TRY(w->flag.ensure(sizeof(int) * 4));
    CUDA_TRY(cudaMemsetAsync(w->flag.p, 0, sizeof(int) * 4, w->st));
    CUDA_TRY(w->tensor_flag.ensure(sizeof(int) * 4));
    CUDA_TRY(cudaMemsetAsync(w->tensor_flag.p, 0, sizeof(int) * 4, w->st));
    int warps = 2 * d->num_snps;
    marginals_kernel<<<(warps * 32 + 255) / 256, 256, 0, w->st>>>(*D, (int*)w->marg[0].p, (int*)w->marg[1].p,
                                                                   (int*)w->flag.p);
    CHECK_LAUNCH();
    ++*launches;
    if (validate) {
        int bad = 0;
        CUDA_TRY(cudaMemcpyAsync(&bad, w->flag.p, sizeof(int), cudaMemcpyDeviceToHost, w->st));
        w->d2h += sizeof(int);
        CUDA_TRY(cudaStreamSynchronize(w->st));
        if (bad)
            return set_error(EPISDET_ERR_INVALID_INPUT,
                             "input planes have padding bits set or overlapping genotype-0/1 planes");
    }
    return EPISDET_OK;
}

episdet_status prepare_slots(Workspace* w, int nslots, int k, Slots* S) {
    CUDA_TRY(w->slots.ensure(sizeof(Cand) * (size_t)nslots * k));
    CUDA_TRY(w->counts.ensure(sizeof(int) * ((size_t)nslots + 1)));
    CUDA_TRY(cudaMemsetAsync(w->counts.p, 0, sizeof(int) * (size_t)nslots, w->st));
    CUDA_TRY(cudaMemsetAsync((int*)w->counts.p + nslots, 0xFF, sizeof(int), w->st));
    S->lists = (Cand*)w->slots.p;
    S->counts = (int*)w->counts.p;
    S->nslots = nslots;
    S->k = k;
    S->gkey = (uint32_t*)((int*)w->counts.p + nslots);
    return EPISDET_OK;
}

static void tri_tiles(int t_first, int nt, std::vector<int2>& out) {
    out.clear();
    for (int a = t_first; a < nt; ++a)
        for (int b = a; b < nt; ++b) out.push_back(make_int2(a, b));
}

// ------------------------------------------------------------ SIMT engine
static episdet_status run_simt(Workspace* w, const DevData& D0, const ScoreTables& T, const episdet_options& o,
                               int fb, int fe, Slots* S, uint64_t* launches, bool progress) {
    DevData D = D0;
    const int M = D.M;
    const int nt = (M + kSimtTileSnps - 1) / kSimtTileSnps;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search3_simt_kernel, kSimtBlockThreads, kSimtSmem3));
    int grid = w->sms * std::max(per_sm, 1);
    episdet_status st = prepare_slots(w, grid, o.top_k, S);
    if (st != EPISDET_OK) return st;
    std::vector<int2> tiles;
    const int bs_lines = (M + 255) / 256;
    if (o.order == 2) {
        tiles.clear();
        for (int a = fb / kSimtTileSnps; a <= (fe - 1) / kSimtTileSnps; ++a)
            for (int b = a; b < nt; ++b) tiles.push_back(make_int2(a, b));
        CUDA_TRY(w->tiles.ensure(sizeof(int2) * tiles.size()));
        CUDA_TRY(cudaMemcpyAsync(w->tiles.p, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, w->st));
        if (progress)
            for (int i = 0; i < bs_lines; ++i) printf("Outer loop iteration %d out of %d\n", i, bs_lines);
        w->h2d += (int64_t)(sizeof(int2) * tiles.size());
        CUDA_TRY(timer_begin(w));
        search2_simt_kernel<<<grid, kSimtBlockThreads, kSimtSmem2, w->st>>>(
            D, T, (const int2*)w->tiles.p, (int)tiles.size(), fb, fe, *S, 0, nullptr, nullptr);
        CHECK_LAUNCH();
        CUDA_TRY(timer_end(w));
        ++*launches;
        return EPISDET_OK;
    }
    // 3-way: pair table (AND cells of every SNP pair with first index >= fb).
    for (int c = 0; c < 2; ++c) {
        CUDA_TRY(w->pair4[c].ensure(sizeof(uint4) * (size_t)M * M));
        D.pair4[c] = (const uint4*)w->pair4[c].p;
    }
    tri_tiles(fb / kSimtTileSnps, nt, tiles);
    std::vector<int2> all3;
    tri_tiles(0, nt, all3);
    size_t need = std::max(tiles.size(), all3.size());
    CUDA_TRY(w->tiles.ensure(sizeof(int2) * need * 2));
    int2* d_pair_tiles = (int2*)w->tiles.p;
    int2* d_tiles3 = d_pair_tiles + tiles.size();
    CUDA_TRY(cudaMemcpyAsync(d_pair_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, w->st));
    CUDA_TRY(cudaMemcpyAsync(d_tiles3, all3.data(), sizeof(int2) * all3.size(), cudaMemcpyHostToDevice, w->st));
    search2_simt_kernel<<<grid, kSimtBlockThreads, kSimtSmem2, w->st>>>(
        D, T, d_pair_tiles, (int)tiles.size(), 0, M, *S, 1, (uint4*)w->pair4[0].p, (uint4*)w->pair4[1].p);
    CHECK_LAUNCH();
    ++*launches;
    // Per-X launches over the (Y-tile, Z-tile) suffix with Y-tile >= tile(X+1).
    std::vector<int> off((size_t)nt + 1, 0);
    for (int t = 0; t < nt; ++t) off[t + 1] = off[t] + (nt - t);
    int xend = std::min(fe, M - 2);
    for (int x = fb; x < xend; ++x) {
        if (progress && x % 256 == 0) printf("Outer loop iteration %d out of %d\n", x / 256, bs_lines);
        int ty0 = (x + 1) / kSimtTileSnps;
        int n3 = off[nt] - off[ty0];
        CUDA_TRY(timer_begin(w));
        search3_simt_kernel<<<grid, kSimtBlockThreads, kSimtSmem3, w->st>>>(D, T, x, d_tiles3 + off[ty0], n3, *S);
        CHECK_LAUNCH();
        CUDA_TRY(timer_end(w));
        ++*launches;
    }
    return EPISDET_OK;
}

// Merge, FP64 re-score, copy back, pick the FP64 optimum.
static episdet_status finish(Workspace* w, const DevData& D, const ScoreTables& T, const episdet_options& o,
                             const Slots& S, episdet_result* r, uint64_t* launches) {
    const int k = o.top_k;
    CUDA_TRY(w->merged.ensure(sizeof(Cand) * (size_t)k));
    CUDA_TRY(w->mcount.ensure(sizeof(int) * 4));
    CUDA_TRY(w->fp64.ensure(sizeof(double) * (size_t)k));
    merge_topk_kernel<<<1, kMergeBlockThreads, kMergeSmem, w->st>>>(S, (Cand*)w->merged.p, (int*)w->mcount.p);
    CHECK_LAUNCH();
    rescore_kernel<<<(k * 32 + 255) / 256, 256, 0, w->st>>>(D, T, o.order, (const Cand*)w->merged.p,
                                                             (const int*)w->mcount.p, (double*)w->fp64.p, nullptr);
    CHECK_LAUNCH();
    *launches += 2;
    std::vector<Cand> cands((size_t)k);
    std::vector<double> f64((size_t)k);
    int cnt = 0;
    CUDA_TRY(cudaMemcpyAsync(cands.data(), w->merged.p, sizeof(Cand) * k, cudaMemcpyDeviceToHost, w->st));
    CUDA_TRY(cudaMemcpyAsync(f64.data(), w->fp64.p, sizeof(double) * k, cudaMemcpyDeviceToHost, w->st));
    CUDA_TRY(cudaMemcpyAsync(&cnt, w->mcount.p, sizeof(int), cudaMemcpyDeviceToHost, w->st));
    int dev_err = 0;
    CUDA_TRY(cudaMemcpyAsync(&dev_err, w->tensor_flag.p, sizeof(int), cudaMemcpyDeviceToHost, w->st));
    CUDA_TRY(cudaEventRecord(w->e1, w->st));
    CUDA_TRY(cudaStreamSynchronize(w->st));
    w->d2h += (int64_t)(sizeof(Cand) + sizeof(double)) * k + 2 * sizeof(int);
    if (dev_err)
        return set_error(EPISDET_ERR_TIMEOUT, "a bounded device wait gave up (code %d); results discarded", dev_err);
    if (cnt < 1) return set_error(EPISDET_ERR_INTERNAL, "no candidate survived the search");
    for (int i = 0; i < cnt; ++i)
        if (std::isnan(f64[i])) return set_error(EPISDET_ERR_INTERNAL, "candidate %d holds an invalid SNP set", i);
    const bool maximize = o.score == EPISDET_SCORE_MI;
    int best = 0;
    for (int i = 1; i < cnt; ++i) {
        bool better = maximize ? f64[i] > f64[best] : f64[i] < f64[best];
        if (f64[i] == f64[best]) better = cands[i].set < cands[best].set;
        if (better) best = i;
    }
    auto unkey = [&](uint64_t s, uint32_t out[3]) {
        if (o.order == 2) {
            out[0] = (uint32_t)(s >> 32);
            out[1] = (uint32_t)(s & 0xFFFFFFFFu);
            out[2] = 0;
        } else {
            out[0] = (uint32_t)((s >> 42) & 0x1FFFFF);
            out[1] = (uint32_t)((s >> 21) & 0x1FFFFF);
            out[2] = (uint32_t)(s & 0x1FFFFF);
        }
    };
    unkey(cands[best].set, r->snps);
    r->score = f64[best];
    r->score_fp32 = key_score(cands[best].key, maximize);
    if (o.order == 2)
        r->packed_indices = (uint64_t)r->snps[0] | ((uint64_t)r->snps[1] << 32);
    else
        r->packed_indices = (uint64_t)r->snps[0] | ((uint64_t)r->snps[1] << 21) | ((uint64_t)r->snps[2] << 42);
    int outn = std::min(cnt, r->top_capacity > 0 ? r->top_capacity : 0);
    for (int i = 0; i < outn; ++i) {
        if (r->top_snps) unkey(cands[i].set, r->top_snps + 3 * (size_t)i);
        if (r->top_fp32) r->top_fp32[i] = key_score(cands[i].key, maximize);
        if (r->top_fp64) r->top_fp64[i] = f64[i];
    }
    r->top_count = outn;
    (void)D;
    (void)T;
    return EPISDET_OK;
}

episdet_status check_options(const episdet_options* in, int M, episdet_options* o) {
    episdet_options d;
    episdet_default_options(&d);
    *o = in ? *in : d;
    if (o->order != 2 && o->order != 3) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "order must be 2 or 3");
    if (o->score != EPISDET_SCORE_K2 && o->score != EPISDET_SCORE_MI)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown score %d", o->score);
    if (o->top_k <= 0) o->top_k = 1024;
    if (o->top_k > kMaxTopK) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "top_k must be <= %d", kMaxTopK);
    if (o->engine < EPISDET_ENGINE_AUTO || o->engine > EPISDET_ENGINE_SIMT)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown engine %d", o->engine);
    if (o->pair_block_snps < 0) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "pair_block_snps must be >= 0");
    if (o->first_end <= 0 || o->first_end > M) o->first_end = M;
    if (o->first_begin < 0 || o->first_begin >= o->first_end)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "empty first-SNP slab [%d,%d)", o->first_begin, o->first_end);
    if (o->first_begin > M - o->order)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "slab [%d,%d) holds no set", o->first_begin, o->first_end);
    return EPISDET_OK;
}

episdet_status check_dataset(const episdet_dataset* d, int order) {
    if (!d || !d->cases || !d->controls) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null dataset");
    if (d->num_snps < order) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "need at least %d SNPs", order);
    if (d->num_snps > (1 << 21) - 1)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "at most 2097151 SNPs (21-bit set packing)");
    if (d->num_cases < 1 || d->num_controls < 1)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "both classes need at least one sample");
    if ((int64_t)d->num_cases + d->num_controls > (1 << 30))
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "too many samples");
    if (d->memory != EPISDET_HOST && d->memory != EPISDET_DEVICE)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown memory kind %d", d->memory);
    return EPISDET_OK;
}

// The tensor engine sums each count over one K segment (a class, or the
// samples of one class with one genotype of the first SNP) in an FP32
// accumulator, exact while the segment holds at most 2^24 samples.  Larger
// classes go to the integer-pipe engine under EPISDET_ENGINE_AUTO and are
// refused for EPISDET_ENGINE_TENSOR.
bool tensor_exact_for(const episdet_dataset* d) {
    return d->num_cases <= kTensorMaxClass && d->num_controls <= kTensorMaxClass;
}

episdet_status check_engine(const episdet_dataset* d, const episdet_options& o) {
    if (o.engine == EPISDET_ENGINE_TENSOR && !tensor_exact_for(d))
        return set_error(EPISDET_ERR_UNSUPPORTED,
                         "the tensor engine counts a class in FP32 accumulators, exact up to %d samples per class "
                         "(got %d cases, %d controls); use EPISDET_ENGINE_AUTO or EPISDET_ENGINE_SIMT",
                         kTensorMaxClass, d->num_cases, d->num_controls);
    return EPISDET_OK;
}

}  // namespace episdet

using namespace episdet;

extern "C" void episdet_default_options(episdet_options* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->order = 3;
    o->score = EPISDET_SCORE_K2;
    o->top_k = 1024;
    o->device = 0;
    o->engine = EPISDET_ENGINE_AUTO;
}

namespace episdet {

// The body of one search; the caller holds w->mu and has validated o.
// ------------------------------------------------------------ autotuning
// The measured choice of triplet instance per shape (EPISDET_FLAG_AUTOTUNE),
// kept for the process and, when EPISDET_TUNE_CACHE names a file, read from it
// once and appended to it: one "order score bucket choice" line per shape,
// bucket = floor(log2(smaller class)).
static std::mutex g_tune_mu;
static std::map<int, int> g_tune;
static bool g_tune_loaded = false;

static int tune_key(int order, int score, int nc, int nn) {
    int m = std::max(1, std::min(nc, nn)), b = 0;
    while (m >>= 1) ++b;
    return (order << 16) | (score << 8) | b;
}

static void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("EPISDET_TUNE_CACHE");
    FILE* f = path && *path ? std::fopen(path, "r") : nullptr;
    if (!f) return;
    char line[128];
    while (std::fgets(line, sizeof(line), f)) {
        int order, score, bucket, choice;
        if (std::sscanf(line, "%d %d %d %d", &order, &score, &bucket, &choice) == 4 && (choice == 0 || choice == 1) &&
            order >= 2 && order <= 3 && score >= 0 && score <= 1 && bucket >= 0 && bucket < 64)
            g_tune[(order << 16) | (score << 8) | bucket] = choice;
    }
    std::fclose(f);
}

static int tune_lookup(int key) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(key);
    return it == g_tune.end() ? -1 : it->second;
}

static void tune_store(int key, int choice) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load_locked();
    g_tune[key] = choice;
    const char* path = std::getenv("EPISDET_TUNE_CACHE");
    if (FILE* f = path && *path ? std::fopen(path, "a") : nullptr) {
        std::fprintf(f, "%d %d %d %d\n", key >> 16, (key >> 8) & 0xFF, key & 0xFF, choice);
        std::fclose(f);
    }
}

// Times both triplet instances on the first 8 first SNPs of this search (two
// rounds, alternating, minimum per instance) and returns the staged one only
// when it is more than 3 % faster (probes share the GPU with any concurrent
// work).  With fewer cases than segment 0 needs to be staged (it holds cases
// only), the plain one is taken without a probe.
static episdet_status tune_probe(Workspace* w, const episdet_dataset* data, const episdet_options& o, int* choice) {
    if (data->num_cases < kStageMinSamples) {
        *choice = 0;
        return EPISDET_OK;
    }
    episdet_options po = o;
    po.flags = (o.flags & ~(EPISDET_FLAG_AUTOTUNE | EPISDET_FLAG_PROGRESS)) | EPISDET_FLAG_TIMING;
    po.first_begin = 0;
    po.first_end = std::min(data->num_snps, 8);
    double best[2] = {1e300, 1e300};
    for (int round = 0; round < 2; ++round)
        for (int c = 0; c < 2; ++c) {
            episdet_result r;
            memset(&r, 0, sizeof(r));
            w->stage_override = c;
            episdet_status st = search_locked(w, data, po, &r);
            w->stage_override = -1;
            if (st != EPISDET_OK) return st;
            best[c] = std::min(best[c], r.count_kernel_ms);
        }
    *choice = best[1] < 0.97 * best[0] ? 1 : 0;
    return EPISDET_OK;
}

episdet_status search_locked(Workspace* w, const episdet_dataset* data, const episdet_options& o,
                             episdet_result* result) {
    auto t0 = std::chrono::steady_clock::now();
    CUDA_TRY(cudaSetDevice(o.device));
    // Triplet instance for this call; reset on every return.
    struct Override {
        Workspace* w;
        ~Override() { w->stage_override = -1; }
    } reset{w};
    episdet_status st0 = check_engine(data, o);
    if (st0 != EPISDET_OK) return st0;
    const bool simt = o.engine == EPISDET_ENGINE_SIMT || !tensor_exact_for(data);
    if ((o.flags & EPISDET_FLAG_AUTOTUNE) && o.order == 3 && !simt) {
        const int key = tune_key(o.order, o.score, data->num_cases, data->num_controls);
        int choice = tune_lookup(key);
        if (choice < 0) {
            episdet_status st = tune_probe(w, data, o, &choice);
            if (st != EPISDET_OK) return st;
            tune_store(key, choice);
        }
        w->stage_override = choice;
    }
    begin_call(w, o);
    uint32_t* keep_snps = result->top_snps;
    float* keep32 = result->top_fp32;
    double* keep64 = result->top_fp64;
    int32_t keepcap = result->top_capacity;
    memset(result, 0, sizeof(*result));
    result->top_snps = keep_snps;
    result->top_fp32 = keep32;
    result->top_fp64 = keep64;
    result->top_capacity = keepcap;

    uint64_t launches = 0;
    DevData D;
    episdet_status st = stage_dataset(w, data, !(o.flags & EPISDET_FLAG_NO_VALIDATE), &D, &launches);
    if (st != EPISDET_OK) return st;
    ScoreTables T;
    st = build_tables(w, o.score, data->num_cases, data->num_controls, &T);
    if (st != EPISDET_OK) return st;
    const int fb = o.first_begin, fe = o.first_end;
    CUDA_TRY(cudaEventRecord(w->e0, w->st));
    Slots S;
    bool progress = (o.flags & EPISDET_FLAG_PROGRESS) != 0;
    if (simt)
        st = run_simt(w, D, T, o, fb, fe, &S, &launches, progress);
    else
        st = run_tensor(w, D, T, o, fb, fe, &S, &launches, progress);
    if (st != EPISDET_OK) return st;
    st = finish(w, D, T, o, S, result, &launches);
    if (st != EPISDET_OK) return st;
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, w->e0, w->e1));
    result->device_ms = ms;
    result->sets_evaluated = sets_in_slab(o.order, data->num_snps, fb, fe);
    result->rounds = reference_rounds(o.order, data->num_snps);
    result->kernel_launches = launches;
    result->count_kernel_launches = w->count_launches;
    result->executed_macs = w->executed_macs;
    result->h2d_bytes = w->h2d;
    result->d2h_bytes = w->d2h;
    if (w->timing) {
        double sum = 0.0;
        for (int i = 0; i + 1 < w->tev_used; i += 2) {
            float t = 0.0f;
            CUDA_TRY(cudaEventElapsedTime(&t, w->tev[i], w->tev[i + 1]));
            sum += t;
            w->launch_ms.push_back(t);
        }
        result->count_kernel_ms = sum;
        // A one-launch search (pairs, SIMT) issues all its MACs in that launch.
        if (w->launch_macs.size() != w->launch_ms.size())
            w->launch_macs.assign(w->launch_ms.size(), w->launch_ms.size() == 1 ? w->executed_macs : 0.0);
    }
    result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return EPISDET_OK;
}

}  // namespace episdet

extern "C" episdet_status episdet_search(const episdet_dataset* data, const episdet_options* opts,
                                         episdet_result* result) {
    clear_error();
    if (!result) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null result");
    if (!data) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null dataset");
    episdet_options o;
    episdet_status st = check_options(opts, data->num_snps, &o);
    if (st != EPISDET_OK) return st;
    st = check_dataset(data, o.order);
    if (st != EPISDET_OK) return st;
    st = check_engine(data, o);
    if (st != EPISDET_OK) return st;
    Workspace* w = nullptr;
    st = get_workspace(o.device, &w);
    if (st != EPISDET_OK) return st;
    std::lock_guard<std::mutex> lock(w->mu);
    return search_locked(w, data, o, result);
}

extern "C" const char* episdet_status_string(episdet_status s) {
    switch (s) {
        case EPISDET_OK: return "ok";
        case EPISDET_ERR_INVALID_ARGUMENT: return "invalid argument";
        case EPISDET_ERR_INVALID_INPUT: return "invalid input planes";
        case EPISDET_ERR_NO_DEVICE: return "no usable device";
        case EPISDET_ERR_CUDA: return "CUDA error";
        case EPISDET_ERR_OUT_OF_MEMORY: return "out of memory";
        case EPISDET_ERR_TIMEOUT: return "device wait timed out";
        case EPISDET_ERR_IO: return "I/O error";
        case EPISDET_ERR_UNSUPPORTED: return "unsupported";
        case EPISDET_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

extern "C" const char* episdet_last_error(void) { return g_err; }
extern "C" int32_t episdet_abi_version(void) { return EPISDET_ABI_VERSION; }

extern "C" episdet_status episdet_release_workspace(int32_t device) {
    if (device < 0 || device >= 64) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "device out of range");
    std::lock_guard<std::mutex> g(g_ws_mu);
    for (int lane = 0; lane < kMaxLanes; ++lane) {
        Workspace* w = g_ws[device][lane];
        if (!w) continue;
        std::lock_guard<std::mutex> l(w->mu);
        cudaSetDevice(device);
        w->release_all();
    }
    return EPISDET_OK;
}

extern "C" int64_t episdet_last_launch_profile(int32_t device, double* ms, double* macs, int64_t cap) {
    if (device < 0 || device >= 64) return 0;
    Workspace* w = nullptr;
    {
        std::lock_guard<std::mutex> g(g_ws_mu);
        w = g_ws[device][0];
    }
    if (!w) return 0;
    std::lock_guard<std::mutex> l(w->mu);
    const int64_t n = (int64_t)w->launch_ms.size();
    for (int64_t i = 0; i < std::min(n, cap); ++i) {
        if (ms) ms[i] = w->launch_ms[(size_t)i];
        if (macs) macs[i] = i < (int64_t)w->launch_macs.size() ? w->launch_macs[(size_t)i] : 0.0;
    }
    return n;
}

extern "C" void episdet_test_fail_allocation(int32_t after) { episdet::g_fail_alloc.store(after > 0 ? after : 0); }

extern "C" int32_t episdet_tuned_stage(int32_t order, int32_t score, int32_t num_cases, int32_t num_controls) {
    return episdet::tune_lookup(episdet::tune_key(order, score, num_cases, num_controls));
}
