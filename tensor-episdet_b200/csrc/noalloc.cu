// noalloc.cu -- a 2-way search that allocates no memory.
//
// Who needs it: callers that cannot let a library call cudaMalloc/cudaFree.
// Typical cases are a process whose memory pool or caching allocator has
// already reserved the GPU's memory (a new cudaMalloc would fail or fragment
// the pool), and pipelines running other streams that cannot absorb the
// device-wide synchronisation cudaFree implies.  episdet_search_pairs_noalloc
// runs the ordinary pairs search (marginals, fused integer-pipe counting with
// K2/MI scoring, candidate merge, FP64 re-score) but keeps every intermediate
// buffer in one file-scope device array of fixed size, kNoAllocScratchBytes.
// The caller provides the input planes already on the device and a host
// result struct; nothing else is allocated, on the device or the host heap.
//
// The array exists once per GPU that loads this library and stays allocated
// until the process exits.  Its device address is looked up once per device
// (cudaGetSymbolAddress, with that device current) on the first call, so the
// first call on a device should not be made while a stream is being captured.
// All calls share the array and it keeps whatever the last call left in it;
// the parts that must start at zero are cleared by every call.  Two calls
// whose GPU work overlapped would race on the array, so calls are serialised
// by a host lock and each call waits for its GPU work before returning, on
// its error paths too.  The looked-up address is kept for the process: after
// a cudaDeviceReset of a device the entry point must not be used on it again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "episdet.h"
#include "host_util.h"
#include "kernels.h"
#include "search_internal.h"

namespace episdet {
namespace noalloc {

// Limits of the fixed scratch (rejected with EPISDET_ERR_INVALID_ARGUMENT beyond them).
constexpr int kMaxSnps = 4096;
constexpr int kMaxSamples = 131072;  // cases + controls
constexpr int kMaxTopKNoAlloc = 1024;
constexpr int kMaxSlots = 320;       // persistent CTAs of the counting kernel
constexpr int kMaxTiles = (kMaxSnps / kSimtTileSnps) * (kMaxSnps / kSimtTileSnps + 1) / 2;
constexpr size_t kNoAllocScratchBytes = 8u << 20;  // 8 MiB per device

// Byte offsets of the regions inside the scratch array (each 256-aligned).
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffMarg = 0;                                                        // 2 x [3][M] int
constexpr size_t kOffFlag = align256(kOffMarg + 2 * 3 * (size_t)kMaxSnps * sizeof(int));
constexpr size_t kOffT32 = align256(kOffFlag + 16);                                   // [N+2] float
constexpr size_t kOffT64 = align256(kOffT32 + (kMaxSamples + 2) * sizeof(float));     // [N+2] double
constexpr size_t kOffTiles = align256(kOffT64 + (kMaxSamples + 2) * sizeof(double));  // [tiles] int2
constexpr size_t kOffSlots = align256(kOffTiles + kMaxTiles * sizeof(int2));          // [slots][k] Cand
constexpr size_t kOffCounts = align256(kOffSlots + (size_t)kMaxSlots * kMaxTopKNoAlloc * sizeof(Cand));
constexpr size_t kOffMerged = align256(kOffCounts + kMaxSlots * sizeof(int));         // [k] Cand
constexpr size_t kOffMcount = align256(kOffMerged + kMaxTopKNoAlloc * sizeof(Cand));
constexpr size_t kOffFp64 = align256(kOffMcount + 16);                                // [k] double
constexpr size_t kEnd = kOffFp64 + kMaxTopKNoAlloc * sizeof(double);
static_assert(kEnd <= kNoAllocScratchBytes, "scratch layout exceeds the array");

static __device__ __align__(256) uint8_t g_scratch[kNoAllocScratchBytes];

// Host-side staging, also fixed size (no heap use per call).
static float h_t32[kMaxSamples + 2];
static double h_t64[kMaxSamples + 2];
static int2 h_tiles[kMaxTiles];
static Cand h_cands[kMaxTopKNoAlloc];
static double h_fp64[kMaxTopKNoAlloc];

static std::mutex g_mu;
static uint8_t* g_dev_scratch[64] = {};  // device address of g_scratch, per device

// Once per device, with that device current.
static episdet_status setup(int device) {
    if (g_dev_scratch[device]) return EPISDET_OK;
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(EPISDET_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a only", device,
                         prop.major, prop.minor);
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    CUDA_TRY(cudaFuncSetAttribute(search2_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSimtSmem2));
    CUDA_TRY(cudaFuncSetAttribute(merge_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMergeSmem));
    g_dev_scratch[device] = (uint8_t*)p;
    return EPISDET_OK;
}

}  // namespace noalloc
}  // namespace episdet

using namespace episdet;
using namespace episdet::noalloc;

static episdet_status search_locked(const episdet_dataset* data, const episdet_options& o, uint8_t* S,
                                    cudaStream_t stream, episdet_result* result);

extern "C" episdet_status episdet_search_pairs_noalloc(const episdet_dataset* data, const episdet_options* opts,
                                                       episdet_result* result) {
    clear_error();
    if (!data || !result) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null dataset or result");
    episdet_options o;
    episdet_status st = check_options(opts, data->num_snps, &o);
    if (st != EPISDET_OK) return st;
    st = check_dataset(data, 2);
    if (st != EPISDET_OK) return st;
    if (o.order != 2) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "the no-alloc entry point searches pairs only");
    if (data->memory != EPISDET_DEVICE)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "the no-alloc entry point needs device-resident planes");
    if (((uintptr_t)data->cases | (uintptr_t)data->controls) & 15)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "device planes must be 16-byte aligned");
    const int M = data->num_snps, nc = data->num_cases, nn = data->num_controls;
    if (M > kMaxSnps || nc + nn > kMaxSamples || o.top_k > kMaxTopKNoAlloc)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT,
                         "no-alloc limits: at most %d SNPs, %d samples (cases + controls) and top_k %d "
                         "(got %d SNPs, %d samples, top_k %d)",
                         kMaxSnps, kMaxSamples, kMaxTopKNoAlloc, M, nc + nn, o.top_k);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(EPISDET_ERR_NO_DEVICE, "no CUDA device");
    }
    if (o.device < 0 || o.device >= ndev || o.device >= 64)
        return set_error(EPISDET_ERR_NO_DEVICE, "device %d not present", o.device);

    std::lock_guard<std::mutex> lock(g_mu);
    CUDA_TRY(cudaSetDevice(o.device));
    st = setup(o.device);
    if (st != EPISDET_OK) return st;
    cudaStream_t stream = (cudaStream_t)(uintptr_t)o.stream;
    st = search_locked(data, o, g_dev_scratch[o.device], stream, result);
    // Whatever failed, no GPU work of this call may still use the shared array
    // once the lock is released (the status of this wait is not the error).
    if (st != EPISDET_OK) cudaStreamSynchronize(stream);
    return st;
}

// The search proper, under g_mu with the device current and the array set up.
static episdet_status search_locked(const episdet_dataset* data, const episdet_options& o, uint8_t* S,
                                    cudaStream_t stream, episdet_result* result) {
    const int M = data->num_snps, nc = data->num_cases, nn = data->num_controls;

    uint32_t* keep_snps = result->top_snps;
    float* keep32 = result->top_fp32;
    double* keep64 = result->top_fp64;
    const int32_t keepcap = result->top_capacity;
    memset(result, 0, sizeof(*result));
    result->top_snps = keep_snps;
    result->top_fp32 = keep32;
    result->top_fp64 = keep64;
    result->top_capacity = keepcap;

    // Inputs, marginals and the input check.
    DevData D;
    memset(&D, 0, sizeof(D));
    D.M = M;
    D.bits[0] = data->cases;
    D.bits[1] = data->controls;
    D.n[0] = nc;
    D.n[1] = nn;
    D.W[0] = episdet_class_words(nc);
    D.W[1] = episdet_class_words(nn);
    int* marg0 = (int*)(S + kOffMarg);
    int* marg1 = marg0 + 3 * M;
    D.marg[0] = marg0;
    D.marg[1] = marg1;
    int* flag = (int*)(S + kOffFlag);
    CUDA_TRY(cudaMemsetAsync(flag, 0, 16, stream));
    uint64_t launches = 0;
    marginals_kernel<<<(2 * M * 32 + 255) / 256, 256, 0, stream>>>(D, marg0, marg1, flag);
    CHECK_LAUNCH();
    ++launches;
    int bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    if (bad && !(o.flags & EPISDET_FLAG_NO_VALIDATE))
        return set_error(EPISDET_ERR_INVALID_INPUT,
                         "input planes have padding bits set or overlapping genotype-0/1 planes");

    // Score tables, the same construction as every other entry point.
    const int N = nc + nn;
    const int size = o.score == EPISDET_SCORE_K2 ? N + 2 : N + 1;
    ScoreTables T;
    memset(&T, 0, sizeof(T));
    if (o.score == EPISDET_SCORE_K2) {
        for (int v = 0; v < size; ++v) {
            double g = lgamma((double)v + 1.0);
            h_t64[v] = g;
            h_t32[v] = (float)g;
        }
    } else {
        T.inv_n32 = (float)(1.0 / (double)N);
        T.inv_n64 = 1.0 / (double)N;
        h_t32[0] = 0.0f;
        h_t64[0] = 0.0;
        for (int v = 1; v < size; ++v) {
            h_t32[v] = (float)log2((double)v * (double)T.inv_n32);
            h_t64[v] = log2((double)v / (double)N);
        }
        double p1 = (double)nc * T.inv_n64, p2 = (double)nn * T.inv_n64;
        T.hy64 = -(p1 * h_t64[nc]) - (p2 * h_t64[nn]);
        T.hy32 = mi_hy32(nc, nn, T.inv_n32, h_t32);
    }
    T.score = o.score;
    T.t32 = (const float*)(S + kOffT32);
    T.t64 = (const double*)(S + kOffT64);
    CUDA_TRY(cudaMemcpyAsync(S + kOffT32, h_t32, sizeof(float) * size, cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(S + kOffT64, h_t64, sizeof(double) * size, cudaMemcpyHostToDevice, stream));

    // Upper-triangular tile list over the first-SNP slab.
    const int fb = o.first_begin, fe = o.first_end;
    const int nt = (M + kSimtTileSnps - 1) / kSimtTileSnps;
    int ntiles = 0;
    for (int a = fb / kSimtTileSnps; a <= (fe - 1) / kSimtTileSnps; ++a)
        for (int b = a; b < nt; ++b) h_tiles[ntiles++] = make_int2(a, b);
    CUDA_TRY(cudaMemcpyAsync(S + kOffTiles, h_tiles, sizeof(int2) * ntiles, cudaMemcpyHostToDevice, stream));

    // Counting with fused scoring, one persistent candidate list per CTA.
    int per_sm = 0, sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search2_simt_kernel, kSimtBlockThreads,
                                                           kSimtSmem2));
    const int grid = std::min(kMaxSlots, sms * std::max(per_sm, 1));
    Slots slots;
    slots.lists = (Cand*)(S + kOffSlots);
    slots.counts = (int*)(S + kOffCounts);
    slots.nslots = grid;
    slots.k = o.top_k;
    slots.gkey = nullptr;
    CUDA_TRY(cudaMemsetAsync(slots.counts, 0, sizeof(int) * grid, stream));
    search2_simt_kernel<<<grid, kSimtBlockThreads, kSimtSmem2, stream>>>(D, T, (const int2*)(S + kOffTiles), ntiles,
                                                                          fb, fe, slots, 0, nullptr, nullptr);
    CHECK_LAUNCH();
    Cand* merged = (Cand*)(S + kOffMerged);
    int* mcount = (int*)(S + kOffMcount);
    double* fp64 = (double*)(S + kOffFp64);
    merge_topk_kernel<<<1, kMergeBlockThreads, kMergeSmem, stream>>>(slots, merged, mcount);
    CHECK_LAUNCH();
    rescore_kernel<<<(o.top_k * 32 + 255) / 256, 256, 0, stream>>>(D, T, 2, merged, mcount, fp64, nullptr);
    CHECK_LAUNCH();
    launches += 3;
    int cnt = 0;
    CUDA_TRY(cudaMemcpyAsync(h_cands, merged, sizeof(Cand) * o.top_k, cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaMemcpyAsync(h_fp64, fp64, sizeof(double) * o.top_k, cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaMemcpyAsync(&cnt, mcount, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    if (cnt < 1) return set_error(EPISDET_ERR_INTERNAL, "no candidate survived the search");
    for (int i = 0; i < cnt; ++i)
        if (std::isnan(h_fp64[i])) return set_error(EPISDET_ERR_INTERNAL, "candidate %d holds an invalid SNP set", i);

    // FP64 optimum, ties to the lowest set.
    const bool maximize = o.score == EPISDET_SCORE_MI;
    int best = 0;
    for (int i = 1; i < cnt; ++i) {
        bool better = maximize ? h_fp64[i] > h_fp64[best] : h_fp64[i] < h_fp64[best];
        if (h_fp64[i] == h_fp64[best]) better = h_cands[i].set < h_cands[best].set;
        if (better) best = i;
    }
    result->snps[0] = (uint32_t)(h_cands[best].set >> 32);
    result->snps[1] = (uint32_t)(h_cands[best].set & 0xFFFFFFFFu);
    result->snps[2] = 0;
    result->packed_indices = (uint64_t)result->snps[0] | ((uint64_t)result->snps[1] << 32);
    result->score = h_fp64[best];
    result->score_fp32 = key_score(h_cands[best].key, maximize);
    const int outn = std::min(cnt, std::max(result->top_capacity, 0));
    for (int i = 0; i < outn; ++i) {
        if (result->top_snps) {
            result->top_snps[3 * i + 0] = (uint32_t)(h_cands[i].set >> 32);
            result->top_snps[3 * i + 1] = (uint32_t)(h_cands[i].set & 0xFFFFFFFFu);
            result->top_snps[3 * i + 2] = 0;
        }
        if (result->top_fp32) result->top_fp32[i] = key_score(h_cands[i].key, maximize);
        if (result->top_fp64) result->top_fp64[i] = h_fp64[i];
    }
    result->top_count = outn;
    int64_t sets = 0;
    for (int a = fb; a < fe; ++a) sets += M - 1 - a;
    result->sets_evaluated = sets;
    const int64_t nb = (M + 255) / 256;
    result->rounds = nb * (nb + 1) / 2;
    result->kernel_launches = launches;
    result->count_kernel_launches = 1;
    return EPISDET_OK;
}
