// tensor.cu -- tcgen05 (5th-generation tensor core) counting engine.
//
// Counting is a matrix product over 0/1 operand rows: for rows a, b (one per
// {SNP, genotype} bit plane) sum_s a[s]*b[s] is the AND-popcount the reference
// computes as (popc a + popc b - popc(a^b))/2 from its CUTLASS XOR GEMM
// (src/helper.cu:636-637, :484-485, :714-750).  Two operand forms:
//   * packed e2m1 (1.0 = nibble 2, two samples per byte), multiplied by
//     tcgen05.mma.cta_group::2.kind::mxf4 with unit block scales and FP32
//     accumulation (exact below 2^24): the pair kernel tc_kernel<true, ...>,
//     used for triplets and for the 2-way search;
//   * 0/1 bytes, multiplied by tcgen05.mma.cta_group::1.kind::i8 (u8 x u8 ->
//     s32): tc_kernel<false, ...>, used for the 3-way pair table.
//
// Pipeline per CTA (one CTA per SM, persistent over a tile list):
//   warp 0      TMA producer: 128-byte K blocks of the A and B row blocks,
//               128-byte swizzle, 4-stage mbarrier ring (no multicast).
//   warp 1      MMA issuer (the even CTA of a pair issues for both),
//               accumulators in TMEM (512 columns).
//   warps 2..9  epilogue: tcgen05.ld of the counts, derivation of the 9 / 27
//               contingency cells, K2 / MI score, per-CTA top-K candidates.
//               No count ever returns to HBM.
//
// Pair-kernel tiles are M = 256 A rows (128 SNPs x 2 planes; each CTA holds
// 128 rows = 64 SNPs) by N = 112 B rows (56 SNPs x 2 planes; each CTA loads 56
// of them); counts are kept per K segment:
//   pairs:    segments {cases, controls}                 -> 2 x 112 columns, two sets
//   triplets: segments {cases, controls} x {X genotype a, X genotype b}
//                                                        -> 4 x 112 columns, one set
// For triplets the sample columns are regrouped per first SNP X by X's
// genotype (xinfo/transpose/regroup kernels below), keeping the two genotypes of X with
// the fewest samples; the third is recovered from the Y-Z pair table exactly
// as the reference recovers genotype 2 (src/helper.cu:494-548).  This replaces
// the materialised X AND Y operand of src/helper.cu:396-425 and reduces the
// tensor work per triplet from 8 N to 4 (N - max_g count(X=g)) MACs.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "device_data.cuh"
#include "host_util.h"
#include "search_internal.h"
#include "tc_ptx.cuh"

namespace episdet {
namespace tc {

constexpr int kTileSnps = 64;
constexpr int kTileRows = 128;
constexpr int kKB = 128;  // bytes per K block: 128 byte samples (pairs), 256 packed e2m1 samples (triplets)
constexpr int kTileBytes = kTileRows * kKB;  // one 128-row operand tile of one K block
// Triplet operands are packed e2m1 (1.0 for a set bit, 0 otherwise), two
// samples per byte, multiplied by kind::mxf4 with unit block scales.
constexpr int kF4PerKB = 2 * kKB;  // samples per triplet K block
constexpr int kZSnpsPair = 56;      // B SNPs per triplet tile (N = 112 rows)
constexpr int kNPair = 2 * kZSnpsPair;
// Packed samples per class region of a regrouped row: two segments padded to
// whole K blocks need at most n + 2 * (kF4PerKB - 1) <= Kc + kClassPad.
constexpr int kClassPad = 2 * kF4PerKB;
constexpr int kCap = 2048;  // k <= kMaxTopK kept plus one step of offers
// Warp 0 issues TMA, warp 1 MMAs; warps 2..9 are the epilogue, two per TMEM
// lane quarter (warp % 4), each taking half of the 128 accumulator columns in
// chunks of 8 columns (4 B SNPs x 2 planes; each lane scores 2 of the 4).
constexpr int kThreads = 320;
constexpr int kEpiThreads = 256;
constexpr int kEpiPerStep = kEpiThreads * 2;
static_assert(kMaxTopK + kEpiPerStep <= kCap, "candidate buffer too small for one step of offers");
// The filtered K2 triplet instances keep their candidate buffer in global
// memory and check its fill once per tile: room for k plus a whole tile's
// offers (each epilogue thread scores 2 sets in each of its 7 chunks).
constexpr int kCapG = 8192;
// Filtered K2 triplet instances: operand K blocks prefetched into L2 this far
// ahead of the stage loads.
constexpr int kPrefetchKb = 8;
constexpr int kEpiPerTile = kEpiThreads * 2 * (kNPair / 16);
static_assert(kMaxTopK + kEpiPerTile <= kCapG, "global candidate buffer too small for one tile of offers");
// Waits for work (operand copies, MMA commits, the scoring warps) give up
// after TcParams::wait_ns.  Drains before exit wait for the copies and MMAs
// still in flight: up to kDrainLimitNs, or kAbortDrainNs once the CTA is
// aborting (a copy the peer CTA never issued must not hold the drain up; the
// pause before exit covers copies still landing).
constexpr uint64_t kDrainLimitNs = 4000000000ull;
constexpr uint64_t kAbortDrainNs = 2000000ull;
constexpr uint64_t kAbortPauseNs = 200000ull;
constexpr uint32_t kIdesc = ptx::idesc_u8(128);
constexpr uint32_t kIdescPair = ptx::idesc_mxf4(kNPair, 256);  // CTA-pair e2m1 MMA, M = 256, N = 112
// TMEM of the pair kernel: four 112-column count segments (triplets: one
// accumulator set of four; pairs: two sets of two), then the block
// scale factors (every byte 1.0 = UE8M0 127) in columns kSfCol .. 511.
constexpr uint32_t kSfCol = 4 * kNPair;

enum Mode { kPairsScore = 0, kPairsStore = 1, kTriplets = 2 };

struct Seg {
    int kb0, kb1;  // K-block range [kb0, kb1)
};

// Per-X sample regrouping: genotypes ga and gb of X are kept (ga the larger
// group), gd (the largest) is derived.
struct XInfo {
    int gd, ga, gb, pad;
    int len[2][2];  // [class][kept genotype] samples
    Seg seg[4];     // [class*2 + kept genotype]
};

constexpr int kMaxGroup = kXGroup;  // first SNPs (X) per triplet launch
constexpr int kStageMin = kStageMinSamples;  // samples of segment 0 from which the staged kernel copies it out
constexpr int kStageClass = 32768;  // class size from which triplet launches use the staged kernel
constexpr int kBand = 12;     // tile-band edge of the triplet tile order

// Tensor maps of a launch, one per X (each X has its own regrouped operand
// rows): m[g] reads 128-row boxes; the CTA-pair kernel also uses m[kMaxGroup + g],
// 64-row boxes of the same rows for its half of the B operand.
struct TmapPack {
    CUtensorMap m[2 * kMaxGroup];
};

// Tiles [cum, next cum) of a launch belong to group member g: X = x, list tiles.
struct GroupDesc {
    const int2* tiles;  // (A tile, B tile) in 64-SNP units
    int cum;
    int x;
    const XInfo* xinfo;
};

// A window of the 3-way pair table: cells of pair (r, col) at
// p[c][(r - r0) * ld + (col - c0)] for class c, rows r >= r0, columns col > r.
struct PairView {
    const uint4* p[2];
    int r0, c0;
    long ld;
};

__device__ __forceinline__ uint4 pair_at(const PairView& v, int c, int r, int col) {
    return __ldg(v.p[c] + (size_t)(r - v.r0) * (size_t)v.ld + (size_t)(col - v.c0));
}

struct TcParams {
    DevData D;
    ScoreTables T;
    Slots S;
    int ngroup;
    int ntiles;  // total over the group
    GroupDesc grp[kMaxGroup];
    int mode;
    Seg seg2[2];
    int first_begin, first_end;
    uint4* pair_out0;
    uint4* pair_out1;
    int out_r0, out_c0;  // store mode: pair (r, col) at pair_out[(r - out_r0) * out_ld + (col - out_c0)]
    long out_ld;
    // Triplets: X-Y and X-Z cells from xv, Y-Z cells from yv (one view of the
    // whole table, or a block of Y rows and the rows of the current X values).
    PairView xv, yv;
    int* err;
    Cand* cbuf;        // kFeatGlobalCands instances: [grid][kCapG] candidate buffers in global memory
    // 2-way label mode: [M][M] AND cells of every pair over all samples of the
    // cohort; the controls' cells are these minus the cases' (no control MMAs).
    const uint4* tot;
    uint64_t wait_ns;  // limit of every wait for work
    const int* hold;   // failure-detection test: a word the scoring warps wait for (nothing sets it), or null
};

// Waits until *word != 0; false after limit_ns.
__device__ __forceinline__ bool wait_word(const int* word, uint64_t limit_ns) {
    const uint64_t t0 = ptx::globaltimer();
    while (*(const volatile int*)word == 0) {
        if (ptx::globaltimer() - t0 > limit_ns) return false;
        __nanosleep(2000);
    }
    return true;
}

// Drain wait for copies or MMAs in flight: gives up after kDrainLimitNs, or
// after kAbortDrainNs once *abort is set.
__device__ __forceinline__ bool drain_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
    if (ptx::mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = ptx::globaltimer();
    for (uint32_t it = 1;; ++it) {
        if (ptx::mbar_try_wait(bar, parity)) return true;
        if ((it & 255) == 0) {
            const uint64_t dt = ptx::globaltimer() - t0;
            if (dt > kDrainLimitNs || (*abort && dt > kAbortDrainNs)) return false;
        }
    }
}

// Features of a kernel instance (a bit mask):
//   kFeatFilter       K2 scoring filter (k2_approx32); only a 32-entry table in
//                     shared memory;
//   kFeatBigStages    stages of four K blocks (one MMA commit per 16 MMAs: a
//                     commit costs the tensor pipe about as much as four MMAs
//                     of this shape, profiles/tcgen05_mma_peak.md), two of them
//                     (2 x 94 KB; three stages of two K blocks ran 2 % slower);
//   kFeatGlobalCands  candidate buffer in a global per-CTA region, its fill
//                     checked once per tile;
//   kFeatMidStages    stages of two K blocks (one commit per 8 MMAs), three of
//                     them: for the MI triplet instance, whose exact scoring
//                     keeps a 32 KB table in shared memory (5 % faster than
//                     four stages of one K block on the 8192 x 65536 MI
//                     workload), and the 2-way instances;
//   kFeatOpPrefetch   operand K blocks prefetched into L2 ahead of the stage loads;
//   kFeatPairPrefetch the Y-Z and X-Z pair-table rows of a tile prefetched into
//                     L2 while its MMAs run.
enum : int {
    kFeatFilter = 1,
    kFeatBigStages = 2,
    kFeatGlobalCands = 4,
    kFeatOpPrefetch = 8,
    kFeatPairPrefetch = 16,
    kFeatMidStages = 32
};

// Shared-memory layout of tc_kernel<PAIR, STAGE, FEAT>.  A K block holds
// 128 bytes of this CTA's 128 A rows and of its B rows: all 128 for one CTA,
// 56 of the pair's 112 for a CTA pair (PAIR), where the other CTA of the pair
// holds the rest.  A stage holds kKbPerStage K blocks and is released by one
// MMA commit.
template <bool PAIR, bool STAGE = false, int FEAT = 0>
struct Cfg {
    static constexpr bool FILTER = (FEAT & kFeatFilter) != 0;
    static constexpr bool GCANDS = (FEAT & kFeatGlobalCands) != 0;
    static constexpr int kKbPerStage = (FEAT & kFeatBigStages) ? 4 : (FEAT & kFeatMidStages) ? 2 : 1;
    static constexpr int kStages = (FEAT & kFeatBigStages) ? 2 : (FEAT & kFeatMidStages) ? 3 : 4;
    static constexpr int kBRows = PAIR ? kZSnpsPair : 128;
    static constexpr int kNSeg = PAIR ? kNPair : 128;      // accumulator columns per count segment
    static constexpr int kZSnps = PAIR ? kZSnpsPair : kTileSnps;  // B SNPs per tile
    static constexpr int kChunks = kNSeg / 16;              // 8-column chunks per epilogue warp
    static constexpr int kKbBytes = kTileBytes + kBRows * kKB;  // A then B of one K block
    static constexpr int kStageBytes = kKbPerStage * kKbBytes;
    static constexpr size_t kSmemTopk = (size_t)kStages * kStageBytes;
    // FP32 score table entries kept in shared memory: kSmallTab (the filter's)
    // or kLoTab (exact scoring of every set).
    static constexpr int kLoEntries = FILTER ? kSmallTab : kLoTab;
    // The candidate buffer: in shared memory, or (GCANDS) in a global per-CTA
    // region, leaving the shared memory to the stages and to L1.
    static constexpr size_t kSmemLo = kSmemTopk + (GCANDS ? 0 : (size_t)kCap * sizeof(Cand));
    // STAGE: count segment 0 of the tile copied out of TMEM as 16-bit counts,
    // [epilogue thread][chunk] x 8 columns.
    static constexpr size_t kSmemStage = kSmemLo + (size_t)kLoEntries * sizeof(float);
    static constexpr size_t kSmemBars = kSmemStage + (STAGE ? (size_t)kEpiThreads * kChunks * sizeof(uint4) : 0);
    static constexpr int kNumBars = 2 * kStages + 5;  // full, empty, tfull[2], tempty[2], drain
    static constexpr size_t kSmemMisc = kSmemBars + ((kNumBars * sizeof(uint64_t) + 63) & ~size_t(63));
    static constexpr size_t kSmemGroup = kSmemMisc + 64;
    static constexpr size_t kSmemTotal = kSmemGroup + 256 + 1024;
    static_assert(kSmemTotal <= 232448, "tc_kernel shared memory exceeds 227 KB");
    static_assert(kKbBytes % 1024 == 0 && kTileBytes % 1024 == 0, "operand tiles must stay 1024-byte aligned");
};

// The configuration of one kernel instance, used by the kernel and by every
// host-side launch and attribute, so the two can never disagree on the layout.
// The K2 triplet instances of large searches (the headline search) filter,
// run stages of four K blocks, keep their candidates in global memory and
// prefetch their pair-table rows; operand prefetch (kFeatOpPrefetch) measured
// slower and is off.  The MI triplet instances run stages of two K blocks with
// their candidates in global memory, the 2-way instances stages of two K
// blocks (15 % faster on 16384 SNPs x 32768 samples); the exact K2 triplet and
// pair-table instances keep the plain layout (stages of two K blocks were 3 %
// slower for exact K2 triplets).
// VAR = 1 selects these features for a K2 triplet instance; the host runs it
// for searches large enough that each CTA scores far more sets than its
// candidate list holds (kFilterMinSetsPerCta), and the plain K2 instance
// (VAR = 0, exact scoring from a shared-memory table) for smaller ones, where
// the filter's warm-up -- every set scored exactly until the lists fill --
// is most of the search.
template <bool PAIR, bool TWO, int SC, int VAR>
constexpr int kInstanceFeat = (PAIR && !TWO && SC == 0 && VAR == 1)
                                  ? (kFeatFilter | kFeatBigStages | kFeatGlobalCands | kFeatPairPrefetch)
                              : (PAIR && !TWO && SC == 1) ? (kFeatMidStages | kFeatGlobalCands)
                              : (PAIR && TWO)             ? kFeatMidStages
                                                          : 0;
template <bool PAIR, bool STAGE, int SC = -1, bool TWO = false, int VAR = 0>
using KCfg = Cfg<PAIR, STAGE, kInstanceFeat<PAIR, TWO, SC, VAR>>;
constexpr double kFilterMinSetsPerCta = 1.0e7;

// Per-launch copy of each group member's segments in shared memory.
struct GroupSm {
    Seg seg[4];
    int ga, gb, x, empty_mask;
    // Pair kernel: when the counts of segment 0 (cases, X = ga) fit 16 bits,
    // the epilogue copies that segment out of TMEM first and releases its
    // columns early, so the next tile's segment-0 MMAs overlap the epilogue.
    int stage_ok, pad;
};
static_assert(sizeof(GroupSm) * kMaxGroup <= 256, "group table size");

__device__ __forceinline__ int group_of(const TcParams& P, int t) {
    int g = 0;
#pragma unroll
    for (int i = 1; i < kMaxGroup; ++i)
        if (i < P.ngroup && t >= P.grp[i].cum) g = i;
    return g;
}

// ------------------------------------------------------------ operand prep
// Packed planes -> 0/1 bytes.  Row r = 2*snp + g holds the cases' bytes in
// [0, Kc) and the controls' in [Kc, Kc + Kn) of a pitch-Kc+Kn row.
__global__ void __launch_bounds__(256) unpack_kernel(DevData D, uint8_t* __restrict__ out, int rows, int pitch) {
    const int Kc = D.W[0] * 32;
    const int chunks = pitch / 16;
    long total = (long)rows * chunks;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        int r = (int)(t / chunks);
        int k = (int)(t % chunks) * 16;
        int c = k < Kc ? 0 : 1;
        int kk = k - (c ? Kc : 0);
        uint32_t word = __ldg(D.bits[c] + (size_t)r * D.W[c] + (kk >> 5));
        uint32_t h = (word >> (16 - (kk & 31))) & 0xFFFFu;
        uint32_t o[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            uint32_t n = (h >> (12 - 4 * e)) & 0xFu;  // 4 samples, first sample in bit 3
            o[e] = ((n >> 3) & 1u) | ((n << 6) & 0x100u) | ((n << 15) & 0x10000u) | ((n << 24) & 0x1000000u);
        }
        *reinterpret_cast<uint4*>(out + (size_t)r * pitch + k) = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// Packed planes -> packed e2m1 operand rows of the 2-way pair kernel, in the
// class-region layout of the regrouped triplet rows (no regrouping): row
// r = 2*snp + g holds the cases from packed sample 0 and the controls from
// packed sample Kc + kClassPad, 1.0 (nibble 2) for a set bit, two samples per
// byte with the even one in the low nibble.  One thread per source word.
__global__ void __launch_bounds__(256) pack_f4_kernel(DevData D, uint8_t* __restrict__ out, int rows, int pitch) {
    const int W0 = D.W[0], W1 = D.W[1], wpr = W0 + W1;
    const int base1 = (W0 * 32 + kClassPad) / 2;  // byte offset of the controls' region
    const long total = (long)rows * wpr;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int r = (int)(t / wpr), w = (int)(t % wpr);
        const int c = w < W0 ? 0 : 1;
        const int ww = w - (c ? W0 : 0);
        const uint32_t word = __ldg(D.bits[c] + (size_t)r * D.W[c] + ww);  // sample ww*32 + i at bit 31 - i
        uint32_t o[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            uint32_t v = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) v |= ((word >> (31 - (8 * e + i))) & 1u) << (4 * i + 1);
            o[e] = v;
        }
        *reinterpret_cast<uint4*>(out + (size_t)r * pitch + (c ? base1 : 0) + (size_t)ww * 16) =
            make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// Block-wide exclusive scan of one int per thread (at most 1024 threads).
__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int* total) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
        int z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xFFFFFFFFu, z, o);
            if (lane >= o) z += y;
        }
        s_warp[lane] = z - w;
        if (lane == 31) *total = z;
    }
    __syncthreads();
    int r = s_warp[warp] + x - v;
    __syncthreads();
    return r;
}

// Per first SNP X and class: which genotype of X to derive (the most frequent
// over both classes), and the ascending sample indices of the two kept ones.
// Regrouping work of the first SNPs X0 .. X0 + gridDim.y - 1 of one launch: member
// m = blockIdx.y owns the XInfo and index lists at base + m * stride bytes.
struct XWork {
    uint8_t* base;     // member 0's XInfo, its index lists info_bytes after it
    size_t stride;     // bytes between members
    size_t info_bytes;
    int x0;
    int max_n;
    __device__ __forceinline__ XInfo* info(int m) const { return reinterpret_cast<XInfo*>(base + m * stride); }
    __device__ __forceinline__ int* idx(int m) const { return reinterpret_cast<int*>(base + m * stride + info_bytes); }
};

constexpr int kXinfoThreads = 256;
__global__ void __launch_bounds__(kXinfoThreads) xinfo_kernel(DevData D, XWork xw) {
    __shared__ int s_warp[32];
    __shared__ int s_total;
    const int c = blockIdx.x;
    const int X = xw.x0 + (int)blockIdx.y;
    XInfo* info = xw.info(blockIdx.y);
    int* idx = xw.idx(blockIdx.y);
    const int max_n = xw.max_n;
    const int M = D.M;
    int tot[3];
#pragma unroll
    for (int g = 0; g < 3; ++g) tot[g] = __ldg(D.marg[0] + g * M + X) + __ldg(D.marg[1] + g * M + X);
    int gd = 0;
    if (tot[1] > tot[gd]) gd = 1;
    if (tot[2] > tot[gd]) gd = 2;
    // Kept genotypes; segment 0 holds the larger group (the pair kernel
    // copies segment 0 out of TMEM early to overlap the next tile's MMAs).
    const int o1 = gd == 0 ? 1 : 0, o2 = gd == 2 ? 1 : 2;
    const int ga = tot[o2] > tot[o1] ? o2 : o1, gb = ga == o1 ? o2 : o1;
    const int W = D.W[c], n = D.n[c];
    const uint32_t* p0 = D.bits[c] + (size_t)X * 2 * W;
    const uint32_t* p1 = p0 + W;
    const int per = (W + blockDim.x - 1) / blockDim.x;
    const int w0 = threadIdx.x * per, w1 = min(W, w0 + per);
    // Class 1's region starts after class 0's Kc + kClassPad packed samples.
    const int base_kb = c == 0 ? 0 : (D.W[0] * 32 + kClassPad) / kF4PerKB;
    int kb = base_kb;
    for (int s = 0; s < 2; ++s) {
        const int g = s == 0 ? ga : gb;
        int cnt = 0;
        for (int w = w0; w < w1; ++w) {
            uint32_t m = g == 0 ? p0[w] : (g == 1 ? p1[w] : ~(p0[w] | p1[w]));
            int lo = w * 32;
            uint32_t valid = (lo + 32 <= n) ? 0xFFFFFFFFu : (lo >= n ? 0u : (0xFFFFFFFFu << (32 - (n - lo))));
            cnt += __popc(m & valid);
        }
        int off = block_exclusive_scan(cnt, s_warp, &s_total);
        int* out = idx + ((size_t)c * 2 + s) * max_n;
        for (int w = w0; w < w1; ++w) {
            uint32_t m = g == 0 ? p0[w] : (g == 1 ? p1[w] : ~(p0[w] | p1[w]));
            int lo = w * 32;
            uint32_t valid = (lo + 32 <= n) ? 0xFFFFFFFFu : (lo >= n ? 0u : (0xFFFFFFFFu << (32 - (n - lo))));
            m &= valid;
            while (m) {
                int lz = __clz(m);
                out[off++] = lo + lz;
                m &= ~(0x80000000u >> lz);
            }
        }
        int len = s_total;
        if (threadIdx.x == 0) {
            info->len[c][s] = len;
            info->seg[c * 2 + s].kb0 = kb;
            info->seg[c * 2 + s].kb1 = kb + (len + kF4PerKB - 1) / kF4PerKB;
        }
        kb += (len + kF4PerKB - 1) / kF4PerKB;
        __syncthreads();
    }
    if (c == 0 && threadIdx.x == 0) {
        info->gd = gd;
        info->ga = ga;
        info->gb = gb;
        info->pad = 0;
    }
}

// Regrouped operand rows for one X: row r, class c, segment s holds the e2m1
// value bit(r, idx[c][s][k]) (1.0 = nibble 2, 0.0 = nibble 0) at packed sample
// position seg.kb0*256 + k, two samples per byte, the even one in the low
// nibble (zero past the segment's length up to its 256-sample end).  Rows
// below row0 are not needed by X.
//
// Output rows of the members of one launch: member m = blockIdx.z writes rows
// [row0[m], nrows_total) of out[m].
struct CmpOut {
    uint8_t* out[kMaxGroup];
    int row0[kMaxGroup];
};

// ------------------------------------------------- sample-major regrouping
// Gathering single bits of the plane rows costs about ten instructions per
// output byte, and a kernel doing that beside the counting kernel slowed it by
// 15 %.  Instead the planes are transposed once per search into sample-major
// words (tt[c][s][q]: bit 31 - i is row 32 q + i at sample s), so that
// gathering a sample is a 128-byte copy, and the gathered block is turned
// back into rows by a 32 x 32 bit transpose in registers (five shuffle
// stages).

// 32 x 32 bit transpose across a warp: lane k returns the word whose bit
// 31 - l is bit 31 - k of lane l's word (the block-swap transpose of
// H. S. Warren, Hacker's Delight, 2nd ed., section 7-3, one stage per
// shuffle distance).
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t a, int lane) {
    uint32_t m = 0x0000FFFFu;
#pragma unroll
    for (int j = 16; j != 0; j >>= 1, m ^= m << j) {
        const uint32_t p = __shfl_xor_sync(0xFFFFFFFFu, a, j);
        if (lane & j) {
            a ^= ((p ^ (a >> j)) & m) << j;
        } else {
            a ^= (a ^ (p >> j)) & m;
        }
    }
    return a;
}

// Rows padded to whole 256-row tiles in the sample-major layout.
constexpr int kTtRows = 256;
__host__ __device__ inline int tt_row_words(int rows) { return (rows + kTtRows - 1) / kTtRows * (kTtRows / 32); }

// Planes of class c -> tt (one warp per 256 rows x 256 samples: eight
// 32-byte reads of eight rows' words per lane, eight 32-byte writes).
constexpr int kTtThreads = 256;
__global__ void __launch_bounds__(kTtThreads) transpose_planes_kernel(DevData D, int c, uint32_t* __restrict__ tt,
                                                                      int rows, int rwp) {
    const int lane = threadIdx.x & 31;
    const int warp = (int)(blockIdx.x * (kTtThreads / 32) + threadIdx.x / 32);
    const int W = D.W[c];
    const int nqb = rwp / 8, nsb = W / 8;
    if (warp >= nqb * nsb) return;  // uniform over the warp
    const int qb = warp % nqb, sb = warp / nqb;
    const uint32_t* __restrict__ bits = D.bits[c];
    uint32_t out[8][8];  // [sample word][row word]
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int r = (qb * 8 + q) * 32 + lane;
        uint4 v0 = make_uint4(0, 0, 0, 0), v1 = v0;
        if (r < rows) {
            const uint4* src = reinterpret_cast<const uint4*>(bits + (size_t)r * W + sb * 8);
            v0 = __ldg(src);
            v1 = __ldg(src + 1);
        }
        const uint32_t v[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
        for (int e = 0; e < 8; ++e) out[e][q] = warp_transpose32(v[e], lane);
    }
    // Lane k now holds, for sample 32 (sb*8 + e) + k, the words of rows
    // 32 (qb*8 + q) .. + 31 (bit 31 - i = row 32 (qb*8 + q) + i).
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        uint4* dst = reinterpret_cast<uint4*>(tt + (size_t)((sb * 8 + e) * 32 + lane) * rwp + qb * 8);
        dst[0] = make_uint4(out[e][0], out[e][1], out[e][2], out[e][3]);
        dst[1] = make_uint4(out[e][4], out[e][5], out[e][6], out[e][7]);
    }
}

// Regrouped operand rows for the members of one launch (the layout above),
// from tt: a work item is kRgRows rows x 256 packed sample positions (one K
// block) of one class region of one member.  Each thread copies the 128 bytes
// of its position's source sample (these rows: one cache line) into shared
// memory; then each lane transposes one 32 rows x 32 positions block in its
// own registers (no shuffles) and writes its 32 rows' 16 bytes, the eight
// lanes of the same rows writing whole 128-byte lines.
constexpr int kRgThreads = 256;
constexpr int kRgRows = 1024;
constexpr int kRgWords = kRgRows / 32;  // row words per position
// [position][row word] with 33 words a position and 4 more each 32 positions,
// so that both the per-position writes and the per-block column reads (lanes
// of 4 row words x 8 position blocks) are free of bank conflicts.
__host__ __device__ constexpr int rg_slot(int pos, int q) { return pos * (kRgWords + 1) + 4 * (pos >> 5) + q; }
constexpr int kRgTBytes = 4 * (rg_slot(kRgThreads - 1, kRgWords - 1) + 1);
// The allocation also keeps the kernel's CTAs off the SMs of a running
// counting CTA (172 KB): the regrouping ran beside the counting kernel at the
// cost of 15 % of the counting rate, more than it saved.
constexpr int kRgSmem = 64 * 1024;
static_assert(kRgTBytes <= kRgSmem, "regroup tile");

// e2m1 nibbles of 8 positions (bit e of b = position e): 1.0 = 2 in nibble e,
// the even position in the low nibble of each byte.  Bit e moves to bit
// 4 e + 1 by three shift-and-mask spreading steps.
__device__ __forceinline__ uint32_t e2m1_nibbles8(uint32_t b) {
    uint32_t v = (b | (b << 12)) & 0x000F000Fu;
    v = (v | (v << 6)) & 0x03030303u;
    v = (v | (v << 3)) & 0x11111111u;
    return v << 1;
}

// 32 x 32 bit transpose of a[0..31] in place: afterwards bit 31 - l of a[k]
// is what bit 31 - k of a[l] was (the block-swap transpose of H. S. Warren,
// Hacker's Delight, 2nd ed., section 7-3).
__device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
    uint32_t m = 0x0000FFFFu;
#pragma unroll
    for (int j = 16; j != 0; j >>= 1, m ^= m << j) {
#pragma unroll
        for (int k = 0; k < 32; k = (k + j + 1) & ~j) {
            const uint32_t t = (a[k] ^ (a[k + j] >> j)) & m;
            a[k] ^= t;
            a[k + j] ^= t << j;
        }
    }
}

// Persistent: a CTA claims work items (member, class K block, row tile) from
// a launch-wide counter (*ctr, zero at launch), skipping those past a
// member's region or below its first row, and loads the next item's source
// samples into registers while it turns the current one into rows.  Claiming
// (rather than a fixed share per CTA) balances the items over CTAs that start
// late: the launch begins on the SMs the previous counting launch frees.
__global__ void __launch_bounds__(kRgThreads, 2)
    regroup_kernel(DevData D, XWork xw, CmpOut co, const uint32_t* __restrict__ tt0, const uint32_t* __restrict__ tt1,
                   int rwp, int rows_total, int pitch, int nmem, int* __restrict__ ctr) {
    extern __shared__ __align__(16) uint32_t s_t[];  // rg_slot(position, row word)
    __shared__ int s_len[kMaxGroup][2][2];           // [member][class][segment]: samples
    __shared__ int s_claim;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t < 4 * nmem) {
        const int m = t >> 2, c = (t >> 1) & 1, sg = t & 1;
        s_len[m][c][sg] = xw.info(m)->len[c][sg];
    }
    __syncthreads();
    const int T0 = (D.W[0] * 32 + kClassPad) / kF4PerKB;
    const int KT = T0 + (D.W[1] * 32 + kClassPad) / kF4PerKB;
    const int RT = (rows_total + kRgRows - 1) / kRgRows;
    const int nitems = nmem * KT * RT;
    // Item i: row tile i % RT, K block (i / RT) % KT of the two class regions,
    // member i / (RT * KT).  Invalid items are skipped (uniformly).
    auto decode = [&](int i, int& m, int& c, int& k0, int& rt) -> bool {
        rt = i % RT;
        const int kt = (i / RT) % KT;
        m = i / (RT * KT);
        c = kt < T0 ? 0 : 1;
        k0 = (kt - (c ? T0 : 0)) * kF4PerKB;
        const int pa = (s_len[m][c][0] + kF4PerKB - 1) / kF4PerKB * kF4PerKB;
        const int pb = (s_len[m][c][1] + kF4PerKB - 1) / kF4PerKB * kF4PerKB;
        return k0 < pa + pb && (rt + 1) * kRgRows > co.row0[m];
    };
    // The next claimed item that is valid (nitems when none is left); called
    // by every thread, between barriers on s_claim.
    auto next_valid = [&](int& m, int& c, int& k0, int& rt) {
        for (;;) {
            if (t == 0) s_claim = atomicAdd(ctr, 1);
            __syncthreads();
            const int i = s_claim;
            __syncthreads();
            if (i >= nitems) return nitems;
            if (decode(i, m, c, k0, rt)) return i;
        }
    };
    // This thread's position of an item: its source sample's 128 bytes of the row tile.
    auto load = [&](int m, int c, int k0, int rt, uint4 (&v)[kRgWords / 4]) {
        const int la = s_len[m][c][0], pa = (la + kF4PerKB - 1) / kF4PerKB * kF4PerKB, lb = s_len[m][c][1];
        const int k = k0 + t;
        const int* __restrict__ idx = xw.idx(m) + (size_t)c * 2 * xw.max_n;
        int src = -1;
        if (k < pa) {
            if (k < la) src = __ldg(idx + k);
        } else if (k - pa < lb) {
            src = __ldg(idx + xw.max_n + (k - pa));
        }
        // Row words past the padded row count (the last tile) read as zero.
        const int nw = min(kRgWords, rwp - rt * kRgWords);
        const uint4* p =
            reinterpret_cast<const uint4*>((c ? tt1 : tt0) + (size_t)max(src, 0) * rwp + rt * kRgWords);
#pragma unroll
        for (int e = 0; e < kRgWords / 4; ++e)
            v[e] = (src >= 0 && 4 * e < nw) ? __ldg(p + e) : make_uint4(0, 0, 0, 0);
    };
    // This lane's block: row word q (rows 32 q .. 32 q + 31 of the tile) and
    // positions 32 j .. 32 j + 31.
    const int q = 4 * w + (lane >> 3), j = lane & 7;
    int m, c, k0, rt;
    int i = next_valid(m, c, k0, rt);
    uint4 v[kRgWords / 4];
    if (i < nitems) load(m, c, k0, rt, v);
    while (i < nitems) {
#pragma unroll
        for (int e = 0; e < kRgWords / 4; ++e) {
            s_t[rg_slot(t, 4 * e)] = v[e].x, s_t[rg_slot(t, 4 * e + 1)] = v[e].y;
            s_t[rg_slot(t, 4 * e + 2)] = v[e].z, s_t[rg_slot(t, 4 * e + 3)] = v[e].w;
        }
        __syncthreads();
        const int cm = m, cc = c, ck0 = k0, crt = rt;
        i = next_valid(m, c, k0, rt);
        if (i < nitems) load(m, c, k0, rt, v);  // lands while this item is turned into rows
        uint32_t a[32];
        // a[p]: bit 31 - r is row 32 q + r at position 32 j + p.
#pragma unroll
        for (int p = 0; p < 32; ++p) a[p] = s_t[rg_slot(32 * j + p, q)];
        transpose32(a);  // a[r]: bit 31 - p is row 32 q + r at position 32 j + p
        const int row0 = co.row0[cm];
        uint8_t* __restrict__ out =
            co.out[cm] + ((cc ? D.W[0] * 32 + kClassPad : 0) + ck0) / 2 + 16 * j;
        const int rbase = crt * kRgRows + 32 * q;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            const uint32_t x = __brev(a[r]);
            const int row = rbase + r;
            if (row >= row0 && row < rows_total)
                *reinterpret_cast<uint4*>(out + (size_t)row * pitch) =
                    make_uint4(e2m1_nibbles8(x & 255u), e2m1_nibbles8((x >> 8) & 255u),
                               e2m1_nibbles8((x >> 16) & 255u), e2m1_nibbles8(x >> 24));
        }
        __syncthreads();  // s_t is refilled next
    }
}

__device__ __forceinline__ void record_error(int* err, int code) { atomicCAS(err, 0, code); }

// ------------------------------------------------------------------ kernel
// PAIR: launched as clusters of two CTAs that share each M = 256 x N = 112
// kind::mxf4 tile (cta_group::2): the even CTA's MMA warp issues for both,
// each CTA holds the accumulators of its 128 A rows and scores them; triplets,
// or pairs with TWO.  Without PAIR: the kind::i8 single-CTA kernel (pair
// table).  STAGE: count segment 0 is copied out of TMEM early (triplets).
// One CTA of ten warps per SM: up to 168 registers a thread (three warps on
// some SM sub-partition).  The regrouping kernel does not share its SMs (its
// shared memory does not fit beside a counting CTA), so nothing else needs
// them; at 144 the filtered K2 instances spilled and ran 2.5 % slower.
// SC: the score fixed at compile time (0 = K2, 1 = MI) or -1 (read at run time).
// TWO: the pair kernel scoring pairs (two class segments, two accumulator sets)
// instead of counting triplets.
// FILTER (the K2 triplet instances): each set's K2 score is first bounded
// without table reads (k2_approx32); only sets that may be better than the
// CTA's current k-th candidate are scored exactly (from the global table),
// so the candidate lists are those of scoring every set.
template <bool PAIR, bool STAGE, int SC = -1, bool TWO = false, int VAR = 0>
__global__ void __launch_bounds__(kThreads, 1)
    tc_kernel(const __grid_constant__ TmapPack tm, const __grid_constant__ TcParams P) {
    static_assert(PAIR || !STAGE, "staging is a pair-kernel mode");
    static_assert(!TWO || (PAIR && !STAGE), "the 2-way pair kernel is the plain pair instance");
    using C = KCfg<PAIR, STAGE, SC, TWO, VAR>;
    constexpr bool FILTER = C::FILTER;
    constexpr bool GCANDS = C::GCANDS;
    constexpr bool OPF = (kInstanceFeat<PAIR, TWO, SC, VAR> & kFeatOpPrefetch) != 0;
    constexpr bool PPF = (kInstanceFeat<PAIR, TWO, SC, VAR> & kFeatPairPrefetch) != 0;
    constexpr int kStages = C::kStages;
    constexpr int kStageBytes = C::kStageBytes;
    constexpr int kKbBytes = C::kKbBytes;
    constexpr int kKbPer = C::kKbPerStage;
    extern __shared__ uint8_t smem_raw[];
    // A launch with less dynamic shared memory than this instance's layout
    // needs is refused before anything touches it (uniform over the CTA and
    // the pair, so no barrier is left waiting).
    {
        uint32_t dyn;
        asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (dyn < (uint32_t)C::kSmemTotal) {
            if (threadIdx.x == 0) record_error(P.err, 7);
            return;
        }
    }
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* stages = smem;
    Cand* tbuf = GCANDS ? P.cbuf + (size_t)blockIdx.x * kCapG : reinterpret_cast<Cand*>(smem + C::kSmemTopk);
    float* s_lo = reinterpret_cast<float*>(smem + C::kSmemLo);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::kSmemBars);
    uint64_t* full = bars;
    uint64_t* empty = bars + kStages;
    uint64_t* tfull = bars + 2 * kStages;
    uint64_t* tempty = bars + 2 * kStages + 2;
    uint64_t* drain = bars + 2 * kStages + 4;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + C::kSmemMisc);
    int* s_abort = reinterpret_cast<int*>(smem + C::kSmemMisc + 4);
    int* s_never = reinterpret_cast<int*>(smem + C::kSmemMisc + 8);  // stays 0: drain waits ignore aborts
    int* s_epi_fail = reinterpret_cast<int*>(smem + C::kSmemMisc + 12);
    int* s_count = reinterpret_cast<int*>(smem + C::kSmemMisc + 16);
    Cand* s_thr = reinterpret_cast<Cand*>(smem + C::kSmemMisc + 32);
    uint4* s_stage = reinterpret_cast<uint4*>(smem + C::kSmemStage);
    volatile int* abort = s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    GroupSm* s_grp = reinterpret_cast<GroupSm*>(smem + C::kSmemGroup);
    const int mode = PAIR ? (TWO ? (int)kPairsScore : (int)kTriplets) : P.mode;
    const int nseg = mode == kTriplets ? 4 : 2;
    const int nbuf = 4 / nseg;
    if (threadIdx.x < P.ngroup) {
        GroupSm gs;
        if (mode == kTriplets) {
            const XInfo* xi = P.grp[threadIdx.x].xinfo;
            for (int s = 0; s < 4; ++s) gs.seg[s] = xi->seg[s];
            gs.ga = xi->ga;
            gs.gb = xi->gb;
        } else {
            gs.seg[0] = P.seg2[0];
            gs.seg[1] = P.seg2[1];
            gs.seg[2] = gs.seg[3] = Seg{0, 0};
            gs.ga = 0;
            gs.gb = 1;
        }
        gs.x = P.grp[threadIdx.x].x;
        gs.empty_mask = 0;
        for (int s = 0; s < 4; ++s)
            if (gs.seg[s].kb1 <= gs.seg[s].kb0) gs.empty_mask |= 1 << s;
        gs.pad = 0;
        // A count of the segment is at most its sample count; short segments
        // are not worth the copy.
        const int len0 = STAGE && mode == kTriplets ? P.grp[threadIdx.x].xinfo->len[0][0] : 0;
        gs.stage_ok = len0 >= kStageMin && len0 <= 65535;
        s_grp[threadIdx.x] = gs;
    }

    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            ptx::mbar_init(&full[i], 1);
            ptx::mbar_init(&empty[i], 1);
        }
        for (int b = 0; b < 2; ++b) {
            ptx::mbar_init(&tfull[b], 1);
            ptx::mbar_init(&tempty[b], PAIR ? 2 * (kEpiThreads / 32) : kEpiThreads);
        }
        ptx::mbar_init(drain, 1);
        *s_abort = 0;
        *s_never = 0;
        *s_epi_fail = 0;
        ptx::fence_barrier_init();
    }
    if (warp == 1) {
        if constexpr (PAIR) {
            ptx::tmem_alloc_pair(s_tmem, 512);
            ptx::tmem_relinquish_pair();
        } else {
            ptx::tmem_alloc(s_tmem, 512);
            ptx::tmem_relinquish();
        }
    }
    if (warp == 0 && lane < P.ngroup) {
        ptx::prefetch_tmap(&tm.m[lane]);
        if (PAIR) ptx::prefetch_tmap(&tm.m[kMaxGroup + lane]);
    }
    // The pair's barriers must be initialised before either CTA touches the other's.
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const int rank = PAIR ? (int)ptx::cluster_ctarank() : 0;
    const int t_first = PAIR ? (int)ptx::cluster_id_x() : (int)blockIdx.x;
    const int t_step = PAIR ? (int)ptx::nclusters_x() : (int)gridDim.x;
    if constexpr (PAIR) {
        // Block scale factors of every pair MMA: 1.0 in each byte of columns
        // kSfCol .. 511 of this CTA's TMEM, written before any MMA is issued.
        if (warp >= 2) {
            const uint32_t sf = tmem + ((uint32_t)((warp & 3) * 32) << 16) + kSfCol + (uint32_t)(((warp - 2) >> 2) * 32);
#pragma unroll
            for (int c = 0; c < 32; c += 8) ptx::tmem_st8_fill(sf + (uint32_t)c, 0x7F7F7F7Fu);
            ptx::tmem_wait_st();
        }
        ptx::tc_fence_before();
        ptx::cluster_sync();
        ptx::tc_fence_after();
    }

    if (warp == 0) {
        // ---------------------------------------------------- TMA producer
        if (lane == 0) {
            uint32_t stage = 0, phase = 0;
            uint32_t pend_phase[kStages];
            bool pend[kStages];
#pragma unroll
            for (int i = 0; i < kStages; ++i) {
                pend[i] = false;
                pend_phase[i] = 0;
            }
            bool ok = true, issued = false;
            // The even CTA arms each stage's full barrier for both CTAs' bytes;
            // the odd CTA's copies count on that barrier too.
            const uint32_t full0 = PAIR ? ptx::mapa(full, 0) : 0u;
            for (int t = t_first; ok && t < P.ntiles; t += t_step) {
                const int g = group_of(P, t);
                const int2 tl = P.grp[g].tiles[t - P.grp[g].cum];
                const Seg* seg = s_grp[g].seg;
                const CUtensorMap* tmap = &tm.m[g];
                const CUtensorMap* tmapb = PAIR ? &tm.m[kMaxGroup + g] : tmap;
                const int arow0 = PAIR ? tl.x * 2 * kTileRows + rank * kTileRows : tl.x * kTileRows;
                const int brow0 = PAIR ? tl.y * kNPair + rank * C::kBRows : tl.y * kTileRows;
                for (int s = 0; ok && s < nseg; ++s) {
                    for (int kb = seg[s].kb0; kb < seg[s].kb1; kb += kKbPer) {
                        // A stage holds up to kKbPer K blocks of one segment.
                        const int nkb = min(kKbPer, seg[s].kb1 - kb);
                        if (!ptx::mbar_wait(&empty[stage], phase ^ 1, abort, P.wait_ns)) {
                            ok = false;
                            break;
                        }
                        uint8_t* sa = stages + (size_t)stage * kStageBytes;
                        if constexpr (OPF) {
                            // The K blocks kPrefetchKb ahead (same segment) into
                            // L2, so that stage loads rarely wait for DRAM.
#pragma unroll
                            for (int j = 0; j < kKbPer; ++j) {
                                const int pk = kb + j + kPrefetchKb;
                                if (j < nkb && pk < seg[s].kb1) {
                                    ptx::tma_prefetch_2d(tmap, pk * kKB, arow0);
                                    ptx::tma_prefetch_2d(tmapb, pk * kKB, brow0);
                                }
                            }
                        }
                        if constexpr (PAIR) {
                            if (rank == 0) ptx::mbar_arrive_expect_tx(&full[stage], (uint32_t)(2 * nkb * kKbBytes));
                            const uint32_t fb = full0 + (uint32_t)(stage * sizeof(uint64_t));
#pragma unroll
                            for (int j = 0; j < kKbPer; ++j)
                                if (j < nkb) {
                                    ptx::tma_load_2d_pair(sa + j * kKbBytes, tmap, (kb + j) * kKB, arow0, fb);
                                    ptx::tma_load_2d_pair(sa + j * kKbBytes + kTileBytes, tmapb, (kb + j) * kKB, brow0,
                                                          fb);
                                }
                        } else {
                            ptx::mbar_arrive_expect_tx(&full[stage], (uint32_t)(nkb * kKbBytes));
#pragma unroll
                            for (int j = 0; j < kKbPer; ++j)
                                if (j < nkb) {
                                    ptx::tma_load_2d(sa + j * kKbBytes, tmap, (kb + j) * kKB, arow0, &full[stage]);
                                    ptx::tma_load_2d(sa + j * kKbBytes + kTileBytes, tmapb, (kb + j) * kKB, brow0,
                                                     &full[stage]);
                                }
                        }
                        issued = true;
                        pend[stage] = !PAIR || rank == 0;  // completions land on the even CTA's barriers
                        pend_phase[stage] = phase;
                        if (++stage == kStages) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
            }
            if (!ok) {
                record_error(P.err, 1);
                *s_abort = 1;
            }
            (void)issued;
            // Never leave with a copy in flight: the even CTA's barriers count
            // both CTAs' copies; the odd CTA's copies of a stage the even CTA
            // never armed land during the pause before exit (see the end).
            for (int i = 0; i < kStages; ++i)
                if (pend[i] && !drain_wait(&full[i], pend_phase[i], abort)) record_error(P.err, 2);
        }
    } else if (warp == 1) {
        // ---------------------------------------------------- MMA issuer
        // (for a CTA pair, the even CTA issues every MMA of the pair)
        if (lane == 0 && rank == 0) {
            uint32_t stage = 0, phase = 0;
            bool ok = true;
            int local = 0;
            for (int t = t_first; ok && t < P.ntiles; t += t_step, ++local) {
                const GroupSm& gs = s_grp[group_of(P, t)];
                const Seg* seg = gs.seg;
                const int b = local % nbuf;
                const uint32_t use = (uint32_t)(local / nbuf);
                // Pair kernel: segment 0's columns are free once both CTAs'
                // epilogues have copied out (or finished with) the previous tile's.
                if constexpr (STAGE) {
                    if (!ptx::mbar_wait_cluster(&tempty[1], (use & 1) ^ 1, abort, P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                }
                // The other segments wait for the whole accumulator set to be
                // drained by both CTAs' epilogues.
                const int late_at = (STAGE && gs.stage_ok) ? 1 : 0;
                const uint32_t dbase = tmem + (uint32_t)(b * nseg * C::kNSeg);
                for (int s = 0; ok && s < nseg; ++s) {
                    if (s == late_at) {
                        const bool freed = PAIR ? ptx::mbar_wait_cluster(&tempty[b], (use & 1) ^ 1, abort, P.wait_ns)
                                                : ptx::mbar_wait(&tempty[b], (use & 1) ^ 1, abort, P.wait_ns);
                        if (!freed) {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                    }
                    const uint32_t dseg = dbase + (uint32_t)(s * C::kNSeg);
                    for (int kb = seg[s].kb0; kb < seg[s].kb1; kb += kKbPer) {
                        const int nkb = min(kKbPer, seg[s].kb1 - kb);
                        if (!ptx::mbar_wait(&full[stage], phase, abort, P.wait_ns)) {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
#pragma unroll
                        for (int j = 0; j < kKbPer; ++j) {
                            if (j >= nkb) break;
                            const uint32_t sa = ptx::smem_u32(stages + (size_t)stage * kStageBytes + j * kKbBytes);
                            const uint64_t ad = ptx::smem_desc_sw128(sa), bd = ptx::smem_desc_sw128(sa + kTileBytes);
#pragma unroll
                            for (int kk = 0; kk < kKB / 32; ++kk) {
                                const uint32_t acc = (kb + j > seg[s].kb0 || kk > 0) ? 1u : 0u;
                                if constexpr (PAIR)
                                    ptx::mma_mxf4_pair(dseg, ad + 2 * kk, bd + 2 * kk, kIdescPair, tmem + kSfCol,
                                                       tmem + kSfCol + 32, acc);
                                else
                                    ptx::mma_u8(dseg, ad + 2 * kk, bd + 2 * kk, kIdesc, acc);
                            }
                        }
                        if constexpr (PAIR)
                            ptx::mma_commit_pair_mc(&empty[stage], 0x3);  // frees the stage in both CTAs
                        else
                            ptx::mma_commit(&empty[stage]);
                        if (++stage == kStages) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
                if (ok) {
                    if constexpr (PAIR)
                        ptx::mma_commit_pair_mc(&tfull[b], 0x3);
                    else
                        ptx::mma_commit(&tfull[b]);
                }
            }
            if (!ok) {
                record_error(P.err, 3);
                *s_abort = 1;
            }
            // Every MMA this thread issued completes before TMEM is released.
            if constexpr (PAIR)
                ptx::mma_commit_pair_mc(drain, 0x1);
            else
                ptx::mma_commit(drain);
            if (!ptx::mbar_wait(drain, 0, s_never, kDrainLimitNs)) record_error(P.err, 4);
        }
    } else {
        // ---------------------------------------------------- epilogue
        const int etid = threadIdx.x - 64;
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int ch0 = ((warp - 2) >> 2) * C::kChunks;  // first of this warp's 8-column chunks
        const int m = q * 32 + lane;
        const int yl = m >> 1, j_own = m & 1;
        const int zoff = j_own ? 2 : 0;
        const BarNamed bar{1, kEpiThreads};
        const bool maximize = SC >= 0 ? SC == 1 : P.T.score == 1;
        const int M = P.D.M;
        LocalTopK<GCANDS ? kCapG : kCap, kEpiThreads> tk{tbuf, s_count, s_thr, P.S.k, etid, P.S.gkey};
        // The candidate buffer takes at most kEpiPerStep offers per chunk; its
        // fill is checked after every chunk.  (Checking less often would need
        // that many more free slots, i.e. a lower fill limit and more sorts.)
        int hi = 0;  // this thread's highest candidate slot + 1 since the last compaction
        const LutShared lut{s_lo, P.T.t32};
        if (mode != kPairsStore) {
            // Low end of the FP32 table (every index the scorer can read is < N + 2).
            const int nlo = min(P.D.n[0] + P.D.n[1] + 2, C::kLoEntries);
            for (int i = etid; i < nlo; i += kEpiThreads) s_lo[i] = __ldg(P.T.t32 + i);
            tk.load(P.S.lists + (size_t)blockIdx.x * P.S.k, P.S.counts[blockIdx.x], bar);
        }
        bool ok = true;
        int local = 0;
        for (int t = t_first; t < P.ntiles; t += t_step, ++local) {
            const int b = local % nbuf;
            const uint32_t use = (uint32_t)(local / nbuf);
            const int g = group_of(P, t);
            const int2 tl = P.grp[g].tiles[t - P.grp[g].cum];
            if constexpr (PPF) {
                // While this tile's MMAs run, bring its Y-Z and X-Z pair-table
                // rows into L2 (one row of 56 entries per thread and class).
                const int bz0 = tl.y * C::kZSnps;
                if (etid < 2 * kTileSnps + 2) {
                    const bool yrow = etid < 2 * kTileSnps;
                    const int c = yrow ? etid / kTileSnps : etid - 2 * kTileSnps;
                    const int row = yrow ? tl.x * 2 * kTileSnps + rank * kTileSnps + etid % kTileSnps : s_grp[g].x;
                    const PairView& v = yrow ? P.yv : P.xv;
                    // Columns past the row only (the view holds no others).
                    const int z0 = max(bz0, row + 1);
                    const int nz = min(bz0 + C::kZSnps, M) - z0;
                    if (row < M && nz > 0)
                        ptx::prefetch_l2(v.p[c] + (size_t)(row - v.r0) * (size_t)v.ld + (size_t)(z0 - v.c0),
                                         (uint32_t)nz * 16u);
                }
            }
            // The decision to leave must be uniform over the 256 epilogue
            // threads (they meet at named barriers), so it is taken after a
            // barrier from a flag only they write.
            if (local == 0 && P.hold && !wait_word(P.hold, P.wait_ns)) *s_epi_fail = 1;
            if (!*(volatile int*)s_epi_fail && !ptx::mbar_wait(&tfull[b], use & 1, abort, P.wait_ns)) *s_epi_fail = 1;
            bar();
            if (*(volatile int*)s_epi_fail) {
                ok = false;
                break;
            }
            ptx::tc_fence_after();
            const int ga = s_grp[g].ga, gb = s_grp[g].gb, emask = s_grp[g].empty_mask;
            const bool stg = STAGE && s_grp[g].stage_ok;
            // This thread's A SNP (pairs: a, triplets: Y); a pair tile spans 128 A SNPs.
            const int arow = PAIR ? tl.x * 2 * kTileSnps + rank * kTileSnps + yl : tl.x * kTileSnps + yl;
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * nseg * C::kNSeg);
            if constexpr (STAGE) {
                if (stg) {
                    // Copy this thread's columns of segment 0 to shared memory
                    // as 16-bit counts, then release them to the next tile's
                    // first MMAs.
                    for (int ch = ch0; ch < ch0 + C::kChunks; ++ch) {
                        uint32_t w[8];
                        __syncwarp();
                        ptx::tmem_ld8(trow + (uint32_t)(ch * 8), w);
                        ptx::tmem_wait_ld();
                        ptx::tmem_regs_ready(w);
                        uint32_t h[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            h[e] = (uint32_t)(int)__uint_as_float(w[2 * e]) |
                                   ((uint32_t)(int)__uint_as_float(w[2 * e + 1]) << 16);
                        s_stage[etid * C::kChunks + (ch - ch0)] = make_uint4(h[0], h[1], h[2], h[3]);
                    }
                    ptx::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) ptx::mbar_arrive_cluster(ptx::mapa(&tempty[1], 0));
                }
            }
            // Per-row constants.
            int ma[2][3] = {{0, 0, 0}, {0, 0, 0}}, mx[2][3] = {{0, 0, 0}, {0, 0, 0}};
            int xy9[2][9];
            const int X = s_grp[g].x;
            const bool row_ok = arow < M && (mode != kTriplets || arow > X);
            // (store mode needs no marginals: the pair-total launch passes none)
            if (row_ok && mode != kPairsStore) {
#pragma unroll
                for (int c = 0; c < 2; ++c) load_marg3(P.D.marg[c], M, arow, ma[c]);
                if (mode == kTriplets) {
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        load_marg3(P.D.marg[c], M, X, mx[c]);
                        pair9_from4(xy9[c], pair_at(P.xv, c, X, arow), mx[c], ma[c]);
                    }
                }
            }
            for (int ch = ch0; ch < ch0 + C::kChunks; ++ch) {
                uint32_t v[4][8];
                __syncwarp();
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (s < nseg) {
                        if (s == 0 && stg) {
                            const uint4 h = s_stage[etid * C::kChunks + (ch - ch0)];
                            const uint32_t hw[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
                            for (int e = 0; e < 8; ++e)
                                v[s][e] = __float_as_uint((float)((hw[e >> 1] >> (16 * (e & 1))) & 0xFFFFu));
                        } else {
                            ptx::tmem_ld8(trow + (uint32_t)(s * C::kNSeg + ch * 8), v[s]);
                        }
                    }
                ptx::tmem_wait_ld();
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (s < nseg) ptx::tmem_regs_ready(v[s]);
                if (ch == ch0 + C::kChunks - 1) {
                    ptx::tc_fence_before();
                    if constexpr (PAIR) {
                        // One arrival per warp, on the even CTA's barriers: the
                        // whole set (b == 0), and segment 0 unless it was staged.
                        __syncwarp();
                        if (lane == 0) {
                            ptx::mbar_arrive_cluster(ptx::mapa(&tempty[b], 0));
                            if (STAGE && !stg) ptx::mbar_arrive_cluster(ptx::mapa(&tempty[1], 0));
                        }
                    } else {
                        ptx::mbar_arrive(&tempty[b]);
                    }
                }
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (s >= nseg || ((emask >> s) & 1))
#pragma unroll
                        for (int e = 0; e < 8; ++e) v[s][e] = 0;
                // Partner lane (other plane of the same A SNP) sends the counts of our 2 B SNPs.
                uint32_t r[4][4];
#pragma unroll
                for (int s = 0; s < 4; ++s)
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        r[s][e] = __shfl_xor_sync(0xFFFFFFFFu, j_own ? v[s][e] : v[s][4 + e], 1);
                Cand thr = *s_thr;
                // FILTER: the smaller of this CTA's and the search-wide k-th
                // best FP32 score so far (+inf until some CTA held k candidates).
                uint32_t thr_key = thr.key;
                if constexpr (FILTER) thr_key = min(thr_key, *(volatile uint32_t*)P.S.gkey);
                const float thr_s = thr_key == 0xFFFFFFFFu ? __int_as_float(0x7F800000) : key_score(thr_key, false);
                (void)thr_s;
#pragma unroll
                for (int z = 0; z < 2; ++z) {
                    const int bsnp = tl.y * C::kZSnps + ch * 4 + zoff + z;
                    // cnt(s, jj, kk): A plane jj, B plane kk, segment s
                    auto cnt = [&](int s, int jj, int kk) -> int {
                        const uint32_t own = j_own ? v[s][4 + 2 * z + kk] : v[s][2 * z + kk];
                        const uint32_t raw = jj == j_own ? own : r[s][2 * z + kk];
                        // Pair counts accumulate in FP32, exact below 2^24.
                        return PAIR ? (int)__uint_as_float(raw) : (int)raw;
                    };
                    if (mode == kPairsStore) {
                        if (row_ok && arow < bsnp && bsnp < M) {
                            const size_t o =
                                (size_t)(arow - P.out_r0) * (size_t)P.out_ld + (size_t)(bsnp - P.out_c0);
                            P.pair_out0[o] = make_uint4(cnt(0, 0, 0), cnt(0, 0, 1), cnt(0, 1, 0), cnt(0, 1, 1));
                            if (P.pair_out1)
                                P.pair_out1[o] = make_uint4(cnt(1, 0, 0), cnt(1, 0, 1), cnt(1, 1, 0), cnt(1, 1, 1));
                        }
                        continue;
                    }
                    if (mode == kPairsScore) {
                        if (!(row_ok && arow < bsnp && bsnp < M && arow >= P.first_begin && arow < P.first_end))
                            continue;
                        int cs[9], cn[9], mb[3];
                        cs[0] = cnt(0, 0, 0);
                        cs[1] = cnt(0, 0, 1);
                        cs[3] = cnt(0, 1, 0);
                        cs[4] = cnt(0, 1, 1);
                        load_marg3(P.D.marg[0], M, bsnp, mb);
                        derive9(cs, ma[0], mb);
                        if (P.tot) {
                            // Label mode: controls = all samples - cases.
                            const uint4 t = __ldg(P.tot + (size_t)arow * M + bsnp);
                            cn[0] = (int)t.x - cs[0];
                            cn[1] = (int)t.y - cs[1];
                            cn[3] = (int)t.z - cs[3];
                            cn[4] = (int)t.w - cs[4];
                        } else {
                            cn[0] = cnt(1, 0, 0);
                            cn[1] = cnt(1, 0, 1);
                            cn[3] = cnt(1, 1, 0);
                            cn[4] = cnt(1, 1, 1);
                        }
                        load_marg3(P.D.marg[1], M, bsnp, mb);
                        derive9(cn, ma[1], mb);
                        float sc = score32_lut<9, LutShared, SC>(P.T, lut, cs, cn);
                        Cand cd;
                        cd.key = score_key(sc, maximize);
                        cd.pad = 0;
                        cd.set = set_key2((uint32_t)arow, (uint32_t)bsnp);
                        tk.offer(cd, thr, hi);
                        continue;
                    }
                    // triplets: X < Y = arow < Z = bsnp
                    if (!(row_ok && arow < bsnp && bsnp < M)) continue;
                    int tab[2][27];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        int mz[3], xz9[9], yz9[9];
                        load_marg3(P.D.marg[c], M, bsnp, mz);
                        const uint4 yz = pair_at(P.yv, c, arow, bsnp);
                        const int yz4[4] = {(int)yz.x, (int)yz.y, (int)yz.z, (int)yz.w};
#pragma unroll
                        for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                            for (int kk = 0; kk < 2; ++kk) {
                                const int g0 = cnt(2 * c, jj, kk), g1 = cnt(2 * c + 1, jj, kk);
                                const int gdv = yz4[jj * 2 + kk] - g0 - g1;
                                tab[c][EPI_C3(0, jj, kk)] = ga == 0 ? g0 : (gb == 0 ? g1 : gdv);
                                tab[c][EPI_C3(1, jj, kk)] = ga == 1 ? g0 : (gb == 1 ? g1 : gdv);
                            }
                        pair9_from4(xz9, pair_at(P.xv, c, X, bsnp), mx[c], mz);
                        pair9_from4(yz9, yz, ma[c], mz);
                        derive27(tab[c], xy9[c], xz9, yz9);
                    }
                    float sc;
                    if constexpr (FILTER) {
                        // Provably worse than the k-th candidate: not offered,
                        // as exact scoring would not have offered it either.
                        if (__fadd_rn(thr_s, P.T.k2_margin) < k2_approx32<27>(s_lo, tab[0], tab[1])) continue;
                        sc = score32_lut<27, LutGlobal, 0>(P.T, LutGlobal{P.T.t32}, tab[0], tab[1]);
                    } else {
                        sc = score32_lut<27, LutShared, SC>(P.T, lut, tab[0], tab[1]);
                    }
                    Cand cd;
                    cd.key = score_key(sc, maximize);
                    cd.pad = 0;
                    cd.set = set_key3((uint32_t)X, (uint32_t)arow, (uint32_t)bsnp);
                    tk.offer(cd, thr, hi);
                }
                if (!GCANDS && mode != kPairsStore) tk.check(hi, kCap - kEpiPerStep, bar);
            }
            if constexpr (GCANDS) tk.check(hi, kCapG - kEpiPerTile, bar);
        }
        if (!ok) {
            record_error(P.err, 5);
            *s_abort = 1;
        } else if (mode != kPairsStore) {
            tk.store(P.S.lists + (size_t)blockIdx.x * P.S.k, P.S.counts + blockIdx.x, bar);
        }
    }
    // Neither CTA of a pair may release TMEM or leave while the pair's MMAs
    // can still read its shared memory or write its accumulators.
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    // After an abort, copies that no barrier of this CTA tracks (its half of a
    // stage the peer never armed) complete within microseconds: pause before
    // either CTA of the pair leaves.
    if (threadIdx.x == 0 && *abort) {
        const uint64_t t0 = ptx::globaltimer();
        while (ptx::globaltimer() - t0 < kAbortPauseNs) __nanosleep(1000);
    }
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    if (warp == 1) {
        ptx::tc_fence_after();
        if constexpr (PAIR)
            ptx::tmem_dealloc_pair(tmem, 512);
        else
            ptx::tmem_dealloc(tmem, 512);
    }
}

}  // namespace tc

// Largest distance |lngamma1_filter(v) - t32[v]| over kSmallTab <= v < size
// (below kSmallTab the filter reads the table itself), as the bits of a
// non-negative float rounded up (their integer order is the float order).
__global__ void __launch_bounds__(256) k2_filter_error_kernel(const float* __restrict__ t32, int size,
                                                               unsigned* __restrict__ out) {
    float worst = 0.0f;
    for (int v = kSmallTab + (int)(blockIdx.x * blockDim.x + threadIdx.x); v < size; v += (int)(gridDim.x * blockDim.x)) {
        const double d = fabs((double)lngamma1_stirling(v) - (double)__ldg(t32 + v));
        worst = fmaxf(worst, __double2float_ru(d));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xFFFFFFFFu, worst, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(worst));
}

// ------------------------------------------------------------------ host
using namespace tc;

episdet_status k2_filter_margin(Workspace* w, int nc, int nn, const float* d_t32, float* margin) {
    const int N = nc + nn, size = N + 2;
    unsigned eps_bits = 0;
    CUDA_TRY(w->flag.ensure(sizeof(int) * 4));
    unsigned* d_out = (unsigned*)w->flag.p + 2;
    CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned), w->st));
    if (size > kSmallTab) {
        k2_filter_error_kernel<<<std::min((size + 255) / 256, 148 * 8), 256, 0, w->st>>>(d_t32, size, d_out);
        CHECK_LAUNCH();
    }
    CUDA_TRY(cudaMemcpyAsync(&eps_bits, d_out, sizeof(unsigned), cudaMemcpyDeviceToHost, w->st));
    CUDA_TRY(cudaStreamSynchronize(w->st));
    float eps;
    memcpy(&eps, &eps_bits, sizeof(eps));
    // |S_fp32 - S_filter| <= 81 eps (81 table reads per 3-way table) + the
    // rounding of both FP32 sums.  Rounding of one sum (27 cells, unit
    // roundoff u = 2^-24): u * (sum_c |a_c| + |b_c| + |s_c|) with a_c the
    // first addition of a cell, b_c the cell term, s_c the running sum; sum_c
    // lnG(n_c + 1) <= lnG(n + 1) per class (superadditivity of ln n!), |b_c| <=
    // (n_c + m_c) ln 2 + ln(N + 1) + 3 (b_c = -ln((n+m+1) C(n+m, n)) up to the
    // table's error), |s_c| <= sum of the |b_c|.
    const double u = std::ldexp(1.0, -24);
    const double lg = std::lgamma((double)nc + 1.0) + std::lgamma((double)nn + 1.0) + 54.0;
    const double bt = (double)N * std::log(2.0) + 27.0 * (std::log((double)N + 2.0) + 3.0);
    const double round1 = u * (lg + 28.0 * bt) * 1.05;
    const double m = 81.0 * (double)eps + 2.0 * round1 + 1.0;
    *margin = std::nextafter((float)m, std::numeric_limits<float>::infinity());
    w->d2h += (int64_t)sizeof(unsigned);
    return EPISDET_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static episdet_status get_encoder() {
    if (g_encode) return EPISDET_OK;
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return set_error(EPISDET_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return EPISDET_OK;
}

// rows x pitch bytes, row-major, 128x128-byte boxes, 128-byte swizzle.
static episdet_status make_tmap(CUtensorMap* m, void* base, uint64_t rows, uint64_t pitch,
                                uint32_t box_rows = kTileRows) {
    cuuint64_t dims[2] = {pitch, rows};
    cuuint64_t strides[1] = {pitch};
    cuuint32_t box[2] = {kKB, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(EPISDET_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return EPISDET_OK;
}

static int grid_for(long work, int threads) {
    long b = (work + threads - 1) / threads;
    return (int)std::min<long>(std::max<long>(b, 1), 148L * 64);
}

// Label-free AND cells of every SNP pair over the n samples of one plane set
// ([M][2][W] words, on the device) into out ([M][M] uint4, pairs a < b): the
// pair-table kernel over a single class.
episdet_status tensor_pair_totals(Workspace* w, const uint32_t* d_planes, int M, int n, uint4* out) {
    episdet_status st = get_encoder();
    if (st != EPISDET_OK) return st;
    CUDA_TRY(w->tensor_flag.ensure(sizeof(int) * 4));
    CUDA_TRY(cudaMemsetAsync(w->tensor_flag.p, 0, sizeof(int) * 4, w->st));
    DevData D;
    memset(&D, 0, sizeof(D));
    D.M = M;
    D.bits[0] = d_planes;
    D.bits[1] = d_planes;  // no second class: W[1] = 0
    D.n[0] = n;
    D.W[0] = episdet_class_words(n);
    const int Kc = D.W[0] * 32, rows = 2 * M, pitch2 = Kc;
    CUDA_TRY(w->planes8.ensure((size_t)rows * pitch2));
    uint8_t* P2 = (uint8_t*)w->planes8.p;
    unpack_kernel<<<grid_for((long)rows * (pitch2 / 16), 256), 256, 0, w->st>>>(D, P2, rows, pitch2);
    CHECK_LAUNCH();
    TmapPack tm2;
    memset(&tm2, 0, sizeof(tm2));
    st = make_tmap(&tm2.m[0], P2, (uint64_t)rows, (uint64_t)pitch2);
    if (st != EPISDET_OK) return st;
    const int nt = (M + kTileSnps - 1) / kTileSnps;
    std::vector<int2> ptiles;
    for (int a = 0; a < nt; ++a)
        for (int b = a; b < nt; ++b) ptiles.push_back(make_int2(a, b));
    CUDA_TRY(w->tiles.ensure(sizeof(int2) * ptiles.size()));
    CUDA_TRY(cudaMemcpyAsync(w->tiles.p, ptiles.data(), sizeof(int2) * ptiles.size(), cudaMemcpyHostToDevice, w->st));
    TcParams p;
    memset(&p, 0, sizeof(p));
    p.D = D;
    p.first_begin = 0;
    p.first_end = M;
    p.err = (int*)w->tensor_flag.p;
    p.wait_ns = 4000ull * 1000000ull;
    p.ngroup = 1;
    p.grp[0] = GroupDesc{(const int2*)w->tiles.p, 0, -1, nullptr};
    p.ntiles = (int)ptiles.size();
    p.mode = kPairsStore;
    p.seg2[0] = Seg{0, Kc / kKB};
    p.seg2[1] = Seg{Kc / kKB, Kc / kKB};
    p.pair_out0 = out;
    p.pair_out1 = nullptr;
    p.out_ld = M;
    tc_kernel<false, false><<<std::max(1, std::min(w->sms, (int)ptiles.size())), kThreads,
                              KCfg<false, false>::kSmemTotal, w->st>>>(tm2, p);
    CHECK_LAUNCH();
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, w->tensor_flag.p, sizeof(int), cudaMemcpyDeviceToHost, w->st));
    CUDA_TRY(cudaStreamSynchronize(w->st));  // the tile list is reused by the next search
    if (err) return set_error(EPISDET_ERR_TIMEOUT, "a bounded device wait gave up (code %d)", err);
    return EPISDET_OK;
}

episdet_status tensor_init_attributes() {
    CUDA_TRY(cudaFuncSetAttribute(regroup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kRgSmem));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<false, false>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, false, 0>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, true, 0>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, false, 0, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, false, 0, false, 1>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, true, 0, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, true, 0, false, 1>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, false, 1>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, true, 1>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, false, 0, true>::kSmemTotal));
    CUDA_TRY(cudaFuncSetAttribute(tc_kernel<true, false, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)KCfg<true, false, 1, true>::kSmemTotal));
    return get_encoder();
}


episdet_status run_tensor(Workspace* w, DevData& D, const ScoreTables& T, const episdet_options& o, int fb, int fe,
                          Slots* S, uint64_t* launches, bool progress) {
    episdet_status st = get_encoder();
    if (st != EPISDET_OK) return st;
    const int M = D.M;
    const int grid = w->sms;
    st = prepare_slots(w, grid, o.top_k, S);
    if (st != EPISDET_OK) return st;
    CUDA_TRY(w->tensor_flag.ensure(sizeof(int) * 4));
    int* d_err = (int*)w->tensor_flag.p;

    const int Kc = D.W[0] * 32, Kn = D.W[1] * 32;
    const int pitch2 = Kc + Kn;
    const int rows = 2 * M;
    const int nt = (M + kTileSnps - 1) / kTileSnps;
    const int bs_lines = (M + 255) / 256;
    std::vector<int2> tiles;
    TcParams p;
    memset(&p, 0, sizeof(p));
    p.D = D;
    p.T = T;
    p.S = *S;
    p.first_begin = fb;
    p.first_end = fe;
    p.err = d_err;
    p.wait_ns = (uint64_t)(o.wait_limit_ms > 0 ? o.wait_limit_ms : 4000) * 1000000ull;
    p.hold = (o.flags & EPISDET_FLAG_INJECT_STALL) ? d_err + 3 : nullptr;
    const bool mi = T.score == EPISDET_SCORE_MI;

    if (o.order == 2) {
        // Pairs on the CTA-pair kind::mxf4 kernel: packed e2m1 rows of every
        // SNP plane, tiles of 128 A SNPs x 56 B SNPs whose B range reaches
        // past the tile's first A SNP, two accumulator sets in TMEM.
        // Label mode (w->label_tot): operand rows of the cases only; the
        // controls' cells come from the label-free pair totals.
        const bool label = w->label_tot != nullptr;
        const int pitchx = (Kc + kClassPad) / 2 + (label ? 0 : (Kn + kClassPad) / 2);
        CUDA_TRY(w->xsub[0].ensure((size_t)rows * pitchx));
        uint8_t* F = (uint8_t*)w->xsub[0].p;
        DevData Dp = D;
        if (label) Dp.W[1] = 0;  // pack class 0 only
        pack_f4_kernel<<<grid_for((long)rows * (Dp.W[0] + Dp.W[1]), 256), 256, 0, w->st>>>(Dp, F, rows, pitchx);
        CHECK_LAUNCH();
        ++*launches;
        TmapPack tmf;
        memset(&tmf, 0, sizeof(tmf));
        st = make_tmap(&tmf.m[0], F, (uint64_t)rows, (uint64_t)pitchx);
        if (st != EPISDET_OK) return st;
        st = make_tmap(&tmf.m[kMaxGroup], F, (uint64_t)rows, (uint64_t)pitchx, kZSnpsPair);
        if (st != EPISDET_OK) return st;
        const int ntb = (M + kZSnpsPair - 1) / kZSnpsPair;
        for (int a = fb / (2 * kTileSnps); a <= (fe - 1) / (2 * kTileSnps); ++a)
            for (int bt = (2 * kTileSnps * a) / kZSnpsPair; bt < ntb; ++bt) tiles.push_back(make_int2(a, bt));
        CUDA_TRY(w->tiles.ensure(sizeof(int2) * tiles.size()));
        CUDA_TRY(cudaMemcpyAsync(w->tiles.p, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, w->st));
        if (progress)
            for (int i = 0; i < bs_lines; ++i) printf("Outer loop iteration %d out of %d\n", i, bs_lines);
        w->h2d += (int64_t)(sizeof(int2) * tiles.size());
        const int kb1 = (Kc + kClassPad) / kF4PerKB;
        p.seg2[0] = Seg{0, (D.n[0] + kF4PerKB - 1) / kF4PerKB};
        p.seg2[1] = label ? Seg{kb1, kb1} : Seg{kb1, kb1 + (D.n[1] + kF4PerKB - 1) / kF4PerKB};
        p.tot = w->label_tot;
        p.ngroup = 1;
        p.grp[0] = GroupDesc{(const int2*)w->tiles.p, 0, -1, nullptr};
        p.ntiles = (int)tiles.size();
        p.mode = kPairsScore;
        auto* const kern2 = mi ? tc_kernel<true, false, 1, true> : tc_kernel<true, false, 0, true>;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(2 * (grid / 2), 1, 1);
        cfg.blockDim = dim3(kThreads, 1, 1);
        cfg.dynamicSmemBytes = mi ? KCfg<true, false, 1, true>::kSmemTotal : KCfg<true, false, 0, true>::kSmemTotal;
        cfg.stream = w->st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int pairs = 0;
        CUDA_TRY(cudaOccupancyMaxActiveClusters(&pairs, kern2, &cfg));
        pairs = std::min(pairs, grid / 2);
        if (pairs < 1) return set_error(EPISDET_ERR_UNSUPPORTED, "no CTA pair of the counting kernel fits on the device");
        // No more clusters than tiles: SMs left idle stay free for concurrent work.
        cfg.gridDim = dim3(2 * std::max(1, std::min(pairs, (int)tiles.size())), 1, 1);
        CUDA_TRY(timer_begin(w));
        CUDA_TRY(cudaLaunchKernelEx(&cfg, kern2, tmf, p));
        CHECK_LAUNCH();
        CUDA_TRY(timer_end(w));
        ++*launches;
        if (w->timing)
            w->executed_macs = (double)tiles.size() * 2.0 * kTileRows * kNPair *
                               (double)(p.seg2[0].kb1 - p.seg2[0].kb0 + p.seg2[1].kb1 - p.seg2[1].kb0) * kF4PerKB;
        return EPISDET_OK;
    }

    CUDA_TRY(w->planes8.ensure((size_t)rows * pitch2));
    uint8_t* P2 = (uint8_t*)w->planes8.p;
    unpack_kernel<<<grid_for((long)rows * (pitch2 / 16), 256), 256, 0, w->st>>>(D, P2, rows, pitch2);
    CHECK_LAUNCH();
    ++*launches;
    TmapPack tm2;
    memset(&tm2, 0, sizeof(tm2));
    st = make_tmap(&tm2.m[0], P2, (uint64_t)rows, (uint64_t)pitch2);
    if (st != EPISDET_OK) return st;

    p.seg2[0] = Seg{0, Kc / kKB};
    p.seg2[1] = Seg{Kc / kKB, pitch2 / kKB};

    // 3-way pair table.  Whole: every pair whose first SNP lies in a tile >=
    // fb's, an [M][M] window per class, filled once.  Y-blocked (when the
    // whole table does not fit beside the other buffers, or as
    // o.pair_block_snps asks): the rows of one block of second SNPs Y at a
    // time ([BY][M - y0] from column y0), plus the rows of the current first
    // SNPs X ([128][M - xt0]); the first SNPs are then swept once per Y block,
    // each pass counting only the triplets whose Y lies in the block (the
    // reference keeps [9][BLOCK_SIZE][M] pair counts per Y block,
    // src/search-triplets.cu:173-176).
    const int nt2 = (M + 2 * kTileSnps - 1) / (2 * kTileSnps);
    const int ntb = (M + kZSnpsPair - 1) / kZSnpsPair;
    const int a_first = (fb + 1) / (2 * kTileSnps);
    const int xend = std::min(fe, M - 2);
    // Regrouped rows: both classes' packed e2m1 regions, 2 samples per byte.
    const int pitchx = (Kc + kClassPad) / 2 + (Kn + kClassPad) / 2;
    const int max_n = std::max(D.n[0], D.n[1]);
    const size_t info_bytes = 256;
    const size_t idx_bytes = sizeof(int) * 4 * (size_t)max_n;
    int blk_tiles = nt2 - a_first;  // A pair tiles (128 Y SNPs) per Y block
    {
        const size_t row_bytes = 2 * sizeof(uint4) * (size_t)M;  // one table row, both classes
        const size_t xrows_bytes = row_bytes * 2 * kTileSnps;
        // The other buffers of the search first (their later ensure calls
        // find them in place); the pair table gets what is left.
        for (DevBuf& d : w->xsub) CUDA_TRY(d.ensure((size_t)rows * pitchx));
        for (int c = 0; c < 2; ++c)
            CUDA_TRY(w->planes_t[c].ensure(sizeof(uint32_t) * (size_t)D.W[c] * 32 * tt_row_words(rows)));
        CUDA_TRY(w->xinfo.ensure((size_t)kXSets * kMaxGroup * (info_bytes + idx_bytes)));
        CUDA_TRY(w->cbuf.ensure(sizeof(Cand) * (size_t)kCapG * grid));
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        // Left for the tile lists, slots, merge buffers and the driver.
        const size_t reserve = std::max<size_t>(tot / 32, (size_t)1 << 30);
        // The pair-table buffers are replaced when they grow, so their memory counts as free.
        const size_t held = w->pair4[0].cap + w->pair4[1].cap + w->pairx[0].cap + w->pairx[1].cap;
        const size_t avail = fr + held > reserve ? fr + held - reserve : 0;
        if (o.pair_block_snps > 0) {
            blk_tiles = std::min(blk_tiles, (o.pair_block_snps + 2 * kTileSnps - 1) / (2 * kTileSnps));
        } else if (row_bytes * (size_t)M > avail) {
            const size_t left = avail > xrows_bytes ? avail - xrows_bytes : 0;
            blk_tiles = (int)std::min<size_t>((size_t)blk_tiles, left / (row_bytes * 2 * kTileSnps));
            if (blk_tiles < 1)
                return set_error(EPISDET_ERR_OUT_OF_MEMORY,
                                 "3-way search of %d SNPs: no 128-row block of the pair table fits in the %.1f GB "
                                 "left beside the operand buffers",
                                 M, (double)avail / 1e9);
        }
    }
    const bool blocked = blk_tiles < nt2 - a_first;
    const int nblk = (nt2 - a_first + blk_tiles - 1) / blk_tiles;
    for (int c = 0; c < 2; ++c) {
        if (blocked) {
            CUDA_TRY(w->pair4[c].ensure(sizeof(uint4) * (size_t)blk_tiles * 2 * kTileSnps * M));
            CUDA_TRY(w->pairx[c].ensure(sizeof(uint4) * (size_t)2 * kTileSnps * M));
        } else {
            CUDA_TRY(w->pair4[c].ensure(sizeof(uint4) * (size_t)M * M));
        }
        D.pair4[c] = (const uint4*)w->pair4[c].p;
    }
    p.D = D;
    // Pair-table tile list: every 64-SNP tile pair (a, b >= a) in order of a,
    // so that the tiles of rows [64 a_lo, 64 a_hi) are one sub-range.
    std::vector<int2> tri;
    std::vector<size_t> tri_off((size_t)nt + 1, 0);
    for (int a = 0; a < nt; ++a) {
        tri_off[a] = tri.size();
        for (int b = a; b < nt; ++b) tri.push_back(make_int2(a, b));
    }
    tri_off[nt] = tri.size();
    // Triplet tile lists, one per (Y block, first A pair tile a0 = (X+1)/128):
    // every (A pair tile a of 128 Y SNPs, B tile b of 56 Z SNPs) with
    // max(a0, first tile of the block) <= a < end of the block, whose Z range
    // reaches past the tile's first Y (b >= bfirst(a)), ordered in bands of
    // about 768 x 784 SNPs so that a wave of concurrent tiles shares few A and
    // B row panels in L2.  First SNPs below the block share one list; lists
    // are built only for the first SNPs of this call's slab.
    constexpr int kBandA = kBand / 2, kBandB = 14;
    auto bfirst = [](int a) { return (2 * kTileSnps * a) / kZSnpsPair; };
    const int a_last = std::min(nt2 - 1, xend / (2 * kTileSnps));  // a0 of the slab's last first SNP
    std::vector<int2> lists;
    std::vector<size_t> list_off((size_t)nblk * (nt2 + 1), 0);
    std::vector<int> list_len((size_t)nblk * (nt2 + 1), 0);
    for (int blk = 0; blk < nblk; ++blk) {
        const int ya0 = a_first + blk * blk_tiles, ya1 = std::min(nt2, ya0 + blk_tiles);
        for (int a0 = a_first; a0 < std::min(ya1, a_last + 1); ++a0) {
            const size_t li = (size_t)blk * (nt2 + 1) + a0;
            if (a0 < ya0 && a0 > a_first) {  // same list as the block's first a0
                list_off[li] = list_off[li - 1];
                list_len[li] = list_len[li - 1];
                continue;
            }
            list_off[li] = lists.size();
            for (int ba = std::max(a0, ya0); ba < ya1; ba += kBandA)
                for (int bb = bfirst(ba); bb < ntb; bb += kBandB)
                    for (int a = ba; a < std::min(ya1, ba + kBandA); ++a)
                        for (int b = std::max(bfirst(a), bb); b < std::min(ntb, bb + kBandB); ++b)
                            lists.push_back(make_int2(a, b));
            list_len[li] = (int)(lists.size() - list_off[li]);
        }
    }
    CUDA_TRY(w->tiles.ensure(sizeof(int2) * (tri.size() + lists.size())));
    int2* d_tri = (int2*)w->tiles.p;
    int2* d_lists = d_tri + tri.size();
    CUDA_TRY(cudaMemcpyAsync(d_tri, tri.data(), sizeof(int2) * tri.size(), cudaMemcpyHostToDevice, w->st));
    CUDA_TRY(cudaMemcpyAsync(d_lists, lists.data(), sizeof(int2) * lists.size(), cudaMemcpyHostToDevice, w->st));
    w->h2d += (int64_t)(sizeof(int2) * (tri.size() + lists.size()));
    // Counts of the pairs of SNP rows [r0, r1) (tile-aligned r0) with every
    // later SNP, stored at (row - r0) * (M - r0) + (col - r0) of out (or at
    // row * M + col when whole).
    auto store_pairs = [&](uint4* out0, uint4* out1, int r0, int r1, bool whole) -> episdet_status {
        const int t0 = r0 / kTileSnps, t1 = std::min(nt, (r1 + kTileSnps - 1) / kTileSnps);
        const int n = (int)(tri_off[t1] - tri_off[t0]);
        p.ngroup = 1;
        p.grp[0] = GroupDesc{d_tri + tri_off[t0], 0, -1, nullptr};
        p.ntiles = n;
        p.mode = kPairsStore;
        p.pair_out0 = out0;
        p.pair_out1 = out1;
        p.out_r0 = whole ? 0 : r0;
        p.out_c0 = whole ? 0 : r0;
        p.out_ld = whole ? M : M - r0;
        tc_kernel<false, false><<<std::max(1, std::min(grid, n)), kThreads, KCfg<false, false>::kSmemTotal, w->st>>>(
            tm2, p);
        CHECK_LAUNCH();
        ++*launches;
        return EPISDET_OK;
    };
    if (!blocked) {
        st = store_pairs((uint4*)w->pair4[0].p, (uint4*)w->pair4[1].p, fb / kTileSnps * kTileSnps, M, true);
        if (st != EPISDET_OK) return st;
        p.xv = PairView{{D.pair4[0], D.pair4[1]}, 0, 0, M};
        p.yv = p.xv;
    }

    // Regrouped operands of the kMaxGroup X values of a launch, and their segment tables.
    for (int i = 0; i < kXSets * kMaxGroup; ++i) CUDA_TRY(w->xsub[i].ensure((size_t)rows * pitchx));
    // kXSets sets of regrouped operands and segment tables: the regrouping of
    // group g + 1 (on aux_st) is queued while the counting launch of group g
    // (on st) runs and starts on the SMs that launch frees at its end, while
    // its last tiles still read group g's set.
    CUDA_TRY(w->xinfo.ensure(kXSets * kMaxGroup * (info_bytes + idx_bytes)));
    TmapPack tmx[kXSets];
    XInfo* d_info[kXSets][kMaxGroup];
    XWork xw[kXSets];
    CmpOut co[kXSets];
    for (int b = 0; b < kXSets; ++b) {
        memset(&tmx[b], 0, sizeof(tmx[b]));
        xw[b].base = (uint8_t*)w->xinfo.p + (size_t)b * kMaxGroup * (info_bytes + idx_bytes);
        xw[b].stride = info_bytes + idx_bytes;
        xw[b].info_bytes = info_bytes;
        xw[b].max_n = max_n;
        for (int i = 0; i < kMaxGroup; ++i) {
            void* buf = w->xsub[b * kMaxGroup + i].p;
            st = make_tmap(&tmx[b].m[i], buf, (uint64_t)rows, (uint64_t)pitchx);
            if (st != EPISDET_OK) return st;
            st = make_tmap(&tmx[b].m[kMaxGroup + i], buf, (uint64_t)rows, (uint64_t)pitchx, kZSnpsPair);
            if (st != EPISDET_OK) return st;
            d_info[b][i] = (XInfo*)(xw[b].base + i * xw[b].stride);
            co[b].out[i] = (uint8_t*)buf;
            co[b].row0[i] = 0;
        }
    }
    p.mode = kTriplets;
    CUDA_TRY(w->cbuf.ensure(sizeof(Cand) * (size_t)kCapG * grid));
    p.cbuf = (Cand*)w->cbuf.p;
    // Large classes make the staged kernel's early release of segment 0 pay
    // (its MMAs then overlap the epilogue); smaller ones run the plain kernel.
    const bool staged = w->stage_override >= 0 ? w->stage_override == 1 : std::min(D.n[0], D.n[1]) >= kStageClass;
    // One instance per score, so each carries only its own scoring code.
    // K2: the filtered instance for searches where every CTA scores far more
    // sets than its candidate list holds (or as the flags force).
    double slab_sets = 0.0;
    for (int x = fb; x < xend; ++x) slab_sets += 0.5 * (double)(M - 1 - x) * (double)(M - 2 - x);
    const bool filt = !mi && (o.flags & EPISDET_FLAG_FILTER_OFF) == 0 &&
                      ((o.flags & EPISDET_FLAG_FILTER_ON) != 0 || slab_sets >= kFilterMinSetsPerCta * (double)grid);
    auto* const kern = mi ? (staged ? tc_kernel<true, true, 1> : tc_kernel<true, false, 1>)
                          : filt ? (staged ? tc_kernel<true, true, 0, false, 1> : tc_kernel<true, false, 0, false, 1>)
                                 : (staged ? tc_kernel<true, true, 0> : tc_kernel<true, false, 0>);
    const size_t ksmem = mi ? (staged ? KCfg<true, true, 1>::kSmemTotal : KCfg<true, false, 1>::kSmemTotal)
                            : filt ? (staged ? KCfg<true, true, 0, false, 1>::kSmemTotal
                                             : KCfg<true, false, 0, false, 1>::kSmemTotal)
                                   : (staged ? KCfg<true, true, 0>::kSmemTotal : KCfg<true, false, 0>::kSmemTotal);
    // CTA pairs: as many clusters of two as can be resident at once.
    int pairs = 0;
    {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(2 * (grid / 2), 1, 1);
        cfg.blockDim = dim3(kThreads, 1, 1);
        cfg.dynamicSmemBytes = ksmem;
        cfg.stream = w->st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CUDA_TRY(cudaOccupancyMaxActiveClusters(&pairs, kern, &cfg));
        pairs = std::min(pairs, grid / 2);
        if (pairs < 1) return set_error(EPISDET_ERR_UNSUPPORTED, "no CTA pair of the counting kernel fits on the device");
    }
    // Sample-major planes for the regrouping, and its persistent grid (as many
    // CTAs as fit on the device at once).
    const int rwp = tt_row_words(rows);
    int rg_per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rg_per_sm, regroup_kernel, kRgThreads, kRgSmem));
    const int rg_ctas = std::max(1, rg_per_sm) * grid;
    int* const rg_ctr = d_err + 2;  // the regrouping's item counter (reset before each launch)
    for (int c = 0; c < 2; ++c) {
        CUDA_TRY(w->planes_t[c].ensure(sizeof(uint32_t) * (size_t)D.W[c] * 32 * rwp));
        const int warps = (rwp / 8) * (D.W[c] / 8);
        transpose_planes_kernel<<<(warps + kTtThreads / 32 - 1) / (kTtThreads / 32), kTtThreads, 0, w->st>>>(
            D, c, (uint32_t*)w->planes_t[c].p, rows, rwp);
        CHECK_LAUNCH();
        ++*launches;
    }
    // The regrouping reads the planes, their transposes and the marginals staged on st.
    CUDA_TRY(cudaEventRecord(w->ev_ready, w->st));
    CUDA_TRY(cudaStreamWaitEvent(w->aux_st, w->ev_ready, 0));
    // Pair tiles each first SNP was counted against, per launch (for the MAC count).
    struct LaunchTiles {
        int x0, gn;
        int len[kMaxGroup];
    };
    std::vector<LaunchTiles> launch_tiles;
    int gi = 0;
    int xt0 = -1;  // first row held in pairx (Y-blocked)
    for (int blk = 0; blk < nblk; ++blk) {
        const int ya0 = a_first + blk * blk_tiles, ya1 = std::min(nt2, ya0 + blk_tiles);
        const int y0 = ya0 * 2 * kTileSnps, y1 = std::min(M, ya1 * 2 * kTileSnps);
        if (blocked) {
            // Y-Z rows of this block (the previous block's launches, on the
            // same stream, have read theirs).
            st = store_pairs((uint4*)w->pair4[0].p, (uint4*)w->pair4[1].p, y0, y1, false);
            if (st != EPISDET_OK) return st;
            p.yv = PairView{{D.pair4[0], D.pair4[1]}, y0, y0, M - y0};
        }
        const int xe = std::min(xend, y1 - 1);  // X < Y < y1
        for (int x0 = fb; x0 < xe; x0 += kMaxGroup) {
            const int gn = std::min(kMaxGroup, xe - x0);
            const int b = gi % kXSets;
            // (Kept aside until the launch: store_pairs below rewrites p.grp.)
            GroupDesc gdesc[kMaxGroup];
            LaunchTiles lt{x0, gn, {0, 0, 0, 0}};
            int cum = 0;
            for (int g = 0; g < gn; ++g) {
                const int x = x0 + g;
                if (progress && x % 256 == 0 && x + 1 >= y0) printf("Outer loop iteration %d out of %d\n", x / 256, bs_lines);
                const size_t li = (size_t)blk * (nt2 + 1) + (x + 1) / (2 * kTileSnps);
                gdesc[g] = GroupDesc{d_lists + list_off[li], cum, x, d_info[b][g]};
                cum += list_len[li];
                lt.len[g] = list_len[li];
            }
            if (cum == 0) continue;
            if (w->timing) launch_tiles.push_back(lt);
            ++gi;
            if (blocked && (xt0 < 0 || x0 < xt0 || x0 + gn > xt0 + 2 * kTileSnps)) {
                // X-Y and X-Z rows of this group's first SNPs (and the next ones').
                xt0 = x0 / kTileSnps * kTileSnps;
                st = store_pairs((uint4*)w->pairx[0].p, (uint4*)w->pairx[1].p, xt0, std::min(M, xt0 + 2 * kTileSnps),
                                 false);
                if (st != EPISDET_OK) return st;
                p.xv = PairView{{(const uint4*)w->pairx[0].p, (const uint4*)w->pairx[1].p}, xt0, xt0, M - xt0};
            }
            // Index lists and regrouped rows of the gn first SNPs, one launch each,
            // into buffer set b once the counting launch that last read it is done.
            if (gi > kXSets) CUDA_TRY(cudaStreamWaitEvent(w->aux_st, w->ev_tc[b], 0));
            xw[b].x0 = x0;
            xinfo_kernel<<<dim3(2, gn), kXinfoThreads, 0, w->aux_st>>>(D, xw[b]);
            CHECK_LAUNCH();
            for (int g = 0; g < gn; ++g)
                co[b].row0[g] = kNPair * bfirst(std::max((x0 + g + 1) / (2 * kTileSnps), ya0));
            CUDA_TRY(cudaMemsetAsync(rg_ctr, 0, sizeof(int), w->aux_st));
            regroup_kernel<<<rg_ctas, kRgThreads, kRgSmem, w->aux_st>>>(
                D, xw[b], co[b], (const uint32_t*)w->planes_t[0].p, (const uint32_t*)w->planes_t[1].p, rwp, rows,
                pitchx, gn, rg_ctr);
            CHECK_LAUNCH();
            CUDA_TRY(cudaEventRecord(w->ev_cmp[b], w->aux_st));
            CUDA_TRY(cudaStreamWaitEvent(w->st, w->ev_cmp[b], 0));
            *launches += 2;
            for (int g = 0; g < gn; ++g) {
                if (gdesc[g].x < 0 || !gdesc[g].xinfo) return set_error(EPISDET_ERR_INTERNAL, "triplet group %d unset", g);
                p.grp[g] = gdesc[g];
            }
            p.ngroup = gn;
            p.ntiles = cum;
            p.mode = kTriplets;
            CUDA_TRY(timer_begin(w));
            {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = 2;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3(2 * std::max(1, std::min(pairs, cum)), 1, 1);
                cfg.blockDim = dim3(kThreads, 1, 1);
                cfg.dynamicSmemBytes = ksmem;
                cfg.stream = w->st;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, tmx[b], p));
            }
            CHECK_LAUNCH();
            CUDA_TRY(timer_end(w));
            CUDA_TRY(cudaEventRecord(w->ev_tc[b], w->st));
            *launches += 1;
        }
    }
    if (w->timing) {
        // Tensor MACs issued: per X, pair tiles x 256 x 112 x the regrouped K extent,
        // which follows from X's genotype counts exactly as xinfo_kernel derives it.
        std::vector<int> mg[2];
        for (int c = 0; c < 2; ++c) {
            mg[c].resize((size_t)3 * M);
            CUDA_TRY(cudaMemcpyAsync(mg[c].data(), D.marg[c], sizeof(int) * 3 * M, cudaMemcpyDeviceToHost, w->st));
        }
        CUDA_TRY(cudaStreamSynchronize(w->st));
        w->d2h += (int64_t)(2 * sizeof(int) * 3 * M);
        auto kext_of = [&](int x) {
            int tot[3];
            for (int g = 0; g < 3; ++g) tot[g] = mg[0][(size_t)g * M + x] + mg[1][(size_t)g * M + x];
            int gd = 0;
            if (tot[1] > tot[gd]) gd = 1;
            if (tot[2] > tot[gd]) gd = 2;
            long kext = 0;
            for (int c = 0; c < 2; ++c)
                for (int g = 0; g < 3; ++g)
                    if (g != gd) kext += ((mg[c][(size_t)g * M + x] + kF4PerKB - 1) / kF4PerKB) * (long)kF4PerKB;
            return kext;
        };
        double macs = 0.0;
        for (const LaunchTiles& lt : launch_tiles) {
            double m = 0.0;
            for (int g = 0; g < lt.gn; ++g) m += (double)lt.len[g] * 2 * kTileRows * kNPair * (double)kext_of(lt.x0 + g);
            w->launch_macs.push_back(m);
            macs += m;
        }
        w->executed_macs = macs;
    }
    return EPISDET_OK;
}

}  // namespace episdet
