// peak_f4.cu -- exactness check and rate of tcgen05.mma kind::mxf4 on B200.
//
//   episdet-peak-f4 [iters]
//   episdet-peak-f4 sweep [iters]
//   episdet-peak-f4 pipe [iters]
//
// The counting engine can hold its 0/1 operand rows as packed e2m1 values
// (0.0 and 1.0, four bits each) instead of unsigned bytes: half the bytes per
// sample and twice the MACs per instruction.  The block scale factors are all
// 1.0 (UE8M0 127), accumulation is FP32, so a count is exact while it stays
// below 2^24.  This program checks that on the device and measures the rate,
// in both instruction forms:
//
//  * cta1: tcgen05.mma.cta_group::1, M = 128, one CTA per SM;
//  * pair: tcgen05.mma.cta_group::2, M = 256 over a cluster of two CTAs (each
//    CTA holds 128 A rows and N/2 B rows; the even CTA issues), the form of
//    the triplet engine;
//
// each with a commit every 16 MMAs and every 4 MMAs (the engine commits once
// per 4-MMA pipeline stage).
//
//  * check: A row i is all 1.0 when i % 3 == 1, B row j all 1.0 when j % 4 != 0
//    (every other value 0), so every D[i][j] must equal the K length or 0 --
//    independent of the swizzle and of the nibble order inside a byte, which A
//    and B share;
//  * rate: back-to-back MMAs on resident tiles, at most 64 in flight.
//  * sweep: the rate over N (112, 128, 224, 256), the commit interval (4, 8,
//    16 MMAs), the number of MMAs in flight, extra commits to a barrier nothing
//    waits on ("sink": the cost of a commit alone, without a wait), and
//    commits of the pair form with and without multicast to the peer CTA.
//  * pipe: the pair form fed the way the counting engine feeds it -- a ring of
//    operand stages filled by a producer warp (TMA tile loads from an
//    L2-resident or a DRAM-sized buffer, or no loads), one commit per stage
//    -- over N, the stage count and the K blocks per stage.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>

#include "tc_ptx.cuh"

using namespace episdet;

namespace {

constexpr int kThreads = 128;
constexpr uint64_t kLimitNs = 2000000000ull;
constexpr int kInFlight = 64;  // MMAs in flight at most
constexpr int kMaxRing = 16;   // commit groups in flight (commit_every >= 4)
constexpr int kSweepRing = 64;  // sweep: commit groups in flight at most

__device__ int g_err;
__device__ unsigned long long g_bad;

__device__ __forceinline__ void mma_mxf4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t sfa, uint32_t sfb, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(
            d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
        : "memory");
}

template <int N, bool PAIR>
constexpr size_t smem_bytes() {
    return 1024 + 16384 + (size_t)(PAIR ? N / 2 : N) * 128 + (kMaxRing + 1) * 8 + 16 + 256;
}

// `groups` groups of `cper` MMAs, one commit per group.  check != 0: the
// exactness check (one accumulator, K = 64 * groups * cper values).
template <int N, bool PAIR>
__global__ void __launch_bounds__(kThreads, 1)
    f4_kernel(int groups, int cper, int check, unsigned long long* cycles) {
    constexpr int kBRows = PAIR ? N / 2 : N;
    // Scale factors: columns sf0 .. 511 of every lane hold bytes of 127 (2^0);
    // the pair form uses the engine's columns 448 .. 511.
    constexpr uint32_t sf0 = PAIR ? 448u : 496u;
    constexpr uint32_t sfb_off = PAIR ? 32u : 8u;
    extern __shared__ uint8_t raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a = sm;          // 128 rows x 128 bytes
    uint8_t* b = sm + 16384;  // kBRows rows x 128 bytes
    uint64_t* bars = reinterpret_cast<uint64_t*>(b + kBRows * 128);  // [0, kMaxRing) ring, [kMaxRing] drain
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + kMaxRing + 1);
    int* s_abort = reinterpret_cast<int*>(s_tmem + 1);
    int* s_never = s_abort + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rank = PAIR ? (int)ptx::cluster_ctarank() : 0;
    // Row-constant operands (a byte holds two e2m1 values: 0x22 = two 1.0).
    // B row j of the pair's N rows is row j - rank * N/2 of CTA `rank`.
    for (int i = threadIdx.x; i < 128 * 128; i += kThreads) a[i] = ((i >> 7) % 3 == 1) ? 0x22 : 0x00;
    for (int i = threadIdx.x; i < kBRows * 128; i += kThreads)
        b[i] = ((rank * kBRows + (i >> 7)) % 4 != 0) ? 0x22 : 0x00;
    if (threadIdx.x == 0) {
        for (int i = 0; i <= kMaxRing; ++i) ptx::mbar_init(&bars[i], 1);
        *s_abort = 0;
        *s_never = 0;
        ptx::fence_barrier_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        if constexpr (PAIR) {
            ptx::tmem_alloc_pair(s_tmem, 512);
            ptx::tmem_relinquish_pair();
        } else {
            ptx::tmem_alloc(s_tmem, 512);
            ptx::tmem_relinquish();
        }
    }
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (uint32_t c = sf0; c < 512u; c += 8) ptx::tmem_st8_fill(lane_base + c, 0x7F7F7F7Fu);
    ptx::tmem_wait_st();
    // Both CTAs' operands and scale factors are in place before the first MMA.
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    ptx::tc_fence_after();
    volatile int* abort = s_abort;
    if (warp == 0 && lane == 0) {
        if (rank == 0) {
            const uint32_t idesc = ptx::idesc_mxf4(N, PAIR ? 256 : 128);
            const uint64_t ad = ptx::smem_desc_sw128(ptx::smem_u32(a)), bd = ptx::smem_desc_sw128(ptx::smem_u32(b));
            const uint32_t sfa = tmem + sf0, sfb = tmem + sf0 + sfb_off;
            const int ring = kInFlight / cper;
            long long t0 = clock64();
            uint32_t ph = 0;
            uint32_t gm = 0;
            for (int g = 0; g < groups; ++g) {
                const int slot = g % ring;
                if (g >= ring) {
                    if (!ptx::mbar_wait(&bars[slot], (ph >> slot) & 1u, abort, kLimitNs)) {
                        atomicExch(&g_err, 1);
                        *s_abort = 1;
                        break;
                    }
                    ph ^= 1u << slot;
                }
                for (int m = 0; m < cper; ++m, ++gm) {
                    const int kk = gm & 3;  // 4 MMAs of K = 64 cover one 128-byte block
                    // Two accumulator regions below the scale factors (one for N = 256).
                    const uint32_t acc = (check || N > 224) ? 0u : ((gm >> 2) & 1u) * (uint32_t)N;
                    const uint32_t first = (check && gm == 0) ? 0u : 1u;
                    if constexpr (PAIR)
                        ptx::mma_mxf4_pair(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, first);
                    else
                        mma_mxf4(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, first);
                }
                if constexpr (PAIR)
                    ptx::mma_commit_pair_mc(&bars[slot], 0x3);  // as the engine: both CTAs' barriers
                else
                    ptx::mma_commit(&bars[slot]);
            }
            if constexpr (PAIR)
                ptx::mma_commit_pair_mc(&bars[kMaxRing], 0x3);
            else
                ptx::mma_commit(&bars[kMaxRing]);
            if (!ptx::mbar_wait(&bars[kMaxRing], 0, s_never, kLimitNs)) atomicExch(&g_err, 2);
            cycles[blockIdx.x] = (unsigned long long)(clock64() - t0);
        } else if (!ptx::mbar_wait(&bars[kMaxRing], 0, s_never, kLimitNs)) {
            atomicExch(&g_err, 3);  // the odd CTA: its accumulators are complete
        }
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const int unit = PAIR ? (int)ptx::cluster_id_x() : (int)blockIdx.x;
    if (check && unit == 0) {
        const float want_one = 64.0f * (float)groups * (float)cper;
        const int row = warp * 32 + lane;
        unsigned long long bad = 0;
        for (int c0 = 0; c0 < N; c0 += 8) {
            uint32_t v[8];
            ptx::tmem_ld8(lane_base + (uint32_t)c0, v);
            ptx::tmem_wait_ld();
            ptx::tmem_regs_ready(v);
            for (int e = 0; e < 8; ++e) {
                const int col = c0 + e;
                const float want = (row % 3 == 1 && col % 4 != 0) ? want_one : 0.0f;
                if (__uint_as_float(v[e]) != want) ++bad;
            }
        }
        if (bad) atomicAdd(&g_bad, bad);
    }
    // Neither CTA of a pair releases TMEM or leaves while the pair's MMAs may
    // still read its shared memory.
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    if (warp == 0) {
        ptx::tc_fence_after();
        if constexpr (PAIR)
            ptx::tmem_dealloc_pair(tmem, 512);
        else
            ptx::tmem_dealloc(tmem, 512);
    }
}


// Sweep kernel: `total` MMAs in groups of `cper`, one ring commit per group,
// at most `inflight` MMAs in flight; with sink > 0 an extra commit every
// `sink` MMAs arrives on a barrier that nothing waits on (its expected count
// is never reached); mc = 0 commits the pair form to the issuing CTA only
// (the odd CTA learns completion from the final multicast commit).
// Pair-form commit that arrives on the issuing CTA's barrier only.
__device__ __forceinline__ void commit_pair_local(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     ptx::smem_u32(bar))
                 : "memory");
}

template <int N, bool PAIR>
constexpr size_t sweep_smem_bytes() {
    return 1024 + 16384 + (size_t)(PAIR ? N / 2 : N) * 128 + (kSweepRing + 2) * 8 + 16 + 256;
}

template <int N, bool PAIR>
__global__ void __launch_bounds__(kThreads, 1)
    sweep_kernel(int total, int cper, int inflight, int sink, int mc, unsigned long long* cycles) {
    constexpr int kBRows = PAIR ? N / 2 : N;
    constexpr uint32_t sf0 = PAIR ? 448u : 496u;
    constexpr uint32_t sfb_off = PAIR ? 32u : 8u;
    extern __shared__ uint8_t raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a = sm;
    uint8_t* b = sm + 16384;
    // [0, kSweepRing) ring, [kSweepRing] drain, [kSweepRing + 1] sink
    uint64_t* bars = reinterpret_cast<uint64_t*>(b + kBRows * 128);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + kSweepRing + 2);
    int* s_abort = reinterpret_cast<int*>(s_tmem + 1);
    int* s_never = s_abort + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rank = PAIR ? (int)ptx::cluster_ctarank() : 0;
    for (int i = threadIdx.x; i < 128 * 128; i += kThreads) a[i] = ((i >> 7) % 3 == 1) ? 0x22 : 0x00;
    for (int i = threadIdx.x; i < kBRows * 128; i += kThreads)
        b[i] = ((rank * kBRows + (i >> 7)) % 4 != 0) ? 0x22 : 0x00;
    if (threadIdx.x == 0) {
        for (int i = 0; i <= kSweepRing; ++i) ptx::mbar_init(&bars[i], 1);
        ptx::mbar_init(&bars[kSweepRing + 1], (1u << 20) - 1);
        *s_abort = 0;
        *s_never = 0;
        ptx::fence_barrier_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        if constexpr (PAIR) {
            ptx::tmem_alloc_pair(s_tmem, 512);
            ptx::tmem_relinquish_pair();
        } else {
            ptx::tmem_alloc(s_tmem, 512);
            ptx::tmem_relinquish();
        }
    }
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (uint32_t c = sf0; c < 512u; c += 8) ptx::tmem_st8_fill(lane_base + c, 0x7F7F7F7Fu);
    ptx::tmem_wait_st();
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    ptx::tc_fence_after();
    volatile int* abort = s_abort;
    if (warp == 0 && lane == 0) {
        if (rank == 0) {
            const uint32_t idesc = ptx::idesc_mxf4(N, PAIR ? 256 : 128);
            const uint64_t ad = ptx::smem_desc_sw128(ptx::smem_u32(a)), bd = ptx::smem_desc_sw128(ptx::smem_u32(b));
            const uint32_t sfa = tmem + sf0, sfb = tmem + sf0 + sfb_off;
            const int ring = inflight / cper;
            const int groups = total / cper;
            long long t0 = clock64();
            uint32_t ph = 0;  // bit i: parity of ring slot i's next phase (ring <= 64: two words)
            uint32_t ph2 = 0;
            uint32_t gm = 0;
            for (int g = 0; g < groups; ++g) {
                const int slot = g % ring;
                if (g >= ring) {
                    uint32_t& w = slot < 32 ? ph : ph2;
                    const uint32_t bit = 1u << (slot & 31);
                    if (!ptx::mbar_wait(&bars[slot], (w & bit) ? 1u : 0u, abort, kLimitNs)) {
                        atomicExch(&g_err, 1);
                        *s_abort = 1;
                        break;
                    }
                    w ^= bit;
                }
                for (int m = 0; m < cper; ++m, ++gm) {
                    const int kk = gm & 3;
                    const uint32_t acc = N > 224 ? 0u : ((gm >> 2) & 1u) * (uint32_t)N;
                    if constexpr (PAIR)
                        ptx::mma_mxf4_pair(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, 1u);
                    else
                        mma_mxf4(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, 1u);
                    if (sink > 0 && (gm + 1) % (uint32_t)sink == 0 && m + 1 < cper) {
                        if constexpr (PAIR)
                            ptx::mma_commit_pair_mc(&bars[kSweepRing + 1], 0x3);
                        else
                            ptx::mma_commit(&bars[kSweepRing + 1]);
                    }
                }
                if constexpr (PAIR) {
                    if (mc)
                        ptx::mma_commit_pair_mc(&bars[slot], 0x3);
                    else
                        commit_pair_local(&bars[slot]);
                } else {
                    ptx::mma_commit(&bars[slot]);
                }
            }
            if constexpr (PAIR)
                ptx::mma_commit_pair_mc(&bars[kSweepRing], 0x3);
            else
                ptx::mma_commit(&bars[kSweepRing]);
            if (!ptx::mbar_wait(&bars[kSweepRing], 0, s_never, kLimitNs)) atomicExch(&g_err, 2);
            cycles[blockIdx.x] = (unsigned long long)(clock64() - t0);
        } else if (!ptx::mbar_wait(&bars[kSweepRing], 0, s_never, kLimitNs)) {
            atomicExch(&g_err, 3);
        }
    }
    ptx::tc_fence_before();
    if constexpr (PAIR)
        ptx::cluster_sync();
    else
        __syncthreads();
    if (warp == 0) {
        ptx::tc_fence_after();
        if constexpr (PAIR)
            ptx::tmem_dealloc_pair(tmem, 512);
        else
            ptx::tmem_dealloc(tmem, 512);
    }
}


// Pipeline kernel (pair form, the engine's structure without its epilogue):
// warp 0 of each CTA produces stages of `kbs` K blocks into a ring of
// `stages` stages (TMA tile loads from a global buffer when tma != 0, else a
// plain arrival), warp 1 of the even CTA waits for each stage, issues its
// 4 * kbs MMAs and commits once to the stage's empty barrier in both CTAs.
constexpr int kPipeMaxStages = 8;

template <int N>
__host__ __device__ constexpr int pipe_kb_bytes() {
    return 16384 + (N / 2) * 128;
}

template <int N>
__global__ void __launch_bounds__(kThreads, 1)
    pipe_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb, int iters, int stages,
                int kbs, int tma, int rows, int pitch, unsigned long long* cycles) {
    constexpr int kKbBytes = pipe_kb_bytes<N>();
    extern __shared__ uint8_t raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    const int stage_bytes = kbs * kKbBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + (size_t)stages * stage_bytes);
    uint64_t* full = bars;
    uint64_t* empty = bars + kPipeMaxStages;
    uint64_t* drain = bars + 2 * kPipeMaxStages;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 2 * kPipeMaxStages + 1);
    int* s_abort = reinterpret_cast<int*>(s_tmem + 1);
    int* s_never = s_abort + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rank = (int)ptx::cluster_ctarank();
    const int cl = (int)ptx::cluster_id_x();
    if (!tma)
        for (int i = threadIdx.x; i < stages * stage_bytes; i += kThreads) sm[i] = (i & 128) ? 0x22 : 0x00;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kPipeMaxStages; ++i) {
            ptx::mbar_init(&full[i], tma ? 1 : 2);
            ptx::mbar_init(&empty[i], 1);
        }
        ptx::mbar_init(drain, 1);
        *s_abort = 0;
        *s_never = 0;
        ptx::fence_barrier_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 1) {
        ptx::tmem_alloc_pair(s_tmem, 512);
        ptx::tmem_relinquish_pair();
    }
    ptx::tc_fence_before();
    ptx::cluster_sync();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (uint32_t c = 448u; c < 512u; c += 8) ptx::tmem_st8_fill(lane_base + c, 0x7F7F7F7Fu);
    ptx::tmem_wait_st();
    ptx::tc_fence_before();
    ptx::cluster_sync();
    ptx::tc_fence_after();
    volatile int* abort = s_abort;
    if (warp == 0 && lane == 0) {
        const uint32_t full0 = ptx::mapa(full, 0);
        bool pend[kPipeMaxStages];
        uint32_t pend_phase[kPipeMaxStages];
        for (int i = 0; i < kPipeMaxStages; ++i) {
            pend[i] = false;
            pend_phase[i] = 0;
        }
        const int xblocks = pitch / 128;
        const int arow = (cl * 256 + rank * 128) % rows;
        const int brow = ((rows / 2 + cl * N) % (rows - 2 * N)) + rank * (N / 2);
        bool ok = true;
        for (int it = 0; it < iters; ++it) {
            const int s = it % stages;
            const uint32_t ph = (uint32_t)(it / stages) & 1u;
            if (!ptx::mbar_wait(&empty[s], ph ^ 1u, abort, kLimitNs)) {
                ok = false;
                break;
            }
            if (tma) {
                uint8_t* sa = sm + (size_t)s * stage_bytes;
                if (rank == 0) ptx::mbar_arrive_expect_tx(&full[s], 2 * (uint32_t)stage_bytes);
                const uint32_t fb = full0 + (uint32_t)(s * sizeof(uint64_t));
                for (int kb = 0; kb < kbs; ++kb) {
                    const int x = ((it * kbs + kb) % xblocks) * 128;
                    ptx::tma_load_2d_pair(sa + kb * kKbBytes, &ma, x, arow, fb);
                    ptx::tma_load_2d_pair(sa + kb * kKbBytes + 16384, &mb, x, brow, fb);
                }
                pend[s] = rank == 0;
                pend_phase[s] = ph;
            } else {
                ptx::mbar_arrive_cluster(full0 + (uint32_t)(s * sizeof(uint64_t)));
            }
        }
        if (!ok) {
            atomicExch(&g_err, 4);
            *s_abort = 1;
            const uint64_t t0 = ptx::globaltimer();
            while (ptx::globaltimer() - t0 < 200000ull) __nanosleep(1000);
        }
        for (int i = 0; i < kPipeMaxStages; ++i)
            if (pend[i] && !ptx::mbar_wait(&full[i], pend_phase[i], s_never, kLimitNs)) atomicExch(&g_err, 5);
    } else if (warp == 1 && lane == 0) {
        if (rank == 0) {
            const uint32_t idesc = ptx::idesc_mxf4(N, 256);
            const uint32_t sfa = tmem + 448u, sfb = tmem + 480u;
            long long t0 = clock64();
            bool ok = true;
            for (int it = 0; it < iters; ++it) {
                const int s = it % stages;
                const uint32_t ph = (uint32_t)(it / stages) & 1u;
                if (!ptx::mbar_wait(&full[s], ph, abort, kLimitNs)) {
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                const uint32_t acc = N > 224 ? 0u : (uint32_t)(it & 1) * (uint32_t)N;
                for (int kb = 0; kb < kbs; ++kb) {
                    const uint32_t sa = ptx::smem_u32(sm + (size_t)s * stage_bytes + kb * kKbBytes);
                    const uint64_t ad = ptx::smem_desc_sw128(sa), bd = ptx::smem_desc_sw128(sa + 16384);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) ptx::mma_mxf4_pair(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, 1u);
                }
                ptx::mma_commit_pair_mc(&empty[s], 0x3);
            }
            if (!ok) {
                atomicExch(&g_err, 6);
                *s_abort = 1;
            }
            ptx::mma_commit_pair_mc(drain, 0x3);
            if (!ptx::mbar_wait(drain, 0, s_never, kLimitNs)) atomicExch(&g_err, 7);
            cycles[blockIdx.x] = (unsigned long long)(clock64() - t0);
        } else if (!ptx::mbar_wait(drain, 0, s_never, kLimitNs)) {
            atomicExch(&g_err, 8);
        }
    }
    ptx::tc_fence_before();
    ptx::cluster_sync();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc_pair(tmem, 512);
    }
}

}  // namespace

#define CK(x)                                                                               \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) {                                                            \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            return 1;                                                                       \
        }                                                                                   \
    } while (0)

template <int N, bool PAIR>
static int launch(int grid, int groups, int cper, int check, unsigned long long* d_cyc) {
    const size_t smem = smem_bytes<N, PAIR>();
    CK(cudaFuncSetAttribute(f4_kernel<N, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = PAIR ? 2 : 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, f4_kernel<N, PAIR>, groups, cper, check, d_cyc));
    CK(cudaGetLastError());
    return 0;
}

// check: one CTA (one pair); rate: one CTA per SM.  iters = 16-MMA units.
template <int N, bool PAIR>
static int run(int sms, int iters, int cper, int check, unsigned long long* d_cyc) {
    const int unit = PAIR ? 2 : 1;
    const int grid = check ? unit : (sms / unit) * unit;
    const int groups = iters * 16 / cper;
    if (!check) {
        if (launch<N, PAIR>(grid, 64 * 16 / cper, cper, 0, d_cyc)) return 1;  // warm-up
        CK(cudaDeviceSynchronize());
    }
    unsigned long long zero = 0;
    CK(cudaMemcpyToSymbol(g_bad, &zero, sizeof(zero)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    if (launch<N, PAIR>(grid, groups, cper, check, d_cyc)) return 1;
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    int err = 0;
    unsigned long long bad = 0, cyc = 0;
    CK(cudaMemcpyFromSymbol(&err, g_err, sizeof(int)));
    CK(cudaMemcpyFromSymbol(&bad, g_bad, sizeof(bad)));
    CK(cudaMemcpy(&cyc, d_cyc, sizeof(cyc), cudaMemcpyDeviceToHost));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    // MACs of one SM: its 128 rows of D (the pair's M = 256 is split over two SMs).
    const double per_sm = (double)groups * cper * 128.0 * N * 64.0;
    const char* form = PAIR ? "pair" : "cta1";
    if (check)
        printf("{\"form\": \"%s\", \"n\": %d, \"mode\": \"check\", \"k_values\": %d, \"bad_cells\": %llu, "
               "\"err\": %d}\n",
               form, N, groups * cper * 64, bad, err);
    else
        printf("{\"form\": \"%s\", \"n\": %d, \"commit_every\": %d, \"mode\": \"rate\", \"ms\": %.3f, "
               "\"tmacs_per_s\": %.1f, \"mac_per_clk_per_sm\": %.0f, \"err\": %d}\n",
               form, N, cper, ms, per_sm * grid / (ms * 1e-3) / 1e12, per_sm / (double)cyc, err);
    return err || bad ? 1 : 0;
}

template <int N, bool PAIR>
static int rates(int sms, int iters, unsigned long long* d_cyc) {
    int rc = run<N, PAIR>(sms, iters, 16, 0, d_cyc);
    rc |= run<N, PAIR>(sms, iters, 4, 0, d_cyc);
    return rc;
}


// One sweep point: every SM busy (one CTA or pair per SM), `units` x 16 MMAs per SM.
template <int N, bool PAIR>
static int sweep_point(int sms, int units, int cper, int inflight, int sink, int mc, unsigned long long* d_cyc) {
    const size_t smem = sweep_smem_bytes<N, PAIR>();
    CK(cudaFuncSetAttribute(sweep_kernel<N, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int unit = PAIR ? 2 : 1;
    const int grid = (sms / unit) * unit;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unit;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int total = units * 16;
    CK(cudaLaunchKernelEx(&cfg, sweep_kernel<N, PAIR>, 1024, cper, inflight, sink, mc, d_cyc));  // warm-up
    CK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    CK(cudaLaunchKernelEx(&cfg, sweep_kernel<N, PAIR>, total, cper, inflight, sink, mc, d_cyc));
    CK(cudaGetLastError());
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    int err = 0;
    unsigned long long cyc = 0;
    CK(cudaMemcpyFromSymbol(&err, g_err, sizeof(int)));
    CK(cudaMemcpy(&cyc, d_cyc, sizeof(cyc), cudaMemcpyDeviceToHost));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    const double per_sm = (double)(total / cper * cper) * 128.0 * N * 64.0;
    printf("{\"form\": \"%s\", \"n\": %d, \"commit_every\": %d, \"inflight\": %d, \"sink_every\": %d, "
           "\"multicast\": %d, \"ms\": %.3f, \"tmacs_per_s\": %.1f, \"mac_per_clk_per_sm\": %.0f, "
           "\"clk_per_mma\": %.1f, \"sm_mhz_implied\": %.0f, \"err\": %d}\n",
           PAIR ? "pair" : "cta1", N, cper, inflight, sink, mc, ms, per_sm * grid / (ms * 1e-3) / 1e12,
           per_sm / (double)cyc, (double)cyc / (double)(total / cper * cper), (double)cyc / (ms * 1e3), err);
    return err ? 1 : 0;
}

static int sweep(int sms, int units, unsigned long long* d_cyc) {
    int rc = 0;
    const int cps[3] = {4, 8, 16};
    for (int c : cps) {
        rc |= sweep_point<112, true>(sms, units, c, 64, 0, 1, d_cyc);
        rc |= sweep_point<128, true>(sms, units, c, 64, 0, 1, d_cyc);
        rc |= sweep_point<224, true>(sms, units, c, 64, 0, 1, d_cyc);
        rc |= sweep_point<256, true>(sms, units, c, 64, 0, 1, d_cyc);
    }
    // The instruction's asymptotic rate: long commit groups (a commit every
    // 32 and 64 MMAs), the form the roofline of the engine is quoted against.
    for (int c = 32; c <= 64; c *= 2) {
        rc |= sweep_point<112, true>(sms, units, c, 128, 0, 1, d_cyc);
        rc |= sweep_point<256, true>(sms, units, c, 128, 0, 1, d_cyc);
    }
    const int inf[3] = {32, 128, 256};
    for (int f : inf) rc |= sweep_point<112, true>(sms, units, 4, f, 0, 1, d_cyc);
    rc |= sweep_point<112, true>(sms, units, 16, 64, 4, 1, d_cyc);
    rc |= sweep_point<112, true>(sms, units, 16, 64, 8, 1, d_cyc);
    rc |= sweep_point<256, true>(sms, units, 16, 64, 4, 1, d_cyc);
    rc |= sweep_point<112, true>(sms, units, 4, 64, 0, 0, d_cyc);
    rc |= sweep_point<112, true>(sms, units, 16, 64, 0, 0, d_cyc);
    rc |= sweep_point<112, false>(sms, units, 4, 64, 0, 1, d_cyc);
    rc |= sweep_point<112, false>(sms, units, 16, 64, 0, 1, d_cyc);
    rc |= sweep_point<112, false>(sms, units, 16, 64, 4, 1, d_cyc);
    return rc;
}


static PFN_cuTensorMapEncodeTiled_v12000 g_enc = nullptr;

static int encode_map(CUtensorMap* m, void* buf, uint64_t rows, uint64_t pitch, uint32_t box_rows) {
    cuuint64_t dims[2] = {pitch, rows};
    cuuint64_t strides[1] = {pitch};
    cuuint32_t box[2] = {128, box_rows};
    cuuint32_t es[2] = {1, 1};
    if (g_enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, buf, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        fprintf(stderr, "tensor map encode failed\n");
        return 1;
    }
    return 0;
}

// One pipeline point: 74 clusters, `units` x 16 MMAs per pair.
template <int N>
static int pipe_point(int sms, int units, int stages, int kbs, int tma, void* buf, int rows, int pitch,
                      unsigned long long* d_cyc) {
    const size_t smem = 1024 + (size_t)stages * kbs * pipe_kb_bytes<N>() + (2 * kPipeMaxStages + 1) * 8 + 16 + 256;
    if (smem > 232448 || stages > kPipeMaxStages) return 0;
    CUtensorMap ma, mb;
    if (encode_map(&ma, buf, (uint64_t)rows, (uint64_t)pitch, 128) || encode_map(&mb, buf, (uint64_t)rows, (uint64_t)pitch, N / 2))
        return 1;
    CK(cudaFuncSetAttribute(pipe_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((sms / 2) * 2);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int iters = units * 4 / kbs;  // stage iterations: units * 16 MMAs
    CK(cudaLaunchKernelEx(&cfg, pipe_kernel<N>, ma, mb, 64, stages, kbs, tma, rows, pitch, d_cyc));  // warm-up
    CK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    CK(cudaLaunchKernelEx(&cfg, pipe_kernel<N>, ma, mb, iters, stages, kbs, tma, rows, pitch, d_cyc));
    CK(cudaGetLastError());
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    int err = 0;
    unsigned long long cyc = 0;
    CK(cudaMemcpyFromSymbol(&err, g_err, sizeof(int)));
    CK(cudaMemcpy(&cyc, d_cyc, sizeof(cyc), cudaMemcpyDeviceToHost));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    const double mmas = (double)iters * kbs * 4;
    const double per_sm = mmas * 128.0 * N * 64.0;
    printf("{\"form\": \"pipe\", \"n\": %d, \"stages\": %d, \"kblocks_per_stage\": %d, \"mma_per_commit\": %d, "
           "\"tma\": \"%s\", \"ms\": %.3f, \"ns_per_mma\": %.1f, \"tmacs_per_s\": %.1f, \"mac_per_clk_per_sm\": %.0f, "
           "\"sm_mhz_implied\": %.0f, \"err\": %d}\n",
           N, stages, kbs, 4 * kbs, tma ? (rows * (size_t)pitch > (256u << 20) ? "dram" : "l2") : "none", ms,
           ms * 1e6 / mmas, per_sm * cfg.gridDim.x / (ms * 1e-3) / 1e12, per_sm / (double)cyc,
           (double)cyc / (ms * 1e3), err);
    return err ? 1 : 0;
}

static int pipe_sweep(int sms, int units, unsigned long long* d_cyc) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    g_enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    if (!g_enc) return 1;
    // L2-resident (32 MiB) and DRAM-streamed (1 GiB) operand sources.
    const int rows_l2 = 8192, pitch_l2 = 4096, rows_dr = 65536, pitch_dr = 16384;
    void* buf = nullptr;
    CK(cudaMalloc(&buf, (size_t)rows_dr * pitch_dr));
    CK(cudaMemset(buf, 0x22, (size_t)rows_dr * pitch_dr));
    int rc = 0;
    const int cfg112[6][2] = {{4, 1}, {8, 1}, {2, 2}, {3, 2}, {4, 2}, {2, 4}};
    for (auto& c : cfg112)
        for (int t = 0; t < 3; ++t)
            rc |= pipe_point<112>(sms, units, c[0], c[1], t > 0, buf, t == 2 ? rows_dr : rows_l2,
                                  t == 2 ? pitch_dr : pitch_l2, d_cyc);
    const int cfg224[4][2] = {{4, 1}, {6, 1}, {2, 2}, {3, 2}};
    for (auto& c : cfg224)
        for (int t = 0; t < 3; ++t)
            rc |= pipe_point<224>(sms, units, c[0], c[1], t > 0, buf, t == 2 ? rows_dr : rows_l2,
                                  t == 2 ? pitch_dr : pitch_l2, d_cyc);
    const int cfg256[3][2] = {{4, 1}, {6, 1}, {3, 2}};
    for (auto& c : cfg256)
        for (int t = 0; t < 3; ++t)
            rc |= pipe_point<256>(sms, units, c[0], c[1], t > 0, buf, t == 2 ? rows_dr : rows_l2,
                                  t == 2 ? pitch_dr : pitch_l2, d_cyc);
    CK(cudaFree(buf));
    return rc;
}

int main(int argc, char** argv) {
    const bool do_sweep = argc > 1 && std::string(argv[1]) == "sweep";
    const bool do_pipe = argc > 1 && std::string(argv[1]) == "pipe";
    const int a0 = (do_sweep || do_pipe) ? 2 : 1;
    int iters = argc > a0 ? atoi(argv[a0]) : 20000;
    if (iters < 64 || iters > 10000000) iters = 20000;
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, 0));
    if (p.major != 10) {
        fprintf(stderr, "needs an sm_100 device\n");
        return 1;
    }
    printf("{\"gpu\": \"%s\", \"sms\": %d}\n", p.name, p.multiProcessorCount);
    const int sms = p.multiProcessorCount;
    unsigned long long* d_cyc = nullptr;
    CK(cudaMalloc(&d_cyc, sizeof(unsigned long long) * sms));
    int rc = 0;
    if (do_sweep || do_pipe) {
        rc = do_sweep ? sweep(sms, iters, d_cyc) : pipe_sweep(sms, iters, d_cyc);
        CK(cudaFree(d_cyc));
        return rc;
    }
    // Exactness first (4096 x 16 MMAs = 4,194,304 values per count).
    rc |= run<128, false>(sms, 4096, 16, 1, d_cyc);
    rc |= run<112, false>(sms, 4096, 16, 1, d_cyc);
    rc |= run<256, false>(sms, 64, 16, 1, d_cyc);
    rc |= run<112, true>(sms, 4096, 16, 1, d_cyc);
    rc |= run<128, true>(sms, 4096, 16, 1, d_cyc);
    rc |= run<256, true>(sms, 64, 16, 1, d_cyc);
    if (rc) return rc;
    rc |= rates<128, false>(sms, iters, d_cyc);
    rc |= rates<112, false>(sms, iters, d_cyc);
    rc |= rates<256, false>(sms, iters, d_cyc);
    rc |= rates<112, true>(sms, iters, d_cyc);
    rc |= rates<128, true>(sms, iters, d_cyc);
    rc |= rates<256, true>(sms, iters, d_cyc);
    CK(cudaFree(d_cyc));
    return rc;
}
