// common.cuh -- device helpers shared by every counting engine: candidate
// keys, the per-CTA top-K buffer, genotype-table derivation and K2/MI scoring.
//
// Scoring follows include/scoring.hpp of hiperbio/tensor-episdet: CALC_K2
// (scoring.hpp:5-7) and CALC_MI (scoring.hpp:9-16) visited cell by cell in
// index order (scoring.hpp:41-45, :78-84).  Every FP operation is an explicit
// round-to-nearest intrinsic so that the result is reproducible bit for bit
// by a CPU running the same sequence (no contraction, no reassociation).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace episdet {

constexpr int kMaxTopK = 1536;

// Candidate: 32-bit orderable FP32 score key (smaller = better for both K2
// and MI) and the lexicographic set key (pairs a<<32|b, triplets
// x<<42|y<<21|z).  Order: key, then set.
struct __align__(16) Cand {
    uint32_t key;
    uint32_t pad;
    uint64_t set;
};

__host__ __device__ inline bool cand_better(const Cand& a, const Cand& b) {
    return a.key < b.key || (a.key == b.key && a.set < b.set);
}

__host__ __device__ inline Cand cand_worst() {
    Cand c;
    c.key = 0xFFFFFFFFu;
    c.pad = 0;
    c.set = ~0ull;
    return c;
}

__device__ inline uint32_t score_key(float s, bool maximize) {
    if (maximize) s = -s;
    uint32_t u = __float_as_uint(s);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__host__ __device__ inline float key_score(uint32_t key, bool maximize) {
    uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
    float s;
#ifdef __CUDA_ARCH__
    s = __uint_as_float(u);
#else
    __builtin_memcpy(&s, &u, 4);
#endif
    return maximize ? -s : s;
}

__host__ __device__ inline uint64_t set_key3(uint32_t x, uint32_t y, uint32_t z) {
    return ((uint64_t)x << 42) | ((uint64_t)y << 21) | (uint64_t)z;
}
__host__ __device__ inline uint64_t set_key2(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | (uint64_t)b; }

// ------------------------------------------------------------------ scoring
struct ScoreTables {
    const float* t32;   // K2: lnGamma(v+1); MI: log2(v/N), index 0 -> 0
    const double* t64;
    float inv_n32;
    float hy32;
    double inv_n64;
    double hy64;
    int score;          // 0 = K2, 1 = MI
    // K2 only: a bound on |FP32 score - k2_approx32 score| over every valid
    // table of this sample count (the scoring filter of the triplet engine).
    float k2_margin;
};

// The FP32 table's first kLoTab entries are also staged in shared memory by
// the tensor epilogue; both lookups return the same value.
constexpr int kLoTab = 8192;

struct LutGlobal {
    const float* __restrict__ t;
    __device__ __forceinline__ float operator()(int v) const { return __ldg(t + v); }
};
struct LutShared {
    const float* s_lo;  // t[0, kLoTab) in shared memory
    const float* __restrict__ t;
    __device__ __forceinline__ float operator()(int v) const { return v < kLoTab ? s_lo[v] : __ldg(t + v); }
};

// FP32 score of one table, scoring.hpp:5-16 (K2 cell term t[ctrl] + t[case] -
// t[ctrl+case+1]; MI terms), cells in index order.  SC: the score when fixed
// at compile time (EPISDET_SCORE_K2 / _MI), -1 to read T.score.
template <int NC, class Lut, int SC = -1>
__device__ __forceinline__ float score32_lut(const ScoreTables& T, const Lut& lut, const int* cs, const int* cn) {
    if (SC == 0 || (SC < 0 && T.score == 0)) {
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < NC; ++c)
            s = __fadd_rn(s, __fsub_rn(__fadd_rn(lut(cn[c]), lut(cs[c])), lut(cn[c] + cs[c] + 1)));
        return fabsf(s);
    }
    float ha = 0.0f, hx = 0.0f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        float pc = __fmul_rn(__int2float_rn(cs[c]), T.inv_n32);
        ha = __fmaf_rn(-pc, lut(cs[c]), ha);
        float pn = __fmul_rn(__int2float_rn(cn[c]), T.inv_n32);
        ha = __fmaf_rn(-pn, lut(cn[c]), ha);
        hx = __fmaf_rn(-__fadd_rn(pc, pn), lut(cs[c] + cn[c]), hx);
    }
    return __fsub_rn(__fadd_rn(hx, T.hy32), ha);
}

// ------------------------------------------------- K2 scoring filter
// lnGamma(v + 1) without a table: the exact FP32 table value for v <
// kSmallTab (from a 32-entry shared-memory copy, one entry per bank, so any
// gather is conflict-free) and above it Stirling's series cut after its
// constant term, (z - 1/2) ln z - z + ln(2 pi) / 2 with z = v + 1 (the next
// term, 1/(12 z), is below 0.0026 there), in FP32 with the hardware log2.
// Every step is an explicit round-to-nearest operation, so the value of a
// given v is the same wherever it is evaluated; the largest distance to the
// FP32 table over 0 <= v <= N + 1 is measured once per sample count
// (k2_filter_margin) and the filter's bound is built from it.
constexpr int kSmallTab = 32;
constexpr float kLn2f = 0.693147182464599609375f;      // ln 2 rounded to float
constexpr float kHalfLn2Pif = 0.918938517570495605469f;  // ln(2 pi) / 2 rounded to float

__device__ __forceinline__ float lngamma1_stirling(int v) {
    const float z = __int2float_rn(v + 1);
    const float lnz = __fmul_rn(__log2f(z), kLn2f);
    return __fmaf_rn(__fsub_rn(z, 0.5f), lnz, __fsub_rn(kHalfLn2Pif, z));
}

__device__ __forceinline__ float lngamma1_filter(const float* s_small, int v) {
    return v < kSmallTab ? s_small[v] : lngamma1_stirling(v);
}

// The K2 score of one table with lngamma1_filter in place of the table, in
// the cell order and operation sequence of score32_lut.  Its distance to the
// exact FP32 score is at most ScoreTables::k2_margin.
template <int NC>
__device__ __forceinline__ float k2_approx32(const float* s_small, const int* cs, const int* cn) {
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < NC; ++c)
        s = __fadd_rn(s, __fsub_rn(__fadd_rn(lngamma1_filter(s_small, cn[c]), lngamma1_filter(s_small, cs[c])),
                                   lngamma1_filter(s_small, cn[c] + cs[c] + 1)));
    return fabsf(s);
}

template <int NC>
__device__ __forceinline__ float score32(const ScoreTables& T, const int* cs, const int* cn) {
    return score32_lut<NC>(T, LutGlobal{T.t32}, cs, cn);
}

template <int NC>
__device__ __forceinline__ double score64(const ScoreTables& T, const int* cs, const int* cn) {
    if (T.score == 0) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double term = __dsub_rn(__dadd_rn(T.t64[cn[c]], T.t64[cs[c]]), T.t64[cn[c] + cs[c] + 1]);
            s = __dadd_rn(s, term);
        }
        return fabs(s);
    }
    double ha = 0.0, hx = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        double pc = __dmul_rn((double)cs[c], T.inv_n64);
        ha = __fma_rn(-pc, T.t64[cs[c]], ha);
        double pn = __dmul_rn((double)cn[c], T.inv_n64);
        ha = __fma_rn(-pn, T.t64[cn[c]], ha);
        hx = __fma_rn(-__dadd_rn(pc, pn), T.t64[cs[c] + cn[c]], hx);
    }
    return __dsub_rn(__dadd_rn(hx, T.hy64), ha);
}

// --------------------------------------------------------------- derivation
// 2-way table, src/helper.cu:634-662: t[i*3+j] for i,j<2 hold the AND cells;
// pa/pb are the genotype counts (g2 = n - g0 - g1) of the two SNPs.
__device__ __forceinline__ void derive9(int t[9], const int pa[3], const int pb[3]) {
    t[0 * 3 + 2] = pa[0] - (t[0 * 3 + 0] + t[0 * 3 + 1]);
    t[1 * 3 + 2] = pa[1] - (t[1 * 3 + 0] + t[1 * 3 + 1]);
    t[2 * 3 + 0] = pb[0] - (t[0 * 3 + 0] + t[1 * 3 + 0]);
    t[2 * 3 + 1] = pb[1] - (t[0 * 3 + 1] + t[1 * 3 + 1]);
    t[2 * 3 + 2] = pa[2] - (t[2 * 3 + 0] + t[2 * 3 + 1]);
}

#define EPI_C3(i, j, k) ((i) * 9 + (j) * 3 + (k))
// 3-way table, src/helper.cu:494-548 with the macros of include/helper.hpp:34-51.
// On entry t holds the 8 AND cells (i,j,k < 2); xy/xz/yz are 9-cell pair tables.
__device__ __forceinline__ void derive27(int t[27], const int xy[9], const int xz[9], const int yz[9]) {
    t[EPI_C3(0, 0, 2)] = xy[0] - (t[EPI_C3(0, 0, 0)] + t[EPI_C3(0, 0, 1)]);
    t[EPI_C3(0, 1, 2)] = xy[1] - (t[EPI_C3(0, 1, 0)] + t[EPI_C3(0, 1, 1)]);
    t[EPI_C3(0, 2, 0)] = xz[0] - (t[EPI_C3(0, 0, 0)] + t[EPI_C3(0, 1, 0)]);
    t[EPI_C3(0, 2, 1)] = xz[1] - (t[EPI_C3(0, 0, 1)] + t[EPI_C3(0, 1, 1)]);
    t[EPI_C3(0, 2, 2)] = xz[2] - (t[EPI_C3(0, 0, 2)] + t[EPI_C3(0, 1, 2)]);
    t[EPI_C3(1, 0, 2)] = xy[3] - (t[EPI_C3(1, 0, 0)] + t[EPI_C3(1, 0, 1)]);
    t[EPI_C3(1, 1, 2)] = xy[4] - (t[EPI_C3(1, 1, 0)] + t[EPI_C3(1, 1, 1)]);
    t[EPI_C3(1, 2, 0)] = xz[3] - (t[EPI_C3(1, 0, 0)] + t[EPI_C3(1, 1, 0)]);
    t[EPI_C3(1, 2, 1)] = xz[4] - (t[EPI_C3(1, 0, 1)] + t[EPI_C3(1, 1, 1)]);
    t[EPI_C3(1, 2, 2)] = xz[5] - (t[EPI_C3(1, 0, 2)] + t[EPI_C3(1, 1, 2)]);
    t[EPI_C3(2, 0, 0)] = yz[0] - (t[EPI_C3(0, 0, 0)] + t[EPI_C3(1, 0, 0)]);
    t[EPI_C3(2, 0, 1)] = yz[1] - (t[EPI_C3(0, 0, 1)] + t[EPI_C3(1, 0, 1)]);
    t[EPI_C3(2, 0, 2)] = xy[6] - (t[EPI_C3(2, 0, 0)] + t[EPI_C3(2, 0, 1)]);
    t[EPI_C3(2, 1, 0)] = yz[3] - (t[EPI_C3(0, 1, 0)] + t[EPI_C3(1, 1, 0)]);
    t[EPI_C3(2, 1, 1)] = yz[4] - (t[EPI_C3(0, 1, 1)] + t[EPI_C3(1, 1, 1)]);
    t[EPI_C3(2, 1, 2)] = xy[7] - (t[EPI_C3(2, 1, 0)] + t[EPI_C3(2, 1, 1)]);
    t[EPI_C3(2, 2, 0)] = xz[6] - (t[EPI_C3(2, 0, 0)] + t[EPI_C3(2, 1, 0)]);
    t[EPI_C3(2, 2, 1)] = xz[7] - (t[EPI_C3(2, 0, 1)] + t[EPI_C3(2, 1, 1)]);
    t[EPI_C3(2, 2, 2)] = xz[8] - (t[EPI_C3(2, 0, 2)] + t[EPI_C3(2, 1, 2)]);
}

// 9-cell pair table from its 4 AND cells and the two SNPs' genotype counts
// (the 2-way derivation of helper.cu:645-662; equal to the masked direct
// count of helper.cu:58-194 for valid inputs).
__device__ __forceinline__ void pair9_from4(int out[9], const uint4& and4, const int ma[3], const int mb[3]) {
    out[0] = (int)and4.x;
    out[1] = (int)and4.y;
    out[3] = (int)and4.z;
    out[4] = (int)and4.w;
    derive9(out, ma, mb);
}

// ------------------------------------------------------- per-CTA top-K list
// Shared-memory candidate buffer of capacity CAP (power of two).  Threads
// offer() candidates better than the local threshold with a shared atomic;
// callers compact() (all NT threads, between barriers) before the buffer can
// overflow.  After compact() the first min(count, K) entries are sorted best
// first and the threshold is the K-th entry.
template <int CAP, int NT>
struct LocalTopK {
    static_assert(CAP > 0 && (CAP & (CAP - 1)) == 0, "compact() is a bitonic sort over a power-of-two buffer");
    Cand* buf;     // [CAP]
    int* count;    // shared scalar
    Cand* thr;     // shared scalar
    int k;
    int tid;
    uint32_t* gkey = nullptr;  // optional: search-wide smallest k-th key (Slots::gkey)

    // `hi` is this thread's highest slot + 1 since the last compaction.  The
    // atomic hands slots out in order, so the largest `hi` over the threads is
    // the buffer's fill; check() reduces it at a barrier.
    __device__ void offer(const Cand& c, const Cand& thr_reg, int& hi) const {
        if (cand_better(c, thr_reg)) {
            int slot = atomicAdd(count, 1);
            buf[slot] = c;
            hi = slot + 1;
        }
    }

    // Compacts when the buffer holds more than `limit` entries (limit >= k).
    // The decision is an OR over the threads' own slots taken at the barrier,
    // so it is exact and the same in every thread even when faster threads
    // already offer again after the barrier.
    template <class Bar>
    __device__ void check(int& hi, int limit, Bar bar) const {
        if (bar.any(hi > limit)) {
            compact(bar);
            hi = 0;
        }
    }

    // Bitonic sort of buf[0..P), P the power of two >= n (at most CAP), with
    // entries >= n set to worst; requires a barrier functor covering exactly
    // the NT participating threads, and every offer of those threads must be
    // ordered before the call by a barrier (so every thread reads the same n).
    template <class Bar>
    __device__ void compact(Bar bar) const {
        int n = *count;
        int P = 2;
        while (P < n) P <<= 1;
        for (int i = n + tid; i < P; i += NT) buf[i] = cand_worst();
        bar();
        for (int kk = 2; kk <= P; kk <<= 1) {
            for (int j = kk >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < P; i += NT) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        Cand a = buf[i], b = buf[ixj];
                        bool up = (i & kk) == 0;
                        if (up ? cand_better(b, a) : cand_better(a, b)) {
                            buf[i] = b;
                            buf[ixj] = a;
                        }
                    }
                }
                bar();
            }
        }
        if (tid == 0) {
            int m = n < k ? n : k;
            *count = m;
            *thr = (m >= k) ? buf[k - 1] : cand_worst();
            if (gkey && m >= k) atomicMin(gkey, buf[k - 1].key);
        }
        bar();
    }

    template <class Bar>
    __device__ void load(const Cand* __restrict__ slot, int slot_count, Bar bar) const {
        for (int i = tid; i < slot_count; i += NT) buf[i] = slot[i];
        if (tid == 0) {
            *count = slot_count;
            *thr = (slot_count >= k) ? slot[k - 1] : cand_worst();
            if (gkey && slot_count >= k) atomicMin(gkey, slot[k - 1].key);
        }
        bar();
    }

    // Every thread's last offers must land before the count is read: callers
    // reach this without a barrier after their final offers.
    template <class Bar>
    __device__ void store(Cand* __restrict__ slot, int* __restrict__ slot_count, Bar bar) const {
        bar();
        compact(bar);
        int n = *count;
        for (int i = tid; i < n; i += NT) slot[i] = buf[i];
        if (tid == 0) *slot_count = n;
    }
};

struct BarAll {
    __device__ void operator()() const { __syncthreads(); }
    __device__ bool any(bool q) const { return __syncthreads_or(q) != 0; }
};

// Named barrier over `n` threads (multiple of 32) of one CTA.
struct BarNamed {
    int id, n;
    __device__ void operator()() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
    // Barrier that also returns whether any participating thread passed q.
    __device__ bool any(bool q) const {
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p, q;\n\t"
            "setp.ne.u32 q, %3, 0;\n\t"
            "bar.red.or.pred p, %1, %2, q;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(r)
            : "r"(id), "r"(n), "r"((uint32_t)q)
            : "memory");
        return r != 0;
    }
};

}  // namespace episdet
