// kernels_simt.cu -- integer-pipe (LOP3 + POPC) counting engine and the
// engine-independent kernels: marginals/validation, top-K merge, FP64 re-score.
//
// The SIMT engine is the straightforward reading of the reference's count
// kernels (src/helper.cu:13-425) fused with its objective kernels
// (src/helper.cu:438-698): counts stay in registers and every set is scored
// in the same kernel.  It is kept beside the tensor-core engine as an
// independent GPU cross-check.
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"
#include "device_data.cuh"
#include "kernels.h"

namespace episdet {

// ------------------------------------------------------------- marginals
// helper.cu:13-52: g0/g1 popcounts per SNP and class, g2 = n - g0 - g1.  The
// same pass checks the input contract: zero padding bits, disjoint planes.
// One warp per (SNP, class); 128-bit loads.
__global__ void __launch_bounds__(256) marginals_kernel(DevData D, int* marg0, int* marg1, int* bad_flag) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int M = D.M;
    if (warp >= 2 * M) return;
    int c = warp / M, snp = warp % M;
    int W = D.W[c], n = D.n[c];
    const uint4* r0 = reinterpret_cast<const uint4*>(D.bits[c] + ((size_t)snp * 2 + 0) * W);
    const uint4* r1 = reinterpret_cast<const uint4*>(D.bits[c] + ((size_t)snp * 2 + 1) * W);
    int c0 = 0, c1 = 0;
    uint32_t bad = 0;
    for (int q = lane; q < W / 4; q += 32) {
        uint4 a = r0[q], b = r1[q];
        uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int w = q * 4 + e;
            int lo = w * 32;
            uint32_t m = (lo + 32 <= n) ? 0xFFFFFFFFu : (lo >= n ? 0u : (0xFFFFFFFFu << (32 - (n - lo))));
            bad |= (av[e] & ~m) | (bv[e] & ~m) | (av[e] & bv[e]);
            c0 += __popc(av[e]);
            c1 += __popc(bv[e]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(0xFFFFFFFFu, c0, o);
        c1 += __shfl_xor_sync(0xFFFFFFFFu, c1, o);
        bad |= __shfl_xor_sync(0xFFFFFFFFu, bad, o);
    }
    if (lane == 0) {
        int* m = c == 0 ? marg0 : marg1;
        m[snp] = c0;
        m[M + snp] = c1;
        m[2 * M + snp] = n - (c0 + c1);
        if (bad) atomicOr(bad_flag, 1);
    }
}

// ------------------------------------------------------------ SIMT 2-way
constexpr int kTS = 32;                // SNPs per tile side
constexpr int kChunk = 32;             // words per K chunk
constexpr int kRowStride = kChunk + 1; // padded shared row (bank spread)
constexpr int kSimtThreads = 256;
constexpr int kSimtCap = 4096;         // local top-K capacity
constexpr int kSimtPerStep = kSimtThreads * 4;
static_assert(kSimtCap - kSimtPerStep >= kMaxTopK, "the fill check needs room for k entries");

__device__ __forceinline__ void simt_load_tile(uint32_t* s, const uint32_t* __restrict__ bits, int W, int M, int snp0,
                                               int chunk) {
    // 64 rows (snp*2+g) x 32 words, 8 uint4 per row.
    for (int idx = threadIdx.x; idx < 64 * 8; idx += kSimtThreads) {
        int r = idx >> 3, q = idx & 7;
        int snp = snp0 + (r >> 1);
        uint4 v = make_uint4(0, 0, 0, 0);
        if (snp < M) v = *reinterpret_cast<const uint4*>(bits + ((size_t)snp * 2 + (r & 1)) * W + chunk * kChunk + q * 4);
        uint32_t* d = s + r * kRowStride + q * 4;
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
    }
}

extern "C" __global__ void __launch_bounds__(kSimtThreads)
    search2_simt_kernel(DevData D, ScoreTables T, const int2* __restrict__ tiles, int ntiles, int first_begin,
                        int first_end, Slots S, int store_pairs, uint4* pair_out0, uint4* pair_out1) {
    extern __shared__ __align__(16) unsigned char smem[];
    Cand* tbuf = reinterpret_cast<Cand*>(smem);
    uint32_t* sA = reinterpret_cast<uint32_t*>(smem + sizeof(Cand) * kSimtCap);
    uint32_t* sB = sA + 64 * kRowStride;
    int* s_count = reinterpret_cast<int*>(sB + 64 * kRowStride);
    Cand* s_thr = reinterpret_cast<Cand*>(s_count + 4);

    LocalTopK<kSimtCap, kSimtThreads> tk{tbuf, s_count, s_thr, S.k, (int)threadIdx.x};
    int hi = 0;  // this thread's highest candidate slot + 1 since the last compaction
    if (!store_pairs) tk.load(S.lists + (size_t)blockIdx.x * S.k, S.counts[blockIdx.x], BarAll());
    const bool maximize = T.score == 1;
    const int ai = threadIdx.x & 15, bi = threadIdx.x >> 4;
    const int M = D.M;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int2 tile = tiles[t];
        int a0 = tile.x * kTS, b0 = tile.y * kTS;
        int cnt[2][2][2][4];  // [class][a][b][ij]
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int x = 0; x < 2; ++x)
#pragma unroll
                for (int y = 0; y < 2; ++y)
#pragma unroll
                    for (int e = 0; e < 4; ++e) cnt[c][x][y][e] = 0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int W = D.W[c];
            for (int ch = 0; ch < W / kChunk; ++ch) {
                __syncthreads();
                simt_load_tile(sA, D.bits[c], W, M, a0, ch);
                simt_load_tile(sB, D.bits[c], W, M, b0, ch);
                __syncthreads();
#pragma unroll 4
                for (int w = 0; w < kChunk; ++w) {
                    uint32_t A[2][2], B[2][2];
#pragma unroll
                    for (int x = 0; x < 2; ++x)
#pragma unroll
                        for (int g = 0; g < 2; ++g) {
                            A[x][g] = sA[((2 * ai + x) * 2 + g) * kRowStride + w];
                            B[x][g] = sB[((2 * bi + x) * 2 + g) * kRowStride + w];
                        }
#pragma unroll
                    for (int x = 0; x < 2; ++x)
#pragma unroll
                        for (int y = 0; y < 2; ++y) {
                            cnt[c][x][y][0] += __popc(A[x][0] & B[y][0]);
                            cnt[c][x][y][1] += __popc(A[x][0] & B[y][1]);
                            cnt[c][x][y][2] += __popc(A[x][1] & B[y][0]);
                            cnt[c][x][y][3] += __popc(A[x][1] & B[y][1]);
                        }
                }
            }
        }
        // epilogue
        Cand thr = *s_thr;
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                int a = a0 + 2 * ai + x, b = b0 + 2 * bi + y;
                bool ok = a < b && b < M && a >= first_begin && a < first_end;
                if (store_pairs) {
                    if (a < b && b < M) {
                        size_t o = (size_t)a * M + b;
                        pair_out0[o] = make_uint4(cnt[0][x][y][0], cnt[0][x][y][1], cnt[0][x][y][2], cnt[0][x][y][3]);
                        pair_out1[o] = make_uint4(cnt[1][x][y][0], cnt[1][x][y][1], cnt[1][x][y][2], cnt[1][x][y][3]);
                    }
                    continue;
                }
                if (!ok) continue;
                int cs[9], cn[9], ma[3], mb[3];
                cs[0] = cnt[0][x][y][0];
                cs[1] = cnt[0][x][y][1];
                cs[3] = cnt[0][x][y][2];
                cs[4] = cnt[0][x][y][3];
                load_marg3(D.marg[0], M, a, ma);
                load_marg3(D.marg[0], M, b, mb);
                derive9(cs, ma, mb);
                cn[0] = cnt[1][x][y][0];
                cn[1] = cnt[1][x][y][1];
                cn[3] = cnt[1][x][y][2];
                cn[4] = cnt[1][x][y][3];
                load_marg3(D.marg[1], M, a, ma);
                load_marg3(D.marg[1], M, b, mb);
                derive9(cn, ma, mb);
                float s = score32<9>(T, cs, cn);
                Cand cd;
                cd.key = score_key(s, maximize);
                cd.pad = 0;
                cd.set = set_key2((uint32_t)a, (uint32_t)b);
                tk.offer(cd, thr, hi);
            }
        if (!store_pairs) tk.check(hi, kSimtCap - kSimtPerStep, BarAll());
    }
    if (!store_pairs) tk.store(S.lists + (size_t)blockIdx.x * S.k, S.counts + blockIdx.x, BarAll());
}

// ------------------------------------------------------------ SIMT 3-way
// One launch per X.  Tile = 32 Y x 32 Z; thread (ai, bi) counts Y in
// {y0+2ai, +1} against Z in {z0+2bi, +1}: 8 AND cells X_i&Y_j&Z_k per
// (Y,Z) and class.  The X_i&Y_j operand of src/helper.cu:396-425 is formed in
// registers and never stored.
extern "C" __global__ void __launch_bounds__(kSimtThreads)
    search3_simt_kernel(DevData D, ScoreTables T, int xsnp, const int2* __restrict__ tiles, int ntiles, Slots S) {
    extern __shared__ __align__(16) unsigned char smem[];
    Cand* tbuf = reinterpret_cast<Cand*>(smem);
    uint32_t* sA = reinterpret_cast<uint32_t*>(smem + sizeof(Cand) * kSimtCap);
    uint32_t* sB = sA + 64 * kRowStride;
    uint32_t* sX = sB + 64 * kRowStride;  // [2][kChunk]
    int* s_count = reinterpret_cast<int*>(sX + 2 * kChunk);
    Cand* s_thr = reinterpret_cast<Cand*>(s_count + 4);

    LocalTopK<kSimtCap, kSimtThreads> tk{tbuf, s_count, s_thr, S.k, (int)threadIdx.x};
    int hi = 0;  // this thread's highest candidate slot + 1 since the last compaction
    tk.load(S.lists + (size_t)blockIdx.x * S.k, S.counts[blockIdx.x], BarAll());
    const bool maximize = T.score == 1;
    const int ai = threadIdx.x & 15, bi = threadIdx.x >> 4;
    const int M = D.M;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int2 tile = tiles[t];
        int y0 = tile.x * kTS, z0 = tile.y * kTS;
        int cnt[2][2][2][8];  // [class][y][z][ijk]
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int x = 0; x < 2; ++x)
#pragma unroll
                for (int y = 0; y < 2; ++y)
#pragma unroll
                    for (int e = 0; e < 8; ++e) cnt[c][x][y][e] = 0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int W = D.W[c];
            const uint32_t* xr = D.bits[c] + (size_t)xsnp * 2 * W;
            for (int ch = 0; ch < W / kChunk; ++ch) {
                __syncthreads();
                simt_load_tile(sA, D.bits[c], W, M, y0, ch);
                simt_load_tile(sB, D.bits[c], W, M, z0, ch);
                if (threadIdx.x < 2 * kChunk) {
                    int g = threadIdx.x / kChunk, w = threadIdx.x % kChunk;
                    sX[threadIdx.x] = xr[(size_t)g * W + ch * kChunk + w];
                }
                __syncthreads();
#pragma unroll 2
                for (int w = 0; w < kChunk; ++w) {
                    uint32_t X0 = sX[w], X1 = sX[kChunk + w];
                    uint32_t Z[2][2];
#pragma unroll
                    for (int y = 0; y < 2; ++y)
#pragma unroll
                        for (int g = 0; g < 2; ++g) Z[y][g] = sB[((2 * bi + y) * 2 + g) * kRowStride + w];
#pragma unroll
                    for (int x = 0; x < 2; ++x) {
                        uint32_t Y0 = sA[((2 * ai + x) * 2 + 0) * kRowStride + w];
                        uint32_t Y1 = sA[((2 * ai + x) * 2 + 1) * kRowStride + w];
                        uint32_t XY[4] = {X0 & Y0, X0 & Y1, X1 & Y0, X1 & Y1};
#pragma unroll
                        for (int y = 0; y < 2; ++y)
#pragma unroll
                            for (int ij = 0; ij < 4; ++ij) {
                                cnt[c][x][y][ij * 2 + 0] += __popc(XY[ij] & Z[y][0]);
                                cnt[c][x][y][ij * 2 + 1] += __popc(XY[ij] & Z[y][1]);
                            }
                    }
                }
            }
        }
        Cand thr = *s_thr;
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                int ys = y0 + 2 * ai + x, zs = z0 + 2 * bi + y;
                if (!(xsnp < ys && ys < zs && zs < M)) continue;
                int tab[2][27];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    int* tt = tab[c];
#pragma unroll
                    for (int i = 0; i < 2; ++i)
#pragma unroll
                        for (int j = 0; j < 2; ++j)
#pragma unroll
                            for (int k = 0; k < 2; ++k) tt[EPI_C3(i, j, k)] = cnt[c][x][y][(i * 2 + j) * 2 + k];
                    int mx[3], my[3], mz[3], xy[9], xz[9], yz[9];
                    load_marg3(D.marg[c], M, xsnp, mx);
                    load_marg3(D.marg[c], M, ys, my);
                    load_marg3(D.marg[c], M, zs, mz);
                    pair9_from4(xy, __ldg(D.pair4[c] + (size_t)xsnp * M + ys), mx, my);
                    pair9_from4(xz, __ldg(D.pair4[c] + (size_t)xsnp * M + zs), mx, mz);
                    pair9_from4(yz, __ldg(D.pair4[c] + (size_t)ys * M + zs), my, mz);
                    derive27(tt, xy, xz, yz);
                }
                float s = score32<27>(T, tab[0], tab[1]);
                Cand cd;
                cd.key = score_key(s, maximize);
                cd.pad = 0;
                cd.set = set_key3((uint32_t)xsnp, (uint32_t)ys, (uint32_t)zs);
                tk.offer(cd, thr, hi);
            }
        tk.check(hi, kSimtCap - kSimtPerStep, BarAll());
    }
    tk.store(S.lists + (size_t)blockIdx.x * S.k, S.counts + blockIdx.x, BarAll());
}

// ------------------------------------------------------------ top-K merge
// Single CTA: merges every slot list into the global best-k, batch by batch
// through an 8192-entry bitonic sort in shared memory.
constexpr int kMergeCap = 8192;
constexpr int kMergeThreads = 1024;
constexpr int kRadixBits = 11;

// In-place ascending bitonic sort of buf[0, n) (n a power of two <= kMergeCap).
__device__ void merge_sort_smem(Cand* buf, int n) {
    for (int kk = 2; kk <= n; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n; i += kMergeThreads) {
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
            __syncthreads();
        }
}

// Exact global top-k of the per-CTA candidate lists, by (key, set).
//
// Radix selection first: three 11-bit histogram passes over the keys of every
// listed candidate find T, the k-th smallest key.  The candidates with key <= T
// contain the top k; they are gathered and sorted alone.  When ties at T
// exceed the buffer the kernel falls back to merging the lists chunk by chunk.
extern "C" __global__ void __launch_bounds__(kMergeThreads) merge_topk_kernel(Slots S, Cand* out, int* out_count) {
    extern __shared__ __align__(16) unsigned char smem[];
    Cand* buf = reinterpret_cast<Cand*>(smem);
    int* hist = reinterpret_cast<int*>(smem);  // aliases buf while selecting
    __shared__ uint32_t s_prefix, s_mask;
    __shared__ int s_need, s_total, s_n;
    const int k = S.k;
    const long total = (long)S.nslots * k;
    auto key_at = [&](long idx, uint32_t& key) -> bool {
        const int s = (int)(idx / k), e = (int)(idx % k);
        if (e >= S.counts[s]) return false;
        key = S.lists[idx].key;
        return true;
    };
    if (threadIdx.x == 0) {
        s_prefix = 0;
        s_mask = 0;
        s_need = k;
        s_total = 0;
    }
    __syncthreads();
    // Number of listed candidates.
    int mine = 0;
    for (long idx = threadIdx.x; idx < total; idx += kMergeThreads) {
        uint32_t key;
        mine += key_at(idx, key) ? 1 : 0;
    }
    atomicAdd(&s_total, mine);
    __syncthreads();
    uint32_t thr = 0xFFFFFFFFu;  // keep everything when there are at most k candidates
    if (s_total > k) {
        for (int pass = 0; pass < 3; ++pass) {
            const int shift = pass == 0 ? 21 : (pass == 1 ? 10 : 0);
            const int bits = pass == 2 ? 10 : kRadixBits;
            const int nb = 1 << bits;
            for (int i = threadIdx.x; i < nb; i += kMergeThreads) hist[i] = 0;
            __syncthreads();
            const uint32_t prefix = s_prefix, mask = s_mask;
            for (long idx = threadIdx.x; idx < total; idx += kMergeThreads) {
                uint32_t key;
                if (key_at(idx, key) && (key & mask) == prefix) atomicAdd(&hist[(key >> shift) & (nb - 1)], 1);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int need = s_need, acc = 0, bin = 0;
                while (acc + hist[bin] < need) acc += hist[bin++];
                s_need = need - acc;
                s_prefix = prefix | ((uint32_t)bin << shift);
                s_mask = mask | ((uint32_t)(nb - 1) << shift);
            }
            __syncthreads();
        }
        thr = s_prefix;  // the k-th smallest key
    }
    // Gather every candidate with key <= thr.
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    for (long idx = threadIdx.x; idx < total; idx += kMergeThreads) {
        uint32_t key;
        if (key_at(idx, key) && key <= thr) {
            const int slot = atomicAdd(&s_n, 1);
            if (slot < kMergeCap) buf[slot] = S.lists[idx];
        }
    }
    __syncthreads();
    const int n = s_n;
    if (n <= kMergeCap) {
        int p2 = 1;
        while (p2 < n) p2 <<= 1;
        for (int i = n + (int)threadIdx.x; i < p2; i += kMergeThreads) buf[i] = cand_worst();
        __syncthreads();
        merge_sort_smem(buf, p2);
        const int r = n < k ? n : k;
        for (int i = threadIdx.x; i < k; i += kMergeThreads) out[i] = i < r ? buf[i] : cand_worst();
        if (threadIdx.x == 0) *out_count = r;
        return;
    }
    // Ties at thr overflow the buffer: merge the lists chunk by chunk.
    const int room = kMergeCap - k;
    __shared__ int s_r;
    if (threadIdx.x == 0) s_r = 0;
    __syncthreads();
    for (long pos = 0; pos < total; pos += room) {
        int r = s_r;
        for (int i = threadIdx.x; i < kMergeCap; i += kMergeThreads) {
            if (i < r) continue;
            long idx = pos + (i - r);
            Cand c = cand_worst();
            if (i - r < room && idx < total) {
                int s = (int)(idx / k), e = (int)(idx % k);
                if (e < S.counts[s]) c = S.lists[idx];
            }
            buf[i] = c;
        }
        __syncthreads();
        merge_sort_smem(buf, kMergeCap);
        if (threadIdx.x == 0) {
            int m = 0;
            while (m < k && buf[m].key != 0xFFFFFFFFu) ++m;
            s_r = m;
        }
        __syncthreads();
    }
    int r = s_r;
    for (int i = threadIdx.x; i < k; i += kMergeThreads) out[i] = i < r ? buf[i] : cand_worst();
    if (threadIdx.x == 0) *out_count = r;
}

// --------------------------------------------------------- FP64 re-score
// One warp per candidate: exact recount of the AND cells from the packed
// planes, derivation as in the objective kernels, FP64 score.
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

extern "C" __global__ void __launch_bounds__(256)
    rescore_kernel(DevData D, ScoreTables T, int order, const Cand* __restrict__ cands, const int* count,
                   double* fp64_out, int* cells_out) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= *count) return;
    Cand cd = cands[warp];
    uint32_t xs, ys, zs;
    if (order == 2) {
        xs = (uint32_t)(cd.set >> 32);
        ys = (uint32_t)(cd.set & 0xFFFFFFFFu);
        zs = 0;
    } else {
        xs = (uint32_t)((cd.set >> 42) & 0x1FFFFF);
        ys = (uint32_t)((cd.set >> 21) & 0x1FFFFF);
        zs = (uint32_t)(cd.set & 0x1FFFFF);
    }
    const int M = D.M;
    // A set outside the dataset (a corrupt candidate) reads no planes: its
    // score is NaN, which the host reports as an internal error.
    const bool valid = order == 2 ? (xs < ys && ys < (uint32_t)M) : (xs < ys && ys < zs && zs < (uint32_t)M);
    if (!valid) {
        if (lane == 0) fp64_out[warp] = __longlong_as_double(0x7FF8000000000000ll);
        return;
    }
    int tab[2][27];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int W = D.W[c];
        const uint32_t* X0 = D.bits[c] + ((size_t)xs * 2 + 0) * W;
        const uint32_t* X1 = X0 + W;
        const uint32_t* Y0 = D.bits[c] + ((size_t)ys * 2 + 0) * W;
        const uint32_t* Y1 = Y0 + W;
        if (order == 2) {
            uint32_t a[4] = {0, 0, 0, 0};
            for (int w = lane; w < W; w += 32) {
                uint32_t x0 = X0[w], x1 = X1[w], y0 = Y0[w], y1 = Y1[w];
                a[0] += __popc(x0 & y0);
                a[1] += __popc(x0 & y1);
                a[2] += __popc(x1 & y0);
                a[3] += __popc(x1 & y1);
            }
            int* tt = tab[c];
            tt[0] = (int)warp_sum(a[0]);
            tt[1] = (int)warp_sum(a[1]);
            tt[3] = (int)warp_sum(a[2]);
            tt[4] = (int)warp_sum(a[3]);
            int ma[3], mb[3];
            load_marg3(D.marg[c], M, xs, ma);
            load_marg3(D.marg[c], M, ys, mb);
            derive9(tt, ma, mb);
        } else {
            const uint32_t* Z0 = D.bits[c] + ((size_t)zs * 2 + 0) * W;
            const uint32_t* Z1 = Z0 + W;
            uint32_t t8[8] = {0, 0, 0, 0, 0, 0, 0, 0}, pxy[4] = {0, 0, 0, 0}, pxz[4] = {0, 0, 0, 0},
                     pyz[4] = {0, 0, 0, 0};
            for (int w = lane; w < W; w += 32) {
                uint32_t x[2] = {X0[w], X1[w]}, y[2] = {Y0[w], Y1[w]}, z[2] = {Z0[w], Z1[w]};
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        pxy[i * 2 + j] += __popc(x[i] & y[j]);
                        pxz[i * 2 + j] += __popc(x[i] & z[j]);
                        pyz[i * 2 + j] += __popc(y[i] & z[j]);
#pragma unroll
                        for (int k = 0; k < 2; ++k) t8[(i * 2 + j) * 2 + k] += __popc(x[i] & y[j] & z[k]);
                    }
            }
            int* tt = tab[c];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int k = 0; k < 2; ++k) tt[EPI_C3(i, j, k)] = (int)warp_sum(t8[(i * 2 + j) * 2 + k]);
            int mx[3], my[3], mz[3], xy[9], xz[9], yz[9];
            load_marg3(D.marg[c], M, xs, mx);
            load_marg3(D.marg[c], M, ys, my);
            load_marg3(D.marg[c], M, zs, mz);
            uint4 v;
            v = make_uint4(warp_sum(pxy[0]), warp_sum(pxy[1]), warp_sum(pxy[2]), warp_sum(pxy[3]));
            pair9_from4(xy, v, mx, my);
            v = make_uint4(warp_sum(pxz[0]), warp_sum(pxz[1]), warp_sum(pxz[2]), warp_sum(pxz[3]));
            pair9_from4(xz, v, mx, mz);
            v = make_uint4(warp_sum(pyz[0]), warp_sum(pyz[1]), warp_sum(pyz[2]), warp_sum(pyz[3]));
            pair9_from4(yz, v, my, mz);
            derive27(tt, xy, xz, yz);
        }
    }
    if (lane == 0) {
        double s = order == 2 ? score64<9>(T, tab[0], tab[1]) : score64<27>(T, tab[0], tab[1]);
        fp64_out[warp] = s;
        if (cells_out) {
            int nc = order == 2 ? 9 : 27;
            for (int c = 0; c < 2; ++c)
                for (int e = 0; e < nc; ++e) cells_out[((size_t)warp * 2 + c) * 27 + e] = tab[c][e];
        }
    }
}

}  // namespace episdet
