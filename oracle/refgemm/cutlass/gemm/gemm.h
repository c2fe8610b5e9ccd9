// Test infrastructure (oracle side): the 1-bit GEMM that CUTLASS 1.3 runs
// for Cutlass_U1_WmmagemmTN (src/helper.cu:714-750 of hiperbio/tensor-episdet),
// restated as a plain CUDA kernel.
//
// Contract, as the reference's call sites use it (src/search-pairs.cu:150-180,
// src/search-triplets.cu:205-235, read by src/helper.cu:468-474 and :632-636):
//   * A is M x K, row-major; B is K x N, column-major; both hold 1-bit
//     elements packed 32 to a word (Vector<bin1_t, 32>);
//   * K counts 1-bit elements (a multiple of 32 here: the classes are padded
//     to 1024 samples); lda and ldb are leading dimensions in 32-bit words;
//   * the binary "multiply-accumulate" of the WMMA b1 operation is XOR then
//     population count, so the product is D[m][n] = sum over k of
//     popc(A[m][k] XOR B[k][n]);
//   * C and D are column-major int matrices (element (m, n) at m + n * ld);
//     D = alpha * product + beta * C (LinearScaling), C not read when beta = 0.
// The kernel stages 32-word slices of 16 A rows and 16 B columns in shared
// memory; every load is bounds-checked, so M and N need not be tile multiples.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../wmma_matrix.h"
#include "wmma_gemm_traits.h"

namespace cutlass {
namespace gemm {

namespace detail {

constexpr int kTile = 16;   // output tile: kTile x kTile, one thread each
constexpr int kSlice = 32;  // words of K per shared-memory slice

// A template so that every translation unit including this header may hold it.
template <int kT>
__global__ void __launch_bounds__(kT* kT)
    xor_popc_gemm_tn(int M, int N, int words, int alpha, const uint32_t* A, long lda, const uint32_t* B, long ldb,
                     int beta, const int* C, long ldc, int* D, long ldd) {
    __shared__ uint32_t sa[kT][kSlice + 1];
    __shared__ uint32_t sb[kT][kSlice + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
    const int tid = ty * kT + tx;
    int acc = 0;
    for (int k0 = 0; k0 < words; k0 += kSlice) {
        for (int e = tid; e < kT * kSlice; e += kT * kT) {
            const int r = e / kSlice, c = e % kSlice, k = k0 + c;
            const int m = m0 + r, n = n0 + r;
            sa[r][c] = (m < M && k < words) ? A[(long)m * lda + k] : 0u;
            sb[r][c] = (n < N && k < words) ? B[(long)n * ldb + k] : 0u;
        }
        __syncthreads();
#pragma unroll 8
        for (int c = 0; c < kSlice; ++c) acc += __popc(sa[ty][c] ^ sb[tx][c]);
        __syncthreads();
    }
    const int m = m0 + ty, n = n0 + tx;
    if (m < M && n < N) {
        int v = alpha * acc;
        if (beta != 0) v += beta * C[(long)m + (long)n * ldc];
        D[(long)m + (long)n * ldd] = v;
    }
}

}  // namespace detail

template <typename Traits_>
struct Gemm {
    typedef Traits_ Traits;
    typedef typename Traits::ScalarA ScalarA;
    typedef typename Traits::ScalarB ScalarB;
    typedef typename Traits::ScalarC ScalarC;
    typedef typename Traits::ScalarD ScalarD;
    typedef typename Traits::Epilogue::Scalar Scalar;
    static_assert(Traits::kLayoutA == MatrixLayout::kRowMajor && Traits::kLayoutB == MatrixLayout::kColumnMajor,
                  "only the TN form that the reference instantiates is restated");
    static_assert(sizeof(ScalarA) == 4 && sizeof(ScalarB) == 4, "operands are 32-bit words of 1-bit elements");

    struct Params {
        int m = 0, n = 0, k = 0;
        Scalar alpha = 0, beta = 0;
        const ScalarA* a = nullptr;
        const ScalarB* b = nullptr;
        const ScalarC* c = nullptr;
        ScalarD* d = nullptr;
        int lda = 0, ldb = 0, ldc = 0, ldd = 0;

        // Returns non-zero for arguments the contract above does not cover.
        int initialize(int m_, int n_, int k_, Scalar alpha_, const ScalarA* a_, int lda_, const ScalarB* b_, int ldb_,
                       Scalar beta_, const ScalarC* c_, int ldc_, ScalarD* d_, int ldd_) {
            if (m_ < 0 || n_ < 0 || k_ < 0 || k_ % 32 != 0) return 1;
            if (lda_ < k_ / 32 || ldb_ < k_ / 32 || ldc_ < m_ || ldd_ < m_) return 1;
            m = m_, n = n_, k = k_, alpha = alpha_, beta = beta_;
            a = a_, b = b_, c = c_, d = d_;
            lda = lda_, ldb = ldb_, ldc = ldc_, ldd = ldd_;
            return 0;
        }
    };

    static void launch(const Params& p, cudaStream_t stream = 0) {
        if (p.m == 0 || p.n == 0) return;
        dim3 block(detail::kTile, detail::kTile);
        dim3 grid((p.n + detail::kTile - 1) / detail::kTile, (p.m + detail::kTile - 1) / detail::kTile);
        detail::xor_popc_gemm_tn<detail::kTile><<<grid, block, 0, stream>>>(
            p.m, p.n, p.k / 32, (int)p.alpha, reinterpret_cast<const uint32_t*>(p.a), p.lda,
            reinterpret_cast<const uint32_t*>(p.b), p.ldb, (int)p.beta, reinterpret_cast<const int*>(p.c), p.ldc,
            reinterpret_cast<int*>(p.d), p.ldd);
    }
};

}  // namespace gemm
}  // namespace cutlass
