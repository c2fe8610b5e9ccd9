// peak_f4.cu -- exactness check and rate of tcgen05.mma kind::mxf4 on B200.
//
//   episdet-peak-f4 [iters]
//
// The counting engine can hold its 0/1 operand rows as packed e2m1 values
// (0.0 and 1.0, four bits each) instead of unsigned bytes: half the bytes per
// sample and twice the MACs per instruction.  The block scale factors are all
// 1.0 (UE8M0 127), accumulation is FP32, so a count is exact while it stays
// below 2^24.  This program checks that on the device and measures the rate:
//
//  * check: A row i is all 1.0 when i % 3 == 1, B row j all 1.0 when j % 4 != 0
//    (every other value 0), so after `chunks` 128-byte K blocks every D[i][j]
//    must equal 256 * chunks or 0 -- independent of the swizzle and of the
//    nibble order inside a byte, which A and B share;
//  * rate: back-to-back M=128 x N x K=64 MMAs on resident tiles.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "tc_ptx.cuh"

using namespace episdet;

namespace {

constexpr int kThreads = 128;
constexpr uint64_t kLimitNs = 2000000000ull;
constexpr uint32_t kSfCol = 496;  // scale-factor columns 496..511, every byte 127 (1.0)

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


// mode 0: exactness check over `iters` K blocks; mode 1: rate.
template <int N>
__global__ void __launch_bounds__(kThreads, 1) f4_kernel(int iters, int mode, unsigned long long* cycles) {
    extern __shared__ uint8_t raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a = sm;          // 128 rows x 128 bytes
    uint8_t* b = sm + 16384;  // N rows x 128 bytes
    uint64_t* bars = reinterpret_cast<uint64_t*>(b + N * 128);  // [0..3] ring, [4] drain
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 8);
    int* s_abort = reinterpret_cast<int*>(s_tmem + 1);
    int* s_never = s_abort + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Row-constant operands (a byte holds two e2m1 values: 0x22 = two 1.0).
    for (int i = threadIdx.x; i < 128 * 128; i += kThreads) a[i] = ((i >> 7) % 3 == 1) ? 0x22 : 0x00;
    for (int i = threadIdx.x; i < N * 128; i += kThreads) b[i] = ((i >> 7) % 4 != 0) ? 0x22 : 0x00;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 5; ++i) ptx::mbar_init(&bars[i], 1);
        *s_abort = 0;
        *s_never = 0;
        ptx::fence_barrier_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        ptx::tmem_alloc(s_tmem, 512);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    // Scale factors: every byte of columns kSfCol .. kSfCol + 15 is 127 (2^0).
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    ptx::tmem_st8_fill(lane_base + kSfCol, 0x7F7F7F7Fu);
    ptx::tmem_st8_fill(lane_base + kSfCol + 8, 0x7F7F7F7Fu);
    ptx::tmem_wait_st();
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    volatile int* abort = s_abort;
    if (warp == 0 && lane == 0) {
        const uint32_t idesc = ptx::idesc_mxf4(N, 128);
        const uint64_t ad = ptx::smem_desc_sw128(ptx::smem_u32(a)), bd = ptx::smem_desc_sw128(ptx::smem_u32(b));
        const uint32_t sfa = tmem + kSfCol, sfb = tmem + kSfCol + 8;
        long long t0 = clock64();
        uint32_t ph = 0;
        for (int it = 0; it < iters; ++it) {
            const int slot = it & 3;
            if (it >= 4) {  // at most 4 groups of 16 MMAs in flight
                if (!ptx::mbar_wait(&bars[slot], (ph >> slot) & 1u, abort, kLimitNs)) {
                    atomicExch(&g_err, 1);
                    *s_abort = 1;
                    break;
                }
                ph ^= 1u << slot;
            }
            for (int m = 0; m < 16; ++m) {
                const int kk = m & 3;  // 4 MMAs of K = 64 cover one 128-byte block
                // Two accumulator regions below the scale-factor columns (one for N = 256).
                const uint32_t acc = (mode == 0 || N > 224) ? 0u : (uint32_t)((m >> 2) & 1) * N;
                const uint32_t first = (mode == 0 && it == 0 && m == 0) ? 0u : 1u;
                mma_mxf4(tmem + acc, ad + 2 * kk, bd + 2 * kk, idesc, sfa, sfb, first);
            }
            ptx::mma_commit(&bars[slot]);
        }
        ptx::mma_commit(&bars[4]);
        if (!ptx::mbar_wait(&bars[4], 0, s_never, kLimitNs)) atomicExch(&g_err, 2);
        cycles[blockIdx.x] = (unsigned long long)(clock64() - t0);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (mode == 0 && blockIdx.x == 0) {
        // Each iteration adds 4 K blocks of 128 bytes = 4 x 256 values.
        const float want_one = 1024.0f * (float)iters;
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
    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, 512);
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

template <int N>
static int run(int sms, int iters, int mode, unsigned long long* d_cyc) {
    const size_t smem = 1024 + 16384 + N * 128 + 256;
    CK(cudaFuncSetAttribute(f4_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = mode == 0 ? 1 : sms;
    if (mode == 1) {
        f4_kernel<N><<<grid, kThreads, smem>>>(64, mode, d_cyc);  // warm-up
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
    }
    unsigned long long zero = 0;
    CK(cudaMemcpyToSymbol(g_bad, &zero, sizeof(zero)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    f4_kernel<N><<<grid, kThreads, smem>>>(iters, mode, d_cyc);
    CK(cudaGetLastError());
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    int err = 0;
    unsigned long long bad = 0, cyc = 0;
    CK(cudaMemcpyFromSymbol(&err, g_err, sizeof(int)));
    CK(cudaMemcpyFromSymbol(&bad, g_bad, sizeof(bad)));
    CK(cudaMemcpy(&cyc, d_cyc, sizeof(cyc), cudaMemcpyDeviceToHost));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    const double per_cta = (double)iters * 16.0 * 128.0 * N * 64.0;
    if (mode == 0)
        printf("{\"n\": %d, \"mode\": \"check\", \"k_values\": %d, \"bad_cells\": %llu, \"err\": %d}\n", N,
               iters * 1024, bad, err);
    else
        printf("{\"n\": %d, \"mode\": \"rate\", \"ms\": %.3f, \"tmacs_per_s\": %.1f, \"mac_per_clk_per_sm\": %.0f, "
               "\"err\": %d}\n",
               N, ms, per_cta * grid / (ms * 1e-3) / 1e12, per_cta / (double)cyc, err);
    return err || bad ? 1 : 0;
}

int main(int argc, char** argv) {
    int iters = argc > 1 ? atoi(argv[1]) : 20000;
    if (iters < 64 || iters > 10000000) iters = 20000;
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, 0));
    if (p.major != 10) {
        fprintf(stderr, "needs an sm_100 device\n");
        return 1;
    }
    printf("{\"gpu\": \"%s\", \"sms\": %d}\n", p.name, p.multiProcessorCount);
    unsigned long long* d_cyc = nullptr;
    CK(cudaMalloc(&d_cyc, sizeof(unsigned long long) * p.multiProcessorCount));
    int rc = 0;
    // Exactness first (one CTA; 4096 iterations = 4,194,304 values per count).
    rc |= run<128>(p.multiProcessorCount, 4096, 0, d_cyc);
    rc |= run<112>(p.multiProcessorCount, 4096, 0, d_cyc);
    rc |= run<256>(p.multiProcessorCount, 64, 0, d_cyc);
    if (rc) return rc;
    rc |= run<128>(p.multiProcessorCount, iters, 1, d_cyc);
    rc |= run<112>(p.multiProcessorCount, iters, 1, d_cyc);
    rc |= run<256>(p.multiProcessorCount, iters, 1, d_cyc);
    CK(cudaFree(d_cyc));
    return rc;
}
