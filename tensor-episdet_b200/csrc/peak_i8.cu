// peak_i8.cu -- microbenchmark of tcgen05.mma.cta_group::1.kind::i8 on B200.
//
//   episdet-peak-i8 [iters]
//
// One CTA per SM issues back-to-back M=128 x N x K=32 unsigned 8-bit MMAs on
// operand tiles resident in shared memory, for N = 128 and 256, and reports
// the dense 8-bit MAC rate of the whole GPU.  A second pass adds a TMA stream
// that writes 32 KB of fresh operand tiles into other shared memory per four
// N=128 MMAs -- the shared-memory write traffic the counting engine's
// producer adds -- to show what a streaming kernel of this shape can reach.
// These are the instruction peaks the engine's roofline is quoted against.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "tc_ptx.cuh"

using namespace episdet;

namespace {

constexpr int kThreads = 128;
constexpr uint64_t kLimitNs = 2000000000ull;

__device__ int g_err;

// mode 0: MMA only, accumulators alternating every 4 MMAs; mode 1: mode 0 plus a
// concurrent TMA stream into a separate buffer; mode 2: every MMA into one
// accumulator; mode 3: accumulators rotating every MMA over 512 / N regions;
// mode 4: as mode 0 but a commit after every 4 MMAs (the engine's stage size).
template <int N>
__global__ void __launch_bounds__(kThreads, 1)
    peak_kernel(const __grid_constant__ CUtensorMap map, int iters, int mode, unsigned long long* cycles) {
    extern __shared__ uint8_t raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    uint8_t* a = sm;                      // 128 x 128 bytes
    uint8_t* b = sm + 16384;              // N x 128 bytes
    uint8_t* stream = b + N * 128;        // 2 x 32 KB landing zone of the TMA stream
    // [0..15] commit ring, [16..17] TMA stream, [18] drain
    uint64_t* bars = reinterpret_cast<uint64_t*>(stream + 65536);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 20);
    int* s_abort = reinterpret_cast<int*>(s_tmem + 1);
    int* s_never = s_abort + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < (16384 + N * 128) / 4; i += kThreads)
        reinterpret_cast<uint32_t*>(sm)[i] = (i * 2654435761u) & 0x01010101u;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 19; ++i) ptx::mbar_init(&bars[i], 1);
        *s_abort = 0;
        *s_never = 0;
        ptx::fence_barrier_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 1) {
        ptx::tmem_alloc(s_tmem, 512);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = *s_tmem;
    volatile int* abort = s_abort;
    if (warp == 0 && lane == 0) {
        const uint32_t idesc = ptx::idesc_u8(N);
        const uint64_t ad = ptx::smem_desc_sw128(ptx::smem_u32(a)), bd = ptx::smem_desc_sw128(ptx::smem_u32(b));
        long long t0 = clock64();
        // Groups of G MMAs, one commit each; at most 64 MMAs in flight.
        const int G = mode == 4 ? 4 : 16, ring = 64 / G, groups = iters * (16 / G);
        uint32_t ph = 0;  // parity bits of the ring's barriers
        for (int it = 0; it < groups; ++it) {
            const int slot = it % ring;
            if (it >= ring) {
                if (!ptx::mbar_wait(&bars[slot], (ph >> slot) & 1u, abort, kLimitNs)) {
                    atomicExch(&g_err, 1);
                    *s_abort = 1;
                    break;
                }
                ph ^= 1u << slot;
            }
            for (int m0 = 0; m0 < G; ++m0) {
                const int m = (it * G + m0) & 15;
                const int kk = m & 3;
                const uint32_t acc = mode == 2 ? 0u : (mode == 3 ? (uint32_t)(m % (512 / N)) : (uint32_t)((m >> 2) & 1));
                ptx::mma_u8(tmem + acc * N, ad + 2 * kk, bd + 2 * kk, idesc, 1u);
            }
            ptx::mma_commit(&bars[slot]);
        }
        ptx::mma_commit(&bars[18]);
        if (!ptx::mbar_wait(&bars[18], 0, s_never, kLimitNs)) atomicExch(&g_err, 2);
        cycles[blockIdx.x] = (unsigned long long)(clock64() - t0);
        *s_abort = 1;  // stops the TMA stream
    } else if (warp == 2 && lane == 0 && mode == 1) {
        uint32_t ph[2] = {0, 0};
        bool issued[2] = {false, false};
        for (int it = 0; !*abort; ++it) {
            const int s = it & 1;
            if (issued[s]) {
                if (!ptx::mbar_wait(&bars[16 + s], ph[s], s_never, kLimitNs)) {
                    atomicExch(&g_err, 3);
                    break;
                }
                ph[s] ^= 1;
            }
            ptx::mbar_arrive_expect_tx(&bars[16 + s], 32768);
            const int row = ((blockIdx.x * 7 + it) % 64) * 128;
            ptx::tma_load_2d(stream + s * 32768, &map, 0, row, &bars[16 + s]);
            ptx::tma_load_2d(stream + s * 32768 + 16384, &map, 128, row, &bars[16 + s]);
            issued[s] = true;
        }
        for (int s = 0; s < 2; ++s)
            if (issued[s] && !ptx::mbar_wait(&bars[16 + s], ph[s], s_never, kLimitNs)) atomicExch(&g_err, 4);
    }
    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
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
static int run(const CUtensorMap& map, int sms, int iters, int mode, unsigned long long* d_cyc, double clock_ghz) {
    const size_t smem = 1024 + 16384 + N * 128 + 65536 + 256;
    CK(cudaFuncSetAttribute(peak_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    peak_kernel<N><<<sms, kThreads, smem>>>(map, 64, mode, d_cyc);  // warm-up
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    peak_kernel<N><<<sms, kThreads, smem>>>(map, iters, mode, d_cyc);
    CK(cudaGetLastError());
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    int err = 0;
    CK(cudaMemcpyFromSymbol(&err, g_err, sizeof(int)));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    const double macs = (double)sms * iters * 16.0 * 128.0 * N * 32.0;
    unsigned long long cyc = 0;
    CK(cudaMemcpy(&cyc, d_cyc, sizeof(cyc), cudaMemcpyDeviceToHost));
    printf("{\"n\": %d, \"mode\": \"%s\", \"ms\": %.3f, \"tmacs_per_s\": %.1f, \"tops\": %.1f, "
           "\"mac_per_clk_per_sm\": %.0f, \"err\": %d}\n",
           N, mode == 1 ? "mma+tma_stream" : (mode == 2 ? "one_accumulator" : (mode == 3 ? "rotating_accumulators" : (mode == 4 ? "commit_every_4" : "mma_only"))), ms, macs / (ms * 1e-3) / 1e12, 2 * macs / (ms * 1e-3) / 1e12,
           (double)iters * 16.0 * 128.0 * N * 32.0 / (double)cyc, err);
    (void)clock_ghz;
    return err;
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
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    auto encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    const uint64_t rows = 8192, pitch = 256;
    void* buf = nullptr;
    CK(cudaMalloc(&buf, rows * pitch));
    CK(cudaMemset(buf, 1, rows * pitch));
    CUtensorMap map;
    cuuint64_t dims[2] = {pitch, rows};
    cuuint64_t strides[1] = {pitch};
    cuuint32_t box[2] = {128, 128};
    cuuint32_t es[2] = {1, 1};
    if (!encode || encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, buf, dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        fprintf(stderr, "tensor map encode failed\n");
        return 1;
    }
    unsigned long long* d_cyc = nullptr;
    CK(cudaMalloc(&d_cyc, sizeof(unsigned long long) * p.multiProcessorCount));
    printf("{\"gpu\": \"%s\", \"sms\": %d}\n", p.name, p.multiProcessorCount);
    int rc = 0;
    rc |= run<128>(map, p.multiProcessorCount, iters, 0, d_cyc, 0);
    rc |= run<256>(map, p.multiProcessorCount, iters, 0, d_cyc, 0);
    rc |= run<128>(map, p.multiProcessorCount, iters, 1, d_cyc, 0);
    rc |= run<256>(map, p.multiProcessorCount, iters, 1, d_cyc, 0);
    rc |= run<64>(map, p.multiProcessorCount, iters, 0, d_cyc, 0);
    rc |= run<64>(map, p.multiProcessorCount, iters, 4, d_cyc, 0);
    for (int mode = 2; mode <= 4; ++mode) {
        rc |= run<128>(map, p.multiProcessorCount, iters, mode, d_cyc, 0);
        rc |= run<256>(map, p.multiProcessorCount, iters, mode, d_cyc, 0);
    }
    return rc;
}
