// dr_peaks.cu -- throughput ceilings of the units the engine's kernels are bound by.
//
// The pod's measured peaks cover the HBM copy bandwidth and a dense bf16 GEMM, neither
// of which binds this engine: the sieve is bound by shared-memory atomics and integer
// issue, the S1/S2 sums by integer issue, FP64 quotient estimates and L2 gathers.
// dr_measure_peaks() times small synthetic kernels of each kind on the device so that
// bench.py can state those kernels' rates against measured ceilings.
#include "../../include/dr_engine.h"
#include "dr_kernels.cuh"

#include <cstdio>

namespace drb {
namespace {

constexpr int kPeakBlock = 1024;
constexpr int kSmemWords = 8192;  // 32 KB of shared words per CTA (2 CTAs per SM)

// 32-bit shared-memory atomicAdd.  pattern 0: lane l of warp w adds to words
// l + 32*(8w + j), j < 8, so the 32 lanes of an instruction hit 32 distinct banks
// (the unit's ceiling).  pattern 1: the sieve's marking pattern, lane l at byte
// j + l*m (m odd, one per warp) advanced by 32*m bytes per step, which leaves the
// bank conflicts that odd strides give.
__global__ void __launch_bounds__(kPeakBlock) peak_atomic_kernel(uint32_t* out, int iters, int pattern) {
    __shared__ uint32_t s[kSmemWords];
    for (int i = threadIdx.x; i < kSmemWords; i += blockDim.x) s[i] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (pattern == 0) {
        uint32_t* p = s + lane + 256u * (warp & 31u);
        for (int k = 0; k < iters; k += 8) {
#pragma unroll
            for (int j = 0; j < 8; ++j) atomicAdd(p + 32 * j, 1u << (8 * (j & 3)));
        }
    } else {
        const uint32_t m = 13u + 2u * warp;
        uint32_t b = lane * m;
        for (int k = 0; k < iters; ++k) {
            atomicAdd(&s[(b >> 2) & (kSmemWords - 1)], 1u << (8 * (b & 3u)));
            b += 32u * m;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < kSmemWords; i += 97) acc += s[i];
        out[blockIdx.x] = acc;
    }
}

// 32-bit integer multiply-add, 8 independent chains per thread.  Each step is
// a <- a*a + c: unlike an affine step, two of these do not compose into one
// multiply-add, so the compiler cannot fold unrolled iterations together.
__global__ void __launch_bounds__(kPeakBlock) peak_imad_kernel(uint32_t* out, int iters) {
    uint32_t a[8];
    const uint32_t c = 0x7F4A7C15u + 2u * blockIdx.x;
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = threadIdx.x + 977u * j + blockIdx.x;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = a[j] * a[j] + c;
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc ^= a[j];
    if (acc == 0x12345678u) out[blockIdx.x] = acc;  // keeps the chains live
}

// FP64 fused multiply-add, 8 independent chains per thread
__global__ void __launch_bounds__(kPeakBlock) peak_dfma_kernel(double* out, int iters) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = 1.0 + 1e-3 * (threadIdx.x + j);
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = __fma_rn(a[j], 0.9999999, 1e-7);
    }
    double acc = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc += a[j];
    if (acc == 12345.0) out[blockIdx.x] = acc;
}

}  // namespace
}  // namespace drb

using namespace drb;

extern "C" int dr_measure_peaks(int device, dr_peaks* out) {
    if (!out) return record_error(DR_ERR_ARG, "dr_measure_peaks: out is NULL");
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return record_error(DR_ERR_CUDA, "dr_measure_peaks: bad device");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int grid = 2 * sms;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    void* buf = nullptr;
    int rc = DR_OK;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaMalloc(&buf, (size_t)grid * sizeof(double)) != cudaSuccess) {
        rc = record_error(DR_ERR_CUDA, "dr_measure_peaks: set-up failed");
    }
    // best of three timed launches after one untimed launch; ops per second
    auto rate = [&](auto launch, double ops) -> double {
        launch();
        float best = 0.0f;
        for (int r = 0; r < 3; ++r) {
            cudaEventRecord(e0, st);
            launch();
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (best == 0.0f || ms < best) best = ms;
        }
        return best > 0.0f ? ops / (best * 1e-3) : 0.0;
    };
    if (rc == DR_OK) {
        const double threads = (double)grid * kPeakBlock;
        const int ia = 16384, ii = 16384, id = 4096;
        out->smem_atomic_per_s = rate([&] { peak_atomic_kernel<<<grid, kPeakBlock, 0, st>>>((uint32_t*)buf, ia, 0); },
                                      threads * ia);
        out->smem_atomic_stride_per_s =
            rate([&] { peak_atomic_kernel<<<grid, kPeakBlock, 0, st>>>((uint32_t*)buf, ia, 1); }, threads * ia);
        out->imad_per_s = rate([&] { peak_imad_kernel<<<grid, kPeakBlock, 0, st>>>((uint32_t*)buf, ii); },
                               threads * ii * 8);
        out->dfma_per_s = rate([&] { peak_dfma_kernel<<<grid, kPeakBlock, 0, st>>>((double*)buf, id); },
                               threads * id * 8);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            char msg[160];
            snprintf(msg, sizeof(msg), "dr_measure_peaks: %s", cudaGetErrorString(e));
            rc = record_error(DR_ERR_CUDA, msg);
        }
    }
    if (buf) cudaFree(buf);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}
