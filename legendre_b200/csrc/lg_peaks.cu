// Compute-side roofline denominators, measured on the device: how many FP64
// FMAs, FP32 FMAs, 32-bit integer multiply-adds and plain 32-bit ALU
// operations (xor, add) the GPU retires per second when every warp slot is
// busy with independent chains of them.  The Model C step kernels are bound
// by instruction issue and the FP64 pipe rather than by HBM, so the bench
// reports their rates against these numbers beside the HBM fraction.
//
// Each thread runs kChains independent chains kUnroll deep per iteration
// (enough independent work to cover the pipes' latencies at full occupancy);
// a never-true store keeps the chains live.  The grid is the device's SM
// count times 8 CTAs of 256 threads (2048 threads per SM).  Times are CUDA
// events on the context's stream, best of three.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "lg_state_view.h"

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;

__global__ void __launch_bounds__(256) peak_dfma_kernel(double* sink, double a, double b, int iters) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3 + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == -1.25) sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) peak_ffma_kernel(float* sink, float a, float b, int iters) {
    float x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == -1.25f) sink[blockIdx.x] = s;
}

// 32-bit integer multiply-add chains (the building block of 64-bit
// multiplies such as SplitMix64's)
__global__ void __launch_bounds__(256) peak_imad_kernel(uint32_t* sink, uint32_t a, uint32_t b, int iters) {
    uint32_t x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x + 977u * k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int k = 0; k < kChains; ++k) x[k] = x[k] * a + b;
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s ^= x[k];
    if (s == 0x9e3779b9u && a == b) sink[blockIdx.x] = s;
}

// plain ALU chains: an xor and an add per element, two operations
__global__ void __launch_bounds__(256) peak_alu_kernel(uint32_t* sink, uint32_t a, uint32_t b, int iters) {
    uint32_t x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x + 977u * k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int k = 0; k < kChains; ++k) x[k] = (x[k] ^ a) + (b + (uint32_t)u);
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s ^= x[k];
    if (s == 0x9e3779b9u && a == b) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" int lg_measure_compute_peaks(lg_ctx* ctx, lg_compute_peaks* out) {
    if (!ctx || !out) return lg::abi_fail(ctx, LG_ERR_INVALID, "bad arguments");
    const int dev = lg::abi_device(ctx);
    cudaStream_t st = lg::abi_stream(ctx);
    cudaError_t e = cudaSetDevice(dev);
    int sms = 0, clock_khz = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, dev);
    if (e != cudaSuccess) return lg::abi_fail(ctx, LG_ERR_CUDA, std::string("device query: ") + cudaGetErrorString(e));
    const int ctas = sms * 8, threads = 256;
    void* sink = nullptr;
    e = cudaMallocAsync(&sink, (size_t)ctas * sizeof(double), st);
    if (e != cudaSuccess) return lg::abi_fail(ctx, LG_ERR_NOMEM, std::string("sink: ") + cudaGetErrorString(e));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // operations per thread per launch: kChains * kUnroll per iteration
    // (two for the ALU kernel's xor and add)
    const double per_iter = (double)kChains * kUnroll;
    const double thread_count = (double)ctas * threads;
    double best[4] = {0.0, 0.0, 0.0, 0.0};
    const int iters[4] = {2048, 4096, 4096, 4096};
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
            cudaEventRecord(e0, st);
            if (k == 0) peak_dfma_kernel<<<ctas, threads, 0, st>>>((double*)sink, 0.9999999, 1e-7, iters[k]);
            if (k == 1) peak_ffma_kernel<<<ctas, threads, 0, st>>>((float*)sink, 0.9999f, 1e-4f, iters[k]);
            if (k == 2) peak_imad_kernel<<<ctas, threads, 0, st>>>((uint32_t*)sink, 0x9e3779b1u, 0x7f4a7c15u, iters[k]);
            if (k == 3) peak_alu_kernel<<<ctas, threads, 0, st>>>((uint32_t*)sink, 0x85ebca6bu, 0xc2b2ae35u, iters[k]);
            lg::abi_count_launch(ctx, 1);
            cudaEventRecord(e1, st);
            e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms > 0.0f) {
                const double ops = thread_count * iters[k] * per_iter * (k == 3 ? 2.0 : 1.0);
                best[k] = std::max(best[k], ops / (ms * 1e-3));
            }
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(sink, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return lg::abi_fail(ctx, LG_ERR_CUDA, std::string("peak kernels: ") + cudaGetErrorString(e));
    out->dfma_per_s = best[0];
    out->ffma_per_s = best[1];
    out->imad_per_s = best[2];
    out->alu_per_s = best[3];
    out->sms = sms;
    out->clock_mhz = clock_khz / 1000.0;
    return LG_OK;
}
