// peak.cu -- live FP64 / FP32 FMA throughput of the current GPU.
//
// The evaluator's hot loop is bound by the FP64 (plain) or FP32+FP64 (mixed)
// pipes, not by HBM or tensor cores, so its roofline denominator is the FMA
// rate this kernel measures: independent FMA chains per thread, enough warps
// to fill every SM, timed with CUDA events.
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/agb.h"

template <typename T, int CHAINS>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b)
{
    T v[CHAINS];
    #pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = (T)(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int c = 0; c < CHAINS; ++c) v[c] = fma(v[c], a, b);
    }
    T s = 0;
    #pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += v[c];
    if (s == (T)12345.678) out[0] = s;   // keeps the chains alive, never true in practice
}

template <typename T>
static int measure(double* tflops, void* stream)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = (cudaStream_t)stream;
    T* out = nullptr;
    if (cudaMallocAsync((void**)&out, sizeof(T), st) != cudaSuccess) return AGB_ERR_DEVICE;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    constexpr int CH = 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chains<T, CH><<<blocks, threads, 0, st>>>(out, iters, (T)0.999999, (T)1e-7);   // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < 5; ++r)
        fma_chains<T, CH><<<blocks, threads, 0, st>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    cudaStreamSynchronize(st);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return AGB_ERR_DEVICE;
    const double flops = 5.0 * 2.0 * (double)blocks * threads * iters * CH;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return AGB_OK;
}

extern "C" int agb_measure_fma_peak(int precision, double* tflops, void* stream)
{
    if (!tflops) return AGB_ERR_ARG;
    return precision == AGB_PREC_MIXED ? measure<float>(tflops, stream)
                                       : measure<double>(tflops, stream);
}
