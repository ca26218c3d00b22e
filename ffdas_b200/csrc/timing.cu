// timing.cu -- kernel timing hooks and the FP32 FMA peak probe.
//
// ffdas_set_kernel_timing / ffdas_get_last_kernel_time let a benchmark time the
// main delay-and-sum kernel of a call with CUDA events on the launching stream
// (the ingest pass is excluded).  ffdas_measure_fp32_peak runs kernels of
// independent FFMA chains and of packed FFMA2 chains sized to fill every SM
// and returns the faster achieved FP32 throughput; it is the denominator of
// the FP32 roofline.
#include <cuda_runtime.h>

#include "core.h"

namespace {

// 8 independent FMA chains per thread, kIters rounds of 8 FMAs each.
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fma_peak_kernel(float *sink, float seed) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.999999f, c = 1e-7f;
#pragma unroll 16
    for (int i = 0; i < kIters; i++) {
        a0 = __fmaf_rn(a0, m, c); a1 = __fmaf_rn(a1, m, c); a2 = __fmaf_rn(a2, m, c); a3 = __fmaf_rn(a3, m, c);
        a4 = __fmaf_rn(a4, m, c); a5 = __fmaf_rn(a5, m, c); a6 = __fmaf_rn(a6, m, c); a7 = __fmaf_rn(a7, m, c);
    }
    float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 12345.678f) sink[blockIdx.x] = s;  // keeps the chains live
}

// The same with packed f32x2 FMAs (FFMA2): 8 independent pair chains per
// thread.  Blackwell issues one packed instruction for two FMAs; whether the
// FP32 pipe also runs them at twice the scalar rate is what this measures.
__global__ void __launch_bounds__(256) fma2_peak_kernel(float *sink, float seed) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = make_float2(seed + threadIdx.x + 2 * k, seed + threadIdx.x + 2 * k + 1);
    const float2 m = make_float2(0.999999f, 0.999999f), c = make_float2(1e-7f, 1e-7f);
#pragma unroll 16
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k].x + a[k].y;
    if (s == 12345.678f) sink[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" {

ffdas_error_t ffdas_set_kernel_timing(ffdas_handle_t h, int enable) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(h->check_device());
    if (enable && !h->ev_start) {
        FFDAS_CUDA(cudaEventCreate(&h->ev_start));
        FFDAS_CUDA(cudaEventCreate(&h->ev_stop));
    }
    h->timing = enable != 0;
    h->timing_recorded = false;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_get_last_kernel_time(ffdas_handle_t h, float *ms) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!ms) return FFDAS_ERROR_NULL_POINTER;
    if (!h->timing || !h->timing_recorded) return FFDAS_ERROR_INVALID_STATE;
    FFDAS_CUDA(cudaEventSynchronize(h->ev_stop));
    FFDAS_CUDA(cudaEventElapsedTime(ms, h->ev_start, h->ev_stop));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_get_last_kernel_units(ffdas_handle_t h, long long *units) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!units) return FFDAS_ERROR_NULL_POINTER;
    if (!h->timing || !h->timing_recorded || !h->units_recorded) return FFDAS_ERROR_INVALID_STATE;
    FFDAS_TRY(h->check_device());
    unsigned long long v = 0ull;
    FFDAS_CUDA(cudaStreamSynchronize(h->stream));
    FFDAS_CUDA(cudaMemcpy(&v, h->unit_count, sizeof(v), cudaMemcpyDeviceToHost));
    *units = (long long)v;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_measure_fp32_peak(ffdas_handle_t h, double *tflops) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!tflops) return FFDAS_ERROR_NULL_POINTER;
    FFDAS_TRY(h->check_device());
    const int blocks = h->sm_count * 8;   // 8 x 256 threads = 64 warps per SM
    float *sink = nullptr;
    FFDAS_TRY(h->alloc((size_t)blocks * sizeof(float), reinterpret_cast<void **>(&sink)));
    cudaEvent_t a, b;
    FFDAS_CUDA(cudaEventCreate(&a));
    FFDAS_CUDA(cudaEventCreate(&b));
    // scalar FFMA chains (8 FMAs per round) and packed FFMA2 chains (16 FMAs
    // per round): the peak is the faster of the two in FMAs per second
    double best_rate = 0.0;
    for (int packed = 0; packed < 2; packed++) {
        float best = 1e30f;
        for (int rep = 0; rep < 6; rep++) {
            cudaEventRecord(a, h->stream);
            if (packed) fma2_peak_kernel<<<blocks, 256, 0, h->stream>>>(sink, 1.0f + rep);
            else fma_peak_kernel<<<blocks, 256, 0, h->stream>>>(sink, 1.0f + rep);
            cudaEventRecord(b, h->stream);
            if (cudaEventSynchronize(b) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0 && ms < best) best = ms;  // first launch is warm-up
        }
        const double flops = 2.0 * (packed ? 16.0 : 8.0) * kIters * 256.0 * blocks;
        best_rate = fmax(best_rate, flops / (best * 1e-3));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->free(sink);
    FFDAS_TRY(ffdas_launch_check(h->stream));
    *tflops = best_rate / 1e12;
    return FFDAS_SUCCESS;
}

}  // extern "C"
