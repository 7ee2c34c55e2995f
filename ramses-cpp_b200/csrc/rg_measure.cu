// rg_measure.cu -- the FP64 peak the face kernel's compute roofline is
// reported against (no reference counterpart; measurement only).
//
// The face kernel is bound by FP64 arithmetic, not by HBM: its roofline in
// FLOP/s needs the device's own FP64 throughput, which no driver-side peak
// file carries.  This kernel keeps every FP64 pipe busy with independent
// fused multiply-add chains (8 per thread, 2 FLOPs each) on the whole GPU and
// is timed with CUDA events on the context's stream.
#include "rg_internal.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_dfma_peak(double seed, double* sink) {
    double a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = seed + 1e-3 * (threadIdx.x + i);
    const double b = 0.999999, c = 1e-7;
#pragma unroll 4
    for (int it = 0; it < kIters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], b, c);
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i];
    if (s == 12345.678) sink[blockIdx.x] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" int rg_measure_fp64_peak(rg_ctx* c, double* tflops) {
    using namespace rg;
    if (!c || !tflops) return RG_ERR_ARG;
    if (c->broken) return set_error(c, RG_ERR_CUDA, c->err);
    cudaSetDevice(c->device);
    const int blocks = c->sm_count * 8, threads = 256;
    double* sink = nullptr;
    if (int rc = check_cuda(c, dev_alloc(c, &sink, sizeof(double) * blocks), "fp64 probe sink")) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; ++w) k_dfma_peak<<<blocks, threads, 0, c->stream>>>(1.0, sink);
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0, c->stream);
        k_dfma_peak<<<blocks, threads, 0, c->stream>>>(1.0 + r, sink);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dev_free(c, sink);
    if (int rc = check_cuda(c, cudaGetLastError(), "fp64 probe")) return rc;
    const double flops = 2.0 * kChains * (double)kIters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "fp64 probe");
}
