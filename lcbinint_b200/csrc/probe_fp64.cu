// FP64 throughput probe: the denominator of the FP64 roofline reported by the
// bench.  Each thread runs independent FMA chains long enough to saturate the
// FP64 pipes; the result is written out so the work cannot be elided.
#include "../../include/lcbinint_b200.h"
#include "lcbi_context.h"

namespace lcbi {

__global__ void __launch_bounds__(256) fp64_fma_kernel(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

} // namespace lcbi

extern "C" int lcbi_gpu_measure_fp64_peak(lcbi_gpu_context* c, double* tflops)
{
    lcbi::Context* ctx = reinterpret_cast<lcbi::Context*>(c);
    if (!ctx || !tflops) return LCBI_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    const int blocks = ctx->sm_count * 8, threads = 256, iters = 4096;
    if (!ctx->ensure(ctx->work[7], (size_t)blocks * threads * sizeof(double))) return LCBI_GPU_ERROR;
    double* out = static_cast<double*>(ctx->work[7].ptr);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        lcbi::fp64_fma_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ctx->check("fp64 probe", cudaGetLastError())) return LCBI_GPU_ERROR;
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return LCBI_OK;
}
