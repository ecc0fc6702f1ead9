// microbench.cu -- peak rates that bound the pair/triplet kernels, measured
// on the device the library runs on (the roofline denominators):
//   PCF_MB_FP32_FMA      FP32 FMA throughput, TFLOP/s (2 flops per FMA)
//   PCF_MB_SMEM_ATOMIC   conflict-free shared-memory u32 atomicAdd, Gop/s
//   PCF_MB_SMEM_ATOMIC_F64 / _U64 / _F32   the same for f64 / u64 / f32 adds
//                        (the weighted histograms' accumulator types)
// Each runs ~10-50 ms, timed with CUDA events on the context stream.
#include "pcf_internal.cuh"
#include "../../include/pcf_bench.h"

namespace {

__global__ void __launch_bounds__(256) k_fma(float *out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[0] = s;  // keeps the chains live
}

template <typename T>
__global__ void __launch_bounds__(256) k_smem_atomic(unsigned *out, int iters) {
    __shared__ T h[256 * 4];
    for (int k = threadIdx.x; k < 256 * 4; k += 256) h[k] = T(0);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T *mine = h + warp * 32 + lane;  // distinct address per lane, no conflicts between lanes
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) atomicAdd(mine + ((k & 3) << 8), T(1));
    }
    __syncthreads();
    if (h[threadIdx.x] == T(123456789)) out[0] = 1;
}

}  // namespace

extern "C" pcf_status pcf_microbench(pcf_ctx *ctx, int which, double *result) {
    if (!ctx || !result) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    PCF_CU(ctx, ctx->d_flag.ensure(64));
    const int blocks = ctx->sm_count * 8, threads = 256;
    float ms = 0.f;
    double ops = 0;
    for (int rep = 0; rep < 2; ++rep) {  // first run warms clocks
        PCF_CU(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        if (which == PCF_MB_FP32_FMA) {
            const int iters = 2048;
            k_fma<<<blocks, threads, 0, ctx->stream>>>(ctx->d_flag.as<float>(), iters, 0.999f, 0.001f);
            ops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        } else if (which >= PCF_MB_SMEM_ATOMIC && which <= PCF_MB_SMEM_ATOMIC_F32) {
            const int iters = 512;
            unsigned *o = ctx->d_flag.as<unsigned>();
            if (which == PCF_MB_SMEM_ATOMIC) k_smem_atomic<unsigned><<<blocks, threads, 0, ctx->stream>>>(o, iters);
            else if (which == PCF_MB_SMEM_ATOMIC_F64) k_smem_atomic<double><<<blocks, threads, 0, ctx->stream>>>(o, iters);
            else if (which == PCF_MB_SMEM_ATOMIC_U64)
                k_smem_atomic<unsigned long long><<<blocks, threads, 0, ctx->stream>>>(o, iters);
            else k_smem_atomic<float><<<blocks, threads, 0, ctx->stream>>>(o, iters);
            ops = 16.0 * (double)iters * blocks * threads;
        } else {
            return PCF_ERR_INVALID_ARG;
        }
        PCF_CU(ctx, cudaGetLastError());
        PCF_CU(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
        PCF_CU(ctx, cudaEventSynchronize(ctx->ev1));
        PCF_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    }
    *result = ops / (ms * 1e-3) / (which == PCF_MB_FP32_FMA ? 1e12 : 1e9);
    return PCF_OK;
}
