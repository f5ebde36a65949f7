// tests/csrc/pipe_rates.cu -- TEST HELPER, NOT PRODUCT CODE.
//
// Throughput of the instructions the stage kernels' costs are made of, in thread operations per
// SM clock, for tests/test_gpu_pipe_rates.py (which compiles this file with nvcc into a temporary
// shared library).  Each kernel runs 8 independent dependency chains per thread over a grid of
// 4 CTAs of 512 threads per SM, so throughput, not latency, is measured.
#include <cuda_runtime.h>

namespace {
constexpr int kChains = 8;

template <int OP>
__global__ void rate_kernel(double* out, int iters, double b, double c) {
    double d[kChains];
    float f[kChains];
    for (int i = 0; i < kChains; i++) {
        d[i] = threadIdx.x * 1e-3 + i;
        f[i] = (float)d[i];
    }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < kChains; i++) {
            if (OP == 0) d[i] = fma(d[i], b, c);                             // FP64 fused multiply-add
            if (OP == 1) d[i] = (double)(float)d[i] * b;                      // FP64 -> FP32 -> FP64 + multiply
            if (OP == 2) f[i] = fmaf(f[i], 1.0001f, 0.5f);                    // FP32 fused multiply-add
            if (OP == 3) {                                                    // FP64 reciprocal seed + add
                double y;
                asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d[i]));
                d[i] = y + c;
            }
            if (OP == 4) d[i] = fmin(fmax(d[i], b), c) + c;                   // library fmin / fmax of doubles
        }
    }
    double s = 0.0;
    for (int i = 0; i < kChains; i++) s += d[i] + (double)f[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int OP>
float time_op(double* out, int blocks, int threads, int iters) {
    cudaEvent_t a, e;
    cudaEventCreate(&a);
    cudaEventCreate(&e);
    rate_kernel<OP><<<blocks, threads>>>(out, iters / 8, 1.0000001, 1e-9);   // warm-up
    cudaEventRecord(a);
    rate_kernel<OP><<<blocks, threads>>>(out, iters, 1.0000001, 1e-9);
    cudaEventRecord(e);
    cudaEventSynchronize(e);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, e);
    cudaEventDestroy(a);
    cudaEventDestroy(e);
    return ms;
}
}  // namespace

// rates[k]: chain iterations per SM clock (thread operations of the op per clock) of op k =
// 0 DFMA, 1 (F2F pair + DMUL), 2 FFMA, 3 (MUFU rcp64 + DADD), 4 (fmin + fmax + DADD), at the SM
// clock the device reports.  Returns a cudaError_t.
extern "C" int pipe_rates(double* rates) {
    int dev = 0, sms = 0, khz = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
    const int blocks = sms * 4, threads = 512, iters = 2048;
    double* out = nullptr;
    cudaError_t err = cudaMalloc(&out, sizeof(double) * blocks * threads);
    if (err != cudaSuccess) return (int)err;
    const float ms[5] = {time_op<0>(out, blocks, threads, iters), time_op<1>(out, blocks, threads, iters),
                         time_op<2>(out, blocks, threads, iters), time_op<3>(out, blocks, threads, iters),
                         time_op<4>(out, blocks, threads, iters)};
    const double ops = (double)blocks * threads * iters * kChains;
    for (int k = 0; k < 5; k++) rates[k] = ops / (ms[k] * 1e-3 * khz * 1e3) / sms;
    err = cudaDeviceSynchronize();
    cudaFree(out);
    return (int)err;
}
