// tests/csrc/rs_special.cu -- TEST HELPER, NOT PRODUCT CODE.
//
// Evaluates the product's FP64 Newton-refined special functions (rs_rcp, rs_rsqrt, rs_sqrt in
// set_b200/csrc/mhd_core.cuh) on the device for tests/test_gpu_special.py, which compiles this
// file with nvcc into a temporary shared library.
#include <cuda_runtime.h>
#include "mhd_core.cuh"

__global__ void rs_kernel(const double* x, double* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[3 * i + 0] = sb::rs_rcp(x[i]);
    out[3 * i + 1] = sb::rs_rsqrt(x[i]);
    out[3 * i + 2] = sb::rs_sqrt(x[i]);
}

// x: n host doubles; out: 3n host doubles (1/x, 1/sqrt(x), sqrt(x)).  Returns a cudaError_t.
extern "C" int rs_eval(const double* x, double* out, long long n) {
    double *dx = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 3 * n);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        rs_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dx, dout, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return (int)e;
}
