// tests/csrc/rs_special.cu -- TEST HELPER, NOT PRODUCT CODE.
//
// Evaluates the product's FP64 Newton-refined special functions (rs_rcp, rs_rsqrt, rs_sqrt in
// set_b200/csrc/mhd_core.cuh), its quotient from a shared reciprocal (div_rn) and its exact
// primitive recovery (prim_from_cons<true>) on the device for tests/test_gpu_special.py, which
// compiles this file with nvcc into a temporary shared library.
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

__global__ void div_kernel(const double* a, const double* b, double* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i + 0] = sb::div_rn(a[i], b[i], __drcp_rn(b[i]));
    out[2 * i + 1] = a[i] / b[i];   // IEEE division
}

__global__ void prim_kernel(const double* U, double* q, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ke, me;
    sb::prim_from_cons<true>(U + 8 * i, q + 8 * i, ke, me);
}

// a, b: n host doubles; out: 2n host doubles (div_rn(a, b), a / b).  Returns a cudaError_t.
extern "C" int div_eval(const double* a, const double* b, double* out, long long n) {
    double *da = nullptr, *db = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&da, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&db, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 2 * n);
    if (e == cudaSuccess) e = cudaMemcpy(da, a, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(db, b, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        div_kernel<<<(unsigned)((n + 255) / 256), 256>>>(da, db, dout, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dout);
    return (int)e;
}

// U: 8n host doubles (conserved states); q: 8n host doubles (primitives).  Returns a cudaError_t.
extern "C" int prim_eval(const double* U, double* q, long long n) {
    double *dU = nullptr, *dq = nullptr;
    cudaError_t e = cudaMalloc(&dU, sizeof(double) * 8 * n);
    if (e == cudaSuccess) e = cudaMalloc(&dq, sizeof(double) * 8 * n);
    if (e == cudaSuccess) e = cudaMemcpy(dU, U, sizeof(double) * 8 * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        prim_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dU, dq, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(q, dq, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost);
    cudaFree(dU);
    cudaFree(dq);
    return (int)e;
}
