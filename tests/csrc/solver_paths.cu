// Test-only kernels: the region-first (LAZY) and branch-free (eager) instantiations of the
// Riemann solvers of set_b200/csrc/mhd_core.cuh side by side on the same face states, and the
// quick pressure-positivity test and the guarded primitive recovery next to the exact recovery.
// Built by tests/test_gpu_solver_paths.py with nvcc for sm_100a into a temporary library.
#include <cuda_runtime.h>
#include "mhd_core.cuh"

using namespace sb;

namespace {

constexpr int kOut = 12;   // F[8], SL, SR, SM, flag

template <typename T, typename S>
__device__ void store(double* o, const T* F, S SL, S SR, S SM, int fl) {
    for (int v = 0; v < 8; v++) o[v] = (double)F[v];
    o[8] = (double)SL;
    o[9] = (double)SR;
    o[10] = (double)SM;
    o[11] = (double)fl;
}

// mode 0: the plain form's FP64 solver (NR, check off); 1: the FP64 recompute's (library special
// functions); 2: FP32 with the star check (the mixed form's n_disc fallback)
template <int NSTATE, bool LAZY>
__global__ void riemann_kernel(const double* q1, const double* q2, int n_disc, int mode, double* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* o = out + kOut * i;
    if (mode == 2) {
        float a[8], b[8], F[8], SL, SR, SM;
        for (int v = 0; v < 8; v++) {
            a[v] = (float)q1[8 * i + v];
            b[v] = (float)q2[8 * i + v];
        }
        const int fl = riemann<float, NSTATE, false, true, true, false, LAZY>(a, b, 0.0f, n_disc, F, SL, SR, SM);
        store(o, F, SL, SR, SM, fl);
        return;
    }
    double F[8], SL, SR, SM;
    int fl;
    if (mode == 0)
        fl = riemann<double, NSTATE, false, false, true, false, LAZY>(q1 + 8 * i, q2 + 8 * i, 0.0, n_disc, F, SL, SR, SM);
    else
        fl = riemann<double, NSTATE, false, false, false, false, LAZY>(q1 + 8 * i, q2 + 8 * i, 0.0, n_disc, F, SL, SR, SM);
    store(o, F, SL, SR, SM, fl);
}

template <int NSTATE, bool LAZY>
__global__ void delta_kernel(const double* q1, const double* q2, double* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double F[8];
    float SL, SR, SM;
    const int fl = riemann_delta<NSTATE, double, LAZY>(q1 + 8 * i, q2 + 8 * i, F, SL, SR, SM);
    store(out + kOut * i, F, SL, SR, SM, fl);
}

// out[2 i] = pressure_surely_positive(U), out[2 i + 1] = the exact recovery's p > 0
__global__ void ptest_kernel(const double* U, int* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double q[8], ke, me;
    prim_from_cons<true>(U + 8 * i, q, ke, me);
    out[2 * i] = pressure_surely_positive(U + 8 * i) ? 1 : 0;
    out[2 * i + 1] = q[4] > 0.0 ? 1 : 0;
}

// out[16 i .. 16 i + 7] = prim_from_cons_guarded(U), out[16 i + 8 ..] = prim_from_cons<true>(U)
__global__ void guarded_kernel(const double* U, double* out, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ke, me;
    prim_from_cons_guarded(U + 8 * i, out + 16 * i);
    prim_from_cons<true>(U + 8 * i, out + 16 * i + 8, ke, me);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int run(void (*launch)(const double*, const double*, double*, long long), const double* q1, const double* q2,
        double* out, long long n) {
    DevBuf a, b, o;
    const size_t qs = sizeof(double) * 8 * n, os = sizeof(double) * kOut * n;
    if (cudaMalloc(&a.p, qs) || cudaMalloc(&b.p, qs) || cudaMalloc(&o.p, os)) return 1;
    if (cudaMemcpy(a.p, q1, qs, cudaMemcpyHostToDevice) || cudaMemcpy(b.p, q2, qs, cudaMemcpyHostToDevice)) return 2;
    launch((const double*)a.p, (const double*)b.p, (double*)o.p, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(out, o.p, os, cudaMemcpyDeviceToHost)) return 4;
    return 0;
}

int g_n_disc = 0, g_mode = 0;

template <int NSTATE, bool LAZY>
void launch_riemann(const double* a, const double* b, double* o, long long n) {
    riemann_kernel<NSTATE, LAZY><<<(unsigned)((n + 255) / 256), 256>>>(a, b, g_n_disc, g_mode, o, n);
}

template <int NSTATE, bool LAZY>
void launch_delta(const double* a, const double* b, double* o, long long n) {
    delta_kernel<NSTATE, LAZY><<<(unsigned)((n + 255) / 256), 256>>>(a, b, o, n);
}

}  // namespace

// Face states q1, q2 ([n][8]: rho, vn, vt1, vt2, p, Bn, Bt1, Bt2, stored B); out [n][12] for the
// region-first and the branch-free instantiation.  nstate 2 or 3.
extern "C" int riemann_pair(const double* q1, const double* q2, long long n, int nstate, int n_disc, int mode,
                            double* out_lazy, double* out_eager) {
    g_n_disc = n_disc;
    g_mode = mode;
    int rc;
    if (nstate == 2) {
        if ((rc = run(launch_riemann<2, true>, q1, q2, out_lazy, n))) return rc;
        return run(launch_riemann<2, false>, q1, q2, out_eager, n);
    }
    if ((rc = run(launch_riemann<3, true>, q1, q2, out_lazy, n))) return rc;
    return run(launch_riemann<3, false>, q1, q2, out_eager, n);
}

extern "C" int delta_pair(const double* q1, const double* q2, long long n, int nstate, double* out_lazy,
                          double* out_eager) {
    int rc;
    if (nstate == 2) {
        if ((rc = run(launch_delta<2, true>, q1, q2, out_lazy, n))) return rc;
        return run(launch_delta<2, false>, q1, q2, out_eager, n);
    }
    if ((rc = run(launch_delta<3, true>, q1, q2, out_lazy, n))) return rc;
    return run(launch_delta<3, false>, q1, q2, out_eager, n);
}

extern "C" int pressure_test(const double* U, long long n, int* out) {
    DevBuf u, o;
    if (cudaMalloc(&u.p, sizeof(double) * 8 * n) || cudaMalloc(&o.p, sizeof(int) * 2 * n)) return 1;
    if (cudaMemcpy(u.p, U, sizeof(double) * 8 * n, cudaMemcpyHostToDevice)) return 2;
    ptest_kernel<<<(unsigned)((n + 255) / 256), 256>>>((const double*)u.p, (int*)o.p, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(out, o.p, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost)) return 4;
    return 0;
}

extern "C" int guarded_recovery(const double* U, long long n, double* out) {
    DevBuf u, o;
    if (cudaMalloc(&u.p, sizeof(double) * 8 * n) || cudaMalloc(&o.p, sizeof(double) * 16 * n)) return 1;
    if (cudaMemcpy(u.p, U, sizeof(double) * 8 * n, cudaMemcpyHostToDevice)) return 2;
    guarded_kernel<<<(unsigned)((n + 255) / 256), 256>>>((const double*)u.p, (double*)o.p, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(out, o.p, sizeof(double) * 16 * n, cudaMemcpyDeviceToHost)) return 4;
    return 0;
}
