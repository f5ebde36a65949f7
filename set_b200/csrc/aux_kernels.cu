// aux_kernels.cu -- initial condition, Cell_par <-> conserved conversions, batched chlld and
// chlld_Q.
#include "setb_internal.cuh"
#include "chlld_q.cuh"

namespace sb {
namespace {

__global__ void lism_init_kernel(const GridGeom g, const double* __restrict__ lism_in, uint64_t seed,
                                 double pert, double* __restrict__ U) {
    __shared__ double lism[8];
    if (threadIdx.x < 8) lism[threadIdx.x] = lism_in[threadIdx.x];
    __syncthreads();
    const long long N = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx);
        const int j = (int)((c / g.nx) % g.ny);
        const int k = (int)(c / ((long long)g.nx * g.ny));
        double u8[8];
        lism_cell(g, lism, seed, pert, i, j, k, u8);
        const long long off = (long long)k * g.ps + (long long)j * g.px + i;
#pragma unroll
        for (int v = 0; v < 8; v++) U[v * g.vs + off] = u8[v];
    }
}

// prim8: [N][8] packed primitives (columns 1..8 of Cell_par) -> conserved SoA
__global__ void prim_to_cons_kernel(const GridGeom g, const double* __restrict__ prim8, double* __restrict__ U) {
    const long long N = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx);
        const int j = (int)((c / g.nx) % g.ny);
        const int k = (int)(c / ((long long)g.nx * g.ny));
        double q[8], u8[8];
        const double2* p2 = reinterpret_cast<const double2*>(prim8 + 8 * c);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const double2 d = p2[v];
            q[2 * v] = d.x;
            q[2 * v + 1] = d.y;
        }
        cons_from_prim_exact(q, u8);
        const long long off = (long long)k * g.ps + (long long)j * g.px + i;
#pragma unroll
        for (int v = 0; v < 8; v++) U[v * g.vs + off] = u8[v];
    }
}

__global__ void cons_to_prim_kernel(const GridGeom g, const double* __restrict__ U, double* __restrict__ prim8) {
    const long long N = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx);
        const int j = (int)((c / g.nx) % g.ny);
        const int k = (int)(c / ((long long)g.nx * g.ny));
        const long long off = (long long)k * g.ps + (long long)j * g.px + i;
        double q[8], u8[8];
#pragma unroll
        for (int v = 0; v < 8; v++) u8[v] = U[v * g.vs + off];
        prim_from_cons_exact(u8, q);
        double2* p2 = reinterpret_cast<double2*>(prim8 + 8 * c);
#pragma unroll
        for (int v = 0; v < 4; v++) p2[v] = make_double2(q[2 * v], q[2 * v + 1]);
    }
}

template <typename T, int NSTATE, bool DELTA = false>
__global__ void chlld_batch_kernel(int64_t n, int n_disc, const double* __restrict__ normals,
                                   const double* __restrict__ w, const double* __restrict__ q1,
                                   const double* __restrict__ q2, double* __restrict__ qqq,
                                   double* __restrict__ speeds, int32_t* __restrict__ flags) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        chlld_general<T, NSTATE, DELTA>(normals + 3 * k, w ? w[k] : 0.0, q1 + 8 * k, q2 + 8 * k, n_disc, qqq + 8 * k,
                             speeds + 3 * k, flags + k);
    }
}

template <int NSTATE>
__global__ void chlld_q_batch_kernel(int64_t n, int n_disc, bool ydar, const double* __restrict__ normals,
                                     const double* __restrict__ w, const double* __restrict__ q1,
                                     const double* __restrict__ q2, double* __restrict__ konvect,
                                     double* __restrict__ qqq, double* __restrict__ speeds,
                                     int32_t* __restrict__ flags) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        chlld_q_general<NSTATE>(normals + 3 * k, w ? w[k] : 0.0, q1 + 9 * k, q2 + 9 * k, n_disc, ydar,
                                konvect ? konvect + 3 * k : nullptr, qqq + 9 * k, speeds + 3 * k, flags + k);
    }
}

int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

}  // namespace

cudaError_t launch_lism_init(const GridGeom& g, const double* lism, uint64_t seed, double pert, double* U,
                             cudaStream_t s) {
    const long long N = (long long)g.nx * g.ny * g.nz;
    lism_init_kernel<<<grid_for(N, 256), 256, 0, s>>>(g, lism, seed, pert, U);
    return cudaGetLastError();
}

cudaError_t launch_prim_to_cons(const GridGeom& g, const double* prim8, double* U, cudaStream_t s) {
    const long long N = (long long)g.nx * g.ny * g.nz;
    prim_to_cons_kernel<<<grid_for(N, 256), 256, 0, s>>>(g, prim8, U);
    return cudaGetLastError();
}

cudaError_t launch_cons_to_prim(const GridGeom& g, const double* U, double* prim8, cudaStream_t s) {
    const long long N = (long long)g.nx * g.ny * g.nz;
    cons_to_prim_kernel<<<grid_for(N, 256), 256, 0, s>>>(g, U, prim8);
    return cudaGetLastError();
}

cudaError_t launch_chlld_batch(int64_t n, int n_state, int n_disc, int precision, const double* normals,
                               const double* w, const double* q1, const double* q2, double* qqq,
                               double* speeds, int32_t* flags, cudaStream_t s) {
    const int g = grid_for(n, 128);
#define SB_LAUNCH(T, NS) chlld_batch_kernel<T, NS><<<g, 128, 0, s>>>(n, n_disc, normals, w, q1, q2, qqq, speeds, flags)
    if (precision == 2) {
        if (n_state == 2) chlld_batch_kernel<double, 2, true><<<g, 128, 0, s>>>(n, n_disc, normals, w, q1, q2, qqq, speeds, flags);
        else chlld_batch_kernel<double, 3, true><<<g, 128, 0, s>>>(n, n_disc, normals, w, q1, q2, qqq, speeds, flags);
    } else if (precision == 1) {
        switch (n_state) {
            case 0: SB_LAUNCH(float, 0); break;
            case 1: SB_LAUNCH(float, 1); break;
            case 2: SB_LAUNCH(float, 2); break;
            default: SB_LAUNCH(float, 3); break;
        }
    } else {
        switch (n_state) {
            case 0: SB_LAUNCH(double, 0); break;
            case 1: SB_LAUNCH(double, 1); break;
            case 2: SB_LAUNCH(double, 2); break;
            default: SB_LAUNCH(double, 3); break;
        }
    }
#undef SB_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_chlld_q_batch(int64_t n, int n_state, int n_disc, bool ydar, const double* normals,
                                 const double* w, const double* q1, const double* q2, double* konvect,
                                 double* qqq, double* speeds, int32_t* flags, cudaStream_t s) {
    const int g = grid_for(n, 128);
#define SB_LAUNCH_Q(NS) \
    chlld_q_batch_kernel<NS><<<g, 128, 0, s>>>(n, n_disc, ydar, normals, w, q1, q2, konvect, qqq, speeds, flags)
    switch (n_state) {
        case 0: SB_LAUNCH_Q(0); break;
        case 1: SB_LAUNCH_Q(1); break;
        case 2: SB_LAUNCH_Q(2); break;
        default: SB_LAUNCH_Q(3); break;
    }
#undef SB_LAUNCH_Q
    return cudaGetLastError();
}

}  // namespace sb
