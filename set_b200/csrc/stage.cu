// stage.cu -- one fused stage of the MHD step on a Cartesian grid, plain FP64 or mixed precision.
//
// Replaces the reference's face kernel + cell kernel pair (CUF_MGD_grans_RK2 /
// CUF_MGD_cell_RK2, SET_Fortran_Cuda_MHD/cuf_solvers.cuf:243-440 and :561-794; Euler variants
// :62-241, :443-558), which exchange fluxes through a 9 x N_gran array in HBM, with a single
// kernel per stage:
//   * a CTA owns a 32 x 7 column of cells and marches along z over lz planes;
//   * each plane (cells + 2-cell x/y halo) is read from the SoA conserved state once, turned into
//     primitives once (FP64 pressure recovery) and kept in a 4-plane shared-memory ring
//     (planes k-1 .. k+2), which is all the z-stencil of the minmod reconstruction needs;
//   * every face of the plane (x, y and the z face k+1/2) is computed once, by one thread, from
//     shared memory, and its flux is applied to both neighbouring cells (the z face k-1/2 is
//     carried in registers from the previous plane);
//   * the conservative update, p floor, source re-imposition and the dt candidate reduction
//     (warp shuffle -> one atomicMin per CTA) are fused; the last CTA rolls the lagged-dt clock.
//
// P = 0, plain form: everything in FP64.
// P = 1, mixed form: the ring holds FP32 primitives (recovered from the FP64 state in FP64),
//   reconstruction and the Riemann solver run in FP32, fluxes are stored in FP32; a face whose
//   selected FP32 state has rho <= 0 or p <= 0 (or a non-finite flux) is recomputed in FP64 from
//   the FP64 state; the flux divergence and the update are FP64, and the second Heun stage (or
//   the Euler step) is a compensated sum with the compensation kept in FP32; dt is reduced in
//   FP64.  Half the shared memory and at most 128 registers give two CTAs per SM.
#include <cfloat>
#include <type_traits>
#include "setb_internal.cuh"

namespace sb {
namespace {

// 32 x 7 cells per CTA and 256 threads: the 711 faces of a plane take three rounds of 256 (a
// 32 x 8 tile has 808 faces, whose fourth round of 40 leaves 6 of 8 warps waiting at the
// barrier; 288 threads would fit 808 faces into three rounds, but a sub-partition holding 3 of
// 9 warps caps FP64 HLLD at 168 registers and spills).  Threads 0..223 own one cell each in the
// update.
constexpr int TX = kTileX, TY = kTileY, NC = TX * TY, NT = kStageThreads;
static_assert(NC <= NT, "one thread per cell in the update");
constexpr int HX = TX + 4, HY = TY + 4, PLANE = HX * HY;
constexpr int NZF = NC;                   // z faces k+1/2 of the column tile
constexpr int NXF = (TX + 1) * TY;        // x faces
constexpr int NYF = TX * (TY + 1);        // y faces
constexpr int NF = NZF + NXF + NYF;
constexpr int RING = 4;

__device__ __forceinline__ int ring_slot(int k) { return (k + 4 * RING) & (RING - 1); }

// FP64 primitive state of global cell (i,j,k) with the boundary rules: inflow beyond x = hi,
// zero-gradient (clamped index) elsewhere.
__device__ __forceinline__ void fetch_prim64(const StageArgs& A, int i, int j, int k, double* q) {
    const GridGeom& g = A.g;
    if (i >= g.nx) {
#pragma unroll
        for (int v = 0; v < 8; v++) q[v] = g.inflow[v];
        return;
    }
    i = max(i, 0);
    j = min(max(j, 0), g.ny - 1);
    k = min(max(k, 0), g.nz - 1);
    const long long off = (long long)k * g.ps + (long long)j * g.px + i;
    double U[8];
#pragma unroll
    for (int v = 0; v < 8; v++) U[v] = __ldg(A.Uin + v * g.vs + off);
    double ke, me;
    prim_from_cons(U, q, ke, me);
}

// Loads plane kk (with halo) of the tile starting at (i0, j0) as primitives into `dst`.
template <typename RT>
__device__ __forceinline__ void load_plane(const StageArgs& A, RT* dst, int i0, int j0, int kk) {
    for (int c = threadIdx.x; c < PLANE; c += NT) {
        const int cx = c % HX, cy = c / HX;
        double q[8];
        fetch_prim64(A, i0 - 2 + cx, j0 - 2 + cy, kk, q);
#pragma unroll
        for (int v = 0; v < 8; v++) dst[v * PLANE + c] = (RT)q[v];
    }
}

// The FP64 recompute of one face of the mixed form (rare path; kept out of line so the FP32
// path keeps its registers).  (i, j, k) is the cell on the high side of the face.
template <int NSTATE, int ORDER>
__device__ __noinline__ int face_fp64(const StageArgs& A, int axis, int i, int j, int k, double* F, double* sl,
                                      double* sr) {
    const int di = axis == 0, dj = axis == 1, dk = axis == 2;
    double c[4][8];
    fetch_prim64(A, i - 2 * di, j - 2 * dj, k - 2 * dk, c[0]);
    fetch_prim64(A, i - di, j - dj, k - dk, c[1]);
    fetch_prim64(A, i, j, k, c[2]);
    fetch_prim64(A, i + di, j + dj, k + dk, c[3]);
    const int pn = 1 + axis, pt1 = axis == 0 ? 2 : 1, pt2 = axis == 2 ? 2 : 3;
    const int perm[8] = {0, pn, pt1, pt2, 4, 4 + pn, 4 + pt1, 4 + pt2};
    double f[4][8];
    for (int s = 0; s < 4; s++)
        for (int v = 0; v < 8; v++) f[s][v] = c[s][perm[v]];
    double q1[8], q2[8], G[8], SM;
    reconstruct<double, ORDER>(f[0], f[1], f[2], f[3], q1, q2);
    const int fl = riemann<double, NSTATE, false, false>(q1, q2, 0.0, A.n_disc, G, *sl, *sr, SM);
    for (int v = 0; v < 8; v++) F[perm[v]] = G[v];
    return fl;
}

// One tile of one stage: the column (bx, by) of TX x TY cells, planes [bz*lz, min(nz, (bz+1)*lz)).
// `total_tiles` is the number of tiles of this solve in the launch; the last one to finish rolls
// the solve's clock.  Called by the single-solve kernel (one tile per CTA) and by the batch
// kernel (tiles of many solves drawn from a work queue); every CTA-wide barrier is reached by all
// threads, and the function ends with one so a CTA may run the next tile immediately.
// Storage and arithmetic types of the two forms: ring (primitives), flux buffer, Riemann math.
template <int P> struct Types {
    using Ring = double;
    using Flux = double;
    using Math = double;
};
template <> struct Types<2> {   // delta form: FP64 states and fluxes, FP32 inside the solver
    using Ring = double;
    using Flux = double;
    using Math = double;
};
template <> struct Types<1> {
#if defined(SB_MIXED_RING_FP64)
    using Ring = double;
#else
    using Ring = float;
#endif
#if defined(SB_MIXED_FLUX_FP64)
    using Flux = double;
#else
    using Flux = float;
#endif
    using Math = float;
};

// FP64 recompute of a face of the delta form from its (FP64) face states; out of line so the
// main path keeps its registers.
template <int NSTATE>
__device__ __noinline__ int face_fp64_states(const double* q1, const double* q2, int n_disc, double* F, double* sl,
                                             double* sr) {
    double SM;
    return riemann<double, NSTATE, false, false>(q1, q2, 0.0, n_disc, F, *sl, *sr, SM);
}

template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT>
__device__ __forceinline__ void run_tile(const StageArgs& A, int bx, int by, int bz, unsigned total_tiles) {
    using RG = typename Types<P>::Ring;
    using FT = typename Types<P>::Flux;
    using RT = typename Types<P>::Math;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RG* ring = reinterpret_cast<RG*>(smem_raw);
    FT* fz = reinterpret_cast<FT*>(ring + RING * 8 * PLANE);   // [8][NZF]
    FT* fx = fz + 8 * NZF;                                      // [8][NXF]
    FT* fy = fx + 8 * NXF;                                      // [8][NYF]
    __shared__ double red[NT / 32];
    __shared__ unsigned long long cnt[5];
    __shared__ bool last_cta;

    const GridGeom& g = A.g;
    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int i0 = bx * TX, j0 = by * TY;
    const int k0 = bz * g.lz;
    const int k1 = min(g.nz, k0 + g.lz);
    const double dt = A.clk->dt_cur;
    if (t < 5) cnt[t] = 0;

    double rate = 0.0;   // max over this thread's real faces of max(|SL|,|SR|)/dist
    unsigned n_recon = 0, n_wave = 0, n_redo = 0;

    // Computes face f of plane k (flattened: z faces, x faces, y faces) into fz/fx/fy.
    // `dup`: the face is also computed by the CTA below (chunk-boundary z face); it still enters
    // the dt candidate (min is idempotent) but not the diagnostic counters.
    auto do_face = [&](int f, int k, bool dup) {
        int axis, cLL, cL, cR, cRR, fxx, fyy, gk;
        const RG *sLL, *sL, *sR, *sRR;
        FT* out;
        int oidx, ostride;
        bool real;
        if (f < NZF) {
            fxx = f % TX;
            fyy = f / TX;
            axis = 2;
            const int c = (fyy + 2) * HX + fxx + 2;
            cLL = cL = cR = cRR = c;
            sLL = ring + ring_slot(k - 1) * 8 * PLANE;
            sL = ring + ring_slot(k) * 8 * PLANE;
            sR = ring + ring_slot(k + 1) * 8 * PLANE;
            sRR = ring + ring_slot(k + 2) * 8 * PLANE;
            out = fz;
            oidx = f;
            ostride = NZF;
            gk = k + 1;
            real = (i0 + fxx < g.nx) && (j0 + fyy < g.ny) && (k + 1 <= g.nz) && (k + 1 >= 0);
        } else if (f < NZF + NXF) {
            const int idx = f - NZF;
            fyy = idx / (TX + 1);
            fxx = idx % (TX + 1);
            axis = 0;
            const int c = (fyy + 2) * HX + fxx;   // cell fxx-2 (tile-local) at halo offset +2
            cLL = c; cL = c + 1; cR = c + 2; cRR = c + 3;
            sLL = sL = sR = sRR = ring + ring_slot(k) * 8 * PLANE;
            out = fx;
            oidx = idx;
            ostride = NXF;
            gk = k;
            real = (i0 + fxx <= g.nx) && (j0 + fyy < g.ny);
        } else {
            const int idx = f - NZF - NXF;
            fyy = idx / TX;
            fxx = idx % TX;
            axis = 1;
            const int c = fyy * HX + fxx + 2;     // row fyy-2 (tile-local)
            cLL = c; cL = c + HX; cR = c + 2 * HX; cRR = c + 3 * HX;
            sLL = sL = sR = sRR = ring + ring_slot(k) * 8 * PLANE;
            out = fy;
            oidx = idx;
            ostride = NYF;
            gk = k;
            real = (i0 + fxx < g.nx) && (j0 + fyy <= g.ny);
        }
        // face-frame permutation of the velocity / B components
        const int pn = 1 + axis;
        const int pt1 = axis == 0 ? 2 : 1;
        const int pt2 = axis == 2 ? 2 : 3;
        RT qLL[8], qL[8], qR[8], qRR[8];
        const int perm[8] = {0, pn, pt1, pt2, 4, 4 + pn, 4 + pt1, 4 + pt2};
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const int o = perm[v] * PLANE;
            qL[v] = (RT)sL[o + cL];
            qR[v] = (RT)sR[o + cR];
            if (v < 5) {
                qLL[v] = (RT)sLL[o + cLL];
                qRR[v] = (RT)sRR[o + cRR];
            } else {
                qLL[v] = RT(0);
                qRR[v] = RT(0);
            }
        }
        RT q1[8], q2[8], F[8];
        reconstruct<RT, ORDER>(qLL, qL, qR, qRR, q1, q2);
        if (real && !dup && (q1[0] < RT(0) || q2[0] < RT(0))) n_recon++;
        int fl;
        double sl, sr;
        if constexpr (P == 2) {
            float SLf, SRf, SMf;
            fl = riemann_delta<NSTATE>(q1, q2, F, SLf, SRf, SMf);
            sl = (double)SLf;
            sr = (double)SRf;
            if (fl & kFlagStar) {
                fl = face_fp64_states<NSTATE>(q1, q2, A.n_disc, F, &sl, &sr);
                if (real && !dup) n_redo++;
            }
        } else {
            RT SL, SR, SM;
            fl = riemann<RT, NSTATE, false, P == 1>(q1, q2, RT(0), A.n_disc, F, SL, SR, SM);
            sl = (double)SL;
            sr = (double)SR;
        }
        const double sq = g.square[axis];
        if (P == 1 && real && (fl & kFlagStar)) {
            double F64[8];
            fl = face_fp64<NSTATE, ORDER>(A, axis, i0 + fxx, j0 + fyy, gk, F64, &sl, &sr);
            if (!dup) n_redo++;
#pragma unroll
            for (int v = 0; v < 8; v++) out[v * ostride + oidx] = (FT)(F64[v] * sq);
        } else {
            if (fl & kFlagWave) {
#pragma unroll
                for (int v = 0; v < 8; v++) F[v] = RT(0);
            }
#pragma unroll
            for (int v = 0; v < 8; v++) out[perm[v] * ostride + oidx] = (FT)(F[v] * (RT)sq);
        }
        if ((fl & kFlagWave) && real && !dup) n_wave++;
        if (WANT_DT && real) rate = fmax(rate, fmax(fabs(sl), fabs(sr)) * g.inv_dist[axis]);
    };

    // ---- the march.  Iteration k0-1 is the prologue: planes k0-2 .. k0+1 and only the z face
    // k0-1/2 (carried into the first update).  Every face goes through the one do_face call
    // site below, so a face's arithmetic does not depend on where a chunk starts.
    for (int kk = k0 - 2; kk <= k0; kk++) load_plane<RG>(A, ring + ring_slot(kk) * 8 * PLANE, i0, j0, kk);
    double fzl[8];
    const int gi = i0 + tx, gj = j0 + ty;
    const bool own = (t < NC) && (gi < g.nx) && (gj < g.ny);
    for (int k = k0 - 1; k < k1; k++) {
        load_plane<RG>(A, ring + ring_slot(k + 2) * 8 * PLANE, i0, j0, k + 2);
        __syncthreads();
        const bool pro = (k < k0);
        const int nf = pro ? NZF : NF;
        for (int f = t; f < nf; f += NT) do_face(f, k, pro && k0 > 0);
        __syncthreads();
        double fzh[8];
#pragma unroll
        for (int v = 0; v < 8; v++) fzh[v] = t < NC ? (double)fz[v * NZF + t] : 0.0;
        if (pro) {
#pragma unroll
            for (int v = 0; v < 8; v++) fzl[v] = fzh[v];
            continue;
        }
        if (own) {
            const long long off = (long long)k * g.ps + (long long)gj * g.px + gi;
            double un[8], qs[8];
            bool reset_comp = false;
            if (source_prim(g, gi, gj, k, qs)) {
                cons_from_prim_exact(qs, un);
                reset_comp = true;
            } else {
                double uin[8], cmp[8];
#pragma unroll
                for (int v = 0; v < 8; v++) {
                    double pot = 0.0;
                    pot = pot - (double)fx[v * NXF + ty * (TX + 1) + tx];
                    pot = pot + (double)fx[v * NXF + ty * (TX + 1) + tx + 1];
                    pot = pot - (double)fy[v * NYF + ty * TX + tx];
                    pot = pot + (double)fy[v * NYF + (ty + 1) * TX + tx];
                    pot = pot - fzl[v];
                    pot = pot + fzh[v];
                    uin[v] = A.Uin[v * g.vs + off];
                    const double inc = dt * (pot * g.inv_vol);
                    if (P != 0 && A.comp) {
                        // compensated sum U_new = base + delta (cuf_solvers.cuf:741-770 as an
                        // increment); the FP32 compensation carries the rounding of the add
                        const double base = KIND == 0 ? uin[v] : A.Ubase[v * g.vs + off];
                        const double delta = KIND == 0 ? -inc : 0.5 * ((uin[v] - base) - inc);
                        const double y = delta - (double)A.comp[v * g.vs + off];
                        const double s = base + y;
                        cmp[v] = (s - base) - y;
                        un[v] = s;
                    } else if (KIND == 0) {
                        un[v] = uin[v] - inc;
                    } else {
                        un[v] = 0.5 * ((A.Ubase[v * g.vs + off] + uin[v]) - inc);
                    }
                }
                if (!(un[0] > 0.0)) {                    // cuf_solvers.cuf:708-711
                    atomicAdd(&cnt[0], 1ull);
                    atomicMin(&A.st->first_bad, (unsigned long long)(gi + (long long)g.nx * (gj + (long long)g.ny * k)));
#pragma unroll
                    for (int v = 0; v < 8; v++) un[v] = uin[v];
                    reset_comp = true;
                } else {
                    double q[8], ke, me;
                    prim_from_cons(un, q, ke, me);
                    if (q[4] <= 0.0) {                    // cuf_solvers.cuf:777-779
                        atomicAdd(&cnt[1], 1ull);
                        un[4] = (kPFloor * kInvG1 + ke) + me;
                        cmp[4] = 0.0;
                    }
                }
                if (P != 0 && A.comp && !reset_comp) {
#pragma unroll
                    for (int v = 0; v < 8; v++) A.comp[v * g.vs + off] = (float)cmp[v];
                }
            }
            if (P != 0 && A.comp && reset_comp) {
#pragma unroll
                for (int v = 0; v < 8; v++) A.comp[v * g.vs + off] = 0.0f;
            }
#pragma unroll
            for (int v = 0; v < 8; v++) A.Uout[v * g.vs + off] = un[v];
        }
#pragma unroll
        for (int v = 0; v < 8; v++) fzl[v] = fzh[v];
    }

    // ---- reductions: counters and the dt candidate
    if (n_recon) atomicAdd(&cnt[2], (unsigned long long)n_recon);
    if (n_wave) atomicAdd(&cnt[3], (unsigned long long)n_wave);
    if (n_redo) atomicAdd(&cnt[4], (unsigned long long)n_redo);
    if (WANT_DT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
        if ((t & 31) == 0) red[t >> 5] = rate;
    }
    __syncthreads();
    if (t == 0) {
        if (WANT_DT) {
            double r = red[0];
#pragma unroll
            for (int w = 1; w < NT / 32; w++) r = fmax(r, red[w]);
            const double cand = fmin(kDtFaceCap, A.cfl / r);   // r == 0 -> +inf -> cap
            atomicMin(&A.clk->dt_next, (unsigned long long)__double_as_longlong(cand));
        }
        if (cnt[0]) atomicAdd(&A.st->n_negdens, cnt[0]);
        if (cnt[1]) atomicAdd(&A.st->n_pfloor, cnt[1]);
        if (cnt[2]) atomicAdd(&A.st->n_recon, cnt[2]);
        if (cnt[3]) atomicAdd(&A.st->n_wave, cnt[3]);
        if (cnt[4]) atomicAdd(&A.st->n_redo, cnt[4]);
        __threadfence();
        const unsigned ticket = atomicAdd(&A.clk->counter, 1u);
        last_cta = (ticket == total_tiles - 1);
    }
    __syncthreads();
    if (last_cta && t == 0) {
        __threadfence();
        DevClock* c = A.clk;
        c->counter = 0;
        if (A.finalize) {
            const unsigned long long nb = atomicExch(&c->dt_next, (unsigned long long)__double_as_longlong(kDtReset));
            c->time_all += c->dt_cur;
            c->dt_last = c->dt_cur;
            c->dt_cur = __longlong_as_double((long long)nb);
            c->steps += 1;
        }
        __threadfence();
    }
    __syncthreads();
}

template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT>
__global__ void __launch_bounds__(NT, P == 1 ? 2 : 1) stage_kernel(const StageArgs A) {
    run_tile<P, NSTATE, ORDER, KIND, WANT_DT>(A, blockIdx.x, blockIdx.y, blockIdx.z,
                                               gridDim.x * gridDim.y * gridDim.z);
}

// Persistent batch kernel: each CTA takes tiles from the work queue until it is empty; the
// tile's solve selects the arguments (copied to shared memory) and the Riemann solver.  The
// items of one solve are counted by its own clock, so every solve keeps its own lagged dt.
template <int P, int ORDER, int KIND, bool WANT_DT>
__global__ void __launch_bounds__(NT, P == 1 ? 2 : 1) batch_stage_kernel(const BatchArgs B) {
    __shared__ __align__(16) StageArgs As;
    __shared__ int4 it;
    constexpr int WORDS = sizeof(StageArgs) / sizeof(unsigned long long);
    static_assert(sizeof(StageArgs) % sizeof(unsigned long long) == 0, "StageArgs must be 8-byte granular");
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned i = atomicAdd(B.queue, 1u);
            it = i < (unsigned)B.n_items ? B.items[i] : make_int4(-1, 0, 0, 0);
        }
        __syncthreads();
        const int4 w = it;
        if (w.x < 0) break;
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(B.inst + w.x);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&As);
        for (int q = threadIdx.x; q < WORDS; q += NT) dst[q] = src[q];
        __syncthreads();
        if (As.n_state == 3)
            run_tile<P, 3, ORDER, KIND, WANT_DT>(As, w.y, w.z, w.w, As.total_tiles);
        else
            run_tile<P, 2, ORDER, KIND, WANT_DT>(As, w.y, w.z, w.w, As.total_tiles);
    }
}

template <int P>
constexpr int smem_bytes() {
    return RING * 8 * PLANE * (int)sizeof(typename Types<P>::Ring) +
           8 * (NZF + NXF + NYF) * (int)sizeof(typename Types<P>::Flux);
}

template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT>
cudaError_t launch_t(const StageArgs& a, cudaStream_t s) {
    auto kern = stage_kernel<P, NSTATE, ORDER, KIND, WANT_DT>;
    const int smem = smem_bytes<P>();
    static bool attr_set = false;   // per process; every device shares the same limit
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, (a.g.nz + a.g.lz - 1) / a.g.lz);
    kern<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int P, int NSTATE>
cudaError_t launch_n(const StageArgs& a, int order, int kind, bool want_dt, cudaStream_t s) {
    if (order == 2) {
        if (kind == 0) return want_dt ? launch_t<P, NSTATE, 2, 0, true>(a, s) : launch_t<P, NSTATE, 2, 0, false>(a, s);
        return launch_t<P, NSTATE, 2, 1, false>(a, s);
    }
    if (kind == 0) return want_dt ? launch_t<P, NSTATE, 1, 0, true>(a, s) : launch_t<P, NSTATE, 1, 0, false>(a, s);
    return launch_t<P, NSTATE, 1, 1, false>(a, s);
}

template <int P>
cudaError_t launch_p(const StageArgs& a, int n_state, int order, int kind, bool want_dt, cudaStream_t s) {
    switch (n_state) {
        case 0: return launch_n<P, 0>(a, order, kind, want_dt, s);
        case 1: return launch_n<P, 1>(a, order, kind, want_dt, s);
        case 2: return launch_n<P, 2>(a, order, kind, want_dt, s);
        default: return launch_n<P, 3>(a, order, kind, want_dt, s);
    }
}

template <int P, int KIND, bool WANT_DT>
cudaError_t batch_attr() {
    return cudaFuncSetAttribute(batch_stage_kernel<P, 2, KIND, WANT_DT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_bytes<P>());
}

}  // namespace

cudaError_t prepare_batch_kernels(int precision) {
    cudaError_t e;
    if (precision == 1) {
        if ((e = batch_attr<1, 0, true>()) != cudaSuccess) return e;
        return batch_attr<1, 1, false>();
    }
    if (precision == 2) {
        if ((e = batch_attr<2, 0, true>()) != cudaSuccess) return e;
        return batch_attr<2, 1, false>();
    }
    if ((e = batch_attr<0, 0, true>()) != cudaSuccess) return e;
    return batch_attr<0, 1, false>();
}

int batch_ctas_per_sm(int precision) { return precision == 1 ? 2 : 1; }

template <int P>
void launch_batch_p(const BatchArgs& b, int kind, bool want_dt, int grid, cudaStream_t s) {
    if (kind == 0 && want_dt) batch_stage_kernel<P, 2, 0, true><<<grid, NT, smem_bytes<P>(), s>>>(b);
    else batch_stage_kernel<P, 2, 1, false><<<grid, NT, smem_bytes<P>(), s>>>(b);
}

cudaError_t launch_batch_stage(const BatchArgs& b, int precision, int kind, bool want_dt, int grid,
                               cudaStream_t s) {
    if (precision == 1) launch_batch_p<1>(b, kind, want_dt, grid, s);
    else if (precision == 2) launch_batch_p<2>(b, kind, want_dt, grid, s);
    else launch_batch_p<0>(b, kind, want_dt, grid, s);
    return cudaGetLastError();
}

int stage_smem_bytes(int precision) {
    return precision == 1 ? smem_bytes<1>() : (precision == 2 ? smem_bytes<2>() : smem_bytes<0>());
}
int stage_fp64_smem_bytes() { return smem_bytes<0>(); }

cudaError_t launch_stage(const StageArgs& a, int precision, int n_state, int order, int kind, bool want_dt,
                         cudaStream_t s) {
    if (precision == 1) return launch_p<1>(a, n_state, order, kind, want_dt, s);
    if (precision == 2)   // the delta form covers HLLC (n_state 2) and HLLD (n_state 3)
        return n_state == 2 ? launch_n<2, 2>(a, order, kind, want_dt, s) : launch_n<2, 3>(a, order, kind, want_dt, s);
    return launch_p<0>(a, n_state, order, kind, want_dt, s);
}

cudaError_t launch_stage_fp64(const StageArgs& a, int n_state, int order, int kind, bool want_dt,
                              cudaStream_t s) {
    return launch_p<0>(a, n_state, order, kind, want_dt, s);
}

}  // namespace sb
