// stage.cu -- one fused stage of the MHD step on a Cartesian grid, plain FP64 or mixed precision.
//
// Replaces the reference's face kernel + cell kernel pair (CUF_MGD_grans_RK2 /
// CUF_MGD_cell_RK2, SET_Fortran_Cuda_MHD/cuf_solvers.cuf:243-440 and :561-794; Euler variants
// :62-241, :443-558), which exchange fluxes through a 9 x N_gran array in HBM, with a single
// kernel per stage:
//   * a CTA owns a 32 x TY column of cells and marches along z over lz planes;
//   * each plane (cells + 2-cell x/y halo) is read from the SoA conserved state once, turned into
//     primitives once (FP64 pressure recovery) and kept in a 4-plane shared-memory ring
//     (planes k-1 .. k+2), which is all the z-stencil of the minmod reconstruction needs;
//   * every face of the plane (x, y and the z face k+1/2) is computed once, by one thread, from
//     shared memory, and its flux is applied to both neighbouring cells (the z face k-1/2 is
//     carried in registers from the previous plane); faces are handed out in warp-sized jobs of
//     one axis, so the face-frame permutation is a compile-time constant;
//   * the conservative update, p floor, source re-imposition and the dt candidate reduction
//     (warp shuffle -> one atomicMin per CTA) are fused; the last CTA rolls the lagged-dt clock.
//
// P = 0, plain form: everything in FP64; the ring holds the field as b = B / sqrt(4 pi), the units
//   the Riemann solver works in, and the primitives are recovered exactly as the oracle does
//   wherever the kinetic and magnetic energies exceed 64 p, within a few ulps elsewhere
//   (prim_from_cons_guarded).
// P = 1, mixed form: the ring holds FP32 primitives (recovered from the FP64 state in FP64),
//   reconstruction and the Riemann solver run in FP32, fluxes are stored in FP32; a face whose
//   selected FP32 state has rho <= 0 or p <= 0 (or a non-finite flux) is recomputed in FP64 from
//   the FP64 state; the flux divergence and the update are FP64, and the second Heun stage (or
//   the Euler step) is a compensated sum with the compensation kept in FP32; dt is reduced in
//   FP64.  Half the shared memory and at most 128 registers give two CTAs per SM.
// P = 2, delta form: FP64 ring and fluxes, the Riemann solver's small differences in FP32.
#include <atomic>
#include <cfloat>
#include <type_traits>
#include "riemann_f32x2.cuh"
#include "setb_internal.cuh"

namespace sb {
namespace {

// Column tile of each form (tile_shape): TX = 32 cells per tile row, one lane per column.  The
// 3 TY + 2 warp jobs of a plane's faces (see run_tile) take three rounds of the CTA's warps
// (32 x 7 cells: 23 jobs over 8 warps; 32 x 11: 35 jobs over 12 warps).  Threads 0..NC-1 own
// one cell each in the update.
template <int P, int SK> struct Tile {   // SK: the launch kind of tile_shape
    static constexpr int TX = kTileX, TY = tile_shape(P, SK).ty, NT = tile_shape(P, SK).threads;
    static constexpr int MINB = tile_shape(P, SK).ctas_per_sm;
    static constexpr int NC = TX * TY;
    static constexpr int HX = TX + 4, HY = TY + 4, PLANE = HX * HY;
    static constexpr int NXF = (TX + 1) * TY;        // x faces
    static constexpr int NYF = TX * (TY + 1);        // y faces
    static_assert(TX == 32, "one lane per tile column");
    static_assert(NC <= NT, "one thread per cell in the update");
};
constexpr int RING = 4;

__device__ __forceinline__ int ring_slot(int k) { return (k + 4 * RING) & (RING - 1); }

// The inflow ghost state beyond x = hi as a primitive ring entry: stored B, or with SB the
// solver's b = B / sqrt(4 pi) (correctly rounded, as prim_from_cons<true, true> forms it).
template <bool SB>
__device__ __forceinline__ void inflow_prim(const GridGeom& g, double* q) {
#pragma unroll
    for (int v = 0; v < 8; v++) q[v] = (SB && v >= 5) ? div_rn(g.inflow[v], kSpi4, kInvSpi4) : g.inflow[v];
}

// FP64 primitive state of global cell (i,j,k) with the boundary rules: inflow beyond x = hi,
// zero-gradient (clamped index) elsewhere.  SB: the field as b (see prim_from_cons).
template <bool EXACT, bool SB = false>
__device__ __forceinline__ void fetch_prim64(const StageArgs& A, int i, int j, int k, double* q) {
    const GridGeom& g = A.g;
    if (i >= g.nx) {
        inflow_prim<SB>(g, q);
        return;
    }
    i = max(i, 0);
    j = min(max(j, 0), g.ny - 1);
    k = min(max(k, 0), g.nz - 1);
    const long long off = (long long)k * g.ps + (long long)j * g.px + i;
    double U[8];
#pragma unroll
    for (int v = 0; v < 8; v++) U[v] = __ldg(A.Uin + v * g.vs + off);
    if constexpr (EXACT) {
        prim_from_cons_guarded<SB>(U, q);
    } else {
        double ke, me;
        prim_from_cons<false, SB>(U, q, ke, me);
    }
}

// Loads plane kk (with halo) of the tile starting at (i0, j0) as primitives into `dst`.
template <int P, int SK, typename RT>
__device__ __forceinline__ void load_plane(const StageArgs& A, RT* dst, int i0, int j0, int kk) {
    constexpr int HX = Tile<P, SK>::HX, PLANE = Tile<P, SK>::PLANE, NT = Tile<P, SK>::NT;
    for (int c = threadIdx.x; c < PLANE; c += NT) {
        const int cx = c % HX, cy = c / HX;
        double q[8];
        fetch_prim64<P != 1, P == 0>(A, i0 - 2 + cx, j0 - 2 + cy, kk, q);
#pragma unroll
        for (int v = 0; v < 8; v++) dst[v * PLANE + c] = (RT)q[v];
    }
}

// ---- plane copies by the tensor-memory accelerator
// One copy per plane: the (kTileX + 4) x (TY + 4) x 1 x 8 box of the state at (i0-2, j0-2, k, 0)
// lands in the staging buffer as [variable][y][x]; its completion is counted on an mbarrier.
// Coordinates outside the grid read zeros (the boundary rules are applied when the plane is
// converted); x = i0 - 2 is even, so the copy starts on a 16-byte boundary.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Non-blocking probe of phase `parity` of the barrier.
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier for at most `limit` SM cycles (0: kCopyWaitCycles,
// < 0: one non-blocking check); false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long limit) {
    if (limit < 0) return mbar_test_wait(bar, parity);
    if (limit == 0) limit = kCopyWaitCycles;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Issued by one thread: expects `bytes` on the barrier and starts the copy.  The caller has
// ordered earlier generic-proxy reads of `dst` before this (barrier + proxy fence).
__device__ __forceinline__ void tma_plane(void* dst, const CUtensorMap* tm, int x, int y, int z, unsigned bytes,
                                          unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
        : "memory");
}

// Primitive plane with the boundary rules from a staged box (conserved, [v][y][x] with row HX):
// inflow beyond x = hi, zero-gradient (clamped index, always inside the box) elsewhere.
template <int P, int SK, typename RT>
__device__ __forceinline__ void convert_plane(const StageArgs& A, const double* stg, RT* dst, int i0, int j0) {
    constexpr int HX = Tile<P, SK>::HX, PLANE = Tile<P, SK>::PLANE, NT = Tile<P, SK>::NT;
    const GridGeom& g = A.g;
    for (int c = threadIdx.x; c < PLANE; c += NT) {
        const int cx = c % HX, cy = c / HX;
        const int i = i0 - 2 + cx, j = j0 - 2 + cy;
        double q[8];
        if (i >= g.nx) {
            inflow_prim<P == 0>(g, q);
        } else {
            const int sx = max(i, 0) - (i0 - 2), sy = min(max(j, 0), g.ny - 1) - (j0 - 2);
            const double* src = stg + sy * HX + sx;
            double U[8];
#pragma unroll
            for (int v = 0; v < 8; v++) U[v] = src[v * PLANE];
            if constexpr (P == 1) {
                double ke, me;
                prim_from_cons<false, false>(U, q, ke, me);
            } else {
                prim_from_cons_guarded<P == 0>(U, q);
            }
        }
#pragma unroll
        for (int v = 0; v < 8; v++) dst[v * PLANE + c] = (RT)q[v];
    }
}

// Face-frame order (normal, t1, t2) of the components of a face normal to axis AX: entry v of
// the face-frame state is natural component face_perm<AX>(v) of (rho, u, v, w, p, Bx, By, Bz).
template <int AX> __host__ __device__ constexpr int face_perm(int v) {
    return (v == 0 || v == 4) ? v
           : (v < 4 ? 0 : 4) + ((v & 3) == 1 ? 1 + AX : ((v & 3) == 2 ? (AX == 0 ? 2 : 1) : (AX == 2 ? 2 : 3)));
}

// face_perm<AX>(v) for an axis known only at run time (the rare FP64 recompute path).
__device__ __forceinline__ int face_perm_dyn(int axis, int v) {
    return axis == 0 ? face_perm<0>(v) : (axis == 1 ? face_perm<1>(v) : face_perm<2>(v));
}

// Face-frame states of the 4-cell stencil of a face normal to AX, from ring cells (component
// planes PLANE apart).  B is first order, so only the inner pair carries it.
template <int AX, int PLANE, typename RG, typename RT>
__device__ __forceinline__ void gather_face(const RG* pLL, const RG* pL, const RG* pR, const RG* pRR, RT* qLL,
                                            RT* qL, RT* qR, RT* qRR) {
#pragma unroll
    for (int v = 0; v < 8; v++) {
        const int o = face_perm<AX>(v) * PLANE;
        qL[v] = (RT)pL[o];
        qR[v] = (RT)pR[o];
        qLL[v] = v < 5 ? (RT)pLL[o] : RT(0);
        qRR[v] = v < 5 ? (RT)pRR[o] : RT(0);
    }
}

// Face-frame flux times the face area into natural component order, components STRIDE apart.
template <int AX, int STRIDE, typename FT, typename RT>
__device__ __forceinline__ void scatter_face(FT* out, const RT* F, RT sq) {
#pragma unroll
    for (int v = 0; v < 8; v++) out[face_perm<AX>(v) * STRIDE] = (FT)(F[v] * sq);
}

// What the out-of-line FP64 recompute of a face needs, passed by value: a reference or pointer to
// the kernel's arguments would make the compiler copy them to local memory and read every field
// from there on the hot path.
struct FetchArgs {
    const double* Uin;
    long long vs, ps, px;
    int nx, ny, nz, n_disc;
    double inflow[8];
};
struct FaceFlux {
    double F[8];   // natural component order
    double sl, sr;
    int fl;
};

__device__ __forceinline__ FetchArgs fetch_args(const StageArgs& A) {
    FetchArgs f;
    f.Uin = A.Uin;
    f.vs = A.g.vs;
    f.ps = A.g.ps;
    f.px = A.g.px;
    f.nx = A.g.nx;
    f.ny = A.g.ny;
    f.nz = A.g.nz;
    f.n_disc = A.n_disc;
#pragma unroll
    for (int v = 0; v < 8; v++) f.inflow[v] = A.g.inflow[v];
    return f;
}

// FP64 primitive state of global cell (i,j,k), boundary rules as fetch_prim64.
__device__ __forceinline__ void fetch_prim64_f(const FetchArgs& f, int i, int j, int k, double* q) {
    if (i >= f.nx) {
#pragma unroll
        for (int v = 0; v < 8; v++) q[v] = f.inflow[v];
        return;
    }
    i = max(i, 0);
    j = min(max(j, 0), f.ny - 1);
    k = min(max(k, 0), f.nz - 1);
    const long long off = (long long)k * f.ps + (long long)j * f.px + i;
    double U[8];
#pragma unroll
    for (int v = 0; v < 8; v++) U[v] = __ldg(f.Uin + v * f.vs + off);
    double ke, me;
    prim_from_cons(U, q, ke, me);
}

// The FP64 recompute of one face of the mixed and delta forms from the FP64 state (rare path;
// kept out of line so the main path keeps its registers), with the library special functions.
// (i, j, k) is the cell on the high side of the face.
template <int NSTATE, int ORDER>
__device__ __noinline__ FaceFlux face_fp64(const FetchArgs fa, int axis, int i, int j, int k) {
    const int di = axis == 0, dj = axis == 1, dk = axis == 2;
    double c[4][8];
    fetch_prim64_f(fa, i - 2 * di, j - 2 * dj, k - 2 * dk, c[0]);
    fetch_prim64_f(fa, i - di, j - dj, k - dk, c[1]);
    fetch_prim64_f(fa, i, j, k, c[2]);
    fetch_prim64_f(fa, i + di, j + dj, k + dk, c[3]);
    const int pn = 1 + axis, pt1 = axis == 0 ? 2 : 1, pt2 = axis == 2 ? 2 : 3;
    const int perm[8] = {0, pn, pt1, pt2, 4, 4 + pn, 4 + pt1, 4 + pt2};
    double f[4][8];
    for (int s = 0; s < 4; s++)
        for (int v = 0; v < 8; v++) f[s][v] = c[s][perm[v]];
    double q1[8], q2[8], G[8], SM;
    reconstruct<double, ORDER>(f[0], f[1], f[2], f[3], q1, q2);
    FaceFlux r;
    r.fl = riemann<double, NSTATE, false, false, false, false, false>(q1, q2, 0.0, fa.n_disc, G, r.sl, r.sr, SM);
    for (int v = 0; v < 8; v++) r.F[perm[v]] = G[v];
    return r;
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
    using Ring = float;
    using Flux = float;
    using Math = float;
};

// `n_waits` counts the completed phases of `bar` and `tma_dead` is set once a plane copy did not
// land within both bounded waits (the thread then reads its planes with plain loads); both are
// per thread and carried across the tiles a CTA runs.
template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT, int SK>
__device__ __forceinline__ void run_tile(const StageArgs& A, int bx, int by, int bz, unsigned total_tiles,
                                         unsigned long long* bar, unsigned& n_waits, bool& tma_dead) {
    using RG = typename Types<P>::Ring;
    using FT = typename Types<P>::Flux;
    using RT = typename Types<P>::Math;
    using C = Tile<P, SK>;
    constexpr int TX = C::TX, TY = C::TY, NC = C::NC, NT = C::NT, HX = C::HX, PLANE = C::PLANE;
    constexpr int NXF = C::NXF, NYF = C::NYF;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // [8][PLANE] staged conserved box; tensor copies land on a 128-byte aligned address.  The
    // alignment pad is an offset from the shared array itself, so every pointer below stays in
    // the shared address space (shared loads and stores with 32-bit addresses, not generic ones).
    const unsigned pad = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
    double* stg = reinterpret_cast<double*>(smem_raw + pad);
    RG* ring = reinterpret_cast<RG*>(stg + 8 * PLANE);
    FT* fx = reinterpret_cast<FT*>(ring + RING * 8 * PLANE);   // [8][NXF]
    FT* fy = fx + 8 * NXF;                                      // [8][NYF]
    __shared__ double red[NT / 32];
    __shared__ unsigned long long cnt[6];
    __shared__ bool last_cta;

    const GridGeom& g = A.g;
    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int i0 = bx * TX, j0 = by * TY;
    const int kb = plane_begin(g), ke = plane_end(g);
    const int k0 = kb + bz * g.lz;
    const int k1 = min(ke, k0 + g.lz);
    const double dt = A.clk->dt_cur;
    const double dt_vol = dt * g.inv_vol;   // dt / cell volume
    if (t < 6) cnt[t] = 0;

    double rate = 0.0;   // max over this thread's real faces of max(|SL|,|SR|)/dist
    unsigned n_recon = 0, n_wave = 0, n_redo = 0, n_tmo = 0;

    // Faces are handed out in warp-sized jobs, so the face axis is uniform across a warp and the
    // face-frame permutation of the components is a compile-time constant of the gather and the
    // scatter (face_perm):
    //   jobs [0, TY)         z faces k+1/2 of tile row `job`, column = lane;
    //   jobs [TY, 2TY)       x faces i-1/2 of tile row `job - TY`, column = lane;
    //   job  2TY             the east x faces (column TX) of tile rows 0 .. TY-1, row = lane;
    //   jobs [2TY+1, 3TY+2)  y faces j-1/2 of tile row `job - 2TY - 1` (TY+1 rows), column = lane.
    // Warp w runs jobs w, w + NW, ...; z job w (round 0) is run by the threads owning the cells of
    // tile row w in the update.  A z flux goes into the ring slot of plane k-1 at its column:
    // only the same thread reads that location in this plane (as the z face's far-left cell), and
    // it reads the flux back before the barrier that precedes the next plane load.  x and y
    // fluxes go to fx / fy.
    // `dup`: the face is also computed by the CTA below (chunk-boundary z face); it still enters
    // the dt candidate (min is idempotent) but not the diagnostic counters.
    static_assert(std::is_same<RG, FT>::value, "z fluxes reuse the ring");
    constexpr int NW = NT / 32;
    constexpr int JZ = TY, JX = 2 * TY + 1, JOBS = 3 * TY + 2;
    static_assert(TY <= NW, "z jobs run in the first round, by the owners of their cells");
    const int lane = t & 31, warp = t >> 5;
    auto do_face = [&](int job, int k, bool dup) {
        int axis, fxx, fyy, gk, oidx, ostride;
        double sq, idist;   // face area and 1/dist of the axis (compile-time index per branch)
        FT* out;
        bool real;
        RT qLL[8], qL[8], qR[8], qRR[8];
        if (job < JZ) {
            axis = 2;
            sq = g.square[2];
            idist = g.inv_dist[2];
            fxx = lane;
            fyy = job;
            const int c = (fyy + 2) * HX + fxx + 2;
            gather_face<2, PLANE>(ring + ring_slot(k - 1) * 8 * PLANE + c, ring + ring_slot(k) * 8 * PLANE + c,
                                  ring + ring_slot(k + 1) * 8 * PLANE + c, ring + ring_slot(k + 2) * 8 * PLANE + c,
                                  qLL, qL, qR, qRR);
            out = ring + ring_slot(k - 1) * 8 * PLANE;
            oidx = c;
            ostride = PLANE;
            gk = k + 1;
            real = (i0 + fxx < g.nx) && (j0 + fyy < g.ny) && (k + 1 <= ke) && (k + 1 >= kb);
        } else if (job < JX) {
            axis = 0;
            sq = g.square[0];
            idist = g.inv_dist[0];
            if (job < 2 * TY) {
                fxx = lane;
                fyy = job - JZ;
            } else {
                if (lane >= TY) return;
                fxx = TX;
                fyy = lane;
            }
            const int c = (fyy + 2) * HX + fxx;   // cell fxx-2 (tile-local) at halo offset +2
            const RG* b = ring + ring_slot(k) * 8 * PLANE + c;
            gather_face<0, PLANE>(b, b + 1, b + 2, b + 3, qLL, qL, qR, qRR);
            out = fx;
            oidx = fyy * (TX + 1) + fxx;
            ostride = NXF;
            gk = k;
            real = (i0 + fxx <= g.nx) && (j0 + fyy < g.ny);
        } else {
            axis = 1;
            sq = g.square[1];
            idist = g.inv_dist[1];
            fxx = lane;
            fyy = job - JX;
            const int c = fyy * HX + fxx + 2;     // row fyy-2 (tile-local)
            const RG* b = ring + ring_slot(k) * 8 * PLANE + c;
            gather_face<1, PLANE>(b, b + HX, b + 2 * HX, b + 3 * HX, qLL, qL, qR, qRR);
            out = fy;
            oidx = fyy * TX + fxx;
            ostride = NYF;
            gk = k;
            real = (i0 + fxx < g.nx) && (j0 + fyy <= g.ny);
        }
        RT q1[8], q2[8], F[8];
        if constexpr (P == 1 && ORDER == 2) reconstruct_f32x2(qLL, qL, qR, qRR, q1, q2);
        else reconstruct<RT, ORDER>(qLL, qL, qR, qRR, q1, q2);
        if (real && !dup && (sb_neg(q1[0]) || sb_neg(q2[0]))) n_recon++;
        int fl;
        double sl, sr;
        if constexpr (P == 2) {
            float SLf, SRf, SMf;
            fl = riemann_delta<NSTATE>(q1, q2, F, SLf, SRf, SMf);
            sl = (double)SLf;
            sr = (double)SRf;
            if (fl & kFlagStar) {   // the same face states, refetched: FP64 throughout
                const FaceFlux r = face_fp64<NSTATE, ORDER>(fetch_args(A), axis, i0 + fxx, j0 + fyy, gk);
                fl = r.fl;
                sl = r.sl;
                sr = r.sr;
#pragma unroll
                for (int v = 0; v < 8; v++) F[v] = r.F[face_perm_dyn(axis, v)];
                if (real && !dup) n_redo++;
            }
        } else {
            RT SL, SR, SM;
            if constexpr (P == 1 && NSTATE >= 2) {
                if (A.n_disc == 0)
                    fl = riemann_f32x2<NSTATE>(q1, q2, F, SL, SR, SM);
                else
                    fl = riemann<RT, NSTATE, false, true, true, false, false>(q1, q2, RT(0), A.n_disc, F, SL, SR, SM);
            } else {
                // the plain form's ring holds b = B / sqrt(4 pi) (BS)
                fl = riemann<RT, NSTATE, false, P == 1, true, P == 0>(q1, q2, RT(0), A.n_disc, F, SL, SR, SM);
            }
            sl = (double)SL;
            sr = (double)SR;
        }

        if (P == 1 && real && (fl & kFlagStar)) {
            const FaceFlux r = face_fp64<NSTATE, ORDER>(fetch_args(A), axis, i0 + fxx, j0 + fyy, gk);
            fl = r.fl;
            sl = r.sl;
            sr = r.sr;
            if (!dup) n_redo++;
#pragma unroll
            for (int v = 0; v < 8; v++) out[v * ostride + oidx] = (FT)(r.F[v] * sq);
        } else {
            // a face no wave-fan region matched gets a zero flux; the warp vote keeps the (never
            // taken in a valid state) zeroing out of the common path
            if (__any_sync(__activemask(), fl & kFlagWave) && (fl & kFlagWave)) {
#pragma unroll
                for (int v = 0; v < 8; v++) F[v] = RT(0);
            }
            if (axis == 2) scatter_face<2, PLANE>(out + oidx, F, (RT)sq);
            else if (axis == 0) scatter_face<0, NXF>(out + oidx, F, (RT)sq);
            else scatter_face<1, NYF>(out + oidx, F, (RT)sq);
        }
        if ((fl & kFlagWave) && real && !dup) n_wave++;
        // compare-and-select maxima (the library fmax of doubles is a far longer sequence); a NaN
        // speed is skipped, as fmax would skip it
        if (WANT_DT && real) rate = sb_max(rate, sb_max(fabs(sl), fabs(sr)) * idist);
    };

    // ---- the march over planes kk = k0-2 .. k1+1.  Plane kk enters ring slot kk; from
    // kk = k0+1 on, iteration k = kk-2 computes the faces of plane k and (from k = k0) updates
    // it.  Iteration k0-1 is the prologue: only the z face k0-1/2 (carried into the first
    // update).  Every face goes through the one do_face call site below, so a face's arithmetic
    // does not depend on where a chunk starts.  With a tensor map, the copy of plane kk+1 is in
    // flight while plane kk's faces and updates run; the last copy issued is plane k1+1.
    const bool use_tma = A.tm_in != nullptr && !tma_dead;
    constexpr unsigned kPlaneBytes = 8u * PLANE * sizeof(double);
    const int kz_last = k1 + 1;
    auto issue_copy = [&](int kk) {
        tma_plane(stg, A.tm_in, i0 - 2, j0 - 2, min(max(kk, 0), g.nz - 1), kPlaneBytes, bar);
    };
    if (use_tma && t == 0) issue_copy(k0 - 2);
    FT fzl[8];       // z fluxes k-1/2 (carried) and k+1/2 of this thread's column
    // centre of this thread's column and its part of the source-sphere test
    const double cxs = cell_coord(g.lo[0], i0 + tx, g.h[0]), cys = cell_coord(g.lo[1], j0 + ty, g.h[1]);
    const double xy2 = dadd(dmul(cxs, cxs), dmul(cys, cys));
    const double rsrc2 = dmul(g.r_src, g.r_src);
    const bool col_src = g.r_src > 0.0 && xy2 < rsrc2;
    const int gi = i0 + tx, gj = j0 + ty;
    const bool own = (t < NC) && (gi < g.nx) && (gj < g.ny);
    for (int kk = k0 - 2; kk <= kz_last; kk++) {
        RG* slot = ring + ring_slot(kk) * 8 * PLANE;
        if (use_tma && !tma_dead) {
            // A wait that runs out is counted (SETB_ETIMEOUT), then the copy gets a second bounded
            // wait to land before the box is read; a copy that never lands switches this thread to
            // plain loads (and thread 0 stops issuing copies), so no read races a late copy.
            bool ok = mbar_wait_bounded(bar, n_waits & 1u, A.copy_wait);
            if (!ok) {
                n_tmo++;
                ok = mbar_wait_bounded(bar, n_waits & 1u, kCopyWaitCycles);
            }
            n_waits++;
            if (ok) convert_plane<P, SK, RG>(A, stg, slot, i0, j0);
            else tma_dead = true;
        }
        if (!use_tma || tma_dead) load_plane<P, SK, RG>(A, slot, i0, j0, kk);
        __syncthreads();
        if (use_tma && !tma_dead && t == 0 && kk < kz_last) issue_copy(kk + 1);
        const int k = kk - 2;
        if (k < k0 - 1) continue;
        const bool pro = (k < k0);
        const int njobs = pro ? JZ : JOBS;
        for (int job = warp; job < njobs; job += NW) do_face(job, k, pro && k0 > kb);
        FT fzh[8];
        {
            const RG* zk = ring + ring_slot(k - 1) * 8 * PLANE + (ty + 2) * HX + tx + 2;
#pragma unroll
            for (int v = 0; v < 8; v++) fzh[v] = t < NC ? zk[v * PLANE] : FT(0);
        }
        __syncthreads();
        if (pro) {
#pragma unroll
            for (int v = 0; v < 8; v++) fzl[v] = fzh[v];
            continue;
        }
        // The plain form's Heun stage 2 streams its base state U^n from HBM, which no plane copy
        // has touched: ask L2 for the next plane's cells now, so their loads one iteration later
        // hit L2 instead of waiting on DRAM (stage 2 at 256^3: 2.78 -> 2.74 ms; the same hint in
        // the mixed form, for U^n and its compensation, measured 1-2 % slower).
        if (P == 0 && KIND == 1 && own && k + 1 < k1) {
            const long long offn = (long long)(k + 1) * g.ps + (long long)gj * g.px + gi;
#pragma unroll
            for (int v = 0; v < 8; v++) asm volatile("prefetch.global.L2 [%0];" ::"l"(A.Ubase + v * g.vs + offn));
        }
        if (own) {
            const long long off = (long long)k * g.ps + (long long)gj * g.px + gi;
            double un[8], qs[8];
            bool reset_comp = false;
            bool is_src = false;
            if (col_src) {   // (x^2 + y^2) + z^2 < r_src^2, rounded as in source_prim
                const double cz = cell_coord(g.lo[2], k + g.koff, g.h[2]);
                const double r2 = dadd(xy2, dmul(cz, cz));
                if (r2 < rsrc2) {
                    source_state(g, cxs, cys, cz, r2, qs);
                    is_src = true;
                }
            }
            if (is_src) {
                cons_from_prim_exact(qs, un);
                reset_comp = true;
            } else {
                double uin[8], cmp[8];
#pragma unroll
                for (int v = 0; v < 8; v++) {
                    double pot;
                    if constexpr (P == 1) {
                        // FP32 fluxes: each opposite-face difference is exact when the two fluxes
                        // are within a factor 2 (Sterbenz) and otherwise rounds relative to the
                        // difference, far below the fluxes' own FP32 rounding; one conversion
                        // per variable instead of six
                        const float ax = fx[v * NXF + ty * (TX + 1) + tx + 1] - fx[v * NXF + ty * (TX + 1) + tx];
                        const float ay = fy[v * NYF + (ty + 1) * TX + tx] - fy[v * NYF + ty * TX + tx];
                        pot = (double)((ax + ay) + (fzh[v] - fzl[v]));
                    } else {
                        // the oracle's sum from zero, 0 - a + b - ...: (0 - a) + b equals b - a
                        // bit for bit, zero signs included
                        pot = (double)fx[v * NXF + ty * (TX + 1) + tx + 1] - (double)fx[v * NXF + ty * (TX + 1) + tx];
                        pot = pot - (double)fy[v * NYF + ty * TX + tx];
                        pot = pot + (double)fy[v * NYF + (ty + 1) * TX + tx];
                        pot = pot - (double)fzl[v];
                        pot = pot + (double)fzh[v];
                    }
                    uin[v] = A.Uin[v * g.vs + off];
                    const double inc = pot * dt_vol;
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
                    atomicMin(&A.st->first_bad,
                              (unsigned long long)(gi + (long long)g.nx * (gj + (long long)g.ny * (k + g.koff))));
#pragma unroll
                    for (int v = 0; v < 8; v++) un[v] = uin[v];
                    reset_comp = true;
                } else if (P == 1 || !pressure_surely_positive(un)) {
                    // the exact recovery (P != 1) only where the quick test cannot clear p > 0
                    double q[8], ke, me;
                    prim_from_cons<P != 1>(un, q, ke, me);
                    if (q[4] <= 0.0) {                    // cuf_solvers.cuf:777-779
                        atomicAdd(&cnt[1], 1ull);
                        un[4] = floor_energy(ke, me);
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
    if (n_tmo) atomicAdd(&cnt[5], (unsigned long long)n_tmo);
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
        if (cnt[5]) atomicAdd(&A.st->n_timeout, cnt[5]);
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
__global__ void __launch_bounds__(Tile<P, KIND>::NT, Tile<P, KIND>::MINB) stage_kernel(const StageArgs A) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar);
    __syncthreads();
    unsigned n_waits = 0;
    bool tma_dead = false;
    run_tile<P, NSTATE, ORDER, KIND, WANT_DT, KIND>(A, blockIdx.x, blockIdx.y, blockIdx.z,
                                                     gridDim.x * gridDim.y * gridDim.z, &bar, n_waits, tma_dead);
}

// Persistent batch kernel: each CTA takes tiles from the work queue until it is empty; the
// tile's solve selects the arguments (copied to shared memory).  One launch covers the solves of
// one Riemann solver (NSTATE), so the kernel holds one solver body.  The items of one solve are
// counted by its own clock, so every solve keeps its own lagged dt.
template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT>
__global__ void __launch_bounds__(Tile<P, kBatchKind>::NT, Tile<P, kBatchKind>::MINB) batch_stage_kernel(const BatchArgs B) {
    __shared__ __align__(16) StageArgs As;
    __shared__ int4 it;
    __shared__ __align__(8) unsigned long long bar;
    constexpr int WORDS = sizeof(StageArgs) / sizeof(unsigned long long);
    static_assert(sizeof(StageArgs) % sizeof(unsigned long long) == 0, "StageArgs must be 8-byte granular");
    if (threadIdx.x == 0) mbar_init(&bar);
    unsigned n_waits = 0;   // completed phases of `bar`, the same count in every thread
    bool tma_dead = false;
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
        for (int q = threadIdx.x; q < WORDS; q += Tile<P, kBatchKind>::NT) dst[q] = src[q];
        __syncthreads();
        run_tile<P, NSTATE, ORDER, KIND, WANT_DT, kBatchKind>(As, w.y, w.z, w.w, As.total_tiles, &bar, n_waits,
                                                              tma_dead);
    }
}

// Dynamic shared memory: alignment slack, staged box (FP64), primitive ring, x / y flux buffers.
template <int P, int SK>
constexpr int smem_bytes() {
    using C = Tile<P, SK>;
    return 128 + 8 * C::PLANE * (int)sizeof(double) + RING * 8 * C::PLANE * (int)sizeof(typename Types<P>::Ring) +
           8 * (C::NXF + C::NYF) * (int)sizeof(typename Types<P>::Flux);
}

template <int P, int NSTATE, int ORDER, int KIND, bool WANT_DT>
cudaError_t launch_t(const StageArgs& a, cudaStream_t s) {
    auto kern = stage_kernel<P, NSTATE, ORDER, KIND, WANT_DT>;
    const int smem = smem_bytes<P, KIND>();
    // The dynamic shared-memory opt-in is a per-device attribute of the kernel: set it once per
    // device ordinal (a bit per device, atomically; two threads that both set it set the same
    // value), and on every launch for ordinals beyond the mask.
    static std::atomic<unsigned long long> attr_set{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!bit || !(attr_set.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(bit, std::memory_order_release);
    }
    constexpr int TX = Tile<P, KIND>::TX, TY = Tile<P, KIND>::TY;
    const int nzu = plane_end(a.g) - plane_begin(a.g);
    dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, (nzu + a.g.lz - 1) / a.g.lz);
    kern<<<grid, Tile<P, KIND>::NT, smem, s>>>(a);
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
    cudaError_t e = cudaFuncSetAttribute(batch_stage_kernel<P, 3, 2, KIND, WANT_DT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes<P, kBatchKind>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(batch_stage_kernel<P, 2, 2, KIND, WANT_DT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_bytes<P, kBatchKind>());
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

int batch_ctas_per_sm(int precision) { return tile_shape(precision, kBatchKind).ctas_per_sm; }

template <int P, int NSTATE>
void launch_batch_pn(const BatchArgs& b, int kind, bool want_dt, int grid, cudaStream_t s) {
    constexpr int NT = Tile<P, kBatchKind>::NT;
    if (kind == 0 && want_dt) batch_stage_kernel<P, NSTATE, 2, 0, true><<<grid, NT, smem_bytes<P, kBatchKind>(), s>>>(b);
    else batch_stage_kernel<P, NSTATE, 2, 1, false><<<grid, NT, smem_bytes<P, kBatchKind>(), s>>>(b);
}

template <int P>
void launch_batch_p(const BatchArgs& b, int n_state, int kind, bool want_dt, int grid, cudaStream_t s) {
    if (n_state == 3) launch_batch_pn<P, 3>(b, kind, want_dt, grid, s);
    else launch_batch_pn<P, 2>(b, kind, want_dt, grid, s);
}

cudaError_t launch_batch_stage(const BatchArgs& b, int precision, int n_state, int kind, bool want_dt, int grid,
                               cudaStream_t s) {
    if (precision == 1) launch_batch_p<1>(b, n_state, kind, want_dt, grid, s);
    else if (precision == 2) launch_batch_p<2>(b, n_state, kind, want_dt, grid, s);
    else launch_batch_p<0>(b, n_state, kind, want_dt, grid, s);
    return cudaGetLastError();
}

int stage_smem_bytes(int precision, int kind) {
    if (precision == 1) return kind == 0 ? smem_bytes<1, 0>() : smem_bytes<1, 1>();
    return precision == 2 ? smem_bytes<2, 0>() : smem_bytes<0, 0>();
}
int stage_fp64_smem_bytes() { return smem_bytes<0, 0>(); }

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
