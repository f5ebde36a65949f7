// setb_internal.cuh -- device-side structures shared by the stage kernels and the host runtime.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "mhd_core.cuh"
#include "setb200.h"

namespace sb {

// Clock of one solve, in device memory.  The reference keeps time_step / time_step2 /
// dev_time_all as device scalars written from the host each step (cuf_kernel.cuf:18-19,
// 789-794); here the last CTA of each step's final kernel rolls the clock on the device, so a
// run of steps needs no host round trip.
// Column tile of the stage kernels: kTileX x ty cells marched along z by `threads` threads,
// `ctas_per_sm` resident per SM; per form (precision 0 plain FP64, 1 mixed, 2 delta) and launch
// (kind 0: Euler step / Heun stage 1; kind 1: Heun stage 2 and every batch launch).  The plain
// and delta forms fit FP64 HLLD in 168 registers (384 threads, 12 warps per SM).  The mixed
// form's first stage runs that shape too; its second stage, which also streams the FP32
// compensation, runs two 256-thread CTAs of at most 128 registers, so one CTA's update overlaps
// the other's faces.
constexpr int kTileX = 32;
struct TileShape {
    int ty, threads, ctas_per_sm;
};
SB_HD constexpr TileShape tile_shape(int precision, int kind) {
    return (precision == 1 && kind == 1) ? TileShape{7, 256, 2} : TileShape{11, 384, 1};
}
// The tile_shape kind every batch launch uses.  The batch kernel holds the HLLC and HLLD bodies;
// in the mixed form the kind-1 shape (two 256-thread CTAs per SM, 128 registers, ~320 B of
// spills) measured 1.5 % faster on the 64-grid ensemble than the kind-0 shape (one 384-thread
// CTA, 168 registers, ~80 B of spills).
constexpr int kBatchKind = 1;

struct DevClock {
    double dt_cur;                  // dt used by the current step (time_step)
    unsigned long long dt_next;     // bits of the running min for the next step (time_step2)
    double time_all;                // dev_time_all
    double dt_last;                 // dt used by the previous step
    unsigned int counter;           // CTAs finished in the running kernel
    unsigned int pad;
    long long steps;
};

struct DevStatus {
    unsigned long long n_negdens, n_pfloor, n_wave, n_recon, n_redo;
    unsigned long long first_bad;   // ULLONG_MAX when none
    unsigned long long n_timeout;   // bounded waits on a plane copy that gave up
};

// Geometry + boundary data of one Cartesian grid.
struct GridGeom {
    int nx, ny, nz, lz;             // lz: z extent of one CTA's march
    int kb, ke, koff;               // z slab: the stage kernels update planes [kb, ke) of the nz
                                    // held (ke = 0: all nz), the others are ghost planes filled by
                                    // the caller; buffer plane k is plane k + koff of the whole
                                    // grid (source-sphere geometry, first-bad-cell index)
    long long vs, ps, px;           // var / plane / row strides of the SoA state (elements);
                                    // device-owned states keep px even and vs a multiple of 32
                                    // (16-byte rows for the tensor copies, 256-byte planes)
    double lo[3], h[3];
    double square[3];               // face areas: hy*hz, hx*hz, hx*hy
    double inv_vol;                 // 1/(hx*hy*hz)
    double inv_dist[3];             // 1/(h/2)
    double inflow[8];               // primitive ghost state beyond x = hi
    double r_src, rho_src, v_src, p_over_rho_src, r_floor;
};

// Scoped NVTX range on the host (header-only NVTX3: a no-op unless a profiler or tracer attaches),
// named after the C entry point, so timelines and ncu --nvtx filters show the library's calls.
struct NvtxRange {
    explicit NvtxRange(const char* name);
    ~NvtxRange();
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Ghost planes on each side of a z slab (the reconstruction stencil reaches two planes).
constexpr int kSlabGhost = 2;
// Updated plane range [kb, ke) of a geometry.
SB_HD int plane_begin(const GridGeom& g) { return g.kb; }
SB_HD int plane_end(const GridGeom& g) { return g.ke > 0 ? g.ke : g.nz; }

struct StageArgs {
    GridGeom g;
    const double* __restrict__ Uin;     // state the fluxes are computed from
    const double* Ubase;                // stage 2: U^n (may alias Uout: read before written, same thread)
    double* Uout;
    DevClock* clk;
    DevStatus* st;
    double cfl;
    int n_disc;
    int finalize;                       // last CTA rolls the clock (Euler, or Heun stage 2)
    float* comp;                        // mixed form: FP32 compensation of the compensated update
                                        // (Euler / Heun stage 2); null = plain update
    unsigned total_tiles;               // batch: tiles of this solve in the launch
    int n_state;                        // batch: per-solve Riemann solver (2 HLLC, 3 HLLD)
    const CUtensorMap* tm_in;           // tensor map of Uin (device memory) for the plane
                                        // copies, box (kTileX + 4, ty + 4, 1, 8) of this form's
                                        // tile; null = planes read with plain loads
    long long copy_wait;                // limit of the first wait for a plane copy, in SM cycles:
                                        // 0 = kCopyWaitCycles, < 0 = one non-blocking check
                                        // (setb_set_copy_wait; tests of the timeout path)
};

// Default limit of a bounded wait on a plane copy (~2 s at 1.965 GHz), and of the second wait
// that lets a late copy land after the first one ran out.
constexpr long long kCopyWaitCycles = 4000000000ll;

// Host-side argument checks shared by every entry point that takes a grid or scheme options
// (capi.cu): SETB_OK or the status to return.
int validate_desc(const setb_cart_desc* d);
int validate_opts(const setb_step_opts* o);
// z extent of one CTA's march for a grid on sm_count SMs (capi.cu).
int choose_lz(const GridGeom& g, int sm_count, int precision, int kind);

// One launch of the batch kernel: tiles of many solves behind one work-queue counter.
struct BatchArgs {
    const StageArgs* inst;              // per-slot arguments of this stage (device array)
    const int4* items;                  // work list: (slot, bx, by, bz), largest solves first
    int n_items;
    unsigned* queue;                    // next item to hand out (zeroed before the launch)
};

// Geometry of cell centres, evaluated with explicitly rounded operations so that host, device
// and every kernel agree bit for bit (FMA contraction would change the source-sphere test).
SB_HD double cell_coord(double lo, int i, double h) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(lo, __dmul_rn((double)i + 0.5, h));
#else
    return lo + ((double)i + 0.5) * h;
#endif
}
SB_HD double dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
SB_HD double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
SB_HD double dsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

// Conserved state from a primitive one, exactly rounded (no contraction): used for initial
// conditions, the re-imposed source state and Cell_par uploads.
SB_HD void cons_from_prim_exact(const double* q, double* U) {
    const double rho = q[0], u = q[1], v = q[2], w = q[3];
    const double bx = q[5] / kSpi4, by = q[6] / kSpi4, bz = q[7] / kSpi4;
    const double ke = dmul(dmul(0.5, rho), dadd(dadd(dmul(u, u), dmul(v, v)), dmul(w, w)));
    const double me = dmul(0.5, dadd(dadd(dmul(bx, bx), dmul(by, by)), dmul(bz, bz)));
    U[0] = rho;
    U[1] = dmul(rho, u);
    U[2] = dmul(rho, v);
    U[3] = dmul(rho, w);
    U[4] = dadd(dadd(q[4] / kG1, ke), me);
    U[5] = q[5];
    U[6] = q[6];
    U[7] = q[7];
}

// Primitive state from a conserved one, exactly rounded with true divisions (Cell_par downloads).
SB_HD void prim_from_cons_exact(const double* U, double* q) {
    const double rho = U[0];
    const double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
    const double bx = U[5] / kSpi4, by = U[6] / kSpi4, bz = U[7] / kSpi4;
    const double ke = dmul(dmul(0.5, rho), dadd(dadd(dmul(u, u), dmul(v, v)), dmul(w, w)));
    const double me = dmul(0.5, dadd(dadd(dmul(bx, bx), dmul(by, by)), dmul(bz, bz)));
    q[0] = rho;
    q[1] = u;
    q[2] = v;
    q[3] = w;
    q[4] = dmul(dsub(dsub(U[4], ke), me), kG1);
    q[5] = U[5];
    q[6] = U[6];
    q[7] = U[7];
}

// Source state (primitive) at cell (i,j,k); false when the cell is outside r_src.
// Source state at centre (x, y, z) with r2 = (x^2 + y^2) + z^2 already below r_src^2.
SB_HD void source_state(const GridGeom& g, double x, double y, double z, double r2, double* q) {
    const double r = sqrt(r2);
    const double re = r > g.r_floor ? r : g.r_floor;
    const double s = g.r_src / re;
    const double rho = dmul(dmul(s, s), g.rho_src);
    q[0] = rho;
    if (r > 0.0) {
        q[1] = dmul(g.v_src, x / r);
        q[2] = dmul(g.v_src, y / r);
        q[3] = dmul(g.v_src, z / r);
    } else {
        q[1] = q[2] = q[3] = 0.0;
    }
    q[4] = dmul(g.p_over_rho_src, rho);
    q[5] = q[6] = q[7] = 0.0;
}

SB_HD bool source_prim(const GridGeom& g, int i, int j, int k, double* q) {
    if (!(g.r_src > 0.0)) return false;
    const double x = cell_coord(g.lo[0], i, g.h[0]);
    const double y = cell_coord(g.lo[1], j, g.h[1]);
    const double z = cell_coord(g.lo[2], k, g.h[2]);
    const double r2 = dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
    if (!(r2 < dmul(g.r_src, g.r_src))) return false;
    source_state(g, x, y, z, r2, q);
    return true;
}

SB_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
SB_HD double unit_draw(uint64_t seed, uint64_t cell, uint64_t which) {
    const uint64_t hsh = splitmix64(splitmix64(seed) ^ (2 * cell + which));
    return dmul((double)(hsh >> 11), 1.0 / 9007199254740992.0);
}

// Seeded initial condition of one cell (primitive).
SB_HD void lism_prim(const GridGeom& g, const double* lism, uint64_t seed, double pert, int i, int j,
                     int k, double* q) {
    if (!source_prim(g, i, j, k, q)) {
        const uint64_t c = (uint64_t)i + (uint64_t)g.nx * ((uint64_t)j + (uint64_t)g.ny * (uint64_t)k);
        const double d1 = dmul(pert, dsub(dmul(2.0, unit_draw(seed, c, 0)), 1.0));
        const double d2 = dmul(pert, dsub(dmul(2.0, unit_draw(seed, c, 1)), 1.0));
        q[0] = dmul(lism[0], dadd(1.0, d1));
        q[1] = lism[1];
        q[2] = lism[2];
        q[3] = lism[3];
        q[4] = dmul(lism[4], dadd(1.0, d2));
        q[5] = lism[5];
        q[6] = lism[6];
        q[7] = lism[7];
    }
}

// Seeded initial condition of one cell (conserved).
SB_HD void lism_cell(const GridGeom& g, const double* lism, uint64_t seed, double pert, int i, int j,
                     int k, double* U) {
    double q[8];
    lism_prim(g, lism, seed, pert, i, j, k, q);
    cons_from_prim_exact(q, U);
}

// Tangent basis (e2, e3) of a face with unit normal nrm, from the field averaged over the two
// sides (the reference's aco construction, Solvers.f90:1236-1273; chlld_Q :323-360), with one
// reciprocal of the norm instead of six divisions (the face-list path measured 5-10 % faster).
SB_HD void face_basis(const double* nrm, const double* q1d, const double* q2d, double* e2, double* e3) {
    const double al = nrm[0], be = nrm[1], ge = nrm[2];
    double bav[3];
    for (int c = 0; c < 3; c++) bav[c] = 0.5 * (q1d[5 + c] + q2d[5 + c]) * kInvSpi4;
    const double bk = bav[0] * al + bav[1] * be + bav[2] * ge;
    double d = (bav[0] * bav[0] + bav[1] * bav[1] + bav[2] * bav[2]) - bk * bk;
    if (d > 1.0e-12) {
        d = sqrt(d);
        const double id = sb_rcp(d);   // one reciprocal for the six components
        e2[0] = (bav[0] - bk * al) * id;
        e2[1] = (bav[1] - bk * be) * id;
        e2[2] = (bav[2] - bk * ge) * id;
        e3[0] = (bav[1] * ge - bav[2] * be) * id;
        e3[1] = (bav[2] * al - bav[0] * ge) * id;
        e3[2] = (bav[0] * be - bav[1] * al) * id;
    } else {
        double ai[3] = {0.0, 0.0, 0.0};
        if (sb_abs(al) < sb_abs(be) && sb_abs(al) < sb_abs(ge)) ai[0] = 1.0;
        else if (sb_abs(be) < sb_abs(ge)) ai[1] = 1.0;
        else ai[2] = 1.0;
        const double aik = ai[0] * al + ai[1] * be + ai[2] * ge;
        d = sqrt(1.0 - aik * aik);
        const double id = sb_rcp(d);
        e2[0] = (ai[0] - aik * al) * id;
        e2[1] = (ai[1] - aik * be) * id;
        e2[2] = (ai[2] - aik * ge) * id;
        e3[0] = (ai[1] * ge - ai[2] * be) * id;
        e3[1] = (ai[2] * al - ai[0] * ge) * id;
        e3[2] = (ai[0] * be - ai[1] * al) * id;
    }
}

// General-normal chlld for a batch of faces: the lab states are rotated into an orthonormal
// face frame (face_basis), solved, and the momentum / B fluxes rotated back.  MOVING = false:
// the caller's face speed w is 0 (the face-list grids), so the face-speed terms are not built.
template <typename T, int NSTATE, bool DELTA = false, bool MOVING = true>
SB_HD void chlld_general(const double* nrm, double w, const double* q1d, const double* q2d, int n_disc,
                          double* qqq, double* sp, int32_t* flag) {
    const double al = nrm[0], be = nrm[1], ge = nrm[2];
    double e2[3], e3[3];
    face_basis(nrm, q1d, q2d, e2, e3);
    T a[8], b[8], F[8], SL, SR, SM;
    const double* qs[2] = {q1d, q2d};
    T* outs[2] = {a, b};
    for (int s = 0; s < 2; s++) {
        const double* q = qs[s];
        T* o = outs[s];
        o[0] = T(q[0]);
        o[4] = T(q[4]);
        o[1] = T(q[1] * al + q[2] * be + q[3] * ge);
        o[2] = T(q[1] * e2[0] + q[2] * e2[1] + q[3] * e2[2]);
        o[3] = T(q[1] * e3[0] + q[2] * e3[1] + q[3] * e3[2]);
        o[5] = T(q[5] * al + q[6] * be + q[7] * ge);
        o[6] = T(q[5] * e2[0] + q[6] * e2[1] + q[7] * e2[2]);
        o[7] = T(q[5] * e3[0] + q[6] * e3[1] + q[7] * e3[2]);
    }
    int fl;
    if (DELTA && sizeof(T) == 8 && w == 0.0 && NSTATE >= 2 && n_disc == 0) {
        float SLf, SRf, SMf;
        double Fd[8];
        fl = riemann_delta<(NSTATE >= 2 ? NSTATE : 3)>((const double*)a, (const double*)b, Fd, SLf, SRf, SMf);
        for (int k = 0; k < 8; k++) F[k] = (T)Fd[k];
        SL = (T)SLf;
        SR = (T)SRf;
        SM = (T)SMf;
        if (fl & kFlagStar) {
            fl = riemann<T, NSTATE, true, false>(a, b, T(w), n_disc, F, SL, SR, SM) | kFlagStar;
        }
    } else {
        fl = riemann<T, NSTATE, MOVING, (sizeof(T) == 4)>(a, b, T(w), n_disc, F, SL, SR, SM);
    }
    if (sizeof(T) == 4 && (fl & kFlagStar)) {
        // the mixed form's rule: a face whose FP32 star state is not positive is redone in FP64
        chlld_general<double, NSTATE, false, MOVING>(nrm, w, q1d, q2d, n_disc, qqq, sp, flag);
        *flag |= kFlagStar;
        return;
    }
    qqq[0] = F[0];
    qqq[4] = F[4];
    const double nn[3] = {al, be, ge};
    for (int c = 0; c < 3; c++) {
        qqq[1 + c] = nn[c] * (double)F[1] + e2[c] * (double)F[2] + e3[c] * (double)F[3];
        qqq[5 + c] = nn[c] * (double)F[5] + e2[c] * (double)F[6] + e3[c] * (double)F[7];
    }
    sp[0] = SL;
    sp[1] = SR;
    sp[2] = SM;
    *flag = fl;
}

// Row pitch and variable stride of a device-owned state of this geometry.
inline void set_device_strides(GridGeom& g) {
    g.px = (g.nx + 1) / 2 * 2;
    g.ps = g.px * g.ny;
    g.vs = (g.ps * g.nz + 31) / 32 * 32;
}

// Encodes the 4-D tensor map (x, y, z, variable) of the FP64 SoA state at `base` with geometry
// g, box (kTileX + 4, ty + 4, 1, 8): one plane of a column tile of ty rows with its 2-cell halo.
// Returns a SETB_* status.
int encode_state_tmap(const GridGeom& g, const double* base, int ty, CUtensorMap* out);

// ---------------------------------------------------------------- face-list grids (facelist.cu)
struct FaceListDev;
int fl_validate(int64_t N, int64_t G, const double* cell_center, const double* cell_volume, const int32_t* cell_gran,
                const double* gran_normal, const double* gran_square, const double* gran_center,
                const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd, const int32_t* gran_type);
int fl_create(FaceListDev** out, int64_t n_cell, int64_t n_gran, const double* cell_center, const double* cell_volume,
              const int32_t* cell_gran, const double* gran_normal, const double* gran_square,
              const double* gran_center, const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd,
              const int32_t* gran_type, const setb_fl_params* p, cudaStream_t s);
void fl_destroy(FaceListDev* f);
// Locality order of a face-list handle: device cell d is the caller's cell perm[d] (0-based);
// null for a null handle.
const int32_t* fl_perm(const FaceListDev* f);
// Uploads the H-atom fluids (Cell_par columns 9..16) of a face list with physics 1; no-op else.
int fl_set_hatom(FaceListDev* f, const double* cell_par, cudaStream_t s);
// One stage on the face list: primitive pass, face fluxes (+ dt candidate when want_dt), cell
// update (kind 0: Euler / Heun stage 1, kind 1: Heun stage 2); a finalizing stage rolls the clock.
cudaError_t fl_launch_stage(const FaceListDev* f, const double* Uin, const double* Ubase, double* Uout, int64_t vs,
                            DevClock* clk, DevStatus* st, const setb_step_opts* o, int kind, bool want_dt,
                            bool finalize, cudaStream_t s);

// ---------------------------------------------------------------- launch entry points
cudaError_t launch_stage_fp64(const StageArgs& a, int n_state, int order, int kind, bool want_dt,
                              cudaStream_t s);
cudaError_t launch_stage(const StageArgs& a, int precision, int n_state, int order, int kind, bool want_dt,
                         cudaStream_t s);
int stage_smem_bytes(int precision, int kind);
cudaError_t launch_batch_stage(const BatchArgs& b, int precision, int n_state, int kind, bool want_dt, int grid,
                               cudaStream_t s);
cudaError_t prepare_batch_kernels(int precision);
int batch_ctas_per_sm(int precision);
cudaError_t launch_lism_init(const GridGeom& g, const double* lism, uint64_t seed, double pert,
                             double* U, cudaStream_t s);
cudaError_t launch_prim_to_cons(const GridGeom& g, const double* prim8, double* U, cudaStream_t s);
cudaError_t launch_cons_to_prim(const GridGeom& g, const double* U, double* prim8, cudaStream_t s);
cudaError_t launch_chlld_batch(int64_t n, int n_state, int n_disc, int precision,
                               const double* normals, const double* w, const double* q1,
                               const double* q2, double* qqq, double* speeds, int32_t* flags,
                               cudaStream_t s);
cudaError_t launch_chlld_q_batch(int64_t n, int n_state, int n_disc, bool ydar, const double* normals,
                                 const double* w, const double* q1, const double* q2, double* konvect,
                                 double* qqq, double* speeds, int32_t* flags, cudaStream_t s);
int stage_fp64_smem_bytes();

}  // namespace sb
