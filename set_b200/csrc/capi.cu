// capi.cu -- host runtime and the C ABI of libsetb200.so (declared in include/setb200.h).
//
// The reference drives its kernels from the Fortran module MY_CUDA: Set_CUDA allocates and
// uploads (cuf_kernel.cuf:351-382), CUDA_START_MGD runs the time loop with 4 launches and 5
// device-wide synchronisations per step (:780-925), Send_data_to_Host downloads (:384-400).
// Here a handle owns the device state and one stream; a step is 2 launches (Heun) or 1
// (Euler) with no host synchronisation, and the lagged dt lives on the device.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "setb200.h"
#include "setb_internal.cuh"
#include "chlld_q.cuh"

using namespace sb;

sb::NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
sb::NvtxRange::~NvtxRange() { nvtxRangePop(); }

struct setb_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    setb_cart_desc desc{};
    GridGeom g{};
    double* buf[2] = {nullptr, nullptr};   // conserved SoA, 8 * vs doubles each
    int cur = 0;                           // buf[cur] holds U^n
    float* comp = nullptr;                 // mixed form: FP32 compensation, 8 * vs floats
    bool comp_clean = false;               // comp holds zeros for the current state
    DevClock* clk = nullptr;
    DevStatus* st = nullptr;
    DevClock* h_clk = nullptr;             // pinned mirrors
    DevStatus* h_st = nullptr;
    CUtensorMap* tmap = nullptr;           // device: [buffer 0/1][tile shape, kShapeTy]
    bool tma_ok[3] = {false, false, false};   // per tile shape: maps encoded (else plain loads)
    FaceListDev* fl = nullptr;             // face-list grid (g is then 1-D: nx = N cells)
    int ctas_per_sm = 1;
    int sm_count = 148;
    long long copy_wait = 0;               // StageArgs::copy_wait of this handle's launches
};

namespace {

#define SB_TRY(expr)                                   \
    do {                                               \
        cudaError_t e_ = (expr);                       \
        if (e_ != cudaSuccess) return SETB_ECUDA;      \
    } while (0)

}  // namespace

int sb::validate_desc(const setb_cart_desc* d) {
    if (!d) return SETB_EINVAL;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->flags != 0) return SETB_EINVAL;
    if ((long long)d->nx * d->ny * d->nz > (1ll << 31)) return SETB_ESIZE;
    for (int a = 0; a < 3; a++)
        if (!(d->hi[a] > d->lo[a])) return SETB_EINVAL;
    if (!(d->inflow[0] > 0.0) || !(d->inflow[4] > 0.0)) return SETB_EINVAL;
    if (d->r_src < 0.0 || (d->r_src > 0.0 && !(d->rho_src > 0.0))) return SETB_EINVAL;
    if (!(d->dt_init > 0.0)) return SETB_EINVAL;
    return SETB_OK;
}

int sb::validate_opts(const setb_step_opts* o) {
    if (!o) return SETB_EINVAL;
    if (o->n_state < 0 || o->n_state > 3) return SETB_EINVAL;
    if (o->n_disc < 0 || o->n_disc > 2) return SETB_EINVAL;
    if (o->order != 1 && o->order != 2) return SETB_EINVAL;
    if (o->scheme != 1 && o->scheme != 2) return SETB_EINVAL;
    if (o->precision < 0 || o->precision > 2) return SETB_EINVAL;
    if (o->precision >= 2 && (o->n_state < 2 || o->n_disc != 0)) return SETB_EINVAL;
    if (o->reserved != 0) return SETB_EINVAL;
    if (!(o->cfl > 0.0)) return SETB_EINVAL;
    return SETB_OK;
}

namespace {

GridGeom make_geom(const setb_cart_desc* d) {
    GridGeom g{};
    g.nx = d->nx;
    g.ny = d->ny;
    g.nz = d->nz;
    set_device_strides(g);   // even row pitch, 256-byte aligned variable planes
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; a++) {
        g.lo[a] = d->lo[a];
        g.h[a] = (d->hi[a] - d->lo[a]) / n[a];
        g.inv_dist[a] = 1.0 / (0.5 * g.h[a]);
    }
    g.square[0] = g.h[1] * g.h[2];
    g.square[1] = g.h[0] * g.h[2];
    g.square[2] = g.h[0] * g.h[1];
    g.inv_vol = 1.0 / (g.h[0] * g.h[1] * g.h[2]);
    for (int v = 0; v < 8; v++) g.inflow[v] = d->inflow[v];
    g.r_src = d->r_src;
    g.rho_src = d->rho_src;
    g.v_src = d->v_src;
    g.p_over_rho_src = d->p_over_rho_src;
    g.r_floor = d->r_floor;
    g.lz = d->nz;
    return g;
}

// The tile heights a handle keeps tensor maps for (plain, mixed stage 2, mixed stage 1 / delta),
// and which one a launch uses.
constexpr int kNumShapes = 3;
constexpr int kShapeTy[kNumShapes] = {tile_shape(0, 0).ty, tile_shape(1, 1).ty, tile_shape(1, 0).ty};
constexpr bool shape_listed(int ty) { return ty == kShapeTy[0] || ty == kShapeTy[1] || ty == kShapeTy[2]; }
static_assert(shape_listed(tile_shape(0, 1).ty) && shape_listed(tile_shape(2, 0).ty) && shape_listed(tile_shape(2, 1).ty),
              "every stage launch's tile height has a tensor map");
int shape_index(int precision, int kind) {
    const int ty = tile_shape(precision, kind).ty;
    return ty == kShapeTy[0] ? 0 : (ty == kShapeTy[1] ? 1 : 2);
}

}  // namespace

// z extent of one CTA's march: balances wave quantisation against the per-chunk prologue
// (4 plane loads + 1 z face, costed as ~1.5 plane iterations).
int sb::choose_lz(const GridGeom& g, int sm_count, int precision, int kind) {
    const TileShape ts = tile_shape(precision, kind);
    const long long cols = (long long)((g.nx + kTileX - 1) / kTileX) * ((g.ny + ts.ty - 1) / ts.ty);
    const long long slots = (long long)sm_count * std::max(ts.ctas_per_sm, 1);
    const int nz = plane_end(g) - plane_begin(g);   // planes the stage kernels update
    double best = 1e300;
    int best_lz = nz;
    for (int c = 1; c <= std::max(1, nz / 8); c++) {
        const int lz = (nz + c - 1) / c;
        const long long ctas = cols * ((nz + lz - 1) / lz);
        const long long waves = (ctas + slots - 1) / slots;
        const double cost = (double)waves * (lz + 1.5);
        if (cost < best - 1e-9) {
            best = cost;
            best_lz = lz;
        }
    }
    return best_lz;
}

namespace {

void clock_reset(setb_handle* h, double time_all) {
    DevClock c{};
    c.dt_cur = h->desc.dt_init;
    c.dt_next = 0;
    double reset = kDtReset;
    std::memcpy(&c.dt_next, &reset, sizeof(double));
    c.time_all = time_all;
    c.dt_last = 0.0;
    c.counter = 0;
    c.steps = 0;
    *h->h_clk = c;
    DevStatus s{};
    s.first_bad = ULLONG_MAX;
    *h->h_st = s;
}

int upload_clock(setb_handle* h) {
    SB_TRY(cudaMemcpyAsync(h->clk, h->h_clk, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    SB_TRY(cudaMemcpyAsync(h->st, h->h_st, sizeof(DevStatus), cudaMemcpyHostToDevice, h->stream));
    SB_TRY(cudaStreamSynchronize(h->stream));
    return SETB_OK;
}

int download_clock(setb_handle* h) {
    SB_TRY(cudaMemcpyAsync(h->h_clk, h->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    SB_TRY(cudaMemcpyAsync(h->h_st, h->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
    SB_TRY(cudaStreamSynchronize(h->stream));
    return SETB_OK;
}

int status_code(const DevStatus& s) {
    if (s.n_timeout) return SETB_ETIMEOUT;
    if (s.n_negdens) return SETB_ENEGDENS;
    if (s.n_wave) return SETB_EWAVES;
    if (s.n_recon) return SETB_ERECON;
    return SETB_OK;
}

void destroy_impl(setb_handle* h) {
    if (!h) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (double* b : h->buf)
        if (b) cudaFree(b);
    if (h->comp) cudaFree(h->comp);
    if (h->clk) cudaFree(h->clk);
    if (h->st) cudaFree(h->st);
    if (h->tmap) cudaFree(h->tmap);
    if (h->fl) fl_destroy(h->fl);
    if (h->h_clk) cudaFreeHost(h->h_clk);
    if (h->h_st) cudaFreeHost(h->h_st);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaSetDevice(prev);
    delete h;
}

// geo: the handle's geometry when it is not the whole grid of d (a z slab)
int create_impl(setb_handle** out, const setb_cart_desc* d, const GridGeom* geo = nullptr) {
    if (!out) return SETB_EINVAL;
    *out = nullptr;
    int rc = validate_desc(d);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SETB_ENODEV;
    setb_handle* h = new (std::nothrow) setb_handle();
    if (!h) return SETB_ENOMEM;
    cudaGetDevice(&h->device);
    h->desc = *d;
    h->g = geo ? *geo : make_geom(d);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) {
        delete h;
        return SETB_ECUDA;
    }
    h->sm_count = prop.multiProcessorCount;
    h->ctas_per_sm = tile_shape(0, 0).ctas_per_sm;
    h->g.lz = choose_lz(h->g, h->sm_count, 0, 0);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return SETB_ECUDA;
    }
    const size_t bytes = sizeof(double) * 8 * (size_t)h->g.vs;
    for (int b = 0; b < 2; b++) {
        if (cudaMalloc(&h->buf[b], bytes) != cudaSuccess) {
            cudaGetLastError();
            destroy_impl(h);
            return SETB_ENOMEM;
        }
        // row padding and the tail of every variable plane stay zero
        if (cudaMemsetAsync(h->buf[b], 0, bytes, h->stream) != cudaSuccess) {
            destroy_impl(h);
            return SETB_ECUDA;
        }
    }
    {
        CUtensorMap tm[2 * kNumShapes] = {};
        for (int shape = 0; shape < kNumShapes; shape++) {
            h->tma_ok[shape] = true;
            for (int b = 0; b < 2; b++)
                if (encode_state_tmap(h->g, h->buf[b], kShapeTy[shape], &tm[kNumShapes * b + shape]) != SETB_OK)
                    h->tma_ok[shape] = false;
        }
        if (cudaMalloc(&h->tmap, sizeof(tm)) != cudaSuccess ||
            cudaMemcpyAsync(h->tmap, tm, sizeof(tm), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
            cudaGetLastError();
            destroy_impl(h);
            return SETB_ENOMEM;
        }
    }
    if (cudaMalloc(&h->clk, sizeof(DevClock)) != cudaSuccess || cudaMalloc(&h->st, sizeof(DevStatus)) != cudaSuccess ||
        cudaMallocHost(&h->h_clk, sizeof(DevClock)) != cudaSuccess ||
        cudaMallocHost(&h->h_st, sizeof(DevStatus)) != cudaSuccess) {
        cudaGetLastError();
        destroy_impl(h);
        return SETB_ENOMEM;
    }
    *out = h;
    return SETB_OK;
}

// Uploads Cell_par columns 1..8 (16 doubles per cell) into buf[cur] through buf[1-cur].  A
// face-list handle keeps its cells in locality order: row d of the device state is the caller's
// cell perm[d].
int upload_cellpar(setb_handle* h, const double* cell_par) {
    h->comp_clean = false;
    const size_t N = (size_t)h->g.nx * h->g.ny * h->g.nz;
    double* stage = h->buf[1 - h->cur];
    if (h->g.kb) {   // z slab: the owned planes only; the ghost planes start as zeros
        const size_t plane = (size_t)h->g.nx * h->g.ny;
        const size_t own = plane * (size_t)(plane_end(h->g) - plane_begin(h->g));
        SB_TRY(cudaMemsetAsync(stage, 0, sizeof(double) * 8 * N, h->stream));
        SB_TRY(cudaMemcpy2DAsync(stage + 8 * plane * (size_t)h->g.kb, 8 * sizeof(double), cell_par, 16 * sizeof(double),
                                 8 * sizeof(double), own, cudaMemcpyHostToDevice, h->stream));
        SB_TRY(launch_prim_to_cons(h->g, stage, h->buf[h->cur], h->stream));
        return SETB_OK;
    }
    if (const int32_t* perm = fl_perm(h->fl)) {
        const int rc = fl_set_hatom(h->fl, cell_par, h->stream);
        if (rc) return rc;
        std::vector<double> tmp(8 * N);
        for (size_t d = 0; d < N; d++) std::memcpy(&tmp[8 * d], cell_par + 16 * (size_t)perm[d], 8 * sizeof(double));
        SB_TRY(cudaMemcpyAsync(stage, tmp.data(), sizeof(double) * 8 * N, cudaMemcpyHostToDevice, h->stream));
        SB_TRY(launch_prim_to_cons(h->g, stage, h->buf[h->cur], h->stream));
        SB_TRY(cudaStreamSynchronize(h->stream));   // tmp is released on return
        return SETB_OK;
    }
    SB_TRY(cudaMemcpy2DAsync(stage, 8 * sizeof(double), cell_par, 16 * sizeof(double), 8 * sizeof(double), N,
                             cudaMemcpyHostToDevice, h->stream));
    SB_TRY(launch_prim_to_cons(h->g, stage, h->buf[h->cur], h->stream));
    return SETB_OK;
}

template <typename T, int NS>
void chlld_host(const double* n, double w, const double* q1, const double* q2, int n_disc, double* qqq,
                double* sp, int32_t* fl) {
    chlld_general<T, NS>(n, w, q1, q2, n_disc, qqq, sp, fl);
}

}  // namespace

extern "C" {

int32_t setb_version(void) { return 100; }

const char* setb_strerror(int32_t code) {
    switch (code) {
        case SETB_OK: return "ok";
        case SETB_EINVAL: return "invalid argument";
        case SETB_ECUDA: return "CUDA runtime error";
        case SETB_ENOMEM: return "device allocation failed or memory budget exceeded";
        case SETB_ENEGDENS: return "cell update produced non-positive density";
        case SETB_EWAVES: return "no wave-fan region matched in the Riemann solver";
        case SETB_ERECON: return "reconstructed face density is negative";
        case SETB_ETIMEOUT: return "bounded device wait gave up";
        case SETB_ENODEV: return "no usable CUDA device";
        case SETB_ESIZE: return "size exceeds the documented maximum";
        case SETB_EIO: return "file I/O or format error";
        case SETB_EBUSY: return "request refused: queue full or admission budget exhausted";
        default: return "unknown status code";
    }
}

int32_t setb_chlld(const int32_t* n_state, const double* al, const double* be, const double* ge, const double* w,
                   const double qqq1[8], const double qqq2[8], double* dsl, double* dsp, double* dsc, double qqq[8],
                   const int32_t* n_disc) {
    if (!n_state || !al || !be || !ge || !w || !qqq1 || !qqq2 || !dsl || !dsp || !dsc || !qqq) return SETB_EINVAL;
    const int nd = n_disc ? *n_disc : 0;
    if (*n_state < 0 || *n_state > 3 || nd < 0 || nd > 2) return SETB_EINVAL;
    const double n[3] = {*al, *be, *ge};
    double sp[3];
    int32_t fl = 0;
    switch (*n_state) {
        case 0: chlld_host<double, 0>(n, *w, qqq1, qqq2, nd, qqq, sp, &fl); break;
        case 1: chlld_host<double, 1>(n, *w, qqq1, qqq2, nd, qqq, sp, &fl); break;
        case 2: chlld_host<double, 2>(n, *w, qqq1, qqq2, nd, qqq, sp, &fl); break;
        default: chlld_host<double, 3>(n, *w, qqq1, qqq2, nd, qqq, sp, &fl); break;
    }
    *dsl = sp[0];
    *dsp = sp[1];
    *dsc = sp[2];
    return (fl & kFlagWave) ? SETB_EWAVES : SETB_OK;
}

int32_t setb_chlld_q(const int32_t* n_state, const double* al, const double* be, const double* ge, const double* w,
                     const double qqq1[9], const double qqq2[9], double* dsl, double* dsp, double* dsc, double qqq[9],
                     const int32_t* null_bn1, const int32_t* n_disc, const int32_t* p_correct_, double* konvect_,
                     const int32_t* ydar_) {
    (void)null_bn1;     // overridden to .False. inside chlld_Q (Solvers.f90:267)
    (void)p_correct_;   // phi_p_correct is set to 1 whatever its value (Solvers.f90:266)
    if (!n_state || !al || !be || !ge || !w || !qqq1 || !qqq2 || !dsl || !dsp || !dsc || !qqq) return SETB_EINVAL;
    const int nd = n_disc ? *n_disc : 0;
    if (*n_state < 0 || *n_state > 3 || nd < 0 || nd > 2) return SETB_EINVAL;
    const bool ydar = ydar_ && *ydar_ != 0;
    const double n[3] = {*al, *be, *ge};
    double sp[3];
    int32_t fl = 0;
    switch (*n_state) {
        case 0: chlld_q_general<0>(n, *w, qqq1, qqq2, nd, ydar, konvect_, qqq, sp, &fl); break;
        case 1: chlld_q_general<1>(n, *w, qqq1, qqq2, nd, ydar, konvect_, qqq, sp, &fl); break;
        case 2: chlld_q_general<2>(n, *w, qqq1, qqq2, nd, ydar, konvect_, qqq, sp, &fl); break;
        default: chlld_q_general<3>(n, *w, qqq1, qqq2, nd, ydar, konvect_, qqq, sp, &fl); break;
    }
    *dsl = sp[0];
    *dsp = sp[1];
    *dsc = sp[2];
    return (fl & kFlagWave) ? SETB_EWAVES : SETB_OK;
}

int32_t setb_chlld_q_batch(int64_t n, int32_t n_state, int32_t n_disc, int32_t ydar, const double* normals,
                           const double* w, const double* q1, const double* q2, double* konvect, double* qqq,
                           double* speeds, int32_t* flags) {
    if (n < 0 || n_state < 0 || n_state > 3 || n_disc < 0 || n_disc > 2) return SETB_EINVAL;
    if (n == 0) return SETB_OK;
    if (!normals || !q1 || !q2 || !qqq || !speeds || !flags) return SETB_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SETB_ENODEV;
    const size_t sn = (size_t)n;
    double *dn = nullptr, *dw = nullptr, *d1 = nullptr, *d2 = nullptr, *dk = nullptr, *dq = nullptr, *ds = nullptr;
    int32_t* df = nullptr;
    cudaStream_t s = nullptr;
    int rc = SETB_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return SETB_ECUDA;
    if (cudaMalloc(&dn, 3 * sn * 8) || (w && cudaMalloc(&dw, sn * 8)) || cudaMalloc(&d1, 9 * sn * 8) ||
        cudaMalloc(&d2, 9 * sn * 8) || (konvect && cudaMalloc(&dk, 3 * sn * 8)) || cudaMalloc(&dq, 9 * sn * 8) ||
        cudaMalloc(&ds, 3 * sn * 8) || cudaMalloc(&df, sn * 4)) {
        cudaGetLastError();
        rc = SETB_ENOMEM;
    }
    if (rc == SETB_OK) {
        bool ok = cudaMemcpyAsync(dn, normals, 3 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  (!w || cudaMemcpyAsync(dw, w, sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess) &&
                  cudaMemcpyAsync(d1, q1, 9 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  cudaMemcpyAsync(d2, q2, 9 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  (!konvect || cudaMemcpyAsync(dk, konvect, 3 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess) &&
                  launch_chlld_q_batch(n, n_state, n_disc, ydar != 0, dn, dw, d1, d2, dk, dq, ds, df, s) ==
                      cudaSuccess &&
                  cudaMemcpyAsync(qqq, dq, 9 * sn * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  cudaMemcpyAsync(speeds, ds, 3 * sn * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  cudaMemcpyAsync(flags, df, sn * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  (!konvect || cudaMemcpyAsync(konvect, dk, 3 * sn * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess) &&
                  cudaStreamSynchronize(s) == cudaSuccess;
        if (!ok) rc = SETB_ECUDA;
    }
    cudaFree(dn);
    cudaFree(dw);
    cudaFree(d1);
    cudaFree(d2);
    cudaFree(dk);
    cudaFree(dq);
    cudaFree(ds);
    cudaFree(df);
    cudaStreamDestroy(s);
    return rc;
}

int32_t setb_chlld_batch(int64_t n, int32_t n_state, int32_t n_disc, int32_t precision, const double* normals,
                         const double* w, const double* q1, const double* q2, double* qqq, double* speeds,
                         int32_t* flags) {
    if (n < 0 || n_state < 0 || n_state > 3 || n_disc < 0 || n_disc > 2 || precision < 0 || precision > 2)
        return SETB_EINVAL;
    if (precision >= 2 && (n_state < 2 || n_disc != 0)) return SETB_EINVAL;
    if (n == 0) return SETB_OK;
    if (!normals || !q1 || !q2 || !qqq || !speeds || !flags) return SETB_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SETB_ENODEV;
    double *dn = nullptr, *dw = nullptr, *d1 = nullptr, *d2 = nullptr, *dq = nullptr, *ds = nullptr;
    int32_t* df = nullptr;
    cudaStream_t s = nullptr;
    int rc = SETB_OK;
    const size_t sn = (size_t)n;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return SETB_ECUDA;
    if (cudaMalloc(&dn, 3 * sn * 8) || (w && cudaMalloc(&dw, sn * 8)) || cudaMalloc(&d1, 8 * sn * 8) ||
        cudaMalloc(&d2, 8 * sn * 8) || cudaMalloc(&dq, 8 * sn * 8) || cudaMalloc(&ds, 3 * sn * 8) ||
        cudaMalloc(&df, sn * 4)) {
        cudaGetLastError();
        rc = SETB_ENOMEM;
    }
    if (rc == SETB_OK) {
        bool ok = cudaMemcpyAsync(dn, normals, 3 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  (!w || cudaMemcpyAsync(dw, w, sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess) &&
                  cudaMemcpyAsync(d1, q1, 8 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  cudaMemcpyAsync(d2, q2, 8 * sn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  launch_chlld_batch(n, n_state, n_disc, precision, dn, dw, d1, d2, dq, ds, df, s) == cudaSuccess &&
                  cudaMemcpyAsync(qqq, dq, 8 * sn * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  cudaMemcpyAsync(speeds, ds, 3 * sn * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  cudaMemcpyAsync(flags, df, sn * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                  cudaStreamSynchronize(s) == cudaSuccess;
        if (!ok) rc = SETB_ECUDA;
    }
    cudaFree(dn);
    cudaFree(dw);
    cudaFree(d1);
    cudaFree(d2);
    cudaFree(dq);
    cudaFree(ds);
    cudaFree(df);
    cudaStreamDestroy(s);
    return rc;
}

int32_t setb_cart_fill_lism(const setb_cart_desc* d, const setb_lism_ic* ic, double* cell_par) {
    int rc = validate_desc(d);
    if (rc) return rc;
    if (!ic || !cell_par) return SETB_EINVAL;
    const GridGeom g = make_geom(d);
    const long long N = (long long)d->nx * d->ny * d->nz;
    for (long long c = 0; c < N; c++) {
        const int i = (int)(c % d->nx);
        const int j = (int)((c / d->nx) % d->ny);
        const int k = (int)(c / ((long long)d->nx * d->ny));
        double q[8];
        lism_prim(g, ic->lism, ic->seed, ic->pert_amp, i, j, k, q);
        for (int v = 0; v < 8; v++) cell_par[16 * c + v] = q[v];
    }
    return SETB_OK;
}

int32_t setb_init_cartesian(setb_handle** out, const setb_cart_desc* d, const double* cell_par) {
    NvtxRange range("setb_init_cartesian");
    if (!cell_par) return SETB_EINVAL;
    int rc = create_impl(out, d);
    if (rc) return rc;
    setb_handle* h = *out;
    clock_reset(h, 0.0);
    rc = upload_cellpar(h, cell_par);
    if (!rc) rc = upload_clock(h);
    if (rc) {
        destroy_impl(h);
        *out = nullptr;
    }
    return rc;
}

int32_t setb_init_facelist(setb_handle** out, int32_t n_cell, int32_t n_gran, const double* cell_par,
                           const double* cell_center, const double* cell_volume, const int32_t* cell_gran,
                           const double* gran_normal, const double* gran_square, const double* gran_center,
                           const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd, const int32_t* gran_type,
                           const setb_fl_params* params) {
    if (!out || !cell_par || !params || n_cell < 1 || n_gran < 1) return SETB_EINVAL;
    *out = nullptr;
    if (!(params->dt_init > 0.0) || params->physics < 0 || params->physics > 1 ||
        params->powell < 0 || params->powell > 2 || (params->powell != 0 && params->physics != 0))
        return SETB_EINVAL;
    if (params->physics == 1)   // the axisymmetric update divides by the radius y
        for (int32_t c = 0; c < n_cell; c++)
            if (!(cell_center[3 * (size_t)c + 1] > 0.0)) return SETB_EINVAL;
    int rc = fl_validate(n_cell, n_gran, cell_center, cell_volume, cell_gran, gran_normal, gran_square, gran_center,
                         gran_neighbour, gran_neighbour_tvd, gran_type);
    if (rc) return rc;
    // the state lives in the handle's buffers as a 1-D "grid" of n_cell cells
    setb_cart_desc d{};
    d.nx = n_cell;
    d.ny = d.nz = 1;
    d.inflow[0] = d.inflow[4] = 1.0;   // unused by face lists (boundaries come from face types)
    for (int a = 0; a < 3; a++) {
        d.lo[a] = 0.0;
        d.hi[a] = 1.0;
    }
    d.r_src = params->r_src;
    d.rho_src = params->rho_src;
    d.v_src = params->v_src;
    d.p_over_rho_src = params->p_over_rho_src;
    d.r_floor = params->r_floor;
    d.dt_init = params->dt_init;
    rc = create_impl(out, &d);
    if (rc) return rc;
    setb_handle* h = *out;
    rc = fl_create(&h->fl, n_cell, n_gran, cell_center, cell_volume, cell_gran, gran_normal, gran_square,
                   gran_center, gran_neighbour, gran_neighbour_tvd, gran_type, params, h->stream);
    if (!rc) {
        clock_reset(h, 0.0);
        rc = upload_cellpar(h, cell_par);
    }
    if (!rc) rc = upload_clock(h);
    if (rc) {
        destroy_impl(h);
        *out = nullptr;
    }
    return rc;
}

int32_t setb_init_cartesian_lism(setb_handle** out, const setb_cart_desc* d, const setb_lism_ic* ic) {
    if (!ic) return SETB_EINVAL;
    int rc = create_impl(out, d);
    if (rc) return rc;
    setb_handle* h = *out;
    clock_reset(h, 0.0);
    double* dl = h->buf[1];   // 8 doubles of scratch for the LISM vector
    rc = SETB_OK;
    if (cudaMemcpyAsync(dl, ic->lism, 8 * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        launch_lism_init(h->g, dl, ic->seed, ic->pert_amp, h->buf[0], h->stream) != cudaSuccess)
        rc = SETB_ECUDA;
    if (!rc) rc = upload_clock(h);
    if (rc) {
        destroy_impl(h);
        *out = nullptr;
    }
    return rc;
}

namespace {
// Enqueues nsteps steps.  When ev is non-null, ev[0..2*nsteps] are recorded before the first
// launch and after every launch (Euler: ev[2s+1] == ev[2s+2] bracket nothing).
// Face-list steps: same stage sequence and events as the Cartesian path, three launches per stage.
int enqueue_fl_steps(setb_handle* h, int32_t nsteps, const setb_step_opts* o, cudaEvent_t* ev) {
    if (o->precision != 0) return SETB_EINVAL;
    h->comp_clean = false;
    if (ev) SB_TRY(cudaEventRecord(ev[0], h->stream));
    for (int s = 0; s < nsteps; s++) {
        double* U = h->buf[h->cur];
        double* W = h->buf[1 - h->cur];
        if (o->scheme == 2) {
            SB_TRY(fl_launch_stage(h->fl, U, nullptr, W, h->g.vs, h->clk, h->st, o, 0, true, false, h->stream));
            if (ev) SB_TRY(cudaEventRecord(ev[2 * s + 1], h->stream));
            SB_TRY(fl_launch_stage(h->fl, W, U, U, h->g.vs, h->clk, h->st, o, 1, false, true, h->stream));
            if (ev) SB_TRY(cudaEventRecord(ev[2 * s + 2], h->stream));
        } else {
            SB_TRY(fl_launch_stage(h->fl, U, nullptr, W, h->g.vs, h->clk, h->st, o, 0, true, true, h->stream));
            if (ev) {
                SB_TRY(cudaEventRecord(ev[2 * s + 1], h->stream));
                SB_TRY(cudaEventRecord(ev[2 * s + 2], h->stream));
            }
            h->cur = 1 - h->cur;
        }
    }
    return SETB_OK;
}

// The mixed form's FP32 compensation: allocated on first use, zeroed when stale.
int prepare_comp(setb_handle* h, int P, float** comp) {
    *comp = nullptr;
    if (P != 0) {
        if (!h->comp) {
            if (cudaMalloc(&h->comp, sizeof(float) * 8 * (size_t)h->g.vs) != cudaSuccess) {
                cudaGetLastError();
                return SETB_ENOMEM;
            }
            h->comp_clean = false;
        }
        if (!h->comp_clean) {
            SB_TRY(cudaMemsetAsync(h->comp, 0, sizeof(float) * 8 * (size_t)h->g.vs, h->stream));
            h->comp_clean = true;
        }
        *comp = h->comp;
    } else {
        h->comp_clean = false;   // plain steps leave the compensation stale
    }
    return SETB_OK;
}

int enqueue_steps(setb_handle* h, int32_t nsteps, const setb_step_opts* o, cudaEvent_t* ev) {
    if (h->fl) return enqueue_fl_steps(h, nsteps, o, ev);
    StageArgs a{};
    a.g = h->g;
    const int P = o->precision;
    const int lz0 = choose_lz(h->g, h->sm_count, P, 0), lz1 = choose_lz(h->g, h->sm_count, P, 1);
    float* comp = nullptr;
    if (const int rc = prepare_comp(h, P, &comp)) return rc;
    a.clk = h->clk;
    a.st = h->st;
    a.cfl = o->cfl;
    a.n_disc = o->n_disc;
    a.copy_wait = h->copy_wait;
    const int shape0 = shape_index(P, 0), shape1 = shape_index(P, 1);
    if (ev) SB_TRY(cudaEventRecord(ev[0], h->stream));
    for (int s = 0; s < nsteps; s++) {
        double* U = h->buf[h->cur];
        double* W = h->buf[1 - h->cur];
        const CUtensorMap* tmU = h->tma_ok[shape0] ? h->tmap + kNumShapes * h->cur + shape0 : nullptr;
        const CUtensorMap* tmW = h->tma_ok[shape1] ? h->tmap + kNumShapes * (1 - h->cur) + shape1 : nullptr;
        if (o->scheme == 2) {
            a.g.lz = lz0;
            a.Uin = U;
            a.tm_in = tmU;
            a.Ubase = nullptr;
            a.Uout = W;
            a.finalize = 0;
            a.comp = nullptr;
            SB_TRY(launch_stage(a, P, o->n_state, o->order, 0, true, h->stream));
            if (ev) SB_TRY(cudaEventRecord(ev[2 * s + 1], h->stream));
            a.g.lz = lz1;
            a.Uin = W;
            a.tm_in = tmW;
            a.Ubase = U;
            a.Uout = U;
            a.finalize = 1;
            a.comp = comp;
            SB_TRY(launch_stage(a, P, o->n_state, o->order, 1, false, h->stream));
            if (ev) SB_TRY(cudaEventRecord(ev[2 * s + 2], h->stream));
        } else {
            a.g.lz = lz0;
            a.Uin = U;
            a.tm_in = tmU;
            a.Ubase = nullptr;
            a.Uout = W;
            a.finalize = 1;
            a.comp = comp;
            SB_TRY(launch_stage(a, P, o->n_state, o->order, 0, true, h->stream));
            if (ev) {
                SB_TRY(cudaEventRecord(ev[2 * s + 1], h->stream));
                SB_TRY(cudaEventRecord(ev[2 * s + 2], h->stream));
            }
            h->cur = 1 - h->cur;
        }
    }
    return SETB_OK;
}
}  // namespace

int32_t setb_step(setb_handle* h, int32_t nsteps, const setb_step_opts* o, double* time_all) {
    NvtxRange range("setb_step");
    if (!h || nsteps < 0 || h->g.kb) return SETB_EINVAL;   // a z slab steps stage by stage
    int rc = validate_opts(o);
    if (rc) return rc;
    cudaSetDevice(h->device);
    rc = enqueue_steps(h, nsteps, o, nullptr);
    if (rc) return rc;
    if (time_all) {
        rc = download_clock(h);
        if (rc) return rc;
        *time_all = h->h_clk->time_all;
        return status_code(*h->h_st);
    }
    return SETB_OK;
}

int32_t setb_step_profiled(setb_handle* h, int32_t nsteps, const setb_step_opts* o, double* time_all,
                           double kernel_ms[2], int32_t launches[2]) {
    NvtxRange range("setb_step_profiled");
    if (!h || nsteps < 0 || !kernel_ms || !launches || h->g.kb) return SETB_EINVAL;
    int rc = validate_opts(o);
    if (rc) return rc;
    cudaSetDevice(h->device);
    std::vector<cudaEvent_t> ev(2 * (size_t)nsteps + 1, nullptr);
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            rc = SETB_ECUDA;
            break;
        }
    if (!rc) rc = enqueue_steps(h, nsteps, o, ev.data());
    kernel_ms[0] = kernel_ms[1] = 0.0;
    launches[0] = nsteps;
    launches[1] = o->scheme == 2 ? nsteps : 0;
    if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = SETB_ECUDA;
    for (int s = 0; s < nsteps && !rc; s++) {
        float a = 0.f, b = 0.f;
        if (cudaEventElapsedTime(&a, ev[2 * s], ev[2 * s + 1]) != cudaSuccess ||
            cudaEventElapsedTime(&b, ev[2 * s + 1], ev[2 * s + 2]) != cudaSuccess) {
            rc = SETB_ECUDA;
            break;
        }
        kernel_ms[0] += a;
        kernel_ms[1] += b;
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (rc) return rc;
    rc = download_clock(h);
    if (rc) return rc;
    if (time_all) *time_all = h->h_clk->time_all;
    return status_code(*h->h_st);
}

int32_t setb_sync(setb_handle* h) {
    if (!h) return SETB_EINVAL;
    cudaSetDevice(h->device);
    int rc = download_clock(h);
    if (rc) return rc;
    return status_code(*h->h_st);
}

int32_t setb_get_state(setb_handle* h, double* cell_par, double* time_all) {
    NvtxRange range("setb_get_state");
    if (!h || !cell_par) return SETB_EINVAL;
    cudaSetDevice(h->device);
    const size_t N = (size_t)h->g.nx * h->g.ny * h->g.nz;
    double* stage = h->buf[1 - h->cur];
    SB_TRY(launch_cons_to_prim(h->g, h->buf[h->cur], stage, h->stream));
    if (const int32_t* perm = fl_perm(h->fl)) {
        std::vector<double> tmp(8 * N);
        SB_TRY(cudaMemcpyAsync(tmp.data(), stage, sizeof(double) * 8 * N, cudaMemcpyDeviceToHost, h->stream));
        SB_TRY(cudaStreamSynchronize(h->stream));
        for (size_t d = 0; d < N; d++) std::memcpy(cell_par + 16 * (size_t)perm[d], &tmp[8 * d], 8 * sizeof(double));
    } else {
        const size_t plane = (size_t)h->g.nx * h->g.ny;   // a z slab returns its owned planes
        const size_t own = plane * (size_t)(plane_end(h->g) - plane_begin(h->g));
        SB_TRY(cudaMemcpy2DAsync(cell_par, 16 * sizeof(double), stage + 8 * plane * (size_t)h->g.kb,
                                 8 * sizeof(double), 8 * sizeof(double), own, cudaMemcpyDeviceToHost, h->stream));
    }
    int rc = download_clock(h);
    if (rc) return rc;
    if (time_all) *time_all = h->h_clk->time_all;
    return SETB_OK;
}

int32_t setb_set_state(setb_handle* h, const double* cell_par, double time_all) {
    NvtxRange range("setb_set_state");
    if (!h || !cell_par) return SETB_EINVAL;
    cudaSetDevice(h->device);
    SB_TRY(cudaStreamSynchronize(h->stream));
    clock_reset(h, time_all);
    int rc = upload_cellpar(h, cell_par);
    if (rc) return rc;
    return upload_clock(h);
}

int32_t setb_copy_state(setb_handle* dst, setb_handle* src) {
    if (!dst || !src) return SETB_EINVAL;
    if (dst->g.nx != src->g.nx || dst->g.ny != src->g.ny || dst->g.nz != src->g.nz || dst->g.vs != src->g.vs)
        return SETB_EINVAL;
    cudaSetDevice(dst->device);
    SB_TRY(cudaStreamSynchronize(src->stream));
    SB_TRY(cudaMemcpyAsync(dst->buf[dst->cur], src->buf[src->cur], sizeof(double) * 8 * (size_t)src->g.vs,
                           cudaMemcpyDeviceToDevice, dst->stream));
    SB_TRY(cudaMemcpyAsync(dst->clk, src->clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, dst->stream));
    SB_TRY(cudaMemcpyAsync(dst->st, src->st, sizeof(DevStatus), cudaMemcpyDeviceToDevice, dst->stream));
    dst->comp_clean = false;
    return SETB_OK;
}

int32_t setb_state_view(setb_handle* h, double** base, int64_t* var_stride, int64_t* plane_stride,
                        int64_t* row_pitch) {
    if (!h) return SETB_EINVAL;
    if (base) *base = h->buf[h->cur];
    if (var_stride) *var_stride = h->g.vs;
    if (plane_stride) *plane_stride = h->g.ps;
    if (row_pitch) *row_pitch = h->g.px;
    return SETB_OK;
}

int32_t setb_get_conserved(setb_handle* h, double* U) {
    if (!h || !U) return SETB_EINVAL;
    cudaSetDevice(h->device);
    const int nown = plane_end(h->g) - plane_begin(h->g);   // a z slab returns its owned planes
    const size_t N = (size_t)h->g.nx * h->g.ny * nown;
    const int32_t* perm = fl_perm(h->fl);
    std::vector<double> tmp(perm ? 8 * N : 0);
    double* dst = perm ? tmp.data() : U;
    for (int v = 0; v < 8; v++)
        SB_TRY(cudaMemcpy2DAsync(dst + v * N, h->g.nx * sizeof(double),
                                 h->buf[h->cur] + v * h->g.vs + (long long)h->g.kb * h->g.ps, h->g.px * sizeof(double),
                                 h->g.nx * sizeof(double), (size_t)h->g.ny * nown, cudaMemcpyDeviceToHost, h->stream));
    SB_TRY(cudaStreamSynchronize(h->stream));
    if (perm)
        for (int v = 0; v < 8; v++)
            for (size_t d = 0; d < N; d++) U[v * N + (size_t)perm[d]] = tmp[v * N + d];
    return SETB_OK;
}

int32_t setb_status(setb_handle* h, setb_diag* out) {
    if (!h || !out) return SETB_EINVAL;
    cudaSetDevice(h->device);
    int rc = download_clock(h);
    if (rc) return rc;
    const DevClock& c = *h->h_clk;
    const DevStatus& s = *h->h_st;
    out->time_all = c.time_all;
    out->dt_next = c.dt_cur;   // the dt the next step will use
    out->dt_last = c.dt_last;
    out->steps = c.steps;
    out->n_negdens = (int64_t)s.n_negdens;
    out->first_bad_cell = s.first_bad == ULLONG_MAX ? -1 : (int64_t)s.first_bad;
    if (out->first_bad_cell >= 0 && fl_perm(h->fl)) out->first_bad_cell = fl_perm(h->fl)[out->first_bad_cell];
    out->n_pfloor = (int64_t)s.n_pfloor;
    out->n_wave_err = (int64_t)s.n_wave;
    out->n_recon_err = (int64_t)s.n_recon;
    out->n_fp64_redo = (int64_t)s.n_redo;
    return SETB_OK;
}

int32_t setb_stream(setb_handle* h, void** stream) {
    if (!h || !stream) return SETB_EINVAL;
    *stream = (void*)h->stream;
    return SETB_OK;
}

// ------------------------------------------------------------------ z slabs
int32_t setb_init_slab(setb_handle** h, const setb_cart_desc* d, int32_t k0, int32_t nz_local,
                       const double* cell_par) {
    if (!h) return SETB_EINVAL;
    *h = nullptr;
    int rc = validate_desc(d);
    if (rc) return rc;
    if (!cell_par || nz_local < 2 || k0 < 0 || (long long)k0 + nz_local > d->nz) return SETB_EINVAL;
    GridGeom g = make_geom(d);   // spacing and face areas of the whole grid
    g.nz = nz_local + 2 * kSlabGhost;
    set_device_strides(g);
    g.kb = kSlabGhost;
    g.ke = nz_local + kSlabGhost;
    g.koff = k0 - kSlabGhost;
    g.lz = g.ke - g.kb;
    rc = create_impl(h, d, &g);
    if (rc) return rc;
    setb_handle* s = *h;
    s->g.lz = choose_lz(s->g, s->sm_count, 0, 0);
    clock_reset(s, 0.0);
    rc = upload_cellpar(s, cell_par);
    if (!rc) rc = upload_clock(s);
    if (rc) {
        destroy_impl(s);
        *h = nullptr;
    }
    return rc;
}

int32_t setb_slab_stage(setb_handle* h, int32_t stage, const setb_step_opts* o) {
    NvtxRange range("setb_slab_stage");
    if (!h || !h->g.kb || (stage != 1 && stage != 2)) return SETB_EINVAL;
    int rc = validate_opts(o);
    if (rc) return rc;
    if (stage == 2 && o->scheme != 2) return SETB_EINVAL;
    cudaSetDevice(h->device);
    const GridGeom& g = h->g;
    const int P = o->precision, kind = stage - 1;
    const int in = stage == 1 ? h->cur : 1 - h->cur;   // buffer index of the stage input
    double* U = h->buf[h->cur];
    double* W = h->buf[1 - h->cur];
    double* X = h->buf[in];
    // ghost planes beyond the whole grid's z ends: copies of the end plane (the clamped index of
    // the single-grid kernel), so a slab reproduces the whole grid bit for bit
    const size_t pitch = sizeof(double) * (size_t)g.vs, width = sizeof(double) * (size_t)g.ps;
    if (g.koff + g.kb == 0)
        for (int p = 0; p < g.kb; p++)
            SB_TRY(cudaMemcpy2DAsync(X + (long long)p * g.ps, pitch, X + (long long)g.kb * g.ps, pitch, width, 8,
                                     cudaMemcpyDeviceToDevice, h->stream));
    if (g.koff + g.ke == h->desc.nz)
        for (int p = g.ke; p < g.nz; p++)
            SB_TRY(cudaMemcpy2DAsync(X + (long long)p * g.ps, pitch, X + (long long)(g.ke - 1) * g.ps, pitch, width, 8,
                                     cudaMemcpyDeviceToDevice, h->stream));
    float* comp = nullptr;
    if ((rc = prepare_comp(h, P, &comp))) return rc;
    const int shape = shape_index(P, kind);
    StageArgs a{};
    a.g = g;
    a.g.lz = choose_lz(g, h->sm_count, P, kind);
    a.clk = h->clk;
    a.st = h->st;
    a.cfl = o->cfl;
    a.n_disc = o->n_disc;
    a.copy_wait = h->copy_wait;
    a.Uin = X;
    a.tm_in = h->tma_ok[shape] ? h->tmap + kNumShapes * in + shape : nullptr;
    if (stage == 1) {
        a.Ubase = nullptr;
        a.Uout = W;
        a.finalize = o->scheme == 1;
        a.comp = o->scheme == 1 ? comp : nullptr;
    } else {
        a.Ubase = U;
        a.Uout = U;
        a.finalize = 1;
        a.comp = comp;
    }
    SB_TRY(launch_stage(a, P, o->n_state, o->order, kind, stage == 1, h->stream));
    if (stage == 1 && o->scheme == 1) h->cur = 1 - h->cur;
    return SETB_OK;
}

int32_t setb_set_copy_wait(setb_handle* h, int64_t cycles) {
    if (!h) return SETB_EINVAL;
    h->copy_wait = cycles;
    return SETB_OK;
}

int32_t setb_slab_view(setb_handle* h, int32_t stage, double** base, int64_t* var_stride, int64_t* plane_stride,
                       int32_t* nz_buffer) {
    if (!h || !h->g.kb || (stage != 1 && stage != 2) || !base || !var_stride || !plane_stride || !nz_buffer)
        return SETB_EINVAL;
    *base = h->buf[stage == 1 ? h->cur : 1 - h->cur];
    *var_stride = h->g.vs;
    *plane_stride = h->g.ps;
    *nz_buffer = h->g.nz;
    return SETB_OK;
}

int32_t setb_slab_dt(setb_handle* h, double** dt_next) {
    if (!h || !h->g.kb || !dt_next) return SETB_EINVAL;
    *dt_next = &h->clk->dt_cur;
    return SETB_OK;
}

int32_t setb_destroy(setb_handle* h) {
    if (!h) return SETB_EINVAL;
    destroy_impl(h);
    return SETB_OK;
}

}  // extern "C"
