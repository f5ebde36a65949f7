// noalloc.cu -- setb_step_noalloc: the Cartesian step for callers that cannot allocate device
// memory through the CUDA runtime.
//
// Who needs it: hosts that own every byte of device memory themselves -- a CUDA Fortran host
// whose state already lives in its own `device` allocatables, or a service that reserves HBM
// up front in its own arena and must not let a library call cudaMalloc (cudaMalloc can
// synchronise the whole device and would carve memory out of space the caller has promised to
// others).  Such a caller passes the state it already owns and gets the step without the
// library allocating anything.
//
// The step's scratch -- the Heun stage buffer U*, the device clock (lagged dt, time, CTA
// counter) and the error counters -- lives in one file-scope __device__ array of fixed size,
// below.  Every GPU that loads the library holds this array until the process exits.
#include <climits>
#include <cstring>
#include <mutex>

#include "setb200.h"
#include "setb_internal.cuh"

namespace sb {
namespace {

// Largest state the scratch holds: var_stride <= kNoAllocMaxCells (64^3 = 262144 cells, the
// size of config C1).  8 planes of U* plus a 256-byte header: 16 MiB + 256 B per GPU.
constexpr long long kNoAllocMaxCells = 262144;
constexpr long long kHeaderDoubles = 32;
static_assert(sizeof(DevClock) + sizeof(DevStatus) <= kHeaderDoubles * sizeof(double), "header too small");

static __device__ __align__(256) double g_noalloc_scratch[kHeaderDoubles + 8 * kNoAllocMaxCells];

// Device address of g_noalloc_scratch per device, resolved once per device.  In host code the
// array's name is only a host-side stand-in, so it must never be passed to a kernel.
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SETB_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return SETB_ENODEV;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        double* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return SETB_ECUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SETB_OK;
}

// Clears the clock and counters that every call must start from.
__global__ void noalloc_clock_init(DevClock* clk, DevStatus* st, double dt, double time_all) {
    DevClock c{};
    c.dt_cur = dt;
    c.dt_next = (unsigned long long)__double_as_longlong(kDtReset);
    c.time_all = time_all;
    c.dt_last = 0.0;
    c.counter = 0;
    c.steps = 0;
    *clk = c;
    DevStatus s{};
    s.first_bad = ULLONG_MAX;
    *st = s;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" int32_t setb_step_noalloc(const setb_cart_desc* d, const setb_step_opts* o, double* U,
                                     int64_t var_stride, int32_t nsteps, double* dt_io, double* time_io,
                                     setb_diag* diag, void* stream) {
    if (!d || !o || !U || !dt_io || !time_io || nsteps < 0) return SETB_EINVAL;
    // the same checks as setb_init_cartesian / setb_step, with the first dt taken from *dt_io
    setb_cart_desc dd = *d;
    dd.dt_init = *dt_io;
    int rc = validate_desc(&dd);
    if (rc == SETB_OK) rc = validate_opts(o);
    if (rc) return rc;
    if (o->precision != 0) return SETB_EINVAL;   // plain FP64 only: no compensation array
    const long long N = (long long)d->nx * d->ny * d->nz;
    if (N > kNoAllocMaxCells || var_stride > kNoAllocMaxCells) return SETB_ESIZE;
    if (var_stride < N) return SETB_EINVAL;

    double* scratch = nullptr;
    rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return SETB_ECUDA;
    DevClock* clk = reinterpret_cast<DevClock*>(scratch);
    DevStatus* st = reinterpret_cast<DevStatus*>(reinterpret_cast<char*>(scratch) + sizeof(DevClock));
    double* W = scratch + kHeaderDoubles;   // U*: 8 planes at the caller's var_stride
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    StageArgs a{};
    a.g.nx = d->nx;
    a.g.ny = d->ny;
    a.g.nz = d->nz;
    a.g.px = d->nx;
    a.g.ps = (long long)d->nx * d->ny;
    a.g.vs = var_stride;
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int ax = 0; ax < 3; ax++) {
        a.g.lo[ax] = d->lo[ax];
        a.g.h[ax] = (d->hi[ax] - d->lo[ax]) / n[ax];
        a.g.inv_dist[ax] = 1.0 / (0.5 * a.g.h[ax]);
    }
    a.g.square[0] = a.g.h[1] * a.g.h[2];
    a.g.square[1] = a.g.h[0] * a.g.h[2];
    a.g.square[2] = a.g.h[0] * a.g.h[1];
    a.g.inv_vol = 1.0 / (a.g.h[0] * a.g.h[1] * a.g.h[2]);
    for (int v = 0; v < 8; v++) a.g.inflow[v] = d->inflow[v];
    a.g.r_src = d->r_src;
    a.g.rho_src = d->rho_src;
    a.g.v_src = d->v_src;
    a.g.p_over_rho_src = d->p_over_rho_src;
    a.g.r_floor = d->r_floor;
    a.g.lz = choose_lz(a.g, sms, 0, 0);   // the handle path's z chunking (same tiles, same faces)
    a.clk = clk;
    a.st = st;
    a.cfl = o->cfl;
    a.n_disc = o->n_disc;

    noalloc_clock_init<<<1, 1, 0, s>>>(clk, st, *dt_io, *time_io);
    if (cudaGetLastError() != cudaSuccess) return SETB_ECUDA;
    double* cur = U;      // holds U^n
    double* other = W;
    for (int k = 0; k < nsteps; k++) {
        cudaError_t e;
        if (o->scheme == 2) {
            a.Uin = cur;
            a.Ubase = nullptr;
            a.Uout = other;
            a.finalize = 0;
            e = launch_stage_fp64(a, o->n_state, o->order, 0, true, s);
            if (e != cudaSuccess) return SETB_ECUDA;
            a.Uin = other;
            a.Ubase = cur;
            a.Uout = cur;
            a.finalize = 1;
            e = launch_stage_fp64(a, o->n_state, o->order, 1, false, s);
        } else {
            a.Uin = cur;
            a.Ubase = nullptr;
            a.Uout = other;
            a.finalize = 1;
            e = launch_stage_fp64(a, o->n_state, o->order, 0, true, s);
            double* t = cur;
            cur = other;
            other = t;
        }
        if (e != cudaSuccess) return SETB_ECUDA;
    }
    // an odd number of Euler steps ends in the scratch: copy the N cells of each plane back (the
    // scratch's plane padding holds whatever an earlier call left there; the caller's padding is
    // never written)
    if (cur != U && cudaMemcpy2DAsync(U, sizeof(double) * (size_t)var_stride, cur, sizeof(double) * (size_t)var_stride,
                                      sizeof(double) * (size_t)N, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return SETB_ECUDA;
    unsigned char hdr[sizeof(DevClock) + sizeof(DevStatus)];
    if (cudaMemcpyAsync(hdr, scratch, sizeof(hdr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return SETB_ECUDA;
    DevClock c;
    DevStatus st_h;
    std::memcpy(&c, hdr, sizeof(DevClock));
    std::memcpy(&st_h, hdr + sizeof(DevClock), sizeof(DevStatus));
    *dt_io = c.dt_cur;
    *time_io = c.time_all;
    if (diag) {
        diag->time_all = c.time_all;
        diag->dt_next = c.dt_cur;
        diag->dt_last = c.dt_last;
        diag->steps = c.steps;
        diag->n_negdens = (int64_t)st_h.n_negdens;
        diag->first_bad_cell = st_h.first_bad == ULLONG_MAX ? -1 : (int64_t)st_h.first_bad;
        diag->n_pfloor = (int64_t)st_h.n_pfloor;
        diag->n_wave_err = (int64_t)st_h.n_wave;
        diag->n_recon_err = (int64_t)st_h.n_recon;
        diag->n_fp64_redo = (int64_t)st_h.n_redo;
    }
    if (st_h.n_timeout) return SETB_ETIMEOUT;
    if (st_h.n_negdens) return SETB_ENEGDENS;
    if (st_h.n_wave) return SETB_EWAVES;
    if (st_h.n_recon) return SETB_ERECON;
    return SETB_OK;
}
