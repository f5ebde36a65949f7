/*
 * setb200.h -- C ABI of the B200-native ideal-MHD step (libsetb200.so).
 *
 * Drop-in boundary for SergeyMSU/SET's FCMHD solver module.  In the reference the boundary is
 * a set of Fortran modules: STORAGE (host arrays, SET_Fortran_Cuda_MHD/Storage_module.f90),
 * MY_CUDA (device arrays, Set_CUDA / CUDA_START_MGD / Send_data_to_Host,
 * SET_Fortran_Cuda_MHD/cuf_kernel.cuf) and Solvers (chlld, SET_Fortran_Cuda_MHD/Solvers.f90).
 * Every entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Every function returns int32_t status, SETB_OK (0) on success; nothing exits or traps.
 *   - Host arrays belong to the caller and are copied in and out; device state belongs to the
 *     handle and stays resident across setb_step calls.
 *   - Cell_par layout: the reference's Cell_par(16, N), Fortran column-major, i.e. 16 doubles
 *     per cell, primitive variables (rho, u, v, w, p, Bx, By, Bz, then 8 H-atom fluid values
 *     that this path carries through untouched).  B is in the reference's stored units: the
 *     solver uses b = B / sqrt(4*pi).  On a Cartesian grid cell (i, j, k) is column
 *     1 + i + nx*(j + ny*k).
 *   - A handle is used by one host thread at a time; each handle owns one CUDA stream.
 */
#ifndef SETB200_H
#define SETB200_H

#include <stdint.h>

#if defined(__GNUC__)
#define SETB_API __attribute__((visibility("default")))
#else
#define SETB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define SETB_OK 0
#define SETB_EINVAL 1     /* bad argument (size, pointer, option)                               */
#define SETB_ECUDA 2      /* CUDA runtime error                                                 */
#define SETB_ENOMEM 3     /* device allocation failed or HBM budget exceeded                    */
#define SETB_ENEGDENS 4   /* a cell update produced rho <= 0 (reference: print + STOP,
                             cuf_solvers.cuf:708-711); the cell keeps its stage input           */
#define SETB_EWAVES 5     /* no wave-fan region matched (reference: STOP, Solvers.f90:1816-1825) */
#define SETB_ERECON 6     /* reconstructed face density < 0 (reference: STOP, cuf_solvers.cuf:414-420) */
#define SETB_ETIMEOUT 7   /* a bounded device-side wait gave up                                 */
#define SETB_ENODEV 8     /* no usable CUDA device                                              */
#define SETB_ESIZE 9      /* size beyond a documented maximum                                   */
#define SETB_EIO 10       /* file I/O or format/sentinel error                                  */
#define SETB_EBUSY 11     /* request refused: queue full or admission budget exhausted          */

typedef struct setb_handle setb_handle;

/* ------------------------------------------------------------------ problem description
 * Uniform Cartesian grid (the reference's face-list geometry with implicit face lists).
 * Boundaries: ghost cells beyond x = hi[0] hold the fixed `inflow` primitive state; every other
 * outer boundary is zero-gradient.  Cells whose centre lies at r < r_src from the origin are
 * re-imposed after every stage with the source state rho = rho_src * (r_src / max(r, r_floor))^2,
 * radial speed v_src, p = p_over_rho_src * rho, B = 0 (the analogue of the inner boundary of
 * cuf_solvers.cuf:614-681).  r_src = 0 disables the source. */
typedef struct {
    int32_t nx, ny, nz;
    int32_t flags;          /* reserved, must be 0                                            */
    double lo[3], hi[3];    /* domain box                                                     */
    double inflow[8];       /* primitive (rho,u,v,w,p,Bx,By,Bz) beyond x = hi[0]              */
    double r_src, rho_src, v_src, p_over_rho_src, r_floor;
    double dt_init;         /* dt of the first step after init / set_state (reference: 2e-9,
                               cuf_kernel.cuf:758)                                            */
} setb_cart_desc;

/* Seeded initial condition: uniform LISM state with +-pert_amp relative perturbations of rho and
 * p drawn by SplitMix64 keyed by (seed, cell index); source state inside r_src. */
typedef struct {
    double lism[8];         /* unperturbed primitive state (rho,u,v,w,p,Bx,By,Bz)             */
    uint64_t seed;
    double pert_amp;
} setb_lism_ic;

/* Scheme options (the reference hard-codes them: metod/n_state = 2 at cuf_solvers.cuf:260,
 * n_disc = 0 at :267, TVD on, RK2 at cuf_kernel.cuf:847-877). */
typedef struct {
    int32_t n_state;    /* 3 HLLD, 2 HLLC, 1 HLL, 0 one-speed Lax (chlld n_state)            */
    int32_t n_disc;     /* chlld n_disc: 0, 1 or 2                                             */
    int32_t order;      /* 1 first order, 2 minmod reconstruction of rho,u,v,w,p              */
    int32_t scheme;     /* 1 forward Euler (CUF_MGD_grans/cells), 2 Heun RK2 (CUF_MGD_*_RK2)  */
    int32_t precision;  /* 0 plain FP64; 1 mixed (FP32 Riemann arithmetic, FP64 state,
                           compensated update, FP64 pressure recovery and dt)                 */
    int32_t reserved;   /* must be 0                                                          */
    double cfl;         /* dt_face = cfl * dist / (max(|SL|,|SR|) + |w|), dist = h/2; the
                           reference's literal is 0.2 (cuf_solvers.cuf:429)                   */
} setb_step_opts;

/* Counters and clocks of a handle (replaces the reference's printed diagnostics). */
typedef struct {
    double time_all;        /* dev_time_all: simulated time                                   */
    double dt_next;         /* time_step2: dt the next step will use                          */
    double dt_last;         /* time_step: dt the last step used                               */
    int64_t steps;          /* steps taken since init / set_state                             */
    int64_t n_negdens;      /* cell updates with rho <= 0                                     */
    int64_t first_bad_cell; /* 0-based cell index of the first such update, -1 if none        */
    int64_t n_pfloor;       /* pressure floors applied (p <= 0 -> 1e-7, cuf_solvers.cuf:777-779) */
    int64_t n_wave_err;     /* faces with no matching wave-fan region                         */
    int64_t n_recon_err;    /* faces with reconstructed rho < 0                               */
    int64_t n_fp64_redo;    /* mixed form: faces recomputed in FP64 after a positivity failure */
} setb_diag;

/* ------------------------------------------------------------------ scalar flux routine
 * Replaces: subroutine chlld(n_state, al, be, ge, w, qqq1, qqq2, dsl, dsp, dsc, qqq, n_disc)
 *           SET_Fortran_Cuda_MHD/Solvers.f90:1144-1147 (host+device).
 * Fortran calling convention (all by reference) so a bind(C) interface can call it directly.
 * n_disc may be NULL (the Fortran OPTIONAL argument, default 0).  Runs on the host. */
SETB_API int32_t setb_chlld(const int32_t* n_state, const double* al, const double* be, const double* ge,
                   const double* w, const double qqq1[8], const double qqq2[8], double* dsl,
                   double* dsp, double* dsc, double qqq[8], const int32_t* n_disc);

/* Batched chlld on the GPU: n independent faces, host arrays, each face k uses normal
 * normals[3k..3k+2], face speed w[k] (NULL = 0), states q1[8k..], q2[8k..]; writes qqq[8k..],
 * speeds[3k..] = (dsl, dsp, dsc) and flags[k] (0 ok, 1 wave-fan failure).
 * precision 0 = FP64 arithmetic, 1 = FP32 arithmetic (the mixed form's solver).
 * Replaces the per-face chlld call inside CUF_MGD_grans_RK2 (cuf_solvers.cuf:423-426). */
SETB_API int32_t setb_chlld_batch(int64_t n, int32_t n_state, int32_t n_disc, int32_t precision,
                         const double* normals, const double* w, const double* q1, const double* q2,
                         double* qqq, double* speeds, int32_t* flags);

/* ------------------------------------------------------------------ passive-scalar flux routine
 * Replaces: subroutine chlld_Q(n_state, al, be, ge, w, qqq1, qqq2, dsl, dsp, dsc, qqq, null_bn1,
 *           n_disc, p_correct_, konvect_, ydar_)   SET_Fortran_Cuda_MHD/Solvers.f90:198-201
 * chlld with a ninth, passively advected variable Q = qqq(9) and an optional second scalar.
 * Fortran calling convention (all by reference); the OPTIONAL arguments null_bn1, n_disc,
 * p_correct_, konvect_ and ydar_ may be NULL.  Fortran LOGICALs are passed as int32 (nonzero =
 * .TRUE.).  null_bn1 and p_correct_ are accepted and, as in the reference (:266-267), change
 * nothing.  konvect_ is the (3,1) array: [0], [1] the scalar's left / right values (in), [2] its
 * flux (out).  ydar_ = .TRUE. takes the left-state branch of the wave fan (:550, :698, :951).
 * Returns SETB_EWAVES where the reference prints and STOPs.  Runs on the host. */
SETB_API int32_t setb_chlld_q(const int32_t* n_state, const double* al, const double* be, const double* ge,
                     const double* w, const double qqq1[9], const double qqq2[9], double* dsl,
                     double* dsp, double* dsc, double qqq[9], const int32_t* null_bn1,
                     const int32_t* n_disc, const int32_t* p_correct_, double* konvect_,
                     const int32_t* ydar_);

/* Batched chlld_Q on the GPU (FP64): n faces, host arrays; face k uses normals[3k..3k+2], w[k]
 * (NULL = 0), q1[9k..], q2[9k..]; konvect (NULL = absent) holds 3 values per face, [3k], [3k+1]
 * in and [3k+2] out.  Writes qqq[9k..], speeds[3k..] = (dsl, dsp, dsc), flags[k] (0 ok, 1 no
 * wave-fan region matched). */
SETB_API int32_t setb_chlld_q_batch(int64_t n, int32_t n_state, int32_t n_disc, int32_t ydar,
                           const double* normals, const double* w, const double* q1, const double* q2,
                           double* konvect, double* qqq, double* speeds, int32_t* flags);

/* ------------------------------------------------------------------ device-resident solver
 * Replaces Set_CUDA (cuf_kernel.cuf:351-382): allocate device state and upload Cell_par. */
SETB_API int32_t setb_init_cartesian(setb_handle** h, const setb_cart_desc* d, const double* cell_par);

/* As setb_init_cartesian, but the seeded initial condition is generated on the device (no host
 * Cell_par, no host-to-device copy of the state). */
SETB_API int32_t setb_init_cartesian_lism(setb_handle** h, const setb_cart_desc* d, const setb_lism_ic* ic);

/* Host-side generator of the same seeded initial condition into a caller Cell_par(16,N);
 * columns 9..16 are left untouched. */
SETB_API int32_t setb_cart_fill_lism(const setb_cart_desc* d, const setb_lism_ic* ic, double* cell_par);

/* Replaces one pass of the CUDA_START_MGD time loop (cuf_kernel.cuf:780-925) for nsteps steps:
 * lagged dt, face fluxes computed once per face, owner-signed conservative update, Euler or
 * Heun RK2.  Runs asynchronously on the handle's stream when time_all is NULL; otherwise waits
 * and writes the simulated time.  Device-side errors are reported by setb_step's return value
 * when it waits, else by the next setb_status / setb_sync. */
SETB_API int32_t setb_step(setb_handle* h, int32_t nsteps, const setb_step_opts* o, double* time_all);

/* As setb_step (always waits), and times every kernel launch with CUDA events recorded on the
 * handle's stream between consecutive launches: kernel_ms[0] = total ms of the first-stage (or
 * Euler) kernels, kernel_ms[1] = total ms of the second-stage kernels; launches[0..1] = counts.
 * Replaces the reference's single event pair around the whole run (cuf_kernel.cuf:760-762,
 * 930-933). */
SETB_API int32_t setb_step_profiled(setb_handle* h, int32_t nsteps, const setb_step_opts* o,
                                    double* time_all, double kernel_ms[2], int32_t launches[2]);

/* Waits for the handle's stream and returns the first device-side error status (or SETB_OK). */
SETB_API int32_t setb_sync(setb_handle* h);

/* Replaces Send_data_to_Host (cuf_kernel.cuf:384-400): download Cell_par columns 1..8 (columns
 * 9..16 of the caller's array are left untouched) and the simulated time. */
SETB_API int32_t setb_get_state(setb_handle* h, double* cell_par, double* time_all);

/* Replaces Fill_data (Storage_module.f90:191-209) as a restart point: upload Cell_par columns
 * 1..8, set the simulated time, reset the lagged dt to dt_init and clear the counters. */
SETB_API int32_t setb_set_state(setb_handle* h, const double* cell_par, double time_all);

/* Copies the resident state, clock and counters of `src` into `dst` on the device (both handles
 * must describe the same grid); used to restart a solve from a stored initial state without a
 * host round trip.  Enqueued on dst's stream after waiting for src's. */
SETB_API int32_t setb_copy_state(setb_handle* dst, setb_handle* src);

/* Device pointers of the conserved state (rho, mx, my, mz, E, Bx, By, Bz), structure of arrays:
 * variable v of cell (i,j,k) is at base[v*var_stride + k*plane_stride + j*row_pitch + i]. */
SETB_API int32_t setb_state_view(setb_handle* h, double** base, int64_t* var_stride, int64_t* plane_stride,
                        int64_t* row_pitch);

/* Downloads the conserved state (rho, mx, my, mz, E, Bx, By, Bz) as 8 packed host planes of
 * N = nx*ny*nz doubles (U[v*N + cell]), the layout the device holds it in. */
SETB_API int32_t setb_get_conserved(setb_handle* h, double* U);

/* Counters and clocks (replaces the reference's prints). Waits for the handle's stream. */
SETB_API int32_t setb_status(setb_handle* h, setb_diag* out);

/* No counterpart in the reference (its kernels have no device-side waits).  Sets how long the
 * handle's stage kernels wait for a plane copy (the tensor copy that stages each z plane into
 * shared memory) before they count the wait as run out: cycles > 0 is the limit in SM clock
 * cycles, 0 restores the default (~2 s), cycles < 0 makes every wait a single non-blocking check
 * (used by tests to drive the error path).  A wait that runs out is reported as SETB_ETIMEOUT by
 * the next call that reads the counters (setb_step with time_all, setb_sync, setb_status); the
 * kernel then gives the copy a second ~2 s wait before it reads the plane, and a copy that never
 * lands switches that thread to plain loads, so the state stays valid.  setb_set_state clears the
 * counters. */
SETB_API int32_t setb_set_copy_wait(setb_handle* h, int64_t cycles);

/* The CUDA stream the handle launches on (as a void* cudaStream_t). */
SETB_API int32_t setb_stream(setb_handle* h, void** stream);

/* ------------------------------------------------------------------ z slabs (one grid on many GPUs)
 * The Cartesian grid d split along z, one slab per rank: the reference runs one grid on one GPU
 * (cuf_kernel.cuf:780-925); this is the multi-GPU form of the same step.  A slab handle owns
 * planes [k0, k0 + nz_local) of d (global sizes, nz_local >= 2) and holds two ghost planes below
 * and above them: buffer planes 0, 1 | owned 2 .. nz_local+1 | nz_local+2, nz_local+3.  One time
 * step is driven stage by stage on the handle's stream:
 *   1. fill the ghost planes of the stage-1 input (setb_slab_view(h, 1, ...)) from the
 *      neighbours' owned edge planes; setb_slab_stage(h, 1, o);
 *   2. (Heun) fill the ghost planes of the stage-2 input (setb_slab_view(h, 2, ...));
 *      setb_slab_stage(h, 2, o);
 *   3. replace the next step's dt (setb_slab_dt) by its minimum over all slabs.
 * Ghost planes beyond the grid's z ends are filled by setb_slab_stage itself (copies of the end
 * plane, the zero-gradient boundary).  With those exchanges the slabs reproduce the single-grid
 * setb_step bit for bit.  setb_get_state / setb_set_state / setb_get_conserved / setb_status /
 * setb_destroy work on a slab handle (state transfers cover the owned planes; the first bad cell
 * is a whole-grid index); setb_step refuses one (SETB_EINVAL).  Diagnostic counters count the two
 * faces on a slab boundary in both slabs. */
SETB_API int32_t setb_init_slab(setb_handle** h, const setb_cart_desc* d, int32_t k0, int32_t nz_local,
                                const double* cell_par /* 16 x (nx*ny*nz_local), owned planes */);
/* Enqueues stage 1 (Euler step or Heun stage 1, with the dt candidate) or stage 2 (Heun stage 2,
 * rolls the clock) on the handle's stream; Euler steps are stage 1 alone. */
SETB_API int32_t setb_slab_stage(setb_handle* h, int32_t stage, const setb_step_opts* o);
/* The device buffer a stage reads (conserved SoA: variable v, buffer plane k, row j, column i at
 * base[v*var_stride + k*plane_stride + j*row_pitch + i]; row_pitch as setb_state_view) and its
 * plane count nz_local + 4.  The buffers swap roles after an Euler step. */
SETB_API int32_t setb_slab_view(setb_handle* h, int32_t stage, double** base, int64_t* var_stride,
                                int64_t* plane_stride, int32_t* nz_buffer);
/* Device address of the dt the next step uses (one double), for a minimum over the slabs after
 * each step (e.g. an in-place NCCL all-reduce with op min on the handle's stream). */
SETB_API int32_t setb_slab_dt(setb_handle* h, double** dt_next);

SETB_API int32_t setb_destroy(setb_handle* h);

/* ------------------------------------------------------------------ face-list grids
 * The reference's own geometry: an explicit list of cells and faces, as Set_CUDA uploads it
 * (cuf_kernel.cuf:351-382) from the STORAGE arrays (Storage_module.f90:20-37), in their Fortran
 * layouts and 1-based numbering:
 *   cell_par     Cell_par(16,N)         primitive state, columns 1..8 used
 *   cell_center  Cell_center(3,N)       cell_volume  Cell_Volume(N)
 *   cell_gran    Cell_gran(6,N)         face numbers of each cell, 0 = none
 *   gran_normal  Gran_normal(3,G)       unit normal, pointing from neighbour 1 to neighbour 2
 *   gran_square  Gran_square(G)         face area
 *   gran_center  Gran_center(3,G)
 *   gran_neighbour      Gran_neighbour(2,G)      cells on each side; neighbour 2 = -1 on a wall
 *   gran_neighbour_tvd  Gran_neighbour_TVD(2,G)  far cells of the TVD stencil, -1 = none
 *   gran_type    Gran_type(G)           1 other, 2 ordinary (a wall when neighbour 2 is -1),
 *                                       3 inner sphere, 4 outer boundary (ghost = cell with its
 *                                       normal velocity clamped to <= -0.1), 5 axis (ghost =
 *                                       cell with v mirrored)  (cuf_solvers.cuf:318-345)
 * The flux of a face is computed once per stage and added to neighbour 1 and subtracted from
 * neighbour 2 (cuf_solvers.cuf:691-703).  A handle made here is driven by setb_step,
 * setb_step_profiled, setb_get_state, setb_set_state, setb_get_conserved, setb_status and
 * setb_destroy like a Cartesian one; it supports precision 0 (plain FP64).  Indices are checked
 * on the host: an index outside its array, a non-positive volume or an unknown face type gives
 * SETB_EINVAL.  The library stores cells in its own locality order (Morton order of the centres,
 * faces by their first cell); every state transfer and the first-bad-cell index use the
 * caller's numbering, only setb_state_view exposes the internal order. */
typedef struct {
    double r_src, rho_src, v_src, p_over_rho_src, r_floor;   /* source sphere, r_src 0 = none  */
    double dt_init;             /* dt of the first step (reference: 2e-9, cuf_kernel.cuf:758)    */
    double face_skip_radius;    /* faces whose neighbour-1 centre is nearer the origin than this
                                   keep their previous flux (reference: 0.02, cuf_solvers.cuf:284);
                                   0 = none                                                      */
    double cell_freeze_radius;  /* cells nearer the origin are not updated (reference: 0.05,
                                   cuf_solvers.cuf:611); 0 = none                                */
    int32_t physics;            /* 0: conservative 3D ideal MHD of all 8 variables.
                                   1: the reference's live cell update, 2D axisymmetric hydro
                                   about the x axis (cuf_solvers.cuf:561-794): rr(2) = y is the
                                   radius, geometric terms rho*v/y..., w = B = 0, charge exchange
                                   with the two H-atom fluids of Cell_par columns 9..16
                                   (Source_MK, cuf_kernel.cuf:215-288), the v clamp near the
                                   axis (:783-785) and the Lax flux on near-axis faces
                                   (cuf_solvers.cuf:293-295).  Cell centres need y > 0.          */
    int32_t powell;             /* physics 0 only.  0: off (the reference: Gran_POTOK(9) = 0,
                                   cuf_solvers.cuf:433).  1: the reference's div-B terms, commented
                                   out there (cuf_solvers.cuf:433, 529-533, 729-733): face flux
                                   Gran_POTOK(9) = 0.5 n.(B1 + B2) * square, sks = its owner-signed
                                   sum over the cell's faces, sources -(B/4pi) sks on the momentum
                                   and -u sks on B (in the flux sum, before the division by the
                                   volume), u and B of the stage input.  2: as 1 plus Powell's
                                   energy source -(u.B/4pi) sks.                                 */
} setb_fl_params;

/* Replaces Set_CUDA for the reference's grid (cuf_kernel.cuf:351-382). */
SETB_API int32_t setb_init_facelist(setb_handle** h, int32_t n_cell, int32_t n_gran, const double* cell_par,
                                    const double* cell_center, const double* cell_volume, const int32_t* cell_gran,
                                    const double* gran_normal, const double* gran_square, const double* gran_center,
                                    const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd,
                                    const int32_t* gran_type, const setb_fl_params* params);

/* ------------------------------------------------------------------ on-disk formats
 * The grid/state stream file the reference's grid generator writes (SET_Gelios/source/
 * Setka.cpp:1158-1567) and its FCMHD host reads (Set_Storage, Storage_module.f90:42-100):
 * unformatted stream, no record markers, native byte order:
 *   real(8) time_all, integer(4) N_cell, integer(4) N_gran, Cell_par(16,N), Cell_center(3,N),
 *   Cell_Volume(N), integer(4) Cell_gran(6,N), Gran_normal(3,G), Gran_square(G), Gran_center(3,G),
 *   integer(4) Gran_neighbour(2,G), integer(4) Gran_neighbour_TVD(2,G), real(8) 121.0,
 *   integer(4) Gran_type(G), real(8) 122.0, Gran_POTOK(9,G), real(8) 123.0
 * and the checkpoint of Save_Storage / Fill_data (Storage_module.f90:160-209):
 *   real(8) time_all, Cell_par(16,N), real(8) 321.0
 * A short file, a wrong sentinel, trailing bytes or counts that differ from the caller's give
 * SETB_EIO (the reference printed the sentinel and went on). */
SETB_API int32_t setb_fcmhd_read_header(const char* path, double* time_all, int32_t* n_cell, int32_t* n_gran);
/* Reads the whole file into caller buffers sized for n_cell / n_gran (from the header);
 * gran_potok (9*G doubles) may be NULL to skip the stored fluxes. */
SETB_API int32_t setb_fcmhd_read(const char* path, int32_t n_cell, int32_t n_gran, double* time_all, double* cell_par,
                                 double* cell_center, double* cell_volume, int32_t* cell_gran, double* gran_normal,
                                 double* gran_square, double* gran_center, int32_t* gran_neighbour,
                                 int32_t* gran_neighbour_tvd, int32_t* gran_type, double* gran_potok);
/* Writes the file; gran_potok NULL writes zero fluxes, as the grid generator does. */
SETB_API int32_t setb_fcmhd_write(const char* path, double time_all, int32_t n_cell, int32_t n_gran,
                                  const double* cell_par, const double* cell_center, const double* cell_volume,
                                  const int32_t* cell_gran, const double* gran_normal, const double* gran_square,
                                  const double* gran_center, const int32_t* gran_neighbour,
                                  const int32_t* gran_neighbour_tvd, const int32_t* gran_type, const double* gran_potok);
/* Replaces Save_Storage / Fill_data (Storage_module.f90:160-209). */
SETB_API int32_t setb_checkpoint_write(const char* path, double time_all, int32_t n_cell, const double* cell_par);
SETB_API int32_t setb_checkpoint_read(const char* path, int32_t n_cell, double* time_all, double* cell_par);

/* ------------------------------------------------------------------ batched solves
 * No counterpart in the reference (one grid per process, cuf_kernel.cuf:351-382).  A batch
 * advances many Cartesian solves of uneven size together: every step is two persistent launches
 * whose CTAs draw 32x8xlz tiles of all active solves from one work queue; each solve keeps its own
 * lagged dt and clock, so a solve's results do not depend on what else is in the batch.  Solves
 * are admitted by HBM footprint and can be added or removed between steps (continuous batching).
 * Supported per solve: n_state 2 (HLLC) or 3 (HLLD), order 2, scheme 2, the batch's precision. */
typedef struct setb_batch setb_batch;

SETB_API int32_t setb_batch_create(setb_batch** b, int32_t max_slots, int32_t precision, int64_t hbm_budget_bytes);
/* Admits one solve (seeded initial condition generated on the device); SETB_EBUSY when no slot
 * is free or its footprint would exceed the budget. */
SETB_API int32_t setb_batch_add(setb_batch* b, const setb_cart_desc* d, const setb_lism_ic* ic,
                                const setb_step_opts* o, int32_t* slot);
SETB_API int32_t setb_batch_remove(setb_batch* b, int32_t slot);
/* Advances every active solve by nsteps (asynchronous; chunks of steps replay a CUDA graph). */
SETB_API int32_t setb_batch_step(setb_batch* b, int32_t nsteps);
/* Steady-state check: rel_change[slot] = sum|rho - rho_prev| / sum|rho| since the previous check
 * of that solve (fixed-order, deterministic reduction), -1 on a solve's first check or for free
 * slots; then rho_prev = rho.  rel_change has max_slots entries.  Waits for the batch. */
SETB_API int32_t setb_batch_check(setb_batch* b, double* rel_change);
SETB_API int32_t setb_batch_get_conserved(setb_batch* b, int32_t slot, double* U);
SETB_API int32_t setb_batch_status(setb_batch* b, int32_t slot, setb_diag* out);
SETB_API int32_t setb_batch_info(setb_batch* b, int64_t* bytes_used, int32_t* active, int32_t* lz, int32_t* grid);
/* Tiling of the batch launches: z-march length lz and persistent CTAs per SM slot multiplier. */
SETB_API int32_t setb_batch_set_tiling(setb_batch* b, int32_t lz, int32_t grid_mult);
/* Autotuner: times `reps` first-stage launches (idempotent on the state) for each candidate
 * tiling on the current membership, keeps the fastest. */
SETB_API int32_t setb_batch_tune(setb_batch* b, int32_t reps, int32_t* lz, int32_t* grid_mult, double* ms);
SETB_API int32_t setb_batch_sync(setb_batch* b);
SETB_API int32_t setb_batch_destroy(setb_batch* b);

/* ------------------------------------------------------------------ solve server
 * No counterpart in the reference.  Continuous batching on one GPU: a server thread owns a batch;
 * requests submitted from any thread are admitted in arrival order, between chunks of
 * `check_every` steps, while their HBM footprint fits the budget; every chunk advances all
 * admitted solves together, runs the steady-state check and retires the solves that reached
 * steady_tol or max_steps.  Destroying the server finishes the admitted and queued solves. */
typedef struct setb_server setb_server;

typedef struct {
    setb_cart_desc desc;
    setb_lism_ic ic;
    setb_step_opts opts;    /* n_state 2 or 3, order 2, scheme 2, the server's precision     */
    int32_t max_steps;      /* step cap, applied at chunk granularity                          */
    int32_t reserved;
    double steady_tol;      /* stop when sum|rho - rho_prev|/sum|rho| between checks < tol (0: off) */
    double* result_U;       /* optional host buffer of 8*N doubles for the final conserved state */
} setb_request;

typedef struct {
    int64_t id;
    int32_t status;         /* SETB_OK, or the error that ended the solve                       */
    int32_t steps;
    int32_t converged;      /* 1 when stopped by steady_tol                                     */
    int32_t reserved;
    double last_change;
    double time_all;
    double t_submit, t_admit, t_done;   /* seconds on the server's steady clock                 */
    setb_diag diag;
} setb_result;

SETB_API int32_t setb_server_create(setb_server** s, int32_t max_slots, int32_t precision, int64_t hbm_budget,
                                    int32_t check_every);
SETB_API int32_t setb_server_submit(setb_server* s, const setb_request* r, int64_t* id);
/* Waits up to timeout_s seconds for request `id`; SETB_ETIMEOUT when it is not done. */
SETB_API int32_t setb_server_wait(setb_server* s, int64_t id, setb_result* out, double timeout_s);
/* Results in completion order not yet polled (at most max). */
SETB_API int32_t setb_server_poll(setb_server* s, setb_result* out, int32_t max, int32_t* n);
SETB_API int32_t setb_server_stats(setb_server* s, int32_t* pending, int32_t* active, int64_t* completed,
                                   int64_t* failed, int32_t* max_active);
SETB_API int32_t setb_server_destroy(setb_server* s);

/* No counterpart in the reference.  A variant of setb_step that allocates nothing, for callers
 * that cannot let a library allocate device memory: hosts that already own the state in their
 * own device arrays (a CUDA Fortran host's `device` allocatables) or that reserve HBM up front in
 * their own arena, where a cudaMalloc inside the library could synchronise the device or take
 * memory promised elsewhere.  The caller passes the conserved state it owns: U is a device
 * pointer to 8 planes (rho, mx, my, mz, E, Bx, By, Bz), plane v at U + v*var_stride, each plane
 * nx*ny*nz doubles with x fastest; it is advanced in place by nsteps steps of `o`.  *dt_io is the
 * dt of the first step on entry (desc->dt_init on a fresh run; desc->dt_init is not used) and the
 * dt of the next step on return; *time_io is the simulated time in and out; diag may be NULL.
 * Runs on `stream` (NULL: the legacy default stream) and is synchronous: it returns after the
 * steps have finished and the clock and counters have been read back.  Arguments are checked as
 * setb_init_cartesian and setb_step check them (precision must be 0).
 *
 * The scratch (the Heun stage buffer, the device clock, the error counters) is one fixed
 * file-scope device array of 16 MiB + 256 B that every GPU loading the library holds until the
 * process exits.  Limit: var_stride <= 262144 (64^3 cells); larger sizes return SETB_ESIZE.
 * Every call shares that array and it keeps the last call's contents: the clock and counters are
 * cleared at the start of each call, and calls that overlap on the GPU (other threads, other
 * streams) race on it.  The first call on a device resolves the array's device address with
 * cudaGetSymbolAddress (once per device, with that device current); make that first call before
 * any stream capture.  No cudaMalloc, cudaFree or other allocating routine is called. */
SETB_API int32_t setb_step_noalloc(const setb_cart_desc* d, const setb_step_opts* o, double* U,
                                   int64_t var_stride, int32_t nsteps, double* dt_io, double* time_io,
                                   setb_diag* diag, void* stream);

SETB_API const char* setb_strerror(int32_t code);

/* Library version, e.g. 100 for 1.0.0. */
SETB_API int32_t setb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SETB200_H */
