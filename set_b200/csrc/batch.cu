// batch.cu -- many Cartesian solves of uneven size advanced together (ensemble / continuous
// batching).  The reference runs one grid per process (cuf_kernel.cuf:351-382); this is new.
//
// * Slots: each admitted solve owns its state (two FP64 buffers, the mixed form's FP32
//   compensation, a density snapshot for steady-state checks) allocated stream-ordered on the
//   batch stream, so admitting or retiring a solve never synchronises the device.  Admission is
//   by HBM footprint against a byte budget.
// * A step is two persistent launches per Riemann solver in use (Heun stages; HLLD solves and
//   HLLC solves in separate launches, so each kernel holds one solver body) whose CTAs draw
//   32x7xlz tiles of those solves from one work-queue counter; each solve counts its own tiles,
//   so each keeps its own lagged dt and clock.  While membership is unchanged the launch sequence of a chunk of steps
//   is replayed from a captured CUDA graph.
// * The z-march length lz and the persistent grid size are chosen by an autotuner that times
//   first-stage launches (idempotent: they read U^n and write the stage buffer only).
// * Steady-state checks reduce |rho - rho_prev| per solve in a fixed order (deterministic), so a
//   solve's trajectory and stopping step are the same alone and in any mix.
#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "setb200.h"
#include "setb_internal.cuh"

using namespace sb;

namespace {

constexpr int kCheckBlocks = 64;     // fixed partial count per solve: deterministic reduction
constexpr int kMaxGraphSteps = 64;   // steps captured in one graph

struct Slot {
    bool active = false;
    setb_cart_desc desc{};
    setb_step_opts opts{};
    GridGeom g{};
    char* mem = nullptr;     // one stream-ordered allocation per slot
    size_t bytes = 0;
    double* U = nullptr;
    double* W = nullptr;
    float* comp = nullptr;
    double* rho_prev = nullptr;
    DevClock* clk = nullptr;
    DevStatus* st = nullptr;
    CUtensorMap* tmap = nullptr;   // [U, W] for the batch's tile shape
    long long steps = 0;
    bool have_prev = false;
};

__global__ void check_partial_kernel(const double* const* rho, double* const* prev, const long long* ncell,
                                     double* partial) {
    // block (b, s): cells [b*chunk, (b+1)*chunk) of solve s, fixed-order tree reduction
    const int s = blockIdx.y, b = blockIdx.x;
    const long long N = ncell[s];
    const long long chunk = (N + kCheckBlocks - 1) / kCheckBlocks;
    const long long c0 = b * chunk, c1 = min(N, c0 + chunk);
    double d = 0.0, a = 0.0;
    for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const double r = rho[s][c];
        d += fabs(r - prev[s][c]);
        a += fabs(r);
        prev[s][c] = r;
    }
    __shared__ double sd[256], sa[256];
    sd[threadIdx.x] = d;
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sd[threadIdx.x] += sd[threadIdx.x + o];
            sa[threadIdx.x] += sa[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * (s * kCheckBlocks + b)] = sd[0];
        partial[2 * (s * kCheckBlocks + b) + 1] = sa[0];
    }
}

__global__ void check_final_kernel(const double* partial, int nsolves, double* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsolves) return;
    double d = 0.0, a = 0.0;
    for (int b = 0; b < kCheckBlocks; b++) {
        d += partial[2 * (s * kCheckBlocks + b)];
        a += partial[2 * (s * kCheckBlocks + b) + 1];
    }
    out[s] = a > 0.0 ? d / a : 0.0;
}

}  // namespace

struct setb_batch {
    int device = 0;
    int precision = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    int64_t budget = 0, used = 0;
    std::vector<Slot> slots;
    // device arrays
    StageArgs* d_inst1 = nullptr;
    StageArgs* d_inst2 = nullptr;
    StageArgs* h_inst = nullptr;   // pinned staging [2 * max_slots]
    int4* d_items = nullptr;
    int4* h_items = nullptr;       // pinned
    size_t items_cap = 0;
    int n_items = 0;               // work items: HLLD solves' [0, n_hlld), HLLC solves' [n_hlld, n_items)
    int n_hlld = 0;
    unsigned* d_queue = nullptr;   // 4 * kMaxGraphSteps counters (2 stages x 2 solvers per step)
    double* d_partial = nullptr;
    double* d_check = nullptr;
    const double** d_rho = nullptr;
    double** d_prev = nullptr;
    long long* d_ncell = nullptr;
    void* h_check_args = nullptr;  // pinned staging for the check kernel arguments
    double* h_check = nullptr;
    // tuning
    int lz = 32;
    int grid_mult = 1;
    // graph cache
    bool dirty = true;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
};

namespace {

#define SB_TRY(expr)                              \
    do {                                          \
        cudaError_t e_ = (expr);                  \
        if (e_ != cudaSuccess) return SETB_ECUDA; \
    } while (0)

// U, W, rho_prev, compensation, then clock (256 B), counters (256 B) and two tensor maps.
size_t slot_bytes(const GridGeom& g) {
    return 2 * sizeof(double) * 8 * (size_t)g.vs + sizeof(float) * 8 * (size_t)g.vs + sizeof(double) * (size_t)g.vs +
           512 + 2 * sizeof(CUtensorMap);
}

GridGeom geom_of(const setb_cart_desc* d) {
    GridGeom g{};
    g.nx = d->nx;
    g.ny = d->ny;
    g.nz = d->nz;
    set_device_strides(g);
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

void drop_graph(setb_batch* b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->graph_steps = 0;
}

// Rebuilds the per-slot stage arguments and the work list (largest solves first).
int rebuild(setb_batch* b) {
    const int ms = (int)b->slots.size();
    std::vector<std::pair<long long, int>> order;
    for (int s = 0; s < ms; s++)
        if (b->slots[s].active) order.push_back({(long long)b->slots[s].g.nx * b->slots[s].g.ny * b->slots[s].g.nz, s});
    std::sort(order.begin(), order.end(), [](auto& x, auto& y) { return x.first > y.first || (x.first == y.first && x.second < y.second); });
    // HLLD solves first, then HLLC solves, each largest first: one launch per solver and stage
    std::stable_partition(order.begin(), order.end(), [&](const std::pair<long long, int>& o) {
        return b->slots[o.second].opts.n_state == 3;
    });
    std::vector<int4> items;
    int n_hlld = 0;
    for (auto& os : order) {
        const int s = os.second;
        Slot& sl = b->slots[s];
        GridGeom g = sl.g;
        g.lz = std::min(b->lz, g.nz);
        const int ty = tile_shape(b->precision, kBatchKind).ty;
        const int ntx = (g.nx + kTileX - 1) / kTileX, nty = (g.ny + ty - 1) / ty, ntz = (g.nz + g.lz - 1) / g.lz;
        for (int bz = 0; bz < ntz; bz++)
            for (int by = 0; by < nty; by++)
                for (int bx = 0; bx < ntx; bx++) items.push_back(make_int4(s, bx, by, bz));
        if (sl.opts.n_state == 3) n_hlld = (int)items.size();
        for (int st = 0; st < 2; st++) {
            StageArgs a{};
            a.g = g;
            a.clk = sl.clk;
            a.st = sl.st;
            a.cfl = sl.opts.cfl;
            a.n_disc = sl.opts.n_disc;
            a.n_state = sl.opts.n_state;
            a.total_tiles = (unsigned)(ntx * nty * ntz);
            if (st == 0) {
                a.Uin = sl.U;
                a.tm_in = sl.tmap;
                a.Ubase = nullptr;
                a.Uout = sl.W;
                a.finalize = 0;
                a.comp = nullptr;
            } else {
                a.Uin = sl.W;
                a.tm_in = sl.tmap ? sl.tmap + 1 : nullptr;
                a.Ubase = sl.U;
                a.Uout = sl.U;
                a.finalize = 1;
                a.comp = b->precision ? sl.comp : nullptr;
            }
            b->h_inst[st * ms + s] = a;
        }
    }
    if (items.size() > b->items_cap) {
        if (b->d_items) cudaFreeAsync(b->d_items, b->stream);
        if (b->h_items) cudaFreeHost(b->h_items);
        b->items_cap = std::max<size_t>(items.size(), 2 * b->items_cap);
        if (cudaMallocAsync(&b->d_items, sizeof(int4) * b->items_cap, b->stream) != cudaSuccess ||
            cudaMallocHost(&b->h_items, sizeof(int4) * b->items_cap) != cudaSuccess) {
            cudaGetLastError();
            b->items_cap = 0;
            return SETB_ENOMEM;
        }
    }
    SB_TRY(cudaStreamSynchronize(b->stream));   // pinned staging buffers are about to be rewritten
    if (!items.empty()) std::memcpy(b->h_items, items.data(), sizeof(int4) * items.size());
    b->n_items = (int)items.size();
    b->n_hlld = n_hlld;
    if (b->n_items) SB_TRY(cudaMemcpyAsync(b->d_items, b->h_items, sizeof(int4) * items.size(), cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(b->d_inst1, b->h_inst, sizeof(StageArgs) * ms, cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(b->d_inst2, b->h_inst + ms, sizeof(StageArgs) * ms, cudaMemcpyHostToDevice, b->stream));
    drop_graph(b);
    b->dirty = false;
    return SETB_OK;
}

int grid_size(const setb_batch* b, int n_items) {
    const int g = b->sm_count * batch_ctas_per_sm(b->precision) * b->grid_mult;
    return std::max(1, std::min(g, std::max(n_items, 1)));
}

// Launches one stage over the work items of one solver (n_state 3: HLLD solves, 2: HLLC solves)
// with queue counter q.
int launch_items(setb_batch* b, int stage, int n_state, unsigned* q) {
    const int first = n_state == 3 ? 0 : b->n_hlld;
    const int n = n_state == 3 ? b->n_hlld : b->n_items - b->n_hlld;
    if (n == 0) return SETB_OK;
    BatchArgs a{stage == 1 ? b->d_inst1 : b->d_inst2, b->d_items + first, n, q};
    SB_TRY(launch_batch_stage(a, b->precision, n_state, stage == 1 ? 0 : 1, stage == 1, grid_size(b, n), b->stream));
    return SETB_OK;
}

// Enqueues nsteps (<= kMaxGraphSteps) steps: one memset of the queue counters, then per step and
// stage one launch per solver that has solves, each with its own counter.
int enqueue(setb_batch* b, int nsteps) {
    SB_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned) * 4 * nsteps, b->stream));
    for (int s = 0; s < nsteps; s++) {
        unsigned* q = b->d_queue + 4 * s;
        int rc;
        if ((rc = launch_items(b, 1, 3, q)) || (rc = launch_items(b, 1, 2, q + 1)) ||
            (rc = launch_items(b, 2, 3, q + 2)) || (rc = launch_items(b, 2, 2, q + 3)))
            return rc;
    }
    return SETB_OK;
}

int run_steps(setb_batch* b, int nsteps) {
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    if (b->n_items == 0) return SETB_OK;
    while (nsteps > 0) {
        const int chunk = std::min(nsteps, kMaxGraphSteps);
        if (chunk >= 8) {   // graph replay; one graph (of the last chunk length) is cached
            if (!b->graph || b->graph_steps != chunk) {
                drop_graph(b);
                cudaGraph_t gr = nullptr;
                SB_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                int rc = enqueue(b, chunk);
                cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
                if (rc || e != cudaSuccess) {
                    if (gr) cudaGraphDestroy(gr);
                    cudaGetLastError();
                    return rc ? rc : SETB_ECUDA;
                }
                e = cudaGraphInstantiate(&b->graph, gr, 0);
                cudaGraphDestroy(gr);
                if (e != cudaSuccess) return SETB_ECUDA;
                b->graph_steps = chunk;
            }
            SB_TRY(cudaGraphLaunch(b->graph, b->stream));
        } else {
            int rc = enqueue(b, chunk);
            if (rc) return rc;
        }
        nsteps -= chunk;
    }
    return SETB_OK;
}

void free_slot(setb_batch* b, Slot& s) {
    if (s.mem) cudaFreeAsync(s.mem, b->stream);
    b->used -= (int64_t)s.bytes;
    s = Slot();
}

}  // namespace

extern "C" {

int32_t setb_batch_create(setb_batch** out, int32_t max_slots, int32_t precision, int64_t hbm_budget) {
    if (!out || max_slots < 1 || max_slots > 65536 || precision < 0 || precision > 2 || hbm_budget <= 0)
        return SETB_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SETB_ENODEV;
    setb_batch* b = new (std::nothrow) setb_batch();
    if (!b) return SETB_ENOMEM;
    cudaGetDevice(&b->device);
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, b->device);
    b->sm_count = prop.multiProcessorCount;
    b->precision = precision;
    b->budget = hbm_budget;
    b->slots.resize(max_slots);
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              prepare_batch_kernels(precision) == cudaSuccess &&
              cudaMalloc(&b->d_inst1, sizeof(StageArgs) * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_inst2, sizeof(StageArgs) * max_slots) == cudaSuccess &&
              cudaMallocHost(&b->h_inst, sizeof(StageArgs) * 2 * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_queue, sizeof(unsigned) * 4 * kMaxGraphSteps) == cudaSuccess &&
              cudaMalloc(&b->d_partial, sizeof(double) * 2 * kCheckBlocks * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_check, sizeof(double) * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_rho, sizeof(double*) * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_prev, sizeof(double*) * max_slots) == cudaSuccess &&
              cudaMalloc(&b->d_ncell, sizeof(long long) * max_slots) == cudaSuccess &&
              cudaMallocHost(&b->h_check_args, (sizeof(double*) * 2 + sizeof(long long)) * max_slots) == cudaSuccess &&
              cudaMallocHost(&b->h_check, sizeof(double) * std::max(max_slots, 8)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        setb_batch_destroy(b);
        return SETB_ENOMEM;
    }
    std::memset(b->h_inst, 0, sizeof(StageArgs) * 2 * max_slots);
    *out = b;
    return SETB_OK;
}

int32_t setb_batch_add(setb_batch* b, const setb_cart_desc* d, const setb_lism_ic* ic, const setb_step_opts* o,
                       int32_t* slot) {
    if (!b || !d || !ic || !o || !slot) return SETB_EINVAL;
    *slot = -1;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->flags != 0 || !(d->dt_init > 0.0)) return SETB_EINVAL;
    if ((o->n_state != 2 && o->n_state != 3) || o->order != 2 || o->scheme != 2 || o->precision != b->precision ||
        o->reserved != 0 || !(o->cfl > 0.0) || o->n_disc < 0 || o->n_disc > 2 || (o->precision == 2 && o->n_disc != 0))
        return SETB_EINVAL;
    cudaSetDevice(b->device);
    int s = -1;
    for (int i = 0; i < (int)b->slots.size(); i++)
        if (!b->slots[i].active) {
            s = i;
            break;
        }
    if (s < 0) return SETB_EBUSY;
    Slot sl;
    sl.desc = *d;
    sl.opts = *o;
    sl.g = geom_of(d);
    sl.bytes = slot_bytes(sl.g);
    if (b->used + (int64_t)sl.bytes > b->budget) return SETB_EBUSY;
    if (cudaMallocAsync((void**)&sl.mem, sl.bytes, b->stream) != cudaSuccess) {
        cudaGetLastError();
        return SETB_ENOMEM;
    }
    const size_t vs = (size_t)sl.g.vs;
    char* p = sl.mem;
    sl.U = reinterpret_cast<double*>(p);
    p += sizeof(double) * 8 * vs;
    sl.W = reinterpret_cast<double*>(p);
    p += sizeof(double) * 8 * vs;
    sl.rho_prev = reinterpret_cast<double*>(p);
    p += sizeof(double) * vs;
    sl.comp = reinterpret_cast<float*>(p);
    p += sizeof(float) * 8 * vs;
    sl.clk = reinterpret_cast<DevClock*>(p);
    sl.st = reinterpret_cast<DevStatus*>(p + 256);
    sl.tmap = reinterpret_cast<CUtensorMap*>(p + 512);
    CUtensorMap tm[2] = {};
    const int ty = tile_shape(b->precision, kBatchKind).ty;
    if (encode_state_tmap(sl.g, sl.U, ty, &tm[0]) != SETB_OK || encode_state_tmap(sl.g, sl.W, ty, &tm[1]) != SETB_OK) {
        sl.tmap = nullptr;   // plain loads for this solve
    }
    // initial condition, clock, counters, compensation (all stream-ordered, no host sync)
    double* dl = sl.W;   // 8 doubles of scratch for the LISM vector
    DevClock c{};
    c.dt_cur = d->dt_init;
    double reset = kDtReset;
    std::memcpy(&c.dt_next, &reset, sizeof(double));
    DevStatus st{};
    st.first_bad = ULLONG_MAX;
    SB_TRY(cudaStreamSynchronize(b->stream));   // the pinned staging area is reused below
    std::memcpy(b->h_check, ic->lism, sizeof(double) * 8);   // h_check holds >= 8 doubles
    SB_TRY(cudaMemsetAsync(sl.U, 0, sizeof(double) * 8 * vs, b->stream));   // zero row padding
    SB_TRY(cudaMemcpyAsync(dl, b->h_check, sizeof(double) * 8, cudaMemcpyHostToDevice, b->stream));
    SB_TRY(launch_lism_init(sl.g, dl, ic->seed, ic->pert_amp, sl.U, b->stream));
    if (sl.tmap) SB_TRY(cudaMemcpyAsync(sl.tmap, tm, sizeof(tm), cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(sl.clk, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(sl.st, &st, sizeof(st), cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemsetAsync(sl.comp, 0, sizeof(float) * 8 * vs, b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    sl.active = true;
    b->used += (int64_t)sl.bytes;
    b->slots[s] = sl;
    b->dirty = true;
    *slot = s;
    return SETB_OK;
}

int32_t setb_batch_remove(setb_batch* b, int32_t slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].active) return SETB_EINVAL;
    cudaSetDevice(b->device);
    free_slot(b, b->slots[slot]);
    b->dirty = true;
    return SETB_OK;
}

int32_t setb_batch_step(setb_batch* b, int32_t nsteps) {
    NvtxRange range("setb_batch_step");
    if (!b || nsteps < 0) return SETB_EINVAL;
    cudaSetDevice(b->device);
    int rc = run_steps(b, nsteps);
    if (rc) return rc;
    for (auto& s : b->slots)
        if (s.active) s.steps += nsteps;
    return SETB_OK;
}

int32_t setb_batch_check(setb_batch* b, double* rel_change) {
    if (!b || !rel_change) return SETB_EINVAL;
    cudaSetDevice(b->device);
    const int ms = (int)b->slots.size();
    std::vector<int> idx;
    for (int s = 0; s < ms; s++) {
        rel_change[s] = -1.0;
        if (b->slots[s].active) idx.push_back(s);
    }
    if (idx.empty()) return SETB_OK;
    SB_TRY(cudaStreamSynchronize(b->stream));
    char* base = static_cast<char*>(b->h_check_args);
    const double** hr = reinterpret_cast<const double**>(base);
    double** hp = reinterpret_cast<double**>(base + sizeof(double*) * ms);
    long long* hn = reinterpret_cast<long long*>(base + 2 * sizeof(double*) * ms);
    const int n = (int)idx.size();
    for (int q = 0; q < n; q++) {
        Slot& sl = b->slots[idx[q]];
        hr[q] = sl.U;   // density plane of U^n
        hp[q] = sl.rho_prev;
        hn[q] = sl.g.ps * sl.g.nz;   // row padding holds zeros in U and in rho_prev
    }
    SB_TRY(cudaMemcpyAsync(b->d_rho, hr, sizeof(double*) * n, cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(b->d_prev, hp, sizeof(double*) * n, cudaMemcpyHostToDevice, b->stream));
    SB_TRY(cudaMemcpyAsync(b->d_ncell, hn, sizeof(long long) * n, cudaMemcpyHostToDevice, b->stream));
    check_partial_kernel<<<dim3(kCheckBlocks, n), 256, 0, b->stream>>>(b->d_rho, b->d_prev, b->d_ncell, b->d_partial);
    check_final_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_partial, n, b->d_check);
    SB_TRY(cudaGetLastError());
    SB_TRY(cudaMemcpyAsync(b->h_check, b->d_check, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    for (int q = 0; q < n; q++) {
        Slot& sl = b->slots[idx[q]];
        rel_change[idx[q]] = sl.have_prev ? b->h_check[q] : -1.0;
        sl.have_prev = true;
    }
    return SETB_OK;
}

int32_t setb_batch_get_conserved(setb_batch* b, int32_t slot, double* U) {
    if (!b || !U || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].active) return SETB_EINVAL;
    cudaSetDevice(b->device);
    const Slot& sl = b->slots[slot];
    const size_t N = (size_t)sl.g.nx * sl.g.ny * sl.g.nz;
    for (int v = 0; v < 8; v++)
        SB_TRY(cudaMemcpy2DAsync(U + v * N, sl.g.nx * sizeof(double), sl.U + v * sl.g.vs, sl.g.px * sizeof(double),
                                 sl.g.nx * sizeof(double), (size_t)sl.g.ny * sl.g.nz, cudaMemcpyDeviceToHost,
                                 b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    return SETB_OK;
}

int32_t setb_batch_status(setb_batch* b, int32_t slot, setb_diag* out) {
    if (!b || !out || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].active) return SETB_EINVAL;
    cudaSetDevice(b->device);
    const Slot& sl = b->slots[slot];
    DevClock c;
    DevStatus s;
    SB_TRY(cudaMemcpyAsync(&c, sl.clk, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    SB_TRY(cudaMemcpyAsync(&s, sl.st, sizeof(s), cudaMemcpyDeviceToHost, b->stream));
    SB_TRY(cudaStreamSynchronize(b->stream));
    out->time_all = c.time_all;
    out->dt_next = c.dt_cur;
    out->dt_last = c.dt_last;
    out->steps = c.steps;
    out->n_negdens = (int64_t)s.n_negdens;
    out->first_bad_cell = s.first_bad == ULLONG_MAX ? -1 : (int64_t)s.first_bad;
    out->n_pfloor = (int64_t)s.n_pfloor;
    out->n_wave_err = (int64_t)s.n_wave;
    out->n_recon_err = (int64_t)s.n_recon;
    out->n_fp64_redo = (int64_t)s.n_redo;
    if (s.n_timeout) return SETB_ETIMEOUT;
    if (s.n_negdens) return SETB_ENEGDENS;
    if (s.n_wave) return SETB_EWAVES;
    if (s.n_recon) return SETB_ERECON;
    return SETB_OK;
}

int32_t setb_batch_info(setb_batch* b, int64_t* bytes_used, int32_t* active, int32_t* lz, int32_t* grid) {
    if (!b) return SETB_EINVAL;
    int n = 0;
    for (auto& s : b->slots) n += s.active ? 1 : 0;
    if (bytes_used) *bytes_used = b->used;
    if (active) *active = n;
    if (lz) *lz = b->lz;
    if (grid) *grid = grid_size(b, b->n_items);
    return SETB_OK;
}

int32_t setb_batch_set_tiling(setb_batch* b, int32_t lz, int32_t grid_mult) {
    if (!b || lz < 1 || grid_mult < 1 || grid_mult > 8) return SETB_EINVAL;
    b->lz = lz;
    b->grid_mult = grid_mult;
    b->dirty = true;
    return SETB_OK;
}

int32_t setb_batch_tune(setb_batch* b, int32_t reps, int32_t* lz_out, int32_t* grid_mult_out, double* ms_out) {
    if (!b || reps < 1) return SETB_EINVAL;
    cudaSetDevice(b->device);
    // save clocks and counters: the timed first-stage launches are idempotent on the state but
    // update the running dt minimum and the counters
    std::vector<std::pair<DevClock, DevStatus>> saved(b->slots.size());
    for (size_t s = 0; s < b->slots.size(); s++)
        if (b->slots[s].active) {
            SB_TRY(cudaMemcpyAsync(&saved[s].first, b->slots[s].clk, sizeof(DevClock), cudaMemcpyDeviceToHost, b->stream));
            SB_TRY(cudaMemcpyAsync(&saved[s].second, b->slots[s].st, sizeof(DevStatus), cudaMemcpyDeviceToHost, b->stream));
        }
    SB_TRY(cudaStreamSynchronize(b->stream));
    const int lzs[] = {8, 16, 32, 64, 1 << 20};
    const int gms[] = {1, 2};
    double best = 1e300;
    int best_lz = b->lz, best_gm = b->grid_mult;
    cudaEvent_t e0, e1;
    SB_TRY(cudaEventCreate(&e0));
    SB_TRY(cudaEventCreate(&e1));
    for (int lz : lzs)
        for (int gm : gms) {
            b->lz = lz;
            b->grid_mult = gm;
            b->dirty = true;
            if (rebuild(b)) continue;
            if (b->n_items == 0) continue;
            auto launch_once = [&]() -> bool {
                if (cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(unsigned), b->stream) != cudaSuccess) return false;
                return launch_items(b, 1, 3, b->d_queue) == SETB_OK && launch_items(b, 1, 2, b->d_queue + 1) == SETB_OK;
            };
            if (!launch_once()) continue;   // warm-up
            cudaEventRecord(e0, b->stream);
            bool ok = true;
            for (int r = 0; r < reps && ok; r++) ok = launch_once();
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ok && ms / reps < best) {
                best = ms / reps;
                best_lz = lz;
                best_gm = gm;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->lz = best_lz;
    b->grid_mult = best_gm;
    b->dirty = true;
    for (size_t s = 0; s < b->slots.size(); s++)
        if (b->slots[s].active) {
            SB_TRY(cudaMemcpyAsync(b->slots[s].clk, &saved[s].first, sizeof(DevClock), cudaMemcpyHostToDevice, b->stream));
            SB_TRY(cudaMemcpyAsync(b->slots[s].st, &saved[s].second, sizeof(DevStatus), cudaMemcpyHostToDevice, b->stream));
        }
    SB_TRY(cudaStreamSynchronize(b->stream));
    if (lz_out) *lz_out = best_lz;
    if (grid_mult_out) *grid_mult_out = best_gm;
    if (ms_out) *ms_out = best;
    return SETB_OK;
}

int32_t setb_batch_sync(setb_batch* b) {
    if (!b) return SETB_EINVAL;
    cudaSetDevice(b->device);
    SB_TRY(cudaStreamSynchronize(b->stream));
    return SETB_OK;
}

int32_t setb_batch_destroy(setb_batch* b) {
    if (!b) return SETB_EINVAL;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (auto& s : b->slots)
        if (s.active) free_slot(b, s);
    if (b->d_items) cudaFreeAsync(b->d_items, b->stream);
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaFree(b->d_inst1);
    cudaFree(b->d_inst2);
    cudaFree(b->d_queue);
    cudaFree(b->d_partial);
    cudaFree(b->d_check);
    cudaFree(b->d_rho);
    cudaFree(b->d_prev);
    cudaFree(b->d_ncell);
    if (b->h_inst) cudaFreeHost(b->h_inst);
    if (b->h_items) cudaFreeHost(b->h_items);
    if (b->h_check_args) cudaFreeHost(b->h_check_args);
    if (b->h_check) cudaFreeHost(b->h_check);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SETB_OK;
}

}  // extern "C"
