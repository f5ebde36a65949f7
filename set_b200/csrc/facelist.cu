// facelist.cu -- the MHD step on the reference's own geometry: an explicit face list.
//
// The reference's GPU solver (SET_Fortran_Cuda_MHD/cuf_solvers.cuf) runs on an unstructured grid
// of cells and faces read from the grid file (Storage_module.f90:20-37): a face kernel
// (CUF_MGD_grans_RK2, :243-440) computes each face's flux once into Gran_POTOK and a cell kernel
// (CUF_MGD_cell_RK2, :561-794) sums the fluxes of its faces with the owner sign.  This file keeps
// that structure, B200-side:
//   * the cell state is conserved SoA FP64 (coalesced in the cell kernel); each stage starts
//     with a pass that writes the primitive state cell-major (8 doubles = 64 B per cell), so a
//     face gathers a cell with four 16-byte loads;
//   * per-face geometry the face kernel needs (the four TVD distances, the reference's "skip"
//     rule) is derived once at set-up, in the same FP64 arithmetic as the reference's per-step
//     computation, so the stage kernels read it instead of recomputing it from cell centres;
//   * the face kernel reduces the dt candidate with warp shuffles and one atomicMin per block;
//     the cell kernel's last block rolls the lagged-dt clock on the device, so a run of steps
//     needs no host round trip;
//   * the face flux array persists between stages: a skipped face keeps its previous flux, as
//     Gran_POTOK does in the reference.
// Physics 0 is the conservative ideal-MHD update of all 8 variables used by the Cartesian path,
// optionally with the div-B terms the reference carries commented out (face flux Gran_POTOK(9),
// sources proportional to its owner-signed sum); physics 1 is the reference's live cell kernel,
// a 2D axisymmetric hydro update with charge exchange.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "setb200.h"
#include "setb_internal.cuh"

namespace sb {

struct FaceListDev {
    int64_t n_cell = 0, n_gran = 0;
    // cells
    double* cell_center = nullptr;   // [N][3]
    double* cell_volume = nullptr;   // [N]
    int32_t* cell_gran = nullptr;    // [N][6], 1-based face numbers, 0 = none
    unsigned char* cell_flag = nullptr;   // bit 0: frozen (not updated)
    // faces
    double* normal = nullptr;        // [G][3]
    double* square = nullptr;        // [G]
    double* geo = nullptr;           // [G][4]: dist = |c_face - c_s1|, df2, dff1, dff2
    int32_t* nb = nullptr;           // [G][2], 1-based, -1 = none
    int32_t* nbt = nullptr;          // [G][2], 1-based, -1 = none
    int32_t* type = nullptr;         // [G]: 0 = skipped, else the reference's face type 1..5,
                                     // plus kLaxFace on the near-axis faces of physics 1
    // work
    double* prim = nullptr;          // [N][8] primitive state of the stage input
    double* flux = nullptr;          // [G][8] face flux * area (persistent)
    GridGeom src{};                  // source-sphere parameters (r_src 0 = none)
    int physics = 0;                 // 0: 3D MHD; 1: the reference's axisymmetric hydro update
    double* hatom = nullptr;         // physics 1: [N][8] H-atom fluids (Cell_par columns 9..16)
    int powell = 0;                  // physics 0: div-B terms (0 off, 1 momentum + induction, 2 + energy)
    double* divb = nullptr;          // powell: [G] div-B face flux * area, Gran_POTOK(9) (persistent)
    // locality order: device cell d holds the caller's cell perm[d] (both 0-based)
    std::vector<int32_t> perm;
};

namespace {

constexpr int kFaceThreads = 128, kCellThreads = 256, kPrimThreads = 256;
constexpr int kLaxFace = 8;   // face-type bit: the reference's Lax flux on near-axis faces

double norm3(const double* x) {
    return std::sqrt((x[0] * x[0] + x[1] * x[1]) + x[2] * x[2]);
}

template <typename T>
cudaError_t upload(T** dst, const T* src, size_t n, cudaStream_t s) {
    cudaError_t e = cudaMalloc(dst, sizeof(T) * std::max<size_t>(n, 1));
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, s);
}

// ------------------------------------------------------------------------------ kernels
__global__ void fl_prim_kernel(int64_t n, const double* __restrict__ U, int64_t vs, double* __restrict__ P) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        double u8[8], q[8], ke, me;
#pragma unroll
        for (int v = 0; v < 8; v++) u8[v] = U[v * vs + c];
        prim_from_cons(u8, q, ke, me);
        double2* p2 = reinterpret_cast<double2*>(P + 8 * c);
#pragma unroll
        for (int v = 0; v < 4; v++) p2[v] = make_double2(q[2 * v], q[2 * v + 1]);
    }
}

// Solvers.f90:141-150 at y = 0: linear(x1,t1,x2,t2,x3,t3,0) = minmod of the two one-sided
// slopes times (0 - x2), plus t2, with ra = 1/(x1 - x2) and rb = 1/(x2 - x3) (geometry, formed
// once per face): the slopes' divisions become multiplications, one rounding from the reference.
__device__ __forceinline__ double linear_rcp(double ra, double t1, double x2, double t2, double rb, double t3) {
    const double d = minmod(dmul(dsub(t1, t2), ra), dmul(dsub(t2, t3), rb));
    return dadd(dmul(d, dsub(0.0, x2)), t2);
}

__device__ __forceinline__ void load_prim(const double* P, int64_t c, double* q) {
    const double2* p2 = reinterpret_cast<const double2*>(P + 8 * c);
#pragma unroll
    for (int v = 0; v < 4; v++) {
        const double2 d = __ldg(p2 + v);
        q[2 * v] = d.x;
        q[2 * v + 1] = d.y;
    }
}

// Source_MK (SET_Fortran_Cuda_MHD/cuf_kernel.cuf:215-288): charge-exchange momentum (x, y) and
// energy sources against two H-atom fluids (rho, u, v, T per fluid in h[0..3], h[4..7]).  The
// reference's default-real literals enter as their single-precision values.
__device__ __forceinline__ void source_mk(const double* q, const double* h, double* out) {
    const double pi = 3.141592653589793;
    const double rho = q[0], u = q[1], v = q[2], p = q[4];
    const double small = (double)0.0000001f;
    const double c_m = __ddiv_rn(64.0, dmul(9.0, pi)), c_u = __ddiv_rn(4.0, pi);
    const double c_s = (double)0.1307345665f;
    const double c_n = (double)(3.0f / 0.4326569f);
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        double rH = h[4 * k], uH = h[4 * k + 1], vH = h[4 * k + 2];
        double pH = dmul(dmul(0.5, h[4 * k + 3]), rH);
        if (rH < small) {
            rH = small;
            pH = 0.0;
        }
        const double du = dsub(u, uH), dv = dsub(v, vH);
        const double th = dadd(__ddiv_rn(p, rho), __ddiv_rn(dmul(2.0, pH), rH));
        const double d2 = dadd(dmul(du, du), dmul(dv, dv));
        const double UM = sqrt(dadd(d2, dmul(c_m, th)));
        const double UH = sqrt(dadd(d2, dmul(c_u, th)));
        const double lg = dsub(1.0, dmul(c_s, log(UM)));
        const double nu = dmul(dmul(dmul(rho, rH), UM), dmul(lg, lg));
        const double cn = dmul(c_n, nu);
        s1 = dadd(s1, dmul(cn, dsub(uH, u)));
        s2 = dadd(s2, dmul(cn, dsub(vH, v)));
        const double ke = __ddiv_rn(dsub(dsub(dadd(dmul(uH, uH), dmul(vH, vH)), dmul(u, u)), dmul(v, v)), 2.0);
        s3 = dadd(s3, dmul(cn, dadd(ke, dmul(__ddiv_rn(UH, UM), dsub(__ddiv_rn(dmul(2.0, pH), rH), __ddiv_rn(p, rho))))));
    }
    out[0] = s1;
    out[1] = s2;
    out[2] = s3;
}

// The reference's live cell update (cuf_solvers.cuf:561-794): 2D axisymmetric hydro about the x
// axis with radius rr(2) = y, w = B = 0, charge exchange, p floor and the near-axis v clamp, in
// the reference's operation order on the primitive state.  Writes the conserved result to un;
// returns 1 for a non-positive density (un = the stage input), 2 when the p floor applied.
template <int KIND>
__device__ __forceinline__ int axisym_update(const double* Uin, const double* Ubase, int64_t vs, int64_t c,
                                             const double* pot, double vol, double x, double y, const double* h,
                                             double t, double* un) {
    const double g = kGamma, gm1 = dsub(kGamma, 1.0);
    double u8[8], q[8], q2[8], ke, me, source[3];
#pragma unroll
    for (int v = 0; v < 8; v++) u8[v] = Uin[v * vs + c];
    prim_from_cons_exact(u8, q);
    if (KIND == 1) {
        double b8[8];
#pragma unroll
        for (int v = 0; v < 8; v++) b8[v] = Ubase[v * vs + c];
        prim_from_cons_exact(b8, q2);
    }
    (void)ke;
    (void)me;
    source_mk(q, h, source);
    const double nq = sqrt(dadd(dadd(dmul(q[1], q[1]), dmul(q[2], q[2])), dmul(q[3], q[3])));
    const double e1 = dadd(__ddiv_rn(q[4], gm1), dmul(dmul(0.5, q[0]), dmul(nq, nq)));
    const double X = dadd(__ddiv_rn(dmul(g, q[4]), gm1), dmul(dmul(q[0], dadd(dmul(q[1], q[1]), dmul(q[2], q[2]))), 0.5));
    const double geo_e = __ddiv_rn(dmul(dmul(t, q[2]), X), y);
    const double div0 = dadd(__ddiv_rn(pot[0], vol), __ddiv_rn(dmul(q[0], q[2]), y));
    double ro3;
    if (KIND == 0) ro3 = dsub(q[0], dmul(t, div0));
    else ro3 = dmul(0.5, dsub(dadd(q2[0], q[0]), dmul(t, div0)));
    if (!(ro3 > 0.0)) {
#pragma unroll
        for (int v = 0; v < 8; v++) un[v] = u8[v];
        return 1;
    }
    const double g1 = __ddiv_rn(dmul(t, pot[1]), vol), g2 = __ddiv_rn(dmul(t, pot[2]), vol);
    const double g4 = __ddiv_rn(dmul(t, pot[4]), vol);
    const double a1 = __ddiv_rn(dmul(dmul(dmul(t, q[0]), q[1]), q[2]), y);
    const double a2 = __ddiv_rn(dmul(dmul(dmul(t, q[0]), q[2]), q[2]), y);
    double u3, v3, p3;
    if (KIND == 0) {
        u3 = __ddiv_rn(dsub(dadd(dsub(dmul(q[0], q[1]), g1), dmul(t, source[0])), a1), ro3);
        v3 = __ddiv_rn(dsub(dadd(dsub(dmul(q[0], q[2]), g2), dmul(t, source[1])), a2), ro3);
        p3 = dmul(dsub(dsub(dadd(dsub(e1, g4), dmul(t, source[2])), geo_e),
                       dmul(dmul(0.5, ro3), dadd(dadd(dmul(u3, u3), dmul(v3, v3)), 0.0))),
                  gm1);
    } else {
        const double nq2 = sqrt(dadd(dadd(dmul(q2[1], q2[1]), dmul(q2[2], q2[2])), dmul(q2[3], q2[3])));
        const double e2 = dadd(__ddiv_rn(q2[4], gm1), dmul(dmul(0.5, q2[0]), dmul(nq2, nq2)));
        u3 = __ddiv_rn(dmul(0.5, dsub(dadd(dsub(dadd(dmul(q2[0], q2[1]), dmul(q[0], q[1])), g1), dmul(t, source[0])), a1)), ro3);
        v3 = __ddiv_rn(dmul(0.5, dsub(dadd(dsub(dadd(dmul(q2[0], q2[2]), dmul(q[0], q[2])), g2), dmul(t, source[1])), a2)), ro3);
        p3 = dmul(dsub(dmul(0.5, dsub(dadd(dsub(dadd(e2, e1), g4), dmul(t, source[2])), geo_e)),
                       dmul(dmul(0.5, ro3), dadd(dadd(dmul(u3, u3), dmul(v3, v3)), 0.0))),
                  gm1);
    }
    int rc = 0;
    if (p3 <= 0.0) {
        p3 = kPFloor;
        rc = 2;
    }
    if (x > (double)0.28f && y < (double)0.07f && v3 < 0.0) v3 = (double)0.01f;
    const double qn[8] = {ro3, u3, v3, 0.0, p3, 0.0, 0.0, 0.0};
    cons_from_prim_exact(qn, un);
    return rc;
}

// One face per thread, cuf_solvers.cuf:243-440 (face speed 0).
template <int NSTATE, int ORDER, bool WANT_DT>
__global__ void __launch_bounds__(kFaceThreads, 4) fl_face_kernel(const FaceListDev m, double cfl, int n_disc,
                                                               DevClock* clk, DevStatus* st) {
    __shared__ double red[kFaceThreads / 32];
    __shared__ unsigned long long cnt[2];
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t gr = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double cand = kDtReset;
    unsigned n_recon = 0, n_wave = 0;
    const int tword = gr < m.n_gran ? m.type[gr] : 0;
    const int type = tword & 7;
    if (type != 0) {
        const int64_t s1 = m.nb[2 * gr] - 1;
        const int32_t s2r = m.nb[2 * gr + 1];
        const double n[3] = {m.normal[3 * gr], m.normal[3 * gr + 1], m.normal[3 * gr + 2]};
        double q1[8], q2[8];
        load_prim(m.prim, s1, q1);
        bool tvd = ORDER == 2;
        if (type == 4) {                          // :318-324 outer boundary
#pragma unroll
            for (int v = 0; v < 8; v++) q2[v] = q1[v];
            if (q2[1] > -0.1) q2[1] = -0.1;
            tvd = false;
        } else if (type == 5) {                   // :325-329 axis
#pragma unroll
            for (int v = 0; v < 8; v++) q2[v] = q1[v];
            q2[2] = -q2[2];
            tvd = false;
        } else if (type == 2 && s2r == -1) {      // :330-345 reflecting wall
            const double vel = dadd(dadd(dmul(n[0], q1[1]), dmul(n[1], q1[2])), dmul(n[2], q1[3]));
#pragma unroll
            for (int v = 0; v < 8; v++) q2[v] = q1[v];
#pragma unroll
            for (int a = 0; a < 3; a++) q2[1 + a] = dsub(dsub(q1[1 + a], dmul(vel, n[a])), dmul(vel, n[a]));
            tvd = false;
        } else {
            load_prim(m.prim, (int64_t)s2r - 1, q2);
        }
        const int32_t ss1 = m.nbt[2 * gr], ss2 = m.nbt[2 * gr + 1];
        const double dist = m.geo[4 * gr];
        if (tvd && ss1 >= 1 && ss2 >= 1) {       // :358-412, linear on the precomputed distances
            const double df1 = dist, df2 = m.geo[4 * gr + 1], dff1 = m.geo[4 * gr + 2], dff2 = m.geo[4 * gr + 3];
            double q11[8], q22[8];
            load_prim(m.prim, (int64_t)ss1 - 1, q11);
            load_prim(m.prim, (int64_t)ss2 - 1, q22);
            double t1[5], t2[5];
#pragma unroll
            // linear(-dff1, q11, -df1, q1, df2, q2) and linear(-dff2, q22, -df2, q2, df1, q1): three
            // reciprocals per face instead of 20 divisions (the face-list path measured 7 % faster)
            const double ra1 = sb_rcp(dsub(-dff1, -df1)), ra2 = sb_rcp(dsub(-dff2, -df2));
            const double rb = sb_rcp(dsub(-df1, df2));   // (-df2) - df1 rounds to the same value
#pragma unroll
            for (int v = 0; v < 5; v++) {
                t1[v] = linear_rcp(ra1, q11[v], -df1, q1[v], rb, q2[v]);
                t2[v] = linear_rcp(ra2, q22[v], -df2, q2[v], rb, q1[v]);
            }
            if (sb_neg(t1[0])) t1[0] = q1[0];
            if (sb_neg(t1[4])) t1[4] = q1[4];
            if (sb_neg(t2[0])) t2[0] = q2[0];
            if (sb_neg(t2[4])) t2[4] = q2[4];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                q1[v] = t1[v];
                q2[v] = t2[v];
            }
        }
        if (sb_neg(q1[0]) || sb_neg(q2[0])) n_recon++;
        double qqq[8], sp[3];
        int32_t fl = 0;
        // the faces do not move (w = 0): no face-speed terms
        if (tword & kLaxFace) chlld_general<double, 0, false, false>(n, 0.0, q1, q2, n_disc, qqq, sp, &fl);   // :293-295
        else chlld_general<double, NSTATE, false, false>(n, 0.0, q1, q2, n_disc, qqq, sp, &fl);
        if (fl & kFlagWave) {
            n_wave++;
#pragma unroll
            for (int v = 0; v < 8; v++) qqq[v] = 0.0;
        }
        const double sq = m.square[gr];
        double2* f2 = reinterpret_cast<double2*>(m.flux + 8 * gr);
#pragma unroll
        for (int v = 0; v < 4; v++) f2[v] = make_double2(qqq[2 * v] * sq, qqq[2 * v + 1] * sq);
        if (m.powell) {   // :433 as commented there: 0.5 * n.(B1 + B2) * square, B of the chlld states
            const double nb = dadd(dadd(dmul(n[0], dadd(q1[5], q2[5])), dmul(n[1], dadd(q1[6], q2[6]))),
                                   dmul(n[2], dadd(q1[7], q2[7])));
            m.divb[gr] = dmul(dmul(0.5, nb), sq);
        }
        // compare-and-select min / max (the library fmin / fmax of doubles are far longer sequences)
        if (WANT_DT) cand = sb_min(kDtFaceCap, cfl * dist * sb_rcp(sb_max(fabs(sp[0]), fabs(sp[1]))));
    }
    if (n_recon) atomicAdd(&cnt[0], (unsigned long long)n_recon);
    if (n_wave) atomicAdd(&cnt[1], (unsigned long long)n_wave);
    if (WANT_DT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cand = fmin(cand, __shfl_xor_sync(0xffffffffu, cand, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cand;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (WANT_DT) {
            double r = red[0];
#pragma unroll
            for (int w = 1; w < kFaceThreads / 32; w++) r = fmin(r, red[w]);
            atomicMin(&clk->dt_next, (unsigned long long)__double_as_longlong(r));
        }
        if (cnt[0]) atomicAdd(&st->n_recon, cnt[0]);
        if (cnt[1]) atomicAdd(&st->n_wave, cnt[1]);
    }
}

// One cell per thread, cuf_solvers.cuf:561-794 as the conservative MHD update: owner-signed sum
// of the face fluxes (:691-703), Euler / Heun stage (:705-770), negative-density check, p floor
// (:777-779), frozen cells (:611) and the re-imposed source sphere.  The last block of a
// finalizing launch rolls the clock.
// PHYS: the physics option; POWELL: the div-B terms are on (their energy term by m.powell ==
// 2).  Compile-time, so a launch carries only its own code (registers set the occupancy of this
// gather-bound kernel).
template <int KIND, int PHYS, bool POWELL>
__global__ void __launch_bounds__(kCellThreads) fl_cell_kernel(const FaceListDev m, const double* __restrict__ Uin,
                                                               const double* Ubase, double* Uout, int64_t vs,
                                                               DevClock* clk, DevStatus* st, int finalize) {
    __shared__ unsigned long long cnt[2];
    __shared__ bool last;
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double dt = clk->dt_cur;
    if (c < m.n_cell) {
        double un[8], qs[8];
        const double x = m.cell_center[3 * c], y = m.cell_center[3 * c + 1], z = m.cell_center[3 * c + 2];
        const double r2 = dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
        if (m.cell_flag[c] & 1) {
#pragma unroll
            for (int v = 0; v < 8; v++) un[v] = KIND == 0 ? Uin[v * vs + c] : Ubase[v * vs + c];
        } else if (PHYS == 0 && m.src.r_src > 0.0 && r2 < dmul(m.src.r_src, m.src.r_src)) {
            source_state(m.src, x, y, z, r2, qs);
            cons_from_prim_exact(qs, un);
        } else if (PHYS == 1) {
            double pot[8];
#pragma unroll
            for (int v = 0; v < 8; v++) pot[v] = 0.0;
            for (int f = 0; f < 6; f++) {
                const int32_t j = m.cell_gran[6 * c + f];
                if (j == 0) continue;
                const int64_t jf = (int64_t)j - 1;
                const bool owner = m.nb[2 * jf] == (int32_t)(c + 1);
                const double2* f2 = reinterpret_cast<const double2*>(m.flux + 8 * jf);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const double2 d = f2[v];
                    pot[2 * v] = owner ? pot[2 * v] + d.x : pot[2 * v] - d.x;
                    pot[2 * v + 1] = owner ? pot[2 * v + 1] + d.y : pot[2 * v + 1] - d.y;
                }
            }
            const int rc = axisym_update<KIND>(Uin, Ubase, vs, c, pot, m.cell_volume[c], x, y, m.hatom + 8 * c, dt, un);
            if (rc == 1) {
                atomicAdd(&cnt[0], 1ull);
                atomicMin(&st->first_bad, (unsigned long long)c);
            } else if (rc == 2) {
                atomicAdd(&cnt[1], 1ull);
            }
        } else {
            double pot[8], sks = 0.0;
#pragma unroll
            for (int v = 0; v < 8; v++) pot[v] = 0.0;
            for (int f = 0; f < 6; f++) {
                const int32_t j = m.cell_gran[6 * c + f];
                if (j == 0) continue;
                const int64_t jf = (int64_t)j - 1;
                const bool owner = m.nb[2 * jf] == (int32_t)(c + 1);
                const double2* f2 = reinterpret_cast<const double2*>(m.flux + 8 * jf);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const double2 d = f2[v];
                    pot[2 * v] = owner ? pot[2 * v] + d.x : pot[2 * v] - d.x;
                    pot[2 * v + 1] = owner ? pot[2 * v + 1] + d.y : pot[2 * v + 1] - d.y;
                }
                if (POWELL) sks = owner ? sks + m.divb[jf] : sks - m.divb[jf];
            }
            if (POWELL) {
                // div-B sources inside the flux sum (cuf_solvers.cuf:529-533 / 729-733, commented
                // there): momentum + (B/4pi) sks, B + u sks, powell 2 energy + (u.B/4pi) sks, with
                // u and B of the stage input (the primitive pass of this stage)
                double q[8];
                load_prim(m.prim, c, q);
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    pot[1 + a] = dadd(pot[1 + a], dmul(q[5 + a] / kCpi4, sks));
                    pot[5 + a] = dadd(pot[5 + a], dmul(q[1 + a], sks));
                }
                if (m.powell == 2) {
                    const double ub = dadd(dadd(dmul(q[1], q[5]), dmul(q[2], q[6])), dmul(q[3], q[7]));
                    pot[4] = dadd(pot[4], dmul(ub / kCpi4, sks));
                }
            }
            // one reciprocal of the volume instead of eight divisions (the face-list path measured
            // 7 % faster); the dt candidate below likewise multiplies by 1/max(|SL|,|SR|)
            const double ivol = sb_rcp(m.cell_volume[c]);
            double uin[8];
#pragma unroll
            for (int v = 0; v < 8; v++) {
                uin[v] = Uin[v * vs + c];
                if (KIND == 0) un[v] = uin[v] - dt * (pot[v] * ivol);
                else un[v] = 0.5 * ((Ubase[v * vs + c] + uin[v]) - dt * (pot[v] * ivol));
            }
            if (!(un[0] > 0.0)) {
                atomicAdd(&cnt[0], 1ull);
                atomicMin(&st->first_bad, (unsigned long long)c);
#pragma unroll
                for (int v = 0; v < 8; v++) un[v] = uin[v];
            } else {
                double q[8], ke, me;
                prim_from_cons(un, q, ke, me);
                if (q[4] <= 0.0) {
                    atomicAdd(&cnt[1], 1ull);
                    un[4] = floor_energy(ke, me);
                }
            }
        }
#pragma unroll
        for (int v = 0; v < 8; v++) Uout[v * vs + c] = un[v];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (cnt[0]) atomicAdd(&st->n_negdens, cnt[0]);
        if (cnt[1]) atomicAdd(&st->n_pfloor, cnt[1]);
        __threadfence();
        last = atomicAdd(&clk->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        clk->counter = 0;
        if (finalize) {
            const unsigned long long nb = atomicExch(&clk->dt_next, (unsigned long long)__double_as_longlong(kDtReset));
            clk->time_all += clk->dt_cur;
            clk->dt_last = clk->dt_cur;
            clk->dt_cur = __longlong_as_double((long long)nb);
            clk->steps += 1;
        }
        __threadfence();
    }
}

template <int NSTATE>
void launch_face_n(const FaceListDev& m, int order, bool want_dt, double cfl, int n_disc, DevClock* clk,
                   DevStatus* st, cudaStream_t s) {
    const unsigned grid = (unsigned)((m.n_gran + kFaceThreads - 1) / kFaceThreads);
    if (order == 2) {
        if (want_dt) fl_face_kernel<NSTATE, 2, true><<<grid, kFaceThreads, 0, s>>>(m, cfl, n_disc, clk, st);
        else fl_face_kernel<NSTATE, 2, false><<<grid, kFaceThreads, 0, s>>>(m, cfl, n_disc, clk, st);
    } else {
        if (want_dt) fl_face_kernel<NSTATE, 1, true><<<grid, kFaceThreads, 0, s>>>(m, cfl, n_disc, clk, st);
        else fl_face_kernel<NSTATE, 1, false><<<grid, kFaceThreads, 0, s>>>(m, cfl, n_disc, clk, st);
    }
}

}  // namespace

// ------------------------------------------------------------------------------ host side
void fl_destroy(FaceListDev* f) {
    if (!f) return;
    void* ptrs[] = {f->cell_center, f->cell_volume, f->cell_gran, f->cell_flag, f->normal, f->square, f->geo,
                    f->nb,          f->nbt,         f->type,      f->prim,      f->flux,   f->hatom,
                    f->divb};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete f;
}

// Host-side check that every index the kernels follow stays inside its array: cell faces in
// 0..G, neighbours in 1..N (neighbour 2 may be -1 only on a ghost face: type 4, 5, or a type-2
// wall), TVD cells in 1..N or -1, face types 1..5, volumes positive.
int fl_validate(int64_t N, int64_t G, const double* cell_center, const double* cell_volume, const int32_t* cell_gran,
                const double* gran_normal, const double* gran_square, const double* gran_center,
                const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd, const int32_t* gran_type) {
    if (N < 1 || G < 1 || !cell_center || !cell_volume || !cell_gran || !gran_normal || !gran_square || !gran_center ||
        !gran_neighbour || !gran_neighbour_tvd || !gran_type)
        return SETB_EINVAL;
    if (N > INT32_MAX - 1 || G > INT32_MAX - 1) return SETB_ESIZE;
    for (int64_t c = 0; c < N; c++) {
        if (!(cell_volume[c] > 0.0)) return SETB_EINVAL;
        for (int f = 0; f < 6; f++) {
            const int32_t j = cell_gran[6 * c + f];
            if (j < 0 || j > G) return SETB_EINVAL;
        }
    }
    for (int64_t g = 0; g < G; g++) {
        const int32_t s1 = gran_neighbour[2 * g], s2 = gran_neighbour[2 * g + 1], t = gran_type[g];
        const int32_t ss1 = gran_neighbour_tvd[2 * g], ss2 = gran_neighbour_tvd[2 * g + 1];
        if (s1 < 1 || s1 > N || t < 1 || t > 5) return SETB_EINVAL;
        const bool ghost = t == 4 || t == 5 || (t == 2 && s2 == -1);
        if (!ghost && (s2 < 1 || s2 > N)) return SETB_EINVAL;
        if ((ss1 != -1 && (ss1 < 1 || ss1 > N)) || (ss2 != -1 && (ss2 < 1 || ss2 > N))) return SETB_EINVAL;
    }
    return SETB_OK;
}

namespace {
// 21-bit spread for a 63-bit Morton code
uint64_t spread3(uint64_t x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
}  // namespace

int fl_create(FaceListDev** out, int64_t N, int64_t G, const double* cell_center_in, const double* cell_volume_in,
              const int32_t* cell_gran_in, const double* gran_normal_in, const double* gran_square_in,
              const double* gran_center_in, const int32_t* gran_neighbour_in, const int32_t* gran_neighbour_tvd_in,
              const int32_t* gran_type_in, const setb_fl_params* p, cudaStream_t s) {
    *out = nullptr;
    if (!p) return SETB_EINVAL;
    int rc = fl_validate(N, G, cell_center_in, cell_volume_in, cell_gran_in, gran_normal_in, gran_square_in,
                         gran_center_in, gran_neighbour_in, gran_neighbour_tvd_in, gran_type_in);
    if (rc) return rc;
    // Locality order: cells along the Morton curve of their centres, faces by their first cell, so
    // the cells a face gathers and the faces a cell gathers sit close in memory whatever the
    // caller's numbering.  cperm[d] = caller's cell of device cell d; fperm likewise for faces.
    std::vector<int32_t> cperm((size_t)N), fperm((size_t)G), cnew((size_t)N), fnew((size_t)G);
    {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int64_t c = 0; c < N; c++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], cell_center_in[3 * c + a]);
                hi[a] = std::max(hi[a], cell_center_in[3 * c + a]);
            }
        std::vector<uint64_t> key((size_t)N);
        for (int64_t c = 0; c < N; c++) {
            uint64_t code = 0;
            for (int a = 0; a < 3; a++) {
                const double span = hi[a] > lo[a] ? hi[a] - lo[a] : 1.0;
                const double u = (cell_center_in[3 * c + a] - lo[a]) / span;
                code |= spread3((uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0))) << a;
            }
            key[c] = code;
        }
        std::iota(cperm.begin(), cperm.end(), 0);
        std::stable_sort(cperm.begin(), cperm.end(), [&](int32_t x, int32_t y) { return key[x] < key[y]; });
        for (int64_t d = 0; d < N; d++) cnew[cperm[d]] = (int32_t)d;
        std::iota(fperm.begin(), fperm.end(), 0);
        std::stable_sort(fperm.begin(), fperm.end(), [&](int32_t x, int32_t y) {
            return cnew[gran_neighbour_in[2 * (int64_t)x] - 1] < cnew[gran_neighbour_in[2 * (int64_t)y] - 1];
        });
        for (int64_t d = 0; d < G; d++) fnew[fperm[d]] = (int32_t)d;
    }
    auto cell_ref = [&](int32_t c1) { return c1 >= 1 ? cnew[c1 - 1] + 1 : c1; };   // 1-based, -1 kept
    std::vector<double> cell_center((size_t)N * 3), cell_volume((size_t)N), gran_normal((size_t)G * 3),
        gran_square((size_t)G), gran_center((size_t)G * 3);
    std::vector<int32_t> cell_gran((size_t)N * 6), gran_neighbour((size_t)G * 2), gran_neighbour_tvd((size_t)G * 2),
        gran_type_v((size_t)G);
    for (int64_t d = 0; d < N; d++) {
        const int64_t c = cperm[d];
        for (int a = 0; a < 3; a++) cell_center[3 * d + a] = cell_center_in[3 * c + a];
        cell_volume[d] = cell_volume_in[c];
        for (int f = 0; f < 6; f++) {
            const int32_t j = cell_gran_in[6 * c + f];
            cell_gran[6 * d + f] = j >= 1 ? fnew[j - 1] + 1 : 0;
        }
    }
    for (int64_t d = 0; d < G; d++) {
        const int64_t g = fperm[d];
        for (int a = 0; a < 3; a++) {
            gran_normal[3 * d + a] = gran_normal_in[3 * g + a];
            gran_center[3 * d + a] = gran_center_in[3 * g + a];
        }
        gran_square[d] = gran_square_in[g];
        for (int b = 0; b < 2; b++) {
            gran_neighbour[2 * d + b] = cell_ref(gran_neighbour_in[2 * g + b]);
            gran_neighbour_tvd[2 * d + b] = cell_ref(gran_neighbour_tvd_in[2 * g + b]);
        }
        gran_type_v[d] = gran_type_in[g];
    }
    const int32_t* gran_type = gran_type_v.data();
    std::vector<double> geo((size_t)G * 4);
    std::vector<int32_t> type((size_t)G);
    for (int64_t g = 0; g < G; g++) {
        const int32_t s1 = gran_neighbour[2 * g], s2 = gran_neighbour[2 * g + 1];
        const int32_t t = gran_type[g];
        const int32_t ss1 = gran_neighbour_tvd[2 * g], ss2 = gran_neighbour_tvd[2 * g + 1];
        const bool ghost = t == 4 || t == 5 || (t == 2 && s2 == -1);
        // distances as the reference forms them each step (cuf_solvers.cuf:290-292, 362-372)
        const double* gc = gran_center.data() + 3 * g;
        const double* c1 = cell_center.data() + 3 * (int64_t)(s1 - 1);
        const double* c2 = ghost ? c1 : cell_center.data() + 3 * (int64_t)(s2 - 1);
        double r[3];
        for (int a = 0; a < 3; a++) r[a] = gc[a] - c1[a];
        geo[4 * g] = norm3(r);
        for (int a = 0; a < 3; a++) r[a] = gc[a] - c2[a];
        geo[4 * g + 1] = norm3(r);
        geo[4 * g + 2] = geo[4 * g + 3] = 0.0;
        if (ss1 >= 1) {
            for (int a = 0; a < 3; a++) r[a] = gc[a] - cell_center[3 * (int64_t)(ss1 - 1) + a];
            geo[4 * g + 2] = norm3(r);
        }
        if (ss2 >= 1) {
            for (int a = 0; a < 3; a++) r[a] = gc[a] - cell_center[3 * (int64_t)(ss2 - 1) + a];
            geo[4 * g + 3] = norm3(r);
        }
        // the reference skips faces whose first cell lies inside its frozen core (:284)
        type[g] = (p->face_skip_radius > 0.0 && norm3(c1) < p->face_skip_radius) ? 0 : t;
        // physics 1: the reference's Lax flux on faces near the axis (cuf_solvers.cuf:293-295)
        if (type[g] && p->physics == 1 && gc[0] > (double)0.22f && gc[1] < (double)0.1f &&
            std::fabs(gran_normal[3 * g]) < (double)0.1f)
            type[g] |= kLaxFace;
    }
    std::vector<unsigned char> flag((size_t)N);
    for (int64_t c = 0; c < N; c++)
        flag[c] = (p->cell_freeze_radius > 0.0 && norm3(cell_center.data() + 3 * c) < p->cell_freeze_radius) ? 1 : 0;

    FaceListDev* f = new (std::nothrow) FaceListDev();
    if (!f) return SETB_ENOMEM;
    f->n_cell = N;
    f->n_gran = G;
    f->src.r_src = p->r_src;
    f->src.rho_src = p->rho_src;
    f->src.v_src = p->v_src;
    f->src.p_over_rho_src = p->p_over_rho_src;
    f->src.r_floor = p->r_floor;
    f->perm = cperm;
    f->physics = p->physics;
    f->powell = p->powell;
    bool ok = upload(&f->cell_center, cell_center.data(), 3 * (size_t)N, s) == cudaSuccess &&
              upload(&f->cell_volume, cell_volume.data(), (size_t)N, s) == cudaSuccess &&
              upload(&f->cell_gran, cell_gran.data(), 6 * (size_t)N, s) == cudaSuccess &&
              upload(&f->cell_flag, flag.data(), (size_t)N, s) == cudaSuccess &&
              upload(&f->normal, gran_normal.data(), 3 * (size_t)G, s) == cudaSuccess &&
              upload(&f->square, gran_square.data(), (size_t)G, s) == cudaSuccess &&
              upload(&f->geo, geo.data(), 4 * (size_t)G, s) == cudaSuccess &&
              upload(&f->nb, gran_neighbour.data(), 2 * (size_t)G, s) == cudaSuccess &&
              upload(&f->nbt, gran_neighbour_tvd.data(), 2 * (size_t)G, s) == cudaSuccess &&
              upload(&f->type, type.data(), (size_t)G, s) == cudaSuccess &&
              cudaMalloc(&f->prim, sizeof(double) * 8 * (size_t)N) == cudaSuccess &&
              cudaMalloc(&f->flux, sizeof(double) * 8 * (size_t)G) == cudaSuccess &&
              (p->physics != 1 || cudaMalloc(&f->hatom, sizeof(double) * 8 * (size_t)N) == cudaSuccess) &&
              cudaMemsetAsync(f->flux, 0, sizeof(double) * 8 * (size_t)G, s) == cudaSuccess &&
              (p->powell == 0 || (cudaMalloc(&f->divb, sizeof(double) * (size_t)G) == cudaSuccess &&
                                  cudaMemsetAsync(f->divb, 0, sizeof(double) * (size_t)G, s) == cudaSuccess)) &&
              cudaStreamSynchronize(s) == cudaSuccess;   // host vectors are released on return
    if (!ok) {
        cudaGetLastError();
        fl_destroy(f);
        return SETB_ENOMEM;
    }
    *out = f;
    return SETB_OK;
}

cudaError_t fl_launch_stage(const FaceListDev* f, const double* Uin, const double* Ubase, double* Uout, int64_t vs,
                            DevClock* clk, DevStatus* st, const setb_step_opts* o, int kind, bool want_dt,
                            bool finalize, cudaStream_t s) {
    const FaceListDev& m = *f;
    const unsigned pgrid = (unsigned)std::min<int64_t>((m.n_cell + kPrimThreads - 1) / kPrimThreads, 148 * 16);
    fl_prim_kernel<<<pgrid, kPrimThreads, 0, s>>>(m.n_cell, Uin, vs, m.prim);
    switch (o->n_state) {
        case 0: launch_face_n<0>(m, o->order, want_dt, o->cfl, o->n_disc, clk, st, s); break;
        case 1: launch_face_n<1>(m, o->order, want_dt, o->cfl, o->n_disc, clk, st, s); break;
        case 2: launch_face_n<2>(m, o->order, want_dt, o->cfl, o->n_disc, clk, st, s); break;
        default: launch_face_n<3>(m, o->order, want_dt, o->cfl, o->n_disc, clk, st, s); break;
    }
    const unsigned cgrid = (unsigned)((m.n_cell + kCellThreads - 1) / kCellThreads);
#define SB_CELL(K, PH, PW) fl_cell_kernel<K, PH, PW><<<cgrid, kCellThreads, 0, s>>>(m, Uin, Ubase, Uout, vs, clk, st, finalize)
    if (m.physics == 1) {
        if (kind == 0) SB_CELL(0, 1, false);
        else SB_CELL(1, 1, false);
    } else if (m.powell) {
        if (kind == 0) SB_CELL(0, 0, true);
        else SB_CELL(1, 0, true);
    } else {
        if (kind == 0) SB_CELL(0, 0, false);
        else SB_CELL(1, 0, false);
    }
#undef SB_CELL
    return cudaGetLastError();
}

}  // namespace sb

namespace sb {
const int32_t* fl_perm(const FaceListDev* f) { return f ? f->perm.data() : nullptr; }
}  // namespace sb

namespace sb {
// Uploads the H-atom fluids (Cell_par columns 9..16, caller numbering) of a physics-1 face list.
int fl_set_hatom(FaceListDev* f, const double* cell_par, cudaStream_t s) {
    if (!f || !f->hatom) return SETB_OK;
    const size_t N = (size_t)f->n_cell;
    std::vector<double> tmp(8 * N);
    for (size_t d = 0; d < N; d++) std::memcpy(&tmp[8 * d], cell_par + 16 * (size_t)f->perm[d] + 8, 8 * sizeof(double));
    if (cudaMemcpyAsync(f->hatom, tmp.data(), sizeof(double) * 8 * N, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return SETB_ECUDA;
    return SETB_OK;
}
}  // namespace sb
