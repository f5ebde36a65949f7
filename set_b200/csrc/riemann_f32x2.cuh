// riemann_f32x2.cuh -- the mixed form's FP32 HLLC / HLLD flux with the left and right states
// carried as pairs through Blackwell's paired FP32 instructions (add / mul / fma .f32x2).
//
// Same algorithm, same formulas and the same wave-fan selection as riemann<float, NSTATE,
// false, true> in mhd_core.cuh (chlld, SET_Fortran_Cuda_MHD/Solvers.f90:1190-1855, face speed 0,
// n_disc 0): everything that chlld computes for both sides of the face -- the B scaling,
// |b|^2, the fast speeds, total pressures, S - u, rho*, the star-state coefficients tv / tb,
// the star velocities and fields, sqrt(rho*) -- is one paired operation for the two sides;
// what follows the wave-fan selection is computed for the selected side alone.
#pragma once
#include "mhd_core.cuh"

namespace sb {

struct F2 {
    float x, y;   // (left, right)
};
__device__ __forceinline__ F2 mk(float a, float b) { return F2{a, b}; }
__device__ __forceinline__ F2 splat(float a) { return F2{a, a}; }
__device__ __forceinline__ float2 f2v(F2 a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ F2 vf2(float2 a) { return F2{a.x, a.y}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return vf2(__fadd2_rn(f2v(a), f2v(b))); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return vf2(__fadd2_rn(f2v(a), f2v(F2{-b.x, -b.y}))); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return vf2(__fmul2_rn(f2v(a), f2v(b))); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return vf2(__ffma2_rn(f2v(a), f2v(b), f2v(c))); }
__device__ __forceinline__ F2 rcp2(F2 a) { return F2{sb_rcp(a.x), sb_rcp(a.y)}; }
__device__ __forceinline__ F2 sqrt2(F2 a) { return F2{sb_sqrt(a.x), sb_sqrt(a.y)}; }
__device__ __forceinline__ F2 rsqrt2(F2 a) { return F2{sb_rsqrt(a.x), sb_rsqrt(a.y)}; }
__device__ __forceinline__ F2 pos2(F2 a) { return F2{fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)}; }
__device__ __forceinline__ float pick(F2 a, bool right) { return right ? a.y : a.x; }

// minmod of each lane (the branch-free FP32 form of mhd_core.cuh's minmod)
__device__ __forceinline__ F2 minmod2(F2 a, F2 b) { return F2{minmod(a.x, b.x), minmod(a.y, b.y)}; }

// The MUSCL-minmod face states of both sides at once (reconstruct() of mhd_core.cuh, second
// order): side L is t_c + 0.5*minmod(t_c - t_f, t_n - t_c) with (t_f, t_c, t_n) = (LL, L, R),
// side R the same with (RR, R, L); each variable's two sides are one f32x2 pair.  Positivity
// fallback of cuf_solvers.cuf:394-406; B stays first order.
__device__ __forceinline__ void reconstruct_f32x2(const float* qLL, const float* qL, const float* qR,
                                                  const float* qRR, float* q1, float* q2) {
#pragma unroll
    for (int v = 0; v < 8; v++) {
        q1[v] = qL[v];
        q2[v] = qR[v];
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        const F2 c = mk(qL[v], qR[v]), fa = mk(qLL[v], qRR[v]), ne = mk(qR[v], qL[v]);
        const F2 r = fma2(splat(0.5f), minmod2(c - fa, ne - c), c);
        q1[v] = r.x;
        q2[v] = r.y;
    }
    if (q1[0] < 0.0f) q1[0] = qL[0];
    if (q1[4] < 0.0f) q1[4] = qL[4];
    if (q2[0] < 0.0f) q2[0] = qR[0];
    if (q2[4] < 0.0f) q2[4] = qR[4];
}

// Face-frame states q = (rho, vn, vt1, vt2, p, Bn, Bt1, Bt2), B in stored units; F in the same
// order (B fluxes in stored units); SL, SR, SM as chlld's dsl, dsp, dsc.  Returns kFlagWave when
// no wave-fan region matched and kFlagStar when the selected state has rho <= 0 or p <= 0 or
// a flux is not finite (the caller then recomputes the face in FP64).
template <int NSTATE>
__device__ __forceinline__ int riemann_f32x2(const float* q1, const float* q2, float* F, float& SLo, float& SRo,
                                             float& SMo) {
    static_assert(NSTATE == 2 || NSTATE == 3, "HLLC or HLLD");
    const float ispi4 = (float)kInvSpi4, half = 0.5f;
    const F2 r = mk(q1[0], q2[0]), u = mk(q1[1], q2[1]), v = mk(q1[2], q2[2]), w = mk(q1[3], q2[3]);
    const F2 p = mk(q1[4], q2[4]);
    const F2 bx = mk(q1[5], q2[5]) * splat(ispi4), by = mk(q1[6], q2[6]) * splat(ispi4);
    const F2 bz = mk(q1[7], q2[7]) * splat(ispi4);

    // fast magnetosonic speeds (Solvers.f90:1282-1306, in the two-square-root form of riemann())
    const F2 ir = rcp2(r);
    const F2 bxx = bx * bx;
    const F2 b2 = fma2(bz, bz, fma2(by, by, bxx));
    const F2 c2 = splat((float)kGamma) * p * ir;
    const F2 s = fma2(b2, ir, c2);
    const F2 disc = pos2(s * s - splat(4.0f) * c2 * (bxx * ir));
    const F2 cf = sqrt2(splat(half) * (s + sqrt2(disc)));
    const F2 pt = fma2(splat(half), b2, p);

    // wave speeds and the contact speed (:1308-1348)
    const F2 um = u - cf, up = u + cf;
    const float SL = fminf(um.x, um.y), SR = fmaxf(up.x, up.y);
    const F2 S = mk(SL, SR);
    const F2 su = S - u;                      // (SL - u1, SR - u2)
    const F2 rsu = r * su;                    // (suL r1, suR r2)
    const F2 rsuu = rsu * u;
    const float idd = sb_rcp(rsu.y - rsu.x);
    const float SM = (((rsuu.y - pt.y) + pt.x) - rsuu.x) * idd;
    SLo = SL;
    SRo = SR;
    SMo = SM;

    // The wave-fan region first (FR, SR < 0, is the last match of the region chain and needs none
    // of the star quantities); the star states and energies only for the star regions.
    float bn = 0.0f;
    F2 ism = splat(0.0f), sum = splat(0.0f), rz = splat(0.0f);
    F2 vz2 = splat(0.0f), vz3 = splat(0.0f);           // star tangential velocity
    F2 bz2 = splat(0.0f), bz3 = splat(0.0f);           // star tangential field
    F2 rzs = splat(0.0f);                              // sqrt(rho*)
    float ptz = 0.0f, sbvz = 0.0f, sbn = 0.0f, SZL = SM, SZR = SM;
    bool ibn = false;
    int region = 6;   // 1: FL, 2: L*, 3: L**, 4: R**, 5: R*, 6: FR, 0: none
    if (!(SR < 0.0f)) {
        const float isrl = sb_rcp(SR - SL);
        bn = (SR * bx.y - SL * bx.x) * isrl;   // HLL average of the normal field
        const F2 sm = S - splat(SM);                       // (SL - SM, SR - SM)
        ism = rcp2(sm);
        sum = su * ism;
        rz = r * sum;                                     // star densities
        if (NSTATE == 2) {   // HLLC (:1465-1567)
            const F2 smu = splat(SM) - u;
            const F2 pzs = fma2(rsu, smu, pt);                // pt + r su (SM - u)
            ptz = half * (pzs.y + pzs.x);
            const F2 m = r * u;
            const F2 f1 = fma2(m, u, pt) - bxx, f2 = m * v - bx * by, f3 = m * w - bx * bz;
            const F2 f6 = u * by - v * bx, f7 = u * bz - w * bx;
            const F2 rv = r * v, rw = r * w;
            const float uz0 = ((SR * r.y - SL * r.x) + m.x - m.y) * isrl;
            const float uz1 = ((SR * m.y - SL * m.x) + f1.x - f1.y) * isrl;
            const float uz2 = ((SR * rv.y - SL * rv.x) + f2.x - f2.y) * isrl;
            const float uz3 = ((SR * rw.y - SL * rw.x) + f3.x - f3.y) * isrl;
            const float uz6 = ((SR * by.y - SL * by.x) + f6.x - f6.y) * isrl;
            const float uz7 = ((SR * bz.y - SL * bz.x) + f7.x - f7.y) * isrl;
            sbvz = ((bn * uz1 + uz6 * uz2) + uz7 * uz3) * sb_rcp(uz0);
            if (fabsf(bn) < (float)kEpsB) {
                vz2 = v;
                vz3 = w;
                bz2 = by * sum;
                bz3 = bz * sum;
            } else {
                const F2 c = splat(bn) * rcp2(rsu);
                vz2 = fma2(by - splat(uz6), c, v);
                vz3 = fma2(bz - splat(uz7), c, w);
                bz2 = splat(uz6);
                bz3 = splat(uz7);
            }
            if (SR < 0.0f) region = 6;
            else if (SM <= 0.0f && SR >= 0.0f) region = 5;
            else if (SL <= 0.0f && SM >= 0.0f) region = 2;
            else if (SL > 0.0f) region = 1;
            else region = 0;
        } else {             // HLLD (:1598-1814)
            const F2 rsupt = rsu * mk(pt.y, pt.x);           // (suL r1 ptR, suR r2 ptL)
            ptz = ((rsupt.y - rsupt.x) + r.x * r.y * su.y * su.x * (u.y - u.x)) * idd;
            const float bn2 = bn * bn;
            const F2 tt = rsu * sm - splat(bn2);             // r su (S - SM) - bn^2
            const F2 itt = rcp2(tt);
            const bool degL = fabsf(tt.x) <= (float)kTtEps, degR = fabsf(tt.y) <= (float)kTtEps;
            F2 tv = (splat(SM) - u) * itt;
            F2 tb = fma2(rsu, su, splat(-bn2)) * itt;        // (r su^2 - bn^2) / tt
            if (degL) tv.x = tb.x = 0.0f;
            if (degR) tv.y = tb.y = 0.0f;
            const F2 nbn = splat(-bn);
            vz2 = fma2(nbn, by * tv, v);
            vz3 = fma2(nbn, bz * tv, w);
            bz2 = by * tb;
            bz3 = bz * tb;
            const F2 isq = rsqrt2(rz);
            rzs = rz * isq;
            const float abn = fabsf(bn);
            if (abn > (float)kEpsB) {
                ibn = true;
                sbn = bn > 0.0f ? 1.0f : -1.0f;
                SZL = SM - abn * isq.x;
                SZR = SM + abn * isq.y;
            }
            if (SR < 0.0f) region = 6;
            else if (SZR <= 0.0f && SR >= 0.0f) region = 5;
            else if (ibn && SM <= 0.0f && SZR >= 0.0f) region = 4;
            else if (ibn && SZL <= 0.0f && SM >= 0.0f) region = 3;
            else if (SL <= 0.0f && SZL >= 0.0f) region = 2;
            else if (SL > 0.0f) region = 1;
            else region = 0;
        }
    }
    int flag = region == 0 ? kFlagWave : 0;
    const bool right = region >= 4;
    const bool use1 = (region >= 2 && region <= 5);
    const bool use2 = (region == 3 || region == 4);

    // the selected side: energy, physical flux, conserved vector (:1368-1404)
    const float rr = pick(r, right), uu = pick(u, right), vv = pick(v, right), ww = pick(w, right);
    const float pp = pick(p, right), bxs = pick(bx, right), bys = pick(by, right), bzs = pick(bz, right);
    const float pts = pick(pt, right), b2s = pick(b2, right);
    const float e = (pp * (float)kInvG1 + rr * (half * ((uu * uu + vv * vv) + ww * ww))) + half * b2s;
    const float sbv = (uu * bxs + vv * bys) + ww * bzs;
    const float m = rr * uu;
    // the two tangential components of each vector, and the flux assembly, as f32x2 pairs
    const F2 vw = mk(vv, ww), bt = mk(bys, bzs);
    const F2 fs23 = fma2(splat(m), vw, splat(-bxs) * bt);   // m v - bx by, m w - bx bz
    const F2 fs67 = fma2(splat(uu), bt, splat(-bxs) * vw);  // u by - v bx, u bz - w bx
    const F2 us23 = splat(rr) * vw;
    F2 Fo[4] = {mk(m, (m * uu + pts) - bxs * bxs), fs23, mk((e + pts) * uu - bxs * sbv, 0.0f), fs67};
    if (use1) {
        // the star state of the selected side and its energy (:1541-1544 / :1650-1656), the
        // double-star state (:1658-1718)
        float vzz2 = 0.0f, vzz3 = 0.0f, bzz2 = 0.0f, bzz3 = 0.0f;
        if (NSTATE == 3 && use2) {
            const float irzss = sb_rcp(rzs.y + rzs.x);
            const float rzps = rzs.y * rzs.x;
            vzz2 = ((rzs.x * vz2.x + rzs.y * vz2.y) + sbn * (bz2.y - bz2.x)) * irzss;
            vzz3 = ((rzs.x * vz3.x + rzs.y * vz3.y) + sbn * (bz3.y - bz3.x)) * irzss;
            bzz2 = ((rzs.x * bz2.y + rzs.y * bz2.x) + sbn * rzps * (vz2.y - vz2.x)) * irzss;
            bzz3 = ((rzs.x * bz3.y + rzs.y * bz3.x) + sbn * rzps * (vz3.y - vz3.x)) * irzss;
        }
        const float sums = pick(sum, right), isms = pick(ism, right);
        const float rzz = pick(rz, right), S1 = right ? SR : SL, S2 = right ? SZR : SZL;
        const float v2s = pick(vz2, right), v3s = pick(vz3, right), b2z = pick(bz2, right), b3z = pick(bz3, right);
        const float sbvS = NSTATE == 2 ? sbvz : (bn * SM + b2z * v2s) + b3z * v3s;
        const float ez = e * sums + (((ptz * SM - pts * uu) + bn * (sbv - sbvS)) * isms);
        float ezz = ez;
        if (NSTATE == 3 && use2) {
            const float sbzz = (bn * SM + bzz2 * vzz2) + bzz3 * vzz3;
            ezz = right ? ez + pick(rzs, true) * sbn * (sbvS - sbzz) : ez - pick(rzs, false) * sbn * (sbvS - sbzz);
        }
        const F2 uz23 = splat(rzz) * mk(v2s, v3s), uzz23 = splat(rzz) * mk(vzz2, vzz3);
        const F2 Us[4] = {mk(rr, m), us23, mk(e, bxs), bt};
        const F2 UZs[4] = {mk(rzz, rzz * SM), uz23, mk(ez, bn), mk(b2z, b3z)};
        const F2 UZZs[4] = {mk(rzz, rzz * SM), uzz23, mk(ezz, bn), mk(bzz2, bzz3)};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            F2 f = Fo[k];
            if (use2) f = fma2(splat(S2), UZZs[k] - UZs[k], f);
            Fo[k] = fma2(splat(S1), UZs[k] - Us[k], f);
        }
        // positivity of the selected star state (rho* > 0, p* = pt* - |b*|^2/2 > 0)
        const float w6 = use2 ? bzz2 : b2z, w7 = use2 ? bzz3 : b3z;
        if (!(rzz > 0.0f) || !(ptz - half * ((bn * bn + w6 * w6) + w7 * w7) > 0.0f)) flag |= kFlagStar;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        F[2 * k] = Fo[k].x;
        F[2 * k + 1] = Fo[k].y;
    }
    // normal-field flux (:1570-1581 / :1828-1839) and B fluxes back to stored units (:1846)
    const float spi4 = (float)kSpi4;
    F[5] = (-fmaxf(fabsf(SL), fabsf(SR)) * (bx.y - bx.x)) * spi4;
    F[6] *= spi4;
    F[7] *= spi4;
    // a non-finite component makes the sum non-finite (finite physical fluxes are far below the
    // FP32 range, so their sum cannot overflow): one test instead of eight
    const F2 s2 = (mk(F[0], F[1]) + mk(F[2], F[3])) + (mk(F[4], F[5]) + mk(F[6], F[7]));
    if (!(fabsf(s2.x + s2.y) < 3.0e38f)) flag |= kFlagStar;
    return flag;
}

}  // namespace sb
