// chlld_q.cuh -- the passive-scalar flux routine chlld_Q (SET_Fortran_Cuda_MHD/Solvers.f90:198-1141)
// for the host and the device.
//
// chlld_Q is chlld with a ninth conserved variable Q (a density-like scalar: its flux is Q vn and
// its star value Q (S - vn)/(S - SM), :483-524, :630-631, :833-834) and an optional second scalar
// passed in konvect_(3,1) (left, right, flux out).  Against chlld it changes
//   * epsb 1e-6 -> 1e-4 (:282) in the HLLC field-degeneracy test and the HLLD Alfven-wave test;
//   * the n_disc = 2 blend of the two wave-speed estimates, 0.75 -> 0.60 (:432);
//   * the HLLC star total pressure, now the HLLD expression (:639-640);
//   * the wave-fan selection: HLL and HLLC are else-if chains led by `SL > wv or ydar` /
//     `SL >= wv or ydar` (:550, :698); HLLD is three successive selections -- (L | L*) led by
//     `SL >= wv or ydar`, then (L** | R**) when |Bn| > epsb, then (R* | R) -- each overriding the
//     one before (:951-1090).
// null_bn1 and p_correct_ are accepted and overridden to .False. / phi = 1 (:266-267), so they
// change nothing.
//
// The face-frame arithmetic follows the design of riemann() in mhd_core.cuh: reciprocals instead
// of repeated divisions, fast speeds from the squared form, and the physical flux, conserved
// vector and star energy formed for the selected side only.  Both passive scalars take the same
// path: HLL gives ((TR sL vL - TL sR vR) + TR TL (sR - sL)) / (TR - TL) - FW; every other region
// is the side flux s v plus S1 (s* - s) with s* = s (S1 - v)/(S1 - SM), the double-star value
// being the star value (:877-880, and the zero SZR term of :1042 for konvect_).
#pragma once
#include "setb_internal.cuh"

namespace sb {

constexpr double kEpsBQ = 1.0e-4;    // Solvers.f90:282
constexpr double kBlendQ = 0.60;     // Solvers.f90:432

// q1, q2: face-frame states (rho, vn, vt1, vt2, p, Bn, Bt1, Bt2), B in stored units.
// s1, s2: the two passive scalars on each side (Q, konvect_).  F[8] (B fluxes in stored units),
// Fs[2], SL / SR / SM.  Returns kFlagWave when no wave-fan region matched.
template <typename T, int NSTATE>
SB_HD int riemann_q(const T* q1, const T* q2, const T* s1, const T* s2, T wv, int n_disc, bool ydar, T* F,
                    T* Fs, T& SLo, T& SRo, T& SMo) {
    const T ispi4 = T(kInvSpi4), ga = T(kGamma), ig1 = T(kInvG1), half = T(0.5);
    const T r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const T bx1 = q1[5] * ispi4, by1 = q1[6] * ispi4, bz1 = q1[7] * ispi4;
    const T r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const T bx2 = q2[5] * ispi4, by2 = q2[6] * ispi4, bz2 = q2[7] * ispi4;

    // fast speeds (:370-394) in the squared form of riemann()
    const T ir1 = sb_rcp(r1), ir2 = sb_rcp(r2);
    const T b2L = (bx1 * bx1 + by1 * by1) + bz1 * bz1, b21 = b2L * ir1, c2L = ga * p1 * ir1, sL = c2L + b21;
    const T cfL = sb_sqrt(half * (sL + sb_sqrt(sb_pos(sL * sL - T(4) * c2L * (bx1 * bx1 * ir1)))));
    const T ptL = p1 + half * b2L;
    const T b2R = (bx2 * bx2 + by2 * by2) + bz2 * bz2, b22 = b2R * ir2, c2R = ga * p2 * ir2, sR = c2R + b22;
    const T cfR = sb_sqrt(half * (sR + sb_sqrt(sb_pos(sR * sR - T(4) * c2R * (bx2 * bx2 * ir2)))));
    const T ptR = p2 + half * b2R;

    // wave speeds (:413-436)
    T SL = sb_min(u1 - cfL, u2 - cfR), SR = sb_max(u1 + cfL, u2 + cfR), cfC = T(0);
    if (n_disc != 0 || NSTATE == 0) {
        const T aC = half * (bx1 * sb_rsqrt(r1) + bx2 * sb_rsqrt(r2));
        const T b2o = half * (b22 + b21);
        const T cC = sb_sqrt(ga * (half * (p2 + p1)) * sb_rcp(half * (r2 + r1)));
        cfC = half * (sb_sqrt(sb_pos(b2o + cC * (cC + T(2) * aC))) + sb_sqrt(sb_pos(b2o + cC * (cC - T(2) * aC))));
        const T vC1 = half * (u1 + u2);
        const T SL1 = sb_min(u1 - cfL, vC1 - cfC), SR1 = sb_max(u2 + cfR, vC1 + cfC);
        if (n_disc == 1) {
            SL = SL1;
            SR = SR1;
        } else if (n_disc == 2) {
            SL = T(kBlendQ) * SL1 + T(1.0 - kBlendQ) * SL;
            SR = T(kBlendQ) * SR1 + T(1.0 - kBlendQ) * SR;
        }
    }
    const T suR = SR - u2, suL = SL - u1;
    const T idd = sb_rcp(suR * r2 - suL * r1);
    const T SM = (((suR * r2 * u2 - ptR) + ptL) - suL * r1 * u1) * idd;
    SLo = SL;
    SRo = SR;
    SMo = SM;
    if (NSTATE == 0) {   // :466-471
        const T TR0 = sb_abs(u1 + u2) * half + cfC;
        SL = -TR0;
        SR = TR0;
    }
    const T isrl = sb_rcp(SR - SL);
    const T bn = (SR * bx2 - SL * bx1) * isrl;   // UZ(6), FL(6) = FR(6) = 0
    int flag = 0;

    if (NSTATE <= 1) {   // :541-621
        const int hr = (SL > wv || ydar) ? 1 : (SL <= wv && wv <= SR) ? 2 : (SR < wv) ? 3 : 0;
        if (hr == 0) flag |= kFlagWave;
        const T TL = hr == 1 ? T(0) : SL, TR = hr == 3 ? T(0) : SR;
        const T a = TR * TL, ib = sb_rcp(TR - TL);
        const T e1 = (p1 * ig1 + r1 * (half * ((u1 * u1 + v1 * v1) + w1 * w1))) + half * b2L;
        const T e2 = (p2 * ig1 + r2 * (half * ((u2 * u2 + v2 * v2) + w2 * w2))) + half * b2R;
        const T sbv1 = (u1 * bx1 + v1 * by1) + w1 * bz1, sbv2 = (u2 * bx2 + v2 * by2) + w2 * bz2;
        const T m1 = r1 * u1, m2 = r2 * u2;
        const T FL[10] = {m1, (m1 * u1 + ptL) - bx1 * bx1, m1 * v1 - bx1 * by1, m1 * w1 - bx1 * bz1,
                          (e1 + ptL) * u1 - bx1 * sbv1, T(0), u1 * by1 - v1 * bx1, u1 * bz1 - w1 * bx1,
                          s1[0] * u1, s1[1] * u1};
        const T FR[10] = {m2, (m2 * u2 + ptR) - bx2 * bx2, m2 * v2 - bx2 * by2, m2 * w2 - bx2 * bz2,
                          (e2 + ptR) * u2 - bx2 * sbv2, T(0), u2 * by2 - v2 * bx2, u2 * bz2 - w2 * bx2,
                          s2[0] * u2, s2[1] * u2};
        const T UL[10] = {r1, m1, r1 * v1, r1 * w1, e1, bx1, by1, bz1, s1[0], s1[1]};
        const T UR[10] = {r2, m2, r2 * v2, r2 * w2, e2, bx2, by2, bz2, s2[0], s2[1]};
        T out[10];
#pragma unroll
        for (int k = 0; k < 10; k++) {
            const T fw = hr == 1   ? wv * UL[k]
                         : hr == 3 ? wv * UR[k]
                                   : wv * (((SR * UR[k] - SL * UL[k]) + FL[k] - FR[k]) * isrl);
            out[k] = ((TR * FL[k] - TL * FR[k]) + a * (UR[k] - UL[k])) * ib - fw;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = out[k];
        Fs[0] = out[8];
        Fs[1] = out[9];
    } else {
        const T isrm = sb_rcp(SR - SM), islm = sb_rcp(SL - SM);
        const T suRm = suR * isrm, suLm = suL * islm;
        const T rzR = r2 * suRm, rzL = r1 * suLm;
        // star total pressure, :639-640 (HLLC) and :817-818 (HLLD)
        const T ptz = ((suR * r2 * ptL - suL * r1 * ptR) + r1 * r2 * suR * suL * (u2 - u1)) * idd;
        T vzL2, vzL3, vzR2, vzR3, bzL2, bzL3, bzR2, bzR3;
        T vzz2 = T(0), vzz3 = T(0), bzz2 = T(0), bzz3 = T(0);
        T SZL = SM, SZR = SM, sbvz = T(0), rzRs = T(0), rzLs = T(0), sbn = T(0);
        int region;   // 1: L, 2: L*, 3: L**, 4: R**, 5: R*, 6: R, 0: none
        if (NSTATE == 2) {   // :624-812
            const T m1 = r1 * u1, m2 = r2 * u2;
            const T FL1 = (m1 * u1 + ptL) - bx1 * bx1, FR1 = (m2 * u2 + ptR) - bx2 * bx2;
            const T FL2 = m1 * v1 - bx1 * by1, FR2 = m2 * v2 - bx2 * by2;
            const T FL3 = m1 * w1 - bx1 * bz1, FR3 = m2 * w2 - bx2 * bz2;
            const T FL6 = u1 * by1 - v1 * bx1, FR6 = u2 * by2 - v2 * bx2;
            const T FL7 = u1 * bz1 - w1 * bx1, FR7 = u2 * bz2 - w2 * bx2;
            const T uz0 = ((SR * r2 - SL * r1) + m1 - m2) * isrl;
            const T uz1 = ((SR * m2 - SL * m1) + FL1 - FR1) * isrl;
            const T uz2 = ((SR * (r2 * v2) - SL * (r1 * v1)) + FL2 - FR2) * isrl;
            const T uz3 = ((SR * (r2 * w2) - SL * (r1 * w1)) + FL3 - FR3) * isrl;
            const T uz6 = ((SR * by2 - SL * by1) + FL6 - FR6) * isrl;
            const T uz7 = ((SR * bz2 - SL * bz1) + FL7 - FR7) * isrl;
            sbvz = ((bn * uz1 + uz6 * uz2) + uz7 * uz3) * sb_rcp(uz0);
            if (sb_abs(bn) < T(kEpsBQ)) {   // :666-675
                vzR2 = v2; vzR3 = w2; vzL2 = v1; vzL3 = w1;
                bzR2 = by2 * suRm; bzR3 = bz2 * suRm;
                bzL2 = by1 * suLm; bzL3 = bz1 * suLm;
            } else {
                const T cR = bn * sb_rcp(suR * r2), cL = bn * sb_rcp(suL * r1);
                vzR2 = v2 + (by2 - uz6) * cR;
                vzR3 = w2 + (bz2 - uz7) * cR;
                vzL2 = v1 + (by1 - uz6) * cL;
                vzL3 = w1 + (bz1 - uz7) * cL;
                bzR2 = uz6; bzR3 = uz7; bzL2 = uz6; bzL3 = uz7;
            }
            region = (SL >= wv || ydar) ? 1 : (SL <= wv && SM >= wv) ? 2 : (SM <= wv && SR >= wv) ? 5 : (SR < wv) ? 6 : 0;
        } else {             // :815-1090
            const T bn2 = bn * bn;
            T tvR = T(0), tbR = T(0), tvL = T(0), tbL = T(0);
            const T ttR = r2 * suR * (SR - SM) - bn2;
            if (!(sb_abs(ttR) <= T(kTtEps))) {
                const T i = sb_rcp(ttR);
                tvR = (SM - u2) * i;
                tbR = (r2 * suR * suR - bn2) * i;
            }
            const T ttL = r1 * suL * (SL - SM) - bn2;
            if (!(sb_abs(ttL) <= T(kTtEps))) {
                const T i = sb_rcp(ttL);
                tvL = (SM - u1) * i;
                tbL = (r1 * suL * suL - bn2) * i;
            }
            vzL2 = v1 - bn * by1 * tvL;
            vzL3 = w1 - bn * bz1 * tvL;
            vzR2 = v2 - bn * by2 * tvR;
            vzR3 = w2 - bn * bz2 * tvR;
            bzL2 = by1 * tbL;
            bzL3 = bz1 * tbL;
            bzR2 = by2 * tbR;
            bzR3 = bz2 * tbR;
            const T isR = sb_rsqrt(rzR), isL = sb_rsqrt(rzL);
            rzRs = rzR * isR;
            rzLs = rzL * isL;
            const T abn = sb_abs(bn);
            const bool ibn = abn > T(kEpsBQ);
            if (ibn) {
                sbn = bn > T(0) ? T(1) : T(-1);
                SZL = SM - abn * isL;
                SZR = SM + abn * isR;
            }
            const int rA = (SL >= wv || ydar) ? 1 : (SL <= wv && SZL >= wv) ? 2 : 0;
            const int rB = !ibn ? 0 : (SZL <= wv && SM >= wv) ? 3 : (SM <= wv && SZR >= wv) ? 4 : 0;
            const int rC = (SZR <= wv && SR >= wv) ? 5 : (SR < wv) ? 6 : 0;
            region = rC ? rC : (rB ? rB : rA);
            if (region == 3 || region == 4) {
                const T irzss = sb_rcp(rzRs + rzLs);
                const T rzps = rzRs * rzLs;
                vzz2 = ((rzLs * vzL2 + rzRs * vzR2) + sbn * (bzR2 - bzL2)) * irzss;
                vzz3 = ((rzLs * vzL3 + rzRs * vzR3) + sbn * (bzR3 - bzL3)) * irzss;
                bzz2 = ((rzLs * bzR2 + rzRs * bzL2) + sbn * rzps * (vzR2 - vzL2)) * irzss;
                bzz3 = ((rzLs * bzR3 + rzRs * bzL3) + sbn * rzps * (vzR3 - vzL3)) * irzss;
            }
        }
        if (region == 0) flag |= kFlagWave;
        const bool right = region >= 4;
        const bool use1 = region >= 2 && region <= 5;
        const bool use2 = region == 3 || region == 4;
        const T r = right ? r2 : r1, u = right ? u2 : u1, v = right ? v2 : v1, w = right ? w2 : w1;
        const T p = right ? p2 : p1, bx = right ? bx2 : bx1, by = right ? by2 : by1, bz = right ? bz2 : bz1;
        const T pt = right ? ptR : ptL, b2 = right ? b2R : b2L;
        const T sum = right ? suRm : suLm, ism = right ? isrm : islm, rz = right ? rzR : rzL;
        const T S1 = right ? SR : SL, S2 = right ? SZR : SZL;
        const T vz2 = right ? vzR2 : vzL2, vz3 = right ? vzR3 : vzL3;
        const T bz2_ = right ? bzR2 : bzL2, bz3_ = right ? bzR3 : bzL3;
        const T e = (p * ig1 + r * (half * ((u * u + v * v) + w * w))) + half * b2;
        const T sbv = (u * bx + v * by) + w * bz;
        const T m = r * u;
        const T sbvS = NSTATE == 2 ? sbvz : (bn * SM + bz2_ * vz2) + bz3_ * vz3;
        const T ez = e * sum + (((ptz * SM - pt * u) + bn * (sbv - sbvS)) * ism);
        T ezz = ez;
        if (NSTATE == 3 && use2) {
            const T sbzz = (bn * SM + bzz2 * vzz2) + bzz3 * vzz3;
            ezz = right ? ez + rzRs * sbn * (sbvS - sbzz) : ez - rzLs * sbn * (sbvS - sbzz);
        }
        const T sa = right ? s2[0] : s1[0], sb = right ? s2[1] : s1[1];
        const T Fx[10] = {m, (m * u + pt) - bx * bx, m * v - bx * by, m * w - bx * bz, (e + pt) * u - bx * sbv,
                          T(0), u * by - v * bx, u * bz - w * bx, sa * u, sb * u};
        const T Ux[10] = {r, m, r * v, r * w, e, bx, by, bz, sa, sb};
        const T UZ[10] = {rz, rz * SM, rz * vz2, rz * vz3, ez, bn, bz2_, bz3_, sa * sum, sb * sum};
        const T UZZ[10] = {rz, rz * SM, rz * vzz2, rz * vzz3, ezz, bn, bzz2, bzz3, sa * sum, sb * sum};
        T out[10];
#pragma unroll
        for (int k = 0; k < 10; k++) {
            T f = Fx[k];
            if (use2) f = f + S2 * (UZZ[k] - UZ[k]);
            if (use1) f = f + S1 * (UZ[k] - Ux[k]);
            out[k] = f - wv * (use2 ? UZZ[k] : (use1 ? UZ[k] : Ux[k]));
        }
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = out[k];
        Fs[0] = out[8];
        Fs[1] = out[9];
        // normal-field flux, :777-788 / :1107-1120
        const T SN = sb_max(sb_abs(SL), sb_abs(SR));
        const T wbn = wv >= SR ? wv * bx2 : (wv <= SL ? wv * bx1 : wv * (bx1 + bx2) * half);
        F[5] = -SN * (bx2 - bx1) - wbn;
    }
    const T spi4 = T(kSpi4);
    F[5] *= spi4;
    F[6] *= spi4;
    F[7] *= spi4;
    return flag;
}

// General-normal chlld_Q: q1d / q2d are the reference's qqq1 / qqq2 (9 values, Q last), kv the
// konvect_(3,1) triplet or nullptr.  Writes qqq[9], sp = (dsl, dsp, dsc), *flag.
template <int NSTATE>
SB_HD void chlld_q_general(const double* nrm, double w, const double* q1d, const double* q2d, int n_disc, bool ydar,
                           double* kv, double* qqq, double* sp, int32_t* flag) {
    const double al = nrm[0], be = nrm[1], ge = nrm[2];
    double e2[3], e3[3];
    face_basis(nrm, q1d, q2d, e2, e3);
    double a[8], b[8], F[8], Fs[2], SL, SR, SM;
    const double* qs[2] = {q1d, q2d};
    double* outs[2] = {a, b};
    for (int s = 0; s < 2; s++) {
        const double* q = qs[s];
        double* o = outs[s];
        o[0] = q[0];
        o[4] = q[4];
        o[1] = q[1] * al + q[2] * be + q[3] * ge;
        o[2] = q[1] * e2[0] + q[2] * e2[1] + q[3] * e2[2];
        o[3] = q[1] * e3[0] + q[2] * e3[1] + q[3] * e3[2];
        o[5] = q[5] * al + q[6] * be + q[7] * ge;
        o[6] = q[5] * e2[0] + q[6] * e2[1] + q[7] * e2[2];
        o[7] = q[5] * e3[0] + q[6] * e3[1] + q[7] * e3[2];
    }
    const double s1[2] = {q1d[8], kv ? kv[0] : 0.0}, s2[2] = {q2d[8], kv ? kv[1] : 0.0};
    *flag = riemann_q<double, NSTATE>(a, b, s1, s2, w, n_disc, ydar, F, Fs, SL, SR, SM);
    qqq[0] = F[0];
    qqq[4] = F[4];
    qqq[8] = Fs[0];
    const double nn[3] = {al, be, ge};
    for (int c = 0; c < 3; c++) {
        qqq[1 + c] = nn[c] * F[1] + e2[c] * F[2] + e3[c] * F[3];
        qqq[5 + c] = nn[c] * F[5] + e2[c] * F[6] + e3[c] * F[7];
    }
    if (kv) kv[2] = Fs[1];
    sp[0] = SL;
    sp[1] = SR;
    sp[2] = SM;
}

}  // namespace sb
