// ============================================================================================
// oracle/oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU, FP64, scalar restatement of SergeyMSU/SET's ideal-MHD finite-volume step, written
// independently of the CUDA kernels in set_b200/csrc.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it, and only as the checker or the timed CPU
// baseline -- never as the thing measured or shipped.
//
// What it restates (paths are inside the reference project):
//   * chlld, all four n_state branches and n_disc 0/1/2 ........ SET_Fortran_Cuda_MHD/Solvers.f90:1144-1859
//   * chlld_Q (chlld + passive scalar Q + konvect_ scalar + ydar) SET_Fortran_Cuda_MHD/Solvers.f90:198-1141
//   * signum / minmod / linear ................................. SET_Fortran_Cuda_MHD/Solvers.f90:109-150
//   * face semantics (TVD of vars 1..5, positivity fallback, dt candidate, flux*square)
//                                                                SET_Fortran_Cuda_MHD/cuf_solvers.cuf:243-440
//   * cell semantics (owner-signed flux sum, Euler / Heun RK2, p floor 1e-7)
//                                                                SET_Fortran_Cuda_MHD/cuf_solvers.cuf:443-558, 561-794
//   * time loop (lagged dt: a step uses the dt reduced in the previous step's first stage;
//     first dt = 2e-9; reset value 1e15) ...................... SET_Fortran_Cuda_MHD/cuf_kernel.cuf:758, 780-925
// on a uniform Cartesian grid whose face lists are implicit (the reference's face-list
// geometry with dist = h/2, df = h/2, dff = 3h/2, square = h_b*h_c, volume = hx*hy*hz), and on
// an explicit face list (orc_fl_run: cells, faces, face types 2/4/5, TVD neighbours).
//
// Parity pinning.  The reference ships no tests, fixtures or golden vectors, and its Fortran
// path cannot be compiled here (no Fortran compiler).  The n_state <= 1 (HLL) branch of chlld,
// which also exercises the shared set-up (rotation basis, fast speeds, SL/SR/SM, FL/FR/UL/UR,
// UZ, rotation back, B scaling), is pinned against the reference's own C++ translation
// Solvers::HLLD_Solver_Alexashov (SET_Gelios/source/Solvers.cpp:92-691, n_state hard-wired to
// 1 at :97), compiled from the reference sources into oracle/_ref by oracle/Makefile.  The
// HLLC and HLLD branches and the Cartesian driver are parity unpinned: they are checked by
// property tests (consistency, mirror symmetry, conservation, B->0 limits) only.
//
// Build: g++ -std=c++17 -O2 -ffp-contract=off -fopenmp (no fast-math), see oracle/Makefile.
// ============================================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

// Storage_module.f90:8-9
const double cpi4 = 12.56637061435917295384;
const double ggg = 5.0 / 3.0;
// cuf_solvers.cuf:778 -- the FP32 literal 0.0000001 promoted to real(8)
const double p_floor = (double)0.0000001f;
// cuf_solvers.cuf:268 -- per-face initial value of the dt candidate (FP32 literal 100000.0)
const double dt_face_cap = (double)100000.0f;
// cuf_kernel.cuf:790 -- value time_step2 is reset to at the start of every step
const double dt_reset = 1000000000000000.0;

// ---------------------------------------------------------------- Solvers.f90:109-123
int signum(double x) {
    if (x > 0) return 1;
    if (x < 0) return -1;
    return 0;
}
// Solvers.f90:126-137
double minmod(double x, double y) {
    if (signum(x) + signum(y) == 0) return 0.0;
    // ((signum(x)+signum(y))/2.0): integer sum converted to default real, divided by 2.0
    return ((double)(float)(signum(x) + signum(y)) / 2.0) * std::min(std::fabs(x), std::fabs(y));
}
// Solvers.f90:141-150
double linear(double x1, double t1, double x2, double t2, double x3, double t3, double y) {
    double d = minmod((t1 - t2) / (x1 - x2), (t2 - t3) / (x2 - x3));
    return d * (y - x2) + t2;
}

// ---------------------------------------------------------------- Solvers.f90:1144-1859
// Returns 0 on success, 1 when the HLLD wave fan matched no region (the reference prints and
// STOPs at Solvers.f90:1816-1825), 2 when HLL/HLLC matched no region (non-finite speeds).
int chlld(int n_state, double al, double be, double ge, double w, const double* qqq1,
          const double* qqq2, double& dsl, double& dsp, double& dsc, double* qqq, int n_disc) {
    const double x0 = 0., x1 = 1., x2 = 2., x3 = 3., x5 = 5.;   // data x0..x9 (:1175)
    double FR[8], FL[8], FW[8], UL[8], UZ[8], UR[8], UZL[8], UZR[8], UZZL[8], UZZR[8], dq[8];
    double vL[3], vR[3], bL[3], bR[3], vzL[3], vzR[3], bzL[3], bzR[3];
    double vzzL[3], vzzR[3], bzzL[3], bzzR[3], aco[3][3], qv[3], qb[3];
    int fw_set = 0;

    const int n_disco = n_disc;                    // :1183-1187
    const double spi4 = std::sqrt(cpi4);           // :1192
    const double eps = 1.0e-12;                    // :1194
    const double epsb = 1.0e-06;                   // :1195
    const double ga = x5 / x3;                     // :1200
    const double g1 = ga - x1;
    const double wv = w;

    double r1 = qqq1[0], u1 = qqq1[1], v1 = qqq1[2], w1 = qqq1[3], p1 = qqq1[4];
    double bx1 = qqq1[5] / spi4, by1 = qqq1[6] / spi4, bz1 = qqq1[7] / spi4;
    double r2 = qqq2[0], u2 = qqq2[1], v2 = qqq2[2], w2 = qqq2[3], p2 = qqq2[4];
    double bx2 = qqq2[5] / spi4, by2 = qqq2[6] / spi4, bz2 = qqq2[7] / spi4;

    double ro = (r2 + r1) / x2;                    // :1226-1233
    double ap = (p2 + p1) / x2;
    double abx = (bx2 + bx1) / x2;
    double aby = (by2 + by1) / x2;
    double abz = (bz2 + bz1) / x2;

    double bk = abx * al + aby * be + abz * ge;    // :1236-1273
    double b2 = abx * abx + aby * aby + abz * abz;
    double d = b2 - bk * bk;
    aco[0][0] = al;
    aco[1][0] = be;
    aco[2][0] = ge;
    if (d > eps) {
        d = std::sqrt(d);
        aco[0][1] = (abx - bk * al) / d;
        aco[1][1] = (aby - bk * be) / d;
        aco[2][1] = (abz - bk * ge) / d;
        aco[0][2] = (aby * ge - abz * be) / d;
        aco[1][2] = (abz * al - abx * ge) / d;
        aco[2][2] = (abx * be - aby * al) / d;
    } else {
        double aix, aiy, aiz;
        if (std::fabs(al) < std::fabs(be) && std::fabs(al) < std::fabs(ge)) {
            aix = x1; aiy = x0; aiz = x0;
        } else if (std::fabs(be) < std::fabs(ge)) {
            aix = x0; aiy = x1; aiz = x0;
        } else {
            aix = x0; aiy = x0; aiz = x1;
        }
        double aik = aix * al + aiy * be + aiz * ge;
        d = std::sqrt(x1 - aik * aik);
        aco[0][1] = (aix - aik * al) / d;
        aco[1][1] = (aiy - aik * be) / d;
        aco[2][1] = (aiz - aik * ge) / d;
        aco[0][2] = (aiy * ge - aiz * be) / d;
        aco[1][2] = (aiz * al - aix * ge) / d;
        aco[2][2] = (aix * be - aiy * al) / d;
    }
    for (int i = 0; i < 3; i++) {                  // :1275-1280
        vL[i] = aco[0][i] * u1 + aco[1][i] * v1 + aco[2][i] * w1;
        vR[i] = aco[0][i] * u2 + aco[1][i] * v2 + aco[2][i] * w2;
        bL[i] = aco[0][i] * bx1 + aco[1][i] * by1 + aco[2][i] * bz1;
        bR[i] = aco[0][i] * bx2 + aco[1][i] * by2 + aco[2][i] * bz2;
    }

    double aaL = bL[0] / std::sqrt(r1);            // :1282-1306
    double b2L = bL[0] * bL[0] + bL[1] * bL[1] + bL[2] * bL[2];
    double b21 = b2L / r1;
    double cL = std::sqrt(ga * p1 / r1);
    double qp = std::sqrt(b21 + cL * (cL + x2 * aaL));
    double qm = std::sqrt(b21 + cL * (cL - x2 * aaL));
    double cfL = (qp + qm) / x2;
    double ptL = p1 + b2L / x2;

    double aaR = bR[0] / std::sqrt(r2);
    double b2R = bR[0] * bR[0] + bR[1] * bR[1] + bR[2] * bR[2];
    double b22 = b2R / r2;
    double cR = std::sqrt(ga * p2 / r2);
    qp = std::sqrt(b22 + cR * (cR + x2 * aaR));
    qm = std::sqrt(b22 + cR * (cR - x2 * aaR));
    double cfR = (qp + qm) / x2;
    double ptR = p2 + b2R / x2;

    double aC = (aaL + aaR) / x2;
    double b2o = (b22 + b21) / x2;
    double cC = std::sqrt(ga * ap / ro);
    qp = std::sqrt(b2o + cC * (cC + x2 * aC));
    qm = std::sqrt(b2o + cC * (cC - x2 * aC));
    double cfC = (qp + qm) / x2;
    double vC1 = (vL[0] + vR[0]) / x2;

    double SL = 0.0, SR = 0.0;                     // :1308-1330
    if (n_disco == 1) {
        SL = std::min((vL[0] - cfL), (vC1 - cfC));
        SR = std::max((vR[0] + cfR), (vC1 + cfC));
    }
    if (n_disco == 0) {
        SL = std::min((vL[0] - cfL), (vR[0] - cfR));
        SR = std::max((vL[0] + cfL), (vR[0] + cfR));
    }
    if (n_disco == 2) {
        double SL_1 = std::min((vL[0] - cfL), (vC1 - cfC));
        double SR_1 = std::max((vR[0] + cfR), (vC1 + cfC));
        double SL_2 = std::min((vL[0] - cfL), (vR[0] - cfR));
        double SR_2 = std::max((vL[0] + cfL), (vR[0] + cfR));
        double oo = 0.75;
        double oo1 = 1.0 - oo;
        SL = oo * SL_1 + oo1 * SL_2;
        SR = oo * SR_1 + oo1 * SR_2;
    }

    double suR = SR - vR[0];                       // :1341-1348
    double suL = SL - vL[0];
    double SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    dsl = SL;
    dsc = SM;
    dsp = SR;

    if (n_state == 0) {                            // :1360-1365
        double TR0 = std::fabs(vL[0] + vR[0]) / x2 + cfC;
        double TL0 = -TR0;
        SR = TR0;
        SL = TL0;
    }

    double upt1 = (u1 * u1 + v1 * v1 + w1 * w1) / x2;   // :1368-1375
    double sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    double upt2 = (u2 * u2 + v2 * v2 + w2 * w2) / x2;
    double sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    double e1 = p1 / g1 + r1 * upt1 + b2L / x2;
    double e2 = p2 / g1 + r2 * upt2 + b2R / x2;

    FL[0] = r1 * vL[0];                            // :1377-1393
    FL[1] = r1 * vL[0] * vL[0] + ptL - bL[0] * bL[0];
    FL[2] = r1 * vL[0] * vL[1] - bL[0] * bL[1];
    FL[3] = r1 * vL[0] * vL[2] - bL[0] * bL[2];
    FL[4] = (e1 + ptL) * vL[0] - bL[0] * sbv1;
    FL[5] = x0;
    FL[6] = vL[0] * bL[1] - vL[1] * bL[0];
    FL[7] = vL[0] * bL[2] - vL[2] * bL[0];
    FR[0] = r2 * vR[0];
    FR[1] = r2 * vR[0] * vR[0] + ptR - bR[0] * bR[0];
    FR[2] = r2 * vR[0] * vR[1] - bR[0] * bR[1];
    FR[3] = r2 * vR[0] * vR[2] - bR[0] * bR[2];
    FR[4] = (e2 + ptR) * vR[0] - bR[0] * sbv2;
    FR[5] = x0;
    FR[6] = vR[0] * bR[1] - vR[1] * bR[0];
    FR[7] = vR[0] * bR[2] - vR[2] * bR[0];

    UL[0] = r1;                                    // :1395-1404
    UL[4] = e1;
    UR[0] = r2;
    UR[4] = e2;
    for (int ik = 0; ik < 3; ik++) {
        UL[ik + 1] = r1 * vL[ik];
        UL[ik + 5] = bL[ik];
        UR[ik + 1] = r2 * vR[ik];
        UR[ik + 5] = bR[ik];
    }
    for (int ik = 0; ik < 8; ik++)                 // :1406-1408
        UZ[ik] = (SR * UR[ik] - SL * UL[ik] + FL[ik] - FR[ik]) / (SR - SL);

    if (n_state <= 1) {                            // :1414-1463  HLL / Lax
        for (int ik = 0; ik < 8; ik++) dq[ik] = UR[ik] - UL[ik];
        double TL = SL, TR = SR;
        if (SL > wv) {
            TL = x0;
            for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UL[ik];
            fw_set = 1;
        }
        if (SL <= wv && wv <= SR) {
            for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UZ[ik];
            fw_set = 1;
        }
        if (SR < wv) {
            TR = x0;
            for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UR[ik];
            fw_set = 1;
        }
        if (!fw_set) return 2;
        double a = TR * TL;
        double b = TR - TL;
        qqq[0] = (TR * FL[0] - TL * FR[0] + a * dq[0]) / b - FW[0];
        qqq[4] = (TR * FL[4] - TL * FR[4] + a * dq[4]) / b - FW[4];
        for (int ik = 1; ik < 4; ik++) qv[ik - 1] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
        for (int ik = 5; ik < 8; ik++) qb[ik - 5] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
        for (int i = 0; i < 3; i++) {
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        return 0;
    }

    if (n_state == 2) {                            // :1465-1596  HLLC
        int hit = 0;
        double suRm = suR / (SR - SM);
        double suLm = suL / (SL - SM);
        double rzR = r2 * suRm;
        double rzL = r1 * suLm;
        vzR[0] = SM;
        vzL[0] = SM;
        double ptzR = ptR + r2 * suR * (SM - vR[0]);
        double ptzL = ptL + r1 * suL * (SM - vL[0]);
        double ptz = (ptzR + ptzL) / x2;
        bzR[0] = UZ[5];
        bzL[0] = UZ[5];
        // :1479-1482 assign UZ(3)/UZ(1), UZ(4)/UZ(1), immediately overwritten at :1484-1487
        vzR[1] = vR[1] + UZ[5] * (bR[1] - UZ[6]) / suR / r2;
        vzR[2] = vR[2] + UZ[5] * (bR[2] - UZ[7]) / suR / r2;
        vzL[1] = vL[1] + UZ[5] * (bL[1] - UZ[6]) / suL / r1;
        vzL[2] = vL[2] + UZ[5] * (bL[2] - UZ[7]) / suL / r1;
        bzR[1] = UZ[6];
        bzR[2] = UZ[7];
        bzL[1] = bzR[1];
        bzL[2] = bzR[2];
        double sbvz = (UZ[5] * UZ[1] + UZ[6] * UZ[2] + UZ[7] * UZ[3]) / UZ[0];
        double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + UZ[5] * (sbv2 - sbvz)) / (SR - SM);
        double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + UZ[5] * (sbv1 - sbvz)) / (SL - SM);
        if (std::fabs(UZ[5]) < epsb) {
            vzR[1] = vR[1];
            vzR[2] = vR[2];
            vzL[1] = vL[1];
            vzL[2] = vL[2];
            bzR[1] = bR[1] * suRm;
            bzR[2] = bR[2] * suRm;
            bzL[1] = bL[1] * suLm;
            bzL[2] = bL[2] * suLm;
        }
        UZL[0] = rzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[4] = ezR;
        for (int ik = 0; ik < 3; ik++) {
            UZL[ik + 1] = vzL[ik] * rzL;
            UZL[ik + 5] = bzL[ik];
            UZR[ik + 1] = vzR[ik] * rzR;
            UZR[ik + 5] = bzR[ik];
        }
        if (SL > wv) {
            qqq[0] = FL[0] - wv * UL[0];
            qqq[4] = FL[4] - wv * UL[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] - wv * UL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] - wv * UL[ik];
            hit = 1;
        }
        if (SL <= wv && SM >= wv) {
            qqq[0] = FL[0] + SL * (rzL - r1) - wv * UZL[0];
            qqq[4] = FL[4] + SL * (ezL - e1) - wv * UZL[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            hit = 1;
        }
        if (SM <= wv && SR >= wv) {
            qqq[0] = FR[0] + SR * (rzR - r2) - wv * UZR[0];
            qqq[4] = FR[4] + SR * (ezR - e2) - wv * UZR[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            hit = 1;
        }
        if (SR < wv) {
            qqq[0] = FR[0] - wv * UR[0];
            qqq[4] = FR[4] - wv * UR[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] - wv * UR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] - wv * UR[ik];
            hit = 1;
        }
        if (!hit) return 2;
        double SN = std::max(std::fabs(SL), std::fabs(SR));   // :1570-1581
        double wbn = x0;
        if (wv >= SR) wbn = wv * bR[0];
        else if (wv <= SL) wbn = wv * bL[0];
        else wbn = wv * (bL[0] + bR[0]) / x2;
        qb[0] = -SN * (bR[0] - bL[0]) - wbn;
        for (int i = 0; i < 3; i++) {
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        return 0;
    }

    if (n_state == 3) {                            // :1598-1855  HLLD
        double ptz = (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                     (suR * r2 - suL * r1);
        vzL[0] = SM;
        vzR[0] = SM;
        vzzL[0] = SM;
        vzzR[0] = SM;
        double suRm = suR / (SR - SM);
        double suLm = suL / (SL - SM);
        double rzR = r2 * suRm;
        double rzL = r1 * suLm;
        double bn = UZ[5];
        double bn2 = bn * bn;
        bzL[0] = bn;
        bzR[0] = bn;
        bzzL[0] = bn;
        bzzR[0] = bn;

        double tvR, tbR, tvL, tbL;
        double ttR = r2 * suR * (SR - SM) - bn2;
        if (std::fabs(ttR) <= 1.0e-09) {
            tvR = x0;
            tbR = x0;
        } else {
            tvR = (SM - vR[0]) / ttR;
            tbR = (r2 * suR * suR - bn2) / ttR;
        }
        double ttL = r1 * suL * (SL - SM) - bn2;
        if (std::fabs(ttL) <= 1.0e-09) {
            tvL = x0;
            tbL = x0;
        } else {
            tvL = (SM - vL[0]) / ttL;
            tbL = (r1 * suL * suL - bn2) / ttL;
        }
        vzL[1] = vL[1] - bn * bL[1] * tvL;
        vzL[2] = vL[2] - bn * bL[2] * tvL;
        vzR[1] = vR[1] - bn * bR[1] * tvR;
        vzR[2] = vR[2] - bn * bR[2] * tvR;
        bzL[1] = bL[1] * tbL;
        bzL[2] = bL[2] * tbL;
        bzR[1] = bR[1] * tbR;
        bzR[2] = bR[2] * tbR;

        double sbvL = bzL[0] * vzL[0] + bzL[1] * vzL[1] + bzL[2] * vzL[2];
        double sbvR = bzR[0] * vzR[0] + bzR[1] * vzR[1] + bzR[2] * vzR[2];
        double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + bn * (sbv2 - sbvR)) / (SR - SM);
        double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + bn * (sbv1 - sbvL)) / (SL - SM);

        double rzzR = rzR;
        double rzzL = rzL;
        double rzRs = std::sqrt(rzR);
        double rzLs = std::sqrt(rzL);
        double rzss = rzRs + rzLs;
        double rzps = rzRs * rzLs;
        double SZL = SM - std::fabs(bn) / rzLs;
        double SZR = SM + std::fabs(bn) / rzRs;
        int ibn = 0;
        double sbn;
        if (std::fabs(bn) > epsb) {
            sbn = std::fabs(bn) / bn;
            ibn = 1;
        } else {
            sbn = x0;
            ibn = 0;
            SZL = SM;
            SZR = SM;
        }
        vzzL[1] = (rzLs * vzL[1] + rzRs * vzR[1] + sbn * (bzR[1] - bzL[1])) / rzss;
        vzzL[2] = (rzLs * vzL[2] + rzRs * vzR[2] + sbn * (bzR[2] - bzL[2])) / rzss;
        vzzR[1] = vzzL[1];
        vzzR[2] = vzzL[2];
        bzzL[1] = (rzLs * bzR[1] + rzRs * bzL[1] + sbn * rzps * (vzR[1] - vzL[1])) / rzss;
        bzzL[2] = (rzLs * bzR[2] + rzRs * bzL[2] + sbn * rzps * (vzR[2] - vzL[2])) / rzss;
        bzzR[1] = bzzL[1];
        bzzR[2] = bzzL[2];
        double sbzz = bzzL[0] * vzzL[0] + bzzL[1] * vzzL[1] + bzzL[2] * vzzL[2];
        double ezzR = ezR + rzRs * sbn * (sbvR - sbzz);
        double ezzL = ezL - rzLs * sbn * (sbvL - sbzz);

        UZL[0] = rzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[4] = ezR;
        for (int ik = 0; ik < 3; ik++) {
            UZL[ik + 1] = vzL[ik] * rzL;
            UZL[ik + 5] = bzL[ik];
            UZR[ik + 1] = vzR[ik] * rzR;
            UZR[ik + 5] = bzR[ik];
        }
        UZZL[0] = rzzL;
        UZZL[4] = ezzL;
        UZZR[0] = rzzR;
        UZZR[4] = ezzR;
        for (int ik = 0; ik < 3; ik++) {
            UZZL[ik + 1] = vzzL[ik] * rzzL;
            UZZL[ik + 5] = bzzL[ik];
            UZZR[ik + 1] = vzzR[ik] * rzzR;
            UZZR[ik + 5] = bzzR[ik];
        }

        int j_ccs = -1;
        if (SL > wv) {
            qqq[0] = FL[0] - wv * UL[0];
            qqq[4] = FL[4] - wv * UL[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] - wv * UL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] - wv * UL[ik];
            j_ccs = 1;
        }
        if (SL <= wv && SZL >= wv) {
            for (int ik : {0, 4}) qqq[ik] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            j_ccs = 2;
        }
        if (ibn == 1) {
            if (SZL <= wv && SM >= wv) {
                for (int ik : {0, 4})
                    qqq[ik] = FL[ik] + SZL * (UZZL[ik] - UZL[ik]) + SL * (UZL[ik] - UL[ik]) - wv * UZZL[ik];
                for (int ik = 1; ik < 4; ik++)
                    qv[ik - 1] = FL[ik] + SZL * (UZZL[ik] - UZL[ik]) + SL * (UZL[ik] - UL[ik]) - wv * UZZL[ik];
                for (int ik = 5; ik < 8; ik++)
                    qb[ik - 5] = FL[ik] + SZL * (UZZL[ik] - UZL[ik]) + SL * (UZL[ik] - UL[ik]) - wv * UZZL[ik];
                j_ccs = 3;
            }
            if (SM <= wv && SZR >= wv) {
                for (int ik : {0, 4})
                    qqq[ik] = FR[ik] + SZR * (UZZR[ik] - UZR[ik]) + SR * (UZR[ik] - UR[ik]) - wv * UZZR[ik];
                for (int ik = 1; ik < 4; ik++)
                    qv[ik - 1] = FR[ik] + SZR * (UZZR[ik] - UZR[ik]) + SR * (UZR[ik] - UR[ik]) - wv * UZZR[ik];
                for (int ik = 5; ik < 8; ik++)
                    qb[ik - 5] = FR[ik] + SZR * (UZZR[ik] - UZR[ik]) + SR * (UZR[ik] - UR[ik]) - wv * UZZR[ik];
                j_ccs = 4;
            }
        }
        if (SZR <= wv && SR >= wv) {
            for (int ik : {0, 4}) qqq[ik] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            j_ccs = 5;
        }
        if (SR < wv) {
            qqq[0] = FR[0] - wv * UR[0];
            qqq[4] = FR[4] - wv * UR[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] - wv * UR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] - wv * UR[ik];
            j_ccs = 6;
        }
        if (j_ccs == -1) return 1;
        double SN = std::max(std::fabs(SL), std::fabs(SR));   // :1828-1839
        double wbn = x0;
        if (wv >= SR) wbn = wv * bR[0];
        else if (wv <= SL) wbn = wv * bL[0];
        else wbn = wv * (bL[0] + bR[0]) / x2;
        qb[0] = -SN * (bR[0] - bL[0]) - wbn;
        for (int i = 0; i < 3; i++) {                          // :1843-1847
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        return 0;
    }
    return 0;   // n_state > 3: the reference leaves qqq untouched
}

// ---------------------------------------------------------------- Solvers.f90:198-1141
// chlld_Q: chlld with a ninth, passively advected variable Q (qqq(9), :293, :303) and an
// optional second passive scalar in konvect_(3,1) = (left value, right value, flux out).  What
// changes results against chlld: epsb = 1e-4 (:282); the n_disc = 2 blend weight 0.60 (:432);
// the HLLC star total pressure by the HLLD formula (:639); the HLL and HLLC wave-fan selection
// as else-if chains that STOP when nothing matched (:550-587, :698-774); `ydar`, which forces
// the left-state branch (:550, :698, :951).  null_bn1 and p_correct_ are read and then
// overridden (phi_p_correct = 1.0 at :266, null_bn = .False. at :267): they have no effect.
// kv is NULL when konvect_ is absent, else kv[0..2] = konvect_(1..3, 1); the declared shape
// (3, 1) makes size(konvect_(1, :)) = 1.
// Returns 0, or 1 when no wave-fan region matched (the reference prints and STOPs).
int chlld_q(int n_state, double al, double be, double ge, double w, const double* qqq1,
            const double* qqq2, double& dsl, double& dsp, double& dsc, double* qqq, int n_disc,
            bool ydar, double* kv) {
    const double x0 = 0., x1 = 1., x2 = 2., x3 = 3., x5 = 5.;
    double FR[9], FL[9], FW[9], UL[9], UZ[9], UR[9], UZL[9], UZR[9], UZZL[9], UZZR[9], dq[9];
    double vL[3], vR[3], bL[3], bR[3], vzL[3], vzR[3], bzL[3], bzR[3];
    double vzzL[3], vzzR[3], bzzL[3], bzzR[3], aco[3][3], qv[3], qb[3];
    double FL_ = 0.0, FR_ = 0.0, UZ_ = 0.0, FW_ = 0.0;

    const int n_disco = n_disc;                    // :269-273
    const double spi4 = std::sqrt(cpi4);           // :279
    const double eps = 1.0e-12;                    // :281
    const double epsb = 1.0e-04;                   // :282
    const double ga = x5 / x3;                     // :287
    const double g1 = ga - x1;
    const double wv = w;

    const double q1 = qqq1[8], r1 = qqq1[0], u1 = qqq1[1], v1 = qqq1[2], w1 = qqq1[3], p1 = qqq1[4];
    const double bx1 = qqq1[5] / spi4, by1 = qqq1[6] / spi4, bz1 = qqq1[7] / spi4;
    const double q2 = qqq2[8], r2 = qqq2[0], u2 = qqq2[1], v2 = qqq2[2], w2 = qqq2[3], p2 = qqq2[4];
    const double bx2 = qqq2[5] / spi4, by2 = qqq2[6] / spi4, bz2 = qqq2[7] / spi4;

    const double ro = (r2 + r1) / x2;              // :313-320
    const double ap = (p2 + p1) / x2;
    const double abx = (bx2 + bx1) / x2, aby = (by2 + by1) / x2, abz = (bz2 + bz1) / x2;

    const double bk = abx * al + aby * be + abz * ge;   // :323-360
    const double b2 = abx * abx + aby * aby + abz * abz;
    double d = b2 - bk * bk;
    aco[0][0] = al;
    aco[1][0] = be;
    aco[2][0] = ge;
    if (d > eps) {
        d = std::sqrt(d);
        aco[0][1] = (abx - bk * al) / d;
        aco[1][1] = (aby - bk * be) / d;
        aco[2][1] = (abz - bk * ge) / d;
        aco[0][2] = (aby * ge - abz * be) / d;
        aco[1][2] = (abz * al - abx * ge) / d;
        aco[2][2] = (abx * be - aby * al) / d;
    } else {
        double aix, aiy, aiz;
        if (std::fabs(al) < std::fabs(be) && std::fabs(al) < std::fabs(ge)) {
            aix = x1; aiy = x0; aiz = x0;
        } else if (std::fabs(be) < std::fabs(ge)) {
            aix = x0; aiy = x1; aiz = x0;
        } else {
            aix = x0; aiy = x0; aiz = x1;
        }
        const double aik = aix * al + aiy * be + aiz * ge;
        d = std::sqrt(x1 - aik * aik);
        aco[0][1] = (aix - aik * al) / d;
        aco[1][1] = (aiy - aik * be) / d;
        aco[2][1] = (aiz - aik * ge) / d;
        aco[0][2] = (aiy * ge - aiz * be) / d;
        aco[1][2] = (aiz * al - aix * ge) / d;
        aco[2][2] = (aix * be - aiy * al) / d;
    }
    for (int i = 0; i < 3; i++) {                  // :363-368
        vL[i] = aco[0][i] * u1 + aco[1][i] * v1 + aco[2][i] * w1;
        vR[i] = aco[0][i] * u2 + aco[1][i] * v2 + aco[2][i] * w2;
        bL[i] = aco[0][i] * bx1 + aco[1][i] * by1 + aco[2][i] * bz1;
        bR[i] = aco[0][i] * bx2 + aco[1][i] * by2 + aco[2][i] * bz2;
    }

    const double aaL = bL[0] / std::sqrt(r1);      // :370-394
    const double b2L = bL[0] * bL[0] + bL[1] * bL[1] + bL[2] * bL[2];
    const double b21 = b2L / r1;
    const double cL = std::sqrt(ga * p1 / r1);
    double qp = std::sqrt(b21 + cL * (cL + x2 * aaL));
    double qm = std::sqrt(b21 + cL * (cL - x2 * aaL));
    const double cfL = (qp + qm) / x2;
    const double ptL = p1 + b2L / x2;
    const double aaR = bR[0] / std::sqrt(r2);
    const double b2R = bR[0] * bR[0] + bR[1] * bR[1] + bR[2] * bR[2];
    const double b22 = b2R / r2;
    const double cR = std::sqrt(ga * p2 / r2);
    qp = std::sqrt(b22 + cR * (cR + x2 * aaR));
    qm = std::sqrt(b22 + cR * (cR - x2 * aaR));
    const double cfR = (qp + qm) / x2;
    const double ptR = p2 + b2R / x2;
    const double aC = (aaL + aaR) / x2;
    const double b2o = (b22 + b21) / x2;
    const double cC = std::sqrt(ga * ap / ro);
    qp = std::sqrt(b2o + cC * (cC + x2 * aC));
    qm = std::sqrt(b2o + cC * (cC - x2 * aC));
    const double cfC = (qp + qm) / x2;
    const double vC1 = (vL[0] + vR[0]) / x2;

    double SL = 0.0, SR = 0.0;                     // :413-436
    if (n_disco == 1) {
        SL = std::min((vL[0] - cfL), (vC1 - cfC));
        SR = std::max((vR[0] + cfR), (vC1 + cfC));
    }
    if (n_disco == 0) {
        SL = std::min((vL[0] - cfL), (vR[0] - cfR));
        SR = std::max((vL[0] + cfL), (vR[0] + cfR));
    }
    if (n_disco == 2) {
        const double SL_1 = std::min((vL[0] - cfL), (vC1 - cfC));
        const double SR_1 = std::max((vR[0] + cfR), (vC1 + cfC));
        const double SL_2 = std::min((vL[0] - cfL), (vR[0] - cfR));
        const double SR_2 = std::max((vL[0] + cfL), (vR[0] + cfR));
        const double oo = 0.60;
        const double oo1 = 1.0 - oo;
        SL = oo * SL_1 + oo1 * SL_2;
        SR = oo * SR_1 + oo1 * SR_2;
    }

    const double suR = SR - vR[0];                 // :447-454
    const double suL = SL - vL[0];
    const double SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    dsl = SL;
    dsc = SM;
    dsp = SR;

    if (n_state == 0) {                            // :466-471
        const double TR0 = std::fabs(vL[0] + vR[0]) / x2 + cfC;
        SR = TR0;
        SL = -TR0;
    }

    const double upt1 = (u1 * u1 + v1 * v1 + w1 * w1) / x2;   // :474-481
    const double sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const double upt2 = (u2 * u2 + v2 * v2 + w2 * w2) / x2;
    const double sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    const double e1 = p1 / g1 + r1 * upt1 + b2L / x2;
    const double e2 = p2 / g1 + r2 * upt2 + b2R / x2;

    FL[0] = r1 * vL[0];                            // :483-511
    FL[8] = q1 * vL[0];
    FL[1] = r1 * vL[0] * vL[0] + ptL - bL[0] * bL[0];
    FL[2] = r1 * vL[0] * vL[1] - bL[0] * bL[1];
    FL[3] = r1 * vL[0] * vL[2] - bL[0] * bL[2];
    FL[4] = (e1 + ptL) * vL[0] - bL[0] * sbv1;
    FL[5] = x0;
    FL[6] = vL[0] * bL[1] - vL[1] * bL[0];
    FL[7] = vL[0] * bL[2] - vL[2] * bL[0];
    if (kv) FL_ = kv[0] * vL[0];
    FR[0] = r2 * vR[0];
    FR[8] = q2 * vR[0];
    FR[1] = r2 * vR[0] * vR[0] + ptR - bR[0] * bR[0];
    FR[2] = r2 * vR[0] * vR[1] - bR[0] * bR[1];
    FR[3] = r2 * vR[0] * vR[2] - bR[0] * bR[2];
    FR[4] = (e2 + ptR) * vR[0] - bR[0] * sbv2;
    FR[5] = x0;
    FR[6] = vR[0] * bR[1] - vR[1] * bR[0];
    FR[7] = vR[0] * bR[2] - vR[2] * bR[0];
    if (kv) FR_ = kv[1] * vR[0];

    UL[0] = r1;                                    // :513-524
    UL[8] = q1;
    UL[4] = e1;
    UR[0] = r2;
    UR[8] = q2;
    UR[4] = e2;
    for (int ik = 0; ik < 3; ik++) {
        UL[ik + 1] = r1 * vL[ik];
        UL[ik + 5] = bL[ik];
        UR[ik + 1] = r2 * vR[ik];
        UR[ik + 5] = bR[ik];
    }
    for (int ik = 0; ik < 9; ik++)                 // :526-528
        UZ[ik] = (SR * UR[ik] - SL * UL[ik] + FL[ik] - FR[ik]) / (SR - SL);
    if (kv) UZ_ = (SR * kv[1] - SL * kv[0] + FL_ - FR_) / (SR - SL);   // :530-534

    if (n_state <= 1) {                            // :541-621  HLL / Lax
        for (int ik = 0; ik < 9; ik++) dq[ik] = UR[ik] - UL[ik];
        double TL = SL, TR = SR;
        if (SL > wv || ydar) {
            TL = x0;
            for (int ik = 0; ik < 9; ik++) FW[ik] = wv * UL[ik];
            if (kv) FW_ = wv * kv[0];
        } else if (SL <= wv && wv <= SR) {
            for (int ik = 0; ik < 9; ik++) FW[ik] = wv * UZ[ik];
            if (kv) FW_ = wv * UZ_;
        } else if (SR < wv) {
            TR = x0;
            for (int ik = 0; ik < 9; ik++) FW[ik] = wv * UR[ik];
            if (kv) FW_ = wv * kv[1];
        } else {
            return 1;                              // :584-587
        }
        const double a = TR * TL;
        const double b = TR - TL;
        qqq[0] = (TR * FL[0] - TL * FR[0] + a * dq[0]) / b - FW[0];
        qqq[8] = (TR * FL[8] - TL * FR[8] + a * dq[8]) / b - FW[8];
        qqq[4] = (TR * FL[4] - TL * FR[4] + a * dq[4]) / b - FW[4];
        for (int ik = 1; ik < 4; ik++) qv[ik - 1] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
        for (int ik = 5; ik < 8; ik++) qb[ik - 5] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
        for (int i = 0; i < 3; i++) {
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        if (kv) kv[2] = (TR * FL_ - TL * FR_ + a * (kv[1] - kv[0])) / b - FW_;   // :609-613
        return 0;
    }

    if (n_state == 2) {                            // :624-812  HLLC
        const double suRm = suR / (SR - SM);
        const double suLm = suL / (SL - SM);
        const double rzR = r2 * suRm, rzL = r1 * suLm;
        const double qzR = q2 * suRm, qzL = q1 * suLm;
        vzR[0] = SM;
        vzL[0] = SM;
        const double ptz = (suR * r2 * ptL - suL * r1 * ptR + 1.0 * r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                           (suR * r2 - suL * r1);  // :639-640, phi_p_correct = 1
        bzR[0] = UZ[5];
        bzL[0] = UZ[5];
        // :645-648 assign UZ(3)/UZ(1), UZ(4)/UZ(1), overwritten at :651-654
        vzR[1] = vR[1] + UZ[5] * (bR[1] - UZ[6]) / suR / r2;
        vzR[2] = vR[2] + UZ[5] * (bR[2] - UZ[7]) / suR / r2;
        vzL[1] = vL[1] + UZ[5] * (bL[1] - UZ[6]) / suL / r1;
        vzL[2] = vL[2] + UZ[5] * (bL[2] - UZ[7]) / suL / r1;
        bzR[1] = UZ[6];
        bzR[2] = UZ[7];
        bzL[1] = bzR[1];
        bzL[2] = bzR[2];
        const double sbvz = (UZ[5] * UZ[1] + UZ[6] * UZ[2] + UZ[7] * UZ[3]) / UZ[0];
        const double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + UZ[5] * (sbv2 - sbvz)) / (SR - SM);
        const double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + UZ[5] * (sbv1 - sbvz)) / (SL - SM);
        if (std::fabs(UZ[5]) < epsb) {             // :666-675
            vzR[1] = vR[1];
            vzR[2] = vR[2];
            vzL[1] = vL[1];
            vzL[2] = vL[2];
            bzR[1] = bR[1] * suRm;
            bzR[2] = bR[2] * suRm;
            bzL[1] = bL[1] * suLm;
            bzL[2] = bL[2] * suLm;
        }
        UZL[0] = rzL;                              // :684-696
        UZL[8] = qzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[8] = qzR;
        UZR[4] = ezR;
        for (int ik = 0; ik < 3; ik++) {
            UZL[ik + 1] = vzL[ik] * rzL;
            UZL[ik + 5] = bzL[ik];
            UZR[ik + 1] = vzR[ik] * rzR;
            UZR[ik + 5] = bzR[ik];
        }
        if (SL >= wv || ydar) {                    // :698-774
            qqq[0] = FL[0] - wv * UL[0];
            qqq[8] = FL[8] - wv * UL[8];
            qqq[4] = FL[4] - wv * UL[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] - wv * UL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] - wv * UL[ik];
            if (kv) kv[2] = FL_ - wv * kv[0];
        } else if (SL <= wv && SM >= wv) {
            qqq[0] = FL[0] + SL * (rzL - r1) - wv * UZL[0];
            qqq[8] = FL[8] + SL * (qzL - q1) - wv * UZL[8];
            qqq[4] = FL[4] + SL * (ezL - e1) - wv * UZL[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik];
            if (kv) kv[2] = FL_ + SL * (kv[0] * suLm - kv[0]) - wv * kv[0] * suLm;
        } else if (SM <= wv && SR >= wv) {
            qqq[0] = FR[0] + SR * (rzR - r2) - wv * UZR[0];
            qqq[8] = FR[8] + SR * (qzR - q2) - wv * UZR[8];
            qqq[4] = FR[4] + SR * (ezR - e2) - wv * UZR[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik];
            if (kv) kv[2] = FR_ + SR * (kv[1] * suRm - kv[1]) - wv * kv[1] * suRm;
        } else if (SR < wv) {
            qqq[0] = FR[0] - wv * UR[0];
            qqq[8] = FR[8] - wv * UR[8];
            qqq[4] = FR[4] - wv * UR[4];
            for (int ik = 1; ik < 4; ik++) qv[ik - 1] = FR[ik] - wv * UR[ik];
            for (int ik = 5; ik < 8; ik++) qb[ik - 5] = FR[ik] - wv * UR[ik];
            if (kv) kv[2] = FR_ - wv * kv[1];
        } else {
            return 1;                              // :769-774
        }
        const double SN = std::max(std::fabs(SL), std::fabs(SR));   // :777-790
        double wbn = x0;
        if (wv >= SR) wbn = wv * bR[0];
        else if (wv <= SL) wbn = wv * bL[0];
        else wbn = wv * (bL[0] + bR[0]) / x2;
        qb[0] = -SN * (bR[0] - bL[0]) - wbn;
        for (int i = 0; i < 3; i++) {              // :796-803
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        return 0;
    }

    if (n_state == 3) {                            // :815-1136  HLLD
        const double ptz = (suR * r2 * ptL - suL * r1 * ptR + 1.0 * r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                           (suR * r2 - suL * r1);
        vzL[0] = SM;
        vzR[0] = SM;
        vzzL[0] = SM;
        vzzR[0] = SM;
        const double suRm = suR / (SR - SM);
        const double suLm = suL / (SL - SM);
        const double rzR = r2 * suRm, rzL = r1 * suLm;
        const double qzR = q2 * suRm, qzL = q1 * suLm;
        const double bn = UZ[5];
        const double bn2 = bn * bn;
        bzL[0] = bn;
        bzR[0] = bn;
        bzzL[0] = bn;
        bzzR[0] = bn;
        double tvR, tbR, tvL, tbL;
        const double ttR = r2 * suR * (SR - SM) - bn2;   // :843-860
        if (std::fabs(ttR) <= 1.0e-09) {
            tvR = x0;
            tbR = x0;
        } else {
            tvR = (SM - vR[0]) / ttR;
            tbR = (r2 * suR * suR - bn2) / ttR;
        }
        const double ttL = r1 * suL * (SL - SM) - bn2;
        if (std::fabs(ttL) <= 1.0e-09) {
            tvL = x0;
            tbL = x0;
        } else {
            tvL = (SM - vL[0]) / ttL;
            tbL = (r1 * suL * suL - bn2) / ttL;
        }
        vzL[1] = vL[1] - bn * bL[1] * tvL;
        vzL[2] = vL[2] - bn * bL[2] * tvL;
        vzR[1] = vR[1] - bn * bR[1] * tvR;
        vzR[2] = vR[2] - bn * bR[2] * tvR;
        bzL[1] = bL[1] * tbL;
        bzL[2] = bL[2] * tbL;
        bzR[1] = bR[1] * tbR;
        bzR[2] = bR[2] * tbR;
        const double sbvL = bzL[0] * vzL[0] + bzL[1] * vzL[1] + bzL[2] * vzL[2];
        const double sbvR = bzR[0] * vzR[0] + bzR[1] * vzR[1] + bzR[2] * vzR[2];
        const double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + bn * (sbv2 - sbvR)) / (SR - SM);
        const double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + bn * (sbv1 - sbvL)) / (SL - SM);
        const double rzzR = rzR, rzzL = rzL;       // :877-888 (the Q square roots there are unused)
        const double qzzR = qzR, qzzL = qzL;
        const double rzRs = std::sqrt(rzR);
        const double rzLs = std::sqrt(rzL);
        const double rzss = rzRs + rzLs;
        const double rzps = rzRs * rzLs;
        double SZL = SM - std::fabs(bn) / rzLs;    // :890-902
        double SZR = SM + std::fabs(bn) / rzRs;
        int ibn;
        double sbn;
        if (std::fabs(bn) > epsb) {
            sbn = std::fabs(bn) / bn;
            ibn = 1;
        } else {
            sbn = x0;
            ibn = 0;
            SZL = SM;
            SZR = SM;
        }
        vzzL[1] = (rzLs * vzL[1] + rzRs * vzR[1] + sbn * (bzR[1] - bzL[1])) / rzss;
        vzzL[2] = (rzLs * vzL[2] + rzRs * vzR[2] + sbn * (bzR[2] - bzL[2])) / rzss;
        vzzR[1] = vzzL[1];
        vzzR[2] = vzzL[2];
        bzzL[1] = (rzLs * bzR[1] + rzRs * bzL[1] + sbn * rzps * (vzR[1] - vzL[1])) / rzss;
        bzzL[2] = (rzLs * bzR[2] + rzRs * bzL[2] + sbn * rzps * (vzR[2] - vzL[2])) / rzss;
        bzzR[1] = bzzL[1];
        bzzR[2] = bzzL[2];
        const double sbzz = bzzL[0] * vzzL[0] + bzzL[1] * vzzL[1] + bzzL[2] * vzzL[2];
        const double ezzR = ezR + rzRs * sbn * (sbvR - sbzz);
        const double ezzL = ezL - rzLs * sbn * (sbvL - sbzz);
        UZL[0] = rzL;                              // :923-947
        UZL[8] = qzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[8] = qzR;
        UZR[4] = ezR;
        UZZL[0] = rzzL;
        UZZL[8] = qzzL;
        UZZL[4] = ezzL;
        UZZR[0] = rzzR;
        UZZR[8] = qzzR;
        UZZR[4] = ezzR;
        for (int ik = 0; ik < 3; ik++) {
            UZL[ik + 1] = vzL[ik] * rzL;
            UZL[ik + 5] = bzL[ik];
            UZR[ik + 1] = vzR[ik] * rzR;
            UZR[ik + 5] = bzR[ik];
            UZZL[ik + 1] = vzzL[ik] * rzzL;
            UZZL[ik + 5] = bzzL[ik];
            UZZR[ik + 1] = vzzR[ik] * rzzR;
            UZZR[ik + 5] = bzzR[ik];
        }
        // :949-1090.  Three selections, each of which overwrites the previous one's result:
        // (L | L*) by an else-if chain with ydar forcing L, then (L** | R**) when the normal
        // field is not degenerate, then (R* | R).  Vars 1, 9, 5 are written as qqq, 2..4 and
        // 6..8 as the face-frame qv / qb.
        int j_ccs = -1;
        auto put = [&](int ik, double v) {
            if (ik >= 1 && ik <= 3) qv[ik - 1] = v;
            else if (ik >= 5 && ik <= 7) qb[ik - 5] = v;
            else qqq[ik] = v;
        };
        if (SL >= wv || ydar) {
            for (int ik = 0; ik < 9; ik++) put(ik, FL[ik] - wv * UL[ik]);
            j_ccs = 1;
            if (kv) kv[2] = FL_ - wv * kv[0];
        } else if (SL <= wv && SZL >= wv) {
            for (int ik = 0; ik < 9; ik++) put(ik, FL[ik] + SL * (UZL[ik] - UL[ik]) - wv * UZL[ik]);
            j_ccs = 2;
            if (kv) kv[2] = FL_ + SL * (kv[0] * suLm - kv[0]) - wv * kv[0] * suLm;
        }
        if (ibn == 1) {
            if (SZL <= wv && SM >= wv) {
                for (int ik = 0; ik < 9; ik++)
                    put(ik, FL[ik] + SZL * (UZZL[ik] - UZL[ik]) + SL * (UZL[ik] - UL[ik]) - wv * UZZL[ik]);
                j_ccs = 3;
                if (kv) kv[2] = FL_ + SL * (kv[0] * suLm - kv[0]) - wv * kv[0] * suLm;
            } else if (SM <= wv && SZR >= wv) {
                for (int ik = 0; ik < 9; ik++)
                    put(ik, FR[ik] + SZR * (UZZR[ik] - UZR[ik]) + SR * (UZR[ik] - UR[ik]) - wv * UZZR[ik]);
                j_ccs = 4;
                // :1042-1043 as written: the SZR term is SZR * (k2 suRm - k2 suRm)
                if (kv)
                    kv[2] = FR_ + SZR * (kv[1] * suRm - kv[1] * suRm) + SR * (kv[1] * suRm - kv[1]) -
                            wv * kv[1] * suRm;
            }
        }
        if (SZR <= wv && SR >= wv) {
            for (int ik = 0; ik < 9; ik++) put(ik, FR[ik] + SR * (UZR[ik] - UR[ik]) - wv * UZR[ik]);
            j_ccs = 5;
            if (kv) kv[2] = FR_ + SR * (kv[1] * suRm - kv[1]) - wv * kv[1] * suRm;
        } else if (SR < wv) {
            for (int ik = 0; ik < 9; ik++) put(ik, FR[ik] - wv * UR[ik]);
            j_ccs = 6;
            if (kv) kv[2] = FR_ - wv * kv[1];
        }
        if (j_ccs == -1) return 1;                 // :1092-1104
        const double SN = std::max(std::fabs(SL), std::fabs(SR));   // :1107-1121
        double wbn = x0;
        if (wv >= SR) wbn = wv * bR[0];
        else if (wv <= SL) wbn = wv * bL[0];
        else wbn = wv * (bL[0] + bR[0]) / x2;
        qb[0] = -SN * (bR[0] - bL[0]) - wbn;
        for (int i = 0; i < 3; i++) {              // :1125-1129
            qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
            qqq[i + 5] = aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2];
            qqq[i + 5] = spi4 * qqq[i + 5];
        }
        return 0;
    }
    return 0;   // n_state > 3: qqq untouched
}

// ------------------------------------------------------------------ conserved <-> primitive
// Conserved U = (rho, rho*u, rho*v, rho*w, E, Bx, By, Bz) with B in the reference's stored
// units; the energy carries |b|^2/2 with b = B/sqrt(4*pi) as chlld does (Solvers.f90:1212-1214,
// 1374).  Pressure recovery follows cuf_solvers.cuf:735-738 with the magnetic term added.
const double spi4g = std::sqrt(cpi4);
const double g1g = ggg - 1.0;

void prim_from_cons(const double* U, double* q) {
    double rho = U[0];
    double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
    double bx = U[5] / spi4g, by = U[6] / spi4g, bz = U[7] / spi4g;
    double ke = 0.5 * rho * ((u * u + v * v) + w * w);
    double me = 0.5 * ((bx * bx + by * by) + bz * bz);
    q[0] = rho;
    q[1] = u;
    q[2] = v;
    q[3] = w;
    q[4] = ((U[4] - ke) - me) * g1g;
    q[5] = U[5];
    q[6] = U[6];
    q[7] = U[7];
}

void cons_from_prim(const double* q, double* U) {
    double rho = q[0], u = q[1], v = q[2], w = q[3];
    double bx = q[5] / spi4g, by = q[6] / spi4g, bz = q[7] / spi4g;
    double ke = 0.5 * rho * ((u * u + v * v) + w * w);
    double me = 0.5 * ((bx * bx + by * by) + bz * bz);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = rho * w;
    U[4] = (q[4] / g1g + ke) + me;
    U[5] = q[5];
    U[6] = q[6];
    U[7] = q[7];
}

}  // namespace

// ============================================================================ C interface
extern "C" {

typedef struct {
    int32_t nx, ny, nz, flags;
    double lo[3], hi[3];
    double inflow[8];
    double r_src, rho_src, v_src, p_over_rho_src, r_floor;
    double dt_init;
} orc_grid;

typedef struct {
    int32_t n_state, n_disc, order, scheme;
    double cfl;
} orc_opts;

typedef struct {
    int64_t n_negdens, first_bad_cell, n_pfloor, n_wave_err, n_recon_err, reserved;
} orc_diag;

typedef struct {
    double time_all;   // dev_time_all
    double dt_next;    // time_step2: the dt the next step will use
    double dt_last;    // time_step: the dt the last step used
} orc_clock;

int orc_chlld(int n_state, double al, double be, double ge, double w, const double* q1,
              const double* q2, double* dsl, double* dsp, double* dsc, double* qqq, int n_disc) {
    return chlld(n_state, al, be, ge, w, q1, q2, *dsl, *dsp, *dsc, qqq, n_disc);
}

// kv: NULL (konvect_ absent) or konvect_(1:3, 1) in / in / out
int orc_chlld_q(int n_state, double al, double be, double ge, double w, const double* q1,
                const double* q2, double* dsl, double* dsp, double* dsc, double* qqq, int n_disc, int ydar,
                double* kv) {
    return chlld_q(n_state, al, be, ge, w, q1, q2, *dsl, *dsp, *dsc, qqq, n_disc, ydar != 0, kv);
}

double orc_minmod(double x, double y) { return minmod(x, y); }
double orc_linear(double x1, double t1, double x2, double t2, double x3, double t3, double y) {
    return linear(x1, t1, x2, t2, x3, t3, y);
}
void orc_prim_from_cons(const double* U, double* q) { prim_from_cons(U, q); }
void orc_cons_from_prim(const double* q, double* U) { cons_from_prim(q, U); }

// ------------------------------------------------------------- seeded initial condition
// SplitMix64 keyed by (seed, global cell index, draw id) so every implementation draws the
// same numbers.  LISM state outside r_src with +-pert_amp relative noise on rho and p; the
// source state inside r_src (the analogue of cuf_solvers.cuf:614-681).
static uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unit_draw(uint64_t seed, uint64_t cell, uint64_t which) {
    uint64_t h = splitmix64(splitmix64(seed) ^ (2 * cell + which));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static void cell_center(const orc_grid* g, int i, int j, int k, double* x) {
    double h0 = (g->hi[0] - g->lo[0]) / g->nx;
    double h1 = (g->hi[1] - g->lo[1]) / g->ny;
    double h2 = (g->hi[2] - g->lo[2]) / g->nz;
    x[0] = g->lo[0] + (i + 0.5) * h0;
    x[1] = g->lo[1] + (j + 0.5) * h1;
    x[2] = g->lo[2] + (k + 0.5) * h2;
}

// Source state (primitive) at a cell centre; returns 0 when the cell is outside r_src.
static int source_prim(const orc_grid* g, const double* x, double* q) {
    if (!(g->r_src > 0.0)) return 0;
    double r2 = (x[0] * x[0] + x[1] * x[1]) + x[2] * x[2];
    if (!(r2 < g->r_src * g->r_src)) return 0;
    double r = std::sqrt(r2);
    double re = std::max(r, g->r_floor);
    double s = g->r_src / re;
    double rho = (s * s) * g->rho_src;
    q[0] = rho;
    if (r > 0.0) {
        q[1] = g->v_src * (x[0] / r);
        q[2] = g->v_src * (x[1] / r);
        q[3] = g->v_src * (x[2] / r);
    } else {
        q[1] = q[2] = q[3] = 0.0;
    }
    q[4] = g->p_over_rho_src * rho;
    q[5] = q[6] = q[7] = 0.0;
    return 1;
}

// lism: unperturbed LISM primitive state (rho,u,v,w,p,Bx,By,Bz).  Output: conserved SoA U[8*N].
void orc_init_lism(const orc_grid* g, const double* lism, uint64_t seed, double pert_amp, double* U) {
    const int64_t N = (int64_t)g->nx * g->ny * g->nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; c++) {
        int i = (int)(c % g->nx);
        int j = (int)((c / g->nx) % g->ny);
        int k = (int)(c / ((int64_t)g->nx * g->ny));
        double x[3], q[8], u8[8];
        cell_center(g, i, j, k, x);
        if (!source_prim(g, x, q)) {
            double d1 = pert_amp * (2.0 * unit_draw(seed, (uint64_t)c, 0) - 1.0);
            double d2 = pert_amp * (2.0 * unit_draw(seed, (uint64_t)c, 1) - 1.0);
            q[0] = lism[0] * (1.0 + d1);
            q[4] = lism[4] * (1.0 + d2);
            q[1] = lism[1];
            q[2] = lism[2];
            q[3] = lism[3];
            q[5] = lism[5];
            q[6] = lism[6];
            q[7] = lism[7];
        }
        cons_from_prim(q, u8);
        for (int v = 0; v < 8; v++) U[v * N + c] = u8[v];
    }
}

// Cell_par(16,N) <-> conserved SoA.  Columns 9..16 are left untouched on output.
void orc_cellpar_to_cons(int64_t N, const double* cell_par, double* U) {
    for (int64_t c = 0; c < N; c++) {
        double u8[8];
        cons_from_prim(cell_par + 16 * c, u8);
        for (int v = 0; v < 8; v++) U[v * N + c] = u8[v];
    }
}
void orc_cons_to_cellpar(int64_t N, const double* U, double* cell_par) {
    for (int64_t c = 0; c < N; c++) {
        double u8[8];
        for (int v = 0; v < 8; v++) u8[v] = U[v * N + c];
        prim_from_cons(u8, cell_par + 16 * c);
    }
}

// ------------------------------------------------------------------------- one stage
// kind 0: Euler / Heun stage 1   Uout = Uin - dt*P/V
// kind 1: Heun stage 2           Uout = 0.5*((Ubase + Uin) - dt*P/V)    (cuf_solvers.cuf:741-770)
// Faces are computed once each and applied to both neighbours with the owner sign of
// cuf_solvers.cuf:691-703: the cell on the low side (s1) adds the flux, the high side subtracts.
// Flux accumulation order per cell: x-low, x-high, y-low, y-high, z-low, z-high.
static void stage(const orc_grid* g, const orc_opts* o, const double* Uin, const double* Ubase,
                  double* Uout, double dt, int kind, int want_dt, double* dt_min, orc_diag* dg,
                  int nthreads) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int64_t N = (int64_t)nx * ny * nz;
    const double h[3] = {(g->hi[0] - g->lo[0]) / nx, (g->hi[1] - g->lo[1]) / ny,
                         (g->hi[2] - g->lo[2]) / nz};
    const double square[3] = {h[1] * h[2], h[0] * h[2], h[0] * h[1]};
    const double volume = h[0] * h[1] * h[2];

    // primitive state of every cell
    std::vector<double> P((size_t)N * 8);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < N; c++) {
        double u8[8];
        for (int v = 0; v < 8; v++) u8[v] = Uin[v * N + c];
        prim_from_cons(u8, &P[(size_t)c * 8]);
    }
    auto prim_at = [&](int i, int j, int k) -> const double* {
        if (i >= nx) return g->inflow;           // fixed inflow beyond x = hi
        i = std::min(std::max(i, 0), nx - 1);    // zero-gradient elsewhere
        j = std::min(std::max(j, 0), ny - 1);
        k = std::min(std::max(k, 0), nz - 1);
        return &P[(size_t)(i + (int64_t)nx * (j + (int64_t)ny * k)) * 8];
    };

    // face flux between cell c-1 and cell c along axis a (stencil c-2..c+1); returns dt cand.
    auto face = [&](int a, int i, int j, int k, double* F, int64_t& nrec, int64_t& nwave) -> double {
        int di = (a == 0), dj = (a == 1), dk = (a == 2);
        const double* qLL = prim_at(i - 2 * di, j - 2 * dj, k - 2 * dk);
        const double* qL = prim_at(i - di, j - dj, k - dk);
        const double* qR = prim_at(i, j, k);
        const double* qRR = prim_at(i + di, j + dj, k + dk);
        double q1[8], q2[8];
        for (int v = 0; v < 8; v++) {
            q1[v] = qL[v];
            q2[v] = qR[v];
        }
        if (o->order == 2) {                     // cuf_solvers.cuf:366-412
            const double df = 0.5 * h[a], dff = 1.5 * h[a];
            double t1[5], t2[5];
            for (int v = 0; v < 5; v++) {
                t1[v] = linear(-dff, qLL[v], -df, qL[v], df, qR[v], 0.0);
                t2[v] = linear(-dff, qRR[v], -df, qR[v], df, qL[v], 0.0);
            }
            if (t1[0] < 0.0) t1[0] = qL[0];
            if (t1[4] < 0.0) t1[4] = qL[4];
            if (t2[0] < 0.0) t2[0] = qR[0];
            if (t2[4] < 0.0) t2[4] = qR[4];
            for (int v = 0; v < 5; v++) {
                q1[v] = t1[v];
                q2[v] = t2[v];
            }
        }
        if (q1[0] < 0.0 || q2[0] < 0.0) nrec++;  // cuf_solvers.cuf:414-420
        double n[3] = {0.0, 0.0, 0.0};
        n[a] = 1.0;
        double dsl, dsp, dsc, pot[8];
        const double wc = 0.0;
        int rc = chlld(o->n_state, n[0], n[1], n[2], wc, q1, q2, dsl, dsp, dsc, pot, o->n_disc);
        if (rc) {
            nwave++;
            for (int v = 0; v < 8; v++) pot[v] = 0.0;
        }
        for (int v = 0; v < 8; v++) F[v] = pot[v] * square[a];   // cuf_solvers.cuf:431
        const double dist = 0.5 * h[a];
        return std::min(dt_face_cap, o->cfl * dist / (std::max(std::fabs(dsl), std::fabs(dsp)) + std::fabs(wc)));
    };

    // z faces of the whole grid (nz+1 planes)
    std::vector<double> FZ((size_t)nx * ny * (nz + 1) * 8);
    double dmin = dt_reset;
    int64_t nrec = 0, nwave = 0, nneg = 0, nfloor = 0, firstbad = -1;
#pragma omp parallel for schedule(static) num_threads(nthreads) reduction(min : dmin) reduction(+ : nrec, nwave)
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                double c = face(2, i, j, k, &FZ[(((size_t)k * ny + j) * nx + i) * 8], nrec, nwave);
                dmin = std::min(dmin, c);
            }

#pragma omp parallel num_threads(nthreads) reduction(min : dmin) reduction(+ : nrec, nwave, nneg, nfloor)
    {
        std::vector<double> FX((size_t)(nx + 1) * ny * 8), FY((size_t)nx * (ny + 1) * 8);
        int64_t local_first = -1;
#pragma omp for schedule(static)
        for (int k = 0; k < nz; k++) {
            for (int j = 0; j < ny; j++)
                for (int i = 0; i <= nx; i++)
                    dmin = std::min(dmin, face(0, i, j, k, &FX[((size_t)j * (nx + 1) + i) * 8], nrec, nwave));
            for (int j = 0; j <= ny; j++)
                for (int i = 0; i < nx; i++)
                    dmin = std::min(dmin, face(1, i, j, k, &FY[((size_t)j * nx + i) * 8], nrec, nwave));
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const int64_t c = i + (int64_t)nx * (j + (int64_t)ny * k);
                    const double* fxl = &FX[((size_t)j * (nx + 1) + i) * 8];
                    const double* fxh = &FX[((size_t)j * (nx + 1) + i + 1) * 8];
                    const double* fyl = &FY[((size_t)j * nx + i) * 8];
                    const double* fyh = &FY[((size_t)(j + 1) * nx + i) * 8];
                    const double* fzl = &FZ[(((size_t)k * ny + j) * nx + i) * 8];
                    const double* fzh = &FZ[(((size_t)(k + 1) * ny + j) * nx + i) * 8];
                    double x[3], qs[8], un[8];
                    cell_center(g, i, j, k, x);
                    if (source_prim(g, x, qs)) {
                        cons_from_prim(qs, un);
                    } else {
                        for (int v = 0; v < 8; v++) {
                            double pot = 0.0;
                            pot = pot - fxl[v];
                            pot = pot + fxh[v];
                            pot = pot - fyl[v];
                            pot = pot + fyh[v];
                            pot = pot - fzl[v];
                            pot = pot + fzh[v];
                            if (kind == 0)
                                un[v] = Uin[v * N + c] - dt * (pot / volume);
                            else
                                un[v] = 0.5 * ((Ubase[v * N + c] + Uin[v * N + c]) - dt * (pot / volume));
                        }
                        if (un[0] <= 0.0) {       // cuf_solvers.cuf:708-711 (STOP in the reference)
                            nneg++;
                            if (local_first < 0) local_first = c;
                            for (int v = 0; v < 8; v++) un[v] = Uin[v * N + c];
                        } else {                 // cuf_solvers.cuf:777-779 pressure floor
                            double q[8];
                            prim_from_cons(un, q);
                            if (q[4] <= 0.0) {
                                nfloor++;
                                q[4] = p_floor;
                                double u2[8];
                                cons_from_prim(q, u2);
                                un[4] = u2[4];
                            }
                        }
                    }
                    for (int v = 0; v < 8; v++) Uout[v * N + c] = un[v];
                }
        }
        if (local_first >= 0) {
#pragma omp critical
            {
                if (firstbad < 0 || local_first < firstbad) firstbad = local_first;
            }
        }
    }
    if (want_dt) *dt_min = std::min(*dt_min, dmin);
    dg->n_recon_err += nrec;
    dg->n_wave_err += nwave;
    dg->n_negdens += nneg;
    dg->n_pfloor += nfloor;
    if (firstbad >= 0 && dg->first_bad_cell < 0) dg->first_bad_cell = firstbad;
}

void orc_clock_init(const orc_grid* g, orc_clock* ck) {
    ck->time_all = 0.0;
    ck->dt_next = g->dt_init;   // cuf_kernel.cuf:758
    ck->dt_last = 0.0;
}

// nsteps time steps, reference loop semantics (cuf_kernel.cuf:780-925). U: conserved SoA.
// Returns the number of steps run.
int orc_run(const orc_grid* g, const orc_opts* o, double* U, orc_clock* ck, int nsteps,
            int nthreads, orc_diag* dg) {
    const int64_t N = (int64_t)g->nx * g->ny * g->nz;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    std::vector<double> W((size_t)N * 8);
    for (int s = 0; s < nsteps; s++) {
        double dt = ck->dt_next;     // time_step = time_step2
        double dmin = dt_reset;      // time_step2 = 1e15
        ck->time_all = ck->time_all + dt;
        ck->dt_last = dt;
        if (o->scheme == 1) {
            stage(g, o, U, nullptr, W.data(), dt, 0, 1, &dmin, dg, nthreads);
            std::memcpy(U, W.data(), sizeof(double) * N * 8);
        } else {
            stage(g, o, U, nullptr, W.data(), dt, 0, 1, &dmin, dg, nthreads);
            stage(g, o, W.data(), U, U, dt, 1, 0, &dmin, dg, nthreads);
        }
        ck->dt_next = dmin;
    }
    return nsteps;
}

// One stage in isolation (for per-stage parity checks).
void orc_stage(const orc_grid* g, const orc_opts* o, const double* Uin, const double* Ubase,
               double* Uout, double dt, int kind, double* dt_min, int nthreads, orc_diag* dg) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    double dmin = dt_reset;
    stage(g, o, Uin, Ubase, Uout, dt, kind, 1, &dmin, dg, nthreads);
    *dt_min = dmin;
}

int orc_max_threads(void) { return omp_get_max_threads(); }

// ============================================================================ face-list grid
// The reference's own geometry (Storage_module.f90:20-37): explicit cells and faces with the
// Fortran layouts Cell_center(3,N), Cell_Volume(N), Cell_gran(6,N) (1-based face numbers, 0 =
// none), Gran_normal(3,G), Gran_square(G), Gran_center(3,G), Gran_neighbour(2,G) and
// Gran_neighbour_TVD(2,G) (1-based cell numbers, -1 = none), Gran_type(G).  The face flux
// array Gran_POTOK(9,G) persists between stages (a skipped face keeps its previous flux).
typedef struct {
    int64_t n_cell, n_gran;
    const double* cell_center;
    const double* cell_volume;
    const int32_t* cell_gran;
    const double* gran_normal;
    const double* gran_square;
    const double* gran_center;
    const int32_t* gran_neighbour;
    const int32_t* gran_neighbour_tvd;
    const int32_t* gran_type;
    double r_src, rho_src, v_src, p_over_rho_src, r_floor;   // source sphere (r_src 0 = none)
    double dt_init;
    double face_skip_radius;    // faces whose first cell has |centre| < this are skipped
    double cell_freeze_radius;  // cells with |centre| < this are not updated
    const double* hatom;        // physics 1: Cell_par columns 9..16 per cell ([N][8]), or null
    int32_t physics;            // 0: 3D MHD conservative update; 1: the reference's axisymmetric
                                // hydro update with charge exchange
    int32_t powell;             // physics 0: 0 off, 1 the reference's commented div-B terms
                                // (cuf_solvers.cuf:433, 529-533), 2 plus the energy term
} orc_facelist;

// SET_Fortran_Cuda_MHD/cuf_kernel.cuf:215-288, Source_MK: charge-exchange momentum (x, y) and
// energy sources of the plasma against two H-atom fluids (rho, u, v, T in Cell_par columns
// 9..12 and 13..16).  Default-real literals are single precision in the reference and enter as
// their promoted values; 3.0/0.4326569 is a single-precision quotient.
static void source_mk(const double* q, const double* h, double* out) {
    const double pi = std::acos(-1.0);
    const double rho = q[0], u = q[1], v = q[2], p = q[4];
    const double small = (double)0.0000001f;
    const double c_m = 64.0 / (9.0 * pi), c_u = 4.0 / pi;
    const double c_s = (double)0.1307345665f;
    const double c_n = (double)(3.0f / 0.4326569f);
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int k = 0; k < 2; k++) {
        double rH = h[4 * k], uH = h[4 * k + 1], vH = h[4 * k + 2];
        double pH = 0.5 * h[4 * k + 3] * rH;
        if (rH < small) {
            rH = small;
            pH = 0.0;
        }
        const double du = u - uH, dv = v - vH;
        const double th = p / rho + 2.0 * pH / rH;
        const double UM = std::sqrt((du * du + dv * dv) + c_m * th);
        const double UH = std::sqrt((du * du + dv * dv) + c_u * th);
        const double sg = (1.0 - c_s * std::log(UM)) * (1.0 - c_s * std::log(UM));
        const double nu = ((rho * rH) * UM) * sg;
        s1 = s1 + (c_n * nu) * (uH - u);
        s2 = s2 + (c_n * nu) * (vH - v);
        s3 = s3 + (c_n * nu) * ((((uH * uH + vH * vH) - u * u) - v * v) / 2.0 + (UH / UM) * (2.0 * pH / rH - p / rho));
    }
    out[0] = s1;
    out[1] = s2;
    out[2] = s3;
}

static double norm3(const double* x) { return std::sqrt((x[0] * x[0] + x[1] * x[1]) + x[2] * x[2]); }

// One face, cuf_solvers.cuf:243-440: boundary ghost by face type, TVD through the far
// neighbours with distance-weighted `linear`, chlld with the face normal, flux * area.
// Returns the dt candidate (dt_face_cap when the face is skipped: it leaves F untouched).
static double fl_face(const orc_facelist* m, const orc_opts* o, const double* P, int64_t gr, double* F,
                      int64_t& nrec, int64_t& nwave) {
    const int64_t s1 = m->gran_neighbour[2 * gr] - 1;
    const int32_t s2r = m->gran_neighbour[2 * gr + 1];
    const int type = m->gran_type[gr];
    const double* c1 = m->cell_center + 3 * s1;
    if (m->face_skip_radius > 0.0 && norm3(c1) < m->face_skip_radius) return dt_face_cap;   // :284
    const double* gc = m->gran_center + 3 * gr;
    const double* n = m->gran_normal + 3 * gr;
    double rast[3];
    for (int a = 0; a < 3; a++) rast[a] = gc[a] - c1[a];
    const double dist = norm3(rast);
    double q1[8], q2[8];
    for (int v = 0; v < 8; v++) q1[v] = P[8 * s1 + v];
    bool tvd = (o->order == 2);
    const double* c2 = c1;
    if (type == 4) {                              // :318-324 outer boundary
        for (int v = 0; v < 8; v++) q2[v] = q1[v];
        if (q2[1] > -0.1) q2[1] = -0.1;
        tvd = false;
    } else if (type == 5) {                       // :325-329 axis
        for (int v = 0; v < 8; v++) q2[v] = q1[v];
        q2[2] = -q2[2];
        tvd = false;
    } else if (type == 2 && s2r == -1) {          // :330-345 reflecting wall
        const double vel = (n[0] * q1[1] + n[1] * q1[2]) + n[2] * q1[3];
        for (int v = 0; v < 8; v++) q2[v] = q1[v];
        for (int a = 0; a < 3; a++) {
            const double vel1 = q1[1 + a] - vel * n[a];
            const double vel2 = vel * n[a];
            q2[1 + a] = vel1 - vel2;
        }
        tvd = false;
    } else {
        const int64_t s2 = s2r - 1;
        for (int v = 0; v < 8; v++) q2[v] = P[8 * s2 + v];
        c2 = m->cell_center + 3 * s2;
    }
    const int32_t ss1 = m->gran_neighbour_tvd[2 * gr], ss2 = m->gran_neighbour_tvd[2 * gr + 1];
    if (tvd && ss1 >= 1 && ss2 >= 1) {           // :358-412
        const double* cs1 = m->cell_center + 3 * (int64_t)(ss1 - 1);
        const double* cs2 = m->cell_center + 3 * (int64_t)(ss2 - 1);
        double r[3];
        for (int a = 0; a < 3; a++) r[a] = gc[a] - c1[a];
        const double df1 = norm3(r);
        for (int a = 0; a < 3; a++) r[a] = gc[a] - c2[a];
        const double df2 = norm3(r);
        for (int a = 0; a < 3; a++) r[a] = gc[a] - cs1[a];
        const double dff1 = norm3(r);
        for (int a = 0; a < 3; a++) r[a] = gc[a] - cs2[a];
        const double dff2 = norm3(r);
        const double* q11 = P + 8 * (int64_t)(ss1 - 1);
        const double* q22 = P + 8 * (int64_t)(ss2 - 1);
        double t1[5], t2[5];
        for (int v = 0; v < 5; v++) {
            t1[v] = linear(-dff1, q11[v], -df1, q1[v], df2, q2[v], 0.0);
            t2[v] = linear(-dff2, q22[v], -df2, q2[v], df1, q1[v], 0.0);
        }
        if (t1[0] < 0.0) t1[0] = q1[0];
        if (t1[4] < 0.0) t1[4] = q1[4];
        if (t2[0] < 0.0) t2[0] = q2[0];
        if (t2[4] < 0.0) t2[4] = q2[4];
        for (int v = 0; v < 5; v++) {
            q1[v] = t1[v];
            q2[v] = t2[v];
        }
    }
    if (q1[0] < 0.0 || q2[0] < 0.0) nrec++;      // :414-420
    double dsl, dsp, dsc, pot[8];
    const double wc = 0.0;
    int metod = o->n_state;
    if (m->physics == 1 && gc[0] > (double)0.22f && gc[1] < (double)0.1f && std::fabs(n[0]) < (double)0.1f)
        metod = 0;                                // :293-295, Lax flux on near-axis faces
    const int rc = chlld(metod, n[0], n[1], n[2], wc, q1, q2, dsl, dsp, dsc, pot, o->n_disc);
    if (rc) {
        nwave++;
        for (int v = 0; v < 8; v++) pot[v] = 0.0;
    }
    const double sq = m->gran_square[gr];
    for (int v = 0; v < 8; v++) F[v] = pot[v] * sq;   // :431
    // :433: 0 live; the commented expression 0.5 * DOT_PRODUCT(Gran_normal, qqq1(6:8) + qqq2(6:8))
    // * square when the div-B terms are on (qqq1 / qqq2: the states given to chlld)
    F[8] = 0.0;
    if (m->powell)
        F[8] = 0.5 * ((n[0] * (q1[5] + q2[5]) + n[1] * (q1[6] + q2[6])) + n[2] * (q1[7] + q2[7])) * sq;
    return std::min(dt_face_cap, o->cfl * dist / (std::max(std::fabs(dsl), std::fabs(dsp)) + std::fabs(wc)));
}

// One stage on a face list (kind 0: Euler / Heun stage 1; kind 1: Heun stage 2).  U: conserved
// SoA U[v*N + c]; F: the persistent Gran_POTOK(9,G).
static void fl_stage(const orc_facelist* m, const orc_opts* o, const double* Uin, const double* Ubase,
                     double* Uout, double* Fl, double dt, int kind, double* dt_min, orc_diag* dg, int nthreads) {
    const int64_t N = m->n_cell, G = m->n_gran;
    std::vector<double> P((size_t)N * 8);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < N; c++) {
        double u8[8];
        for (int v = 0; v < 8; v++) u8[v] = Uin[v * N + c];
        prim_from_cons(u8, &P[(size_t)c * 8]);
    }
    double dmin = dt_reset;
    int64_t nrec = 0, nwave = 0, nneg = 0, nfloor = 0, firstbad = -1;
#pragma omp parallel for schedule(static) num_threads(nthreads) reduction(min : dmin) reduction(+ : nrec, nwave)
    for (int64_t gr = 0; gr < G; gr++) dmin = std::min(dmin, fl_face(m, o, P.data(), gr, Fl + 9 * gr, nrec, nwave));
    orc_grid sg{};   // the source sphere, through the Cartesian helper
    sg.r_src = m->r_src;
    sg.rho_src = m->rho_src;
    sg.v_src = m->v_src;
    sg.p_over_rho_src = m->p_over_rho_src;
    sg.r_floor = m->r_floor;
#pragma omp parallel num_threads(nthreads) reduction(+ : nneg, nfloor)
    {
        int64_t local_first = -1;
#pragma omp for schedule(static)
        for (int64_t c = 0; c < N; c++) {
            const double* x = m->cell_center + 3 * c;
            double un[8], qs[8];
            if (m->cell_freeze_radius > 0.0 && norm3(x) < m->cell_freeze_radius) {   // :611
                for (int v = 0; v < 8; v++) un[v] = kind == 0 ? Uin[v * N + c] : Ubase[v * N + c];
            } else if (m->physics == 0 && source_prim(&sg, x, qs)) {
                cons_from_prim(qs, un);
            } else if (m->physics == 1) {
                // cuf_solvers.cuf:561-794: the axisymmetric hydro update of the primitive state,
                // restated with the reference's operation order; rr(2) = y
                double pot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int f = 0; f < 6; f++) {
                    const int32_t j = m->cell_gran[6 * c + f];
                    if (j == 0) continue;
                    const double* Fj = Fl + 9 * (int64_t)(j - 1);
                    const bool owner = m->gran_neighbour[2 * (int64_t)(j - 1)] == (int32_t)(c + 1);
                    for (int v = 0; v < 8; v++) pot[v] = owner ? pot[v] + Fj[v] : pot[v] - Fj[v];
                }
                double q[8], q2[8], u8[8], source[3];
                for (int v = 0; v < 8; v++) u8[v] = Uin[v * N + c];
                prim_from_cons(u8, q);                               // qqq: the stage input
                if (kind == 1) {
                    for (int v = 0; v < 8; v++) u8[v] = Ubase[v * N + c];
                    prim_from_cons(u8, q2);                          // qqq2: Cell_par
                }
                source_mk(q, m->hatom + 8 * c, source);
                const double vol = m->cell_volume[c], y = x[1], t = dt;
                const double nq = std::sqrt((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]);
                const double e1 = q[4] / (ggg - 1.0) + 0.5 * q[0] * (nq * nq);
                const double geo_e = (t * q[2]) * (ggg * q[4] / (ggg - 1) + q[0] * (q[1] * q[1] + q[2] * q[2]) * 0.5) / y;
                double ro3, u3, v3, p3;
                if (kind == 0) {
                    ro3 = q[0] - t * (pot[0] / vol + q[0] * q[2] / y);
                } else {
                    ro3 = 0.5 * (q2[0] + q[0] - t * (pot[0] / vol + q[0] * q[2] / y));
                }
                if (ro3 <= 0.0) {                                    // :708-711 (STOP there)
                    nneg++;
                    if (local_first < 0) local_first = c;
                    for (int v = 0; v < 8; v++) un[v] = Uin[v * N + c];
                } else {
                    if (kind == 0) {
                        u3 = ((((q[0] * q[1] - t * (pot[1]) / vol) + t * source[0]) - ((t * q[0]) * q[1]) * q[2] / y)) / ro3;
                        v3 = ((((q[0] * q[2] - t * (pot[2]) / vol) + t * source[1]) - ((t * q[0]) * q[2]) * q[2] / y)) / ro3;
                        p3 = ((((e1 - t * (pot[4]) / vol) + t * source[2]) - geo_e) - 0.5 * ro3 * ((u3 * u3 + v3 * v3) + 0.0)) * (ggg - 1.0);
                    } else {
                        const double nq2 = std::sqrt((q2[1] * q2[1] + q2[2] * q2[2]) + q2[3] * q2[3]);
                        const double e2 = q2[4] / (ggg - 1.0) + 0.5 * q2[0] * (nq2 * nq2);
                        u3 = 0.5 * ((((q2[0] * q2[1] + q[0] * q[1]) - t * (pot[1]) / vol) + t * source[0]) - ((t * q[0]) * q[1]) * q[2] / y) / ro3;
                        v3 = 0.5 * ((((q2[0] * q2[2] + q[0] * q[2]) - t * (pot[2]) / vol) + t * source[1]) - ((t * q[0]) * q[2]) * q[2] / y) / ro3;
                        p3 = (0.5 * ((((e2 + e1) - t * (pot[4]) / vol) + t * source[2]) - geo_e) - 0.5 * ro3 * ((u3 * u3 + v3 * v3) + 0.0)) * (ggg - 1.0);
                    }
                    if (p3 <= 0.0) {                                 // :777-779
                        nfloor++;
                        p3 = p_floor;
                    }
                    if (x[0] > (double)0.28f && x[1] < (double)0.07f && v3 < 0.0) v3 = (double)0.01f;   // :783-785
                    const double qn[8] = {ro3, u3, v3, 0.0, p3, 0.0, 0.0, 0.0};
                    cons_from_prim(qn, un);
                }
            } else {
                double pot[8] = {0, 0, 0, 0, 0, 0, 0, 0}, sks = 0.0;
                for (int f = 0; f < 6; f++) {                                         // :691-703
                    const int32_t j = m->cell_gran[6 * c + f];
                    if (j == 0) continue;
                    const double* Fj = Fl + 9 * (int64_t)(j - 1);
                    const bool owner = m->gran_neighbour[2 * (int64_t)(j - 1)] == (int32_t)(c + 1);
                    for (int v = 0; v < 8; v++) pot[v] = owner ? pot[v] + Fj[v] : pot[v] - Fj[v];
                    sks = owner ? sks + Fj[8] : sks - Fj[8];
                }
                if (m->powell) {
                    // :529-533 / :729-733 (commented there): w3 carries + (qqq(8)/cpi4) * sks and
                    // B carries + qqq(2..4) * sks inside the flux sum; the same for every momentum
                    // component; powell 2 adds the energy term (u.B/cpi4) * sks.  qqq: the stage
                    // input's primitive state.
                    const double* q = &P[(size_t)c * 8];
                    for (int a = 0; a < 3; a++) {
                        pot[1 + a] += (q[5 + a] / cpi4) * sks;
                        pot[5 + a] += q[1 + a] * sks;
                    }
                    if (m->powell == 2) pot[4] += (((q[1] * q[5] + q[2] * q[6]) + q[3] * q[7]) / cpi4) * sks;
                }
                const double vol = m->cell_volume[c];
                for (int v = 0; v < 8; v++) {
                    if (kind == 0)
                        un[v] = Uin[v * N + c] - dt * (pot[v] / vol);
                    else
                        un[v] = 0.5 * ((Ubase[v * N + c] + Uin[v * N + c]) - dt * (pot[v] / vol));
                }
                if (un[0] <= 0.0) {
                    nneg++;
                    if (local_first < 0) local_first = c;
                    for (int v = 0; v < 8; v++) un[v] = Uin[v * N + c];
                } else {
                    double q[8];
                    prim_from_cons(un, q);
                    if (q[4] <= 0.0) {
                        nfloor++;
                        q[4] = p_floor;
                        double u2[8];
                        cons_from_prim(q, u2);
                        un[4] = u2[4];
                    }
                }
            }
            for (int v = 0; v < 8; v++) Uout[v * N + c] = un[v];
        }
        if (local_first >= 0) {
#pragma omp critical
            {
                if (firstbad < 0 || local_first < firstbad) firstbad = local_first;
            }
        }
    }
    *dt_min = std::min(*dt_min, dmin);
    dg->n_recon_err += nrec;
    dg->n_wave_err += nwave;
    dg->n_negdens += nneg;
    dg->n_pfloor += nfloor;
    if (firstbad >= 0 && dg->first_bad_cell < 0) dg->first_bad_cell = firstbad;
}

// nsteps on a face list with the reference's loop semantics (lagged dt); F: Gran_POTOK(9,G),
// persistent across calls.
int orc_fl_run(const orc_facelist* m, const orc_opts* o, double* U, double* F, orc_clock* ck, int nsteps,
               int nthreads, orc_diag* dg) {
    const int64_t N = m->n_cell;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    std::vector<double> W((size_t)N * 8);
    for (int s = 0; s < nsteps; s++) {
        const double dt = ck->dt_next;
        double dmin = dt_reset;
        ck->time_all = ck->time_all + dt;
        ck->dt_last = dt;
        if (o->scheme == 1) {
            fl_stage(m, o, U, nullptr, W.data(), F, dt, 0, &dmin, dg, nthreads);
            std::memcpy(U, W.data(), sizeof(double) * N * 8);
        } else {
            fl_stage(m, o, U, nullptr, W.data(), F, dt, 0, &dmin, dg, nthreads);
            double dummy = dt_reset;
            fl_stage(m, o, W.data(), U, U, F, dt, 1, &dummy, dg, nthreads);
        }
        ck->dt_next = dmin;
    }
    return nsteps;
}

}  // extern "C"
