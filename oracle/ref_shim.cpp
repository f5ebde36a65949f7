// oracle/ref_shim.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// C entry points around three of the reference's own C++ Riemann solvers in
// SET_Gelios/source/Solvers.cpp.  oracle/Makefile compiles this shim together with that source
// file, in place, into oracle/_ref/libgelios_hll.so.  Tests and tests/golden/make_golden.py use
// them to pin the oracle's restatement of chlld (SET_Fortran_Cuda_MHD/Solvers.f90:1144-1859):
//
//   ref_gelios_hll    Solvers::HLLD_Solver_Alexashov (:92-691): a translation of chlld with
//                     n_state hard-wired to 1 (HLL, :97).  Pins chlld's shared set-up and its
//                     HLL branch bit for bit.
//   ref_gelios_hllc   Solvers::HLLC_Aleksashov (:1324-1639): chlld's n_state = 2 branch with
//                     B = 0, n_disc = 0 and a fixed face (w = 0): the same rotation basis, Davis
//                     speeds, SM, ptz average and star states (Solvers.f90:1465-1596).  Pins the
//                     HLLC branch bit for bit.
//   ref_korolkov_hlld Solvers::HLLDQ_Korolkov (:1642-2185) with metod = 3, a second author's
//                     HLLD for axis-aligned normals and w = 0.  Its wave-speed estimate, fast-speed
//                     formula and degeneracy thresholds differ from chlld's, so it is a
//                     tolerance cross-check of the HLLD star and double-star states, not a pin.
//
// Variable orders: chlld takes (rho,u,v,w,p,Bx,By,Bz) and returns (rho,mx,my,mz,E,Bx,By,Bz);
// the shim maps each reference function's own order to that one.
#include <vector>
#include "Solvers.h"

extern "C" {

// HLLD_Solver_Alexashov takes (rho,p,u,v,w,Bx,By,Bz) (:110-127) and returns
// (rho,mx,my,mz,Bx,By,Bz,E) after the swap at :372-376.  Callers must pass states with
// SL < SM < SR: the reference function calls exit() otherwise (:228-252).
double ref_gelios_hll(const double* q1, const double* q2, const double* n, double w, double dist, double* qqq,
                      double* dsl, double* dsp, double* dsc) {
    std::vector<double> a = {q1[0], q1[4], q1[1], q1[2], q1[3], q1[5], q1[6], q1[7]};
    std::vector<double> b = {q2[0], q2[4], q2[1], q2[2], q2[3], q2[5], q2[6], q2[7]};
    std::vector<double> nn = {n[0], n[1], n[2]};
    std::vector<double> out(8, 0.0);
    Solvers s;
    double t = s.HLLD_Solver_Alexashov(a, b, nn, out, *dsl, *dsp, *dsc, w, dist);
    qqq[0] = out[0];
    qqq[1] = out[1];
    qqq[2] = out[2];
    qqq[3] = out[3];
    qqq[4] = out[7];
    qqq[5] = out[4];
    qqq[6] = out[5];
    qqq[7] = out[6];
    return t;
}

// HLLC_Aleksashov takes the hydro states as scalars (rho, p, u, v, w per side) and returns the
// five fluxes (rho, mx, my, mz, E) in P[0..4]; it has no field and no face speed.  The B entries
// of q1/q2 are ignored (the caller passes B = 0 to compare with chlld).
double ref_gelios_hllc(const double* q1, const double* q2, const double* n, double rad, double* qqq5) {
    Solvers s;
    return s.HLLC_Aleksashov(q1[0], q1[4], q1[1], q1[2], q1[3], q2[0], q2[4], q2[1], q2[2], q2[3], qqq5, n[0], n[1],
                             n[2], rad);
}

// HLLDQ_Korolkov takes (rho, Q, p, v1..3, B1..3) per side, B in stored units, an axis-aligned
// unit normal, and returns (rho, mx, my, mz, Bx, By, Bz, E) in P after its final swap plus the
// passive-scalar flux PQ.  metod 3 is HLLD, metod 2 its HLLC variant.
double ref_korolkov(int metod, const double* q1, double Q1, const double* q2, double Q2, const double* n, double rad,
                    double* qqq, double* pq) {
    Solvers s;
    double P[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double PQ = 0.0;
    double t = s.HLLDQ_Korolkov(q1[0], Q1, q1[4], q1[1], q1[2], q1[3], q1[5], q1[6], q1[7], q2[0], Q2, q2[4], q2[1],
                                q2[2], q2[3], q2[5], q2[6], q2[7], P, PQ, n[0], n[1], n[2], rad, metod);
    qqq[0] = P[0];
    qqq[1] = P[1];
    qqq[2] = P[2];
    qqq[3] = P[3];
    qqq[4] = P[7];
    qqq[5] = P[4];
    qqq[6] = P[5];
    qqq[7] = P[6];
    *pq = PQ;
    return t;
}

}  // extern "C"
