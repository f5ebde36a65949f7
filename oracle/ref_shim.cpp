// oracle/ref_shim.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A C entry point around the reference's own C++ solver Solvers::HLLD_Solver_Alexashov
// (SET_Gelios/source/Solvers.cpp:92-691), which is a translation of chlld
// (SET_Fortran_Cuda_MHD/Solvers.f90:1144-1859) with n_state hard-wired to 1 (HLL, :97).
// oracle/Makefile compiles this shim together with the reference source file, in place, into
// oracle/_ref/libgelios_hll.so.  Tests use it to pin the oracle's HLL branch.
//
// Variable orders: chlld takes (rho,u,v,w,p,Bx,By,Bz) and returns (rho,mx,my,mz,E,Bx,By,Bz);
// HLLD_Solver_Alexashov takes (rho,p,u,v,w,Bx,By,Bz) (:110-127) and returns
// (rho,mx,my,mz,Bx,By,Bz,E) after the swap at :372-376.  The shim maps both ways.
// Callers must pass states with SL < SM < SR: the reference function calls exit() otherwise
// (:228-252).
#include <vector>
#include "Solvers.h"

extern "C" double ref_gelios_hll(const double* q1, const double* q2, const double* n, double w,
                                 double dist, double* qqq, double* dsl, double* dsp, double* dsc) {
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
