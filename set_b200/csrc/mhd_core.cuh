// mhd_core.cuh -- the per-face and per-cell arithmetic of the MHD step, written once for the
// device and the host, templated on the arithmetic type (double for the plain form, float for
// the Riemann arithmetic of the mixed form).
//
// The algorithm is chlld (SET_Fortran_Cuda_MHD/Solvers.f90:1144-1859) with these B200-side
// design choices, each exact in real arithmetic and differing from the reference only by
// rounding:
//   * Faces of the Cartesian grid are axis-aligned, so states arrive already in the face frame
//     (normal, t1, t2) = a permutation of (x, y, z).  The reference's tangent rotation basis
//     aco (Solvers.f90:1236-1280) is not built: every chlld formula treats the two tangential
//     components as a 2-vector (componentwise updates, dot products, sums of squares), so the
//     flux is the same in any orthonormal tangent basis.
//   * Divisions by a common denominator become one reciprocal and multiplies; /2 becomes *0.5
//     (exact); B/sqrt(4*pi) becomes B*(1/sqrt(4*pi)).
//   * Only the quantities the selected n_state branch reads are formed (e.g. HLLD needs UZ(6)
//     alone of the HLL average UZ).
//   * The overlapping "last match wins" IF blocks of the wave-fan selection (:1521-1567,
//     :1722-1814) are evaluated as the equivalent else-if chain in reverse order.
#pragma once
#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define SB_HD __host__ __device__ __forceinline__
#else
#define SB_HD inline
#endif

namespace sb {

// Storage_module.f90:8-9 and the derived constants, as correctly rounded doubles.
constexpr double kCpi4 = 12.566370614359172;        // 4*pi
constexpr double kSpi4 = 3.5449077018110318;        // sqrt(4*pi)
constexpr double kInvSpi4 = 0.28209479177387814;    // 1/sqrt(4*pi)
constexpr double kGamma = 1.6666666666666667;       // 5/3
constexpr double kG1 = 0.6666666666666667;          // 5/3 - 1
constexpr double kInvG1 = 1.4999999999999998;       // 1/(5/3 - 1)
constexpr double kPFloor = 1.0000000116860974e-07;  // FP32 literal 0.0000001 (cuf_solvers.cuf:778)
constexpr double kDtFaceCap = 100000.0;             // cuf_solvers.cuf:268
constexpr double kDtReset = 1.0e15;                 // cuf_kernel.cuf:790
constexpr double kEpsB = 1.0e-6;                    // Solvers.f90:1195
constexpr double kTtEps = 1.0e-9;                   // Solvers.f90:1625,1634

enum : int { kFlagWave = 1, kFlagStar = 2 };

// ------------------------------------------------------------------ elementary functions
// FP64: IEEE square root and correctly rounded reciprocal.  FP32 (the mixed form's Riemann
// arithmetic): the special-function unit's approximations (PTX sqrt / rcp / rsqrt .approx.ftz,
// a few ulp, subnormals flushed -- states here are far from the FP32 subnormal range).
SB_HD double sb_sqrt(double x) { return sqrt(x); }
SB_HD float sb_sqrt(float x) {
#if defined(__CUDA_ARCH__)
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return std::sqrt(x);
#endif
}
SB_HD double sb_rcp(double x) {
#if defined(__CUDA_ARCH__)
    return __drcp_rn(x);
#else
    return 1.0 / x;
#endif
}
SB_HD float sb_rcp(float x) {
#if defined(__CUDA_ARCH__)
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / x;
#endif
}
SB_HD double sb_rsqrt(double x) {
#if defined(__CUDA_ARCH__)
    return rsqrt(x);
#else
    return 1.0 / std::sqrt(x);
#endif
}
SB_HD float sb_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / std::sqrt(x);
#endif
}
// The Riemann solver's special functions.  FP32: the approximations above.  FP64 on the device:
// the FP64 approximate instructions (relative error ~1e-6, measured) refined by one third-order
// step each -- 1/x = y (1 + e + e^2) with e = 1 - x y, and 1/sqrt(x) = y (1 + e/2 + 3e^2/8) with
// e = 1 - x y^2 (the truncated binomial series: ~e^3 ~ 2^-60 before the final rounding; e is
// formed with one rounding of x y, ~2^-54 relative) -- and sqrt(x) = x * (1/sqrt(x)).  Domain:
// positive normal x whose result is normal (the approximate instructions flush subnormals);
// there 1/x and 1/sqrt(x) are within one ulp and sqrt(x) within two, mostly correctly rounded
// (tests/test_gpu_special.py checks 2^20 inputs over 1e-300..1e300).  At 0 and +-inf 1/x and
// 1/sqrt(x) give NaN; at subnormals 1/x gives NaN and 1/sqrt(x) +inf (sqrt(0) = 0).  Every
// argument the flux passes them is a positive density, a sum of squares under sb_pos, or a
// wave-speed difference that a valid state keeps away from zero (SR - SL >= cfL + cfR > 0; the
// star denominators tt are screened against 1e-9 before the reciprocal); a state that is already
// invalid (rho <= 0) is reported by the cell update's counters either way.  Three (1/x), five
// (1/sqrt(x)) and six (sqrt(x)) FP64 operations after the seed: fewer than the correctly rounded
// library forms, on the pipe that bounds the plain form.  The guarded primitive recovery's cheap
// path uses rs_rcp too; the exact recovery, the mixed form and the out-of-line FP64 recomputes
// keep the library forms.  On the host all
// three are the IEEE operations.
SB_HD double rs_rcp(double x) {
#if defined(__CUDA_ARCH__)
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
#else
    return 1.0 / x;
#endif
}
SB_HD double rs_rsqrt(double x) {
#if defined(__CUDA_ARCH__)
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    return fma(y, e * fma(0.375, e, 0.5), y);
#else
    return 1.0 / std::sqrt(x);
#endif
}
SB_HD double rs_sqrt(double x) {
#if defined(__CUDA_ARCH__)
    const double r = x * rs_rsqrt(x);
    return x == 0.0 ? x : r;   // the seed of 0 is infinite
#else
    return std::sqrt(x);
#endif
}
SB_HD float rs_rcp(float x) { return sb_rcp(x); }
SB_HD float rs_rsqrt(float x) { return sb_rsqrt(x); }
SB_HD float rs_sqrt(float x) { return sb_sqrt(x); }
// NR = false selects the library forms (riemann's FP64 recompute inside the mixed and delta
// kernels, whose schedules measured faster that way).
template <bool NR, typename T> SB_HD T fr_rcp(T x) {
    if constexpr (NR) return rs_rcp(x);
    else return sb_rcp(x);
}
template <bool NR, typename T> SB_HD T fr_rsqrt(T x) {
    if constexpr (NR) return rs_rsqrt(x);
    else return sb_rsqrt(x);
}
template <bool NR, typename T> SB_HD T fr_sqrt(T x) {
    if constexpr (NR) return rs_sqrt(x);
    else return sb_sqrt(x);
}

// |x| is a sign-bit operation on the device; sb_pos of a double tests the sign on the integer
// pipes (the FP64 pipe is the plain form's bottleneck): the same value for every non-NaN x.
template <typename T> SB_HD T sb_abs(T x) {
#if defined(__CUDA_ARCH__)
    return fabs(x);
#else
    return x < T(0) ? -x : x;
#endif
}
template <typename T> SB_HD T sb_min(T a, T b) { return b < a ? b : a; }
template <typename T> SB_HD T sb_max(T a, T b) { return a < b ? b : a; }
template <typename T> SB_HD T sb_pos(T x) {
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) return __double_as_longlong(x) > 0 ? x : T(0);
#endif
    return x > T(0) ? x : T(0);
}
// x < 0; a double on the device is tested by its sign bit (integer pipes), which differs from
// the comparison only at -0 and at NaNs with the sign bit set -- values no valid density or
// pressure takes.
template <typename T> SB_HD bool sb_neg(T x) {
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) return __double_as_longlong(x) < 0;
#endif
    return x < T(0);
}

// Solvers.f90:126-137: (signum(x)+signum(y))/2 * min(|x|,|y|).  On the device it is branch-free
// (the same value for every finite a, b, except that a zero result may carry a sign); in the FP64
// stage kernel the compare-and-branch form cost 16 % of the plain form's time (A/B on one box:
// 2.41 -> 2.81 G cell-updates/s at 256^3), through divergent branches in the 30 minmods per cell
// and stage.  FP32: |minmod| = max(0, min(|a|, b * sign(a))) with the sign of a.  FP64 works on
// the bit patterns, on the integer pipes: the FP64 pipe is the plain form's bottleneck, and
// minmod's value is one of its arguments (or zero), so no FP64 operation is needed -- with the
// signs of a and b different the result is 0, else the argument of smaller magnitude (magnitudes
// of doubles order like their bit patterns with the sign bit cleared).
template <typename T> SB_HD T minmod(T a, T b) {
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 4) {
        return copysignf(fmaxf(0.0f, fminf(fabsf(a), b * copysignf(1.0f, a))), a);
    } else {
        const long long A = __double_as_longlong(a), B = __double_as_longlong(b);
        const unsigned long long kMag = 0x7fffffffffffffffull;
        const long long m = ((unsigned long long)A & kMag) < ((unsigned long long)B & kMag) ? A : B;
        return (A ^ B) < 0 ? 0.0 : __longlong_as_double(m);
    }
#endif
    if (a > T(0) && b > T(0)) return sb_min(a, b);
    if (a < T(0) && b < T(0)) return sb_max(a, b);
    return T(0);
}

// ------------------------------------------------------------------ conserved -> primitive
// Explicitly rounded FP64 operations (no FMA contraction), for arithmetic that must match a
// host evaluation bit for bit.
SB_HD double rn_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
SB_HD double rn_add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
SB_HD double rn_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
// a / b rounded to nearest, given y = RN(1/b): q = RN(a y), the remainder r = a - b q is exact
// under FMA, and RN(q + r y) = RN(a / b) (Markstein's quotient theorem: y within half an ulp of
// 1/b and q within one ulp of a/b; IBM J. Res. Dev. 34(1), 1990).  Three operations per quotient
// after one shared reciprocal; tests/test_gpu_special.py compares it with IEEE division.
SB_HD double div_rn(double a, double b, double y) {
#if defined(__CUDA_ARCH__)
    const double q = __dmul_rn(a, y);
    // the sign of q is the quotient's (a zero numerator keeps its sign, which the correction
    // step's zero sum would drop)
    return copysign(__fma_rn(__fma_rn(-q, b, a), y, q), q);
#else
    (void)y;
    return a / b;
#endif
}

// U = (rho, mx, my, mz, E, Bx, By, Bz), B in stored units, E carrying |B/sqrt(4pi)|^2/2.
// Pressure recovery: p = ((E - rho|v|^2/2) - |b|^2/2)(gamma-1)  (cuf_solvers.cuf:735-738 with the
// magnetic term of the conservative MHD energy).
// EXACT (the plain form's default): the velocities and b are the correctly rounded quotients
// U[1..3] / rho and B / sqrt(4 pi), and ke, me, p are evaluated in the written order with every
// operation rounded, so the primitive state equals the host evaluation (the oracle's) bit for
// bit.  Pressure recovery cancels where the flow is hypersonic (the solar-wind source's outflow
// runs at Mach ~77, where rho|v|^2/2 is ~3000 times p): there one ulp in a velocity moves p by
// ~1e-12 relative, so a step computed from a differently rounded p differs from another correct
// FP64 step by more than 1e-12 per cell.  !EXACT: one one-ulp reciprocal (rs_rcp) and
// multiplies, with contraction (the mixed form, which rounds the result to FP32).
// SB: q[5..7] = b = B / sqrt(4 pi) (the field in the units the Riemann solver works in) instead of
// the stored B.
template <bool EXACT = true, bool SB = false>
SB_HD void prim_from_cons(const double* U, double* q, double& ke, double& me) {
    const double rho = U[0];
    const double ir = EXACT ? sb_rcp(rho) : rs_rcp(rho);   // Markstein's quotients need RN(1/rho)
    double u, v, w, bx, by, bz;
    if (EXACT) {
        u = div_rn(U[1], rho, ir);
        v = div_rn(U[2], rho, ir);
        w = div_rn(U[3], rho, ir);
        bx = div_rn(U[5], kSpi4, kInvSpi4);
        by = div_rn(U[6], kSpi4, kInvSpi4);
        bz = div_rn(U[7], kSpi4, kInvSpi4);
        ke = rn_mul(rn_mul(0.5, rho), rn_add(rn_add(rn_mul(u, u), rn_mul(v, v)), rn_mul(w, w)));
        me = rn_mul(0.5, rn_add(rn_add(rn_mul(bx, bx), rn_mul(by, by)), rn_mul(bz, bz)));
        q[4] = rn_mul(rn_sub(rn_sub(U[4], ke), me), kG1);
    } else {
        u = U[1] * ir;
        v = U[2] * ir;
        w = U[3] * ir;
        bx = U[5] * kInvSpi4;
        by = U[6] * kInvSpi4;
        bz = U[7] * kInvSpi4;
        ke = 0.5 * rho * ((u * u + v * v) + w * w);
        me = 0.5 * ((bx * bx + by * by) + bz * bz);
        q[4] = ((U[4] - ke) - me) * kG1;
    }
    q[0] = rho;
    q[1] = u;
    q[2] = v;
    q[3] = w;
    q[5] = SB ? bx : U[5];
    q[6] = SB ? by : U[6];
    q[7] = SB ? bz : U[7];
}
// The exact recovery where it matters, at about half its cost elsewhere: velocities and b from a
// one-ulp reciprocal (rs_rcp) and multiplies, ke, me, p with contraction.  Each velocity and b is
// then within 4 ulps of the exact quotient and p within about 12 (ke + me) / p + 2 E / p ulps of
// the exact recovery's; where the kinetic and magnetic energies exceed 64 p (the hypersonic
// outflow of the source, where one ulp of a velocity moves p by ~1e-12), or p is not positive or
// not finite, the exact recovery is run instead, so the state differs from the oracle's by at
// most ~1e-13 relative in p and 4 ulps elsewhere.  SB as prim_from_cons.
template <bool SB = false>
SB_HD void prim_from_cons_guarded(const double* U, double* q) {
    const double rho = U[0];
    const double ir = rs_rcp(rho);
    const double u = U[1] * ir, v = U[2] * ir, w = U[3] * ir;
    const double bx = U[5] * kInvSpi4, by = U[6] * kInvSpi4, bz = U[7] * kInvSpi4;
    const double ke = 0.5 * rho * ((u * u + v * v) + w * w);
    const double me = 0.5 * ((bx * bx + by * by) + bz * bz);
    const double p = ((U[4] - ke) - me) * kG1;
    if (!(ke + me <= 64.0 * p)) {
        double ke2, me2;
        prim_from_cons<true, SB>(U, q, ke2, me2);
        return;
    }
    q[0] = rho;
    q[1] = u;
    q[2] = v;
    q[3] = w;
    q[4] = p;
    q[5] = SB ? bx : U[5];
    q[6] = SB ? by : U[6];
    q[7] = SB ? bz : U[7];
}

// Total energy at the pressure floor, (p_floor/(gamma-1) + ke) + me: the oracle's cons_from_prim
// of the floored state (cuf_solvers.cuf:777-779), with ke, me from prim_from_cons<true>.
constexpr double kPFloorE = kPFloor / kG1;
SB_HD double floor_energy(double ke, double me) { return rn_add(rn_add(kPFloorE, ke), me); }

// A sufficient test that the exact recovery's pressure, ((E - ke) - me)(gamma - 1), is positive,
// at a third of its cost.  X' = (E - |m|^2/(2 rho)) - |B|^2/(8 pi) with a reciprocal of one ulp
// differs from the exact recovery's (E - ke) - me by at most ~17 units of 2^-53 times
// |E| + ke + me (ke, me carry at most 6-7 roundings each, X' at most 7; two subtractions
// each), so X' above 2^-48 (|E| + ke' + me') -- plus 1e-300 against subnormal magnitudes -- means
// the exact pressure is positive and the pressure floor does not apply.  Otherwise the caller
// runs the exact recovery.
SB_HD bool pressure_surely_positive(const double* U) {
    const double ir = rs_rcp(U[0]);
    const double m2 = (U[1] * U[1] + U[2] * U[2]) + U[3] * U[3];
    const double b2 = (U[5] * U[5] + U[6] * U[6]) + U[7] * U[7];
    const double ke = 0.5 * m2 * ir;
    const double me = b2 * (0.5 * kInvSpi4 * kInvSpi4);
    const double x = (U[4] - ke) - me;
    return x > 0x1p-48 * ((sb_abs(U[4]) + ke) + me) + 1e-300;
}

// ------------------------------------------------------------------ Riemann solver
// Face-frame states q = (rho, vn, vt1, vt2, p, Bn, Bt1, Bt2), B in stored units.
// Output F in the same order (B fluxes in stored units, not multiplied by the face area),
// SL, SR, SM (chlld's dsl, dsp, dsc).  wv is the face speed (used only when MOVING).
// Returns a bit set: kFlagWave when no wave-fan region matched (the reference STOPs),
// kFlagStar (CHECK_STAR only) when the selected state has rho <= 0 or p <= 0 or F is not finite.
// BS: the states carry b = B / sqrt(4 pi) already (q[5..7]), so the solver skips its scaling.
// LAZY (HLLC / HLLD): skip what the selected wave-fan region does not read (the FP64 stage
// kernels); !LAZY evaluates every region's quantities branch-free and selects, which needs fewer
// registers where the solver is a rare path of a kernel whose register budget it would set.
template <typename T, int NSTATE, bool MOVING, bool CHECK_STAR, bool NR = true, bool BS = false,
          bool LAZY = true>
SB_HD int riemann(const T* q1, const T* q2, T wv, int n_disc, T* F, T& SLo, T& SRo, T& SMo) {
    const T ispi4 = T(kInvSpi4);
    const T ga = T(kGamma);
    const T ig1 = T(kInvG1);
    const T g1 = T(kG1);
    const T half = T(0.5);
    if (!MOVING) wv = T(0);

    const T r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const T bx1 = BS ? q1[5] : q1[5] * ispi4, by1 = BS ? q1[6] : q1[6] * ispi4, bz1 = BS ? q1[7] : q1[7] * ispi4;
    const T r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const T bx2 = BS ? q2[5] : q2[5] * ispi4, by2 = BS ? q2[6] : q2[6] * ispi4, bz2 = BS ? q2[7] : q2[7] * ispi4;

    // fast magnetosonic speeds, Solvers.f90:1282-1306.  The reference forms
    // cf = (sqrt(b2/r + c(c + 2a)) + sqrt(b2/r + c(c - 2a)))/2 with c = sqrt(ga p/r),
    // a = bn/sqrt(r); squaring gives the same speed as
    // cf^2 = (c^2 + b2/r + sqrt((c^2 + b2/r)^2 - 4 c^2 bn^2/r))/2, which needs two square roots
    // per side instead of three plus a reciprocal square root.
    const T ir1 = fr_rcp<NR>(r1), ir2 = fr_rcp<NR>(r2);
    const T b2L = (bx1 * bx1 + by1 * by1) + bz1 * bz1;
    const T b21 = b2L * ir1;
    const T c2L = ga * p1 * ir1;
    const T sL = c2L + b21;
    const T cfL = fr_sqrt<NR>(half * (sL + fr_sqrt<NR>(sb_pos(sL * sL - T(4) * c2L * (bx1 * bx1 * ir1)))));
    const T ptL = p1 + half * b2L;
    const T b2R = (bx2 * bx2 + by2 * by2) + bz2 * bz2;
    const T b22 = b2R * ir2;
    const T c2R = ga * p2 * ir2;
    const T sR = c2R + b22;
    const T cfR = fr_sqrt<NR>(half * (sR + fr_sqrt<NR>(sb_pos(sR * sR - T(4) * c2R * (bx2 * bx2 * ir2)))));
    const T ptR = p2 + half * b2R;

    // wave-speed estimates, :1308-1330
    T SL = sb_min(u1 - cfL, u2 - cfR);
    T SR = sb_max(u1 + cfL, u2 + cfR);
    T cfC = T(0), vC1 = T(0);
    if (n_disc != 0 || NSTATE == 0) {
        const T aC = half * (bx1 * fr_rsqrt<NR>(r1) + bx2 * fr_rsqrt<NR>(r2));
        const T b2o = half * (b22 + b21);
        const T cC = fr_sqrt<NR>(ga * (half * (p2 + p1)) * fr_rcp<NR>(half * (r2 + r1)));
        cfC = half * (fr_sqrt<NR>(sb_pos(b2o + cC * (cC + T(2) * aC))) +
                      fr_sqrt<NR>(sb_pos(b2o + cC * (cC - T(2) * aC))));
        vC1 = half * (u1 + u2);
        if (n_disc == 1) {
            SL = sb_min(u1 - cfL, vC1 - cfC);
            SR = sb_max(u2 + cfR, vC1 + cfC);
        } else if (n_disc == 2) {
            const T SL1 = sb_min(u1 - cfL, vC1 - cfC), SR1 = sb_max(u2 + cfR, vC1 + cfC);
            const T SL2 = sb_min(u1 - cfL, u2 - cfR), SR2 = sb_max(u1 + cfL, u2 + cfR);
            SL = T(0.75) * SL1 + T(0.25) * SL2;
            SR = T(0.75) * SR1 + T(0.25) * SR2;
        }
    }
    const T suR = SR - u2, suL = SL - u1;
    const T idd = fr_rcp<NR>(suR * r2 - suL * r1);
    const T SM = (((suR * r2 * u2 - ptR) + ptL) - suL * r1 * u1) * idd;
    SLo = SL;
    SRo = SR;
    SMo = SM;
    if (NSTATE == 0) {   // one-speed Lax, :1360-1365
        const T TR0 = sb_abs(u1 + u2) * half + cfC;
        SL = -TR0;
        SR = TR0;
    }

    int flag = 0;
    if (NSTATE <= 1) {   // :1414-1463, with the left/right energies, fluxes and states of :1368-1404
        const T isrl = fr_rcp<NR>(SR - SL);
        const T e1 = (p1 * ig1 + r1 * (half * ((u1 * u1 + v1 * v1) + w1 * w1))) + half * b2L;
        const T e2 = (p2 * ig1 + r2 * (half * ((u2 * u2 + v2 * v2) + w2 * w2))) + half * b2R;
        const T sbv1 = (u1 * bx1 + v1 * by1) + w1 * bz1;
        const T sbv2 = (u2 * bx2 + v2 * by2) + w2 * bz2;
        const T m1 = r1 * u1, m2 = r2 * u2;
        T FL[8], FR[8], UL[8], UR[8];
        FL[0] = m1;
        FL[1] = (m1 * u1 + ptL) - bx1 * bx1;
        FL[2] = m1 * v1 - bx1 * by1;
        FL[3] = m1 * w1 - bx1 * bz1;
        FL[4] = (e1 + ptL) * u1 - bx1 * sbv1;
        FL[5] = T(0);
        FL[6] = u1 * by1 - v1 * bx1;
        FL[7] = u1 * bz1 - w1 * bx1;
        FR[0] = m2;
        FR[1] = (m2 * u2 + ptR) - bx2 * bx2;
        FR[2] = m2 * v2 - bx2 * by2;
        FR[3] = m2 * w2 - bx2 * bz2;
        FR[4] = (e2 + ptR) * u2 - bx2 * sbv2;
        FR[5] = T(0);
        FR[6] = u2 * by2 - v2 * bx2;
        FR[7] = u2 * bz2 - w2 * bx2;
        UL[0] = r1; UL[1] = m1; UL[2] = r1 * v1; UL[3] = r1 * w1; UL[4] = e1;
        UL[5] = bx1; UL[6] = by1; UL[7] = bz1;
        UR[0] = r2; UR[1] = m2; UR[2] = r2 * v2; UR[3] = r2 * w2; UR[4] = e2;
        UR[5] = bx2; UR[6] = by2; UR[7] = bz2;
        T TL = SL, TR = SR;
        if (SL > wv) TL = T(0);
        if (SR < wv) TR = T(0);
        const T a = TR * TL;
        const T ib = fr_rcp<NR>(TR - TL);
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = ((TR * FL[k] - TL * FR[k]) + a * (UR[k] - UL[k])) * ib;
        if (MOVING) {
            // FW: last matching block wins (:1422-1438)
#pragma unroll
            for (int k = 0; k < 8; k++) {
                T fw;
                if (SR < wv) fw = wv * UR[k];
                else if (SL <= wv && wv <= SR) fw = wv * ((SR * UR[k] - SL * UL[k] + FL[k] - FR[k]) * isrl);
                else fw = wv * UL[k];
                F[k] = F[k] - fw;
            }
        }
        if (!(SL > wv) && !(SL <= wv && wv <= SR) && !(SR < wv)) flag |= kFlagWave;
    } else {
        // The wave-fan region is found first and (LAZY) everything else is formed only where the
        // selected region reads it.  The region chains of :1521-1567 and :1722-1814 (last match
        // wins) end with FR (SR < wv), so SR < wv selects FR whatever the other speeds are: no HLL
        // average, star density or Alfven speed is needed there.  FL (SL > wv) holds only when no later region
        // matches, so it is decided with the others.  The star states (:1465-1567 / :1598-1718)
        // and the star energy are formed for the star regions alone, a side's single-star state
        // for the regions that read it; the energy, physical flux and conserved vector
        // (:1368-1404) for the selected side alone.
        int region = 6;   // 1: FL, 2: L*, 3: L**, 4: R**, 5: R*, 6: FR, 0: none
        T isrl = T(0), bn = T(0), isrm = T(0), islm = T(0), suRm = T(0), suLm = T(0), rzR = T(0), rzL = T(0);
        T rzRs = T(0), rzLs = T(0), sbn = T(0), SZL = SM, SZR = SM;
        T isR = T(0), isL = T(0);
        bool ibn = false;
        if (!LAZY || !(SR < wv)) {
            isrl = fr_rcp<NR>(SR - SL);
            bn = (SR * bx2 - SL * bx1) * isrl;   // HLL average of the normal field, UZ(6) (:1406-1408)
            isrm = fr_rcp<NR>(SR - SM);
            islm = fr_rcp<NR>(SL - SM);
            suRm = suR * isrm;
            suLm = suL * islm;
            rzR = r2 * suRm;
            rzL = r1 * suLm;
            if (NSTATE == 2) {   // HLLC, :1521-1567
                if (SR < wv) region = 6;
                else if (SM <= wv && SR >= wv) region = 5;
                else if (SL <= wv && SM >= wv) region = 2;
                else if (SL > wv) region = 1;
                else region = 0;
            } else {             // HLLD, :1660-1676, :1722-1814
                isR = fr_rsqrt<NR>(rzR);   // 1/sqrt(rho*) and sqrt(rho*) = rho*/sqrt(rho*)
                isL = fr_rsqrt<NR>(rzL);
                rzRs = rzR * isR;
                rzLs = rzL * isL;
                const T abn = sb_abs(bn);
                if (abn > T(kEpsB)) {
                    ibn = true;
                    sbn = bn > T(0) ? T(1) : T(-1);
                    SZL = SM - abn * isL;
                    SZR = SM + abn * isR;
                }
                if (SR < wv) region = 6;
                else if (SZR <= wv && SR >= wv) region = 5;
                else if (ibn && SM <= wv && SZR >= wv) region = 4;
                else if (ibn && SZL <= wv && SM >= wv) region = 3;
                else if (SL <= wv && SZL >= wv) region = 2;
                else if (SL > wv) region = 1;
                else region = 0;
            }
        }
        if (region == 0) flag |= kFlagWave;
        const bool right = region >= 4;
        const bool use1 = (region >= 2 && region <= 5);
        const bool use2 = (region == 3 || region == 4);
        // the selected side
        const T r = right ? r2 : r1, u = right ? u2 : u1, v = right ? v2 : v1, w = right ? w2 : w1;
        const T p = right ? p2 : p1, bx = right ? bx2 : bx1, by = right ? by2 : by1, bz = right ? bz2 : bz1;
        const T pt = right ? ptR : ptL, b2 = right ? b2R : b2L;
        const T e = (p * ig1 + r * (half * ((u * u + v * v) + w * w))) + half * b2;
        const T sbv = (u * bx + v * by) + w * bz;
        const T m = r * u;
        T Fs[8], Us[8];
        Fs[0] = m;
        Fs[1] = (m * u + pt) - bx * bx;
        Fs[2] = m * v - bx * by;
        Fs[3] = m * w - bx * bz;
        Fs[4] = (e + pt) * u - bx * sbv;
        Fs[5] = T(0);
        Fs[6] = u * by - v * bx;
        Fs[7] = u * bz - w * bx;
        Us[0] = r; Us[1] = m; Us[2] = r * v; Us[3] = r * w; Us[4] = e;
        Us[5] = bx; Us[6] = by; Us[7] = bz;
        T W[8];   // the state whose flux is returned (for the face-speed term and the check)
#pragma unroll
        for (int k = 0; k < 8; k++) {
            F[k] = Fs[k];
            W[k] = Us[k];
        }
        if (!LAZY || use1) {
            T vzL2 = T(0), vzL3 = T(0), vzR2 = T(0), vzR3 = T(0);
            T bzL2 = T(0), bzL3 = T(0), bzR2 = T(0), bzR3 = T(0);
            T vzz2 = T(0), vzz3 = T(0), bzz2 = T(0), bzz3 = T(0);
            T ptz;        // total pressure of the star states
            T sbvz = T(0);
            if (NSTATE == 2) {   // HLLC, :1465-1558
                ptz = half * ((ptR + r2 * suR * (SM - u2)) + (ptL + r1 * suL * (SM - u1)));
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
                sbvz = ((bn * uz1 + uz6 * uz2) + uz7 * uz3) * fr_rcp<NR>(uz0);
                if (sb_abs(bn) < T(kEpsB)) {
                    vzR2 = v2; vzR3 = w2; vzL2 = v1; vzL3 = w1;
                    bzR2 = by2 * suRm; bzR3 = bz2 * suRm;
                    bzL2 = by1 * suLm; bzL3 = bz1 * suLm;
                } else {
                    const T cR = bn * fr_rcp<NR>(suR * r2), cL = bn * fr_rcp<NR>(suL * r1);
                    vzR2 = v2 + (by2 - uz6) * cR;
                    vzR3 = w2 + (bz2 - uz7) * cR;
                    vzL2 = v1 + (by1 - uz6) * cL;
                    vzL3 = w1 + (bz1 - uz7) * cL;
                    bzR2 = uz6; bzR3 = uz7; bzL2 = uz6; bzL3 = uz7;
                }
            } else {             // HLLD, :1598-1718
                ptz = ((suR * r2 * ptL - suL * r1 * ptR) + r1 * r2 * suR * suL * (u2 - u1)) * idd;
                const T bn2 = bn * bn;
                if (!LAZY || region <= 4) {   // L*, L**, R**: the left single-star state
                    T tvL = T(0), tbL = T(0);
                    const T ttL = r1 * suL * (SL - SM) - bn2;
                    if (!(sb_abs(ttL) <= T(kTtEps))) {
                        const T i = fr_rcp<NR>(ttL);
                        tvL = (SM - u1) * i;
                        tbL = (r1 * suL * suL - bn2) * i;
                    }
                    vzL2 = v1 - bn * by1 * tvL;
                    vzL3 = w1 - bn * bz1 * tvL;
                    bzL2 = by1 * tbL;
                    bzL3 = bz1 * tbL;
                }
                if (!LAZY || region >= 3) {   // L**, R**, R*: the right single-star state
                    T tvR = T(0), tbR = T(0);
                    const T ttR = r2 * suR * (SR - SM) - bn2;
                    if (!(sb_abs(ttR) <= T(kTtEps))) {
                        const T i = fr_rcp<NR>(ttR);
                        tvR = (SM - u2) * i;
                        tbR = (r2 * suR * suR - bn2) * i;
                    }
                    vzR2 = v2 - bn * by2 * tvR;
                    vzR3 = w2 - bn * bz2 * tvR;
                    bzR2 = by2 * tbR;
                    bzR3 = bz2 * tbR;
                }
                if (use2) {
                    const T irzss = fr_rcp<NR>(rzRs + rzLs);
                    const T rzps = rzRs * rzLs;
                    vzz2 = ((rzLs * vzL2 + rzRs * vzR2) + sbn * (bzR2 - bzL2)) * irzss;
                    vzz3 = ((rzLs * vzL3 + rzRs * vzR3) + sbn * (bzR3 - bzL3)) * irzss;
                    bzz2 = ((rzLs * bzR2 + rzRs * bzL2) + sbn * rzps * (vzR2 - vzL2)) * irzss;
                    bzz3 = ((rzLs * bzR3 + rzRs * bzL3) + sbn * rzps * (vzR3 - vzL3)) * irzss;
                }
            }
            const T sum = right ? suRm : suLm, ism = right ? isrm : islm;
            const T rz = right ? rzR : rzL;
            const T S1 = right ? SR : SL;
            const T S2 = right ? SZR : SZL;
            const T vz2 = right ? vzR2 : vzL2, vz3 = right ? vzR3 : vzL3;
            const T bz2_ = right ? bzR2 : bzL2, bz3_ = right ? bzR3 : bzL3;
            // star energy of the selected side (:1541-1544 / :1650-1656) and its double star
            // (:1710-1718)
            const T sbvS = NSTATE == 2 ? sbvz : (bn * SM + bz2_ * vz2) + bz3_ * vz3;
            const T ez = e * sum + (((ptz * SM - pt * u) + bn * (sbv - sbvS)) * ism);
            T ezz = ez;
            if (NSTATE == 3 && use2) {
                const T sbzz = (bn * SM + bzz2 * vzz2) + bzz3 * vzz3;
                ezz = right ? ez + rzRs * sbn * (sbvS - sbzz) : ez - rzLs * sbn * (sbvS - sbzz);
            }
            T UZs[8], UZZs[8];
            UZs[0] = rz; UZs[1] = rz * SM; UZs[2] = rz * vz2; UZs[3] = rz * vz3; UZs[4] = ez;
            UZs[5] = bn; UZs[6] = bz2_; UZs[7] = bz3_;
            UZZs[0] = rz; UZZs[1] = rz * SM; UZZs[2] = rz * vzz2; UZZs[3] = rz * vzz3; UZZs[4] = ezz;
            UZZs[5] = bn; UZZs[6] = bzz2; UZZs[7] = bzz3;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                T f = Fs[k];
                if (use2) f = f + S2 * (UZZs[k] - UZs[k]);
                if (LAZY || use1) f = f + S1 * (UZs[k] - Us[k]);
                W[k] = use2 ? UZZs[k] : (LAZY || use1 ? UZs[k] : Us[k]);
                F[k] = f;
            }
            if (CHECK_STAR && (LAZY || use1)) {
                // positivity of the selected star state: rho* > 0 and p* = pt* - |b*|^2/2 > 0 (the
                // gas pressure from the star total pressure avoids the kinetic-energy cancellation
                // of E - rho|v|^2/2); FL / FR themselves are the reconstructed, positive states
                const T bb = (bn * bn + W[6] * W[6]) + W[7] * W[7];
                if (!(rz > T(0)) || !(ptz - half * bb > T(0))) flag |= kFlagStar;
            }
        }
        if (MOVING) {
#pragma unroll
            for (int k = 0; k < 8; k++) F[k] = F[k] - wv * W[k];
        }
        // normal-field flux, :1570-1581 / :1828-1839
        const T SN = sb_max(sb_abs(SL), sb_abs(SR));
        T wbn = T(0);
        if (MOVING) {
            if (wv >= SR) wbn = wv * bx2;
            else if (wv <= SL) wbn = wv * bx1;
            else wbn = wv * (bx1 + bx2) * half;
        }
        F[5] = -SN * (bx2 - bx1) - wbn;
    }
    // B fluxes back to stored units (:1846)
    const T spi4 = T(kSpi4);
    F[5] *= spi4;
    F[6] *= spi4;
    F[7] *= spi4;
    if (CHECK_STAR) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (!(sb_abs(F[k]) < T(3.0e38))) flag |= kFlagStar;
    }
    return flag;
}

// ------------------------------------------------------------------ delta-form solver
// The same HLLD (NSTATE 3) / HLLC-without-field (NSTATE 2) flux, arranged so that FP32 only
// computes small quantities.  In FP32 arithmetic on full-magnitude states every flux carries
// ~6e-8 |F| of rounding whatever its storage; here FP32 evaluates the wave speeds, the jumps
// across the face and the differences between each star state and its side state, all in closed
// form:
//   SM - u1 = (suR r2 du - dpt) / (suR r2 - suL r1),      SM - u2 = (suL r1 du - dpt) / (...)
//   rho*L - r1 = r1 (SM - u1) / (SL - SM),                tb - 1 = r suL (SM - u1) / tt
//   pt* - ptL = (r1 r2 suR suL du - suL r1 dpt) / (...), bn - bx1 = SR dbx / (SR - SL)
//   e*L - e1 = ((e1 + pt*)(SM - u1) + (pt* - ptL) u1 + bn (v.b - v*.b*)) / (SL - SM)
// and likewise for the double-star states (Solvers.f90:1600-1718).  The flux is
// F = F_side + S2 (U** - U*) + S1 (U* - U_side); delta_core returns the bracketed part (the
// dissipation of the selected side, FP32) and the caller adds the physical flux of that side.
struct DeltaIn {   // FP32 side values (b = B / sqrt(4 pi)), their jumps, energies, total pressure
    float r1, u1, v1, w1, p1, bx1, by1, bz1, b2L, e1, ptL;
    float r2, u2, v2, w2, p2, bx2, by2, bz2, b2R, e2;
    float du, dv, dw, dbx, dby, dbz, dpt;
};

// The fast magnetosonic speeds of the two sides (as riemann()), from d's r, p, bx and |b|^2.
SB_HD void delta_fast_speeds(const DeltaIn& d, float& cfL, float& cfR) {
    typedef float f;
    const f ga = (f)kGamma, half = 0.5f;
    const f ir1 = sb_rcp(d.r1), ir2 = sb_rcp(d.r2);
    const f c2L = ga * d.p1 * ir1, c2R = ga * d.p2 * ir2;
    const f sL = c2L + d.b2L * ir1, sR = c2R + d.b2R * ir2;
    cfL = sb_sqrt(half * (sL + sb_sqrt(sb_pos(sL * sL - 4.0f * c2L * (d.bx1 * d.bx1 * ir1)))));
    cfR = sb_sqrt(half * (sR + sb_sqrt(sb_pos(sR * sR - 4.0f * c2R * (d.bx2 * d.bx2 * ir2)))));
}

// Returns kFlagWave / kFlagStar like riemann() and sets `right` (the selected side) and c[8]:
// the flux minus the physical flux of the selected side, c[5] the whole normal-field flux.
// cfL, cfR: delta_fast_speeds of d.
template <int NSTATE>
SB_HD int delta_core(const DeltaIn& d, float cfL, float cfR, float* c, bool& right, float& SLo, float& SRo,
                     float& SMo) {
    typedef float f;
    const f fr1 = d.r1, fu1 = d.u1, fv1 = d.v1, fw1 = d.w1, fr2 = d.r2, fu2 = d.u2, fv2 = d.v2, fw2 = d.w2;
    const f fbx1 = d.bx1, fby1 = d.by1, fbz1 = d.bz1, fbx2 = d.bx2, fby2 = d.by2, fbz2 = d.bz2;
    const f du = d.du, dv = d.dv, dw = d.dw, dbx = d.dbx, dby = d.dby, dbz = d.dbz, dpt = d.dpt;
    const f half = 0.5f;

    // speeds relative to each side: SL - u1 = min(-cfL, du - cfR), SR - u2 = max(cfL - du, cfR)
    const f suL = sb_min(-cfL, du - cfR);
    const f suR = sb_max(cfL - du, cfR);
    const f SL = fu1 + suL, SR = fu2 + suR;
    const f iden = sb_rcp(suR * fr2 - suL * fr1);
    const f dL = (suR * fr2 * du - dpt) * iden;   // SM - u1
    const f dR = (suL * fr1 * du - dpt) * iden;   // SM - u2
    const f SM = fu1 + dL;
    SLo = SL;
    SRo = SR;
    SMo = SM;
    const f slm = suL - dL, srm = suR - dR;       // SL - SM, SR - SM
    const f islm = sb_rcp(slm), isrm = sb_rcp(srm);
    const f D0L = fr1 * dL * islm, D0R = fr2 * dR * isrm;   // rho* - rho
    const f rzL = fr1 + D0L, rzR = fr2 + D0R;

    f DL[8], DR[8], DDL[8], DDR[8];   // U* - U_side, U** - U*
    f SZL = SM, SZR = SM, ptz, bn = 0.0f, bz2L = 0.f, bz3L = 0.f, bz2R = 0.f, bz3R = 0.f;
    f bzz2 = 0.f, bzz3 = 0.f;
    bool ibn = false;
    int region;
    if (NSTATE == 2) {   // HLLC without field: v* = v, B* = 0
        const f ptz_m_ptL = half * ((dpt + fr2 * suR * dR) + fr1 * suL * dL);
        const f ptz_m_ptR = ptz_m_ptL - dpt;
        ptz = d.ptL + ptz_m_ptL;
        DL[0] = D0L; DL[1] = D0L * SM + fr1 * dL; DL[2] = D0L * fv1; DL[3] = D0L * fw1;
        DL[4] = ((d.e1 + ptz) * dL + ptz_m_ptL * fu1) * islm;
        DR[0] = D0R; DR[1] = D0R * SM + fr2 * dR; DR[2] = D0R * fv2; DR[3] = D0R * fw2;
        DR[4] = ((d.e2 + ptz) * dR + ptz_m_ptR * fu2) * isrm;
#pragma unroll
        for (int k = 5; k < 8; k++) DL[k] = DR[k] = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; k++) DDL[k] = DDR[k] = 0.0f;
        if (SR < 0.0f) region = 6;
        else if (SM <= 0.0f && SR >= 0.0f) region = 5;
        else if (SL <= 0.0f && SM >= 0.0f) region = 2;
        else if (SL > 0.0f) region = 1;
        else region = 0;
    } else {             // HLLD
        const f isrl = sb_rcp(SR - SL);
        const f bnL = SR * dbx * isrl, bnR = SL * dbx * isrl;   // bn - bx1, bn - bx2
        bn = fbx1 + bnL;
        const f bn2 = bn * bn;
        const f ptz_m_ptL = (fr1 * fr2 * suR * suL * du - suL * fr1 * dpt) * iden;
        const f ptz_m_ptR = ptz_m_ptL - dpt;
        ptz = d.ptL + ptz_m_ptL;
        // left star
        const f ttL = fr1 * suL * slm - bn2;
        f tvL = 0.0f, tbL = -1.0f;   // tv and tb - 1 (degenerate: tv = tb = 0)
        if (!(sb_abs(ttL) <= (f)kTtEps)) {
            const f i = sb_rcp(ttL);
            tvL = dL * i;
            tbL = fr1 * suL * dL * i;
        }
        const f dvL2 = -bn * fby1 * tvL, dvL3 = -bn * fbz1 * tvL;   // v* - v
        const f dbL2 = fby1 * tbL, dbL3 = fbz1 * tbL;                // b* - b
        const f vzL2 = fv1 + dvL2, vzL3 = fw1 + dvL3;
        bz2L = fby1 + dbL2;
        bz3L = fbz1 + dbL3;
        const f dsL = -(dL * fbx1 + SM * bnL) - (fv1 * dbL2 + dvL2 * bz2L) - (fw1 * dbL3 + dvL3 * bz3L);
        DL[0] = D0L; DL[1] = D0L * SM + fr1 * dL; DL[2] = D0L * vzL2 + fr1 * dvL2; DL[3] = D0L * vzL3 + fr1 * dvL3;
        DL[4] = ((d.e1 + ptz) * dL + ptz_m_ptL * fu1 + bn * dsL) * islm;
        DL[5] = bnL; DL[6] = dbL2; DL[7] = dbL3;
        // right star
        const f ttR = fr2 * suR * srm - bn2;
        f tvR = 0.0f, tbR = -1.0f;
        if (!(sb_abs(ttR) <= (f)kTtEps)) {
            const f i = sb_rcp(ttR);
            tvR = dR * i;
            tbR = fr2 * suR * dR * i;
        }
        const f dvR2 = -bn * fby2 * tvR, dvR3 = -bn * fbz2 * tvR;
        const f dbR2 = fby2 * tbR, dbR3 = fbz2 * tbR;
        const f vzR2 = fv2 + dvR2, vzR3 = fw2 + dvR3;
        bz2R = fby2 + dbR2;
        bz3R = fbz2 + dbR3;
        const f dsR = -(dR * fbx2 + SM * bnR) - (fv2 * dbR2 + dvR2 * bz2R) - (fw2 * dbR3 + dvR3 * bz3R);
        DR[0] = D0R; DR[1] = D0R * SM + fr2 * dR; DR[2] = D0R * vzR2 + fr2 * dvR2; DR[3] = D0R * vzR3 + fr2 * dvR3;
        DR[4] = ((d.e2 + ptz) * dR + ptz_m_ptR * fu2 + bn * dsR) * isrm;
        DR[5] = bnR; DR[6] = dbR2; DR[7] = dbR3;
        // double star
        const f isR = sb_rsqrt(rzR), isL = sb_rsqrt(rzL);
        const f rzRs = rzR * isR, rzLs = rzL * isL;
        const f abn = sb_abs(bn);
        f sbn = 0.0f;
        if (abn > (f)kEpsB) {
            ibn = true;
            sbn = bn > 0.0f ? 1.0f : -1.0f;
            SZL = SM - abn * isL;
            SZR = SM + abn * isR;
        }
        const f irzss = sb_rcp(rzRs + rzLs), rzps = rzRs * rzLs;
        const f dvRL2 = (dv + dvR2) - dvL2, dvRL3 = (dw + dvR3) - dvL3;   // vR* - vL*
        const f dbRL2 = (dby + dbR2) - dbL2, dbRL3 = (dbz + dbR3) - dbL3;   // bR* - bL*
        const f ddvL2 = (rzRs * dvRL2 + sbn * dbRL2) * irzss, ddvL3 = (rzRs * dvRL3 + sbn * dbRL3) * irzss;
        const f ddbL2 = (rzLs * dbRL2 + sbn * rzps * dvRL2) * irzss, ddbL3 = (rzLs * dbRL3 + sbn * rzps * dvRL3) * irzss;
        const f ddvR2 = ddvL2 - dvRL2, ddvR3 = ddvL3 - dvRL3, ddbR2 = ddbL2 - dbRL2, ddbR3 = ddbL3 - dbRL3;
        bzz2 = bz2L + ddbL2;
        bzz3 = bz3L + ddbL3;
        const f dszL = -(vzL2 * ddbL2 + ddvL2 * bzz2) - (vzL3 * ddbL3 + ddvL3 * bzz3);   // sbvL - sbzz
        const f dszR = -(vzR2 * ddbR2 + ddvR2 * bzz2) - (vzR3 * ddbR3 + ddvR3 * bzz3);   // sbvR - sbzz
        DDL[0] = 0.f; DDL[1] = 0.f; DDL[2] = rzL * ddvL2; DDL[3] = rzL * ddvL3; DDL[4] = -rzLs * sbn * dszL;
        DDL[5] = 0.f; DDL[6] = ddbL2; DDL[7] = ddbL3;
        DDR[0] = 0.f; DDR[1] = 0.f; DDR[2] = rzR * ddvR2; DDR[3] = rzR * ddvR3; DDR[4] = rzRs * sbn * dszR;
        DDR[5] = 0.f; DDR[6] = ddbR2; DDR[7] = ddbR3;
        if (SR < 0.0f) region = 6;
        else if (SZR <= 0.0f && SR >= 0.0f) region = 5;
        else if (ibn && SM <= 0.0f && SZR >= 0.0f) region = 4;
        else if (ibn && SZL <= 0.0f && SM >= 0.0f) region = 3;
        else if (SL <= 0.0f && SZL >= 0.0f) region = 2;
        else if (SL > 0.0f) region = 1;
        else region = 0;
    }
    int flag = region == 0 ? kFlagWave : 0;
    right = region >= 4;
    const bool use1 = (region >= 2 && region <= 5), use2 = (region == 3 || region == 4);
    // positivity of the selected star state (rho* > 0, p* = pt* - |b*|^2 / 2 > 0)
    if (use1) {
        const f rz = right ? rzR : rzL;
        const f b2 = use2 ? bzz2 : (right ? bz2R : bz2L), b3 = use2 ? bzz3 : (right ? bz3R : bz3L);
        if (!(rz > 0.0f) || !(ptz - half * ((bn * bn + b2 * b2) + b3 * b3) > 0.0f)) flag |= kFlagStar;
    }
    const f S1 = right ? SR : SL, S2 = right ? SZR : SZL;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        f ck = 0.0f;
        if (use2) ck = S2 * (right ? DDR[k] : DDL[k]);
        if (use1) ck = ck + S1 * (right ? DR[k] : DL[k]);
        c[k] = ck;
    }
    c[5] = NSTATE == 3 ? -sb_max(sb_abs(SL), sb_abs(SR)) * dbx : 0.0f;
    if (!(sb_abs(SL) < 3.0e38f) || !(sb_abs(SR) < 3.0e38f)) flag |= kFlagStar;
    return flag;
}

// Delta form on face states held in type D (FP64 in the delta form): side values rounded to
// FP32, jumps formed in D then rounded, and the physical flux of the selected side in D.
// kFlagStar also when NSTATE 2 sees a magnetic field (the delta form covers hydro HLLC only) --
// the caller then recomputes the face in FP64.  LAZY: FR faces skip the star states (below).
template <int NSTATE, typename D = double, bool LAZY = true>
SB_HD int riemann_delta(const D* q1, const D* q2, D* F, float& SLo, float& SRo, float& SMo) {
    typedef float f;
    const D ispi4 = D(kInvSpi4);
    const D r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const D bx1 = q1[5] * ispi4, by1 = q1[6] * ispi4, bz1 = q1[7] * ispi4;
    const D r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const D bx2 = q2[5] * ispi4, by2 = q2[6] * ispi4, bz2 = q2[7] * ispi4;
    const D b2L = (bx1 * bx1 + by1 * by1) + bz1 * bz1;
    const D b2R = (bx2 * bx2 + by2 * by2) + bz2 * bz2;
    const D ptL = p1 + D(0.5) * b2L, ptR = p2 + D(0.5) * b2R;
    if (NSTATE == 2 && (b2L != D(0) || b2R != D(0))) return kFlagStar;
    // First the values the wave speeds and SM need.  SR < 0 selects FR (the last match of the
    // region chain) whatever the star states are, and FR's flux is the right side's physical flux
    // with c = 0 but the normal-field term, so the remaining conversions and the star states are
    // made only where some other region may be selected.
    DeltaIn d;
    d.r1 = (f)r1; d.u1 = (f)u1; d.p1 = (f)p1; d.bx1 = (f)bx1; d.b2L = (f)b2L;
    d.r2 = (f)r2; d.u2 = (f)u2; d.p2 = (f)p2; d.bx2 = (f)bx2; d.b2R = (f)b2R;
    d.du = (f)(u2 - u1);
    d.dbx = (f)(bx2 - bx1);
    d.dpt = (f)(ptR - ptL);
    float cfL, cfR;
    delta_fast_speeds(d, cfL, cfR);
    float c[8];
    bool right = true;
    int flag;
    D e1 = D(0), e2 = D(0);
    const f suR = sb_max(cfL - d.du, cfR);
    const f SR = d.u2 + suR;
    if (LAZY && SR < 0.0f) {
        const f suL = sb_min(-cfL, d.du - cfR);
        const f SL = d.u1 + suL;
        const f iden = sb_rcp(suR * d.r2 - suL * d.r1);
        SLo = SL;
        SRo = SR;
        SMo = d.u1 + (suR * d.r2 * d.du - d.dpt) * iden;
#pragma unroll
        for (int k = 0; k < 8; k++) c[k] = 0.0f;
        c[5] = NSTATE == 3 ? -sb_max(sb_abs(SL), sb_abs(SR)) * d.dbx : 0.0f;
        flag = (!(sb_abs(SL) < 3.0e38f) || !(sb_abs(SR) < 3.0e38f)) ? kFlagStar : 0;
        e2 = (p2 * D(kInvG1) + r2 * (D(0.5) * ((u2 * u2 + v2 * v2) + w2 * w2))) + D(0.5) * b2R;
    } else {
        e1 = (p1 * D(kInvG1) + r1 * (D(0.5) * ((u1 * u1 + v1 * v1) + w1 * w1))) + D(0.5) * b2L;
        e2 = (p2 * D(kInvG1) + r2 * (D(0.5) * ((u2 * u2 + v2 * v2) + w2 * w2))) + D(0.5) * b2R;
        d.v1 = (f)v1; d.w1 = (f)w1; d.by1 = (f)by1; d.bz1 = (f)bz1; d.e1 = (f)e1; d.ptL = (f)ptL;
        d.v2 = (f)v2; d.w2 = (f)w2; d.by2 = (f)by2; d.bz2 = (f)bz2; d.e2 = (f)e2;
        d.dv = (f)(v2 - v1); d.dw = (f)(w2 - w1);
        d.dby = (f)(by2 - by1); d.dbz = (f)(bz2 - bz1);
        flag = delta_core<NSTATE>(d, cfL, cfR, c, right, SLo, SRo, SMo);
    }
    // physical flux of the selected side
    const D r = right ? r2 : r1, u = right ? u2 : u1, v = right ? v2 : v1, w = right ? w2 : w1;
    const D bx = right ? bx2 : bx1, by = right ? by2 : by1, bz = right ? bz2 : bz1;
    const D pt = right ? ptR : ptL, e = right ? e2 : e1;
    const D m = r * u;
    F[0] = m + (D)c[0];
    F[1] = ((m * u + pt) - bx * bx) + (D)c[1];
    F[2] = (m * v - bx * by) + (D)c[2];
    F[3] = (m * w - bx * bz) + (D)c[3];
    F[4] = ((e + pt) * u - bx * ((u * bx + v * by) + w * bz)) + (D)c[4];
    F[5] = (D)c[5] * D(kSpi4);
    F[6] = ((u * by - v * bx) + (D)c[6]) * D(kSpi4);
    F[7] = ((u * bz - w * bx) + (D)c[7]) * D(kSpi4);
    return flag;
}

// MUSCL-minmod face value of cell c toward its neighbour n with the far cell f on the other
// side: t_c + 0.5*minmod(t_c - t_f, t_n - t_c).  On the Cartesian grid this is the reference's
// linear(-3h/2, t_f, -h/2, t_c, h/2, t_n, 0) (Solvers.f90:141-150, cuf_solvers.cuf:389-392).
template <typename T> SB_HD T muscl(T tf, T tc, T tn) { return tc + T(0.5) * minmod(tc - tf, tn - tc); }

// Face states from the 4-cell stencil (face-frame order), with the positivity fallback of
// cuf_solvers.cuf:394-406.  Only rho, vn, vt1, vt2, p are reconstructed; B stays first order.
template <typename T, int ORDER>
SB_HD void reconstruct(const T* qLL, const T* qL, const T* qR, const T* qRR, T* q1, T* q2) {
#pragma unroll
    for (int v = 0; v < 8; v++) {
        q1[v] = qL[v];
        q2[v] = qR[v];
    }
    if (ORDER == 2) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
            q1[v] = muscl(qLL[v], qL[v], qR[v]);
            q2[v] = muscl(qRR[v], qR[v], qL[v]);
        }
        if (sb_neg(q1[0])) q1[0] = qL[0];
        if (sb_neg(q1[4])) q1[4] = qL[4];
        if (sb_neg(q2[0])) q2[0] = qR[0];
        if (sb_neg(q2[4])) q2[4] = qR[4];
    }
}

}  // namespace sb
