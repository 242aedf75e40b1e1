// fvm2d_math.cuh -- per-cell and per-interface arithmetic of the split step.
//
// One sweep treats its direction as "normal" (n) and the other as
// "tangential" (t): a cell is (rho, p, un, ut).  In an x-sweep un = u; in a
// y-sweep un = v, exactly as the reference's anti-transposed copy swaps the
// u and v slots (src/basicFuns.cuh:249-262).
//
// The functions below keep the reference's operation order: with FMA
// contraction off (-fmad=false) an FP64 build rounds every operation in the
// same order as the reference built the same way, so the two agree bit for
// bit.  The product build contracts (the nvcc default, as the reference's own
// build does) and is checked against the reference within a relative L1
// tolerance.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include <type_traits>

#ifndef FVM2D_VARIANT
#error "define FVM2D_VARIANT (the namespace of this build of the kernels) first"
#endif

namespace fvm2d {
namespace FVM2D_VARIANT {

template <typename Real>
struct Cell {
    Real rho, p, un, ut;
};

template <typename Real>
__device__ __forceinline__ Real rmin(Real a, Real b) { return (b < a) ? b : a; }
template <typename Real>
__device__ __forceinline__ Real rmax(Real a, Real b) { return (a < b) ? b : a; }
// single precision: the min/max instructions (equal to the selects unless an
// argument is NaN)
__device__ __forceinline__ float rmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
// 1/x and 1/sqrt(x).
//
// Builds that define FVM2D_FAST_RCP (the FP64 product build, and the FP64
// wave speed of the FP32 build) take the hardware's approximate seeds --
// PTX rcp.approx.ftz.f64 and rsqrt.approx.ftz.f64, about 20 correct bits --
// and refine each by one third-order step (Householder's method of order 3),
// written from the series
//   1/x       = r / (1 - e)       = r (1 + e + e^2 + ...),         e = 1 - x r
//   1/sqrt(x) = y / sqrt(1 - e)   = y (1 + e/2 + 3 e^2/8 + ...),   e = 1 - x y^2
// truncated after the quadratic term: the relative error falls from about
// 2^-20 to about 2^-58, below the rounding of the result, so the results are
// within a couple of ulp of correctly rounded ones (not bit-identical: that
// build is held to the reference within a relative L1 tolerance; a further
// Newton step towards correct rounding was measured to leave its distance
// from the oracle no smaller, 5% slower).  Each costs the seed and three to
// five FP64 operations instead of a full IEEE division or square-root
// sequence.  The
// seeds flush subnormal arguments to zero, so the arguments must be normal
// numbers: the solver's reciprocals take densities, pressures, sound speeds
// and their products, which are, in any state that is not degenerate
// (vacuum) or corrupt; the wave speed, whose velocity part can be
// arbitrarily small, clamps its arguments (wave_speed).  Other builds use
// IEEE division and CUDA's rsqrt (1 ulp); rsqrtf is within 2 ulp; the
// dual-number overloads live with the dual type, and other number types
// divide.
#if defined(FVM2D_FAST_RCP)
__device__ __forceinline__ double rcp_seed(double x)
{
#if defined(__CUDA_ARCH__)
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
#else
    return (1.0 / x) * (1.0 + 0x1p-21);  // host builds of this file (tests): a seed 2^-21 off
#endif
}
__device__ __forceinline__ double rsqrt_seed(double x)
{
#if defined(__CUDA_ARCH__)
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
#else
    return (1.0 / sqrt(x)) * (1.0 - 0x1p-21);
#endif
}
__device__ __forceinline__ double rrcp(double x)
{
    const double r = rcp_seed(x);
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ double rrsqrt(double x)
{
    const double y = rsqrt_seed(x);
    const double e = fma(-(x * y), y, 1.0);
    return fma(y, e * fma(e, 0.375, 0.5), y);
}
#else
__device__ __forceinline__ double rrcp(double x) { return 1.0 / x; }
__device__ __forceinline__ double rrsqrt(double x) { return ::rsqrt(x); }
#endif
__device__ __forceinline__ float rrcp(float x) { return 1.0f / x; }
__device__ __forceinline__ float rrsqrt(float x) { return ::rsqrtf(x); }
template <typename Real>
__device__ __forceinline__ Real rrcp(Real x) { return Real(1) / x; }

// Generalized-minmod slope of one component from its left (m), centre (c)
// and right (p) values.  src/basicFuns.cuh:49-68.
template <typename Real>
__device__ __forceinline__ Real limited_slope(Real m, Real c, Real p, Real rh, Real alpha)
{
    Real central = (p - m) * Real(0.5) * rh;
    Real back = (c - m) * rh * alpha;
    Real fwd = (p - c) * rh * alpha;
    Real p13 = central * fwd, p23 = back * fwd;
    if (p13 > Real(0) && p23 > Real(0)) {
        Real sign = (central <= Real(0)) ? Real(-1) : Real(1);
        return sign * rmin(fabs(central), rmin(fabs(back), fabs(fwd)));
    }
    return Real(0);
}

// Interface state W = (rho, p, un, ut, e) and its time derivative Wt.
template <typename Real>
struct Interface {
    Real rho, p, un, ut, e;
    Real rho_t, p_t, un_t, ut_t, e_t;
};

// Relaxation GRP at one interface from the left/right face states (L, R)
// and the slopes of the two cells (sL, sR).  src/basicFuns.cuh:86-189.
// The star-region coefficients k_l, k_r, d_l, d_r read the velocity before
// it receives the star value (basicFuns.cuh:151-155 see the initial 0.0 of
// basicFuns.cuh:110); the literal `u0` keeps that.
template <typename Real>
__device__ __forceinline__ Interface<Real> relaxation_grp(const Cell<Real> &L, const Cell<Real> &R,
                                                          const Cell<Real> &sL, const Cell<Real> &sR,
                                                          Real g)
{
    const Real rho_l = L.rho, pi_l = L.p, u_l = L.un, v_l = L.ut;
    const Real rho_r = R.rho, pi_r = R.p, u_r = R.un, v_r = R.ut;
    const Real rho_lx = sL.rho, pi_lx = sL.p, u_lx = sL.un, v_lx = sL.ut;
    const Real rho_rx = sR.rho, pi_rx = sR.p, u_rx = sR.un, v_rx = sR.ut;
    const Real one = Real(1), two = Real(2), half = Real(0.5), zero = Real(0);

    Real e_l = pi_l / rho_l / (g - one);
    Real e_r = pi_r / rho_r / (g - one);
    Real e_lx = pi_lx / rho_l / (g - one) - pi_l * rho_lx / rho_l / rho_l / (g - one);
    Real e_rx = pi_rx / rho_r / (g - one) - pi_r * rho_rx / rho_r / rho_r / (g - one);
    Real c_lx = half * sqrt(g / pi_l / rho_l) * (pi_l * rho_lx + rho_l * pi_lx);
    Real c_rx = half * sqrt(g / pi_r / rho_r) * (pi_r * rho_rx + rho_r * pi_rx);

    Interface<Real> o;
    Real c_l, c_r;
    Real a_l = sqrt(g * pi_l / rho_l), a_r = sqrt(g * pi_r / rho_r);
    Real kappa = (g + one) / two;
    if (pi_r >= pi_l) {
        c_l = rho_l * (a_l + kappa * rmax(zero, (pi_r - pi_l) / rho_r / a_r + u_l - u_r));
        c_r = rho_r * (a_r + kappa * rmax(zero, (pi_l - pi_r) / c_l + u_l - u_r));
    } else {
        c_r = rho_r * (a_r + kappa * rmax(zero, (pi_l - pi_r) / rho_l / a_l + u_l - u_r));
        c_l = rho_l * (a_l + kappa * rmax(zero, (pi_r - pi_l) / c_r + u_l - u_r));
    }

    if (u_l - c_l / rho_l >= zero) {
        // the whole wave fan moves right: left state (basicFuns.cuh:129-137)
        Real rho = rho_l, pi = pi_l, u = u_l;
        o.rho = rho_l; o.p = pi_l; o.un = u_l; o.ut = v_l; o.e = e_l;
        o.rho_t = -rho * u_lx - u * rho_lx;
        o.un_t = -u * u_lx - pi_lx / rho;
        o.e_t = -u * e_lx - pi / rho * u_lx;
        o.ut_t = -u * v_lx;
        o.p_t = -u * pi_lx - c_l * c_l / rho_l * u_lx;
    } else if (u_r + c_r / rho_r <= zero) {
        // the whole wave fan moves left: right state (basicFuns.cuh:138-146)
        Real rho = rho_r, pi = pi_r, u = u_r;
        o.rho = rho_r; o.p = pi_r; o.un = u_r; o.ut = v_r; o.e = e_r;
        o.rho_t = -rho * u_rx - u * rho_rx;
        o.un_t = -u * u_rx - pi_rx / rho;
        o.e_t = -u * e_rx - pi / rho * u_rx;
        o.ut_t = -u * v_rx;
        o.p_t = -u * pi_rx - c_r * c_r / rho * u_rx;
    } else {
        // star region (basicFuns.cuh:147-186)
        const Real u0 = zero;
        Real u_m = (u_l * c_l + u_r * c_r + pi_l - pi_r) / (c_l + c_r);
        Real pi_m = ((u_l - u_r) * c_l * c_r + c_l * pi_r + c_r * pi_l) / (c_l + c_r);
        Real k_l = -pi_lx - c_l * u_lx + half * (u0 - u_l) * c_lx;
        Real k_r = -pi_rx + c_r * u_rx - half * (u0 - u_r) * c_rx;
        Real d_l = Real(-2.0) * c_l * c_l / rho_l * u_lx - two * c_l / rho_l * pi_lx + c_l / rho_l * (u0 - u_l) * c_lx;
        Real d_r = two * c_r * c_r / rho_r * u_rx - two * c_r / rho_r * pi_rx + c_r / rho_r * (u_r - u0) * c_rx;
        Real Dpi_Dt = (c_r * d_l - c_l * d_r) / two / (c_l + c_r);
        Real pi = pi_m, u = u_m, rho, e;
        o.p = pi_m;
        o.un = u_m;
        if (u <= zero) {
            Real rho_mr = c_r / (u_r - u_m + c_r / rho_r);
            Real e_mr = e_r + (pi_m - pi_r) * (pi_m + pi_r) / two / c_r / c_r;
            rho = rho_mr;
            e = e_mr;
            o.ut = v_r;
            o.rho_t = -u * rho * rho * rho / (rho_r * c_r * c_r) * (c_r * c_r / rho_r / rho_r * rho_rx - c_r * u_rx + Real(1.5) * (u - u_r) * c_rx) + rho * rho * rho / (c_r * c_r * c_r) * (u + c_r / rho) * Dpi_Dt;
            o.p_t = one / (c_l + c_r) * (c_l * c_r / rho_l * (one + u * rho / c_r) * k_l - c_l * c_r / rho_r * (one - u * rho / c_l) * k_r);
            o.un_t = one / (c_l + c_r) * (c_l / rho_l * (one + u * rho / c_r) * k_l + c_r / rho_r * (one - u * rho * c_l / c_r / c_r) * k_r);
            o.e_t = -u * rho / rho_r / c_r / c_r / c_r * (-pi_r * c_r * pi_rx + c_r * c_r * c_r * e_rx + two * (e_r - e) * c_r * c_r * c_rx) + pi / c_r / c_r * o.p_t;
            Real v_x = rho / rho_r * v_rx;
            o.ut_t = -u * v_x;
        } else {
            Real rho_ml = c_l / (u_m - u_l + c_l / rho_l);
            Real e_ml = e_l + (pi_m - pi_l) * (pi_m + pi_l) / two / c_l / c_l;
            rho = rho_ml;
            e = e_ml;
            o.ut = v_l;
            o.rho_t = -u * rho * rho * rho / (rho_l * c_l * c_l) * (c_l * c_l / rho_l / rho_l * rho_lx + c_l * u_lx + Real(1.5) * (u - u_l) * c_lx) - rho * rho * rho / (c_l * c_l * c_l) * (u - c_l / rho) * Dpi_Dt;
            o.p_t = one / (c_l + c_r) * (c_l * c_r / rho_l * (one + u * rho / c_r) * k_l - c_l * c_r / rho_r * (one - u * rho / c_l) * k_r);
            o.un_t = one / (c_l + c_r) * (c_l / rho_l * (one + u * rho * c_r / c_l / c_l) * k_l + c_r / rho_r * (one - u * rho / c_l) * k_r);
            o.e_t = -u * rho / rho_l / c_l / c_l / c_l * (-pi_l * c_l * pi_lx + c_l * c_l * c_l * e_lx + two * (e_l - e) * c_l * c_l * c_lx) + pi / c_l / c_l * o.p_t;
            Real v_x = rho / rho_l * v_lx;
            o.ut_t = -u * v_x;
        }
        o.rho = rho;
        o.e = e;
    }
    return o;
}

// Midpoint flux F(W) + k/2 dF/dt in the sweep's conserved ordering
// (mass, normal momentum, energy, tangential momentum).
// src/basicFuns.cuh:14-34.
template <typename Real>
__device__ __forceinline__ Cell<Real> midpoint_flux(const Interface<Real> &w, Real k)
{
    const Real rho = w.rho, pi = w.p, u = w.un, v = w.ut, e = w.e;
    const Real rho_t = w.rho_t, pi_t = w.p_t, u_t = w.un_t, v_t = w.ut_t, e_t = w.e_t;
    const Real two = Real(2);
    Cell<Real> F;
    F.rho = rho * u + k / two * (rho * u_t + u * rho_t);
    F.p = rho * u * u + pi + k / two * (rho_t * u * u + two * rho * u * u_t + pi_t);
    F.un = rho * u * (e + u * u / two + v * v / two) + pi * u + k / two * (rho_t * u * e + rho * u_t * e + rho * u * e_t + rho_t * u * u * u / two + Real(1.5) * rho * u * u * u_t + rho_t * u * v * v / two + rho * u * v * v_t + rho * u_t * v * v / two + pi_t * u + pi * u_t);
    F.ut = rho * u * v + k / two * (rho * u_t * v + u * rho_t * v + u * rho * v_t);
    return F;
}

// Conservative update of one cell, primitive in and out:
// W = cons(U); W -= (F_R - F_L) * lambda; U = prim(W).
// src/basicFuns.cuh:195-212, 240-244.  Field slots of the flux Cell are
// (mass, normal momentum, energy, tangential momentum).
template <typename Real>
__device__ __forceinline__ Cell<Real> conservative_update(const Cell<Real> &U, const Cell<Real> &FL,
                                                          const Cell<Real> &FR, Real lambda, Real g)
{
    const Real one = Real(1), two = Real(2);
    Real m0 = U.rho;
    Real m1 = U.rho * U.un;
    Real m2 = U.p / (g - one) + U.rho * (U.un * U.un + U.ut * U.ut) / two;
    Real m3 = U.rho * U.ut;
    m0 = m0 - (FR.rho - FL.rho) * lambda;
    m1 = m1 - (FR.p - FL.p) * lambda;
    m2 = m2 - (FR.un - FL.un) * lambda;
    m3 = m3 - (FR.ut - FL.ut) * lambda;
    Cell<Real> o;
    o.rho = m0;
    o.p = (g - one) * (m2 - m1 * m1 / m0 / two - m3 * m3 / m0 / two);
    o.un = m1 / m0;
    o.ut = m3 / m0;
    return o;
}

// ---------------------------------------------------------------------------
// Arithmetic policies.  A sweep kernel calls Phys::interface_flux once per
// interface and Phys::update once per cell.
//
// RefOrder: the reference's expressions in the reference's order (above).
// Hoisted:  the same mathematics with the reciprocals hoisted and shared
//           (1/rho_l and 1/rho_r from one division; 1/(rho a) per side as
//           1/sqrt(g p rho), with a = g p/(rho a); the second side's 1/c and
//           1/(c_l + c_r) from one division; 1/c of the first side and
//           1/rho_star: 4 divisions and 2 reciprocal square roots per
//           interface in the star region, 3 and 2 when the wave fan is
//           one-sided, where the reference's expressions divide by a
//           variable 61 times (27-28) and take 4 square roots),
//           sqrt(g/(p rho)) rewritten as g/(rho a), and the midpoint flux
//           written through the mass flux
//           m = rho u and its time derivative; the limiter tests signs on
//           the raw differences and scales its minimum once, and h/2 is
//           folded into the face states.  Rounding differs from the
//           reference at the ulp level; results are checked against the
//           reference within a relative L1 tolerance.
// ---------------------------------------------------------------------------
template <typename Real>
struct SweepConsts {
    Real h, rh, alpha, g;  // spacing, 1/h, limiter parameter, gamma
    Real k, lambda;        // dt and dt/h
    Real igm1, kappa;      // 1/(gamma-1), (gamma+1)/2   (Hoisted only)
    // 1/(gamma-1) and gamma-1 as hi + lo pairs of the arithmetic type (lo = 0
    // unless Real is float), for the compensated FP32 update: it converts p
    // to E and back once per sweep, and with the rounded constants alone
    // (2.5f and 1.4f - 1 for gamma 1.4) every round trip scales the internal
    // energy by 1 - 6e-8, a bias that grows with the number of sweeps
    Real igm1_lo, gm1, gm1_lo;
    Real lambda_lo;  // dt/h - lambda (0 unless Real is float): the FP64 update of residual builds
};

// The part of x that Real does not hold: 0 unless Real is float.
template <typename Real>
__host__ __device__ inline double lo_part(double x)
{
    if constexpr (std::is_same<Real, float>::value)
        return x - double(float(x));
    else
        return 0.0;
}

// The constants of gamma in SweepConsts.
template <typename Real>
__host__ __device__ inline void set_gamma_consts(SweepConsts<Real> &K, double gamma)
{
    const double gm1 = gamma - 1.0, igm1 = 1.0 / gm1;
    K.g = Real(gamma);
    K.igm1 = Real(igm1);
    K.igm1_lo = Real(lo_part<Real>(igm1));
    K.gm1 = Real(gm1);
    K.gm1_lo = Real(lo_part<Real>(gm1));
    K.kappa = Real((gamma + 1.0) / 2.0);
}

template <typename Real>
__device__ __forceinline__ Cell<Real> cell_slope(const Cell<Real> &m, const Cell<Real> &c, const Cell<Real> &p,
                                                 const SweepConsts<Real> &K)
{
    Cell<Real> s;
    s.rho = limited_slope(m.rho, c.rho, p.rho, K.rh, K.alpha);
    s.p = limited_slope(m.p, c.p, p.p, K.rh, K.alpha);
    s.un = limited_slope(m.un, c.un, p.un, K.rh, K.alpha);
    s.ut = limited_slope(m.ut, c.ut, p.ut, K.rh, K.alpha);
    return s;
}

// Face states of the interface between cells L and R: U_L + s_L h/2 and
// U_R - s_R h/2 (src/basicFuns.cuh:69-70).
template <typename Real>
__device__ __forceinline__ void face_states(const Cell<Real> &UL, const Cell<Real> &UR, const Cell<Real> &sL,
                                            const Cell<Real> &sR, Real h, Cell<Real> &fL, Cell<Real> &fR)
{
    fL.rho = UL.rho + sL.rho * h * Real(0.5);
    fL.p = UL.p + sL.p * h * Real(0.5);
    fL.un = UL.un + sL.un * h * Real(0.5);
    fL.ut = UL.ut + sL.ut * h * Real(0.5);
    fR.rho = UR.rho - sR.rho * h * Real(0.5);
    fR.p = UR.p - sR.p * h * Real(0.5);
    fR.un = UR.un - sR.un * h * Real(0.5);
    fR.ut = UR.ut - sR.ut * h * Real(0.5);
}

struct RefOrder {
    template <typename Real>
    __device__ static __forceinline__ Cell<Real> slope(const Cell<Real> &m, const Cell<Real> &c, const Cell<Real> &p,
                                                       const SweepConsts<Real> &K)
    {
        return cell_slope(m, c, p, K);
    }
    template <typename Real>
    __device__ static __forceinline__ Cell<Real> interface_flux(const Cell<Real> &UL, const Cell<Real> &UR,
                                                                const Cell<Real> &sL, const Cell<Real> &sR,
                                                                const SweepConsts<Real> &K)
    {
        Cell<Real> fL, fR;
        face_states(UL, UR, sL, sR, K.h, fL, fR);
        return midpoint_flux(relaxation_grp(fL, fR, sL, sR, K.g), K.k);
    }
    template <typename Real>
    __device__ static __forceinline__ Cell<Real> update(const Cell<Real> &U, const Cell<Real> &FL,
                                                        const Cell<Real> &FR, const SweepConsts<Real> &K)
    {
        return conservative_update(U, FL, FR, K.lambda, K.g);
    }
};

// Generalized minmod on raw differences: the reference's sign tests on the
// scaled differences are sign tests on the differences themselves (rh and
// alpha are positive), and the minimum is scaled once.
template <typename Real>
__device__ __forceinline__ Real limited_slope_hoisted(Real m, Real c, Real p, Real hrh, Real rha)
{
    const Real d1 = c - m, d2 = p - c, dc = p - m;
    if (dc * d2 > Real(0) && d1 * d2 > Real(0)) {
        const Real a = rmin(fabs(dc) * hrh, rha * rmin(fabs(d1), fabs(d2)));
        return dc <= Real(0) ? -a : a;
    }
    return Real(0);
}

// Double precision: the same result with one product and one test.  d1 d2 > 0
// implies dc d2 > 0: d1, d2 nonzero of one sign puts m, c, p in strict order,
// so dc = fl(p - m) has that sign and |dc| >= |d1| (rounding is monotonic),
// hence |dc d2| >= |d1 d2| > 0; then dc != 0 and the result takes its sign.
// The branch skips the minima where the slope is zero (constant regions):
// measured 2.4% off the FP64 step at 4096^2, where computing them
// unconditionally (a select) cost 7%.
__device__ __forceinline__ double limited_slope_hoisted(double m, double c, double p, double hrh, double rha)
{
    const double d1 = c - m, d2 = p - c, dc = p - m;
    if (d1 * d2 > 0.0) return copysign(rmin(fabs(dc) * hrh, rha * rmin(fabs(d1), fabs(d2))), dc);
    return 0.0;
}

// Single precision: the same choices with the min/max and sign instructions
// (they differ from the selects above only when an argument is NaN); the
// sign test is d1 d2 > 0 alone, for the reason given above.
__device__ __forceinline__ float limited_slope_hoisted(float m, float c, float p, float hrh, float rha)
{
    const float d1 = c - m, d2 = p - c, dc = p - m;
    const float a = fminf(fabsf(dc) * hrh, rha * fminf(fabsf(d1), fabsf(d2)));
    return d1 * d2 > 0.f ? copysignf(a, dc) : 0.f;
}

struct Hoisted {
    template <typename Real>
    __device__ static __forceinline__ Cell<Real> slope(const Cell<Real> &m, const Cell<Real> &c, const Cell<Real> &p,
                                                       const SweepConsts<Real> &K)
    {
        Cell<Real> s;
        const Real hrh = K.rh * Real(0.5), rha = K.rh * K.alpha;
        s.rho = limited_slope_hoisted(m.rho, c.rho, p.rho, hrh, rha);
        s.p = limited_slope_hoisted(m.p, c.p, p.p, hrh, rha);
        s.un = limited_slope_hoisted(m.un, c.un, p.un, hrh, rha);
        s.ut = limited_slope_hoisted(m.ut, c.ut, p.ut, hrh, rha);
        return s;
    }
    template <typename Real>
    __device__ static __forceinline__ Interface<Real> grp(const Cell<Real> &L, const Cell<Real> &R,
                                                          const Cell<Real> &sL, const Cell<Real> &sR,
                                                          const SweepConsts<Real> &K)
    {
        const Real one = Real(1), half = Real(0.5), zero = Real(0);
        const Real g = K.g, igm1 = K.igm1, kappa = K.kappa;
        const Real rho_l = L.rho, pi_l = L.p, u_l = L.un, v_l = L.ut;
        const Real rho_r = R.rho, pi_r = R.p, u_r = R.un, v_r = R.ut;
        const Real rho_lx = sL.rho, pi_lx = sL.p, u_lx = sL.un, v_lx = sL.ut;
        const Real rho_rx = sR.rho, pi_rx = sR.p, u_rx = sR.un, v_rx = sR.ut;

        // 1/rho_l and 1/rho_r from one division
        const Real irlr = rrcp(rho_l * rho_r);
        const Real irl = rho_r * irlr, irr = rho_l * irlr;
        const Real e_l = pi_l * irl * igm1, e_r = pi_r * irr * igm1;
        const Real e_lx = (pi_lx - pi_l * rho_lx * irl) * irl * igm1;
        const Real e_rx = (pi_rx - pi_r * rho_rx * irr) * irr * igm1;
        // 1/(rho a) = 1/sqrt(g p rho) and a = sqrt(g p / rho) = g p / sqrt(g p rho):
        // one reciprocal square root per side
        const Real il = rrsqrt(g * pi_l * rho_l), ir = rrsqrt(g * pi_r * rho_r);
        const Real a_l = g * pi_l * il, a_r = g * pi_r * ir;
        const Real c_lx = half * g * (pi_l * rho_lx + rho_l * pi_lx) * il;
        const Real c_rx = half * g * (pi_r * rho_rx + rho_r * pi_rx) * ir;
        const Real du = u_l - u_r;
        // the side computed second gets its reciprocal and 1/(c_l + c_r)
        // from one division
        Real c_l, c_r, icl, icr, isum;
        if (pi_r >= pi_l) {
            c_l = rho_l * (a_l + kappa * rmax(zero, (pi_r - pi_l) * ir + du));
            icl = rrcp(c_l);
            c_r = rho_r * (a_r + kappa * rmax(zero, (pi_l - pi_r) * icl + du));
            const Real sc = c_l + c_r, q = rrcp(c_r * sc);
            icr = sc * q;
            isum = c_r * q;
        } else {
            c_r = rho_r * (a_r + kappa * rmax(zero, (pi_l - pi_r) * il + du));
            icr = rrcp(c_r);
            c_l = rho_l * (a_l + kappa * rmax(zero, (pi_r - pi_l) * icr + du));
            const Real sc = c_l + c_r, q = rrcp(c_l * sc);
            icl = sc * q;
            isum = c_l * q;
        }
        const Real sl = c_l * irl, sr = c_r * irr;  // c/rho: the fan's edge speeds relative to u
        Interface<Real> o;
        if (u_l - sl >= zero) {
            o.rho = rho_l; o.p = pi_l; o.un = u_l; o.ut = v_l; o.e = e_l;
            o.rho_t = -rho_l * u_lx - u_l * rho_lx;
            o.un_t = -u_l * u_lx - pi_lx * irl;
            o.e_t = -u_l * e_lx - pi_l * irl * u_lx;
            o.ut_t = -u_l * v_lx;
            o.p_t = -u_l * pi_lx - c_l * sl * u_lx;
        } else if (u_r + sr <= zero) {
            o.rho = rho_r; o.p = pi_r; o.un = u_r; o.ut = v_r; o.e = e_r;
            o.rho_t = -rho_r * u_rx - u_r * rho_rx;
            o.un_t = -u_r * u_rx - pi_rx * irr;
            o.e_t = -u_r * e_rx - pi_r * irr * u_rx;
            o.ut_t = -u_r * v_rx;
            o.p_t = -u_r * pi_rx - c_r * sr * u_rx;
        } else {
            const Real u = (u_l * c_l + u_r * c_r + pi_l - pi_r) * isum;
            const Real pm = (du * c_l * c_r + c_l * pi_r + c_r * pi_l) * isum;
            const Real k_l = -pi_lx - c_l * u_lx - half * u_l * c_lx;
            const Real k_r = -pi_rx + c_r * u_rx + half * u_r * c_rx;
            const Real d_l = sl * (Real(-2) * (c_l * u_lx + pi_lx) - u_l * c_lx);
            const Real d_r = sr * (Real(2) * (c_r * u_rx - pi_rx) + u_r * c_rx);
            const Real Dp = (c_r * d_l - c_l * d_r) * half * isum;
            o.p = pm;
            o.un = u;
            if (u <= zero) {
                const Real irho = (u_r - u + sr) * icr;
                const Real rho = rrcp(irho);
                const Real icr2 = icr * icr;
                const Real e = e_r + (pm - pi_r) * (pm + pi_r) * half * icr2;
                const Real rho3 = rho * rho * rho, urho = u * rho;
                o.rho = rho; o.e = e; o.ut = v_r;
                o.rho_t = -u * rho3 * irr * icr2 * (sr * sr * rho_rx - c_r * u_rx + Real(1.5) * (u - u_r) * c_rx) +
                          rho3 * icr2 * icr * (u + c_r * irho) * Dp;
                o.p_t = isum * (c_r * sl * (one + urho * icr) * k_l - c_l * sr * (one - urho * icl) * k_r);
                o.un_t = isum * (sl * (one + urho * icr) * k_l + sr * (one - urho * c_l * icr2) * k_r);
                o.e_t = -urho * irr * (e_rx - pi_r * pi_rx * icr2 + Real(2) * (e_r - e) * c_rx * icr) + pm * icr2 * o.p_t;
                o.ut_t = -urho * irr * v_rx;
            } else {
                const Real irho = (u - u_l + sl) * icl;
                const Real rho = rrcp(irho);
                const Real icl2 = icl * icl;
                const Real e = e_l + (pm - pi_l) * (pm + pi_l) * half * icl2;
                const Real rho3 = rho * rho * rho, urho = u * rho;
                o.rho = rho; o.e = e; o.ut = v_l;
                o.rho_t = -u * rho3 * irl * icl2 * (sl * sl * rho_lx + c_l * u_lx + Real(1.5) * (u - u_l) * c_lx) -
                          rho3 * icl2 * icl * (u - c_l * irho) * Dp;
                o.p_t = isum * (c_r * sl * (one + urho * icr) * k_l - c_l * sr * (one - urho * icl) * k_r);
                o.un_t = isum * (sl * (one + urho * c_r * icl2) * k_l + sr * (one - urho * icl) * k_r);
                o.e_t = -urho * irl * (e_lx - pi_l * pi_lx * icl2 + Real(2) * (e_l - e) * c_lx * icl) + pm * icl2 * o.p_t;
                o.ut_t = -urho * irl * v_lx;
            }
        }
        return o;
    }

    template <typename Real>
    __device__ static __forceinline__ Cell<Real> interface_flux(const Cell<Real> &UL, const Cell<Real> &UR,
                                                                const Cell<Real> &sL, const Cell<Real> &sR,
                                                                const SweepConsts<Real> &K)
    {
        const Real hh = K.h * Real(0.5);
        Cell<Real> fL, fR;  // U_L + s_L h/2, U_R - s_R h/2 with h/2 folded in
        fL.rho = fma(sL.rho, hh, UL.rho);
        fL.p = fma(sL.p, hh, UL.p);
        fL.un = fma(sL.un, hh, UL.un);
        fL.ut = fma(sL.ut, hh, UL.ut);
        fR.rho = fma(-sR.rho, hh, UR.rho);
        fR.p = fma(-sR.p, hh, UR.p);
        fR.un = fma(-sR.un, hh, UR.un);
        fR.ut = fma(-sR.ut, hh, UR.ut);
        const Interface<Real> w = grp(fL, fR, sL, sR, K);
        // F + k/2 dF/dt through m = rho u and m_t = d(rho u)/dt (the product
        // rule applied to src/basicFuns.cuh:28-33)
        const Real hk = K.k * Real(0.5);
        const Real m = w.rho * w.un, m_t = w.rho * w.un_t + w.un * w.rho_t;
        const Real es = w.e + Real(0.5) * (w.un * w.un + w.ut * w.ut);
        Cell<Real> F;
        F.rho = m + hk * m_t;
        F.p = m * w.un + w.p + hk * (m_t * w.un + m * w.un_t + w.p_t);
        F.un = m * es + w.p * w.un +
               hk * (m_t * es + m * (w.e_t + w.un * w.un_t + w.ut * w.ut_t) + w.p_t * w.un + w.p * w.un_t);
        F.ut = m * w.ut + hk * (m_t * w.ut + m * w.ut_t);
        return F;
    }

    template <typename Real>
    __device__ static __forceinline__ Cell<Real> update(const Cell<Real> &U, const Cell<Real> &FL,
                                                        const Cell<Real> &FR, const SweepConsts<Real> &K)
    {
        const Real half = Real(0.5);
        Real m0 = U.rho;
        Real m1 = U.rho * U.un;
        Real m2 = U.p * K.igm1 + half * U.rho * (U.un * U.un + U.ut * U.ut);
        Real m3 = U.rho * U.ut;
        m0 -= (FR.rho - FL.rho) * K.lambda;
        m1 -= (FR.p - FL.p) * K.lambda;
        m2 -= (FR.un - FL.un) * K.lambda;
        m3 -= (FR.ut - FL.ut) * K.lambda;
        const Real ir = rrcp(m0);
        Cell<Real> o;
        o.rho = m0;
        o.un = m1 * ir;
        o.ut = m3 * ir;
        o.p = (K.g - Real(1)) * (m2 - half * (m1 * m1 + m3 * m3) * ir);
        return o;
    }
};

// ---------------------------------------------------------------------------
// Compensated conservative update for FP32 storage.  The cell's conserved
// vector and its update are carried as unevaluated sums hi + lo built from
// error-free transformations (TwoSum, and TwoProd through fma), so the sum
// W - lambda (F_R - F_L) loses nothing to rounding before the primitive
// variables are recovered; the recovery divides and subtracts with the same
// residual terms.  The only roundings left are the flux difference itself and
// the final rounding of each primitive to its FP32 plane.
// ---------------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ void two_sum(Real a, Real b, Real &s, Real &e)
{
    s = a + b;
    const Real bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

template <typename Real>
__device__ __forceinline__ void two_prod(Real a, Real b, Real &p, Real &e)
{
    p = a * b;
    e = fma(a, b, -p);
}

struct HoistedCompensated : Hoisted {
    template <typename Real>
    __device__ static __forceinline__ Cell<Real> update(const Cell<Real> &U, const Cell<Real> &FL,
                                                        const Cell<Real> &FR, const SweepConsts<Real> &K)
    {
        const Real half = Real(0.5);
        // conserved vector of the cell: (rho, rho un, E, rho ut) as hi + lo
        Real m1, m1e, m3, m3e;
        two_prod(U.rho, U.un, m1, m1e);
        two_prod(U.rho, U.ut, m3, m3e);
        Real ka, kae, kb, kbe, kin, kine;
        two_prod(m1, U.un, ka, kae);
        two_prod(m3, U.ut, kb, kbe);
        two_sum(ka, kb, kin, kine);
        kine += kae + kbe + m1e * U.un + m3e * U.ut;  // rho (un^2 + ut^2) = kin + kine
        Real pe, pee, E, Ee;
        two_prod(U.p, K.igm1, pe, pee);
        pee = fma(U.p, K.igm1_lo, pee);  // p / (gamma - 1) = pe + pee
        two_sum(pe, half * kin, E, Ee);
        Ee += pee + half * kine;
        // W - lambda (F_R - F_L), compensated
        Real s0, e0, s1, e1, s2, e2, s3, e3;
        two_sum(U.rho, -(FR.rho - FL.rho) * K.lambda, s0, e0);
        two_sum(m1, -(FR.p - FL.p) * K.lambda, s1, e1);
        two_sum(E, -(FR.un - FL.un) * K.lambda, s2, e2);
        two_sum(m3, -(FR.ut - FL.ut) * K.lambda, s3, e3);
        e1 += m1e;
        e2 += Ee;
        e3 += m3e;
        // primitives from (s + e)
        Cell<Real> o;
        o.rho = s0 + e0;
        const Real ir = Real(1) / o.rho;
        const Real qu = s1 * ir, qv = s3 * ir;
        o.un = fma(fma(-qu, o.rho, s1) + e1, ir, qu);
        o.ut = fma(fma(-qv, o.rho, s3) + e3, ir, qv);
        Real ku, kue, kv, kve, k2, k2e;
        two_prod(s1, o.un, ku, kue);
        two_prod(s3, o.ut, kv, kve);
        two_sum(ku, kv, k2, k2e);
        k2e += kue + kve + e1 * o.un + e3 * o.ut;  // m . u = k2 + k2e
        Real d, de;
        two_sum(s2, -half * k2, d, de);
        const Real ei = d + (de + e2 - half * k2e);  // internal energy
        o.p = fma(K.gm1, ei, K.gm1_lo * ei);        // (gamma - 1) ei with the constant's low part
        return o;
    }
};

// |(u, v)| + sqrt(gamma p / rho) in the array's own (u, v) order.
// src/basicFuns.cuh:223-224.
template <typename Real>
__device__ __forceinline__ double wave_speed(Real rho, Real p, Real u, Real v, double g)
{
    double du = double(u), dv = double(v);
#if defined(FVM2D_FAST_RCP)
    // sqrt(q) = q / sqrt(q) and sqrt(g p / rho) = |g p| / sqrt(g p rho):
    // two reciprocal square roots, no division.  The reciprocal square root
    // wants a normal argument: q below 2^-998 (zero and the subnormal squares
    // of vanishing velocities ahead of a wave included) takes that bound, so
    // the speed stays below 2^-499 (0 for q = 0), which adds nothing to the
    // maximum; g p rho is clamped to [2^-998, 2^998], which changes nothing
    // but degenerate states (vacuum, or pressure and density both below
    // 1e-150), and where it is negative or NaN the sound speed is NaN, as the
    // reference's square root makes it (a NaN never wins the maximum)
    // (every product and sum is rounded on its own -- no contraction choice
    // left to the compiler -- so the init, final-sweep and ghost kernels give
    // the same bits for the same cell, and a resumed run the same dt)
    const double q = fma(du, du, __dmul_rn(dv, dv));
    const double velo = __dmul_rn(q, rrsqrt(fmax(q, 0x1p-998)));
    const double gp = __dmul_rn(g, double(p)), gpr = __dmul_rn(gp, double(rho));
    const double c = __dmul_rn(fabs(gp), rrsqrt(fmin(fmax(gpr, 0x1p-998), 0x1p998)));
    return __dadd_rn(velo, gpr >= 0.0 ? c : nan(""));
#else
    double velo = sqrt(du * du + dv * dv);
    double c = sqrt(g * double(p) / double(rho));
    return fabs(velo) + c;
#endif
}

} // namespace FVM2D_VARIANT
} // namespace fvm2d
