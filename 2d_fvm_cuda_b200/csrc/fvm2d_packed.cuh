// fvm2d_packed.cuh -- the FP32 physics with sm_100's packed two-wide FP32
// instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn): pairs of independent
// single-precision operations issue as one instruction.  Used where the pairs
// come naturally: the face states (two field pairs per side) and the
// compensated conservative update (the conserved vector as (rho, rho un) and
// (E, rho ut), the momenta as (rho un, rho ut)).  Packing the limiter's field
// pairs or the relaxation GRP's left/right set-up as well was measured
// slower (the pairing moves and registers cost more than they save), so the
// GRP and limiter stay those of HoistedCompensated.  Same mathematics as
// HoistedCompensated; rounding differs at the FP32 ulp level.
#pragma once

#include "fvm2d_math.cuh"

namespace fvm2d {
namespace FVM2D_VARIANT {

__device__ __forceinline__ float2 p2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// TwoSum on two pairs at once: s + e = a + b exactly, per lane.
__device__ __forceinline__ void two_sum2(float2 a, float2 b, float2 &s, float2 &e)
{
    s = add2(a, b);
    const float2 bb = sub2(s, a);
    e = add2(sub2(a, sub2(s, bb)), sub2(b, bb));
}

struct PackedCompensated : HoistedCompensated {
    // Hoisted::interface_flux with the face states as two packed pairs
    __device__ static __forceinline__ Cell<float> interface_flux(const Cell<float> &UL, const Cell<float> &UR,
                                                                 const Cell<float> &sL, const Cell<float> &sR,
                                                                 const SweepConsts<float> &K)
    {
        const float2 hh = p2(K.h * 0.5f, K.h * 0.5f), mh = p2(-K.h * 0.5f, -K.h * 0.5f);
        const float2 l01 = fma2(p2(sL.rho, sL.p), hh, p2(UL.rho, UL.p));
        const float2 l23 = fma2(p2(sL.un, sL.ut), hh, p2(UL.un, UL.ut));
        const float2 r01 = fma2(p2(sR.rho, sR.p), mh, p2(UR.rho, UR.p));
        const float2 r23 = fma2(p2(sR.un, sR.ut), mh, p2(UR.un, UR.ut));
        const Cell<float> fL = {l01.x, l01.y, l23.x, l23.y}, fR = {r01.x, r01.y, r23.x, r23.y};
        const Interface<float> w = grp(fL, fR, sL, sR, K);
        const float hk = K.k * 0.5f;
        const float m = w.rho * w.un, m_t = w.rho * w.un_t + w.un * w.rho_t;
        const float es = w.e + 0.5f * (w.un * w.un + w.ut * w.ut);
        Cell<float> F;
        F.rho = m + hk * m_t;
        F.p = m * w.un + w.p + hk * (m_t * w.un + m * w.un_t + w.p_t);
        F.un = m * es + w.p * w.un + hk * (m_t * es + m * (w.e_t + w.un * w.un_t + w.ut * w.ut_t) + w.p_t * w.un + w.p * w.un_t);
        F.ut = m * w.ut + hk * (m_t * w.ut + m * w.ut_t);
        return F;
    }

    // HoistedCompensated::update with the conserved vector handled as the
    // pairs (rho, rho un), (E, rho ut) and the momenta as (rho un, rho ut)
    __device__ static __forceinline__ Cell<float> update(const Cell<float> &U, const Cell<float> &FL,
                                                         const Cell<float> &FR, const SweepConsts<float> &K)
    {
        const float2 uv = p2(U.un, U.ut), rr = p2(U.rho, U.rho);
        // (m1, m3) = rho (un, ut) and their errors; (ka, kb) = (m1 un, m3 ut)
        const float2 m13 = mul2(rr, uv);
        const float2 m13e = fma2(rr, uv, p2(-m13.x, -m13.y));
        const float2 kab = mul2(m13, uv);
        const float2 kabe = fma2(m13, uv, p2(-kab.x, -kab.y));
        float kin, kine;
        two_sum(kab.x, kab.y, kin, kine);
        const float2 kt = fma2(m13e, uv, kabe);
        kine += kt.x + kt.y;  // rho (un^2 + ut^2) = kin + kine
        float pe, pee, E, Ee;
        two_prod(U.p, K.igm1, pe, pee);
        pee = fmaf(U.p, K.igm1_lo, pee);  // p / (gamma - 1) = pe + pee
        two_sum(pe, 0.5f * kin, E, Ee);
        Ee += pee + 0.5f * kine;
        // W - lambda (F_R - F_L) on the pairs (rho, m1) and (E, m3)
        const float2 ml = p2(-K.lambda, -K.lambda);
        const float2 d01 = mul2(sub2(p2(FR.rho, FR.p), p2(FL.rho, FL.p)), ml);
        const float2 d23 = mul2(sub2(p2(FR.un, FR.ut), p2(FL.un, FL.ut)), ml);
        float2 s01, e01, s23, e23;
        two_sum2(p2(U.rho, m13.x), d01, s01, e01);
        two_sum2(p2(E, m13.y), d23, s23, e23);
        const float2 e13 = add2(p2(e01.y, e23.y), m13e);  // momenta errors
        const float e2 = e23.x + Ee;
        // primitives from (s + e)
        Cell<float> o;
        o.rho = s01.x + e01.x;
        const float ir = 1.0f / o.rho;
        const float2 s13 = p2(s01.y, s23.y), ir2 = p2(ir, ir);
        const float2 q = mul2(s13, ir2);
        const float2 uvn = fma2(add2(fma2(q, p2(-o.rho, -o.rho), s13), e13), ir2, q);
        o.un = uvn.x;
        o.ut = uvn.y;
        const float2 k = mul2(s13, uvn);
        const float2 ke = fma2(s13, uvn, p2(-k.x, -k.y));
        float k2, k2e;
        two_sum(k.x, k.y, k2, k2e);
        const float2 kt2 = fma2(e13, uvn, ke);
        k2e += kt2.x + kt2.y;  // m . u = k2 + k2e
        float d, de;
        two_sum(s23.x, -0.5f * k2, d, de);
        const float ei = d + (de + e2 - 0.5f * k2e);  // internal energy
        o.p = fmaf(K.gm1, ei, K.gm1_lo * ei);        // (gamma - 1) ei with the constant's low part
        return o;
    }
};

// The FP32 physics of the build with residual planes (FVM2D_FP32_RESIDUAL):
// slopes and fluxes from the FP32 values as PackedCompensated computes them;
// the conservative update of a cell from its stored hi + lo in FP64, with
// dt/h, 1/(gamma-1) and gamma-1 as hi + lo pairs, the result returned
// unrounded for the caller to split into the two planes.  (An FP64 update
// costs fewer instructions than the compensated FP32 one, and the FP64 pipe
// is otherwise idle in these sweeps.)
struct PackedResidual : PackedCompensated {
    static constexpr bool kSplitStorage = true;
    __device__ static __forceinline__ Cell<double> update_split(const Cell<float> &U, const Cell<float> &L,
                                                                const Cell<float> &FL, const Cell<float> &FR,
                                                                const SweepConsts<float> &K)
    {
        const double rho = double(U.rho) + double(L.rho), p = double(U.p) + double(L.p);
        const double un = double(U.un) + double(L.un), ut = double(U.ut) + double(L.ut);
        const double lam = double(K.lambda) + double(K.lambda_lo);
        const double igm1 = double(K.igm1) + double(K.igm1_lo), gm1 = double(K.gm1) + double(K.gm1_lo);
        double m0 = rho, m1 = rho * un, m3 = rho * ut;
        double m2 = fma(p, igm1, 0.5 * (m1 * un + m3 * ut));
        // W - lambda (F_R - F_L), the flux differences exact in FP64 (FP32
        // differences measured 1% faster, but across the jet's strong
        // gradients they doubled this build's distance from FP64)
        m0 = fma(double(FL.rho) - double(FR.rho), lam, m0);
        m1 = fma(double(FL.p) - double(FR.p), lam, m1);
        m2 = fma(double(FL.un) - double(FR.un), lam, m2);
        m3 = fma(double(FL.ut) - double(FR.ut), lam, m3);
        const double ir = rrcp(m0);
        Cell<double> o;
        o.rho = m0;
        o.un = m1 * ir;
        o.ut = m3 * ir;
        o.p = gm1 * (m2 - 0.5 * (m1 * o.un + m3 * o.ut));
        return o;
    }
};

} // namespace FVM2D_VARIANT
} // namespace fvm2d
