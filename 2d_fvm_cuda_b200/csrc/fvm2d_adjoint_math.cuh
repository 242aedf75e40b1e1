// fvm2d_adjoint_math.cuh -- reverse-mode (adjoint) versions of the per-cell
// and per-interface arithmetic of one sweep, for the builds with shared
// reciprocals (Hoisted in fvm2d_math.cuh), in the arithmetic type FVM2D_REAL.  Each function recomputes the
// forward values it needs and then applies the transposed Jacobian of the
// forward statements in reverse order.  Branches (limiter selection, wave
// cases, max(0, .)) follow the forward values, so the derivative is the one
// of the branch taken (almost everywhere).  dt is an input, not a variable:
// the time step is fixed while differentiating.
#pragma once

#include "fvm2d_math.cuh"

namespace fvm2d {
namespace FVM2D_VARIANT {

using A = FVM2D_REAL;

struct Cell5 {
    A rho, p, un, ut, e;
};

// ---- limiter -------------------------------------------------------------
// s = Hoisted::slope's limiter (limited_slope_hoisted) on (m, c, p): which
// difference was selected (0 none, 1 central, 2 backward, 3 forward), for the
// adjoint.  Same tests and tie order (d1 d2 > 0 alone: it implies dc d2 > 0).
__device__ __forceinline__ int slope_choice(A m, A c, A p, A rh, A alpha)
{
    const A d1 = c - m, d2 = p - c, dc = p - m;
    if (!(d1 * d2 > A(0))) return 0;
    const A a1 = fabs(d1), a2 = fabs(d2);
    const A inner = (rh * alpha) * ((a2 < a1) ? a2 : a1);
    if (!(inner < fabs(dc) * (rh * A(0.5)))) return 1;
    return (a2 < a1) ? 3 : 2;
}

// Adds the adjoint of one slope component (sbar) to its three cells.
__device__ __forceinline__ void slope_adjoint(int choice, A sbar, A rh, A alpha, A &mbar, A &cbar, A &pbar)
{
    if (choice == 1) {
        pbar += A(0.5) * rh * sbar;
        mbar -= A(0.5) * rh * sbar;
    } else if (choice == 2) {
        cbar += rh * alpha * sbar;
        mbar -= rh * alpha * sbar;
    } else if (choice == 3) {
        pbar += rh * alpha * sbar;
        cbar -= rh * alpha * sbar;
    }
}

// ---- conservative update ---------------------------------------------------
// Adjoint of Hoisted::update.  Given the output adjoint Ub (rho, p, un, ut),
// adds the adjoint of the input cell to Uin_b and returns the adjoint of the
// post-update conserved vector m' (slots mass, normal momentum, energy,
// tangential momentum); the flux adjoints are then +lambda mb' for F_L and
// -lambda mb' for F_R.
__device__ __forceinline__ Cell<A> update_adjoint(const Cell<A> &U, const Cell<A> &FL, const Cell<A> &FR,
                                                  const SweepConsts<A> &K, const Cell<A> &Ub, Cell<A> &Uin_b)
{
    const A half = A(0.5), gm1 = K.g - A(1);
    // forward
    const A m1 = U.rho * U.un, m3 = U.rho * U.ut;
    const A n0 = U.rho - (FR.rho - FL.rho) * K.lambda;
    const A n1 = m1 - (FR.p - FL.p) * K.lambda;
    const A n3 = m3 - (FR.ut - FL.ut) * K.lambda;
    const A ir = rrcp(n0);
    // reverse of the primitive recovery
    A n0b = Ub.rho, n1b = ir * Ub.un, n3b = ir * Ub.ut, n2b = gm1 * Ub.p;
    A irb = n1 * Ub.un + n3 * Ub.ut;
    n1b += -gm1 * n1 * ir * Ub.p;
    n3b += -gm1 * n3 * ir * Ub.p;
    irb += -gm1 * half * (n1 * n1 + n3 * n3) * Ub.p;
    n0b += -ir * ir * irb;
    // m' = m - lambda (F_R - F_L): dm = dm'
    // conserved from primitive
    Uin_b.rho += n0b + U.un * n1b + U.ut * n3b + half * (U.un * U.un + U.ut * U.ut) * n2b;
    Uin_b.un += U.rho * n1b + U.rho * U.un * n2b;
    Uin_b.ut += U.rho * n3b + U.rho * U.ut * n2b;
    Uin_b.p += K.igm1 * n2b;
    Cell<A> mb;
    mb.rho = n0b;
    mb.p = n1b;
    mb.un = n2b;
    mb.ut = n3b;
    return mb;
}

// ---- interface: face states, relaxation GRP, midpoint flux -------------------
// Adjoint of Hoisted::interface_flux(UL, UR, sL, sR): given the flux adjoint
// Fb (slots mass, normal momentum, energy, tangential momentum), adds the
// adjoints of the two cells and the two slopes.
__device__ __forceinline__ void interface_flux_adjoint(const Cell<A> &UL, const Cell<A> &UR, const Cell<A> &sL,
                                                       const Cell<A> &sR, const SweepConsts<A> &K, const Cell<A> &Fb,
                                                       Cell<A> &ULb, Cell<A> &URb, Cell<A> &sLb, Cell<A> &sRb)
{
    const A one = A(1), half = A(0.5), zero = A(0), two = A(2), onehalf = A(1.5);
    const A g = K.g, igm1 = K.igm1, kappa = K.kappa, hk = K.k * half, hh = K.h * half;
    // ---- forward: face states ----
    const A rho_l = fma(sL.rho, hh, UL.rho), pi_l = fma(sL.p, hh, UL.p);
    const A u_l = fma(sL.un, hh, UL.un), v_l = fma(sL.ut, hh, UL.ut);
    const A rho_r = fma(-sR.rho, hh, UR.rho), pi_r = fma(-sR.p, hh, UR.p);
    const A u_r = fma(-sR.un, hh, UR.un), v_r = fma(-sR.ut, hh, UR.ut);
    const A rho_lx = sL.rho, pi_lx = sL.p, u_lx = sL.un, v_lx = sL.ut;
    const A rho_rx = sR.rho, pi_rx = sR.p, u_rx = sR.un, v_rx = sR.ut;
    // ---- forward: Hoisted::grp, its reciprocals formed as it forms them
    // (the reverse below uses only what they are: irl = 1/rho_l,
    // il = 1/(rho_l a_l), a_l = sqrt(g pi_l / rho_l), icl = 1/c_l,
    // isum = 1/(c_l + c_r), and the same on the right) ----
    const A irlr = rrcp(rho_l * rho_r);
    const A irl = rho_r * irlr, irr = rho_l * irlr;
    const A e_l = pi_l * irl * igm1, e_r = pi_r * irr * igm1;
    const A X_l = pi_lx - pi_l * rho_lx * irl, X_r = pi_rx - pi_r * rho_rx * irr;
    const A e_lx = X_l * irl * igm1, e_rx = X_r * irr * igm1;
    const A il = rrsqrt(g * pi_l * rho_l), ir = rrsqrt(g * pi_r * rho_r);
    const A a_l = g * pi_l * il, a_r = g * pi_r * ir;
    const A Y_l = pi_l * rho_lx + rho_l * pi_lx, Y_r = pi_r * rho_rx + rho_r * pi_rx;
    const A c_lx = half * g * Y_l * il, c_rx = half * g * Y_r * ir;
    const A du = u_l - u_r;
    const bool right_first = pi_r >= pi_l;
    A zl_arg, zr_arg, c_l, c_r, icl, icr, isum;
    if (right_first) {
        zl_arg = (pi_r - pi_l) * ir + du;
        c_l = rho_l * (a_l + kappa * rmax(zero, zl_arg));
        icl = rrcp(c_l);
        zr_arg = (pi_l - pi_r) * icl + du;
        c_r = rho_r * (a_r + kappa * rmax(zero, zr_arg));
        const A sc = c_l + c_r, q = rrcp(c_r * sc);
        icr = sc * q;
        isum = c_r * q;
    } else {
        zr_arg = (pi_l - pi_r) * il + du;
        c_r = rho_r * (a_r + kappa * rmax(zero, zr_arg));
        icr = rrcp(c_r);
        zl_arg = (pi_r - pi_l) * icr + du;
        c_l = rho_l * (a_l + kappa * rmax(zero, zl_arg));
        const A sc = c_l + c_r, q = rrcp(c_l * sc);
        icl = sc * q;
        isum = c_l * q;
    }
    const A zl = rmax(zero, zl_arg), zr = rmax(zero, zr_arg);
    const A sl = c_l * irl, sr = c_r * irr;
    const int wave = (u_l - sl >= zero) ? 0 : ((u_r + sr <= zero) ? 1 : 2);  // left, right, star
    Cell5 W, Wt;
    // star-region intermediates (used only when wave == 2)
    A u = 0, pm = 0, k_l = 0, k_r = 0, H = 0, G = 0, d_l = 0, d_r = 0, Dp = 0;
    A irho = 0, rho = 0, ic2 = 0, rho3 = 0, urho = 0, A1 = 0, B1 = 0, C1 = 0, P = 0, V = 0, Q = 0, T1 = 0, T2 = 0;
    bool star_right = false;
    if (wave == 0) {
        W = {rho_l, pi_l, u_l, v_l, e_l};
        Wt.rho = -rho_l * u_lx - u_l * rho_lx;
        Wt.un = -u_l * u_lx - pi_lx * irl;
        Wt.e = -u_l * e_lx - pi_l * irl * u_lx;
        Wt.ut = -u_l * v_lx;
        Wt.p = -u_l * pi_lx - c_l * sl * u_lx;
    } else if (wave == 1) {
        W = {rho_r, pi_r, u_r, v_r, e_r};
        Wt.rho = -rho_r * u_rx - u_r * rho_rx;
        Wt.un = -u_r * u_rx - pi_rx * irr;
        Wt.e = -u_r * e_rx - pi_r * irr * u_rx;
        Wt.ut = -u_r * v_rx;
        Wt.p = -u_r * pi_rx - c_r * sr * u_rx;
    } else {
        u = (u_l * c_l + u_r * c_r + pi_l - pi_r) * isum;
        pm = (du * c_l * c_r + c_l * pi_r + c_r * pi_l) * isum;
        k_l = -pi_lx - c_l * u_lx - half * u_l * c_lx;
        k_r = -pi_rx + c_r * u_rx + half * u_r * c_rx;
        H = A(-2) * (c_l * u_lx + pi_lx) - u_l * c_lx;
        G = two * (c_r * u_rx - pi_rx) + u_r * c_rx;
        d_l = sl * H;
        d_r = sr * G;
        Dp = (c_r * d_l - c_l * d_r) * half * isum;
        star_right = u <= zero;
        if (star_right) {
            irho = (u_r - u + sr) * icr;
            rho = rrcp(irho);
            ic2 = icr * icr;
            const A e = e_r + (pm - pi_r) * (pm + pi_r) * half * ic2;
            rho3 = rho * rho * rho;
            urho = u * rho;
            P = sr * sr * rho_rx - c_r * u_rx + onehalf * (u - u_r) * c_rx;
            V = u + c_r * irho;
            T1 = rho3 * irr * ic2;
            T2 = rho3 * ic2 * icr;
            A1 = one + urho * icr;
            B1 = one - urho * c_l * ic2;
            C1 = one - urho * icl;
            Q = e_rx - pi_r * pi_rx * ic2 + two * (e_r - e) * c_rx * icr;
            W = {rho, pm, u, v_r, e};
            Wt.rho = -u * T1 * P + T2 * V * Dp;
            Wt.p = isum * (c_r * sl * A1 * k_l - c_l * sr * C1 * k_r);
            Wt.un = isum * (sl * A1 * k_l + sr * B1 * k_r);
            Wt.e = -urho * irr * Q + pm * ic2 * Wt.p;
            Wt.ut = -urho * irr * v_rx;
        } else {
            irho = (u - u_l + sl) * icl;
            rho = rrcp(irho);
            ic2 = icl * icl;
            const A e = e_l + (pm - pi_l) * (pm + pi_l) * half * ic2;
            rho3 = rho * rho * rho;
            urho = u * rho;
            P = sl * sl * rho_lx + c_l * u_lx + onehalf * (u - u_l) * c_lx;
            V = u - c_l * irho;
            T1 = rho3 * irl * ic2;
            T2 = rho3 * ic2 * icl;
            A1 = one + urho * icr;
            B1 = one + urho * c_r * ic2;  // the left case's factor of k_l in un_t
            C1 = one - urho * icl;
            Q = e_lx - pi_l * pi_lx * ic2 + two * (e_l - e) * c_lx * icl;
            W = {rho, pm, u, v_l, e};
            Wt.rho = -u * T1 * P - T2 * V * Dp;
            Wt.p = isum * (c_r * sl * A1 * k_l - c_l * sr * C1 * k_r);
            Wt.un = isum * (sl * B1 * k_l + sr * C1 * k_r);
            Wt.e = -urho * irl * Q + pm * ic2 * Wt.p;
            Wt.ut = -urho * irl * v_lx;
        }
    }
    // ---- reverse: midpoint flux ----
    // F.rho = m + hk mt; F.p = m un + p + hk (mt un + m un_t + p_t);
    // F.un (energy) = m es + p un + hk (mt es + m q + p_t un + p un_t);
    // F.ut = m ut + hk (mt ut + m ut_t), with m = rho un, mt = rho un_t + un rho_t,
    // es = e + (un^2 + ut^2)/2, q = e_t + un un_t + ut ut_t
    Cell5 Wb, Wtb;
    {
        const A m = W.rho * W.un, mt = W.rho * Wt.un + W.un * Wt.rho;
        const A es = W.e + half * (W.un * W.un + W.ut * W.ut);
        const A q = Wt.e + W.un * Wt.un + W.ut * Wt.ut;
        const A hr = hk * Fb.rho, hp = hk * Fb.p, he = hk * Fb.un, hu = hk * Fb.ut;
        const A mb = Fb.rho + W.un * Fb.p + Wt.un * hp + es * Fb.un + q * he + W.ut * Fb.ut + Wt.ut * hu;
        const A mtb = hr + W.un * hp + es * he + W.ut * hu;
        const A esb = m * Fb.un + mt * he, qb = m * he;
        Wb.rho = Wt.un * mtb + W.un * mb;
        Wb.p = Fb.p + W.un * Fb.un + Wt.un * he;
        Wb.un = m * Fb.p + mt * hp + W.p * Fb.un + Wt.p * he + Wt.un * qb + W.un * esb + Wt.rho * mtb + W.rho * mb;
        Wb.ut = m * Fb.ut + mt * hu + Wt.ut * qb + W.ut * esb;
        Wb.e = esb;
        Wtb.rho = W.un * mtb;
        Wtb.p = hp + W.un * he;
        Wtb.un = m * hp + W.p * he + W.un * qb + W.rho * mtb;
        Wtb.ut = m * hu + W.ut * qb;
        Wtb.e = qb;
    }
    // ---- reverse: Hoisted::grp ----
    A rho_lb = 0, pi_lb = 0, u_lb = 0, v_lb = 0, rho_rb = 0, pi_rb = 0, u_rb = 0, v_rb = 0;
    A rho_lxb = 0, pi_lxb = 0, u_lxb = 0, v_lxb = 0, rho_rxb = 0, pi_rxb = 0, u_rxb = 0, v_rxb = 0;
    A irlb = 0, irrb = 0, e_lb = 0, e_rb = 0, e_lxb = 0, e_rxb = 0, c_lxb = 0, c_rxb = 0;
    A c_lb = 0, c_rb = 0, iclb = 0, icrb = 0, slb = 0, srb = 0, dub = 0;
    if (wave == 0) {
        // W = left face state; Wt: rho_t = -rho_l u_lx - u_l rho_lx, un_t = -u_l u_lx - pi_lx irl,
        // e_t = -u_l e_lx - pi_l irl u_lx, ut_t = -u_l v_lx, p_t = -u_l pi_lx - c_l sl u_lx
        const A tp = -Wtb.p, te = -Wtb.e, tn = -Wtb.un, tr = -Wtb.rho;
        rho_lb += Wb.rho + u_lx * tr;
        pi_lb += Wb.p + irl * u_lx * te;
        u_lb += Wb.un + pi_lx * tp - v_lx * Wtb.ut + e_lx * te + u_lx * tn + rho_lx * tr;
        v_lb += Wb.ut;
        e_lb += Wb.e;
        pi_lxb += u_l * tp + irl * tn;
        c_lb += sl * u_lx * tp;
        slb += c_l * u_lx * tp;
        u_lxb += c_l * sl * tp + pi_l * irl * te + u_l * tn + rho_l * tr;
        v_lxb += -u_l * Wtb.ut;
        e_lxb += u_l * te;
        irlb += pi_l * u_lx * te + pi_lx * tn;
        rho_lxb += u_l * tr;
    } else if (wave == 1) {
        const A tp = -Wtb.p, te = -Wtb.e, tn = -Wtb.un, tr = -Wtb.rho;
        rho_rb += Wb.rho + u_rx * tr;
        pi_rb += Wb.p + irr * u_rx * te;
        u_rb += Wb.un + pi_rx * tp - v_rx * Wtb.ut + e_rx * te + u_rx * tn + rho_rx * tr;
        v_rb += Wb.ut;
        e_rb += Wb.e;
        pi_rxb += u_r * tp + irr * tn;
        c_rb += sr * u_rx * tp;
        srb += c_r * u_rx * tp;
        u_rxb += c_r * sr * tp + pi_r * irr * te + u_r * tn + rho_r * tr;
        v_rxb += -u_r * Wtb.ut;
        e_rxb += u_r * te;
        irrb += pi_r * u_rx * te + pi_rx * tn;
        rho_rxb += u_r * tr;
    } else {
        // The star state's side s (right if u <= 0, else left), written once for
        // both sides with sg = +1 (right) or -1 (left):
        //   irho = (sg (u_s - u) + s_s) ic_s, rho = 1/irho, ic2 = ic_s^2,
        //   e = e_s + (pm^2 - pi_s^2)/2 ic2, rho3 = rho^3, urho = u rho,
        //   P = s_s^2 rho_sx - sg c_s u_sx + 1.5 (u - u_s) c_sx, V = u + sg c_s irho,
        //   T1 = rho3 ir_s ic2, T2 = rho3 ic2 ic_s, Q = e_sx - pi_s pi_sx ic2 + 2 (e_s - e) c_sx ic_s,
        //   rho_t = -u T1 P + sg T2 V Dp, e_t = -urho ir_s Q + pm ic2 p_t, ut_t = -urho ir_s v_sx,
        //   p_t = isum (c_r sl A1 k_l - c_l sr C1 k_r), A1 = 1 + urho icr, C1 = 1 - urho icl,
        //   un_t = isum (sl a k_l + sr b k_r), with (a, b) = (A1, B1) on the right and (B1, C1)
        //   on the left, B1 = 1 - sg urho c_o ic2 (c_o the other side's c).
        const bool R = star_right;
        const A sg = R ? one : -one;
        const A u_s = R ? u_r : u_l, s_s = R ? sr : sl, ic_s = R ? icr : icl, ir_s = R ? irr : irl;
        const A c_s = R ? c_r : c_l, c_o = R ? c_l : c_r, pi_s = R ? pi_r : pi_l, pi_sx = R ? pi_rx : pi_lx;
        const A e_s = R ? e_r : e_l, c_sx = R ? c_rx : c_lx, rho_sx = R ? rho_rx : rho_lx;
        const A u_sx = R ? u_rx : u_lx, v_sx = R ? v_rx : v_lx;
        A ub = Wb.un, pmb = Wb.p, rhob = Wb.rho, eb = Wb.e, p_tb = Wtb.p, Dpb = 0;
        A k_lb = 0, k_rb = 0, urhob = 0, ic2b = 0, ir_sb = 0, ic_sb = 0, c_sb = 0, c_ob = 0;
        A u_sb = 0, s_sb = 0, pi_sb = 0, pi_sxb = 0, e_sb = 0, e_sxb = 0, c_sxb = 0, rho_sxb = 0, u_sxb = 0;
        const A v_sxb = -urho * ir_s * Wtb.ut;
        // ut_t and e_t
        const A tt = -(v_sx * Wtb.ut + Q * Wtb.e);
        urhob += ir_s * tt;
        ir_sb += urho * tt;
        const A Qb = -urho * ir_s * Wtb.e;
        const A cpe = Wt.p * Wtb.e;
        pmb += ic2 * cpe;
        ic2b += pm * cpe;
        p_tb += pm * ic2 * Wtb.e;
        // Q
        e_sxb += Qb;
        const A dq = -ic2 * Qb;
        pi_sb += pi_sx * dq;
        pi_sxb += pi_s * dq;
        ic2b += -pi_s * pi_sx * Qb;
        const A fq = two * c_sx * ic_s * Qb;
        e_sb += fq;
        eb -= fq;
        const A gq = two * (e_s - W.e) * Qb;
        c_sxb += ic_s * gq;
        ic_sb += c_sx * gq;
        // un_t
        const A iu = isum * Wtb.un;
        const A a = R ? A1 : B1, b = R ? B1 : C1;
        slb += a * k_l * iu;
        k_lb += sl * a * iu;
        srb += b * k_r * iu;
        k_rb += sr * b * iu;
        const A ab = sl * k_l * iu, bb = sr * k_r * iu;
        A A1b = R ? ab : A(0), C1b = R ? A(0) : bb;
        const A B1b = R ? bb : ab;
        const A hb = -sg * B1b;  // B1 = 1 - sg urho c_o ic2
        urhob += c_o * ic2 * hb;
        c_ob += urho * ic2 * hb;
        ic2b += urho * c_o * hb;
        // p_t
        const A ip = isum * p_tb;
        const A LL = c_r * sl, L2 = A1 * k_l, RR = c_l * sr, R2 = C1 * k_r;
        const A x1 = ip * L2, x2 = ip * LL, x3 = -ip * R2, x4 = -ip * RR;
        c_rb += sl * x1;
        slb += c_r * x1;
        A1b += k_l * x2;
        k_lb += A1 * x2;
        c_lb += sr * x3;
        srb += c_l * x3;
        C1b += k_r * x4;
        k_rb += C1 * x4;
        urhob += icr * A1b - icl * C1b;
        icrb += urho * A1b;
        iclb -= urho * C1b;
        // rho_t
        const A y1 = -Wtb.rho * T1, y2 = sg * Wtb.rho * T2;
        ub += P * y1;
        const A Pb = u * y1, Vb = Dp * y2;
        Dpb += V * y2;
        const A T1b = -u * P * Wtb.rho, T2b = sg * V * Dp * Wtb.rho;
        const A zt = ir_s * T1b + ic_s * T2b, w = rho3 * ic2;
        A rho3b = ic2 * zt;
        ic2b += rho3 * zt;
        ir_sb += w * T1b;
        ic_sb += w * T2b;
        // P
        s_sb += two * s_s * rho_sx * Pb;
        rho_sxb += s_s * s_s * Pb;
        c_sb += -sg * u_sx * Pb;
        u_sxb += -sg * c_s * Pb;
        const A kp = onehalf * c_sx * Pb;
        ub += kp;
        u_sb -= kp;
        c_sxb += onehalf * (u - u_s) * Pb;
        // V
        ub += Vb;
        c_sb += sg * irho * Vb;
        A irhob = sg * c_s * Vb;
        // urho, rho3
        ub += rho * urhob;
        rhob += u * urhob + A(3) * rho * rho * rho3b;
        // e, ic2
        e_sb += eb;
        pmb += pm * ic2 * eb;
        pi_sb -= pi_s * ic2 * eb;
        ic2b += half * (pm * pm - pi_s * pi_s) * eb;
        ic_sb += two * ic_s * ic2b;
        // rho = 1/irho, irho = (sg (u_s - u) + s_s) ic_s
        irhob -= rho * rho * rhob;
        const A vi = ic_s * irhob;
        u_sb += sg * vi;
        ub -= sg * vi;
        s_sb += vi;
        ic_sb += (sg * (u_s - u) + s_s) * irhob;
        // back to the two sides
        if (R) {
            v_rb += Wb.ut; v_rxb += v_sxb; u_rb += u_sb; srb += s_sb; icrb += ic_sb; irrb += ir_sb;
            c_rb += c_sb; c_lb += c_ob; pi_rb += pi_sb; pi_rxb += pi_sxb; e_rb += e_sb; e_rxb += e_sxb;
            c_rxb += c_sxb; rho_rxb += rho_sxb; u_rxb += u_sxb;
        } else {
            v_lb += Wb.ut; v_lxb += v_sxb; u_lb += u_sb; slb += s_sb; iclb += ic_sb; irlb += ir_sb;
            c_lb += c_sb; c_rb += c_ob; pi_lb += pi_sb; pi_lxb += pi_sxb; e_lb += e_sb; e_lxb += e_sxb;
            c_lxb += c_sxb; rho_lxb += rho_sxb; u_lxb += u_sxb;
        }
        // Dp = (c_r d_l - c_l d_r) isum / 2
        const A hD = half * isum * Dpb;
        c_rb += d_l * hD;
        c_lb -= d_r * hD;
        const A d_lb = c_r * hD, d_rb = -c_l * hD;
        // d_r = sr G ; G = 2 (c_r u_rx - pi_rx) + u_r c_rx
        srb += G * d_rb;
        const A Gb = sr * d_rb;
        c_rb += two * u_rx * Gb;
        u_rxb += two * c_r * Gb;
        pi_rxb -= two * Gb;
        u_rb += c_rx * Gb;
        c_rxb += u_r * Gb;
        // d_l = sl H ; H = -2 (c_l u_lx + pi_lx) - u_l c_lx
        slb += H * d_lb;
        const A Hb = sl * d_lb;
        c_lb -= two * u_lx * Hb;
        u_lxb -= two * c_l * Hb;
        pi_lxb -= two * Hb;
        u_lb -= c_lx * Hb;
        c_lxb -= u_l * Hb;
        // k_r = -pi_rx + c_r u_rx + u_r c_rx / 2 ; k_l = -pi_lx - c_l u_lx - u_l c_lx / 2
        pi_rxb -= k_rb;
        c_rb += u_rx * k_rb;
        u_rxb += c_r * k_rb;
        u_rb += half * c_rx * k_rb;
        c_rxb += half * u_r * k_rb;
        pi_lxb -= k_lb;
        c_lb -= u_lx * k_lb;
        u_lxb -= c_l * k_lb;
        u_lb -= half * c_lx * k_lb;
        c_lxb -= half * u_l * k_lb;
        // pm = (du c_l c_r + c_l pi_r + c_r pi_l) isum
        const A ipm = isum * pmb;
        dub += c_l * c_r * ipm;
        c_lb += (du * c_r + pi_r) * ipm;
        c_rb += (du * c_l + pi_l) * ipm;
        pi_rb += c_l * ipm;
        pi_lb += c_r * ipm;
        // u = (u_l c_l + u_r c_r + pi_l - pi_r) isum
        const A iub = isum * ub;
        u_lb += c_l * iub;
        c_lb += u_l * iub;
        u_rb += c_r * iub;
        c_rb += u_r * iub;
        pi_lb += iub;
        pi_rb -= iub;
        // isum = 1/(c_l + c_r): each quantity X = bracket isum above gives
        // bracket * Xb = X (c_l + c_r) Xb to isum's adjoint, and
        // d isum / d c = -isum^2, so c_l and c_r receive -isum sum(X Xb)
        const A sb = -isum * (u * ub + pm * pmb + Wt.p * p_tb + Wt.un * Wtb.un + Dp * Dpb);
        c_lb += sb;
        c_rb += sb;
    }
    // sl = c_l irl ; sr = c_r irr
    c_lb += irl * slb;
    irlb += c_l * slb;
    c_rb += irr * srb;
    irrb += c_r * srb;
    // relaxation speeds (the order of the forward branch, reversed)
    A a_lb = 0, a_rb = 0, ilb = 0, irb = 0;
    if (right_first) {
        c_rb += -icr * icr * icrb;
        rho_rb += (a_r + kappa * zr) * c_rb;
        a_rb += rho_r * c_rb;
        if (zr_arg > zero) {
            const A zb = rho_r * kappa * c_rb;
            pi_lb += icl * zb;
            pi_rb -= icl * zb;
            iclb += (pi_l - pi_r) * zb;
            dub += zb;
        }
        c_lb += -icl * icl * iclb;
        rho_lb += (a_l + kappa * zl) * c_lb;
        a_lb += rho_l * c_lb;
        if (zl_arg > zero) {
            const A zb = rho_l * kappa * c_lb;
            pi_rb += ir * zb;
            pi_lb -= ir * zb;
            irb += (pi_r - pi_l) * zb;
            dub += zb;
        }
    } else {
        c_lb += -icl * icl * iclb;
        rho_lb += (a_l + kappa * zl) * c_lb;
        a_lb += rho_l * c_lb;
        if (zl_arg > zero) {
            const A zb = rho_l * kappa * c_lb;
            pi_rb += icr * zb;
            pi_lb -= icr * zb;
            icrb += (pi_r - pi_l) * zb;
            dub += zb;
        }
        c_rb += -icr * icr * icrb;
        rho_rb += (a_r + kappa * zr) * c_rb;
        a_rb += rho_r * c_rb;
        if (zr_arg > zero) {
            const A zb = rho_r * kappa * c_rb;
            pi_lb += il * zb;
            pi_rb -= il * zb;
            ilb += (pi_l - pi_r) * zb;
            dub += zb;
        }
    }
    // du = u_l - u_r
    u_lb += dub;
    u_rb -= dub;
    // c_lx = g Y_l il / 2 ; Y_l = pi_l rho_lx + rho_l pi_lx  (and the right side)
    {
        const A Ylb = half * g * il * c_lxb, Yrb = half * g * ir * c_rxb;
        ilb += half * g * Y_l * c_lxb;
        irb += half * g * Y_r * c_rxb;
        pi_lb += rho_lx * Ylb;
        rho_lxb += pi_l * Ylb;
        rho_lb += pi_lx * Ylb;
        pi_lxb += rho_l * Ylb;
        pi_rb += rho_rx * Yrb;
        rho_rxb += pi_r * Yrb;
        rho_rb += pi_rx * Yrb;
        pi_rxb += rho_r * Yrb;
    }
    // il = 1/(rho_l a_l) ; ir = 1/(rho_r a_r)
    {
        const A Dl = -il * il * ilb, Dr = -ir * ir * irb;
        rho_lb += a_l * Dl;
        a_lb += rho_l * Dl;
        rho_rb += a_r * Dr;
        a_rb += rho_r * Dr;
    }
    // a = sqrt(g pi irho); 1/a = rho il
    {
        const A al = half * a_lb * rho_l * il, ar = half * a_rb * rho_r * ir;
        pi_lb += g * irl * al;
        irlb += g * pi_l * al;
        pi_rb += g * irr * ar;
        irrb += g * pi_r * ar;
    }
    // e_x = X irho igm1 ; X = pi_x - pi rho_x irho
    {
        const A Xlb = irl * igm1 * e_lxb, Xrb = irr * igm1 * e_rxb;
        irlb += X_l * igm1 * e_lxb;
        irrb += X_r * igm1 * e_rxb;
        pi_lxb += Xlb;
        pi_lb += -rho_lx * irl * Xlb;
        rho_lxb += -pi_l * irl * Xlb;
        irlb += -pi_l * rho_lx * Xlb;
        pi_rxb += Xrb;
        pi_rb += -rho_rx * irr * Xrb;
        rho_rxb += -pi_r * irr * Xrb;
        irrb += -pi_r * rho_rx * Xrb;
    }
    // e = pi irho igm1
    pi_lb += irl * igm1 * e_lb;
    irlb += pi_l * igm1 * e_lb;
    pi_rb += irr * igm1 * e_rb;
    irrb += pi_r * igm1 * e_rb;
    // irho = 1/rho
    rho_lb += -irl * irl * irlb;
    rho_rb += -irr * irr * irrb;
    // ---- reverse: face states ----
    ULb.rho += rho_lb;
    ULb.p += pi_lb;
    ULb.un += u_lb;
    ULb.ut += v_lb;
    URb.rho += rho_rb;
    URb.p += pi_rb;
    URb.un += u_rb;
    URb.ut += v_rb;
    sLb.rho += rho_lxb + hh * rho_lb;
    sLb.p += pi_lxb + hh * pi_lb;
    sLb.un += u_lxb + hh * u_lb;
    sLb.ut += v_lxb + hh * v_lb;
    sRb.rho += rho_rxb - hh * rho_rb;
    sRb.p += pi_rxb - hh * pi_rb;
    sRb.un += u_rxb - hh * u_rb;
    sRb.ut += v_rxb - hh * v_rb;
}

} // namespace FVM2D_VARIANT
} // namespace fvm2d
