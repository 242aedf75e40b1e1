// fvm2d_adjoint_math.cuh -- reverse-mode (adjoint) versions of the per-cell
// and per-interface arithmetic of one sweep, for the FP64 build with shared
// reciprocals (Hoisted in fvm2d_math.cuh).  Each function recomputes the
// forward values it needs and then applies the transposed Jacobian of the
// forward statements in reverse order.  Branches (limiter selection, wave
// cases, max(0, .)) follow the forward values, so the derivative is the one
// of the branch taken (almost everywhere).  dt is an input, not a variable:
// the time step is fixed while differentiating.
#pragma once

#include "fvm2d_math.cuh"

namespace fvm2d {
namespace FVM2D_VARIANT {

using A = double;

struct Cell5 {
    A rho, p, un, ut, e;
};

// ---- limiter -------------------------------------------------------------
// s = limited_slope(m, c, p): which difference was selected (0 none,
// 1 central, 2 backward, 3 forward), for the adjoint.  Same tests and tie
// order as limited_slope.
__device__ __forceinline__ int slope_choice(A m, A c, A p, A rh, A alpha)
{
    const A central = (p - m) * A(0.5) * rh;
    const A back = (c - m) * rh * alpha;
    const A fwd = (p - c) * rh * alpha;
    if (!(central * fwd > A(0) && back * fwd > A(0))) return 0;
    const A ac = fabs(central), ab = fabs(back), af = fabs(fwd);
    const A inner = (af < ab) ? af : ab;
    if (!(inner < ac)) return 1;
    return (af < ab) ? 3 : 2;
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
    const A ir = A(1) / n0;
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
    const A rho_l = UL.rho + sL.rho * K.h * half, pi_l = UL.p + sL.p * K.h * half;
    const A u_l = UL.un + sL.un * K.h * half, v_l = UL.ut + sL.ut * K.h * half;
    const A rho_r = UR.rho - sR.rho * K.h * half, pi_r = UR.p - sR.p * K.h * half;
    const A u_r = UR.un - sR.un * K.h * half, v_r = UR.ut - sR.ut * K.h * half;
    const A rho_lx = sL.rho, pi_lx = sL.p, u_lx = sL.un, v_lx = sL.ut;
    const A rho_rx = sR.rho, pi_rx = sR.p, u_rx = sR.un, v_rx = sR.ut;
    // ---- forward: Hoisted::grp ----
    const A irl = one / rho_l, irr = one / rho_r;
    const A e_l = pi_l * irl * igm1, e_r = pi_r * irr * igm1;
    const A X_l = pi_lx - pi_l * rho_lx * irl, X_r = pi_rx - pi_r * rho_rx * irr;
    const A e_lx = X_l * irl * igm1, e_rx = X_r * irr * igm1;
    const A a_l = sqrt(g * pi_l * irl), a_r = sqrt(g * pi_r * irr);
    const A il = one / (rho_l * a_l), ir = one / (rho_r * a_r);
    const A Y_l = pi_l * rho_lx + rho_l * pi_lx, Y_r = pi_r * rho_rx + rho_r * pi_rx;
    const A c_lx = half * g * Y_l * il, c_rx = half * g * Y_r * ir;
    const A du = u_l - u_r;
    const bool right_first = pi_r >= pi_l;
    A zl_arg, zr_arg, c_l, c_r, icl, icr;
    if (right_first) {
        zl_arg = (pi_r - pi_l) * ir + du;
        c_l = rho_l * (a_l + kappa * rmax(zero, zl_arg));
        icl = one / c_l;
        zr_arg = (pi_l - pi_r) * icl + du;
        c_r = rho_r * (a_r + kappa * rmax(zero, zr_arg));
        icr = one / c_r;
    } else {
        zr_arg = (pi_l - pi_r) * il + du;
        c_r = rho_r * (a_r + kappa * rmax(zero, zr_arg));
        icr = one / c_r;
        zl_arg = (pi_r - pi_l) * icr + du;
        c_l = rho_l * (a_l + kappa * rmax(zero, zl_arg));
        icl = one / c_l;
    }
    const A zl = rmax(zero, zl_arg), zr = rmax(zero, zr_arg);
    const A sl = c_l * irl, sr = c_r * irr;
    const int wave = (u_l - sl >= zero) ? 0 : ((u_r + sr <= zero) ? 1 : 2);  // left, right, star
    Cell5 W, Wt;
    // star-region intermediates (used only when wave == 2)
    A isum = 0, u = 0, pm = 0, k_l = 0, k_r = 0, H = 0, G = 0, d_l = 0, d_r = 0, Dp = 0;
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
        isum = one / (c_l + c_r);
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
            rho = one / irho;
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
            rho = one / irho;
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
    Cell5 Wb = {0, 0, 0, 0, 0}, Wtb = {0, 0, 0, 0, 0};
    {
        const A m = W.rho * W.un, mt = W.rho * Wt.un + W.un * Wt.rho;
        const A es = W.e + half * (W.un * W.un + W.ut * W.ut);
        const A q = Wt.e + W.un * Wt.un + W.ut * Wt.ut;
        A mb = 0, mtb = 0, esb = 0, qb = 0;
        // F.ut = m ut + hk (mt ut + m ut_t)
        mb += (W.ut + hk * Wt.ut) * Fb.ut;
        Wb.ut += (m + hk * mt) * Fb.ut;
        mtb += hk * W.ut * Fb.ut;
        Wtb.ut += hk * m * Fb.ut;
        // F.un (energy) = m es + p un + hk (mt es + m q + p_t un + p un_t)
        mb += (es + hk * q) * Fb.un;
        esb += (m + hk * mt) * Fb.un;
        Wb.p += (W.un + hk * Wt.un) * Fb.un;
        Wb.un += (W.p + hk * Wt.p) * Fb.un;
        mtb += hk * es * Fb.un;
        qb += hk * m * Fb.un;
        Wtb.p += hk * W.un * Fb.un;
        Wtb.un += hk * W.p * Fb.un;
        // q = e_t + un un_t + ut ut_t
        Wtb.e += qb;
        Wb.un += Wt.un * qb;
        Wtb.un += W.un * qb;
        Wb.ut += Wt.ut * qb;
        Wtb.ut += W.ut * qb;
        // F.p (normal momentum) = m un + p + hk (mt un + m un_t + p_t)
        mb += (W.un + hk * Wt.un) * Fb.p;
        Wb.un += (m + hk * mt) * Fb.p;
        Wb.p += Fb.p;
        mtb += hk * W.un * Fb.p;
        Wtb.un += hk * m * Fb.p;
        Wtb.p += hk * Fb.p;
        // F.rho (mass) = m + hk mt
        mb += Fb.rho;
        mtb += hk * Fb.rho;
        // es = e + (un^2 + ut^2)/2
        Wb.e += esb;
        Wb.un += W.un * esb;
        Wb.ut += W.ut * esb;
        // mt = rho un_t + un rho_t ; m = rho un
        Wb.rho += Wt.un * mtb + W.un * mb;
        Wtb.un += W.rho * mtb;
        Wb.un += Wt.rho * mtb + W.rho * mb;
        Wtb.rho += W.un * mtb;
    }
    // ---- reverse: Hoisted::grp ----
    A rho_lb = 0, pi_lb = 0, u_lb = 0, v_lb = 0, rho_rb = 0, pi_rb = 0, u_rb = 0, v_rb = 0;
    A rho_lxb = 0, pi_lxb = 0, u_lxb = 0, v_lxb = 0, rho_rxb = 0, pi_rxb = 0, u_rxb = 0, v_rxb = 0;
    A irlb = 0, irrb = 0, e_lb = 0, e_rb = 0, e_lxb = 0, e_rxb = 0, c_lxb = 0, c_rxb = 0;
    A c_lb = 0, c_rb = 0, iclb = 0, icrb = 0, slb = 0, srb = 0, dub = 0;
    if (wave == 0) {
        rho_lb += Wb.rho;
        pi_lb += Wb.p;
        u_lb += Wb.un;
        v_lb += Wb.ut;
        e_lb += Wb.e;
        // p_t = -u_l pi_lx - c_l sl u_lx
        u_lb += -pi_lx * Wtb.p;
        pi_lxb += -u_l * Wtb.p;
        c_lb += -sl * u_lx * Wtb.p;
        slb += -c_l * u_lx * Wtb.p;
        u_lxb += -c_l * sl * Wtb.p;
        // ut_t = -u_l v_lx
        u_lb += -v_lx * Wtb.ut;
        v_lxb += -u_l * Wtb.ut;
        // e_t = -u_l e_lx - pi_l irl u_lx
        u_lb += -e_lx * Wtb.e;
        e_lxb += -u_l * Wtb.e;
        pi_lb += -irl * u_lx * Wtb.e;
        irlb += -pi_l * u_lx * Wtb.e;
        u_lxb += -pi_l * irl * Wtb.e;
        // un_t = -u_l u_lx - pi_lx irl
        u_lb += -u_lx * Wtb.un;
        u_lxb += -u_l * Wtb.un;
        pi_lxb += -irl * Wtb.un;
        irlb += -pi_lx * Wtb.un;
        // rho_t = -rho_l u_lx - u_l rho_lx
        rho_lb += -u_lx * Wtb.rho;
        u_lxb += -rho_l * Wtb.rho;
        u_lb += -rho_lx * Wtb.rho;
        rho_lxb += -u_l * Wtb.rho;
    } else if (wave == 1) {
        rho_rb += Wb.rho;
        pi_rb += Wb.p;
        u_rb += Wb.un;
        v_rb += Wb.ut;
        e_rb += Wb.e;
        u_rb += -pi_rx * Wtb.p;
        pi_rxb += -u_r * Wtb.p;
        c_rb += -sr * u_rx * Wtb.p;
        srb += -c_r * u_rx * Wtb.p;
        u_rxb += -c_r * sr * Wtb.p;
        u_rb += -v_rx * Wtb.ut;
        v_rxb += -u_r * Wtb.ut;
        u_rb += -e_rx * Wtb.e;
        e_rxb += -u_r * Wtb.e;
        pi_rb += -irr * u_rx * Wtb.e;
        irrb += -pi_r * u_rx * Wtb.e;
        u_rxb += -pi_r * irr * Wtb.e;
        u_rb += -u_rx * Wtb.un;
        u_rxb += -u_r * Wtb.un;
        pi_rxb += -irr * Wtb.un;
        irrb += -pi_rx * Wtb.un;
        rho_rb += -u_rx * Wtb.rho;
        u_rxb += -rho_r * Wtb.rho;
        u_rb += -rho_rx * Wtb.rho;
        rho_rxb += -u_r * Wtb.rho;
    } else {
        A ub = Wb.un, pmb = Wb.p, rhob = Wb.rho, eb = Wb.e;
        A isumb = 0, k_lb = 0, k_rb = 0, Dpb = 0, urhob = 0, rho3b = 0, irhob = 0, ic2b = 0;
        A A1b = 0, B1b = 0, C1b = 0, Pb = 0, Vb = 0, Qb = 0, T1b = 0, T2b = 0;
        A p_tb = Wtb.p;
        if (star_right) {
            v_rb += Wb.ut;
            // ut_t = -urho irr v_rx
            urhob += -irr * v_rx * Wtb.ut;
            irrb += -urho * v_rx * Wtb.ut;
            v_rxb += -urho * irr * Wtb.ut;
            // e_t = -urho irr Q + pm ic2 p_t
            urhob += -irr * Q * Wtb.e;
            irrb += -urho * Q * Wtb.e;
            Qb += -urho * irr * Wtb.e;
            pmb += ic2 * Wt.p * Wtb.e;
            ic2b += pm * Wt.p * Wtb.e;
            p_tb += pm * ic2 * Wtb.e;
            // Q = e_rx - pi_r pi_rx ic2 + 2 (e_r - e) c_rx icr
            e_rxb += Qb;
            pi_rb += -pi_rx * ic2 * Qb;
            pi_rxb += -pi_r * ic2 * Qb;
            ic2b += -pi_r * pi_rx * Qb;
            e_rb += two * c_rx * icr * Qb;
            eb += -two * c_rx * icr * Qb;
            c_rxb += two * (e_r - W.e) * icr * Qb;
            icrb += two * (e_r - W.e) * c_rx * Qb;
            // un_t = isum (sl A1 k_l + sr B1 k_r)
            isumb += (sl * A1 * k_l + sr * B1 * k_r) * Wtb.un;
            slb += isum * A1 * k_l * Wtb.un;
            A1b += isum * sl * k_l * Wtb.un;
            k_lb += isum * sl * A1 * Wtb.un;
            srb += isum * B1 * k_r * Wtb.un;
            B1b += isum * sr * k_r * Wtb.un;
            k_rb += isum * sr * B1 * Wtb.un;
            // B1 = 1 - urho c_l ic2
            urhob += -c_l * ic2 * B1b;
            c_lb += -urho * ic2 * B1b;
            ic2b += -urho * c_l * B1b;
        } else {
            v_lb += Wb.ut;
            urhob += -irl * v_lx * Wtb.ut;
            irlb += -urho * v_lx * Wtb.ut;
            v_lxb += -urho * irl * Wtb.ut;
            urhob += -irl * Q * Wtb.e;
            irlb += -urho * Q * Wtb.e;
            Qb += -urho * irl * Wtb.e;
            pmb += ic2 * Wt.p * Wtb.e;
            ic2b += pm * Wt.p * Wtb.e;
            p_tb += pm * ic2 * Wtb.e;
            // Q = e_lx - pi_l pi_lx ic2 + 2 (e_l - e) c_lx icl
            e_lxb += Qb;
            pi_lb += -pi_lx * ic2 * Qb;
            pi_lxb += -pi_l * ic2 * Qb;
            ic2b += -pi_l * pi_lx * Qb;
            e_lb += two * c_lx * icl * Qb;
            eb += -two * c_lx * icl * Qb;
            c_lxb += two * (e_l - W.e) * icl * Qb;
            iclb += two * (e_l - W.e) * c_lx * Qb;
            // un_t = isum (sl B1 k_l + sr C1 k_r), B1 = 1 + urho c_r ic2
            isumb += (sl * B1 * k_l + sr * C1 * k_r) * Wtb.un;
            slb += isum * B1 * k_l * Wtb.un;
            B1b += isum * sl * k_l * Wtb.un;
            k_lb += isum * sl * B1 * Wtb.un;
            srb += isum * C1 * k_r * Wtb.un;
            C1b += isum * sr * k_r * Wtb.un;
            k_rb += isum * sr * C1 * Wtb.un;
            urhob += c_r * ic2 * B1b;
            c_rb += urho * ic2 * B1b;
            ic2b += urho * c_r * B1b;
        }
        // p_t = isum (c_r sl A1 k_l - c_l sr C1 k_r)   (both star cases)
        isumb += (c_r * sl * A1 * k_l - c_l * sr * C1 * k_r) * p_tb;
        c_rb += isum * sl * A1 * k_l * p_tb;
        slb += isum * c_r * A1 * k_l * p_tb;
        A1b += isum * c_r * sl * k_l * p_tb;
        k_lb += isum * c_r * sl * A1 * p_tb;
        c_lb += -isum * sr * C1 * k_r * p_tb;
        srb += -isum * c_l * C1 * k_r * p_tb;
        C1b += -isum * c_l * sr * k_r * p_tb;
        k_rb += -isum * c_l * sr * C1 * p_tb;
        // A1 = 1 + urho icr ; C1 = 1 - urho icl
        urhob += icr * A1b - icl * C1b;
        icrb += urho * A1b;
        iclb += -urho * C1b;
        if (star_right) {
            // rho_t = -u T1 P + T2 V Dp
            ub += -T1 * P * Wtb.rho;
            T1b += -u * P * Wtb.rho;
            Pb += -u * T1 * Wtb.rho;
            T2b += V * Dp * Wtb.rho;
            Vb += T2 * Dp * Wtb.rho;
            Dpb += T2 * V * Wtb.rho;
            // T1 = rho3 irr ic2 ; T2 = rho3 ic2 icr
            rho3b += irr * ic2 * T1b + ic2 * icr * T2b;
            irrb += rho3 * ic2 * T1b;
            ic2b += rho3 * irr * T1b + rho3 * icr * T2b;
            icrb += rho3 * ic2 * T2b;
            // P = sr^2 rho_rx - c_r u_rx + 1.5 (u - u_r) c_rx
            srb += two * sr * rho_rx * Pb;
            rho_rxb += sr * sr * Pb;
            c_rb += -u_rx * Pb;
            u_rxb += -c_r * Pb;
            ub += onehalf * c_rx * Pb;
            u_rb += -onehalf * c_rx * Pb;
            c_rxb += onehalf * (u - u_r) * Pb;
            // V = u + c_r irho
            ub += Vb;
            c_rb += irho * Vb;
            irhob += c_r * Vb;
        } else {
            // rho_t = -u T1 P - T2 V Dp
            ub += -T1 * P * Wtb.rho;
            T1b += -u * P * Wtb.rho;
            Pb += -u * T1 * Wtb.rho;
            T2b += -V * Dp * Wtb.rho;
            Vb += -T2 * Dp * Wtb.rho;
            Dpb += -T2 * V * Wtb.rho;
            // T1 = rho3 irl ic2 ; T2 = rho3 ic2 icl
            rho3b += irl * ic2 * T1b + ic2 * icl * T2b;
            irlb += rho3 * ic2 * T1b;
            ic2b += rho3 * irl * T1b + rho3 * icl * T2b;
            iclb += rho3 * ic2 * T2b;
            // P = sl^2 rho_lx + c_l u_lx + 1.5 (u - u_l) c_lx
            slb += two * sl * rho_lx * Pb;
            rho_lxb += sl * sl * Pb;
            c_lb += u_lx * Pb;
            u_lxb += c_l * Pb;
            ub += onehalf * c_lx * Pb;
            u_lb += -onehalf * c_lx * Pb;
            c_lxb += onehalf * (u - u_l) * Pb;
            // V = u - c_l irho
            ub += Vb;
            c_lb += -irho * Vb;
            irhob += -c_l * Vb;
        }
        // urho = u rho ; rho3 = rho^3
        ub += rho * urhob;
        rhob += u * urhob + A(3) * rho * rho * rho3b;
        if (star_right) {
            // e = e_r + (pm^2 - pi_r^2)/2 ic2
            e_rb += eb;
            pmb += pm * ic2 * eb;
            pi_rb += -pi_r * ic2 * eb;
            ic2b += half * (pm * pm - pi_r * pi_r) * eb;
            // ic2 = icr^2
            icrb += two * icr * ic2b;
            // rho = 1/irho ; irho = (u_r - u + sr) icr
            irhob += -rho * rho * rhob;
            u_rb += icr * irhob;
            ub += -icr * irhob;
            srb += icr * irhob;
            icrb += (u_r - u + sr) * irhob;
        } else {
            e_lb += eb;
            pmb += pm * ic2 * eb;
            pi_lb += -pi_l * ic2 * eb;
            ic2b += half * (pm * pm - pi_l * pi_l) * eb;
            iclb += two * icl * ic2b;
            // irho = (u - u_l + sl) icl
            irhob += -rho * rho * rhob;
            ub += icl * irhob;
            u_lb += -icl * irhob;
            slb += icl * irhob;
            iclb += (u - u_l + sl) * irhob;
        }
        // Dp = (c_r d_l - c_l d_r) isum / 2
        c_rb += d_l * half * isum * Dpb;
        c_lb += -d_r * half * isum * Dpb;
        A d_lb = c_r * half * isum * Dpb, d_rb = -c_l * half * isum * Dpb;
        isumb += (c_r * d_l - c_l * d_r) * half * Dpb;
        // d_r = sr G ; G = 2 (c_r u_rx - pi_rx) + u_r c_rx
        srb += G * d_rb;
        const A Gb = sr * d_rb;
        c_rb += two * u_rx * Gb;
        u_rxb += two * c_r * Gb;
        pi_rxb += -two * Gb;
        u_rb += c_rx * Gb;
        c_rxb += u_r * Gb;
        // d_l = sl H ; H = -2 (c_l u_lx + pi_lx) - u_l c_lx
        slb += H * d_lb;
        const A Hb = sl * d_lb;
        c_lb += -two * u_lx * Hb;
        u_lxb += -two * c_l * Hb;
        pi_lxb += -two * Hb;
        u_lb += -c_lx * Hb;
        c_lxb += -u_l * Hb;
        // k_r = -pi_rx + c_r u_rx + u_r c_rx / 2
        pi_rxb += -k_rb;
        c_rb += u_rx * k_rb;
        u_rxb += c_r * k_rb;
        u_rb += half * c_rx * k_rb;
        c_rxb += half * u_r * k_rb;
        // k_l = -pi_lx - c_l u_lx - u_l c_lx / 2
        pi_lxb += -k_lb;
        c_lb += -u_lx * k_lb;
        u_lxb += -c_l * k_lb;
        u_lb += -half * c_lx * k_lb;
        c_lxb += -half * u_l * k_lb;
        // pm = (du c_l c_r + c_l pi_r + c_r pi_l) isum
        dub += c_l * c_r * isum * pmb;
        c_lb += (du * c_r + pi_r) * isum * pmb;
        c_rb += (du * c_l + pi_l) * isum * pmb;
        pi_rb += c_l * isum * pmb;
        pi_lb += c_r * isum * pmb;
        isumb += (du * c_l * c_r + c_l * pi_r + c_r * pi_l) * pmb;
        // u = (u_l c_l + u_r c_r + pi_l - pi_r) isum
        u_lb += c_l * isum * ub;
        c_lb += u_l * isum * ub;
        u_rb += c_r * isum * ub;
        c_rb += u_r * isum * ub;
        pi_lb += isum * ub;
        pi_rb += -isum * ub;
        isumb += (u_l * c_l + u_r * c_r + pi_l - pi_r) * ub;
        // isum = 1/(c_l + c_r)
        const A sb = -isum * isum * isumb;
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
