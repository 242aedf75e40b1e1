// math_host.cpp -- the per-cell and per-interface arithmetic of the sweep
// kernels (2d_fvm_cuda_b200/csrc/fvm2d_math.cuh) compiled for the host with
// g++, so that the CPU tests can check the arithmetic policies against one
// another without a GPU: the shared-reciprocal forms (Hoisted,
// HoistedCompensated) against the reference-order form (RefOrder), in double
// and in single precision.  tests/test_math_host.py builds it and calls it
// through ctypes.
//
// It also holds the hand-written adjoint of the interface flux, the update
// and the limiter (csrc/fvm2d_adjoint_math.cuh) and a dual-number tangent of
// the forward (csrc/fvm2d_dual.cuh), for a per-interface dot-product test of
// the adjoint.
//
// The device code takes 1/sqrt(x) from CUDA's rsqrt/rsqrtf and the FP32 build
// its paired single-precision operations from sm_100's two-wide instructions,
// which exist only in device code; here they are 1/sqrt(x) and two
// correctly rounded scalar operations (what the two-wide instructions do
// lane by lane).  The dual type's warp shuffles are declared for the
// compiler and never called.
#include <cmath>

#include <cuda_runtime.h>

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
// correctly rounded products and sums that the compiler may not contract
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline float2 __fadd2_rn(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
static inline float2 __fmul2_rn(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
static inline float2 __ffma2_rn(float2 a, float2 b, float2 c)
{
    return make_float2(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y));
}
template <typename T>
static inline T __shfl_down_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_up_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_sync(unsigned, T v, int) { return v; }

#define FVM2D_VARIANT host
#define FVM2D_REAL double
#include "../2d_fvm_cuda_b200/csrc/fvm2d_adjoint_math.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_dual.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_packed.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_split.cuh"

// A number that counts the operations done on it, to state how many
// divisions and square roots each policy spends per interface.
namespace opcount {
struct Counts {
    // div2: divisions by the constant 2, which a compiler turns into products
    long add, mul, div, div2, sqrt, rsqrt, fma, cmp;
};
static Counts g_counts;
struct Num {
    double v;
    Num() : v(0.0) {}
    Num(double x) : v(x) {}
    explicit operator double() const { return v; }
};
inline Num operator+(Num a, Num b) { ++g_counts.add; return Num(a.v + b.v); }
inline Num operator-(Num a, Num b) { ++g_counts.add; return Num(a.v - b.v); }
inline Num operator-(Num a) { return Num(-a.v); }
inline Num operator*(Num a, Num b) { ++g_counts.mul; return Num(a.v * b.v); }
inline Num operator/(Num a, Num b)
{
    ++(b.v == 2.0 ? g_counts.div2 : g_counts.div);
    return Num(a.v / b.v);
}
inline Num &operator+=(Num &a, Num b) { return a = a + b; }
inline Num &operator-=(Num &a, Num b) { return a = a - b; }
inline bool operator<(Num a, Num b) { ++g_counts.cmp; return a.v < b.v; }
inline bool operator>(Num a, Num b) { ++g_counts.cmp; return a.v > b.v; }
inline bool operator<=(Num a, Num b) { ++g_counts.cmp; return a.v <= b.v; }
inline bool operator>=(Num a, Num b) { ++g_counts.cmp; return a.v >= b.v; }
inline Num sqrt(Num a) { ++g_counts.sqrt; return Num(std::sqrt(a.v)); }
inline Num rrsqrt(Num a) { ++g_counts.rsqrt; return Num(1.0 / std::sqrt(a.v)); }
inline Num fabs(Num a) { return Num(std::fabs(a.v)); }
inline Num fma(Num a, Num b, Num c) { ++g_counts.fma; return Num(std::fma(a.v, b.v, c.v)); }
} // namespace opcount

using namespace fvm2d::host;
using fvm2d::ad::Dual;

namespace {

template <typename Real>
Cell<Real> cell(const double *p)
{
    return Cell<Real>{Real(p[0]), Real(p[1]), Real(p[2]), Real(p[3])};
}

template <typename Real>
void put(const Cell<Real> &c, double *o)
{
    o[0] = double(c.rho);
    o[1] = double(c.p);
    o[2] = double(c.un);
    o[3] = double(c.ut);
}

// h, k, gamma, alpha -> the sweep constants as the kernels form them
template <typename Real>
SweepConsts<Real> consts(const double *k4)
{
    const double h = k4[0], k = k4[1], g = k4[2], alpha = k4[3];
    SweepConsts<Real> K;
    K.h = Real(h);
    K.rh = Real(1.0 / h);
    K.alpha = Real(alpha);
    set_gamma_consts(K, g);
    K.k = Real(k);
    K.lambda = Real(k / h);
    K.lambda_lo = Real(lo_part<Real>(k / h));
    return K;
}

template <typename Real>
void put_interface(const Interface<Real> &w, double *o)
{
    const Real v[10] = {w.rho, w.p, w.un, w.ut, w.e, w.rho_t, w.p_t, w.un_t, w.ut_t, w.e_t};
    for (int i = 0; i < 10; ++i) o[i] = double(v[i]);
}

template <typename Real>
int grp_n(int policy, long n, const double *in, const double *k4, double *out)
{
    const SweepConsts<Real> K = consts<Real>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 16 * i;
        const Cell<Real> L = cell<Real>(p), R = cell<Real>(p + 4), sL = cell<Real>(p + 8), sR = cell<Real>(p + 12);
        if (policy == 0)
            put_interface(relaxation_grp(L, R, sL, sR, K.g), out + 10 * i);
        else if (policy == 1)
            put_interface(Hoisted::grp(L, R, sL, sR, K), out + 10 * i);
        else
            return 1;
    }
    return 0;
}

template <typename Real>
int flux_n(int policy, long n, const double *in, const double *k4, double *out)
{
    const SweepConsts<Real> K = consts<Real>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 16 * i;
        const Cell<Real> UL = cell<Real>(p), UR = cell<Real>(p + 4), sL = cell<Real>(p + 8),
                         sR = cell<Real>(p + 12);
        if (policy == 0)
            put(RefOrder::interface_flux(UL, UR, sL, sR, K), out + 4 * i);
        else if (policy == 1)
            put(Hoisted::interface_flux(UL, UR, sL, sR, K), out + 4 * i);
        else if constexpr (sizeof(Real) == 4) {
            if (policy != 3) return 1;
            put(PackedCompensated::interface_flux(UL, UR, sL, sR, K), out + 4 * i);
        } else {
            return 1;
        }
    }
    return 0;
}

template <typename Real>
int update_n(int policy, long n, const double *in, const double *k4, double *out)
{
    const SweepConsts<Real> K = consts<Real>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i;
        const Cell<Real> U = cell<Real>(p), FL = cell<Real>(p + 4), FR = cell<Real>(p + 8);
        if (policy == 0)
            put(RefOrder::update(U, FL, FR, K), out + 4 * i);
        else if (policy == 1)
            put(Hoisted::update(U, FL, FR, K), out + 4 * i);
        else if (policy == 2)
            put(HoistedCompensated::update(U, FL, FR, K), out + 4 * i);
        else if constexpr (sizeof(Real) == 4) {
            if (policy != 3) return 1;
            put(PackedCompensated::update(U, FL, FR, K), out + 4 * i);
        } else {
            return 1;
        }
    }
    return 0;
}

template <typename Real>
int slope_n(int policy, long n, const double *in, const double *k4, double *out)
{
    const SweepConsts<Real> K = consts<Real>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i;
        const Cell<Real> m = cell<Real>(p), c = cell<Real>(p + 4), q = cell<Real>(p + 8);
        if (policy == 0)
            put(RefOrder::slope(m, c, q, K), out + 4 * i);
        else if (policy == 1)
            put(Hoisted::slope(m, c, q, K), out + 4 * i);
        else
            return 1;
    }
    return 0;
}

Cell<Dual> dual_cell(const double *p, const double *d)
{
    return Cell<Dual>{Dual(p[0], d[0]), Dual(p[1], d[1]), Dual(p[2], d[2]), Dual(p[3], d[3])};
}

void put_tangent(const Cell<Dual> &c, double *o)
{
    o[0] = c.rho.d;
    o[1] = c.p.d;
    o[2] = c.un.d;
    o[3] = c.ut.d;
}

} // namespace

// Every entry: `policy` 0 = RefOrder, 1 = Hoisted, 2 = HoistedCompensated
// (update only), 3 = PackedCompensated (flux and update, 32 bits only: the
// FP32 build's physics); `bits` 64 or 32 is the arithmetic (inputs rounded
// to it);
// k4 = (h, dt, gamma, alpha).  Returns 0, or 1 for an unknown policy/bits.
extern "C" {

// n interfaces from face states: in n x 16 (L, R, sL, sR as rho, p, un, ut);
// out n x 10 (rho, p, un, ut, e and their time derivatives).
int mh_grp(int policy, int bits, long n, const double *in, const double *k4, double *out)
{
    if (bits == 64) return grp_n<double>(policy, n, in, k4, out);
    if (bits == 32) return grp_n<float>(policy, n, in, k4, out);
    return 1;
}

// n interface fluxes from the two cells and their slopes: in n x 16 (UL, UR,
// sL, sR); out n x 4 (mass, normal momentum, energy, tangential momentum).
int mh_flux(int policy, int bits, long n, const double *in, const double *k4, double *out)
{
    if (bits == 64) return flux_n<double>(policy, n, in, k4, out);
    if (bits == 32) return flux_n<float>(policy, n, in, k4, out);
    return 1;
}

// n cell updates: in n x 12 (U, F_L, F_R); out n x 4 primitives.
int mh_update(int policy, int bits, long n, const double *in, const double *k4, double *out)
{
    if (bits == 64) return update_n<double>(policy, n, in, k4, out);
    if (bits == 32) return update_n<float>(policy, n, in, k4, out);
    return 1;
}

// n limited slopes: in n x 12 (left, centre, right cells); out n x 4.
int mh_slope(int policy, int bits, long n, const double *in, const double *k4, double *out)
{
    if (bits == 64) return slope_n<double>(policy, n, in, k4, out);
    if (bits == 32) return slope_n<float>(policy, n, in, k4, out);
    return 1;
}

// The limiter of one component, n triples (m, c, p) in `in` (n x 3), with
// hrh, rha in k2: out n x 2 = (the form the sweeps compile for the type --
// the double or float overload --, the generic template form).  bits 64 or
// 32.
int mh_limiter_forms(int bits, long n, const double *in, const double *k2, double *out)
{
    for (long i = 0; i < n; ++i) {
        const double *q = in + 3 * i;
        if (bits == 64) {
            out[2 * i] = limited_slope_hoisted(q[0], q[1], q[2], k2[0], k2[1]);
            out[2 * i + 1] = limited_slope_hoisted<double>(q[0], q[1], q[2], k2[0], k2[1]);
        } else if (bits == 32) {
            const float m = float(q[0]), c = float(q[1]), p = float(q[2]), a = float(k2[0]), b = float(k2[1]);
            out[2 * i] = limited_slope_hoisted(m, c, p, a, b);
            out[2 * i + 1] = limited_slope_hoisted<float>(m, c, p, a, b);
        } else {
            return 1;
        }
    }
    return 0;
}

// ---- derivatives (FP64, shared-reciprocal forms) ----------------------------
// Tangents (dual numbers through Hoisted) and adjoints (the hand-written
// reverse the VJP kernels run) of the same maps, one interface or cell per
// row.  dir / w are the tangent directions / output adjoints, in the layout
// of the inputs / outputs above.

// d flux: in, dir n x 16 -> out n x 4
int mh_flux_jvp(long n, const double *in, const double *dir, const double *k4, double *out)
{
    const SweepConsts<Dual> K = consts<Dual>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 16 * i, *d = dir + 16 * i;
        put_tangent(Hoisted::interface_flux(dual_cell(p, d), dual_cell(p + 4, d + 4), dual_cell(p + 8, d + 8),
                                            dual_cell(p + 12, d + 12), K),
                    out + 4 * i);
    }
    return 0;
}

// flux adjoint: in n x 16, w n x 4 -> out n x 16
int mh_flux_vjp(long n, const double *in, const double *w, const double *k4, double *out)
{
    const SweepConsts<double> K = consts<double>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 16 * i;
        Cell<double> b[4] = {};
        interface_flux_adjoint(cell<double>(p), cell<double>(p + 4), cell<double>(p + 8), cell<double>(p + 12), K,
                               cell<double>(w + 4 * i), b[0], b[1], b[2], b[3]);
        for (int q = 0; q < 4; ++q) put(b[q], out + 16 * i + 4 * q);
    }
    return 0;
}

// d update: in, dir n x 12 (U, F_L, F_R) -> out n x 4
int mh_update_jvp(long n, const double *in, const double *dir, const double *k4, double *out)
{
    const SweepConsts<Dual> K = consts<Dual>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i, *d = dir + 12 * i;
        put_tangent(Hoisted::update(dual_cell(p, d), dual_cell(p + 4, d + 4), dual_cell(p + 8, d + 8), K),
                    out + 4 * i);
    }
    return 0;
}

// update adjoint: in n x 12, w n x 4 -> out n x 12 (U, F_L, F_R); the flux
// adjoints are +lambda and -lambda times the conserved vector's adjoint
int mh_update_vjp(long n, const double *in, const double *w, const double *k4, double *out)
{
    const SweepConsts<double> K = consts<double>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i;
        double *o = out + 12 * i;
        Cell<double> Ub = {};
        const Cell<double> mb = update_adjoint(cell<double>(p), cell<double>(p + 4), cell<double>(p + 8), K,
                                               cell<double>(w + 4 * i), Ub);
        put(Ub, o);
        const Cell<double> fl = {K.lambda * mb.rho, K.lambda * mb.p, K.lambda * mb.un, K.lambda * mb.ut};
        put(fl, o + 4);
        const Cell<double> fr = {-fl.rho, -fl.p, -fl.un, -fl.ut};
        put(fr, o + 8);
    }
    return 0;
}

// d slopes: in, dir n x 12 (left, centre, right) -> out n x 4
int mh_slope_jvp(long n, const double *in, const double *dir, const double *k4, double *out)
{
    const SweepConsts<Dual> K = consts<Dual>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i, *d = dir + 12 * i;
        put_tangent(Hoisted::slope(dual_cell(p, d), dual_cell(p + 4, d + 4), dual_cell(p + 8, d + 8), K),
                    out + 4 * i);
    }
    return 0;
}

// slope adjoint: in n x 12, w n x 4 -> out n x 12
int mh_slope_vjp(long n, const double *in, const double *w, const double *k4, double *out)
{
    const SweepConsts<double> K = consts<double>(k4);
    for (long i = 0; i < n; ++i) {
        const double *p = in + 12 * i, *wi = w + 4 * i;
        double *o = out + 12 * i;
        for (int q = 0; q < 12; ++q) o[q] = 0.0;
        for (int f = 0; f < 4; ++f) {
            const int ch = slope_choice(p[f], p[4 + f], p[8 + f], K.rh, K.alpha);
            slope_adjoint(ch, wi[f], K.rh, K.alpha, o[f], o[4 + f], o[8 + f]);
        }
    }
    return 0;
}

// Operations of one evaluation for policy 0 = RefOrder or 1 = Hoisted:
// what = 0 the GRP alone (face states in, 16 doubles as for mh_grp), 1 the
// whole interface flux (cells and slopes in, as for mh_flux: face states,
// GRP, midpoint flux), 2 the four limited slopes of a cell (12 doubles as for
// mh_slope), 3 the conservative update (12 doubles as for mh_update; policy
// 2 = HoistedCompensated counts the compensated one).  counts: additions and subtractions,
// multiplications, divisions (by a variable), divisions by the constant 2,
// square roots, reciprocal square roots, fused multiply-adds, comparisons.  Constant operands formed once per sweep
// (SweepConsts) are not counted.
// The residual storage's split of each x (fvm2d_split.cuh): out[3k] = hi,
// out[3k+1] = the residual's value, out[3k+2] = 1 when splitting hi + lo
// again gives the same hi and lo bits.
int mh_split(long n, const double *x, double *out)
{
    for (long k = 0; k < n; ++k) {
        float hi, hi2;
        unsigned short lo, lo2;
        fvm2d::split_value(x[k], hi, lo);
        fvm2d::split_value(fvm2d::join_value(hi, lo), hi2, lo2);
        out[3 * k] = hi;
        out[3 * k + 1] = fvm2d::bf16_value(lo);
        out[3 * k + 2] = (memcmp(&hi, &hi2, 4) == 0 && lo == lo2) ? 1.0 : 0.0;
    }
    return 0;
}

int mh_count(int policy, int what, const double *in, const double *k4, long *counts)
{
    using opcount::Num;
    const Cell<Num> L = cell<Num>(in), R = cell<Num>(in + 4), sL = cell<Num>(in + 8), sR = cell<Num>(in + 12);
    const SweepConsts<Num> K = consts<Num>(k4);
    opcount::g_counts = {};
    if (policy == 0 && what == 0)
        relaxation_grp(L, R, sL, sR, K.g);
    else if (policy == 1 && what == 0)
        Hoisted::grp(L, R, sL, sR, K);
    else if (policy == 0 && what == 1)
        RefOrder::interface_flux(L, R, sL, sR, K);
    else if (policy == 1 && what == 1)
        Hoisted::interface_flux(L, R, sL, sR, K);
    else if (what == 2 && policy <= 1)
        policy == 0 ? RefOrder::slope(L, R, sL, K) : Hoisted::slope(L, R, sL, K);
    else if (what == 3 && policy == 0)
        RefOrder::update(L, R, sL, K);
    else if (what == 3 && policy == 1)
        Hoisted::update(L, R, sL, K);
    else if (what == 3 && policy == 2)
        HoistedCompensated::update(L, R, sL, K);
    else
        return 1;
    const opcount::Counts &c = opcount::g_counts;
    const long v[8] = {c.add, c.mul, c.div, c.div2, c.sqrt, c.rsqrt, c.fma, c.cmp};
    for (int i = 0; i < 8; ++i) counts[i] = v[i];
    return 0;
}

} // extern "C"
