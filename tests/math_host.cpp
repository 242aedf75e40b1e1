// math_host.cpp -- the per-cell and per-interface arithmetic of the sweep
// kernels (2d_fvm_cuda_b200/csrc/fvm2d_math.cuh) compiled for the host with
// g++, so that the CPU tests can check the arithmetic policies against one
// another without a GPU: the shared-reciprocal forms (Hoisted,
// HoistedCompensated) against the reference-order form (RefOrder), in double
// and in single precision.  tests/test_math_host.py builds it and calls it
// through ctypes.
//
// The device code takes 1/sqrt(x) from CUDA's rsqrt/rsqrtf, which exist only
// in device code; here they are 1/sqrt(x) in the host's arithmetic.
#include <cmath>

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }

#define FVM2D_VARIANT host
#include "../2d_fvm_cuda_b200/csrc/fvm2d_math.cuh"

using namespace fvm2d::host;

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
    K.g = Real(g);
    K.k = Real(k);
    K.lambda = Real(k / h);
    K.igm1 = Real(1.0 / (g - 1.0));
    K.kappa = Real((g + 1.0) / 2.0);
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
        else
            return 1;
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
        else
            return 1;
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

} // namespace

// Every entry: `policy` 0 = RefOrder, 1 = Hoisted, 2 = HoistedCompensated
// (update only); `bits` 64 or 32 is the arithmetic (inputs rounded to it);
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

} // extern "C"
