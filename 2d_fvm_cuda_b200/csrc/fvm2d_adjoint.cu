// fvm2d_adjoint.cu -- reverse-mode (adjoint) step of the FP64 build with shared
// reciprocals, for fixed dt.
//
// The step is U' = ghost((Y(X(U)) + X(Y(U))) / 2).  Its adjoint, given the
// adjoint lb' of U', is
//   Vb = ghost^T lb'           (ring values are copies of interior cells)
//   A2b = B2b = Vb / 2
//   A1b = Y^T(A1) A2b ;  UbA = X^T(U) A1b      (branch A)
//   B1b = X^T(B1) B2b ;  UbB = Y^T(U) B1b      (branch B)
//   lb  = UbA + UbB
// with A1 = X(U) and B1 = Y(U) recomputed from U.  The transpose of a sweep
// runs as four gathers over the array, one thread per cell or interface of a
// line, so no value is accumulated by more than one thread:
//   1. interface fluxes F (forward)
//   2. per cell: adjoint of the conservative update -> the cell's direct part
//      and the adjoint mb of its post-update conserved vector
//   3. per interface: flux adjoint Fb = lambda (mb_right - mb_left), then the
//      adjoint of face states, relaxation GRP and midpoint flux -> adjoints of
//      the two cells and the two slopes it used
//   4. per cell: gather the direct part, the two interfaces' face-state parts
//      and the limiter adjoint of the three slopes that read the cell
// Only the ghost transpose adds with atomics (several ring cells may copy the
// same interior cell).
#define FVM2D_VARIANT adj
#include "fvm2d_adjoint_math.cuh"
#include "fvm2d_adjoint.h"
#include "fvm2d_kernels.cuh"

namespace fvm2d {
namespace adj {

using Phys = Hoisted;
constexpr int ANT = 256;

struct SweepGeom {
    int nx, ny, dir;  // dir 0: x-sweep; 1: y-sweep (line position l = ny-1-j, (un, ut) = (v, u))
    __device__ __forceinline__ int L() const { return dir == 0 ? nx : ny; }
    __device__ __forceinline__ int NC() const { return dir == 0 ? ny : nx; }
    __device__ __forceinline__ int x(int l, int c) const { return dir == 0 ? l : c; }
    __device__ __forceinline__ int y(int l, int c) const { return dir == 0 ? c : ny - 1 - l; }
    __device__ __forceinline__ int fn() const { return dir == 0 ? 2 : 3; }
    __device__ __forceinline__ int ft() const { return dir == 0 ? 3 : 2; }
};

// (l, c) of this thread: lines run along threadIdx.x for x-sweeps so that
// global accesses stay coalesced, across threadIdx.x for y-sweeps.
__device__ __forceinline__ bool thread_lc(const SweepGeom &G, int &l, int &c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    l = G.dir == 0 ? i : j;
    c = G.dir == 0 ? j : i;
    return l < G.L() && c < G.NC();
}

__device__ __forceinline__ Cell<A> ld(const Field<A> &F, const SweepGeom &G, int l, int c)
{
    return load_cell(F, G.x(l, c), G.y(l, c), G.fn(), G.ft());
}
__device__ __forceinline__ void st(const Field<A> &F, const SweepGeom &G, int l, int c, const Cell<A> &v)
{
    store_cell(F, G.x(l, c), G.y(l, c), G.fn(), G.ft(), v);
}
// flux-slot quantities (mass, normal momentum, energy, tangential momentum) are
// stored in plane order 0..3 without the u/v mapping
__device__ __forceinline__ Cell<A> ldf(const Field<A> &F, const SweepGeom &G, int l, int c)
{
    return load_cell(F, G.x(l, c), G.y(l, c), 2, 3);
}
__device__ __forceinline__ void stf(const Field<A> &F, const SweepGeom &G, int l, int c, const Cell<A> &v)
{
    store_cell(F, G.x(l, c), G.y(l, c), 2, 3, v);
}

__device__ __forceinline__ Cell<A> zero_cell() { return {0.0, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ Cell<A> add(const Cell<A> &a, const Cell<A> &b)
{
    return {a.rho + b.rho, a.p + b.p, a.un + b.un, a.ut + b.ut};
}

struct SweepParams {
    SweepGeom G;
    SweepConsts<A> K;
};

__device__ __forceinline__ Cell<A> slope_at(const Field<A> &U, const SweepParams &P, int l, int c)
{
    return cell_slope(ld(U, P.G, l - 1, c), ld(U, P.G, l, c), ld(U, P.G, l + 1, c), P.K);
}

// 1. interface fluxes: F(l) for the interface between cells l-1 and l
__global__ void __launch_bounds__(ANT) flux_kernel(Field<A> U, Field<A> F, SweepParams P)
{
    int l, c;
    if (!thread_lc(P.G, l, c) || l < 2 || l > P.G.L() - 2) return;
    const Cell<A> sm = slope_at(U, P, l - 1, c), s0 = slope_at(U, P, l, c);
    stf(F, P.G, l, c, Phys::interface_flux(ld(U, P.G, l - 1, c), ld(U, P.G, l, c), sm, s0, P.K));
}

// forward update of a sweep from the fluxes (recomputes A1 = X(U), B1 = Y(U))
__global__ void __launch_bounds__(ANT) update_kernel(Field<A> U, Field<A> F, Field<A> out, SweepParams P)
{
    int l, c;
    if (!thread_lc(P.G, l, c)) return;
    const Cell<A> u = ld(U, P.G, l, c);
    if (l >= 2 && l <= P.G.L() - 3)
        st(out, P.G, l, c, Phys::update(u, ldf(F, P.G, l, c), ldf(F, P.G, l + 1, c), P.K));
    else
        st(out, P.G, l, c, u);
}

// 2. per cell: adjoint of the update
__global__ void __launch_bounds__(ANT) update_adjoint_kernel(Field<A> U, Field<A> F, Field<A> Ub_out, Field<A> Up,
                                                             Field<A> Mb, SweepParams P)
{
    int l, c;
    if (!thread_lc(P.G, l, c)) return;
    const Cell<A> ub = ld(Ub_out, P.G, l, c);
    if (l >= 2 && l <= P.G.L() - 3) {
        Cell<A> part = zero_cell();
        const Cell<A> mb =
            update_adjoint(ld(U, P.G, l, c), ldf(F, P.G, l, c), ldf(F, P.G, l + 1, c), P.K, ub, part);
        st(Up, P.G, l, c, part);
        stf(Mb, P.G, l, c, mb);
    } else {  // pass-through cell
        st(Up, P.G, l, c, ub);
        stf(Mb, P.G, l, c, zero_cell());
    }
}

// 3. per interface: adjoint of face states, GRP and flux
__global__ void __launch_bounds__(ANT) interface_adjoint_kernel(Field<A> U, Field<A> Mb, Field<A> ULb, Field<A> URb,
                                                                Field<A> sLb, Field<A> sRb, SweepParams P)
{
    int l, c;
    if (!thread_lc(P.G, l, c) || l < 2 || l > P.G.L() - 2) return;
    const Cell<A> mr = ldf(Mb, P.G, l, c), ml = ldf(Mb, P.G, l - 1, c);
    const A lam = P.K.lambda;
    // the interface is F_L of cell l (+lambda) and F_R of cell l-1 (-lambda)
    const Cell<A> Fb = {lam * (mr.rho - ml.rho), lam * (mr.p - ml.p), lam * (mr.un - ml.un), lam * (mr.ut - ml.ut)};
    const Cell<A> sm = slope_at(U, P, l - 1, c), s0 = slope_at(U, P, l, c);
    Cell<A> a = zero_cell(), b = zero_cell(), sa = zero_cell(), sb = zero_cell();
    interface_flux_adjoint(ld(U, P.G, l - 1, c), ld(U, P.G, l, c), sm, s0, P.K, Fb, a, b, sa, sb);
    st(ULb, P.G, l, c, a);
    st(URb, P.G, l, c, b);
    st(sLb, P.G, l, c, sa);
    st(sRb, P.G, l, c, sb);
}

// 4. per cell: gather every contribution to the adjoint of the sweep input
__global__ void __launch_bounds__(ANT) gather_kernel(Field<A> U, Field<A> Up, Field<A> ULb, Field<A> URb,
                                                     Field<A> sLb, Field<A> sRb, Field<A> Ub_in, SweepParams P)
{
    int l, c;
    if (!thread_lc(P.G, l, c)) return;
    const int L = P.G.L();
    auto iface = [&](int j) { return j >= 2 && j <= L - 2; };
    Cell<A> r = ld(Up, P.G, l, c);
    if (iface(l)) r = add(r, ld(URb, P.G, l, c));          // right cell of interface l
    if (iface(l + 1)) r = add(r, ld(ULb, P.G, l + 1, c));  // left cell of interface l+1
    // slopes j = l-1, l, l+1 read this cell
    for (int j = l - 1; j <= l + 1; ++j) {
        if (j < 1 || j > L - 2) continue;
        Cell<A> sb = zero_cell();
        if (iface(j)) sb = add(sb, ld(sRb, P.G, j, c));          // slope j as the right slope of interface j
        if (iface(j + 1)) sb = add(sb, ld(sLb, P.G, j + 1, c));  // ... and the left slope of interface j+1
        const Cell<A> um = ld(U, P.G, j - 1, c), u0 = ld(U, P.G, j, c), up = ld(U, P.G, j + 1, c);
        const A um4[4] = {um.rho, um.p, um.un, um.ut}, u04[4] = {u0.rho, u0.p, u0.un, u0.ut};
        const A up4[4] = {up.rho, up.p, up.un, up.ut}, sb4[4] = {sb.rho, sb.p, sb.un, sb.ut};
        A out[4] = {0, 0, 0, 0};
        for (int f = 0; f < 4; ++f) {
            A mb = 0, cb = 0, pb = 0;
            slope_adjoint(slope_choice(um4[f], u04[f], up4[f], P.K.rh, P.K.alpha), sb4[f], P.K.rh, P.K.alpha, mb,
                          cb, pb);
            out[f] = (l == j - 1) ? mb : (l == j ? cb : pb);
        }
        r = add(r, Cell<A>{out[0], out[1], out[2], out[3]});
    }
    st(Ub_in, P.G, l, c, r);
}

// ---- ghost ring transpose ------------------------------------------------
// Interior source of ring cell (i, j) as the forward fill reads it (rows
// first, then columns; ghostCellPresets.cuh): returns false for a constant
// (inflow states), else (si, sj) and the sign applied to v.
__device__ __forceinline__ bool row_source(int strategy, int nx, int ny, int i, int j, int &si, int &sj, A &vs)
{
    si = i;
    vs = 1.0;
    switch (strategy) {
    case OUTFLOW:
    case JET:
        sj = j < 2 ? 2 : ny - 3;
        return true;
    case JET800:
        sj = j < 2 ? 2 : (j == ny - 2 ? ny - 3 : ny - 4);
        return true;
    case PERIODIC:
        sj = j == 0 ? ny - 4 : j == 1 ? ny - 3 : j == ny - 2 ? 2 : 3;
        return true;
    case REFLECTIVE_TB:
        sj = j == 0 ? 3 : j == 1 ? 2 : j == ny - 2 ? ny - 3 : ny - 4;
        vs = -1.0;
        return true;
    default:  // REFLECTIVE, DOUBLE_MACH
        if (j == 0 || j == 1) return false;
        if (j == ny - 1) {
            if (i <= nx / 24) sj = j - 2;
            else sj = j - 3, vs = -1.0;
            return true;
        }
        sj = j - 1;
        if (i > nx / 24) vs = -1.0;
        return true;
    }
}

__device__ __forceinline__ bool ring_source(int strategy, int nx, int ny, int i, int j, int &si, int &sj, A &vs)
{
    const bool gcol = i < 2 || i >= nx - 2, grow = j < 2 || j >= ny - 2;
    if (!gcol) return row_source(strategy, nx, ny, i, j, si, sj, vs);
    int ci;
    const bool left = i < 2;
    switch (strategy) {
    case OUTFLOW:
    case REFLECTIVE_TB:
        ci = left ? 2 : nx - 3;
        break;
    case JET:
    case JET800:
        if (left) return false;
        ci = nx - 3;
        break;
    case PERIODIC:
        ci = i == 0 ? nx - 4 : i == 1 ? nx - 3 : i == nx - 2 ? 2 : 3;
        break;
    default:
        return false;
    }
    if (grow) return row_source(strategy, nx, ny, ci, j, si, sj, vs);
    si = ci;
    sj = j;
    vs = 1.0;
    return true;
}

struct GhostGeom {
    int nx, ny, strategy;
};

__device__ __forceinline__ bool on_ring(const GhostGeom &g, int i, int j)
{
    return i < 2 || i >= g.nx - 2 || j < 2 || j >= g.ny - 2;
}

// Vb = lb with the ring zeroed
__global__ void ghost_adjoint_copy(Field<A> lb, Field<A> Vb, GhostGeom g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const bool ring = on_ring(g, i, j);
    for (int f = 0; f < 4; ++f) Vb.at(f, i, j) = ring ? 0.0 : lb.at(f, i, j);
}

// Vb(source) += sign * lb(ring cell)
__global__ void ghost_adjoint_scatter(Field<A> lb, Field<A> Vb, GhostGeom g)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nrow = 4 * g.nx, ncol = 4 * (g.ny - 4);
    if (k >= nrow + ncol) return;
    int i, j;
    if (k < nrow) {
        const int r = k / g.nx;
        i = k % g.nx;
        j = r < 2 ? r : g.ny - 4 + r;
    } else {
        const int q = k - nrow, r = q / (g.ny - 4);
        j = 2 + q % (g.ny - 4);
        i = r < 2 ? r : g.nx - 4 + r;
    }
    int si, sj;
    A vs;
    if (!ring_source(g.strategy, g.nx, g.ny, i, j, si, sj, vs)) return;
    atomicAdd(&Vb.at(0, si, sj), lb.at(0, i, j));
    atomicAdd(&Vb.at(1, si, sj), lb.at(1, i, j));
    atomicAdd(&Vb.at(2, si, sj), lb.at(2, i, j));
    atomicAdd(&Vb.at(3, si, sj), vs * lb.at(3, i, j));
}

// out = a * x + b * y over the 4 planes
__global__ void axpby_kernel(Field<A> x, Field<A> y, Field<A> out, A a, A b, int nx, int ny)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    for (int f = 0; f < 4; ++f) out.at(f, i, j) = a * x.at(f, i, j) + b * y.at(f, i, j);
}

} // namespace adj

// ---- host entry --------------------------------------------------------------
namespace {

using adj::A;

adj::SweepParams sweep_params(const AdjointLaunch &L, int dir)
{
    adj::SweepParams P;
    P.G.nx = L.nx;
    P.G.ny = L.ny;
    P.G.dir = dir;
    const double h = dir == 0 ? L.hx : L.hy;
    P.K.h = h;
    P.K.rh = dir == 0 ? L.rhx : L.rhy;
    P.K.alpha = L.alpha;
    P.K.g = L.gamma;
    P.K.k = L.dt;
    P.K.lambda = L.dt / h;
    P.K.igm1 = 1.0 / (L.gamma - 1.0);
    P.K.kappa = (L.gamma + 1.0) / 2.0;
    return P;
}

adj::Field<A> fld(double *p, const AdjointLaunch &L)
{
    adj::Field<A> f;
    f.base = p;
    f.plane = L.plane;
    f.pitch = L.pitch;
    return f;
}

dim3 sweep_grid(const AdjointLaunch &L, int dir)
{
    const int L_ = dir == 0 ? L.nx : L.ny, NC = dir == 0 ? L.ny : L.nx;
    // x-sweeps: lines along threadIdx.x; y-sweeps: cross index along threadIdx.x
    return dir == 0 ? dim3((L_ + 31) / 32, (NC + 7) / 8) : dim3((NC + 31) / 32, (L_ + 7) / 8);
}

// out = sweep_dir(U)
void forward_sweep(const AdjointLaunch &L, int dir, double *U, double *out, cudaStream_t s)
{
    const adj::SweepParams P = sweep_params(L, dir);
    const dim3 g = sweep_grid(L, dir), b(32, 8);
    adj::flux_kernel<<<g, b, 0, s>>>(fld(U, L), fld(L.work[0], L), P);
    adj::update_kernel<<<g, b, 0, s>>>(fld(U, L), fld(L.work[0], L), fld(out, L), P);
}

// Ub_in = (d sweep_dir / dU at U)^T Ub_out
void adjoint_sweep(const AdjointLaunch &L, int dir, double *U, double *Ub_out, double *Ub_in, cudaStream_t s)
{
    const adj::SweepParams P = sweep_params(L, dir);
    const dim3 g = sweep_grid(L, dir), b(32, 8);
    double *F = L.work[0], *Up = L.work[1], *Mb = L.work[2];
    double *ULb = L.work[3], *URb = L.work[4], *sLb = L.work[5], *sRb = L.work[6];
    adj::flux_kernel<<<g, b, 0, s>>>(fld(U, L), fld(F, L), P);
    adj::update_adjoint_kernel<<<g, b, 0, s>>>(fld(U, L), fld(F, L), fld(Ub_out, L), fld(Up, L), fld(Mb, L), P);
    adj::interface_adjoint_kernel<<<g, b, 0, s>>>(fld(U, L), fld(Mb, L), fld(ULb, L), fld(URb, L), fld(sLb, L),
                                                  fld(sRb, L), P);
    adj::gather_kernel<<<g, b, 0, s>>>(fld(U, L), fld(Up, L), fld(ULb, L), fld(URb, L), fld(sLb, L), fld(sRb, L),
                                       fld(Ub_in, L), P);
}

} // namespace

cudaError_t adjoint_step(const AdjointLaunch &L, cudaStream_t s)
{
    const dim3 g2((L.nx + 31) / 32, (L.ny + 7) / 8), b2(32, 8);
    adj::GhostGeom gg{L.nx, L.ny, L.strategy};
    double *A1 = L.state[0], *B1 = L.state[1], *H = L.state[2], *T1 = L.state[3], *T2 = L.state[4],
           *T3 = L.state[5];
    // recompute the first sweeps of both branches
    forward_sweep(L, 0, L.U, A1, s);
    forward_sweep(L, 1, L.U, B1, s);
    // ghost fill and average, transposed: H = ghost^T(lb_out) / 2
    adj::ghost_adjoint_copy<<<g2, b2, 0, s>>>(fld(L.lb_out, L), fld(H, L), gg);
    const int ring = 4 * L.nx + 4 * (L.ny - 4);
    adj::ghost_adjoint_scatter<<<(ring + 255) / 256, 256, 0, s>>>(fld(L.lb_out, L), fld(H, L), gg);
    adj::axpby_kernel<<<g2, b2, 0, s>>>(fld(H, L), fld(H, L), fld(H, L), 0.5, 0.0, L.nx, L.ny);
    // branch A: A2 = Y(A1), A1 = X(U)
    adjoint_sweep(L, 1, A1, H, T1, s);
    adjoint_sweep(L, 0, L.U, T1, T2, s);
    // branch B: B2 = X(B1), B1 = Y(U)
    adjoint_sweep(L, 0, B1, H, T1, s);
    adjoint_sweep(L, 1, L.U, T1, T3, s);
    adj::axpby_kernel<<<g2, b2, 0, s>>>(fld(T2, L), fld(T3, L), fld(L.lb_in, L), 1.0, 1.0, L.nx, L.ny);
    return cudaGetLastError();
}

} // namespace fvm2d
