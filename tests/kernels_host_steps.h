// kernels_host_steps.h -- whole sweeps, steps and sweep transposes composed
// from the library's device code, as its launchers compose them, for the
// host builds of the CPU tests.  Include after the device headers of one
// variant (FVM2D_VARIANT, FVM2D_REAL) and a using-directive for it.
#pragma once

#include <type_traits>
#include <vector>

namespace {

// Four planes of pitch nx for a (ny, nx) array.
template <typename R>
struct Planes {
    int nx = 0, ny = 0;
    long long plane = 0;
    std::vector<R> v;
    Planes() = default;
    Planes(int nx_, int ny_) : nx(nx_), ny(ny_), plane((long long)nx_ * ny_), v(4 * plane, R(0.0)) {}
    Field<R> field() { return Field<R>{v.data(), plane, nx}; }
};

template <typename R>
SweepArgs<R> sweep_args(Planes<R> &src, Planes<R> &dst, Planes<R> *flux, double h, double alpha, double gamma)
{
    SweepArgs<R> a;
    a.src = src.field();
    a.dst = dst.field();
    a.comb = a.dst;
    a.flux = flux ? flux->field() : Field<R>{nullptr, src.plane, src.nx};
    a.nx = src.nx;
    a.ny = src.ny;
    a.h = h;
    a.rh = 1.0 / h;
    a.alpha = alpha;
    a.gamma = gamma;
    a.ctl = nullptr;
    a.xchunks = 2;  // two chunks of 32 cells per x item: the chunk carry is exercised
    return a;
}

// x-sweep src -> dst through x_item on one emulated warp (FINAL: dst holds
// branch A and is averaged in place); TAPE stores the interface fluxes.
template <typename R, bool FINAL, bool TAPE, class Phys = Hoisted>
void x_sweep(Planes<R> &src, Planes<R> &dst, Planes<R> *flux, double h, double dt, double alpha, double gamma)
{
    const SweepArgs<R> a = sweep_args(src, dst, flux, h, alpha, gamma);
    const SweepConsts<R> K = sweep_consts(a, dt);
    const int nseg = fvm2d::x_items_per_row(a.nx, a.xchunks);
    const long long nwork = (long long)nseg * a.ny;
    emu::launch(dim3(1), dim3(32), true, [&] {
        double vmax = 0.0;
        int bad = 0;
        for (long long w = 0; w < nwork; ++w)
            x_item<R, Phys, FINAL>(a, K, int(w / nseg), int(w % nseg), nseg, int(threadIdx.x), vmax, bad);
    });
}

// y-sweep src -> dst through y_item, segments of T interfaces.
template <typename R, bool TAPE, class Phys = Hoisted>
void y_sweep(Planes<R> &src, Planes<R> &dst, Planes<R> *flux, double h, double dt, double alpha, double gamma, int T)
{
    const SweepArgs<R> a = sweep_args(src, dst, flux, h, alpha, gamma);
    const SweepConsts<R> K = sweep_consts(a, dt);
    const int ncw = (a.nx + 31) / 32, nseg = y_segments(a.ny, T);
    for (int seg = 0; seg < nseg; ++seg)
        for (int cw = 0; cw < ncw; ++cw)
            for (int lane = 0; lane < 32; ++lane) y_item<R, Phys>(a, K, seg, nseg, cw, lane, T);
}

// One split step U -> out of the shared-reciprocal build, in the kernels'
// order (X(U) -> A, Y(U) -> B, Y(A) -> out, X(B) averaged with out, ghost
// fill of out at t + dt); TAPE keeps A, B and the four sweeps' fluxes.
template <typename R, bool TAPE, class Phys = Hoisted>
void forward_step(Planes<R> &U, Planes<R> &A, Planes<R> &B, Planes<R> &out, Planes<R> *flux, int strategy, double t,
                  double dt, double hx, double hy, double alpha, double gamma, int T)
{
    x_sweep<R, false, TAPE, Phys>(U, A, TAPE ? &flux[0] : nullptr, hx, dt, alpha, gamma);
    y_sweep<R, TAPE, Phys>(U, B, TAPE ? &flux[1] : nullptr, hy, dt, alpha, gamma, T);
    y_sweep<R, TAPE, Phys>(A, out, TAPE ? &flux[2] : nullptr, hy, dt, alpha, gamma, T);
    x_sweep<R, true, TAPE, Phys>(B, out, TAPE ? &flux[3] : nullptr, hx, dt, alpha, gamma);
    GhostArgs<R> g;
    g.U = out.field();
    g.nx = U.nx;
    g.ny = U.ny;
    g.strategy = strategy;
    g.gamma = gamma;
    g.ctl = nullptr;
    g.plan = fvm2d::PlanParams{};
    g.row0 = 0;
    g.gny = U.ny;
    g.fill_top = g.fill_bottom = 1;
    for (int k = 0; k < 4 * U.nx + 4 * (U.ny - 4); ++k) ghost_cell(g, k, t + dt);
}

template <typename R>
void cells_to(Planes<R> &P, const double *cells, const double *tangent)
{
    for (long long c = 0; c < P.plane; ++c)
        for (int f = 0; f < 4; ++f) {
            if constexpr (std::is_same_v<R, Dual>)
                P.v[f * P.plane + c] = R(cells[4 * c + f], tangent[4 * c + f]);
            else
                P.v[f * P.plane + c] = R(cells[4 * c + f]);
        }
}

// The sweep transposes' constants, formed as the adjoint step's launcher
// forms them (the forward's sweep_consts: lambda = dt / h).
SweepConsts<A> adjoint_consts(double h, double dt, double alpha, double gamma)
{
    SweepConsts<A> K;
    K.h = h;
    K.rh = 1.0 / h;
    K.alpha = alpha;
    set_gamma_consts(K, gamma);
    K.k = dt;
    K.lambda = dt / h;
    K.lambda_lo = 0.0;
    return K;
}

// out = (d sweep_dir at U)^T ub (+ addend), with the grids the launcher uses
// (adjoint_x_kernel grid-strides, here one block of 128 threads).
void transpose(int dir, Planes<A> &U, Planes<A> &F, Planes<A> &ub, Planes<A> &out, Planes<A> *addend, double h,
               double dt, double alpha, double gamma)
{
    SweepT g;
    g.U = U.field();
    g.F = F.field();
    g.ub = ub.field();
    g.out = out.field();
    g.addend = addend ? addend->field() : Field<A>{nullptr, U.plane, U.nx};
    g.nx = U.nx;
    g.ny = U.ny;
    g.K = adjoint_consts(h, dt, alpha, gamma);
    if (dir == 0)
        emu::launch(dim3(1), dim3(ANT), true, [&] { adjoint_x_kernel(g); });
    else
        emu::launch(dim3((U.nx + kTileCols - 1) / kTileCols, (U.ny + kLineOut - 1) / kLineOut), dim3(ANT), true,
                    [&] { adjoint_y_kernel(g); });
}


} // namespace
