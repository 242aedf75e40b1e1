// kernels_host.cpp -- the device code of the step's kernels compiled for the
// host with g++ from 2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh and
// fvm2d_adjoint.inc, so that the CPU tests can compare it with the oracle
// and with itself without a GPU: the ghost-ring rules (ghost_cell), the
// step-size plan (plan_step), the wave speed, the sweep work items (x_item,
// y_item) with the kernels' item numbering, whole solves through the
// single-problem kernels, the frame renderer and PNG writer, the batched kernels
// (fvm2d_batch.cuh) over several problems, and the adjoint step's kernels
// (adjoint_x_kernel, adjoint_y_kernel, the ghost transposes) against a
// dual-number tangent of the forward items.  tests/test_kernels_host.py
// builds it and calls it through ctypes.
//
// The CUDA built-ins are emulated on the host by cuda_host_emu.h; the sweeps,
// steps and transposes are composed in kernels_host_steps.h.
#include "cuda_host_emu.h"

#define FVM2D_VARIANT host
#define FVM2D_REAL double
#include "../2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_dual.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_adjoint.inc"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_packed.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_batch.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_io.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_transfer.cuh"

using namespace fvm2d::host;
using fvm2d::ad::Dual;

#include "kernels_host_steps.h"

// chunks of 32 cells per x-sweep item used by the functions below
static int g_xchunks = 2;
extern "C" int kh_set_xchunks(int c)
{
    if (c < 1) return 1;
    g_xchunks = c;
    return 0;
}

using fvm2d::PlanParams;
using fvm2d::StepControl;

extern "C" {

// The ghost fill of ghost_kernel on a (ny, nx, 4) array of (rho, p, u, v)
// cells, in place: every ring cell from ghost_cell at time t in the row frame
// (row0, gny, fill_top, fill_bottom).  *vmax: the ring cells' largest wave
// speed, as the kernel folds it into the step's maximum.
int kh_ghost(double *cells, int nx, int ny, int strategy, double gamma, double t, int row0, int gny, int fill_top,
             int fill_bottom, double *vmax)
{
    if (nx < 6 || ny < 6) return 1;
    const long long plane = (long long)nx * ny;
    std::vector<double> P(4 * plane);
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) P[f * plane + c] = cells[4 * c + f];
    GhostArgs<double> a;
    a.U.base = P.data();
    a.U.plane = plane;
    a.U.pitch = nx;
    a.nx = nx;
    a.ny = ny;
    a.strategy = strategy;
    a.gamma = gamma;
    a.ctl = nullptr;
    a.plan = PlanParams{};
    a.row0 = row0;
    a.gny = gny;
    a.fill_top = fill_top;
    a.fill_bottom = fill_bottom;
    double m = 0.0;
    for (int k = 0; k < 4 * nx + 4 * (ny - 4); ++k) m = std::fmax(m, ghost_cell(a, k, t));
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) cells[4 * c + f] = P[f * plane + c];
    *vmax = m;
    return 0;
}

// plan_step on a control record with committed time t, wave-speed max smax,
// `steps` of `step_limit` and the done flag.  out: dt, active, done.
int kh_plan(double t, double smax, int steps, int step_limit, int done, double t_end, double cfl, double hmin,
            double fixed_dt, double *dt, int *active, int *done_out)
{
    StepControl c{};
    c.t = t;
    c.smax_last = smax;
    c.steps = steps;
    c.step_limit = step_limit;
    c.done = done;
    c.dt = -1.0;
    PlanParams p{t_end, cfl, hmin, fixed_dt};
    plan_step(&c, p);
    *dt = c.dt;
    *active = c.active;
    *done_out = c.done;
    return 0;
}

// Wave speed |(u, v)| + sqrt(gamma p / rho) of n cells (n x 4).
int kh_wave_speed(long n, const double *cells, double gamma, double *out)
{
    for (long i = 0; i < n; ++i) {
        const double *c = cells + 4 * i;
        out[i] = wave_speed(c[0], c[1], c[2], c[3], gamma);
    }
    return 0;
}

// One sweep of a (ny, nx, 4) state through the kernels' work items: dir 0
// runs x_item over every (row, 30-cell segment) item with a 32-thread warp,
// dir 1 runs y_item over every (32-column, T-interface segment) item, lane by
// lane (y items exchange nothing).  final (x only): the final sweep, which
// averages with `comb` (branch A) in place, as the kernel does: `out` starts
// as `comb` and is both read and written.  policy 0 = RefOrder, 1 = Hoisted.
// Cells the items do not write are left NaN in `out` (or `comb`'s values).
int kh_sweep(int policy, int dir, int final, int T, const double *in, const double *comb, double *out, int nx,
             int ny, double h, double dt, double alpha, double gamma)
{
    if (nx < 6 || ny < 6 || (dir == 1 && T < 3) || (final && dir != 0)) return 1;
    const long long plane = (long long)nx * ny;
    if (final && !comb) return 1;
    std::vector<double> S(4 * plane), D(4 * plane, NAN);
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) {
            S[f * plane + c] = in[4 * c + f];
            if (final) D[f * plane + c] = comb[4 * c + f];
        }
    SweepArgs<double> a;
    a.src = Field<double>{S.data(), plane, nx};
    a.dst = Field<double>{D.data(), plane, nx};
    a.comb = a.dst;
    a.flux = Field<double>{nullptr, plane, nx};
    a.xchunks = g_xchunks;
    a.nx = nx;
    a.ny = ny;
    a.h = h;
    a.rh = 1.0 / h;
    a.alpha = alpha;
    a.gamma = gamma;
    a.ctl = nullptr;
    const SweepConsts<double> K = sweep_consts(a, dt);
    if (dir == 0) {
        const int nseg = fvm2d::x_items_per_row(nx, a.xchunks);
        const long long nwork = (long long)nseg * ny;
        emu::launch(dim3(1), dim3(32), true, [&] {
            const int lane = int(threadIdx.x);
            double vmax = 0.0;
            int bad = 0;
            for (long long w = 0; w < nwork; ++w) {
                const int y = int(w / nseg), seg = int(w % nseg);
                static double xring[kXRingChunks * 128];  // one warp's ring
                if (policy == 3 && final)
                    x_item<double, RefOrder, true, 4>(a, K, y, seg, nseg, lane, vmax, bad, xring);
                else if (policy == 3)
                    x_item<double, RefOrder, false, 4>(a, K, y, seg, nseg, lane, vmax, bad, xring);
                else if (policy == 0 && final)
                    x_item<double, RefOrder, true>(a, K, y, seg, nseg, lane, vmax, bad);
                else if (policy == 0)
                    x_item<double, RefOrder, false>(a, K, y, seg, nseg, lane, vmax, bad);
                else if (final)
                    x_item<double, Hoisted, true>(a, K, y, seg, nseg, lane, vmax, bad);
                else
                    x_item<double, Hoisted, false>(a, K, y, seg, nseg, lane, vmax, bad);
            }
        });
    } else {
        const int ncw = (nx + 31) / 32, nseg = y_segments(ny, T);
        // policy 2: RefOrder items that stream their columns through the
        // shared-memory ring (one ring per lane, as per thread on the GPU)
        std::vector<double> ring(kYRingRows * 4 * 32);
        for (int seg = 0; seg < nseg; ++seg)
            for (int cw = 0; cw < ncw; ++cw)
                for (int lane = 0; lane < 32; ++lane) {
                    if (policy == 0)
                        y_item<double, RefOrder>(a, K, seg, nseg, cw, lane, T);
                    else if (policy == 2)
                        y_item<double, RefOrder, 4>(a, K, seg, nseg, cw, lane, T, ring.data() + lane, 32);
                    else
                        y_item<double, Hoisted>(a, K, seg, nseg, cw, lane, T);
                }
    }
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) out[4 * c + f] = D[f * plane + c];
    return 0;
}

// Tangent of one split step of the shared-reciprocal build at a (ny, nx, 4)
// state `cells` along `dir`, from the forward work items run on dual numbers:
// out = the step's result, out_t = its tangent.  T: y segment length.
int kh_step_jvp(const double *cells, const double *dir, int nx, int ny, int strategy, double t, double dt,
                double width, double height, double alpha, double gamma, int T, double *out, double *out_t)
{
    if (nx < 6 || ny < 6) return 1;
    Planes<Dual> U(nx, ny), A(nx, ny), B(nx, ny), V(nx, ny);
    cells_to(U, cells, dir);
    forward_step<Dual, false>(U, A, B, V, nullptr, strategy, t, dt, width / nx, height / ny, alpha, gamma, T);
    for (long long c = 0; c < V.plane; ++c)
        for (int f = 0; f < 4; ++f) {
            out[4 * c + f] = V.v[f * V.plane + c].v;
            out_t[4 * c + f] = V.v[f * V.plane + c].d;
        }
    return 0;
}

// Adjoint of the same step: the taped forward on doubles, then the adjoint
// step's kernels in the launcher's order (ghost transpose into H, then
// Y^T(A1) and X^T(U) for branch A, X^T(B1) and Y^T(U) for branch B, summed):
// in_b = (d step at cells)^T out_b.
int kh_step_vjp(const double *cells, const double *out_b, int nx, int ny, int strategy, double t, double dt,
                double width, double height, double alpha, double gamma, int T, double *in_b)
{
    if (nx < 6 || ny < 6) return 1;
    const double hx = width / nx, hy = height / ny;
    Planes<double> U(nx, ny), A1(nx, ny), B1(nx, ny), V(nx, ny);
    Planes<double> flux[4] = {Planes<double>(nx, ny), Planes<double>(nx, ny), Planes<double>(nx, ny),
                              Planes<double>(nx, ny)};
    cells_to(U, cells, nullptr);
    forward_step<double, true>(U, A1, B1, V, flux, strategy, t, dt, hx, hy, alpha, gamma, T);
    Planes<double> lb(nx, ny), H(nx, ny), T1(nx, ny), T2(nx, ny), out(nx, ny);
    cells_to(lb, out_b, nullptr);
    const GhostGeom gg{nx, ny, strategy};
    Field<double> lbf = lb.field(), Hf = H.field();
    emu::launch(dim3((nx + 31) / 32, (ny + 7) / 8), dim3(32, 8), false,
                [&] { ghost_adjoint_copy(lbf, Hf, gg, 0.5); });
    const int ring = 4 * nx + 4 * (ny - 4);
    emu::launch(dim3((ring + 255) / 256), dim3(256), false, [&] { ghost_adjoint_scatter(lbf, Hf, gg, 0.5); });
    transpose(1, A1, flux[2], H, T1, nullptr, hy, dt, alpha, gamma);
    transpose(0, U, flux[0], T1, T2, nullptr, hx, dt, alpha, gamma);
    transpose(0, B1, flux[3], H, T1, nullptr, hx, dt, alpha, gamma);
    transpose(1, U, flux[1], T1, out, &T2, hy, dt, alpha, gamma);
    for (long long c = 0; c < out.plane; ++c)
        for (int f = 0; f < 4; ++f) in_b[4 * c + f] = out.v[f * out.plane + c];
    return 0;
}

// One sweep in the FP32 build's arithmetic (FP32 planes, PackedCompensated
// physics, the float overloads of the limiter): dir 0 x, 1 y (T interfaces
// per segment); final (x only) averages with comb in place.
int kh_sweep32(int dir, int final, int T, const double *in, const double *comb, double *out, int nx, int ny,
               double h, double dt, double alpha, double gamma)
{
    if (nx < 6 || ny < 6 || (dir == 1 && T < 3) || (final && (dir != 0 || !comb))) return 1;
    Planes<float> S(nx, ny), D(nx, ny);
    cells_to(S, in, nullptr);
    if (final) cells_to(D, comb, nullptr);
    if (dir == 0 && final)
        x_sweep<float, true, false, PackedCompensated>(S, D, nullptr, h, dt, alpha, gamma);
    else if (dir == 0)
        x_sweep<float, false, false, PackedCompensated>(S, D, nullptr, h, dt, alpha, gamma);
    else
        y_sweep<float, false, PackedCompensated>(S, D, nullptr, h, dt, alpha, gamma, T);
    for (long long c = 0; c < D.plane; ++c)
        for (int f = 0; f < 4; ++f) out[4 * c + f] = double(D.v[f * D.plane + c]);
    return 0;
}

// A batch of np problems solved by the batched kernels in the reference
// order (RefOrder), launched as the batch runtime launches them: the initial
// wave-speed kernel, then per step the x, y, y and final x sweeps over all
// problems' items and the ghost kernel, until every problem's loop has ended
// (or max_steps steps).  Problem p is nx[p] x ny[p] cells, `cells` the
// problems' (ny, nx, 4) states one after another; params[7p..7p+6] = width,
// height, t_end, cfl, alpha, gamma, strategy.  The descriptors are laid out
// as the batch runtime lays them out (rows padded to 32, u/a/b buffers per
// problem, prefix counts of items and blocks); grid_x, grid_y: blocks of the
// sweep launches (chunks of items per warp).
int kh_batch_solve(int np, const int *nx, const int *ny, const double *params, const double *cells, int T,
                   int grid_x, int grid_y, int max_steps, double *out_cells, double *out_t, int *out_steps)
{
    constexpr int kSweepThreads = 128, kGhostThreads = 256, kInitThreads = 256;
    std::vector<fvm2d::BatchProblem> P(np);
    std::vector<long long> x0(np + 1, 0), y0(np + 1, 0), off(np + 1, 0);
    std::vector<int> rb0(np + 1, 0), ib0(np + 1, 0);
    for (int p = 0; p < np; ++p) {
        if (nx[p] < 6 || ny[p] < 6) return 1;
        fvm2d::BatchProblem &q = P[p];
        std::memset(&q, 0, sizeof q);
        const double *pr = params + 7 * p;
        q.pitch = (nx[p] + 31) / 32 * 32;
        q.plane = (long long)q.pitch * ny[p];
        q.u = off[p];
        q.a = off[p] + 4 * q.plane;
        q.b = off[p] + 8 * q.plane;
        off[p + 1] = off[p] + 12 * q.plane;
        q.nx = nx[p];
        q.ny = ny[p];
        q.strategy = int(pr[6]);
        q.hx = pr[0] / double(nx[p]);
        q.hy = pr[1] / double(ny[p]);
        q.rhx = 1.0 / q.hx;
        q.rhy = 1.0 / q.hy;
        q.alpha = pr[4];
        q.gamma = pr[5];
        q.plan.t_end = pr[2];
        q.plan.cfl = pr[3];
        q.plan.hmin = (q.hy < q.hx) ? q.hy : q.hx;
        q.plan.fixed_dt = 0.0;
        q.xchunks = g_xchunks;
        q.nsegx = fvm2d::x_items_per_row(nx[p], g_xchunks);
        q.ncw = (nx[p] + 31) / 32;
        q.T = T;
        q.nsegy = y_segments(ny[p], T);
        q.ring = 4 * nx[p] + 4 * (ny[p] - 4);
        x0[p + 1] = x0[p] + (long long)q.nsegx * ny[p];
        y0[p + 1] = y0[p] + (long long)q.ncw * q.nsegy;
        rb0[p + 1] = rb0[p] + (q.ring + kGhostThreads - 1) / kGhostThreads;
        const long long n = (long long)nx[p] * ny[p];
        ib0[p + 1] = ib0[p] + int((n + fvm2d::kBatchInitCells - 1) / fvm2d::kBatchInitCells);
    }
    std::vector<double> base(off[np], 0.0);
    std::vector<StepControl> ctl(np);
    long long c0 = 0;
    for (int p = 0; p < np; ++p) {
        std::memset(&ctl[p], 0, sizeof(StepControl));
        ctl[p].step_limit = max_steps;
        for (int y = 0; y < ny[p]; ++y)
            for (int x = 0; x < nx[p]; ++x)
                for (int f = 0; f < 4; ++f)
                    base[P[p].u + f * P[p].plane + (long long)y * P[p].pitch + x] =
                        cells[c0 + 4 * ((long long)y * nx[p] + x) + f];
        c0 += 4LL * nx[p] * ny[p];
    }
    BatchArgs<double> b;
    b.base = base.data();
    b.prob = P.data();
    b.ctl = ctl.data();
    b.x0 = x0.data();
    b.y0 = y0.data();
    b.rb0 = rb0.data();
    b.ib0 = ib0.data();
    b.np = np;
    const long long xt = x0[np], yt = y0[np];
    emu::launch(dim3(ib0[np]), dim3(kInitThreads), true, [&] { batch_init_kernel<double, kInitThreads>(b); });
    for (int step = 0; step < max_steps; ++step) {
        bool any = false;
        for (int p = 0; p < np; ++p) any |= ctl[p].active != 0;
        if (!any) break;
        emu::launch(dim3(grid_x), dim3(kSweepThreads), true,
                    [&] { batch_sweep_x_kernel<double, RefOrder, false, kSweepThreads, 1>(b, xt, 0); });
        for (int stage = 1; stage <= 2; ++stage)
            emu::launch(dim3(grid_y), dim3(kSweepThreads), false,
                        [&] { batch_sweep_y_kernel<double, RefOrder, kSweepThreads, 1>(b, yt, stage); });
        emu::launch(dim3(grid_x), dim3(kSweepThreads), true,
                    [&] { batch_sweep_x_kernel<double, RefOrder, true, kSweepThreads, 1>(b, xt, 3); });
        emu::launch(dim3(rb0[np]), dim3(kGhostThreads), true, [&] { batch_ghost_kernel<double, kGhostThreads>(b); });
    }
    c0 = 0;
    for (int p = 0; p < np; ++p) {
        for (int y = 0; y < ny[p]; ++y)
            for (int x = 0; x < nx[p]; ++x)
                for (int f = 0; f < 4; ++f)
                    out_cells[c0 + 4 * ((long long)y * nx[p] + x) + f] =
                        base[P[p].u + f * P[p].plane + (long long)y * P[p].pitch + x];
        c0 += 4LL * nx[p] * ny[p];
        out_t[p] = ctl[p].t;
        out_steps[p] = ctl[p].steps;
    }
    return 0;
}

} // extern "C"

// The body of kh_solve for a storage type R and physics Phys; SPLIT: the
// states hold residual planes after the FP32 planes (fvm2d_split.cuh).
template <typename R, class Phys, bool SPLIT>
static int solve_impl(const double *cells, int nx, int ny, double width, double height, double t_end, double cfl,
                      double alpha, double gamma, int strategy, int T, int blocks, int max_steps, double *out,
                      double *t, int *steps, int *first_bad)
{
    constexpr int kNT = 128, kGhostNT = 256, kInitNT = 256;
    if (nx < 6 || ny < 6 || blocks < 1) return 1;
    const int pitch = (nx + 31) / 32 * 32;
    const long long plane = (long long)pitch * ny;
    const long long per_state = (SPLIT ? 6 : 4) * plane;  // 4 FP32 planes + 4 planes of 16-bit residuals
    std::vector<R> Uv(per_state, R(0.0)), Av(per_state, R(0.0)), Bv(per_state, R(0.0));
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            for (int f = 0; f < 4; ++f) {
                const long long k = f * plane + (long long)y * pitch + x;
                const double v = cells[4 * ((long long)y * nx + x) + f];
                if constexpr (SPLIT)
                    fvm2d::split_planes(Uv.data(), plane).put(k, v);
                else
                    Uv[k] = R(v);
            }
    const Field<R> U{Uv.data(), plane, pitch}, A{Av.data(), plane, pitch}, B{Bv.data(), plane, pitch};
    StepControl ctl;
    std::memset(&ctl, 0, sizeof ctl);
    ctl.step_limit = max_steps;
    const double hx = width / nx, hy = height / ny;
    const PlanParams plan{t_end, cfl, hy < hx ? hy : hx, 0.0};
    auto args = [&](const Field<R> &src, const Field<R> &dst, int dir) {
        SweepArgs<R> a;
        a.src = src;
        a.dst = dst;
        a.comb = dst;
        a.flux = Field<R>{nullptr, plane, pitch};
        a.xchunks = g_xchunks;
        a.nx = nx;
        a.ny = ny;
        a.h = dir == 0 ? hx : hy;
        a.rh = 1.0 / a.h;
        a.alpha = alpha;
        a.gamma = gamma;
        a.ctl = &ctl;
        return a;
    };
    GhostArgs<R> g;
    g.U = U;
    g.nx = nx;
    g.ny = ny;
    g.strategy = strategy;
    g.gamma = gamma;
    g.ctl = &ctl;
    g.plan = plan;
    g.row0 = 0;
    g.gny = ny;
    g.fill_top = g.fill_bottom = 1;
    g.residual = SPLIT;
    const int ring = 4 * nx + 4 * (ny - 4);
    emu::launch(dim3(2), dim3(kInitNT), true, [&] { init_kernel<R, kInitNT>(U, nx, ny, gamma, &ctl, plan); });
    for (int k = 0; k < max_steps && ctl.active; ++k) {
        const SweepArgs<R> ax = args(U, A, 0), ay = args(U, B, 1), aya = args(A, U, 1), axf = args(B, U, 0);
        emu::launch(dim3(blocks), dim3(kNT), true, [&] { sweep_x_kernel<R, Phys, false, kNT, 1>(ax); });
        emu::launch(dim3(blocks), dim3(kNT), false, [&] { sweep_y_kernel<R, Phys, kNT, 1>(ay, T); });
        emu::launch(dim3(blocks), dim3(kNT), false, [&] { sweep_y_kernel<R, Phys, kNT, 1>(aya, T); });
        emu::launch(dim3(blocks), dim3(kNT), true, [&] { sweep_x_kernel<R, Phys, true, kNT, 1>(axf); });
        emu::launch(dim3((ring + kGhostNT - 1) / kGhostNT), dim3(kGhostNT), true,
                    [&] { ghost_kernel<R, kGhostNT>(g); });
    }
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            for (int f = 0; f < 4; ++f) {
                const long long k = f * plane + (long long)y * pitch + x;
                double v;
                if constexpr (SPLIT)
                    v = fvm2d::split_planes(Uv.data(), plane).get(k);
                else
                    v = double(Uv[k]);
                out[4 * ((long long)y * nx + x) + f] = v;
            }
    *t = ctl.t;
    *steps = ctl.steps;
    *first_bad = ctl.first_bad;
    return 0;
}

extern "C" {

// A solve through the single-problem kernels in the reference order
// (RefOrder), launched as a solver's step graphs launch them: init_kernel,
// then per step sweep_x_kernel, sweep_y_kernel twice, the final
// sweep_x_kernel and ghost_kernel, on `blocks` blocks of 128 threads per
// sweep (grid-stride), until the control record ends the loop or max_steps.
// out: final state; t, steps and the health record's first bad step.
int kh_solve(const double *cells, int nx, int ny, double width, double height, double t_end, double cfl,
             double alpha, double gamma, int strategy, int T, int blocks, int max_steps, double *out, double *t,
             int *steps, int *first_bad)
{
    return solve_impl<double, RefOrder, false>(cells, nx, ny, width, height, t_end, cfl, alpha, gamma, strategy, T,
                                               blocks, max_steps, out, t, steps, first_bad);
}

// kh_solve through the builds' own physics: 0 the FP64 default (Hoisted),
// 1 FP32 (PackedCompensated), 2 FP32 with residual planes (PackedResidual).
int kh_solve_build(int build, const double *cells, int nx, int ny, double width, double height, double t_end,
                   double cfl, double alpha, double gamma, int strategy, int T, int blocks, int max_steps, double *out,
                   double *t, int *steps, int *first_bad)
{
    if (build == 0)
        return solve_impl<double, Hoisted, false>(cells, nx, ny, width, height, t_end, cfl, alpha, gamma, strategy, T,
                                                  blocks, max_steps, out, t, steps, first_bad);
    if (build == 1)
        return solve_impl<float, PackedCompensated, false>(cells, nx, ny, width, height, t_end, cfl, alpha, gamma,
                                                           strategy, T, blocks, max_steps, out, t, steps, first_bad);
    if (build == 2)
        return solve_impl<float, PackedResidual, true>(cells, nx, ny, width, height, t_end, cfl, alpha, gamma,
                                                       strategy, T, blocks, max_steps, out, t, steps, first_bad);
    return 1;
}

// A frame of a (ny, nx, 4) state as a solver writes one: the density range
// reduced by density_range_blocks over `blocks` blocks of 256 threads, the
// colours by render_density, the file by write_png_rgb.  Returns 0, or 2 when
// the file cannot be written.
int kh_frame(const double *cells, int nx, int ny, int blocks, const char *path)
{
    constexpr int kNT = 256;
    if (nx < 1 || ny < 1 || blocks < 1) return 1;
    const int pitch = (nx + 31) / 32 * 32;
    std::vector<double> rho((size_t)pitch * ny, 0.0);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) rho[(size_t)y * pitch + x] = cells[4 * ((size_t)y * nx + x)];
    std::vector<float> parts(2 * blocks);
    std::vector<unsigned char> rgb(3 * (size_t)nx * ny);
    emu::launch(dim3(blocks), dim3(kNT), true, [&] {
        fvm2d::io::density_range_blocks<double, kNT>(rho.data(), pitch, nx, ny, parts.data());
    });
    emu::launch(dim3(3), dim3(kNT), false, [&] {
        fvm2d::io::render_density<double>(rho.data(), pitch, nx, ny, parts.data(), blocks, rgb.data());
    });
    return fvm2d::io::write_png_rgb(path, nx, ny, rgb.data()) ? 0 : 2;
}

// The conserved totals as fvm2d_get_conserved_totals computes them
// (conserved_partials over `blocks` blocks of 256 threads, then
// conserved_sum) on a (ny, nx, 4) array of (rho, p, u, v) cells, stored
// first as the solver stores them: storage 0 FP64 planes, 1 FP32 planes,
// 2 FP32 planes with residuals, rows `pitch` elements apart.  totals: mass,
// x momentum, y momentum, energy times `area`.
int kh_totals(const double *cells, int nx, int ny, int pitch, int storage, int blocks, double gamma, double area,
              double *totals)
{
    constexpr int kNT = 256;
    if (nx < 6 || ny < 6 || pitch < nx || blocks < 1 || storage < 0 || storage > 2) return 1;
    const long long plane = (long long)pitch * ny;
    std::vector<double> d(storage == 0 ? 4 * plane : 0);
    std::vector<float> f(storage == 0 ? 0 : 6 * plane);  // FP32 planes, then room for the residual block
    std::vector<double> partial(4 * (size_t)blocks), sum(4);
    auto run = [&](auto st) {
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                for (int q = 0; q < 4; ++q) st.put(q * plane + (long long)y * pitch + x, cells[4 * ((size_t)y * nx + x) + q]);
        emu::launch(dim3(blocks), dim3(kNT), true, [&] {
            fvm2d::conserved_partials<decltype(st), kNT>(st, nx, ny, pitch, plane, gamma, partial.data());
        });
        emu::launch(dim3(1), dim3(32), false, [&] { fvm2d::conserved_sum(partial.data(), blocks, area, sum.data()); });
    };
    if (storage == 0)
        run(fvm2d::Planes<double>{d.data()});
    else if (storage == 1)
        run(fvm2d::Planes<float>{f.data()});
    else
        run(fvm2d::split_planes(f.data(), plane));
    for (int q = 0; q < 4; ++q) totals[q] = sum[q];
    return 0;
}

} // extern "C"
