/*
 * ref_host.cpp -- runs the reference's own kernels (src/basicFuns.cuh,
 * src/ghostCellPresets.cuh, compiled unchanged for the host through
 * ref_shim.h) in the launch sequence of RGRP_2D_CUDA::solve()
 * (src/wrappers.cuh:154-306).  Built by oracle/Makefile into
 * oracle/_ref/libref_host.so straight from the reference sources.
 *
 * TEST INFRASTRUCTURE ONLY: it pins the C restatement (fvm2d_oracle.c), makes
 * the golden fixtures (tests/golden/make_golden.py) and is the timed CPU
 * baseline of bench.py ("kind": "reference").
 *
 * The solve loop itself (wrappers.cuh) cannot be compiled on the host because
 * it includes OpenCV, so its sequence is restated here call for call:
 * maxPropagtingSpeed + max reduction + dt rule, device copy, branch A
 * (x-sweep, rotate, y-sweep, rotate back), branch B (rotate, y-sweep, rotate
 * back, x-sweep), combineResults, time advance, ghost fill.
 *
 * Launch emulation: every kernel runs over the same 16x16 blocks and grids as
 * wrappers.cuh:187-189; blocks are spread over OpenMP threads (the kernels
 * are independent per thread except the ghost fills).  The ghost-fill kernels
 * read cells that other threads of the same warp write earlier in program
 * order (ghostCellPresets.cuh:112-144: the column phase of a corner reads a
 * row-phase result); on the GPU those threads run in lock step, so the
 * column phase sees the row-phase values.  A serial host loop would not, so
 * each ghost kernel is run twice: the fills are idempotent once their
 * sources are final, and the second pass reads the row-phase results exactly
 * as the GPU does.
 */
#include "basicFuns.cuh"

#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

thread_local uint3 threadIdx, blockIdx;
thread_local dim3 blockDim;

namespace {

int g_threads = 0;

template <class F>
void launch(dim3 grid, dim3 block, F &&kernel)
{
    const long nblocks = (long)grid.x * grid.y;
#pragma omp parallel for schedule(static) num_threads(g_threads > 0 ? g_threads : omp_get_max_threads())
    for (long b = 0; b < nblocks; ++b) {
        blockDim = block;
        blockIdx = make_uint3((unsigned)(b % grid.x), (unsigned)(b / grid.x), 0);
        for (unsigned ty = 0; ty < block.y; ++ty)
            for (unsigned tx = 0; tx < block.x; ++tx) {
                threadIdx = make_uint3(tx, ty, 0);
                kernel();
            }
    }
}

template <class F>
void launch_serial(dim3 grid, dim3 block, F &&kernel)
{
    blockDim = block;
    for (unsigned by = 0; by < grid.y; ++by)
        for (unsigned bx = 0; bx < grid.x; ++bx) {
            blockIdx = make_uint3(bx, by, 0);
            for (unsigned ty = 0; ty < block.y; ++ty)
                for (unsigned tx = 0; tx < block.x; ++tx) {
                    threadIdx = make_uint3(tx, ty, 0);
                    kernel();
                }
        }
}

struct Solver {
    int Nx, Ny;
    double width, height, CFL, alpha, gamma, endTime;
    int strategy;
    std::vector<vec5d> u, u_copy, lr, uut, lr_y, uut_y, uy, slope, slope_y;
    std::vector<double> speed;
    std::vector<int> edited, edited_y;
    dim3 block{16, 16}, grid, grid_y;
    double cTime = 0.0;

    Solver(int nx, int ny) : Nx(nx), Ny(ny)
    {
        size_t n = (size_t)nx * ny;
        u.resize(n); u_copy.resize(n); uy.resize(n);
        lr.resize((n + ny) * 2); uut.resize((n + ny) * 2);
        lr_y.resize((n + nx) * 2); uut_y.resize((n + nx) * 2);
        slope.resize(n); slope_y.resize(n); speed.resize(n);
        edited.resize((n + ny) * 2); edited_y.resize((n + ny) * 2);
        grid = dim3((nx + 15) / 16, (ny + 15) / 16);
        grid_y = dim3((ny + 15) / 16, (nx + 15) / 16);
    }

    void x_sweep(vec5d *U, int nx, int ny, double w, vec5d *S, vec5d *LR, vec5d *UUT, int *ed, double dt, dim3 g)
    {
        launch(g, block, [&] { MUSCL_rel_RP_GRP(U, S, nx, ny, alpha, w, LR); });
        launch(g, block, [&] { rel_RP_posi_fix(U, S, LR, nx, ny, UUT, ed, gamma); });
        launch(g, block, [&] { forward_x_dir(U, UUT, nx, ny, w, dt, gamma); });
    }

    void rotate(vec5d *in, vec5d *out, int nx, int ny, dim3 g)
    {
        launch(g, block, [&] { rotate_and_flip_vertically(in, out, nx, ny); });
    }

    /* returns 1 when the loop of wrappers.cuh:196 has ended */
    int step()
    {
        if (!(cTime < endTime)) return 1;
        launch(grid, block, [&] { maxPropagtingSpeed(u.data(), speed.data(), Nx, Ny, gamma); });
        double max_speed = -std::numeric_limits<double>::infinity();
        for (double s : speed) max_speed = (max_speed < s) ? s : max_speed;
        double h = std::min(width / double(Nx), height / double(Ny));
        double dt = std::min(CFL * h / max_speed, endTime - cTime);
        if (h / max_speed < 1e-20) return 1;

        u_copy = u;
        x_sweep(u.data(), Nx, Ny, width, slope.data(), lr.data(), uut.data(), edited.data(), dt, grid);
        rotate(u.data(), uy.data(), Nx, Ny, grid);
        x_sweep(uy.data(), Ny, Nx, height, slope_y.data(), lr_y.data(), uut_y.data(), edited_y.data(), dt, grid_y);
        rotate(uy.data(), u.data(), Ny, Nx, grid_y);

        rotate(u_copy.data(), uy.data(), Nx, Ny, grid);
        x_sweep(uy.data(), Ny, Nx, height, slope_y.data(), lr_y.data(), uut_y.data(), edited_y.data(), dt, grid_y);
        rotate(uy.data(), u_copy.data(), Ny, Nx, grid_y);
        x_sweep(u_copy.data(), Nx, Ny, width, slope.data(), lr.data(), uut.data(), edited.data(), dt, grid);

        launch(grid, block, [&] { combineResults(u.data(), u_copy.data(), Nx, Ny); });
        cTime += dt;

        vec5d *U = u.data();
        for (int pass = 0; pass < 2; ++pass) {
            switch (strategy) {
            case 0: launch_serial(grid, block, [&] { set_ghost_cells(U, Nx, Ny, width, height, cTime); }); break;
            case 2: launch_serial(grid, block, [&] { set_ghost_cells_jet(U, Nx, Ny, width, height, cTime); }); break;
            case 3: launch_serial(grid, block, [&] { set_ghost_cells_jet800(U, Nx, Ny, width, height, cTime); }); break;
            default: launch_serial(grid, block, [&] { set_ghost_cells_2Mach(U, Nx, Ny, width, height, cTime); }); break;
            }
        }
        return 0;
    }
};

void load(Solver &s, const double *U4)
{
    for (size_t k = 0; k < s.u.size(); ++k)
        s.u[k] = vec5d(U4[4 * k], U4[4 * k + 1], U4[4 * k + 2], U4[4 * k + 3], 0.0);
}

void store(const Solver &s, double *U4)
{
    for (size_t k = 0; k < s.u.size(); ++k)
        for (int c = 0; c < 4; ++c) U4[4 * k + c] = s.u[k][c];
}

} // namespace

extern "C" {

void ref_set_threads(int n) { g_threads = n; }

/* Runs the loop from t = t0 for at most max_steps steps (max_steps < 0: until
 * the loop ends) on U4 = (ny, nx, 4) doubles in place.  The strategy codes
 * follow wrappers.cuh:17-24 (0 outflow, 1 reflective, 2 jet, 3 jet800,
 * 4 doubleMach); 1 and 4 both run the double-Mach kernel as
 * wrappers.cuh:277-280 does.  Returns 0; *steps and *t report progress. */
int ref_run(double *U4, int nx, int ny, double width, double height,
            double cfl, double alpha, double gamma, double t_end, int strategy,
            double t0, int max_steps, int *steps, double *t)
{
    /* set_ghost_cells (ghostCellPresets.cuh:106-145) has no bounds check and
     * its corner reads are warp-local only when both sizes are multiples of
     * the 16x16 block, so the reference is run on such sizes only. */
    if (strategy < 0 || strategy > 4 || nx < 16 || ny < 16 || nx % 16 || ny % 16) return 1;
    Solver s(nx, ny);
    s.width = width; s.height = height; s.CFL = cfl; s.alpha = alpha;
    s.gamma = gamma; s.endTime = t_end; s.strategy = strategy; s.cTime = t0;
    load(s, U4);
    int k = 0;
    while (max_steps < 0 || k < max_steps) {
        if (s.step()) break;
        ++k;
    }
    store(s, U4);
    if (steps) *steps = k;
    if (t) *t = s.cTime;
    return 0;
}

} // extern "C"
