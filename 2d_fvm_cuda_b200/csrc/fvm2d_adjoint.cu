// fvm2d_adjoint.cu -- reverse-mode (adjoint) step of the FP64 build with shared
// reciprocals, for fixed dt.
//
// The step is U' = ghost((Y(X(U)) + X(Y(U))) / 2).  Its adjoint, given the
// adjoint lb' of U', is
//   H   = ghost^T lb' / 2      (ring values are copies of interior cells)
//   A1b = Y^T(A1) H ;  UbA = X^T(U) A1b      (branch A, A1 = X(U))
//   B1b = X^T(B1) H ;  UbB = Y^T(U) B1b      (branch B, B1 = Y(U))
//   lb  = UbA + UbB
// A1, B1 and the interface fluxes of the four sweeps come from the forward
// step's tape (fp64::enqueue_step_taped), so no forward sweep is rerun.
//
// A sweep's transpose is one kernel.  A warp holds 32 consecutive positions
// of a line, one per lane, and does in registers, exchanging neighbours by
// shuffles: the limited slope of its cell, the adjoint of its cell's
// conservative update (from the taped fluxes), the adjoint of its interface
// (face states, relaxation GRP and midpoint flux, recomputed forward and then
// reversed), the limiter's adjoint of its slope, and finally the gather of
// every part that reaches its cell.  An output depends on positions up to
// three away, so lanes 3..28 (26 positions) are exact and work items overlap
// by six positions; no value is accumulated by two threads.  x-lines are read
// straight from global memory (coalesced along rows); y-lines go through a
// shared-memory tile of 8 columns x 32 positions that is loaded and stored
// row by row.  Only the ghost ring's transpose adds with atomics (several
// ring cells may copy the same interior cell).
#define FVM2D_VARIANT adj
#include "fvm2d_adjoint_math.cuh"
#include "fvm2d_adjoint.h"
#include "fvm2d_kernels.cuh"

namespace fvm2d {
namespace adj {

constexpr int ANT = 128;         // threads per block of the sweep transposes
constexpr int kLineOut = 26;     // exact positions per 32-lane item (lanes 3..28)
constexpr int kTileCols = 8;     // columns of a y-line tile
constexpr int kTileStride = kTileCols + 1;  // odd stride: conflict-free column reads

__device__ __forceinline__ Cell<A> zero_cell() { return {0.0, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ Cell<A> add(const Cell<A> &a, const Cell<A> &b)
{
    return {a.rho + b.rho, a.p + b.p, a.un + b.un, a.ut + b.ut};
}

// Adjoint of one sweep at line position c of a line of L cells, one position
// per lane: U is the cell swept, ub the adjoint of the sweep's output there,
// F the taped flux of interface c-1/2 (zero where c is not an interface).
// Returns the adjoint of the sweep's input at c; exact on lanes 3..28.
// Ranges follow the forward sweep: slopes 1..L-2, interfaces 2..L-2, updated
// cells 2..L-3; the others pass through.
__device__ __forceinline__ Cell<A> line_adjoint(const Cell<A> &U, const Cell<A> &ub, const Cell<A> &F, int c, int L,
                                                const SweepConsts<A> &K)
{
    const Cell<A> Um = shfl_up(U), Up = shfl_down(U);
    const bool has_slope = c >= 1 && c <= L - 2;
    const bool iface = c >= 2 && c <= L - 2;
    Cell<A> s = zero_cell();
    if (has_slope) s = Hoisted::slope(Um, U, Up, K);
    const Cell<A> sm = shfl_up(s);
    const Cell<A> FR = shfl_down(F);
    // the cell's conservative update
    Cell<A> r = zero_cell(), mb = zero_cell();
    if (c >= 2 && c <= L - 3)
        mb = update_adjoint(U, F, FR, K, ub, r);
    else
        r = ub;
    const Cell<A> mbm = shfl_up(mb);
    // interface c-1/2: the flux leaves cell c-1 (-lambda) and enters cell c (+lambda)
    Cell<A> a = zero_cell(), b = zero_cell(), sa = zero_cell(), sb = zero_cell();
    if (iface) {
        const A lam = K.lambda;
        const Cell<A> Fb = {lam * (mb.rho - mbm.rho), lam * (mb.p - mbm.p), lam * (mb.un - mbm.un),
                            lam * (mb.ut - mbm.ut)};
        interface_flux_adjoint(Um, U, sm, s, K, Fb, a, b, sa, sb);
    }
    r = add(r, b);                // right cell of interface c-1/2
    r = add(r, shfl_down(a));     // left cell of interface c+1/2
    // slope c: right slope of interface c-1/2, left slope of interface c+1/2
    const Cell<A> sbar = add(sb, shfl_down(sa));
    Cell<A> mbar = zero_cell(), cbar = zero_cell(), pbar = zero_cell();
    if (has_slope) {
        slope_adjoint(slope_choice(Um.rho, U.rho, Up.rho, K.rh, K.alpha), sbar.rho, K.rh, K.alpha, mbar.rho, cbar.rho,
                      pbar.rho);
        slope_adjoint(slope_choice(Um.p, U.p, Up.p, K.rh, K.alpha), sbar.p, K.rh, K.alpha, mbar.p, cbar.p, pbar.p);
        slope_adjoint(slope_choice(Um.un, U.un, Up.un, K.rh, K.alpha), sbar.un, K.rh, K.alpha, mbar.un, cbar.un,
                      pbar.un);
        slope_adjoint(slope_choice(Um.ut, U.ut, Up.ut, K.rh, K.alpha), sbar.ut, K.rh, K.alpha, mbar.ut, cbar.ut,
                      pbar.ut);
    }
    r = add(r, cbar);             // slope c
    r = add(r, shfl_up(pbar));    // slope c-1 (this cell is its right cell)
    r = add(r, shfl_down(mbar));  // slope c+1 (this cell is its left cell)
    return r;
}

struct SweepT {
    Field<A> U, F, ub, out, addend;  // addend.base may be null
    int nx, ny;
    adj::SweepConsts<A> K;
};

// out = X^T ub (+ addend).  Work item: row y, positions 26 seg - 3 .. 26 seg + 28.
__global__ void __launch_bounds__(ANT, 2) adjoint_x_kernel(SweepT g)
{
    const int lane = threadIdx.x & 31;
    const int nseg = (g.nx + kLineOut - 1) / kLineOut;
    const long long nwork = (long long)nseg * g.ny;
    const long long wstride = (long long)gridDim.x * (ANT / 32);
    for (long long w = (long long)blockIdx.x * (ANT / 32) + threadIdx.x / 32; w < nwork; w += wstride) {
        const int y = int(w / nseg), seg = int(w % nseg);
        const int c = kLineOut * seg + lane - 3;
        const bool in = c >= 0 && c < g.nx;
        const int xc = min(max(c, 0), g.nx - 1);
        const Cell<A> U = load_cell(g.U, xc, y, 2, 3);
        const Cell<A> ub = in ? load_cell(g.ub, xc, y, 2, 3) : zero_cell();
        const Cell<A> F = (c >= 2 && c <= g.nx - 2) ? load_cell(g.F, c, y, 2, 3) : zero_cell();
        Cell<A> r = line_adjoint(U, ub, F, c, g.nx, g.K);
        if (lane >= 3 && lane <= 28 && in) {
            if (g.addend.base) r = add(r, load_cell(g.addend, c, y, 2, 3));
            store_cell(g.out, c, y, 2, 3, r);
        }
    }
}

// out = Y^T ub (+ addend).  Block: columns 8 bx .. 8 bx + 7, line positions
// 26 by - 3 .. 26 by + 28 (position l is row ny-1-l; (un, ut) = (v, u)).
__global__ void __launch_bounds__(ANT, 2) adjoint_y_kernel(SweepT g)
{
    __shared__ A sU[4][32][kTileStride], sB[4][32][kTileStride], sF[4][32][kTileStride];
    const int x0 = blockIdx.x * kTileCols, l0 = blockIdx.y * kLineOut - 3;
    const int nx = g.nx, ny = g.ny;
    for (int q = threadIdx.x; q < 32 * kTileCols; q += ANT) {
        const int k = q / kTileCols, col = q % kTileCols;
        const int x = min(x0 + col, nx - 1), l = l0 + k;
        const int j = ny - 1 - min(max(l, 0), ny - 1);
        const Cell<A> U = load_cell(g.U, x, j, 3, 2);
        const Cell<A> ub = (l >= 0 && l < ny) ? load_cell(g.ub, x, j, 3, 2) : zero_cell();
        const Cell<A> F = (l >= 2 && l <= ny - 2) ? load_cell(g.F, x, j, 2, 3) : zero_cell();
        sU[0][k][col] = U.rho; sU[1][k][col] = U.p; sU[2][k][col] = U.un; sU[3][k][col] = U.ut;
        sB[0][k][col] = ub.rho; sB[1][k][col] = ub.p; sB[2][k][col] = ub.un; sB[3][k][col] = ub.ut;
        sF[0][k][col] = F.rho; sF[1][k][col] = F.p; sF[2][k][col] = F.un; sF[3][k][col] = F.ut;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x / 32;
    for (int col = warp; col < kTileCols; col += ANT / 32) {
        const Cell<A> U = {sU[0][lane][col], sU[1][lane][col], sU[2][lane][col], sU[3][lane][col]};
        const Cell<A> ub = {sB[0][lane][col], sB[1][lane][col], sB[2][lane][col], sB[3][lane][col]};
        const Cell<A> F = {sF[0][lane][col], sF[1][lane][col], sF[2][lane][col], sF[3][lane][col]};
        const Cell<A> r = line_adjoint(U, ub, F, l0 + lane, ny, g.K);
        // each warp owns its columns: the result replaces its own ub entry
        sB[0][lane][col] = r.rho; sB[1][lane][col] = r.p; sB[2][lane][col] = r.un; sB[3][lane][col] = r.ut;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 32 * kTileCols; q += ANT) {
        const int k = q / kTileCols, col = q % kTileCols;
        const int x = x0 + col, l = l0 + k;
        if (k < 3 || k > 28 || x >= nx || l >= ny) continue;
        const int j = ny - 1 - l;
        Cell<A> r = {sB[0][k][col], sB[1][k][col], sB[2][k][col], sB[3][k][col]};
        if (g.addend.base) r = add(r, load_cell(g.addend, x, j, 3, 2));
        store_cell(g.out, x, j, 3, 2, r);
    }
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

// Vb = scale * lb with the ring zeroed
__global__ void ghost_adjoint_copy(Field<A> lb, Field<A> Vb, GhostGeom g, A scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const bool ring = on_ring(g, i, j);
    for (int f = 0; f < 4; ++f) Vb.at(f, i, j) = ring ? 0.0 : scale * lb.at(f, i, j);
}

// Vb(source) += scale * sign * lb(ring cell)
__global__ void ghost_adjoint_scatter(Field<A> lb, Field<A> Vb, GhostGeom g, A scale)
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
    atomicAdd(&Vb.at(0, si, sj), scale * lb.at(0, i, j));
    atomicAdd(&Vb.at(1, si, sj), scale * lb.at(1, i, j));
    atomicAdd(&Vb.at(2, si, sj), scale * lb.at(2, i, j));
    atomicAdd(&Vb.at(3, si, sj), scale * vs * lb.at(3, i, j));
}

} // namespace adj

// ---- host entry --------------------------------------------------------------
namespace {

using adj::A;

adj::Field<A> fld(const double *p, const AdjointLaunch &L)
{
    adj::Field<A> f;
    f.base = const_cast<double *>(p);
    f.plane = L.plane;
    f.pitch = L.pitch;
    return f;
}

adj::SweepConsts<A> consts(const AdjointLaunch &L, int dir)
{
    adj::SweepConsts<A> K;
    const double h = dir == 0 ? L.hx : L.hy;
    K.h = h;
    K.rh = dir == 0 ? L.rhx : L.rhy;
    K.alpha = L.alpha;
    K.g = L.gamma;
    K.k = L.dt;
    K.lambda = L.dt / h;
    K.igm1 = 1.0 / (L.gamma - 1.0);
    K.kappa = (L.gamma + 1.0) / 2.0;
    return K;
}

int g_sms = 0, g_occ_x = 1;

// out = (d sweep_dir / dU at U)^T ub (+ addend)
void sweep_transpose(const AdjointLaunch &L, int dir, const double *U, const double *F, const double *ub,
                     double *out, const double *addend, cudaStream_t s)
{
    adj::SweepT g;
    g.U = fld(U, L);
    g.F = fld(F, L);
    g.ub = fld(ub, L);
    g.out = fld(out, L);
    g.addend = fld(addend, L);
    g.nx = L.nx;
    g.ny = L.ny;
    g.K = consts(L, dir);
    if (dir == 0) {
        const long long items = (long long)((L.nx + adj::kLineOut - 1) / adj::kLineOut) * L.ny;
        long long blocks = (items + adj::ANT / 32 - 1) / (adj::ANT / 32);
        const long long cap = (long long)g_occ_x * g_sms;
        adj::adjoint_x_kernel<<<int(blocks < cap ? blocks : cap), adj::ANT, 0, s>>>(g);
    } else {
        const dim3 grid((L.nx + adj::kTileCols - 1) / adj::kTileCols, (L.ny + adj::kLineOut - 1) / adj::kLineOut);
        adj::adjoint_y_kernel<<<grid, adj::ANT, 0, s>>>(g);
    }
}

} // namespace

cudaError_t adjoint_prepare()
{
    if (g_sms) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ_x, adj::adjoint_x_kernel, adj::ANT, 0))) return e;
    if (g_occ_x < 1) g_occ_x = 1;
    g_sms = sms;
    return cudaSuccess;
}

cudaError_t adjoint_step(const AdjointLaunch &L, cudaStream_t s)
{
    if (cudaError_t e = adjoint_prepare()) return e;
    double *H = L.work[0], *T1 = L.work[1], *T2 = L.work[2];
    // ghost fill and average, transposed: H = ghost^T(lb_out) / 2
    const dim3 g2((L.nx + 31) / 32, (L.ny + 7) / 8), b2(32, 8);
    const adj::GhostGeom gg{L.nx, L.ny, L.strategy};
    adj::ghost_adjoint_copy<<<g2, b2, 0, s>>>(fld(L.lb_out, L), fld(H, L), gg, 0.5);
    const int ring = 4 * L.nx + 4 * (L.ny - 4);
    adj::ghost_adjoint_scatter<<<(ring + 255) / 256, 256, 0, s>>>(fld(L.lb_out, L), fld(H, L), gg, 0.5);
    // branch A: A2 = Y(A1), A1 = X(U)
    sweep_transpose(L, 1, L.A1, L.flux[2], H, T1, nullptr, s);
    sweep_transpose(L, 0, L.U, L.flux[0], T1, T2, nullptr, s);
    // branch B: B2 = X(B1), B1 = Y(U); the sum of both branches is written at once
    sweep_transpose(L, 0, L.B1, L.flux[3], H, T1, nullptr, s);
    sweep_transpose(L, 1, L.U, L.flux[1], T1, L.lb_in, T2, s);
    return cudaGetLastError();
}

} // namespace fvm2d
