/*
 * fvm2d_oracle.c -- CPU restatement of the reference's split 2D Euler step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see the header.
 * Every routine cites the reference file:line whose arithmetic it restates.
 * Expressions keep the reference's evaluation order because FP64 parity with
 * contraction off is bit-exact only when every rounding happens in the same
 * order; the structure around them (row-local scratch, OpenMP over rows,
 * 4-double cells) is this oracle's own.
 */
#include "fvm2d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;

void orc_set_threads(int n) { g_threads = n; }

static int nthreads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

static double dmin(double a, double b) { return (b < a) ? b : a; }
static double dmax(double a, double b) { return (a < b) ? b : a; }

/* Limited slope of one cell from its two neighbours: central, backward and
 * forward differences scaled by 1/h (the last two by alpha) combined by the
 * generalized minmod.  basicFuns.cuh:49-68. */
void orc_slope(const double *Um, const double *U0, const double *Up,
               double h, double alpha, double s[4])
{
    for (int c = 0; c < 4; ++c) {
        double central = (Up[c] - Um[c]) * 0.5 * (1.0 / h);
        double back = (U0[c] - Um[c]) * (1.0 / h) * alpha;
        double fwd = (Up[c] - U0[c]) * (1.0 / h) * alpha;
        double p13 = central * fwd, p23 = back * fwd;
        if (p13 > 0.0 && p23 > 0.0) {
            double sign = (central <= 0.0) ? -1.0 : 1.0;
            s[c] = sign * dmin(fabs(central), dmin(fabs(back), fabs(fwd)));
        } else {
            s[c] = 0.0;
        }
    }
}

/* Relaxation GRP at one interface: left/right face states and the slopes of
 * the two cells give the sampled interface state W = (rho, p, u, v, e) and
 * its time derivative Wt.  basicFuns.cuh:86-189.  The star-region
 * coefficients read `u` before it is assigned the star velocity
 * (basicFuns.cuh:151-155 use the initial 0.0 of basicFuns.cuh:110); that is
 * reproduced by the literal 0.0 below. */
void orc_grp(const double L[4], const double R[4], const double sL[4],
             const double sR[4], double g, double W[5], double Wt[5])
{
    const double rho_l = L[0], pi_l = L[1], u_l = L[2], v_l = L[3];
    const double rho_r = R[0], pi_r = R[1], u_r = R[2], v_r = R[3];
    const double rho_lx = sL[0], pi_lx = sL[1], u_lx = sL[2], v_lx = sL[3];
    const double rho_rx = sR[0], pi_rx = sR[1], u_rx = sR[2], v_rx = sR[3];

    double e_l = pi_l / rho_l / (g - 1.0);
    double e_r = pi_r / rho_r / (g - 1.0);
    double e_lx = pi_lx / rho_l / (g - 1.0) - pi_l * rho_lx / rho_l / rho_l / (g - 1.0);
    double e_rx = pi_rx / rho_r / (g - 1.0) - pi_r * rho_rx / rho_r / rho_r / (g - 1.0);
    double c_lx = 0.5 * sqrt(g / pi_l / rho_l) * (pi_l * rho_lx + rho_l * pi_lx);
    double c_rx = 0.5 * sqrt(g / pi_r / rho_r) * (pi_r * rho_rx + rho_r * pi_rx);

    double rho, pi, u, v, e, rho_t, pi_t, u_t, v_t, e_t;
    double c_l, c_r;
    double a_l = sqrt(g * pi_l / rho_l), a_r = sqrt(g * pi_r / rho_r);
    double kappa = (g + 1.0) / 2.0;

    /* relaxation (Lagrangian) wave speeds, basicFuns.cuh:115-127 */
    if (pi_r >= pi_l) {
        c_l = rho_l * (a_l + kappa * dmax(0.0, (pi_r - pi_l) / rho_r / a_r + u_l - u_r));
        c_r = rho_r * (a_r + kappa * dmax(0.0, (pi_l - pi_r) / c_l + u_l - u_r));
    } else {
        c_r = rho_r * (a_r + kappa * dmax(0.0, (pi_l - pi_r) / rho_l / a_l + u_l - u_r));
        c_l = rho_l * (a_l + kappa * dmax(0.0, (pi_r - pi_l) / c_r + u_l - u_r));
    }

    if (u_l - c_l / rho_l >= 0.0) {
        /* whole fan moves right: left state, basicFuns.cuh:129-137 */
        rho = rho_l; pi = pi_l; u = u_l; v = v_l; e = e_l;
        rho_t = -rho * u_lx - u * rho_lx;
        u_t = -u * u_lx - pi_lx / rho;
        e_t = -u * e_lx - pi / rho * u_lx;
        v_t = -u * v_lx;
        pi_t = -u * pi_lx - c_l * c_l / rho_l * u_lx;
    } else if (u_r + c_r / rho_r <= 0.0) {
        /* whole fan moves left: right state, basicFuns.cuh:138-146 */
        rho = rho_r; pi = pi_r; u = u_r; v = v_r; e = e_r;
        rho_t = -rho * u_rx - u * rho_rx;
        u_t = -u * u_rx - pi_rx / rho;
        e_t = -u * e_rx - pi / rho * u_rx;
        v_t = -u * v_rx;
        pi_t = -u * pi_rx - c_r * c_r / rho * u_rx;
    } else {
        /* star region, basicFuns.cuh:147-186 */
        const double u0 = 0.0; /* value `u` holds at basicFuns.cuh:151-155 */
        double u_m = (u_l * c_l + u_r * c_r + pi_l - pi_r) / (c_l + c_r);
        double pi_m = ((u_l - u_r) * c_l * c_r + c_l * pi_r + c_r * pi_l) / (c_l + c_r);
        double k_l = -pi_lx - c_l * u_lx + 0.5 * (u0 - u_l) * c_lx;
        double k_r = -pi_rx + c_r * u_rx - 0.5 * (u0 - u_r) * c_rx;
        double d_l = -2.0 * c_l * c_l / rho_l * u_lx - 2.0 * c_l / rho_l * pi_lx + c_l / rho_l * (u0 - u_l) * c_lx;
        double d_r = 2.0 * c_r * c_r / rho_r * u_rx - 2.0 * c_r / rho_r * pi_rx + c_r / rho_r * (u_r - u0) * c_rx;
        double Dpi_Dt = (c_r * d_l - c_l * d_r) / 2.0 / (c_l + c_r);
        pi = pi_m;
        u = u_m;
        if (u <= 0.0) {
            double rho_mr = c_r / (u_r - u_m + c_r / rho_r);
            double e_mr = e_r + (pi_m - pi_r) * (pi_m + pi_r) / 2.0 / c_r / c_r;
            rho = rho_mr;
            e = e_mr;
            v = v_r;
            rho_t = -u * rho * rho * rho / (rho_r * c_r * c_r) * (c_r * c_r / rho_r / rho_r * rho_rx - c_r * u_rx + 1.5 * (u - u_r) * c_rx) + rho * rho * rho / (c_r * c_r * c_r) * (u + c_r / rho) * Dpi_Dt;
            pi_t = 1.0 / (c_l + c_r) * (c_l * c_r / rho_l * (1 + u * rho / c_r) * k_l - c_l * c_r / rho_r * (1 - u * rho / c_l) * k_r);
            u_t = 1.0 / (c_l + c_r) * (c_l / rho_l * (1 + u * rho / c_r) * k_l + c_r / rho_r * (1 - u * rho * c_l / c_r / c_r) * k_r);
            e_t = -u * rho / rho_r / c_r / c_r / c_r * (-pi_r * c_r * pi_rx + c_r * c_r * c_r * e_rx + 2.0 * (e_r - e) * c_r * c_r * c_rx) + pi / c_r / c_r * pi_t;
            double v_x = rho / rho_r * v_rx;
            v_t = -u * v_x;
        } else {
            double rho_ml = c_l / (u_m - u_l + c_l / rho_l);
            double e_ml = e_l + (pi_m - pi_l) * (pi_m + pi_l) / 2.0 / c_l / c_l;
            rho = rho_ml;
            e = e_ml;
            v = v_l;
            rho_t = -u * rho * rho * rho / (rho_l * c_l * c_l) * (c_l * c_l / rho_l / rho_l * rho_lx + c_l * u_lx + 1.5 * (u - u_l) * c_lx) - rho * rho * rho / (c_l * c_l * c_l) * (u - c_l / rho) * Dpi_Dt;
            pi_t = 1.0 / (c_l + c_r) * (c_l * c_r / rho_l * (1 + u * rho / c_r) * k_l - c_l * c_r / rho_r * (1 - u * rho / c_l) * k_r);
            u_t = 1.0 / (c_l + c_r) * (c_l / rho_l * (1 + u * rho * c_r / c_l / c_l) * k_l + c_r / rho_r * (1 - u * rho / c_l) * k_r);
            e_t = -u * rho / rho_l / c_l / c_l / c_l * (-pi_l * c_l * pi_lx + c_l * c_l * c_l * e_lx + 2.0 * (e_l - e) * c_l * c_l * c_lx) + pi / c_l / c_l * pi_t;
            double v_x = rho / rho_l * v_lx;
            v_t = -u * v_x;
        }
    }
    W[0] = rho; W[1] = pi; W[2] = u; W[3] = v; W[4] = e;
    Wt[0] = rho_t; Wt[1] = pi_t; Wt[2] = u_t; Wt[3] = v_t; Wt[4] = e_t;
}

/* Midpoint flux F(W) + k/2 dF/dt(W, Wt) in the sweep's conserved ordering
 * (rho u, rho u^2 + p, energy flux, rho u v).  basicFuns.cuh:14-34. */
void orc_flux(const double W[5], const double Wt[5], double k, double F[4])
{
    const double rho = W[0], pi = W[1], u = W[2], v = W[3], e = W[4];
    const double rho_t = Wt[0], pi_t = Wt[1], u_t = Wt[2], v_t = Wt[3], e_t = Wt[4];
    F[0] = rho * u + k / 2.0 * (rho * u_t + u * rho_t);
    F[1] = rho * u * u + pi + k / 2.0 * (rho_t * u * u + 2.0 * rho * u * u_t + pi_t);
    F[2] = rho * u * (e + u * u / 2.0 + v * v / 2.0) + pi * u + k / 2.0 * (rho_t * u * e + rho * u_t * e + rho * u * e_t + rho_t * u * u * u / 2.0 + 1.5 * rho * u * u * u_t + rho_t * u * v * v / 2.0 + rho * u * v * v_t + rho * u_t * v * v / 2.0 + pi_t * u + pi * u_t);
    F[3] = rho * u * v + k / 2.0 * (rho * u_t * v + u * rho_t * v + u * rho * v_t);
}

/* One x-sweep of one row of n cells (stride 4 doubles) in place.
 * Slopes and face values: basicFuns.cuh:37-72 for 1 <= i <= n-2.
 * Interface i-1/2 for 2 <= i <= n-2: basicFuns.cuh:75-192.
 * Update of 2 <= i <= n-3: basicFuns.cuh:229-246.
 * scratch holds 4n (slopes) + 8n (faces) + 5n + 5n (interface state and
 * derivative) doubles. */
static void sweep_row(double *row, int n, double h, double dt, double alpha,
                      double g, double *scratch)
{
    double *slope = scratch;           /* [n][4] */
    double *faceL = slope + 4 * n;     /* [n][4]  left face of cell i  = right state of interface i-1/2 */
    double *faceR = faceL + 4 * n;     /* [n][4]  right face of cell i = left state of interface i+1/2 */
    double *Wi = faceR + 4 * n;        /* [n][5]  interface i-1/2 state */
    double *Wti = Wi + 5 * n;          /* [n][5]  interface i-1/2 time derivative */

    for (int i = 1; i <= n - 2; ++i) {
        double *s = slope + 4 * i;
        orc_slope(row + 4 * (i - 1), row + 4 * i, row + 4 * (i + 1), h, alpha, s);
        for (int c = 0; c < 4; ++c) {
            faceL[4 * i + c] = row[4 * i + c] - s[c] * h * 0.5;
            faceR[4 * i + c] = row[4 * i + c] + s[c] * h * 0.5;
        }
    }
    for (int i = 2; i <= n - 2; ++i)
        orc_grp(faceR + 4 * (i - 1), faceL + 4 * i, slope + 4 * (i - 1), slope + 4 * i,
                g, Wi + 5 * i, Wti + 5 * i);
    for (int i = 2; i <= n - 3; ++i) {
        double FL[4], FR[4], C[4];
        double *U = row + 4 * i;
        orc_flux(Wi + 5 * i, Wti + 5 * i, dt, FL);
        orc_flux(Wi + 5 * (i + 1), Wti + 5 * (i + 1), dt, FR);
        /* primitive -> conserved (rho, rho u, E, rho v), basicFuns.cuh:195-202 */
        C[0] = U[0];
        C[1] = U[0] * U[2];
        C[2] = U[1] / (g - 1.0) + U[0] * (U[2] * U[2] + U[3] * U[3]) / 2.0;
        C[3] = U[0] * U[3];
        double lambda = dt / h;
        for (int c = 0; c < 4; ++c)
            C[c] = C[c] - (FR[c] - FL[c]) * lambda;
        /* conserved -> primitive, basicFuns.cuh:205-212 */
        U[0] = C[0];
        U[1] = (g - 1.0) * (C[2] - C[1] * C[1] / C[0] / 2.0 - C[3] * C[3] / C[0] / 2.0);
        U[2] = C[1] / C[0];
        U[3] = C[3] / C[0];
    }
}

void orc_sweep_x(double *U, int nx, int ny, double width, double dt,
                 double alpha, double gamma)
{
    double h = width / (double)nx;
    int nt = nthreads();
#pragma omp parallel num_threads(nt)
    {
        double *scratch = (double *)malloc(sizeof(double) * 22 * (size_t)nx);
#pragma omp for schedule(static)
        for (int j = 0; j < ny; ++j)
            sweep_row(U + (size_t)4 * nx * j, nx, h, dt, alpha, gamma, scratch);
        free(scratch);
    }
}

/* out[(nx-1-x) * ny + (ny-1-y)] = in[y * nx + x] with slots 2,3 swapped.
 * basicFuns.cuh:249-262.  Applying it to the result with (ny, nx) is the
 * identity. */
static void anti_transpose(const double *in, double *out, int nx, int ny)
{
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const double *a = in + 4 * ((size_t)y * nx + x);
            double *b = out + 4 * ((size_t)(nx - 1 - x) * ny + (ny - 1 - y));
            b[0] = a[0]; b[1] = a[1]; b[2] = a[3]; b[3] = a[2];
        }
}

void orc_sweep_y(double *U, int nx, int ny, double height, double dt,
                 double alpha, double gamma)
{
    double *T = (double *)malloc(sizeof(double) * 4 * (size_t)nx * ny);
    anti_transpose(U, T, nx, ny);
    orc_sweep_x(T, ny, nx, height, dt, alpha, gamma);
    anti_transpose(T, U, ny, nx);
    free(T);
}

double orc_max_speed(const double *U, int nx, int ny, double gamma)
{
    double m = -INFINITY;
    for (size_t k = 0; k < (size_t)nx * ny; ++k) {
        const double *c = U + 4 * k;
        double velo = sqrt(c[2] * c[2] + c[3] * c[3]);
        double a = sqrt(gamma * c[1] / c[0]);
        double s = fabs(velo) + a;
        m = (m < s) ? s : m;  /* thrust::maximum keeps the larger; NaN never wins */
    }
    return m;
}

/* ---- ghost-cell presets: rows first, then columns ---------------------- */

#define CELL(U, i, j) ((U) + 4 * ((size_t)(j) * nx + (i)))

static void set4(double *d, double a, double b, double c, double e)
{
    d[0] = a; d[1] = b; d[2] = c; d[3] = e;
}

static void copy4(double *d, const double *s) { memcpy(d, s, 4 * sizeof(double)); }

/* Rows 0,1 <- 2 and ny-2 <- ny-3; row ny-1 <- ny-3 (outflow, jet) or
 * ny-4 (jet800).  ghostCellPresets.cuh:112-127, 156-171, 204-219. */
static void rows_outflow(double *U, int nx, int ny, int last_src)
{
    for (int i = 0; i < nx; ++i) {
        copy4(CELL(U, i, 0), CELL(U, i, 2));
        copy4(CELL(U, i, 1), CELL(U, i, 2));
        copy4(CELL(U, i, ny - 2), CELL(U, i, ny - 3));
        copy4(CELL(U, i, ny - 1), CELL(U, i, last_src));
    }
}

static void cols_outflow_right(double *U, int nx, int ny)
{
    for (int j = 0; j < ny; ++j) {
        copy4(CELL(U, nx - 2, j), CELL(U, nx - 3, j));
        copy4(CELL(U, nx - 1, j), CELL(U, nx - 3, j));
    }
}

void orc_ghost(double *U, int nx, int ny, double width, double height,
               double t, int strategy)
{
    (void)width; (void)height;
    switch (strategy) {
    case ORC_OUTFLOW: /* ghostCellPresets.cuh:106-145 */
        rows_outflow(U, nx, ny, ny - 3);
        for (int j = 0; j < ny; ++j) {
            copy4(CELL(U, 0, j), CELL(U, 2, j));
            copy4(CELL(U, 1, j), CELL(U, 2, j));
        }
        cols_outflow_right(U, nx, ny);
        break;
    case ORC_JET: /* ghostCellPresets.cuh:148-193 */
        rows_outflow(U, nx, ny, ny - 3);
        for (int j = 0; j < ny; ++j) {
            int in_jet = (j >= 2 * ny / 5 + 1 && j <= 3 * ny / 5);
            for (int i = 0; i < 2; ++i) {
                if (in_jet) set4(CELL(U, i, j), 5.0, 0.4127, 800.0, 0.0);
                else set4(CELL(U, i, j), 0.5, 0.4127, 0.0, 0.0);
            }
        }
        cols_outflow_right(U, nx, ny);
        break;
    case ORC_JET800: /* ghostCellPresets.cuh:196-241 */
        rows_outflow(U, nx, ny, ny - 4);
        for (int j = 0; j < ny; ++j) {
            int in_jet = (j >= 9 * ny / 10);
            for (int i = 0; i < 2; ++i) {
                if (in_jet) set4(CELL(U, i, j), 1.4, 1.0, 800.0, 0.0);
                else set4(CELL(U, i, j), 0.14, 1.0, 0.0, 0.0);
            }
        }
        cols_outflow_right(U, nx, ny);
        break;
    case ORC_PERIODIC: /* new preset: two-layer wrap */
        for (int i = 0; i < nx; ++i) {
            copy4(CELL(U, i, 0), CELL(U, i, ny - 4));
            copy4(CELL(U, i, 1), CELL(U, i, ny - 3));
            copy4(CELL(U, i, ny - 2), CELL(U, i, 2));
            copy4(CELL(U, i, ny - 1), CELL(U, i, 3));
        }
        for (int j = 0; j < ny; ++j) {
            copy4(CELL(U, 0, j), CELL(U, nx - 4, j));
            copy4(CELL(U, 1, j), CELL(U, nx - 3, j));
            copy4(CELL(U, nx - 2, j), CELL(U, 2, j));
            copy4(CELL(U, nx - 1, j), CELL(U, 3, j));
        }
        break;
    case ORC_REFLECTIVE_TB: /* new preset: mirrored rows with v negated, transmissive columns */
        for (int i = 0; i < nx; ++i) {
            static const int dst[4] = {0, 1, -2, -1};
            static const int src[4] = {3, 2, -3, -4};
            for (int k = 0; k < 4; ++k) {
                int jd = dst[k] < 0 ? ny + dst[k] : dst[k];
                int js = src[k] < 0 ? ny + src[k] : src[k];
                double *d = CELL(U, i, jd);
                copy4(d, CELL(U, i, js));
                d[3] = -d[3];
            }
        }
        for (int j = 0; j < ny; ++j) {
            copy4(CELL(U, 0, j), CELL(U, 2, j));
            copy4(CELL(U, 1, j), CELL(U, 2, j));
        }
        cols_outflow_right(U, nx, ny);
        break;
    default: { /* ORC_REFLECTIVE, ORC_DOUBLE_MACH: ghostCellPresets.cuh:48-103 */
        const double post[4] = {8, 116.5, 4.125 * sqrt(3.0), -4.125};
        const double pre[4] = {1.4, 1, 0, 0};
        double temp = (double)ny / sqrt(3.0);
        double dist = (double)ny * 20 * t / sqrt(3.0);
        int shock_i = nx / 24 + (int)temp + (int)dist;
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                double *d = CELL(U, i, j);
                if (j == 0 || j == 1) {
                    copy4(d, (i <= shock_i) ? post : pre);
                } else if (j == ny - 1) {
                    if (i <= nx / 24) copy4(d, CELL(U, i, j - 2));
                    else { copy4(d, CELL(U, i, j - 3)); d[3] = -d[3]; }
                } else if (j == ny - 2) {
                    copy4(d, CELL(U, i, j - 1));
                    if (i > nx / 24) d[3] = -d[3];
                }
            }
        }
        for (int j = 0; j < ny; ++j) {
            copy4(CELL(U, 0, j), post);
            copy4(CELL(U, 1, j), post);
            copy4(CELL(U, nx - 2, j), pre);
            copy4(CELL(U, nx - 1, j), pre);
        }
        break;
    }
    }
}

#undef CELL

/* wrappers.cuh:196-207 */
int orc_dt(const double *U, const orc_params *p, double t, double *dt)
{
    if (!(t < p->t_end)) return 1;
    double smax = orc_max_speed(U, p->nx, p->ny, p->gamma);
    double h = dmin(p->width / (double)p->nx, p->height / (double)p->ny);
    *dt = dmin(p->cfl * h / smax, p->t_end - t);
    if (h / smax < 1e-20) return 1;
    return 0;
}

/* wrappers.cuh:209-281 */
int orc_step(double *U, const orc_params *p, double *t, double *dt_out)
{
    double dt;
    if (orc_dt(U, p, *t, &dt)) return 1;
    size_t n = (size_t)4 * p->nx * p->ny;
    double *B = (double *)malloc(sizeof(double) * n);
    memcpy(B, U, sizeof(double) * n);
    /* branch A: Y(X(U)) */
    orc_sweep_x(U, p->nx, p->ny, p->width, dt, p->alpha, p->gamma);
    orc_sweep_y(U, p->nx, p->ny, p->height, dt, p->alpha, p->gamma);
    /* branch B: X(Y(U)) */
    orc_sweep_y(B, p->nx, p->ny, p->height, dt, p->alpha, p->gamma);
    orc_sweep_x(B, p->nx, p->ny, p->width, dt, p->alpha, p->gamma);
    /* primitive average, basicFuns.cuh:264-274 */
    for (size_t k = 0; k < n; ++k) U[k] = (U[k] + B[k]) * 0.5;
    free(B);
    *t += dt;
    orc_ghost(U, p->nx, p->ny, p->width, p->height, *t, p->strategy);
    if (dt_out) *dt_out = dt;
    return 0;
}

int orc_solve(double *U, const orc_params *p, int max_steps, int *steps,
              double *t)
{
    int k = 0;
    double tt = 0.0;
    while (max_steps < 0 || k < max_steps) {
        if (orc_step(U, p, &tt, NULL)) break;
        ++k;
    }
    if (steps) *steps = k;
    if (t) *t = tt;
    return 0;
}
