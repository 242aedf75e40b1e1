/*
 * fvm2d_oracle.h -- CPU restatement of the reference's split 2D Euler step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it.  The product library never
 * links or calls it, and there is no CPU fallback through it.
 *
 * Parity: pinned.  The restatement is checked bit-for-bit against the
 * reference's own kernels (src/basicFuns.cuh, src/ghostCellPresets.cuh)
 * compiled for the host (oracle/_ref, recipe in oracle/Makefile) and against
 * the golden fixtures in tests/golden/ generated from that build.
 *
 * State layout: (ny, nx, 4) row-major doubles, cell (i, j) at
 * ((j * nx) + i) * 4, fields (rho, p, u, v) -- the first four slots of the
 * reference's vec5d (src/ghostCellPresets.cuh:4-45; slot 4 never feeds the
 * arithmetic because vec5d's operators only touch slots 0-3).
 *
 * Build with contraction off (-ffp-contract=off): every expression keeps the
 * reference's operation order so a no-FMA build of the reference and of the
 * CUDA kernels agree with it bit for bit.
 */
#ifndef FVM2D_ORACLE_H
#define FVM2D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Ghost-cell strategies.  0..4 are the reference's enum class
 * ghostCellStrategy (src/wrappers.cuh:17-24) in declaration order; 5 and 6
 * are presets the reference does not have. */
enum {
    ORC_OUTFLOW = 0,
    ORC_REFLECTIVE = 1,   /* reference dispatches this to the double-Mach kernel (wrappers.cuh:277-280) */
    ORC_JET = 2,
    ORC_JET800 = 3,
    ORC_DOUBLE_MACH = 4,
    ORC_PERIODIC = 5,
    ORC_REFLECTIVE_TB = 6
};

typedef struct {
    int nx, ny;            /* cells incl. the two ghost layers on each side */
    double width, height;  /* extent of the whole array, ghosts included */
    double cfl, alpha, gamma, t_end;
    int strategy;
} orc_params;

/* max over all cells of |(u,v)| + sqrt(gamma p / rho)  (basicFuns.cuh:215-226) */
double orc_max_speed(const double *U, int nx, int ny, double gamma);

/* One reference x-sweep in place: MUSCL slopes (basicFuns.cuh:37-72), the
 * relaxation GRP at every interior interface (basicFuns.cuh:75-192) and the
 * conservative update of columns 2..nx-3 (basicFuns.cuh:229-246). */
void orc_sweep_x(double *U, int nx, int ny, double width, double dt,
                 double alpha, double gamma);

/* One reference y-sweep in place: anti-transpose with u<->v
 * (basicFuns.cuh:249-262), x-sweep of the transposed array with spacing
 * height/ny, anti-transpose back (wrappers.cuh:217-225). */
void orc_sweep_y(double *U, int nx, int ny, double height, double dt,
                 double alpha, double gamma);

/* Ghost fill for one strategy at time t, rows first then columns
 * (ghostCellPresets.cuh:48-241 plus the two new presets). */
void orc_ghost(double *U, int nx, int ny, double width, double height,
               double t, int strategy);

/* dt rule of wrappers.cuh:196-207.  Returns 1 when the loop ends (t >= t_end
 * or the step-size guard fires), else 0 with *dt set. */
int orc_dt(const double *U, const orc_params *p, double t, double *dt);

/* One full step of wrappers.cuh:196-284 in place:
 * U <- ghost( (Y(X(U)) + X(Y(U))) / 2 ) with t advanced by dt.
 * Returns 1 if the loop has ended (nothing done), else 0. */
int orc_step(double *U, const orc_params *p, double *t, double *dt_out);

/* Run the loop until it ends or max_steps steps (max_steps < 0: no cap). */
int orc_solve(double *U, const orc_params *p, int max_steps, int *steps,
              double *t);

/* Point routines exposed for unit tests. */
void orc_slope(const double *Um, const double *U0, const double *Up,
               double h, double alpha, double s[4]);
void orc_grp(const double L[4], const double R[4], const double sL[4],
             const double sR[4], double gamma, double W[5], double Wt[5]);
void orc_flux(const double W[5], const double Wt[5], double k, double F[4]);

/* Thread count used by the OpenMP loops (<=0: OpenMP default). */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
