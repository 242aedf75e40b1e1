/*
 * fvm2d.h -- C ABI of the B200 split 2D Euler solver (libfvm2d.so).
 *
 * The reference exposes one C++ class, RGRP_2D_CUDA, header-only in
 * src/wrappers.cuh:26-65, with enum class ghostCellStrategy at
 * src/wrappers.cuh:17-24.  Each entry point below replaces one of its
 * members (cited), with plain pointers and sizes so any language can bind it.
 * include/rgrp_2d_cuda.hpp rebuilds the reference's C++ class on top of this
 * ABI for drop-in source compatibility.
 *
 * Conventions
 *  - Every call returns an int status (FVM2D_OK on success) and never throws;
 *    fvm2d_last_error() gives a message for the calling thread's last failure.
 *  - A handle belongs to the CUDA device current when it was created and owns
 *    one CUDA stream; it is not thread-safe.  All its calls return with their
 *    device work finished (the solve is synchronous, as the reference's is).
 *  - States are `ny` rows of `nx` cells, row-major, including the two ghost
 *    layers on every side (src/wrappers.cuh:67-78).  A host cell is `stride`
 *    doubles: stride 4 is (rho, p, u, v); stride 5 is the reference's vec5d
 *    (src/ghostCellPresets.cuh:4-45), whose fifth slot is ignored on input
 *    and written as 0 on output.  Pointers may be host (pageable or pinned)
 *    or device memory.
 *  - Axis convention (src/basicFuns.cuh:249-262): +u toward increasing column
 *    i, +v toward decreasing row j.
 */
#ifndef FVM2D_H
#define FVM2D_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FVM2D_OK 0
#define FVM2D_ERR_INVALID 1  /* bad argument or unsupported size */
#define FVM2D_ERR_CUDA 2     /* a CUDA call failed (no device, out of memory, ...) */
#define FVM2D_ERR_STATE 3    /* call out of order: no state uploaded yet */

/* Ghost-cell strategies.  0..4 are ghostCellStrategy (src/wrappers.cuh:17-24)
 * with the reference's dispatch (src/wrappers.cuh:265-280): REFLECTIVE and
 * DOUBLE_MACH both run the double-Mach preset.  PERIODIC and REFLECTIVE_TB
 * have no reference counterpart. */
enum fvm2d_ghost_strategy {
    FVM2D_OUTFLOW = 0,       /* src/ghostCellPresets.cuh:106-145 */
    FVM2D_REFLECTIVE = 1,    /* src/ghostCellPresets.cuh:48-103 (as the reference dispatches it) */
    FVM2D_JET = 2,           /* src/ghostCellPresets.cuh:148-193 */
    FVM2D_JET800 = 3,        /* src/ghostCellPresets.cuh:196-241 */
    FVM2D_DOUBLE_MACH = 4,   /* src/ghostCellPresets.cuh:48-103 */
    FVM2D_PERIODIC = 5,      /* two-layer wrap in both directions */
    FVM2D_REFLECTIVE_TB = 6  /* mirrored top/bottom rows with v negated, transmissive columns */
};

/* Arithmetic modes (no reference counterpart: the reference has one FP64 build). */
enum fvm2d_precision {
    FVM2D_FP64 = 0,          /* FP64, shared reciprocals and FMA: the fast default, within the
                                reference tolerance (relative L1 1e-10) */
    FVM2D_FP64_STRICT = 1,   /* FP64, the reference's operation order, no contraction: bit-exact
                                with the reference built -fmad=false */
    FVM2D_FP64_REFORDER = 2, /* FP64, the reference's operation order with FMA contraction, as the
                                reference's own (default) build computes */
    FVM2D_FP32 = 3,          /* FP32 state planes and arithmetic with a compensated conservative
                                update; wave-speed max, dt and time stay FP64.  Host-side states
                                remain doubles (converted on upload and download). */
    FVM2D_FP32_RESIDUAL = 4  /* FP32 slopes and fluxes; each stored value is an FP32 plane value
                                plus a 16-bit (bfloat16) residual, about 31 significant bits
                                in 6 bytes, and the conservative update runs
                                in FP64 on hi + lo.  Solver handles only (no batches, no
                                differentiation). */
};

typedef struct fvm2d_solver fvm2d_solver;

/* Message for the calling thread's last failed call ("" if none). */
const char *fvm2d_last_error(void);

/* Library version string. */
const char *fvm2d_version(void);

/* Creates a solver for an nx x ny array (ghosts included, nx, ny >= 6, and
 * nx rounded up to a multiple of 32 times ny below 2^31) on the current CUDA
 * device.  Replaces RGRP_2D_CUDA(const vector<vector<vec5d>>&)
 * (src/wrappers.cuh:67-78) together with fvm2d_set_state, and the sizes of
 * setRPInitialData (src/wrappers.cuh:80-85).  Defaults as the reference
 * (src/wrappers.cuh:49-52): width = height = 1, end time 0, CFL 0.5,
 * alpha 1.9, gamma 1.4, outflow. */
int fvm2d_create(fvm2d_solver **out, int nx, int ny);

/* Releases the handle and its device memory.  Replaces the per-solve
 * cudaFree calls and clear() (src/wrappers.cuh:292-303, 347-353). */
int fvm2d_destroy(fvm2d_solver *s);

/* setSpatialLayout (src/wrappers.cuh:110-114): extent of the whole array,
 * ghosts included; h_x = width/nx, h_y = height/ny. */
int fvm2d_set_spatial_layout(fvm2d_solver *s, double width, double height);

/* setTimeLayout(endTime, CFL) (src/wrappers.cuh:116-120). */
int fvm2d_set_time_layout(fvm2d_solver *s, double end_time, double cfl);

/* setTimeLayout(endTime) (src/wrappers.cuh:122-125). */
int fvm2d_set_end_time(fvm2d_solver *s, double end_time);

/* setCFL (src/wrappers.cuh:127-130). */
int fvm2d_set_cfl(fvm2d_solver *s, double cfl);

/* setAlpha (src/wrappers.cuh:132-135): limiter parameter of the generalized minmod. */
int fvm2d_set_alpha(fvm2d_solver *s, double alpha);

/* setGamma (src/wrappers.cuh:137-140). */
int fvm2d_set_gamma(fvm2d_solver *s, double gamma);

/* setGhostCellStrategy (src/wrappers.cuh:142-145); strategy is an
 * fvm2d_ghost_strategy value. */
int fvm2d_set_ghost_strategy(fvm2d_solver *s, int strategy);

/* Selects the arithmetic build (fvm2d_precision); an uploaded state is kept
 * (converted when the storage type changes).  No reference counterpart. */
int fvm2d_set_precision(fvm2d_solver *s, int precision);

/* Uploads a state of ny x nx cells of `stride` doubles (4 or 5).  Replaces the
 * constructor's copy of U0 (src/wrappers.cuh:67-78) and the H2D copy in
 * solve() (src/wrappers.cuh:185).  Resets time and step counters of the
 * current run to zero. */
int fvm2d_set_state(fvm2d_solver *s, const double *cells, int stride);

/* The state as four planes, [4][ny][nx] doubles (rho, p, u, v), from or into
 * host or device memory (a (4, ny, nx) tensor, say).  No reference
 * counterpart: the reference takes vec5d rows only. */
int fvm2d_set_state_planes(fvm2d_solver *s, const double *planes);
int fvm2d_get_state_planes(fvm2d_solver *s, double *planes);

/* setRPInitialData (src/wrappers.cuh:80-108): four constant states (4 doubles
 * each: rho, p, u, v) split at column nx/2 and row ny/2 -- U2 | U1 over U3 | U4. */
int fvm2d_set_rp_initial_data(fvm2d_solver *s, const double *U1, const double *U2,
                              const double *U3, const double *U4);

/* Downloads the current state into ny x nx cells of `stride` doubles.
 * Replaces the D2H copy and result of solve() (src/wrappers.cuh:290-305). */
int fvm2d_get_state(fvm2d_solver *s, double *cells, int stride);

/* solve() (src/wrappers.cuh:154-306): runs the time loop from t = 0 on the
 * current state until the end time (or the step-size guard of
 * src/wrappers.cuh:204-207).  The result stays in the handle; like the
 * reference, a second call starts again from t = 0 on the previous result. */
int fvm2d_solve(fvm2d_solver *s);

/* Advances the current run by at most nsteps steps from its current time,
 * stopping early at the end time.  *steps_done (may be NULL) receives the
 * steps taken.  No reference counterpart (step granularity for checks and
 * benchmarks). */
int fvm2d_advance(fvm2d_solver *s, int nsteps, int *steps_done);

/* Health of the run (no reference counterpart: the reference checks
 * nothing).  *first_bad_step receives the number, counted from 1 since the
 * state was set, of the first step that left an interior cell with NaN or a
 * non-positive density or pressure; 0 if none has.  The run goes on either
 * way, as the reference's does. */
int fvm2d_get_health(fvm2d_solver *s, int *first_bad_step);

/* Conserved totals of the current state (no reference counterpart: the
 * reference has no diagnostics).  totals[0..3] (host or device memory)
 * receive the mass, x momentum, y momentum and energy of the interior cells
 * (rows and columns 2 .. n-3; for a row slab, its own rows), each the sum of
 * rho, rho u, rho v and p / (gamma - 1) + rho (u^2 + v^2) / 2 times the cell
 * area, computed in FP64 whatever the precision of the state, in a fixed
 * order: the same state gives the same bits.  The split step conserves the
 * mass exactly up to rounding; momentum and energy only up to the average of
 * the two split orders being taken in primitive variables
 * (src/basicFuns.cuh:264-274). */
int fvm2d_get_conserved_totals(fvm2d_solver *s, double *totals);

/* ---- frames and state files -----------------------------------------------
 * Frame recording replaces RGRP_2D_CUDA::setRecordModel / writeStagesTo_png
 * (src/wrappers.cuh:147-152, 253-260, 323-345): with recording on,
 * fvm2d_solve writes <dir>/<k>.png after step k for k = 0, gap, 2 gap, ...
 * (k counts from 0), density mapped to viridis over its min..max range.  The
 * frame shows the state after the step's ghost fill (the reference's, before
 * it).  PNG files are written without OpenCV or zlib (stored deflate). */
int fvm2d_set_record_model(fvm2d_solver *s, int on, int gap_per_frame, const char *dir);

/* The current density as a viridis PNG, as the recorder writes it. */
int fvm2d_write_frame_png(fvm2d_solver *s, const char *path);

/* State files (no reference counterpart): "FVM2DST1", int32 nx, int32 ny,
 * double t, int64 steps, then ny*nx cells of (rho, p, u, v) doubles.
 * fvm2d_read_state needs a solver of the same nx, ny; it sets the state, the
 * time and the step count, so fvm2d_advance continues the saved run. */
int fvm2d_write_state(fvm2d_solver *s, const char *path);
int fvm2d_read_state(fvm2d_solver *s, const char *path);

/* ---- row slabs (no reference counterpart) ---------------------------------
 * One problem split by rows across processes (2d_fvm_cuda_b200/slab.py): each
 * process holds a slab with two halo rows per inner edge, exchanges them
 * between steps and steps with a dt agreed across processes. */

/* One step with the caller's dt (the CFL rule applied by the caller, e.g.
 * over all slabs).  The ghost fill and time advance are as in fvm2d_advance. */
int fvm2d_advance_dt(fvm2d_solver *s, double dt);

/* Max over the cells of the current state of |(u, v)| + sqrt(gamma p / rho),
 * the quantity of the reference's CFL rule (src/basicFuns.cuh:215-226,
 * src/wrappers.cuh:198-202); halo rows of a slab are left out after a step. */
int fvm2d_get_wave_speed_max(fvm2d_solver *s, double *smax);

/* The array is rows row0 .. row0+ny-1 of a problem of ny_global rows whose
 * height is the spatial layout's: the row spacing is height / ny_global, the
 * presets see global row numbers, and they fill the top ghost rows (0, 1)
 * only if fill_top and the bottom ones only if fill_bottom.  Ring rows they do
 * not fill are halo rows, left out of the wave-speed max (their values are
 * the caller's to replace before the next step).  ny_global = 0 restores a
 * whole problem. */
int fvm2d_set_row_frame(fvm2d_solver *s, int row0, int ny_global, int fill_top, int fill_bottom);

/* Rows j0 .. j0+nrows-1 of the state as [4][nrows][nx] doubles (planes rho,
 * p, u, v), from or into host or device memory. */
int fvm2d_get_rows(fvm2d_solver *s, int j0, int nrows, double *rows);
int fvm2d_set_rows(fvm2d_solver *s, int j0, int nrows, const double *rows);

/* Asynchronous slab steps, for slabs on several devices whose halo exchange
 * and wave-speed reduction run on the device (NCCL, say): the calls below
 * only enqueue work on the handle's stream (*stream from fvm2d_get_stream, a
 * cudaStream_t) and return at once.  The caller enqueues its exchange and
 * reduction on that same stream between them, so no step waits on the host.
 *
 * fvm2d_get_rows_async / fvm2d_set_rows_async: as fvm2d_get_rows /
 * fvm2d_set_rows, device memory only.
 * fvm2d_slab_begin: starts a run from t = 0 with no step limit and writes
 * this slab's wave-speed max of the current state to *smax_out (device
 * memory, one double).
 * fvm2d_slab_step: one step whose dt follows the reference's rule
 * (src/wrappers.cuh:196-207) from *smax_in (device memory: the max over all
 * slabs of what fvm2d_slab_begin or the previous fvm2d_slab_step wrote) and
 * the handle's time, then writes this slab's wave-speed max of the new state
 * to *smax_out.  A step after the loop has ended (the end time reached)
 * does nothing.
 * fvm2d_slab_sync: waits for the stream and reads back the time, the steps
 * taken since fvm2d_slab_begin and whether the loop has ended. */
int fvm2d_get_stream(fvm2d_solver *s, void **stream);
int fvm2d_get_rows_async(fvm2d_solver *s, int j0, int nrows, double *rows);
int fvm2d_set_rows_async(fvm2d_solver *s, int j0, int nrows, const double *rows);
int fvm2d_slab_begin(fvm2d_solver *s, double *smax_out);
int fvm2d_slab_step(fvm2d_solver *s, const double *smax_in, double *smax_out);
int fvm2d_slab_sync(fvm2d_solver *s, double *t, int *steps, int *done);

/* getComputationTime_ms (src/wrappers.cuh:308-311): wall time of the last
 * solve()/advance() loop in milliseconds. */
int fvm2d_get_computation_time_ms(fvm2d_solver *s, double *ms);

/* getTimeStagesCount (src/wrappers.cuh:313-316): steps taken by all solve()
 * and advance() calls since the handle was created (the reference never
 * resets its counter either, src/wrappers.cuh:252). */
int fvm2d_get_time_stages_count(fvm2d_solver *s, long long *count);

/* Time and step count of the current run (no reference counterpart; the
 * reference keeps them in solve()'s locals, src/wrappers.cuh:191-196). */
int fvm2d_get_time(fvm2d_solver *s, double *t, int *steps, double *last_dt);

/* CUDA-event time (on the handle's stream) of the last solve()/advance()
 * loop, and the number of kernels it launched (graph replays launch every
 * captured kernel; steps after the loop ends exit at once).  No reference
 * counterpart: the reference times its loop on the host only
 * (src/wrappers.cuh:193,286-288). */
int fvm2d_get_run_stats(fvm2d_solver *s, double *device_ms, long long *kernel_launches);

/* Runs up to nsteps steps one at a time outside the graph, with CUDA events
 * between the five kernels of a step (sweep X, sweep Y, sweep Y, final sweep X
 * + average, ghost ring); kernel_ms[0..4] receive their mean durations in
 * milliseconds and *steps_done the steps taken.  Advances the state like
 * fvm2d_advance.  No reference counterpart (diagnostics). */
int fvm2d_profile_kernels(fvm2d_solver *s, int nsteps, double *kernel_ms, int *steps_done);

/* The current device's FP64 rate in TFLOP/s (2 flops per fused multiply-add):
 * a fully occupied grid of independent FMA chains, best of ten CUDA-event
 * timed launches (*ms_per_launch, may be NULL, receives that launch's time).
 * The FP64-pipe roofline of the sweeps is quoted against it.  No reference
 * counterpart (diagnostics). */
int fvm2d_measure_fp64_peak(double *tflops, double *ms_per_launch);

/* The FP64 product build's reciprocal and reciprocal square root (hardware
 * seeds refined by one third-order step instead of IEEE division and
 * square root) on n arguments in device memory: rcp[k] ~ 1/x[k],
 * rsqrt_out[k] ~ 1/sqrt(x[k]).  For tests of their error bound (within a
 * couple of ulp of the correctly rounded values).  No reference counterpart
 * (diagnostics). */
int fvm2d_eval_reciprocals(const double *x, long long n, double *rcp, double *rsqrt_out);

/* ---- differentiation (no reference counterpart) ----------------------------
 * Derivatives of the step with respect to the state, at a fixed step size so
 * the CFL maximum is not differentiated: fvm2d_forward / fvm2d_vjp on the
 * FVM2D_FP64 or FVM2D_FP32 build, fvm2d_jvp on FVM2D_FP64.  Branches of the
 * limiter and of the Riemann solver contribute the derivative of the branch
 * taken (almost everywhere). */

/* dt > 0: every step of this handle uses dt (no CFL rule; the run is bounded
 * by its step count, not by the end time).  0 restores the reference's CFL
 * rule. */
int fvm2d_set_fixed_dt(fvm2d_solver *s, double dt);

/* Tangent-linear model: advances the state nsteps steps and carries the
 * tangent (ny x nx cells of `stride` doubles) along; tangent_out receives the
 * tangent of the final state.  Requires FVM2D_FP64 and a fixed dt. */
int fvm2d_jvp(fvm2d_solver *s, int nsteps, const double *tangent_in, double *tangent_out, int stride);

/* Advances the state nsteps steps keeping `checkpoints` evenly spaced
 * copies of it (sqrt(nsteps) is the usual choice) for fvm2d_vjp; the last
 * segment, the first one the reverse needs, is taped as it runs.
 * checkpoints = FVM2D_FULL_TAPE keeps instead the whole tape: every step's
 * input state, X(U), Y(U) and interface fluxes, 7 states per step (8.4 MB x 7
 * per step at 512^2 in FP64), written by the forward steps themselves, so
 * that fvm2d_vjp recomputes nothing and may be called several times for one
 * forward.  Fails with FVM2D_ERR_INVALID when the tape does not fit in the
 * device's free memory. */
#define FVM2D_FULL_TAPE 0
int fvm2d_forward(fvm2d_solver *s, int nsteps, int checkpoints);

/* Adjoint of the last fvm2d_forward: given the cotangent of its final state,
 * returns in cotangent_out the cotangent of its initial state (the
 * vector-Jacobian product), recomputing each segment from its checkpoint (or
 * reading the full tape) and running the hand-written reverse step backwards
 * through it.  The state and time are those after fvm2d_forward when it
 * returns.  Changing a parameter (end time, CFL, alpha, gamma, preset,
 * layout, precision, row frame, step size) after a full-tape forward
 * discards its tape. */
int fvm2d_vjp(fvm2d_solver *s, const double *cotangent_in, double *cotangent_out, int stride);

/* With checkpoints, fvm2d_forward tapes its last segment as it runs and
 * fvm2d_vjp recomputes the others.  on != 0 (the default): where the device
 * has room for two segments' tapes, segment k-1 is recomputed on a second
 * stream while segment k is reversed; 0: one tape buffer, recompute and
 * reverse taking turns (half the tape memory).  The gradient is the same. */
int fvm2d_set_vjp_overlap(fvm2d_solver *s, int on);

/* ---- batched form (no reference counterpart) -------------------------------
 * Many independent problems of different sizes advance together: every stage
 * of the step is one launch covering all problems, each problem with its own
 * dt, end time and ghost preset, and the time loop is captured in CUDA
 * graphs.  Results match the same problems solved one by one with the same
 * precision bit for bit. */
typedef struct fvm2d_batch fvm2d_batch;

/* A batch of nproblems problems; problem p is nx[p] x ny[p] cells (ghosts
 * included, >= 6 each) on the current device.  Per-problem defaults as
 * fvm2d_create. */
int fvm2d_batch_create(fvm2d_batch **out, int nproblems, const int *nx, const int *ny);
int fvm2d_batch_destroy(fvm2d_batch *b);

/* The setters of the solver (setSpatialLayout, setTimeLayout, setAlpha,
 * setGamma, setGhostCellStrategy; src/wrappers.cuh:110-145) for problem p. */
int fvm2d_batch_set_problem(fvm2d_batch *b, int p, double width, double height, double t_end, double cfl,
                            double alpha, double gamma, int strategy);

/* Arithmetic build for all problems (fvm2d_precision); uploaded states are kept. */
int fvm2d_batch_set_precision(fvm2d_batch *b, int precision);

/* State of problem p in and out, as fvm2d_set_state / fvm2d_get_state. */
int fvm2d_batch_set_state(fvm2d_batch *b, int p, const double *cells, int stride);
int fvm2d_batch_get_state(fvm2d_batch *b, int p, double *cells, int stride);

/* Runs every problem from t = 0 to its end time (solve() of each,
 * src/wrappers.cuh:154-306, all at once). */
int fvm2d_batch_solve(fvm2d_batch *b);

/* Time reached and steps taken by problem p in the last solve. */
int fvm2d_batch_get_time(fvm2d_batch *b, int p, double *t, int *steps);

/* CUDA-event time of the last solve, kernels launched, and cell updates done
 * (sum over problems of nx * ny * steps). */
int fvm2d_batch_get_run_stats(fvm2d_batch *b, double *device_ms, long long *kernel_launches,
                              long long *cell_updates);

/* Times trial_steps steps of the batch for each candidate y-sweep segment
 * length (16, 32, 64 interfaces) and sweep grid size (1, 2, 4 times the
 * resident blocks), keeps the fastest and restores the states; reports the
 * choice. */
int fvm2d_batch_autotune(fvm2d_batch *b, int trial_steps, int *segment_interfaces, int *grid_blocks);

/* Largest nx * ny that fvm2d_advance_noalloc accepts. */
#define FVM2D_NOALLOC_MAX_CELLS 262144

/* Advances a state that lives in the caller's device memory by up to nsteps
 * FP64 split steps from time t0, without allocating any device memory.  No
 * counterpart in the reference (whose solve() allocates all its buffers).
 *
 * For callers that must not call cudaMalloc/cudaFree: applications whose
 * device memory belongs to their own allocator or fixed-budget arena, and
 * latency-critical loops that cannot pay for an allocation that may
 * synchronize the device.  The intermediate buffers of the sweeps and the
 * step-control record live in one static device array of the library, sized
 * for FVM2D_NOALLOC_MAX_CELLS cells (16 MiB + 256 B per GPU that loads the
 * library, held until exit); larger states are rejected with
 * FVM2D_ERR_INVALID.
 *
 * state_in, state_out: device memory, 4 planes (rho, p, u, v) of ny x nx
 *   doubles each, row-major, planes back to back; they may be the same
 *   buffer, but two buffers that overlap only in part are rejected with
 *   FVM2D_ERR_INVALID.  The result (and the whole ring of ghost cells) lands
 *   in state_out.
 * Parameters as the solver setters (fvm2d_set_spatial_layout, ...), t_end
 *   bounding the run as the reference's end time does; *t_out and
 *   *steps_out (may be NULL) receive the time reached and the steps taken.
 * stream: a cudaStream_t (NULL for the default stream); the call returns
 *   after the work on it has finished.  Steps are enqueued in groups of 32
 *   with a read of the step-control record after each group, so a run that
 *   reaches t_end early stops within 32 steps of it: nsteps may be a generous
 *   upper bound.
 * The call waits for its own work, so it cannot run inside a stream capture:
 *   a call on a stream that is being captured is rejected with
 *   FVM2D_ERR_INVALID.
 * The first call on each device finds the device address of the static
 * array and sets kernel attributes.  All calls share the array: calls whose
 * GPU work overlaps race on it, so serialize them. */
int fvm2d_advance_noalloc(const double *state_in, double *state_out, int nx, int ny, double width, double height,
                          double t_end, double cfl, double alpha, double gamma, int strategy, double t0,
                          int nsteps, void *stream, double *t_out, int *steps_out);

#ifdef __cplusplus
}
#endif
#endif /* FVM2D_H */
