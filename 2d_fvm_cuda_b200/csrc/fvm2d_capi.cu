// fvm2d_capi.cu -- host runtime behind include/fvm2d.h.
//
// A handle owns, on one device:
//   U        the state: 4 planes (rho, p, u, v), rows padded to `pitch`
//            elements (a multiple of 32) so every row starts 256-byte aligned;
//   scratch  two more state-sized buffers (A, B) that the sweeps write, also
//            used as the staging area for uploads and downloads;
//   ctl      the device-resident StepControl of the time loop;
//   CUDA graphs of 16 steps and of 1 step (5 kernels each) replayed until
//   the control record says the loop has ended, so the only host round trip
//   is one 64-byte read per graph replay (the reference reads the max wave
//   speed back and synchronizes 17 times per step, src/wrappers.cuh:196-284);
//   and, allocated on first use, the differentiation workspaces (dual-number
//   states of fvm2d_jvp; checkpoints, one segment's tape (or, for a
//   full-tape forward, every step's) and the adjoint states of
//   fvm2d_forward / fvm2d_vjp, with graphs of a full segment).
#include "../../include/fvm2d.h"
#include "fvm2d_io.cuh"
#include "fvm2d_adjoint.h"
#include "fvm2d_control.h"
#include "fvm2d_dual.cuh"
#include "fvm2d_transfer.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <new>
#include <string>
#include <utility>
#include <vector>

using fvm2d::LaunchConfig;
using fvm2d::StepControl;
using fvm2d::aos_to_soa;
using fvm2d::conserved_partials;
using fvm2d::conserved_sum;
using fvm2d::convert_planes;
using fvm2d::is_device_pointer;
using fvm2d::rows_in;
using fvm2d::rows_out;
using fvm2d::soa_to_aos;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    // clear a pending error that is not sticky (a failed allocation, say), so
    // that it is not reported again by the next call's launch checks
    cudaGetLastError();
    return fail(FVM2D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                   \
    } while (0)

// An NVTX range over a library call (visible in nsys / ncu; no cost without
// a profiler attached).
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

struct Variant {
    cudaError_t (*prepare)();
    cudaError_t (*init)(const LaunchConfig &, cudaStream_t);
    cudaError_t (*plan)(const LaunchConfig &, cudaStream_t);
    cudaError_t (*step)(const LaunchConfig &, cudaStream_t, cudaEvent_t *);
    cudaError_t (*plan_from)(const LaunchConfig &, cudaStream_t, const double *);
};

#define FVM2D_VARIANT_ENTRY(ns)                                                                        \
    {fvm2d::ns::prepare, fvm2d::ns::enqueue_init, fvm2d::ns::enqueue_plan, fvm2d::ns::enqueue_step,     \
     fvm2d::ns::enqueue_plan_from}
const Variant kVariants[] = {FVM2D_VARIANT_ENTRY(fp64), FVM2D_VARIANT_ENTRY(fp64_strict),
                             FVM2D_VARIANT_ENTRY(fp64_reforder), FVM2D_VARIANT_ENTRY(fp32),
                             FVM2D_VARIANT_ENTRY(fp32r)};
// the tangent-linear build (dual numbers), used by fvm2d_jvp only
const Variant kJvp = FVM2D_VARIANT_ENTRY(jvp);
#undef FVM2D_VARIANT_ENTRY

using fvm2d::ad::Dual;

// (value planes, tangent planes) <-> dual planes
__global__ void pack_dual(const double *__restrict__ v, const double *__restrict__ t, Dual *__restrict__ out, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        out[k] = Dual(v[k], t[k]);
}

__global__ void unpack_dual(const Dual *__restrict__ in, double *__restrict__ v, double *__restrict__ t, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        v[k] = in[k].v;
        t[k] = in[k].d;
    }
}

// Element type of the state planes for a precision: FP32 stores floats (and
// FP32_RESIDUAL floats followed by 16-bit residual planes), the FP64 builds
// doubles.  Host-side states are always doubles.
bool is_fp32(int precision) { return precision == FVM2D_FP32; }
bool float_planes(int precision) { return precision == FVM2D_FP32 || precision == FVM2D_FP32_RESIDUAL; }
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Storage of a precision's state planes: 0 doubles, 1 floats, 2 floats with
// 16-bit residual planes; and the bytes of one state.
int storage_of(int precision) { return precision == FVM2D_FP32 ? 1 : precision == FVM2D_FP32_RESIDUAL ? 2 : 0; }
size_t state_bytes(int precision, long long plane)
{
    static const size_t per_element[3] = {sizeof(double), sizeof(float), sizeof(float) + sizeof(unsigned short)};
    return (size_t)4 * plane * per_element[storage_of(precision)];
}

// Calls f with the storage policy (fvm2d_split.cuh) of a state buffer of the
// given precision, for the transfer kernels.
template <class F>
void with_planes(int precision, const void *state, long long plane, F &&f)
{
    void *U = const_cast<void *>(state);
    if (precision == FVM2D_FP32)
        f(fvm2d::Planes<float>{static_cast<float *>(U)});
    else if (precision == FVM2D_FP32_RESIDUAL)
        f(fvm2d::split_planes(U, plane));
    else
        f(fvm2d::Planes<double>{static_cast<double *>(U)});
}

} // namespace

int fvm2d::report_error(int code, const char *msg) { return fail(code, msg); }

struct fvm2d_solver {
    int device = 0;
    int nx = 0, ny = 0, pitch = 0;
    long long plane = 0;
    double width = 1.0, height = 1.0, t_end = 0.0, cfl = 0.5, alpha = 1.9, gamma = 1.4;
    int strategy = FVM2D_OUTFLOW;
    int precision = FVM2D_FP64;
    cudaStream_t stream = nullptr;
    double *U = nullptr;
    double *scratch = nullptr;  // A then B
    StepControl *ctl = nullptr;
    StepControl *ctl_h = nullptr;  // pinned mirror
    // replayed graphs: kGraphSteps[g] steps each; built on first use for the
    // current precision and parameters, dropped by every setter
    static constexpr int kGraphSteps[2] = {16, 1};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_variant = -1;
    bool have_state = false;
    bool need_init = true;
    double fixed_dt = 0.0;        // > 0: differentiation runs step with this constant dt
    int row0 = 0, ny_global = 0, fill_top = 1, fill_bottom = 1;  // row frame of a slab (fvm2d_set_row_frame)
    bool record_on = false;       // frames during fvm2d_solve (fvm2d_set_record_model)
    int record_gap = 10;
    std::string record_dir = ".";
    // differentiation workspaces (allocated on first use)
    void *dual = nullptr;         // 3 state buffers of dual numbers (jvp)
    char *ckpt = nullptr;         // checkpoints of fvm2d_forward (states of the build's type)
    char *tape = nullptr;         // one or two segments' steps, recomputed by fvm2d_vjp (or every step,
                                  // written by a full-tape fvm2d_forward): per step its input state, X(U),
                                  // Y(U) and the fluxes of its four sweeps
    char *adj = nullptr;          // adjoint work: 2 adjoints, 3 work states, the saved final state
    size_t ck_bytes = 0, tape_bytes = 0, adj_bytes = 0;
    int ck_count = 0, ck_len = 0, fwd_steps = -1, fwd_precision = -1;
    bool full_tape = false;       // the last fvm2d_forward kept every step's tape
    // the graphs of a full checkpoint segment: its taped recompute into tape
    // buffer b ([b]), its reverse from tape buffer b starting from adjoint
    // buffer a ([2 + 2b + a]), and its untaped forward steps ([6], for
    // fvm2d_forward); built for vjp_len steps and vjp_bufs tape buffers
    cudaGraphExec_t vjp_graph[7] = {};
    int vjp_len = 0, vjp_bufs = 0;
    bool last_taped = false;      // the checkpointed forward taped its last segment (fvm2d_vjp skips its recompute)
    bool vjp_overlap = true;      // fvm2d_set_vjp_overlap: two tape buffers where they fit
    // with two tape buffers fvm2d_vjp recomputes the next segment on `aux`
    // while the current one is reversed on `stream`; vjp_ev[b] marks tape
    // buffer b filled, vjp_ev[2 + b] free again, vjp_ev[4] the start
    cudaStream_t aux = nullptr;
    cudaEvent_t vjp_ev[5] = {};
    // the adjoint step's fork stream and events (AdjointLaunch::fork)
    cudaStream_t fork = nullptr;
    cudaEvent_t fork_ev[2] = {};
    std::vector<double> ck_t;     // time at each checkpoint
    double last_ms = 0.0;         // wall time of the last loop (the reference's timer)
    double last_device_ms = 0.0;  // CUDA-event time of the last loop on the stream
    long long last_launches = 0;  // kernels launched by the last loop
    long long total_steps = 0;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;

    LaunchConfig config() const
    {
        LaunchConfig c;
        c.nx = nx;
        c.ny = ny;
        c.pitch = pitch;
        c.plane = plane;
        c.U = U;
        c.A = scratch;
        c.B = scratch + 4 * plane;
        c.ctl = ctl;
        c.hx = width / double(nx);
        c.hy = height / double(ny_global > 0 ? ny_global : ny);  // a slab keeps the problem's row spacing
        c.rhx = 1.0 / c.hx;
        c.rhy = 1.0 / c.hy;
        c.alpha = alpha;
        c.gamma = gamma;
        c.strategy = strategy;
        c.plan.t_end = t_end;
        c.plan.cfl = cfl;
        c.plan.hmin = (c.hy < c.hx) ? c.hy : c.hx;
        c.plan.fixed_dt = fixed_dt;
        c.row0 = row0;
        c.ny_global = ny_global;
        c.fill_top = fill_top;
        c.fill_bottom = fill_bottom;
        return c;
    }

    void drop_graph()
    {
        for (auto &g : graph) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
        graph_variant = -1;
        drop_vjp_graphs();
        last_taped = false;  // taped with the former parameters
        if (full_tape) {  // a parameter changed: the tape no longer belongs to this solver's step
            full_tape = false;
            fwd_steps = -1;
        }
    }

    void drop_vjp_graphs()
    {
        for (auto &g : vjp_graph) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
        vjp_len = 0;
        vjp_bufs = 0;
    }

    // Captures what `enqueue` puts on the stream into *out.
    template <class F>
    int capture(cudaGraphExec_t *out, F &&enqueue)
    {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue();
        cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
        cudaError_t e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            *out = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        return FVM2D_OK;
    }

    int build_graphs()
    {
        if (graph_variant == precision && graph[0] && graph[1]) return FVM2D_OK;
        drop_graph();
        const LaunchConfig c = config();
        for (int which = 0; which < 2; ++which) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaSuccess;
            for (int k = 0; k < kGraphSteps[which] && e == cudaSuccess; ++k)
                e = kVariants[precision].step(c, stream, nullptr);
            cudaError_t e2 = cudaStreamEndCapture(stream, &g);
            if (e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return cuda_fail(e, "capture of the step kernels");
            }
            if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&graph[which], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                graph[which] = nullptr;
                return cuda_fail(e, "cudaGraphInstantiate");
            }
        }
        graph_variant = precision;
        return FVM2D_OK;
    }

    // Replays the step graphs until the control record says no step is in
    // flight.  The record on the device must already be planned; `first`
    // kernels (init or plan) were enqueued just before.
    // `budget` bounds the steps this loop may start; the long graph is
    // replayed while at least its length remains, then the one-step graph.
    int loop(int first, long long budget)
    {
        int rc = build_graphs();
        if (rc) return rc;
        auto t0 = std::chrono::high_resolution_clock::now();
        long long launches = first;
        for (;;) {
            const int which = budget >= kGraphSteps[0] ? 0 : 1;
            CK(cudaGraphLaunch(graph[which], stream));
            budget -= kGraphSteps[which];
            launches += (long long)kGraphSteps[which] * fvm2d::kStepKernels;
            CK(cudaMemcpyAsync(ctl_h, ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            if (!ctl_h->active) break;
        }
        CK(cudaEventRecord(ev_end, stream));
        CK(cudaEventSynchronize(ev_end));
        auto t1 = std::chrono::high_resolution_clock::now();
        last_ms = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() / 1000.0;
        float dms = 0.f;
        CK(cudaEventElapsedTime(&dms, ev_begin, ev_end));
        last_device_ms = dms;
        last_launches = launches;
        return FVM2D_OK;
    }

    int upload_control()
    {
        CK(cudaMemcpyAsync(ctl, ctl_h, sizeof(StepControl), cudaMemcpyHostToDevice, stream));
        return FVM2D_OK;
    }
};

namespace {

int check(fvm2d_solver *s)
{
    if (!s) return fail(FVM2D_ERR_INVALID, "null solver handle");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return FVM2D_OK;
}

int upload(fvm2d_solver *s, const double *cells, int stride)
{
    const size_t bytes = sizeof(double) * (size_t)s->nx * s->ny * stride;
    const cudaMemcpyKind kind = is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(s->scratch, cells, bytes, kind, s->stream));
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        aos_to_soa<<<148 * 4, 256, 0, s->stream>>>(s->scratch, stride, st, s->nx, s->ny, s->pitch, s->plane);
    });
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    s->have_state = true;
    s->need_init = true;
    std::memset(s->ctl_h, 0, sizeof(StepControl));
    return FVM2D_OK;
}

} // namespace

extern "C" {
#pragma GCC visibility push(default)

const char *fvm2d_last_error(void) { return g_err.c_str(); }

const char *fvm2d_version(void) { return "fvm2d-b200 0.1 (sm_100a)"; }

int fvm2d_create(fvm2d_solver **out, int nx, int ny)
{
    if (!out) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (nx < 6 || ny < 6) return fail(FVM2D_ERR_INVALID, "nx and ny must be at least 6 (two ghost layers per side)");
    if ((long long)nx * ny > (1ll << 31) - 1) return fail(FVM2D_ERR_INVALID, "nx * ny must stay below 2^31");
    if ((long long)((nx + 31) / 32 * 32) * ny > (1ll << 31) - 1)
        return fail(FVM2D_ERR_INVALID, "the padded plane, round_up(nx, 32) * ny, must stay below 2^31");
    fvm2d_solver *s = new (std::nothrow) fvm2d_solver();
    if (!s) return fail(FVM2D_ERR_INVALID, "out of host memory");
    cudaError_t e = cudaGetDevice(&s->device);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(e, "cudaGetDevice");
    }
    s->nx = nx;
    s->ny = ny;
    s->pitch = (nx + 31) / 32 * 32;
    s->plane = (long long)s->pitch * ny;
    const size_t state_bytes = sizeof(double) * 4 * (size_t)s->plane;
    int rc = FVM2D_OK;
    do {
        for (int v = 0; v < kNumVariants && !rc; ++v)
            if ((e = kVariants[v].prepare()) != cudaSuccess) rc = cuda_fail(e, "kernel attributes");
        if (rc) break;
        if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking))) { rc = cuda_fail(e, "cudaStreamCreate"); break; }
        if ((e = cudaMalloc(&s->U, state_bytes))) { rc = cuda_fail(e, "cudaMalloc(state)"); break; }
        if ((e = cudaMalloc(&s->scratch, 2 * state_bytes))) { rc = cuda_fail(e, "cudaMalloc(scratch)"); break; }
        if ((e = cudaMalloc(&s->ctl, sizeof(StepControl)))) { rc = cuda_fail(e, "cudaMalloc(control)"); break; }
        if ((e = cudaMallocHost(&s->ctl_h, sizeof(StepControl)))) { rc = cuda_fail(e, "cudaMallocHost"); break; }
        if ((e = cudaEventCreate(&s->ev_begin)) || (e = cudaEventCreate(&s->ev_end))) { rc = cuda_fail(e, "cudaEventCreate"); break; }
        std::memset(s->ctl_h, 0, sizeof(StepControl));
        if ((e = cudaMemsetAsync(s->U, 0, state_bytes, s->stream))) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((e = cudaMemsetAsync(s->scratch, 0, 2 * state_bytes, s->stream))) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((e = cudaMemsetAsync(s->ctl, 0, sizeof(StepControl), s->stream))) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((e = cudaStreamSynchronize(s->stream))) { rc = cuda_fail(e, "cudaStreamSynchronize"); break; }
    } while (0);
    if (rc) {
        fvm2d_destroy(s);
        return rc;
    }
    *out = s;
    return FVM2D_OK;
}

int fvm2d_destroy(fvm2d_solver *s)
{
    if (!s) return FVM2D_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->drop_graph();
    if (s->U) cudaFree(s->U);
    if (s->scratch) cudaFree(s->scratch);
    if (s->ctl) cudaFree(s->ctl);
    if (s->ctl_h) cudaFreeHost(s->ctl_h);
    if (s->dual) cudaFree(s->dual);
    if (s->ckpt) cudaFree(s->ckpt);
    if (s->tape) cudaFree(s->tape);
    if (s->adj) cudaFree(s->adj);
    if (s->ev_begin) cudaEventDestroy(s->ev_begin);
    if (s->ev_end) cudaEventDestroy(s->ev_end);
    for (auto &e : s->vjp_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : s->fork_ev)
        if (e) cudaEventDestroy(e);
    if (s->fork) {
        cudaStreamSynchronize(s->fork);
        cudaStreamDestroy(s->fork);
    }
    if (s->aux) {
        cudaStreamSynchronize(s->aux);
        cudaStreamDestroy(s->aux);
    }
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FVM2D_OK;
}

#define SETTER(name, field, type, cond, msg)                                  \
    int name(fvm2d_solver *s, type v)                                          \
    {                                                                          \
        if (int rc = check(s)) return rc;                                      \
        if (!(cond)) return fail(FVM2D_ERR_INVALID, msg);                      \
        s->field = v;                                                          \
        s->drop_graph();                                                       \
        return FVM2D_OK;                                                       \
    }

SETTER(fvm2d_set_end_time, t_end, double, v == v, "end time must be a number")
SETTER(fvm2d_set_cfl, cfl, double, v > 0.0, "CFL must be positive")
SETTER(fvm2d_set_alpha, alpha, double, v == v, "alpha must be a number")
SETTER(fvm2d_set_gamma, gamma, double, v > 1.0, "gamma must exceed 1")
SETTER(fvm2d_set_ghost_strategy, strategy, int, v >= FVM2D_OUTFLOW && v <= FVM2D_REFLECTIVE_TB,
       "unknown ghost-cell strategy")
int fvm2d_set_precision(fvm2d_solver *s, int v)
{
    if (int rc = check(s)) return rc;
    if (!(v >= 0 && v < kNumVariants)) return fail(FVM2D_ERR_INVALID, "unknown precision");
    if (s->have_state && storage_of(v) != storage_of(s->precision)) {
        // keep the current state: convert its planes to the new storage type
        const long long n = 4 * s->plane;
        with_planes(s->precision, s->U, s->plane, [&](auto from) {
            with_planes(v, s->scratch, s->plane, [&](auto to) {
                convert_planes<<<148 * 4, 256, 0, s->stream>>>(from, to, n);
            });
        });
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(s->U, s->scratch, state_bytes(v, s->plane), cudaMemcpyDeviceToDevice, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    s->precision = v;
    s->drop_graph();
    return FVM2D_OK;
}

int fvm2d_set_spatial_layout(fvm2d_solver *s, double width, double height)
{
    if (int rc = check(s)) return rc;
    if (!(width > 0.0 && height > 0.0)) return fail(FVM2D_ERR_INVALID, "width and height must be positive");
    s->width = width;
    s->height = height;
    s->drop_graph();
    return FVM2D_OK;
}

int fvm2d_set_time_layout(fvm2d_solver *s, double end_time, double cfl)
{
    if (int rc = fvm2d_set_end_time(s, end_time)) return rc;
    return fvm2d_set_cfl(s, cfl);
}

int fvm2d_set_state(fvm2d_solver *s, const double *cells, int stride)
{
    Range range_("fvm2d_set_state");
    if (int rc = check(s)) return rc;
    if (!cells) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    return upload(s, cells, stride);
}

int fvm2d_set_state_planes(fvm2d_solver *s, const double *planes)
{
    if (int rc = check(s)) return rc;
    if (!planes) return fail(FVM2D_ERR_INVALID, "null state pointer");
    CK(cudaMemcpyAsync(s->scratch, planes, sizeof(double) * 4 * (size_t)s->nx * s->ny, cudaMemcpyDefault, s->stream));
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        rows_in<<<148 * 4, 256, 0, s->stream>>>(st, s->plane, s->pitch, 0, s->ny, s->nx, s->scratch);
    });
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    s->have_state = true;
    s->need_init = true;
    std::memset(s->ctl_h, 0, sizeof(StepControl));
    return FVM2D_OK;
}

int fvm2d_get_state_planes(fvm2d_solver *s, double *planes)
{
    if (int rc = check(s)) return rc;
    if (!planes) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    return fvm2d_get_rows(s, 0, s->ny, planes);
}

int fvm2d_set_rp_initial_data(fvm2d_solver *s, const double *U1, const double *U2, const double *U3,
                              const double *U4)
{
    if (int rc = check(s)) return rc;
    if (!U1 || !U2 || !U3 || !U4) return fail(FVM2D_ERR_INVALID, "null quadrant state");
    std::vector<double> cells;
    try {
        cells.resize((size_t)s->nx * s->ny * 4);
    } catch (...) {
        return fail(FVM2D_ERR_INVALID, "out of host memory");
    }
    for (int j = 0; j < s->ny; ++j)
        for (int i = 0; i < s->nx; ++i) {
            // src/wrappers.cuh:90-105
            const double *q = (i < s->nx / 2) ? (j < s->ny / 2 ? U2 : U3) : (j < s->ny / 2 ? U1 : U4);
            std::memcpy(&cells[((size_t)j * s->nx + i) * 4], q, 4 * sizeof(double));
        }
    return upload(s, cells.data(), 4);
}

int fvm2d_get_state(fvm2d_solver *s, double *cells, int stride)
{
    Range range_("fvm2d_get_state");
    if (int rc = check(s)) return rc;
    if (!cells) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        soa_to_aos<<<148 * 4, 256, 0, s->stream>>>(st, s->nx, s->ny, s->pitch, s->plane, stride, s->scratch);
    });
    CK(cudaGetLastError());
    const size_t bytes = sizeof(double) * (size_t)s->nx * s->ny * stride;
    const cudaMemcpyKind kind = is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(cells, s->scratch, bytes, kind, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FVM2D_OK;
}

static int write_frame(fvm2d_solver *s, const char *path);

// fvm2d_solve with frames: one after the first step, then one every `gap`
// steps, named by the index of the step they follow (src/wrappers.cuh:
// 194-195, 253-263); the frame shows the state after that step's ghost fill.
static int solve_recording(fvm2d_solver *s)
{
    std::error_code ec;
    std::filesystem::create_directories(s->record_dir, ec);
    StepControl *c = s->ctl_h;
    const LaunchConfig cfg = s->config();
    auto t0 = std::chrono::high_resolution_clock::now();
    double device_ms = 0.0;
    long long launches = 0;
    int target = 1;
    c->step_limit = target;
    if (int rc = s->upload_control()) return rc;
    CK(cudaEventRecord(s->ev_begin, s->stream));
    CK(kVariants[s->precision].init(cfg, s->stream));
    s->need_init = false;
    for (;;) {
        if (int rc = s->loop(1, target - c->steps)) return rc;
        device_ms += s->last_device_ms;
        launches += s->last_launches;
        if (c->steps == target) {
            const std::string path = s->record_dir + "/" + std::to_string(target - 1) + ".png";
            if (int rc = write_frame(s, path.c_str())) return rc;
        }
        if (c->done || c->steps < target || s->record_gap <= 0) break;
        target += s->record_gap;
        c->step_limit = target;
        c->active = 0;
        if (int rc = s->upload_control()) return rc;
        CK(cudaEventRecord(s->ev_begin, s->stream));
        CK(kVariants[s->precision].plan(cfg, s->stream));
    }
    if (s->record_gap <= 0 && !c->done) {  // the reference records only its first step then
        c->step_limit = INT_MAX;
        c->active = 0;
        if (int rc = s->upload_control()) return rc;
        CK(cudaEventRecord(s->ev_begin, s->stream));
        CK(kVariants[s->precision].plan(cfg, s->stream));
        if (int rc = s->loop(1, LLONG_MAX)) return rc;
        device_ms += s->last_device_ms;
        launches += s->last_launches;
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    s->last_ms = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() / 1000.0;
    s->last_device_ms = device_ms;
    s->last_launches = launches;
    return FVM2D_OK;
}

int fvm2d_solve(fvm2d_solver *s)
{
    Range range_("fvm2d_solve");
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    StepControl *c = s->ctl_h;
    std::memset(c, 0, sizeof(StepControl));
    c->step_limit = INT_MAX;
    const LaunchConfig cfg = s->config();
    if (int rc = s->build_graphs()) return rc;
    if (s->record_on) {
        if (int rc = solve_recording(s)) return rc;
        s->total_steps += c->steps;
        return FVM2D_OK;
    }
    if (int rc = s->upload_control()) return rc;
    CK(cudaEventRecord(s->ev_begin, s->stream));
    CK(kVariants[s->precision].init(cfg, s->stream));
    s->need_init = false;
    if (int rc = s->loop(1, LLONG_MAX)) return rc;
    s->total_steps += c->steps;
    return FVM2D_OK;
}

int fvm2d_advance(fvm2d_solver *s, int nsteps, int *steps_done)
{
    Range range_("fvm2d_advance");
    if (steps_done) *steps_done = 0;
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (nsteps < 0) return fail(FVM2D_ERR_INVALID, "nsteps must be non-negative");
    StepControl *c = s->ctl_h;
    const int before = c->steps;
    c->step_limit = (before > INT_MAX - nsteps) ? INT_MAX : before + nsteps;
    c->done = 0;
    c->active = 0;
    if (int rc = s->upload_control()) return rc;
    const LaunchConfig cfg = s->config();
    if (int rc = s->build_graphs()) return rc;
    CK(cudaEventRecord(s->ev_begin, s->stream));
    if (s->need_init) {
        CK(kVariants[s->precision].init(cfg, s->stream));
        s->need_init = false;
    } else {
        CK(kVariants[s->precision].plan(cfg, s->stream));
    }
    if (int rc = s->loop(1, nsteps)) return rc;
    s->total_steps += c->steps - before;
    if (steps_done) *steps_done = c->steps - before;
    return FVM2D_OK;
}

int fvm2d_advance_dt(fvm2d_solver *s, double dt)
{
    Range range_("fvm2d_advance_dt");
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(FVM2D_ERR_INVALID, "dt must be positive and finite");
    const LaunchConfig cfg = s->config();
    if (int rc = s->build_graphs()) return rc;
    StepControl *c = s->ctl_h;
    if (s->need_init) {  // wave-speed max of the fresh state; the device record becomes the reference
        CK(kVariants[s->precision].init(cfg, s->stream));
        s->need_init = false;
        CK(cudaMemcpyAsync(c, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    c->dt = dt;
    c->active = 1;
    c->done = 0;
    c->step_limit = c->steps + 1;
    if (int rc = s->upload_control()) return rc;
    CK(cudaEventRecord(s->ev_begin, s->stream));
    CK(cudaGraphLaunch(s->graph[1], s->stream));
    CK(cudaMemcpyAsync(c, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaEventRecord(s->ev_end, s->stream));
    CK(cudaEventSynchronize(s->ev_end));
    float dms = 0.f;
    CK(cudaEventElapsedTime(&dms, s->ev_begin, s->ev_end));
    s->last_device_ms = dms;
    s->last_launches = fvm2d::kStepKernels;
    s->total_steps += 1;
    return FVM2D_OK;
}

int fvm2d_get_wave_speed_max(fvm2d_solver *s, double *smax)
{
    if (int rc = check(s)) return rc;
    if (!smax) return fail(FVM2D_ERR_INVALID, "null output pointer");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (s->need_init) {
        CK(kVariants[s->precision].init(s->config(), s->stream));
        s->need_init = false;
        CK(cudaMemcpyAsync(s->ctl_h, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    *smax = s->ctl_h->smax_last;
    return FVM2D_OK;
}

int fvm2d_set_row_frame(fvm2d_solver *s, int row0, int ny_global, int fill_top, int fill_bottom)
{
    if (int rc = check(s)) return rc;
    if (ny_global == 0) {
        row0 = 0;
        fill_top = fill_bottom = 1;
    } else if (row0 < 0 || ny_global < row0 + s->ny) {
        return fail(FVM2D_ERR_INVALID, "the slab must lie inside the global rows: 0 <= row0, row0 + ny <= ny_global");
    }
    s->row0 = row0;
    s->ny_global = ny_global;
    s->fill_top = fill_top ? 1 : 0;
    s->fill_bottom = fill_bottom ? 1 : 0;
    s->drop_graph();
    return FVM2D_OK;
}

static int rows_check(fvm2d_solver *s, int j0, int nrows, const void *buf)
{
    if (int rc = check(s)) return rc;
    if (!buf) return fail(FVM2D_ERR_INVALID, "null row buffer");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (j0 < 0 || nrows < 1 || j0 + nrows > s->ny) return fail(FVM2D_ERR_INVALID, "rows out of range");
    return FVM2D_OK;
}

int fvm2d_get_rows(fvm2d_solver *s, int j0, int nrows, double *rows)
{
    if (int rc = rows_check(s, j0, nrows, rows)) return rc;
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        rows_out<<<148 * 4, 256, 0, s->stream>>>(st, s->plane, s->pitch, j0, nrows, s->nx, s->scratch);
    });
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rows, s->scratch, sizeof(double) * 4 * (size_t)nrows * s->nx, cudaMemcpyDefault, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FVM2D_OK;
}

int fvm2d_set_rows(fvm2d_solver *s, int j0, int nrows, const double *rows)
{
    if (int rc = rows_check(s, j0, nrows, rows)) return rc;
    CK(cudaMemcpyAsync(s->scratch, rows, sizeof(double) * 4 * (size_t)nrows * s->nx, cudaMemcpyDefault, s->stream));
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        rows_in<<<148 * 4, 256, 0, s->stream>>>(st, s->plane, s->pitch, j0, nrows, s->nx, s->scratch);
    });
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    return FVM2D_OK;
}

// ---- row slabs on several devices: asynchronous steps ------------------------
// The calls below enqueue on the handle's stream and return at once; the
// caller orders its own work (a halo exchange, a max-reduction over the slabs,
// e.g. NCCL on a torch stream wrapping fvm2d_get_stream's stream) on the same
// stream, so a slab step never waits on the host.

int fvm2d_get_stream(fvm2d_solver *s, void **stream)
{
    if (int rc = check(s)) return rc;
    if (!stream) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *stream = static_cast<void *>(s->stream);
    return FVM2D_OK;
}

int fvm2d_get_rows_async(fvm2d_solver *s, int j0, int nrows, double *rows)
{
    if (int rc = rows_check(s, j0, nrows, rows)) return rc;
    if (!is_device_pointer(rows)) return fail(FVM2D_ERR_INVALID, "the row buffer must be device memory");
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        rows_out<<<148 * 4, 256, 0, s->stream>>>(st, s->plane, s->pitch, j0, nrows, s->nx, rows);
    });
    CK(cudaGetLastError());
    return FVM2D_OK;
}

int fvm2d_set_rows_async(fvm2d_solver *s, int j0, int nrows, const double *rows)
{
    if (int rc = rows_check(s, j0, nrows, rows)) return rc;
    if (!is_device_pointer(rows)) return fail(FVM2D_ERR_INVALID, "the row buffer must be device memory");
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        rows_in<<<148 * 4, 256, 0, s->stream>>>(st, s->plane, s->pitch, j0, nrows, s->nx, rows);
    });
    CK(cudaGetLastError());
    return FVM2D_OK;
}

int fvm2d_slab_begin(fvm2d_solver *s, double *smax_out)
{
    Range range_("fvm2d_slab_begin");
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (!smax_out || !is_device_pointer(smax_out)) return fail(FVM2D_ERR_INVALID, "smax_out must be device memory");
    StepControl *c = s->ctl_h;
    std::memset(c, 0, sizeof(StepControl));
    c->step_limit = INT_MAX;
    if (int rc = s->upload_control()) return rc;
    if (int rc = s->build_graphs()) return rc;
    CK(kVariants[s->precision].init(s->config(), s->stream));
    s->need_init = false;
    CK(cudaMemcpyAsync(smax_out, &s->ctl->smax_last, sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    return FVM2D_OK;
}

int fvm2d_slab_step(fvm2d_solver *s, const double *smax_in, double *smax_out)
{
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (!smax_in || !smax_out || !is_device_pointer(smax_in) || !is_device_pointer(smax_out))
        return fail(FVM2D_ERR_INVALID, "smax_in and smax_out must be device memory");
    if (s->graph_variant != s->precision || !s->graph[1])
        return fail(FVM2D_ERR_STATE, "fvm2d_slab_begin must come first (and again after a setter)");
    CK(kVariants[s->precision].plan_from(s->config(), s->stream, smax_in));
    CK(cudaGraphLaunch(s->graph[1], s->stream));
    CK(cudaMemcpyAsync(smax_out, &s->ctl->smax_last, sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    s->total_steps += 1;
    return FVM2D_OK;
}

int fvm2d_slab_sync(fvm2d_solver *s, double *t, int *steps, int *done)
{
    if (int rc = check(s)) return rc;
    CK(cudaMemcpyAsync(s->ctl_h, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (t) *t = s->ctl_h->t;
    if (steps) *steps = s->ctl_h->steps;
    if (done) *done = s->ctl_h->done;
    return FVM2D_OK;
}

// ---- frames and state files ---------------------------------------------------
static int write_frame(fvm2d_solver *s, const char *path)
{
    constexpr int NT = 256;
    const long long n = (long long)s->nx * s->ny;
    long long blocks = (n + NT - 1) / NT;
    if (blocks > 148 * 4) blocks = 148 * 4;
    float *parts = reinterpret_cast<float *>(s->scratch);
    unsigned char *rgb = reinterpret_cast<unsigned char *>(s->scratch) + 4096 * sizeof(float);
    if (float_planes(s->precision)) {  // the density's FP32 plane (residuals left out of a frame)
        const float *rho = reinterpret_cast<const float *>(s->U);
        fvm2d::io::density_range_blocks<float, NT><<<(int)blocks, NT, 0, s->stream>>>(rho, s->pitch, s->nx, s->ny, parts);
        fvm2d::io::render_density<float><<<148 * 4, 256, 0, s->stream>>>(rho, s->pitch, s->nx, s->ny, parts, (int)blocks,
                                                                        rgb);
    } else {
        fvm2d::io::density_range_blocks<double, NT><<<(int)blocks, NT, 0, s->stream>>>(s->U, s->pitch, s->nx, s->ny, parts);
        fvm2d::io::render_density<double><<<148 * 4, 256, 0, s->stream>>>(s->U, s->pitch, s->nx, s->ny, parts, (int)blocks,
                                                                         rgb);
    }
    CK(cudaGetLastError());
    std::vector<unsigned char> host((size_t)n * 3);
    CK(cudaMemcpyAsync(host.data(), rgb, host.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (!fvm2d::io::write_png_rgb(path, s->nx, s->ny, host.data()))
        return fail(FVM2D_ERR_INVALID, (std::string("cannot write ") + path).c_str());
    return FVM2D_OK;
}

int fvm2d_write_frame_png(fvm2d_solver *s, const char *path)
{
    if (int rc = check(s)) return rc;
    if (!path) return fail(FVM2D_ERR_INVALID, "null path");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    return write_frame(s, path);
}

int fvm2d_set_record_model(fvm2d_solver *s, int on, int gap_per_frame, const char *dir)
{
    if (int rc = check(s)) return rc;
    s->record_on = on != 0;
    s->record_gap = gap_per_frame;
    s->record_dir = dir ? dir : ".";
    return FVM2D_OK;
}

int fvm2d_write_state(fvm2d_solver *s, const char *path)
{
    if (int rc = check(s)) return rc;
    if (!path) return fail(FVM2D_ERR_INVALID, "null path");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    std::vector<double> cells((size_t)s->nx * s->ny * 4);
    if (int rc = fvm2d_get_state(s, cells.data(), 4)) return rc;
    fvm2d::io::StateFileHeader hd;
    std::memcpy(hd.magic, "FVM2DST1", 8);
    hd.nx = s->nx;
    hd.ny = s->ny;
    hd.t = s->ctl_h->t;
    hd.steps = s->ctl_h->steps;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(FVM2D_ERR_INVALID, (std::string("cannot open ") + path).c_str());
    const bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1 &&
                    std::fwrite(cells.data(), sizeof(double), cells.size(), f) == cells.size();
    if (std::fclose(f) != 0 || !ok) return fail(FVM2D_ERR_INVALID, (std::string("cannot write ") + path).c_str());
    return FVM2D_OK;
}

int fvm2d_read_state(fvm2d_solver *s, const char *path)
{
    if (int rc = check(s)) return rc;
    if (!path) return fail(FVM2D_ERR_INVALID, "null path");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(FVM2D_ERR_INVALID, (std::string("cannot open ") + path).c_str());
    fvm2d::io::StateFileHeader hd;
    std::vector<double> cells((size_t)s->nx * s->ny * 4);
    const bool head = std::fread(&hd, sizeof hd, 1, f) == 1 && std::memcmp(hd.magic, "FVM2DST1", 8) == 0;
    const bool size = head && hd.nx == s->nx && hd.ny == s->ny;
    const bool body = size && std::fread(cells.data(), sizeof(double), cells.size(), f) == cells.size();
    std::fclose(f);
    if (!head) return fail(FVM2D_ERR_INVALID, "not an fvm2d state file");
    if (!size) return fail(FVM2D_ERR_INVALID, "the state file's nx, ny differ from the solver's");
    if (!body) return fail(FVM2D_ERR_INVALID, "the state file is truncated");
    if (int rc = fvm2d_set_state(s, cells.data(), 4)) return rc;
    s->ctl_h->t = hd.t;  // fvm2d_advance continues from the saved time and step count
    s->ctl_h->steps = int(hd.steps);
    return FVM2D_OK;
}

int fvm2d_get_health(fvm2d_solver *s, int *first_bad_step)
{
    if (int rc = check(s)) return rc;
    if (!first_bad_step) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *first_bad_step = s->ctl_h->first_bad;
    return FVM2D_OK;
}

int fvm2d_get_conserved_totals(fvm2d_solver *s, double *totals)
{
    Range range_("fvm2d_get_conserved_totals");
    if (int rc = check(s)) return rc;
    if (!totals) return fail(FVM2D_ERR_INVALID, "null output pointer");
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    constexpr int NT = 256;
    const long long cells = (long long)(s->nx - 4) * (s->ny - 4);
    const int blocks = (int)std::min<long long>(148 * 4, (cells + NT - 1) / NT);
    // the per-block partials, then the totals, in the sweep buffers (idle
    // between steps; everything runs in order on the handle's stream)
    double *partial = s->scratch, *sum = s->scratch + 4 * (long long)blocks;
    with_planes(s->precision, s->U, s->plane, [&](auto st) {
        conserved_partials<decltype(st), NT>
            <<<blocks, NT, 0, s->stream>>>(st, s->nx, s->ny, s->pitch, s->plane, s->gamma, partial);
    });
    CK(cudaGetLastError());
    const LaunchConfig c = s->config();
    conserved_sum<<<1, 32, 0, s->stream>>>(partial, blocks, c.hx * c.hy, sum);
    CK(cudaGetLastError());
    const cudaMemcpyKind kind = is_device_pointer(totals) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(totals, sum, 4 * sizeof(double), kind, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FVM2D_OK;
}

int fvm2d_get_computation_time_ms(fvm2d_solver *s, double *ms)
{
    if (int rc = check(s)) return rc;
    if (!ms) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *ms = s->last_ms;
    return FVM2D_OK;
}

int fvm2d_get_time_stages_count(fvm2d_solver *s, long long *count)
{
    if (int rc = check(s)) return rc;
    if (!count) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *count = s->total_steps;
    return FVM2D_OK;
}

int fvm2d_get_time(fvm2d_solver *s, double *t, int *steps, double *last_dt)
{
    if (int rc = check(s)) return rc;
    if (t) *t = s->ctl_h->t;
    if (steps) *steps = s->ctl_h->steps;
    if (last_dt) *last_dt = s->ctl_h->dt;
    return FVM2D_OK;
}

int fvm2d_get_run_stats(fvm2d_solver *s, double *device_ms, long long *kernel_launches)
{
    if (int rc = check(s)) return rc;
    if (device_ms) *device_ms = s->last_device_ms;
    if (kernel_launches) *kernel_launches = s->last_launches;
    return FVM2D_OK;
}

int fvm2d_profile_kernels(fvm2d_solver *s, int nsteps, double *kernel_ms, int *steps_done)
{
    Range range_("fvm2d_profile_kernels");
    if (steps_done) *steps_done = 0;
    if (int rc = check(s)) return rc;
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (nsteps < 1 || !kernel_ms) return fail(FVM2D_ERR_INVALID, "nsteps must be positive and kernel_ms non-null");
    cudaEvent_t ev[fvm2d::kStepKernels + 1] = {};
    for (auto &e : ev) CK(cudaEventCreate(&e));
    double acc[fvm2d::kStepKernels] = {};
    int done = 0, rc = FVM2D_OK;
    StepControl *c = s->ctl_h;
    const LaunchConfig cfg = s->config();
    for (int k = 0; k < nsteps && rc == FVM2D_OK; ++k) {
        const int before = c->steps;
        c->step_limit = before + 1;
        c->done = 0;
        c->active = 0;
        cudaError_t e;
        if ((rc = s->upload_control())) break;
        e = s->need_init ? kVariants[s->precision].init(cfg, s->stream) : kVariants[s->precision].plan(cfg, s->stream);
        s->need_init = false;
        if (!e) e = kVariants[s->precision].step(cfg, s->stream, ev);
        if (!e) e = cudaMemcpyAsync(c, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream);
        if (!e) e = cudaStreamSynchronize(s->stream);
        if (e) { rc = cuda_fail(e, "profiled step"); break; }
        if (c->steps == before) break;  // the loop has ended: nothing ran
        ++done;
        for (int q = 0; q < fvm2d::kStepKernels; ++q) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[q], ev[q + 1]);
            acc[q] += ms;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    s->total_steps += done;
    for (int q = 0; q < fvm2d::kStepKernels; ++q) kernel_ms[q] = done ? acc[q] / done : 0.0;
    if (steps_done) *steps_done = done;
    return FVM2D_OK;
}

// ---- differentiation -------------------------------------------------------

int fvm2d_set_vjp_overlap(fvm2d_solver *s, int on)
{
    if (int rc = check(s)) return rc;
    s->vjp_overlap = on != 0;
    s->drop_vjp_graphs();
    s->last_taped = false;  // the buffer it sits in follows the buffer count
    return FVM2D_OK;
}

int fvm2d_set_fixed_dt(fvm2d_solver *s, double dt)
{
    if (int rc = check(s)) return rc;
    if (!(dt >= 0.0)) return fail(FVM2D_ERR_INVALID, "dt must be non-negative");
    s->fixed_dt = dt;
    s->fwd_steps = -1;
    s->drop_graph();
    return FVM2D_OK;
}

static int diff_ready(fvm2d_solver *s)
{
    if (!s->have_state) return fail(FVM2D_ERR_STATE, "no state has been set");
    if (s->precision != FVM2D_FP64 && s->precision != FVM2D_FP32)
        return fail(FVM2D_ERR_INVALID, "differentiation runs on the FVM2D_FP64 or FVM2D_FP32 build");
    if (!(s->fixed_dt > 0.0)) return fail(FVM2D_ERR_INVALID, "set a fixed step size first (fvm2d_set_fixed_dt)");
    return FVM2D_OK;
}

// Bytes of one state of the current build (4 planes of `plane` values).
static size_t state_bytes_of(const fvm2d_solver *s)
{
    return state_bytes(s->precision, s->plane);
}

// (Re)allocates *buf to at least `bytes`; `grew` tells whether it moved.
static int ensure(char *&buf, size_t &cap, size_t bytes, bool &grew)
{
    grew = false;
    if (bytes <= cap) return FVM2D_OK;
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    CK(cudaMalloc(&buf, bytes));
    cap = bytes;
    grew = true;
    return FVM2D_OK;
}

// Copies host or device cells (stride doubles) into 4 planes at dst, of the
// current build's type, staging through the sweep buffers.
static int cells_to_planes(fvm2d_solver *s, const double *cells, int stride, void *dst)
{
    const size_t bytes = sizeof(double) * (size_t)s->nx * s->ny * stride;
    const cudaMemcpyKind kind = is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(s->scratch, cells, bytes, kind, s->stream));
    with_planes(s->precision, dst, s->plane, [&](auto st) {
        aos_to_soa<<<148 * 4, 256, 0, s->stream>>>(s->scratch, stride, st, s->nx, s->ny, s->pitch, s->plane);
    });
    CK(cudaGetLastError());
    return FVM2D_OK;
}

static int planes_to_cells(fvm2d_solver *s, const void *src, double *cells, int stride)
{
    with_planes(s->precision, src, s->plane, [&](auto st) {
        soa_to_aos<<<148 * 4, 256, 0, s->stream>>>(st, s->nx, s->ny, s->pitch, s->plane, stride, s->scratch);
    });
    CK(cudaGetLastError());
    const size_t bytes = sizeof(double) * (size_t)s->nx * s->ny * stride;
    const cudaMemcpyKind kind = is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(cells, s->scratch, bytes, kind, s->stream));
    return FVM2D_OK;
}

int fvm2d_jvp(fvm2d_solver *s, int nsteps, const double *tangent_in, double *tangent_out, int stride)
{
    Range range_("fvm2d_jvp");
    if (int rc = check(s)) return rc;
    if (int rc = diff_ready(s)) return rc;
    if (s->precision != FVM2D_FP64) return fail(FVM2D_ERR_INVALID, "fvm2d_jvp runs on the FP64 build (FVM2D_FP64)");
    if (!tangent_in || !tangent_out) return fail(FVM2D_ERR_INVALID, "null tangent pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    if (nsteps < 0) return fail(FVM2D_ERR_INVALID, "nsteps must be non-negative");
    const long long n4 = 4 * s->plane;
    if (!s->dual) CK(cudaMalloc(&s->dual, 3 * n4 * sizeof(Dual)));
    Dual *dU = static_cast<Dual *>(s->dual), *dA = dU + n4, *dB = dA + n4;
    double *T = reinterpret_cast<double *>(dB);  // tangent planes, before packing and after unpacking
    if (int rc = cells_to_planes(s, tangent_in, stride, T)) return rc;
    pack_dual<<<148 * 4, 256, 0, s->stream>>>(s->U, T, dU, n4);
    CK(cudaGetLastError());
    LaunchConfig c = s->config();
    c.U = dU;
    c.A = dA;
    c.B = dB;
    StepControl *h = s->ctl_h;
    const int before = h->steps;
    h->step_limit = before + nsteps;
    h->done = 0;
    h->active = 0;
    if (int rc = s->upload_control()) return rc;
    CK(kJvp.init(c, s->stream));
    for (int k = 0; k < nsteps; ++k) CK(kJvp.step(c, s->stream, nullptr));
    CK(cudaMemcpyAsync(h, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
    unpack_dual<<<148 * 4, 256, 0, s->stream>>>(dU, s->U, T, n4);
    CK(cudaGetLastError());
    if (int rc = planes_to_cells(s, T, tangent_out, stride)) return rc;
    CK(cudaStreamSynchronize(s->stream));
    s->need_init = true;  // the state changed outside the FP64 graphs' bookkeeping
    s->total_steps += h->steps - before;
    s->fwd_steps = -1;
    return FVM2D_OK;
}

constexpr int kTapeStates = 7;  // per taped step: U, X(U), Y(U), the fluxes of its 4 sweeps

// State q of taped step j in tape buffer `buf` (buffers of ck_len steps).
static char *tape_at(const fvm2d_solver *s, int buf, int j, int q, size_t sb)
{
    return s->tape + (((size_t)buf * s->ck_len + j) * kTapeStates + q) * sb;
}

// Enqueues on `st` m taped steps (control planned) from the state in slot 0
// of tape buffer `buf`: step j reads slot j's input state, fills the rest of
// slot j and writes its result as slot j+1's input state, the last step's
// into U.
static int taped_steps(fvm2d_solver *s, const LaunchConfig &c, int m, int buf, cudaStream_t st)
{
    const size_t sb = state_bytes_of(s);
    auto taped_step = is_fp32(s->precision) ? fvm2d::fp32::enqueue_step_taped : fvm2d::fp64::enqueue_step_taped;
    for (int j = 0; j < m; ++j) {
        LaunchConfig cj = c;
        cj.U = tape_at(s, buf, j, 0, sb);
        cj.A = tape_at(s, buf, j, 1, sb);
        cj.B = tape_at(s, buf, j, 2, sb);
        void *const flux[4] = {tape_at(s, buf, j, 3, sb), tape_at(s, buf, j, 4, sb), tape_at(s, buf, j, 5, sb),
                               tape_at(s, buf, j, 6, sb)};
        void *const out =
            j + 1 < m ? static_cast<void *>(tape_at(s, buf, j + 1, 0, sb)) : static_cast<void *>(s->U);
        CK(taped_step(cj, st, flux, out));
    }
    return FVM2D_OK;
}

// The control record of a recomputed segment: time t, nothing committed, the
// fixed step dt planned.  Written by a kernel on the recompute's stream, so
// each segment's record travels with its own launch (a host-side record
// copied asynchronously could be overwritten by the next segment's before
// the copy runs).
__global__ void segment_control(StepControl *c, double t, double dt)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        c->t = t;
        c->dt = dt;
        c->smax_last = 0.0;
        c->smax_bits = 0ull;
        c->steps = 0;
        c->step_limit = INT_MAX;
        c->active = 1;
        c->done = 0;
        c->ticket = 0u;
        c->first_bad = 0;
    }
}

// fvm2d_forward with FVM2D_FULL_TAPE: the forward steps are the taped ones.
static int forward_full_tape(fvm2d_solver *s, int nsteps)
{
    const size_t sb = state_bytes_of(s);
    const size_t need = (size_t)nsteps * kTapeStates * sb;
    if (need > s->tape_bytes) {
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        if (need > free_b + s->tape_bytes) {
            char msg[160];
            std::snprintf(msg, sizeof msg, "the full tape needs %.2f GB, more than the device's free memory: use checkpoints",
                          need / 1e9);
            return fail(FVM2D_ERR_INVALID, msg);
        }
    }
    s->full_tape = false;
    s->fwd_steps = -1;
    bool grew;
    if (int rc = ensure(s->tape, s->tape_bytes, need, grew)) return rc;
    if (grew) s->drop_vjp_graphs();
    if (int rc = s->build_graphs()) return rc;  // as fvm2d_forward, so a later advance keeps the tape
    StepControl *h = s->ctl_h;
    h->step_limit = INT_MAX;
    h->done = 0;
    h->active = 0;
    if (int rc = s->upload_control()) return rc;
    const LaunchConfig c = s->config();
    CK(s->need_init ? kVariants[s->precision].init(c, s->stream) : kVariants[s->precision].plan(c, s->stream));
    s->need_init = false;
    CK(cudaMemcpyAsync(tape_at(s, 0, 0, 0, sb), s->U, sb, cudaMemcpyDeviceToDevice, s->stream));
    if (int rc = taped_steps(s, c, nsteps, 0, s->stream)) return rc;
    CK(cudaMemcpyAsync(h, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->ck_count = 1;
    s->ck_len = nsteps;
    s->fwd_steps = nsteps;
    s->fwd_precision = s->precision;
    s->full_tape = true;
    s->total_steps += nsteps;
    return FVM2D_OK;
}

// Steps of checkpoint segment k when nsteps are split into `count` segments
// of at most len steps: the first one takes the remainder, so the last one,
// which the forward tapes and the reverse meets first, is a full segment
// (and its recompute never waits on a shorter reverse).
static int segment_steps(int nsteps, int len, int count, int k)
{
    return k == 0 ? nsteps - (count - 1) * len : len;
}

// adjoint workspace: two adjoints, three work states, the saved final state,
// the fourth work state of the fork stream's branch
constexpr int kAdjStates = 7;

// The adjoint step's launch parameters for this handle; the tape and
// adjoint pointers are filled per step.
static fvm2d::AdjointLaunch adjoint_launch_of(const fvm2d_solver *s, size_t sb)
{
    fvm2d::AdjointLaunch L{};
    L.nx = s->nx;
    L.ny = s->ny;
    L.pitch = s->pitch;
    L.plane = s->plane;
    L.strategy = s->strategy;
    const LaunchConfig c = s->config();
    L.hx = c.hx;
    L.hy = c.hy;
    L.rhx = c.rhx;
    L.rhy = c.rhy;
    L.alpha = s->alpha;
    L.gamma = s->gamma;
    L.dt = s->fixed_dt;
    for (int k = 0; k < 3; ++k) L.work[k] = s->adj + (2 + k) * sb;
    L.work[3] = s->adj + 6 * sb;
    L.fork = s->fork;
    L.fork_ev[0] = s->fork_ev[0];
    L.fork_ev[1] = s->fork_ev[1];
    return L;
}

// The adjoint step's fork stream and its events (created once per handle).
static int ensure_fork(fvm2d_solver *s)
{
    if (s->fork) return FVM2D_OK;
    CK(cudaStreamCreateWithFlags(&s->fork, cudaStreamNonBlocking));
    for (auto &e : s->fork_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return FVM2D_OK;
}

// Enqueues on `st` the reverse of m steps taped in buffer `buf`, starting
// from adjoint buffer `from` (0 or 1 of the workspace); the result lands in
// `from` for even m, in the other buffer for odd m.
static int reverse_steps(fvm2d_solver *s, int m, int buf, int from, cudaStream_t st)
{
    const size_t sb = state_bytes_of(s);
    auto adjoint_step = is_fp32(s->precision) ? fvm2d::adj32::adjoint_step : fvm2d::adj::adjoint_step;
    fvm2d::AdjointLaunch L = adjoint_launch_of(s, sb);
    char *a = s->adj + from * sb, *b = s->adj + (1 - from) * sb;
    for (int j = m - 1; j >= 0; --j) {
        L.U = tape_at(s, buf, j, 0, sb);
        L.A1 = tape_at(s, buf, j, 1, sb);
        L.B1 = tape_at(s, buf, j, 2, sb);
        for (int q = 0; q < 4; ++q) L.flux[q] = tape_at(s, buf, j, 3 + q, sb);
        L.lb_out = a;
        L.lb_in = b;
        CK(adjoint_step(L, st));
        std::swap(a, b);
    }
    return FVM2D_OK;
}

// Workspace of a checkpointed reverse (ck_count segments of ck_len steps):
// the adjoint states and the tape buffers -- two where the device has room
// for the second (segment k-1 is then recomputed on the aux stream while
// segment k is reversed), else one -- with the aux stream, its events and
// the graphs of a full segment's recompute and reverse.  *bufs is 1 or 2.
static int vjp_workspace(fvm2d_solver *s, int *bufs)
{
    const size_t sb = state_bytes_of(s);
    const size_t seg_bytes = (size_t)s->ck_len * kTapeStates * sb;
    *bufs = 1;
    if (s->ck_count > 1 && s->vjp_overlap) {
        if (s->tape_bytes >= 2 * seg_bytes) {
            *bufs = 2;
        } else {
            size_t free_b = 0, total_b = 0;
            CK(cudaMemGetInfo(&free_b, &total_b));
            const size_t margin = (size_t)256 << 20;  // left to the rest of the process
            const size_t adj_need = s->adj_bytes >= kAdjStates * sb ? 0 : kAdjStates * sb;
            if (2 * seg_bytes + adj_need + margin <= free_b + s->tape_bytes) *bufs = 2;
        }
    }
    bool grew_tape, grew_adj;
    if (int rc = ensure(s->tape, s->tape_bytes, *bufs * seg_bytes, grew_tape)) return rc;
    if (int rc = ensure(s->adj, s->adj_bytes, kAdjStates * sb, grew_adj)) return rc;
    if (grew_tape || grew_adj) s->drop_vjp_graphs();
    if (grew_tape) s->last_taped = false;
    if (int rc = ensure_fork(s)) return rc;
    if (*bufs == 2 && !s->aux) {
        // default priority: the recompute fills the SM room the reverse's
        // blocks leave (measured: at the device's higher priority the VJP
        // took 1% longer)
        CK(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
        for (auto &e : s->vjp_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // graphs of a full segment, kept while the handle's parameters, build and
    // buffers stay the same
    if (s->ck_count > 1 && (s->vjp_len != s->ck_len || s->vjp_bufs != *bufs)) {
        s->drop_vjp_graphs();
        CK(is_fp32(s->precision) ? fvm2d::adj32::adjoint_prepare() : fvm2d::adj::adjoint_prepare());
        const LaunchConfig c = s->config();
        const int len = s->ck_len;
        if (int rc = s->capture(&s->vjp_graph[6], [&] {
                for (int j = 0; j < len; ++j) CK(kVariants[s->precision].step(c, s->stream, nullptr));
                return FVM2D_OK;
            }))
            return rc;
        for (int b = 0; b < *bufs; ++b) {
            if (int rc = s->capture(&s->vjp_graph[b], [&] { return taped_steps(s, c, len, b, s->stream); }))
                return rc;
            for (int a = 0; a < 2; ++a)
                if (int rc = s->capture(&s->vjp_graph[2 + 2 * b + a], [&] { return reverse_steps(s, len, b, a, s->stream); }))
                    return rc;
        }
        s->vjp_len = len;
        s->vjp_bufs = *bufs;
    }
    return FVM2D_OK;
}

int fvm2d_forward(fvm2d_solver *s, int nsteps, int checkpoints)
{
    Range range_("fvm2d_forward");
    if (int rc = check(s)) return rc;
    if (int rc = diff_ready(s)) return rc;
    if (nsteps < 1 || checkpoints < 0)
        return fail(FVM2D_ERR_INVALID, "nsteps must be positive and checkpoints positive or FVM2D_FULL_TAPE");
    if (checkpoints == FVM2D_FULL_TAPE) return forward_full_tape(s, nsteps);
    if (checkpoints > nsteps) checkpoints = nsteps;
    const int len = (nsteps + checkpoints - 1) / checkpoints;
    const int count = (nsteps + len - 1) / len;
    const size_t sb = state_bytes_of(s);
    bool grew;
    if (int rc = ensure(s->ckpt, s->ck_bytes, (size_t)count * sb, grew)) return rc;
    if (int rc = s->build_graphs()) return rc;  // the step graphs of the fixed-dt build
    s->fwd_steps = -1;
    s->full_tape = false;
    s->last_taped = false;
    s->ck_count = count;
    s->ck_len = len;
    // the last segment, the first one the reverse needs, is taped as it runs
    // (as revolve schedules do), so fvm2d_vjp does not recompute it
    int bufs = 1;
    if (count > 1)
        if (int rc = vjp_workspace(s, &bufs)) return rc;
    StepControl *h = s->ctl_h;
    h->step_limit = INT_MAX;
    h->done = 0;
    h->active = 0;
    if (int rc = s->upload_control()) return rc;
    const LaunchConfig c = s->config();
    CK(s->need_init ? kVariants[s->precision].init(c, s->stream) : kVariants[s->precision].plan(c, s->stream));
    s->need_init = false;
    s->ck_t.assign(count, 0.0);
    double t = h->t;
    for (int k = 0; k < count; ++k) {
        s->ck_t[k] = t;
        CK(cudaMemcpyAsync(s->ckpt + k * sb, s->U, sb, cudaMemcpyDeviceToDevice, s->stream));
        const int m = segment_steps(nsteps, len, count, k);
        if (count > 1 && k == count - 1) {
            const int b = k % bufs;
            CK(cudaMemcpyAsync(tape_at(s, b, 0, 0, sb), s->U, sb, cudaMemcpyDeviceToDevice, s->stream));
            if (m == s->vjp_len) {
                CK(cudaGraphLaunch(s->vjp_graph[b], s->stream));
            } else if (int rc = taped_steps(s, c, m, b, s->stream)) {
                return rc;
            }
            for (int q = 0; q < m; ++q) t = t + s->fixed_dt;
            continue;
        }
        if (count > 1 && m == s->vjp_len) {  // a full segment: one graph of its steps
            CK(cudaGraphLaunch(s->vjp_graph[6], s->stream));
            for (int q = 0; q < m; ++q) t = t + s->fixed_dt;
            continue;
        }
        for (int j = 0; j < m;) {
            const int which = m - j >= fvm2d_solver::kGraphSteps[0] ? 0 : 1;
            CK(cudaGraphLaunch(s->graph[which], s->stream));
            for (int q = 0; q < fvm2d_solver::kGraphSteps[which]; ++q) t = t + s->fixed_dt;  // as the device adds
            j += fvm2d_solver::kGraphSteps[which];
        }
    }
    CK(cudaMemcpyAsync(h, s->ctl, sizeof(StepControl), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->fwd_steps = nsteps;
    s->fwd_precision = s->precision;
    s->last_taped = count > 1;
    s->total_steps += nsteps;
    return FVM2D_OK;
}

int fvm2d_vjp(fvm2d_solver *s, const double *cotangent_in, double *cotangent_out, int stride)
{
    Range range_("fvm2d_vjp");
    if (int rc = check(s)) return rc;
    if (int rc = diff_ready(s)) return rc;
    if (s->fwd_steps < 0 || s->fwd_precision != s->precision)
        return fail(FVM2D_ERR_STATE, "fvm2d_vjp reverses the last fvm2d_forward of this build: call it first");
    if (!cotangent_in || !cotangent_out) return fail(FVM2D_ERR_INVALID, "null cotangent pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    const size_t sb = state_bytes_of(s);
    int bufs = 1;
    if (s->full_tape) {
        bool grew_adj;
        if (int rc = ensure(s->adj, s->adj_bytes, kAdjStates * sb, grew_adj)) return rc;
        if (grew_adj) s->drop_vjp_graphs();
        if (int rc = ensure_fork(s)) return rc;
    } else if (int rc = vjp_workspace(s, &bufs)) {
        return rc;
    }
    char *const saved = s->adj + 5 * sb;
    int lam = 0;  // adjoint buffer holding the current adjoint
    const StepControl after = *s->ctl_h;
    CK(cudaMemcpyAsync(saved, s->U, sb, cudaMemcpyDeviceToDevice, s->stream));
    if (int rc = cells_to_planes(s, cotangent_in, stride, s->adj)) return rc;
    const int count = s->ck_count;
    auto seg_len = [&](int k) { return segment_steps(s->fwd_steps, s->ck_len, count, k); };
    if (s->full_tape) {  // the forward taped every step: reverse only
        if (int rc = reverse_steps(s, s->fwd_steps, 0, lam, s->stream)) return rc;
        lam ^= s->fwd_steps & 1;
    } else {
        // segment k is taped in buffer k % bufs
        auto recompute_segment = [&](int k, cudaStream_t st) -> int {
            if (k == count - 1 && s->last_taped) return FVM2D_OK;  // taped by the forward
            const int m = seg_len(k), b = k % bufs;
            CK(cudaMemcpyAsync(tape_at(s, b, 0, 0, sb), s->ckpt + k * sb, sb, cudaMemcpyDeviceToDevice, st));
            segment_control<<<1, 32, 0, st>>>(s->ctl, s->ck_t[k], s->fixed_dt);
            CK(cudaGetLastError());
            if (m == s->vjp_len) {
                CK(cudaGraphLaunch(s->vjp_graph[b], st));
            } else if (int rc = taped_steps(s, s->config(), m, b, st)) {
                return rc;
            }
            return FVM2D_OK;
        };
        auto reverse_segment = [&](int k, cudaStream_t st) -> int {
            const int m = seg_len(k), b = k % bufs;
            if (m == s->vjp_len) {
                CK(cudaGraphLaunch(s->vjp_graph[2 + 2 * b + lam], st));
            } else if (int rc = reverse_steps(s, m, b, lam, st)) {
                return rc;
            }
            lam ^= m & 1;
            return FVM2D_OK;
        };
        if (bufs == 1) {
            for (int k = count - 1; k >= 0; --k) {
                if (int rc = recompute_segment(k, s->stream)) return rc;
                if (int rc = reverse_segment(k, s->stream)) return rc;
            }
        } else {
            // aux: recompute(K-1), recompute(K-2), ...; stream: reverse(K-1),
            // reverse(K-2), ...  reverse(k) waits for recompute(k) (buffer
            // filled); recompute(k-1) waits for reverse(k+1), the last user
            // of its buffer.  The recomputes own the control record and U
            // (restored from `saved` below, after the last wait).
            cudaEvent_t *const filled = s->vjp_ev, *const freed = s->vjp_ev + 2, start = s->vjp_ev[4];
            CK(cudaEventRecord(start, s->stream));
            CK(cudaStreamWaitEvent(s->aux, start, 0));
            if (int rc = recompute_segment(count - 1, s->aux)) return rc;
            CK(cudaEventRecord(filled[(count - 1) % 2], s->aux));
            for (int k = count - 1; k >= 0; --k) {
                CK(cudaStreamWaitEvent(s->stream, filled[k % 2], 0));
                if (int rc = reverse_segment(k, s->stream)) return rc;
                CK(cudaEventRecord(freed[k % 2], s->stream));
                if (k > 0) {
                    if (k + 1 < count) CK(cudaStreamWaitEvent(s->aux, freed[(k + 1) % 2], 0));
                    if (int rc = recompute_segment(k - 1, s->aux)) return rc;
                    CK(cudaEventRecord(filled[(k - 1) % 2], s->aux));
                }
            }
        }
        s->last_taped = false;  // its buffer has been reused (or will be by the next call)
    }
    if (int rc = planes_to_cells(s, s->adj + lam * sb, cotangent_out, stride)) return rc;
    CK(cudaMemcpyAsync(s->U, saved, sb, cudaMemcpyDeviceToDevice, s->stream));
    *s->ctl_h = after;
    if (int rc = s->upload_control()) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return FVM2D_OK;
}

#pragma GCC visibility pop
} // extern "C"
