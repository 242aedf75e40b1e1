// fvm2d_noalloc.cu -- fvm2d_advance_noalloc: the FP64 split step for callers
// that cannot allocate device memory.
//
// Who needs it: code that must not call cudaMalloc/cudaFree itself -- a host
// application whose device memory is owned by its own allocator or arena
// with a fixed budget (an allocation behind its back breaks its accounting),
// or a latency-critical loop that cannot pay for cudaMalloc/cudaFree, which
// may synchronize the device.  Such a caller already holds the state in its
// own device memory; this entry point advances it using only memory that
// exists for the whole life of the library.
//
// The sweeps need two state-sized intermediate buffers and the step-control
// record.  Here they live in one file-scope device array, `g_scratch`, sized
// for at most kNoAllocMaxCells cells; every GPU that loads the library holds
// that array (16 MiB + 256 B) until the process exits.  Every call uses the
// same array: calls whose work overlaps on the GPU (on different streams, or
// from different host threads) race on it and must be serialized by the
// caller.  The array keeps whatever the previous call left; the control
// record, the only part that must start from known values, is rewritten at
// the start of every call.
//
// A call waits for its own work (it reads the step-control record back
// between groups of steps), so it cannot be made while its stream is being
// captured into a CUDA graph; such a call is refused.
#include "../../include/fvm2d.h"
#include "fvm2d_control.h"

#include <climits>
#include <mutex>
#include <string>

namespace {

constexpr long long kNoAllocMaxCells = FVM2D_NOALLOC_MAX_CELLS;
constexpr long long kScratchDoubles = 8 * kNoAllocMaxCells;  // intermediate states A and B
constexpr long long kControlDoubles = 32;                     // 256 bytes for the StepControl record
static_assert(sizeof(fvm2d::StepControl) <= kControlDoubles * sizeof(double), "control record does not fit");

// The only device memory this entry point touches besides the caller's.
static __device__ __align__(256) double g_scratch[kScratchDoubles + kControlDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};  // device address of g_scratch, per device

// Steps enqueued between two reads of the control record: a run that reaches
// its end time early stops within this many (empty) steps of it.
constexpr int kStepsPerCheck = 32;

int fail(int code, const std::string &msg) { return fvm2d::report_error(code, msg.c_str()); }

int cuda_fail(cudaError_t e, const char *what)
{
    // clear a pending error that is not sticky (a failed allocation, say), so
    // that it is not reported again by the next call's launch checks
    cudaGetLastError();
    return fail(FVM2D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Sets the control record for a run of at most `nsteps` steps from time t0.
__global__ void reset_control(fvm2d::StepControl *c, double t0, int nsteps)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->t = t0;
    c->dt = 0.0;
    c->smax_last = 0.0;
    c->smax_bits = 0ull;
    c->steps = 0;
    c->step_limit = nsteps;
    c->active = 0;
    c->done = 0;
    c->ticket = 0u;
    c->first_bad = 0;
}

// Once per device, with that device current: the device address of
// g_scratch (the host-side name is only a stand-in and must never be passed
// to a kernel) and the kernels' shared-memory attributes.
int setup_device(int dev, double **scratch)
{
    if (dev < 0 || dev >= kMaxDevices) return fail(FVM2D_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        if ((e = fvm2d::fp64::prepare()) != cudaSuccess) return cuda_fail(e, "kernel attributes");
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *scratch = g_scratch_ptr[dev];
    return FVM2D_OK;
}

} // namespace

extern "C" {
#pragma GCC visibility push(default)

int fvm2d_advance_noalloc(const double *state_in, double *state_out, int nx, int ny, double width, double height,
                          double t_end, double cfl, double alpha, double gamma, int strategy, double t0,
                          int nsteps, void *stream, double *t_out, int *steps_out)
{
    if (t_out) *t_out = t0;
    if (steps_out) *steps_out = 0;
    if (!state_in || !state_out) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (nx < 6 || ny < 6) return fail(FVM2D_ERR_INVALID, "nx and ny must be at least 6 (two ghost layers per side)");
    if ((long long)nx * ny > kNoAllocMaxCells)
        return fail(FVM2D_ERR_INVALID, "nx * ny = " + std::to_string((long long)nx * ny) +
                                           " exceeds the allocation-free limit of " +
                                           std::to_string(kNoAllocMaxCells) + " cells");
    if (nsteps < 0) return fail(FVM2D_ERR_INVALID, "nsteps must be non-negative");
    if (strategy < FVM2D_OUTFLOW || strategy > FVM2D_REFLECTIVE_TB) return fail(FVM2D_ERR_INVALID, "unknown ghost-cell strategy");
    if (!(width > 0.0 && height > 0.0 && cfl > 0.0 && gamma > 1.0))
        return fail(FVM2D_ERR_INVALID, "width, height and cfl must be positive and gamma above 1");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    double *scratch = nullptr;
    if (int rc = setup_device(dev, &scratch)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(s, &capturing))) return cuda_fail(e, "cudaStreamIsCapturing");
    if (capturing != cudaStreamCaptureStatusNone)
        return fail(FVM2D_ERR_INVALID, "fvm2d_advance_noalloc waits for its work and cannot run inside a stream capture");

    const long long plane = (long long)nx * ny;
    {
        // the same buffer, or two that do not overlap: a partial overlap would
        // make the input copy below read cells it has already overwritten
        const char *in0 = reinterpret_cast<const char *>(state_in), *out0 = reinterpret_cast<const char *>(state_out);
        const long long bytes = (long long)sizeof(double) * 4 * plane;
        if (in0 != out0 && in0 < out0 + bytes && out0 < in0 + bytes)
            return fail(FVM2D_ERR_INVALID, "state_in and state_out overlap without being the same buffer");
    }
    if (state_out != state_in &&
        (e = cudaMemcpyAsync(state_out, state_in, sizeof(double) * 4 * plane, cudaMemcpyDeviceToDevice, s)))
        return cuda_fail(e, "copy of the input state");

    fvm2d::LaunchConfig c;
    c.nx = nx;
    c.ny = ny;
    c.pitch = nx;
    c.plane = plane;
    c.U = state_out;
    c.A = scratch;
    c.B = scratch + 4 * plane;
    c.ctl = reinterpret_cast<fvm2d::StepControl *>(scratch + kScratchDoubles);
    c.hx = width / double(nx);
    c.hy = height / double(ny);
    c.rhx = 1.0 / c.hx;
    c.rhy = 1.0 / c.hy;
    c.alpha = alpha;
    c.gamma = gamma;
    c.strategy = strategy;
    c.plan.t_end = t_end;
    c.plan.cfl = cfl;
    c.plan.hmin = (c.hy < c.hx) ? c.hy : c.hx;
    c.plan.fixed_dt = 0.0;

    reset_control<<<1, 32, 0, s>>>(c.ctl, t0, nsteps);
    if ((e = cudaGetLastError())) return cuda_fail(e, "control reset");
    if ((e = fvm2d::fp64::enqueue_init(c, s))) return cuda_fail(e, "init kernel");
    // groups of steps, each followed by a read of the control record: once the
    // run has reached t_end (or nsteps) no further steps are enqueued
    fvm2d::StepControl out;
    int queued = 0;
    do {
        const int n = (nsteps - queued < kStepsPerCheck) ? nsteps - queued : kStepsPerCheck;
        for (int k = 0; k < n; ++k)
            if ((e = fvm2d::fp64::enqueue_step(c, s, nullptr))) return cuda_fail(e, "step kernels");
        queued += n;
        if ((e = cudaMemcpyAsync(&out, c.ctl, sizeof(out), cudaMemcpyDeviceToHost, s)))
            return cuda_fail(e, "control read");
        if ((e = cudaStreamSynchronize(s))) return cuda_fail(e, "cudaStreamSynchronize");
    } while (out.active && queued < nsteps);
    if (t_out) *t_out = out.t;
    if (steps_out) *steps_out = out.steps;
    return FVM2D_OK;
}

#pragma GCC visibility pop
} // extern "C"
