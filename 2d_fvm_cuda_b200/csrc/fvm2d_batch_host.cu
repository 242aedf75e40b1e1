// fvm2d_batch_host.cu -- host runtime of the batched form (fvm2d_batch_* in
// include/fvm2d.h).
//
// All problems of a batch share one allocation: problem p owns three
// consecutive state-sized regions (U, A, B), each 4 planes of pitch_p x ny_p
// doubles; FP32 planes start at the same byte addresses and fill the first
// half of each region.  A step is five launches covering every problem (x-sweep, y-sweep,
// y-sweep, final x-sweep, ghost ring); each problem carries its own dt, time
// and end time in its control record, and its items are skipped once its loop
// has ended.  The step is captured in CUDA graphs (16 steps and 1 step) that
// are replayed until no problem has a step in flight; each replay reads the
// control records back (64 bytes per problem).  fvm2d_batch_autotune times
// candidate y-segment lengths and sweep grid sizes on the batch itself and
// keeps the fastest.
//
// Per problem, a batch gives the bits of a single solve in the
// contraction-free build; in the builds with FMA contraction the two agree to
// rounding (the compiler may contract the same inlined arithmetic differently
// in the batched and the single-problem kernels).
#include <nvtx3/nvToolsExt.h>
#include "../../include/fvm2d.h"
#include "fvm2d_batch_control.h"
#include "fvm2d_transfer.cuh"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using fvm2d::BatchLaunch;
using fvm2d::BatchProblem;
using fvm2d::StepControl;

namespace {

int fail(int code, const std::string &msg) { return fvm2d::report_error(code, msg.c_str()); }

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

struct BatchVariant {
    cudaError_t (*prepare)(int *, int *);
    cudaError_t (*init)(const BatchLaunch &, cudaStream_t);
    cudaError_t (*plan)(const BatchLaunch &, cudaStream_t);
    cudaError_t (*step)(const BatchLaunch &, cudaStream_t);
};

const BatchVariant kBatchVariants[] = {
    {fvm2d::fp64::batch_prepare, fvm2d::fp64::batch_enqueue_init, fvm2d::fp64::batch_enqueue_plan,
     fvm2d::fp64::batch_enqueue_step},
    {fvm2d::fp64_strict::batch_prepare, fvm2d::fp64_strict::batch_enqueue_init, fvm2d::fp64_strict::batch_enqueue_plan,
     fvm2d::fp64_strict::batch_enqueue_step},
    {fvm2d::fp64_reforder::batch_prepare, fvm2d::fp64_reforder::batch_enqueue_init,
     fvm2d::fp64_reforder::batch_enqueue_plan, fvm2d::fp64_reforder::batch_enqueue_step},
    {fvm2d::fp32::batch_prepare, fvm2d::fp32::batch_enqueue_init, fvm2d::fp32::batch_enqueue_plan,
     fvm2d::fp32::batch_enqueue_step},
};
constexpr int kNumBatchVariants = sizeof(kBatchVariants) / sizeof(kBatchVariants[0]);

constexpr int kGhostThreads = 256;
constexpr int kGraphSteps[2] = {16, 1};

int y_segments(int ny, int T) { return (ny - 4 + T - 2) / (T - 1); }

} // namespace

struct fvm2d_batch {
    int device = 0, np = 0, precision = FVM2D_FP64;
    cudaStream_t stream = nullptr;
    std::vector<int> nx, ny, pitch, strategy;
    std::vector<double> width, height, t_end, cfl, alpha, gamma;
    std::vector<long long> off;  // element offset of problem p's U region
    std::vector<char> have_state;
    long long total_elems = 0;   // doubles in the allocation
    double *base = nullptr;
    BatchProblem *prob_d = nullptr;
    StepControl *ctl_d = nullptr, *ctl_h = nullptr;
    long long *x0_d = nullptr, *y0_d = nullptr;
    int *rb0_d = nullptr, *ib0_d = nullptr;
    BatchLaunch L{};
    bool dirty = true;  // descriptors must be rebuilt and uploaded
    // problems whose sweep items are in the item lists: all at the start of a
    // run; problems whose loop has ended are dropped from the lists (and the
    // step graphs re-captured) once they hold a sizeable share of the items,
    // so the static split of items over warps keeps every warp on live work
    std::vector<char> listed;
    int T = 32;         // y-sweep interfaces per segment
    int xchunks = 8;    // x-sweep chunks of 32 cells per item (set with the descriptors)
    int grid_x = 0, grid_y = 0;
    int occ_x = 1, occ_y = 1;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_variant = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0, last_device_ms = 0.0;
    long long last_launches = 0, last_cell_updates = 0;

    void drop_graphs()
    {
        for (auto &g : graph) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
        graph_variant = -1;
    }

    long long plane(int p) const { return (long long)pitch[p] * ny[p]; }

    // Host descriptors and prefix counts -> device.
    int upload_descriptors()
    {
        if (!dirty) return FVM2D_OK;
        std::vector<BatchProblem> P(np);
        std::vector<int> rb0(np + 1, 0), ib0(np + 1, 0);
        // one x-item length for the batch: the longest that still gives
        // every resident warp a couple of items over all problems
        xchunks = 8;
        for (;;) {
            long long items = 0;
            for (int p = 0; p < np; ++p) items += (long long)fvm2d::x_items_per_row(nx[p], xchunks) * ny[p];
            if (xchunks == 1 || items >= 2ll * occ_x * 4) break;
            xchunks /= 2;
        }
        if ((int)listed.size() != np) listed.assign(np, 1);
        // offsets in elements of the storage type: FP32 planes start at the
        // same byte addresses as FP64 planes would (the layout is in doubles)
        const long long scale = (precision == FVM2D_FP32) ? 2 : 1;
        for (int p = 0; p < np; ++p) {
            BatchProblem &q = P[p];
            std::memset(&q, 0, sizeof(q));
            q.plane = plane(p);
            q.u = scale * off[p];
            q.a = scale * (off[p] + 4 * q.plane);
            q.b = scale * (off[p] + 8 * q.plane);
            q.pitch = pitch[p];
            q.nx = nx[p];
            q.ny = ny[p];
            q.strategy = strategy[p];
            q.hx = width[p] / double(nx[p]);
            q.hy = height[p] / double(ny[p]);
            q.rhx = 1.0 / q.hx;
            q.rhy = 1.0 / q.hy;
            q.alpha = alpha[p];
            q.gamma = gamma[p];
            q.plan.t_end = t_end[p];
            q.plan.cfl = cfl[p];
            q.plan.hmin = (q.hy < q.hx) ? q.hy : q.hx;
            q.plan.fixed_dt = 0.0;
            q.xchunks = xchunks;
            q.nsegx = fvm2d::x_items_per_row(nx[p], xchunks);
            q.ncw = (nx[p] + 31) / 32;
            q.T = T;
            q.nsegy = y_segments(ny[p], T);
            q.ring = 4 * nx[p] + 4 * (ny[p] - 4);
            rb0[p + 1] = rb0[p] + (q.ring + kGhostThreads - 1) / kGhostThreads;
            const long long cells = (long long)nx[p] * ny[p];
            ib0[p + 1] = ib0[p] + int((cells + fvm2d::kBatchInitCells - 1) / fvm2d::kBatchInitCells);
        }
        CK(cudaMemcpyAsync(prob_d, P.data(), sizeof(BatchProblem) * np, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(rb0_d, rb0.data(), sizeof(int) * (np + 1), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(ib0_d, ib0.data(), sizeof(int) * (np + 1), cudaMemcpyHostToDevice, stream));
        if (int rc = upload_items()) return rc;
        L.base = base;
        L.prob = prob_d;
        L.ctl = ctl_d;
        L.x0 = x0_d;
        L.y0 = y0_d;
        L.rb0 = rb0_d;
        L.ib0 = ib0_d;
        L.np = np;
        L.ring_blocks = rb0[np];
        L.init_blocks = ib0[np];
        L.grid_x = grid_x;
        L.grid_y = grid_y;
        dirty = false;
        drop_graphs();
        return FVM2D_OK;
    }

    // Sweep items of one row or column group of problem p.
    long long x_items(int p) const { return (long long)fvm2d::x_items_per_row(nx[p], xchunks) * ny[p]; }
    long long y_items(int p) const { return (long long)((nx[p] + 31) / 32) * y_segments(ny[p], T); }

    // Item prefix counts of the listed problems (others get no items) -> device.
    int upload_items()
    {
        std::vector<long long> x0(np + 1, 0), y0(np + 1, 0);
        for (int p = 0; p < np; ++p) {
            x0[p + 1] = x0[p] + (listed[p] ? x_items(p) : 0);
            y0[p + 1] = y0[p] + (listed[p] ? y_items(p) : 0);
        }
        CK(cudaMemcpyAsync(x0_d, x0.data(), sizeof(long long) * (np + 1), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(y0_d, y0.data(), sizeof(long long) * (np + 1), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
        L.x_total = x0[np];
        L.y_total = y0[np];
        return FVM2D_OK;
    }

    // After a graph replay: drops the problems whose loop has ended from the
    // item lists once they hold at least a quarter of the listed x items.
    int compact_items()
    {
        long long ended = 0;
        for (int p = 0; p < np; ++p)
            if (listed[p] && !ctl_h[p].active) ended += x_items(p);
        if (ended == 0 || 4 * ended < L.x_total) return FVM2D_OK;
        for (int p = 0; p < np; ++p)
            if (!ctl_h[p].active) listed[p] = 0;
        if (int rc = upload_items()) return rc;
        drop_graphs();
        return build_graphs();
    }

    int build_graphs()
    {
        if (graph_variant == precision && graph[0] && graph[1]) return FVM2D_OK;
        drop_graphs();
        for (int which = 0; which < 2; ++which) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaSuccess;
            for (int k = 0; k < kGraphSteps[which] && e == cudaSuccess; ++k) e = kBatchVariants[precision].step(L, stream);
            cudaError_t e2 = cudaStreamEndCapture(stream, &g);
            if (e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return cuda_fail(e, "capture of the batched step");
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

    // Resets every problem's run to t = 0 with at most `limit` steps, plans the
    // first steps on the device and replays the step graphs until no problem
    // has a step in flight.
    int run(int limit)
    {
        if (int rc = upload_descriptors()) return rc;
        if (std::count(listed.begin(), listed.end(), 0)) {  // every problem's items back in the lists
            listed.assign(np, 1);
            if (int rc = upload_items()) return rc;
            drop_graphs();
        }
        if (int rc = build_graphs()) return rc;
        std::vector<int> before(np);
        for (int p = 0; p < np; ++p) {
            std::memset(&ctl_h[p], 0, sizeof(StepControl));
            ctl_h[p].step_limit = limit;
        }
        CK(cudaMemcpyAsync(ctl_d, ctl_h, sizeof(StepControl) * np, cudaMemcpyHostToDevice, stream));
        auto t0 = std::chrono::high_resolution_clock::now();
        CK(cudaEventRecord(ev0, stream));
        CK(kBatchVariants[precision].init(L, stream));
        long long launches = 1;
        long long budget = limit;
        for (;;) {
            const int which = budget >= kGraphSteps[0] ? 0 : 1;
            CK(cudaGraphLaunch(graph[which], stream));
            budget -= kGraphSteps[which];
            launches += (long long)kGraphSteps[which] * fvm2d::kStepKernels;
            CK(cudaMemcpyAsync(ctl_h, ctl_d, sizeof(StepControl) * np, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            bool any = false;
            for (int p = 0; p < np && !any; ++p) any = ctl_h[p].active != 0;
            if (!any) break;
            if (int rc = compact_items()) return rc;
        }
        CK(cudaEventRecord(ev1, stream));
        CK(cudaEventSynchronize(ev1));
        auto t1 = std::chrono::high_resolution_clock::now();
        float dms = 0.f;
        CK(cudaEventElapsedTime(&dms, ev0, ev1));
        last_device_ms = dms;
        last_ms = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() / 1000.0;
        last_launches = launches;
        last_cell_updates = 0;
        for (int p = 0; p < np; ++p) last_cell_updates += (long long)nx[p] * ny[p] * ctl_h[p].steps;
        return FVM2D_OK;
    }

    int convert_states(int to)
    {
        for (int p = 0; p < np; ++p) {
            if (!have_state[p]) continue;
            const long long n = 4 * plane(p);
            double *U = base + off[p], *S = base + off[p] + 4 * plane(p);
            if (to == FVM2D_FP32)
                fvm2d::convert_planes<<<148 * 4, 256, 0, stream>>>(fvm2d::Planes<double>{U},
                                                                    fvm2d::Planes<float>{reinterpret_cast<float *>(S)}, n);
            else
                fvm2d::convert_planes<<<148 * 4, 256, 0, stream>>>(fvm2d::Planes<float>{reinterpret_cast<float *>(U)},
                                                                    fvm2d::Planes<double>{S}, n);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(U, S, n * (to == FVM2D_FP32 ? sizeof(float) : sizeof(double)), cudaMemcpyDeviceToDevice,
                               stream));
        }
        CK(cudaStreamSynchronize(stream));
        return FVM2D_OK;
    }
};

namespace {

int check(fvm2d_batch *b)
{
    if (!b) return fail(FVM2D_ERR_INVALID, "null batch handle");
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return FVM2D_OK;
}

int check_problem(fvm2d_batch *b, int p)
{
    if (int rc = check(b)) return rc;
    if (p < 0 || p >= b->np) return fail(FVM2D_ERR_INVALID, "problem index out of range");
    return FVM2D_OK;
}

} // namespace

extern "C" {
#pragma GCC visibility push(default)

int fvm2d_batch_create(fvm2d_batch **out, int nproblems, const int *nx, const int *ny)
{
    if (!out) return fail(FVM2D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (nproblems < 1 || !nx || !ny) return fail(FVM2D_ERR_INVALID, "need at least one problem and its sizes");
    for (int p = 0; p < nproblems; ++p) {
        if (nx[p] < 6 || ny[p] < 6) return fail(FVM2D_ERR_INVALID, "every nx and ny must be at least 6");
        if ((long long)nx[p] * ny[p] > (1ll << 31) - 1) return fail(FVM2D_ERR_INVALID, "nx * ny must stay below 2^31");
        if ((long long)((nx[p] + 31) / 32 * 32) * ny[p] > (1ll << 31) - 1)
            return fail(FVM2D_ERR_INVALID, "the padded plane, round_up(nx, 32) * ny, must stay below 2^31");
    }
    fvm2d_batch *b = new (std::nothrow) fvm2d_batch();
    if (!b) return fail(FVM2D_ERR_INVALID, "out of host memory");
    int rc = FVM2D_OK;
    cudaError_t e;
    do {
        try {
            b->np = nproblems;
            b->nx.assign(nx, nx + nproblems);
            b->ny.assign(ny, ny + nproblems);
            b->pitch.resize(nproblems);
            b->off.resize(nproblems);
            b->strategy.assign(nproblems, FVM2D_OUTFLOW);
            b->width.assign(nproblems, 1.0);
            b->height.assign(nproblems, 1.0);
            b->t_end.assign(nproblems, 0.0);
            b->cfl.assign(nproblems, 0.5);
            b->alpha.assign(nproblems, 1.9);
            b->gamma.assign(nproblems, 1.4);
            b->have_state.assign(nproblems, 0);
        } catch (...) {
            rc = fail(FVM2D_ERR_INVALID, "out of host memory");
            break;
        }
        long long total = 0;
        for (int p = 0; p < nproblems; ++p) {
            b->pitch[p] = (nx[p] + 31) / 32 * 32;
            b->off[p] = total;
            total += 12 * b->plane(p);  // U, A, B
        }
        b->total_elems = total;
        if ((e = cudaGetDevice(&b->device))) { rc = cuda_fail(e, "cudaGetDevice"); break; }
        for (int v = 0; v < kNumBatchVariants && !rc; ++v) {
            int ox = 0, oy = 0;
            if ((e = kBatchVariants[v].prepare(&ox, &oy))) rc = cuda_fail(e, "kernel attributes");
            if (v == 0) b->occ_x = ox, b->occ_y = oy;
        }
        if (rc) break;
        if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking))) { rc = cuda_fail(e, "cudaStreamCreate"); break; }
        if ((e = cudaMalloc(&b->base, sizeof(double) * total))) { rc = cuda_fail(e, "cudaMalloc(batch states)"); break; }
        if ((e = cudaMalloc(&b->prob_d, sizeof(BatchProblem) * nproblems))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&b->ctl_d, sizeof(StepControl) * nproblems))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaMallocHost(&b->ctl_h, sizeof(StepControl) * nproblems))) { rc = cuda_fail(e, "cudaMallocHost"); break; }
        if ((e = cudaMalloc(&b->x0_d, sizeof(long long) * (nproblems + 1)))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&b->y0_d, sizeof(long long) * (nproblems + 1)))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&b->rb0_d, sizeof(int) * (nproblems + 1)))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&b->ib0_d, sizeof(int) * (nproblems + 1)))) { rc = cuda_fail(e, "cudaMalloc"); break; }
        if ((e = cudaEventCreate(&b->ev0)) || (e = cudaEventCreate(&b->ev1))) { rc = cuda_fail(e, "cudaEventCreate"); break; }
        std::memset(b->ctl_h, 0, sizeof(StepControl) * nproblems);
        if ((e = cudaMemsetAsync(b->base, 0, sizeof(double) * total, b->stream))) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((e = cudaMemsetAsync(b->ctl_d, 0, sizeof(StepControl) * nproblems, b->stream))) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((e = cudaStreamSynchronize(b->stream))) { rc = cuda_fail(e, "cudaStreamSynchronize"); break; }
    } while (0);
    if (rc) {
        fvm2d_batch_destroy(b);
        return rc;
    }
    *out = b;
    return FVM2D_OK;
}

int fvm2d_batch_destroy(fvm2d_batch *b)
{
    if (!b) return FVM2D_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->drop_graphs();
    cudaFree(b->base);
    cudaFree(b->prob_d);
    cudaFree(b->ctl_d);
    if (b->ctl_h) cudaFreeHost(b->ctl_h);
    cudaFree(b->x0_d);
    cudaFree(b->y0_d);
    cudaFree(b->rb0_d);
    cudaFree(b->ib0_d);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FVM2D_OK;
}

int fvm2d_batch_set_problem(fvm2d_batch *b, int p, double width, double height, double t_end, double cfl, double alpha,
                            double gamma, int strategy)
{
    if (int rc = check_problem(b, p)) return rc;
    if (!(width > 0.0 && height > 0.0 && cfl > 0.0 && gamma > 1.0) || t_end != t_end || alpha != alpha)
        return fail(FVM2D_ERR_INVALID, "width, height and cfl must be positive, gamma above 1");
    if (strategy < FVM2D_OUTFLOW || strategy > FVM2D_REFLECTIVE_TB) return fail(FVM2D_ERR_INVALID, "unknown ghost-cell strategy");
    b->width[p] = width;
    b->height[p] = height;
    b->t_end[p] = t_end;
    b->cfl[p] = cfl;
    b->alpha[p] = alpha;
    b->gamma[p] = gamma;
    b->strategy[p] = strategy;
    b->dirty = true;
    return FVM2D_OK;
}

int fvm2d_batch_set_precision(fvm2d_batch *b, int precision)
{
    if (int rc = check(b)) return rc;
    if (precision < 0 || precision >= kNumBatchVariants) return fail(FVM2D_ERR_INVALID, "unknown precision");
    if ((precision == FVM2D_FP32) != (b->precision == FVM2D_FP32)) {
        if (int rc = b->convert_states(precision)) return rc;
        b->dirty = true;  // element offsets depend on the storage type
    }
    b->precision = precision;
    b->drop_graphs();
    return FVM2D_OK;
}

int fvm2d_batch_set_state(fvm2d_batch *b, int p, const double *cells, int stride)
{
    if (int rc = check_problem(b, p)) return rc;
    if (!cells) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    double *U = b->base + b->off[p], *S = U + 4 * b->plane(p);  // staging: the problem's A and B regions
    const size_t bytes = sizeof(double) * (size_t)b->nx[p] * b->ny[p] * stride;
    const cudaMemcpyKind kind = fvm2d::is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(S, cells, bytes, kind, b->stream));
    if (b->precision == FVM2D_FP32)
        fvm2d::aos_to_soa<<<148 * 4, 256, 0, b->stream>>>(S, stride, fvm2d::Planes<float>{reinterpret_cast<float *>(U)},
                                                           b->nx[p], b->ny[p], b->pitch[p], b->plane(p));
    else
        fvm2d::aos_to_soa<<<148 * 4, 256, 0, b->stream>>>(S, stride, fvm2d::Planes<double>{U}, b->nx[p], b->ny[p],
                                                           b->pitch[p], b->plane(p));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(b->stream));
    b->have_state[p] = 1;
    return FVM2D_OK;
}

int fvm2d_batch_get_state(fvm2d_batch *b, int p, double *cells, int stride)
{
    if (int rc = check_problem(b, p)) return rc;
    if (!cells) return fail(FVM2D_ERR_INVALID, "null state pointer");
    if (stride != 4 && stride != 5) return fail(FVM2D_ERR_INVALID, "stride must be 4 or 5 doubles per cell");
    if (!b->have_state[p]) return fail(FVM2D_ERR_STATE, "no state has been set for this problem");
    double *U = b->base + b->off[p], *S = U + 4 * b->plane(p);
    if (b->precision == FVM2D_FP32)
        fvm2d::soa_to_aos<<<148 * 4, 256, 0, b->stream>>>(fvm2d::Planes<float>{reinterpret_cast<float *>(U)}, b->nx[p],
                                                           b->ny[p], b->pitch[p], b->plane(p), stride, S);
    else
        fvm2d::soa_to_aos<<<148 * 4, 256, 0, b->stream>>>(fvm2d::Planes<double>{U}, b->nx[p], b->ny[p], b->pitch[p],
                                                           b->plane(p), stride, S);
    CK(cudaGetLastError());
    const size_t bytes = sizeof(double) * (size_t)b->nx[p] * b->ny[p] * stride;
    const cudaMemcpyKind kind = fvm2d::is_device_pointer(cells) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(cells, S, bytes, kind, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return FVM2D_OK;
}

int fvm2d_batch_solve(fvm2d_batch *b)
{
    nvtxRangePushA("fvm2d_batch_solve");
    struct Pop { ~Pop() { nvtxRangePop(); } } pop_;
    if (int rc = check(b)) return rc;
    for (int p = 0; p < b->np; ++p)
        if (!b->have_state[p]) return fail(FVM2D_ERR_STATE, "every problem needs a state before solving");
    return b->run(INT_MAX);
}

int fvm2d_batch_get_time(fvm2d_batch *b, int p, double *t, int *steps)
{
    if (int rc = check_problem(b, p)) return rc;
    if (t) *t = b->ctl_h[p].t;
    if (steps) *steps = b->ctl_h[p].steps;
    return FVM2D_OK;
}

int fvm2d_batch_get_run_stats(fvm2d_batch *b, double *device_ms, long long *kernel_launches, long long *cell_updates)
{
    if (int rc = check(b)) return rc;
    if (device_ms) *device_ms = b->last_device_ms;
    if (kernel_launches) *kernel_launches = b->last_launches;
    if (cell_updates) *cell_updates = b->last_cell_updates;
    return FVM2D_OK;
}

int fvm2d_batch_autotune(fvm2d_batch *b, int trial_steps, int *segment_interfaces, int *grid_blocks)
{
    if (int rc = check(b)) return rc;
    for (int p = 0; p < b->np; ++p)
        if (!b->have_state[p]) return fail(FVM2D_ERR_STATE, "every problem needs a state before tuning");
    if (trial_steps < 1) return fail(FVM2D_ERR_INVALID, "trial_steps must be positive");
    // keep the states: every trial starts from them
    double *saved = nullptr;
    const size_t per_elem = (b->precision == FVM2D_FP32) ? sizeof(float) : sizeof(double);
    size_t bytes = 0;
    for (int p = 0; p < b->np; ++p) bytes += 4 * b->plane(p) * per_elem;
    CK(cudaMalloc(&saved, bytes));
    auto copy_states = [&](bool save) -> cudaError_t {
        size_t o = 0;
        for (int p = 0; p < b->np; ++p) {
            const size_t n = 4 * b->plane(p) * per_elem;
            char *U = reinterpret_cast<char *>(b->base + b->off[p]);
            char *K = reinterpret_cast<char *>(saved) + o;
            cudaError_t e = cudaMemcpyAsync(save ? K : U, save ? U : K, n, cudaMemcpyDeviceToDevice, b->stream);
            if (e) return e;
            o += n;
        }
        return cudaStreamSynchronize(b->stream);
    };
    cudaError_t e = copy_states(true);
    int best_T = b->T, best_g = 0;
    double best = 1e300;
    int rc = FVM2D_OK;
    const int Ts[] = {16, 32, 64};
    const int mults[] = {1, 2, 4};
    for (int ti = 0; ti < 3 && !e && !rc; ++ti)
        for (int mi = 0; mi < 3 && !e && !rc; ++mi) {
            b->T = Ts[ti];
            b->grid_x = mults[mi] * b->occ_x;
            b->grid_y = mults[mi] * b->occ_y;
            b->dirty = true;
            if ((rc = b->run(trial_steps))) break;
            const double ms = b->last_device_ms;
            if (ms < best) best = ms, best_T = Ts[ti], best_g = mults[mi];
            e = copy_states(false);
        }
    cudaFree(saved);
    if (rc) return rc;
    if (e) return cuda_fail(e, "state copy during tuning");
    b->T = best_T;
    b->grid_x = best_g * b->occ_x;
    b->grid_y = best_g * b->occ_y;
    b->dirty = true;
    std::memset(b->ctl_h, 0, sizeof(StepControl) * b->np);
    if (segment_interfaces) *segment_interfaces = best_T;
    if (grid_blocks) *grid_blocks = b->grid_x;
    return FVM2D_OK;
}

#pragma GCC visibility pop
} // extern "C"
