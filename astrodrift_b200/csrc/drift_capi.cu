// drift_capi.cu -- the C ABI declared in include/drift_b200.h.
//
// Host-side validation, launch geometry, a library-owned persistent device
// context (stream and grow-only buffers per device) and the host-buffer path
// that pipelines particle chunks: copy-in, integration and copy-out of
// different chunks overlap on two streams.  In the reference every stage
// creates a CUDA context, JIT-loads the module and copies a zeroed output
// buffer to the device (src/dispatch/gpu/cuda_oxide.rs:9-86); none of that is
// repeated here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <chrono>
#include <thread>
#include <vector>

#include "drift_b200.h"
#include "drift_bulge_table.h"
#include "drift_launch_args.cuh"
#include "drift_trace.h"

namespace drift {
void fill_bulge_table(double s, BulgeTable *t)
{
    fill_bulge_table_impl(s, t->c, BULGE_PIECES, BULGE_PIECE_DEG);
}
}  // namespace drift

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DRIFT_ERROR_OUT_OF_MEMORY : DRIFT_ERROR_CUDA;
}

#define DRIFT_CUDA_TRY(expr, what)                 \
    do {                                           \
        cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

constexpr int64_t DEFAULT_MAX_STEPS = 100000000;  // 10^8 attempts per particle
constexpr int DEFAULT_BLOCK = 128;
constexpr size_t CURSOR_BYTES = 256;  // one 8-byte cursor, padded to an allocation granule

// Device buffer that only grows.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need)
    {
        if (need <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, need);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T>
    T *as() const
    {
        return static_cast<T *>(ptr);
    }
};

struct HostBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need)
    {
        if (need <= bytes) return cudaSuccess;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMallocHost(&ptr, need);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    void release()
    {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// State of the host path on one device: two streams and grow-only device
// and page-locked buffers.  The implicit context of each device is created
// on first use and kept for the life of the process; explicit ones
// (drift_context_create) are freed by drift_context_destroy.
struct DeviceContext {
    int device = -1;
    int sm_count = 0;
    std::mutex mu;  // serialises host-buffer calls that share the buffers below
    cudaStream_t streams[2] = {nullptr, nullptr};
    cudaStream_t poll_stream = nullptr;  // streamed copy-out: reads the chunk counters
    cudaEvent_t done[2] = {nullptr, nullptr};
    DevBuf y0, grid, out[2], yfin, status, err, acc, rej, cursor, origins;
    DevBuf src_traj, src_table, src_origins;  // drift_origin_table_host
    HostBuf stage[2];
    HostBuf poll;  // streamed copy-out: the chunk completion counters, read back

    DevBuf *dev_bufs[14] = {&y0, &grid, &out[0], &out[1], &yfin, &status, &err, &acc, &rej, &cursor,
                            &origins, &src_traj, &src_table, &src_origins};

    // Streams and events on `device` (which must be current).
    int init(int dev);
    size_t device_bytes() const
    {
        size_t b = 0;
        for (const DevBuf *d : dev_bufs) b += d->bytes;
        return b;
    }
    size_t pinned_bytes() const { return stage[0].bytes + stage[1].bytes + poll.bytes; }
    // Waits for the streams and frees every buffer, stream and event (device current).
    void release()
    {
        for (int i = 0; i < 2; i++)
            if (streams[i]) cudaStreamSynchronize(streams[i]);
        for (DevBuf *d : dev_bufs) d->release();
        poll.release();
        if (poll_stream) {
            cudaStreamSynchronize(poll_stream);
            cudaStreamDestroy(poll_stream);
            poll_stream = nullptr;
        }
        for (int i = 0; i < 2; i++) {
            stage[i].release();
            if (done[i]) cudaEventDestroy(done[i]);
            if (streams[i]) cudaStreamDestroy(streams[i]);
            done[i] = nullptr;
            streams[i] = nullptr;
        }
    }
};

std::mutex g_ctx_mu;
std::vector<DeviceContext *> g_ctx;

int current_context(DeviceContext **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(DRIFT_ERROR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_ctx_mu);
    if ((int)g_ctx.size() <= dev) g_ctx.resize(dev + 1, nullptr);
    if (!g_ctx[dev]) {
        auto *c = new DeviceContext();
        int rc = c->init(dev);
        if (rc) {
            c->release();
            delete c;
            return rc;
        }
        g_ctx[dev] = c;
    }
    *out = g_ctx[dev];
    return DRIFT_SUCCESS;
}

int DeviceContext::init(int dev)
{
    device = dev;
    DRIFT_CUDA_TRY(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev),
                   "cudaDeviceGetAttribute");
    for (int i = 0; i < 2; i++) {
        DRIFT_CUDA_TRY(cudaStreamCreateWithFlags(&streams[i], cudaStreamNonBlocking), "cudaStreamCreate");
        DRIFT_CUDA_TRY(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    DRIFT_CUDA_TRY(cudaStreamCreateWithFlags(&poll_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    return DRIFT_SUCCESS;
}

// Makes `device` current for one scope and restores the caller's device.
struct ScopedDevice {
    int saved = -1;
    bool switched = false;
    explicit ScopedDevice(int device)
    {
        if (cudaGetDevice(&saved) == cudaSuccess && saved != device) switched = cudaSetDevice(device) == cudaSuccess;
        cudaGetLastError();
    }
    ~ScopedDevice()
    {
        if (switched) cudaSetDevice(saved);
    }
};

bool is_finite_value(double v) { return std::isfinite(v); }

// A force model's own consistency (its pointers are checked by the caller).
int validate_model(const drift_force_model *m)
{
    if (!m) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "potential kind DRIFT_POT_MODEL needs force_model");
    if (m->n_static < 0 || m->n_static > DRIFT_MAX_COMPONENTS || m->n_groups < 0 ||
        m->n_groups > DRIFT_MAX_COMPONENTS)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "a force model has at most " + std::to_string(DRIFT_MAX_COMPONENTS) +
                        " stationary parts and source groups");
    double alpha = 0.0;
    bool bovy = false;
    for (int i = 0; i < m->n_static; i++) {
        const int k = m->statics[i].kind;
        if (k < DRIFT_POT_KEPLER || k > DRIFT_POT_KEPLER_CARTESIAN)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown kind of a force model's stationary part");
        if (k == DRIFT_POT_BOVY) {
            if (bovy && m->statics[i].bulge_alpha != alpha)
                return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the Bovy parts of a force model must share bulge_alpha");
            bovy = true;
            alpha = m->statics[i].bulge_alpha;
        }
    }
    int64_t need = 0;
    for (int g = 0; g < m->n_groups; g++) {
        const drift_source_group &G = m->groups[g];
        if (G.kind != DRIFT_POT_KEPLER_CARTESIAN && G.kind != DRIFT_POT_PLUMMER)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                        "only Kepler and Plummer potentials can currently be attached to particles");
        if (G.first < 0 || G.count < 0) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "negative source range");
        need = std::max(need, G.first + G.count);
    }
    if (m->n_groups > 0) {
        if (need > m->n_sources) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "source ranges exceed n_sources");
        if (m->n_segments < 1 || !m->origins)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "moving sources need an origin table (n_segments >= 1)");
        if (!is_finite_value(m->t0) || !is_finite_value(m->dt) || m->dt == 0.0)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the origin table needs finite t0 and a nonzero dt");
    }
    return DRIFT_SUCCESS;
}

// The bulge table a model needs (from its first Bovy part), or none.
void fill_model_bulge(const drift_force_model &m, drift::BulgeTable *t)
{
    for (int i = 0; i < m.n_static; i++)
        if (m.statics[i].kind == DRIFT_POT_BOVY) {
            drift::fill_bulge_table(1.5 - 0.5 * m.statics[i].bulge_alpha, t);
            return;
        }
}

int validate(const drift_launch *L, bool device_pointers)
{
    if (!L) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "launch is NULL");
    if (L->method != DRIFT_DOPR54 && L->method != DRIFT_DOP853)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown method");
    if (L->precision != DRIFT_PRECISION_EXACT && L->precision != DRIFT_PRECISION_FMA)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown precision");
    if (L->schedule != DRIFT_SCHEDULE_PLAIN && L->schedule != DRIFT_SCHEDULE_PERSISTENT &&
        L->schedule != DRIFT_SCHEDULE_ORDERED)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown schedule");
    if (L->schedule == DRIFT_SCHEDULE_ORDERED && L->n > (int64_t)UINT32_MAX)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the ordered schedule supports at most 2^32 - 1 particles");
    const int max_block = std::min(drift::max_threads_exact(), drift::max_threads_fma());
    if (L->block_size != 0 && (L->block_size < 32 || L->block_size > max_block || L->block_size % 32))
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "block_size must be 0 or a multiple of 32 in [32, " + std::to_string(max_block) + "]");
    const int k = L->potential.kind;
    if (k < DRIFT_POT_KEPLER || k > DRIFT_POT_MODEL)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown potential kind");
    if (k == DRIFT_POT_MODEL) {
        int rc = validate_model(L->force_model);
        if (rc) return rc;
        if (L->force_model->n_groups > 0 && device_pointers &&
            reinterpret_cast<uintptr_t>(L->force_model->origins) % 8)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the origin table must be 8-byte aligned");
        if (L->tape) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the step tape supports single potentials");
    }
    if (L->n < 1) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "n must be >= 1");
    if (L->n > (int64_t(1) << 40)) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "n is too large");
    if (L->nt < 2 || L->nt > INT32_MAX - 1)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "nt must be in [2, 2^31 - 2]");
    if (!L->y0) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "y0 is NULL");
    if (L->y0_layout != DRIFT_Y0_ROWS && L->y0_layout != DRIFT_Y0_COLUMNS)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown y0_layout");
    if (L->y0_layout == DRIFT_Y0_COLUMNS && L->y0_stride != 0 && L->y0_stride < L->n)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "y0_stride must be 0 or at least n");
    if (!L->ts && !L->t_end) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "either ts or t_end is required");
    if (!L->ts && !is_finite_value(L->t0)) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "t0 must be finite");
    if (!is_finite_value(L->rtol_ln) || !is_finite_value(L->atol_ln))
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "tolerances must be finite logarithms");
    if (device_pointers &&
        (reinterpret_cast<uintptr_t>(L->y0) % (L->y0_layout == DRIFT_Y0_ROWS ? 16 : 8) ||
         (L->out && reinterpret_cast<uintptr_t>(L->out) % 16) ||
         (L->y_final && reinterpret_cast<uintptr_t>(L->y_final) % 16)))
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "y0 (rows), out and y_final must be 16-byte aligned, y0 columns 8-byte aligned");
    if (L->tape) {
        if (!device_pointers)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the step tape is a device buffer (device entry points only)");
        if (L->method != DRIFT_DOP853)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the step tape is recorded by DOP853 only");
        if (L->tape_steps < 1 || L->tape_steps > (int64_t(1) << 40) / std::max<int64_t>(L->n, 1))
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "tape_steps must be >= 1 (and n * tape_steps <= 2^40)");
        if (L->tape_stride > DRIFT_MAX_TAPE_STRIDE)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                        "tape_stride must be at most " + std::to_string(DRIFT_MAX_TAPE_STRIDE));
        if (reinterpret_cast<uintptr_t>(L->tape) % 16)
            return fail(DRIFT_ERROR_INVALID_ARGUMENT, "the tape must be 16-byte aligned");
    }
    return DRIFT_SUCCESS;
}

int block_of(const drift_launch *L)
{
    if (L->block_size) return L->block_size;
    return std::min(DEFAULT_BLOCK, std::min(drift::max_threads_exact(), drift::max_threads_fma()));
}

drift::KernelArgs make_args(const drift_launch *L)
{
    drift::KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = L->n;
    a.y0 = L->y0;
    a.nt = (int32_t)L->nt;
    a.persistent = L->schedule != DRIFT_SCHEDULE_PLAIN;
    a.ts = L->ts;
    a.t0 = L->t0;
    a.t_end = L->t_end;
    a.out = L->out;
    a.y_final = L->y_final;
    // The reference's DOP853 exponentiates the logarithmic tolerances at the
    // start of every particle (dop853.rs:340-341); the same host libm exp is
    // applied once here.
    a.rtol = std::exp(L->rtol_ln);
    a.atol = std::exp(L->atol_ln);
    a.tol54.e_rtol = a.rtol;
    a.tol54.e_atol = a.atol;
    a.dt_one = L->dt_one;
    a.max_steps = L->max_steps > 0 ? L->max_steps : DEFAULT_MAX_STEPS;
    a.timeout_ns = L->timeout_s > 0 ? (uint64_t)(L->timeout_s * 1e9) : 0;
    a.status = L->status;
    a.err_code = L->err_code;
    a.n_accepted = L->n_accepted;
    a.n_rejected = L->n_rejected;
    a.tape = L->tape;
    a.tape_steps = L->tape_steps;
    a.arbitrary_times = L->arbitrary_times != 0;
    a.tape_stride = L->tape_stride;
    a.sparse_output = L->nt <= drift::SPARSE_OUTPUT_NT;
    a.y0_stride = L->y0_layout == DRIFT_Y0_COLUMNS ? (L->y0_stride ? L->y0_stride : L->n) : 0;
    a.potential = L->potential;
    if (L->potential.kind == DRIFT_POT_BOVY)
        drift::fill_bulge_table(1.5 - 0.5 * L->potential.bulge_alpha, &a.bulge);
    if (L->potential.kind == DRIFT_POT_MODEL) {
        a.model = *L->force_model;
        fill_model_bulge(a.model, &a.bulge);
    }
    return a;
}

cudaError_t launch_args(const drift::KernelArgs &a, int method, int precision, int grid, int block,
                        cudaStream_t s)
{
    return precision == DRIFT_PRECISION_EXACT ? drift::launch_exact(a, method, grid, block, s)
                                              : drift::launch_fma(a, method, grid, block, s);
}

// Workspace of a request: [cursor, 256 B][ordered: bucket counts 1 KiB]
// [ordered: queue, 4 B per particle][ordered: cost keys, 1 B per particle].
size_t workspace_bytes(const drift_launch *L)
{
    if (L->schedule == DRIFT_SCHEDULE_PERSISTENT) return CURSOR_BYTES;
    if (L->schedule == DRIFT_SCHEDULE_ORDERED) {
        size_t b = CURSOR_BYTES + 1024 + 5 * (size_t)L->n;
        return (b + 255) / 256 * 256;
    }
    return 0;
}

int grid_for(int sm_count, const drift_launch *L, int64_t n, int block, int *grid)
{
    int64_t blocks = (n + block - 1) / block;
    if (L->schedule != DRIFT_SCHEDULE_PLAIN) {
        int per_sm = 0;
        cudaError_t e = L->precision == DRIFT_PRECISION_EXACT
                            ? drift::occupancy_exact(L->method, L->potential.kind, block, L->tape != nullptr,
                                                     &per_sm)
                            : drift::occupancy_fma(L->method, L->potential.kind, block, L->tape != nullptr,
                                                   &per_sm);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        int64_t cap = (int64_t)std::max(per_sm, 1) * sm_count;
        blocks = std::min(blocks, cap);
    }
    if (blocks > INT32_MAX) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "too many particles for one launch");
    *grid = (int)blocks;
    return DRIFT_SUCCESS;
}

// Launch prepared kernel arguments `a` for request geometry `L` (n = all
// particles of the launch) with `ws` (workspace_bytes(L) bytes, 256-byte
// aligned) as scratch.  Every launch clears the parts that must start at 0.
int launch_args_on_workspace(int sm_count, const drift_launch *L, drift::KernelArgs &a, void *ws,
                             cudaStream_t s)
{
    const int block = block_of(L);
    int grid = 0;
    int rc = grid_for(sm_count, L, L->n, block, &grid);
    if (rc) return rc;
    if (a.persistent) {
        char *base = static_cast<char *>(ws);
        a.cursor = reinterpret_cast<unsigned long long *>(base);
        DRIFT_CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(unsigned long long), s), "cudaMemsetAsync");
        if (L->schedule == DRIFT_SCHEDULE_ORDERED) {
            unsigned *counts = reinterpret_cast<unsigned *>(base + CURSOR_BYTES);
            uint32_t *order = reinterpret_cast<uint32_t *>(base + CURSOR_BYTES + 1024);
            uint8_t *keys = reinterpret_cast<uint8_t *>(order + L->n);
            DRIFT_CUDA_TRY(drift::build_order(a, L->method, keys, counts, order, sm_count, s),
                           "ordering kernels");
            a.order = order;
        }
    }
    DRIFT_CUDA_TRY(launch_args(a, L->method, L->precision, grid, block, s), "kernel launch");
    return DRIFT_SUCCESS;
}

int launch_on_workspace(int sm_count, const drift_launch *L, void *ws, cudaStream_t s)
{
    drift::KernelArgs a = make_args(L);
    return launch_args_on_workspace(sm_count, L, a, ws, s);
}

// A batch of requests sharing method, precision, schedule, block size,
// potential, tolerances and step limits, as one launch over their
// concatenated particles.  Request i occupies [first_i, first_i + n_i).
int check_batch(const drift_launch *R, int32_t count)
{
    if (!R || count < 1 || count > drift::MAX_BATCH)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "a batch holds 1 to " + std::to_string(drift::MAX_BATCH) + " requests");
    for (int32_t i = 0; i < count; i++) {
        int rc = validate(&R[i], true);
        if (rc) return rc;
        if (R[i].tape) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "batched launches record no step tape");
        const drift_launch &A = R[0], &B = R[i];
        if (B.method != A.method || B.precision != A.precision || B.schedule != A.schedule ||
            B.block_size != A.block_size || std::memcmp(&B.potential, &A.potential, sizeof(A.potential)) ||
            B.rtol_ln != A.rtol_ln || B.atol_ln != A.atol_ln || B.dt_one != A.dt_one ||
            B.max_steps != A.max_steps || B.timeout_s != A.timeout_s ||
            (B.arbitrary_times != 0) != (A.arbitrary_times != 0) ||
            (A.potential.kind == DRIFT_POT_MODEL && B.force_model != A.force_model))
            return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                        "batched requests must share method, precision, schedule, block size, "
                        "potential (and force model), tolerances, first step and limits");
    }
    return DRIFT_SUCCESS;
}

int launch_batch(int sm_count, const drift_launch *R, int32_t count, void *ws, cudaStream_t s)
{
    drift::KernelArgs a = make_args(&R[0]);
    drift_launch geometry = R[0];
    int64_t first = 0;
    a.nsegs = count;
    for (int32_t i = 0; i < count; i++) {
        drift::Segment &S = a.segs[i];
        S.first = first;
        S.n = R[i].n;
        S.y0 = R[i].y0;
        S.y0_stride = R[i].y0_layout == DRIFT_Y0_COLUMNS ? (R[i].y0_stride ? R[i].y0_stride : R[i].n) : 0;
        S.ts = R[i].ts;
        S.t0 = R[i].t0;
        S.t_end = R[i].t_end;
        S.nt = (int32_t)R[i].nt;
        S.out = R[i].out;
        S.y_final = R[i].y_final;
        S.status = R[i].status;
        S.err_code = R[i].err_code;
        S.n_accepted = R[i].n_accepted;
        S.n_rejected = R[i].n_rejected;
        first += R[i].n;
        if (R[i].nt > drift::SPARSE_OUTPUT_NT) a.sparse_output = 0;
    }
    a.n = first;
    geometry.n = first;
    return launch_args_on_workspace(sm_count, &geometry, a, ws, s);
}

int launch_device(DeviceContext *ctx, const drift_launch *L, void *ws, cudaStream_t s)
{
    return launch_on_workspace(ctx->sm_count, L, ws, s);
}

bool is_pinned(const void *p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

}  // namespace

// Shared with the request server (drift_server.cu).
int drift_internal_launch_batch(int sm_count, const drift_launch *R, int32_t count, void *ws,
                                cudaStream_t s)
{
    int rc = check_batch(R, count);
    if (rc) return rc;
    return launch_batch(sm_count, R, count, ws, s);
}

int drift_internal_fail(int code, const char *msg) { return fail(code, msg); }

extern "C" {

int drift_abi_version(void) { return DRIFT_ABI_VERSION; }

const char *drift_result_string(int code)
{
    switch (code) {
    case DRIFT_SUCCESS: return "success";
    case DRIFT_ERROR_INVALID_ARGUMENT: return "invalid argument";
    case DRIFT_ERROR_CUDA: return "CUDA error";
    case DRIFT_ERROR_WORKSPACE: return "workspace too small";
    case DRIFT_ERROR_NO_DEVICE: return "no CUDA device";
    case DRIFT_ERROR_OUT_OF_MEMORY: return "out of device memory";
    case DRIFT_ERROR_TIMEOUT: return "timed out";
    case DRIFT_ERROR_CANCELLED: return "cancelled";
    default: return "unknown error";
    }
}

const char *drift_last_error(void) { return g_last_error.c_str(); }

// Series / continued-fraction lower incomplete gamma (Numerical Recipes 3rd
// ed. section 6.2), host copy used to normalise the bulge.
static double host_lower_gamma(double s, double x, double gamma_s)
{
    const double eps = 1.1102230246251565e-16;
    const double fpmin = 1e-300;
    if (!(x > 0.0)) return 0.0;
    double prefactor = std::exp(s * std::log(x) - x);
    if (x < s + 1.0) {
        double ap = s, del = 1.0 / s, sum = del;
        for (int n = 0; n < 500; ++n) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (std::fabs(del) < std::fabs(sum) * eps) break;
        }
        return sum * prefactor;
    }
    double b = x + 1.0 - s, c = 1.0 / fpmin, d = 1.0 / b, h = d;
    for (int i = 1; i < 500; ++i) {
        double an = -i * (i - s);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < fpmin) d = fpmin;
        c = b + an / c;
        if (std::fabs(c) < fpmin) c = fpmin;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < eps) break;
    }
    return gamma_s - prefactor * h;
}

int drift_potential_bovy(drift_potential *p, double alpha, double rc, double bulge_force_at_1,
                         double mn_amp, double mn_a, double mn_b, double nfw_amp, double nfw_a)
{
    if (!p) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "potential is NULL");
    if (!(alpha < 3.0) || !(rc > 0.0) || !is_finite_value(bulge_force_at_1))
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "bulge needs alpha < 3, rc > 0 and a finite force");
    std::memset(p, 0, sizeof(*p));
    p->kind = DRIFT_POT_BOVY;
    p->bulge_alpha = alpha;
    p->bulge_rc = rc;
    double s = 1.5 - 0.5 * alpha;
    p->bulge_gamma_s = std::tgamma(s);
    p->bulge_k = bulge_force_at_1 / host_lower_gamma(s, 1.0 / (rc * rc), p->bulge_gamma_s);
    p->mn_amp = mn_amp;
    p->mn_a = mn_a;
    p->mn_b = mn_b;
    p->nfw_amp = nfw_amp;
    p->nfw_a = nfw_a;
    return DRIFT_SUCCESS;
}

int drift_query_workspace(const drift_launch *launch, size_t *bytes)
{
    if (!launch || !bytes) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    *bytes = workspace_bytes(launch);
    return DRIFT_SUCCESS;
}

int drift_integrate(const drift_launch *launch, void *stream)
{
    drift::TraceRange trace("drift integrate");
    int rc = validate(launch, true);
    if (rc) return rc;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    const size_t need = workspace_bytes(launch);
    if (need) {
        if (!launch->workspace || launch->workspace_bytes < need ||
            reinterpret_cast<uintptr_t>(launch->workspace) % 8)
            return fail(DRIFT_ERROR_WORKSPACE, "this schedule needs an 8-byte aligned workspace of " +
                                                   std::to_string(need) + " bytes (drift_query_workspace)");
    }
    return launch_device(ctx, launch, launch->workspace, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// drift_integrate_noalloc: drift_integrate for callers that cannot allocate
// device memory.  Its only scratch -- the persistent schedule's claim cursor
// -- lives in the fixed array below, which the module carries for as long as
// the library is loaded on a device.
// ---------------------------------------------------------------------------

static __device__ __align__(256) unsigned char g_noalloc_scratch[DRIFT_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch in the calling thread's current
// context.  In host code the array's name is only a host-side stand-in;
// kernels must receive this address instead.  It is looked up on every call
// (a host-side table lookup once the module is loaded, no allocation): an
// address saved from an earlier call would be stale after a device reset or
// under another context on the same device.
int noalloc_scratch(void **out)
{
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    *out = ptr;
    return DRIFT_SUCCESS;
}

}  // namespace

extern "C" int drift_integrate_noalloc(const drift_launch *launch, void *stream)
{
    int rc = validate(launch, true);
    if (rc) return rc;
    size_t need = 0;
    rc = drift_query_workspace(launch, &need);
    if (rc) return rc;
    if (need > DRIFT_NOALLOC_SCRATCH_BYTES)
        return fail(DRIFT_ERROR_WORKSPACE,
                    "drift_integrate_noalloc: this request needs " + std::to_string(need) +
                        " bytes of scratch but the library's fixed scratch holds " +
                        std::to_string((size_t)DRIFT_NOALLOC_SCRATCH_BYTES) +
                        "; use drift_integrate with a caller-provided workspace");
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(DRIFT_ERROR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    void *scratch = nullptr;
    rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    int sm_count = 0;
    DRIFT_CUDA_TRY(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device),
                   "cudaDeviceGetAttribute");
    // The array keeps the previous call's contents; launch_on_workspace clears
    // what must start at zero on the caller's stream.
    rc = launch_on_workspace(sm_count, launch, scratch, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    return DRIFT_SUCCESS;
}

extern "C" {

int drift_integrate_batch(const drift_launch *requests, int32_t count, void *stream)
{
    int rc = check_batch(requests, count);
    if (rc) return rc;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    if (requests[0].schedule != DRIFT_SCHEDULE_PLAIN) {
        drift_launch all = requests[0];
        all.n = 0;
        for (int32_t i = 0; i < count; i++) all.n += requests[i].n;
        const size_t need = workspace_bytes(&all);
        if (!requests[0].workspace || requests[0].workspace_bytes < need ||
            reinterpret_cast<uintptr_t>(requests[0].workspace) % 8)
            return fail(DRIFT_ERROR_WORKSPACE, "this batch needs an 8-byte aligned requests[0].workspace of " +
                                                   std::to_string(need) + " bytes");
    }
    return launch_batch(ctx->sm_count, requests, count, requests[0].workspace,
                        static_cast<cudaStream_t>(stream));
}

int drift_force(const drift_potential *potential, int64_t n, const double *xyz, double *acc,
                void *stream)
{
    return drift_force_precision(potential, DRIFT_PRECISION_EXACT, n, xyz, acc, stream);
}

int drift_force_precision(const drift_potential *potential, int32_t precision, int64_t n,
                          const double *xyz, double *acc, void *stream)
{
    if (!potential || !xyz || !acc || n < 0)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_force: NULL pointer or negative n");
    if (precision != DRIFT_PRECISION_EXACT && precision != DRIFT_PRECISION_FMA)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown precision");
    const int k = potential->kind;
    if (k < DRIFT_POT_KEPLER || k > DRIFT_POT_KEPLER_CARTESIAN)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown potential kind");
    if (n == 0) return DRIFT_SUCCESS;
    DeviceContext *ctx = nullptr;
    int rc = current_context(&ctx);
    if (rc) return rc;
    int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sm_count * 8);
    drift::BulgeTable table;
    std::memset(&table, 0, sizeof(table));
    if (k == DRIFT_POT_BOVY) drift::fill_bulge_table(1.5 - 0.5 * potential->bulge_alpha, &table);
    DRIFT_CUDA_TRY(precision == DRIFT_PRECISION_FMA
                       ? drift::force_fma(*potential, n, xyz, acc, table, (int)blocks,
                                          static_cast<cudaStream_t>(stream))
                       : drift::force_exact(*potential, n, xyz, acc, table, (int)blocks,
                                            static_cast<cudaStream_t>(stream)),
                   "force kernel launch");
    return DRIFT_SUCCESS;
}

int drift_force_model_eval(const drift_force_model *model, int64_t n, double t, const double *xyz,
                           double *acc, void *stream)
{
    if (!xyz || !acc || n < 0)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_force_model_eval: NULL pointer or negative n");
    int rc = validate_model(model);
    if (rc) return rc;
    if (n == 0) return DRIFT_SUCCESS;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sm_count * 8);
    drift::BulgeTable table;
    std::memset(&table, 0, sizeof(table));
    fill_model_bulge(*model, &table);
    DRIFT_CUDA_TRY(drift::model_force_exact(*model, table, t, n, xyz, acc, (int)blocks,
                                            static_cast<cudaStream_t>(stream)),
                   "model force kernel launch");
    return DRIFT_SUCCESS;
}

int drift_origin_table(const drift_force_model *source_model, int64_t n_sources, int64_t nt, double t0,
                       double dt, const double *trajectory, double *origins, void *stream)
{
    if (!trajectory || !origins || n_sources < 1 || nt < 2)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "drift_origin_table: NULL pointer, n_sources < 1 or nt < 2");
    if (!is_finite_value(t0) || !is_finite_value(dt) || dt == 0.0)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_origin_table: t0 finite and dt nonzero required");
    int rc = validate_model(source_model);
    if (rc) return rc;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    drift::BulgeTable table;
    std::memset(&table, 0, sizeof(table));
    fill_model_bulge(*source_model, &table);
    DRIFT_CUDA_TRY(drift::origin_table_exact(*source_model, table, n_sources, nt, t0, dt, trajectory, origins,
                                             static_cast<cudaStream_t>(stream)),
                   "origin table kernel launch");
    return DRIFT_SUCCESS;
}

int drift_origin_table_host(const drift_force_model *source_model, int64_t n_sources, int64_t nt, double t0,
                            double dt, const double *trajectory, double *origins)
{
    if (!trajectory || !origins || n_sources < 1 || nt < 2)
        return fail(DRIFT_ERROR_INVALID_ARGUMENT,
                    "drift_origin_table_host: NULL pointer, n_sources < 1 or nt < 2");
    int rc = validate_model(source_model);
    if (rc) return rc;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaStream_t s = ctx->streams[0];
    drift_force_model m = *source_model;
    if (m.n_groups > 0) {
        const size_t b = (size_t)m.n_segments * m.n_sources * 18 * sizeof(double);
        DRIFT_CUDA_TRY(ctx->src_origins.ensure(b), "cudaMalloc(source origins)");
        DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->src_origins.ptr, m.origins, b, cudaMemcpyHostToDevice, s),
                       "H2D source origins");
        m.origins = ctx->src_origins.as<double>();
    }
    const size_t tb = (size_t)nt * n_sources * 6 * sizeof(double);
    const size_t ob = (size_t)(nt - 1) * n_sources * 18 * sizeof(double);
    DRIFT_CUDA_TRY(ctx->src_traj.ensure(tb), "cudaMalloc(source trajectory)");
    DRIFT_CUDA_TRY(ctx->src_table.ensure(ob), "cudaMalloc(origin table)");
    DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->src_traj.ptr, trajectory, tb, cudaMemcpyHostToDevice, s),
                   "H2D source trajectory");
    rc = drift_origin_table(&m, n_sources, nt, t0, dt, ctx->src_traj.as<double>(), ctx->src_table.as<double>(),
                            s);
    if (rc) return rc;
    DRIFT_CUDA_TRY(cudaMemcpyAsync(origins, ctx->src_table.ptr, ob, cudaMemcpyDeviceToHost, s), "D2H origin table");
    DRIFT_CUDA_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return DRIFT_SUCCESS;
}

int drift_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "ptr is NULL");
    cudaError_t e = cudaMallocHost(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    return DRIFT_SUCCESS;
}

int drift_host_free(void *ptr)
{
    cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFreeHost");
    return DRIFT_SUCCESS;
}

}  // extern "C"

static int host_integrate(DeviceContext *ctx, const drift_launch *L);

// Requests above this many particles may take the streamed copy-out.
#ifndef DRIFT_STREAMED_MIN_PARTICLES
#define DRIFT_STREAMED_MIN_PARTICLES 65536
#endif
constexpr int64_t STREAMED_MIN_PARTICLES = DRIFT_STREAMED_MIN_PARTICLES;
// Particle chunks of a streamed copy-out: between STREAMED_MIN_CHUNKS and
// STREAMED_CHUNKS, each holding about STREAMED_PER_LANE particles per
// resident thread, so that a chunk lasts many particle lifetimes and the
// particles that must go first (those that outlast a chunk's share of the
// launch) stay few.  Measured end to end with page-locked buffers: the
// uneven Bovy workload (2^22 particles, compute-bound) 13.04 s per pass at
// 4 particles per thread per chunk (18 chunks), 12.54 s at 16 (4 chunks),
// against 12.29 s for the device pass alone; the Plummer workload (2^20
// particles, bound by the 10 GB device-to-host copy) 217 ms at 6 chunks and
// 275 ms at 1 chunk, whose copy then waits for the whole launch.
constexpr int STREAMED_CHUNKS = 32;
constexpr int STREAMED_MIN_CHUNKS = 4;
#ifndef DRIFT_STREAMED_PER_LANE
#define DRIFT_STREAMED_PER_LANE 16
#endif
constexpr int64_t STREAMED_PER_LANE = DRIFT_STREAMED_PER_LANE;

static size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// The streamed copy-out of drift_integrate_host (the request's trajectory
// destination is page-locked and fits the device whole).  One launch
// integrates every particle into a full (nt, n, 6) device array; its queue
// (drift::build_order_chunked) runs the particles that outlast a chunk's
// share of the launch first, then chunk 0's particles longest first, then
// chunk 1's, and so on, and every particle counts itself done in its chunk's
// counter (4 to 32 chunks, see STREAMED_PER_LANE).  This thread reads the
// counters back every 200 microseconds (a small copy on a stream of its own,
// so that reading never waits behind a chunk's copy) and queues each
// finished chunk's trajectory copy on the second stream as soon as its
// counter is full, so the copy-out overlaps the rest of the launch and only
// the last chunks' copies remain after it.  The loop ends when every chunk
// is copied; once the launch's completion event fires, whatever is left is
// copied at once, so a launch that ends early (an error, a timeout) never
// leaves the loop waiting.
static int stream_copy_out(DeviceContext *ctx, const drift_launch *L)
{
    drift::TraceRange trace("drift host streamed copy-out");
    const int64_t n = L->n;
    const int64_t nt = L->nt;
    const size_t row = 6 * sizeof(double);
    cudaStream_t s0 = ctx->streams[0], s1 = ctx->streams[1];

    drift_launch shape = *L;
    shape.schedule = DRIFT_SCHEDULE_ORDERED;
    const int block = block_of(&shape);
    int grid = 0;
    int rc = grid_for(ctx->sm_count, &shape, n, block, &grid);
    if (rc) return rc;
    const int64_t lanes = (int64_t)grid * block;
    const int64_t want = std::max<int64_t>(STREAMED_MIN_CHUNKS,
                                           std::min<int64_t>(STREAMED_CHUNKS, n / (lanes * STREAMED_PER_LANE)));
    const int64_t chunk_len = ((n + want - 1) / want + 127) / 128 * 128;
    const int nchunks = (int)((n + chunk_len - 1) / chunk_len);
    const size_t scratch = drift::chunked_order_scratch(nchunks);
    const size_t ws = CURSOR_BYTES + scratch + align256(nchunks * sizeof(unsigned)) + align256(4 * (size_t)n) +
                      align256((size_t)n);
    DRIFT_CUDA_TRY(ctx->out[0].ensure((size_t)nt * n * row), "cudaMalloc(trajectory)");
    DRIFT_CUDA_TRY(ctx->cursor.ensure(ws), "cudaMalloc(workspace)");
    DRIFT_CUDA_TRY(ctx->poll.ensure(nchunks * sizeof(unsigned)), "cudaMallocHost(chunk counters)");

    // inputs
    drift_force_model model_dev{};
    drift_launch sub = *L;
    if (L->potential.kind == DRIFT_POT_MODEL) {
        model_dev = *L->force_model;
        if (model_dev.n_groups > 0) {
            const size_t bytes = (size_t)model_dev.n_segments * model_dev.n_sources * 18 * sizeof(double);
            DRIFT_CUDA_TRY(ctx->origins.ensure(bytes), "cudaMalloc(origins)");
            DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->origins.ptr, model_dev.origins, bytes, cudaMemcpyHostToDevice, s0),
                           "H2D origins");
            model_dev.origins = ctx->origins.as<double>();
        }
        sub.force_model = &model_dev;
    }
    const bool columns = L->y0_layout == DRIFT_Y0_COLUMNS;
    if (columns) {
        const size_t spitch = (size_t)(L->y0_stride ? L->y0_stride : n) * sizeof(double);
        DRIFT_CUDA_TRY(cudaMemcpy2DAsync(ctx->y0.ptr, n * sizeof(double), L->y0, spitch, n * sizeof(double), 6,
                                         cudaMemcpyHostToDevice, s0),
                       "H2D y0 columns");
    } else {
        DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->y0.ptr, L->y0, n * row, cudaMemcpyHostToDevice, s0), "H2D y0");
    }
    const size_t grid_bytes = L->ts ? nt * sizeof(double) : n * sizeof(double);
    DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->grid.ptr, L->ts ? (const void *)L->ts : (const void *)L->t_end,
                                   grid_bytes, cudaMemcpyHostToDevice, s0),
                   "H2D grid");
    sub.y0 = ctx->y0.as<double>();
    sub.y0_stride = columns ? n : 0;
    sub.ts = L->ts ? ctx->grid.as<double>() : nullptr;
    sub.t_end = L->ts ? nullptr : ctx->grid.as<double>();
    sub.out = ctx->out[0].as<double>();
    sub.y_final = L->y_final ? ctx->yfin.as<double>() : nullptr;
    sub.status = L->status ? ctx->status.as<uint8_t>() : nullptr;
    sub.err_code = L->err_code ? ctx->err.as<int32_t>() : nullptr;
    sub.n_accepted = L->n_accepted ? ctx->acc.as<uint32_t>() : nullptr;
    sub.n_rejected = L->n_rejected ? ctx->rej.as<uint32_t>() : nullptr;
    sub.schedule = DRIFT_SCHEDULE_ORDERED;

    // the chunk-ordered queue and the launch, on stream 0
    char *base = static_cast<char *>(ctx->cursor.ptr);
    unsigned *counts = reinterpret_cast<unsigned *>(base + CURSOR_BYTES);
    unsigned *split = counts + 256;
    unsigned *chunk_counts = split + 1;
    unsigned *done = reinterpret_cast<unsigned *>(base + CURSOR_BYTES + scratch);
    uint32_t *order = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(done) + align256(nchunks * sizeof(unsigned)));
    uint8_t *keys = reinterpret_cast<uint8_t *>(order) + align256(4 * (size_t)n);
    drift::KernelArgs a = make_args(&sub);
    a.persistent = 1;
    a.cursor = reinterpret_cast<unsigned long long *>(base);
    a.chunk_done = done;
    a.chunk_len = chunk_len;
    DRIFT_CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(unsigned long long), s0), "cudaMemsetAsync");
    DRIFT_CUDA_TRY(cudaMemsetAsync(done, 0, nchunks * sizeof(unsigned), s0), "cudaMemsetAsync");
    // the counters are read (poll stream) only after they are cleared
    DRIFT_CUDA_TRY(cudaEventRecord(ctx->done[1], s0), "cudaEventRecord");
    DRIFT_CUDA_TRY(cudaStreamWaitEvent(ctx->poll_stream, ctx->done[1], 0), "cudaStreamWaitEvent");
    DRIFT_CUDA_TRY(drift::build_order_chunked(a, sub.method, keys, counts, split, chunk_counts, order, chunk_len,
                                              nchunks, lanes, ctx->sm_count, s0),
                   "ordering kernels");
    a.order = order;
    DRIFT_CUDA_TRY(launch_args(a, sub.method, sub.precision, grid, block, s0), "kernel launch");
    DRIFT_CUDA_TRY(cudaEventRecord(ctx->done[0], s0), "cudaEventRecord");

    // copy-out as chunks complete, on stream 1
    const unsigned *seen = static_cast<const unsigned *>(ctx->poll.ptr);
    std::vector<char> copied(nchunks, 0);
    int remaining = nchunks;
    while (remaining > 0) {
        const cudaError_t q = cudaEventQuery(ctx->done[0]);
        if (q != cudaSuccess && q != cudaErrorNotReady) return cuda_fail(q, "integration launch");
        const bool launch_done = q == cudaSuccess;
        if (launch_done) {
            DRIFT_CUDA_TRY(cudaStreamWaitEvent(s1, ctx->done[0], 0), "cudaStreamWaitEvent");
        } else {
            cudaGetLastError();  // clears the not-ready status
            DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->poll.ptr, done, nchunks * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                           ctx->poll_stream),
                           "D2H chunk counters");
            DRIFT_CUDA_TRY(cudaStreamSynchronize(ctx->poll_stream), "cudaStreamSynchronize");
        }
        for (int c = 0; c < nchunks; c++) {
            if (copied[c]) continue;
            const int64_t c0 = (int64_t)c * chunk_len;
            const int64_t cn = std::min(chunk_len, n - c0);
            if (!launch_done && (int64_t)seen[c] < cn) continue;
            DRIFT_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<char *>(L->out) + c0 * row, n * row,
                                             sub.out + c0 * 6, n * row, cn * row, nt, cudaMemcpyDeviceToHost, s1),
                           "D2H trajectory chunk");
            copied[c] = 1;
            remaining--;
        }
        if (remaining > 0) std::this_thread::sleep_for(std::chrono::microseconds(200));
    }

    // per-particle outputs once the launch is done
    if (L->y_final)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->y_final, ctx->yfin.ptr, n * row, cudaMemcpyDeviceToHost, s0), "D2H y_final");
    if (L->status)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->status, ctx->status.ptr, n, cudaMemcpyDeviceToHost, s0), "D2H status");
    if (L->err_code)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->err_code, ctx->err.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s0),
                       "D2H err");
    if (L->n_accepted)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->n_accepted, ctx->acc.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s0),
                       "D2H accepted");
    if (L->n_rejected)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->n_rejected, ctx->rej.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s0),
                       "D2H rejected");
    DRIFT_CUDA_TRY(cudaStreamSynchronize(s0), "cudaStreamSynchronize");
    DRIFT_CUDA_TRY(cudaStreamSynchronize(s1), "cudaStreamSynchronize");
    return DRIFT_SUCCESS;
}

extern "C" {

int drift_integrate_host(const drift_launch *L)
{
    int rc = validate(L, false);
    if (rc) return rc;
    DeviceContext *ctx = nullptr;
    rc = current_context(&ctx);
    if (rc) return rc;
    return host_integrate(ctx, L);
}

}  // extern "C"

// The host path on a given context (its device current, the launch valid).
static int host_integrate_locked(DeviceContext *ctx, const drift_launch *L);

static int host_integrate(DeviceContext *ctx, const drift_launch *L)
{
    std::lock_guard<std::mutex> lock(ctx->mu);
    const int rc = host_integrate_locked(ctx, L);
    if (rc != DRIFT_SUCCESS) {
        // An error can leave the launch and copies into the caller's buffers
        // in flight: they end before the caller sees the error (and may free
        // those buffers).  A device fault makes these waits return at once.
        for (cudaStream_t st : {ctx->streams[0], ctx->streams[1], ctx->poll_stream})
            if (st) cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    return rc;
}

static int host_integrate_locked(DeviceContext *ctx, const drift_launch *L)
{
    int rc = DRIFT_SUCCESS;
    drift::TraceRange trace("drift host integrate");

    const int64_t n = L->n;
    const int64_t nt = L->nt;
    const size_t row = 6 * sizeof(double);

    // Whole-request buffers: initial states, grid, per-particle outputs.
    DRIFT_CUDA_TRY(ctx->y0.ensure(n * row), "cudaMalloc(y0)");
    const size_t grid_bytes = L->ts ? nt * sizeof(double) : n * sizeof(double);
    DRIFT_CUDA_TRY(ctx->grid.ensure(grid_bytes), "cudaMalloc(grid)");
    if (L->y_final) DRIFT_CUDA_TRY(ctx->yfin.ensure(n * row), "cudaMalloc(y_final)");
    if (L->status) DRIFT_CUDA_TRY(ctx->status.ensure(n), "cudaMalloc(status)");
    if (L->err_code) DRIFT_CUDA_TRY(ctx->err.ensure(n * sizeof(int32_t)), "cudaMalloc(err)");
    if (L->n_accepted) DRIFT_CUDA_TRY(ctx->acc.ensure(n * sizeof(uint32_t)), "cudaMalloc(acc)");
    if (L->n_rejected) DRIFT_CUDA_TRY(ctx->rej.ensure(n * sizeof(uint32_t)), "cudaMalloc(rej)");
    // (the per-slot workspace is sized once the chunk length is known)

    // Streamed copy-out (large persistent or ordered requests into page-locked
    // memory whose whole trajectory fits the device): one launch over every
    // particle with a queue that completes particle chunks in order, each
    // chunk copied out as soon as it is done (stream_copy_out below).
    // Otherwise, trajectory chunks: particles [c0, c0 + cn) write a
    // (nt, cn, 6) device block that is copied out row by row into the
    // caller's (nt, n, 6) array while the next chunk integrates.
    const bool out_pinned = L->out && is_pinned(L->out);
    size_t free_b = 0, total_b = 0;
    if (L->out) DRIFT_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t out_bytes = L->out ? (size_t)nt * n * row : 0;
    const bool streamed = out_pinned && L->schedule != DRIFT_SCHEDULE_PLAIN && n > STREAMED_MIN_PARTICLES &&
                          out_bytes <= (free_b + ctx->out[0].bytes) / 10 * 6;
    if (streamed) return stream_copy_out(ctx, L);
    int64_t chunk = n;
    if (L->out) {
        const size_t budget = std::min<size_t>(free_b / 4, size_t(8) << 30);
        int64_t by_mem = (int64_t)(budget / (nt * row));
        // Several chunks when the output is large, so the device->host copy
        // of one chunk overlaps the integration of the next; the copy of the
        // whole output usually takes longer than its integration, and only
        // the first chunk's integration is not hidden behind a copy.
        const int64_t parts = n > 524288 ? 16 : (n > 65536 ? 4 : 1);
        int64_t target = (n + parts - 1) / parts;
        chunk = std::max<int64_t>(1, std::min(target, by_mem));
        if (chunk < n) chunk = std::max<int64_t>(128, chunk / 128 * 128);
        chunk = std::min(chunk, n);
        for (int i = 0; i < 2; i++)
            DRIFT_CUDA_TRY(ctx->out[i].ensure(chunk * nt * row), "cudaMalloc(out chunk)");
    }
    drift_launch chunk_req = *L;
    chunk_req.n = chunk;
    const size_t ws_slot = std::max<size_t>(workspace_bytes(&chunk_req), CURSOR_BYTES);
    DRIFT_CUDA_TRY(ctx->cursor.ensure(2 * ws_slot), "cudaMalloc(workspace)");
    if (L->out && !out_pinned)
        for (int i = 0; i < 2; i++)
            DRIFT_CUDA_TRY(ctx->stage[i].ensure(chunk * nt * row), "cudaMallocHost(stage)");

    cudaStream_t s0 = ctx->streams[0];
    // A force model's origin table is a host array here: its device copy
    // lives in the context.
    drift_force_model model_dev{};
    if (L->potential.kind == DRIFT_POT_MODEL) {
        model_dev = *L->force_model;
        if (model_dev.n_groups > 0) {
            const size_t bytes = (size_t)model_dev.n_segments * model_dev.n_sources * 18 * sizeof(double);
            DRIFT_CUDA_TRY(ctx->origins.ensure(bytes), "cudaMalloc(origins)");
            DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->origins.ptr, model_dev.origins, bytes, cudaMemcpyHostToDevice, s0),
                           "H2D origins");
            model_dev.origins = ctx->origins.as<double>();
        }
    }
    const bool columns = L->y0_layout == DRIFT_Y0_COLUMNS;
    if (columns) {
        // six columns, packed to a stride of n on the device
        const size_t spitch = (size_t)(L->y0_stride ? L->y0_stride : n) * sizeof(double);
        DRIFT_CUDA_TRY(cudaMemcpy2DAsync(ctx->y0.ptr, n * sizeof(double), L->y0, spitch, n * sizeof(double), 6,
                                         cudaMemcpyHostToDevice, s0),
                       "H2D y0 columns");
    } else {
        DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->y0.ptr, L->y0, n * row, cudaMemcpyHostToDevice, s0), "H2D y0");
    }
    DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->grid.ptr, L->ts ? (const void *)L->ts : (const void *)L->t_end,
                                   grid_bytes, cudaMemcpyHostToDevice, s0),
                   "H2D grid");
    DRIFT_CUDA_TRY(cudaEventRecord(ctx->done[0], s0), "cudaEventRecord");
    DRIFT_CUDA_TRY(cudaStreamWaitEvent(ctx->streams[1], ctx->done[0], 0), "cudaStreamWaitEvent");

    int64_t chunk_index = 0;
    int64_t pending_c0[2] = {-1, -1}, pending_cn[2] = {0, 0};
    auto drain_stage = [&](int slot) -> int {
        // Move a finished pageable-destination chunk from pinned staging.
        if (pending_c0[slot] < 0) return DRIFT_SUCCESS;
        DRIFT_CUDA_TRY(cudaEventSynchronize(ctx->done[slot]), "cudaEventSynchronize");
        const int64_t c0 = pending_c0[slot], cn = pending_cn[slot];
        const char *src = static_cast<const char *>(ctx->stage[slot].ptr);
        char *dst = reinterpret_cast<char *>(L->out);
        for (int64_t k = 0; k < nt; k++)
            std::memcpy(dst + (k * n + c0) * row, src + k * cn * row, cn * row);
        pending_c0[slot] = -1;
        return DRIFT_SUCCESS;
    };

    for (int64_t c0 = 0; c0 < n; c0 += chunk, chunk_index++) {
        drift::TraceRange chunk_trace("drift host chunk");
        const int slot = (int)(chunk_index & 1);
        cudaStream_t s = ctx->streams[slot];
        const int64_t cn = std::min(chunk, n - c0);
        if (L->out && !out_pinned) {
            rc = drain_stage(slot);
            if (rc) return rc;
        }
        drift_launch sub = *L;
        sub.n = cn;
        if (L->potential.kind == DRIFT_POT_MODEL) sub.force_model = &model_dev;
        sub.y0 = columns ? ctx->y0.as<double>() + c0 : ctx->y0.as<double>() + c0 * 6;
        sub.y0_stride = columns ? n : 0;
        sub.ts = L->ts ? ctx->grid.as<double>() : nullptr;
        sub.t_end = L->ts ? nullptr : ctx->grid.as<double>() + c0;
        sub.out = L->out ? ctx->out[slot].as<double>() : nullptr;
        sub.y_final = L->y_final ? ctx->yfin.as<double>() + c0 * 6 : nullptr;
        sub.status = L->status ? ctx->status.as<uint8_t>() + c0 : nullptr;
        sub.err_code = L->err_code ? ctx->err.as<int32_t>() + c0 : nullptr;
        sub.n_accepted = L->n_accepted ? ctx->acc.as<uint32_t>() + c0 : nullptr;
        sub.n_rejected = L->n_rejected ? ctx->rej.as<uint32_t>() + c0 : nullptr;
        rc = launch_device(ctx, &sub, static_cast<char *>(ctx->cursor.ptr) + slot * ws_slot, s);
        if (rc) return rc;
        if (L->out) {
            if (out_pinned) {
                DRIFT_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<char *>(L->out) + c0 * row, n * row,
                                                 sub.out, cn * row, cn * row, nt,
                                                 cudaMemcpyDeviceToHost, s),
                               "D2H trajectories");
            } else {
                DRIFT_CUDA_TRY(cudaMemcpyAsync(ctx->stage[slot].ptr, sub.out, cn * nt * row,
                                               cudaMemcpyDeviceToHost, s),
                               "D2H trajectories");
                DRIFT_CUDA_TRY(cudaEventRecord(ctx->done[slot], s), "cudaEventRecord");
                pending_c0[slot] = c0;
                pending_cn[slot] = cn;
            }
        }
    }
    for (int slot = 0; slot < 2; slot++) {
        if (L->out && !out_pinned) {
            rc = drain_stage(slot);
            if (rc) return rc;
        }
    }
    // Per-particle outputs once every chunk is done.
    drift::TraceRange tail_trace("drift host copy-out and wait");
    DRIFT_CUDA_TRY(cudaEventRecord(ctx->done[1], ctx->streams[1]), "cudaEventRecord");
    DRIFT_CUDA_TRY(cudaStreamWaitEvent(s0, ctx->done[1], 0), "cudaStreamWaitEvent");
    if (L->y_final)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->y_final, ctx->yfin.ptr, n * row, cudaMemcpyDeviceToHost, s0), "D2H y_final");
    if (L->status)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->status, ctx->status.ptr, n, cudaMemcpyDeviceToHost, s0), "D2H status");
    if (L->err_code)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->err_code, ctx->err.ptr, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s0), "D2H err");
    if (L->n_accepted)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->n_accepted, ctx->acc.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s0), "D2H accepted");
    if (L->n_rejected)
        DRIFT_CUDA_TRY(cudaMemcpyAsync(L->n_rejected, ctx->rej.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s0), "D2H rejected");
    DRIFT_CUDA_TRY(cudaStreamSynchronize(s0), "cudaStreamSynchronize");
    DRIFT_CUDA_TRY(cudaStreamSynchronize(ctx->streams[1]), "cudaStreamSynchronize");
    return DRIFT_SUCCESS;
}

struct drift_context {
    DeviceContext c;
};

extern "C" {

int drift_context_create(int32_t device, drift_context **out)
{
    if (!out) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_context_create: out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
        cudaGetLastError();
        return fail(DRIFT_ERROR_NO_DEVICE, "no CUDA device");
    }
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(DRIFT_ERROR_NO_DEVICE, "no current CUDA device");
    }
    if (dev >= count) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "no such CUDA device");
    ScopedDevice on(dev);
    auto *ctx = new drift_context();
    int rc = ctx->c.init(dev);
    if (rc) {
        ctx->c.release();
        delete ctx;
        return rc;
    }
    *out = ctx;
    return DRIFT_SUCCESS;
}

int drift_context_integrate_host(drift_context *ctx, const drift_launch *L)
{
    if (!ctx) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_context_integrate_host: context is NULL");
    int rc = validate(L, false);
    if (rc) return rc;
    ScopedDevice on(ctx->c.device);
    return host_integrate(&ctx->c, L);
}

int drift_context_memory(drift_context *ctx, size_t *device_bytes, size_t *pinned_bytes)
{
    if (!ctx) return fail(DRIFT_ERROR_INVALID_ARGUMENT, "drift_context_memory: context is NULL");
    std::lock_guard<std::mutex> lock(ctx->c.mu);
    if (device_bytes) *device_bytes = ctx->c.device_bytes();
    if (pinned_bytes) *pinned_bytes = ctx->c.pinned_bytes();
    return DRIFT_SUCCESS;
}

int drift_context_destroy(drift_context *ctx)
{
    if (!ctx) return DRIFT_SUCCESS;
    {
        std::lock_guard<std::mutex> lock(ctx->c.mu);
        ScopedDevice on(ctx->c.device);
        ctx->c.release();
    }
    delete ctx;
    return DRIFT_SUCCESS;
}

int drift_galpy_dopr54(const double *state0, const double *times, double *state_out, int64_t n,
                       int64_t nt, double rtol, double atol, double dt_one_init, void *stream)
{
    drift_launch L;
    std::memset(&L, 0, sizeof(L));
    L.method = DRIFT_DOPR54;
    L.precision = DRIFT_PRECISION_EXACT;
    L.schedule = DRIFT_SCHEDULE_PLAIN;
    L.potential.kind = DRIFT_POT_KEPLER;
    L.potential.amp = 1.0;
    L.n = n;
    L.y0 = state0;
    L.nt = nt;
    L.ts = times;
    L.out = state_out;
    L.rtol_ln = rtol;
    L.atol_ln = atol;
    L.dt_one = dt_one_init;
    return drift_integrate(&L, stream);
}

int drift_galpy_dop853(const double *state0, const double *times, double *state_out, int64_t n,
                       int64_t nt, double rtol, double atol, void *stream)
{
    drift_launch L;
    std::memset(&L, 0, sizeof(L));
    L.method = DRIFT_DOP853;
    L.precision = DRIFT_PRECISION_EXACT;
    L.schedule = DRIFT_SCHEDULE_PLAIN;
    L.potential.kind = DRIFT_POT_KEPLER;
    L.potential.amp = 1.0;
    L.n = n;
    L.y0 = state0;
    L.nt = nt;
    L.ts = times;
    L.out = state_out;
    L.rtol_ln = rtol;
    L.atol_ln = atol;
    L.dt_one = DRIFT_INITIAL_STEP_SENTINEL;
    return drift_integrate(&L, stream);
}

}  // extern "C"
