// drift_server.cu -- resident request server with continuous batching.
//
// A scheduler thread owns a device memory pool, a set of streams and the
// queue of submitted requests.  Whenever a stream is free it forms a batch:
// the oldest pending request plus every later pending request that can share
// its launch (same method, precision, schedule, potential, tolerances and
// limits), as long as the batch fits the device-memory budget.  A request larger than the
// remaining budget is admitted in particle chunks.  Each batch copies its
// inputs in, runs one batched integration launch (drift_integrate_batch's
// kernel path), copies trajectories and per-particle outputs back into the
// requests' host buffers and frees its memory, all ordered on its stream, so
// requests that arrive while others are on the GPU start as soon as a stream
// and memory free up and their kernels overlap the running ones.  Completion
// is signalled from the stream (cudaLaunchHostFunc) to the scheduler, which
// wakes waiters.  No counterpart exists in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "drift_b200.h"
#include "drift_trace.h"
#include "drift_launch_args.cuh"

// Internal launcher shared with drift_capi.cu.
int drift_internal_launch_batch(int sm_count, const drift_launch *R, int32_t count, void *ws,
                                cudaStream_t s);
int drift_internal_fail(int code, const char *msg);

namespace {

using Clock = std::chrono::steady_clock;
constexpr size_t ALIGN = 256;
constexpr size_t CURSOR = 256;

size_t align_up(size_t b) { return (b + ALIGN - 1) / ALIGN * ALIGN; }

struct Request {
    uint64_t ticket = 0;
    drift_launch L{};          // host pointers owned by the caller
    int64_t admitted = 0;      // particles [0, admitted) handed to batches
    int64_t finished = 0;      // particles whose batch completed
    int result = DRIFT_SUCCESS;
    bool done = false;
    Clock::time_point submitted, completed;
};

// One chunk of one request inside a batch.
struct Piece {
    Request *req;
    int64_t c0, cn;
    size_t off_y0, off_grid, off_out, off_fin, off_st, off_err, off_acc, off_rej;
};

struct Batch {
    int slot = -1;
    void *dmem = nullptr;
    size_t bytes = 0;
    std::vector<Piece> pieces;
    std::atomic<bool> complete{false};
};

// Bytes a chunk of cn particles of request L needs on the device.
size_t piece_bytes(const drift_launch &L, int64_t cn)
{
    size_t b = align_up(cn * 48);                                   // y0
    b += align_up(L.ts ? L.nt * sizeof(double) : cn * sizeof(double));  // grid
    if (L.out) b += align_up((size_t)L.nt * cn * 48);
    if (L.y_final) b += align_up(cn * 48);
    if (L.status) b += align_up(cn);
    if (L.err_code) b += align_up(cn * 4);
    if (L.n_accepted) b += align_up(cn * 4);
    if (L.n_rejected) b += align_up(cn * 4);
    return b;
}

// Schedule a request runs under inside a batch: ordered stays ordered, the
// rest share a persistent claim queue.
int batch_schedule(const drift_launch &L)
{
    return L.schedule == DRIFT_SCHEDULE_ORDERED ? DRIFT_SCHEDULE_ORDERED : DRIFT_SCHEDULE_PERSISTENT;
}

// Scratch at the front of a batch's allocation: the claim cursor, and for
// the ordered schedule the bucket counts and the queue and keys of all its
// particles (the layout drift_integrate_batch expects).
size_t scratch_bytes(int schedule, int64_t particles)
{
    if (schedule != DRIFT_SCHEDULE_ORDERED) return CURSOR;
    return align_up(CURSOR + 1024 + 5 * (size_t)particles);
}

bool compatible(const drift_launch &A, const drift_launch &B)
{
    return A.method == B.method && A.precision == B.precision && A.block_size == B.block_size &&
           batch_schedule(A) == batch_schedule(B) &&
           !std::memcmp(&A.potential, &B.potential, sizeof(A.potential)) && A.rtol_ln == B.rtol_ln &&
           A.atol_ln == B.atol_ln && A.dt_one == B.dt_one && A.max_steps == B.max_steps &&
           A.timeout_s == B.timeout_s && (A.arbitrary_times != 0) == (B.arbitrary_times != 0);
}

}  // namespace

struct drift_server {
    drift_server_options opts{};
    int device = -1;
    int sm_count = 0;
    int reserve_sms = 0;         // SMs large batches leave free
    int64_t small_particles = 0; // batches this small count as small
    size_t budget = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<bool> slot_busy;

    std::mutex mu;
    std::condition_variable cv_work;  // scheduler wake-up
    std::condition_variable cv_done;  // waiters
    std::deque<Request *> pending;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    std::vector<std::unique_ptr<Batch>> inflight;
    size_t bytes_inflight = 0;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    std::string last_error;

    drift_server_stats stats{};

    static void CUDART_CB on_batch_done(void *p)
    {
        auto *pair = static_cast<std::pair<drift_server *, Batch *> *>(p);
        drift_server *s = pair->first;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            pair->second->complete = true;
        }
        s->cv_work.notify_all();
        delete pair;
    }

    // Called with mu held: retire completed batches.
    void retire()
    {
        for (size_t i = 0; i < inflight.size();) {
            Batch *b = inflight[i].get();
            if (!b->complete) {
                i++;
                continue;
            }
            for (Piece &p : b->pieces) {
                p.req->finished += p.cn;
                if (p.req->finished == p.req->L.n && !p.req->done) {
                    p.req->done = true;
                    p.req->completed = Clock::now();
                    stats.requests_completed++;
                    stats.particles_completed += p.req->L.n;
                }
            }
            bytes_inflight -= b->bytes;
            slot_busy[b->slot] = false;
            inflight.erase(inflight.begin() + i);
            cv_done.notify_all();
        }
    }

    // Called with mu held: form and launch one batch on a free slot.
    // Returns false when nothing could be admitted.
    bool admit()
    {
        int slot = -1;
        for (int i = 0; i < (int)slot_busy.size(); i++)
            if (!slot_busy[i]) {
                slot = i;
                break;
            }
        if (slot < 0 || pending.empty()) return false;
        slot = -1;  // chosen once the batch's size is known
        Request *head = pending.front();
        auto batch = std::make_unique<Batch>();
        size_t room = budget > bytes_inflight ? budget - bytes_inflight : 0;
        const int schedule = batch_schedule(head->L);
        size_t used = 0;  // piece bytes; the scratch goes in front of them
        int64_t particles = 0;
        std::vector<Request *> taken;
        for (Request *r : pending) {
            if ((int)batch->pieces.size() >= drift::MAX_BATCH) break;
            if (particles >= opts.max_batch_particles) break;
            if (!compatible(head->L, r->L)) continue;
            int64_t remaining = r->L.n - r->admitted;
            int64_t cn = std::min<int64_t>(remaining, opts.max_batch_particles - particles);
            // shrink to the memory that is left
            while (cn > 0 && scratch_bytes(schedule, particles + cn) + used + piece_bytes(r->L, cn) > room)
                cn = cn > 256 ? cn / 2 : cn - 1;
            if (cn <= 0) {
                if (r == head) {
                    if (inflight.empty() && scratch_bytes(schedule, 1) + piece_bytes(r->L, 1) > budget) {
                        // Not even one particle fits the whole budget.
                        r->result = DRIFT_ERROR_OUT_OF_MEMORY;
                        r->done = true;
                        r->completed = Clock::now();
                        pending.pop_front();
                        cv_done.notify_all();
                        return !pending.empty();
                    }
                    break;  // keep FIFO order for the head: wait for memory
                }
                continue;
            }
            Piece p{};
            p.req = r;
            p.c0 = r->admitted;
            p.cn = cn;
            size_t off = used;
            p.off_y0 = off;
            off += align_up(cn * 48);
            p.off_grid = off;
            off += align_up(r->L.ts ? r->L.nt * sizeof(double) : cn * sizeof(double));
            p.off_out = off;
            if (r->L.out) off += align_up((size_t)r->L.nt * cn * 48);
            p.off_fin = off;
            if (r->L.y_final) off += align_up(cn * 48);
            p.off_st = off;
            if (r->L.status) off += align_up(cn);
            p.off_err = off;
            if (r->L.err_code) off += align_up(cn * 4);
            p.off_acc = off;
            if (r->L.n_accepted) off += align_up(cn * 4);
            p.off_rej = off;
            if (r->L.n_rejected) off += align_up(cn * 4);
            used = off;
            r->admitted += cn;
            particles += cn;
            batch->pieces.push_back(p);
            if (r->admitted == r->L.n) taken.push_back(r);
            if (r != head && cn < remaining) break;
        }
        if (batch->pieces.empty()) return false;
        for (Request *r : taken) pending.erase(std::find(pending.begin(), pending.end(), r));
        const size_t scratch = scratch_bytes(schedule, particles);
        for (Piece &p : batch->pieces)
            for (size_t *o : {&p.off_y0, &p.off_grid, &p.off_out, &p.off_fin, &p.off_st, &p.off_err,
                              &p.off_acc, &p.off_rej})
                *o += scratch;
        used += scratch;

        // Small batches run on the high-priority stream 0 and may use every
        // SM; large ones use the other streams and leave the reserve free.
        const bool small = particles <= small_particles;
        if (small && !slot_busy[0]) slot = 0;
        for (int i = 1; slot < 0 && i < (int)slot_busy.size(); i++)
            if (!slot_busy[i]) slot = i;
        if (slot < 0) slot = 0;  // only stream 0 is free
        const int launch_sms = small ? sm_count : std::max(1, sm_count - reserve_sms);

        cudaStream_t s = streams[slot];
        void *dmem = nullptr;
        if (cudaMallocFromPoolAsync(&dmem, used, pool, s) != cudaSuccess) {
            cudaGetLastError();
            // give the pieces back and wait for memory
            for (Piece &p : batch->pieces) p.req->admitted = p.c0;
            for (auto it = taken.rbegin(); it != taken.rend(); ++it) pending.push_front(*it);
            return false;
        }
        batch->slot = slot;
        batch->dmem = dmem;
        batch->bytes = used;
        char *base = static_cast<char *>(dmem);

        std::vector<drift_launch> sub(batch->pieces.size());
        for (size_t i = 0; i < batch->pieces.size(); i++) {
            Piece &p = batch->pieces[i];
            const drift_launch &L = p.req->L;
            drift_launch &D = sub[i];
            D = L;
            D.n = p.cn;
            D.y0 = reinterpret_cast<double *>(base + p.off_y0);
            cudaMemcpyAsync((void *)D.y0, L.y0 + p.c0 * 6, p.cn * 48, cudaMemcpyHostToDevice, s);
            if (L.ts) {
                D.ts = reinterpret_cast<double *>(base + p.off_grid);
                D.t_end = nullptr;
                cudaMemcpyAsync((void *)D.ts, L.ts, L.nt * sizeof(double), cudaMemcpyHostToDevice, s);
            } else {
                D.t_end = reinterpret_cast<double *>(base + p.off_grid);
                cudaMemcpyAsync((void *)D.t_end, L.t_end + p.c0, p.cn * sizeof(double),
                                cudaMemcpyHostToDevice, s);
            }
            D.out = L.out ? reinterpret_cast<double *>(base + p.off_out) : nullptr;
            D.y_final = L.y_final ? reinterpret_cast<double *>(base + p.off_fin) : nullptr;
            D.status = L.status ? reinterpret_cast<uint8_t *>(base + p.off_st) : nullptr;
            D.err_code = L.err_code ? reinterpret_cast<int32_t *>(base + p.off_err) : nullptr;
            D.n_accepted = L.n_accepted ? reinterpret_cast<uint32_t *>(base + p.off_acc) : nullptr;
            D.n_rejected = L.n_rejected ? reinterpret_cast<uint32_t *>(base + p.off_rej) : nullptr;
            D.schedule = schedule;
            D.workspace = base;
            D.workspace_bytes = scratch;
        }
        drift::TraceRange trace("drift server batch");
        int rc = drift_internal_launch_batch(launch_sms, sub.data(), (int32_t)sub.size(), base, s);
        for (size_t i = 0; i < batch->pieces.size(); i++) {
            Piece &p = batch->pieces[i];
            const drift_launch &L = p.req->L;
            const drift_launch &D = sub[i];
            if (rc != DRIFT_SUCCESS) p.req->result = rc;
            if (L.out)
                cudaMemcpy2DAsync(L.out + p.c0 * 6, L.n * 48, D.out, p.cn * 48, p.cn * 48, L.nt,
                                  cudaMemcpyDeviceToHost, s);
            if (L.y_final)
                cudaMemcpyAsync(L.y_final + p.c0 * 6, D.y_final, p.cn * 48, cudaMemcpyDeviceToHost, s);
            if (L.status) cudaMemcpyAsync(L.status + p.c0, D.status, p.cn, cudaMemcpyDeviceToHost, s);
            if (L.err_code)
                cudaMemcpyAsync(L.err_code + p.c0, D.err_code, p.cn * 4, cudaMemcpyDeviceToHost, s);
            if (L.n_accepted)
                cudaMemcpyAsync(L.n_accepted + p.c0, D.n_accepted, p.cn * 4, cudaMemcpyDeviceToHost, s);
            if (L.n_rejected)
                cudaMemcpyAsync(L.n_rejected + p.c0, D.n_rejected, p.cn * 4, cudaMemcpyDeviceToHost, s);
            stats.bytes_to_device += p.cn * 48;
            if (L.out) stats.bytes_to_host += (size_t)L.nt * p.cn * 48;
        }
        cudaFreeAsync(dmem, s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            for (Piece &p : batch->pieces) p.req->result = DRIFT_ERROR_CUDA;
        slot_busy[slot] = true;
        bytes_inflight += used;
        stats.batches_launched++;
        stats.pieces_launched += batch->pieces.size();
        stats.peak_bytes_in_flight = std::max<uint64_t>(stats.peak_bytes_in_flight, bytes_inflight);
        Batch *raw = batch.get();
        inflight.push_back(std::move(batch));
        auto *ctx = new std::pair<drift_server *, Batch *>(this, raw);
        if (cudaLaunchHostFunc(s, &drift_server::on_batch_done, ctx) != cudaSuccess) {
            cudaGetLastError();
            cudaStreamSynchronize(s);
            raw->complete = true;
            delete ctx;
        }
        return true;
    }

    void run()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(mu);
        while (true) {
            retire();
            if (stop && inflight.empty()) break;
            bool progressed = false;
            if (!stop)
                while (admit()) progressed = true;
            if (!progressed)
                cv_work.wait_for(lock, std::chrono::milliseconds(5));
        }
    }
};

extern "C" {

int drift_server_create(const drift_server_options *options, drift_server **out)
{
    if (!out) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "out is NULL");
    auto s = std::make_unique<drift_server>();
    drift_server_options o{};
    o.memory_fraction = 0.5;
    o.streams = 4;
    o.max_batch_particles = int64_t(1) << 20;
    o.sm_reserve_percent = 0;
    if (options) {
        o.sm_reserve_percent = std::min(std::max(options->sm_reserve_percent, 0), 50);
        if (options->memory_fraction > 0) o.memory_fraction = std::min(options->memory_fraction, 0.95);
        if (options->streams > 0) o.streams = std::min(options->streams, 32);
        if (options->max_batch_particles > 0) o.max_batch_particles = options->max_batch_particles;
        o.memory_bytes = options->memory_bytes;
    }
    s->opts = o;
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        cudaGetLastError();
        return drift_internal_fail(DRIFT_ERROR_NO_DEVICE, "no CUDA device");
    }
    if (options && options->select_device) {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || options->device < 0 || options->device >= count) {
            cudaGetLastError();
            return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "no such CUDA device");
        }
        s->device = options->device;
    }
    // every call below, and the scheduler thread, work on the server's device
    int caller_device = -1;
    cudaGetDevice(&caller_device);
    cudaSetDevice(s->device);
    struct RestoreDevice {
        int d;
        ~RestoreDevice()
        {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{caller_device};
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
    s->reserve_sms = s->sm_count * o.sm_reserve_percent / 100;
    // a small batch fits the reserve at 256 particles per SM
    s->small_particles = std::max<int64_t>(int64_t(s->reserve_sms) * 256, 1);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return drift_internal_fail(DRIFT_ERROR_CUDA, "cudaMemGetInfo failed");
    }
    s->budget = o.memory_bytes > 0 ? std::min<size_t>(o.memory_bytes, free_b)
                                   : (size_t)(o.memory_fraction * (double)free_b);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return drift_internal_fail(DRIFT_ERROR_CUDA, "cudaMemPoolCreate failed");
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    s->streams.resize(o.streams);
    s->slot_busy.assign(o.streams, false);
    int lowest = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&lowest, &greatest);
    for (size_t i = 0; i < s->streams.size(); i++)
        if (cudaStreamCreateWithPriority(&s->streams[i], cudaStreamNonBlocking, i == 0 ? greatest : lowest) !=
            cudaSuccess) {
            cudaGetLastError();
            return drift_internal_fail(DRIFT_ERROR_CUDA, "cudaStreamCreate failed");
        }
    s->stats.memory_budget = s->budget;
    drift_server *raw = s.release();
    raw->worker = std::thread([raw] { raw->run(); });
    *out = raw;
    return DRIFT_SUCCESS;
}

int drift_server_submit(drift_server *s, const drift_launch *request, uint64_t *ticket)
{
    if (!s || !request || !ticket)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    const drift_launch &L = *request;
    if (L.n < 1 || L.nt < 2 || !L.y0 || (!L.ts && !L.t_end) || L.schedule < DRIFT_SCHEDULE_PLAIN ||
        L.schedule > DRIFT_SCHEDULE_ORDERED || L.tape ||
        L.method < DRIFT_DOPR54 || L.method > DRIFT_DOP853 || L.precision < 0 || L.precision > 1 ||
        L.potential.kind < DRIFT_POT_KEPLER || L.potential.kind > DRIFT_POT_KEPLER_CARTESIAN)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "invalid request");
    if (L.y0_layout != DRIFT_Y0_ROWS)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "the server takes y0 as (n, 6) rows");
    auto r = std::make_unique<Request>();
    r->L = L;
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->pending.push_back(r.get());
    s->requests[r->ticket] = std::move(r);
    s->stats.requests_submitted++;
    s->cv_work.notify_all();
    return DRIFT_SUCCESS;
}

int drift_server_wait(drift_server *s, uint64_t ticket, double timeout_s, int *request_result,
                      double *latency_s)
{
    if (!s) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "server is NULL");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end())
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown ticket");
    Request *r = it->second.get();
    auto pred = [r] { return r->done; };
    if (timeout_s > 0) {
        if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), pred))
            return drift_internal_fail(DRIFT_ERROR_TIMEOUT, "request still running");
    } else {
        s->cv_done.wait(lock, pred);
    }
    if (request_result) *request_result = r->result;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->completed - r->submitted).count();
    s->requests.erase(it);
    return DRIFT_SUCCESS;
}

int drift_server_stats_get(drift_server *s, drift_server_stats *out)
{
    if (!s || !out) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->requests_pending = s->pending.size();
    out->batches_in_flight = s->inflight.size();
    out->bytes_in_flight = s->bytes_inflight;
    out->bytes_pending = 0;
    for (const Request *r : s->pending) out->bytes_pending += piece_bytes(r->L, r->L.n - r->admitted);
    out->device = s->device;
    out->reserved = 0;
    return DRIFT_SUCCESS;
}

int drift_server_destroy(drift_server *s)
{
    if (!s) return DRIFT_SUCCESS;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        for (Request *r : s->pending) {
            if (r->admitted == 0) {
                r->result = DRIFT_ERROR_CANCELLED;
                r->done = true;
                r->completed = Clock::now();
            }
        }
        s->pending.clear();
        s->cv_done.notify_all();
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return DRIFT_SUCCESS;
}

}  // extern "C"
