// drift_server.cu -- resident request server with continuous batching.
//
// A scheduler thread owns the queue of submitted requests and a device
// memory pool; one worker thread per stream runs the batches.  Whenever a
// stream is free the scheduler forms a batch: the oldest pending request plus
// every later pending request that can share its launch (same method,
// precision, schedule, potential, tolerances and limits), as long as the
// batch fits the device-memory budget.  A request larger than the remaining
// budget is admitted in particle chunks.  The stream's worker then copies
// the batch's inputs in, runs one batched integration launch
// (drift_integrate_batch's kernel path), copies trajectories and
// per-particle outputs back into the requests' host buffers, frees its
// memory and waits for its stream, so requests that arrive while others are
// on the GPU start as soon as a stream and memory free up and their kernels
// overlap the running ones.
//
// Locking: the mutex guards the queue, the requests' bookkeeping and the
// statistics, and no thread holds it across a CUDA call.  A worker blocked
// in a copy into pageable host memory (which returns only when its kernel
// has finished) or in its stream wait holds up nobody but its own stream:
// the scheduler keeps admitting batches on the other streams, and submit,
// wait, cancel and stats calls proceed.  No counterpart exists in the
// reference.
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
    bool cancelled = false;    // no further particles are admitted
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
    size_t bytes = 0;           // device bytes (scratch + pieces)
    size_t scratch = 0;         // scratch bytes at the front of dmem
    int schedule = DRIFT_SCHEDULE_PERSISTENT;
    int launch_sms = 0;
    std::vector<Piece> pieces;
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

    // One worker per stream; `job` is handed over under mu.
    struct Worker {
        std::thread thread;
        std::condition_variable cv;
        std::unique_ptr<Batch> job;
        bool busy = false;       // a batch is planned for or running on this stream
    };
    std::vector<std::unique_ptr<Worker>> workers;

    std::mutex mu;
    std::condition_variable cv_work;  // scheduler wake-up
    std::condition_variable cv_done;  // waiters
    std::condition_variable cv_idle;  // destroy: the last waiter has left
    int waiters = 0;                  // threads inside drift_server_wait(_any)
    std::deque<Request *> pending;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    size_t bytes_inflight = 0;
    int batches_inflight = 0;
    uint64_t next_ticket = 1;
    bool stop = false;          // no further admissions (destroy)
    bool quit = false;          // workers exit once idle
    std::thread scheduler;

    drift_server_stats stats{};

    // With mu held: a request ends once every particle it will run has
    // finished (all of them, or the admitted ones after a cancellation).
    void maybe_complete(Request *r)
    {
        if (r->done) return;
        const int64_t target = r->cancelled ? r->admitted : r->L.n;
        if (r->finished < target) return;
        if (r->cancelled) r->result = DRIFT_ERROR_CANCELLED;
        r->done = true;
        r->completed = Clock::now();
        stats.requests_completed++;
        stats.particles_completed += r->finished;
        cv_done.notify_all();
    }

    // With mu held: the pieces of a batch that never ran go back to their
    // requests (the scheduler plans one batch at a time, so they are the
    // last particles admitted of each request).
    void give_back(Batch &b)
    {
        for (auto it = b.pieces.rbegin(); it != b.pieces.rend(); ++it) {
            Request *r = it->req;
            r->admitted = it->c0;
            if (!r->cancelled && std::find(pending.begin(), pending.end(), r) == pending.end())
                pending.push_front(r);
            maybe_complete(r);
        }
    }

    // With mu held: form one batch for a free stream.  Its pieces are taken
    // from the queue and its bytes reserved; returns nullptr when nothing can
    // be admitted now.
    std::unique_ptr<Batch> plan()
    {
        int free_slot = -1;
        for (int i = 0; i < (int)workers.size(); i++)
            if (!workers[i]->busy) {
                free_slot = i;
                break;
            }
        while (!pending.empty() && pending.front()->cancelled) pending.pop_front();
        if (free_slot < 0 || pending.empty()) return nullptr;
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
            if (r->cancelled || !compatible(head->L, r->L)) continue;
            int64_t remaining = r->L.n - r->admitted;
            int64_t cn = std::min<int64_t>(remaining, opts.max_batch_particles - particles);
            // shrink to the memory that is left
            while (cn > 0 && scratch_bytes(schedule, particles + cn) + used + piece_bytes(r->L, cn) > room)
                cn = cn > 256 ? cn / 2 : cn - 1;
            if (cn <= 0) {
                if (r == head) {
                    if (batches_inflight == 0 && scratch_bytes(schedule, 1) + piece_bytes(r->L, 1) > budget) {
                        // Not even one particle fits the whole budget.
                        r->result = DRIFT_ERROR_OUT_OF_MEMORY;
                        r->done = true;
                        r->completed = Clock::now();
                        pending.pop_front();
                        cv_done.notify_all();
                        return plan();
                    }
                    break;  // keep FIFO order for the head: wait for memory
                }
                continue;
            }
            Piece pc{};
            pc.req = r;
            pc.c0 = r->admitted;
            pc.cn = cn;
            size_t off = used;
            pc.off_y0 = off;
            off += align_up(cn * 48);
            pc.off_grid = off;
            off += align_up(r->L.ts ? r->L.nt * sizeof(double) : cn * sizeof(double));
            pc.off_out = off;
            if (r->L.out) off += align_up((size_t)r->L.nt * cn * 48);
            pc.off_fin = off;
            if (r->L.y_final) off += align_up(cn * 48);
            pc.off_st = off;
            if (r->L.status) off += align_up(cn);
            pc.off_err = off;
            if (r->L.err_code) off += align_up(cn * 4);
            pc.off_acc = off;
            if (r->L.n_accepted) off += align_up(cn * 4);
            pc.off_rej = off;
            if (r->L.n_rejected) off += align_up(cn * 4);
            used = off;
            r->admitted += cn;
            particles += cn;
            batch->pieces.push_back(pc);
            if (r->admitted == r->L.n) taken.push_back(r);
            if (r != head && cn < remaining) break;
        }
        if (batch->pieces.empty()) return nullptr;
        for (Request *r : taken) pending.erase(std::find(pending.begin(), pending.end(), r));
        const size_t scratch = scratch_bytes(schedule, particles);
        for (Piece &pc : batch->pieces)
            for (size_t *o : {&pc.off_y0, &pc.off_grid, &pc.off_out, &pc.off_fin, &pc.off_st, &pc.off_err,
                              &pc.off_acc, &pc.off_rej})
                *o += scratch;
        used += scratch;

        // Small batches run on the high-priority stream 0 and may use every
        // SM; large ones use the other streams and leave the reserve free.
        const bool small = particles <= small_particles;
        int slot = -1;
        if (small && !workers[0]->busy) slot = 0;
        for (int i = 1; slot < 0 && i < (int)workers.size(); i++)
            if (!workers[i]->busy) slot = i;
        if (slot < 0) slot = 0;  // only stream 0 is free
        batch->slot = slot;
        batch->bytes = used;
        batch->scratch = scratch;
        batch->schedule = schedule;
        batch->launch_sms = small ? sm_count : std::max(1, sm_count - reserve_sms);
        workers[slot]->busy = true;
        bytes_inflight += used;
        batches_inflight++;
        return batch;
    }

    // Without mu: every CUDA call of one batch on its stream, ending with a
    // wait for the stream.  Returns the batch's drift_result.
    int execute(Batch &b)
    {
        cudaStream_t s = streams[b.slot];
        char *base = static_cast<char *>(b.dmem);
        std::vector<drift_launch> sub(b.pieces.size());
        for (size_t i = 0; i < b.pieces.size(); i++) {
            Piece &pc = b.pieces[i];
            const drift_launch &L = pc.req->L;
            drift_launch &D = sub[i];
            D = L;
            D.n = pc.cn;
            D.y0 = reinterpret_cast<double *>(base + pc.off_y0);
            cudaMemcpyAsync((void *)D.y0, L.y0 + pc.c0 * 6, pc.cn * 48, cudaMemcpyHostToDevice, s);
            if (L.ts) {
                D.ts = reinterpret_cast<double *>(base + pc.off_grid);
                D.t_end = nullptr;
                cudaMemcpyAsync((void *)D.ts, L.ts, L.nt * sizeof(double), cudaMemcpyHostToDevice, s);
            } else {
                D.t_end = reinterpret_cast<double *>(base + pc.off_grid);
                cudaMemcpyAsync((void *)D.t_end, L.t_end + pc.c0, pc.cn * sizeof(double),
                                cudaMemcpyHostToDevice, s);
            }
            D.out = L.out ? reinterpret_cast<double *>(base + pc.off_out) : nullptr;
            D.y_final = L.y_final ? reinterpret_cast<double *>(base + pc.off_fin) : nullptr;
            D.status = L.status ? reinterpret_cast<uint8_t *>(base + pc.off_st) : nullptr;
            D.err_code = L.err_code ? reinterpret_cast<int32_t *>(base + pc.off_err) : nullptr;
            D.n_accepted = L.n_accepted ? reinterpret_cast<uint32_t *>(base + pc.off_acc) : nullptr;
            D.n_rejected = L.n_rejected ? reinterpret_cast<uint32_t *>(base + pc.off_rej) : nullptr;
            D.schedule = b.schedule;
            D.workspace = base;
            D.workspace_bytes = b.scratch;
        }
        drift::TraceRange trace("drift server batch");
        int rc = drift_internal_launch_batch(b.launch_sms, sub.data(), (int32_t)sub.size(), base, s);
        if (rc == DRIFT_SUCCESS) {
            for (size_t i = 0; i < b.pieces.size(); i++) {
                Piece &pc = b.pieces[i];
                const drift_launch &L = pc.req->L;
                const drift_launch &D = sub[i];
                if (L.out)
                    cudaMemcpy2DAsync(L.out + pc.c0 * 6, L.n * 48, D.out, pc.cn * 48, pc.cn * 48, L.nt,
                                      cudaMemcpyDeviceToHost, s);
                if (L.y_final)
                    cudaMemcpyAsync(L.y_final + pc.c0 * 6, D.y_final, pc.cn * 48, cudaMemcpyDeviceToHost, s);
                if (L.status) cudaMemcpyAsync(L.status + pc.c0, D.status, pc.cn, cudaMemcpyDeviceToHost, s);
                if (L.err_code)
                    cudaMemcpyAsync(L.err_code + pc.c0, D.err_code, pc.cn * 4, cudaMemcpyDeviceToHost, s);
                if (L.n_accepted)
                    cudaMemcpyAsync(L.n_accepted + pc.c0, D.n_accepted, pc.cn * 4, cudaMemcpyDeviceToHost, s);
                if (L.n_rejected)
                    cudaMemcpyAsync(L.n_rejected + pc.c0, D.n_rejected, pc.cn * 4, cudaMemcpyDeviceToHost, s);
            }
        }
        cudaFreeAsync(b.dmem, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = cudaGetLastError();
        else cudaGetLastError();
        if (rc == DRIFT_SUCCESS && e != cudaSuccess) rc = DRIFT_ERROR_CUDA;
        return rc;
    }

    void work(int slot)
    {
        cudaSetDevice(device);
        Worker &w = *workers[slot];
        std::unique_lock<std::mutex> lock(mu);
        while (true) {
            w.cv.wait(lock, [&] { return w.job != nullptr || quit; });
            if (!w.job) break;  // quit with nothing to do
            std::unique_ptr<Batch> b = std::move(w.job);
            lock.unlock();
            const int rc = execute(*b);
            lock.lock();
            for (Piece &pc : b->pieces) {
                if (rc != DRIFT_SUCCESS) pc.req->result = rc;
                pc.req->finished += pc.cn;
                stats.bytes_to_device += pc.cn * 48;
                if (pc.req->L.out) stats.bytes_to_host += (size_t)pc.req->L.nt * pc.cn * 48;
                maybe_complete(pc.req);
            }
            bytes_inflight -= b->bytes;
            batches_inflight--;
            w.busy = false;
            cv_work.notify_all();
        }
    }

    void run()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(mu);
        while (true) {
            if (stop && batches_inflight == 0) break;
            std::unique_ptr<Batch> b = stop ? nullptr : plan();
            if (!b) {
                cv_work.wait_for(lock, std::chrono::milliseconds(5));
                continue;
            }
            // The allocation is the scheduler's only CUDA call; it runs
            // without the mutex.  Only this thread plans batches, so the
            // pieces are still the last particles admitted if they must be
            // given back.
            lock.unlock();
            void *dmem = nullptr;
            cudaError_t e = cudaMallocFromPoolAsync(&dmem, b->bytes, pool, streams[b->slot]);
            if (e != cudaSuccess) cudaGetLastError();
            lock.lock();
            if (e != cudaSuccess) {
                give_back(*b);
                bytes_inflight -= b->bytes;
                batches_inflight--;
                workers[b->slot]->busy = false;
                cv_work.wait_for(lock, std::chrono::milliseconds(5));  // wait for memory
                continue;
            }
            b->dmem = dmem;
            stats.batches_launched++;
            stats.pieces_launched += b->pieces.size();
            stats.peak_bytes_in_flight = std::max<uint64_t>(stats.peak_bytes_in_flight, bytes_inflight);
            Worker &w = *workers[b->slot];
            w.job = std::move(b);
            w.cv.notify_one();
        }
    }
};

// Counts a thread inside a wait for drift_server_destroy, which frees the
// server only once every waiter has left.  Constructed after the wait's lock
// and so destroyed while it is still held.
struct WaiterScope {
    drift_server *s;
    explicit WaiterScope(drift_server *srv) : s(srv) { s->waiters++; }
    ~WaiterScope()
    {
        if (--s->waiters == 0) s->cv_idle.notify_all();
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
    for (int i = 0; i < (int)raw->streams.size(); i++) raw->workers.push_back(std::make_unique<drift_server::Worker>());
    for (int i = 0; i < (int)raw->streams.size(); i++)
        raw->workers[i]->thread = std::thread([raw, i] { raw->work(i); });
    raw->scheduler = std::thread([raw] { raw->run(); });
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
    WaiterScope scope(s);
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

int drift_server_wait_any(drift_server *s, const uint64_t *tickets, int32_t count, double timeout_s,
                          int32_t *index, int *request_result, double *latency_s)
{
    if (!s || !tickets || !index || count < 1)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument or empty ticket list");
    std::unique_lock<std::mutex> lock(s->mu);
    WaiterScope scope(s);
    std::vector<Request *> rs((size_t)count);
    for (int32_t i = 0; i < count; i++) {
        auto it = s->requests.find(tickets[i]);
        if (it == s->requests.end())
            return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown ticket");
        rs[i] = it->second.get();
    }
    // The earliest completion among the finished requests, so that a client
    // retiring one request at a time sees them in completion order.
    int32_t found = -1;
    auto pred = [&] {
        for (int32_t i = 0; i < count; i++)
            if (rs[i]->done && (found < 0 || rs[i]->completed < rs[found]->completed)) found = i;
        return found >= 0;
    };
    if (timeout_s > 0) {
        if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), pred))
            return drift_internal_fail(DRIFT_ERROR_TIMEOUT, "every request still running");
    } else {
        s->cv_done.wait(lock, pred);
    }
    Request *r = rs[found];
    *index = found;
    if (request_result) *request_result = r->result;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->completed - r->submitted).count();
    s->requests.erase(r->ticket);
    return DRIFT_SUCCESS;
}

int drift_server_stats_get(drift_server *s, drift_server_stats *out)
{
    if (!s || !out) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->requests_pending = s->pending.size();
    out->batches_in_flight = s->batches_inflight;
    out->bytes_in_flight = s->bytes_inflight;
    out->bytes_pending = 0;
    for (const Request *r : s->pending) out->bytes_pending += piece_bytes(r->L, r->L.n - r->admitted);
    out->device = s->device;
    out->reserved = 0;
    return DRIFT_SUCCESS;
}

int drift_server_cancel(drift_server *s, uint64_t ticket)
{
    if (!s) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "server is NULL");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end())
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown ticket");
    Request *r = it->second.get();
    if (r->done) return DRIFT_SUCCESS;  // already finished: its result stands
    r->cancelled = true;
    auto pos = std::find(s->pending.begin(), s->pending.end(), r);
    if (pos != s->pending.end()) s->pending.erase(pos);
    s->maybe_complete(r);  // ends now unless some of its particles are on the GPU
    s->cv_work.notify_all();
    return DRIFT_SUCCESS;
}

int drift_server_destroy(drift_server *s)
{
    if (!s) return DRIFT_SUCCESS;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        for (Request *r : s->pending) {
            r->cancelled = true;
            s->maybe_complete(r);
        }
        s->pending.clear();
        s->cv_done.notify_all();
    }
    s->cv_work.notify_all();
    if (s->scheduler.joinable()) s->scheduler.join();  // returns once no batch is in flight
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->quit = true;
        for (auto &w : s->workers) w->cv.notify_all();
    }
    for (auto &w : s->workers)
        if (w->thread.joinable()) w->thread.join();
    {
        // Every request has ended (cancelled, or its batches finished), so
        // each thread still inside a wait is on its way out.
        std::unique_lock<std::mutex> lock(s->mu);
        s->cv_idle.wait(lock, [s] { return s->waiters == 0; });
    }
    for (auto st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return DRIFT_SUCCESS;
}

}  // extern "C"
