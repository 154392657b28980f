// drift_kernels.cuh -- integration kernels, compiled once per precision mode.
//
// The including translation unit defines DRIFT_PRECISION_NS (the namespace
// that receives this unit's launch function) and is compiled either with
// -fmad=false (stage arithmetic rounds like the reference) or -fmad=true.
//
// One thread integrates one particle at a time.  In the plain schedule
// thread g takes particle g and exits when it is done (the reference's
// one-thread-per-particle launch, kernels/src/lib.rs:143-216).  In the
// persistent schedule the grid is sized to the resident capacity of the GPU
// and a thread that finishes takes the next particle from a device-wide
// cursor (one atomic per warp-group of requesters), so particles whose step
// counts differ by orders of magnitude keep every lane busy until the queue
// drains.
#pragma once

#include <algorithm>
#include <type_traits>

#include "drift_dop853.cuh"
#include "drift_dopr54.cuh"
#include "drift_launch_args.cuh"

#ifndef DRIFT_PRECISION_NS
#error "DRIFT_PRECISION_NS must name the precision namespace"
#endif

namespace drift {
namespace DRIFT_PRECISION_NS {

__device__ __forceinline__ int64_t claim_particle(unsigned long long *cursor)
{
    // Warp-aggregated claim: the lanes that need work right now share one
    // atomic and take consecutive queue positions.
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(cursor, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    unsigned below = mask & ((1u << lane) - 1u);
    return (int64_t)(base + (unsigned long long)__popc(below));
}

// Batched launches: the request whose particles [first, first + n) hold
// particle p (the last segment whose first index is <= p).
__device__ __forceinline__ int segment_of(const KernelArgs &a, int64_t p)
{
    int lo = 0, hi = a.nsegs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (a.segs[mid].first <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// The potential functor of a launch: the descriptor's potential, or the
// summed force model held in the kernel's parameter space.
template <class Pot>
__device__ __forceinline__ Pot make_pot(const KernelArgs &a, const double *table)
{
    return Pot(a.potential, table);
}
template <>
__device__ __forceinline__ Composite make_pot<Composite>(const KernelArgs &a, const double *table)
{
    return Composite(&a.model, table);
}

// Potentials that read the bulge table staged in shared memory.
template <class Pot>
__host__ __device__ constexpr bool needs_bulge_table()
{
    return std::is_same<Pot, Bovy>::value || std::is_same<Pot, Composite>::value;
}


// Launch bounds of the integration kernels: at most DRIFT_MAX_THREADS
// threads per block, and registers allocated so that a given number of such
// blocks can be resident on one SM.  Registers are allocated per scheduler
// (16K each), so the choices are two warps per scheduler (up to 255
// registers), three (168) or four (128).  Measured on full workloads
// (throughput, not the tail of a slice):
//   DOP853, light forces: DRIFT_MIN_BLOCKS_DOP853 = 2 blocks of 128; the step
//     fits in about 250 registers with rcont5..8 held in registers (the
//     Plummer workload, 2^20 particles: 67.2 ms per pass, against 70.2 ms
//     with them parked in shared memory and 71.7 ms at 3 blocks).
//   DOP853, Bovy and force models: DRIFT_MIN_BLOCKS_DOP853_HEAVY = 3 (168
//     registers, a few hundred bytes of spills): the uneven Bovy workload,
//     2^22 particles, 12.36 s per pass against 12.93 s at 2 blocks (a
//     2^18-particle slice, whose pass is its slowest particle, prefers 2).
//   DOPR54: DRIFT_MIN_BLOCKS_PER_SM = 3 (the Kepler configuration: 7.15 ms
//     against 7.22 ms at 2).
#ifndef DRIFT_MAX_THREADS
#define DRIFT_MAX_THREADS 128
#endif
#ifndef DRIFT_MIN_BLOCKS_PER_SM
#define DRIFT_MIN_BLOCKS_PER_SM 3
#endif
#ifndef DRIFT_MIN_BLOCKS_DOP853
#define DRIFT_MIN_BLOCKS_DOP853 2
#endif
#ifndef DRIFT_MIN_BLOCKS_DOP853_HEAVY
#define DRIFT_MIN_BLOCKS_DOP853_HEAVY 3
#endif

template <int METHOD, class Pot>
struct LaunchShape {
    static constexpr int threads = DRIFT_MAX_THREADS;
    static constexpr int min_blocks =
        METHOD != DRIFT_DOP853 ? DRIFT_MIN_BLOCKS_PER_SM
                               : (compact_extra_stages<Pot>() ? DRIFT_MIN_BLOCKS_DOP853_HEAVY : DRIFT_MIN_BLOCKS_DOP853);
};

// Dynamic shared memory per block: the DOP853 rcont parking tile (24
// doubles per thread, column-major by thread), then the Bovy tables.
__host__ __device__ constexpr size_t smem_bytes(int method, int kind, int block)
{
    return (method == DRIFT_DOP853 ? 24 * sizeof(double) * block : 0) +
           ((kind == DRIFT_POT_BOVY || kind == DRIFT_POT_MODEL) ? BOVY_SMEM_DOUBLES * sizeof(double) : 0);
}

// TAPE (DOP853 only): record every accepted step of every particle in
// a.tape for the adjoint pass; a particle whose tape is full stops with
// DRIFT_PARTICLE_TAPE_FULL.
template <int METHOD, class Pot, bool TAPE = false>
__global__ void __launch_bounds__(LaunchShape<METHOD, Pot>::threads, LaunchShape<METHOD, Pot>::min_blocks)
    integrate_kernel(const __grid_constant__ KernelArgs a)
{
    static_assert(!TAPE || METHOD == DRIFT_DOP853, "the step tape is recorded by DOP853 only");
    extern __shared__ __align__(16) double smem[];
    // [park tile (DOP853)][Bovy tables (Bovy, force models)]
    volatile double *park = smem + threadIdx.x;
    double *table = smem + (METHOD == DRIFT_DOP853 ? 24 * blockDim.x : 0);
    if (needs_bulge_table<Pot>()) {
        stage_bovy_tables(table, a.bulge);
        __syncthreads();
    }
    const Pot pot = make_pot<Pot>(a, table);
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t deadline = a.timeout_ns ? global_timer_ns() + a.timeout_ns : 0;

    Dop853Lane<Pot> l853;
    Dopr54Lane<Pot> l54;
    TimeMajorOut out;
    out.base = a.out;
    out.y_final = a.y_final;
    out.n = a.n;
    out.nt = a.nt;
    Grid grid;
    grid.ts = a.ts;
    grid.t0 = a.t0;
    grid.nt = a.nt;
    grid.t_end = 0.0;

    int64_t pid = -1;
    int64_t attempts = 0;
    uint32_t nacc = 0, nrej = 0;
    bool active = false;

    int32_t seg = 0;  // batched launches: request of the current particle

    auto start = [&](int64_t p) {
        const double *y0p;
        int64_t stride;
        if (a.nsegs) {
            seg = segment_of(a, p);
            const Segment &S = a.segs[seg];
            p -= S.first;
            grid.ts = S.ts;
            grid.t0 = S.t0;
            grid.nt = S.nt;
            grid.t_end = S.ts ? 0.0 : S.t_end[p];
            out.base = S.out;
            out.y_final = S.y_final;
            out.n = S.n;
            out.nt = S.nt;
            stride = S.y0_stride;
            y0p = stride ? S.y0 + p : S.y0 + p * 6;
        } else {
            if (!a.ts) grid.t_end = __ldg(a.t_end + p);
            stride = a.y0_stride;
            y0p = stride ? a.y0 + p : a.y0 + p * 6;
        }
        pid = p;
        out.pid = p;
        double y0[6];
        if (stride) {
#pragma unroll
            for (int i = 0; i < 6; i++) y0[i] = __ldg(y0p + i * stride);
        } else {
            const double2 *src = reinterpret_cast<const double2 *>(y0p);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                double2 v = __ldg(src + i);
                y0[2 * i] = v.x;
                y0[2 * i + 1] = v.y;
            }
        }
        if (METHOD == DRIFT_DOP853)
            l853.begin(pot, y0, grid, a.rtol, a.atol, out);
        else
            l54.begin(pot, y0, grid, a.dt_one, a.tol54, out, a.arbitrary_times != 0);
        attempts = 0;
        nacc = 0;
        nrej = 0;
        active = true;
    };

    auto finish = [&](int status) {
        if (status != DRIFT_PARTICLE_OK) {
            // Samples the integration did not reach are marked NaN.
            double nan6[6];
#pragma unroll
            for (int i = 0; i < 6; i++) nan6[i] = __longlong_as_double(0x7ff8000000000000LL);
            int32_t first = (METHOD == DRIFT_DOP853) ? l853.next + 1 : l54.ii + 1;
            for (int32_t k = first; k < grid.nt; k++) out.write(k, nan6);
        }
        int32_t code = 0;
        if (METHOD == DRIFT_DOPR54) {
            code = l54.err;
            if (status == DRIFT_PARTICLE_OK && (code & 1)) status = DRIFT_PARTICLE_MIN_STEP;
        }
        uint8_t *st = a.status;
        int32_t *ec = a.err_code;
        uint32_t *na = a.n_accepted, *nr = a.n_rejected;
        if (a.nsegs) {
            const Segment &S = a.segs[seg];
            st = S.status;
            ec = S.err_code;
            na = S.n_accepted;
            nr = S.n_rejected;
        }
        if (st) st[pid] = (uint8_t)status;
        if (ec) ec[pid] = code;
        if (na) na[pid] = nacc;
        if (nr) nr[pid] = nrej;
        if (a.chunk_done) {
            // every write of this particle is visible before it counts as done
            __threadfence();
            atomicAdd(a.chunk_done + pid / a.chunk_len, 1u);
        }
        active = false;
    };

    // Warp-uniform control: every lane of the warp stays in the loop until
    // no lane has work, and the vote at the top of each iteration makes the
    // lanes reconverge before the next step, so one step instruction stream
    // serves all particles of the warp.
    bool exhausted = false;  // no further particle for this lane
    if (!a.persistent) {
        if (gtid < a.n)
            start(gtid);
        else
            exhausted = true;
    }
    while (true) {
        if (a.persistent && !active && !exhausted) {
            int64_t p = claim_particle(a.cursor);
            if (p < a.n)
                start(a.order ? (int64_t)__ldg(a.order + p) : p);
            else
                exhausted = true;
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (!active) continue;
        bool done = (METHOD == DRIFT_DOP853) ? l853.done : l54.done;
        if (done) {
            finish(DRIFT_PARTICLE_OK);
            if (!a.persistent) exhausted = true;
            continue;
        }
        if (attempts >= a.max_steps) {
            finish(DRIFT_PARTICLE_MAX_STEPS);
            if (!a.persistent) exhausted = true;
            continue;
        }
        if (deadline != 0 && (attempts & 63) == 0 && global_timer_ns() > deadline) {
            finish(DRIFT_PARTICLE_TIMEOUT);
            if (!a.persistent) exhausted = true;
            continue;
        }
        if (TAPE && (int64_t)nacc >= a.tape_steps) {
            finish(DRIFT_PARTICLE_TAPE_FULL);
            if (!a.persistent) exhausted = true;
            continue;
        }
        attempts++;
        bool accepted;
        if (METHOD == DRIFT_DOP853) {
            if (TAPE) {
                double *row, *h_slot = nullptr;
                if (a.tape_stride <= 1) {
                    row = a.tape + (pid * a.tape_steps + nacc) * 8;
                } else {
                    const int64_t m = a.tape_stride;
                    const int64_t ncp = (a.tape_steps + m - 1) / m;
                    double *block = a.tape + pid * (ncp * 8 + ((a.tape_steps + 1) & ~int64_t(1)));
                    row = (nacc % m == 0) ? block + (nacc / m) * 8 : nullptr;
                    h_slot = block + ncp * 8 + nacc;
                }
                accepted = l853.template step<true>(pot, grid, a.rtol, a.atol, out, park, row, h_slot,
                                                    a.sparse_output != 0);
            } else {
                accepted = l853.step(pot, grid, a.rtol, a.atol, out, park, nullptr, nullptr, a.sparse_output != 0);
            }
            if (!accepted && l853.nonfinite_run >= DOP853_NONFINITE_LIMIT) {
                nrej++;
                finish(DRIFT_PARTICLE_NONFINITE);
                if (!a.persistent) exhausted = true;
                continue;
            }
        } else {
            accepted = l54.step(pot, grid, a.tol54, out);
        }
        if (accepted)
            nacc++;
        else
            nrej++;
    }
}

// ---- longest-first queue (ordered schedule) ------------------------------
//
// Cost estimate of a particle: number of dynamical times in its time span,
// |t_end - t0| * sqrt(|F| / r + (v / r)^2), plus nt / 4 for the output
// intervals DOPR54 must land on.  Keys are 4 buckets per octave of cost;
// bucket 0 holds the most expensive particles.
constexpr int ORDER_BUCKETS = 256;

template <class Pot>
__global__ void __launch_bounds__(256) rank_kernel(const __grid_constant__ KernelArgs a, int method,
                                                   uint8_t *keys, unsigned *counts)
{
    __shared__ unsigned hist[ORDER_BUCKETS];
    __shared__ __align__(16) double table[BOVY_SMEM_DOUBLES];
    for (int i = threadIdx.x; i < ORDER_BUCKETS; i += blockDim.x) hist[i] = 0;
    if (needs_bulge_table<Pot>()) stage_bovy_tables(table, a.bulge);
    __syncthreads();
    const Pot pot = make_pot<Pot>(a, table);
    for (int64_t pid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pid < a.n;
         pid += (int64_t)gridDim.x * blockDim.x) {
        double y[6];
        double span, t_start;
        int64_t nt = a.nt;
        auto load = [&](const double *base, int64_t stride, int64_t p) {
#pragma unroll
            for (int i = 0; i < 6; i++) y[i] = stride ? base[p + i * stride] : base[p * 6 + i];
        };
        if (a.nsegs) {
            const Segment &S = a.segs[segment_of(a, pid)];
            const int64_t p = pid - S.first;
            load(S.y0, S.y0_stride, p);
            nt = S.nt;
            span = S.ts ? fabs(__ldg(S.ts + S.nt - 1) - __ldg(S.ts)) : fabs(__ldg(S.t_end + p) - S.t0);
            t_start = S.ts ? __ldg(S.ts) : S.t0;
        } else {
            load(a.y0, a.y0_stride, pid);
            span = a.ts ? fabs(__ldg(a.ts + a.nt - 1) - __ldg(a.ts)) : fabs(__ldg(a.t_end + pid) - a.t0);
            t_start = a.ts ? __ldg(a.ts) : a.t0;
        }
        double ax, ay, az;
        force_at(pot, t_start, y[0], y[1], y[2], ax, ay, az);
        double r2 = fmax(y[0] * y[0] + y[1] * y[1] + y[2] * y[2], 1e-300);
        double v2 = y[3] * y[3] + y[4] * y[4] + y[5] * y[5];
        double f = sqrt(ax * ax + ay * ay + az * az);
        double cost = span * sqrt(f * rsqrt(r2) + v2 / r2);
        if (method == DRIFT_DOPR54) cost += 0.25 * (double)nt;
        int key = 0;
        if (cost > 0.0 && cost < 1e300) key = min(max((int)floor(4.0 * log2(cost)) + 128, 0), ORDER_BUCKETS - 1);
        else if (!(cost > 0.0)) key = 0;
        else key = ORDER_BUCKETS - 1;
        keys[pid] = (uint8_t)key;
        atomicAdd(&hist[ORDER_BUCKETS - 1 - key], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ORDER_BUCKETS; i += blockDim.x)
        if (hist[i]) atomicAdd(&counts[i], hist[i]);
}

// Exclusive prefix sum of the 256 bucket counts, in place (one block of 256).
__global__ void __launch_bounds__(256) order_scan_kernel(unsigned *counts)
{
    __shared__ unsigned v[ORDER_BUCKETS];
    const int i = threadIdx.x;
    v[i] = counts[i];
    __syncthreads();
    for (int off = 1; off < ORDER_BUCKETS; off <<= 1) {
        unsigned add = i >= off ? v[i - off] : 0u;
        __syncthreads();
        v[i] += add;
        __syncthreads();
    }
    counts[i] = i ? v[i - 1] : 0u;
}

// order[offset[bucket]++] = pid, one atomic per (warp, bucket) group.
__global__ void __launch_bounds__(256) order_scatter_kernel(int64_t n, const uint8_t *keys,
                                                            unsigned *offsets, uint32_t *order)
{
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = base + threadIdx.x;
        const bool valid = pid < n;
        const int bucket = valid ? ORDER_BUCKETS - 1 - keys[pid] : -1 - (int)(threadIdx.x & 31);
        const unsigned peers = __match_any_sync(0xffffffffu, bucket);
        if (valid) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(peers) - 1;
            unsigned pos = 0;
            if (lane == leader) pos = atomicAdd(&offsets[bucket], (unsigned)__popc(peers));
            pos = __shfl_sync(peers, pos, leader);
            order[pos + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)pid;
        }
    }
}

// ---- chunk-ordered queue (streamed copy-out) -----------------------------
//
// Bucket b of the rank histogram holds particles of cost about
// 2^((127.5 - b) / 4) (key = 255 - b = floor(4 log2 cost) + 128).  One
// thread finds the first bucket whose cost is below total / (lanes x
// nchunks): particles in buckets before it last longer than a chunk's share
// of the launch and go first; the rest are queued chunk by chunk.
__global__ void __launch_bounds__(32) chunk_split_kernel(const unsigned *counts, double lanes_x_chunks,
                                                         unsigned *split)
{
    if (threadIdx.x != 0) return;
    double total = 0.0;
    for (int b = 0; b < ORDER_BUCKETS; b++) total += (double)counts[b] * exp2((127.5 - b) * 0.25);
    const double threshold = total / lanes_x_chunks;
    unsigned k = ORDER_BUCKETS;
    for (int b = 0; b < ORDER_BUCKETS; b++)
        if (exp2((127.5 - b) * 0.25) < threshold) {
            k = b;
            break;
        }
    *split = k;
}

__device__ __forceinline__ int chunk_bucket(int64_t pid, const uint8_t *keys, int64_t chunk_len, unsigned split)
{
    const int b = ORDER_BUCKETS - 1 - keys[pid];
    const int cls = (unsigned)b < split ? 0 : 1 + (int)(pid / chunk_len);
    return cls * ORDER_BUCKETS + b;
}

__global__ void __launch_bounds__(256) chunk_hist_kernel(int64_t n, const uint8_t *keys, int64_t chunk_len,
                                                         const unsigned *split, unsigned *chunk_counts)
{
    const unsigned k = *split;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = base + threadIdx.x;
        const bool valid = pid < n;
        const int id = valid ? chunk_bucket(pid, keys, chunk_len, k) : -1 - (int)(threadIdx.x & 31);
        const unsigned peers = __match_any_sync(0xffffffffu, id);
        if (valid && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&chunk_counts[id], (unsigned)__popc(peers));
    }
}

// Exclusive prefix sum of `count` entries in place (one block of 1024).
__global__ void __launch_bounds__(1024) chunk_scan_kernel(unsigned *v, int count)
{
    __shared__ unsigned tile[1024];
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < count; base += 1024) {
        const int i = base + threadIdx.x;
        const unsigned x = i < count ? v[i] : 0u;
        tile[threadIdx.x] = x;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const unsigned add = threadIdx.x >= off ? tile[threadIdx.x - off] : 0u;
            __syncthreads();
            tile[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < count) v[i] = carry + tile[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == 1023) carry += tile[1023];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) chunk_scatter_kernel(int64_t n, const uint8_t *keys, int64_t chunk_len,
                                                            const unsigned *split, unsigned *offsets,
                                                            uint32_t *order)
{
    const unsigned k = *split;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = base + threadIdx.x;
        const bool valid = pid < n;
        const int id = valid ? chunk_bucket(pid, keys, chunk_len, k) : -1 - (int)(threadIdx.x & 31);
        const unsigned peers = __match_any_sync(0xffffffffu, id);
        if (valid) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(peers) - 1;
            unsigned pos = 0;
            if (lane == leader) pos = atomicAdd(&offsets[id], (unsigned)__popc(peers));
            pos = __shfl_sync(peers, pos, leader);
            order[pos + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)pid;
        }
    }
}

inline cudaError_t launch_rank(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts, int grid,
                               cudaStream_t stream)
{
    switch (a.potential.kind) {
    case DRIFT_POT_KEPLER: rank_kernel<KeplerGalpy><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_PLUMMER: rank_kernel<Plummer><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_BOVY: rank_kernel<Bovy><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_KEPLER_CARTESIAN:
        rank_kernel<KeplerCartesian><<<grid, 256, 0, stream>>>(a, method, keys, counts);
        break;
    case DRIFT_POT_MODEL: rank_kernel<Composite><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

inline cudaError_t build_order_chunked_impl(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                                            unsigned *split, unsigned *chunk_counts, uint32_t *order,
                                            int64_t chunk_len, int nchunks, int64_t lanes, int sm_count,
                                            cudaStream_t stream)
{
    const int entries = (nchunks + 1) * ORDER_BUCKETS;
    cudaError_t e = cudaMemsetAsync(counts, 0, ORDER_BUCKETS * sizeof(unsigned), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(chunk_counts, 0, entries * sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>((a.n + 255) / 256, (int64_t)sm_count * 8);
    e = launch_rank(a, method, keys, counts, grid, stream);
    if (e != cudaSuccess) return e;
    chunk_split_kernel<<<1, 32, 0, stream>>>(counts, (double)lanes * nchunks, split);
    chunk_hist_kernel<<<grid, 256, 0, stream>>>(a.n, keys, chunk_len, split, chunk_counts);
    chunk_scan_kernel<<<1, 1024, 0, stream>>>(chunk_counts, entries);
    chunk_scatter_kernel<<<grid, 256, 0, stream>>>(a.n, keys, chunk_len, split, chunk_counts, order);
    return cudaGetLastError();
}

inline cudaError_t build_order_impl(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                                    uint32_t *order, int sm_count, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(counts, 0, ORDER_BUCKETS * sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>((a.n + 255) / 256, (int64_t)sm_count * 8);
    switch (a.potential.kind) {
    case DRIFT_POT_KEPLER: rank_kernel<KeplerGalpy><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_PLUMMER: rank_kernel<Plummer><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_BOVY: rank_kernel<Bovy><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    case DRIFT_POT_KEPLER_CARTESIAN:
        rank_kernel<KeplerCartesian><<<grid, 256, 0, stream>>>(a, method, keys, counts);
        break;
    case DRIFT_POT_MODEL: rank_kernel<Composite><<<grid, 256, 0, stream>>>(a, method, keys, counts); break;
    default: return cudaErrorInvalidValue;
    }
    order_scan_kernel<<<1, ORDER_BUCKETS, 0, stream>>>(counts);
    order_scatter_kernel<<<grid, 256, 0, stream>>>(a.n, keys, counts, order);
    return cudaGetLastError();
}

template <class Pot>
__global__ void __launch_bounds__(256) force_kernel(drift_potential p, int64_t n, const double *xyz,
                                                    double *acc, const __grid_constant__ BulgeTable bt)
{
    __shared__ __align__(16) double table[BOVY_SMEM_DOUBLES];
    if (std::is_same<Pot, Bovy>::value) {
        stage_bovy_tables(table, bt);
        __syncthreads();
    }
    const Pot pot(p, table);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ax, ay, az;
        pot.force(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], ax, ay, az);
        acc[3 * i] = ax;
        acc[3 * i + 1] = ay;
        acc[3 * i + 2] = az;
    }
}

inline cudaError_t force_impl(const drift_potential &p, int64_t n, const double *xyz, double *acc,
                              const BulgeTable &bt, int grid, cudaStream_t stream)
{
    switch (p.kind) {
    case DRIFT_POT_KEPLER: force_kernel<KeplerGalpy><<<grid, 256, 0, stream>>>(p, n, xyz, acc, bt); break;
    case DRIFT_POT_PLUMMER: force_kernel<Plummer><<<grid, 256, 0, stream>>>(p, n, xyz, acc, bt); break;
    case DRIFT_POT_BOVY: force_kernel<Bovy><<<grid, 256, 0, stream>>>(p, n, xyz, acc, bt); break;
    case DRIFT_POT_KEPLER_CARTESIAN:
        force_kernel<KeplerCartesian><<<grid, 256, 0, stream>>>(p, n, xyz, acc, bt);
        break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Acceleration of a force model at time t (drift_force_model_eval).
__global__ void __launch_bounds__(256) model_force_kernel(const __grid_constant__ drift_force_model m,
                                                          const __grid_constant__ BulgeTable bt, double t,
                                                          int64_t n, const double *xyz, double *acc)
{
    __shared__ __align__(16) double table[BOVY_SMEM_DOUBLES];
    stage_bovy_tables(table, bt);
    __syncthreads();
    const Composite pot(&m, table);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ax, ay, az;
        pot.force_t(t, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], ax, ay, az);
        acc[3 * i] = ax;
        acc[3 * i + 1] = ay;
        acc[3 * i + 2] = az;
    }
}

// One thread per (segment k, source j): accelerations at both ends from the
// sources' own force model, then the quintic Hermite coefficients of each
// axis, written as origins[(k * n_sources + j) * 18 + 6 * axis + c].
__global__ void __launch_bounds__(256) origin_table_kernel(const __grid_constant__ drift_force_model m,
                                                           const __grid_constant__ BulgeTable bt,
                                                           int64_t n_sources, int64_t nt, double t0,
                                                           double dt, const double *traj, double *origins)
{
    __shared__ __align__(16) double table[BOVY_SMEM_DOUBLES];
    stage_bovy_tables(table, bt);
    __syncthreads();
    const Composite pot(&m, table);
    const int64_t total = (nt - 1) * n_sources;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = w / n_sources, j = w - k * n_sources;
        const double *q0 = traj + (k * n_sources + j) * 6;
        const double *q1 = traj + ((k + 1) * n_sources + j) * 6;
        const double ta = t0 + dt * (double)k;
        const double tb = t0 + dt * (double)(k + 1);
        double a0[3], a1[3];
        pot.force_t(ta, q0[0], q0[1], q0[2], a0[0], a0[1], a0[2]);
        pot.force_t(tb, q1[0], q1[1], q1[2], a1[0], a1[1], a1[2]);
        double *c = origins + w * 18;
        for (int axis = 0; axis < 3; axis++)
            hermite5(q0[axis], q0[3 + axis], a0[axis], q1[axis], q1[3 + axis], a1[axis], dt, c + 6 * axis);
    }
}

// Host-side launcher for this precision unit.
inline cudaError_t launch_impl(const KernelArgs &a, int method, int grid, int block,
                               cudaStream_t stream)
{
    const int kind = a.potential.kind;
#define DRIFT_LAUNCH(M, P)                                                                   \
    do {                                                                                     \
        if (M == DRIFT_DOP853 && a.tape)                                                     \
            integrate_kernel<DRIFT_DOP853, P, true>                                          \
                <<<grid, block, smem_bytes(M, kind, block), stream>>>(a);                    \
        else                                                                                 \
            integrate_kernel<M, P><<<grid, block, smem_bytes(M, kind, block), stream>>>(a); \
        return cudaGetLastError();                                                           \
    } while (0)
#define DRIFT_POT_SWITCH(M)                                                      \
    switch (kind) {                                                              \
    case DRIFT_POT_KEPLER: DRIFT_LAUNCH(M, KeplerGalpy);                         \
    case DRIFT_POT_PLUMMER: DRIFT_LAUNCH(M, Plummer);                            \
    case DRIFT_POT_BOVY: DRIFT_LAUNCH(M, Bovy);                                  \
    case DRIFT_POT_KEPLER_CARTESIAN: DRIFT_LAUNCH(M, KeplerCartesian);           \
    case DRIFT_POT_MODEL: DRIFT_LAUNCH(M, Composite);                            \
    default: return cudaErrorInvalidValue;                                       \
    }
    if (method == DRIFT_DOP853) {
        DRIFT_POT_SWITCH(DRIFT_DOP853);
    } else {
        DRIFT_POT_SWITCH(DRIFT_DOPR54);
    }
#undef DRIFT_POT_SWITCH
#undef DRIFT_LAUNCH
}

inline int max_threads_impl() { return DRIFT_MAX_THREADS; }

inline cudaError_t occupancy_impl(int method, int kind, int block, bool tape, int *blocks_per_sm)
{
#define DRIFT_OCC(M, P)                                                                     \
    return (M == DRIFT_DOP853 && tape)                                                      \
               ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(                             \
                     blocks_per_sm, integrate_kernel<DRIFT_DOP853, P, true>, block,         \
                     smem_bytes(M, kind, block))                                            \
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(                             \
                     blocks_per_sm, integrate_kernel<M, P>, block, smem_bytes(M, kind, block))
#define DRIFT_OCC_SWITCH(M)                                                     \
    switch (kind) {                                                             \
    case DRIFT_POT_KEPLER: DRIFT_OCC(M, KeplerGalpy);                           \
    case DRIFT_POT_PLUMMER: DRIFT_OCC(M, Plummer);                              \
    case DRIFT_POT_BOVY: DRIFT_OCC(M, Bovy);                                    \
    case DRIFT_POT_KEPLER_CARTESIAN: DRIFT_OCC(M, KeplerCartesian);             \
    case DRIFT_POT_MODEL: DRIFT_OCC(M, Composite);                              \
    default: return cudaErrorInvalidValue;                                      \
    }
    if (method == DRIFT_DOP853) {
        DRIFT_OCC_SWITCH(DRIFT_DOP853);
    } else {
        DRIFT_OCC_SWITCH(DRIFT_DOPR54);
    }
#undef DRIFT_OCC_SWITCH
#undef DRIFT_OCC
}

}  // namespace DRIFT_PRECISION_NS
}  // namespace drift
