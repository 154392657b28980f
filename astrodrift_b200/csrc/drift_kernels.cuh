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

// Launch bounds of the integration kernels: at most DRIFT_MAX_THREADS
// threads per block, and registers allocated so that DRIFT_MIN_BLOCKS_PER_SM
// such blocks can be resident on one SM.
#ifndef DRIFT_MAX_THREADS
#define DRIFT_MAX_THREADS 128
#endif
#ifndef DRIFT_MIN_BLOCKS_PER_SM
#define DRIFT_MIN_BLOCKS_PER_SM 3
#endif

// Dynamic shared memory per block: the DOP853 rcont parking tile (24
// doubles per thread, column-major by thread), then the Bovy bulge table.
__host__ __device__ constexpr size_t smem_bytes(int method, int kind, int block)
{
    return (method == DRIFT_DOP853 ? 24 * sizeof(double) * block : 0) +
           (kind == DRIFT_POT_BOVY ? sizeof(BulgeTable) : 0);
}

template <int METHOD, class Pot>
__global__ void __launch_bounds__(DRIFT_MAX_THREADS, DRIFT_MIN_BLOCKS_PER_SM)
    integrate_kernel(const __grid_constant__ KernelArgs a)
{
    extern __shared__ double smem[];
    // [park tile (DOP853)][bulge table (Bovy)]
    volatile double *park = smem + threadIdx.x;
    double *table = smem + (METHOD == DRIFT_DOP853 ? 24 * blockDim.x : 0);
    if (std::is_same<Pot, Bovy>::value) {
        for (int i = threadIdx.x; i < BULGE_TABLE_SIZE; i += blockDim.x) table[i] = a.bulge.c[i];
        __syncthreads();
    }
    const Pot pot(a.potential, table);
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

    auto start = [&](int64_t p) {
        pid = p;
        out.pid = p;
        if (!a.ts) grid.t_end = __ldg(a.t_end + p);
        double y0[6];
        const double2 *src = reinterpret_cast<const double2 *>(a.y0 + p * 6);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double2 v = __ldg(src + i);
            y0[2 * i] = v.x;
            y0[2 * i + 1] = v.y;
        }
        if (METHOD == DRIFT_DOP853)
            l853.begin(pot, y0, grid, a.rtol, a.atol, out);
        else
            l54.begin(pot, y0, grid, a.dt_one, a.tol54, out);
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
            for (int32_t k = first; k < a.nt; k++) out.write(k, nan6);
        }
        int32_t code = 0;
        if (METHOD == DRIFT_DOPR54) {
            code = l54.err;
            if (status == DRIFT_PARTICLE_OK && (code & 1)) status = DRIFT_PARTICLE_MIN_STEP;
        }
        if (a.status) a.status[pid] = (uint8_t)status;
        if (a.err_code) a.err_code[pid] = code;
        if (a.n_accepted) a.n_accepted[pid] = nacc;
        if (a.n_rejected) a.n_rejected[pid] = nrej;
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
                start(p);
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
        attempts++;
        bool accepted;
        if (METHOD == DRIFT_DOP853) {
            accepted = l853.step(pot, grid, a.rtol, a.atol, out, park);
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

template <class Pot>
__global__ void __launch_bounds__(256) force_kernel(drift_potential p, int64_t n, const double *xyz,
                                                    double *acc, const __grid_constant__ BulgeTable bt)
{
    __shared__ double table[BULGE_TABLE_SIZE];
    if (std::is_same<Pot, Bovy>::value) {
        for (int i = threadIdx.x; i < BULGE_TABLE_SIZE; i += blockDim.x) table[i] = bt.c[i];
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

// Host-side launcher for this precision unit.
inline cudaError_t launch_impl(const KernelArgs &a, int method, int grid, int block,
                               cudaStream_t stream)
{
    const int kind = a.potential.kind;
#define DRIFT_LAUNCH(M, P)                                                       \
    do {                                                                         \
        integrate_kernel<M, P><<<grid, block, smem_bytes(M, kind, block), stream>>>(a); \
        return cudaGetLastError();                                               \
    } while (0)
#define DRIFT_POT_SWITCH(M)                                                      \
    switch (kind) {                                                              \
    case DRIFT_POT_KEPLER: DRIFT_LAUNCH(M, KeplerGalpy);                         \
    case DRIFT_POT_PLUMMER: DRIFT_LAUNCH(M, Plummer);                            \
    case DRIFT_POT_BOVY: DRIFT_LAUNCH(M, Bovy);                                  \
    case DRIFT_POT_KEPLER_CARTESIAN: DRIFT_LAUNCH(M, KeplerCartesian);           \
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

inline cudaError_t occupancy_impl(int method, int kind, int block, int *blocks_per_sm)
{
#define DRIFT_OCC(M, P)                                                                     \
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                   \
        blocks_per_sm, integrate_kernel<M, P>, block, smem_bytes(M, kind, block))
#define DRIFT_OCC_SWITCH(M)                                                     \
    switch (kind) {                                                             \
    case DRIFT_POT_KEPLER: DRIFT_OCC(M, KeplerGalpy);                           \
    case DRIFT_POT_PLUMMER: DRIFT_OCC(M, Plummer);                              \
    case DRIFT_POT_BOVY: DRIFT_OCC(M, Bovy);                                    \
    case DRIFT_POT_KEPLER_CARTESIAN: DRIFT_OCC(M, KeplerCartesian);             \
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
