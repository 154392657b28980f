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

template <int METHOD, class Pot>
__global__ void __launch_bounds__(128) integrate_kernel(KernelArgs a)
{
    const Pot pot(a.potential);
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t deadline = a.timeout_ns ? global_timer_ns() + a.timeout_ns : 0;

    Dop853Lane<Pot> l853;
    Dopr54Lane<Pot> l54;
    TimeMajorOut out;
    out.base = a.out;
    out.n = a.n;
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
        if (a.y_final) {
            double2 *dst = reinterpret_cast<double2 *>(a.y_final + pid * 6);
            dst[0] = make_double2(out.last[0], out.last[1]);
            dst[1] = make_double2(out.last[2], out.last[3]);
            dst[2] = make_double2(out.last[4], out.last[5]);
        }
        active = false;
    };

    if (!a.persistent) {
        if (gtid >= a.n) return;
        start(gtid);
    }

    while (true) {
        if (!active) {
            if (!a.persistent) break;
            int64_t p = claim_particle(a.cursor);
            if (p >= a.n) break;
            start(p);
        }
        bool done = (METHOD == DRIFT_DOP853) ? l853.done : l54.done;
        if (done) {
            finish(DRIFT_PARTICLE_OK);
            continue;
        }
        if (attempts >= a.max_steps) {
            finish(DRIFT_PARTICLE_MAX_STEPS);
            continue;
        }
        if (deadline != 0 && (attempts & 63) == 0 && global_timer_ns() > deadline) {
            finish(DRIFT_PARTICLE_TIMEOUT);
            continue;
        }
        attempts++;
        bool accepted;
        if (METHOD == DRIFT_DOP853) {
            accepted = l853.step(pot, grid, a.rtol, a.atol, out);
            if (!accepted && l853.nonfinite_run >= DOP853_NONFINITE_LIMIT) {
                nrej++;
                finish(DRIFT_PARTICLE_NONFINITE);
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

// Host-side launcher for this precision unit.
inline cudaError_t launch_impl(const KernelArgs &a, int method, int grid, int block,
                               cudaStream_t stream)
{
    const int kind = a.potential.kind;
#define DRIFT_LAUNCH(M, P)                                                       \
    do {                                                                         \
        integrate_kernel<M, P><<<grid, block, 0, stream>>>(a);                   \
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

inline cudaError_t occupancy_impl(int method, int kind, int block, int *blocks_per_sm)
{
#define DRIFT_OCC(M, P)                                                                     \
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm,                     \
                                                         integrate_kernel<M, P>, block, 0)
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
