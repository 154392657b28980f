// drift_common.cuh -- small shared pieces of the integrator kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "drift_math.cuh"
#include "drift_potentials.cuh"

namespace drift {

// dop853.rs:286-299: comparisons without fmin/fmax NaN semantics.
__device__ __forceinline__ double c_min(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double c_max(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double custom_sign(double x, double y)
{
    return y > 0.0 ? fabs(x) : -fabs(x);
}

// Output grid of one particle: either a shared array of nt times, or the
// uniform grid t0..t_end with nt points sampled as OutputGrid::sample does
// (shared/src/config.rs:57-66; exact end point).
struct Grid {
    const double *ts;
    double t0, t_end;
    int32_t nt;
    __device__ __forceinline__ double at(int32_t k) const
    {
        if (ts) return __ldg(ts + k);
        if (k == nt - 1) return t_end;
        return t0 + (t_end - t0) * (double)k / (double)(nt - 1);
    }
};

// 1: trajectory samples are written with streaming (evict-first) stores;
// 0: with ordinary write-back stores.
#ifndef DRIFT_STREAMING_STORES
#define DRIFT_STREAMING_STORES 1
#endif

__device__ __forceinline__ void store6(double *dst, const double *v)
{
    double2 *p = reinterpret_cast<double2 *>(dst);
#if DRIFT_STREAMING_STORES
    __stcs(p + 0, make_double2(v[0], v[1]));
    __stcs(p + 1, make_double2(v[2], v[3]));
    __stcs(p + 2, make_double2(v[4], v[5]));
#else
    p[0] = make_double2(v[0], v[1]);
    p[1] = make_double2(v[2], v[3]);
    p[2] = make_double2(v[4], v[5]);
#endif
}

// Writes one 6-vector of particle `pid` at output slot k of a time-major
// (nt, n, 6) array with 16-byte vector stores (48 B per sample, aligned);
// the sample at the last output time is also the particle's final state.
struct TimeMajorOut {
    double *base;     // NULL: trajectories not requested
    double *y_final;  // NULL: final states not requested
    int64_t n;
    int64_t pid;
    int32_t nt;
    __device__ __forceinline__ void write(int32_t k, const double *v) const
    {
        if (base) store6(base + ((int64_t)k * n + pid) * 6, v);
        if (y_final && k == nt - 1) store6(y_final + pid * 6, v);
    }
};

__device__ __forceinline__ uint64_t global_timer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

}  // namespace drift
