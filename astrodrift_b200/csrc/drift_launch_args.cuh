// drift_launch_args.cuh -- parameter block shared by the kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "drift_b200.h"
#include "drift_dopr54.cuh"
#include "drift_composite.cuh"
#include "drift_potentials.cuh"

namespace drift {

// Requests one batched launch can carry; the table travels in the kernel's
// parameter space (MAX_BATCH x 112 bytes), so no device table is needed.
constexpr int MAX_BATCH = DRIFT_MAX_BATCH;  // from drift_b200.h

// One request of a batched launch: particles [first, first + n) of the
// launch's index space, with the request's own inputs, grid and outputs.
struct Segment {
    int64_t first;
    int64_t n;
    const double *y0;         // (n, 6) rows, or 6 columns of y0_stride
    int64_t y0_stride;        // 0: rows; > 0: column stride (elements)
    const double *ts;         // shared grid of this request, or NULL
    double t0;                // per-particle grid start (ts == NULL)
    const double *t_end;      // (n) per-particle grid ends (ts == NULL)
    int32_t nt;
    int32_t reserved;
    double *out;              // (nt, n, 6) or NULL
    double *y_final;          // (n, 6) or NULL
    uint8_t *status;
    int32_t *err_code;
    uint32_t *n_accepted;
    uint32_t *n_rejected;
};

// Grids with at most this many output times count as sparse: DOP853 then
// skips the dense-output stages of steps that emit no sample.  (With dense
// grids most warps emit somewhere in most steps, and warps that take and
// skip the block at different times thrash the instruction cache.)
#ifndef DRIFT_SPARSE_OUTPUT_NT
#define DRIFT_SPARSE_OUTPUT_NT 8
#endif
constexpr int SPARSE_OUTPUT_NT = DRIFT_SPARSE_OUTPUT_NT;

// Everything a launch needs, passed by value as the kernel parameter.
struct KernelArgs {
    int64_t n;
    const double *y0;         // (n, 6) rows, or 6 columns of y0_stride
    int64_t y0_stride;        // 0: rows; > 0: column stride (elements)
    int32_t nt;
    int32_t persistent;       // 0: plain schedule, 1: persistent schedule
    const double *ts;         // shared grid or NULL
    double t0;                // per-particle grid start
    const double *t_end;      // per-particle grid end (when ts == NULL)
    double *out;              // (nt, n, 6) or NULL
    double *y_final;          // (n, 6) or NULL
    double rtol, atol;        // DOP853: exp(ln tolerance), formed on the host
    Dopr54Tol tol54;          // DOPR54: exp(ln tolerance), formed on the host
    double dt_one;            // DOPR54 first step or the estimate sentinel
    int64_t max_steps;
    uint64_t timeout_ns;      // per-thread device-time budget from its start, 0 = none
    uint8_t *status;
    int32_t *err_code;
    uint32_t *n_accepted;
    uint32_t *n_rejected;
    unsigned long long *cursor;  // persistent schedule queue position (workspace)
    const uint32_t *order;       // ordered schedule: queue position -> particle, or NULL
    double *tape;                // DOP853 step tape (t_old, h, y_old[6]) per accepted step, or NULL
    int64_t tape_steps;          // tape rows per particle
    int32_t nsegs;               // batched launch: requests in segs[], 0 = single request
    int32_t arbitrary_times;     // DOPR54: intervals end at ts[i + 1]
    int32_t tape_stride;         // step tape layout (see drift_launch.tape_stride)
    int32_t sparse_output;       // every grid has <= SPARSE_OUTPUT_NT times (see Dop853Lane::step)
    // Streamed copy-out (host path): particle p, once finished, counts itself
    // in chunk_done[p / chunk_len]; NULL = no counting.
    unsigned *chunk_done;
    int64_t chunk_len;
    drift_potential potential;
    BulgeTable bulge;            // Bovy (or a force model with Bovy parts): incomplete gamma table
    drift_force_model model;     // potential.kind == DRIFT_POT_MODEL: the summed force
    Segment segs[MAX_BATCH];  // batched launch: the request table (kernel parameter space)
};

// Fill the bulge table for exponent s (host, extended precision).
void fill_bulge_table(double s, BulgeTable *t);

// Per-precision launchers (one translation unit each).
cudaError_t launch_exact(const KernelArgs &a, int method, int grid, int block,
                         cudaStream_t stream);
cudaError_t launch_fma(const KernelArgs &a, int method, int grid, int block,
                       cudaStream_t stream);
cudaError_t occupancy_exact(int method, int kind, int block, bool tape, int *blocks_per_sm);
int max_threads_exact();
int max_threads_fma();
// Longest-first queue for the ordered schedule: fills order[0..n) with the
// particles in decreasing estimated cost.  `counts` holds 256 uint32 and
// `keys` n bytes of scratch.
cudaError_t build_order(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                        uint32_t *order, int sm_count, cudaStream_t stream);
// Longest-first queue for a streamed launch whose particles are copied out
// chunk by chunk: particles too long to finish within one chunk's share of
// the launch go first (longest first), then chunk 0's particles longest
// first, then chunk 1's, and so on, so that the chunks complete in order.
// Scratch: counts 256 + split 1 + chunk_counts (nchunks + 1) * 256 uint32,
// keys n bytes.  `lanes` is the launch's resident thread count.
cudaError_t build_order_chunked(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                                unsigned *split, unsigned *chunk_counts, uint32_t *order, int64_t chunk_len,
                                int nchunks, int64_t lanes, int sm_count, cudaStream_t stream);
// Scratch bytes build_order_chunked needs beside the queue (counts, split
// and chunk counts, 256-byte aligned).
inline size_t chunked_order_scratch(int nchunks)
{
    return ((256 + 1 + (size_t)(nchunks + 1) * 256) * sizeof(unsigned) + 255) / 256 * 256;
}
cudaError_t force_exact(const drift_potential &p, int64_t n, const double *xyz, double *acc,
                        const BulgeTable &bt, int grid, cudaStream_t stream);
cudaError_t force_fma(const drift_potential &p, int64_t n, const double *xyz, double *acc,
                      const BulgeTable &bt, int grid, cudaStream_t stream);
// Force model at time t (exact unit).
cudaError_t model_force_exact(const drift_force_model &m, const BulgeTable &bt, double t, int64_t n,
                              const double *xyz, double *acc, int grid, cudaStream_t stream);
// Quintic Hermite origin table of n_sources sources from their trajectory
// (nt, n_sources, 6) on the uniform grid t0 + k dt, accelerations from the
// sources' own force model (exact unit).
cudaError_t origin_table_exact(const drift_force_model &source_model, const BulgeTable &bt,
                               int64_t n_sources, int64_t nt, double t0, double dt,
                               const double *trajectory, double *origins, cudaStream_t stream);
cudaError_t occupancy_fma(int method, int kind, int block, bool tape, int *blocks_per_sm);

}  // namespace drift
