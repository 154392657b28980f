/*
 * drift_b200.h -- C ABI of the B200 batched Dormand-Prince test-particle integrator.
 *
 * This is the host->device boundary of the lbparticles/astrodrift ("drift")
 * integration path.  In the reference that boundary is the per-backend
 *   backend::launch(kernel, input_state, times, output_state)
 * (src/dispatch/gpu/cuda_oxide.rs:9-86, src/dispatch/gpu/rust_cuda.rs:10-91)
 * calling the device kernels
 *   galpy_dopr54(state0, times, state_out, n, nt, rtol, atol, dt_one_init)
 *   galpy_dop853(state0, times, state_out, n, nt, rtol, atol)
 * (kernels/src/lib.rs:143-173 and :188-216).  Every entry point below uses
 * plain pointers and sizes only.  Tolerances are natural logarithms, exactly
 * as the reference kernels receive them (src/integrators/galpy/mod.rs:19-24).
 *
 * Layouts: initial states are (n, 6) row-major [x, y, z, vx, vy, vz];
 * trajectories are time-major (nt, n, 6), as write_time_major_state writes
 * them (kernels/src/lib.rs:18-33).
 *
 * Threading: calls are thread-safe; device work is ordered on the stream the
 * caller passes (NULL = the legacy default stream).
 */
#ifndef DRIFT_B200_H
#define DRIFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DRIFT_ABI_VERSION 5

/* Sentinel that asks DOPR54 for galpy's RK4 initial-step estimate
 * (src/integrators/galpy/mod.rs:8). */
#define DRIFT_INITIAL_STEP_SENTINEL (-9999.99)

typedef enum {
    DRIFT_DOPR54 = 0, /* galpy bovy_rk.c DOPR54 (src/integrators/galpy/dopr54.rs) */
    DRIFT_DOP853 = 1  /* galpy leung_dop853.c DOP853 (src/integrators/galpy/dop853.rs) */
} drift_method;

typedef enum {
    /* galpy's cylindrical point-mass force, the force both reference
     * integrators evaluate (src/integrators/galpy/dopr54.rs:75-88). */
    DRIFT_POT_KEPLER = 0,
    /* shared/src/potential.rs:241-262 */
    DRIFT_POT_PLUMMER = 1,
    /* bulge + Miyamoto-Nagai disk + NFW halo (shared/src/potential.rs:87-176),
     * with a power-law-with-cutoff bulge */
    DRIFT_POT_BOVY = 2,
    /* KeplerPotential::force, Cartesian (shared/src/potential.rs:217-239) */
    DRIFT_POT_KEPLER_CARTESIAN = 3,
    /* The sum described by drift_launch.force_model: stationary potentials
     * plus potentials attached to moving particle groups. */
    DRIFT_POT_MODEL = 4
} drift_potential_kind;

typedef enum {
    /* No multiply-add contraction: the stage arithmetic rounds exactly like
     * the reference's Rust code (which never contracts). */
    DRIFT_PRECISION_EXACT = 0,
    /* Multiply-adds fused: fewer FP64 instructions, results differ from the
     * reference at the last-bit level. */
    DRIFT_PRECISION_FMA = 1
} drift_precision;

typedef enum {
    /* One particle per thread for the life of the launch. */
    DRIFT_SCHEDULE_PLAIN = 0,
    /* Persistent grid; a thread that finishes its particle takes the next one
     * from a device-wide cursor (needs workspace). */
    DRIFT_SCHEDULE_PERSISTENT = 1,
    /* Persistent grid fed longest-first: each particle's cost is estimated
     * from its time span and dynamical frequency at t0, and particles are
     * claimed in decreasing cost (workspace grows by 5 bytes per particle). */
    DRIFT_SCHEDULE_ORDERED = 2
} drift_schedule;

/* Return codes of every entry point. */
typedef enum {
    DRIFT_SUCCESS = 0,
    DRIFT_ERROR_INVALID_ARGUMENT = 1,
    DRIFT_ERROR_CUDA = 2,
    DRIFT_ERROR_WORKSPACE = 3,
    DRIFT_ERROR_NO_DEVICE = 4,
    DRIFT_ERROR_OUT_OF_MEMORY = 5,
    DRIFT_ERROR_TIMEOUT = 6,
    DRIFT_ERROR_CANCELLED = 7
} drift_result;

/* Per-particle status codes written to drift_launch.status. */
typedef enum {
    DRIFT_PARTICLE_OK = 0,
    /* DOPR54 hit galpy's minimum step (init/10^4) or a NaN step and forced an
     * accept; galpy's error code is odd (src/integrators/galpy/dopr54.rs:407-418). */
    DRIFT_PARTICLE_MIN_STEP = 1,
    /* The max_steps cap ended the integration (the reference has no cap). */
    DRIFT_PARTICLE_MAX_STEPS = 2,
    /* DOP853's error estimate stayed non-finite for 64 consecutive attempts. */
    DRIFT_PARTICLE_NONFINITE = 3,
    /* The launch deadline passed before this particle finished. */
    DRIFT_PARTICLE_TIMEOUT = 4,
    /* The step tape (drift_launch.tape) was full before the particle finished. */
    DRIFT_PARTICLE_TAPE_FULL = 5
} drift_particle_status;

/* Potential descriptor.  Fields a kind does not use are ignored. */
typedef struct {
    int32_t kind;          /* drift_potential_kind */
    int32_t reserved;
    double amp;            /* Kepler / Plummer mass (G = 1) */
    double b;              /* Plummer radius */
    double mn_amp, mn_a, mn_b;   /* Miyamoto-Nagai disk */
    double nfw_amp, nfw_a;       /* NFW halo */
    double bulge_alpha;    /* bulge density slope, rho ~ r^-alpha exp(-(r/rc)^2) */
    double bulge_rc;       /* bulge cutoff radius */
    double bulge_k;        /* F_r = -bulge_k gamma(s, r^2/rc^2) / r^2, s = 1.5 - alpha/2 */
    double bulge_gamma_s;  /* complete Gamma(s) */
} drift_potential;

/* ---- force models: a stage's force from the container graph ------------
 * A stage's particles feel the sum of every potential their container
 * requires (src/tree/mod.rs:89-110): stationary backgrounds, and potentials
 * attached to particle groups integrated in earlier stages, which move along
 * those groups' trajectories (the reference's CustomKepler / CustomPlummer
 * recipes and CustomOrigin, shared/src/model.rs:183-234,
 * shared/src/potential.rs:264-356).  A moving source particle's position
 * between two output times is the quintic Hermite interpolant of its
 * position, velocity and acceleration at both ends (drift_origin_table). */

/* Largest number of summed stationary potentials, and of source groups
 * (shared/src/lib.rs:21: at most 11 model components). */
#define DRIFT_MAX_COMPONENTS 11

/* A particle group whose particles each carry a point-mass (Kepler,
 * Cartesian form) or Plummer potential. */
typedef struct {
    int32_t kind;          /* DRIFT_POT_KEPLER_CARTESIAN or DRIFT_POT_PLUMMER */
    int32_t reserved;
    double amp;            /* mass of each source particle */
    double b;              /* Plummer radius */
    int64_t first;         /* this group's sources are origins [first, first + count) */
    int64_t count;
} drift_source_group;

typedef struct {
    int32_t n_static;      /* stationary potentials, summed in order */
    int32_t n_groups;      /* moving source groups, summed after them in order */
    drift_potential statics[DRIFT_MAX_COMPONENTS];   /* kinds 0..3; Bovy parts share alpha */
    drift_source_group groups[DRIFT_MAX_COMPONENTS];
    int64_t n_sources;     /* all source particles */
    int64_t n_segments;    /* origin table: segment k covers [t0 + k dt, t0 + (k+1) dt] */
    double t0, dt;
    const double *origins; /* (n_segments, n_sources, 18): per axis the 6 coefficients of
                            * x(s) = c0 + s (c1 + s (c2 + s (c3 + s (c4 + s c5)))),
                            * s = (t - t0)/dt - k; device pointer for device entry points,
                            * host pointer for drift_integrate_host.  Times outside
                            * [t0, t0 + n_segments dt] use the nearest segment. */
} drift_force_model;

/* One integration request.  Pointers are DEVICE pointers for drift_integrate
 * and HOST pointers for drift_integrate_host. */
typedef struct {
    int32_t method;        /* drift_method */
    int32_t precision;     /* drift_precision */
    int32_t schedule;      /* drift_schedule */
    int32_t block_size;    /* threads per block; 0 = library default */
    drift_potential potential;
    int64_t n;             /* particles, >= 1 */
    const double *y0;      /* (n, 6) initial states */
    int64_t nt;            /* output times per particle, >= 2 */
    const double *ts;      /* (nt) shared output grid, or NULL ... */
    double t0;             /* ... then particle i uses the nt-point uniform grid */
    const double *t_end;   /*     t0 .. t_end[i] (shared/src/config.rs:57-66) */
    double *out;           /* (nt, n, 6) trajectories, or NULL */
    double *y_final;       /* (n, 6) state at the last output time, or NULL */
    double rtol_ln;        /* ln(rtol) */
    double atol_ln;        /* ln(atol) */
    double dt_one;         /* DOPR54 first step; DRIFT_INITIAL_STEP_SENTINEL = estimate */
    int64_t max_steps;     /* step attempts per particle before MAX_STEPS; <= 0 = 10^8 */
    double timeout_s;      /* device-time budget of the launch; <= 0 = none */
    uint8_t *status;       /* (n) drift_particle_status, or NULL */
    int32_t *err_code;     /* (n) galpy DOPR54 error code, or NULL */
    uint32_t *n_accepted;  /* (n) accepted steps, or NULL */
    uint32_t *n_rejected;  /* (n) rejected steps, or NULL */
    void *workspace;       /* device scratch for the persistent and ordered schedules */
    size_t workspace_bytes;
    /* DOP853 step tape for drift_integrate_adjoint, or NULL (device entry
     * points only; not with batched launches).  tape_steps bounds the
     * accepted steps of one particle; the layout follows tape_stride below
     * and takes drift_tape_doubles(tape_steps, tape_stride) doubles per
     * particle. */
    double *tape;
    int64_t tape_steps;
    /* With potential.kind == DRIFT_POT_MODEL: the summed force (see
     * drift_force_model); otherwise ignored. */
    const drift_force_model *force_model;
    /* DOPR54 only: 0 = every output interval spans ts[1] - ts[0] from where
     * the previous one ended (galpy's uniform-grid semantics, the reference's
     * behaviour); 1 = interval i ends exactly at ts[i + 1], so the shared grid
     * may hold arbitrary strictly monotone times.  DOP853's dense output
     * handles arbitrary times either way. */
    int32_t arbitrary_times;
    /* Step tape layout.  <= 1: every accepted step j of particle i is a row
     * of 8 doubles (t_old, h, y_old[6]) at tape[(i * tape_steps + j) * 8].
     * m in 2..DRIFT_MAX_TAPE_STRIDE: checkpoints -- particle i's block starts
     * at tape + i * drift_tape_doubles(tape_steps, m); step j = c m is a row
     * (t_old, h, y_old[6]) at block + c * 8, and every step's h sits at
     * block + ceil(tape_steps / m) * 8 + j.  The adjoint recomputes the
     * m - 1 states between checkpoints: about 8 + 64 / m bytes per step
     * instead of 64, for one extra forward step per step. */
    int32_t tape_stride;
    /* Layout of y0.  DRIFT_Y0_ROWS (0, default): (n, 6) rows
     * [x, y, z, vx, vy, vz], the reference's InputState (src/state/mod.rs:7-25).
     * DRIFT_Y0_COLUMNS: six columns of y0_stride doubles, component c of
     * particle i at y0[c * y0_stride + i] (y0_stride 0 means n): one tensor
     * per coordinate, as column-major hosts hold them.  The request server
     * takes rows only. */
    int32_t y0_layout;
    int32_t reserved;
    int64_t y0_stride;
} drift_launch;

enum { DRIFT_Y0_ROWS = 0, DRIFT_Y0_COLUMNS = 1 };

#define DRIFT_MAX_TAPE_STRIDE 16

/* Doubles of step tape per particle for a tape_steps / tape_stride pair. */
static inline int64_t drift_tape_doubles(int64_t tape_steps, int32_t tape_stride)
{
    if (tape_stride <= 1) return tape_steps * 8;
    return (tape_steps + tape_stride - 1) / tape_stride * 8 + ((tape_steps + 1) & ~(int64_t)1);
}

/* Library / device information. */
int drift_abi_version(void);
const char *drift_result_string(int code);
/* Message of the last failing call on this thread ("" if none). */
const char *drift_last_error(void);

/* Page-locked host memory for drift_integrate_host buffers: with pinned
 * trajectory buffers the copy-out of one particle chunk overlaps the
 * integration of the next. */
int drift_host_alloc(size_t bytes, void **ptr);
int drift_host_free(void *ptr);

/* Fill a drift_potential for the Bovy composite from physical parameters
 * (bulge slope alpha, cutoff rc, bulge radial force at r = 1; disk amp, a, b;
 * halo amp, a).  Host-only arithmetic. */
int drift_potential_bovy(drift_potential *p, double alpha, double rc, double bulge_force_at_1,
                         double mn_amp, double mn_a, double mn_b, double nfw_amp,
                         double nfw_a);

/* Bytes of device workspace drift_integrate needs for this request. */
int drift_query_workspace(const drift_launch *launch, size_t *bytes);

/* Integrate on the device; all pointers are device pointers.  Replaces the
 * launch inside backend::launch (src/dispatch/gpu/cuda_oxide.rs:40-73). */
int drift_integrate(const drift_launch *launch, void *stream);

/* Integrate from host buffers: copies in, launches, copies results out and
 * synchronises.  Replaces the whole backend::launch
 * (src/dispatch/gpu/cuda_oxide.rs:9-86), with a library-owned persistent
 * context instead of one context per call.  Large requests are processed in
 * particle chunks whose copies overlap the integration of other chunks. */
int drift_integrate_host(const drift_launch *launch);

/* Explicit host-path contexts.  drift_integrate_host uses one implicit
 * context per device, created on first use and kept until the process exits,
 * whose grow-only buffers can hold gigabytes after a large request.  An
 * explicit context owns its own streams and buffers:
 * drift_context_destroy frees them, and host threads with separate contexts
 * run host-path integrations on one device concurrently (calls on one
 * context are serialised).  The reference creates and drops a CUDA context
 * on every call instead (src/dispatch/gpu/cuda_oxide.rs:16-28).
 * device < 0 selects the caller's current device. */
typedef struct drift_context drift_context;
int drift_context_create(int32_t device, drift_context **context);
/* drift_integrate_host on the context's device, streams and buffers. */
int drift_context_integrate_host(drift_context *context, const drift_launch *launch);
/* Device and page-locked host bytes the context's buffers hold now. */
int drift_context_memory(drift_context *context, size_t *device_bytes, size_t *pinned_bytes);
/* Waits for the context's work and frees it; NULL is a no-op. */
int drift_context_destroy(drift_context *context);

/* Largest number of requests one drift_integrate_batch launch carries. */
#define DRIFT_MAX_BATCH 64

/* Several requests as one launch over their concatenated particles, with one
 * claim queue, so small requests share the GPU instead of each launching a
 * mostly idle grid.  Device pointers.  The requests must share method,
 * precision, schedule, block size, potential, tolerances, first step and
 * limits; each has its own particles, output grid and output buffers.  A
 * persistent or ordered batch uses requests[0].workspace, of
 * drift_query_workspace's size for one request holding all the batch's
 * particles; the ordered schedule ranks the particles of all requests
 * together (most expensive first).  No counterpart in the
 * reference, which launches one kernel per stage
 * (src/dispatch/gpu.rs:157-178). */
int drift_integrate_batch(const drift_launch *requests, int32_t count, void *stream);

/* Acceleration of the potential at n positions: xyz (n, 3) -> acc (n, 3),
 * device pointers, the same force code the integrators inline (rounded
 * without multiply-add contraction).  The reference exposes the force only
 * through its Potential trait (shared/src/potential.rs:41-44). */
int drift_force(const drift_potential *potential, int64_t n, const double *xyz, double *acc,
                void *stream);
/* The same, rounded as the chosen precision unit's integrators round
 * (drift_precision): DRIFT_PRECISION_FMA gives the contraction unit's force,
 * with its few-ulp powers. */
int drift_force_precision(const drift_potential *potential, int32_t precision, int64_t n,
                          const double *xyz, double *acc, void *stream);

/* Origin table of moving sources (no counterpart in the reference, whose
 * CustomOrigin tables are never built: shared/src/model.rs:193-199).
 * trajectory (nt, n_sources, 6): the sources' states at the uniform times
 * t0 + k dt, k = 0..nt-1, as their own stage produced them; source_model:
 * the force that stage integrated in (its accelerations at the samples
 * complete the Hermite data).  Writes origins (nt - 1, n_sources, 18).
 * Device pointers. */
int drift_origin_table(const drift_force_model *source_model, int64_t n_sources, int64_t nt,
                       double t0, double dt, const double *trajectory, double *origins,
                       void *stream);

/* drift_origin_table with host pointers (trajectory, origins, and the
 * source model's own origin table when it has moving sources); synchronous. */
int drift_origin_table_host(const drift_force_model *source_model, int64_t n_sources, int64_t nt,
                            double t0, double dt, const double *trajectory, double *origins);

/* Acceleration of a force model at time t: xyz (n, 3) -> acc (n, 3), device
 * pointers, rounded without multiply-add contraction like drift_force. */
int drift_force_model_eval(const drift_force_model *model, int64_t n, double t,
                           const double *xyz, double *acc, void *stream);

/* ---- captured launch graphs (no counterpart in the reference) ----------
 * drift_graph_create records drift_integrate(launch) on `stream` (not the
 * legacy default stream) by stream capture: the cursor reset, the ordering
 * kernels and the integration kernel, with the launch's pointers and values
 * as they are now.  drift_graph_launch replays that sequence with one call;
 * change the buffers' contents in place between replays, not the launch. */
typedef struct drift_graph drift_graph;
int drift_graph_create(const drift_launch *launch, void *stream, drift_graph **graph);
int drift_graph_launch(drift_graph *graph, void *stream);
int drift_graph_destroy(drift_graph *graph);

/* ---- launch autotuner (no counterpart in the reference) -----------------
 * Times every block size (32, 64, 96, 128) under every schedule on the first
 * `sample` particles of a device-pointer launch (0: 16384), in scratch
 * buffers of its own, and returns the fastest.  Results are cached per
 * workload class (method, precision, potential kind, grid kind, nt and n
 * rounded to powers of two); `cached` tells whether this call measured.
 * The launch's own outputs are not written. */
typedef struct {
    int32_t block_size;
    int32_t schedule;
    double seconds;        /* the winner's time on the sample */
    double candidates[12]; /* plain, persistent, ordered x block 32..128 */
    int64_t sample;
    int32_t cached;
    int32_t reserved;
} drift_tuning;
int drift_autotune(const drift_launch *launch, int64_t sample, drift_tuning *best);

/* ---- discrete adjoint (no counterpart in the reference) ----------------- */

/* Largest number of potential parameters with a gradient:
 *   Kepler (both forms): amp
 *   Plummer:             amp, b
 *   Bovy:                mn_amp, mn_a, mn_b, nfw_amp, nfw_a, bulge_k */
#define DRIFT_ADJOINT_MAX_PARAMS 6

/* Reverse pass of a taped DOP853 integration.  The trajectory `out` of a
 * drift_integrate call with a tape is a function of y0 and the potential
 * parameters through the recorded steps (the step sizes are held fixed, so
 * this is the exact derivative of the discrete map that produced `out`).
 * Given the cotangent grad_out of `out`, the kernel replays every particle's
 * steps in reverse from the tape, recomputing each step's stages, and writes
 *   grad_y0[i]     = d<grad_out, out> / d y0[i]
 *   grad_params[i] = d<grad_out[:, i], out[:, i]> / d params   (per particle;
 *                    the gradient of the whole trajectory is their sum).
 * Particles whose forward status is not DRIFT_PARTICLE_OK get NaN rows.  The
 * output grid must be monotone in the direction of integration.  Device
 * pointers. */
typedef struct {
    int32_t method;            /* DRIFT_DOP853 */
    int32_t block_size;        /* 0 = library default */
    drift_potential potential; /* as in the forward launch */
    int64_t n;
    int64_t nt;
    const double *ts;          /* grid exactly as in the forward launch */
    double t0;
    const double *t_end;
    const double *tape;        /* the forward launch's tape, tape_steps and tape_stride */
    int64_t tape_steps;
    const uint32_t *n_accepted;/* (n) from the forward launch */
    const uint8_t *status;     /* (n) from the forward launch */
    const double *grad_out;    /* (nt, n, 6) cotangent of the trajectory */
    double *grad_y0;           /* (n, 6) */
    double *grad_params;       /* (n, DRIFT_ADJOINT_MAX_PARAMS), or NULL */
    int32_t tape_stride;
    int32_t reserved;
} drift_adjoint_launch;

int drift_integrate_adjoint(const drift_adjoint_launch *adjoint, void *stream);

/* Bytes of device scratch that drift_integrate_noalloc owns (per device). */
#define DRIFT_NOALLOC_SCRATCH_BYTES 4096

/* drift_integrate for callers that cannot allocate device memory.
 *
 * No counterpart in the reference (its launch path allocates and frees
 * buffers on every call).  Some callers of this library own every byte of
 * device memory themselves and cannot call cudaMalloc: a host application
 * whose memory pool has reserved the GPU in advance, a real-time loop where
 * an allocation's implicit synchronisation would stall the pipeline, or a
 * plugin running inside another runtime that forbids allocation.  For them
 * this entry point takes the same request as drift_integrate, with device
 * pointers for every input and output, and allocates nothing: the scratch
 * the kernels need (the persistent schedule's claim cursor; for the ordered
 * schedule also its longest-first queue, 5 bytes per particle) lives in a
 * fixed DRIFT_NOALLOC_SCRATCH_BYTES array inside the library, which every
 * GPU that loads the library holds until the process exits.
 * launch->workspace is ignored.
 *
 * Limits and rules:
 *  - a request whose drift_query_workspace size exceeds
 *    DRIFT_NOALLOC_SCRATCH_BYTES is rejected with DRIFT_ERROR_WORKSPACE
 *    (plain and persistent requests always fit; ordered requests fit up to
 *    563 particles);
 *  - every call looks up the array's device address in the calling
 *    thread's current context (the device the call runs on must be
 *    current), so the address stays right after a device reset or under
 *    another context; the first call on a device also loads the library's
 *    kernels there, so make that first call before any CUDA stream capture;
 *  - every call shares the one array and clears the part that must start
 *    at zero before its launch, so calls whose kernels overlap on the GPU
 *    (different streams, or different host threads) race with each other:
 *    order them on one stream or serialise them. */
int drift_integrate_noalloc(const drift_launch *launch, void *stream);

/* ---- Request server (continuous batching) -------------------------------
 *
 * A resident server keeps a device memory pool, several streams and a
 * scheduler thread.  Submitted requests (host pointers, which must stay
 * valid until the request completes) are admitted by free device memory:
 * whenever a stream is free, the oldest pending request and every later one
 * that can share its launch (same method, precision, potential, tolerances
 * and limits) form one batched launch, and requests larger than the free
 * budget run in particle chunks.  Requests that arrive while others run start
 * as soon as a stream and memory free up; their kernels overlap the running
 * ones.  Each stream has its own worker thread, and no lock is held across
 * a CUDA call: a copy into a pageable result buffer (which returns only once
 * its kernel has finished) holds up only its own stream, never admission,
 * other streams or the submit/wait/cancel/stats calls.  Page-locked buffers
 * (drift_host_alloc) still copy faster.  Results are identical to
 * drift_integrate_host's for the same request.  No counterpart in the
 * reference (which runs one blocking call per stage). */
typedef struct drift_server drift_server;

typedef struct {
    double memory_fraction;      /* of the device's free memory at creation; default 0.5 */
    size_t memory_bytes;         /* absolute budget, overrides the fraction when > 0 */
    int32_t streams;             /* batches in flight; default 4 */
    /* Percent of the SMs (0 to 50) that large batches leave to newly
     * admitted small ones, which run on the highest-priority stream: bounds
     * how long a small request waits behind a long one, at the price of the
     * long one's speed.  Default 0 (none). */
    int32_t sm_reserve_percent;
    int64_t max_batch_particles; /* particles per launch; default 2^20 */
    /* select_device != 0: the server's pool, streams and kernels live on
     * CUDA device `device`; 0 (default): on the caller's current device. */
    int32_t select_device;
    int32_t device;
} drift_server_options;

typedef struct {
    uint64_t requests_submitted, requests_completed, requests_pending;
    uint64_t particles_completed;
    uint64_t batches_launched, pieces_launched, batches_in_flight;
    uint64_t bytes_to_device, bytes_to_host;
    uint64_t memory_budget, bytes_in_flight, peak_bytes_in_flight;
    uint64_t bytes_pending;  /* device bytes the queued, not yet admitted particles need */
    int32_t device;          /* the server's CUDA device */
    int32_t reserved;
} drift_server_stats;

int drift_server_create(const drift_server_options *options, drift_server **server);
/* Plain or persistent schedule; the request's workspace is ignored. */
int drift_server_submit(drift_server *server, const drift_launch *request, uint64_t *ticket);
/* Blocks until the request completes (timeout_s <= 0: no limit; else
 * DRIFT_ERROR_TIMEOUT).  request_result receives the request's drift_result,
 * latency_s the time from submission to completion.  Releases the ticket. */
int drift_server_wait(drift_server *server, uint64_t ticket, double timeout_s, int *request_result,
                      double *latency_s);
/* Blocks until any of `count` requests completes (timeout_s as above) and
 * releases that one ticket: *index receives its position in `tickets` (the
 * earliest completion when several have finished), request_result and
 * latency_s as drift_server_wait.  The other tickets stay valid.  A client
 * holding a fixed set of result buffers retires whichever request finishes
 * first instead of the oldest one. */
int drift_server_wait_any(drift_server *server, const uint64_t *tickets, int32_t count, double timeout_s,
                          int32_t *index, int *request_result, double *latency_s);
int drift_server_stats_get(drift_server *server, drift_server_stats *stats);
/* Cancels one request: none of its particles that are not yet on the GPU
 * will run.  Particles already admitted finish (their results are written
 * to the request's buffers), and then the request ends with result
 * DRIFT_ERROR_CANCELLED, which drift_server_wait reports; a request with
 * nothing on the GPU ends at once.  Cancelling a request that has already
 * finished changes nothing.  The ticket stays valid until waited for. */
int drift_server_cancel(drift_server *server, uint64_t ticket);
/* Cancels pending requests (their waiters receive DRIFT_ERROR_CANCELLED),
 * finishes the batches in flight and frees the server.  Waits already in
 * progress on other threads return (their request's result, or
 * DRIFT_ERROR_CANCELLED) before the server is freed; no call on the server
 * may begin once destroy has been called. */
int drift_server_destroy(drift_server *server);

/* The reference kernel signatures (kernels/src/lib.rs:143-173, 188-216):
 * galpy Kepler force, shared output grid, plain schedule, exact precision.
 * Device pointers; tolerances are natural logarithms. */
int drift_galpy_dopr54(const double *state0, const double *times, double *state_out, int64_t n,
                       int64_t nt, double rtol, double atol, double dt_one_init, void *stream);
int drift_galpy_dop853(const double *state0, const double *times, double *state_out, int64_t n,
                       int64_t nt, double rtol, double atol, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DRIFT_B200_H */
