/*
 * drift_oracle.h -- CPU oracle for the batched Dormand-Prince test-particle path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * CPU integrators (lbparticles/astrodrift `src/integrators/galpy/dopr54.rs`
 * and `src/integrators/galpy/dop853.rs`, themselves ports of galpy v1.11.2
 * `bovy_rk.c` / `leung_dop853.c`).  It keeps their operation order and calls
 * glibc libm for every transcendental, so that it reproduces the reference's
 * bits.  Only the test-suite, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product library never links it.
 *
 * Pinning: `tests/test_oracle.py` checks the DOPR54 golden tail recorded in
 * the reference (`tests/galpy_integrator_tests.rs:35-42`) bit for bit.
 */
#ifndef DRIFT_ORACLE_H
#define DRIFT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Potential kinds.  KEPLER is galpy's cylindrical point-mass force, the one
 * the reference integrators actually evaluate (dopr54.rs:118-131,
 * dop853.rs:33-59).  PLUMMER follows shared/src/potential.rs:254-261.  BOVY is
 * bulge + Miyamoto-Nagai disk + NFW halo summed in that order
 * (shared/src/potential.rs:117-124), with the disk and halo formulas of
 * shared/src/potential.rs:138-175 and a power-law bulge with exponential
 * cutoff whose enclosed-mass force replaces the reference's table stub.
 * KEPLER_CARTESIAN is KeplerPotential::force (shared/src/potential.rs:229-238),
 * the force behind the reference's earlier DOPR54 golden tail. */
enum {
    ORACLE_POT_KEPLER = 0,
    ORACLE_POT_PLUMMER = 1,
    ORACLE_POT_BOVY = 2,
    ORACLE_POT_KEPLER_CARTESIAN = 3,
    ORACLE_POT_MODEL = 4    /* the sum described by oracle_potential.model */
};

enum { ORACLE_DOPR54 = 0, ORACLE_DOP853 = 1 };

enum {
    ORACLE_OK = 0,
    ORACLE_MAX_STEPS = 2
};

typedef struct {
    int32_t kind;
    int32_t pad_;
    double amp;          /* Kepler / Plummer mass (G = 1)               */
    double b;            /* Plummer scale radius                        */
    double mn_amp, mn_a, mn_b;
    double nfw_amp, nfw_a;
    double bulge_alpha;  /* density slope                               */
    double bulge_rc;     /* cutoff radius                               */
    double bulge_k;      /* F_r = -bulge_k * gamma(s, r^2/rc^2) / r^2   */
    double bulge_gamma_s;/* complete Gamma(s), s = 1.5 - alpha/2        */
    const struct oracle_model *model; /* ORACLE_POT_MODEL only                */
} oracle_potential;

/* A stage's summed force: stationary potentials, then potentials attached to
 * moving source particles (Kepler, Cartesian form, or Plummer), each placed at
 * its quintic Hermite origin (see oracle_origin_table).  Mirrors the device's
 * drift_force_model and its evaluation order. */
typedef struct {
    int32_t kind;         /* ORACLE_POT_KEPLER_CARTESIAN or ORACLE_POT_PLUMMER */
    int32_t pad_;
    double amp, b;
    int64_t first, count;
} oracle_source_group;

typedef struct oracle_model {
    int32_t n_static, n_groups;
    oracle_potential statics[11];
    oracle_source_group groups[11];
    int64_t n_sources, n_segments;
    double t0, dt;
    const double *origins;  /* (n_segments, n_sources, 18) */
} oracle_model;

/* Force at time t (stationary kinds ignore t). */
void oracle_force_t(const oracle_potential *p, double t, double x, double y, double z,
                    double *ax, double *ay, double *az);

/* Quintic Hermite origin table of n_sources sources from their trajectory
 * (nt, n_sources, 6) at the times t0 + k dt; accelerations from `source_pot`
 * (the force the sources were integrated in).  Writes (nt-1, n_sources, 18). */
void oracle_origin_table(const oracle_potential *source_pot, int64_t n_sources, int64_t nt, double t0,
                         double dt, const double *trajectory, double *origins);

typedef struct {
    int64_t accepted;    /* steps that advanced the solution            */
    int64_t rejected;    /* steps whose error estimate was refused      */
    int64_t rhs;         /* right-hand-side (force) evaluations         */
} oracle_stats;

/* Lower incomplete gamma function gamma(s, x), series / continued fraction
 * (Numerical Recipes, 3rd ed., section 6.2). */
double oracle_lower_gamma(double s, double x, double gamma_s);

/* Fill the bulge constants of a Bovy potential from its physical parameters:
 * density slope alpha, cutoff radius rc, and the radial force at r = 1. */
void oracle_bovy_setup(oracle_potential *p, double alpha, double rc, double force_at_1,
                       double mn_amp, double mn_a, double mn_b, double nfw_amp, double nfw_a);

void oracle_force(const oracle_potential *p, double x, double y, double z,
                  double *ax, double *ay, double *az);

/* One particle.  `t` holds the nt output times, `result` receives nt*6
 * values.  Tolerances are natural logarithms, as in the reference.  max_steps
 * <= 0 means unlimited (the reference's behaviour).  Returns an ORACLE_*
 * status; `err` receives galpy's DOPR54 error code (odd on step underflow). */
int oracle_dopr54(const oracle_potential *p, const double yo[6], int nt, double dt_one,
                  const double *t, double rtol_ln, double atol_ln, int64_t max_steps,
                  double *result, int *err, oracle_stats *stats);

int oracle_dop853(const oracle_potential *p, const double y0[6], int nt, const double *t,
                  double rtol_ln, double atol_ln, int64_t max_steps, double *result,
                  oracle_stats *stats);

/* oracle_dop853 that also records its accepted steps: row j of `tape`
 * (8 doubles) is (t_old, h, y_old[6]) of accepted step j, for the first
 * tape_steps accepted steps (stats->accepted counts all of them).  The same
 * record the device integrator writes for the adjoint pass. */
int oracle_dop853_tape(const oracle_potential *p, const double y0[6], int nt, const double *t,
                       double rtol_ln, double atol_ln, int64_t max_steps, double *result,
                       oracle_stats *stats, double *tape, int64_t tape_steps);

/* Batch driver: restates src/dispatch/cpu.rs:53-89 (per-particle loop and
 * time-major scatter into (nt, n, 6)).  Either `ts` (shared grid of nt times)
 * or `t_end` (per-particle end times on the grid t0..t_end[i] with nt points,
 * sampled as shared/src/config.rs:57-66) is given.  Uses `threads` OpenMP
 * threads.  Per-particle outputs may be NULL.  Returns the number of
 * particles whose status is not ORACLE_OK.  arbitrary_times (DOPR54): each
 * output interval ends exactly at ts[i + 1] instead of spanning ts[1] - ts[0]
 * from the previous end (the device's drift_launch.arbitrary_times). */
int64_t oracle_integrate_batch(int method, const oracle_potential *p, int64_t n,
                               const double *y0, int nt, const double *ts, double t0,
                               const double *t_end, double rtol_ln, double atol_ln,
                               double dt_one, int64_t max_steps, double *out,
                               int32_t *status, int32_t *err, int64_t *accepted,
                               int64_t *rejected, int64_t *rhs, int threads,
                               int arbitrary_times);

/* OutputGrid::sample (shared/src/config.rs:57-66). */
double oracle_grid_sample(double start, double end, int64_t steps, int64_t index);

#ifdef __cplusplus
}
#endif

#endif
