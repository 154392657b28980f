/*
 * drift_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see drift_oracle.h).
 *
 * A plain-C restatement of the reference's CPU integrators:
 *   DOPR54: lbparticles/astrodrift src/integrators/galpy/dopr54.rs
 *           (rk4_onestep :135-208, rk4_estimate_step :210-368,
 *            dopr54_onestep :370-460, dopr54_actualstep :462-659,
 *            dopr54 :670-778)
 *   DOP853: src/integrators/galpy/dop853.rs:316-783 with the tableau of
 *           :105-264 and the helpers c_min/c_max/custom_sign of :286-299.
 * Operation order follows those files expression by expression and every
 * transcendental goes through glibc libm, so with -ffp-contract=off the
 * results are the reference's bits.  The right-hand side is generalised from
 * the hard-coded Kepler callback to a potential descriptor.
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp).
 */
#include "drift_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DIM 6

/* ------------------------------------------------------------------ */
/* Potentials                                                          */
/* ------------------------------------------------------------------ */

/* Lower incomplete gamma gamma(s, x) by the power series for x < s + 1 and by
 * the modified-Lentz continued fraction for Gamma(s, x) otherwise (Numerical
 * Recipes 3rd ed. section 6.2).  `gamma_s` is the complete Gamma(s).  The
 * device implementation runs the same recurrences with the same stopping
 * rules. */
double oracle_lower_gamma(double s, double x, double gamma_s)
{
    const double eps = 1.1102230246251565e-16; /* 2^-53 */
    const double fpmin = 1e-300;
    if (!(x > 0.0)) return 0.0;
    double prefactor = exp(s * log(x) - x);
    if (x < s + 1.0) {
        double ap = s;
        double del = 1.0 / s;
        double sum = del;
        for (int n = 0; n < 500; ++n) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * eps) break;
        }
        return sum * prefactor;
    }
    double b = x + 1.0 - s;
    double c = 1.0 / fpmin;
    double d = 1.0 / b;
    double h = d;
    for (int i = 1; i < 500; ++i) {
        double an = -i * (i - s);
        b += 2.0;
        d = an * d + b;
        if (fabs(d) < fpmin) d = fpmin;
        c = b + an / c;
        if (fabs(c) < fpmin) c = fpmin;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) < eps) break;
    }
    return gamma_s - prefactor * h;
}

/* The bulge force's incomplete gamma.  The operation counter (opcount.cpp)
 * redefines this name to tally each evaluation as one special-function call,
 * like pow, exp and log, since its loop lengths depend on the argument. */
#ifndef ORACLE_BULGE_GAMMA
#define ORACLE_BULGE_GAMMA oracle_lower_gamma
#endif

void oracle_bovy_setup(oracle_potential *p, double alpha, double rc, double force_at_1,
                       double mn_amp, double mn_a, double mn_b, double nfw_amp, double nfw_a)
{
    memset(p, 0, sizeof(*p));
    p->kind = ORACLE_POT_BOVY;
    p->bulge_alpha = alpha;
    p->bulge_rc = rc;
    double s = 1.5 - 0.5 * alpha;
    p->bulge_gamma_s = tgamma(s);
    /* F_r(1) = -bulge_k * gamma(s, 1/rc^2) / 1  ==  -force_at_1 */
    p->bulge_k = force_at_1 / oracle_lower_gamma(s, 1.0 / (rc * rc), p->bulge_gamma_s);
    p->mn_amp = mn_amp;
    p->mn_a = mn_a;
    p->mn_b = mn_b;
    p->nfw_amp = nfw_amp;
    p->nfw_a = nfw_a;
}

/* galpy's cylindrical point-mass force, dopr54.rs:75-88.  The reference has
 * the mass fixed at 1; `amp` scales it and reproduces those bits at amp = 1. */
static void kepler_galpy(double amp, double x, double y, double z, double *ax, double *ay,
                         double *az)
{
    double cylindrical_radius = sqrt(x * x + y * y);
    double sin_phi = y / cylindrical_radius;
    double cos_phi = x / cylindrical_radius;
    double radius_squared = cylindrical_radius * cylindrical_radius + z * z;
    double p = amp * pow(radius_squared, -1.5);
    double radial_force = -cylindrical_radius * p;
    double phi_torque = 0.0;
    *ax = cos_phi * radial_force - 1.0 / cylindrical_radius * sin_phi * phi_torque;
    *ay = sin_phi * radial_force + 1.0 / cylindrical_radius * cos_phi * phi_torque;
    *az = -z * p;
}

/* Cartesian point mass, KeplerPotential::force (shared/src/potential.rs:229-238). */
static void kepler_cartesian(double amp, double x, double y, double z, double *ax, double *ay,
                             double *az)
{
    double r2 = x * x + y * y + z * z;
    double r = sqrt(r2);
    double inv_r3 = 1.0 / (r2 * r);
    double ar = -amp * inv_r3;
    *ax = ar * x;
    *ay = ar * y;
    *az = ar * z;
}

/* shared/src/potential.rs:254-261 */
static void plummer(double amp, double b, double x, double y, double z, double *ax,
                    double *ay, double *az)
{
    double r2 = x * x + y * y + z * z;
    double ar = -amp * pow(r2 + (b * b), -1.5);
    *ax = ar * x;
    *ay = ar * y;
    *az = ar * z;
}

/* shared/src/potential.rs:138-151 */
static void miyamoto_nagai(double amp, double a, double b, double x, double y, double z,
                           double *ax, double *ay, double *az)
{
    double r2 = pow(x, 2.) + pow(y, 2.);
    double r = sqrt(r2);
    double z2 = pow(z, 2.);
    double b2 = pow(b, 2.);
    double sqrtz2b2 = sqrt(z2 + b2);
    double pyth = pow(a + sqrtz2b2, 2.);
    double denom = pow(pyth + r2, 3. / 2.);
    double ar = -amp * (r / denom);
    *ax = ar * (x / r);
    *ay = ar * (y / r);
    *az = -amp * (z * (a + sqrtz2b2)) / (sqrtz2b2 * denom);
}

/* shared/src/potential.rs:165-175 */
static void nfw(double amp, double a, double x, double y, double z, double *ax, double *ay,
                double *az)
{
    double r2 = pow(x, 2.) + pow(y, 2.) + pow(z, 2.);
    double r = sqrt(r2);
    double ar = -amp * (log(1. + r / a) - r / (a + r)) / r2;
    *ax = ar * (x / r);
    *ay = ar * (y / r);
    *az = ar * (z / r);
}

/* Power-law bulge with exponential cutoff, rho ~ r^-alpha exp(-(r/rc)^2).
 * Enclosed mass ~ gamma(1.5 - alpha/2, r^2/rc^2), so
 *   F = -k gamma(s, r^2/rc^2) / r^3 * (x, y, z).
 * The reference's stand-in (shared/src/potential.rs:178-215) is a broken
 * table stub; the r2 == 0 guard is kept from it. */
static void bulge(const oracle_potential *p, double x, double y, double z, double *ax,
                  double *ay, double *az)
{
    double r2 = x * x + y * y + z * z;
    if (r2 == 0.0) {
        *ax = 0.0;
        *ay = 0.0;
        *az = 0.0;
        return;
    }
    double r = sqrt(r2);
    double s = 1.5 - 0.5 * p->bulge_alpha;
    double g = ORACLE_BULGE_GAMMA(s, r2 / (p->bulge_rc * p->bulge_rc), p->bulge_gamma_s);
    double ar_over_r = -p->bulge_k * g / (r2 * r);
    *ax = ar_over_r * x;
    *ay = ar_over_r * y;
    *az = ar_over_r * z;
}

void oracle_force(const oracle_potential *p, double x, double y, double z, double *ax,
                  double *ay, double *az)
{
    switch (p->kind) {
    case ORACLE_POT_KEPLER:
        kepler_galpy(p->amp, x, y, z, ax, ay, az);
        return;
    case ORACLE_POT_PLUMMER:
        plummer(p->amp, p->b, x, y, z, ax, ay, az);
        return;
    case ORACLE_POT_BOVY: {
        /* combine_potentials!(bulge, disk, halo): ((bulge + disk) + halo),
         * shared/src/potential.rs:64-85, 117-124 */
        double bx, by, bz, dx, dy, dz, hx, hy, hz;
        bulge(p, x, y, z, &bx, &by, &bz);
        miyamoto_nagai(p->mn_amp, p->mn_a, p->mn_b, x, y, z, &dx, &dy, &dz);
        nfw(p->nfw_amp, p->nfw_a, x, y, z, &hx, &hy, &hz);
        *ax = (bx + dx) + hx;
        *ay = (by + dy) + hy;
        *az = (bz + dz) + hz;
        return;
    }
    case ORACLE_POT_KEPLER_CARTESIAN:
        kepler_cartesian(p->amp, x, y, z, ax, ay, az);
        return;
    default:
        *ax = *ay = *az = NAN;
    }
}

/* ------------------------------------------------------------------ */
/* Force models: stationary parts plus moving sources                  */
/* ------------------------------------------------------------------ */

static void hermite5(double x0, double v0, double a0, double x1, double v1, double a1, double h,
                     double *c)
{
    const double hh = h * h;
    const double d = x1 - x0;
    c[0] = x0;
    c[1] = h * v0;
    c[2] = 0.5 * (hh * a0);
    c[3] = 10.0 * d - h * (6.0 * v0 + 4.0 * v1) - hh * (1.5 * a0 - 0.5 * a1);
    c[4] = -15.0 * d + h * (8.0 * v0 + 7.0 * v1) + hh * (1.5 * a0 - a1);
    c[5] = 6.0 * d - 3.0 * h * (v0 + v1) - hh * (0.5 * a0 - 0.5 * a1);
}

static double quintic(const double *c, double s)
{
    return c[0] + s * (c[1] + s * (c[2] + s * (c[3] + s * (c[4] + s * c[5]))));
}

static void model_force(const oracle_model *m, double t, double x, double y, double z, double *ax,
                        double *ay, double *az)
{
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 0; i < m->n_static; i++) {
        double fx, fy, fz;
        oracle_force(&m->statics[i], x, y, z, &fx, &fy, &fz);
        sx = sx + fx;
        sy = sy + fy;
        sz = sz + fz;
    }
    if (m->n_groups > 0) {
        const double u = (t - m->t0) / m->dt;
        double kf = floor(u);
        kf = fmin(fmax(kf, 0.0), (double)(m->n_segments - 1));
        const double s = u - kf;
        const double *row = m->origins + (int64_t)kf * m->n_sources * 18;
        for (int g = 0; g < m->n_groups; g++) {
            const oracle_source_group *G = &m->groups[g];
            for (int64_t j = G->first; j < G->first + G->count; j++) {
                const double *c = row + j * 18;
                const double dx = x - quintic(c, s);
                const double dy = y - quintic(c + 6, s);
                const double dz = z - quintic(c + 12, s);
                double fx, fy, fz;
                if (G->kind == ORACLE_POT_PLUMMER)
                    plummer(G->amp, G->b, dx, dy, dz, &fx, &fy, &fz);
                else
                    kepler_cartesian(G->amp, dx, dy, dz, &fx, &fy, &fz);
                sx = sx + fx;
                sy = sy + fy;
                sz = sz + fz;
            }
        }
    }
    *ax = sx;
    *ay = sy;
    *az = sz;
}

void oracle_force_t(const oracle_potential *p, double t, double x, double y, double z, double *ax,
                    double *ay, double *az)
{
    if (p->kind == ORACLE_POT_MODEL)
        model_force(p->model, t, x, y, z, ax, ay, az);
    else
        oracle_force(p, x, y, z, ax, ay, az);
}

void oracle_origin_table(const oracle_potential *source_pot, int64_t n_sources, int64_t nt, double t0,
                         double dt, const double *trajectory, double *origins)
{
    for (int64_t k = 0; k + 1 < nt; k++)
        for (int64_t j = 0; j < n_sources; j++) {
            const double *q0 = trajectory + (k * n_sources + j) * 6;
            const double *q1 = trajectory + ((k + 1) * n_sources + j) * 6;
            const double ta = t0 + dt * (double)k;
            const double tb = t0 + dt * (double)(k + 1);
            double a0[3], a1[3];
            oracle_force_t(source_pot, ta, q0[0], q0[1], q0[2], &a0[0], &a0[1], &a0[2]);
            oracle_force_t(source_pot, tb, q1[0], q1[1], q1[2], &a1[0], &a1[1], &a1[2]);
            double *c = origins + (k * n_sources + j) * 18;
            for (int axis = 0; axis < 3; axis++)
                hermite5(q0[axis], q0[3 + axis], a0[axis], q1[axis], q1[3 + axis], a1[axis], dt,
                         c + 6 * axis);
        }
}

/* kepler_rhs, dopr54.rs:59-73: a = (v, F(t, x)). */
static void rhs(const oracle_potential *p, double t, const double *q, double *a,
                oracle_stats *st)
{
    double ax, ay, az;
    oracle_force_t(p, t, q[0], q[1], q[2], &ax, &ay, &az);
    a[0] = q[3];
    a[1] = q[4];
    a[2] = q[5];
    a[3] = ax;
    a[4] = ay;
    a[5] = az;
    st->rhs++;
}

/* ------------------------------------------------------------------ */
/* DOPR54 (galpy bovy_rk.c as ported in dopr54.rs)                     */
/* ------------------------------------------------------------------ */

#define MAX_STEPCHANGE_POWERTWO 3.0
#define MIN_STEPCHANGE_POWERTWO (-3.0)
#define MAX_STEPREDUCE 10000.0
#define MAX_DT_REDUCE 10000.0

/* dopr54.rs:135-208 */
static void rk4_onestep(const oracle_potential *p, const double *yn, double *yn1, double tn,
                        double dt, double *ynk, double *a, oracle_stats *st)
{
    int i;
    rhs(p, tn, yn, a, st);
    for (i = 0; i < DIM; i++) yn1[i] += dt * a[i] / 6.0;
    for (i = 0; i < DIM; i++) ynk[i] = yn[i] + dt * a[i] / 2.0;
    rhs(p, tn + dt / 2.0, ynk, a, st);
    for (i = 0; i < DIM; i++) yn1[i] += dt * a[i] / 3.0;
    for (i = 0; i < DIM; i++) ynk[i] = yn[i] + dt * a[i] / 2.0;
    rhs(p, tn + dt / 2.0, ynk, a, st);
    for (i = 0; i < DIM; i++) yn1[i] += dt * a[i] / 3.0;
    for (i = 0; i < DIM; i++) ynk[i] = yn[i] + dt * a[i];
    rhs(p, tn + dt, ynk, a, st);
    for (i = 0; i < DIM; i++) yn1[i] += dt * a[i] / 6.0;
}

/* dopr54.rs:210-368 */
static double rk4_estimate_step(const oracle_potential *p, const double *yo, double dt,
                                const double *t, double rtol, double atol, oracle_stats *st)
{
    double err = 2.0;
    double to = t[0];
    double init_dt = dt;
    double yn[DIM], y1[DIM], y21[DIM], y2[DIM], ynk[DIM], a[DIM], scale[DIM];
    int i;

    double max_val = log(fabs(yo[0]));
    for (i = 1; i < DIM; i++) {
        double v = log(fabs(yo[i]));
        if (v > max_val) max_val = v;
    }
    double c = fmax(atol, rtol + max_val);
    double s = log(exp(atol - c) + exp(rtol + max_val - c)) + c;
    for (i = 0; i < DIM; i++) scale[i] = s;

    while (err > 1.0) {
        for (i = 0; i < DIM; i++) yn[i] = yo[i];
        for (i = 0; i < DIM; i++) y1[i] = yo[i];
        for (i = 0; i < DIM; i++) y21[i] = yo[i];
        rk4_onestep(p, yn, y1, to, dt, ynk, a, st);
        rk4_onestep(p, yn, y21, to, dt / 2.0, ynk, a, st);
        for (i = 0; i < DIM; i++) y2[i] = y21[i];
        rk4_onestep(p, y21, y2, to + dt / 2.0, dt / 2.0, ynk, a, st);
        err = 0.0;
        for (i = 0; i < DIM; i++) {
            double diff = y1[i] - y2[i];
            double term = exp(2.0 * log(fabs(diff)) - 2.0 * scale[i]);
            err += term;
        }
        err = sqrt(err / (double)DIM);
        double factor = ceil(pow(err, 1.0 / 5.0));
        if (factor > 1.0 && init_dt / dt * factor < MAX_DT_REDUCE)
            dt /= factor;
        else
            break;
    }
    return dt;
}

/* dopr54.rs:462-659.  Returns the next step size; *advanced tells whether the
 * step was taken. */
static double dopr54_actualstep(const oracle_potential *p, double *yo, double dt, double *to,
                                double rtol, double atol, double *a1, double *a, double *k1,
                                double *k2, double *k3, double *k4, double *k5, double *k6,
                                double *yn1, double *yerr, double *ynk, int accept,
                                int *advanced, oracle_stats *st)
{
    const double C2 = 0.2;
    const double C3 = 0.3;
    const double C4 = 0.8;
    const double C5 = 8.0 / 9.0;
    const double A21 = 0.2;
    const double A31 = 3.0 / 40.0;
    const double A41 = 44.0 / 45.0;
    const double A51 = 19372.0 / 6561.0;
    const double A61 = 9017.0 / 3168.0;
    const double A71 = 35.0 / 384.0;
    const double A32 = 9.0 / 40.0;
    const double A42 = -56.0 / 15.0;
    const double A52 = -25360.0 / 2187.0;
    const double A62 = -355.0 / 33.0;
    const double A43 = 32.0 / 9.0;
    const double A53 = 64448.0 / 6561.0;
    const double A63 = 46732.0 / 5247.0;
    const double A73 = 500.0 / 1113.0;
    const double A54 = -212.0 / 729.0;
    const double A64 = 49.0 / 176.0;
    const double A74 = 125.0 / 192.0;
    const double A65 = -5103.0 / 18656.0;
    const double A75 = -2187.0 / 6784.0;
    const double A76 = 11.0 / 84.0;
    const double B1 = 35.0 / 384.0;
    const double B3 = 500.0 / 1113.0;
    const double B4 = 125.0 / 192.0;
    const double B5 = -2187.0 / 6784.0;
    const double B6 = 11.0 / 84.0;
    const double BE1 = B1 - 5179.0 / 57600.0;
    const double BE3 = B3 - 7571.0 / 16695.0;
    const double BE4 = B4 - 393.0 / 640.0;
    const double BE5 = B5 + 92097.0 / 339200.0;
    const double BE6 = B6 - 187.0 / 2100.0;
    const double BE7 = -1.0 / 40.0;
    int i;

    for (i = 0; i < DIM; i++) yn1[i] = yo[i];
    for (i = 0; i < DIM; i++) a[i] = a1[i];
    for (i = 0; i < DIM; i++) {
        k1[i] = dt * a[i];
        yn1[i] += B1 * k1[i];
        yerr[i] = BE1 * k1[i];
        ynk[i] = yo[i] + A21 * k1[i];
    }
    rhs(p, *to + C2 * dt, ynk, a, st);
    for (i = 0; i < DIM; i++) {
        k2[i] = dt * a[i];
        ynk[i] = yo[i] + A31 * k1[i] + A32 * k2[i];
    }
    rhs(p, *to + C3 * dt, ynk, a, st);
    for (i = 0; i < DIM; i++) {
        k3[i] = dt * a[i];
        yn1[i] += B3 * k3[i];
        yerr[i] += BE3 * k3[i];
        ynk[i] = yo[i] + A41 * k1[i] + A42 * k2[i] + A43 * k3[i];
    }
    rhs(p, *to + C4 * dt, ynk, a, st);
    for (i = 0; i < DIM; i++) {
        k4[i] = dt * a[i];
        yn1[i] += B4 * k4[i];
        yerr[i] += BE4 * k4[i];
        ynk[i] = yo[i] + A51 * k1[i] + A52 * k2[i] + A53 * k3[i] + A54 * k4[i];
    }
    rhs(p, *to + C5 * dt, ynk, a, st);
    for (i = 0; i < DIM; i++) {
        k5[i] = dt * a[i];
        yn1[i] += B5 * k5[i];
        yerr[i] += BE5 * k5[i];
        ynk[i] = yo[i] + A61 * k1[i] + A62 * k2[i] + A63 * k3[i] + A64 * k4[i] + A65 * k5[i];
    }
    rhs(p, *to + dt, ynk, a, st);
    for (i = 0; i < DIM; i++) {
        k6[i] = dt * a[i];
        yn1[i] += B6 * k6[i];
        yerr[i] += BE6 * k6[i];
        ynk[i] = yo[i] + A71 * k1[i] + A73 * k3[i] + A74 * k4[i] + A75 * k5[i] + A76 * k6[i];
    }
    rhs(p, *to + dt, ynk, a, st);
    for (i = 0; i < DIM; i++) yerr[i] += BE7 * dt * a[i];

    double max_val = log(fabs(yo[0]));
    for (i = 1; i < DIM; i++) {
        double v = log(fabs(yo[i]));
        if (v > max_val) max_val = v;
    }
    double c = fmax(atol, rtol + max_val);
    double s = log(exp(atol - c) + exp(rtol + max_val - c)) + c;

    double err = 0.0;
    for (i = 0; i < DIM; i++) err += exp(2.0 * log(fabs(yerr[i])) - 2.0 * s);
    err = sqrt(err / (double)DIM);

    double corr = 0.85 * pow(err, -0.2);
    double powertwo = round(log(corr) / log(2.0));
    if (powertwo > MAX_STEPCHANGE_POWERTWO)
        powertwo = MAX_STEPCHANGE_POWERTWO;
    else if (powertwo < MIN_STEPCHANGE_POWERTWO)
        powertwo = MIN_STEPCHANGE_POWERTWO;

    *advanced = 0;
    if (powertwo >= 0.0 || accept != 0) {
        for (i = 0; i < DIM; i++) {
            a1[i] = a[i];
            yo[i] = yn1[i];
        }
        *to += dt;
        *advanced = 1;
    }
    return dt * pow(2.0, powertwo);
}

static int dopr54_run(const oracle_potential *p, const double yo_in[6], int nt, double dt_one,
                      const double *t, double rtol, double atol, int64_t max_steps,
                      double *result, int *err, oracle_stats *stats, int arbitrary_times)
{
    double a[DIM], a1[DIM], k1[DIM], k2[DIM], k3[DIM], k4[DIM], k5[DIM], k6[DIM];
    double yo[DIM], yn[DIM], yn1[DIM], yerr[DIM], ynk[DIM];
    oracle_stats local = {0, 0, 0};
    oracle_stats *st = stats ? stats : &local;
    int i, ii;
    int64_t attempts = 0;
    int status = ORACLE_OK;

    memcpy(yo, yo_in, sizeof(yo));
    memset(result, 0, sizeof(double) * (size_t)nt * DIM);
    /* save_rk(dim, yo, result) */
    for (i = 0; i < DIM; i++) result[i] = yo[i];
    *err = 0;
    for (i = 0; i < DIM; i++) yn[i] = yo[i];

    double dt = t[1] - t[0];
    if (dt_one == -9999.99) dt_one = rk4_estimate_step(p, yo, dt, t, rtol, atol, st);

    double to = t[0];
    rhs(p, to, yn, a1, st);

    for (ii = 0; ii < nt - 1; ii++) {
        /* dopr54_onestep, dopr54.rs:370-460 */
        double init_dt_one = dt_one;
        double init_to = to;
        /* arbitrary_times: the interval ends at t[ii + 1]; otherwise it spans
         * dt from where the previous one ended (bovy_rk's uniform grid). */
        const double end = arbitrary_times ? t[ii + 1] : init_to + dt;
        while ((dt >= 0.0 && to < end) || (dt < 0.0 && to > end)) {
            int accept = 0;
            int advanced;
            if (init_dt_one / dt_one > MAX_STEPREDUCE || dt_one != dt_one) {
                dt_one = init_dt_one / MAX_STEPREDUCE;
                accept = 1;
                if (*err % 2 == 0) *err += 1;
            }
            if (dt >= 0.0 && dt_one > (end - to)) dt_one = end - to;
            if (dt < 0.0 && dt_one < (end - to)) dt_one = end - to;
            if (max_steps > 0 && attempts >= max_steps) {
                status = ORACLE_MAX_STEPS;
                goto done;
            }
            attempts++;
            dt_one = dopr54_actualstep(p, yn, dt_one, &to, rtol, atol, a1, a, k1, k2, k3, k4,
                                       k5, k6, yn1, yerr, ynk, accept, &advanced, st);
            if (advanced)
                st->accepted++;
            else
                st->rejected++;
        }
        for (i = 0; i < DIM; i++) result[(size_t)(ii + 1) * DIM + i] = yn[i];
    }
done:
    return status;
}

/* ------------------------------------------------------------------ */
/* DOP853 (galpy leung_dop853.c as ported in dop853.rs)                */
/* ------------------------------------------------------------------ */

static const double UROUND = 2.3e-16;

static const double C2 = 0.526001519587677318785587544488e-1;
static const double C3 = 0.789002279381515978178381316732e-1;
static const double C4 = 0.118350341907227396726757197510;
static const double C5 = 0.281649658092772603273242802490;
static const double C6 = 0.333333333333333333333333333333;
static const double C7 = 0.25;
static const double C8 = 0.307692307692307692307692307692;
static const double C9 = 0.651282051282051282051282051282;
static const double C10 = 0.6;
static const double C11 = 0.857142857142857142857142857142;
static const double C14 = 0.1;
static const double C15 = 0.2;
static const double C16 = 0.777777777777777777777777777778;

static const double A21 = 5.26001519587677318785587544488e-2;
static const double A31 = 1.97250569845378994544595329183e-2;
static const double A32 = 5.91751709536136983633785987549e-2;
static const double A41 = 2.95875854768068491816892993775e-2;
static const double A43 = 8.87627564304205475450678981324e-2;
static const double A51 = 2.41365134159266685502369798665e-1;
static const double A53 = -8.84549479328286085344864962717e-1;
static const double A54 = 9.24834003261792003115737966543e-1;
static const double A61 = 3.7037037037037037037037037037e-2;
static const double A64 = 1.70828608729473871279604482173e-1;
static const double A65 = 1.25467687566822425016691814123e-1;
static const double A71 = 3.7109375e-2;
static const double A74 = 1.70252211019544039314978060272e-1;
static const double A75 = 6.02165389804559606850219397283e-2;
static const double A76 = -1.7578125e-2;
static const double A81 = 3.70920001185047927108779319836e-2;
static const double A84 = 1.70383925712239993810214054705e-1;
static const double A85 = 1.07262030446373284651809199168e-1;
static const double A86 = -1.53194377486244017527936158236e-2;
static const double A87 = 8.27378916381402288758473766002e-3;
static const double A91 = 6.24110958716075717114429577812e-1;
static const double A94 = -3.36089262944694129406857109825e0;
static const double A95 = -8.68219346841726006818189891453e-1;
static const double A96 = 2.75920996994467083049415600797e1;
static const double A97 = 2.01540675504778934086186788979e1;
static const double A98 = -4.34898841810699588477366255144e1;
static const double A101 = 4.77662536438264365890433908527e-1;
static const double A104 = -2.48811461997166764192642586468e0;
static const double A105 = -5.90290826836842996371446475743e-1;
static const double A106 = 2.12300514481811942347288949897e1;
static const double A107 = 1.52792336328824235832596922938e1;
static const double A108 = -3.32882109689848629194453265587e1;
static const double A109 = -2.03312017085086261358222928593e-2;
static const double A111 = -9.3714243008598732571704021658e-1;
static const double A114 = 5.18637242884406370830023853209e0;
static const double A115 = 1.09143734899672957818500254654e0;
static const double A116 = -8.14978701074692612513997267357e0;
static const double A117 = -1.85200656599969598641566180701e1;
static const double A118 = 2.27394870993505042818970056734e1;
static const double A119 = 2.49360555267965238987089396762e0;
static const double A1110 = -3.0467644718982195003823669022e0;
static const double A121 = 2.27331014751653820792359768449e0;
static const double A124 = -1.05344954667372501984066689879e1;
static const double A125 = -2.00087205822486249909675718444e0;
static const double A126 = -1.79589318631187989172765950534e1;
static const double A127 = 2.79488845294199600508499808837e1;
static const double A128 = -2.85899827713502369474065508674e0;
static const double A129 = -8.87285693353062954433549289258e0;
static const double A1210 = 1.23605671757943030647266201528e1;
static const double A1211 = 6.43392746015763530355970484046e-1;
static const double A141 = 5.61675022830479523392909219681e-2;
static const double A147 = 2.53500210216624811088794765333e-1;
static const double A148 = -2.46239037470802489917441475441e-1;
static const double A149 = -1.24191423263816360469010140626e-1;
static const double A1410 = 1.5329179827876569731206322685e-1;
static const double A1411 = 8.20105229563468988491666602057e-3;
static const double A1412 = 7.56789766054569976138603589584e-3;
static const double A1413 = -8.298e-3;
static const double A151 = 3.18346481635021405060768473261e-2;
static const double A156 = 2.83009096723667755288322961402e-2;
static const double A157 = 5.35419883074385676223797384372e-2;
static const double A158 = -5.49237485713909884646569340306e-2;
static const double A1511 = -1.08347328697249322858509316994e-4;
static const double A1512 = 3.82571090835658412954920192323e-4;
static const double A1513 = -3.40465008687404560802977114492e-4;
static const double A1514 = 1.41312443674632500278074618366e-1;
static const double A161 = -4.28896301583791923408573538692e-1;
static const double A166 = -4.69762141536116384314449447206e0;
static const double A167 = 7.68342119606259904184240953878e0;
static const double A168 = 4.06898981839711007970213554331e0;
static const double A169 = 3.56727187455281109270669543021e-1;
static const double A1613 = -1.39902416515901462129418009734e-3;
static const double A1614 = 2.9475147891527723389556272149e0;
static const double A1615 = -9.15095847217987001081870187138e0;

static const double B1 = 5.42937341165687622380535766363e-2;
static const double B6 = 4.45031289275240888144113950566;
static const double B7 = 1.89151789931450038304281599044;
static const double B8 = -5.8012039600105847814672114227;
static const double B9 = 3.1116436695781989440891606237e-1;
static const double B10 = -1.52160949662516078556178806805e-1;
static const double B11 = 2.01365400804030348374776537501e-1;
static const double B12 = 4.47106157277725905176885569043e-2;
static const double BHH1 = 0.244094488188976377952755905512;
static const double BHH2 = 0.733846688281611857341361741547;
static const double BHH3 = 0.220588235294117647058823529412e-1;

static const double D41 = -0.84289382761090128651353491142e1;
static const double D46 = 0.56671495351937776962531783590;
static const double D47 = -0.30689499459498916912797304727e1;
static const double D48 = 0.23846676565120698287728149680e1;
static const double D49 = 0.21170345824450282767155149946e1;
static const double D410 = -0.87139158377797299206789907490;
static const double D411 = 0.22404374302607882758541771650e1;
static const double D412 = 0.63157877876946881815570249290;
static const double D413 = -0.88990336451333310820698117400e-1;
static const double D414 = 0.18148505520854727256656404962e2;
static const double D415 = -0.91946323924783554000451984436e1;
static const double D416 = -0.44360363875948939664310572000e1;
static const double D51 = 0.10427508642579134603413151009e2;
static const double D56 = 0.24228349177525818288430175319e3;
static const double D57 = 0.16520045171727028198505394887e3;
static const double D58 = -0.37454675472269020279518312152e3;
static const double D59 = -0.22113666853125306036270938578e2;
static const double D510 = 0.77334326684722638389603898808e1;
static const double D511 = -0.30674084731089398182061213626e2;
static const double D512 = -0.93321305264302278729567221706e1;
static const double D513 = 0.15697238121770843886131091075e2;
static const double D514 = -0.31139403219565177677282850411e2;
static const double D515 = -0.93529243588444783865713862664e1;
static const double D516 = 0.35816841486394083752465898540e2;
static const double D61 = 0.19985053242002433820987653617e2;
static const double D66 = -0.38703730874935176555105901742e3;
static const double D67 = -0.18917813819516756882830838328e3;
static const double D68 = 0.52780815920542364900561016686e3;
static const double D69 = -0.11573902539959630126141871134e2;
static const double D610 = 0.68812326946963000169666922661e1;
static const double D611 = -0.10006050966910838403183860980e1;
static const double D612 = 0.77771377980534432092869265740;
static const double D613 = -0.27782057523535084065932004339e1;
static const double D614 = -0.60196695231264120758267380846e2;
static const double D615 = 0.84320405506677161018159903784e2;
static const double D616 = 0.11992291136182789328035130030e2;
static const double D71 = -0.25693933462703749003312586129e2;
static const double D76 = -0.15418974869023643374053993627e3;
static const double D77 = -0.23152937917604549567536039109e3;
static const double D78 = 0.35763911791061412378285349910e3;
static const double D79 = 0.93405324183624310003907691704e2;
static const double D710 = -0.37458323136451633156875139351e2;
static const double D711 = 0.10409964950896230045147246184e3;
static const double D712 = 0.29840293426660503123344363579e2;
static const double D713 = -0.43533456590011143754432175058e2;
static const double D714 = 0.96324553959188282948394950600e2;
static const double D715 = -0.39177261675615439165231486172e2;
static const double D716 = -0.14972683625798562581422125276e3;

static const double ER1 = 0.1312004499419488073250102996e-1;
static const double ER6 = -0.1225156446376204440720569753e1;
static const double ER7 = -0.4957589496572501915214079952;
static const double ER8 = 0.1664377182454986536961530415e1;
static const double ER9 = -0.3503288487499736816886487290;
static const double ER10 = 0.3341791187130174790297318841;
static const double ER11 = 0.8192320648511571246570742613e-1;
static const double ER12 = -0.2235530786388629525884427845e-1;

int oracle_dopr54(const oracle_potential *p, const double yo_in[6], int nt, double dt_one,
                  const double *t, double rtol, double atol, int64_t max_steps,
                  double *result, int *err, oracle_stats *stats)
{
    return dopr54_run(p, yo_in, nt, dt_one, t, rtol, atol, max_steps, result, err, stats, 0);
}

static double c_min(double a, double b) { return a < b ? a : b; }
static double c_max(double a, double b) { return a > b ? a : b; }
static double custom_sign(double x, double y) { return y > 0.0 ? fabs(x) : -fabs(x); }

static int dop853_run(const oracle_potential *p, const double y0_in[6], int nt, const double *t,
                      double rtol_ln, double atol_ln, int64_t max_steps, double *result,
                      oracle_stats *stats, double *tape, int64_t tape_steps)
{
    const int dim = DIM;
    oracle_stats local = {0, 0, 0};
    oracle_stats *st = stats ? stats : &local;
    double y0[DIM], yy1[DIM], yy_temp[DIM];
    double k1[DIM], k2[DIM], k3[DIM], k4[DIM], k5[DIM], k6[DIM], k7[DIM], k8[DIM], k9[DIM],
        k10[DIM];
    double rcont1[DIM], rcont2[DIM], rcont3[DIM], rcont4[DIM], rcont5[DIM], rcont6[DIM],
        rcont7[DIM], rcont8[DIM];
    int i;
    int64_t attempts = 0;

    memcpy(y0, y0_in, sizeof(y0));
    memset(result, 0, sizeof(double) * (size_t)nt * DIM);

    double rtol = exp(rtol_ln);
    double atol = exp(atol_ln);
    const double safe = 0.9;
    const double beta = 0.0;
    double facold = 1.0e-4;
    const double expo1 = 1.0 / 8.0 - beta * 0.2;
    const double facc1 = 1.0 / 0.333;
    const double facc2 = 1.0 / 6.0;
    double hmax = t[nt - 1] - t[0];
    double pos_neg = custom_sign(1.0, hmax);

    for (i = 0; i < dim; i++) result[i] = y0[i];
    size_t result_offset = dim;

    rhs(p, t[0], y0, k1, st);

    double dnf = 0.0, dny = 0.0;
    for (i = 0; i < dim; i++) {
        double sk = atol + rtol * fabs(y0[i]);
        double sqr = k1[i] / sk;
        dnf += sqr * sqr;
        sqr = y0[i] / sk;
        dny += sqr * sqr;
    }
    double h = custom_sign(c_min(sqrt(dny / dnf) * 0.01, fabs(hmax)), pos_neg);
    for (i = 0; i < dim; i++) k3[i] = y0[i] + h * k1[i];
    rhs(p, t[0] + h, k3, k2, st);
    double der2 = 0.0;
    for (i = 0; i < dim; i++) {
        double sk = atol + rtol * fabs(y0[i]);
        double sqr = (k2[i] - k1[i]) / sk;
        der2 += sqr * sqr;
    }
    der2 = sqrt(der2) / h;
    double der12 = c_max(fabs(der2), sqrt(dnf));
    double h1 = pow(0.01 / der12, 1.0 / 8.0);
    h = custom_sign(c_min(100.0 * fabs(h), c_min(fabs(h1), fabs(hmax))), pos_neg);

    int reject = 0;
    double t_current = t[0];
    double t_old = t[0];
    double t_old_older;
    int finished_user_t_ii = 0;

    while (finished_user_t_ii < nt - 1) {
        if (max_steps > 0 && attempts >= max_steps) return ORACLE_MAX_STEPS;
        attempts++;
        h = pos_neg * c_max(fabs(h), 1e3 * UROUND);

        for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * A21 * k1[i];
        rhs(p, t_current + C2 * h, yy1, k2, st);
        for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * (A31 * k1[i] + A32 * k2[i]);
        rhs(p, t_current + C3 * h, yy1, k3, st);
        for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * (A41 * k1[i] + A43 * k3[i]);
        rhs(p, t_current + C4 * h, yy1, k4, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A51 * k1[i] + A53 * k3[i] + A54 * k4[i]);
        rhs(p, t_current + C5 * h, yy1, k5, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A61 * k1[i] + A64 * k4[i] + A65 * k5[i]);
        rhs(p, t_current + C6 * h, yy1, k6, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A71 * k1[i] + A74 * k4[i] + A75 * k5[i] + A76 * k6[i]);
        rhs(p, t_current + C7 * h, yy1, k7, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] +
                     h * (A81 * k1[i] + A84 * k4[i] + A85 * k5[i] + A86 * k6[i] + A87 * k7[i]);
        rhs(p, t_current + C8 * h, yy1, k8, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A91 * k1[i] + A94 * k4[i] + A95 * k5[i] + A96 * k6[i] +
                                  A97 * k7[i] + A98 * k8[i]);
        rhs(p, t_current + C9 * h, yy1, k9, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A101 * k1[i] + A104 * k4[i] + A105 * k5[i] + A106 * k6[i] +
                                  A107 * k7[i] + A108 * k8[i] + A109 * k9[i]);
        rhs(p, t_current + C10 * h, yy1, k10, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A111 * k1[i] + A114 * k4[i] + A115 * k5[i] + A116 * k6[i] +
                                  A117 * k7[i] + A118 * k8[i] + A119 * k9[i] + A1110 * k10[i]);
        rhs(p, t_current + C11 * h, yy1, k2, st);
        for (i = 0; i < dim; i++)
            yy1[i] = y0[i] + h * (A121 * k1[i] + A124 * k4[i] + A125 * k5[i] + A126 * k6[i] +
                                  A127 * k7[i] + A128 * k8[i] + A129 * k9[i] + A1210 * k10[i] +
                                  A1211 * k2[i]);

        t_old_older = t_old;
        t_old = t_current;
        t_current = t_current + h;

        rhs(p, t_current, yy1, k3, st);

        for (i = 0; i < dim; i++) {
            k4[i] = B1 * k1[i] + B6 * k6[i] + B7 * k7[i] + B8 * k8[i] + B9 * k9[i] +
                    B10 * k10[i] + B11 * k2[i] + B12 * k3[i];
            k5[i] = y0[i] + h * k4[i];
        }

        double err = 0.0, err2 = 0.0;
        for (i = 0; i < dim; i++) {
            double sk = atol + rtol * c_max(fabs(y0[i]), fabs(k5[i]));
            double erri = k4[i] - BHH1 * k1[i] - BHH2 * k9[i] - BHH3 * k3[i];
            double sqr = erri / sk;
            err2 += sqr * sqr;
            erri = ER1 * k1[i] + ER6 * k6[i] + ER7 * k7[i] + ER8 * k8[i] + ER9 * k9[i] +
                   ER10 * k10[i] + ER11 * k2[i] + ER12 * k3[i];
            sqr = erri / sk;
            err += sqr * sqr;
        }
        double deno = err + 0.01 * err2;
        if (deno <= 0.0) deno = 1.0;
        err = fabs(h) * err * sqrt(1.0 / (deno * (double)dim));

        double fac11 = pow(err, expo1);
        double fac = fac11 / pow(facold, beta);
        fac = c_max(facc2, c_min(facc1, fac / safe));
        double hnew = h / fac;

        if (err <= 1.0) {
            if (tape && st->accepted < tape_steps) {
                double *row = tape + st->accepted * 8;
                row[0] = t_old;
                row[1] = h;
                for (i = 0; i < dim; i++) row[2 + i] = y0[i];
            }
            st->accepted++;
            facold = c_max(err, 1.0e-4);
            rhs(p, t_current, k5, k4, st);

            for (i = 0; i < dim; i++) {
                rcont1[i] = y0[i];
                double ydiff = k5[i] - y0[i];
                rcont2[i] = ydiff;
                double bspl = h * k1[i] - ydiff;
                rcont3[i] = bspl;
                rcont4[i] = ydiff - h * k4[i] - bspl;
                rcont5[i] = D41 * k1[i] + D46 * k6[i] + D47 * k7[i] + D48 * k8[i] +
                            D49 * k9[i] + D410 * k10[i] + D411 * k2[i] + D412 * k3[i];
                rcont6[i] = D51 * k1[i] + D56 * k6[i] + D57 * k7[i] + D58 * k8[i] +
                            D59 * k9[i] + D510 * k10[i] + D511 * k2[i] + D512 * k3[i];
                rcont7[i] = D61 * k1[i] + D66 * k6[i] + D67 * k7[i] + D68 * k8[i] +
                            D69 * k9[i] + D610 * k10[i] + D611 * k2[i] + D612 * k3[i];
                rcont8[i] = D71 * k1[i] + D76 * k6[i] + D77 * k7[i] + D78 * k8[i] +
                            D79 * k9[i] + D710 * k10[i] + D711 * k2[i] + D712 * k3[i];
            }

            for (i = 0; i < dim; i++)
                yy1[i] = y0[i] + h * (A141 * k1[i] + A147 * k7[i] + A148 * k8[i] +
                                      A149 * k9[i] + A1410 * k10[i] + A1411 * k2[i] +
                                      A1412 * k3[i] + A1413 * k4[i]);
            rhs(p, t_old + C14 * h, yy1, k10, st);
            for (i = 0; i < dim; i++)
                yy1[i] = y0[i] + h * (A151 * k1[i] + A156 * k6[i] + A157 * k7[i] +
                                      A158 * k8[i] + A1511 * k2[i] + A1512 * k3[i] +
                                      A1513 * k4[i] + A1514 * k10[i]);
            rhs(p, t_old + C15 * h, yy1, k2, st);
            for (i = 0; i < dim; i++)
                yy1[i] = y0[i] + h * (A161 * k1[i] + A166 * k6[i] + A167 * k7[i] +
                                      A168 * k8[i] + A169 * k9[i] + A1613 * k4[i] +
                                      A1614 * k10[i] + A1615 * k2[i]);
            rhs(p, t_old + C16 * h, yy1, k3, st);

            for (i = 0; i < dim; i++) {
                rcont5[i] = h * (rcont5[i] + D413 * k4[i] + D414 * k10[i] + D415 * k2[i] +
                                 D416 * k3[i]);
                rcont6[i] = h * (rcont6[i] + D513 * k4[i] + D514 * k10[i] + D515 * k2[i] +
                                 D516 * k3[i]);
                rcont7[i] = h * (rcont7[i] + D613 * k4[i] + D614 * k10[i] + D615 * k2[i] +
                                 D616 * k3[i]);
                rcont8[i] = h * (rcont8[i] + D713 * k4[i] + D714 * k10[i] + D715 * k2[i] +
                                 D716 * k3[i]);
                k1[i] = k4[i];
                y0[i] = k5[i];
            }

            while (finished_user_t_ii < nt - 1 &&
                   pos_neg * t[finished_user_t_ii + 1] < pos_neg * t_current) {
                double s = (t[finished_user_t_ii + 1] - t_old) / h;
                double s1 = 1.0 - s;
                for (i = 0; i < dim; i++)
                    yy_temp[i] =
                        rcont1[i] +
                        s * (rcont2[i] +
                             s1 * (rcont3[i] +
                                   s * (rcont4[i] +
                                        s1 * (rcont5[i] +
                                              s * (rcont6[i] + s1 * (rcont7[i] + s * rcont8[i]))))));
                memcpy(result + result_offset, yy_temp, sizeof(yy_temp));
                result_offset += dim;
                finished_user_t_ii += 1;
            }

            hnew = fabs(hnew) > fabs(hmax) ? pos_neg * hmax : hnew;
            if (reject != 0) hnew = pos_neg * c_min(fabs(hnew), fabs(h));
            reject = 0;
        } else {
            st->rejected++;
            hnew = h / c_min(facc1, fac11 / safe);
            reject = 1;
            t_current = t_old;
            t_old = t_old_older;
        }
        h = hnew;
    }
    return ORACLE_OK;
}

int oracle_dop853(const oracle_potential *p, const double y0_in[6], int nt, const double *t,
                  double rtol_ln, double atol_ln, int64_t max_steps, double *result,
                  oracle_stats *stats)
{
    return dop853_run(p, y0_in, nt, t, rtol_ln, atol_ln, max_steps, result, stats, NULL, 0);
}

int oracle_dop853_tape(const oracle_potential *p, const double y0_in[6], int nt, const double *t,
                       double rtol_ln, double atol_ln, int64_t max_steps, double *result,
                       oracle_stats *stats, double *tape, int64_t tape_steps)
{
    return dop853_run(p, y0_in, nt, t, rtol_ln, atol_ln, max_steps, result, stats, tape,
                      tape_steps);
}

/* ------------------------------------------------------------------ */
/* Batch driver (src/dispatch/cpu.rs:53-89)                            */
/* ------------------------------------------------------------------ */

double oracle_grid_sample(double start, double end, int64_t steps, int64_t index)
{
    if (index == steps - 1) return end;
    return start + (end - start) * (double)index / (double)(steps - 1);
}

int64_t oracle_integrate_batch(int method, const oracle_potential *p, int64_t n,
                               const double *y0, int nt, const double *ts, double t0,
                               const double *t_end, double rtol_ln, double atol_ln,
                               double dt_one, int64_t max_steps, double *out,
                               int32_t *status, int32_t *err, int64_t *accepted,
                               int64_t *rejected, int64_t *rhs_count, int threads,
                               int arbitrary_times)
{
    int64_t failures = 0;
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads) reduction(+ : failures)
    {
        double *traj = (double *)malloc(sizeof(double) * (size_t)nt * DIM);
        double *times = (double *)malloc(sizeof(double) * (size_t)nt);
#pragma omp for schedule(dynamic, 4)
        for (int64_t pid = 0; pid < n; pid++) {
            const double *tp = ts;
            if (!ts) {
                for (int k = 0; k < nt; k++) times[k] = oracle_grid_sample(t0, t_end[pid], nt, k);
                tp = times;
            }
            oracle_stats st = {0, 0, 0};
            int e = 0;
            int s;
            if (method == ORACLE_DOPR54)
                s = dopr54_run(p, y0 + pid * DIM, nt, dt_one, tp, rtol_ln, atol_ln, max_steps,
                               traj, &e, &st, arbitrary_times);
            else
                s = oracle_dop853(p, y0 + pid * DIM, nt, tp, rtol_ln, atol_ln, max_steps, traj,
                                  &st);
            if (out)
                for (int k = 0; k < nt; k++)
                    memcpy(out + ((size_t)k * (size_t)n + (size_t)pid) * DIM, traj + (size_t)k * DIM,
                           sizeof(double) * DIM);
            if (status) status[pid] = s;
            if (err) err[pid] = e;
            if (accepted) accepted[pid] = st.accepted;
            if (rejected) rejected[pid] = st.rejected;
            if (rhs_count) rhs_count[pid] = st.rhs;
            if (s != ORACLE_OK || e != 0) failures++;
        }
        free(traj);
        free(times);
    }
    return failures;
}
