// drift_dopr54.cuh -- per-thread DOPR54 integrator (one particle per thread).
//
// Follows galpy's bovy_rk.c as ported in the reference
// (src/integrators/galpy/dopr54.rs): RK4 initial-step estimate (:210-368),
// sub-steps clipped to land on each output time (dopr54_onestep :370-460),
// the Dormand-Prince 5(4) stages with FSAL (dopr54_actualstep :462-655) and
// a step size that only ever changes by a power of two in [-3, 3].
//
// Step-size control.  The reference forms the error norm in log space:
//   max_val = max_i ln|y_i|, c = max(atol, rtol + max_val),
//   s = ln(e^(atol-c) + e^(rtol+max_val-c)) + c,
//   err = sqrt(mean_i exp(2 ln|yerr_i| - 2 s)),
//   p = clamp(round(ln(0.85 err^-0.2) / ln 2), -3, 3)
// (15 logs, 8 exps and 2 pows per step).  With M = max_i |y_i| and
// sc = e^atol + e^rtol M, the same quantities are e^s = sc and
// err^2 = mean_i (yerr_i / sc)^2, so
//   p = clamp(round(log2(0.85) - 0.1 log2(err^2)), -3, 3),
// one log2 per step.  p is an integer; the two forms can only disagree when
// the argument of round() lies within about 1e-14 of a half-integer.  The
// special values map identically: err = 0 gives p = +3, err = inf gives
// p = -3 and a NaN err leaves p NaN, which rejects the step and makes the
// next step size NaN as in the reference.  The RK4 estimate's
// ceil(err^(1/5)) is evaluated the same way.
#pragma once

#include "drift_common.cuh"
#include "drift_composite.cuh"

namespace drift {
namespace dopr54c {
constexpr double C2 = 0.2;
constexpr double C3 = 0.3;
constexpr double C4 = 0.8;
constexpr double C5 = 8.0 / 9.0;
constexpr double A21 = 0.2;
constexpr double A31 = 3.0 / 40.0;
constexpr double A41 = 44.0 / 45.0;
constexpr double A51 = 19372.0 / 6561.0;
constexpr double A61 = 9017.0 / 3168.0;
constexpr double A71 = 35.0 / 384.0;
constexpr double A32 = 9.0 / 40.0;
constexpr double A42 = -56.0 / 15.0;
constexpr double A52 = -25360.0 / 2187.0;
constexpr double A62 = -355.0 / 33.0;
constexpr double A43 = 32.0 / 9.0;
constexpr double A53 = 64448.0 / 6561.0;
constexpr double A63 = 46732.0 / 5247.0;
constexpr double A73 = 500.0 / 1113.0;
constexpr double A54 = -212.0 / 729.0;
constexpr double A64 = 49.0 / 176.0;
constexpr double A74 = 125.0 / 192.0;
constexpr double A65 = -5103.0 / 18656.0;
constexpr double A75 = -2187.0 / 6784.0;
constexpr double A76 = 11.0 / 84.0;
constexpr double B1 = 35.0 / 384.0;
constexpr double B3 = 500.0 / 1113.0;
constexpr double B4 = 125.0 / 192.0;
constexpr double B5 = -2187.0 / 6784.0;
constexpr double B6 = 11.0 / 84.0;
constexpr double BE1 = B1 - 5179.0 / 57600.0;
constexpr double BE3 = B3 - 7571.0 / 16695.0;
constexpr double BE4 = B4 - 393.0 / 640.0;
constexpr double BE5 = B5 + 92097.0 / 339200.0;
constexpr double BE6 = B6 - 187.0 / 2100.0;
constexpr double BE7 = -1.0 / 40.0;
constexpr double MAX_STEPCHANGE_POWERTWO = 3.0;
constexpr double MIN_STEPCHANGE_POWERTWO = -3.0;
constexpr double MAX_STEPREDUCE = 10000.0;
constexpr double MAX_DT_REDUCE = 10000.0;
constexpr double LOG2_085 = -0.23446525363702297;  // log2(0.85)
}  // namespace dopr54c

// Tolerance constants of one launch, derived on the host with the host libm:
// rtol/atol are the natural logs the reference passes; e_rtol/e_atol their
// exponentials.
struct Dopr54Tol {
    double e_rtol, e_atol;
};

template <class Pot>
struct Dopr54Lane {
    double yn[6];  // current solution
    double a1[6];  // f(yn), carried across steps (FSAL)
    double to;     // current time
    double dt;     // output interval (t[1] - t[0])
    double dt_one; // current step size
    double init_to, init_dt_one;
    double end;    // end of the current output interval
    bool arbitrary;  // intervals end at ts[ii + 1] (else every interval spans dt)
    int32_t ii;    // index of the interval being integrated
    int32_t err;   // galpy error code
    bool done;

    // a = f(t, q) = (v, F(t, x)); stationary potentials ignore t.
    __device__ __forceinline__ void rhs(const Pot &pot, double t, const double *q, double *a) const
    {
        a[0] = q[3];
        a[1] = q[4];
        a[2] = q[5];
        force_at(pot, t, q[0], q[1], q[2], a[3], a[4], a[5]);
    }

    // 1 / (e^atol + e^rtol max_i |y_i|), the reciprocal of e^s.
    __device__ __forceinline__ static double inv_scale(const double *y, const Dopr54Tol &tol)
    {
        double m = fabs(y[0]);
#pragma unroll
        for (int i = 1; i < 6; i++) {
            double v = fabs(y[i]);
            if (v > m) m = v;
        }
#if DRIFT_EXACT_ARITH
        return 1.0 / (tol.e_atol + tol.e_rtol * m);
#else
        return fast_rcp(tol.e_atol + tol.e_rtol * m);
#endif
    }

    // rk4_onestep (dopr54.rs:135-208): yn1 += RK4 increment of step dt.
    __device__ __forceinline__ void rk4_onestep(const Pot &pot, double tn, const double *yv, double *yn1,
                                                double dtv) const
    {
        double a[6], ynk[6];
        rhs(pot, tn, yv, a);
#pragma unroll
        for (int i = 0; i < 6; i++) yn1[i] += dtv * a[i] / 6.0;
#pragma unroll
        for (int i = 0; i < 6; i++) ynk[i] = yv[i] + dtv * a[i] / 2.0;
        rhs(pot, tn + dtv / 2.0, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) yn1[i] += dtv * a[i] / 3.0;
#pragma unroll
        for (int i = 0; i < 6; i++) ynk[i] = yv[i] + dtv * a[i] / 2.0;
        rhs(pot, tn + dtv / 2.0, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) yn1[i] += dtv * a[i] / 3.0;
#pragma unroll
        for (int i = 0; i < 6; i++) ynk[i] = yv[i] + dtv * a[i];
        rhs(pot, tn + dtv, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) yn1[i] += dtv * a[i] / 6.0;
    }

    // rk4_estimate_step (dopr54.rs:210-368).
    __device__ __forceinline__ double rk4_estimate_step(const Pot &pot, double t0, double dtv,
                                                        const Dopr54Tol &tol) const
    {
        using namespace dopr54c;
        const double init_dt = dtv;
        const double isc = inv_scale(yn, tol);
        for (int trial = 0; trial < 64; trial++) {
            double y1[6], y21[6], y2[6];
#pragma unroll
            for (int i = 0; i < 6; i++) {
                y1[i] = yn[i];
                y21[i] = yn[i];
            }
            rk4_onestep(pot, t0, yn, y1, dtv);
            rk4_onestep(pot, t0, yn, y21, dtv / 2.0);
#pragma unroll
            for (int i = 0; i < 6; i++) y2[i] = y21[i];
            rk4_onestep(pot, t0 + dtv / 2.0, y21, y2, dtv / 2.0);
            double q = 0.0;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double r = (y1[i] - y2[i]) * isc;
                q += r * r;
            }
            q = q / 6.0;
            // factor = ceil(err^(1/5)) with err^2 = q
            double factor = ceil(exp2(0.1 * log2(q)));
            if (factor > 1.0 && init_dt / dtv * factor < MAX_DT_REDUCE)
                dtv /= factor;
            else
                break;
        }
        return dtv;
    }

    // dopr54.rs:670-770 set-up; writes y0 as output sample 0.
    template <class Out>
    // arbitrary_times: interval i ends exactly at ts[i + 1] (output times
    // need not be uniform); otherwise every interval spans ts[1] - ts[0]
    // from where the previous one ended, as galpy's bovy_rk does.
    __device__ __forceinline__ void begin(const Pot &pot, const double *y0, const Grid &grid,
                                          double dt_one_init, const Dopr54Tol &tol, Out &out,
                                          bool arbitrary_times = false)
    {
        arbitrary = arbitrary_times;
#pragma unroll
        for (int i = 0; i < 6; i++) yn[i] = y0[i];
        out.write(0, yn);
        err = 0;
        double t0 = grid.at(0);
        dt = grid.at(1) - t0;
        dt_one = dt_one_init;
        if (dt_one == -9999.99) dt_one = rk4_estimate_step(pot, t0, dt, tol);
        to = t0;
        rhs(pot, to, yn, a1);
        ii = 0;
        done = (grid.nt < 2);
        init_to = to;
        init_dt_one = dt_one;
        end = arbitrary ? grid.at(1) : init_to + dt;
        close_intervals(grid, out);
    }

    __device__ __forceinline__ bool inside_interval() const
    {
        return (dt >= 0.0 && to < end) || (dt < 0.0 && to > end);
    }

    // End of dopr54_onestep's loop: save the state for every interval whose
    // end has been reached and open the next one.
    template <class Out>
    __device__ __forceinline__ void close_intervals(const Grid &grid, Out &out)
    {
        while (!done && !inside_interval()) {
            out.write(ii + 1, yn);
            ii += 1;
            if (ii >= grid.nt - 1) {
                done = true;
            } else {
                init_to = to;
                init_dt_one = dt_one;
                end = arbitrary ? grid.at(ii + 1) : init_to + dt;
            }
        }
    }

    // One pass of dopr54_onestep's loop body plus dopr54_actualstep.
    // Returns true when the step advanced the solution.
    template <class Out>
    __device__ __forceinline__ bool step(const Pot &pot, const Grid &grid, const Dopr54Tol &tol,
                                         Out &out)
    {
        using namespace dopr54c;
        int accept = 0;
        if (init_dt_one / dt_one > MAX_STEPREDUCE || dt_one != dt_one) {
            dt_one = init_dt_one / MAX_STEPREDUCE;
            accept = 1;
            if (err % 2 == 0) err += 1;
        }
        if (dt >= 0.0 && dt_one > (end - to)) dt_one = end - to;
        if (dt < 0.0 && dt_one < (end - to)) dt_one = end - to;

        const double h = dt_one;
        double yn1[6], yerr[6], ynk[6], a[6];
        double k1[6], k2[6], k3[6], k4[6], k5[6], k6[6];
#pragma unroll
        for (int i = 0; i < 6; i++) yn1[i] = yn[i];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k1[i] = h * a1[i];
            yn1[i] += B1 * k1[i];
            yerr[i] = BE1 * k1[i];
            ynk[i] = yn[i] + A21 * k1[i];
        }
        rhs(pot, to + C2 * h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k2[i] = h * a[i];
            ynk[i] = yn[i] + A31 * k1[i] + A32 * k2[i];
        }
        rhs(pot, to + C3 * h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k3[i] = h * a[i];
            yn1[i] += B3 * k3[i];
            yerr[i] += BE3 * k3[i];
            ynk[i] = yn[i] + A41 * k1[i] + A42 * k2[i] + A43 * k3[i];
        }
        rhs(pot, to + C4 * h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k4[i] = h * a[i];
            yn1[i] += B4 * k4[i];
            yerr[i] += BE4 * k4[i];
            ynk[i] = yn[i] + A51 * k1[i] + A52 * k2[i] + A53 * k3[i] + A54 * k4[i];
        }
        rhs(pot, to + C5 * h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k5[i] = h * a[i];
            yn1[i] += B5 * k5[i];
            yerr[i] += BE5 * k5[i];
            ynk[i] = yn[i] + A61 * k1[i] + A62 * k2[i] + A63 * k3[i] + A64 * k4[i] + A65 * k5[i];
        }
        rhs(pot, to + h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            k6[i] = h * a[i];
            yn1[i] += B6 * k6[i];
            yerr[i] += BE6 * k6[i];
            ynk[i] = yn[i] + A71 * k1[i] + A73 * k3[i] + A74 * k4[i] + A75 * k5[i] + A76 * k6[i];
        }
        rhs(pot, to + h, ynk, a);
#pragma unroll
        for (int i = 0; i < 6; i++) yerr[i] += BE7 * h * a[i];

        const double isc = inv_scale(yn, tol);
        double q = 0.0;
#pragma unroll
        for (int i = 0; i < 6; i++) {
            double r = yerr[i] * isc;
            q += r * r;
        }
#if DRIFT_EXACT_ARITH
        q = q / 6.0;
#else
        q = q * (1.0 / 6.0);
#endif
        double powertwo = round(LOG2_085 - 0.1 * unit_log2_for_rounding(q));
        if (powertwo > MAX_STEPCHANGE_POWERTWO)
            powertwo = MAX_STEPCHANGE_POWERTWO;
        else if (powertwo < MIN_STEPCHANGE_POWERTWO)
            powertwo = MIN_STEPCHANGE_POWERTWO;

        bool advanced = false;
        if (powertwo >= 0.0 || accept != 0) {
#pragma unroll
            for (int i = 0; i < 6; i++) {
                a1[i] = a[i];
                yn[i] = yn1[i];
            }
            to += h;
            advanced = true;
        }
        // dt * pow(2, powertwo) with powertwo an integer in [-3, 3]: a
        // product with an exact power of two, which rounds (subnormal results)
        // and overflows exactly as scalbn does.  NaN stays NaN.
        dt_one = (powertwo == powertwo)
                     ? h * __longlong_as_double((long long)(1023 + (int)powertwo) << 52)
                     : powertwo;
        close_intervals(grid, out);
        return advanced;
    }
};

}  // namespace drift
