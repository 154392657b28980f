// drift_potentials.cuh -- fused force evaluation for the integrator kernels.
//
// Each potential is a functor with a device `force(x, y, z, ax, ay, az)`; the
// integrators are templated on it so the force is inlined into every stage.
// Formulas and their evaluation order follow the reference:
//   KeplerGalpy     src/integrators/galpy/dopr54.rs:75-88 (the force both
//                   reference integrators evaluate, amp fixed at 1 there)
//   KeplerCartesian shared/src/potential.rs:229-238
//   Plummer         shared/src/potential.rs:254-261
//   Bovy            shared/src/potential.rs:117-124 = ((bulge + disk) + halo),
//                   disk :138-151, halo :165-175, bulge = power law with
//                   exponential cutoff (enclosed-mass force).
// pow(., -1.5) and pow(., 1.5) go through the correctly rounded routines of
// drift_math.cuh instead of a general pow.
#pragma once

#include "drift_math.cuh"
#include "drift_b200.h"

// DRIFT_FORCE_NOINLINE: keep one out-of-line copy of each force body instead
// of inlining it at every stage (the integrators evaluate it up to 17 times
// per step, and the inlined copies compete for instruction cache).
#ifdef DRIFT_FORCE_NOINLINE
#define DRIFT_FORCE_FN __noinline__
#else
#define DRIFT_FORCE_FN __forceinline__
#endif

namespace drift {

struct KeplerGalpy {
    double amp;
    __host__ __device__ explicit KeplerGalpy(const drift_potential &p) : amp(p.amp) {}
    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
        double cylindrical_radius = sqrt(x * x + y * y);
        double sin_phi = y / cylindrical_radius;
        double cos_phi = x / cylindrical_radius;
        double radius_squared = cylindrical_radius * cylindrical_radius + z * z;
        double p = amp * pow_m1p5(radius_squared);
        double radial_force = -cylindrical_radius * p;
        // The reference adds (1/R) * sin_phi * phi_torque with phi_torque = 0.
        // For every R >= 0 that term equals sin_phi * 0.0 (a signed zero, or
        // NaN exactly when sin_phi is NaN), so the division is dropped.
        ax = cos_phi * radial_force - sin_phi * 0.0;
        ay = sin_phi * radial_force + cos_phi * 0.0;
        az = -z * p;
    }
};

struct KeplerCartesian {
    double amp;
    __host__ __device__ explicit KeplerCartesian(const drift_potential &p) : amp(p.amp) {}
    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
        double r2 = x * x + y * y + z * z;
        double r = sqrt(r2);
        double inv_r3 = 1.0 / (r2 * r);
        double ar = -amp * inv_r3;
        ax = ar * x;
        ay = ar * y;
        az = ar * z;
    }
};

struct Plummer {
    double amp, b2;
    __host__ __device__ explicit Plummer(const drift_potential &p) : amp(p.amp), b2(p.b * p.b) {}
    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
        double r2 = x * x + y * y + z * z;
        double ar = -amp * pow_m1p5(r2 + b2);
        ax = ar * x;
        ay = ar * y;
        az = ar * z;
    }
};

// Lower incomplete gamma gamma(s, x): power series for x < s + 1, modified
// Lentz continued fraction for Gamma(s, x) otherwise (Numerical Recipes 3rd
// ed. section 6.2).  Same recurrences and stopping rules as the host oracle.
__device__ __forceinline__ double lower_gamma(double s, double x, double gamma_s)
{
    const double eps = 1.1102230246251565e-16;  // 2^-53
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
    if (prefactor == 0.0) return gamma_s;  // Gamma(s, x) underflows: gamma == Gamma(s)
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

struct Bovy {
    double mn_amp, mn_a, mn_b2;
    double nfw_amp, nfw_a;
    double bulge_s, bulge_rc2, bulge_k, bulge_gamma_s;
    __host__ __device__ explicit Bovy(const drift_potential &p)
        : mn_amp(p.mn_amp), mn_a(p.mn_a), mn_b2(p.mn_b * p.mn_b), nfw_amp(p.nfw_amp),
          nfw_a(p.nfw_a), bulge_s(1.5 - 0.5 * p.bulge_alpha), bulge_rc2(p.bulge_rc * p.bulge_rc),
          bulge_k(p.bulge_k), bulge_gamma_s(p.bulge_gamma_s)
    {
    }

    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
        // bulge
        double bx = 0.0, by = 0.0, bz = 0.0;
        double r2s = x * x + y * y + z * z;
        if (r2s != 0.0) {
            double r = sqrt(r2s);
            double g = lower_gamma(bulge_s, r2s / bulge_rc2, bulge_gamma_s);
            double ar_over_r = -bulge_k * g / (r2s * r);
            bx = ar_over_r * x;
            by = ar_over_r * y;
            bz = ar_over_r * z;
        }
        // Miyamoto-Nagai disk
        double dx, dy, dz;
        {
            double r2 = x * x + y * y;
            double r = sqrt(r2);
            double z2 = z * z;
            double sqrtz2b2 = sqrt(z2 + mn_b2);
            double apz = mn_a + sqrtz2b2;
            double pyth = apz * apz;
            double denom = pow_1p5(pyth + r2);
            double ar = -mn_amp * (r / denom);
            dx = ar * (x / r);
            dy = ar * (y / r);
            dz = -mn_amp * (z * apz) / (sqrtz2b2 * denom);
        }
        // NFW halo
        double hx, hy, hz;
        {
            double r2 = r2s;
            double r = sqrt(r2);
            double ar = -nfw_amp * (log(1. + r / nfw_a) - r / (nfw_a + r)) / r2;
            hx = ar * (x / r);
            hy = ar * (y / r);
            hz = ar * (z / r);
        }
        ax = (bx + dx) + hx;
        ay = (by + dy) + hy;
        az = (bz + dz) + hz;
    }
};

}  // namespace drift
