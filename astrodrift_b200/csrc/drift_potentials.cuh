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
//                   exponential cutoff (enclosed-mass force).  In FMA mode
//                   (DRIFT_EXACT_ARITH 0) the disk and halo use reciprocals
//                   and a few-ulp rsqrt instead of the reference's
//                   divisions, the bulge and halo share one inverse radius
//                   and one radial sum, and ln / exp come from shared-memory
//                   tables.
// pow(., -1.5) and pow(., 1.5) go through the routines of drift_math.cuh
// instead of a general pow: correctly rounded in the exact unit, within a
// few ulps in the contraction unit, which also takes the Bovy force's log
// and exp from drift_math.cuh's table forms (log_tab, exp_tab).
#pragma once

#include "drift_math.cuh"
#include "drift_b200.h"

#ifndef DRIFT_EXACT_ARITH
#define DRIFT_EXACT_ARITH 1
#endif

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
    __host__ __device__ KeplerGalpy(const drift_potential &p, const double * = nullptr) : amp(p.amp) {}
    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
#if DRIFT_EXACT_ARITH
        double cylindrical_radius = sqrt(x * x + y * y);
        double sin_phi = y / cylindrical_radius;
        double cos_phi = x / cylindrical_radius;
        double radius_squared = cylindrical_radius * cylindrical_radius + z * z;
        double p = amp * unit_pow_m1p5(radius_squared);
        double radial_force = -cylindrical_radius * p;
        // The reference adds (1/R) * sin_phi * phi_torque with phi_torque = 0.
        // For every R >= 0 that term equals sin_phi * 0.0 (a signed zero, or
        // NaN exactly when sin_phi is NaN), so the division is dropped.
        ax = cos_phi * radial_force - sin_phi * 0.0;
        ay = sin_phi * radial_force + cos_phi * 0.0;
        az = -z * p;
#else
        // cos(phi) (-R p) = -x p wherever R > 0: no square root or division
        // on the dependency chain; on the z axis (R = 0) the cylindrical
        // form's NaN is kept.
        const double R2 = x * x + y * y;
        const double p = amp * unit_pow_m1p5(fma(z, z, R2));
        const double nan_if_axis = R2 > 0.0 ? 1.0 : __longlong_as_double(0x7ff8000000000000LL);
        ax = -x * p * nan_if_axis;
        ay = -y * p * nan_if_axis;
        az = -z * p;
#endif
    }
};

struct KeplerCartesian {
    double amp;
    __host__ __device__ KeplerCartesian(const drift_potential &p, const double * = nullptr) : amp(p.amp) {}
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
    __host__ __device__ Plummer(const drift_potential &p, const double * = nullptr)
        : amp(p.amp), b2(p.b * p.b)
    {
    }
    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
        double r2 = x * x + y * y + z * z;
        double ar = -amp * unit_pow_m1p5(r2 + b2);
        ax = ar * x;
        ay = ar * y;
        az = ar * z;
    }
};

// Lower incomplete gamma gamma(s, x) of the bulge at fixed cost.
//
// The host oracle follows Numerical Recipes (series / continued fraction);
// those loops run a data-dependent number of divisions, which diverges across
// the lanes of a warp.  The device evaluates the same function as
//   gamma(s, x) = x^s E(x),  E(x) = sum_n (-x)^n / (n! (s + n))  (x < 40),
// E being entire (E(x) = int_0^1 u^(s-1) e^(-x u) du), from a table built on
// the host in extended precision: Taylor expansions of E around the centres
// 1, 3, ..., 39, degree 17 in t = x - centre, |t| <= 1.  Every derivative
// obeys |E^(k)(x)| <= min(1 / (s + k), Gamma(s + k) / x^(s + k)), so the
// omitted terms stay below 1e-16 of E over [0, 40].  Every lane runs the
// same Horner sum and one power; for x >= 40, gamma = Gamma(s)
// (Gamma(s, 40) < 1e-15 Gamma(s) for s <= 1.5).
constexpr int BULGE_PIECES = 20;
constexpr int BULGE_PIECE_DEG = 17;  // odd: a piece's 18 coefficients load as 9 pairs
constexpr int BULGE_TABLE_SIZE = BULGE_PIECES * (BULGE_PIECE_DEG + 1);
constexpr double BULGE_X_CONST = 40.0;

struct BulgeTable {
    double c[BULGE_TABLE_SIZE];
};

// Shared-memory tables of the Bovy force, staged once per block (16-byte
// aligned): the bulge table's Taylor pieces, then the contraction unit's log
// and exp tables (drift_math.cuh).
constexpr int BOVY_SMEM_DOUBLES = BULGE_TABLE_SIZE + MATH_TABLE_DOUBLES;

__device__ __forceinline__ void stage_bovy_tables(double *smem, const BulgeTable &bt)
{
    for (int i = threadIdx.x; i < BULGE_TABLE_SIZE; i += blockDim.x) smem[i] = bt.c[i];
    for (int i = threadIdx.x; i < MATH_TABLE_DOUBLES; i += blockDim.x)
        smem[BULGE_TABLE_SIZE + i] = math_table_entry(i);
}

// x^s from ln and exp: the library functions in the exact unit, the tables
// (staged after the bulge table) in the contraction unit.
__device__ __forceinline__ double bulge_power(const double *table, double s, double x)
{
#if DRIFT_EXACT_ARITH
    (void)table;
    return exp(s * log(x));
#else
    const double *T = table + BULGE_TABLE_SIZE;
    return exp_tab(T, s * log_tab(T, x));
#endif
}

// `table` is the Bovy tables staged in shared memory: each lane reads its
// own piece, and differing addresses do not serialise there.
__device__ __forceinline__ double bulge_lower_gamma(const double *table, double s, double x, double gamma_s)
{
    if (x < BULGE_X_CONST) {
        const int j = min((int)(x * 0.5), BULGE_PIECES - 1);
        const double t = x - (2.0 * j + 1.0);
        // A piece is 18 doubles (144 bytes, 16-byte aligned), read as 9
        // pairs.  The degree-17 polynomial is evaluated as two halves,
        // p = P_lo(t) + t^9 P_hi(t) with P_lo = c0..c8 and P_hi = c9..c17,
        // whose Horner chains (8 multiply-adds each) run side by side: half
        // the dependent latency of one 17-term chain for four extra
        // multiplications.
        static_assert(BULGE_PIECE_DEG == 17, "the split below assumes 18 coefficients");
        const double2 *c = reinterpret_cast<const double2 *>(table + j * (BULGE_PIECE_DEG + 1));
        const double2 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3], c4 = c[4], c5 = c[5], c6 = c[6],
                      c7 = c[7], c8 = c[8];
        // P_lo: c0 .. c8 = c0.x c0.y c1.x c1.y c2.x c2.y c3.x c3.y c4.x
        double lo = fma(c4.x, t, c3.y);
        lo = fma(lo, t, c3.x);
        lo = fma(lo, t, c2.y);
        lo = fma(lo, t, c2.x);
        lo = fma(lo, t, c1.y);
        lo = fma(lo, t, c1.x);
        lo = fma(lo, t, c0.y);
        lo = fma(lo, t, c0.x);
        // P_hi: c9 .. c17 = c4.y c5.x c5.y c6.x c6.y c7.x c7.y c8.x c8.y
        double hi = fma(c8.y, t, c8.x);
        hi = fma(hi, t, c7.y);
        hi = fma(hi, t, c7.x);
        hi = fma(hi, t, c6.y);
        hi = fma(hi, t, c6.x);
        hi = fma(hi, t, c5.y);
        hi = fma(hi, t, c5.x);
        hi = fma(hi, t, c4.y);
        const double t2 = t * t, t4 = t2 * t2, t9 = (t4 * t4) * t;
        return bulge_power(table, s, x) * fma(hi, t9, lo);
    }
    return gamma_s;
}

struct Bovy {
    double mn_amp, mn_a, mn_b2;
    double nfw_amp, nfw_a;
    double bulge_s, bulge_rc2, bulge_k, bulge_gamma_s;
    double inv_rc2, inv_nfw_a;  // contraction unit: reciprocals formed once
    const double *table;   // BulgeTable staged in shared memory
    __device__ Bovy(const drift_potential &p, const double *bulge_table)
        : mn_amp(p.mn_amp), mn_a(p.mn_a), mn_b2(p.mn_b * p.mn_b), nfw_amp(p.nfw_amp),
          nfw_a(p.nfw_a), bulge_s(1.5 - 0.5 * p.bulge_alpha), bulge_rc2(p.bulge_rc * p.bulge_rc),
          bulge_k(p.bulge_k), bulge_gamma_s(p.bulge_gamma_s),
          inv_rc2(1.0 / (p.bulge_rc * p.bulge_rc)), inv_nfw_a(1.0 / p.nfw_a), table(bulge_table)
    {
    }

    __device__ DRIFT_FORCE_FN void force(double x, double y, double z, double &ax, double &ay,
                                          double &az) const
    {
#if DRIFT_EXACT_ARITH
        // bulge
        double bx = 0.0, by = 0.0, bz = 0.0;
        double r2s = x * x + y * y + z * z;
        if (r2s != 0.0) {
            double r = sqrt(r2s);
            double g = bulge_lower_gamma(table, bulge_s, r2s / bulge_rc2, bulge_gamma_s);
            double ar_over_r = -bulge_k * g / (r2s * r);
            bx = ar_over_r * x;
            by = ar_over_r * y;
            bz = ar_over_r * z;
        }
        // Miyamoto-Nagai disk
        double dx, dy, dz;
        {
            double r2 = x * x + y * y;
            double z2 = z * z;
            double r = sqrt(r2);
            double sqrtz2b2 = sqrt(z2 + mn_b2);
            double apz = mn_a + sqrtz2b2;
            double pyth = apz * apz;
            double denom = unit_pow_1p5(pyth + r2);
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
#else
        // One inverse radius serves the bulge and the halo, whose radial
        // accelerations are summed into one a_r / r before the disk is added
        // (fewer live temporaries than three separate vectors: the uneven
        // Bovy workload 12.40 -> 12.15 s per pass).
        const double r2s = x * x + y * y + z * z;
        const double inv_r = rsqrt_few_ulp(r2s);
        const double inv_r3 = inv_r * inv_r * inv_r;
        double ar_over_r;
        {
            // NFW halo
            const double r = r2s * inv_r;
            const double u = r * inv_nfw_a;
            const double term = log_tab(table + BULGE_TABLE_SIZE, 1. + u) - u * fast_rcp(1.0 + u);
            ar_over_r = -nfw_amp * term;
        }
        if (r2s != 0.0) {
            // bulge
            const double g = bulge_lower_gamma(table, bulge_s, r2s * inv_rc2, bulge_gamma_s);
            ar_over_r = fma(-bulge_k, g, ar_over_r);
        }
        ar_over_r *= inv_r3;
        // Miyamoto-Nagai disk: a_R x/R == -amp x / D with
        // D = (R^2 + (a + sqrt(z^2 + b^2))^2)^(3/2)
        const double r2 = x * x + y * y;
        const double zb2 = z * z + mn_b2;
        const double inv_sz = rsqrt_few_ulp(zb2);
        const double apz = fma(zb2, inv_sz, mn_a);
        const double m_over_d = -mn_amp * unit_pow_m1p5(fma(apz, apz, r2));
        ax = (m_over_d + ar_over_r) * x;
        ay = (m_over_d + ar_over_r) * y;
        az = fma(m_over_d * apz, z * inv_sz, ar_over_r * z);
#endif
    }
};

}  // namespace drift
