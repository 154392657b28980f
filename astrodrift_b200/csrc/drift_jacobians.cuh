// drift_jacobians.cuh -- force Jacobians and parameter derivatives for the
// discrete adjoint.
//
// For a force a(x; p) = -grad Phi the Jacobian J = da/dx is symmetric, so the
// vector-Jacobian product the adjoint needs, J^T w, is J w.  Each functor's
// `vjp(x, y, z, w, jw, dp)` returns J w in jw[3] and adds w . da/dp_j to
// dp[j] for the potential's parameters, in the order
//   Kepler (both forms): amp
//   Plummer:             amp, b
//   Bovy:                mn_amp, mn_a, mn_b, nfw_amp, nfw_a, bulge_k
// Used by the adjoint only, which is compiled with contraction: powers,
// logs, exps, inverse square roots and reciprocals are the few-ulp forms of
// drift_math.cuh (ln and exp from the tables staged beside the bulge table).
// The formulas are the analytic derivatives of the forces in
// drift_potentials.cuh (shared/src/potential.rs:126-176, 229-262 and the
// galpy-cylindrical Kepler force of src/integrators/galpy/dopr54.rs:75-88,
// which equals -amp x / r^3 wherever R > 0).
#pragma once

#include "drift_potentials.cuh"

namespace drift {

// Point mass, -amp x / r^3:
//   J w = -amp (w / r^3 - 3 x (x.w) / r^5),  da/damp = -x / r^3.
struct KeplerJac {
    double amp;
    __host__ __device__ KeplerJac(const drift_potential &p, const double * = nullptr) : amp(p.amp) {}
    __device__ __forceinline__ void vjp(double x, double y, double z, const double *w, double *jw,
                                        double *dp) const
    {
        double r2 = x * x + y * y + z * z;
        double r = sqrt(r2);
        double ir3 = 1.0 / (r2 * r);
        double xw = x * w[0] + y * w[1] + z * w[2];
        double c = 3.0 * xw * ir3 / r2;
        jw[0] = -amp * (w[0] * ir3 - x * c);
        jw[1] = -amp * (w[1] * ir3 - y * c);
        jw[2] = -amp * (w[2] * ir3 - z * c);
        dp[0] += -xw * ir3;
    }
};

// Plummer, -amp x q^-3/2 with q = r^2 + b^2:
//   J w = -amp (w q^-3/2 - 3 x (x.w) q^-5/2),
//   da/damp = -x q^-3/2,  da/db = 3 amp b x q^-5/2.
struct PlummerJac {
    double amp, b;
    __host__ __device__ PlummerJac(const drift_potential &p, const double * = nullptr) : amp(p.amp), b(p.b) {}
    __device__ __forceinline__ void vjp(double x, double y, double z, const double *w, double *jw,
                                        double *dp) const
    {
        double q = x * x + y * y + z * z + b * b;
        double q15 = 1.0 / (q * sqrt(q));
        double q25 = q15 / q;
        double xw = x * w[0] + y * w[1] + z * w[2];
        double c = 3.0 * xw * q25;
        jw[0] = -amp * (w[0] * q15 - x * c);
        jw[1] = -amp * (w[1] * q15 - y * c);
        jw[2] = -amp * (w[2] * q15 - z * c);
        dp[0] += -xw * q15;
        dp[1] += 3.0 * amp * b * xw * q25;
    }
};

// Bovy composite: bulge + Miyamoto-Nagai disk + NFW halo.
//
// Disk: zeta = sqrt(z^2 + b^2), A = a + zeta, D = R^2 + A^2,
//   a = -amp D^-3/2 g with g = (x, y, A z / zeta) = grad(D) / 2,
//   J w = -amp (D^-3/2 (w_x, w_y, h w_z) - 3 D^-5/2 g (g.w)),
//   h = z^2 / zeta^2 + A b^2 / zeta^3 (= d g_z / dz),
//   da/da_mn = -amp (D^-3/2 (0, 0, z / zeta) - 3 A D^-5/2 g),
//   da/db_mn = -amp (-D^-3/2 (0, 0, a b z / zeta^3) - 3 A (b / zeta) D^-5/2 g).
// Halo: m(r) = ln(1 + r/a) - r / (a + r), a = -amp m x / r^3, m' = r / (a + r)^2,
//   J w = -amp (m (w / r^3 - 3 x (x.w) / r^5) + x (x.w) / (r^3 (a + r)^2)),
//   dm/da = -r^2 / (a (a + r)^2).
// Bulge: G(r) = gamma(s, r^2 / rc^2), a = -k G x / r^3,
//   G'(r) = (r^2/rc^2)^(s-1) exp(-r^2/rc^2) 2 r / rc^2,
//   J w = -k (G (w / r^3 - 3 x (x.w) / r^5) + G' x (x.w) / r^4).
struct BovyJac {
    double mn_amp, mn_a, mn_b;
    double nfw_amp, nfw_a;
    double bulge_s, bulge_rc2, bulge_k, bulge_gamma_s;
    double inv_nfw_a, inv_rc2;  // reciprocals formed once
    const double *table;
    __device__ BovyJac(const drift_potential &p, const double *bulge_table)
        : mn_amp(p.mn_amp), mn_a(p.mn_a), mn_b(p.mn_b), nfw_amp(p.nfw_amp), nfw_a(p.nfw_a),
          bulge_s(1.5 - 0.5 * p.bulge_alpha), bulge_rc2(p.bulge_rc * p.bulge_rc), bulge_k(p.bulge_k),
          bulge_gamma_s(p.bulge_gamma_s), inv_nfw_a(1.0 / p.nfw_a),
          inv_rc2(1.0 / (p.bulge_rc * p.bulge_rc)), table(bulge_table)
    {
    }
    __device__ __forceinline__ void vjp(double x, double y, double z, const double *w, double *jw,
                                        double *dp) const
    {
        const double *T = table + BULGE_TABLE_SIZE;  // ln / exp tables (drift_math.cuh)
        const double xw = x * w[0] + y * w[1] + z * w[2];
        const double r2 = x * x + y * y + z * z;
        jw[0] = jw[1] = jw[2] = 0.0;
        // disk
        {
            double zeta2 = z * z + mn_b * mn_b;
            double izeta = rsqrt_few_ulp(zeta2);
            double zeta = zeta2 * izeta;
            double A = mn_a + zeta;
            double D = x * x + y * y + A * A;
            double d15 = unit_pow_m1p5(D);
            double d25 = d15 * fast_rcp(D);
            double gz = A * z * izeta;
            double gw = x * w[0] + y * w[1] + gz * w[2];
            double h = z * z / zeta2 + A * mn_b * mn_b * izeta * izeta * izeta;
            double c = 3.0 * d25 * gw;
            jw[0] += -mn_amp * (d15 * w[0] - c * x);
            jw[1] += -mn_amp * (d15 * w[1] - c * y);
            jw[2] += -mn_amp * (d15 * h * w[2] - c * gz);
            dp[0] += -d15 * gw;
            dp[1] += -mn_amp * (d15 * w[2] * z * izeta - 3.0 * A * d25 * gw);
            dp[2] += -mn_amp * (-d15 * mn_a * mn_b * z * w[2] * izeta * izeta * izeta -
                                3.0 * A * mn_b * izeta * d25 * gw);
        }
        if (r2 != 0.0) {
            const double inv_r = rsqrt_few_ulp(r2);
            const double r = r2 * inv_r;
            const double ir3 = inv_r * inv_r * inv_r;
            const double c3 = 3.0 * xw * ir3 * (inv_r * inv_r);
            // halo
            {
                double apr = nfw_a + r;
                double inv_apr = fast_rcp(apr);
                double m = log_tab(T, 1.0 + r * inv_nfw_a) - r * inv_apr;
                double e = xw * ir3 * (inv_apr * inv_apr);
                jw[0] += -nfw_amp * (m * (w[0] * ir3 - x * c3) + x * e);
                jw[1] += -nfw_amp * (m * (w[1] * ir3 - y * c3) + y * e);
                jw[2] += -nfw_amp * (m * (w[2] * ir3 - z * c3) + z * e);
                dp[3] += -m * xw * ir3;
                dp[4] += nfw_amp * xw * inv_r * inv_nfw_a * (inv_apr * inv_apr);
            }
            // bulge
            {
                double u = r2 * inv_rc2;
                double G = bulge_lower_gamma(table, bulge_s, u, bulge_gamma_s);
                double Gp = exp_tab(T, (bulge_s - 1.0) * log_tab(T, u) - u) * 2.0 * r * inv_rc2;
                double e = Gp * xw * ir3 * inv_r;
                jw[0] += -bulge_k * (G * (w[0] * ir3 - x * c3) + x * e);
                jw[1] += -bulge_k * (G * (w[1] * ir3 - y * c3) + y * e);
                jw[2] += -bulge_k * (G * (w[2] * ir3 - z * c3) + z * e);
                dp[5] += -G * xw * ir3;
            }
        }
    }
};

}  // namespace drift
