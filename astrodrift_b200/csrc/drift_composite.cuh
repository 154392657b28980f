// drift_composite.cuh -- the summed, time-dependent force of a stage
// (drift_force_model): stationary potentials plus potentials attached to the
// particles of groups integrated in earlier stages.
//
// The reference's model (src/tree/mod.rs:89-110) lists, for every stage,
// the recipes of the containers it requires; a particle group created with
// `particles(potential, istate)` becomes a CustomKepler / CustomPlummer
// recipe whose force is the sum of the attached potential over the group's
// particles, each placed at its interpolated position at time t
// (shared/src/potential.rs:264-356).  The reference leaves the construction
// unfinished (shared/src/model.rs:193-199, 225-231); here the positions come
// from the earlier stage's trajectory through quintic Hermite segments
// (position, velocity and acceleration matched at both ends of each output
// interval), so the source moves on a C2 curve that is exact to O(dt^6).
//
// Evaluation order (kept by the oracle): stationary parts in order, then
// every source of every group in order, each added to a running sum that
// starts at 0.  A model with one stationary part therefore reproduces that
// potential's force bit for bit.
#pragma once

#include "drift_potentials.cuh"

namespace drift {

// Stationary potentials ignore t; the composite uses it.
template <class Pot>
struct is_time_dependent {
    static constexpr bool value = false;
};

// Quintic Hermite segment of one axis: x(0) = x0, x'(0) = h v0, x''(0) = h^2 a0
// and the same at s = 1, as coefficients of x(s) = c0 + s(c1 + ... + s c5).
__host__ __device__ __forceinline__ void hermite5(double x0, double v0, double a0, double x1, double v1,
                                                  double a1, double h, double *c)
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

__host__ __device__ __forceinline__ double quintic(const double *c, double s)
{
    return c[0] + s * (c[1] + s * (c[2] + s * (c[3] + s * (c[4] + s * c[5]))));
}

struct Composite {
    const drift_force_model *m;  // in the kernel's parameter space
    const double *table;         // bulge table (shared memory) for Bovy parts

    __device__ Composite(const drift_force_model *model, const double *bulge_table)
        : m(model), table(bulge_table)
    {
    }

    __device__ DRIFT_FORCE_FN void force_t(double t, double x, double y, double z, double &ax,
                                           double &ay, double &az) const
    {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        const int ns = m->n_static;
        for (int i = 0; i < ns; i++) {
            const drift_potential &p = m->statics[i];
            double fx = 0.0, fy = 0.0, fz = 0.0;
            switch (p.kind) {
            case DRIFT_POT_KEPLER: KeplerGalpy(p).force(x, y, z, fx, fy, fz); break;
            case DRIFT_POT_PLUMMER: Plummer(p).force(x, y, z, fx, fy, fz); break;
            case DRIFT_POT_BOVY: Bovy(p, table).force(x, y, z, fx, fy, fz); break;
            case DRIFT_POT_KEPLER_CARTESIAN: KeplerCartesian(p).force(x, y, z, fx, fy, fz); break;
            default: break;
            }
            sx = sx + fx;
            sy = sy + fy;
            sz = sz + fz;
        }
        const int ng = m->n_groups;
        if (ng > 0) {
            const double u = (t - m->t0) / m->dt;
            double kf = floor(u);
            kf = fmin(fmax(kf, 0.0), (double)(m->n_segments - 1));
            const double s = u - kf;
            const double *row = m->origins + (int64_t)kf * m->n_sources * 18;
            for (int g = 0; g < ng; g++) {
                const drift_source_group &G = m->groups[g];
                const bool plummer = G.kind == DRIFT_POT_PLUMMER;
                drift_potential sp;
                sp.amp = G.amp;
                sp.b = G.b;
                const Plummer pl(sp);
                const KeplerCartesian kc(sp);
                for (int64_t j = G.first; j < G.first + G.count; j++) {
                    const double *c = row + j * 18;
                    const double dx = x - quintic(c, s);
                    const double dy = y - quintic(c + 6, s);
                    const double dz = z - quintic(c + 12, s);
                    double fx, fy, fz;
                    if (plummer)
                        pl.force(dx, dy, dz, fx, fy, fz);
                    else
                        kc.force(dx, dy, dz, fx, fy, fz);
                    sx = sx + fx;
                    sy = sy + fy;
                    sz = sz + fz;
                }
            }
        }
        ax = sx;
        ay = sy;
        az = sz;
    }
};

template <>
struct is_time_dependent<Composite> {
    static constexpr bool value = true;
};

// The force of any potential at time t (stationary potentials ignore t).
template <class Pot>
__device__ __forceinline__ void force_at(const Pot &pot, double t, double x, double y, double z, double &ax,
                                         double &ay, double &az)
{
    if constexpr (is_time_dependent<Pot>::value)
        pot.force_t(t, x, y, z, ax, ay, az);
    else
        pot.force(x, y, z, ax, ay, az);
}

}  // namespace drift
