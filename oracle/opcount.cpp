// opcount.cpp -- exact operation counts of the oracle's arithmetic (test
// infrastructure: it produces the algorithmic work figures the benchmark's
// roofline divides by; nothing here is on the product path).
//
// The oracle's C restatement is compiled here as C++ with every `double`
// replaced by a scalar that tallies its operations under the counting
// convention of the roofline: + - * / and sqrt are one flop each (the
// oracle has no fused multiply-add); pow, exp and log are transcendental
// calls, tallied apart, and so is the Bovy bulge's lower incomplete gamma
// (a series or continued fraction whose length depends on its argument);
// pow(x, 2) is one multiplication; comparisons, fabs, fmin/fmax, floor/ceil/round and
// sign changes are not counted.  The scalar converts to other arithmetic
// types only explicitly, so a libm call without a counting overload below
// fails to compile instead of escaping the tally.
//
// Output: one line per particle integration,
//   <case> <accepted> <rejected> <samples> <flops> <pow> <exp> <log> <sqrt> <gamma>
// from which oracle/roofline_counts.py fits the cost per accepted step,
// rejected step, emitted sample and particle.
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <random>
#include <vector>

namespace opcount {

struct Tally {
    uint64_t add = 0, mul = 0, div = 0, sqrt = 0, pow = 0, exp = 0, log = 0, gamma = 0;
    uint64_t flops() const { return add + mul + div + sqrt; }
};
Tally g;

struct Num {
    double v;
    Num() = default;
    constexpr Num(double x) : v(x) {}
    template <class T>
    explicit constexpr operator T() const
    {
        return (T)v;
    }
};

inline Num operator+(Num a, Num b) { g.add++; return Num(a.v + b.v); }
inline Num operator-(Num a, Num b) { g.add++; return Num(a.v - b.v); }
inline Num operator*(Num a, Num b) { g.mul++; return Num(a.v * b.v); }
inline Num operator/(Num a, Num b) { g.div++; return Num(a.v / b.v); }
inline Num operator-(Num a) { return Num(-a.v); }
inline Num operator+(Num a) { return a; }
inline Num &operator+=(Num &a, Num b) { return a = a + b; }
inline Num &operator-=(Num &a, Num b) { return a = a - b; }
inline Num &operator*=(Num &a, Num b) { return a = a * b; }
inline Num &operator/=(Num &a, Num b) { return a = a / b; }
inline bool operator<(Num a, Num b) { return a.v < b.v; }
inline bool operator>(Num a, Num b) { return a.v > b.v; }
inline bool operator<=(Num a, Num b) { return a.v <= b.v; }
inline bool operator>=(Num a, Num b) { return a.v >= b.v; }
inline bool operator==(Num a, Num b) { return a.v == b.v; }
inline bool operator!=(Num a, Num b) { return a.v != b.v; }
inline bool operator!(Num a) { return !a.v; }

inline Num sqrt(Num x) { g.sqrt++; return Num(std::sqrt(x.v)); }
// pow(x, 2.0) is x * x exactly (the reference squares that way in the disk
// and halo): one multiplication, not a transcendental call.
inline Num pow(Num x, Num y)
{
    if (y.v == 2.0)
        g.mul++;
    else
        g.pow++;
    return Num(std::pow(x.v, y.v));
}
inline Num exp(Num x) { g.exp++; return Num(std::exp(x.v)); }
inline Num log(Num x) { g.log++; return Num(std::log(x.v)); }
inline Num tgamma(Num x) { return Num(std::tgamma(x.v)); }
inline Num fabs(Num x) { return Num(std::fabs(x.v)); }
inline Num fmax(Num a, Num b) { return Num(std::fmax(a.v, b.v)); }
inline Num fmin(Num a, Num b) { return Num(std::fmin(a.v, b.v)); }
inline Num floor(Num x) { return Num(std::floor(x.v)); }
inline Num ceil(Num x) { return Num(std::ceil(x.v)); }
inline Num round(Num x) { return Num(std::round(x.v)); }
inline bool isfinite(Num x) { return std::isfinite(x.v); }
inline bool isnan(Num x) { return std::isnan(x.v); }

}  // namespace opcount

// The bulge's incomplete gamma, tallied as one call (defined below).
opcount::Num opcount_bulge_gamma(opcount::Num s, opcount::Num x, opcount::Num gamma_s);
#define ORACLE_BULGE_GAMMA opcount_bulge_gamma

#define double opcount::Num
#include "drift_oracle.c"
#undef double

opcount::Num opcount_bulge_gamma(opcount::Num s, opcount::Num x, opcount::Num gamma_s)
{
    const opcount::Tally saved = opcount::g;
    const opcount::Num v = oracle_lower_gamma(s, x, gamma_s);
    opcount::g = saved;
    opcount::g.gamma++;
    return v;
}

namespace {

using opcount::g;
using opcount::Num;

void report(const char *name, const oracle_stats &st, int samples, const opcount::Tally &t)
{
    printf("%s %lld %lld %d %llu %llu %llu %llu %llu %llu\n", name, (long long)st.accepted,
           (long long)st.rejected, samples, (unsigned long long)t.flops(), (unsigned long long)t.pow,
           (unsigned long long)t.exp, (unsigned long long)t.log, (unsigned long long)t.sqrt,
           (unsigned long long)t.gamma);
}

// Seeded initial states like the benchmark's: Plummer (amp = b = 1) bound
// orbits and near-circular Kepler orbits away from the z axis.
void initial_state(std::mt19937_64 &rng, bool plummer, double *y)
{
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::normal_distribution<double> n(0.0, 1.0);
    const double r = plummer ? 0.2 + 2.0 * u(rng) : 0.5 + 1.5 * u(rng);
    double d[3] = {n(rng), n(rng), 0.3 * n(rng)};
    const double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double w[3] = {-d[1], d[0], 0.2 * n(rng)};
    const double wn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    const double vc = plummer ? r / std::pow(r * r + 1.0, 0.75) : std::sqrt(1.0 / r);
    const double f = plummer ? 0.6 + 0.5 * u(rng) : 0.9 + 0.2 * u(rng);
    for (int i = 0; i < 3; i++) {
        y[i] = r * d[i] / dn;
        y[3 + i] = f * vc * w[i] / wn;
    }
}

// Seeded disc orbits in the Bovy composite (natural units): R in [0.1, 4],
// z ~ 0.1 R, speeds within 20 % of circular in the plane.
void bovy_initial_state(std::mt19937_64 &rng, const oracle_potential &p, double *y)
{
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::normal_distribution<double> n(0.0, 1.0);
    const double R = 0.1 * std::exp(u(rng) * std::log(40.0));
    const double phi = 2.0 * M_PI * u(rng);
    Num ax, ay, az;
    oracle_force(&p, Num(R), Num(0.0), Num(0.0), &ax, &ay, &az);
    const double vc = std::sqrt(R * std::fabs(ax.v));
    const double vt = vc * (1.0 + 0.1 * n(rng)), vr = 0.1 * vc * n(rng), vz = 0.1 * vc * n(rng);
    y[0] = R * std::cos(phi);
    y[1] = R * std::sin(phi);
    y[2] = 0.1 * R * n(rng);
    y[3] = vr * std::cos(phi) - vt * std::sin(phi);
    y[4] = vr * std::sin(phi) + vt * std::cos(phi);
    y[5] = vz;
}

void dop853_case(const char *name, int kind, double rtol, int nt, double t_end, int particles,
                 uint64_t seed)
{
    oracle_potential p;
    memset(&p, 0, sizeof(p));
    p.kind = kind;
    p.amp = 1.0;
    p.b = 1.0;
    if (kind == ORACLE_POT_BOVY)  // the benchmark composite (the library's Bovy defaults)
        oracle_bovy_setup(&p, Num(1.8), Num(1.9 / 8.0), Num(0.05), Num(0.7574802019), Num(3.0 / 8.0),
                          Num(0.28 / 8.0), Num(4.852230533528), Num(16.0 / 8.0));
    std::mt19937_64 rng(seed);
    std::vector<Num> t(nt), out((size_t)nt * 6);
    for (int k = 0; k < nt; k++) t[k] = Num(t_end * k / (nt - 1));
    for (int i = 0; i < particles; i++) {
        double y[6];
        if (kind == ORACLE_POT_BOVY)
            bovy_initial_state(rng, p, y);
        else
            initial_state(rng, kind == ORACLE_POT_PLUMMER, y);
        Num y0[6];
        for (int c = 0; c < 6; c++) y0[c] = Num(y[c]);
        oracle_stats st;
        memset(&st, 0, sizeof(st));
        const Num rl(std::log(rtol));
        g = opcount::Tally();
        dop853_run(&p, y0, nt, t.data(), rl, rl, 100000000, out.data(), &st, nullptr, 0);
        report(name, st, nt - 1, g);
    }
}

void dopr54_case(const char *name, double rtol, int nt, double t_end, int particles, uint64_t seed,
                 double dt_one)
{
    oracle_potential p;
    memset(&p, 0, sizeof(p));
    p.kind = ORACLE_POT_KEPLER;
    p.amp = 1.0;
    std::mt19937_64 rng(seed);
    std::vector<Num> t(nt), out((size_t)nt * 6);
    for (int k = 0; k < nt; k++) t[k] = Num(t_end * k / (nt - 1));
    for (int i = 0; i < particles; i++) {
        double y[6];
        initial_state(rng, false, y);
        Num y0[6];
        for (int c = 0; c < 6; c++) y0[c] = Num(y[c]);
        oracle_stats st;
        memset(&st, 0, sizeof(st));
        int err = 0;
        const Num rl(std::log(rtol));
        g = opcount::Tally();
        dopr54_run(&p, y0, nt, Num(dt_one), t.data(), rl, rl, 100000000, out.data(), &err, &st, 0);
        report(name, st, nt - 1, g);
    }
}

}  // namespace

int main()
{
    // Different tolerances, grids and spans give independent mixes of
    // accepted steps, rejected steps and samples for the fit.
    const double rtols[3] = {1e-8, 1e-10, 1e-12};
    const int nts[3] = {11, 101, 201};
    const double spans[3] = {5.0, 20.0, 60.0};
    uint64_t seed = 1;
    for (double rtol : rtols) {
        for (int nt : nts) {
            dop853_case("dop853_plummer", ORACLE_POT_PLUMMER, rtol, nt, 20.0, 6, seed++);
            dop853_case("dop853_kepler", ORACLE_POT_KEPLER, rtol, nt, 20.0, 6, seed++);
            dop853_case("dop853_bovy", ORACLE_POT_BOVY, rtol, nt, 20.0, 6, seed++);
        }
        // DOPR54 lands every substep sequence on the interval's end, and
        // whether the last step of an interval is shortened depends on the
        // orbit (one subtraction more); a single interval keeps that to
        // exactly one shortened step per particle.  A fixed first step skips
        // the RK4 step-size search, whose iteration count depends on the
        // particle.
        for (double span : spans) dopr54_case("dopr54_kepler", rtol, 2, span, 6, seed++, 1e-3);
    }
    return 0;
}
