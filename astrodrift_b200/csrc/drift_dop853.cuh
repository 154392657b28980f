// drift_dop853.cuh -- per-thread DOP853 integrator (one particle per thread).
//
// Arithmetic follows galpy's leung_dop853.c as ported in the reference
// (src/integrators/galpy/dop853.rs:316-783): Hairer initial step (:383-417),
// 12-stage step (:425-595), Hairer error norm (:597-619), controller with
// safe = 0.9, facc1 = 1/0.333, facc2 = 1/6, beta = 0 (:621-624, :765-781),
// FSAL + three extra stages + rcont1..8 on accept (:626-745) and dense output
// of every requested time strictly before t_current (:747-763).  Expressions
// keep the reference's association so that, compiled without multiply-add
// contraction, each stage rounds as the reference does.
//
// The state that outlives a step (y, k1 = f(y), h, t, flags) lives in
// registers; stage vectors are locals of `step` so the compiler can reuse
// their registers across stages.  On accept the eight-term partial sums of
// rcont5..8 must survive the three extra stages: in registers, or for the
// heavy forces (whose kernels have fewer registers per thread) parked in
// this thread's column of a shared-memory tile (RcontPark).
//
// DRIFT_EXACT_ARITH (set by the including translation unit): 1 keeps every
// division of the reference's error norm; 0 multiplies by one reciprocal per
// component instead.
#pragma once

#include <type_traits>

#include "drift_common.cuh"
#include "drift_composite.cuh"

#ifndef DRIFT_EXACT_ARITH
#define DRIFT_EXACT_ARITH 1
#endif

namespace drift {
namespace dop853c {
constexpr double UROUND = 2.3e-16;
constexpr double A21 = 5.26001519587677318785587544488e-2;
constexpr double A31 = 1.97250569845378994544595329183e-2;
constexpr double A32 = 5.91751709536136983633785987549e-2;
constexpr double A41 = 2.95875854768068491816892993775e-2;
constexpr double A43 = 8.87627564304205475450678981324e-2;
constexpr double A51 = 2.41365134159266685502369798665e-1;
constexpr double A53 = -8.84549479328286085344864962717e-1;
constexpr double A54 = 9.24834003261792003115737966543e-1;
constexpr double A61 = 3.7037037037037037037037037037e-2;
constexpr double A64 = 1.70828608729473871279604482173e-1;
constexpr double A65 = 1.25467687566822425016691814123e-1;
constexpr double A71 = 3.7109375e-2;
constexpr double A74 = 1.70252211019544039314978060272e-1;
constexpr double A75 = 6.02165389804559606850219397283e-2;
constexpr double A76 = -1.7578125e-2;
constexpr double A81 = 3.70920001185047927108779319836e-2;
constexpr double A84 = 1.70383925712239993810214054705e-1;
constexpr double A85 = 1.07262030446373284651809199168e-1;
constexpr double A86 = -1.53194377486244017527936158236e-2;
constexpr double A87 = 8.27378916381402288758473766002e-3;
constexpr double A91 = 6.24110958716075717114429577812e-1;
constexpr double A94 = -3.36089262944694129406857109825e0;
constexpr double A95 = -8.68219346841726006818189891453e-1;
constexpr double A96 = 2.75920996994467083049415600797e1;
constexpr double A97 = 2.01540675504778934086186788979e1;
constexpr double A98 = -4.34898841810699588477366255144e1;
constexpr double A101 = 4.77662536438264365890433908527e-1;
constexpr double A104 = -2.48811461997166764192642586468e0;
constexpr double A105 = -5.90290826836842996371446475743e-1;
constexpr double A106 = 2.12300514481811942347288949897e1;
constexpr double A107 = 1.52792336328824235832596922938e1;
constexpr double A108 = -3.32882109689848629194453265587e1;
constexpr double A109 = -2.03312017085086261358222928593e-2;
constexpr double A111 = -9.3714243008598732571704021658e-1;
constexpr double A114 = 5.18637242884406370830023853209e0;
constexpr double A115 = 1.09143734899672957818500254654e0;
constexpr double A116 = -8.14978701074692612513997267357e0;
constexpr double A117 = -1.85200656599969598641566180701e1;
constexpr double A118 = 2.27394870993505042818970056734e1;
constexpr double A119 = 2.49360555267965238987089396762e0;
constexpr double A1110 = -3.0467644718982195003823669022e0;
constexpr double A121 = 2.27331014751653820792359768449e0;
constexpr double A124 = -1.05344954667372501984066689879e1;
constexpr double A125 = -2.00087205822486249909675718444e0;
constexpr double A126 = -1.79589318631187989172765950534e1;
constexpr double A127 = 2.79488845294199600508499808837e1;
constexpr double A128 = -2.85899827713502369474065508674e0;
constexpr double A129 = -8.87285693353062954433549289258e0;
constexpr double A1210 = 1.23605671757943030647266201528e1;
constexpr double A1211 = 6.43392746015763530355970484046e-1;
constexpr double A141 = 5.61675022830479523392909219681e-2;
constexpr double A147 = 2.53500210216624811088794765333e-1;
constexpr double A148 = -2.46239037470802489917441475441e-1;
constexpr double A149 = -1.24191423263816360469010140626e-1;
constexpr double A1410 = 1.5329179827876569731206322685e-1;
constexpr double A1411 = 8.20105229563468988491666602057e-3;
constexpr double A1412 = 7.56789766054569976138603589584e-3;
constexpr double A1413 = -8.298e-3;
constexpr double A151 = 3.18346481635021405060768473261e-2;
constexpr double A156 = 2.83009096723667755288322961402e-2;
constexpr double A157 = 5.35419883074385676223797384372e-2;
constexpr double A158 = -5.49237485713909884646569340306e-2;
constexpr double A1511 = -1.08347328697249322858509316994e-4;
constexpr double A1512 = 3.82571090835658412954920192323e-4;
constexpr double A1513 = -3.40465008687404560802977114492e-4;
constexpr double A1514 = 1.41312443674632500278074618366e-1;
constexpr double A161 = -4.28896301583791923408573538692e-1;
constexpr double A166 = -4.69762141536116384314449447206e0;
constexpr double A167 = 7.68342119606259904184240953878e0;
constexpr double A168 = 4.06898981839711007970213554331e0;
constexpr double A169 = 3.56727187455281109270669543021e-1;
constexpr double A1613 = -1.39902416515901462129418009734e-3;
constexpr double A1614 = 2.9475147891527723389556272149e0;
constexpr double A1615 = -9.15095847217987001081870187138e0;
constexpr double B1 = 5.42937341165687622380535766363e-2;
constexpr double B6 = 4.45031289275240888144113950566;
constexpr double B7 = 1.89151789931450038304281599044;
constexpr double B8 = -5.8012039600105847814672114227;
constexpr double B9 = 3.1116436695781989440891606237e-1;
constexpr double B10 = -1.52160949662516078556178806805e-1;
constexpr double B11 = 2.01365400804030348374776537501e-1;
constexpr double B12 = 4.47106157277725905176885569043e-2;
constexpr double BHH1 = 0.244094488188976377952755905512;
constexpr double BHH2 = 0.733846688281611857341361741547;
constexpr double BHH3 = 0.220588235294117647058823529412e-1;
constexpr double D41 = -0.84289382761090128651353491142e1;
constexpr double D46 = 0.56671495351937776962531783590;
constexpr double D47 = -0.30689499459498916912797304727e1;
constexpr double D48 = 0.23846676565120698287728149680e1;
constexpr double D49 = 0.21170345824450282767155149946e1;
constexpr double D410 = -0.87139158377797299206789907490;
constexpr double D411 = 0.22404374302607882758541771650e1;
constexpr double D412 = 0.63157877876946881815570249290;
constexpr double D413 = -0.88990336451333310820698117400e-1;
constexpr double D414 = 0.18148505520854727256656404962e2;
constexpr double D415 = -0.91946323924783554000451984436e1;
constexpr double D416 = -0.44360363875948939664310572000e1;
constexpr double D51 = 0.10427508642579134603413151009e2;
constexpr double D56 = 0.24228349177525818288430175319e3;
constexpr double D57 = 0.16520045171727028198505394887e3;
constexpr double D58 = -0.37454675472269020279518312152e3;
constexpr double D59 = -0.22113666853125306036270938578e2;
constexpr double D510 = 0.77334326684722638389603898808e1;
constexpr double D511 = -0.30674084731089398182061213626e2;
constexpr double D512 = -0.93321305264302278729567221706e1;
constexpr double D513 = 0.15697238121770843886131091075e2;
constexpr double D514 = -0.31139403219565177677282850411e2;
constexpr double D515 = -0.93529243588444783865713862664e1;
constexpr double D516 = 0.35816841486394083752465898540e2;
constexpr double D61 = 0.19985053242002433820987653617e2;
constexpr double D66 = -0.38703730874935176555105901742e3;
constexpr double D67 = -0.18917813819516756882830838328e3;
constexpr double D68 = 0.52780815920542364900561016686e3;
constexpr double D69 = -0.11573902539959630126141871134e2;
constexpr double D610 = 0.68812326946963000169666922661e1;
constexpr double D611 = -0.10006050966910838403183860980e1;
constexpr double D612 = 0.77771377980534432092869265740;
constexpr double D613 = -0.27782057523535084065932004339e1;
constexpr double D614 = -0.60196695231264120758267380846e2;
constexpr double D615 = 0.84320405506677161018159903784e2;
constexpr double D616 = 0.11992291136182789328035130030e2;
constexpr double D71 = -0.25693933462703749003312586129e2;
constexpr double D76 = -0.15418974869023643374053993627e3;
constexpr double D77 = -0.23152937917604549567536039109e3;
constexpr double D78 = 0.35763911791061412378285349910e3;
constexpr double D79 = 0.93405324183624310003907691704e2;
constexpr double D710 = -0.37458323136451633156875139351e2;
constexpr double D711 = 0.10409964950896230045147246184e3;
constexpr double D712 = 0.29840293426660503123344363579e2;
constexpr double D713 = -0.43533456590011143754432175058e2;
constexpr double D714 = 0.96324553959188282948394950600e2;
constexpr double D715 = -0.39177261675615439165231486172e2;
constexpr double D716 = -0.14972683625798562581422125276e3;
constexpr double ER1 = 0.1312004499419488073250102996e-1;
constexpr double ER6 = -0.1225156446376204440720569753e1;
constexpr double ER7 = -0.4957589496572501915214079952;
constexpr double ER8 = 0.1664377182454986536961530415e1;
constexpr double ER9 = -0.3503288487499736816886487290;
constexpr double ER10 = 0.3341791187130174790297318841;
constexpr double ER11 = 0.8192320648511571246570742613e-1;
constexpr double ER12 = -0.2235530786388629525884427845e-1;
// Stage times c_i (the node of stage i is t + c_i h).
constexpr double C2 = 0.526001519587677318785587544488e-1;
constexpr double C3 = 0.789002279381515978178381316732e-1;
constexpr double C4 = 0.118350341907227396726757197510;
constexpr double C5 = 0.281649658092772603273242802490;
constexpr double C6 = 0.333333333333333333333333333333;
constexpr double C7 = 0.25;
constexpr double C8 = 0.307692307692307692307692307692;
constexpr double C9 = 0.651282051282051282051282051282;
constexpr double C10 = 0.6;
constexpr double C11 = 0.857142857142857142857142857142;
constexpr double C14 = 0.1;
constexpr double C15 = 0.2;
constexpr double C16 = 0.777777777777777777777777777778;
constexpr double SAFE = 0.9;
constexpr double FACC1 = 1.0 / 0.333;
constexpr double FACC2 = 1.0 / 6.0;
}  // namespace dop853c

// Consecutive non-finite error estimates after which a particle is stopped
// with DRIFT_PARTICLE_NONFINITE.  The reference keeps rejecting at the floor
// step h = 1e3 * UROUND forever in that situation.
constexpr int DOP853_NONFINITE_LIMIT = 64;


// Potentials whose force is large enough that the accept branch evaluates
// its three extra stages from one call site instead of three inlined copies.
template <class Pot>
__host__ __device__ constexpr bool compact_extra_stages()
{
    return std::is_same<Pot, Bovy>::value || std::is_same<Pot, Composite>::value;
}

// Where the eight-term partial sums of rcont5..8 wait out the three extra
// stages of an accepted step.  The heavy forces' kernels run three blocks of
// 128 per SM (168 registers) and park them in this thread's column of a
// shared-memory tile; the others run two blocks (up to 255 registers), which
// hold them in registers (the Plummer workload: 67.2 against 70.2 ms per pass).
struct RcontPark {
    volatile double *p;
    int stride;
    __device__ __forceinline__ void put(int j, int i, double v) { p[(j * 6 + i) * stride] = v; }
    __device__ __forceinline__ double get(int j, int i) const { return p[(j * 6 + i) * stride]; }
};
struct RcontRegs {
    double v[24];
    __device__ __forceinline__ void put(int j, int i, double x) { v[j * 6 + i] = x; }
    __device__ __forceinline__ double get(int j, int i) const { return v[j * 6 + i]; }
};

template <class Pot>
struct Dop853Lane {
    double y[6];   // current solution (y0 in the reference)
    double k1[6];  // f(y), carried across steps (FSAL)
    double h;
    double t_cur;
    double hmax;
    double pos_neg;
    int32_t next;         // finished_user_t_ii
    double t_next;        // output time next + 1 (valid while next < nt - 1)
    int32_t reject;
    int32_t nonfinite_run;
    bool done;

    // a = f(t, q) = (v, F(t, x)); stationary potentials ignore t.
    __device__ __forceinline__ void rhs(const Pot &pot, double t, const double *q, double *a) const
    {
        a[0] = q[3];
        a[1] = q[4];
        a[2] = q[5];
        force_at(pot, t, q[0], q[1], q[2], a[3], a[4], a[5]);
    }

    // dop853.rs:340-424: tolerances, Hairer's initial step, bookkeeping.
    // Writes y0 as output sample 0.
    template <class Out>
    __device__ __forceinline__ void begin(const Pot &pot, const double *y0, const Grid &grid,
                                          double rtol, double atol, Out &out)
    {
        using namespace dop853c;
#pragma unroll
        for (int i = 0; i < 6; i++) y[i] = y0[i];
        out.write(0, y);
        double t0 = grid.at(0);
        hmax = grid.at(grid.nt - 1) - t0;
        pos_neg = custom_sign(1.0, hmax);
        done = (grid.nt < 2);

        rhs(pot, t0, y, k1);
        double dnf = 0.0, dny = 0.0;
#pragma unroll
        for (int i = 0; i < 6; i++) {
            double sk = atol + rtol * fabs(y[i]);
            double sqr = k1[i] / sk;
            dnf += sqr * sqr;
            sqr = y[i] / sk;
            dny += sqr * sqr;
        }
        double hh = custom_sign(c_min(sqrt(dny / dnf) * 0.01, fabs(hmax)), pos_neg);
        double k2[6], k3[6];
#pragma unroll
        for (int i = 0; i < 6; i++) k3[i] = y[i] + hh * k1[i];
        rhs(pot, t0 + hh, k3, k2);
        double der2 = 0.0;
#pragma unroll
        for (int i = 0; i < 6; i++) {
            double sk = atol + rtol * fabs(y[i]);
            double sqr = (k2[i] - k1[i]) / sk;
            der2 += sqr * sqr;
        }
        der2 = sqrt(der2) / hh;
        double der12 = c_max(fabs(der2), sqrt(dnf));
        double h1 = unit_root8(0.01 / der12);
        h = custom_sign(c_min(100.0 * fabs(hh), c_min(fabs(h1), fabs(hmax))), pos_neg);
        reject = 0;
        next = 0;
        t_next = grid.nt > 1 ? grid.at(1) : 0.0;
        nonfinite_run = 0;
        t_cur = t0;
    }

    // One step attempt (dop853.rs:425-782).  Returns true when accepted.
    // `park` is this thread's column of a [24][blockDim.x] shared tile.
    // TAPE: an accepted step also writes (t_old, h, y_old[6]) to tape_row
    // (when not NULL) and h to h_slot (when not NULL).
    template <bool TAPE = false, class Out>
    __device__ __forceinline__ bool step(const Pot &pot, const Grid &grid, double rtol,
                                         double atol, Out &out, volatile double *park,
                                         double *tape_row = nullptr, double *h_slot = nullptr,
                                         bool sparse_output = false)
    {
        using namespace dop853c;
        const int RCONT_STRIDE = blockDim.x;
        h = pos_neg * c_max(fabs(h), 1e3 * UROUND);
        double yy1[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], k8[6], k9[6], k10[6];

#pragma unroll
        for (int i = 0; i < 6; i++) yy1[i] = y[i] + h * A21 * k1[i];
        rhs(pot, t_cur + C2 * h, yy1, k2);
#pragma unroll
        for (int i = 0; i < 6; i++) yy1[i] = y[i] + h * (A31 * k1[i] + A32 * k2[i]);
        rhs(pot, t_cur + C3 * h, yy1, k3);
#pragma unroll
        for (int i = 0; i < 6; i++) yy1[i] = y[i] + h * (A41 * k1[i] + A43 * k3[i]);
        rhs(pot, t_cur + C4 * h, yy1, k4);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A51 * k1[i] + A53 * k3[i] + A54 * k4[i]);
        rhs(pot, t_cur + C5 * h, yy1, k5);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A61 * k1[i] + A64 * k4[i] + A65 * k5[i]);
        rhs(pot, t_cur + C6 * h, yy1, k6);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A71 * k1[i] + A74 * k4[i] + A75 * k5[i] + A76 * k6[i]);
        rhs(pot, t_cur + C7 * h, yy1, k7);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] +
                     h * (A81 * k1[i] + A84 * k4[i] + A85 * k5[i] + A86 * k6[i] + A87 * k7[i]);
        rhs(pot, t_cur + C8 * h, yy1, k8);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A91 * k1[i] + A94 * k4[i] + A95 * k5[i] + A96 * k6[i] +
                                 A97 * k7[i] + A98 * k8[i]);
        rhs(pot, t_cur + C9 * h, yy1, k9);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A101 * k1[i] + A104 * k4[i] + A105 * k5[i] + A106 * k6[i] +
                                 A107 * k7[i] + A108 * k8[i] + A109 * k9[i]);
        rhs(pot, t_cur + C10 * h, yy1, k10);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A111 * k1[i] + A114 * k4[i] + A115 * k5[i] + A116 * k6[i] +
                                 A117 * k7[i] + A118 * k8[i] + A119 * k9[i] + A1110 * k10[i]);
        rhs(pot, t_cur + C11 * h, yy1, k2);
#pragma unroll
        for (int i = 0; i < 6; i++)
            yy1[i] = y[i] + h * (A121 * k1[i] + A124 * k4[i] + A125 * k5[i] + A126 * k6[i] +
                                 A127 * k7[i] + A128 * k8[i] + A129 * k9[i] + A1210 * k10[i] +
                                 A1211 * k2[i]);
        const double t_old = t_cur;
        const double t_new = t_cur + h;
        rhs(pot, t_new, yy1, k3);

#pragma unroll
        for (int i = 0; i < 6; i++) {
            k4[i] = B1 * k1[i] + B6 * k6[i] + B7 * k7[i] + B8 * k8[i] + B9 * k9[i] +
                    B10 * k10[i] + B11 * k2[i] + B12 * k3[i];
            k5[i] = y[i] + h * k4[i];
        }

        double err = 0.0, err2 = 0.0;
#pragma unroll
        for (int i = 0; i < 6; i++) {
            double sk = atol + rtol * c_max(fabs(y[i]), fabs(k5[i]));
#if !DRIFT_EXACT_ARITH
            double inv_sk = fast_rcp(sk);
#endif
            double erri = k4[i] - BHH1 * k1[i] - BHH2 * k9[i] - BHH3 * k3[i];
#if DRIFT_EXACT_ARITH
            double sqr = erri / sk;
#else
            double sqr = erri * inv_sk;
#endif
            err2 += sqr * sqr;
            erri = ER1 * k1[i] + ER6 * k6[i] + ER7 * k7[i] + ER8 * k8[i] + ER9 * k9[i] +
                   ER10 * k10[i] + ER11 * k2[i] + ER12 * k3[i];
#if DRIFT_EXACT_ARITH
            sqr = erri / sk;
#else
            sqr = erri * inv_sk;
#endif
            err += sqr * sqr;
        }
        double deno = err + 0.01 * err2;
        if (deno <= 0.0) deno = 1.0;
#if DRIFT_EXACT_ARITH
        err = fabs(h) * err * sqrt(1.0 / (deno * 6.0));
#else
        // the contraction unit divides by reciprocal estimates (a few ulps)
        err = fabs(h) * err * rsqrt(deno * 6.0);
#endif

        // fac11 = err^expo1 with expo1 = 1/8; beta = 0 makes the facold
        // factor pow(facold, 0) = 1.
        double fac11 = unit_root8(err);
#if DRIFT_EXACT_ARITH
        double fac = c_max(FACC2, c_min(FACC1, fac11 / SAFE));
        double hnew = h / fac;
#else
        constexpr double INV_SAFE = 1.0 / SAFE;
        double fac = c_max(FACC2, c_min(FACC1, fac11 * INV_SAFE));
        double hnew = h * fast_rcp(fac);
#endif

        if (err <= 1.0) {
            nonfinite_run = 0;
            if (TAPE) {
                if (tape_row) {
                    double2 *row = reinterpret_cast<double2 *>(tape_row);
                    row[0] = make_double2(t_old, h);
                    row[1] = make_double2(y[0], y[1]);
                    row[2] = make_double2(y[2], y[3]);
                    row[3] = make_double2(y[4], y[5]);
                }
                if (h_slot) *h_slot = h;
            }
            rhs(pot, t_new, k5, k4);  // FSAL: k4 = f(t_new, y_new)

            // The three extra stages and rcont1..8 serve only the dense output
            // of this step.  On sparse grids (a launch-uniform flag) a lane
            // with no requested time in (t_old, t_new) skips them; emitted
            // samples are unchanged.
            const bool skip_dense =
                sparse_output && !(next < grid.nt - 1 && pos_neg * t_next < pos_neg * t_new);
            if (!skip_dense) {
                std::conditional_t<compact_extra_stages<Pot>(), RcontPark, RcontRegs> parked;
                if constexpr (compact_extra_stages<Pot>()) parked = RcontPark{park, RCONT_STRIDE};

#pragma unroll
                for (int i = 0; i < 6; i++) {
                    parked.put(0, i,
                        D41 * k1[i] + D46 * k6[i] + D47 * k7[i] + D48 * k8[i] + D49 * k9[i] +
                        D410 * k10[i] + D411 * k2[i] + D412 * k3[i]);
                    parked.put(1, i,
                        D51 * k1[i] + D56 * k6[i] + D57 * k7[i] + D58 * k8[i] + D59 * k9[i] +
                        D510 * k10[i] + D511 * k2[i] + D512 * k3[i]);
                    parked.put(2, i,
                        D61 * k1[i] + D66 * k6[i] + D67 * k7[i] + D68 * k8[i] + D69 * k9[i] +
                        D610 * k10[i] + D611 * k2[i] + D612 * k3[i]);
                    parked.put(3, i,
                        D71 * k1[i] + D76 * k6[i] + D77 * k7[i] + D78 * k8[i] + D79 * k9[i] +
                        D710 * k10[i] + D711 * k2[i] + D712 * k3[i]);
                }
                if constexpr (compact_extra_stages<Pot>()) {
                    // Stages 14..16 around one force call site: for the heavy
                    // forces the step body, inlined once per force evaluation,
                    // otherwise overflows the instruction cache.
#pragma unroll 1
                    for (int e = 14; e <= 16; e++) {
                        double tq;
                        if (e == 14) {
#pragma unroll
                            for (int i = 0; i < 6; i++)
                                yy1[i] = y[i] + h * (A141 * k1[i] + A147 * k7[i] + A148 * k8[i] +
                                                     A149 * k9[i] + A1410 * k10[i] + A1411 * k2[i] +
                                                     A1412 * k3[i] + A1413 * k4[i]);
                            tq = t_old + C14 * h;
                        } else if (e == 15) {
#pragma unroll
                            for (int i = 0; i < 6; i++)
                                yy1[i] = y[i] + h * (A151 * k1[i] + A156 * k6[i] + A157 * k7[i] +
                                                     A158 * k8[i] + A1511 * k2[i] + A1512 * k3[i] +
                                                     A1513 * k4[i] + A1514 * k10[i]);
                            tq = t_old + C15 * h;
                        } else {
#pragma unroll
                            for (int i = 0; i < 6; i++)
                                yy1[i] = y[i] + h * (A161 * k1[i] + A166 * k6[i] + A167 * k7[i] +
                                                     A168 * k8[i] + A169 * k9[i] + A1613 * k4[i] +
                                                     A1614 * k10[i] + A1615 * k2[i]);
                            tq = t_old + C16 * h;
                        }
                        double f[6];
                        rhs(pot, tq, yy1, f);
#pragma unroll
                        for (int i = 0; i < 6; i++) {
                            if (e == 14)
                                k10[i] = f[i];
                            else if (e == 15)
                                k2[i] = f[i];
                            else
                                k3[i] = f[i];
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 6; i++)
                        yy1[i] = y[i] + h * (A141 * k1[i] + A147 * k7[i] + A148 * k8[i] + A149 * k9[i] +
                                             A1410 * k10[i] + A1411 * k2[i] + A1412 * k3[i] +
                                             A1413 * k4[i]);
                    rhs(pot, t_old + C14 * h, yy1, k10);
#pragma unroll
                    for (int i = 0; i < 6; i++)
                        yy1[i] = y[i] + h * (A151 * k1[i] + A156 * k6[i] + A157 * k7[i] + A158 * k8[i] +
                                             A1511 * k2[i] + A1512 * k3[i] + A1513 * k4[i] +
                                             A1514 * k10[i]);
                    rhs(pot, t_old + C15 * h, yy1, k2);
#pragma unroll
                    for (int i = 0; i < 6; i++)
                        yy1[i] = y[i] + h * (A161 * k1[i] + A166 * k6[i] + A167 * k7[i] + A168 * k8[i] +
                                             A169 * k9[i] + A1613 * k4[i] + A1614 * k10[i] +
                                             A1615 * k2[i]);
                    rhs(pot, t_old + C16 * h, yy1, k3);
                }

                // rcont1..4 (dop853.rs:636-642) need only y, y_new, k1 and k4,
                // so they are formed here, after the extra stages.
                double r1[6], r2[6], r3[6], r4[6], r5[6], r6[6], r7[6], r8[6];
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    r5[i] = h * (parked.get(0, i) + D413 * k4[i] + D414 * k10[i] +
                                 D415 * k2[i] + D416 * k3[i]);
                    r6[i] = h * (parked.get(1, i) + D513 * k4[i] + D514 * k10[i] +
                                 D515 * k2[i] + D516 * k3[i]);
                    r7[i] = h * (parked.get(2, i) + D613 * k4[i] + D614 * k10[i] +
                                 D615 * k2[i] + D616 * k3[i]);
                    r8[i] = h * (parked.get(3, i) + D713 * k4[i] + D714 * k10[i] +
                                 D715 * k2[i] + D716 * k3[i]);
                    r1[i] = y[i];
                    double ydiff = k5[i] - y[i];
                    r2[i] = ydiff;
                    double bspl = h * k1[i] - ydiff;
                    r3[i] = bspl;
                    r4[i] = ydiff - h * k4[i] - bspl;
                }

                // Dense output of every requested time strictly before t_current.
#if !DRIFT_EXACT_ARITH
                const double inv_h = fast_rcp(h);
#endif
                // The next output time is formed once per emitted sample
                // (t_next), not once per step: for per-particle grids that
                // is a division (OutputGrid::sample) saved in every step.
                while (next < grid.nt - 1) {
                    const double tk = t_next;
                    if (!(pos_neg * tk < pos_neg * t_new)) break;
#if DRIFT_EXACT_ARITH
                    double s = (tk - t_old) / h;
#else
                    double s = (tk - t_old) * inv_h;
#endif
                    double s1 = 1.0 - s;
                    double yy[6];
#pragma unroll
                    for (int i = 0; i < 6; i++)
                        yy[i] = r1[i] +
                                s * (r2[i] +
                                     s1 * (r3[i] +
                                           s * (r4[i] +
                                                s1 * (r5[i] + s * (r6[i] + s1 * (r7[i] + s * r8[i]))))));
                    out.write(next + 1, yy);
                    next += 1;
                    if (next < grid.nt - 1) t_next = grid.at(next + 1);
                }
            }
#pragma unroll
            for (int i = 0; i < 6; i++) {
                k1[i] = k4[i];
                y[i] = k5[i];
            }
            t_cur = t_new;
            done = (next >= grid.nt - 1);

            hnew = fabs(hnew) > fabs(hmax) ? pos_neg * hmax : hnew;
            if (reject != 0) hnew = pos_neg * c_min(fabs(hnew), fabs(h));
            reject = 0;
            h = hnew;
            return true;
        }
#if DRIFT_EXACT_ARITH
        hnew = h / c_min(FACC1, fac11 / SAFE);
#else
        hnew = h * fast_rcp(c_min(FACC1, fac11 * INV_SAFE));
#endif
        reject = 1;
        nonfinite_run = isfinite(err) ? 0 : nonfinite_run + 1;
        h = hnew;
        return false;
    }
};

}  // namespace drift
