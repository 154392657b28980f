// drift_bulge_table.h -- host construction of the bulge's incomplete-gamma
// table (layout and evaluation in drift_potentials.cuh, bulge_lower_gamma).
//
// gamma(s, x) = x^s E(x) with E(x) = int_0^1 u^(s-1) e^(-x u) du, entire.
// Its derivatives are E^(k)(x) = (-1)^k I_k(x) with
//   I_k(x) = int_0^1 u^(s-1+k) e^(-x u) du = gamma(s+k, x) / x^(s+k)
//          = e^-x sum_n x^n / ((s+k) (s+k+1) ... (s+k+n)),
// a series of positive terms (no cancellation).  Piece j holds the Taylor
// coefficients E^(k)(c) / k!, k = 0..deg, around the centre c = 2j + 1,
// computed in x87 extended precision (64-bit significand).
#pragma once

#include <cmath>

namespace drift {

inline void fill_bulge_table_impl(double s_in, double *out, int pieces, int deg)
{
    typedef long double ld;
    const ld s = s_in;
    for (int j = 0; j < pieces; j++) {
        const ld c = 2.0L * j + 1.0L;
        const ld e = expl(-c);
        ld fact = 1.0L;
        for (int k = 0; k <= deg; k++) {
            if (k > 0) fact *= k;
            ld term = 1.0L / (s + k), sum = term;
            for (int n = 1; n < 4000; n++) {
                term *= c / (s + k + n);
                sum += term;
                if (term < sum * 1e-22L) break;
            }
            const ld v = e * sum / fact;
            out[j * (deg + 1) + k] = (double)((k & 1) ? -v : v);
        }
    }
}

}  // namespace drift
