// drift_bulge_table.h -- host construction of the bulge's incomplete-gamma
// table (layout and evaluation in drift_potentials.cuh, bulge_lower_gamma).
//
// Computed in x87 extended precision (64-bit significand):
//   series coefficients a_n = 1 / (s (s+1) ... (s+n)), n = 0..series_deg;
//   for each centre c = first_centre + 2j the Taylor coefficients of gamma(s, .):
//     coefficient 0 = gamma(s, c) = c^s e^-c sum_n a_n c^n (positive series),
//     coefficient k = f^(k-1)(c) / k!  with f(x) = x^(s-1) e^-x, and by Leibniz
//     f^(m)(x) = e^-x sum_i C(m,i) (-1)^(m-i) g_i x^(s-1-i),
//     g_i = (s-1)(s-2)...(s-i).
#pragma once

#include <cmath>

namespace drift {

inline void fill_bulge_table_impl(double s_in, double *out, int series_deg, int pieces,
                                  int piece_deg, double first_centre)
{
    typedef long double ld;
    const ld s = s_in;
    ld a = 1.0L / s;
    out[0] = (double)a;
    for (int n = 1; n <= series_deg; n++) {
        a /= (s + n);
        out[n] = (double)a;
    }
    double *piece = out + series_deg + 1;
    for (int j = 0; j < pieces; j++) {
        const ld c = (ld)first_centre + 2.0L * j;
        ld term = 1.0L / s, sum = term;
        for (int n = 1; n < 2000; n++) {
            term *= c / (s + n);
            sum += term;
            if (term < sum * 1e-24L) break;
        }
        const ld e = expl(-c);
        double *pc = piece + j * (piece_deg + 1);
        pc[0] = (double)(powl(c, s) * e * sum);
        ld fact = 1.0L;
        for (int k = 1; k <= piece_deg; k++) {
            const int m = k - 1;
            fact *= k;
            ld fm = 0.0L, binom = 1.0L, g = 1.0L;
            for (int i = 0; i <= m; i++) {
                if (i > 0) {
                    binom = binom * (m - i + 1) / i;
                    g *= (s - i);
                }
                const ld sign = ((m - i) & 1) ? -1.0L : 1.0L;
                fm += sign * binom * g * powl(c, s - 1.0L - i);
            }
            pc[k] = (double)(e * fm / fact);
        }
    }
}

}  // namespace drift
