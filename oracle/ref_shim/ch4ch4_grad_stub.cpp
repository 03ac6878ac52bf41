/* Stand-in for the CH4-CH4 2-body gradient polynomial of the reference.
 *
 * The reference declares
 *   poly_2b_A1B4_A1B4_deg4_exp0_v1x::eval(const double a[1345],
 *                                          const double x[45], double g[45])
 * (potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1x.h:82) and lists its source in
 * src/Makefile.am:33, but the file itself is absent from the repository (it is
 * named in .MISSING_LARGE_BLOBS).  The energy-only program
 * eval(a, x) (poly_2b_A1B4_A1B4_deg4_exp0_v1.cpp) is present.
 *
 * The polynomial has total degree 4, so along any single variable x_j it is a
 * polynomial of degree <= 4 in x_j.  The five-point central difference
 *   f'(0) = [f(-2h) - 8 f(-h) + 8 f(h) - f(2h)] / (12 h)
 * is exact for polynomials of degree <= 4 (its truncation term is
 * h^4 f^(5) / 30), so this gives dP/dx_j exactly up to rounding.  The step
 * h = 1/16 is a power of two so that x_j +- h and x_j +- 2h carry no extra
 * representation error beyond the final rounding of the sum.
 *
 * This is test infrastructure for the oracle build only.
 */
#include "potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1x.h"

namespace x2b_A1B4_A1B4_deg4_exp0 {

double poly_2b_A1B4_A1B4_deg4_exp0_v1x::eval(const double a[1345], const double x[45], double g[45]) {
    const double h = 0.0625;
    double xs[45];
    for (int j = 0; j < 45; ++j) xs[j] = x[j];
    for (int j = 0; j < 45; ++j) {
        const double x0 = x[j];
        xs[j] = x0 - 2.0 * h;
        const double fm2 = eval(a, xs);
        xs[j] = x0 - h;
        const double fm1 = eval(a, xs);
        xs[j] = x0 + h;
        const double fp1 = eval(a, xs);
        xs[j] = x0 + 2.0 * h;
        const double fp2 = eval(a, xs);
        xs[j] = x0;
        g[j] = ((fm2 - fp2) + 8.0 * (fp1 - fm1)) / (12.0 * h);
    }
    return eval(a, x);
}

}  // namespace x2b_A1B4_A1B4_deg4_exp0
