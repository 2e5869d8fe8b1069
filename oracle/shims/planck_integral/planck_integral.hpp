// Stand-in for the `planck_integral` module STORM clones unpinned
// (install_deps.sh:58).  Normalised Planck integral
//     planck_integral(a, b) = 15/pi^4 * int_a^b x^3 / (e^x - 1) dx,
// evaluated with the two classical series used by Clark (1987): the
// Bernoulli-number expansion for small x and the exponential tail series
//     int_x^inf t^3/(e^t-1) dt = sum_n e^{-n x} (x^3/n + 3x^2/n^2 + 6x/n^3 + 6/n^4)
// for large x.  Written for this project from those published series.
#ifndef STORM_SHIM_PLANCK_INTEGRAL_HPP
#define STORM_SHIM_PLANCK_INTEGRAL_HPP
#include <cmath>
namespace planck_integral {
namespace detail {
constexpr double kPi = 3.14159265358979323846;
inline double norm() { return 15.0 / (kPi * kPi * kPi * kPi); }
// int_0^x t^3/(e^t-1) dt = sum_k B_k x^(k+3) / (k! (k+3)), valid for x < 2 pi.
inline double small_series(double x) {
    static const double B[] = {1.0, -0.5, 1.0 / 6.0, 0.0, -1.0 / 30.0, 0.0, 1.0 / 42.0, 0.0, -1.0 / 30.0, 0.0,
                               5.0 / 66.0, 0.0, -691.0 / 2730.0, 0.0, 7.0 / 6.0, 0.0, -3617.0 / 510.0, 0.0,
                               43867.0 / 798.0, 0.0, -174611.0 / 330.0};
    double sum = 0.0, xp = x * x * x, fact = 1.0;
    for (int k = 0; k <= 20; ++k) {
        if (k > 0) { fact *= k; xp *= x; }
        if (B[k] != 0.0) sum += B[k] * xp / (fact * (k + 3));
    }
    return sum;
}
inline double tail_series(double x) {
    double sum = 0.0;
    for (int n = 1; n < 100000; ++n) {
        double e = std::exp(-n * x);
        if (e == 0.0) break;
        double dn = n;
        double term = e * (x * x * x / dn + 3.0 * x * x / (dn * dn) + 6.0 * x / (dn * dn * dn) + 6.0 / (dn * dn * dn * dn));
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}
constexpr double kSwitch = 0.5;
inline double cumulative(double x) {   // 15/pi^4 * int_0^x
    if (!(x > 0.0)) return 0.0;
    if (x < kSwitch) return norm() * small_series(x);
    return 1.0 - norm() * tail_series(x);
}
} // namespace detail
inline double planck_integral(double a, double b) {
    if (a >= detail::kSwitch && b >= detail::kSwitch)
        return detail::norm() * (detail::tail_series(a) - detail::tail_series(b));
    return detail::cumulative(b) - detail::cumulative(a);
}
} // namespace planck_integral
#endif
