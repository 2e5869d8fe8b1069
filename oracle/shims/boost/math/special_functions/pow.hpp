// Stand-in for Boost.Math's compile-time integer power, written for this project
// (Boost is not installed here).  Exponentiation by squaring with the same
// association as Boost's documented positive_power recursion:
//   pow<2>(x) = x*x, pow<3>(x) = (x*x)*x, pow<4>(x) = (x*x)*(x*x).
// STORM uses pow<3> and pow<4> (radiation/RadiationIMC.hpp:1649, 2058;
// boundary/SideTemperature.hpp:117).
#ifndef STORM_SHIM_BOOST_MATH_POW_HPP
#define STORM_SHIM_BOOST_MATH_POW_HPP
namespace boost { namespace math {
namespace shim_detail {
template <int N, int Odd = N % 2> struct positive_power;
template <> struct positive_power<0, 0> { template <class T> static T result(T) { return T(1); } };
template <int N> struct positive_power<N, 0> {
    template <class T> static T result(T base) { T p = positive_power<N / 2>::result(base); return p * p; }
};
template <int N> struct positive_power<N, 1> {
    template <class T> static T result(T base) {
        if (N == 1) return base;
        T p = positive_power<N / 2>::result(base); return base * p * p;
    }
};
} // namespace shim_detail
template <int N, class T> inline T pow(T base) { return shim_detail::positive_power<N>::result(base); }
}} // namespace boost::math
#endif
