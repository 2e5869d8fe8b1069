// Stand-in for boost::random::mt19937_64 (an unused member of
// CombPopulationControl, population/CombPopulationControl.hpp:31).
#ifndef STORM_SHIM_BOOST_MT_HPP
#define STORM_SHIM_BOOST_MT_HPP
#include <random>
namespace boost { namespace random { using mt19937_64 = std::mt19937_64; }}
#endif
