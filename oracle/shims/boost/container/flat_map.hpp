// Stand-in for boost::container::flat_map (only find/end/operator[] are used,
// manager/MonteCarloManagerSerial.hpp:46-70).  Ordered-map semantics.
#ifndef STORM_SHIM_BOOST_FLAT_MAP_HPP
#define STORM_SHIM_BOOST_FLAT_MAP_HPP
#include <map>
namespace boost { namespace container {
template <class K, class V> using flat_map = std::map<K, V>;
}} // namespace boost::container
#endif
