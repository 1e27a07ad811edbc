// Test infrastructure (oracle): boost::unordered_map stand-in for building the
// reference's CPU path without Boost.  A thin alias over std::unordered_map whose
// default hasher is the shim's boost::hash (covers std::vector<int> and
// std::pair<int,int> keys).  Self-written; NOT Boost source.
#ifndef ORACLE_BOOST_SHIM_UNORDERED_MAP_HPP
#define ORACLE_BOOST_SHIM_UNORDERED_MAP_HPP

#include <cassert>
#include <climits>
#include <cstring>
#include <algorithm>
#include <unordered_map>

#include "functional/hash.hpp"

namespace boost {
template <class K, class V, class H = boost::hash<K>, class E = std::equal_to<K>>
using unordered_map = std::unordered_map<K, V, H, E>;
} // namespace boost

#endif
