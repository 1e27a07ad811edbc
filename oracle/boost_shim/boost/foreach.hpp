// Test infrastructure (oracle): BOOST_FOREACH stand-in (C++11 range-for).
// Self-written; NOT Boost source.
#ifndef ORACLE_BOOST_SHIM_FOREACH_HPP
#define ORACLE_BOOST_SHIM_FOREACH_HPP
#include <cassert>
#include <climits>
#include <cstring>
#include <algorithm>
#define BOOST_FOREACH(VAR, COL) for (VAR : COL)
#endif
