// Test infrastructure (oracle): a minimal, self-written stand-in for the part of
// Boost's hashing API that the reference's CPU path uses (hash_value over a block
// vector, hash_combine, and a default boost::hash functor).  Boost is not installed
// in this image; this file is NOT Boost source.  Iteration order of hash maps keyed
// with it differs from real Boost, which changes node numbering in the reference's
// decision diagrams but not layer sizes or the enumerated Pareto frontier.
#ifndef ORACLE_BOOST_SHIM_HASH_HPP
#define ORACLE_BOOST_SHIM_HASH_HPP

#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <utility>
#include <vector>

namespace boost {

// 64-bit mixer (splitmix64 finaliser, public domain) used to spread hash bits.
inline std::size_t shim_mix(std::uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return static_cast<std::size_t>(x ^ (x >> 31));
}

template <class T> struct hash;

template <class T> inline std::size_t hash_value(const T &v) { return hash<T>()(v); }

template <class T> inline void hash_combine(std::size_t &seed, const T &v) {
    seed = shim_mix(static_cast<std::uint64_t>(seed) * 31u + hash_value(v));
}

template <class T> struct hash {
    std::size_t operator()(const T &v) const { return std::hash<T>()(v); }
};

template <class T, class A> struct hash<std::vector<T, A>> {
    std::size_t operator()(const std::vector<T, A> &v) const {
        std::size_t seed = v.size();
        for (typename std::vector<T, A>::const_iterator it = v.begin(); it != v.end(); ++it) {
            hash_combine(seed, *it);
        }
        return seed;
    }
};

template <class A, class B> struct hash<std::pair<A, B>> {
    std::size_t operator()(const std::pair<A, B> &p) const {
        std::size_t seed = 0;
        hash_combine(seed, p.first);
        hash_combine(seed, p.second);
        return seed;
    }
};

} // namespace boost

#endif
