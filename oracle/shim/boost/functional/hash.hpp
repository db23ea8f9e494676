// Minimal stand-in for boost::hash<std::pair<A,B>> used as an unordered_map
// hasher by the reference's tensor classes (never used on the MTTKRP path).
// Test infrastructure for building the reference as an oracle.
#pragma once
#include <cstddef>
#include <functional>
#include <utility>
namespace boost {
template <class T> struct hash : std::hash<T> {};
template <class A, class B> struct hash<std::pair<A, B>> {
  std::size_t operator()(const std::pair<A, B>& p) const {
    std::size_t h = std::hash<A>()(p.first);
    return h ^ (std::hash<B>()(p.second) + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2));
  }
};
}
