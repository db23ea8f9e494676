// Minimal stand-in for the one Boost.Sort entry point the reference's
// format builders call (boost::sort::sample_sort). Boost is not installed in
// this image. The stand-in is a STABLE sort, which makes the reference's
// otherwise unstable parallel sort deterministic: ties keep their prior order.
// This header is test infrastructure for building the reference as an oracle.
#pragma once
#include <algorithm>
namespace boost { namespace sort {
template <class It, class Cmp>
inline void sample_sort(It first, It last, Cmp cmp) { std::stable_sort(first, last, cmp); }
template <class It>
inline void sample_sort(It first, It last) { std::stable_sort(first, last); }
} }
