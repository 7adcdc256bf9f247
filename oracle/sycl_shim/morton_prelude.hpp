// Forced-include prelude for checker builds of the reference's Morton configuration.
// TEST INFRASTRUCTURE ONLY.
//
// With SFC_TYPE_MORTON the reference does not compile as shipped: src/hlbvh.hpp names
// uint128_t (55, 67, 100) and _DIST_SHIFT (1044-1045), which only sfc.peano_hilbert.hpp
// declares, and build_tree / build_bvh name KEY_TOTAL_BITS and to_sort_key (858, 2212).
// These declarations give them the values the Peano-Hilbert header gives for
// floating-point coordinates: _DIST_SHIFT = 0 (sfc.peano_hilbert.hpp:192), a 63-bit key
// (3 x 21 bits), and an identity sort key for the single-word Morton key.
#pragma once
#include <cstdint>
namespace fasttree {
struct uint128_t {
    uint64_t lo = 0, hi = 0;
    constexpr uint128_t() = default;
    constexpr uint128_t(uint64_t h, uint64_t l) : lo(l), hi(h) {}
    constexpr uint128_t(uint64_t v) : lo(v), hi(0) {}
};
constexpr int        _DIST_SHIFT    = 0;
static constexpr int KEY_TOTAL_BITS = 63;
inline uint64_t      to_sort_key(uint64_t k) { return k; }
} // namespace fasttree
