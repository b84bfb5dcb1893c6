// nb_morton.h — 3-D Morton keys, 21 bits per axis, x in the lowest bit of each
// triple: the same key as core/include/nabla/mesh/morton.hpp:19-48 (the map
// must be bit-exact). Implemented with a byte-wise spread table instead of the
// reference's shift-mask cascade.
#pragma once
#include <cstdint>

namespace nb {

// Spread the 8 bits of a byte so bit b lands at bit 3b (24-bit result).
__host__ __device__ constexpr uint32_t spread_byte3(uint32_t v) {
  uint32_t r = 0;
  for (int b = 0; b < 8; ++b) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

__host__ __device__ inline uint64_t morton_spread3(uint32_t a) {
  a &= 0x1fffffu;
  return static_cast<uint64_t>(spread_byte3(a & 0xffu)) |
         (static_cast<uint64_t>(spread_byte3((a >> 8) & 0xffu)) << 24) |
         (static_cast<uint64_t>(spread_byte3((a >> 16) & 0x1fu)) << 48);
}

__host__ __device__ inline uint32_t morton_gather3(uint64_t x) {
  uint32_t r = 0;
  for (int b = 0; b < 21; ++b) r |= static_cast<uint32_t>((x >> (3 * b)) & 1u) << b;
  return r;
}

__host__ __device__ inline uint64_t morton_encode(uint32_t x, uint32_t y, uint32_t z) {
  return morton_spread3(x) | (morton_spread3(y) << 1) | (morton_spread3(z) << 2);
}

__host__ __device__ inline void morton_decode(uint64_t c, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = morton_gather3(c);
  y = morton_gather3(c >> 1);
  z = morton_gather3(c >> 2);
}

}  // namespace nb
