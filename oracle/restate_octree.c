/* restate_octree.c — TEST INFRASTRUCTURE ONLY: the oracle's restatement of the
 * reference's integer octree maps.
 *
 * Morton keys follow core/include/nabla/mesh/morton.hpp:19-48 (21 bits per
 * axis, x in bit 0, y in bit 1, z in bit 2 of each triple). The bit spreading
 * here is a plain per-bit loop (a different method from the reference's
 * magic-number shifts) so that the two are independent checks of one map.
 */
#include "orc.h"

uint64_t orc_morton_encode(uint32_t x, uint32_t y, uint32_t z) {
  uint64_t code = 0;
  for (int b = 0; b < 21; ++b) {
    code |= (uint64_t)((x >> b) & 1u) << (3 * b);
    code |= (uint64_t)((y >> b) & 1u) << (3 * b + 1);
    code |= (uint64_t)((z >> b) & 1u) << (3 * b + 2);
  }
  return code;
}

void orc_morton_decode(uint64_t code, uint32_t* x, uint32_t* y, uint32_t* z) {
  uint32_t a = 0, b = 0, c = 0;
  for (int k = 0; k < 21; ++k) {
    a |= (uint32_t)((code >> (3 * k)) & 1u) << k;
    b |= (uint32_t)((code >> (3 * k + 1)) & 1u) << k;
    c |= (uint32_t)((code >> (3 * k + 2)) & 1u) << k;
  }
  *x = a;
  *y = b;
  *z = c;
}
