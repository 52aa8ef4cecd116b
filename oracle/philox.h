/*
 * philox.h -- TEST INFRASTRUCTURE ONLY (oracle copy).
 *
 * Philox4x32-10, the counter-based generator of Salmon, Moraes, Dror and
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11), restated from
 * the paper: ten rounds of two 32x32->64 multiplications with round-key
 * bumps by the Weyl constants.  The engine has its own copy; tests pin both
 * to the published known-answer vectors.
 *
 * The draws of the effective-domain rebuild are keyed by the replica seed
 * and indexed by (molecule, rebuild number, purpose, word): see
 * mdn_oracle.cpp, which states the layout the engine must follow.
 */
#ifndef MDN_ORACLE_PHILOX_H
#define MDN_ORACLE_PHILOX_H
#include <cmath>
#include <cstdint>

namespace orc {

struct U4 {
  uint32_t v[4];
};

inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * c.v[0];
    uint64_t p1 = (uint64_t)M1 * c.v[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    U4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

/* uniform in (0, 1) from one 32-bit word */
inline double u01(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

/* Box-Muller: two standard normals from two words */
inline void box_muller(uint32_t a, uint32_t b, double* z0, double* z1) {
  double r = std::sqrt(-2.0 * std::log(u01(a)));
  double t = 6.283185307179586 * u01(b);
  *z0 = r * std::cos(t);
  *z1 = r * std::sin(t);
}

}  // namespace orc
#endif
