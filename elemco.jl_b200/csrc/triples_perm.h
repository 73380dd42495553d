// triples_perm.h — orderings of an element's three indices, shared by the
// (T) energy kernels.
#pragma once

namespace ecg {
namespace dev {

// Permutations s of (0,1,2) in the order (012)(021)(102)(120)(201)(210).
__host__ __device__ constexpr int perm3(int q, int d) {
  return q == 0   ? d
         : q == 1 ? (d == 0 ? 0 : 3 - d)
         : q == 2 ? (d == 2 ? 2 : 1 - d)
         : q == 3 ? (d == 0 ? 1 : d == 1 ? 2 : 0)
         : q == 4 ? (d == 0 ? 2 : d - 1)
                  : 2 - d;
}
__host__ __device__ constexpr int perm3_index(int t0, int t1) {
  return 2 * t0 + (t0 == 0 ? (t1 == 2) : t0 == 1 ? (t1 == 2) : (t1 == 1));
}
// X terms: K at (a,b,c) (a,c,b) (c,b,a) (b,a,c) (c,a,b) (b,c,a), weights 4 -2 -2 -2 1 1
__host__ __device__ constexpr int xp(int r, int d) {
  return r == 0   ? d
         : r == 1 ? (d == 0 ? 0 : 3 - d)
         : r == 2 ? 2 - d
         : r == 3 ? (d == 2 ? 2 : 1 - d)
         : r == 4 ? (d == 0 ? 2 : d - 1)
                  : (d == 2 ? 0 : d + 1);
}
// For the ordering q of an element, the ordering that X term r reads.
__host__ __device__ constexpr int xcomp(int q, int r) {
  return perm3_index(perm3(q, xp(r, 0)), perm3(q, xp(r, 1)));
}
// Parity of ordering q: (012)(120)(201) even, (021)(102)(210) odd.  For an
// element in ordering q the transposed orderings (weight -2) are the three of
// the other parity and the cyclic ones (weight 1) the two others of its own,
// so X_q = 3 k_q + (sum of k over q's parity) - 2 (sum over the other).
__host__ __device__ constexpr int perm3_parity(int q) {
  return ((perm3(q, 0) > perm3(q, 1)) + (perm3(q, 0) > perm3(q, 2)) + (perm3(q, 1) > perm3(q, 2))) & 1;
}
constexpr bool x_parity_rule() {
  for (int q = 0; q < 6; ++q) {
    if (xcomp(q, 0) != q) return false;
    for (int r = 1; r < 6; ++r) {
      const int p = xcomp(q, r);
      if (p == q || (r <= 3) == (perm3_parity(p) == perm3_parity(q))) return false;
    }
  }
  return true;
}
static_assert(x_parity_rule(), "X term orderings follow the parity rule");
// Index of the ordered position pair (x, y), x != y, in [0, 6).
__host__ __device__ constexpr int pair_index(int x, int y) { return 2 * x + (y > x ? y - 1 : y); }


}  // namespace dev
}  // namespace ecg
