// Velocity order and moment basis of the colour-gradient model (host and device).
#pragma once

#include "lbm_internal.h"

namespace lbm {
namespace cg {

// CG velocity order (CG3:188-196): opposite pairs are adjacent (1,2), (3,4), ...
__host__ __device__ constexpr int ex(int k) {
  return (k == 1 || k == 7 || k == 9 || k == 11 || k == 13) ? 1
         : (k == 2 || k == 8 || k == 10 || k == 12 || k == 14) ? -1
                                                                 : 0;
}
__host__ __device__ constexpr int ey(int k) {
  return (k == 3 || k == 7 || k == 10 || k == 15 || k == 17) ? 1
         : (k == 4 || k == 8 || k == 9 || k == 16 || k == 18) ? -1
                                                                : 0;
}
__host__ __device__ constexpr int ez(int k) {
  return (k == 5 || k == 11 || k == 14 || k == 15 || k == 18) ? 1
         : (k == 6 || k == 12 || k == 13 || k == 16 || k == 17) ? -1
                                                                  : 0;
}
// storage row (single-phase direction index) of CG direction k
__host__ __device__ constexpr int row(int k) {
  return k <= 7 ? k
                : (k == 8 ? 10 : k == 9 ? 9 : k == 10 ? 8 : k == 11 ? 15 : k == 12 ? 18 : k == 13 ? 17
                               : k == 14 ? 16 : k == 15 ? 11 : k == 16 ? 14 : k == 17 ? 13 : 12);
}
// CG direction of storage row q (inverse of row)
__host__ __device__ constexpr int of_row(int q) {
  return q <= 7 ? q
                : (q == 8 ? 10 : q == 9 ? 9 : q == 10 ? 8 : q == 11 ? 15 : q == 12 ? 18 : q == 13 ? 17
                               : q == 14 ? 16 : q == 15 ? 11 : q == 16 ? 14 : q == 17 ? 13 : 12);
}
// Moments of even degree (they depend only on f_0 and the opposite-pair
// sums) and of odd degree (only on the pair differences), in the column
// order of the FP32 back-transform blocks: 0, 1, 2, 9 .. 15 and 3 .. 8,
// 16, 17, 18.
__host__ __device__ constexpr int even_moment(int c) { return c < 3 ? c : c + 6; }
__host__ __device__ constexpr int odd_moment(int c) { return c < 6 ? c + 3 : c + 10; }

// the scaled CG moment basis (CG3:63-83) as polynomials of e
__host__ __device__ constexpr int mcoef(int k, int q) {
  const int x = ex(q), y = ey(q), z = ez(q);
  const int c2 = x * x + y * y + z * z;
  switch (k) {
    case 0: return 1;
    case 1: return c2 - 1;
    case 2: return 3 * c2 * c2 - 6 * c2 + 1;
    case 3: return x;
    case 4: return (3 * c2 - 5) * x;
    case 5: return y;
    case 6: return (3 * c2 - 5) * y;
    case 7: return z;
    case 8: return (3 * c2 - 5) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (2 * c2 - 3) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (2 * c2 - 3) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    default: return (x * x - y * y) * z;
  }
}

}  // namespace cg

}  // namespace lbm
