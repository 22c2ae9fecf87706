// MRT constants: the moment matrix, its inverse and the relaxation rates.
#include <cmath>
#include <utility>

#include "cg_basis.h"
#include "lbm_internal.h"

namespace lbm {

namespace {

// Full-pivot Gauss-Jordan inversion in place.  The reference computes M^-1
// with this algorithm (SP3:797-836) and hard-codes its output as hex literals
// in the collision (SP3:1745-1779).  The pivot search (first strictly larger
// |a| in a row-major scan of the trailing block), the row/column swaps and
// the update order are kept the same because they fix the rounding of every
// entry, and the FP64 kernel reproduces the reference bit for bit only with
// the same M^-1.
template <int N>
bool gauss_jordan_full_pivot(double (&a)[N][N]) {
  int piv_r[N], piv_c[N];
  for (int k = 0; k < N; k++) {
    double amax = 0.0;
    for (int i = k; i < N; i++)
      for (int j = k; j < N; j++)
        if (std::fabs(a[i][j]) > amax) {
          amax = std::fabs(a[i][j]);
          piv_r[k] = i;
          piv_c[k] = j;
        }
    if (std::fabs(amax) < 1e-12) return false;
    if (piv_r[k] != k)
      for (int j = 0; j < N; j++) std::swap(a[k][j], a[piv_r[k]][j]);
    if (piv_c[k] != k)
      for (int i = 0; i < N; i++) std::swap(a[i][k], a[i][piv_c[k]]);
    a[k][k] = 1 / a[k][k];
    const double d = a[k][k];
    for (int j = 0; j < N; j++)
      if (j != k) a[k][j] *= d;
    for (int i = 0; i < N; i++) {
      if (i == k) continue;
      for (int j = 0; j < N; j++)
        if (j != k) a[i][j] -= a[i][k] * a[k][j];
    }
    for (int i = 0; i < N; i++)
      if (i != k) a[i][k] *= -d;
  }
  for (int k = N - 1; k >= 0; k--) {
    if (piv_c[k] != k)
      for (int j = 0; j < N; j++) std::swap(a[k][j], a[piv_c[k]][j]);
    if (piv_r[k] != k)
      for (int i = 0; i < N; i++) std::swap(a[i][k], a[i][piv_r[k]]);
  }
  return true;
}

}  // namespace

// Inverse of the colour-gradient basis; the reference hard-codes this
// algorithm's output in its collision too (CG3:3081-3117).
bool build_cg_inverse(double MI[kQ][kQ]) {
  double a[kQ][kQ];
  for (int k = 0; k < kQ; k++)
    for (int q = 0; q < kQ; q++) a[k][q] = cg::mcoef(k, q);
  if (!gauss_jordan_full_pivot<kQ>(a)) return false;
  for (int k = 0; k < kQ; k++)
    for (int q = 0; q < kQ; q++) MI[k][q] = a[k][q];
  return true;
}

// Rates of `init` (SP3:1286-1322) for a lattice of spacing dx and step dt.
bool build_mrt_constants(double nu, MrtConstants* out, double dx, double dt) {
  for (int k = 0; k < kQ; k++)
    for (int q = 0; q < kQ; q++) out->M[k][q] = mcoef(k, q);
  for (int k = 0; k < kQ; k++)
    for (int q = 0; q < kQ; q++) out->MI[k][q] = out->M[k][q];
  if (!gauss_jordan_full_pivot<kQ>(out->MI)) return false;
  const double lat_c = dx / dt;
  const double c_s2 = lat_c * lat_c / 3;
  const double tau = nu / (c_s2 * dt) + 0.5;
  const double s_v = 1 / tau;
  const double s_o = 8 * (2 - s_v) / (8 - s_v);
  const bool viscous[kQ] = {false, true, true, false, false, false, false, false, false, true,
                            true,  true, true, true,  true,  true,  false, false, false};
  const bool conserved[kQ] = {true, false, false, true, false, true, false, true, false, false,
                              false, false, false, false, false, false, false, false, false};
  for (int k = 0; k < kQ; k++) out->S[k] = conserved[k] ? 0.0 : (viscous[k] ? s_v : s_o);
  out->s_v = s_v;
  out->s_o = s_o;
  return true;
}

Lattice make_lattice(double dx, double dt) {
  Lattice l;
  l.dx = dx;
  l.dt = dt;
  l.c = dx / dt;  // SP3:1292-1294
  l.ic = 1.0 / l.c;
  l.cs2 = l.c * l.c / 3;
  l.c2 = l.c * l.c;  // feq (SP3:1387)
  l.c4 = l.c2 * l.c2;
  l.on = (l.c != 1.0 || dt != 1.0) ? 1 : 0;
  return l;
}

}  // namespace lbm
