// FP64 single-phase kernel that reproduces the reference collision bit for bit.
//
// This translation unit is compiled with -fmad=false: every a*b+c that is
// written as such stays two correctly rounded operations, as in the reference
// built without FMA contraction.  The work per node is the reference's own
// arithmetic (SP3:1423-1779):
//   Guo force per direction, f_eq per direction, then per moment k
//   m_k = M_k . f, F_k = (1 - S_k/2) M_k . G, meq_k = M_k . f_eq,
//   m*_k = m_k - S_k (m_k - meq_k) + dt F_k;   f*_q = MI_q . m*
// with MI the Gauss-Jordan inverse the reference hard-codes.  Every sum keeps
// its terms and their order; what changes is only work whose result is
// determined without it:
//  * a term whose factor is exactly zero (a zero entry of M or MI, a zero
//    velocity component e_a of a direction, a force component the kernel is
//    specialised for being zero) adds +-0 to a sum and is left out -- it could
//    only flip the sign of an intermediate zero, which no later +, -, * turns
//    into a different non-zero value;
//  * a product by a power-of-two coefficient of M or MI is exact, so product
//    and sum are issued as one fma (one rounding, the same as the sum's);
//  * values that the reference recomputes per direction and that are equal
//    bit for bit (the Guo terms of opposite directions, the force terms of
//    directions with the same e_x) are computed once;
//  * the 19 moments of f are accumulated column by column while the pulled
//    populations arrive: each row still adds its terms in ascending index
//    order, so every m_k is the same chain of roundings, and the 19 pulled
//    values are dead once the columns are done (the kernel holds 19 moment
//    accumulators instead of f, f_eq and G at once);
//  * the conserved moments (S_k = 0) keep m_k: m_k - 0 (m_k - meq_k) = m_k.
// Streaming is a pull through the table instead of the reference's push
// through nei_loc, which moves values without arithmetic.
#include <utility>

#include "bc_kernels.cuh"
#include "mi_pattern.h"  // generated at build time from mrt.cpp's M^-1

namespace lbm {

__constant__ double c_MI[kQ * kQ];

cudaError_t set_mi_constant(const double* mi361, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_MI, mi361, sizeof(double) * kQ * kQ, 0, cudaMemcpyHostToDevice, st);
}

bool mi_pattern_matches(const double* mi361) {
  for (int q = 0; q < kQ; q++)
    for (int j = 0; j < kQ; j++) {
      const double v = mi361[q * kQ + j];
      int e;
      const bool nz = v != 0.0, p2 = nz && std::fabs(std::frexp(v, &e)) == 0.5;
      if (nz != (((mi_nonzero_row(q) >> j) & 1u) != 0) || p2 != (((mi_pow2_row(q) >> j) & 1u) != 0)) return false;
    }
  return true;
}

namespace {

__host__ __device__ constexpr int first_col(int k) {
  for (int j = 0; j < kQ; j++)
    if (mcoef(k, j) != 0) return j;
  return kQ;
}
__host__ __device__ constexpr bool pow2_coef(int c) {
  const int a = c < 0 ? -c : c;
  return a > 1 && (a & (a - 1)) == 0;
}
__host__ __device__ constexpr bool macro_rows_are_moments() {
  // rho = sum f and j = sum e f in the macro step are rows 0, 3, 5, 7 of M
  for (int q = 0; q < kQ; q++)
    if (mcoef(0, q) != 1 || mcoef(3, q) != cx(q) || mcoef(5, q) != cy(q) || mcoef(7, q) != cz(q)) return false;
  return first_col(0) == 0;
}
static_assert(macro_rows_are_moments(), "moment rows 0, 3, 5, 7 must be rho, j_x, j_y, j_z");
__host__ __device__ constexpr bool conserved_moment(int k) { return k == 0 || k == 3 || k == 5 || k == 7; }
__host__ __device__ constexpr bool mi_nz(int q, int j) { return ((mi_nonzero_row(q) >> j) & 1u) != 0; }
__host__ __device__ constexpr bool mi_p2(int q, int j) { return ((mi_pow2_row(q) >> j) & 1u) != 0; }
__host__ __device__ constexpr bool mi_rows_start_at_zero() {
  for (int q = 0; q < kQ; q++)
    if (!mi_nz(q, 0) || mi_p2(q, 0)) return false;
  return true;
}
static_assert(mi_rows_start_at_zero(), "every row of M^-1 starts with a non-zero, non-power-of-two entry");

__device__ __forceinline__ double srate(int k, double sv, double so) {
  const bool viscous = (k == 1 || k == 2 || (k >= 9 && k <= 15));
  return viscous ? sv : so;
}

// Every structural choice below (which coefficient is zero, a power of two or
// the first of its row; which direction leads its opposite pair) is a
// template parameter decided with if constexpr, so the kernel holds only the
// arithmetic that remains.
using QSeq = std::make_integer_sequence<int, kQ>;

// One term M_kj v of row k, added in ascending j.
template <int K, int J>
__device__ __forceinline__ void moment_term(double& acc, const double v) {
  constexpr int c = mcoef(K, J);
  if constexpr (c == 0) {
    return;
  } else if constexpr (J == first_col(K)) {
    if constexpr (c == 1)
      acc = v;
    else if constexpr (c == -1)
      acc = -v;
    else
      acc = (double)c * v;
  } else if constexpr (c == 1) {
    acc = acc + v;
  } else if constexpr (c == -1) {
    acc = acc - v;
  } else if constexpr (pow2_coef(c)) {
    acc = fma((double)c, v, acc);  // c*v is exact: one rounding, as c*v then +
  } else {
    acc = acc + (double)c * v;
  }
}

// Column J of the moment sums: acc_k (+)= M_kJ v for every row k.
template <int J, int... K>
__device__ __forceinline__ void moment_column_(double (&acc)[kQ], const double v, std::integer_sequence<int, K...>) {
  (moment_term<K, J>(acc[K], v), ...);
}
template <int J>
__device__ __forceinline__ void moment_column(double (&acc)[kQ], const double v) {
  moment_column_<J>(acc, v, QSeq{});
}
template <int... J>
__device__ __forceinline__ void moments_by_column(double (&acc)[kQ], const double (&f)[kQ],
                                                  std::integer_sequence<int, J...>) {
  (moment_column<J>(acc, f[J]), ...);
}

// Row K of the moment sums, M_K . v, terms in ascending index order.
template <int K, int... J>
__device__ __forceinline__ double moment_row_(const double (&v)[kQ], std::integer_sequence<int, J...>) {
  double acc = 0.0;
  (moment_term<K, J>(acc, v[J]), ...);
  return acc;
}
template <int K>
__device__ __forceinline__ double moment_row(const double (&v)[kQ]) {
  return moment_row_<K>(v, QSeq{});
}

// e_Q . a over the non-zero components of e_Q, in the order x, y, z (the
// reference's e[0]*a0 + e[1]*a1 + e[2]*a2 with its zero products left out).
template <int Q>
__device__ __forceinline__ double edot(double ax, double ay, double az) {
  constexpr int x = cx(Q), y = cy(Q), z = cz(Q);
  static_assert(x != 0 || y != 0 || z != 0, "edot of the rest direction");
  double s;
  if constexpr (x != 0) s = x > 0 ? ax : -ax;
  if constexpr (y != 0) {
    if constexpr (x == 0)
      s = y > 0 ? ay : -ay;
    else
      s = y > 0 ? s + ay : s - ay;
  }
  if constexpr (z != 0) {
    if constexpr (x == 0 && y == 0)
      s = z > 0 ? az : -az;
    else
      s = z > 0 ? s + az : s - az;
  }
  return s;
}

// A direction of each opposite pair: the one whose first non-zero component
// is positive.
__host__ __device__ constexpr bool leads_pair(int q) {
  return q != 0 && (cx(q) > 0 || (cx(q) == 0 && (cy(q) > 0 || (cy(q) == 0 && cz(q) > 0))));
}

// f_eq of feq() (SP3:1382-1391): w rho (1 + 3 eu / c2 + 4.5 eu eu / c4 -
// 1.5 uv / c2) with eu = e lat_c . u.  On the default lattice c2 = c4 = 1 and
// the divisions are left out (LAT = false); e lat_c . u is e . (lat_c u),
// each product (+-lat_c) u_a being exactly +-(lat_c u_a).  For the opposite
// direction eu is exactly -eu, so 3 eu / c2 changes sign and 4.5 eu eu / c4
// is the same value.
template <bool LAT, int Q>
__device__ __forceinline__ void equilibrium_pair(double rho, double cux, double cuy, double cuz, double t_uv,
                                                 const Lattice& L, double (&feq)[kQ]) {
  if constexpr (leads_pair(Q)) {
    const double eu = edot<Q>(cux, cuy, cuz);
    double t3 = 3.0 * eu, t45 = 4.5 * eu * eu;
    if constexpr (LAT) {
      t3 = t3 / L.c2;
      t45 = t45 / L.c4;
    }
    const double wr = weight(Q) * rho;
    feq[Q] = wr * (1.0 + t3 + t45 - t_uv);
    feq[opp(Q)] = wr * (1.0 - t3 + t45 - t_uv);
  }
}
template <bool LAT, int... Q>
__device__ __forceinline__ void equilibrium_(double rho, double ux, double uy, double uz, const Lattice& L,
                                             double (&feq)[kQ], std::integer_sequence<int, Q...>) {
  const double uv = ux * ux + uy * uy + uz * uz;
  double t_uv = 1.5 * uv;
  if constexpr (LAT) t_uv = t_uv / L.c2;
  feq[0] = weight(0) * rho * (1.0 - t_uv);
  const double cux = LAT ? L.c * ux : ux, cuy = LAT ? L.c * uy : uy, cuz = LAT ? L.c * uz : uz;
  (equilibrium_pair<LAT, Q>(rho, cux, cuy, cuz, t_uv, L, feq), ...);
}

// Guo forcing GuoF[q] = w_q (lm0 + lm1) (SP3:1432-1510, c_l = lat_c):
//   lm0 = ((e_x c_l - u_x) g_x + (e_y c_l - u_y) g_y + (e_z c_l - u_z) g_z) / c_s2
//   lm1 = (e c_l . u)(e c_l . g) / (c_s2 c_s2)
// (e.u)(e.g) is the same for q and its opposite (both factors change sign),
// so lm1 is divided once per pair.  GX: g_y = g_z = 0, so lm0 depends on
// e_x alone (three values) and lm1 vanishes for e_x = 0.  The default
// lattice (c_l = 1) uses the constants below; LAT = true takes c_l, c_s2
// from the step's lattice (the GX form is not built for it).
constexpr double kCs2 = 1.0 * 1.0 / 3;
constexpr double kCs4 = kCs2 * kCs2;

template <int Q>
__device__ __forceinline__ void guo_pair_x(double ux, double uy, double uz, double gx, double l0p, double l0z,
                                           double l0m, double (&guo)[kQ]) {
  if constexpr (Q == 0 || (!leads_pair(Q) && cx(Q) == 0)) {
    // e_x = 0 (the rest direction included): lm1 = (e.u)(+-0) / c_s4 = +-0
    guo[Q] = weight(Q) * l0z;
  } else if constexpr (leads_pair(Q) && cx(Q) == 0) {
    guo[Q] = weight(Q) * l0z;
  } else if constexpr (leads_pair(Q)) {  // e_x = +1, its opposite e_x = -1
    const double l1 = (edot<Q>(ux, uy, uz) * gx) / kCs4;
    guo[Q] = weight(Q) * (l0p + l1);
    guo[opp(Q)] = weight(Q) * (l0m + l1);
  }
}
template <int Q>
__device__ __forceinline__ void guo_pair_any(double ux, double uy, double uz, double gx, double gy, double gz,
                                             const double (&tx)[3], const double (&ty)[3], const double (&tz)[3],
                                             double (&guo)[kQ]) {
  if constexpr (leads_pair(Q)) {
    constexpr int o = opp(Q);
    const double l1 = (edot<Q>(ux, uy, uz) * edot<Q>(gx, gy, gz)) / kCs4;
    const double l0q = ((tx[cx(Q) + 1] + ty[cy(Q) + 1]) + tz[cz(Q) + 1]) / kCs2;
    const double l0o = ((tx[cx(o) + 1] + ty[cy(o) + 1]) + tz[cz(o) + 1]) / kCs2;
    guo[Q] = weight(Q) * (l0q + l1);
    guo[o] = weight(Q) * (l0o + l1);
  }
}
template <int Q>
__device__ __forceinline__ void guo_pair_lat(double cux, double cuy, double cuz, double cgx, double cgy, double cgz,
                                             const double (&tx)[3], const double (&ty)[3], const double (&tz)[3],
                                             double cs2, double cs4, double (&guo)[kQ]) {
  if constexpr (leads_pair(Q)) {
    constexpr int o = opp(Q);
    const double l1 = (edot<Q>(cux, cuy, cuz) * edot<Q>(cgx, cgy, cgz)) / cs4;
    const double l0q = ((tx[cx(Q) + 1] + ty[cy(Q) + 1]) + tz[cz(Q) + 1]) / cs2;
    const double l0o = ((tx[cx(o) + 1] + ty[cy(o) + 1]) + tz[cz(o) + 1]) / cs2;
    guo[Q] = weight(Q) * (l0q + l1);
    guo[o] = weight(Q) * (l0o + l1);
  }
}
template <bool GX, bool LAT, int... Q>
__device__ __forceinline__ void guo_force_(double ux, double uy, double uz, double gx, double gy, double gz,
                                           const Lattice& L, double (&guo)[kQ], std::integer_sequence<int, Q...>) {
  if constexpr (LAT) {
    static_assert(!GX, "the lattice form is built for the general force only");
    const double c = L.c, cs2 = L.cs2, cs4 = L.cs2 * L.cs2;
    // (e_a c_l - u_a) g_a for e_a = -1, 0, +1; 0 c_l - u_a is -u_a
    const double tx[3] = {(-c - ux) * gx, (-ux) * gx, (c - ux) * gx};
    const double ty[3] = {(-c - uy) * gy, (-uy) * gy, (c - uy) * gy};
    const double tz[3] = {(-c - uz) * gz, (-uz) * gz, (c - uz) * gz};
    guo[0] = weight(0) * (((tx[1] + ty[1]) + tz[1]) / cs2);
    (guo_pair_lat<Q>(c * ux, c * uy, c * uz, c * gx, c * gy, c * gz, tx, ty, tz, cs2, cs4, guo), ...);
  } else if constexpr (GX) {
    const double l0p = ((1.0 - ux) * gx) / kCs2;
    const double l0z = ((-ux) * gx) / kCs2;
    const double l0m = ((-1.0 - ux) * gx) / kCs2;
    (guo_pair_x<Q>(ux, uy, uz, gx, l0p, l0z, l0m, guo), ...);
  } else {
    const double tx[3] = {(-1.0 - ux) * gx, (-ux) * gx, (1.0 - ux) * gx};
    const double ty[3] = {(-1.0 - uy) * gy, (-uy) * gy, (1.0 - uy) * gy};
    const double tz[3] = {(-1.0 - uz) * gz, (-uz) * gz, (1.0 - uz) * gz};
    guo[0] = weight(0) * (((tx[1] + ty[1]) + tz[1]) / kCs2);
    (guo_pair_any<Q>(ux, uy, uz, gx, gy, gz, tx, ty, tz, guo), ...);
  }
}

// Relaxation of moment K: the non-conserved moments relax towards meq; every
// moment gets its forcing term (dt = 1).
template <int K>
__device__ __forceinline__ void relax_eq(double& m, const double (&feq)[kQ], double sv, double so) {
  if constexpr (!conserved_moment(K)) {
    const double S = srate(K, sv, so);
    m = m - S * (m - moment_row<K>(feq));
  }
}
template <bool LAT, int K>
__device__ __forceinline__ void relax_force(double& m, const double (&guo)[kQ], double sv, double so, double dt) {
  double fh = moment_row<K>(guo);
  if constexpr (!conserved_moment(K)) fh *= (1 - 0.5 * srate(K, sv, so));
  if constexpr (LAT)
    m = m + dt * fh;
  else
    m = m + fh;  // dt = 1
}

// Back-transform row Q: f*_Q = MI_Q . m, the non-zero entries in ascending j.
template <int Q, int J>
__device__ __forceinline__ void mi_term(double& s, const double (&m)[kQ]) {
  if constexpr (J == 0) {
    s = c_MI[Q * kQ] * m[0];
  } else if constexpr (mi_nz(Q, J)) {
    if constexpr (mi_p2(Q, J))
      s = fma(c_MI[Q * kQ + J], m[J], s);  // exact product: one rounding
    else
      s = s + c_MI[Q * kQ + J] * m[J];
  }
}
template <int Q, int... J>
__device__ __forceinline__ double mi_row(const double (&m)[kQ], std::integer_sequence<int, J...>) {
  double s;
  (mi_term<Q, J>(s, m), ...);
  return s;
}

template <bool GX, bool LAT, int... K>
__device__ __forceinline__ void collide_moments_(double (&m)[kQ], double rho, double ux, double uy, double uz,
                                                 const StepArgs& a, int p, std::integer_sequence<int, K...>) {
  {
    double feq[kQ];
    equilibrium_<LAT>(rho, ux, uy, uz, a.lat, feq, QSeq{});
    (relax_eq<K>(m[K], feq, a.s_v, a.s_o), ...);
  }
  {
    double guo[kQ];
    guo_force_<GX, LAT>(ux, uy, uz, a.gx, a.gy, a.gz, a.lat, guo, QSeq{});
    (relax_force<LAT, K>(m[K], guo, a.s_v, a.s_o, a.lat.dt), ...);
  }
  double* __restrict__ dst = static_cast<double*>(a.dst_pop) + p;
  const size_t np = (size_t)a.npad;
  ((dst[(size_t)K * np] = mi_row<K>(m, QSeq{})), ...);
}

// Relaxation in moment space and back-transform for one node whose moments
// m = M f (accumulated by the caller) and macro values are known; writes the
// 19 post-collision populations of node p.
template <bool GX, bool LAT = false>
__device__ __forceinline__ void collide_moments(double (&m)[kQ], double rho, double ux, double uy, double uz,
                                                const StepArgs& a, int p) {
  collide_moments_<GX, LAT>(m, rho, ux, uy, uz, a, p, QSeq{});
}

}  // namespace

__device__ __forceinline__ void pull_f64(const StepArgs& a, int p, double (&f)[kQ]) {
  const double* __restrict__ src = static_cast<const double*>(a.src_pop);
  f[0] = __ldg(src + p);
#pragma unroll
  for (int q = 1; q < kQ; q++) f[q] = __ldg(src + __ldg(a.table + (size_t)(q - 1) * a.npad + p));
}

__device__ __forceinline__ void macro_in_out(const StepArgs& a, int p, bool given, bool write, const double (&f)[kQ],
                                             double& rho, double& ux, double& uy, double& uz) {
  if (given) {
    const double* r = static_cast<const double*>(a.rho_in);
    const double* u = static_cast<const double*>(a.u_in);
    rho = r[p];
    ux = u[p];
    uy = u[a.npad + p];
    uz = u[2 * a.npad + p];
  } else if (a.lat.on) {
    macro_faithful_lat(f, a.lat.c, a.lat.dt * a.gx / 2, a.lat.dt * a.gy / 2, a.lat.dt * a.gz / 2, rho, ux, uy, uz);
  } else {
    macro_faithful(f, a.gx / 2, a.gy / 2, a.gz / 2, rho, ux, uy, uz);
  }
  if (write) {
    static_cast<double*>(a.rho_out)[p] = rho;
    double* u = static_cast<double*>(a.u_out);
    u[p] = ux;
    u[a.npad + p] = uy;
    u[2 * a.npad + p] = uz;
  }
}

// Resident blocks per SM asked of the register allocator: 16 warps (128
// registers, no spills) for 128-512 threads; 24 warps for 64-thread blocks
// (80 registers with a few spills) -- the autotuner times both.
constexpr int f64_min_blocks(int bs) { return bs == 64 ? 12 : 512 / bs; }

// One node per thread.  The macro step of the reference (comput_macro_variables,
// SP3:2414-2439) is rho = sum f and u = (j + dt g/2) / rho.  On the default
// lattice rho and j are the sums of moment rows 0, 3, 5, 7, so it reads them
// from the accumulated moments; with a self-defined lattice (LAT) j sums the
// products e_a lat_c f_q, each rounded, in direction order, which the kernel
// accumulates beside the moments.
template <int BS, bool GIVEN, bool WRITE, bool GX, bool LAT>
__global__ void __launch_bounds__(BS, f64_min_blocks(BS)) step_f64_faithful(StepArgs a) {
  const int p = blockIdx.x * BS + threadIdx.x;
  if (p >= a.n_main) return;
  double m[kQ];
  double jx = 0.0, jy = 0.0, jz = 0.0;
  {
    double f[kQ];
    pull_f64(a, p, f);
    moments_by_column(m, f, QSeq{});
    if constexpr (LAT && !GIVEN) lattice_momentum(f, a.lat.c, jx, jy, jz);
  }
  double rho, ux, uy, uz;
  if (GIVEN) {
    const double* r = static_cast<const double*>(a.rho_in);
    const double* u = static_cast<const double*>(a.u_in);
    rho = r[p];
    ux = u[p];
    uy = u[a.npad + p];
    uz = u[2 * a.npad + p];
  } else if constexpr (LAT) {
    rho = m[0];
    ux = (jx + a.lat.dt * a.gx / 2) / rho;
    uy = (jy + a.lat.dt * a.gy / 2) / rho;
    uz = (jz + a.lat.dt * a.gz / 2) / rho;
  } else {
    rho = m[0];
    ux = (m[3] + a.gx / 2) / rho;
    uy = (m[5] + a.gy / 2) / rho;
    uz = (m[7] + a.gz / 2) / rho;
  }
  if (WRITE) {
    static_cast<double*>(a.rho_out)[p] = rho;
    double* u = static_cast<double*>(a.u_out);
    u[p] = ux;
    u[a.npad + p] = uy;
    u[2 * a.npad + p] = uz;
  }
  if (a.snap_dst != nullptr && p >= a.snap_begin) {
    // nodes read by a face rule record their pulled state (pulled again:
    // the source array is read-only during the launch)
    double f[kQ];
    pull_f64(a, p, f);
    snap_write(a.snap_dst, a.nsnap, p - a.snap_begin, f, rho, ux, uy, uz);
  }
  collide_moments<GX, LAT>(m, rho, ux, uy, uz, a, p);
}

// Face nodes: pull, the boundary rules, macro step, record, collision.  With
// a.bnd_f set: only the populations after the rules (current state).  LAT:
// a self-defined lattice (the rules' equilibria, the macro step and the
// collision on it).
template <bool GIVEN, bool FINAL, bool LAT>
__global__ void __launch_bounds__(128) bc_f64_faithful(BcArgs a) {
  const int b = blockIdx.x * 128 + threadIdx.x;
  const int p = a.s.n_main + b;
  if (p >= a.s.n) return;
  double f[kQ];
  pull_f64(a.s, p, f);
  if (!GIVEN) bc_apply(a, b, f, a.s.lat);
  if (FINAL) {
    const size_t nb = (size_t)(a.s.n - a.s.n_main);
#pragma unroll
    for (int q = 0; q < kQ; q++) a.bnd_f[(size_t)q * nb + b] = f[q];
    return;
  }
  double rho, ux, uy, uz;
  macro_in_out(a.s, p, GIVEN, a.s.rho_out != nullptr, f, rho, ux, uy, uz);
  snap_write(a.s.snap_dst, a.s.nsnap, p - a.s.snap_begin, f, rho, ux, uy, uz);
  double m[kQ];
  moments_by_column(m, f, QSeq{});
  collide_moments<false, LAT>(m, rho, ux, uy, uz, a.s, p);
}

template <bool LAT>
static void launch_bc_f64(const BcArgs& a, int grid, cudaStream_t st) {
  if (a.bnd_f)
    bc_f64_faithful<false, true, LAT><<<grid, 128, 0, st>>>(a);
  else if (a.s.rho_in != nullptr)
    bc_f64_faithful<true, false, LAT><<<grid, 128, 0, st>>>(a);
  else
    bc_f64_faithful<false, false, LAT><<<grid, 128, 0, st>>>(a);
}

cudaError_t launch_boundary_f64(const BcArgs& a, cudaStream_t st) {
  const int nb = a.s.n - a.s.n_main;
  if (nb <= 0) return cudaSuccess;
  const int grid = (nb + 127) / 128;
  if (a.s.lat.on)
    launch_bc_f64<true>(a, grid, st);
  else
    launch_bc_f64<false>(a, grid, st);
  return cudaGetLastError();
}

// final pass of the diagnostics reduction (shared by all kinds)
__global__ void reduce_final_kernel(const double* __restrict__ partials, int nblocks, double* __restrict__ result) {
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] = (i == 3) ? fmax(acc[i], partials[(size_t)b * 8 + i]) : acc[i] + partials[(size_t)b * 8 + i];
  block_reduce8(acc, result, smem);
}

template <int BS, bool GX, bool LAT>
static cudaError_t launch_f64_bs(const StepArgs& a, cudaStream_t st) {
  const int grid = (a.n_main + BS - 1) / BS;
  if (grid == 0) return cudaSuccess;
  const bool given = a.rho_in != nullptr, write = a.rho_out != nullptr;
  if (given && write)
    step_f64_faithful<BS, true, true, GX, LAT><<<grid, BS, 0, st>>>(a);
  else if (given)
    step_f64_faithful<BS, true, false, GX, LAT><<<grid, BS, 0, st>>>(a);
  else if (write)
    step_f64_faithful<BS, false, true, GX, LAT><<<grid, BS, 0, st>>>(a);
  else
    step_f64_faithful<BS, false, false, GX, LAT><<<grid, BS, 0, st>>>(a);
  return cudaGetLastError();
}

template <int BS>
static cudaError_t launch_f64_force(const StepArgs& a, cudaStream_t st) {
  // a self-defined lattice: the general lattice arithmetic; force along x
  // only (every configuration of the benchmarks): the specialised Guo terms;
  // any other force: the general ones
  if (a.lat.on) return launch_f64_bs<BS, false, true>(a, st);
  if (a.gy == 0.0 && a.gz == 0.0) return launch_f64_bs<BS, true, false>(a, st);
  return launch_f64_bs<BS, false, false>(a, st);
}

cudaError_t launch_step_f64(const StepArgs& a, int block, cudaStream_t st) {
  switch (block) {
    case 64: return launch_f64_force<64>(a, st);
    case 128: return launch_f64_force<128>(a, st);
    case 512: return launch_f64_force<512>(a, st);
    default: return launch_f64_force<256>(a, st);
  }
}

cudaError_t reduce_f64(const ReduceArgs& a, cudaStream_t st) { return reduce_dispatch<Store::F64>(a, st); }
cudaError_t export_f64(const void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad, double* out,
                       cudaStream_t st, int n_main, const double* bnd_f) {
  return export_dispatch<Store::F64>(pop, table, ref_of, n, npad, 1.0, out, st, n_main, bnd_f);
}
cudaError_t import_f64(void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad, const double* in,
                       cudaStream_t st) {
  return import_dispatch<Store::F64>(pop, table, ref_of, n, npad, 1.0, in, st);
}
cudaError_t import_macro_f64(void* rho, void* u, const int32_t* ref_of, int n, int npad, const double* rho_in,
                             const double* u_in, cudaStream_t st) {
  return import_macro_dispatch<Store::F64>(rho, u, ref_of, n, npad, rho_in, u_in, st);
}

}  // namespace lbm
