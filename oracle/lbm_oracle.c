/*
 * lbm_oracle.c -- CPU restatement of the reference's sparse D3Q19 MRT
 * single-phase update, written as TEST INFRASTRUCTURE.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker.  The product library
 * (liblbm.so) never links it.
 *
 * Every function restates the algorithm of
 *   Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp (abbrev. SP3)
 * at one rank, in the reference's own floating-point operation order (built
 * with -ffp-contract=off), so its results are pinned bit-exactly against the
 * reference compiled from source (oracle/_ref/libref_sp3.so) and against the
 * committed golden fixtures in tests/golden/.
 *
 * Layout conventions (same as the reference):
 *   node ids are 1-based, id 0 is an unused dummy row;
 *   populations are AoS double f[(count+1)*19];
 *   velocity is AoS double u[(count+1)*3];
 *   coor[id] = i*ny*nz + j*nz + k   (z fastest, SP3:1065-1071);
 *   the in-memory mask is uint8 mask[x + nx*(y + ny*z)] (x fastest, the
 *   order of the reference's ASCII geometry file, SP3:935-943).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define Q19 19

/* D3Q19 velocity set, weights and opposite directions: SP3:167-180. */
static const int E19[Q19][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                {0, 0, 1},  {0, 0, -1}, {1, 1, 0},  {-1, 1, 0}, {1, -1, 0},
                                {-1, -1, 0}, {0, 1, 1},  {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
                                {1, 0, 1},  {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1}};
static const int OPP19[Q19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

static double w19(int q) {
  if (q == 0) return 1.0 / 3.0;
  if (q <= 6) return 1.0 / 18.0;
  return 1.0 / 36.0;
}

/* d'Humieres moment matrix (SP3:64-83).  Row k is built from the velocity
 * set with the standard polynomial definitions rather than typed in:
 *   0 rho, 1 e, 2 eps, 3/5/7 j, 4/6/8 q, 9 3pxx, 10 3pixx, 11 pww, 12 piww,
 *   13 pxy, 14 pyz, 15 pxz, 16-18 m_x, m_y, m_z. */
void orc_moment_matrix(double M[Q19][Q19]) {
  for (int q = 0; q < Q19; q++) {
    const int x = E19[q][0], y = E19[q][1], z = E19[q][2];
    const int c2 = x * x + y * y + z * z;
    M[0][q] = 1;
    M[1][q] = 19 * c2 - 30;
    M[2][q] = (21 * c2 * c2 - 53 * c2 + 24) / 2;
    M[3][q] = x;
    M[4][q] = (5 * c2 - 9) * x;
    M[5][q] = y;
    M[6][q] = (5 * c2 - 9) * y;
    M[7][q] = z;
    M[8][q] = (5 * c2 - 9) * z;
    M[9][q] = 3 * x * x - c2;
    M[10][q] = (3 * c2 - 5) * (3 * x * x - c2);
    M[11][q] = y * y - z * z;
    M[12][q] = (3 * c2 - 5) * (y * y - z * z);
    M[13][q] = x * y;
    M[14][q] = y * z;
    M[15][q] = x * z;
    M[16][q] = (y * y - z * z) * x;
    M[17][q] = (z * z - x * x) * y;
    M[18][q] = (x * x - y * y) * z;
  }
}

/* In-place matrix inverse by Gauss-Jordan elimination with full pivoting,
 * restating `inverse` (SP3:797-836), which the reference also used offline to
 * print the hex literals of M^-1 it hard-codes in `collision` (SP3:1745-1779,
 * generator Single_Phase_3D/M_Inv_Calculation_For_SP.cpp).  The same pivot
 * rule (first strictly larger |a_ij| in row-major scan of the trailing block)
 * and the same update order are required for a bit-identical M^-1.
 * Returns 1 on success, 0 if singular (|pivot| < 1e-12). */
int orc_invert(double* a, int n) {
  int prow[128], pcol[128];
  if (n > 128) return 0;
  for (int k = 0; k < n; k++) {
    double best = 0.0;
    for (int i = k; i < n; i++)
      for (int j = k; j < n; j++) {
        const double v = fabs(a[i * n + j]);
        if (v > best) {
          best = v;
          prow[k] = i;
          pcol[k] = j;
        }
      }
    if (fabs(best) < 1e-12) return 0;
    if (prow[k] != k)
      for (int j = 0; j < n; j++) {
        const double t = a[k * n + j];
        a[k * n + j] = a[prow[k] * n + j];
        a[prow[k] * n + j] = t;
      }
    if (pcol[k] != k)
      for (int i = 0; i < n; i++) {
        const double t = a[i * n + k];
        a[i * n + k] = a[i * n + pcol[k]];
        a[i * n + pcol[k]] = t;
      }
    a[k * n + k] = 1 / a[k * n + k];
    for (int j = 0; j < n; j++)
      if (j != k) a[k * n + j] *= a[k * n + k];
    for (int i = 0; i < n; i++)
      if (i != k)
        for (int j = 0; j < n; j++)
          if (j != k) a[i * n + j] -= a[i * n + k] * a[k * n + j];
    for (int i = 0; i < n; i++)
      if (i != k) a[i * n + k] *= -a[k * n + k];
  }
  for (int k = n - 1; k >= 0; k--) {
    for (int j = 0; j < n; j++)
      if (pcol[k] != k) {
        const double t = a[k * n + j];
        a[k * n + j] = a[pcol[k] * n + j];
        a[pcol[k] * n + j] = t;
      }
    for (int i = 0; i < n; i++)
      if (prow[k] != k) {
        const double t = a[i * n + k];
        a[i * n + k] = a[i * n + prow[k]];
        a[i * n + prow[k]] = t;
      }
  }
  return 1;
}

/* M and M^-1 as flat 19x19 row-major arrays. */
int orc_mrt_matrices(double* M_out, double* MI_out) {
  double M[Q19][Q19];
  orc_moment_matrix(M);
  memcpy(M_out, M, sizeof(M));
  memcpy(MI_out, M, sizeof(M));
  return orc_invert(MI_out, Q19);
}

/* Relaxation rates (SP3:1278-1322): tau = nu/(c_s^2 dt) + 0.5, s_v = 1/tau,
 * s_o = 8(2-s_v)/(8-s_v), S = [0,s_v,s_v,0,s_o,0,s_o,0,s_o,s_v x7,s_o x3]. */
void orc_rates(double nu, double* S) {
  const double lat_c = 1.0, dt = 1.0;
  const double c_s2 = lat_c * lat_c / 3;
  const double tau_f = nu / (c_s2 * dt) + 0.5;
  const double s_v = 1 / tau_f;
  const double s_o = 8 * (2 - s_v) / (8 - s_v);
  const double r[Q19] = {0, s_v, s_v, 0, s_o, 0, s_o, 0, s_o, s_v, s_v, s_v, s_v, s_v, s_v, s_v, s_o, s_o, s_o};
  memcpy(S, r, sizeof(r));
}

/* Porosity over the whole box (SP3:1009-1020 with par_per_* = 0). */
double orc_porosity(const uint8_t* mask, int nx, int ny, int nz) {
  long pores = 0;
  for (long c = 0; c < (long)nx * ny * nz; c++) pores += (mask[c] == 0);
  return (double)pores / (double)((long)nx * ny * nz);
}

/* Fluid-node compaction (SP3:1018-1071 at one rank; Partition_Solid
 * SP3:3799-3819 and 4011-4021 assign every pore to partition 1):
 * pore cells numbered 1.. in k-outer, j, i-inner order (x fastest);
 * coor[id] = i*ny*nz + j*nz + k.  Returns the number of fluid nodes; coor may
 * be NULL to count only. */
int orc_compact(const uint8_t* mask, int nx, int ny, int nz, int32_t* coor) {
  int count = 0;
  if (coor) coor[0] = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (mask[i + (long)nx * (j + (long)ny * k)] == 0) {
          count++;
          if (coor) coor[count] = i * ny * nz + j * nz + k;
        }
  return count;
}

/* Push-style neighbour table nei_loc[id][q] (SP3:1099-1151 at one rank):
 * the fluid id at x + e_q with periodic wrap on every axis, or 0 when that
 * cell is solid (halfway bounce-back into direction LR[q]).  Row 0 is zero. */
void orc_nei_loc(const uint8_t* mask, int nx, int ny, int nz, const int32_t* coor, int count,
                 int32_t* nei) {
  int32_t* id = (int32_t*)calloc((size_t)nx * ny * nz, sizeof(int32_t));
  for (int c = 1; c <= count; c++) {
    const int i = coor[c] / (ny * nz), j = (coor[c] % (ny * nz)) / nz, k = coor[c] % nz;
    id[i + (long)nx * (j + (long)ny * k)] = c;
  }
  memset(nei, 0, sizeof(int32_t) * Q19);
  for (int c = 1; c <= count; c++) {
    const int i = coor[c] / (ny * nz), j = (coor[c] % (ny * nz)) / nz, k = coor[c] % nz;
    for (int q = 0; q < Q19; q++) {
      int ip = i + E19[q][0], jp = j + E19[q][1], kp = k + E19[q][2];
      if (ip < 0) ip = nx - 1;
      if (ip >= nx) ip = 0;
      if (jp < 0) jp = ny - 1;
      if (jp >= ny) jp = 0;
      if (kp < 0) kp = nz - 1;
      if (kp >= nz) kp = 0;
      nei[(long)c * Q19 + q] = id[ip + (long)nx * (jp + (long)ny * kp)];
    }
  }
  free(id);
}

/* Equilibrium `feq` (SP3:1382-1394) with lat_c = 1. */
static inline double feq_ref(int q, double rho, const double* u) {
  const double c2 = 1.0 * 1.0, c4 = c2 * c2;
  const double eu = (double)E19[q][0] * u[0] + (double)E19[q][1] * u[1] + (double)E19[q][2] * u[2];
  const double uv = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  return w19(q) * rho * (1.0 + 3.0 * eu / c2 + 4.5 * eu * eu / c4 - 1.5 * uv / c2);
}

/* `init` (SP3:1278-1380): rho = 1, u = u_init, f = feq(rho, u). */
void orc_sp_init(int count, const double* u_init, double* rho, double* u, double* f) {
  memset(f, 0, sizeof(double) * Q19);
  memset(u, 0, sizeof(double) * 3);
  rho[0] = 0.0;
  for (int c = 1; c <= count; c++) {
    for (int d = 0; d < 3; d++) u[(long)c * 3 + d] = u_init[d];
    rho[c] = 1.0;
    for (int q = 0; q < Q19; q++) f[(long)c * Q19 + q] = feq_ref(q, 1.0, &u[(long)c * 3]);
  }
}

/* Row-vector product sum_j A[r][j] x[j] in index order, skipping exact zeros
 * (adding a +-0 product never changes a running sum's value). */
static inline double rowdot(const double* A, int r, const double* x) {
  double s = 0.0;
  int started = 0;
  for (int j = 0; j < Q19; j++) {
    const double a = A[r * Q19 + j];
    if (a == 0.0) continue;
    if (!started) {
      s = a * x[j];
      started = 1;
    } else {
      s = s + a * x[j];
    }
  }
  return s;
}

/* One reference time step at one rank: `collision` (SP3:1398-1819: Guo force,
 * moment-space relaxation, back-transform with M^-1, push-stream with
 * halfway bounce-back through nei_loc) followed by `comput_macro_variables`
 * (SP3:2401-2446: f <- F, rho = sum f, u = (sum e f + dt g/2)/rho, u0 <- old u).
 * MI must be the matrix from orc_mrt_matrices. */
void orc_sp_step(int count, const int32_t* nei, const double* M, const double* MI, const double* S,
                 double gx, double gy, double gz, double* rho, double* u, double* u0, double* f,
                 double* F) {
  const double c_l = 1.0, dt = 1.0;
  const double c_s2 = c_l * c_l / 3;
  const double g[3] = {gx, gy, gz};
  for (int c = 1; c <= count; c++) {
    const double* uc = &u[(long)c * 3];
    const double* fc = &f[(long)c * Q19];
    double guo[Q19], fe[Q19], ml[Q19], mi[Q19];
    for (int q = 0; q < Q19; q++) {
      const double ex = (double)E19[q][0] * c_l, ey = (double)E19[q][1] * c_l, ez = (double)E19[q][2] * c_l;
      const double lm0 = ((ex - uc[0]) * g[0] + (ey - uc[1]) * g[1] + (ez - uc[2]) * g[2]) / c_s2;
      const double lm1 = (ex * uc[0] + ey * uc[1] + ez * uc[2]) * (ex * g[0] + ey * g[1] + ez * g[2]) /
                         (c_s2 * c_s2);
      guo[q] = w19(q) * (lm0 + lm1);
      fe[q] = feq_ref(q, rho[c], uc);
    }
    for (int k = 0; k < Q19; k++) {
      double m = rowdot(M, k, fc);
      double fh = rowdot(M, k, guo);
      const double me = rowdot(M, k, fe);
      fh *= (1 - 0.5 * S[k]);
      ml[k] = m - S[k] * (m - me) + dt * fh;
    }
    for (int q = 0; q < Q19; q++) mi[q] = rowdot(MI, q, ml);
    for (int q = 0; q < Q19; q++) {
      const int32_t d = nei[(long)c * Q19 + q];
      if (d > 0)
        F[(long)d * Q19 + q] = mi[q];
      else
        F[(long)c * Q19 + OPP19[q]] = mi[q];
    }
  }
  for (int c = 1; c <= count; c++) {
    double* uc = &u[(long)c * 3];
    for (int d = 0; d < 3; d++) u0[(long)c * 3 + d] = uc[d];
    double r = 0, ux = 0, uy = 0, uz = 0;
    for (int q = 0; q < Q19; q++) {
      const double v = F[(long)c * Q19 + q];
      f[(long)c * Q19 + q] = v;
      r += v;
      ux += (double)E19[q][0] * v;
      uy += (double)E19[q][1] * v;
      uz += (double)E19[q][2] * v;
    }
    rho[c] = r;
    uc[0] = (ux + dt * g[0] / 2) / r;
    uc[1] = (uy + dt * g[1] / 2) / r;
    uc[2] = (uz + dt * g[2] / 2) / r;
  }
}

/* `Error` (SP3:3118-3196) at one rank.  Note the reference loop runs
 * i = 1 .. count-1 and so leaves out the last node (SP3:3141).  Writes u_max
 * and the mean pore speed sum|u| / (nx ny nz phi). */
double orc_sp_error(int count, const double* u, const double* u0, int nx, int ny, int nz,
                    double porosity, double* umax_out, double* uave_out) {
  double t1 = 0, t2 = 0, t3 = 0, um = 0;
  for (int c = 1; c < count; c++) {
    const double* a = &u[(long)c * 3];
    const double* b = &u0[(long)c * 3];
    t1 += (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
    t2 += a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    t3 += sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    if (a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > um) um = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  }
  t1 = sqrt(t1);
  t2 = sqrt(t2);
  if (umax_out) *umax_out = sqrt(um);
  if (uave_out) *uave_out = t3 / (nx * ny * nz * porosity);
  return t1 / (t2 + 1e-30);
}

/* `Comput_Perm` (SP3:3518-3648) at one rank, whole-box window, no pressure
 * boundary (dp = 0): Q = sum u, k_d = Q_d / V * nu / g_d, u_ave = |Q|/(V phi).
 * perm_prev holds the previous permeability (the reference's Permia); the
 * return value is the relative change along direction perdir (1..3). */
double orc_sp_perm(int count, const double* u, int nx, int ny, int nz, double porosity, double nu,
                   double gx, double gy, double gz, int perdir, double* perm_prev, double* uave_out) {
  double Q[3] = {0, 0, 0};
  for (int c = 1; c <= count; c++)
    for (int d = 0; d < 3; d++) Q[d] += u[(long)c * 3 + d];
  const int V = nx * ny * nz;
  const double dp = 0;
  double perm[3];
  perm[0] = Q[0] / V * nu / (gx + dp);
  perm[1] = Q[1] / V * nu / (gy + dp);
  perm[2] = Q[2] / V * nu / (gz + dp);
  const int d = (perdir >= 1 && perdir <= 3) ? perdir - 1 : 0;
  const double err = (perm[d] - perm_prev[d]) / perm_prev[d];
  for (int i = 0; i < 3; i++) perm_prev[i] = perm[i];
  const double ax = Q[0] / (V * porosity), ay = Q[1] / (V * porosity), az = Q[2] / (V * porosity);
  if (uave_out) *uave_out = sqrt(ax * ax + ay * ay + az * az);
  return err;
}
