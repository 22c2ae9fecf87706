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
static void sp_boundaries(int count, const int32_t* nei, const double* M, const double* MI, int sub_bc,
                          const int* pre, const double* p, const int* vel, const double* v,
                          const int32_t* lists, const int* len, const double* rho, const double* u,
                          const double* f, double* F);

void orc_sp_step_bc(int count, const int32_t* nei, const double* M, const double* MI, const double* S,
                    double gx, double gy, double gz, double* rho, double* u, double* u0, double* f, double* F,
                    int sub_bc, const int* pre, const double* p, const int* vel, const double* v,
                    const int32_t* lists, const int* len);

void orc_sp_step(int count, const int32_t* nei, const double* M, const double* MI, const double* S,
                 double gx, double gy, double gz, double* rho, double* u, double* u0, double* f,
                 double* F) {
  orc_sp_step_bc(count, nei, M, MI, S, gx, gy, gz, rho, u, u0, f, F, 0, NULL, NULL, NULL, NULL, NULL, NULL);
}

/* As orc_sp_step, with the reference's pressure and velocity boundaries
 * applied between streaming and the macro step (SP3:580-585); pre/p/vel/v are
 * NULL for none.  Faces of pre, p, vel, v in INPUT.dat order xp, xn, yp, yn,
 * zp, zn; lists/len are the six boundary-node lists of orc_face_list in the
 * order xn, xp, yn, yp, zn, zp, concatenated. */
void orc_sp_step_bc(int count, const int32_t* nei, const double* M, const double* MI, const double* S,
                    double gx, double gy, double gz, double* rho, double* u, double* u0, double* f, double* F,
                    int sub_bc, const int* pre, const double* p, const int* vel, const double* v,
                    const int32_t* lists, const int* len) {
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
  if (lists) sp_boundaries(count, nei, M, MI, sub_bc, pre, p, vel, v, lists, len, rho, u, f, F);
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

/* Boundary-node list of one face (SP3:1164-1222 at one rank): the pore cells
 * of the face in the reference's loop order, as fluid ids.  face: 0 x=0
 * (bclx, k outer, j inner), 1 x=nx-1 (bcrx), 2 y=0 (bcly, k outer, i inner),
 * 3 y=ny-1 (bcry), 4 z=0 (bclz, j outer, i inner), 5 z=nz-1 (bcrz).  Returns
 * the length; out may be NULL to count only. */
int orc_face_list(const uint8_t* mask, int nx, int ny, int nz, int face, int32_t* out) {
  int32_t* id = (int32_t*)calloc((size_t)nx * ny * nz, sizeof(int32_t));
  int count = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (mask[i + (long)nx * (j + (long)ny * k)] == 0) id[i + (long)nx * (j + (long)ny * k)] = ++count;
  const int axis = face / 2, side = face % 2;
  const int n0 = axis == 0 ? nz : (axis == 1 ? nz : ny);  /* outer loop extent */
  const int n1 = axis == 0 ? ny : nx;                      /* inner loop extent */
  int len = 0;
  for (int a = 0; a < n0; a++)
    for (int b = 0; b < n1; b++) {
      int i, j, k;
      if (axis == 0) { i = side ? nx - 1 : 0; j = b; k = a; }
      else if (axis == 1) { i = b; j = side ? ny - 1 : 0; k = a; }
      else { i = b; j = a; k = side ? nz - 1 : 0; }
      const int32_t c = id[i + (long)nx * (j + (long)ny * k)];
      if (c > 0) {
        if (out) out[len] = c;
        len++;
      }
    }
  free(id);
  return len;
}

/* `boundary_pressure` (SP3:2656-3116) then `boundary_velocity`
 * (SP3:2450-2655) at one rank, each called only when one of its faces is on
 * (SP3:580-585).  They overwrite post-streaming F of the face nodes from the
 * previous step's f, rho, u (the reference calls them before the macro step)
 * and, for Sub_BC 2 velocity faces, from F itself.  Kept as the reference
 * has them:
 *   - pressure Sub_BC 1: a node whose inward neighbour is solid writes the
 *     rest-state equilibrium into the i-th node of the y=ny-1 list, whatever
 *     face it belongs to (SP3:2733-2790); an index past that list's end is
 *     outside the reference's array and is skipped here;
 *   - pressure Sub_BC 3 takes the non-equilibrium part from the -y neighbour
 *     (nei_loc[.][4]) on every face (SP3:3000-3110), row 0 when that is solid;
 *   - velocity Sub_BC 2: the x flags drive the z faces with the z velocities
 *     and the z flags the x faces (SP3:2556-2591).
 * Face order of every pass: pressure yp, yn, xp, xn, zp, zn; velocity Sub_BC
 * 0/1 yn, yp, zn, zp, xn, xp; Sub_BC 2 and 3 yp, yn, then (as above) x, z. */
static void sp_boundaries(int count, const int32_t* nei, const double* M, const double* MI, int sub_bc,
                          const int* pre, const double* p, const int* vel, const double* v,
                          const int32_t* lists, const int* len, const double* rho, const double* u,
                          const double* f, double* F) {
  (void)count;
  const int32_t* L[6];
  int off = 0;
  for (int s = 0; s < 6; s++) {
    L[s] = lists + off;
    off += len[s];
  }
  /* INPUT order index (xp, xn, yp, yn, zp, zn) -> list slot (xn, xp, yn, yp, zn, zp) and the push
   * direction towards the inside */
  static const int slot_of[6] = {1, 0, 3, 2, 5, 4};
  static const int dir_in[6] = {2, 1, 4, 3, 6, 5};
  const double zero[3] = {0.0, 0.0, 0.0};
  int any_pre = 0, any_vel = 0;
  for (int s = 0; s < 6; s++) {
    any_pre |= pre && pre[s] == 1;
    any_vel |= vel && vel[s] == 1;
  }
  if (any_pre) {
    static const int order[6] = {2, 3, 0, 1, 4, 5}; /* yp, yn, xp, xn, zp, zn */
    for (int oi = 0; oi < 6; oi++) {
      const int fc = order[oi];
      if (pre[fc] != 1) continue;
      const int32_t* lst = L[slot_of[fc]];
      const int n = len[slot_of[fc]];
      const double rb = p[fc];
      for (int i = 0; i < n; i++) {
        const int32_t b = lst[i];
        const int32_t nb = nei[(long)b * Q19 + dir_in[fc]];
        double* Fb = &F[(long)b * Q19];
        if (sub_bc == 0) {
          for (int ks = 0; ks < Q19; ks++) Fb[ks] = feq_ref(ks, rb, zero);
        } else if (sub_bc == 1) {
          if (nb > 0) {
            for (int ks = 0; ks < Q19; ks++) Fb[ks] = feq_ref(ks, rb, &u[(long)nb * 3]);
          } else if (i < len[3]) {
            double* Ft = &F[(long)L[3][i] * Q19];
            for (int ks = 0; ks < Q19; ks++) Ft[ks] = feq_ref(ks, rb, zero);
          }
        } else if (sub_bc == 2) {
          if (nb > 0) {
            double ml[Q19];
            for (int mi = 0; mi < Q19; mi++) {
              ml[mi] = 0;
              for (int mj = 0; mj < Q19; mj++) ml[mi] += M[mi * Q19 + mj] * f[(long)nb * Q19 + mj];
            }
            ml[0] = rb;
            for (int mi = 0; mi < Q19; mi++) {
              Fb[mi] = 0;
              for (int mj = 0; mj < Q19; mj++) Fb[mi] += MI[mi * Q19 + mj] * ml[mj];
            }
          } else {
            for (int ks = 0; ks < Q19; ks++) Fb[ks] = feq_ref(ks, rb, zero);
          }
        } else if (sub_bc == 3) {
          if (nb > 0) {
            const int32_t n4 = nei[(long)b * Q19 + 4];
            for (int ks = 0; ks < Q19; ks++)
              Fb[ks] = feq_ref(ks, rb, &u[(long)nb * 3]) + f[(long)n4 * Q19 + ks] -
                       feq_ref(ks, rho[nb], &u[(long)nb * 3]);
          } else {
            for (int ks = 0; ks < Q19; ks++) Fb[ks] = feq_ref(ks, rb, zero);
          }
        }
      }
    }
  }
  if (any_vel) {
    double uf[6][3];
    for (int s = 0; s < 6; s++) {
      uf[s][0] = uf[s][1] = uf[s][2] = 0.0;
      uf[s][s / 2] = v[s];
    }
    if (sub_bc == 0 || sub_bc == 1) {
      static const int order[6] = {3, 2, 5, 4, 1, 0}; /* yn, yp, zn, zp, xn, xp */
      for (int oi = 0; oi < 6; oi++) {
        const int fc = order[oi];
        if (vel[fc] != 1) continue;
        const int32_t* lst = L[slot_of[fc]];
        for (int i = 0; i < len[slot_of[fc]]; i++)
          for (int ks = 0; ks < Q19; ks++) F[(long)lst[i] * Q19 + ks] = feq_ref(ks, 1.0, uf[fc]);
      }
    } else if (sub_bc == 2) {
      /* (flag, face whose list, velocity and incoming sign are used) */
      static const int flag_of[6] = {2, 3, 0, 1, 4, 5};  /* yp, yn, xp, xn, zp, zn flags */
      static const int face_of[6] = {2, 3, 4, 5, 0, 1};  /* yp, yn, zp, zn, xp, xn faces */
      for (int oi = 0; oi < 6; oi++) {
        if (vel[flag_of[oi]] != 1) continue;
        const int fc = face_of[oi];
        const int axis = fc / 2, plus = (fc % 2) == 0;
        const int32_t* lst = L[slot_of[fc]];
        for (int i = 0; i < len[slot_of[fc]]; i++) {
          double* Fb = &F[(long)lst[i] * Q19];
          for (int ks = 0; ks < Q19; ks++) {
            const int e = E19[ks][axis];
            if (plus ? e < 0 : e > 0)
              Fb[ks] = feq_ref(OPP19[ks], 1.0, uf[fc]) - Fb[OPP19[ks]] + feq_ref(ks, 1.0, uf[fc]);
          }
        }
      }
    } else if (sub_bc == 3) {
      static const int order[6] = {2, 3, 0, 1, 4, 5}; /* yp, yn, xp, xn, zp, zn */
      for (int oi = 0; oi < 6; oi++) {
        const int fc = order[oi];
        if (vel[fc] != 1) continue;
        const int32_t* lst = L[slot_of[fc]];
        for (int i = 0; i < len[slot_of[fc]]; i++) {
          const int32_t b = lst[i];
          const int32_t nb = nei[(long)b * Q19 + dir_in[fc]];
          for (int ks = 0; ks < Q19; ks++)
            if (nb > 0) F[(long)b * Q19 + ks] = feq_ref(ks, rho[nb], uf[fc]);
        }
      }
    }
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

/* `Comput_Perm` (SP3:3518-3648) at one rank, whole-box window: Q = sum u,
 * k_d = Q_d / V * nu / (g_d + dp), u_ave = |Q|/(V phi).  dp is the pressure
 * gradient term, 0 without pressure boundaries (in_BC = 0) and otherwise
 * |p_+ - p_-| c_s^2 / L along perdir (SP3:3543-3556, see orc_sp_dp).
 * perm_prev holds the previous permeability (the reference's Permia); the
 * return value is the relative change along direction perdir (1..3). */
double orc_sp_perm_dp(int count, const double* u, int nx, int ny, int nz, double porosity, double nu,
                      double gx, double gy, double gz, double dp, int perdir, double* perm_prev,
                      double* uave_out) {
  double Q[3] = {0, 0, 0};
  for (int c = 1; c <= count; c++)
    for (int d = 0; d < 3; d++) Q[d] += u[(long)c * 3 + d];
  const int V = nx * ny * nz;
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

double orc_sp_perm(int count, const double* u, int nx, int ny, int nz, double porosity, double nu,
                   double gx, double gy, double gz, int perdir, double* perm_prev, double* uave_out) {
  return orc_sp_perm_dp(count, u, nx, ny, nz, porosity, nu, gx, gy, gz, 0.0, perdir, perm_prev, uave_out);
}

/* dp of Comput_Perm (SP3:3543-3556) for the whole box: in_bc = 0 gives 0;
 * else |p_+ - p_-| * c_s^2 / (extent along perdir) / dx with c_s^2 = 1/3,
 * dx = 1; p in INPUT.dat order xp, xn, yp, yn, zp, zn. */
double orc_sp_dp(int in_bc, int perdir, const double* p, int nx, int ny, int nz) {
  if (in_bc == 0) return 0.0;
  const double c_s2 = 1.0 * 1.0 / 3;
  const double dx = 1.0;
  switch (perdir) {
    case 2: return fabs(p[2] - p[3]) * c_s2 / (ny - 1 - 0 + 1) / dx;
    case 3: return fabs(p[4] - p[5]) * c_s2 / (nz - 1 - 0 + 1) / dx;
    default: return fabs(p[0] - p[1]) * c_s2 / (nx - 1 - 0 + 1) / dx;
  }
}

/* `Comput_Grop_Perm` (SP:4886-5091) at one rank: for each division d, the
 * n_sub[d]^3 cubes of edge size[d] whose first low corner is corner[3*d..];
 * cube (a, b, c) (loop order a = x outer, b = y, c = z inner) spans
 * [corner + (a, b, c) * size, + size - 1] on each axis.  Per cube:
 * Q = sum of u over the fluid nodes inside (id order), perm_d = Q_d / size^3
 * * nu / (g_d + dp), porosity = pores / size^3; written to out as
 * (perm_x, perm_y, perm_z, porosity).  SP's dp uses the whole box:
 * |p_+ - p_-| c_s^2 / (N+1) / dx (SP:4928-4941).  Returns the number of cubes. */
int orc_sp_group_perm(int count, const double* u, const int32_t* coor, int nx, int ny, int nz, double nu, double gx,
                      double gy, double gz, double dp, int ndiv, const int* n_sub, const int* size,
                      const int* corner, double* out) {
  (void)nx;
  int cube = 0;
  for (int d = 0; d < ndiv; d++) {
    const int vol = size[d] * size[d] * size[d];
    for (int a = 0; a < n_sub[d]; a++)
      for (int b = 0; b < n_sub[d]; b++)
        for (int c = 0; c < n_sub[d]; c++) {
          const int xn = corner[3 * d + 0] + a * size[d], xp = corner[3 * d + 0] + a * size[d] + size[d] - 1;
          const int yn = corner[3 * d + 1] + b * size[d], yp = corner[3 * d + 1] + b * size[d] + size[d] - 1;
          const int zn = corner[3 * d + 2] + c * size[d], zp = corner[3 * d + 2] + c * size[d] + size[d] - 1;
          double Q[3] = {0, 0, 0};
          int pores = 0;
          for (int i = 1; i <= count; i++) {
            const int si = coor[i] / (ny * nz), sj = (coor[i] % (ny * nz)) / nz, sm = coor[i] % nz;
            if (si >= xn && si <= xp && sj >= yn && sj <= yp && sm >= zn && sm <= zp) {
              Q[0] += u[(long)i * 3 + 0];
              Q[1] += u[(long)i * 3 + 1];
              Q[2] += u[(long)i * 3 + 2];
              pores += 1;
            }
          }
          out[cube * 4 + 0] = Q[0] / (vol) * (nu) / (gx + dp);
          out[cube * 4 + 1] = Q[1] / (vol) * (nu) / (gy + dp);
          out[cube * 4 + 2] = Q[2] / (vol) * (nu) / (gz + dp);
          out[cube * 4 + 3] = (double)pores / vol;
          cube++;
        }
  }
  return cube;
}
