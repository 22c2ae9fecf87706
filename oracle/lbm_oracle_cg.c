/*
 * lbm_oracle_cg.c -- CPU restatement of the reference's colour-gradient
 * two-phase update, TEST INFRASTRUCTURE (see lbm_oracle.c for the rules).
 *
 * Restates MP_3D/Multi_Component_CG_MPI_SPARSE_Software_3DPartition.cpp
 * ("CG3") at one rank for fully periodic runs: compaction and nei_loc in the
 * CG velocity order, M^-1 of the scaled CG basis, init with the phase field
 * from a file, and per step `collision` (colour gradient, Guo force masked by
 * phase, MRT with the surface-tension terms in m_eq and psi-interpolated
 * viscosity, push stream, equilibrium colour distributions with recolouring,
 * colour scatter-add) followed by `comput_macro_variables`.  Same operation
 * order as the reference (built with -ffp-contract=off); pinned bit for bit
 * against the reference compiled from source.
 *
 * Layouts: 1-based ids, row 0 unused; f AoS [(count+1)*19] in CG direction
 * order; u [(count+1)*3]; scalars [(count+1)].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int orc_invert(double* a, int n);

/* CG velocity order, weights and opposites (CG3:188-206). */
static const int ECG[19][3] = {{0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                               {0, 0, 1},   {0, 0, -1},  {1, 1, 0},  {-1, -1, 0}, {1, -1, 0},
                               {-1, 1, 0},  {1, 0, 1},   {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1},
                               {0, 1, 1},   {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};
static const int LRCG[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

static double wcg(int q) { return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }

/* The CG basis (CG3:63-83) as polynomials of e in the CG order. */
void orc_cg_moment_matrix(double* M) {
  for (int q = 0; q < 19; q++) {
    const int x = ECG[q][0], y = ECG[q][1], z = ECG[q][2];
    const int c2 = x * x + y * y + z * z;
    double r[19];
    r[0] = 1;
    r[1] = c2 - 1;
    r[2] = 3 * c2 * c2 - 6 * c2 + 1;
    r[3] = x;
    r[4] = (3 * c2 - 5) * x;
    r[5] = y;
    r[6] = (3 * c2 - 5) * y;
    r[7] = z;
    r[8] = (3 * c2 - 5) * z;
    r[9] = 3 * x * x - c2;
    r[10] = (2 * c2 - 3) * (3 * x * x - c2);
    r[11] = y * y - z * z;
    r[12] = (2 * c2 - 3) * (y * y - z * z);
    r[13] = x * y;
    r[14] = y * z;
    r[15] = x * z;
    r[16] = (y * y - z * z) * x;
    r[17] = (z * z - x * x) * y;
    r[18] = (x * x - y * y) * z;
    for (int k = 0; k < 19; k++) M[k * 19 + q] = r[k];
  }
}

int orc_cg_matrices(double* M, double* MI) {
  orc_cg_moment_matrix(M);
  memcpy(MI, M, sizeof(double) * 361);
  return orc_invert(MI, 19);
}

/* nei_loc with the CG velocity order (CG3 Parallelize_Geometry, same
 * construction as SP3:1099-1151). */
void orc_cg_nei_loc(const uint8_t* mask, int nx, int ny, int nz, const int32_t* coor, int count, int32_t* nei) {
  int32_t* id = (int32_t*)calloc((size_t)nx * ny * nz, sizeof(int32_t));
  for (int c = 1; c <= count; c++) {
    const int i = coor[c] / (ny * nz), j = (coor[c] % (ny * nz)) / nz, k = coor[c] % nz;
    id[i + (long)nx * (j + (long)ny * k)] = c;
  }
  memset(nei, 0, sizeof(int32_t) * 19);
  for (int c = 1; c <= count; c++) {
    const int i = coor[c] / (ny * nz), j = (coor[c] % (ny * nz)) / nz, k = coor[c] % nz;
    for (int q = 0; q < 19; q++) {
      int ip = i + ECG[q][0], jp = j + ECG[q][1], kp = k + ECG[q][2];
      if (ip < 0) ip = nx - 1;
      if (ip >= nx) ip = 0;
      if (jp < 0) jp = ny - 1;
      if (jp >= ny) jp = 0;
      if (kp < 0) kp = nz - 1;
      if (kp >= nz) kp = 0;
      nei[(long)c * 19 + q] = id[ip + (long)nx * (jp + (long)ny * kp)];
    }
  }
  free(id);
}

typedef struct orc_cg_params {
  double nu_l, nu_g;      /* niu_l, niu_g */
  double psi_solid;       /* ContactAngle_parameter */
  double cap_a;           /* CapA */
  double g[3];            /* gxs, gys, gzs */
  int body_force_phase;   /* bodyforce_apply */
  double flux_psi;        /* rel_perm_psi */
  double flux_umax;       /* rel_perm_psi2 */
} orc_cg_params;

/* viscosity interpolation constants (CG3 init: delta = 0.1) */
typedef struct {
  double wl, wg, lg0, l1, l2, g1, g2, delta;
} cg_visc;

static cg_visc cg_visc_of(const orc_cg_params* p) {
  cg_visc v;
  const double c_s2 = 1.0 * 1.0 / 3, dt = 1.0;
  v.delta = 0.1;
  v.wl = 1.0 / (p->nu_l / (c_s2 * dt) + 0.5);
  v.wg = 1.0 / (p->nu_g / (c_s2 * dt) + 0.5);
  v.lg0 = 2 * v.wl * v.wg / (v.wl + v.wg);
  v.l1 = 2 * (v.wl - v.lg0) / v.delta;
  v.l2 = -v.l1 / (2 * v.delta);
  v.g1 = 2 * (v.lg0 - v.wg) / v.delta;
  v.g2 = v.g1 / (2 * v.delta);
  return v;
}

/* `feq` of CG3 (CG3:2520-2545): M^-1 applied to the incompressible
 * equilibrium moments, summed from 0 in index order. */
static double feq_cg(const double* MI, int k, double rho, const double* u) {
  double meq[19];
  const double rho_0 = 1.0;
  for (int s = 0; s < 19; s++) meq[s] = 0;
  const double ux = u[0], uy = u[1], uz = u[2];
  meq[0] = rho;
  meq[3] = rho_0 * ux;
  meq[5] = rho_0 * uy;
  meq[7] = rho_0 * uz;
  meq[1] = rho_0 * (ux * ux + uy * uy + uz * uz);
  meq[9] = rho_0 * (2 * ux * ux - uy * uy - uz * uz);
  meq[11] = rho_0 * (uy * uy - uz * uz);
  meq[13] = rho_0 * ux * uy;
  meq[14] = rho_0 * uy * uz;
  meq[15] = rho_0 * ux * uz;
  double f = 0;
  for (int j = 0; j < 19; j++) f += MI[k * 19 + j] * meq[j];
  return f;
}

/* `init` with ini_Sat < 0 (CG3:2360-2380): psi from the phase file (stored as
 * float, CG3:2121), rho = 1, u = 0, rho_r = (psi rho + rho)/2, rho_b = rho - rho_r,
 * f = feq(rho, u). psi_in is in compaction order [count+1]. */
void orc_cg_init(int count, const double* MI, const float* psi_in, double* rho, double* u, double* f, double* psi,
                 double* rho_r, double* rho_b) {
  const double u0[3] = {0, 0, 0};
  memset(f, 0, sizeof(double) * 19);
  memset(u, 0, sizeof(double) * 3);
  rho[0] = psi[0] = rho_r[0] = rho_b[0] = 0;
  for (int i = 1; i <= count; i++) {
    u[i * 3 + 0] = u[i * 3 + 1] = u[i * 3 + 2] = 0.0;
    psi[i] = psi_in[i];
    rho[i] = 1.0;
    rho_r[i] = (psi[i] * rho[i] + rho[i]) / 2;
    rho_b[i] = rho[i] - rho_r[i];
    for (int lm = 0; lm < 19; lm++) f[(long)i * 19 + lm] = feq_cg(MI, lm, rho[i], u0);
  }
}

static inline double rowdot_cg(const double* A, int r, const double* x) {
  double s = 0.0;
  int started = 0;
  for (int j = 0; j < 19; j++) {
    const double a = A[r * 19 + j];
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

/* One reference step: `collision` (CG3:2546-3290) then
 * `comput_macro_variables` (CG3:3316-3370).  rhor/rhob are the scatter
 * accumulators (zeroed by the macro step). */
void orc_cg_step(int count, const int32_t* nei, const double* M, const double* MI, const orc_cg_params* p,
                 double* rho, double* u, double* u0, double* f, double* F, double* psi, double* rho_r,
                 double* rho_b, double* rhor, double* rhob) {
  const double c_l = 1.0, dt = 1.0, lat_c = 1.0;
  const double c_s2 = lat_c * lat_c / 3;
  const double c2 = lat_c * lat_c, c4 = c2 * c2;
  const double rho_0 = 1.0;
  const cg_visc V = cg_visc_of(p);
  double S[19];
  S[0] = 0; S[3] = 0; S[5] = 0; S[7] = 0;
  for (int ci = 1; ci <= count; ci++) {
    double C[3] = {0, 0, 0};
    int ind_S = 0;
    for (int t = 0; t < 19; t++) {
      const int32_t nb = nei[(long)ci * 19 + t];
      const double ps = nb > 0 ? psi[nb] : p->psi_solid;
      if (nb == 0) ind_S = 1;
      for (int d = 0; d < 3; d++) C[d] += 3.0 / (lat_c * lat_c * dt) * wcg(t) * (double)ECG[t][d] * ps;
    }
    const double* uc = &u[(long)ci * 3];
    const double uu = uc[0] * uc[0] + uc[1] * uc[1] + uc[2] * uc[2];
    if ((sqrt((rho_r[ci] - rho_b[ci]) * (rho_r[ci] - rho_b[ci])) >= 0.9) && (ind_S == 1)) {
      C[0] = 0;
      C[1] = 0;
      C[2] = 0;
    }
    const double cc = sqrt(C[0] * C[0] + C[1] * C[1] + C[2] * C[2]);
    double nx, ny, nz;
    if (cc > 0) {
      nx = C[0] / cc;
      ny = C[1] / cc;
      nz = C[2] / cc;
    } else {
      nx = 0;
      ny = 0;
      nz = 0;
    }
    double guo[19];
    if (((p->body_force_phase == 1) && (psi[ci] < p->flux_psi)) ||
        ((p->body_force_phase == -1) && (psi[ci] > -p->flux_psi))) {
      for (int q = 0; q < 19; q++) guo[q] = 0.0;
    } else {
      const double* g = p->g;
      for (int q = 0; q < 19; q++) {
        const double ex = (double)ECG[q][0] * c_l, ey = (double)ECG[q][1] * c_l, ez = (double)ECG[q][2] * c_l;
        const double lm0 = ((ex - uc[0]) * g[0] + (ey - uc[1]) * g[1] + (ez - uc[2]) * g[2]) / c_s2;
        const double lm1 = (ex * uc[0] + ey * uc[1] + ez * uc[2]) * (ex * g[0] + ey * g[1] + ez * g[2]) / (c_s2 * c_s2);
        guo[q] = wcg(q) * (lm0 + lm1);
      }
    }
    const double ux = uc[0], uy = uc[1], uz = uc[2];
    double meq[19];
    for (int k = 0; k < 19; k++) meq[k] = 0;
    meq[0] = rho[ci];
    meq[3] = rho_0 * ux;
    meq[5] = rho_0 * uy;
    meq[7] = rho_0 * uz;
    meq[1] = rho_0 * (ux * ux + uy * uy + uz * uz) + p->cap_a * cc;
    meq[9] = rho_0 * (2 * ux * ux - uy * uy - uz * uz) + 0.5 * p->cap_a * cc * (2 * nx * nx - ny * ny - nz * nz);
    meq[11] = rho_0 * (uy * uy - uz * uz) + 0.5 * p->cap_a * cc * (ny * ny - nz * nz);
    meq[13] = rho_0 * ux * uy + 0.5 * p->cap_a * cc * (nx * ny);
    meq[14] = rho_0 * uy * uz + 0.5 * p->cap_a * cc * (ny * nz);
    meq[15] = rho_0 * ux * uz + 0.5 * p->cap_a * cc * (nx * nz);
    double s_v;
    const double ps = psi[ci];
    if (ps > 0) {
      if (ps > V.delta)
        s_v = V.wl;
      else
        s_v = V.lg0 + V.l1 * ps + V.l2 * ps * ps;
    } else {
      if (ps < -V.delta)
        s_v = V.wg;
      else
        s_v = V.lg0 + V.g1 * ps + V.g2 * ps * ps;
    }
    const double s_other = 8 * (2 - s_v) / (8 - s_v);
    S[1] = s_v; S[2] = s_v; S[4] = s_other; S[6] = s_other; S[8] = s_other; S[9] = s_v;
    S[10] = s_v; S[11] = s_v; S[12] = s_v; S[13] = s_v; S[14] = s_v; S[15] = s_v; S[16] = s_other;
    S[17] = s_other; S[18] = s_other;
    const double* fc = &f[(long)ci * 19];
    double ml[19], mi[19];
    for (int k = 0; k < 19; k++) {
      double m = rowdot_cg(M, k, fc);
      double fh = rowdot_cg(M, k, guo);
      fh *= (1 - 0.5 * S[k]);
      ml[k] = m - S[k] * (m - meq[k]) + dt * fh;
    }
    for (int q = 0; q < 19; q++) mi[q] = rowdot_cg(MI, q, ml);
    double gr[19], gb[19];
    for (int q = 0; q < 19; q++) {
      const int32_t d = nei[(long)ci * 19 + q];
      if (d > 0)
        F[(long)d * 19 + q] = mi[q];
      else
        F[(long)ci * 19 + LRCG[q]] = mi[q];
      const double eu = (double)ECG[q][0] * uc[0] + (double)ECG[q][1] * uc[1] + (double)ECG[q][2] * uc[2];
      gr[q] = wcg(q) * rho_r[ci] * (1 + 3 * eu / c2 + 4.5 * eu * eu / c4 - 1.5 * uu / c2);
      gb[q] = wcg(q) * rho_b[ci] * (1 + 3 * eu / c2 + 4.5 * eu * eu / c4 - 1.5 * uu / c2);
    }
    if (cc > 0)
      for (int kk = 1; kk < 19; kk += 2) {
        const double ef = ECG[kk][0] * C[0] + ECG[kk][1] * C[1] + ECG[kk][2] * C[2];
        double cp = gr[kk] < gr[kk + 1] ? gr[kk] : gr[kk + 1];
        cp = cp < gb[kk] ? cp : gb[kk];
        cp = cp < gb[kk + 1] ? cp : gb[kk + 1];
        cp *= ef / cc;
        gr[kk] += cp;
        gr[kk + 1] -= cp;
        gb[kk] -= cp;
        gb[kk + 1] += cp;
      }
    for (int q = 0; q < 19; q++) {
      const int32_t d = nei[(long)ci * 19 + q];
      if (d > 0) {
        rhor[d] += gr[q];
        rhob[d] += gb[q];
      } else {
        rhor[ci] += gr[q];
        rhob[ci] += gb[q];
      }
    }
  }
  for (int i = 1; i <= count; i++) {
    double* uc = &u[(long)i * 3];
    for (int d = 0; d < 3; d++) u0[(long)i * 3 + d] = uc[d];
    double r = 0, x = 0, y = 0, z = 0;
    for (int k = 0; k < 19; k++) {
      const double v = F[(long)i * 19 + k];
      f[(long)i * 19 + k] = v;
      r += v;
      x += (double)ECG[k][0] * v;
      y += (double)ECG[k][1] * v;
      z += (double)ECG[k][2] * v;
    }
    rho[i] = r;
    rho_r[i] = rhor[i];
    rho_b[i] = rhob[i];
    rhor[i] = 0;
    rhob[i] = 0;
    uc[0] = (x + dt * p->g[0] / 2) / r;
    uc[1] = (y + dt * p->g[1] / 2) / r;
    uc[2] = (z + dt * p->g[2] / 2) / r;
    psi[i] = (rho_r[i] - rho_b[i]) / (rho_r[i] + rho_b[i]);
  }
}

/* `Comput_Perm` (CG3:5116-5284), whole box, dp = 0: phase fluxes over nodes
 * with |u| < flux_umax; liquid psi >= flux_psi, gas psi <= -flux_psi. */
double orc_cg_perm(int count, const double* u, const double* psi, int nx, int ny, int nz, double porosity,
                   const orc_cg_params* p, double* per_l, double* per_g, double* uave_out) {
  double Ql[3] = {0, 0, 0}, Qg[3] = {0, 0, 0};
  for (int i = 1; i <= count; i++) {
    const double* a = &u[(long)i * 3];
    if (sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) < p->flux_umax) {
      if (psi[i] >= p->flux_psi)
        for (int d = 0; d < 3; d++) Ql[d] += a[d];
      if (psi[i] <= -p->flux_psi)
        for (int d = 0; d < 3; d++) Qg[d] += a[d];
    }
  }
  const int V = nx * ny * nz;
  const double dp = 0;
  double pl[3], pg[3];
  for (int d = 0; d < 3; d++) {
    pl[d] = Ql[d] / V * (p->nu_l) / (p->g[d] + dp);
    pg[d] = Qg[d] / V * (p->nu_g) / (p->g[d] + dp);
  }
  const double vx = (Ql[0] + Qg[0]) / V, vy = (Ql[1] + Qg[1]) / V, vz = (Ql[2] + Qg[2]) / V;
  if (uave_out)
    *uave_out = sqrt((vx / porosity) * (vx / porosity) + (vy / porosity) * (vy / porosity) +
                     (vz / porosity) * (vz / porosity));
  const double err = (pl[0] - per_l[0]) / per_l[0];
  for (int d = 0; d < 3; d++) {
    per_l[d] = pl[d];
    per_g[d] = pg[d];
  }
  return err;
}

/* `Comput_Saturation` (CG3:5286-5370), whole box: share of psi >= 0. */
double orc_cg_saturation(int count, const double* psi, int nx, int ny, int nz, double porosity) {
  double sl = 0;
  for (int i = 1; i <= count; i++)
    if (psi[i] >= 0) sl += 1;
  return sl / (nx * ny * nz * porosity);
}
