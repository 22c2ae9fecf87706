/*
 * Oracle harness (test infrastructure only): compiles the reference
 * single-phase sparse solver Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp
 * ("SP3") unmodified, from where it lies, into oracle/_ref/libref_sp3.so, and
 * exposes its own functions and globals through a small C ABI so tests and the
 * CPU-baseline leg of bench.py can drive the reference's CPU path directly.
 *
 * The reference's main() (SP3:258-795) is renamed away; the functions below do
 * what main does for one rank, in the same order:
 *   Parallelize_Geometry (SP3:862)  -> mask read, Partition_Solid, Solid2/coor,
 *                                      nei_loc (SP3:1018-1151)
 *   allocation of rho/u/f/F/u0     (SP3:440-482, index 0 unused)
 *   Comput_MI (SP3:838), init (SP3:1278)
 *   loop body: collision (SP3:1398), boundary_pressure (SP3:2656) and
 *              boundary_velocity (SP3:2450) when a face has one (SP3:580-585),
 *              comput_macro_variables (SP3:2401)
 *   reporting: Error (SP3:3118), Comput_Perm (SP3:3518)
 * The INPUT.dat parse is replaced by setting the same globals from arguments:
 * ref_sp3_set_boundaries sets Sub_BC, in_BC and the pressure/velocity faces
 * (default: none, the fully periodic path); lattice_v=0, nnf_module=0,
 * par_per_*=0.
 */
#define main lbm_reference_sp3_main
#include SP3_SOURCE
#undef main

#include <cstdint>

/* The reference's globals have common names (error, init, n, M, S, e, w ...)
 * that collide with libc and the host process; the library is built with
 * -fvisibility=hidden -Wl,-Bsymbolic so they bind to this file's own
 * definitions, and only the entry points below are exported. */


namespace {
double* h_rho = nullptr;
double** h_u = nullptr;
double** h_f = nullptr;
double** h_F = nullptr;
double** h_u0 = nullptr;
double h_Permia[3] = {0.0, 0.0, 0.0};
// faces in INPUT.dat order: xp, xn, yp, yn, zp, zn
int g_perdir = 1, g_sub_bc = 0, g_in_bc = 0, g_pre[6] = {0, 0, 0, 0, 0, 0}, g_vel[6] = {0, 0, 0, 0, 0, 0};
double g_p[6] = {0, 0, 0, 0, 0, 0}, g_v[6] = {0, 0, 0, 0, 0, 0};

double** alloc_rows(int count, int width) {
  double** p = new double*[count + 1];
  p[0] = new double[(size_t)(count + 1) * width]();
  for (int i = 1; i <= count; i++) p[i] = p[i - 1] + width;
  return p;
}
}  // namespace

#pragma GCC visibility push(default)
extern "C" {

/* Pressure/velocity boundary settings used by the next ref_sp3_create (the
 * INPUT.dat lines SP3:299-305, 318).  Faces in the order xp, xn, yp, yn, zp,
 * zn; pre/vel 1 = on; p = boundary density, v = normal velocity; perdir =
 * PerDir of Comput_Perm. */
void ref_sp3_set_boundaries(int sub_bc, int in_bc, const int* pre, const double* p, const int* vel,
                            const double* v, int perdir) {
  g_perdir = perdir;
  g_sub_bc = sub_bc;
  g_in_bc = in_bc;
  for (int i = 0; i < 6; i++) {
    g_pre[i] = pre ? pre[i] : 0;
    g_p[i] = p ? p[i] : 0.0;
    g_vel[i] = vel ? vel[i] : 0;
    g_v[i] = v ? v[i] : 0.0;
  }
}

/* Builds geometry, compaction, neighbour table and the initial state exactly as
 * the reference main does at one rank.  Returns Count (number of fluid nodes). */
int ref_sp3_create(const char* mask_path, int nx, int ny, int nz, int is_binary,
                   double nu, double gx_in, double gy_in, double gz_in) {
  std::strncpy(filename, mask_path, 127);
  filename[127] = 0;
  NX = nx - 1; NY = ny - 1; NZ = nz - 1;           /* SP3:343 */
  decbin = is_binary;
  in_vis = nu;
  gx = gx_in; gy = gy_in; gz = gz_in;
  inivx = inivy = inivz = 0.0;
  in_BC = g_in_bc; PerDir = g_perdir; lattice_v = 0; nnf_module = 0;
  Sub_BC = g_sub_bc;
  pre_xp = g_pre[0]; pre_xn = g_pre[1]; pre_yp = g_pre[2]; pre_yn = g_pre[3]; pre_zp = g_pre[4]; pre_zn = g_pre[5];
  p_xp = g_p[0]; p_xn = g_p[1]; p_yp = g_p[2]; p_yn = g_p[3]; p_zp = g_p[4]; p_zn = g_p[5];
  vel_xp = g_vel[0]; vel_xn = g_vel[1]; vel_yp = g_vel[2]; vel_yn = g_vel[3]; vel_zp = g_vel[4]; vel_zn = g_vel[5];
  v_xp = g_v[0]; v_xn = g_v[1]; v_yp = g_v[2]; v_yn = g_v[3]; v_zp = g_v[4]; v_zn = g_v[5];
  par_per_x = par_per_y = par_per_z = 0;
  mirX = mirY = mirZ = 0;

  Parallelize_Geometry();
  h_rho = new double[Count + 1]();
  h_u = alloc_rows(Count, 3);
  h_f = alloc_rows(Count, 19);
  h_F = alloc_rows(Count, 19);
  h_u0 = alloc_rows(Count, 3);
  h_Permia[0] = h_Permia[1] = h_Permia[2] = 0.0;
  Comput_MI(M, MI);
  init(h_rho, h_u, h_f, Solid);
  return Count;
}

/* n iterations of the reference loop body (SP3:571-590). */
void ref_sp3_step(int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    collision(h_rho, h_u, h_f, h_F, nullptr, Solid, nullptr, nullptr);
    if ((1 - pre_xp) * (1 - pre_xn) * (1 - pre_yp) * (1 - pre_yn) * (1 - pre_zp) * (1 - pre_zn) == 0)
      boundary_pressure(pre_xp, p_xp, pre_xn, p_xn, pre_yp, p_yp, pre_yn, p_yn, pre_zp, p_zp, pre_zn, p_zn, h_f, h_F,
                        h_u, h_rho, Solid);
    if ((1 - vel_xp) * (1 - vel_xn) * (1 - vel_yp) * (1 - vel_yn) * (1 - vel_zp) * (1 - vel_zn) == 0)
      boundary_velocity(vel_xp, v_xp, vel_xn, v_xn, vel_yp, v_yp, vel_yn, v_yn, vel_zp, v_zp, vel_zn, v_zn, h_f, h_F,
                        h_rho, h_u, Solid);
    comput_macro_variables(h_rho, h_u, h_u0, h_f, h_F, nullptr, Solid);
  }
}

/* The boundary-node lists the reference builds (SP3:1164-1222): face 0..5 =
 * xn (bclx), xp (bcrx), yn (bcly), yp (bcry), zn (bclz), zp (bcrz).  Returns
 * the length; writes the ids when out is not null. */
int ref_sp3_get_face_list(int face, int32_t* out) {
  int* lists[6] = {bclx, bcrx, bcly, bcry, bclz, bcrz};
  int lens[6] = {bclxn, bcrxn, bclyn, bcryn, bclzn, bcrzn};
  if (face < 0 || face > 5) return -1;
  if (out)
    for (int i = 0; i < lens[face]; i++) out[i] = lists[face][i];
  return lens[face];
}

/* Error (SP3:3118): returns the relative L2 change of u; u_max and the
 * mean-speed u_ave it writes are returned through the pointers. */
double ref_sp3_error(double* umax_out, double* uave_out) {
  double vmax = 0.0, uave = 0.0;
  double e = Error(h_u, h_u0, &vmax, &uave);
  if (umax_out) *umax_out = vmax;
  if (uave_out) *uave_out = uave;
  return e;
}

/* Comput_Perm (SP3:3518): permeability components and |Q|/(V*phi). */
double ref_sp3_perm(double* perm3_out, double* uave_out) {
  double e = Comput_Perm(h_u, h_Permia, PerDir, nullptr);
  if (perm3_out) for (int d = 0; d < 3; d++) perm3_out[d] = h_Permia[d];
  if (uave_out) *uave_out = u_ave;
  return e;
}

int ref_sp3_count() { return Count; }
double ref_sp3_porosity() { return porosity; }
double ref_sp3_s_v() { return s_v; }

void ref_sp3_get_coor(int32_t* out) {
  for (int i = 0; i <= Count; i++) out[i] = (i == 0) ? 0 : coor[i];
}
void ref_sp3_get_nei_loc(int32_t* out) {
  for (int i = 1; i <= Count; i++)
    for (int q = 0; q < 19; q++) out[(size_t)i * 19 + q] = nei_loc[i][q];
  for (int q = 0; q < 19; q++) out[q] = 0;
}
void ref_sp3_get_f(double* out) {
  std::memcpy(out, h_f[0], sizeof(double) * (size_t)(Count + 1) * 19);
}
void ref_sp3_set_f(const double* in) {
  std::memcpy(h_f[0], in, sizeof(double) * (size_t)(Count + 1) * 19);
}
void ref_sp3_get_u(double* out) {
  std::memcpy(out, h_u[0], sizeof(double) * (size_t)(Count + 1) * 3);
}
void ref_sp3_set_u(const double* in) {
  std::memcpy(h_u[0], in, sizeof(double) * (size_t)(Count + 1) * 3);
}
void ref_sp3_get_rho(double* out) {
  std::memcpy(out, h_rho, sizeof(double) * (size_t)(Count + 1));
}
void ref_sp3_set_rho(const double* in) {
  std::memcpy(h_rho, in, sizeof(double) * (size_t)(Count + 1));
}
void ref_sp3_get_M(double* out) {
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 19; j++) out[i * 19 + j] = M[i][j];
}
void ref_sp3_get_MI(double* out) {
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 19; j++) out[i * 19 + j] = MI[i][j];
}
}
#pragma GCC visibility pop
