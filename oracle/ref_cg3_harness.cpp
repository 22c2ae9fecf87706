/*
 * Oracle harness (test infrastructure only): compiles the reference
 * colour-gradient two-phase solver
 * MP_3D/Multi_Component_CG_MPI_SPARSE_Software_3DPartition.cpp ("CG3")
 * unmodified, from where it lies, into oracle/_ref/libref_cg3.so and exposes
 * its own functions and globals through a small C ABI.
 *
 * The functions below do what its main (CG3:322-1010) does at one rank for a
 * fully periodic run with the initial phase field read from a file
 * (ini_Sat = -1): Parallelize_Geometry (geometry, compaction, nei_loc, phase
 * file), allocation, Comput_MI, init (CG3:2208), then per step collision
 * (CG3:2546) + comput_macro_variables (CG3:3316); reports are
 * Comput_Perm (CG3:5116) and Comput_Saturation (CG3:5286).  Pressure/velocity
 * and psi boundaries, the stabiliser, dynamic inputs and the relative
 * permeability drivers are switched off.
 */
#define main lbm_reference_cg3_main
#include CG3_SOURCE
#undef main

#include <cstdint>

namespace {
double *c_rho = nullptr, *c_rho_r = nullptr, *c_rho_b = nullptr, *c_rhor = nullptr, *c_rhob = nullptr,
       *c_psi = nullptr;
double **c_u = nullptr, **c_f = nullptr, **c_F = nullptr, **c_u0 = nullptr;
int* c_SupInv = nullptr;
double c_Per_l[3] = {0, 0, 0}, c_Per_g[3] = {0, 0, 0};

double** rows(int count, int width) {
  double** p = new double*[count + 1];
  p[0] = new double[(size_t)(count + 1) * width]();
  for (int i = 1; i <= count; i++) p[i] = p[i - 1] + width;
  return p;
}
}  // namespace

#pragma GCC visibility push(default)
// mixture injection settings for the next ref_cg3_create (0 = off)
static int h_mix_thickness = 0;
static double h_mix_portion = 0.5;

extern "C" {

void ref_cg3_set_mixture(int thickness, double portion) {
  h_mix_thickness = thickness;
  h_mix_portion = portion;
}

int ref_cg3_create(const char* mask_path, const char* psi_path, int nx, int ny, int nz, int is_binary,
                   double nu_l, double nu_g, double psi_solid, double cap_a, double gx_in, double gy_in,
                   double gz_in, int body_force_phase, double flux_psi, double flux_umax) {
  std::strncpy(filename, mask_path, 127);
  filename[127] = 0;
  std::strncpy(filenamepsi, psi_path, 127);
  filenamepsi[127] = 0;
  NX = nx - 1; NY = ny - 1; NZ = nz - 1;
  decbin = is_binary;
  in_BC = 0; in_psi_BC = 0;
  psi_xp = psi_xn = psi_yp = psi_yn = psi_zp = psi_zn = 0;
  pre_xp = pre_xn = pre_yp = pre_yn = pre_zp = pre_zn = 0;
  vel_xp = vel_xn = vel_yp = vel_yn = vel_zp = vel_zn = 0;
  gx = gx_in; gy = gy_in; gz = gz_in;
  niu_l = nu_l; niu_g = nu_g;
  ContactAngle_parameter = psi_solid;
  CapA = cap_a;
  inivx = inivy = inivz = 0.0;
  PerDir = 1; lattice_v = 0;
  stab = 0; stab_time = 0;
  ini_Sat = -1; ini_buf = 0;
  rel_perm_psi = flux_psi; rel_perm_psi2 = flux_umax;
  par_per_x = par_per_y = par_per_z = 0;
  mix_psi_thickness = h_mix_thickness; protion_w = h_mix_portion; zero_sigma_thickness = 0;
  bodyforce_apply = body_force_phase;
  pressure_change = 0; pressure_change2 = 0; input_dynamic = 0;
  rel_perm_id_dir = 0; rel_perm_chan_num = 0;
  mirX = mirY = mirZ = 0;
  Zoom = 1;

  Parallelize_Geometry();
  c_rho = new double[Count + 1]();
  c_rho_r = new double[Count + 1]();
  c_rho_b = new double[Count + 1]();
  c_rhor = new double[Count + 1]();
  c_rhob = new double[Count + 1]();
  c_psi = new double[Count + 1]();
  c_u = rows(Count, 3);
  c_f = rows(Count, 19);
  c_F = rows(Count, 19);
  c_u0 = rows(Count, 3);
  c_SupInv = new int[Count + 1]();
  c_Per_l[0] = c_Per_l[1] = c_Per_l[2] = 0;
  c_Per_g[0] = c_Per_g[1] = c_Per_g[2] = 0;
  Comput_MI(M, MI);
  init(c_rho, c_u, c_f, c_psi, c_rho_r, c_rho_b, c_rhor, c_rhob, c_SupInv);
  return Count;
}

void ref_cg3_step(int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    collision(c_rho, c_u, c_f, c_F, c_psi, c_rho_r, c_rho_b, c_rhor, c_rhob, c_SupInv, Solid, nullptr, nullptr);
    comput_macro_variables(c_rho, c_u, c_u0, c_f, c_F, c_rho_r, c_rho_b, c_rhor, c_rhob, c_psi, c_SupInv);
  }
}

/* Comput_Perm: phase permeabilities (x,y,z for each phase) and u_ave. */
double ref_cg3_perm(double* perm_l, double* perm_g, double* uave_out) {
  double e = Comput_Perm(c_psi, c_u, c_Per_l, c_Per_g, PerDir, c_SupInv);
  for (int d = 0; d < 3; d++) {
    if (perm_l) perm_l[d] = c_Per_l[d];
    if (perm_g) perm_g[d] = c_Per_g[d];
  }
  if (uave_out) *uave_out = u_ave;
  return e;
}

double ref_cg3_saturation() { return Comput_Saturation(c_psi, Solid, c_SupInv); }

int ref_cg3_count() { return Count; }
double ref_cg3_porosity() { return porosity; }

void ref_cg3_get_coor(int32_t* out) {
  for (int i = 0; i <= Count; i++) out[i] = (i == 0) ? 0 : coor[i];
}
void ref_cg3_get_nei_loc(int32_t* out) {
  for (int q = 0; q < 19; q++) out[q] = 0;
  for (int i = 1; i <= Count; i++)
    for (int q = 0; q < 19; q++) out[(size_t)i * 19 + q] = nei_loc[i][q];
}
void ref_cg3_get_f(double* out) { std::memcpy(out, c_f[0], sizeof(double) * (size_t)(Count + 1) * 19); }
void ref_cg3_get_u(double* out) { std::memcpy(out, c_u[0], sizeof(double) * (size_t)(Count + 1) * 3); }
void ref_cg3_get_scalars(double* rho, double* psi, double* rho_r, double* rho_b) {
  const size_t b = sizeof(double) * (size_t)(Count + 1);
  if (rho) std::memcpy(rho, c_rho, b);
  if (psi) std::memcpy(psi, c_psi, b);
  if (rho_r) std::memcpy(rho_r, c_rho_r, b);
  if (rho_b) std::memcpy(rho_b, c_rho_b, b);
}
void ref_cg3_get_M(double* out) {
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 19; j++) out[i * 19 + j] = M[i][j];
}
void ref_cg3_get_MI(double* out) {
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 19; j++) out[i * 19 + j] = MI[i][j];
}
}
#pragma GCC visibility pop
