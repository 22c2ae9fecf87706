// lbm_sp -- drop-in driver for the single-phase sparse solver.
//
//   lbm_sp INPUT.dat [checkpoint_prefix] [--precision f64|f32|f16|f64fast]
//          [--ordering reference|morton|hilbert|brick|auto] [--stop-on-convergence]
//
// Runs the time loop of Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp
// (main, SP3:258-795) on the GPU through liblbm.so and produces the same side
// effects: Results.txt (previous and current report blocks, SP3:596-660),
// Permeability_error_local_Perm.txt, bodyforce.txt, Velocity_ave_max.txt,
// LBM_Geometry.vtk, LBM_velocity_Vector_<n>.vtk / LBM_Density_<n>.vtk at
// freVe / freDe, LBM_checkpoint_* at fre_backup and at the end,
// Velocity_for_solute_<n>.0.bin at vel_sol, General_Results.txt, and the
// reference's stop rules (NaN, five reports with u_max >= 10).  With
// --stop-on-convergence it also applies the slab solver's stop test
// |(u_ave_prev - u_ave)/u_ave_prev| < 1e-7 (SP:812-816).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "lbm.h"

namespace {

int parse_precision(const std::string& s) {
  if (s == "f32") return LBM_PREC_F32;
  if (s == "f16") return LBM_PREC_F16;
  if (s == "f64fast") return LBM_PREC_F64_FAST;
  return LBM_PREC_F64;
}
int parse_ordering(const std::string& s) {
  if (s == "morton") return LBM_ORDER_MORTON;
  if (s == "hilbert") return LBM_ORDER_HILBERT;
  if (s == "brick") return LBM_ORDER_BRICK;
  if (s == "auto") return LBM_ORDER_AUTO;
  return LBM_ORDER_REFERENCE;
}

struct Clock {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

void hms(double s, int* h, int* m, int* sec) {
  if (!(s >= 0) || s > 1e9) s = 0;
  *h = int(s / 3600);
  *m = int((s - *h * 3600) / 60);
  *sec = int(s - (*h * 3600 + *m * 60));
}

int die(const char* what) {
  std::cerr << what << ": " << lbm_last_error() << std::endl;
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: lbm_sp INPUT.dat [checkpoint_prefix] [--precision f64|f32|f16|f64fast] "
                 "[--ordering reference|morton|hilbert|brick|auto] [--stop-on-convergence]"
              << std::endl;
    return 2;
  }
  std::string pfix = "./";
  int precision = LBM_PREC_F64, ordering = LBM_ORDER_REFERENCE;
  bool stop_conv = false;
  for (int a = 2; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--precision" && a + 1 < argc)
      precision = parse_precision(argv[++a]);
    else if (s == "--ordering" && a + 1 < argc)
      ordering = parse_ordering(argv[++a]);
    else if (s == "--stop-on-convergence")
      stop_conv = true;
    else if (a == 2)
      pfix = s;
  }
  Clock clock;
  lbm_input in;
  lbm_handle* h = nullptr;
  if (lbm_create_from_input(argv[1], precision, ordering, &h, &in) != LBM_OK) return die("lbm_create_from_input");
  const int nx = in.nx, ny = in.ny, nz = in.nz;
  const int NY = ny - 1;
  const std::string out = in.output_path;
  if (in.mode_backup_ini != 0 && lbm_read_checkpoint(h, pfix.c_str(), in.mode_backup_ini) != LBM_OK)
    return die("lbm_read_checkpoint");
  std::cout << std::endl << "INITIALIZATION COMPLETED" << std::endl << std::endl;

  if (in.out_mode == 1 || in.fre_ve >= 0 || in.fre_de >= 0) {
    std::vector<uint8_t> mask((size_t)nx * ny * nz);
    if (lbm_read_mask(in.geometry_file, nx, ny, nz, in.decbin, mask.data()) != LBM_OK) return die("lbm_read_mask");
    if (in.out_mode == 1) {
      // Geometry_Par (SP3:3249-3283): the partition index of each cell, 1 for
      // every pore cell of a one-device solve and 0 for solids.
      std::vector<uint8_t> part(mask.size());
      for (size_t c = 0; c < mask.size(); c++) part[c] = mask[c] == 0;
      if (lbm_write_vtk_geometry(part.data(), nx, ny, nz, (out + "LBM_Geometry_Mesh.vtk").c_str()) != LBM_OK)
        return die("lbm_write_vtk_geometry");
    }
    if ((in.fre_ve >= 0 || in.fre_de >= 0) &&
        lbm_write_vtk_geometry(mask.data(), nx, ny, nz, (out + "LBM_Geometry.vtk").c_str()) != LBM_OK)
      return die("lbm_write_vtk_geometry");
  }
  const std::string f_res = out + "Results.txt", f_perm = out + "Permeability_error_local_Perm.txt",
                    f_bf = out + "bodyforce.txt", f_vel = out + "Velocity_ave_max.txt";
  { std::ofstream(f_res, std::ios::trunc); }
  if (in.wr_per == 1) { std::ofstream(f_perm, std::ios::trunc); }
  { std::ofstream(f_bf, std::ios::out); }
  { std::ofstream(f_vel, std::ios::out); }

  const double reso2k = in.reso * in.reso * 1000;
  // init's lattice (SP3:1286-1298): dx, dt of a self-defined lattice
  // velocity, else 1; s_v = 1 / tau_f with tau_f = nu / (c_s^2 dt) + 0.5
  const double dt = in.lattice_v == 1 ? in.dt_input : 1.0, dx = in.lattice_v == 1 ? in.dx_input : 1.0;
  const double lat_c = dx / dt, c_s2 = lat_c * lat_c / 3;
  const double s_v = 1 / (in.in_vis / (c_s2 * dt) + 0.5);
  double perm[3] = {0, 0, 0}, error_perm = 0, u_max = 0, error = 0, u_ave = 0, pre_u_ave = 0, Re = 0;
  int the = 0, tme = 0, tse = 0, th = 0, tm = 0, ts = 0;
  int u_max_ref = 0;
  const int fre_re = in.fre_re > 0 ? in.fre_re : 1;
  int count = 0;
  double porosity = 0;
  long long done = 0;
  lbm_info(h, &count, &porosity, &done);
  std::vector<double> rho((size_t)count + 1);

  auto block = [&](std::ostream& o, long long nn) {
    o << "The" << nn << "th computation result:" << std::endl;
    o << "The permiability is: " << perm[0] * reso2k << ", " << perm[1] * reso2k << ", " << perm[2] * reso2k
      << std::endl;
    o << "The relative error of permiability computing is: " << error_perm << std::endl;
    o << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re=" << Re
      << "     Courant Number=" << u_max * dt / dx << std::endl;
    o << "The max relative error of velocity is: " << std::setiosflags(std::ios::scientific) << error << std::endl;
  };

  long long n = 0;
  for (n = 0; n <= in.n_max;) {
    // advance to the end of step n, where n is the next reporting step
    long long next = ((n + fre_re - 1) / fre_re) * fre_re;  // first n' >= n with n' % freRe == 0
    if (next > in.n_max) next = in.n_max;
    if (lbm_step(h, (int)(next - n + 1)) != LBM_OK) return die("lbm_step");
    n = next;
    if (n % fre_re != 0) {
      n++;
      continue;
    }
    {
      std::ofstream fin(f_res, std::ios::out);
      block(fin, n - fre_re);
      fin << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
      fin << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
      fin << std::endl;
    }
    pre_u_ave = u_ave;
    lbm_diag d;
    if (lbm_reduce(h, &d) != LBM_OK) return die("lbm_reduce");
    error = d.u_rel_change;
    u_max = d.u_max;
    if (u_max >= 10.0) u_max_ref += 1;
    error_perm = d.perm_rel_change;
    for (int i = 0; i < 3; i++) perm[i] = d.perm[i];
    u_ave = d.u_ave;
    {
      const double finish = clock.now();
      hms(n > 0 ? (in.n_max - n) * (finish / n) : 0.0, &th, &tm, &ts);
      hms(finish, &the, &tme, &tse);
      std::ofstream fin(f_res, std::ios::app);
      Re = u_ave * (NY + 1) / (1.0 / 3.0 * (1 / s_v - 0.5));
      block(fin, n);
      fin << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
      fin << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
      fin << std::endl;
    }
    if (in.wr_per == 1) {
      std::ofstream finfs(f_perm, std::ios::app);
      const int dir = (in.perdir >= 1 && in.perdir <= 3) ? in.perdir - 1 : 0;
      finfs << perm[dir] * reso2k << " " << error_perm << " " << std::endl;
    }
    { std::ofstream(f_bf, std::ios::app) << in.gx << std::endl; }
    {
      std::ofstream(f_vel, std::ios::app) << u_ave << "  " << u_max << " " << error << "  "
                                          << std::abs((pre_u_ave - u_ave) / (u_ave + 1e-20)) << std::endl;
    }
    if (lbm_get_fields(h, rho.data(), nullptr) != LBM_OK) return die("lbm_get_fields");
    std::cout << "The" << n << "th computation result:" << std::endl;
    std::cout << "The Density of point(NX/2,NY/2,NZ/2) is: " << std::setprecision(6) << rho[count / 2] << std::endl;
    std::cout << "The permiability is: " << perm[0] * reso2k << ", " << perm[1] * reso2k << ", " << perm[2] * reso2k
              << std::endl;
    std::cout << "The relative error of permiability computing is: " << error_perm << std::endl;
    std::cout << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re=" << Re
              << "     Courant Number=" << u_max * dt / dx << std::endl;
    std::cout << "The average velocity is: " << std::setprecision(6) << u_ave << std::endl;
    std::cout << "The max relative error of uv is: " << std::setiosflags(std::ios::scientific) << error << std::endl;
    std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    std::cout << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
    std::cout << std::endl;  // like the reference, stdout stays in scientific notation from here on

    std::ostringstream tag;
    tag << n;
    if (in.fre_de > 0 && n % in.fre_de == 0 && n > 0 &&
        lbm_write_vtk_density(h, (out + "LBM_Density_" + tag.str() + ".vtk").c_str()) != LBM_OK)
      return die("lbm_write_vtk_density");
    if (in.fre_ve > 0 && n % in.fre_ve == 0 && n > 0 &&
        lbm_write_vtk_velocity(h, (out + "LBM_velocity_Vector_" + tag.str() + ".vtk").c_str()) != LBM_OK)
      return die("lbm_write_vtk_velocity");
    if (in.fre_backup > 0 && n % in.fre_backup == 0 && n > 0 && lbm_write_checkpoint(h, out.c_str(), n) != LBM_OK)
      return die("lbm_write_checkpoint");
    if (in.vel_sol > 0 && n % in.vel_sol == 0 && n > 0 &&
        lbm_write_velocity_for_solute_ordered(h, (out + "Velocity_for_solute_" + tag.str() + ".0.bin").c_str(),
                                              LBM_SOLUTE_ORDER_XFAST) != LBM_OK)
      return die("lbm_write_velocity_for_solute");
    if (error != error) {
      std::cout << "PROGRAM STOP" << std::endl;
      break;
    }
    if (u_max_ref >= 5) {
      std::cout << "PROGRAM STOP DUE TO HIGH VELOCITY" << std::endl;
      break;
    }
    if (stop_conv && std::abs((pre_u_ave - u_ave) / pre_u_ave) < 1e-7) break;
    n++;
  }
  if (in.fre_backup >= 0 && lbm_write_checkpoint(h, out.c_str(), in.n_max) != LBM_OK)
    return die("lbm_write_checkpoint");
  std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
  std::cout << "Accuracy: " << 1e-9 << " Second" << std::endl;
  {
    std::ofstream fin(f_res, std::ios::app);
    fin << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    fin << "Accuracy: " << 1e-9 << " Second" << std::endl;
  }
  {
    std::ofstream fin(out + "General_Results.txt", std::ios::app);
    fin << in.geometry_file << "  " << perm[0] * reso2k << " " << perm[1] * reso2k << " " << perm[2] * reso2k
        << std::endl;
    fin << std::endl;
  }
  lbm_destroy(h);
  return 0;
}
