// lbm_st7 -- drop-in driver for the D3Q7 solute (passive scalar) solver.
//
//   lbm_st7 INPUT.dat [prefix] [--ranks N] [--precision f64|f32] [--lattice 7|19]
// (--lattice 19: the D3Q19 solute program, Solute_Transport_MPI_Software_
// Spars.cpp, "ST19": the same program with the 19-velocity lattice, 19
// columns in its g checkpoints, and bodyforce.txt emptied at start)
//
// Runs the time loop of Single_Phase_3D/Solute_Transport_MPI_Software_Spars_6V.cpp
// (main, ST7:187-730) on one GPU through liblbm.so.  The reference is an
// x-slab MPI program whose input and output files are per rank; --ranks N
// names the rank count of the run being replaced (the one that wrote the
// Velocity_for_solute_<sol_ini_n>.<rank>.bin files it reads), and the driver
// reads and writes the per-rank files of that decomposition
// (lbm_slab_partition).  Side effects, at the reference's steps:
// Results_solute.txt (previous and current report blocks, ST7:526-585),
// LBM_Geometry.vtk, LBM_velocity_Vector_<n>.vtk and LBM_psi_<n>.vtk in the
// Out_Mode 1 layout (z, y, x dimensions, one value per line, ST7:2235-2553,
// 3150-3296) or the Out_Mode 0 layout (x fastest, ST7:2695-3150), and
// LBM_checkpoint_{psi,fg}_<n>.<rank>.bin_input at fre_backup (Backup,
// ST7:3681-3714), the dispersion statistics of Sub_Dis 1-3 (plane sums of the
// concentration along x, y or z in Statistical_data_concentration_<X|Y|Z>_<n>.sta
// and the dispersion coefficient in bodyforce.txt, Statistical_psi
// ST7:3442-3638); USE BACKUP DATA restarts from those files in the working
// directory (Backup_init, ST7:3716-3802).
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

int die_msg(const std::string& what) {
  std::cerr << what << std::endl;
  return 1;
}

bool read_doubles(const std::string& path, double* dst, size_t n) {
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) return false;
  const size_t r = std::fread(dst, sizeof(double), n, fp);
  std::fclose(fp);
  return r == n;
}

bool write_doubles(const std::string& path, const double* src, size_t n) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const size_t w = std::fwrite(src, sizeof(double), n, fp);
  std::fclose(fp);
  return w == n;
}

// The decomposition the per-rank files follow: rank r's nodes are its slab's
// pore cells with i outer, j, k inner (the slab programs' compaction), each
// mapped to the library's reference id (pore cells numbered x fastest).
struct Slabs {
  int nranks = 1;
  std::vector<int> first_x;                 // [nranks+1]
  std::vector<std::vector<int32_t>> ids;    // per rank: reference ids in local order
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: lbm_st7 INPUT.dat [prefix] [--ranks N] [--precision f64|f32] [--lattice 7|19]" << std::endl;
    return 2;
  }
  std::string pfix = "./";
  int precision = LBM_PREC_F64, nranks = 1, lattice = 7;
  for (int a = 2; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--precision" && a + 1 < argc)
      precision = std::string(argv[++a]) == "f32" ? LBM_PREC_F32 : LBM_PREC_F64;
    else if (s == "--ranks" && a + 1 < argc)
      nranks = std::atoi(argv[++a]);
    else if (s == "--lattice" && a + 1 < argc)
      lattice = std::atoi(argv[++a]);
    else if (a == 2)
      pfix = s;
  }
  if (nranks < 1) return die_msg("--ranks must be at least 1");
  if (lattice != 7 && lattice != 19) return die_msg("--lattice is 7 or 19");
  const int W = lattice;  // columns of a g checkpoint row
  Clock clock;
  lbm_st7_input in;
  if (lbm_read_st7_input(argv[1], &in) != LBM_OK) return die("lbm_read_st7_input");
  // what the reference's loop does not run or this driver does not support
  if (in.lattice_v == 1 && !(in.dx_input > 0 && in.dt_input > 0))
    return die_msg("lattice_v: dx and dt must be positive");
  if (in.sub_dis > 0 && in.fre_dis == 0) return die_msg("freDis = 0: the reference takes n % 0; use -1 or a positive interval");
  if (in.fre_re <= 0) return die_msg("freRe must be positive");
  if (in.fre_ve == 0 || in.fre_psi == 0 || in.fre_backup == 0)
    return die_msg("freVe / frePsi / fre_backup = 0: the reference takes n % 0; use -1 or a positive interval");
  const int nx = in.nx, ny = in.ny, nz = in.nz;
  const size_t cells = (size_t)nx * ny * nz;
  const std::string out = in.output_path;

  std::vector<uint8_t> mask(cells);
  if (lbm_read_mask(in.geometry_file, nx, ny, nz, in.decbin, mask.data()) != LBM_OK) return die("lbm_read_mask");
  std::vector<double> c0(cells);
  if (lbm_read_phase(in.conc_file, nx, ny, nz, c0.data()) != LBM_OK) return die("lbm_read_phase");
  std::vector<int32_t> ref_id(cells, 0);  // reference id of each pore cell, x fastest
  int count = 0;
  for (size_t c = 0; c < cells; c++)
    if (mask[c] == 0) ref_id[c] = ++count;
  Slabs sl;
  sl.nranks = nranks;
  sl.first_x.assign(nranks + 1, 0);
  if (lbm_slab_partition(mask.data(), nx, ny, nz, nranks, sl.first_x.data()) != LBM_OK)
    return die("lbm_slab_partition");
  sl.ids.resize(nranks);
  for (int r = 0; r < nranks; r++)
    for (int i = sl.first_x[r]; i < sl.first_x[r + 1]; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
          const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
          if (mask[c] == 0) sl.ids[r].push_back(ref_id[c]);
        }

  // Backup_input_v (ST7:3640-3667): each rank reads its Count*3 velocities
  std::vector<double> u((size_t)(count + 1) * 3, 0.0);
  for (int r = 0; r < nranks; r++) {
    std::ostringstream name;
    name << pfix << "Velocity_for_solute_" << in.sol_ini_n << "." << r << ".bin";
    std::vector<double> lsu(sl.ids[r].size() * 3);
    if (!read_doubles(name.str(), lsu.data(), lsu.size()))
      return die_msg("file open error on " + name.str() + " (or shorter than Count*3 doubles)");
    for (size_t s = 0; s < sl.ids[r].size(); s++)
      for (int d = 0; d < 3; d++) u[(size_t)sl.ids[r][s] * 3 + d] = lsu[s * 3 + d];
  }
  lbm_st7_params p{};
  p.diffusivity = in.nu_s;
  p.precision = precision;
  p.device = 0;
  lbm_st7_handle* h = nullptr;
  if ((lattice == 19 ? lbm_st19_create(&p, mask.data(), nx, ny, nz, u.data(), c0.data(), &h)
                     : lbm_st7_create(&p, mask.data(), nx, ny, nz, u.data(), c0.data(), &h)) != LBM_OK)
    return die("lbm_st7_create");
  // init: dx = dt = 1 / Zoom (Zoom = 1), or the INPUT file's dx, dt with
  // lattice_v (ST7:1259-1274)
  const double dx = in.lattice_v == 1 ? in.dx_input : 1.0, dt = in.lattice_v == 1 ? in.dt_input : 1.0;
  if (in.lattice_v == 1 && lbm_st7_set_lattice(h, dx, dt) != LBM_OK) return die("lbm_st7_set_lattice");
  if (in.mode_backup_ini != 0) {
    // Backup_init reads LBM_checkpoint_{psi,fg}_<m>.<rank>.bin_input from the
    // working directory, without the output prefix (ST7:3735-3740)
    std::vector<double> c((size_t)count + 1, 0.0), g((size_t)(count + 1) * W, 0.0);
    for (int r = 0; r < nranks; r++) {
      const size_t nr = sl.ids[r].size();
      std::ostringstream n3, n5;
      n3 << "LBM_checkpoint_psi_" << in.mode_backup_ini << "." << r << ".bin_input";
      n5 << "LBM_checkpoint_fg_" << in.mode_backup_ini << "." << r << ".bin_input";
      std::vector<double> pr(nr + 1), gr((nr + 1) * W);
      if (!read_doubles(n3.str(), pr.data(), pr.size())) return die_msg("file open error on" + n3.str());
      if (!read_doubles(n5.str(), gr.data(), gr.size())) return die_msg("file open error on" + n5.str());
      for (size_t s = 0; s < nr; s++) {
        const int32_t id = sl.ids[r][s];
        c[id] = pr[s + 1];
        for (int q = 0; q < W; q++) g[(size_t)id * W + q] = gr[(s + 1) * W + q];
      }
    }
    if (lbm_st7_set_state(h, g.data(), c.data()) != LBM_OK) return die("lbm_st7_set_state");
  }
  std::cout << std::endl << "INITIALIZATION COMPLETED" << std::endl << std::endl;

  // cell values in the two layouts: Out_Mode 1 walks i outer, k inner with
  // the dimensions written z, y, x; Out_Mode 0 walks x fastest
  const bool mode1 = in.out_mode == 1;
  auto header = [&](std::ofstream& o, const char* title) {
    o << "# vtk DataFile Version 2.0" << std::endl;
    o << title << std::endl;
    o << "ASCII" << std::endl;
    o << "DATASET STRUCTURED_POINTS" << std::endl;
    if (mode1)
      o << "DIMENSIONS         " << nz << "         " << ny << "         " << nx << std::endl;
    else
      o << "DIMENSIONS         " << nx << "         " << ny << "         " << nz << std::endl;
    o << "ORIGIN 0 0 0" << std::endl;
    o << "SPACING 1 1 1" << std::endl;
    o << "POINT_DATA     " << nx * ny * nz << std::endl;
  };
  auto for_cells = [&](auto&& visit) {
    if (mode1) {
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) visit(i + (size_t)nx * (j + (size_t)ny * k));
    } else {
      for (size_t c = 0; c < cells; c++) visit(c);
    }
  };
  {
    // Geometry / Geometry_b (ST7:2235-2377, 2695-2790): 1 on solids, 0 on pores
    std::ofstream o(out + "LBM_Geometry.vtk");
    header(o, "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Solid-Geometry");
    o << "SCALARS sample_scalars float" << std::endl;
    o << "LOOKUP_TABLE default" << std::endl;
    for_cells([&](size_t c) { o << (mask[c] == 0 ? 0 : 1) << std::endl; });
  }
  const std::string f_res = out + "Results_solute.txt";
  { std::ofstream(f_res, std::ios::trunc); }
  // the D3Q19 program empties bodyforce.txt at start (ST19:518), the D3Q7 one
  // only appends to it
  if (lattice == 19) std::ofstream(out + "bodyforce.txt", std::ios::trunc);

  // Error (ST7:2159-2233) on the fixed velocity: every rank skips its last
  // node (its loop stops at Count - 1); rank sums are added in rank order
  double u_max_e = 0, u_ave_e = 0;
  {
    double v_max = 0, u_compt = 0;
    for (int r = 0; r < nranks; r++) {
      double temp3 = 0, m2 = 0;
      const size_t nr = sl.ids[r].size();
      for (size_t s = 0; s + 1 < nr; s++) {
        const double* v = &u[(size_t)sl.ids[r][s] * 3];
        temp3 += std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] > m2) m2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      }
      const double um = std::sqrt(m2);
      if (um > v_max) v_max = um;
      u_compt += temp3;
    }
    u_compt /= (double)cells;
    u_max_e = v_max;
    u_ave_e = u_compt;
  }
  const double lat_c = dx / dt, c_s2 = lat_c * lat_c / 3;
  // psi_total (ST7:1083-1105): every rank sums the initial concentration of
  // its pore cells (i, j, k order, the float values), rank 0 adds the ranks
  double psi_total = 0;
  {
    for (int r = 0; r < nranks; r++) {
      double part = 0;
      for (int i = sl.first_x[r]; i < sl.first_x[r + 1]; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) {
            const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
            if (mask[c] == 0) part += c0[c];
          }
      psi_total += part;
    }
  }
  // the statistics window: an axis without a partial window spans the box (ST7:853-858)
  const int win[6] = {in.par_per_x ? in.per_xn : 0, in.par_per_x ? in.per_xp : nx - 1,
                      in.par_per_y ? in.per_yn : 0, in.par_per_y ? in.per_yp : ny - 1,
                      in.par_per_z ? in.per_zn : 0, in.par_per_z ? in.per_zp : nz - 1};
  double dispersion = 0, disp_pre = 0;
  // Statistical_psi: plane sums of C along the axis, in the reference's
  // summation order (a plane along x lies in one rank; along y or z every
  // rank sums its slab and rank 0 adds the ranks)
  auto statistics = [&](long long m, const std::vector<double>& conc) -> bool {
    const int ax = in.sub_dis - 1;
    if (ax < 0 || ax > 2) return true;
    const int len = ax == 0 ? nx : (ax == 1 ? ny : nz);
    std::vector<double> s_psi(len, 0.0);
    if (ax == 0) {
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) {
            const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
            if (mask[c] == 0) s_psi[i] += conc[ref_id[c]];
          }
    } else {
      std::vector<double> part(len);
      for (int r = 0; r < nranks; r++) {
        std::fill(part.begin(), part.end(), 0.0);
        for (int a2 = 0; a2 < len; a2++)
          for (int i = sl.first_x[r]; i < sl.first_x[r + 1]; i++)
            for (int b = 0; b < (ax == 1 ? nz : ny); b++) {
              const int j = ax == 1 ? a2 : b, k = ax == 1 ? b : a2;
              const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
              if (mask[c] == 0) part[a2] += conc[ref_id[c]];
            }
        for (int a2 = 0; a2 < len; a2++) s_psi[a2] += part[a2];
      }
    }
    std::ostringstream name;
    name << out << "Statistical_data_concentration_" << "XYZ"[ax] << "_" << m << ".sta";
    std::ofstream o(name.str());
    if (!o) return false;
    double EX = 0, EX2 = 0;
    for (int i = win[2 * ax]; i <= win[2 * ax + 1]; i++) {
      o << s_psi[i] << std::endl;
      EX += i * dx * s_psi[i] / psi_total;
      EX2 += (i * dx * i * dx) * s_psi[i] / psi_total;
    }
    const double DX = EX2 - EX * EX;
    dispersion = (DX - disp_pre) * 0.5 / (in.fre_dis * dt);
    disp_pre = DX;
    return true;
  };
  const double s_v = 1 / (in.nu / (c_s2 * dt) + 0.5);
  double u_max = 0, u_ave = 0, Re = 0;
  int the = 0, tme = 0, tse = 0, th = 0, tm = 0, ts = 0;
  auto block = [&](std::ostream& o, long long nn) {
    o << "The" << nn << "th computation result:" << std::endl;
    o << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re=" << Re << std::endl;
    o << "Peclet Number=" << u_max * dx / in.nu_s << "     Courant Number=" << u_max * dt / dx << std::endl;
    o << "The averaged velocity is: " << u_ave << std::endl;
    o << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    o << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
    o << std::endl;
  };
  std::vector<double> conc((size_t)count + 1);

  long long n = 0;
  while (n <= in.n_max) {
    long long last = ((n + in.fre_re - 1) / in.fre_re) * in.fre_re;
    if (last > in.n_max) last = in.n_max;
    if (lbm_st7_step(h, (int)(last - n + 1)) != LBM_OK) return die("lbm_st7_step");
    n = last;
    if (n % in.fre_re != 0) {
      n++;
      continue;
    }
    {
      std::ofstream fin(f_res, std::ios::out);
      block(fin, n - in.fre_re);
    }
    u_max = u_max_e;
    u_ave = u_ave_e;
    {
      const double finish = clock.now();
      Re = u_ave * ny / (1.0 / 3.0 * (1 / s_v - 0.5));
      hms(n > 0 ? (in.n_max - n) * (finish / n) : 0.0, &th, &tm, &ts);
      hms(finish, &the, &tme, &tse);
      std::ofstream fin(f_res, std::ios::app);
      block(fin, n);
    }
    std::cout << "The" << n << "th computation result:" << std::endl;
    std::cout << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re=" << Re << std::endl;
    std::cout << "Peclet Number=" << u_max * dx / in.nu_s << "     Courant Number=" << u_max * dt / dx << std::endl;
    std::cout << "The averaged velocity is: " << u_ave << std::endl;
    std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    std::cout << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
    std::cout << std::endl;

    std::ostringstream tag;
    tag << n;
    if (in.fre_ve >= 0 && n % in.fre_ve == 0) {
      std::ofstream o(out + "LBM_velocity_Vector_" + tag.str() + ".vtk");
      header(o, "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Velocity");
      o << "VECTORS sample_vectors double" << std::endl;
      o << std::endl;
      for_cells([&](size_t c) {
        const double* v = &u[(size_t)ref_id[c] * 3];
        const bool pore = mask[c] == 0;
        if (mode1) {
          if (pore)
            o << v[2] << " " << v[1] << " " << v[0] << std::endl;
          else
            o << 0.0 << " " << 0.0 << " " << 0.0 << std::endl;
        } else {
          if (pore)
            o << v[0] << " " << v[1] << " " << v[2] << " " << std::endl;
          else
            o << 0.0 << " " << 0.0 << " " << 0.0 << " " << std::endl;
        }
      });
    }
    const bool stats = in.fre_dis >= 0 && n % in.fre_dis == 0 && in.sub_dis > 0;
    const bool want_c = (in.fre_psi >= 0 && n % in.fre_psi == 0) ||
                        (in.fre_backup >= 0 && n % in.fre_backup == 0 && n > 0) || stats;
    if (want_c && lbm_st7_get_concentration(h, conc.data()) != LBM_OK) return die("lbm_st7_get_concentration");
    if (in.fre_psi >= 0 && n % in.fre_psi == 0) {
      std::ofstream o(out + "LBM_psi_" + tag.str() + ".vtk");
      header(o, "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Solid-Density");
      o << "SCALARS sample_scalars float" << std::endl;
      o << "LOOKUP_TABLE default" << std::endl;
      for_cells([&](size_t c) { o << (mask[c] == 0 ? conc[ref_id[c]] : in.ref_psi) << std::endl; });
    }
    if (stats) {
      if (!statistics(n, conc)) return die_msg("cannot write the statistics of step " + tag.str());
      if (n > in.ini_psi) {
        // appended without emptying the file first, as the reference does (ST7:510-517, 682-686)
        std::ofstream(out + "bodyforce.txt", std::ios::app) << dispersion << "  " << disp_pre << std::endl;
      }
    }
    if (in.fre_backup >= 0 && n % in.fre_backup == 0 && n > 0) {
      std::vector<double> g((size_t)(count + 1) * W);
      if (lbm_st7_get_populations(h, g.data()) != LBM_OK) return die("lbm_st7_get_populations");
      for (int r = 0; r < nranks; r++) {
        const size_t nr = sl.ids[r].size();
        std::vector<double> pr(nr + 1, 0.0), gr((nr + 1) * W, 0.0);
        for (size_t s = 0; s < nr; s++) {
          const int32_t id = sl.ids[r][s];
          pr[s + 1] = conc[id];
          for (int q = 0; q < W; q++) gr[(s + 1) * W + q] = g[(size_t)id * W + q];
        }
        std::ostringstream n3, n5;
        n3 << out << "LBM_checkpoint_psi_" << n << "." << r << ".bin_input";
        n5 << out << "LBM_checkpoint_fg_" << n << "." << r << ".bin_input";
        if (!write_doubles(n3.str(), pr.data(), pr.size()) || !write_doubles(n5.str(), gr.data(), gr.size()))
          return die_msg("cannot write the checkpoint of step " + tag.str());
      }
    }
    n++;
  }
  std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
  std::cout << "Accuracy: " << 1e-9 << " Second" << std::endl;
  {
    std::ofstream fin(f_res, std::ios::app);
    fin << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    fin << "Accuracy: " << 1e-9 << " Second" << std::endl;
  }
  lbm_st7_destroy(h);
  return 0;
}
