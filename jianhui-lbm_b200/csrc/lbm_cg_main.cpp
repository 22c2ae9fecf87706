// lbm_cg -- drop-in driver for the colour-gradient two-phase sparse solver.
//
//   lbm_cg INPUT.dat [checkpoint_prefix] [--precision f64|f32] [--seed N]
//
// Runs the time loop of MP_3D/Multi_Component_CG_MPI_SPARSE_Software_3DPartition.cpp
// (main, CG3:336-1100) on the GPU through liblbm.so and produces the same side
// effects: Results.txt (previous and current report blocks, CG3:896-1005),
// Relative_Permeability_Component1/2.txt, bodyforce.txt, Velocity_ave_max.txt,
// the emptied Capillary_Pressure.txt and Imb_Drai_Rel_Perm.txt,
// LBM_Geometry.vtk / LBM_Geometry_Mesh.vtk, LBM_Density_<n>.vtk,
// LBM_velocity_Vector_<n>.vtk and LBM_psi_<n>.vtk at freDe / freVe / frePsi,
// LBM_checkpoint_* at fre_backup and at the end, and the stop after five
// reports with u_max >= 10.  Parameter schedules run between steps: the
// stabiliser's force switch at stab_time (CG3:851-852), the force or pressure
// ramps of pressure_change (pressure_bodyforce_change, CG3:1252-1420), the
// surface-tension change of rel_perm_ift (CG3:892-893) and the least-squares
// fit of the relative permeabilities (Least_Square_Rel_Perm, CG3:1201-1250)
// and the capillary-pressure stepping (pressure_capillary, CG3:1427-1600),
// and with input_dynamic the INPUT file read again every update_fre steps
// (input_update, CG3:859-861, 5765-5925).
// Pressure and velocity faces (boundary_pressure / boundary_velocity,
// CG3:868-876) follow the face densities these schedules move.
#include <algorithm>
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

// Body force and face pressures the run is at (gxs.., p_xn..).
struct Drive {
  double g[3];
  double p_n[3], p_p[3];
};

// pressure_bodyforce_change (CG3:1252-1420) at step n: piecewise-linear
// ramps through five (step, p_n, p_p, force) points along the axis
// pressure_change names.  Kept as written: the first segment of the y and z
// ramps starts from gx, and the fifth segment is taken for every step in
// (pre_chan_3, pre_chan_5].  Returns true when the force changed.
bool ramp(const lbm_cg_input& in, long long n, const double g_in[3], const double p_n0[3], const double p_p0[3],
          Drive* d) {
  const int a = in.pressure_change - 1;
  if (a < 0 || a > 2) return false;
  const int* c = in.pre_chan;
  const double *pn = in.pre_chan_pn, *pp = in.pre_chan_pp, *f = in.pre_chan_f;
  const bool pressure = in.pre_chan_pb == 1;
  const double g_before = d->g[a];
  auto seg = [&](double pn0, double pp0, double f0, int k, double den, double c_hi) {
    const double s = 1 - (double)(c_hi - n) / den;
    if (pressure) {
      d->p_n[a] = pn0 + (pn[k] - pn0) * s;
      d->p_p[a] = pp0 + (pp[k] - pp0) * s;
    } else {
      d->g[a] = f0 + (f[k] - (k == 0 ? g_in[a] : f0)) * s;
    }
  };
  if (n <= c[0]) seg(p_n0[a], p_p0[a], g_in[0], 0, (double)c[0], c[0]);
  if (n <= c[1] && n > c[0]) seg(pn[0], pp[0], f[0], 1, (double)(c[1] - c[0]), c[1]);
  if (n <= c[2] && n > c[1]) seg(pn[1], pp[1], f[1], 2, (double)(c[2] - c[1]), c[2]);
  if (n <= c[3] && n > c[2]) seg(pn[2], pp[2], f[2], 3, (double)(c[3] - c[2]), c[3]);
  if (n <= c[4] && n > c[2]) seg(pn[3], pp[3], f[3], 4, (double)(c[4] - c[3]), c[4]);
  return !pressure && !(d->g[a] == g_before || (d->g[a] != d->g[a] && g_before != g_before));
}

// Whether any ramp segment covers step n.
bool ramp_at(const lbm_cg_input& in, long long n) {
  if (in.pressure_change < 1 || in.pressure_change > 3) return false;
  const int* c = in.pre_chan;
  return n <= c[0] || (n <= c[1] && n > c[0]) || (n <= c[2] && n > c[1]) || (n <= c[3] && n > c[2]) ||
         (n <= c[4] && n > c[2]);
}

// pressure_capillary (CG3:1427-1600): capillary-pressure stepping.  From
// step start to start + interval_pre the force (or the face pressures) along
// the axis of pressure_change2 ramps by 1/chan_no of the way to its target;
// then, once the saturation changed by less than sat_cri_d between reports
// for sat_cri reports after the first such one, the reached value becomes
// the new base, the point (S_l, 1 - S_l, force x length or |dp|/3) goes to
// Capillary_Pressure.txt and the next ramp starts, chan_no times.
struct Capillary {
  bool on = false;
  int a = 0;
  bool pressure = false;
  double pre_in = 0, pre_ip = 0;
  int error_sat = 0, ind = 0, num = 0;
  long long start = 0;
  bool ramping(const lbm_cg_input& in, long long n) const {
    return on && num < in.chan_no && n <= start + in.interval_pre;
  }
};

// One step's update; returns true when the force changed.
bool capillary_step(const lbm_cg_input& in, Capillary& cp, long long n, double S_l, double S_l_r, double gbase[3],
                    double p_n0[3], double p_p0[3], Drive* d, const std::string& f_cap, const int len[3]) {
  if (!cp.on) return false;
  const int a = cp.a;
  const double err = std::abs((S_l_r - S_l) / S_l);
  const long long lim = cp.start + in.interval_pre;
  if (err < in.sat_cri_d && n % in.fre_re == 0 && n > lim && cp.num < in.chan_no) {
    if (cp.ind == 1) {
      cp.error_sat += 1;
    } else {
      cp.error_sat = 0;
      cp.ind = 1;
    }
  } else if (err >= in.sat_cri_d && n % in.fre_re == 0 && n > lim && cp.num < in.chan_no) {
    cp.ind = 0;
    cp.error_sat = 0;
  }
  bool changed = false;
  if (n <= lim && cp.num < in.chan_no) {
    const double s = 1 - (double)(lim - n) / in.interval_pre;
    if (cp.pressure) {
      d->p_n[a] = p_n0[a] + cp.pre_in * s;
      d->p_p[a] = p_p0[a] + cp.pre_ip * s;
    } else {
      const double before = d->g[a];
      d->g[a] = gbase[a] + cp.pre_in * s;
      changed = !(d->g[a] == before);
    }
  }
  if (cp.error_sat >= in.sat_cri) {
    cp.error_sat = 0;
    cp.ind = 0;
    cp.start = n;
    cp.num++;
    std::ofstream fc(f_cap, std::ios::app);
    if (cp.pressure) {
      p_n0[a] = d->p_n[a];
      p_p0[a] = d->p_p[a];
      fc << S_l << " " << 1 - S_l << " " << std::abs(d->p_p[a] - d->p_n[a]) / 3 << std::endl;
    } else {
      gbase[a] = d->g[a];
      fc << S_l << " " << 1 - S_l << " " << d->g[a] * len[a] << std::endl;
    }
  }
  return changed;
}

// Least_Square_Rel_Perm (CG3:1201-1250): a line through the last
// num_least_square values (newest first) evaluated at the newest point.
struct LeastSquares {
  std::vector<double> l, g;
  double rel_l = 0, rel_g = 0, slope_l = 0, slope_g = 0;
  void push(double per_l, double per_g) {
    const int m = (int)l.size();
    for (int i = m - 1; i > 0; i--) {
      l[i] = l[i - 1];
      g[i] = g[i - 1];
    }
    l[0] = per_l;
    g[0] = per_g;
    double xs = 0.0, sl = 0.0, sg = 0.0;
    for (int i = 0; i < m; i++) {
      xs += (double)i;
      sl += l[i];
      sg += g[i];
    }
    sl /= (double)m;
    sg /= (double)m;
    xs /= (double)m;
    double s2l = 0.0, s2g = 0.0, sb = 0.0;
    for (int i = 0; i < m; i++) {
      s2l += (i - xs) * (l[i] - sl);
      s2g += (i - xs) * (g[i] - sg);
      sb += (i - xs) * (i - xs);
    }
    slope_l = s2l / sb;
    slope_g = s2g / sb;
    rel_l = sl - slope_l * xs;
    rel_g = sg - slope_g * xs;
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: lbm_cg INPUT.dat [checkpoint_prefix] [--precision f64|f32] [--seed N]" << std::endl;
    return 2;
  }
  std::string pfix = "./";
  int precision = LBM_PREC_F64;
  unsigned long long seed = 0;  // random initial phase and random phase faces
  for (int a = 2; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--precision" && a + 1 < argc)
      precision = std::string(argv[++a]) == "f32" ? LBM_PREC_F32 : LBM_PREC_F64;
    else if (s == "--seed" && a + 1 < argc)
      seed = std::stoull(argv[++a]);
    else if (a == 2)
      pfix = s;
  }
  Clock clock;
  lbm_cg_input in;
  lbm_cg_handle* h = nullptr;
  if (lbm_cg_create_from_input_seeded(argv[1], precision, seed, &h, &in) != LBM_OK)
    return die("lbm_cg_create_from_input");
  const int nx = in.nx, ny = in.ny, nz = in.nz;
  const std::string out = in.output_path;

  if (in.out_mode == 1 || in.fre_ve >= 0 || in.fre_de >= 0) {
    std::vector<uint8_t> mask((size_t)nx * ny * nz);
    if (lbm_read_mask(in.geometry_file, nx, ny, nz, in.decbin, mask.data()) != LBM_OK) return die("lbm_read_mask");
    if (in.out_mode == 1) {
      // Geometry_Par (CG3:4803-4838): the partition index of each cell, 1 for
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
  // init computes the saturation of the initial phase (CG3:2454); a restart
  // (Backup_init, CG3:5438-5690) leaves it at 0
  double S_l = 0, Sd_l = 0, Sd_g = 0;
  lbm_cg_diag d;
  if (in.mode_backup_ini == 0) {
    if (lbm_cg_reduce(h, &d) != LBM_OK) return die("lbm_cg_reduce");
    S_l = d.saturation;
  } else if (lbm_cg_read_checkpoint(h, pfix.c_str(), in.mode_backup_ini) != LBM_OK) {
    return die("lbm_cg_read_checkpoint");
  }
  std::cout << std::endl << "INITIALIZATION COMPLETED" << std::endl << std::endl;

  const std::string f_res = out + "Results.txt", f_rel1 = out + "Relative_Permeability_Component1.txt",
                    f_rel2 = out + "Relative_Permeability_Component2.txt", f_bf = out + "bodyforce.txt",
                    f_vel = out + "Velocity_ave_max.txt";
  { std::ofstream(f_res, std::ios::trunc); }
  { std::ofstream(out + "Capillary_Pressure.txt", std::ios::trunc); }
  { std::ofstream(out + "Imb_Drai_Rel_Perm.txt", std::ios::trunc); }
  if (in.wr_per == 1) { std::ofstream(f_rel1, std::ios::trunc); }
  { std::ofstream(f_bf, std::ios::out); }
  { std::ofstream(f_rel2, std::ios::out); }
  { std::ofstream(f_vel, std::ios::out); }

  double rk = in.reso * in.reso * 1000 / in.permeability;  // lattice permeability -> relative
  const double dt = 1.0, dx = 1.0;
  const int NY1 = ny;  // NY + 1
  const bool stab = in.stab == 1;
  Drive drv;
  drv.g[0] = stab ? 0.0 : in.gx;
  drv.g[1] = stab ? 0.0 : in.gy;
  drv.g[2] = stab ? 0.0 : in.gz;
  double p_n0[3] = {in.p_xn, in.p_yn, in.p_zn}, p_p0[3] = {in.p_xp, in.p_yp, in.p_zp};
  double gbase[3] = {in.gx, in.gy, in.gz};  // gx, gy, gz: moved by the capillary stepping
  const int len[3] = {nx, ny, nz};
  Capillary cap;
  if (in.pressure_change2 >= 1 && in.pressure_change2 <= 3) {
    // CG3:560-576
    cap.on = true;
    cap.a = in.pressure_change2 - 1;
    cap.pressure = in.pre_chan_pb2 == 1;
    if (cap.pressure) {
      cap.pre_in = (in.pre_chan_pns - p_n0[cap.a]) / (double)in.chan_no;
      cap.pre_ip = (in.pre_chan_pps - p_p0[cap.a]) / (double)in.chan_no;
    } else {
      cap.pre_in = (in.pre_chan_fs - gbase[cap.a]) / (double)in.chan_no;
    }
  }
  const std::string f_cap = out + "Capillary_Pressure.txt";
  for (int a = 0; a < 3; a++) {
    drv.p_n[a] = p_n0[a];
    drv.p_p[a] = p_p0[a];
  }
  double cap_a = in.cap_a;
  double Per_l[3] = {0, 0, 0}, Per_g[3] = {0, 0, 0};
  const double Per_l_local[3] = {0, 0, 0}, Per_g_local[3] = {0, 0, 0};  // never computed by the reference
  double error = 0, u_max = 0, u_ave = 0, pre_u_ave = 0, capillary = 0, error_per = 0, S_l_r = 0;
  double Re_l = 0, Re_g = 0;
  int the = 0, tme = 0, tse = 0, th = 0, tm = 0, ts = 0;
  int u_max_ref = 0;
  LeastSquares ls;
  ls.l.assign(in.num_least_square > 0 ? in.num_least_square : 0, 0.0);
  ls.g.assign(ls.l.size(), 0.0);
  // Comput_Perm's direction (CG3:5138-5147, 5229-5242) and the rate files'
  // (CG3:1009-1034): PerDir 2 -> y, 3 -> z, anything else -> x; the
  // least-squares call (CG3:938-946) takes z for anything but 1 and 2
  const int dir = in.perdir == 2 ? 1 : in.perdir == 3 ? 2 : 0;
  const int ls_dir = in.perdir == 1 ? 0 : in.perdir == 2 ? 1 : 2;
  int count = 0;
  double porosity = 0;
  lbm_cg_info(h, &count, &porosity, nullptr, nullptr);
  // Imbibition / drainage control (rel_perm_id_dir, CG3:615-621, 1121-1200,
  // 2467-2484): target saturations sw[i] = (i + 1) / (chan + 1) rising (1) or
  // (chan - i) / (chan + 1) falling (2); the first target is the first one the
  // initial saturation has not passed.  At a report, once the saturation
  // passes the target the phase field is written, and the next target
  // becomes the threshold of the random phase faces (ini_Sat).  The
  // reference reads past its target array once every target is passed; here
  // nothing more happens then.
  const int chan = in.rel_perm_id_dir > 0 ? in.rel_perm_chan_num : 0;
  std::vector<double> sw((size_t)std::max(chan, 0));
  for (int i = 0; i < chan; i++)
    sw[i] = in.rel_perm_id_dir == 1 ? (double)(i + 1) * (1.0 / (chan + 1)) : (double)(chan - i) * (1.0 / (chan + 1));
  // init sets the control up (CG3:2339-2345, 2467-2484); after a restart
  // (Backup_init) its state stays zero and it never acts
  int id_ids = 0, id_mode = in.mode_backup_ini == 0 ? 1 : 0;
  if (chan > 0 && id_mode == 1) {
    while (id_ids < chan && (in.rel_perm_id_dir == 1 ? S_l > sw[id_ids] : S_l < sw[id_ids])) id_ids++;
  }
  const int pf[6] = {in.psi_xp, in.psi_xn, in.psi_yp, in.psi_yn, in.psi_zp, in.psi_zn};
  std::vector<double> rho((size_t)count + 1);

  auto block = [&](std::ostream& o, long long nn) {
    o << "The" << nn << "th computation result:" << std::endl;
    o << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re_l=" << Re_l << "   Re_g=" << Re_g
      << std::endl;
    o << "Courant Number=" << u_max * dt / dx << "\t Capillary Num=" << capillary << std::endl;
    o << "The max relative error of velocity is: " << std::setiosflags(std::ios::scientific) << error << std::endl;
    o << "The relative permeability of component 1 is " << Per_l[0] * rk << ", " << Per_l[1] * rk << ", "
      << Per_l[2] * rk << std::endl;
    o << "The relative permeability of component 2 is " << Per_g[0] * rk << ", " << Per_g[1] * rk << ", "
      << Per_g[2] * rk << std::endl;
    o << "The LEAST SQUARED relative permeability of component 1 is " << ls.rel_l << std::endl;
    o << "The LEAST SQUARED relative permeability of component 2 is " << ls.rel_g << std::endl;
    o << "Satuation of Component 1: " << S_l << ", " << "The satuation of Component 2: " << 1 - S_l << std::endl;
    o << "The relative error of permiability computing is: " << error_per << std::endl;
    o << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    o << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
  };

  // face densities p_xp..p_zn as the ramps move them, and whether the face
  // rules run (from stab_time with the stabiliser, CG3:868)
  const double v_face[6] = {in.v_xp, in.v_xn, in.v_yp, in.v_yn, in.v_zp, in.v_zn};
  bool faces_on = !(stab && in.stab_time > 0);
  double rho_set[6] = {in.p_xp, in.p_xn, in.p_yp, in.p_yn, in.p_zp, in.p_zn};
  auto sync_faces = [&](bool force) {
    const double r[6] = {drv.p_p[0], drv.p_n[0], drv.p_p[1], drv.p_n[1], drv.p_p[2], drv.p_n[2]};
    bool same = !force;
    for (int f = 0; f < 6; f++) same = same && r[f] == rho_set[f];
    if (same) return true;
    for (int f = 0; f < 6; f++) rho_set[f] = r[f];
    return lbm_cg_set_faces(h, rho_set, v_face, faces_on ? 1 : 0) == LBM_OK;
  };

  // output_psi (CG3:5022-5114) with its title lines (CG3:5058-5059)
  auto write_psi = [&](long long step) {
    std::ostringstream v, t, tag;
    tag << step;
    v << " - " << in.nu_l << " " << in.nu_g << " " << in.contact_angle << " " << cap_a;
    t << "J.Yang Lattice Boltzmann Simulation 3D MC- " << S_l << " " << porosity << " " << in.reso << " "
      << drv.g[0] << " " << drv.p_p[0] << " " << drv.p_n[0];
    return lbm_cg_write_vtk_psi(h, (out + "LBM_psi_" + tag.str() + ".vtk").c_str(), v.str().c_str(),
                                t.str().c_str()) == LBM_OK;
  };
  long long n = 0;
  while (n <= in.n_max) {
    if (stab && n == in.stab_time) {
      // CG3:851-852, before this step's collision
      for (int k = 0; k < 3; k++) drv.g[k] = gbase[k];
      if (lbm_cg_set_body_force(h, drv.g[0], drv.g[1], drv.g[2], LBM_CG_FORCE_BEFORE_COLLISION) != LBM_OK)
        return die("lbm_cg_set_body_force");
      faces_on = true;
      if (!sync_faces(true)) return die("lbm_cg_set_faces");
    }
    // last step of this chunk: the next report, the step before the
    // stabiliser switch, or a ramp step (ramps run one step at a time)
    long long last = n;
    if (!ramp_at(in, n) && !cap.ramping(in, n)) {
      last = ((n + in.fre_re - 1) / in.fre_re) * in.fre_re;
      if (last > in.n_max) last = in.n_max;
      if (stab && in.stab_time > n && in.stab_time - 1 < last) last = in.stab_time - 1;
      if (in.input_dynamic > 0) last = std::min(last, ((n + in.update_fre - 1) / in.update_fre) * in.update_fre);
      for (long long k = n + 1; k <= last; k++)
        if (ramp_at(in, k) || cap.ramping(in, k)) {
          last = k - 1;
          break;
        }
    }
    if (lbm_cg_step(h, (int)(last - n + 1)) != LBM_OK) return die("lbm_cg_step");
    n = last;
    // pressure_bodyforce_change then pressure_capillary, between this step's
    // collision and its macro step (CG3:854-858)
    const bool moved = ramp(in, n, gbase, p_n0, p_p0, &drv);
    const bool moved2 = capillary_step(in, cap, n, S_l, S_l_r, gbase, p_n0, p_p0, &drv, f_cap, len);
    if ((moved || moved2) &&
        lbm_cg_set_body_force(h, drv.g[0], drv.g[1], drv.g[2], LBM_CG_FORCE_BEFORE_MACRO) != LBM_OK)
      return die("lbm_cg_set_body_force");
    if (in.input_dynamic > 0 && n % in.update_fre == 0) {
      // input_update (CG3:859-861, 5765-5925): the file read again; n_max,
      // the body force (gx = gxs), wall colour, CapA, permeability, report
      // and output intervals and the flux thresholds take its values
      lbm_cg_input up;
      if (lbm_read_cg_input(argv[1], &up) != LBM_OK) return die("lbm_read_cg_input (input update)");
      in.n_max = up.n_max;
      gbase[0] = drv.g[0] = in.gx = up.gx;
      gbase[1] = drv.g[1] = in.gy = up.gy;
      gbase[2] = drv.g[2] = in.gz = up.gz;
      in.contact_angle = up.contact_angle;
      cap_a = in.cap_a = up.cap_a;
      in.permeability = up.permeability;
      rk = in.reso * in.reso * 1000 / in.permeability;
      in.fre_re = up.fre_re;
      in.fre_ve = up.fre_ve;
      in.fre_de = up.fre_de;
      in.fre_psi = up.fre_psi;
      in.rel_perm_psi = up.rel_perm_psi;
      in.rel_perm_psi2 = up.rel_perm_psi2;
      if (lbm_cg_input_update(h, &in) != LBM_OK) return die("lbm_cg_input_update");
    }
    if (!sync_faces(false)) return die("lbm_cg_set_faces");
    if (n % in.fre_re != 0) {
      n++;
      continue;
    }
    if (in.rel_perm_ift > 0 && in.rel_perm_ift == n) {
      cap_a = in.vary_ift;
      if (lbm_cg_set_cap_a(h, cap_a) != LBM_OK) return die("lbm_cg_set_cap_a");
    }
    {
      std::ofstream fin(f_res, std::ios::out);
      Re_l = u_ave * NY1 / in.nu_l;
      Re_g = u_ave * NY1 / in.nu_g;
      block(fin, n - in.fre_re);
      fin << std::endl;
    }
    pre_u_ave = u_ave;
    if (lbm_cg_reduce(h, &d) != LBM_OK) return die("lbm_cg_reduce");
    // Error (CG3:4683-4750)
    error = d.u_rel_change;
    u_max = d.u_max;
    if (u_max >= 10.0) u_max_ref += 1;
    // Comput_Perm (CG3:5116-5284)
    error_per = (d.perm_l[dir] - Per_l[dir]) / Per_l[dir];
    for (int a = 0; a < 3; a++) {
      Per_l[a] = d.perm_l[a];
      Per_g[a] = d.perm_g[a];
    }
    capillary = d.capillary;
    u_ave = d.u_ave;
    // Comput_Saturation (CG3:5286-5400)
    S_l_r = S_l;
    S_l = d.saturation;
    Sd_l = d.sd_l;
    Sd_g = d.sd_g;
    if (in.least_square > 0) ls.push(Per_l[ls_dir] * rk, Per_g[ls_dir] * rk);
    // Rel_Perm_Imb_Dra (CG3:1121-1200), after the least-squares fit
    if (chan > 0 && id_mode > 0 && id_ids < chan) {
      if (id_mode == 1 && (in.rel_perm_id_dir == 1 ? S_l > sw[id_ids] : S_l < sw[id_ids])) id_mode = 2;
      if (id_mode == 2) {
        if (!write_psi(n)) return die("lbm_cg_write_vtk_psi");
        id_ids++;
        if (id_ids < chan) {
          id_mode = 1;
          if (lbm_cg_set_random(h, sw[id_ids], seed) != LBM_OK || lbm_cg_set_phase_faces(h, pf) != LBM_OK)
            return die("lbm_cg_set_phase_faces");
        }
      }
    }
    {
      const double finish = clock.now();
      hms(n > 0 ? (in.n_max - n) * (finish / n) : 0.0, &th, &tm, &ts);
      hms(finish, &the, &tme, &tse);
      std::ofstream fin(f_res, std::ios::app);
      Re_l = u_ave * NY1 / in.nu_l;
      Re_g = u_ave * NY1 / in.nu_g;
      block(fin, n);
      fin << std::endl;
    }
    if (in.wr_per == 1) {
      const double pn = drv.p_n[dir], pp = drv.p_p[dir], gs = drv.g[dir];
      {
        std::ofstream f1(f_rel1, std::ios::app);
        f1 << Per_l[dir] * rk << " " << S_l << " " << Per_l_local[dir] * rk << " " << 1 - S_l << " " << pn << " "
           << pp << " " << gs << " " << ls.rel_l << std::endl;
      }
      std::ofstream f2(f_rel2, std::ios::app);
      f2 << Per_g[dir] * rk << " " << 1 - S_l << " " << Per_g_local[dir] * rk << " " << S_l << " " << ls.rel_g << " "
         << ls.slope_l << " " << std::endl;
    }
    {
      std::ofstream(f_bf, std::ios::app) << S_l << " " << 1 - S_l << " " << std::abs((S_l_r - S_l) / (S_l + 1e-20))
                                         << " " << Sd_l << " " << Sd_g << std::endl;
    }
    {
      std::ofstream(f_vel, std::ios::app) << u_ave << " " << u_max << "  " << error << "  "
                                          << std::abs((pre_u_ave - u_ave) / (u_ave + 1e-20)) << std::endl;
    }
    if (lbm_cg_get_fields(h, rho.data(), nullptr, nullptr, nullptr, nullptr) != LBM_OK) return die("lbm_cg_get_fields");
    std::cout << "The" << n << "th computation result:" << std::endl;
    std::cout << "The Density of point(NX/2,NY/2,NZ/2) is: " << std::setprecision(6) << rho[count / 2] << std::endl;
    std::cout << "The Maximum velocity is: " << std::setprecision(6) << u_max << "   Re_l=" << Re_l
              << "   Re_g=" << Re_g << std::endl;
    std::cout << "Courant Number=" << u_max * dt / dx << "\t Capillary Num=" << capillary << std::endl;
    std::cout << "The max relative error of uv is: " << std::setiosflags(std::ios::scientific) << error << std::endl;
    std::cout << "The relative permeability of component 1 is " << Per_l[0] * rk << ", " << Per_l[1] * rk << ", "
              << Per_l[2] * rk << std::endl;
    std::cout << "The relative permeability of component 2 is " << Per_g[0] * rk << ", " << Per_g[1] * rk << ", "
              << Per_g[2] * rk << std::endl;
    std::cout << "The LEAST SQUARED relative permeability of component 1 is " << ls.rel_l << std::endl;
    std::cout << "The LEAST SQUARED relative permeability of component 2 is " << ls.rel_g << std::endl;
    std::cout << "Satuation of Component 1: " << S_l << ", " << "The satuation of Component 2: " << 1 - S_l
              << std::endl;
    std::cout << "The relative error of permiability computing is: " << error_per << std::endl;
    std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    std::cout << "The expected completion time is " << th << "h" << tm << "m" << ts << "s" << std::endl;
    std::cout << std::endl;  // like the reference, stdout stays in scientific notation from here on

    std::ostringstream tag;
    tag << n;
    if (in.fre_de > 0 && n % in.fre_de == 0 && n > 0 &&
        lbm_cg_write_vtk_density(h, (out + "LBM_Density_" + tag.str() + ".vtk").c_str()) != LBM_OK)
      return die("lbm_cg_write_vtk_density");
    if (in.fre_ve > 0 && n % in.fre_ve == 0 && n > 0 &&
        lbm_cg_write_vtk_velocity(h, (out + "LBM_velocity_Vector_" + tag.str() + ".vtk").c_str()) != LBM_OK)
      return die("lbm_cg_write_vtk_velocity");
    if (in.fre_psi >= 0 && n % in.fre_psi == 0 && !write_psi(n)) return die("lbm_cg_write_vtk_psi");
    if (in.fre_backup > 0 && n % in.fre_backup == 0 && n > 0 && lbm_cg_write_checkpoint(h, out.c_str(), n) != LBM_OK)
      return die("lbm_cg_write_checkpoint");
    if (u_max_ref >= 5) {
      std::cout << "PROGRAM STOP DUE TO HIGH VELOCITY" << std::endl;
      break;
    }
    n++;
  }
  if (in.fre_backup >= 0 && lbm_cg_write_checkpoint(h, out.c_str(), in.n_max) != LBM_OK)
    return die("lbm_cg_write_checkpoint");
  std::cout << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
  std::cout << "Accuracy: " << 1e-9 << " Second" << std::endl;
  {
    std::ofstream fin(f_res, std::ios::app);
    fin << "Elapsed time is " << the << "h" << tme << "m" << tse << "s" << std::endl;
    fin << "Accuracy: " << 1e-9 << " Second" << std::endl;
  }
  lbm_cg_destroy(h);
  return 0;
}
