// Reference file formats written from a solver's state: ASCII VTK structured
// points (SP3:3205-3468, CG3:4840-5114) and the per-rank raw checkpoints
// (SP3:3469-3516, 3652-3767; CG3:5438-5745).  Numbers are formatted by std::ostream with its default
// settings, as the reference's writers do.
#include <cstdio>
#include <iomanip>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "lbm_internal.h"

using namespace lbm;

namespace {

void vtk_header(std::ofstream& out, const char* title, int nx, int ny, int nz) {
  out << "# vtk DataFile Version 2.0" << std::endl;
  out << title << std::endl;
  out << "ASCII" << std::endl;
  out << "DATASET STRUCTURED_POINTS" << std::endl;
  out << "DIMENSIONS         " << nx << "         " << ny << "         " << nz << std::endl;
  out << "ORIGIN 0 0 0" << std::endl;
  out << "SPACING 1 1 1" << std::endl;
  out << "POINT_DATA     " << nx * ny * nz << std::endl;
}

lbm_status read_raw(const std::string& path, void* dst, size_t bytes) {
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) return fail(LBM_ERR_IO, "file open error on " + path);
  const size_t r = std::fread(dst, 1, bytes, fp);
  std::fclose(fp);
  if (r != bytes) return fail(LBM_ERR_FORMAT, path + ": shorter than the solver's state");
  return LBM_OK;
}

lbm_status write_raw(const std::string& path, const void* src, size_t bytes) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return fail(LBM_ERR_IO, "cannot write " + path);
  const size_t w = std::fwrite(src, 1, bytes, fp);
  std::fclose(fp);
  if (w != bytes) return fail(LBM_ERR_IO, "short write to " + path);
  return LBM_OK;
}

std::string ckpt_name(const char* prefix, const char* what, long long m) {
  std::ostringstream s;
  s << (prefix ? prefix : "") << "LBM_checkpoint_" << what << "_" << m << ".0.bin_input";
  return s.str();
}

// output_velocity (SP3:3286-3377, CG3:4840-4931): one "ux uy uz" line per
// cell, "0 0 0" on solids; u in reference id order (pore cells x fastest).
lbm_status vtk_velocity(const char* path, const uint8_t* mask, int nx, int ny, int nz, const double* u) {
  std::ofstream out(path);
  if (!out) return fail(LBM_ERR_IO, std::string("cannot write ") + path);
  vtk_header(out, "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Velocity", nx, ny, nz);
  out << "VECTORS sample_vectors double" << std::endl;
  out << std::endl;
  size_t id = 0;  // pore cells in x-fastest order are the reference ids 1..count
  const size_t cells = (size_t)nx * ny * nz;
  for (size_t c = 0; c < cells; c++) {
    if (mask[c] != 0) {
      out << 0 << " " << 0 << " " << 0 << std::endl;
    } else {
      ++id;
      out << u[id * 3 + 0] << " ";
      out << u[id * 3 + 1] << " ";
      out << u[id * 3 + 2] << std::endl;
    }
  }
  out.close();
  return out ? LBM_OK : fail(LBM_ERR_IO, std::string("write failed: ") + path);
}

// One scalar per cell on one line, `solid` on solid cells (output_density
// SP3:3379-3466 and CG3:4933-5020 with 1 on solids; output_psi CG3:5022-5114
// with 0 on solids and 2 significant digits from the first pore cell on).
lbm_status vtk_scalars(const char* path, const char* version_suffix, const char* title, const uint8_t* mask, int nx,
                       int ny, int nz, const double* v, double solid, int digits) {
  std::ofstream out(path);
  if (!out) return fail(LBM_ERR_IO, std::string("cannot write ") + path);
  out << "# vtk DataFile Version 2.0" << version_suffix << std::endl;
  out << title << std::endl;
  out << "ASCII" << std::endl;
  out << "DATASET STRUCTURED_POINTS" << std::endl;
  out << "DIMENSIONS         " << nx << "         " << ny << "         " << nz << std::endl;
  out << "ORIGIN 0 0 0" << std::endl;
  out << "SPACING 1 1 1" << std::endl;
  out << "POINT_DATA     " << nx * ny * nz << std::endl;
  out << "SCALARS sample_scalars float" << std::endl;
  out << "LOOKUP_TABLE default" << std::endl;
  size_t id = 0;
  const size_t cells = (size_t)nx * ny * nz;
  for (size_t c = 0; c < cells; c++) {
    if (mask[c] != 0) {
      out << solid << " ";
    } else {
      if (digits > 0) out << std::setprecision(digits);
      out << v[++id] << " ";
    }
  }
  out.close();
  return out ? LBM_OK : fail(LBM_ERR_IO, std::string("write failed: ") + path);
}

}  // namespace

extern "C" {

// Geometry (SP3:3205-3247): 0 for pore, 1 for solid, x fastest.
lbm_status lbm_write_vtk_geometry(const uint8_t* mask, int nx, int ny, int nz, const char* path) {
  if (!mask || !path) return fail(LBM_ERR_ARG, "lbm_write_vtk_geometry: null argument");
  std::ofstream out(path);
  if (!out) return fail(LBM_ERR_IO, std::string("cannot write ") + path);
  vtk_header(out, "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Solid-Geometry", nx, ny, nz);
  out << "SCALARS sample_scalars float" << std::endl;
  out << "LOOKUP_TABLE default" << std::endl;
  const size_t cells = (size_t)nx * ny * nz;
  for (size_t c = 0; c < cells; c++) out << (mask[c] == 0 ? 0 : 1) << " ";
  out.close();
  return out ? LBM_OK : fail(LBM_ERR_IO, std::string("write failed: ") + path);
}

lbm_status lbm_write_vtk_velocity(lbm_handle* h, const char* path) {
  if (!h || !path) return fail(LBM_ERR_ARG, "lbm_write_vtk_velocity: null argument");
  int count = 0, nx, ny, nz;
  double por;
  long long step;
  lbm_status st = lbm_info(h, &count, &por, &step);
  if (st != LBM_OK) return st;
  std::vector<double> u((size_t)(count + 1) * 3);
  if ((st = lbm_get_fields(h, nullptr, u.data())) != LBM_OK) return st;
  const uint8_t* mask = lbm_internal_mask(h, &nx, &ny, &nz);
  return vtk_velocity(path, mask, nx, ny, nz, u.data());
}

lbm_status lbm_write_vtk_density(lbm_handle* h, const char* path) {
  if (!h || !path) return fail(LBM_ERR_ARG, "lbm_write_vtk_density: null argument");
  int count = 0, nx, ny, nz;
  double por;
  long long step;
  lbm_status st = lbm_info(h, &count, &por, &step);
  if (st != LBM_OK) return st;
  std::vector<double> rho((size_t)(count + 1));
  if ((st = lbm_get_fields(h, rho.data(), nullptr)) != LBM_OK) return st;
  const uint8_t* mask = lbm_internal_mask(h, &nx, &ny, &nz);
  return vtk_scalars(path, "", "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Solid-Density", mask, nx, ny, nz,
                     rho.data(), 1.0, 0);
}

// Backup (SP3:3469-3516): raw doubles including the unused row 0.
lbm_status lbm_write_checkpoint(lbm_handle* h, const char* prefix, long long m) {
  if (!h) return fail(LBM_ERR_ARG, "lbm_write_checkpoint: null handle");
  int count = 0;
  double por;
  long long step;
  lbm_status st = lbm_info(h, &count, &por, &step);
  if (st != LBM_OK) return st;
  const size_t n1 = (size_t)count + 1;
  std::vector<double> rho(n1), u(n1 * 3), f(n1 * kQ);
  if ((st = lbm_get_fields(h, rho.data(), u.data())) != LBM_OK) return st;
  if ((st = lbm_get_populations(h, f.data())) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "velocity", m), u.data(), u.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "rho", m), rho.data(), rho.size() * sizeof(double))) != LBM_OK) return st;
  return write_raw(ckpt_name(prefix, "f", m), f.data(), f.size() * sizeof(double));
}

// Backup_init (SP3:3652-3767): restores rho, u, f; the next step uses them.
lbm_status lbm_read_checkpoint(lbm_handle* h, const char* prefix, long long m) {
  if (!h) return fail(LBM_ERR_ARG, "lbm_read_checkpoint: null handle");
  int count = 0;
  double por;
  long long step;
  lbm_status st = lbm_info(h, &count, &por, &step);
  if (st != LBM_OK) return st;
  const size_t n1 = (size_t)count + 1;
  std::vector<double> rho(n1), u(n1 * 3), f(n1 * kQ);
  if ((st = read_raw(ckpt_name(prefix, "rho", m), rho.data(), rho.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "velocity", m), u.data(), u.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "f", m), f.data(), f.size() * sizeof(double))) != LBM_OK) return st;
  return lbm_set_state(h, rho.data(), u.data(), f.data());
}

// Colour-gradient writers: the velocity / density VTK share the single-phase
// formats; the phase VTK takes its title lines from the caller.
lbm_status lbm_cg_write_vtk_velocity(lbm_cg_handle* h, const char* path) {
  if (!h || !path) return fail(LBM_ERR_ARG, "lbm_cg_write_vtk_velocity: null argument");
  int count = 0, nx, ny, nz;
  lbm_status st = lbm_cg_info(h, &count, nullptr, nullptr, nullptr);
  if (st != LBM_OK) return st;
  std::vector<double> u((size_t)(count + 1) * 3);
  if ((st = lbm_cg_get_fields(h, nullptr, u.data(), nullptr, nullptr, nullptr)) != LBM_OK) return st;
  const uint8_t* mask = lbm_cg_internal_mask(h, &nx, &ny, &nz);
  return vtk_velocity(path, mask, nx, ny, nz, u.data());
}

lbm_status lbm_cg_write_vtk_density(lbm_cg_handle* h, const char* path) {
  if (!h || !path) return fail(LBM_ERR_ARG, "lbm_cg_write_vtk_density: null argument");
  int count = 0, nx, ny, nz;
  lbm_status st = lbm_cg_info(h, &count, nullptr, nullptr, nullptr);
  if (st != LBM_OK) return st;
  std::vector<double> rho((size_t)(count + 1));
  if ((st = lbm_cg_get_fields(h, rho.data(), nullptr, nullptr, nullptr, nullptr)) != LBM_OK) return st;
  const uint8_t* mask = lbm_cg_internal_mask(h, &nx, &ny, &nz);
  return vtk_scalars(path, "", "J.Yang Lattice Boltzmann Simulation 3D Single Phase-Solid-Density", mask, nx, ny, nz,
                     rho.data(), 1.0, 0);
}

lbm_status lbm_cg_write_vtk_psi(lbm_cg_handle* h, const char* path, const char* version_suffix, const char* title) {
  if (!h || !path) return fail(LBM_ERR_ARG, "lbm_cg_write_vtk_psi: null argument");
  int count = 0, nx, ny, nz;
  lbm_status st = lbm_cg_info(h, &count, nullptr, nullptr, nullptr);
  if (st != LBM_OK) return st;
  std::vector<double> psi((size_t)(count + 1));
  if ((st = lbm_cg_get_fields(h, nullptr, nullptr, psi.data(), nullptr, nullptr)) != LBM_OK) return st;
  const uint8_t* mask = lbm_cg_internal_mask(h, &nx, &ny, &nz);
  return vtk_scalars(path, version_suffix ? version_suffix : "", title ? title : "", mask, nx, ny, nz, psi.data(), 0.0,
                     2);
}

// Backup (CG3:5693-5745): u, rho, psi, f, rho_r, rho_b as raw doubles with row 0.
lbm_status lbm_cg_write_checkpoint(lbm_cg_handle* h, const char* prefix, long long m) {
  if (!h) return fail(LBM_ERR_ARG, "lbm_cg_write_checkpoint: null handle");
  int count = 0;
  lbm_status st = lbm_cg_info(h, &count, nullptr, nullptr, nullptr);
  if (st != LBM_OK) return st;
  const size_t n1 = (size_t)count + 1;
  std::vector<double> rho(n1), u(n1 * 3), psi(n1), rr(n1), rb(n1), f(n1 * kQ);
  if ((st = lbm_cg_get_fields(h, rho.data(), u.data(), psi.data(), rr.data(), rb.data())) != LBM_OK) return st;
  if ((st = lbm_cg_get_populations(h, f.data())) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "velocity", m), u.data(), u.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "rho", m), rho.data(), rho.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "psi", m), psi.data(), psi.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "f", m), f.data(), f.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = write_raw(ckpt_name(prefix, "rhor", m), rr.data(), rr.size() * sizeof(double))) != LBM_OK) return st;
  return write_raw(ckpt_name(prefix, "rhob", m), rb.data(), rb.size() * sizeof(double));
}

// Backup_init (CG3:5438-5690): psi, rho_r, rho_b and f restored; rho and u
// follow from f at the next step.
lbm_status lbm_cg_read_checkpoint(lbm_cg_handle* h, const char* prefix, long long m) {
  if (!h) return fail(LBM_ERR_ARG, "lbm_cg_read_checkpoint: null handle");
  int count = 0;
  lbm_status st = lbm_cg_info(h, &count, nullptr, nullptr, nullptr);
  if (st != LBM_OK) return st;
  const size_t n1 = (size_t)count + 1;
  std::vector<double> rho(n1), u(n1 * 3), psi(n1), rr(n1), rb(n1), f(n1 * kQ);
  if ((st = read_raw(ckpt_name(prefix, "rho", m), rho.data(), rho.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "velocity", m), u.data(), u.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "psi", m), psi.data(), psi.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "f", m), f.data(), f.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "rhor", m), rr.data(), rr.size() * sizeof(double))) != LBM_OK) return st;
  if ((st = read_raw(ckpt_name(prefix, "rhob", m), rb.data(), rb.size() * sizeof(double))) != LBM_OK) return st;
  return lbm_cg_set_state(h, f.data(), psi.data(), rr.data(), rb.data());
}

}  // extern "C"
