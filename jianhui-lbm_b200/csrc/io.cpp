// INPUT.dat and geometry-file readers (the reference's L0/L1 formats).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "lbm_internal.h"

namespace lbm {

namespace {

// The reference reads each INPUT line as `fin >> values...; fin.getline(...)`:
// leading whitespace and newlines are skipped by operator>>, the rest of the
// line after the values is a comment.  Separator lines are consumed by a bare
// getline.
class LineReader {
 public:
  explicit LineReader(std::istream& in) : in_(in) {}
  template <typename... Ts>
  bool line(Ts&... vals) {
    bool ok = true;
    (void)std::initializer_list<int>{(ok = ok && static_cast<bool>(in_ >> vals), 0)...};
    skip();
    return ok;
  }
  bool word(char* buf, size_t cap) {
    std::string s;
    if (!(in_ >> s)) return false;
    std::strncpy(buf, s.c_str(), cap - 1);
    buf[cap - 1] = 0;
    skip();
    return true;
  }
  void skip() {
    in_.clear();
    in_.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  }

 private:
  std::istream& in_;
};

}  // namespace

// Field order of SP3:283-340 (identical in SP:255-308).
lbm_status read_input_file(const char* path, lbm_input* o) {
  if (!path || !o) return fail(LBM_ERR_ARG, "lbm_read_input: null argument");
  std::ifstream fin(path);
  if (!fin) return fail(LBM_ERR_IO, std::string("cannot open input file ") + path);
  std::memset(o, 0, sizeof(*o));
  LineReader r(fin);
  bool ok = true;
  r.skip();
  ok &= r.word(o->geometry_file, sizeof(o->geometry_file));
  ok &= r.line(o->nx, o->ny, o->nz);
  ok &= r.line(o->n_max);
  ok &= r.line(o->reso);
  ok &= r.line(o->in_bc);
  ok &= r.line(o->gx, o->gy, o->gz);
  ok &= r.line(o->pre_xp, o->p_xp, o->pre_xn, o->p_xn);
  ok &= r.line(o->pre_yp, o->p_yp, o->pre_yn, o->p_yn);
  ok &= r.line(o->pre_zp, o->p_zp, o->pre_zn, o->p_zn);
  ok &= r.line(o->vel_xp, o->v_xp, o->vel_xn, o->v_xn);
  ok &= r.line(o->vel_yp, o->v_yp, o->vel_yn, o->v_yn);
  ok &= r.line(o->vel_zp, o->v_zp, o->vel_zn, o->v_zn);
  ok &= r.line(o->in_vis);
  ok &= r.line(o->inivx, o->inivy, o->inivz);
  r.skip();
  ok &= r.line(o->wr_per);
  ok &= r.line(o->perdir);
  ok &= r.line(o->fre_re);
  ok &= r.line(o->out_mode);
  ok &= r.line(o->fre_ve);
  ok &= r.line(o->fre_de);
  r.skip();
  ok &= r.line(o->lattice_v, o->dx_input, o->dt_input);
  ok &= r.word(o->output_path, sizeof(o->output_path));
  ok &= r.line(o->sub_bc);
  ok &= r.line(o->loc_perm);
  ok &= r.line(o->par_per_x, o->par_per_y, o->par_per_z);
  ok &= r.line(o->per_xp, o->per_xn);
  ok &= r.line(o->per_yp, o->per_yn);
  ok &= r.line(o->per_zp, o->per_zn);
  r.skip();
  ok &= r.line(o->fre_backup);
  ok &= r.line(o->mode_backup_ini);
  ok &= r.line(o->vel_sol);
  r.skip();
  ok &= r.line(o->gperm);
  ok &= r.line(o->n_gperm[0], o->n_gperm[1], o->n_gperm[2], o->n_gperm[3]);
  ok &= r.line(o->size_gperm[0], o->size_gperm[1], o->size_gperm[2], o->size_gperm[3]);
  for (int i = 0; i < 4; i++) ok &= r.line(o->c_gperm[i][0], o->c_gperm[i][1], o->c_gperm[i][2]);
  r.skip();
  ok &= r.line(o->decbin);
  r.skip();
  ok &= r.line(o->nnf_module);
  ok &= r.line(o->nnf_m, o->nnf_n);
  if (!ok) return fail(LBM_ERR_FORMAT, std::string("malformed input file ") + path);
  if (o->nx <= 0 || o->ny <= 0 || o->nz <= 0)
    return fail(LBM_ERR_FORMAT, "input file: non-positive grid size");
  return LBM_OK;
}

// Field order of the colour-gradient program's INPUT file (CG3:372-474).
lbm_status read_cg_input_file(const char* path, lbm_cg_input* o) {
  if (!path || !o) return fail(LBM_ERR_ARG, "lbm_read_cg_input: null argument");
  std::ifstream fin(path);
  if (!fin) return fail(LBM_ERR_IO, std::string("cannot open input file ") + path);
  std::memset(o, 0, sizeof(*o));
  LineReader r(fin);
  bool ok = true;
  r.skip();
  ok &= r.word(o->geometry_file, sizeof(o->geometry_file));
  ok &= r.word(o->phase_file, sizeof(o->phase_file));
  ok &= r.line(o->nx, o->ny, o->nz);
  ok &= r.line(o->n_max);
  ok &= r.line(o->reso);
  ok &= r.line(o->in_bc);
  ok &= r.line(o->in_psi_bc);
  ok &= r.line(o->gx, o->gy, o->gz);
  ok &= r.line(o->pre_xp, o->p_xp, o->pre_xn, o->p_xn);
  ok &= r.line(o->pre_yp, o->p_yp, o->pre_yn, o->p_yn);
  ok &= r.line(o->pre_zp, o->p_zp, o->pre_zn, o->p_zn);
  ok &= r.line(o->vel_xp, o->v_xp, o->vel_xn, o->v_xn);
  ok &= r.line(o->vel_yp, o->v_yp, o->vel_yn, o->v_yn);
  ok &= r.line(o->vel_zp, o->v_zp, o->vel_zn, o->v_zn);
  ok &= r.line(o->psi_xp, o->psi_xn);
  ok &= r.line(o->psi_yp, o->psi_yn);
  ok &= r.line(o->psi_zp, o->psi_zn);
  ok &= r.line(o->nu_l);
  ok &= r.line(o->nu_g);
  ok &= r.line(o->contact_angle);
  ok &= r.line(o->cap_a);
  ok &= r.line(o->inivx, o->inivy, o->inivz);
  ok &= r.line(o->permeability);
  r.skip();
  ok &= r.line(o->wr_per);
  ok &= r.line(o->perdir);
  ok &= r.line(o->fre_re);
  ok &= r.line(o->out_mode);
  ok &= r.line(o->fre_ve);
  ok &= r.line(o->fre_de);
  ok &= r.line(o->fre_psi);
  r.skip();
  ok &= r.line(o->lattice_v, o->dx_input, o->dt_input);
  ok &= r.word(o->output_path, sizeof(o->output_path));
  ok &= r.line(o->sub_bc);
  ok &= r.line(o->stab, o->stab_time);
  ok &= r.line(o->ini_sat);
  ok &= r.line(o->ini_buf);
  ok &= r.line(o->rel_perm_psi, o->rel_perm_psi2);
  ok &= r.line(o->par_per_x, o->par_per_y, o->par_per_z);
  ok &= r.line(o->per_xp, o->per_xn);
  ok &= r.line(o->per_yp, o->per_yn);
  ok &= r.line(o->per_zp, o->per_zn);
  r.skip();
  ok &= r.line(o->fre_backup);
  ok &= r.line(o->mode_backup_ini);
  r.skip();
  ok &= r.line(o->decbin);
  r.skip();
  ok &= r.line(o->pressure_change, o->pre_chan_pb);
  for (int i = 0; i < 5; i++) ok &= r.line(o->pre_chan[i], o->pre_chan_pn[i], o->pre_chan_pp[i], o->pre_chan_f[i]);
  ok &= r.line(o->bodyforce_apply);
  r.skip();
  ok &= r.line(o->pressure_change2, o->pre_chan_pb2, o->interval_pre);
  ok &= r.line(o->pre_chan_pns, o->pre_chan_pps, o->pre_chan_fs, o->chan_no, o->sat_cri);
  ok &= r.line(o->sat_cri_d);
  r.skip();
  ok &= r.line(o->least_square, o->num_least_square);
  r.skip();
  ok &= r.line(o->rel_perm_id_dir, o->rel_perm_chan_num);
  ok &= r.line(o->rel_perm_ift, o->vary_ift);
  ok &= r.line(o->input_dynamic, o->update_fre);
  r.skip();
  ok &= r.line(o->mix_psi_thickness);
  ok &= r.line(o->protion_w);
  ok &= r.line(o->zero_sigma_thickness);
  if (!ok) return fail(LBM_ERR_FORMAT, std::string("malformed input file ") + path);
  if (o->nx <= 0 || o->ny <= 0 || o->nz <= 0)
    return fail(LBM_ERR_FORMAT, "input file: non-positive grid size");
  return LBM_OK;
}

// Field order of the solute program's INPUT file (ST7:219-280).
lbm_status read_st7_input_file(const char* path, lbm_st7_input* o) {
  if (!path || !o) return fail(LBM_ERR_ARG, "lbm_read_st7_input: null argument");
  std::ifstream fin(path);
  if (!fin) return fail(LBM_ERR_IO, std::string("cannot open input file ") + path);
  std::memset(o, 0, sizeof(*o));
  LineReader r(fin);
  bool ok = true;
  r.skip();
  ok &= r.word(o->geometry_file, sizeof(o->geometry_file));
  ok &= r.word(o->conc_file, sizeof(o->conc_file));
  ok &= r.line(o->nx, o->ny, o->nz);
  ok &= r.line(o->n_max);
  ok &= r.line(o->reso);
  ok &= r.line(o->in_bc);
  ok &= r.line(o->buoyancy, o->ref_psi);
  ok &= r.line(o->gravity);
  ok &= r.line(o->gx, o->gy, o->gz);
  ok &= r.line(o->pre_xp, o->p_xp, o->pre_xn, o->p_xn);
  ok &= r.line(o->pre_yp, o->p_yp, o->pre_yn, o->p_yn);
  ok &= r.line(o->pre_zp, o->p_zp, o->pre_zn, o->p_zn);
  ok &= r.line(o->vel_xp, o->v_xp, o->vel_xn, o->v_xn);
  ok &= r.line(o->vel_yp, o->v_yp, o->vel_yn, o->v_yn);
  ok &= r.line(o->vel_zp, o->v_zp, o->vel_zn, o->v_zn);
  ok &= r.line(o->sol_c_xp, o->c_xp, o->sol_c_xn, o->c_xn);
  ok &= r.line(o->sol_c_yp, o->c_yp, o->sol_c_yn, o->c_yn);
  ok &= r.line(o->sol_c_zp, o->c_zp, o->sol_c_zn, o->c_zn);
  ok &= r.line(o->sol_zf_xp, o->zf_xp, o->sol_zf_xn, o->zf_xn);
  ok &= r.line(o->sol_zf_yp, o->zf_yp, o->sol_zf_yn, o->zf_yn);
  ok &= r.line(o->sol_zf_zp, o->zf_zp, o->sol_zf_zn, o->zf_zn);
  ok &= r.line(o->nu);
  ok &= r.line(o->nu_s);
  ok &= r.line(o->inivx, o->inivy, o->inivz);
  r.skip();
  ok &= r.line(o->wr_per);
  ok &= r.line(o->perdir);
  ok &= r.line(o->fre_re);
  ok &= r.line(o->out_mode);
  ok &= r.line(o->fre_ve);
  ok &= r.line(o->fre_de);
  ok &= r.line(o->fre_psi);
  ok &= r.line(o->sub_dis, o->fre_dis);
  r.skip();
  ok &= r.line(o->lattice_v, o->dx_input, o->dt_input);
  ok &= r.word(o->output_path, sizeof(o->output_path));
  ok &= r.line(o->sub_bc);
  ok &= r.line(o->sub_bc_psi);
  ok &= r.line(o->ini_psi);
  ok &= r.line(o->par_per_x, o->par_per_y, o->par_per_z);
  ok &= r.line(o->per_xp, o->per_xn);
  ok &= r.line(o->per_yp, o->per_yn);
  ok &= r.line(o->per_zp, o->per_zn);
  r.skip();
  ok &= r.line(o->fre_backup);
  ok &= r.line(o->mode_backup_ini);
  ok &= r.line(o->sol_ini_n);
  r.skip();
  r.skip();
  ok &= r.line(o->decbin);
  if (!ok) return fail(LBM_ERR_FORMAT, std::string("malformed input file ") + path);
  if (o->nx <= 0 || o->ny <= 0 || o->nz <= 0)
    return fail(LBM_ERR_FORMAT, "input file: non-positive grid size");
  return LBM_OK;
}

// Phase file (CG3:2144-2150): nx*ny*nz numbers, k outer / j / i inner, each
// stored as float.
lbm_status read_phase_file(const char* path, int nx, int ny, int nz, double* out) {
  if (!path || !out || nx <= 0 || ny <= 0 || nz <= 0) return fail(LBM_ERR_ARG, "lbm_read_phase: bad argument");
  std::ifstream fin(path);
  if (!fin) return fail(LBM_ERR_IO, std::string("the concentration file (") + path + ") does not exist");
  const size_t cells = (size_t)nx * ny * nz;
  for (size_t c = 0; c < cells; c++) {
    float v;
    if (!(fin >> v))
      return fail(LBM_ERR_FORMAT, std::string("phase file ") + path + ": " + std::to_string(c) + " values, expected " +
                                      std::to_string(cells));
    out[c] = (double)v;
  }
  return LBM_OK;
}

// decbin 0: whitespace-separated integer tokens, k outer / j / i inner; any
// non-zero token is solid (SP3:929-943 reads into Solid, Partition_Solid
// SP3:3818-3819 treats Solid == 0 as pore).  decbin 1: raw int32 C-order
// [i][j][k] (SP3:947-961).
lbm_status read_mask_file(const char* path, int nx, int ny, int nz, int decbin, uint8_t* mask) {
  if (!path || !mask || nx <= 0 || ny <= 0 || nz <= 0) return fail(LBM_ERR_ARG, "lbm_read_mask: bad argument");
  const size_t cells = (size_t)nx * ny * nz;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(LBM_ERR_IO, std::string("the pore geometry file (") + path + ") does not exist");
  if (decbin == 0) {
    std::vector<char> buf(1 << 20);
    size_t c = 0;
    bool in_tok = false;
    long long val = 0;
    size_t got;
    while (c < cells && (got = std::fread(buf.data(), 1, buf.size(), fp)) > 0) {
      for (size_t i = 0; i < got && c < cells; i++) {
        const char ch = buf[i];
        if (ch >= '0' && ch <= '9') {
          val = val * 10 + (ch - '0');
          in_tok = true;
        } else if (ch == '-' && !in_tok) {
          // a sign is part of the token; negative values count as solid
        } else {
          if (in_tok) {  // token order is the mask's x-fastest memory order
            mask[c] = (val != 0) ? 1 : 0;
            c++;
          } else if (!(ch == ' ' || ch == '\n' || ch == '\r' || ch == '\t')) {
            std::fclose(fp);
            return fail(LBM_ERR_FORMAT, std::string("geometry file ") + path + ": unexpected character");
          }
          in_tok = false;
          val = 0;
        }
      }
    }
    if (in_tok && c < cells) {
      mask[c] = (val != 0) ? 1 : 0;
      c++;
    }
    std::fclose(fp);
    if (c < cells)
      return fail(LBM_ERR_FORMAT, std::string("geometry file ") + path + ": " + std::to_string(c) + " tokens, expected " +
                                      std::to_string(cells));
    return LBM_OK;
  }
  std::vector<int32_t> raw(cells);
  const size_t got = std::fread(raw.data(), sizeof(int32_t), cells, fp);
  std::fclose(fp);
  if (got != cells)
    return fail(LBM_ERR_FORMAT, std::string("geometry file ") + path + ": shorter than nx*ny*nz int32 values");
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++)
        mask[i + (size_t)nx * (j + (size_t)ny * k)] = raw[((size_t)i * ny + j) * nz + k] != 0 ? 1 : 0;
  return LBM_OK;
}

}  // namespace lbm
