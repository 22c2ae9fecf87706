// Host-visible structures and launchers of the colour-gradient kernels.
#pragma once

#include "lbm_internal.h"

namespace lbm {

struct CgParams {
  double psi_solid, cap_a;
  double g[3];   // body force of this step's collision (Guo forcing)
  double gm[3];  // body force of the macro step folded into this step's collide
                 // (u = (j + gm/2)/rho of the previous step; equals g except
                 // right after a force change that precedes a collision)
  int body_force_phase;
  double flux_psi;
  double u0[3];  // velocity of the initial state (inivx..z, CG3:2357-2362): rho = 1, u = u0
  // viscosity interpolation (CG3 init, delta = 0.1)
  double wl, wg, lg0, l1, l2, g1, g2, delta;
  // pressure/velocity faces: rules on at this step, face densities and
  // velocities (xp, xn, yp, yn, zp, zn)
  int faces;
  double face_rho[6];
  double face_u[6][3];
  // [npad] 1 = node in the zero-surface-tension layer of the mixture
  // injection (meq without the CapA |C| terms, CG3:2854-2867), or null
  const uint8_t* zero_sigma;
};

struct CgArgs {
  const void* f_src;  // [19][npad] post-collision f of the previous step
  void* f_dst;
  void* gr;           // [19][npad] recoloured red distributions (at their source node), FP64
  void* gb;
  void* rec;          // FP32: [2][npad] float4 per-node colour record (rho_r, rho_b, ux, uy | uz, unit colour gradient)
  const int32_t* table;
  const uint8_t* corder;  // [19][npad] colour summation order (FP64), or null
  int n, npad;
  void* psi;          // [npad] current phase field
  void* rho_r;
  void* rho_b;
  int given;          // first step after init: rho = 1, u = 0
  CgParams p;
  void* u_out;        // [3][npad] this step's pre-collision u, or null (Error's u0)
};

struct CgReduceArgs {
  const void* f;  // current post-collision f
  const int32_t* table;
  const void* psi;
  int n, npad;
  int given;
  double u0[3];  // u of the initial state
  double g[3];
  double flux_psi, flux_umax;
  double* rho_out;  // optional [npad] internal order
  double* u_out;    // optional [3][npad]
  double* partials;
  double* result;   // Ql(3), count(psi >= 0), Qg(3), mass
  // Error and the saturation position sums: null u_prev -> no change
  const void* u_prev;      // [3][npad]
  const int32_t* axis;     // [npad] coordinate along perdir, or null
  double* partials2;
  double* result2;         // |du|^2, |u|^2, |u|, max |u|^2, sd_l, sd_g, 0, 0
  const uint8_t* win;      // [npad] 1 = node inside the permeability window, or null (all)
};

// Pressure/velocity faces of the two-phase model: the record pass stores f,
// rho, u of the nodes the rules read ([23][nsnap] doubles); the face pass
// applies the rules to the face nodes' pulled populations in place.
struct CgBcArgs {
  void* f;                  // [19][npad] populations whose pulled state is acted on
  const int32_t* table;
  int npad;
  const int32_t* nodes;     // [nface] face nodes (internal index)
  const int32_t* op_off;    // [nface + 1]
  const BcOp* ops;
  int nface;
  const int32_t* snap_nodes;  // [nsnap] nodes the rules read
  double* rec;              // [23][nsnap]: f_0..f_18 (CG order), rho, ux, uy, uz
  int nsnap;
  int given;                // record pass: rho = 1, u = u0 (initial state)
  double u0[3];
  double gm[3];             // record pass: force of the macro step
  double face_rho[6];       // xp, xn, yp, yn, zp, zn
  double face_u[6][3];
};
cudaError_t cg_bc_record(bool f64, const CgBcArgs& a, cudaStream_t st);
cudaError_t cg_bc_faces(bool f64, const CgBcArgs& a, cudaStream_t st);

cudaError_t cg_set_mi_f64(const double* mi, cudaStream_t st);
cudaError_t cg_set_mi_f32(const double* mi, cudaStream_t st);
// whether the FP32 back-transform's build-time zero pattern fits this inverse
bool cg_block_pattern_matches(const double* mi);
cudaError_t cg_colour_f64(const CgArgs& a, cudaStream_t st);
cudaError_t cg_colour_f32(const CgArgs& a, cudaStream_t st);
cudaError_t cg_collide_f64(const CgArgs& a, cudaStream_t st);
cudaError_t cg_collide_f32(const CgArgs& a, cudaStream_t st);
cudaError_t cg_reduce_f64(const CgReduceArgs& a, int nblocks, cudaStream_t st);
cudaError_t cg_reduce_f32(const CgReduceArgs& a, int nblocks, cudaStream_t st);
bool build_cg_inverse(double MI[kQ][kQ]);
// f in the CG direction order, reference layout [(count+1)*19]
cudaError_t cg_export_f(bool f64, const void* f, const int32_t* table, const int32_t* ref_of, int n, int npad,
                        double* out, cudaStream_t st);
// Constant-phase faces: nodes[i] (internal index) takes psi0[i] after the
// colour pass, rho_r = (psi0 + 1)/2, rho_b = 1 - rho_r.
// out[i] = psi[src[i]] (src >= 0) or val[i]: the values of the face rules,
// read before any face node is written
cudaError_t cg_phase_faces_gather(bool f64, const int32_t* src, const double* val, int nface, const void* psi,
                                  double* out, cudaStream_t st);
cudaError_t cg_phase_faces(bool f64, const int32_t* nodes, const double* psi0, int nface, void* psi, void* rho_r,
                           void* rho_b, cudaStream_t st);
cudaError_t cg_import_f(bool f64, void* f, const int32_t* table, const int32_t* ref_of, int n, int npad,
                        const double* in, cudaStream_t st);

}  // namespace lbm
