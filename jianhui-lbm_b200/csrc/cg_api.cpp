// C ABI of the colour-gradient two-phase solver (lbm_cg_*).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cg_api.h"
#include "cg_basis.h"

namespace lbm {

lbm_status read_cg_input_file(const char* path, lbm_cg_input* o);
lbm_status read_phase_file(const char* path, int nx, int ny, int nz, double* out);
lbm_status read_mask_file(const char* path, int nx, int ny, int nz, int decbin, uint8_t* mask);

namespace {

struct Dev {
  void* p = nullptr;
  size_t bytes = 0;
  ~Dev() {
    if (p) lbm::dev_free(p);
  }
  cudaError_t alloc(size_t b) {
    if (p) lbm::dev_free(p);
    p = nullptr;
    bytes = b;
    return b ? lbm::dev_alloc(&p, b) : cudaSuccess;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

constexpr int kCgGraphSteps = 16;

// Draw k (0-based) of the seeded generator that stands in for the
// reference's clock-seeded rand(): the splitmix64 output (Steele, Lea and
// Flood 2014) of the state seed + (k + 1) * 0x9E3779B97F4A7C15, shifted right
// by 33 bits -- a non-negative 31-bit integer, as rand() returns.
unsigned long long cg_draw(unsigned long long seed, unsigned long long k) {
  unsigned long long z = seed + (k + 1) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return z >> 33;
}

}  // namespace
}  // namespace lbm

using namespace lbm;

struct lbm_cg_handle {
  lbm_cg_params prm{};
  bool f64 = true;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // with pressure/velocity faces: the face and record passes of a step run
  // on `side`, beside the colour pass (ev_fork: the step's start on the main
  // stream, ev_faces: rules applied, ev_rec: record written)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_faces = nullptr, ev_rec = nullptr;
  std::vector<uint8_t> mask;
  Geometry geo;
  double MI[kQ][kQ];
  CgParams cp{};
  Dev f[2], gr, gb, rec, table, corder, psi, rho_r, rho_b, ref_of, partials, result;
  Dev u_prev, axis, partials2, result2;  // Error's u0 and the saturation position sums
  Dev win;                                // permeability window flags, or none
  Dev face_nodes, face_psi0;              // phase-face nodes and their constant values
  Dev face_src, face_tmp;                 // copied-phase faces: source node per entry (-1: constant), values
  bool face_copy = false;                 // some face node copies another node's phase
  // psi / rho_r / rho_b already hold the pending macro step's colour pass
  // (a reader ran it); the next step uses them instead of running it again,
  // so that a phase-face change between steps acts from the next macro step
  // on, as the reference's settings change after comput_macro_variables
  bool colour_done = false;
  double rand_sat = -1.0;                 // ini_Sat: threshold of the random phase faces
  unsigned long long rand_seed = 0;       // seed of the random phase faces
  Dev zero_sigma;                         // zero-surface-tension layer flags, or none
  int nface = 0;
  std::vector<double> psi0;               // initial phase per node (internal order), as read
  long long window_volume = 0;            // divisor of the fluxes and the saturation
  bool uprev_valid = false;
  // pressure/velocity faces (bc_nface = 0: none).  The rules of a step are
  // applied to the state it leaves when that state is next used: by the
  // following step or by a reader (faces_pending), so that a face density
  // set between steps acts on the step just run, as the reference changes
  // p_* between collision and boundary_pressure.
  lbm_boundary bc{};
  Dev bc_nodes, bc_off, bc_ops, bc_snap, bc_rec;
  int bc_nface = 0, bc_nsnap = 0;
  bool faces_pending = false;
  int perdir = 1;
  int cur = 0;
  // 1: initial state (rho = 1, u = 0, psi / rho_r / rho_b given);
  // 2: restored state (psi / rho_r / rho_b given, rho and u from f);
  // 0: running (the colour pass recomputes psi / rho_r / rho_b)
  int given = 1;
  long long step = 0;
  double perm_prev = 0.0;
  double last_ms = 0.0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  CgParams graph_cp{};  // parameters the graphs were captured with
  ~lbm_cg_handle() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : {ev_fork, ev_faces, ev_rec})
      if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
  size_t s() const { return f64 ? 8 : 4; }
};

namespace {

CgArgs cg_args(lbm_cg_handle* h, int c, int given, bool write_u = false) {
  CgArgs a{};
  a.u_out = write_u ? h->u_prev.p : nullptr;
  a.f_src = h->f[c].p;
  a.f_dst = h->f[1 - c].p;
  a.gr = h->gr.p;
  a.gb = h->gb.p;
  a.rec = h->rec.p;
  a.table = h->table.as<int32_t>();
  a.corder = h->f64 ? h->corder.as<uint8_t>() : nullptr;
  a.n = h->geo.count;
  a.npad = h->geo.npad;
  a.psi = h->psi.p;
  a.rho_r = h->rho_r.p;
  a.rho_b = h->rho_b.p;
  a.given = given == 1;
  a.p = h->cp;
  return a;
}

// The colour pass (psi, rho_r, rho_b of the pending macro step) and the
// constant-phase faces that comput_macro_variables applies after it.
cudaError_t colour_pass(lbm_cg_handle* h, const CgArgs& a) {
  cudaError_t e = h->f64 ? cg_colour_f64(a, h->stream) : cg_colour_f32(a, h->stream);
  if (e == cudaSuccess && h->nface > 0) {
    const double* vals = h->face_psi0.as<double>();
    if (h->face_copy) {
      e = cg_phase_faces_gather(h->f64, h->face_src.as<int32_t>(), vals, h->nface, h->psi.p,
                                h->face_tmp.as<double>(), h->stream);
      vals = h->face_tmp.as<double>();
    }
    if (e == cudaSuccess)
      e = cg_phase_faces(h->f64, h->face_nodes.as<int32_t>(), vals, h->nface, h->psi.p, h->rho_r.p, h->rho_b.p,
                         h->stream);
  }
  return e;
}

CgBcArgs bc_args(lbm_cg_handle* h, int c) {
  CgBcArgs b{};
  b.f = h->f[c].p;
  b.table = h->table.as<int32_t>();
  b.npad = h->geo.npad;
  b.nodes = h->bc_nodes.as<int32_t>();
  b.op_off = h->bc_off.as<int32_t>();
  b.ops = h->bc_ops.as<BcOp>();
  b.nface = h->bc_nface;
  b.snap_nodes = h->bc_snap.as<int32_t>();
  b.rec = h->bc_rec.as<double>();
  b.nsnap = h->bc_nsnap;
  for (int d = 0; d < 3; d++) b.gm[d] = h->cp.gm[d];
  for (int f = 0; f < 6; f++) {
    b.face_rho[f] = h->cp.face_rho[f];
    for (int d = 0; d < 3; d++) b.face_u[f][d] = h->cp.face_u[f][d];
  }
  return b;
}

// The rules of the step that produced state c (pending), then the record of
// state c that this step's rules will read when they are on.  On the side
// stream: ev_faces marks the rules applied, ev_rec the record written.
cudaError_t face_passes(lbm_cg_handle* h, int c, int given, bool pending) {
  CgBcArgs b = bc_args(h, c);
  cudaError_t e = cudaSuccess;
  if (pending) e = cg_bc_faces(h->f64, b, h->side);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev_faces, h->side);
  if (e == cudaSuccess && h->cp.faces) {
    b.given = given == 1;
    for (int d = 0; d < 3; d++) b.u0[d] = h->cp.u0[d];
    e = cg_bc_record(h->f64, b, h->side);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->ev_rec, h->side);
  return e;
}

// Applies the pending rules to the current state before it is read.
cudaError_t resolve_faces(lbm_cg_handle* h) {
  if (!h->faces_pending) return cudaSuccess;
  h->faces_pending = false;
  return cg_bc_faces(h->f64, bc_args(h, h->cur), h->stream);
}

// One step.  With faces the step forks: the face pass (it writes only face
// nodes' slots of state c) and the record pass (it reads state c) run on the
// side stream while the colour pass (it reads the colour record and writes
// psi, rho_r, rho_b) runs on the main stream; the collide pass waits for the
// rules, and the step ends when the record is written too, so that the next
// step (or any other reader or writer of the state) starts after both.
cudaError_t one_cg_step(lbm_cg_handle* h, int c, int given, bool write_u, bool pending, bool colour_done = false) {
  const CgArgs a = cg_args(h, c, given, write_u);
  cudaError_t e = cudaSuccess;
  const bool faces = h->bc_nface > 0;
  if (faces) {
    e = cudaEventRecord(h->ev_fork, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
    if (e == cudaSuccess) e = face_passes(h, c, given, pending);
  }
  if (e == cudaSuccess && !given && !colour_done) e = colour_pass(h, a);
  if (e == cudaSuccess && faces) e = cudaStreamWaitEvent(h->stream, h->ev_faces, 0);
  if (e != cudaSuccess) return e;
  e = h->f64 ? cg_collide_f64(a, h->stream) : cg_collide_f32(a, h->stream);
  if (e == cudaSuccess && faces) e = cudaStreamWaitEvent(h->stream, h->ev_rec, 0);
  return e;
}

bool same_params(const CgParams& a, const CgParams& b) {
  bool same = a.psi_solid == b.psi_solid && a.cap_a == b.cap_a && a.body_force_phase == b.body_force_phase &&
              a.flux_psi == b.flux_psi && a.faces == b.faces && a.zero_sigma == b.zero_sigma;
  for (int d = 0; d < 3; d++) same = same && a.g[d] == b.g[d] && a.gm[d] == b.gm[d];
  for (int f = 0; f < 6; f++) {
    same = same && a.face_rho[f] == b.face_rho[f];
    for (int d = 0; d < 3; d++) same = same && a.face_u[f][d] == b.face_u[f][d];
  }
  return same;
}

void drop_graphs(lbm_cg_handle* h) {
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Chains of kCgGraphSteps running steps, captured with the steady parameters
// (gm = g); a parameter change drops them.  Every captured step applies the
// previous step's rules when the faces are on, so a chain starts from a
// state whose rules are pending exactly when the faces are on.
lbm_status cg_graph(lbm_cg_handle* h, int c0) {
  CgParams steady = h->cp;
  for (int d = 0; d < 3; d++) steady.gm[d] = steady.g[d];
  if (!same_params(steady, h->graph_cp)) drop_graphs(h);
  if (h->graph[c0]) return LBM_OK;
  h->graph_cp = steady;
  const CgParams saved = h->cp;
  h->cp = steady;
  cudaGraph_t g = nullptr;
  LBM_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  int c = c0;
  for (int s = 0; s < kCgGraphSteps && err == cudaSuccess; s++) {
    err = one_cg_step(h, c, 0, false, steady.faces != 0);
    c = 1 - c;
  }
  h->cp = saved;
  const cudaError_t end = cudaStreamEndCapture(h->stream, &g);
  if (err != cudaSuccess || end != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(LBM_ERR_CUDA, std::string("cg graph capture: ") + cudaGetErrorString(err ? err : end));
  }
  const cudaError_t ie = cudaGraphInstantiate(&h->graph[c0], g, 0);
  cudaGraphDestroy(g);
  LBM_CUDA_TRY(ie);
  return LBM_OK;
}

// Colour summation order of the reference's scatter (CG3:3507-3570): the
// contributions to rho_r(x) arrive in ascending source-node id, and for one
// source in ascending push direction (CG order).
void build_colour_order(const Geometry& g, std::vector<uint8_t>& order) {
  const int n = g.count, npad = g.npad;
  order.assign((size_t)kQ * npad, 0);
  for (int x = 0; x < n; x++) {
    long long key[kQ];
    int qs[kQ];
    for (int q = 0; q < kQ; q++) {
      int src_node, mi;
      if (q == 0) {
        src_node = x;
        mi = 0;
      } else {
        const int32_t s = g.src[(size_t)(q - 1) * npad + x];
        const int sq = s / npad, m = s % npad;
        if (sq == q) {
          src_node = m;
          mi = cg::of_row(q);
        } else {
          src_node = x;
          mi = cg::of_row(opp(q));
        }
      }
      key[q] = (long long)g.ref_of[src_node] * kQ + mi;
      qs[q] = q;
    }
    std::sort(qs, qs + kQ, [&](int a, int b) { return key[a] < key[b]; });
    for (int k = 0; k < kQ; k++) order[(size_t)k * npad + x] = (uint8_t)qs[k];
  }
}

lbm_status cg_check(lbm_cg_handle* h) {
  if (!h) return fail(LBM_ERR_ARG, "null cg handle");
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  return LBM_OK;
}

// Runs the colour pass (when the state is not the initial one) and the
// diagnostics reduction; optional macro fields in internal order.
lbm_status cg_reduce_raw(lbm_cg_handle* h, double r[8], double* rho_out, double* u_out, double* r2 = nullptr) {
  LBM_CUDA_TRY(resolve_faces(h));
  if (!h->given && !h->colour_done) {
    const CgArgs a = cg_args(h, h->cur, 0);
    LBM_CUDA_TRY(colour_pass(h, a));
    h->colour_done = true;
  }
  CgReduceArgs ra{};
  ra.f = h->f[h->cur].p;
  ra.table = h->table.as<int32_t>();
  ra.psi = h->psi.p;
  ra.n = h->geo.count;
  ra.npad = h->geo.npad;
  ra.given = h->given == 1;
  for (int d = 0; d < 3; d++) ra.u0[d] = h->cp.u0[d];
  for (int d = 0; d < 3; d++) ra.g[d] = h->cp.gm[d];  // the pending macro step's force
  ra.flux_psi = h->prm.flux_psi;
  ra.flux_umax = h->prm.flux_umax;
  ra.rho_out = rho_out;
  ra.u_out = u_out;
  ra.partials = h->partials.as<double>();
  ra.result = h->result.as<double>();
  ra.u_prev = (!h->given && h->uprev_valid) ? h->u_prev.p : nullptr;
  ra.axis = h->axis.as<int32_t>();
  ra.partials2 = h->partials2.as<double>();
  ra.result2 = h->result2.as<double>();
  ra.win = h->win.as<uint8_t>();
  const int nb = reduce_blocks(h->geo.count);
  LBM_CUDA_TRY(h->f64 ? cg_reduce_f64(ra, nb, h->stream) : cg_reduce_f32(ra, nb, h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(r, ra.result, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (r2) LBM_CUDA_TRY(cudaMemcpyAsync(r2, ra.result2, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

}  // namespace

extern "C" {

lbm_status lbm_cg_create(const lbm_cg_params* p, const uint8_t* mask, const double* psi_cells, int nx, int ny,
                         int nz, lbm_cg_handle** out) {
  return lbm_cg_create_bc(p, nullptr, mask, psi_cells, nx, ny, nz, out);
}

lbm_status lbm_cg_create_bc(const lbm_cg_params* p, const lbm_boundary* bc, const uint8_t* mask,
                            const double* psi_cells, int nx, int ny, int nz, lbm_cg_handle** out) {
  if (!p || !mask || !psi_cells || !out || nx <= 0 || ny <= 0 || nz <= 0)
    return fail(LBM_ERR_ARG, "lbm_cg_create: bad argument");
  if (bc) {
    for (int f = 0; f < 6; f++)
      if ((bc->pressure[f] != 0 && bc->pressure[f] != 1) || (bc->velocity[f] != 0 && bc->velocity[f] != 1))
        return fail(LBM_ERR_ARG, "lbm_cg_create: face flags must be 0 or 1");
    if (bc_active(*bc) && (bc->sub_bc < 0 || bc->sub_bc > 3))
      return fail(LBM_ERR_ARG, "lbm_cg_create: Sub_BC must be 0..3");
  }
  *out = nullptr;
  if (!(p->nu_l > 0) || !(p->nu_g > 0)) return fail(LBM_ERR_ARG, "lbm_cg_create: viscosities must be positive");
  if (p->precision != LBM_PREC_F64 && p->precision != LBM_PREC_F32)
    return fail(LBM_ERR_ARG, "lbm_cg_create: precision must be F64 or F32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
  auto h = std::make_unique<lbm_cg_handle>();
  h->prm = *p;
  h->f64 = p->precision == LBM_PREC_F64;
  h->device = p->device;
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  LBM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev0));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev1));
  const size_t cells = (size_t)nx * ny * nz;
  h->mask.assign(mask, mask + cells);
  Geometry& g = h->geo;
  compact_reference(mask, nx, ny, nz, &g);
  if (g.count == 0) return fail(LBM_ERR_ARG, "geometry has no pore cells");
  order_nodes(mask, LBM_ORDER_REFERENCE, &g);
  // with pressure/velocity faces: the nodes a rule reads, then the nodes a
  // rule writes, after all others (each class in reference order), so that
  // the face passes' threads take consecutive nodes.  The reference's order
  // runs x fastest, which puts the nodes of an x face about a row of x
  // apart: there each of the passes' loads was a DRAM access of its own
  // (56 MB read per pass for 19 K face nodes on 128^3).
  if (bc) {
    BcPlan plan;
    bc_partition(mask, *bc, &g, &plan);
  }
  build_pull_table(mask, &g);
  if (!build_cg_inverse(h->MI)) return fail(LBM_ERR_ARG, "colour-gradient basis inversion failed");

  // constants of init (CG3:2226-2260)
  CgParams& cp = h->cp;
  if (bc) {
    h->bc = *bc;
    cp.faces = 1;
    for (int f = 0; f < 6; f++) {
      cp.face_rho[f] = bc->rho[f];
      cp.face_u[f][f / 2] = bc->vel[f];
    }
  }
  cp.psi_solid = p->psi_solid;
  cp.cap_a = p->cap_a;
  cp.g[0] = cp.gm[0] = p->gx;
  cp.g[1] = cp.gm[1] = p->gy;
  cp.g[2] = cp.gm[2] = p->gz;
  h->window_volume = (long long)nx * ny * nz;
  cp.body_force_phase = p->body_force_phase;
  cp.flux_psi = p->flux_psi;
  const double c_s2 = 1.0 * 1.0 / 3, dt = 1.0;
  cp.delta = 0.1;
  cp.wl = 1.0 / (p->nu_l / (c_s2 * dt) + 0.5);
  cp.wg = 1.0 / (p->nu_g / (c_s2 * dt) + 0.5);
  cp.lg0 = 2 * cp.wl * cp.wg / (cp.wl + cp.wg);
  cp.l1 = 2 * (cp.wl - cp.lg0) / cp.delta;
  cp.l2 = -cp.l1 / (2 * cp.delta);
  cp.g1 = 2 * (cp.lg0 - cp.wg) / cp.delta;
  cp.g2 = cp.g1 / (2 * cp.delta);

  const int n = g.count, npad = g.npad;
  const size_t s = h->s();
  for (auto& b : h->f) LBM_CUDA_TRY(b.alloc((size_t)kQ * npad * s));
  if (h->f64) {
    LBM_CUDA_TRY(h->gr.alloc((size_t)kQ * npad * s));
    LBM_CUDA_TRY(h->gb.alloc((size_t)kQ * npad * s));
  } else {
    LBM_CUDA_TRY(h->rec.alloc((size_t)8 * npad * sizeof(float)));
  }
  LBM_CUDA_TRY(h->table.alloc((size_t)18 * npad * sizeof(int32_t)));
  LBM_CUDA_TRY(h->psi.alloc((size_t)npad * s));
  LBM_CUDA_TRY(h->rho_r.alloc((size_t)npad * s));
  LBM_CUDA_TRY(h->rho_b.alloc((size_t)npad * s));
  LBM_CUDA_TRY(h->ref_of.alloc((size_t)n * sizeof(int32_t)));
  LBM_CUDA_TRY(h->partials.alloc((size_t)reduce_blocks(n) * 8 * sizeof(double)));
  LBM_CUDA_TRY(h->result.alloc(8 * sizeof(double)));
  LBM_CUDA_TRY(h->partials2.alloc((size_t)reduce_blocks(n) * 8 * sizeof(double)));
  LBM_CUDA_TRY(h->result2.alloc(8 * sizeof(double)));
  LBM_CUDA_TRY(h->u_prev.alloc((size_t)3 * npad * s));
  {
    // coordinate of every node along perdir, for the saturation position sums
    h->perdir = (p->perdir >= 1 && p->perdir <= 3) ? p->perdir : 1;
    std::vector<int32_t> ax(npad, 0);
    for (int x = 0; x < n; x++) {
      const int c = g.coor[g.ref_of[x]];  // i*ny*nz + j*nz + k
      const int i = c / (ny * nz), j = (c % (ny * nz)) / nz, k = c % nz;
      ax[x] = h->perdir == 1 ? i : (h->perdir == 2 ? j : k);
    }
    LBM_CUDA_TRY(h->axis.alloc((size_t)npad * sizeof(int32_t)));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->axis.p, ax.data(), sizeof(int32_t) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  LBM_CUDA_TRY(cudaMemcpyAsync(h->table.p, g.src.data(), sizeof(int32_t) * 18 * (size_t)npad,
                               cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->ref_of.p, g.ref_of.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                               h->stream));
  std::vector<uint8_t> order;
  // the FP64 inverse also serves the Sub_BC 2 pressure rule of both precisions
  LBM_CUDA_TRY(cg_set_mi_f64(&h->MI[0][0], h->stream));
  if (h->f64) {
    build_colour_order(g, order);
    LBM_CUDA_TRY(h->corder.alloc(order.size()));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->corder.p, order.data(), order.size(), cudaMemcpyHostToDevice, h->stream));
  } else {
    if (!cg_block_pattern_matches(&h->MI[0][0]))
      return fail(LBM_ERR_STATE, "colour-gradient M^-1 does not have the pattern the FP32 kernel was built for; "
                                 "rebuild the library");
    LBM_CUDA_TRY(cg_set_mi_f32(&h->MI[0][0], h->stream));
  }
  BcLists bl;
  if (bc) bc_node_lists(*bc, g, &bl);
  if (!bl.nodes.empty()) {
    h->bc_nface = (int)bl.nodes.size();
    h->bc_nsnap = (int)bl.snap_nodes.size();
    LBM_CUDA_TRY(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    for (cudaEvent_t* ev : {&h->ev_fork, &h->ev_faces, &h->ev_rec})
      LBM_CUDA_TRY(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    LBM_CUDA_TRY(h->bc_nodes.alloc(bl.nodes.size() * sizeof(int32_t)));
    LBM_CUDA_TRY(h->bc_off.alloc(bl.op_off.size() * sizeof(int32_t)));
    LBM_CUDA_TRY(h->bc_ops.alloc(bl.ops.size() * sizeof(BcOp)));
    LBM_CUDA_TRY(h->bc_snap.alloc(std::max<size_t>(bl.snap_nodes.size(), 1) * sizeof(int32_t)));
    LBM_CUDA_TRY(h->bc_rec.alloc((size_t)(kQ + 4) * std::max(h->bc_nsnap, 1) * sizeof(double)));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_nodes.p, bl.nodes.data(), bl.nodes.size() * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_off.p, bl.op_off.data(), bl.op_off.size() * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_ops.p, bl.ops.data(), bl.ops.size() * sizeof(BcOp), cudaMemcpyHostToDevice,
                                 h->stream));
    if (!bl.snap_nodes.empty())
      LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_snap.p, bl.snap_nodes.data(), bl.snap_nodes.size() * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemsetAsync(h->bc_rec.p, 0, h->bc_rec.bytes, h->stream));
  }
  // init (CG3:2360-2380): f = feq(1, 0) = first column of M^-1 in CG order,
  // psi from the phase file as float, rho_r = (psi + 1)/2, rho_b = 1 - rho_r
  double f0[kQ];
  for (int q = 0; q < kQ; q++) f0[q] = h->MI[cg::of_row(q)][0];
  LBM_CUDA_TRY(launch_init_uniform(h->f64 ? Store::F64 : Store::F32, h->f[0].p, h->table.as<int32_t>(), n, npad, 1.0,
                                   f0, h->stream));
  std::vector<double> ps(npad, 0.0), rr(npad, 0.0), rb(npad, 0.0);
  for (int x = 0; x < n; x++) {
    const int c = g.coor[g.ref_of[x]];  // i*ny*nz + j*nz + k
    const int i = c / (ny * nz), j = (c % (ny * nz)) / nz, k = c % nz;
    const double v = (double)(float)psi_cells[i + (size_t)nx * (j + (size_t)ny * k)];
    const double rho = 1.0;
    ps[x] = v;
    rr[x] = (v * rho + rho) / 2;
    rb[x] = rho - rr[x];
  }
  h->psi0.assign(ps.begin(), ps.begin() + n);
  if (h->f64) {
    LBM_CUDA_TRY(cudaMemcpyAsync(h->psi.p, ps.data(), sizeof(double) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->rho_r.p, rr.data(), sizeof(double) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->rho_b.p, rb.data(), sizeof(double) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<float> a(ps.begin(), ps.end()), b(rr.begin(), rr.end()), c(rb.begin(), rb.end());
    LBM_CUDA_TRY(cudaMemcpyAsync(h->psi.p, a.data(), sizeof(float) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->rho_r.p, b.data(), sizeof(float) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->rho_b.p, c.data(), sizeof(float) * npad, cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  if (h->gr.p) LBM_CUDA_TRY(cudaMemsetAsync(h->gr.p, 0, h->gr.bytes, h->stream));
  if (h->gb.p) LBM_CUDA_TRY(cudaMemsetAsync(h->gb.p, 0, h->gb.bytes, h->stream));
  if (h->rec.p) LBM_CUDA_TRY(cudaMemsetAsync(h->rec.p, 0, h->rec.bytes, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = h.release();
  return LBM_OK;
}

lbm_status lbm_cg_step(lbm_cg_handle* h, int nsteps) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (nsteps < 0) return fail(LBM_ERR_ARG, "lbm_cg_step: negative step count");
  if (nsteps == 0) return LBM_OK;
  int left = nsteps;
  // the first step runs alone after init or restore, when a reader already
  // ran the pending macro step's colour pass, and when a force change falls
  // between the pending macro step and the next collision
  bool special = h->given != 0 || h->colour_done;
  for (int d = 0; d < 3; d++) special = special || h->cp.gm[d] != h->cp.g[d];
  // ... and when the state's pending rules differ from what a chain assumes
  const bool faces_on = h->bc_nface > 0 && h->cp.faces;
  special = special || (h->bc_nface > 0 && h->faces_pending != faces_on);
  if (left - (special ? 1 : 0) - 1 >= kCgGraphSteps) {
    const int c0 = h->cur;
    for (int c = 0; c < 2; c++)
      if ((st = cg_graph(h, c)) != LBM_OK) return st;
    h->cur = c0;
  }
  LBM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  if (special) {
    LBM_CUDA_TRY(one_cg_step(h, h->cur, h->given, left == 1, h->faces_pending, h->colour_done));
    h->cur = 1 - h->cur;
    h->given = 0;
    for (int d = 0; d < 3; d++) h->cp.gm[d] = h->cp.g[d];
    left--;
  }
  while (left - 1 >= kCgGraphSteps) {
    LBM_CUDA_TRY(cudaGraphLaunch(h->graph[h->cur], h->stream));
    left -= kCgGraphSteps;  // even chain: parity unchanged
  }
  // the last step also writes its pre-collision u (Error's u0 of the next report)
  while (left > 0) {
    LBM_CUDA_TRY(one_cg_step(h, h->cur, 0, left == 1, faces_on));
    h->cur = 1 - h->cur;
    left--;
  }
  h->faces_pending = faces_on;
  h->uprev_valid = true;
  h->colour_done = false;
  LBM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  LBM_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0;
  LBM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_ms = ms;
  h->step += nsteps;
  return LBM_OK;
}

lbm_status lbm_cg_reduce(lbm_cg_handle* h, lbm_cg_diag* out) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!out) return fail(LBM_ERR_ARG, "lbm_cg_reduce: null output");
  double r[8], r2[8];
  if ((st = cg_reduce_raw(h, r, nullptr, nullptr, r2)) != LBM_OK) return st;
  const Geometry& g = h->geo;
  // fluxes and saturation over the window volume, Error over the box; the
  // porosity is the window's pore fraction (CG3:1851, 5217-5227, 5361)
  const double V = (double)g.nx * g.ny * g.nz, Vw = (double)h->window_volume, phi = g.porosity;
  // pressure-gradient term (CG3:5137-5149): |p_+ - p_-| c_s^2 / (N + 1) / dx
  // along PerDir (x for anything but 2 and 3), when in_BC is set
  double dp = 0.0;
  if (h->bc.in_bc != 0) {
    const int a = h->prm.perdir == 2 ? 1 : h->prm.perdir == 3 ? 2 : 0;
    const int ext[3] = {g.nx, g.ny, g.nz};
    const double c_s2 = 1.0 * 1.0 / 3, dx = 1.0;
    dp = std::fabs(h->cp.face_rho[2 * a] - h->cp.face_rho[2 * a + 1]) * c_s2 / ext[a] / dx;
  }
  const double* gg = h->cp.gm;  // gxs when the macro step ran
  std::memset(out, 0, sizeof(*out));
  out->step = h->step;
  for (int d = 0; d < 3; d++) {
    out->q_l[d] = r[d];
    out->q_g[d] = r[4 + d];
    out->perm_l[d] = r[d] / Vw * h->prm.nu_l / (gg[d] + dp);      // CG3:5217-5222
    out->perm_g[d] = r[4 + d] / Vw * h->prm.nu_g / (gg[d] + dp);
  }
  const double vx = (r[0] + r[4]) / Vw, vy = (r[1] + r[5]) / Vw, vz = (r[2] + r[6]) / Vw;
  out->u_ave = std::sqrt((vx / phi) * (vx / phi) + (vy / phi) * (vy / phi) + (vz / phi) * (vz / phi));
  out->capillary = std::sqrt(vx * vx + vy * vy + vz * vz) / phi * h->prm.nu_l / h->cp.cap_a;
  out->saturation = r[3] / (Vw * phi);  // CG3:5361
  out->mass = r[7];
  const int dir = h->perdir - 1;
  out->perm_rel_change = (out->perm_l[dir] - h->perm_prev) / h->perm_prev;  // CG3:5235-5246
  h->perm_prev = out->perm_l[dir];
  out->u_max = std::sqrt(r2[3]);                                         // CG3:4709-4745
  out->u_rel_change = std::sqrt(r2[0]) / (std::sqrt(r2[1]) + 1e-30);
  out->u_mean_speed = r2[2] / V;
  out->sd_l = r2[4];
  out->sd_g = r2[5];
  return LBM_OK;
}

lbm_status lbm_cg_get_fields(lbm_cg_handle* h, double* rho, double* u, double* psi, double* rho_r, double* rho_b) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  const int n = h->geo.count, npad = h->geo.npad;
  Dev rint, uint_, rref, uref;
  LBM_CUDA_TRY(rint.alloc((size_t)npad * sizeof(double)));
  LBM_CUDA_TRY(uint_.alloc((size_t)3 * npad * sizeof(double)));
  LBM_CUDA_TRY(rref.alloc((size_t)(n + 1) * sizeof(double)));
  LBM_CUDA_TRY(uref.alloc((size_t)(n + 1) * 3 * sizeof(double)));
  double r[8];
  if ((st = cg_reduce_raw(h, r, rint.as<double>(), uint_.as<double>())) != LBM_OK) return st;
  LBM_CUDA_TRY(cudaMemsetAsync(rref.p, 0, rref.bytes, h->stream));
  LBM_CUDA_TRY(cudaMemsetAsync(uref.p, 0, uref.bytes, h->stream));
  LBM_CUDA_TRY(launch_export_macro(rint.as<double>(), uint_.as<double>(), h->ref_of.as<int32_t>(), n, npad,
                                   rref.as<double>(), uref.as<double>(), h->stream));
  if (rho) LBM_CUDA_TRY(cudaMemcpyAsync(rho, rref.p, rref.bytes, cudaMemcpyDeviceToHost, h->stream));
  if (u) LBM_CUDA_TRY(cudaMemcpyAsync(u, uref.p, uref.bytes, cudaMemcpyDeviceToHost, h->stream));
  // scalar fields: internal order equals reference order - 1 for this solver
  std::vector<double> tmp(npad);
  std::vector<float> tmpf(npad);
  double* outs[3] = {psi, rho_r, rho_b};
  Dev* srcs[3] = {&h->psi, &h->rho_r, &h->rho_b};
  for (int i = 0; i < 3; i++) {
    if (!outs[i]) continue;
    if (h->f64) {
      LBM_CUDA_TRY(cudaMemcpyAsync(tmp.data(), srcs[i]->p, sizeof(double) * npad, cudaMemcpyDeviceToHost, h->stream));
      LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    } else {
      LBM_CUDA_TRY(cudaMemcpyAsync(tmpf.data(), srcs[i]->p, sizeof(float) * npad, cudaMemcpyDeviceToHost, h->stream));
      LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
      for (int x = 0; x < npad; x++) tmp[x] = tmpf[x];
    }
    outs[i][0] = 0.0;
    for (int x = 0; x < n; x++) outs[i][h->geo.ref_of[x]] = tmp[x];
  }
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status lbm_cg_get_populations(lbm_cg_handle* h, double* f) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!f) return fail(LBM_ERR_ARG, "lbm_cg_get_populations: null output");
  LBM_CUDA_TRY(resolve_faces(h));
  const int n = h->geo.count;
  Dev o;
  LBM_CUDA_TRY(o.alloc((size_t)(n + 1) * kQ * sizeof(double)));
  LBM_CUDA_TRY(cudaMemsetAsync(o.p, 0, o.bytes, h->stream));
  LBM_CUDA_TRY(cg_export_f(h->f64, h->f[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n, h->geo.npad,
                           o.as<double>(), h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(f, o.p, o.bytes, cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status lbm_cg_set_body_force(lbm_cg_handle* h, double gx, double gy, double gz, int timing) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (timing != LBM_CG_FORCE_BEFORE_MACRO && timing != LBM_CG_FORCE_BEFORE_COLLISION)
    return fail(LBM_ERR_ARG, "lbm_cg_set_body_force: unknown timing");
  const double g[3] = {gx, gy, gz};
  for (int d = 0; d < 3; d++) {
    h->cp.g[d] = g[d];
    if (timing == LBM_CG_FORCE_BEFORE_MACRO) h->cp.gm[d] = g[d];
  }
  h->prm.gx = gx;
  h->prm.gy = gy;
  h->prm.gz = gz;
  return LBM_OK;
}

lbm_status lbm_cg_set_faces(lbm_cg_handle* h, const double rho[6], const double vel[6], int active) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!rho || !vel) return fail(LBM_ERR_ARG, "lbm_cg_set_faces: null argument");
  for (int f = 0; f < 6; f++) {
    h->cp.face_rho[f] = rho[f];
    h->bc.rho[f] = rho[f];
    h->bc.vel[f] = vel[f];
    for (int d = 0; d < 3; d++) h->cp.face_u[f][d] = d == f / 2 ? vel[f] : 0.0;
  }
  h->cp.faces = active != 0;
  return LBM_OK;
}

lbm_status lbm_cg_set_cap_a(lbm_cg_handle* h, double cap_a) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  h->cp.cap_a = cap_a;
  h->prm.cap_a = cap_a;
  return LBM_OK;
}

// feq of the colour-gradient program on the host (CG3:2503-2540), the same
// operations as cg_feq in cg_faithful.cu: row k of M^-1 applied to the
// equilibrium moments, summed from j = 0.
static double cg_feq_host(const double (&mi)[kQ][kQ], int k, double rho, double ux, double uy, double uz) {
  const double rho_0 = 1.0;
  double meq[kQ] = {};
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
  double feq = 0.0;
  for (int j = 0; j < kQ; j++) feq = feq + mi[k][j] * meq[j];
  return feq;
}

lbm_status lbm_cg_set_initial_velocity(lbm_cg_handle* h, double ux, double uy, double uz) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (h->given != 1) return fail(LBM_ERR_STATE, "lbm_cg_set_initial_velocity: only before the first step");
  // init (CG3:2357-2400): u = (inivx, inivy, inivz) and f = feq(1, u) at
  // every node; the first collision takes rho = 1, u = u0
  double f0[kQ];
  for (int q = 0; q < kQ; q++) f0[q] = cg_feq_host(h->MI, cg::of_row(q), 1.0, ux, uy, uz);
  LBM_CUDA_TRY(launch_init_uniform(h->f64 ? Store::F64 : Store::F32, h->f[h->cur].p, h->table.as<int32_t>(),
                                   h->geo.count, h->geo.npad, 1.0, f0, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->cp.u0[0] = ux;
  h->cp.u0[1] = uy;
  h->cp.u0[2] = uz;
  drop_graphs(h);
  return LBM_OK;
}

lbm_status lbm_cg_input_update(lbm_cg_handle* h, const lbm_cg_input* in) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!in) return fail(LBM_ERR_ARG, "lbm_cg_input_update: null input");
  // input_update (CG3:5765-5925): the wall colour, CapA and the flux
  // thresholds from the next collision on; gxs = gx already for this step's
  // macro step, like a ramp
  h->cp.psi_solid = h->prm.psi_solid = in->contact_angle;
  h->cp.cap_a = h->prm.cap_a = in->cap_a;
  h->cp.flux_psi = h->prm.flux_psi = in->rel_perm_psi;
  h->prm.flux_umax = in->rel_perm_psi2;
  return lbm_cg_set_body_force(h, in->gx, in->gy, in->gz, LBM_CG_FORCE_BEFORE_MACRO);
}

lbm_status lbm_cg_set_window(lbm_cg_handle* h, const int window[6], int restrict_nodes) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!window) return fail(LBM_ERR_ARG, "lbm_cg_set_window: null window");
  Geometry& g = h->geo;
  bool whole = true;
  for (int i = 0; i < 6; i++) whole = whole && window[i] < 0;
  if (whole) {
    h->window_volume = (long long)g.nx * g.ny * g.nz;
    g.porosity = (double)g.count / (double)h->window_volume;
    h->win.alloc(0);
    return LBM_OK;
  }
  h->window_volume = (long long)(window[1] - window[0] + 1) * (window[3] - window[2] + 1) * (window[5] - window[4] + 1);
  // the porosity becomes the window's pore fraction (CG3:1835-1851)
  std::vector<uint8_t> in((size_t)g.npad, 0);
  long long pores = 0;
  for (int x = 0; x < g.count; x++) {
    const int c = g.coor[g.ref_of[x]];  // i*ny*nz + j*nz + k
    const int i = c / (g.ny * g.nz), j = (c % (g.ny * g.nz)) / g.nz, k = c % g.nz;
    in[x] = i >= window[0] && i <= window[1] && j >= window[2] && j <= window[3] && k >= window[4] && k <= window[5];
    pores += in[x];
  }
  g.porosity = h->window_volume > 0 ? (double)pores / (double)h->window_volume : 0.0;
  if (!restrict_nodes) {
    h->win.alloc(0);
    return LBM_OK;
  }
  LBM_CUDA_TRY(h->win.alloc(in.size()));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->win.p, in.data(), in.size(), cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status lbm_cg_set_random(lbm_cg_handle* h, double ini_sat, unsigned long long seed) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  h->rand_sat = ini_sat;
  h->rand_seed = seed;
  return LBM_OK;
}

// Phase faces of comput_macro_variables (in_psi_BC = 1, CG3:3386-3700), after
// the macro step's psi, in the reference's order: the faces x-, x+, y-, y+,
// z-, z+, each walking its node list (x faces: z outer, y inner; y faces: z
// outer, x inner; z faces: y outer, x inner; CG3:2029-2101):
//   1  the node takes its initial phase;
//   2  the node takes the phase of its +x neighbour (periodic), which may be a
//      face node already set earlier in the walk; a node whose +x neighbour
//      is solid resets every node of the face list to its initial phase and
//      the walk goes on;
//   3  the node takes +1 when draw % 10000 / 10000 < ini_Sat, else -1, with
//      the face draws numbered from 0 in walk order at every macro step (the
//      reference reseeds from the clock at the start of the macro step,
//      CG3:3321; here a fixed seed, lbm_cg_set_random);
// rho_r = (psi + 1) / 2, rho_b = 1 - rho_r.  The walk is resolved here once:
// the final value of every face node is either a constant (its initial
// phase, a draw) or the phase some node had before the walk (flag 2 chains),
// so every step gathers those values and then writes the face nodes.
lbm_status lbm_cg_set_phase_faces(lbm_cg_handle* h, const int faces[6]) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!faces) return fail(LBM_ERR_ARG, "lbm_cg_set_phase_faces: null faces");
  for (int f = 0; f < 6; f++)
    if (faces[f] < 0 || faces[f] > 3)
      return fail(LBM_ERR_ARG, "lbm_cg_set_phase_faces: a face is 0 (off), 1 (initial phase), 2 (phase of the +x "
                               "neighbour) or 3 (random)");
  if (!h->given && !h->colour_done) {
    // the pending macro step keeps the faces it was computed under
    LBM_CUDA_TRY(resolve_faces(h));
    LBM_CUDA_TRY(colour_pass(h, cg_args(h, h->cur, 0)));
    h->colour_done = true;
  }
  const Geometry& g = h->geo;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  std::vector<int32_t> at((size_t)nx * ny * nz, -1);  // cell (i*ny*nz + j*nz + k) -> node
  for (int x = 0; x < g.count; x++) at[g.coor[g.ref_of[x]]] = x;
  auto node = [&](int i, int j, int k) { return at[((size_t)i * ny + j) * nz + k]; };
  // value of a node in the walk: kind 0 = its phase before the walk (src), 1 = constant (val)
  struct Sym {
    int8_t kind;
    int32_t src;
    double val;
  };
  std::vector<Sym> cur((size_t)g.count);
  for (int x = 0; x < g.count; x++) cur[x] = Sym{0, x, 0.0};
  std::vector<uint8_t> touched((size_t)g.count, 0);
  int slot = 0;
  // walk order x-, x+, y-, y+, z-, z+ (faces[] is in INPUT order xp, xn, yp, yn, zp, zn)
  const int order[6] = {1, 0, 3, 2, 5, 4};
  for (int o = 0; o < 6; o++) {
    const int f = order[o], flag = faces[f];
    if (!flag) continue;
    std::vector<int32_t> list;
    if (f <= 1) {
      const int i = f == 1 ? 0 : nx - 1;
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          if (node(i, j, k) >= 0) list.push_back(node(i, j, k));
    } else if (f <= 3) {
      const int j = f == 3 ? 0 : ny - 1;
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++)
          if (node(i, j, k) >= 0) list.push_back(node(i, j, k));
    } else {
      const int k = f == 5 ? 0 : nz - 1;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
          if (node(i, j, k) >= 0) list.push_back(node(i, j, k));
    }
    for (int32_t x : list) touched[x] = 1;
    if (flag == 1) {
      for (int32_t x : list) cur[x] = Sym{1, -1, h->psi0[x]};
    } else if (flag == 2) {
      for (size_t ii = 0; ii < list.size(); ii++) {
        const int c = g.coor[g.ref_of[list[ii]]];
        const int i = c / (ny * nz), j = (c % (ny * nz)) / nz, k = c % nz;
        const int nb = node((i + 1) % nx, j, k);
        if (nb >= 0) {
          cur[list[ii]] = cur[nb];
        } else {
          for (int32_t x : list) cur[x] = Sym{1, -1, h->psi0[x]};
        }
      }
    } else {
      for (int32_t x : list) {
        const double r = (double)(cg_draw(h->rand_seed, (unsigned long long)slot++) % 10000) / 10000;
        cur[x] = Sym{1, -1, r < h->rand_sat ? 1.0 : -1.0};
      }
    }
  }
  std::vector<int32_t> nodes, src;
  std::vector<double> vals;
  bool copy = false;
  for (int x = 0; x < g.count; x++) {
    if (!touched[x]) continue;
    const Sym& s = cur[x];
    if (s.kind == 0 && s.src == x) continue;  // a flag-2 chain back to its own phase
    nodes.push_back(x);
    src.push_back(s.kind == 0 ? s.src : -1);
    vals.push_back(s.kind == 0 ? 0.0 : s.val);
    copy = copy || s.kind == 0;
  }
  h->nface = (int)nodes.size();
  h->face_copy = copy;
  if (h->nface > 0) {
    LBM_CUDA_TRY(h->face_nodes.alloc(nodes.size() * sizeof(int32_t)));
    LBM_CUDA_TRY(h->face_psi0.alloc(vals.size() * sizeof(double)));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->face_nodes.p, nodes.data(), nodes.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                 h->stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->face_psi0.p, vals.data(), vals.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
    if (copy) {
      LBM_CUDA_TRY(h->face_src.alloc(src.size() * sizeof(int32_t)));
      LBM_CUDA_TRY(h->face_tmp.alloc(vals.size() * sizeof(double)));
      LBM_CUDA_TRY(cudaMemcpyAsync(h->face_src.p, src.data(), src.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                   h->stream));
    }
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  drop_graphs(h);  // the chains captured so far do not apply these faces
  return LBM_OK;
}

lbm_status lbm_cg_set_state(lbm_cg_handle* h, const double* f, const double* psi, const double* rho_r,
                            const double* rho_b) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (!f || !psi || !rho_r || !rho_b) return fail(LBM_ERR_ARG, "lbm_cg_set_state: null argument");
  const int n = h->geo.count, npad = h->geo.npad;
  Dev in;
  const size_t fbytes = (size_t)(n + 1) * kQ * sizeof(double);
  LBM_CUDA_TRY(in.alloc(fbytes));
  LBM_CUDA_TRY(cudaMemcpyAsync(in.p, f, fbytes, cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cg_import_f(h->f64, h->f[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n, npad,
                           in.as<double>(), h->stream));
  // scalar fields: internal order equals reference order - 1 for this solver
  const double* srcs[3] = {psi, rho_r, rho_b};
  Dev* dsts[3] = {&h->psi, &h->rho_r, &h->rho_b};
  std::vector<double> d(npad, 0.0);
  std::vector<float> fl(npad, 0.f);
  for (int i = 0; i < 3; i++) {
    for (int x = 0; x < n; x++) d[x] = srcs[i][h->geo.ref_of[x]];
    if (h->f64) {
      LBM_CUDA_TRY(cudaMemcpyAsync(dsts[i]->p, d.data(), sizeof(double) * npad, cudaMemcpyHostToDevice, h->stream));
    } else {
      for (int x = 0; x < npad; x++) fl[x] = (float)d[x];
      LBM_CUDA_TRY(cudaMemcpyAsync(dsts[i]->p, fl.data(), sizeof(float) * npad, cudaMemcpyHostToDevice, h->stream));
    }
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  h->given = 2;
  h->colour_done = false;
  h->uprev_valid = false;
  h->faces_pending = false;  // the state given is the one after its step's rules
  return LBM_OK;
}

lbm_status lbm_read_cg_input(const char* path, lbm_cg_input* out) { return read_cg_input_file(path, out); }

lbm_status lbm_read_phase(const char* path, int nx, int ny, int nz, double* out) {
  return read_phase_file(path, nx, ny, nz, out);
}

// Initial phase of the mixture injection (psi_mixture_ini, CG3:6151-6350).
// In the plane x = thickness, pore cells next to a solid cell are marked
// wetting (up to portion x the plane's pore count), starting at the plane's
// centre and walking square rings outwards; a second pass of rings marks
// cells next to a solid or an already marked cell (the cells it marks only
// count as marked after the pass).  The neighbours looked at are CG
// directions 0..17 (the cell itself included, direction 18 = (0,-1,1) not),
// within the box (no wrap).  Every cell with x <= thickness whose column
// (thickness, y, z) is an unmarked pore starts in component B (psi = -1),
// every other cell in component A (psi = +1).  The reference walks the rings
// up to max(ny, nz)/2 and reads outside the plane when ny != nz; cells outside
// the plane count here as not pore.
lbm_status lbm_cg_mixture_phase(const uint8_t* mask, int nx, int ny, int nz, int thickness, double portion,
                                double* psi_out) {
  if (!mask || !psi_out || nx <= 0 || ny <= 0 || nz <= 0)
    return fail(LBM_ERR_ARG, "lbm_cg_mixture_phase: bad argument");
  if (thickness <= 0 || thickness >= nx)
    return fail(LBM_ERR_ARG, "lbm_cg_mixture_phase: thickness must lie in 1..nx-1");
  const int ci = thickness;
  auto solid = [&](int i, int j, int k) { return mask[((size_t)k * ny + j) * nx + i] != 0; };
  // state of the plane x = ci: 1 solid, 0 pore, 2 marked, -2 marked in this ring pass
  std::vector<int> s2((size_t)ny * nz);
  auto at = [&](int j, int k) -> int& { return s2[(size_t)j * nz + k]; };
  int fluid_sum = 0;
  for (int j = 0; j < ny; j++)
    for (int k = 0; k < nz; k++) {
      at(j, k) = solid(ci, j, k) ? 1 : 0;
      fluid_sum += at(j, k) == 0;
    }
  const int nw_node = (int)(fluid_sum * portion);
  int marked = 0;
  // state of any cell of the box: the plane's own state, elsewhere the mask
  auto state = [&](int i, int j, int k) { return i == ci ? at(j, k) : (solid(i, j, k) ? 1 : 0); };
  auto next_to = [&](int j, int k, bool level2) {
    for (int ls = 0; ls < 18; ls++) {
      const int li = ci + cg::ex(ls), lj = j + cg::ey(ls), lk = k + cg::ez(ls);
      if (li < 0 || li >= nx || lj < 0 || lj >= ny || lk < 0 || lk >= nz) continue;
      const int v = state(li, lj, lk);
      if (level2 ? v > 0 : v == 1) return true;
    }
    return false;
  };
  auto visit = [&](int j, int k, bool level2) {
    if (j < 0 || j >= ny || k < 0 || k >= nz || at(j, k) != 0) return;
    if (next_to(j, k, level2) && marked < nw_node) {
      at(j, k) = level2 ? -2 : 2;
      marked++;
    }
  };
  const int ceny = ny / 2, cenz = nz / 2;
  const int rad_max = std::max(ny / 2, nz / 2);
  visit(ceny, cenz, false);
  for (int pass = 0; pass < 2; pass++) {
    const bool level2 = pass == 1;
    for (int rad = 1; marked < nw_node && rad < rad_max; rad++) {
      for (int k = cenz - rad; k <= cenz + rad; k += 2 * rad)
        for (int j = ceny - rad; j <= ceny + rad; j++) visit(j, k, level2);
      for (int j = ceny - rad; j <= ceny + rad; j += 2 * rad)
        for (int k = cenz - rad; k <= cenz + rad; k++) visit(j, k, level2);
    }
  }
  for (auto& v : s2)
    if (v == -2) v = 2;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) psi_out[((size_t)k * ny + j) * nx + i] = (i <= ci && at(j, k) == 0) ? -1.0 : 1.0;
  return LBM_OK;
}

lbm_status lbm_cg_set_zero_sigma(lbm_cg_handle* h, int x_last) {
  lbm_status st = cg_check(h);
  if (st != LBM_OK) return st;
  if (x_last < 0) {
    h->zero_sigma.alloc(0);
    h->cp.zero_sigma = nullptr;
    return LBM_OK;
  }
  const Geometry& g = h->geo;
  std::vector<uint8_t> flag((size_t)g.npad, 0);
  for (int x = 0; x < g.count; x++) {
    const int c = g.coor[g.ref_of[x]];  // i*ny*nz + j*nz + k
    flag[x] = c / (g.ny * g.nz) <= x_last;
  }
  LBM_CUDA_TRY(h->zero_sigma.alloc(flag.size()));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->zero_sigma.p, flag.data(), flag.size(), cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->cp.zero_sigma = h->zero_sigma.as<uint8_t>();
  return LBM_OK;
}

lbm_status lbm_cg_create_from_input(const char* input_path, int precision, lbm_cg_handle** out,
                                    lbm_cg_input* parsed_out) {
  return lbm_cg_create_from_input_seeded(input_path, precision, 0ULL, out, parsed_out);
}

lbm_status lbm_cg_create_from_input_seeded(const char* input_path, int precision, unsigned long long seed,
                                           lbm_cg_handle** out, lbm_cg_input* parsed_out) {
  if (!out) return fail(LBM_ERR_ARG, "lbm_cg_create_from_input: null output");
  *out = nullptr;
  lbm_cg_input in;
  lbm_status st = read_cg_input_file(input_path, &in);
  if (st != LBM_OK) return st;
  if (parsed_out) *parsed_out = in;
  // the phase read from file (CG3:2355-2380)
  const int pre[6] = {in.pre_xp, in.pre_xn, in.pre_yp, in.pre_yn, in.pre_zp, in.pre_zn};
  const int vel[6] = {in.vel_xp, in.vel_xn, in.vel_yp, in.vel_yn, in.vel_zp, in.vel_zn};
  for (int f = 0; f < 6; f++)
    if ((pre[f] != 0 && pre[f] != 1) || (vel[f] != 0 && vel[f] != 1))
      return fail(LBM_ERR_ARG, "pre_* / vel_*: face flags must be 0 or 1");
  const int pf[6] = {in.psi_xp, in.psi_xn, in.psi_yp, in.psi_yn, in.psi_zp, in.psi_zn};
  for (int f = 0; f < 6; f++)
    if (in.in_psi_bc == 1 && (pf[f] < 0 || pf[f] > 3))
      return fail(LBM_ERR_ARG, "psi_xp..psi_zn: a phase face is 0, 1 (initial phase), 2 (+x neighbour) or 3 (random)");
  if (in.mix_psi_thickness > 0 && in.mix_psi_thickness >= in.nx)
    return fail(LBM_ERR_ARG, "mix_psi_thickness must be smaller than nx");
  if (in.lattice_v != 0) return fail(LBM_ERR_ARG, "lattice_v: self-defined lattice velocity is not supported");
  if (in.rel_perm_id_dir < 0 || in.rel_perm_id_dir > 2)
    return fail(LBM_ERR_ARG, "rel_perm_id_dir: 0 (off), 1 (imbibition) or 2 (drainage)");
  if (in.rel_perm_id_dir > 0 && in.rel_perm_chan_num <= 0)
    return fail(LBM_ERR_ARG, "rel_perm_id_dir: rel_perm_chan_num must be positive");
  if (in.input_dynamic > 0 && in.update_fre <= 0)
    return fail(LBM_ERR_ARG, "input_dynamic: the update interval must be positive (the reference takes n % update_fre)");
  // the imbibition / drainage control turns the phase faces on in init
  // (CG3:2339-2345); a restart (Backup_init) skips it
  if (in.rel_perm_id_dir > 0 && in.mode_backup_ini == 0) in.in_psi_bc = 1;
  if (in.pressure_change2 < 0 || in.pressure_change2 > 3)
    return fail(LBM_ERR_ARG, "pressure_change2: the capillary-pressure axis is 0 (off) or 1..3");
  if (in.pressure_change2 > 0 && (in.chan_no <= 0 || in.interval_pre <= 0))
    return fail(LBM_ERR_ARG, "pressure_change2: chan_no and interval_pre must be positive");
  if (in.fre_re <= 0) return fail(LBM_ERR_ARG, "freRe must be positive");
  if (in.fre_psi == 0) return fail(LBM_ERR_ARG, "frePsi = 0: the reference takes n % 0; use -1 or a positive interval");
  if (in.least_square > 0 && in.num_least_square < 2)
    return fail(LBM_ERR_ARG, "num_least_square must be at least 2 for the least-squares fit");
  const size_t cells = (size_t)in.nx * in.ny * in.nz;
  std::vector<uint8_t> mask(cells);
  std::vector<double> psi(cells);
  // file paths are relative to the working directory, as in the reference
  if ((st = read_mask_file(in.geometry_file, in.nx, in.ny, in.nz, in.decbin, mask.data())) != LBM_OK) return st;
  if (in.mix_psi_thickness > 0) {
    // mixture injection: the initial phase is built from the geometry and
    // the phase file is not read (CG3:2117-2128)
    if ((st = lbm_cg_mixture_phase(mask.data(), in.nx, in.ny, in.nz, in.mix_psi_thickness, in.protion_w,
                                   psi.data())) != LBM_OK)
      return st;
  } else if (in.ini_sat >= 0) {
    // random initial phase (init, CG3:2384-2455): one draw per fluid node in
    // id order, +1 when draw % 10000 / 10000 < ini_Sat; with a partial
    // permeability window and a buffer phase (ini_buf = +-1), the nodes
    // outside the window on a windowed axis take the buffer phase.  The
    // reference seeds from the clock (CG3:2232); here the seed is given.
    Geometry order;
    compact_reference(mask.data(), in.nx, in.ny, in.nz, &order);
    const int nyz = in.ny * in.nz;
    for (int id = 1; id <= order.count; id++) {
      const int c = order.coor[id];  // i*ny*nz + j*nz + k
      const int i = c / nyz, j = (c % nyz) / in.nz, k = c % in.nz;
      const double r = (double)(cg_draw(seed, (unsigned long long)(id - 1)) % 10000) / 10000;
      double v = r < in.ini_sat ? 1.0 : -1.0;
      const bool outside = (in.par_per_x > 0 && (i < in.per_xn || i > in.per_xp)) ||
                           (in.par_per_y > 0 && (j < in.per_yn || j > in.per_yp)) ||
                           (in.par_per_z > 0 && (k < in.per_zn || k > in.per_zp));
      if (outside && (in.ini_buf == 1 || in.ini_buf == -1)) v = in.ini_buf;
      psi[((size_t)k * in.ny + j) * in.nx + i] = v;
    }
  } else if ((st = read_phase_file(in.phase_file, in.nx, in.ny, in.nz, psi.data())) != LBM_OK) {
    return st;
  }
  lbm_cg_params p{};
  p.nu_l = in.nu_l;
  p.nu_g = in.nu_g;
  p.psi_solid = in.contact_angle;  // CG3:2355
  p.cap_a = in.cap_a;
  const bool stab = in.stab == 1;  // gxs = 0 until stab_time (CG3:2375-2378)
  p.gx = stab ? 0.0 : in.gx;
  p.gy = stab ? 0.0 : in.gy;
  p.gz = stab ? 0.0 : in.gz;
  p.body_force_phase = in.bodyforce_apply;
  p.flux_psi = in.rel_perm_psi;
  p.flux_umax = in.rel_perm_psi2;
  p.precision = precision;
  p.device = 0;
  p.perdir = in.perdir;
  // pressure/velocity faces, their rules from stab_time when the stabiliser
  // is on (CG3:868)
  lbm_boundary bc{};
  bc.sub_bc = in.sub_bc;
  bc.in_bc = in.in_bc;
  const double rho_f[6] = {in.p_xp, in.p_xn, in.p_yp, in.p_yn, in.p_zp, in.p_zn};
  const double vel_f[6] = {in.v_xp, in.v_xn, in.v_yp, in.v_yn, in.v_zp, in.v_zn};
  for (int f = 0; f < 6; f++) {
    bc.pressure[f] = pre[f];
    bc.velocity[f] = vel[f];
    bc.rho[f] = rho_f[f];
    bc.vel[f] = vel_f[f];
  }
  lbm_cg_handle* h = nullptr;
  if ((st = lbm_cg_create_bc(&p, &bc, mask.data(), psi.data(), in.nx, in.ny, in.nz, &h)) != LBM_OK) return st;
  if (stab && in.stab_time > 0) h->cp.faces = 0;
  if (in.par_per_x || in.par_per_y || in.par_per_z) {
    // an axis without a partial window spans the whole box (CG3:1707-1712);
    // the sums are limited to the window when one of par_per_* is 1
    // (CG3:5156, 5307)
    const int w[6] = {in.par_per_x ? in.per_xn : 0, in.par_per_x ? in.per_xp : in.nx - 1,
                      in.par_per_y ? in.per_yn : 0, in.par_per_y ? in.per_yp : in.ny - 1,
                      in.par_per_z ? in.per_zn : 0, in.par_per_z ? in.per_zp : in.nz - 1};
    const int restrict_nodes = (in.par_per_x - 1) * (in.par_per_y - 1) * (in.par_per_z - 1) == 0;
    if ((st = lbm_cg_set_window(h, w, restrict_nodes)) != LBM_OK) {
      lbm_cg_destroy(h);
      return st;
    }
  }
  if (in.in_psi_bc == 1 && (pf[0] || pf[1] || pf[2] || pf[3] || pf[4] || pf[5])) {
    if ((st = lbm_cg_set_random(h, in.ini_sat, seed)) != LBM_OK || (st = lbm_cg_set_phase_faces(h, pf)) != LBM_OK) {
      lbm_cg_destroy(h);
      return st;
    }
  }
  // the surface tension is off in the layer x <= zero_sigma_thickness while
  // the mixture injects at the x- face (CG3:2854-2855)
  if (in.mix_psi_thickness > 0 && in.psi_xn > 0) {
    if ((st = lbm_cg_set_zero_sigma(h, in.zero_sigma_thickness)) != LBM_OK) {
      lbm_cg_destroy(h);
      return st;
    }
  }
  // the initial velocity of init (CG3:2357-2362); a restart's checkpoint
  // replaces the state afterwards, as Backup_init does after init
  if (in.inivx != 0 || in.inivy != 0 || in.inivz != 0) {
    if ((st = lbm_cg_set_initial_velocity(h, in.inivx, in.inivy, in.inivz)) != LBM_OK) {
      lbm_cg_destroy(h);
      return st;
    }
  }
  *out = h;
  return LBM_OK;
}

const uint8_t* lbm_cg_internal_mask(lbm_cg_handle* h, int* nx, int* ny, int* nz) {
  *nx = h->geo.nx;
  *ny = h->geo.ny;
  *nz = h->geo.nz;
  return h->mask.data();
}

lbm_status lbm_cg_info(lbm_cg_handle* h, int* count, double* porosity, long long* step, double* last_step_ms) {
  if (!h) return fail(LBM_ERR_ARG, "null cg handle");
  if (count) *count = h->geo.count;
  if (porosity) *porosity = h->geo.porosity;
  if (step) *step = h->step;
  if (last_step_ms) *last_step_ms = h->last_ms;
  return LBM_OK;
}

void lbm_cg_destroy(lbm_cg_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
}

}  // extern "C"
