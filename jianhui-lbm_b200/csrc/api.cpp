// C ABI of the single-phase solver (include/lbm.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "lbm_internal.h"
#include "setup.h"

namespace lbm {

lbm_status read_input_file(const char* path, lbm_input* o);
cudaError_t launch_box_sums(const int32_t* cell_idx, const double* u, int npad, int nx, int ny, const int32_t* boxes,
                            int nbox, int chunks, double* partials, double* out, cudaStream_t st);
lbm_status read_mask_file(const char* path, int nx, int ny, int nz, int decbin, uint8_t* mask);

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
lbm_status fail(lbm_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

static Store store_of(int precision) {
  switch (precision) {
    case LBM_PREC_F64: return Store::F64;
    case LBM_PREC_F32: return Store::F32;
    case LBM_PREC_F16: return Store::F16;
    default: return Store::F64D;
  }
}

// feq of `feq` (SP3:1382-1394) on the lattice L (elat = e lat_c).
static double feq_ref(int q, double rho, const double* u, const Lattice& L) {
  const double c2 = L.c2, c4 = L.c4;
  const double ex = (double)cx(q) * L.c, ey = (double)cy(q) * L.c, ez = (double)cz(q) * L.c;
  const double eu = ex * u[0] + ey * u[1] + ez * u[2];
  const double uv = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  return weight(q) * rho * (1.0 + 3.0 * eu / c2 + 4.5 * eu * eu / c4 - 1.5 * uv / c2);
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
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

// Allocator whose value-less construct leaves the element uninitialised, so
// that resizing a byte vector that is overwritten at once does not first
// zero it on one thread.
template <class T>
struct UninitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = UninitAlloc<U>;
  };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) {}
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    if constexpr (sizeof...(A) == 0)
      ::new ((void*)p) U;
    else
      ::new ((void*)p) U(std::forward<A>(a)...);
  }
};

// Copies the caller's mask into dst and counts its pore cells (value 0) in
// one pass split over a few threads: at 256^3 a serial copy and a serial
// count took 2-8 and 5-8 ms of lbm_create.
long long copy_mask_count_pores(const uint8_t* src, size_t cells, uint8_t* dst) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max(1u, std::min(8u, hw ? hw : 1u));
  const size_t min_part = size_t(1) << 20;
  const int parts = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, cells / min_part));
  std::vector<long long> pores(parts, 0);
  auto work = [&](int t) {
    const size_t lo = cells * t / parts, hi = cells * (t + 1) / parts;
    std::memcpy(dst + lo, src + lo, hi - lo);
    long long c = 0;
    for (size_t i = lo; i < hi; i++) c += (src[i] == 0);
    pores[t] = c;
  };
  std::vector<std::thread> th;
  for (int t = 1; t < parts; t++) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  long long total = 0;
  for (long long c : pores) total += c;
  return total;
}

}  // namespace lbm

using namespace lbm;

struct lbm_handle {
  lbm_params prm{};
  Store kind = Store::F32;
  std::vector<uint8_t, UninitAlloc<uint8_t>> mask;
  Geometry geo;
  MrtConstants mrt{};
  Lattice lat;  // self-defined lattice velocity (lbm_set_lattice); default lattice otherwise
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // with pressure/velocity faces the face kernel of a step runs on `side`
  // beside the step kernel (ev_fork: the step's start, ev_bc: faces done)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_bc = nullptr;
  DevBuf pop[2], table, ref_of, window, rho_given, u_given, rho_prev, u_prev, partials, result;
  // pressure/velocity faces: plan, per-step records (ping-pong like pop),
  // operations, M^-1 for the moment rule, post-rule populations of the state
  BcPlan bc;
  DevBuf snap[2], bc_ops, bc_off, bc_mi, bnd_f;
  // dense cell -> internal index map for box sums, built on first use
  DevBuf cell_idx;
  bool cell_idx_valid = false;
  // compact pull table of the step kernel (built after every layout); the
  // fraction of (warp, direction) pairs that keep reading the full table
  DevBuf ct_base, ct_off, ct_wide;
  bool ct_ok = false;
  bool ct_on = false;  // the int32 table unless chosen (lbm_set_table_mode, lbm_autotune)
  double ct_wide_frac = 1.0;
  // field export: device buffers kept between calls
  DevBuf x_rint, x_uint, x_rref, x_uref;
  int cur = 0;
  long long step = 0;
  bool given_macro = true;  // next step / reduce takes rho, u from rho_given / u_given
  bool uprev_valid = false;
  double perm_prev[3] = {0, 0, 0};
  int overspeed = 0;
  int block = 256;
  int ordering = LBM_ORDER_REFERENCE;
  int last_p = -1;
  double fp16_scale = 1.0;
  double last_ms = 0.0;
  // captured step chains, one per starting buffer
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_steps = 0;
  // false when the layout was built on the device and the host copies of the
  // compaction / node order (needed only for exports and re-layouts) are not
  // built yet
  bool host_geo = true;

  ~lbm_handle() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_bc) cudaEventDestroy(ev_bc);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
  size_t mac_bytes() const { return (kind == Store::F64 || kind == Store::F64D) ? 8 : 4; }
  void drop_graphs() {
    for (auto& g : graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
};

namespace lbm {
const uint8_t* lbm_internal_mask(lbm_handle* h, int* nx, int* ny, int* nz) {
  *nx = h->geo.nx;
  *ny = h->geo.ny;
  *nz = h->geo.nz;
  return h->mask.data();
}
}  // namespace lbm

namespace {

// Compact form of the pull table (read by the step kernel; the other kernels
// keep reading the int32 table).
lbm_status build_compact_table(lbm_handle* h) {
  const int npad = h->geo.npad;
  h->ct_ok = false;
  if (!h->ct_base.p) {
    LBM_CUDA_TRY(h->ct_base.alloc((size_t)18 * (npad / 32) * sizeof(int32_t)));
    LBM_CUDA_TRY(h->ct_off.alloc((size_t)18 * npad * sizeof(uint16_t)));
    LBM_CUDA_TRY(h->ct_wide.alloc(sizeof(unsigned long long)));
  }
  LBM_CUDA_TRY(launch_compact_table(h->table.as<int32_t>(), h->geo.count, npad, h->ct_base.as<int32_t>(),
                                    h->ct_off.as<uint16_t>(), h->ct_wide.as<unsigned long long>(), h->stream));
  unsigned long long wide = 0;
  LBM_CUDA_TRY(cudaMemcpyAsync(&wide, h->ct_wide.p, sizeof(wide), cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->ct_wide_frac = (double)wide / (18.0 * (npad / 32));
  h->ct_ok = true;
  h->drop_graphs();
  return LBM_OK;
}

// Table bytes the step kernel reads per node.
double table_bytes_per_node(const lbm_handle* h) {
  if (!(h->ct_ok && h->ct_on)) return 18.0 * 4.0;
  return 18.0 * 2.0 + 18.0 * 4.0 / 32.0 + h->ct_wide_frac * 18.0 * 4.0;
}

lbm_status upload_layout(lbm_handle* h) {
  Geometry& g = h->geo;
  const size_t npad = (size_t)g.npad;
  LBM_CUDA_TRY(cudaMemcpyAsync(h->table.p, g.src.data(), sizeof(int32_t) * 18 * npad, cudaMemcpyHostToDevice,
                               h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->ref_of.p, g.ref_of.data(), sizeof(int32_t) * (size_t)std::max(g.count, 1),
                               cudaMemcpyHostToDevice, h->stream));
  if (!g.in_window.empty()) {
    if (!h->window.p) LBM_CUDA_TRY(h->window.alloc((size_t)g.count));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->window.p, g.in_window.data(), (size_t)g.count, cudaMemcpyHostToDevice, h->stream));
  }
  h->last_p = g.count > 0 ? g.int_of[g.count] : -1;
  h->drop_graphs();
  h->cell_idx_valid = false;
  // the compact form is built when it is first chosen (lbm_set_table_mode,
  // lbm_autotune) or asked about (lbm_table_info); a new layout rebuilds it
  // only when it is in use
  h->ct_ok = false;
  return h->ct_on ? build_compact_table(h) : LBM_OK;
}

// Host copies of the compaction and node order, built on first need.
void ensure_host_geometry(lbm_handle* h) {
  if (h->host_geo) return;
  const int nx = h->geo.nx, ny = h->geo.ny, nz = h->geo.nz;
  Geometry g;
  compact_reference(h->mask.data(), nx, ny, nz, &g);
  order_nodes(h->mask.data(), h->ordering, &g);
  h->geo.coor = std::move(g.coor);
  h->geo.ref_of = std::move(g.ref_of);
  h->geo.int_of = std::move(g.int_of);
  h->host_geo = true;
}

lbm_status upload_bc(lbm_handle* h) {
  const BcPlan& b = h->bc;
  if (!b.active) return LBM_OK;
  if (!h->side) {
    LBM_CUDA_TRY(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    LBM_CUDA_TRY(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    LBM_CUDA_TRY(cudaEventCreateWithFlags(&h->ev_bc, cudaEventDisableTiming));
  }
  const int n = h->geo.count;
  const size_t nsnap = (size_t)std::max(n - b.snap_begin, 1), nbnd = (size_t)std::max(n - b.n_main, 1);
  for (auto& sb : h->snap) {
    if (sb.bytes != kSnapRows * nsnap * sizeof(double)) LBM_CUDA_TRY(sb.alloc(kSnapRows * nsnap * sizeof(double)));
    LBM_CUDA_TRY(cudaMemsetAsync(sb.p, 0, sb.bytes, h->stream));
  }
  if (h->bnd_f.bytes != (size_t)kQ * nbnd * sizeof(double)) LBM_CUDA_TRY(h->bnd_f.alloc((size_t)kQ * nbnd * sizeof(double)));
  LBM_CUDA_TRY(h->bc_ops.alloc(std::max<size_t>(b.ops.size(), 1) * sizeof(BcOp)));
  LBM_CUDA_TRY(h->bc_off.alloc(b.op_off.size() * sizeof(int32_t)));
  if (!b.ops.empty())
    LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_ops.p, b.ops.data(), b.ops.size() * sizeof(BcOp), cudaMemcpyHostToDevice,
                                 h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_off.p, b.op_off.data(), b.op_off.size() * sizeof(int32_t),
                               cudaMemcpyHostToDevice, h->stream));
  if (!h->bc_mi.p) {
    LBM_CUDA_TRY(h->bc_mi.alloc(kQ * kQ * sizeof(double)));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->bc_mi.p, &h->mrt.MI[0][0], kQ * kQ * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
  }
  // host copies of the plan arrays must outlive the asynchronous copies
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status layout(lbm_handle* h, int ordering) {
  ensure_host_geometry(h);
  order_nodes(h->mask.data(), ordering, &h->geo);
  bc_partition(h->mask.data(), h->prm.bc, &h->geo, &h->bc);
  build_pull_table(h->mask.data(), &h->geo);
  set_window(h->prm.window, &h->geo);
  h->ordering = ordering;
  lbm_status st = upload_layout(h);
  if (st != LBM_OK) return st;
  return upload_bc(h);
}

lbm_status alloc_device(lbm_handle* h) {
  const size_t npad = (size_t)h->geo.npad;
  const size_t s = store_bytes(h->kind);
  for (auto& b : h->pop) LBM_CUDA_TRY(b.alloc(kQ * npad * s));
  LBM_CUDA_TRY(h->table.alloc(18 * npad * sizeof(int32_t)));
  LBM_CUDA_TRY(h->ref_of.alloc(std::max<size_t>(h->geo.count, 1) * sizeof(int32_t)));
  LBM_CUDA_TRY(h->rho_given.alloc(npad * h->mac_bytes()));
  LBM_CUDA_TRY(h->u_given.alloc(3 * npad * h->mac_bytes()));
  LBM_CUDA_TRY(h->rho_prev.alloc(npad * h->mac_bytes()));
  LBM_CUDA_TRY(h->u_prev.alloc(3 * npad * h->mac_bytes()));
  LBM_CUDA_TRY(h->partials.alloc((size_t)reduce_blocks(h->geo.count) * 8 * sizeof(double)));
  LBM_CUDA_TRY(h->result.alloc(8 * sizeof(double)));
  return LBM_OK;
}

lbm_status init_state(lbm_handle* h) {
  double feq[kQ];
  for (int q = 0; q < kQ; q++) feq[q] = feq_ref(q, 1.0, h->prm.u_init, h->lat);
  LBM_CUDA_TRY(launch_init_uniform(h->kind, h->pop[0].p, h->table.as<int32_t>(), h->geo.count, h->geo.npad,
                                   h->fp16_scale, feq, h->stream));
  LBM_CUDA_TRY(launch_fill_macro(h->kind, h->rho_given.p, h->u_given.p, h->geo.count, h->geo.npad, 1.0,
                                 h->prm.u_init, h->stream));
  h->cur = 0;
  h->step = 0;
  h->given_macro = true;
  h->uprev_valid = false;
  h->perm_prev[0] = h->perm_prev[1] = h->perm_prev[2] = 0.0;
  h->overspeed = 0;
  return LBM_OK;
}

// The force as the step and reduce kernels take it: g itself for the FP64
// reference kernel, dt g / lat_c for the kernels that work in units of lat_c
// (g on the default lattice).
void kernel_force(const lbm_handle* h, double* gx, double* gy, double* gz) {
  const double s = (h->lat.on && h->kind != Store::F64) ? h->lat.dt / h->lat.c : 1.0;
  *gx = h->lat.on ? h->prm.gx * s : h->prm.gx;
  *gy = h->lat.on ? h->prm.gy * s : h->prm.gy;
  *gz = h->lat.on ? h->prm.gz * s : h->prm.gz;
}

StepArgs step_args(lbm_handle* h, bool write) {
  StepArgs a{};
  a.src_pop = h->pop[h->cur].p;
  a.dst_pop = h->pop[1 - h->cur].p;
  a.table = h->table.as<int32_t>();
  a.n = h->geo.count;
  a.npad = h->geo.npad;
  a.rho_in = h->given_macro ? h->rho_given.p : nullptr;
  a.u_in = h->given_macro ? h->u_given.p : nullptr;
  a.rho_out = write ? h->rho_prev.p : nullptr;
  a.u_out = write ? h->u_prev.p : nullptr;
  kernel_force(h, &a.gx, &a.gy, &a.gz);
  a.lat = h->lat;
  a.s_v = h->mrt.s_v;
  a.s_o = h->mrt.s_o;
  a.fp16_scale = h->fp16_scale;
  const int n = h->geo.count;
  a.n_main = h->bc.active ? h->bc.n_main : n;
  if (h->ct_ok && h->ct_on) {
    a.ct_base = h->ct_base.as<int32_t>();
    a.ct_off = h->ct_off.as<uint16_t>();
    a.nwarps = h->geo.npad / 32;
  }
  a.snap_begin = h->bc.active ? h->bc.snap_begin : n;
  a.nsnap = std::max(n - a.snap_begin, 1);
  a.snap_dst = h->bc.active ? h->snap[1 - h->cur].as<double>() : nullptr;
  return a;
}

// Arguments of the face-node kernel for a step whose step arguments are s and
// whose source buffers have parity c.
BcArgs bc_args(lbm_handle* h, const StepArgs& s, int c) {
  BcArgs b{};
  b.s = s;
  b.snap_src = h->snap[c].as<double>();
  b.op_off = h->bc_off.as<int32_t>();
  b.ops = h->bc_ops.as<BcOp>();
  b.mi = h->bc_mi.as<double>();
  const lbm_boundary& bc = h->prm.bc;
  // face velocities in units of lat_c for the deviation-storage kernels
  const bool scale = h->lat.on && h->kind != Store::F64;
  for (int f = 0; f < 6; f++) {
    b.face_rho[f] = bc.rho[f];
    b.face_u[f][0] = b.face_u[f][1] = b.face_u[f][2] = 0.0;
    b.face_u[f][f / 2] = scale ? bc.vel[f] * h->lat.ic : bc.vel[f];
  }
  b.bnd_f = nullptr;
  return b;
}

// One step: the step kernel over [0, n_main) and, with faces, the face kernel
// over [n_main, n).  The two write disjoint nodes of the new state and of the
// record (the step kernel the nodes below n_main, the face kernel the rest)
// and read only the previous step's, so the face kernel runs on the side
// stream beside the step kernel and the step ends when both have.
cudaError_t launch_full_step(lbm_handle* h, const StepArgs& a, int c) {
  if (!h->bc.active) return launch_step(h->kind, a, h->block, h->stream);
  cudaError_t e = cudaEventRecord(h->ev_fork, h->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
  if (e == cudaSuccess) e = launch_boundary(h->kind, bc_args(h, a, c), h->side);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev_bc, h->side);
  if (e == cudaSuccess) e = launch_step(h->kind, a, h->block, h->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, h->ev_bc, 0);
  return e;
}

// Face nodes of the current state after their rules, for reductions and
// exports (the state itself is the post-collision populations of the last
// step; the reference's f of face nodes is the result of the rules).
lbm_status finalize_faces(lbm_handle* h, int* n_main, const double** bnd_f) {
  *n_main = h->geo.count;
  *bnd_f = nullptr;
  if (!h->bc.active || h->given_macro) return LBM_OK;
  StepArgs s = step_args(h, false);
  s.rho_in = s.u_in = nullptr;
  BcArgs b = bc_args(h, s, h->cur);
  b.bnd_f = h->bnd_f.as<double>();
  LBM_CUDA_TRY(launch_boundary(h->kind, b, h->stream));
  *n_main = h->bc.n_main;
  *bnd_f = h->bnd_f.as<double>();
  return LBM_OK;
}

lbm_status one_step(lbm_handle* h, bool write) {
  const StepArgs a = step_args(h, write);
  LBM_CUDA_TRY(launch_full_step(h, a, h->cur));
  h->cur = 1 - h->cur;
  h->given_macro = false;
  h->step++;
  return LBM_OK;
}

constexpr int kGraphSteps = 16;  // even: a replay leaves the buffer parity unchanged

lbm_status ensure_graph(lbm_handle* h) {
  if (h->graph[h->cur]) return LBM_OK;
  cudaGraph_t g = nullptr;
  const int cur0 = h->cur;
  LBM_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int c = cur0;
  cudaError_t err = cudaSuccess;
  for (int s = 0; s < kGraphSteps && err == cudaSuccess; s++) {
    StepArgs a = step_args(h, false);
    a.src_pop = h->pop[c].p;
    a.dst_pop = h->pop[1 - c].p;
    a.rho_in = a.u_in = nullptr;
    if (h->bc.active) a.snap_dst = h->snap[1 - c].as<double>();
    err = launch_full_step(h, a, c);
    c = 1 - c;
  }
  const cudaError_t end = cudaStreamEndCapture(h->stream, &g);
  if (err != cudaSuccess || end != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(LBM_ERR_CUDA, std::string("graph capture failed: ") +
                                  cudaGetErrorString(err != cudaSuccess ? err : end));
  }
  const cudaError_t inst = cudaGraphInstantiate(&h->graph[cur0], g, 0);
  cudaGraphDestroy(g);
  LBM_CUDA_TRY(inst);
  h->graph_steps = kGraphSteps;
  return LBM_OK;
}

lbm_status run_steps(lbm_handle* h, int nsteps) {
  if (nsteps <= 0) return LBM_OK;
  lbm_status st;
  // capture the step chains before the start event: capture and instantiation
  // are host work and must not count as step time
  if (nsteps - (h->given_macro ? 1 : 0) - 1 >= kGraphSteps) {
    const int cur0 = h->cur;
    for (int parity = 0; parity < 2; parity++) {
      h->cur = parity;
      if ((st = ensure_graph(h)) != LBM_OK) {
        h->cur = cur0;
        return st;
      }
    }
    h->cur = cur0;
  }
  LBM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  int left = nsteps;
  if (h->given_macro) {
    if ((st = one_step(h, left == 1)) != LBM_OK) return st;
    left--;
  }
  // all but the last step through captured chains, the last one writes the
  // pre-collision macro fields (the velocity one step before the new state)
  while (left - 1 >= kGraphSteps) {
    if ((st = ensure_graph(h)) != LBM_OK) return st;
    LBM_CUDA_TRY(cudaGraphLaunch(h->graph[h->cur], h->stream));
    h->step += kGraphSteps;
    left -= kGraphSteps;
  }
  while (left > 0) {
    if ((st = one_step(h, left == 1)) != LBM_OK) return st;
    left--;
  }
  h->uprev_valid = true;
  LBM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  LBM_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  LBM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_ms = ms;
  return LBM_OK;
}

// Error + Comput_Perm on the device; optional macro fields (internal order).
lbm_status reduce_raw(lbm_handle* h, double r[8], double* rho_out_int, double* u_out_int) {
  ReduceArgs a{};
  a.pop = h->pop[h->cur].p;
  a.table = h->table.as<int32_t>();
  a.n = h->geo.count;
  a.npad = h->geo.npad;
  a.rho_in = h->given_macro ? h->rho_given.p : nullptr;
  a.u_in = h->given_macro ? h->u_given.p : nullptr;
  a.u_prev = (!h->given_macro && h->uprev_valid) ? h->u_prev.p : nullptr;
  a.last_p = h->last_p;
  a.window = h->geo.in_window.empty() ? nullptr : h->window.as<uint8_t>();
  kernel_force(h, &a.gx, &a.gy, &a.gz);
  a.lat = h->lat;
  a.fp16_scale = h->fp16_scale;
  a.rho_out = rho_out_int;
  a.u_out = u_out_int;
  a.partials = h->partials.as<double>();
  a.result = h->result.as<double>();
  lbm_status st = finalize_faces(h, &a.n_main, &a.bnd_f);
  if (st != LBM_OK) return st;
  LBM_CUDA_TRY(launch_reduce(h->kind, a, h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(r, a.result, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

void fill_diag(lbm_handle* h, const double r[8], lbm_diag* d) {
  const Geometry& g = h->geo;
  std::memset(d, 0, sizeof(*d));
  d->step = h->step;
  const double t1 = std::sqrt(r[0]), t2 = std::sqrt(r[1]);
  d->u_rel_change = t1 / (t2 + 1e-30);                                   // SP3:3149-3151
  d->u_max = std::sqrt(r[3]);                                             // SP3:3152
  d->u_mean_speed = r[2] / ((double)g.nx * g.ny * g.nz * g.porosity);    // SP3:3183
  const double V = (double)g.window_volume;
  // pressure-gradient term of Comput_Perm (SP3:3543-3556): |p_+ - p_-| c_s^2 / L / dx
  double dp = 0.0;
  if (h->prm.bc.in_bc != 0) {
    const int dir = (h->prm.perdir >= 1 && h->prm.perdir <= 3) ? h->prm.perdir - 1 : 0;
    const int* w = h->prm.window;
    const bool full = w[0] < 0 && w[1] < 0 && w[2] < 0 && w[3] < 0 && w[4] < 0 && w[5] < 0;
    const int ext[3] = {g.nx, g.ny, g.nz};
    const int L = full ? ext[dir] : w[2 * dir + 1] - w[2 * dir] + 1;
    const double c_s2 = h->lat.cs2, dx = h->lat.dx;
    dp = std::fabs(h->prm.bc.rho[2 * dir] - h->prm.bc.rho[2 * dir + 1]) * c_s2 / L / dx;
  }
  const double gg[3] = {h->prm.gx, h->prm.gy, h->prm.gz};
  double perm[3];
  for (int i = 0; i < 3; i++) perm[i] = r[4 + i] / V * h->prm.nu / (gg[i] + dp);  // SP3:3611-3613
  const int dir = (h->prm.perdir >= 1 && h->prm.perdir <= 3) ? h->prm.perdir - 1 : 0;
  d->perm_rel_change = (perm[dir] - h->perm_prev[dir]) / h->perm_prev[dir];  // SP3:3615-3626
  for (int i = 0; i < 3; i++) {
    d->perm[i] = perm[i];
    h->perm_prev[i] = perm[i];
  }
  const double ax = r[4] / (V * g.porosity), ay = r[5] / (V * g.porosity), az = r[6] / (V * g.porosity);
  d->u_ave = std::sqrt(ax * ax + ay * ay + az * az);  // SP3:3634-3638
  d->mass = r[7];
  d->porosity = g.porosity;
  d->nan_detected = (d->u_rel_change != d->u_rel_change) ? 1 : 0;
}

lbm_status check_handle(lbm_handle* h) {
  if (!h) return fail(LBM_ERR_ARG, "null handle");
  if (cudaSetDevice(h->device) != cudaSuccess) return fail(LBM_ERR_CUDA, "cudaSetDevice failed");
  return LBM_OK;
}

}  // namespace

extern "C" {

const char* lbm_last_error(void) { return g_last_error.c_str(); }

const char* lbm_status_string(lbm_status s) {
  switch (s) {
    case LBM_OK: return "ok";
    case LBM_ERR_ARG: return "invalid argument";
    case LBM_ERR_IO: return "i/o error";
    case LBM_ERR_OOM: return "out of memory";
    case LBM_ERR_CUDA: return "cuda error";
    case LBM_ERR_NAN: return "non-finite velocity";
    case LBM_ERR_NOT_CONVERGED: return "not converged";
    case LBM_ERR_FORMAT: return "malformed input";
    case LBM_ERR_STATE: return "invalid state";
    case LBM_ERR_OVERSPEED: return "velocity above 10 (reference stop rule)";
    case LBM_ERR_NO_DEVICE: return "no cuda device";
  }
  return "unknown status";
}

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

void lbm_params_default(lbm_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->nu = 0.1;
  p->gx = 1e-6;
  p->precision = LBM_PREC_F32;
  p->ordering = LBM_ORDER_REFERENCE;
  p->block_size = 256;
  p->perdir = 1;
  for (int i = 0; i < 6; i++) p->window[i] = -1;
  p->fp16_scale = 0.0;
  p->device = 0;
}

lbm_status lbm_read_input(const char* path, lbm_input* out) { return read_input_file(path, out); }

lbm_status lbm_read_mask(const char* path, int nx, int ny, int nz, int decbin, uint8_t* mask_out) {
  return read_mask_file(path, nx, ny, nz, decbin, mask_out);
}

lbm_status lbm_create(const lbm_params* p, const uint8_t* mask, int nx, int ny, int nz, lbm_handle** out) {
  if (!p || !mask || !out || nx <= 0 || ny <= 0 || nz <= 0) return fail(LBM_ERR_ARG, "lbm_create: bad argument");
  *out = nullptr;
  if ((long long)nx * ny * nz > (1LL << 31) - 1) return fail(LBM_ERR_ARG, "lbm_create: grid exceeds 2^31 cells");
  if (!(p->nu > 0.0)) return fail(LBM_ERR_ARG, "lbm_create: viscosity must be positive");
  if (p->precision < LBM_PREC_F64 || p->precision > LBM_PREC_F64_FAST)
    return fail(LBM_ERR_ARG, "lbm_create: unknown precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
  if (p->device < 0 || p->device >= ndev) return fail(LBM_ERR_ARG, "lbm_create: bad device ordinal");
  auto h = std::make_unique<lbm_handle>();
  h->prm = *p;
  h->device = p->device;
  h->kind = store_of(p->precision);
  h->block = (p->block_size == 64 || p->block_size == 128 || p->block_size == 256 || p->block_size == 512)
                 ? p->block_size
                 : 256;
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  LBM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev0));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev1));
  const size_t ncells = (size_t)nx * ny * nz;
  h->mask.resize(ncells);
  const long long pores = copy_mask_count_pores(mask, ncells, h->mask.data());
  if (!build_mrt_constants(p->nu, &h->mrt)) return fail(LBM_ERR_ARG, "moment matrix inversion failed");
  if (h->kind == Store::F64) {
    if (!mi_pattern_matches(&h->mrt.MI[0][0]))
      return fail(LBM_ERR_STATE, "M^-1 does not have the pattern the FP64 kernel was built for; rebuild the library");
    LBM_CUDA_TRY(set_mi_constant(&h->mrt.MI[0][0], h->stream));
  }
  if (h->kind == Store::F16) {
    double sc = p->fp16_scale;
    if (!(sc > 0)) {
      const double gmax = std::fmax(std::fabs(p->gx), std::fmax(std::fabs(p->gy), std::fabs(p->gz)));
      const double target = gmax > 0 ? 10.0 * p->nu / gmax : 1024.0;
      sc = std::exp2(std::round(std::log2(target)));
      sc = std::fmin(std::fmax(sc, 1.0), 16777216.0);
    }
    h->fp16_scale = sc;
  }
  const int ord = p->ordering == LBM_ORDER_AUTO ? LBM_ORDER_REFERENCE : p->ordering;
  const bool full_window = p->window[0] < 0 && p->window[1] < 0 && p->window[2] < 0 && p->window[3] < 0 &&
                           p->window[4] < 0 && p->window[5] < 0;
  const bool on_device = ord == LBM_ORDER_REFERENCE && full_window && !bc_active(p->bc);
  if (on_device) {
    // count only; numbering and table are built on the device
    const size_t cells = ncells;
    Geometry& g = h->geo;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.count = (int)pores;
    g.npad = std::max(256, (int)(((pores + 255) / 256) * 256));
    g.porosity = (double)pores / (double)cells;
    g.window_volume = (int)cells;
    h->host_geo = false;
  } else {
    compact_reference(h->mask.data(), nx, ny, nz, &h->geo);
  }
  if (h->geo.count == 0) return fail(LBM_ERR_ARG, "geometry has no pore cells");
  if ((long long)h->geo.npad * kQ > (1LL << 31) - 1) return fail(LBM_ERR_ARG, "too many fluid nodes for int32 table");
  lbm_status st;
  if ((st = alloc_device(h.get())) != LBM_OK) return st;
  if (on_device) {
    // the indexing's scratch (5 bytes per cell) lives in the second
    // population array, which nothing reads before the first step writes it
    SetupScratch scratch;
    scratch.borrow(h->pop[1].p, h->pop[1].bytes, (long long)nx * ny * nz, h->geo.count);
    if ((st = device_index_reference(h->mask.data(), nx, ny, nz, h->geo.count, h->table.as<int32_t>(), h->geo.npad,
                                     0, h->ref_of.as<int32_t>(), scratch, h->stream)) != LBM_OK)
      return st;
    h->ordering = LBM_ORDER_REFERENCE;
    h->last_p = h->geo.count - 1;
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));  // before the scratch is freed
  } else if ((st = layout(h.get(), ord)) != LBM_OK) {
    return st;
  }
  if ((st = init_state(h.get())) != LBM_OK) return st;
  // the process's staging memory for field reads (pinned once per device)
  LBM_CUDA_TRY(stage_pool_prime());
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = h.release();
  if (p->ordering == LBM_ORDER_AUTO) {
    int o, b;
    double ml;
    st = lbm_autotune(*out, 20, &o, &b, &ml);
    if (st != LBM_OK) {
      lbm_destroy(*out);
      *out = nullptr;
      return st;
    }
  }
  return LBM_OK;
}

lbm_status lbm_create_from_input(const char* input_path, int precision, int ordering, lbm_handle** out,
                                 lbm_input* parsed_out) {
  lbm_input in;
  lbm_status st = read_input_file(input_path, &in);
  if (st != LBM_OK) return st;
  if (parsed_out) *parsed_out = in;
  if (in.nnf_module != 0) return fail(LBM_ERR_ARG, "non-Newtonian module is not supported");
  if (in.lattice_v == 1 && !(in.dx_input > 0 && in.dt_input > 0))
    return fail(LBM_ERR_ARG, "lattice_v: dx and dt must be positive");
  std::vector<uint8_t> mask((size_t)in.nx * in.ny * in.nz);
  // the geometry path is relative to the working directory, as in the reference
  st = read_mask_file(in.geometry_file, in.nx, in.ny, in.nz, in.decbin, mask.data());
  if (st != LBM_OK) return st;
  lbm_params p;
  lbm_params_default(&p);
  p.nu = in.in_vis;
  p.gx = in.gx;
  p.gy = in.gy;
  p.gz = in.gz;
  p.u_init[0] = in.inivx;
  p.u_init[1] = in.inivy;
  p.u_init[2] = in.inivz;
  p.precision = precision;
  p.ordering = ordering;
  p.perdir = in.perdir;
  // pressure / velocity faces (SP3:299-305, 318), INPUT.dat order xp, xn, yp, yn, zp, zn
  p.bc.sub_bc = in.sub_bc;
  p.bc.in_bc = in.in_bc;
  const int pre[6] = {in.pre_xp, in.pre_xn, in.pre_yp, in.pre_yn, in.pre_zp, in.pre_zn};
  const double prho[6] = {in.p_xp, in.p_xn, in.p_yp, in.p_yn, in.p_zp, in.p_zn};
  const int vel[6] = {in.vel_xp, in.vel_xn, in.vel_yp, in.vel_yn, in.vel_zp, in.vel_zn};
  const double vv[6] = {in.v_xp, in.v_xn, in.v_yp, in.v_yn, in.v_zp, in.v_zn};
  for (int f = 0; f < 6; f++) {
    p.bc.pressure[f] = pre[f];
    p.bc.rho[f] = prho[f];
    p.bc.velocity[f] = vel[f];
    p.bc.vel[f] = vv[f];
  }
  if (in.par_per_x || in.par_per_y || in.par_per_z) {
    // SP3:1005-1010: an axis without a partial window spans the whole box
    p.window[0] = in.par_per_x ? in.per_xn : 0;
    p.window[1] = in.par_per_x ? in.per_xp : in.nx - 1;
    p.window[2] = in.par_per_y ? in.per_yn : 0;
    p.window[3] = in.par_per_y ? in.per_yp : in.ny - 1;
    p.window[4] = in.par_per_z ? in.per_zn : 0;
    p.window[5] = in.par_per_z ? in.per_zp : in.nz - 1;
  }
  if ((st = lbm_create(&p, mask.data(), in.nx, in.ny, in.nz, out)) != LBM_OK) return st;
  // self-defined lattice velocity (SP3:1286-1296; lattice_v == 1 as in the
  // reference's init)
  if (in.lattice_v == 1 && (st = lbm_set_lattice(*out, in.dx_input, in.dt_input)) != LBM_OK) {
    lbm_destroy(*out);
    *out = nullptr;
  }
  return st;
}

lbm_status lbm_set_lattice(lbm_handle* h, double dx, double dt) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!(dx > 0) || !(dt > 0) || !std::isfinite(dx / dt)) return fail(LBM_ERR_ARG, "lbm_set_lattice: dx and dt must be positive");
  if (h->step != 0 || !h->given_macro) return fail(LBM_ERR_STATE, "lbm_set_lattice: call before the first step");
  MrtConstants m;
  if (!build_mrt_constants(h->prm.nu, &m, dx, dt)) return fail(LBM_ERR_ARG, "moment matrix inversion failed");
  h->lat = make_lattice(dx, dt);
  h->mrt.s_v = m.s_v;
  h->mrt.s_o = m.s_o;
  for (int k = 0; k < kQ; k++) h->mrt.S[k] = m.S[k];
  h->drop_graphs();
  if ((st = init_state(h)) != LBM_OK) return st;
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

void lbm_destroy(lbm_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
}

lbm_status lbm_step(lbm_handle* h, int nsteps) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (nsteps < 0) return fail(LBM_ERR_ARG, "lbm_step: negative step count");
  return run_steps(h, nsteps);
}

lbm_status lbm_reduce(lbm_handle* h, lbm_diag* out) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!out) return fail(LBM_ERR_ARG, "lbm_reduce: null output");
  double r[8];
  if ((st = reduce_raw(h, r, nullptr, nullptr)) != LBM_OK) return st;
  fill_diag(h, r, out);
  return LBM_OK;
}

lbm_status lbm_run_to_convergence(lbm_handle* h, double tol, int check_every, int max_steps, lbm_diag* out) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (check_every <= 0 || max_steps < 0 || !(tol > 0)) return fail(LBM_ERR_ARG, "lbm_run_to_convergence: bad argument");
  lbm_diag d{};
  double prev = 0.0;
  bool have_prev = false;
  while (h->step < max_steps) {
    const int k = (int)std::min<long long>(check_every, max_steps - h->step);
    if ((st = run_steps(h, k)) != LBM_OK) return st;
    double r[8];
    if ((st = reduce_raw(h, r, nullptr, nullptr)) != LBM_OK) return st;
    fill_diag(h, r, &d);
    if (out) *out = d;
    if (d.nan_detected) return fail(LBM_ERR_NAN, "non-finite velocity (reference: PROGRAM STOP)");
    if (d.u_max >= 10.0 && ++h->overspeed >= 5) return fail(LBM_ERR_OVERSPEED, "velocity above 10 five times");
    if (have_prev && std::fabs((prev - d.u_ave) / prev) < tol) {
      d.converged = 1;
      if (out) *out = d;
      return LBM_OK;
    }
    prev = d.u_ave;
    have_prev = true;
  }
  if (out) *out = d;
  return fail(LBM_ERR_NOT_CONVERGED, "step cap reached before the convergence tolerance");
}

lbm_status lbm_info(lbm_handle* h, int* count, double* porosity, long long* step) {
  if (!h) return fail(LBM_ERR_ARG, "null handle");
  if (count) *count = h->geo.count;
  if (porosity) *porosity = h->geo.porosity;
  if (step) *step = h->step;
  return LBM_OK;
}

lbm_status lbm_get_fields(lbm_handle* h, double* rho, double* u) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  const int n = h->geo.count, npad = h->geo.npad;
  DevBuf &rint = h->x_rint, &uint_ = h->x_uint, &rref = h->x_rref, &uref = h->x_uref;
  if (!rint.p) LBM_CUDA_TRY(rint.alloc((size_t)npad * sizeof(double)));
  if (!uint_.p) LBM_CUDA_TRY(uint_.alloc((size_t)3 * npad * sizeof(double)));
  if (!rref.p) LBM_CUDA_TRY(rref.alloc((size_t)(n + 1) * sizeof(double)));
  if (!uref.p) LBM_CUDA_TRY(uref.alloc((size_t)(n + 1) * 3 * sizeof(double)));
  double r[8];
  const double pp[3] = {h->perm_prev[0], h->perm_prev[1], h->perm_prev[2]};
  if ((st = reduce_raw(h, r, rint.as<double>(), uint_.as<double>())) != LBM_OK) return st;
  for (int i = 0; i < 3; i++) h->perm_prev[i] = pp[i];
  LBM_CUDA_TRY(cudaMemsetAsync(rref.p, 0, rref.bytes, h->stream));
  LBM_CUDA_TRY(cudaMemsetAsync(uref.p, 0, uref.bytes, h->stream));
  LBM_CUDA_TRY(launch_export_macro(rint.as<double>(), uint_.as<double>(), h->ref_of.as<int32_t>(), n, npad,
                                   rref.as<double>(), uref.as<double>(), h->stream));
  if (rho) LBM_CUDA_TRY(d2h_staged(rho, rref.p, rref.bytes, h->stream));
  if (u) LBM_CUDA_TRY(d2h_staged(u, uref.p, uref.bytes, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status lbm_get_populations(lbm_handle* h, double* f) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!f) return fail(LBM_ERR_ARG, "lbm_get_populations: null output");
  const int n = h->geo.count;
  DevBuf out;  // 152 B per node: not kept between calls
  LBM_CUDA_TRY(out.alloc((size_t)(n + 1) * kQ * sizeof(double)));
  LBM_CUDA_TRY(cudaMemsetAsync(out.p, 0, out.bytes, h->stream));
  int n_main;
  const double* bnd_f;
  if ((st = finalize_faces(h, &n_main, &bnd_f)) != LBM_OK) return st;
  LBM_CUDA_TRY(launch_export_pop(h->kind, h->pop[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n,
                                 h->geo.npad, h->fp16_scale, out.as<double>(), h->stream, n_main, bnd_f));
  LBM_CUDA_TRY(d2h_staged(f, out.p, out.bytes, h->stream));
  return LBM_OK;
}

lbm_status lbm_set_state(lbm_handle* h, const double* rho, const double* u, const double* f) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!rho || !u || !f) return fail(LBM_ERR_ARG, "lbm_set_state: null input");
  const int n = h->geo.count;
  DevBuf fin, rin, uin;
  LBM_CUDA_TRY(fin.alloc((size_t)(n + 1) * kQ * sizeof(double)));
  LBM_CUDA_TRY(rin.alloc((size_t)(n + 1) * sizeof(double)));
  LBM_CUDA_TRY(uin.alloc((size_t)(n + 1) * 3 * sizeof(double)));
  LBM_CUDA_TRY(cudaMemcpyAsync(fin.p, f, fin.bytes, cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(rin.p, rho, rin.bytes, cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(uin.p, u, uin.bytes, cudaMemcpyHostToDevice, h->stream));
  LBM_CUDA_TRY(launch_import_pop(h->kind, h->pop[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n,
                                 h->geo.npad, h->fp16_scale, fin.as<double>(), h->stream));
  LBM_CUDA_TRY(launch_import_macro(h->kind, h->rho_given.p, h->u_given.p, h->ref_of.as<int32_t>(), n, h->geo.npad,
                                   rin.as<double>(), uin.as<double>(), h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->given_macro = true;
  h->uprev_valid = false;
  return LBM_OK;
}

lbm_status lbm_export_compaction(lbm_handle* h, int32_t* coor) {
  if (!h || !coor) return fail(LBM_ERR_ARG, "lbm_export_compaction: null argument");
  ensure_host_geometry(h);
  std::memcpy(coor, h->geo.coor.data(), sizeof(int32_t) * (size_t)(h->geo.count + 1));
  return LBM_OK;
}

lbm_status lbm_export_table(lbm_handle* h, int32_t* nei_loc) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!nei_loc) return fail(LBM_ERR_ARG, "lbm_export_table: null output");
  // round-trip through the device copy so the exported table is the one the kernels read
  ensure_host_geometry(h);
  Geometry g = h->geo;
  g.src.assign((size_t)18 * g.npad, 0);
  LBM_CUDA_TRY(cudaMemcpyAsync(g.src.data(), h->table.p, sizeof(int32_t) * 18 * (size_t)g.npad, cudaMemcpyDeviceToHost,
                               h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  pull_to_push(g, nei_loc);
  return LBM_OK;
}

lbm_status lbm_last_step_ms(lbm_handle* h, double* ms) {
  if (!h || !ms) return fail(LBM_ERR_ARG, "null argument");
  *ms = h->last_ms;
  return LBM_OK;
}

lbm_status lbm_release_cached_memory(void) {
  LBM_CUDA_TRY(dev_pool_trim());
  return LBM_OK;
}

lbm_status lbm_memory(lbm_handle* h, size_t* device_bytes, double* bytes_per_lu) {
  if (!h) return fail(LBM_ERR_ARG, "null handle");
  if (device_bytes) {
    size_t b = 0;
    for (const DevBuf* d : {&h->pop[0], &h->pop[1], &h->table, &h->ref_of, &h->window, &h->rho_given, &h->u_given,
                            &h->rho_prev, &h->u_prev, &h->partials, &h->result, &h->snap[0], &h->snap[1],
                            &h->bc_ops, &h->bc_off, &h->bc_mi, &h->bnd_f, &h->ct_base, &h->ct_off})
      b += d->bytes;
    *device_bytes = b;
  }
  if (bytes_per_lu) *bytes_per_lu = 2.0 * kQ * (double)store_bytes(h->kind) + table_bytes_per_node(h);
  return LBM_OK;
}

lbm_status lbm_set_table_mode(lbm_handle* h, int compact) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (compact != 0 && compact != 1) return fail(LBM_ERR_ARG, "lbm_set_table_mode: mode must be 0 or 1");
  if (compact && !h->ct_ok && (st = build_compact_table(h)) != LBM_OK) return st;
  if (h->ct_on != (compact == 1)) h->drop_graphs();
  h->ct_on = compact == 1;
  return LBM_OK;
}

lbm_status lbm_table_info(lbm_handle* h, int* compact, double* table_bytes_per_node_out, double* wide_fraction) {
  if (!h) return fail(LBM_ERR_ARG, "null handle");
  if (wide_fraction && !h->ct_ok) {
    lbm_status st = check_handle(h);
    if (st == LBM_OK) st = build_compact_table(h);
    if (st != LBM_OK) return st;
  }
  if (compact) *compact = (h->ct_ok && h->ct_on) ? 1 : 0;
  if (table_bytes_per_node_out) *table_bytes_per_node_out = table_bytes_per_node(h);
  if (wide_fraction) *wide_fraction = h->ct_wide_frac;
  return LBM_OK;
}

lbm_status lbm_autotune(lbm_handle* h, int trial_steps, int* ordering_out, int* block_out, double* mlups_out) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (trial_steps <= 0) trial_steps = 20;
  const int n = h->geo.count;
  // save the state in reference layout (device side)
  DevBuf fsave, rsave, usave;
  LBM_CUDA_TRY(fsave.alloc((size_t)(n + 1) * kQ * sizeof(double)));
  LBM_CUDA_TRY(rsave.alloc((size_t)h->geo.npad * sizeof(double)));
  LBM_CUDA_TRY(usave.alloc((size_t)3 * h->geo.npad * sizeof(double)));
  LBM_CUDA_TRY(cudaMemsetAsync(fsave.p, 0, fsave.bytes, h->stream));
  {
    int n_main;
    const double* bnd_f;
    if ((st = finalize_faces(h, &n_main, &bnd_f)) != LBM_OK) return st;
    LBM_CUDA_TRY(launch_export_pop(h->kind, h->pop[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n,
                                   h->geo.npad, h->fp16_scale, fsave.as<double>(), h->stream, n_main, bnd_f));
  }
  DevBuf rref, uref;
  LBM_CUDA_TRY(rref.alloc((size_t)(n + 1) * sizeof(double)));
  LBM_CUDA_TRY(uref.alloc((size_t)(n + 1) * 3 * sizeof(double)));
  // With pressure/velocity faces the restored state restarts as a given one
  // (populations after the face rules plus their macro fields): the per-step
  // records the next step's rules read are overwritten by the trial steps.
  const bool given = h->given_macro || h->bc.active;
  if (given) {
    // the given macro fields are part of the state: round-trip them too
    double r[8];
    const double pp[3] = {h->perm_prev[0], h->perm_prev[1], h->perm_prev[2]};
    if ((st = reduce_raw(h, r, rsave.as<double>(), usave.as<double>())) != LBM_OK) return st;
    for (int i = 0; i < 3; i++) h->perm_prev[i] = pp[i];
    LBM_CUDA_TRY(launch_export_macro(rsave.as<double>(), usave.as<double>(), h->ref_of.as<int32_t>(), n, h->geo.npad,
                                     rref.as<double>(), uref.as<double>(), h->stream));
  }
  const long long step0 = h->step;
  const int cur0 = h->cur;
  const bool uprev0 = h->uprev_valid;
  const int orders[4] = {LBM_ORDER_REFERENCE, LBM_ORDER_MORTON, LBM_ORDER_HILBERT, LBM_ORDER_BRICK};
  const int blocks[4] = {128, 256, 512, 64};
  // every candidate once, then the three fastest again with four times the
  // steps (single short trials of near-equal candidates are at the mercy of
  // clock and power-cap noise)
  struct Cand {
    int o, b, ct;
    double ml;
  };
  std::vector<Cand> cands;
  auto time_cand = [&](const Cand& c, int steps, double* ml) -> lbm_status {
    h->block = c.b;
    h->ct_on = c.ct == 1;
    h->drop_graphs();
    h->given_macro = false;  // timing only; the state is restored below
    h->cur = 0;
    lbm_status s2;
    if ((s2 = run_steps(h, 2)) != LBM_OK) return s2;  // warm-up
    if ((s2 = run_steps(h, steps)) != LBM_OK) return s2;
    *ml = (double)n * steps / (h->last_ms * 1e3);
    return LBM_OK;
  };
  for (int oi = 0; oi < 4; oi++) {
    if ((st = layout(h, orders[oi])) != LBM_OK) return st;
    if (!h->ct_ok && (st = build_compact_table(h)) != LBM_OK) return st;
    for (int bi = 0; bi < 4; bi++)
      for (int ct = 0; ct < (h->ct_ok ? 2 : 1); ct++) {
        Cand c{orders[oi], blocks[bi], ct, 0.0};
        if ((st = time_cand(c, trial_steps, &c.ml)) != LBM_OK) return st;
        cands.push_back(c);
      }
  }
  std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.ml > y.ml; });
  if (cands.size() > 3) cands.resize(3);
  double best = -1.0;
  int best_o = h->ordering, best_b = h->block;
  bool best_ct = h->ct_on;
  for (Cand& c : cands) {
    if ((st = layout(h, c.o)) != LBM_OK) return st;
    if (c.ct == 1 && !h->ct_ok && (st = build_compact_table(h)) != LBM_OK) return st;
    if ((st = time_cand(c, 4 * trial_steps, &c.ml)) != LBM_OK) return st;
    if (c.ml > best) {
      best = c.ml;
      best_o = c.o;
      best_b = c.b;
      best_ct = c.ct == 1;
    }
  }
  if ((st = layout(h, best_o)) != LBM_OK) return st;
  if (best_ct && !h->ct_ok && (st = build_compact_table(h)) != LBM_OK) return st;
  h->block = best_b;
  h->ct_on = best_ct && h->ct_ok;
  h->drop_graphs();
  h->cur = cur0;
  LBM_CUDA_TRY(launch_import_pop(h->kind, h->pop[h->cur].p, h->table.as<int32_t>(), h->ref_of.as<int32_t>(), n,
                                 h->geo.npad, h->fp16_scale, fsave.as<double>(), h->stream));
  if (given)
    LBM_CUDA_TRY(launch_import_macro(h->kind, h->rho_given.p, h->u_given.p, h->ref_of.as<int32_t>(), n, h->geo.npad,
                                     rref.as<double>(), uref.as<double>(), h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->step = step0;
  h->given_macro = given;
  h->uprev_valid = false;
  (void)uprev0;
  if (ordering_out) *ordering_out = best_o;
  if (block_out) *block_out = best_b;
  if (mlups_out) *mlups_out = best;
  return LBM_OK;
}


// ------------------------------------------------------------ box sums
lbm_status lbm_box_sums(lbm_handle* h, int nbox, const int32_t* boxes, double* out) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (nbox < 0 || (nbox > 0 && (!boxes || !out))) return fail(LBM_ERR_ARG, "lbm_box_sums: bad argument");
  if (nbox == 0) return LBM_OK;
  if (nbox > 65535) return fail(LBM_ERR_ARG, "lbm_box_sums: at most 65535 boxes per call");
  const Geometry& g = h->geo;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  // clip to the grid; an empty box sums to zero
  std::vector<int32_t> clipped((size_t)nbox * 6);
  std::vector<int> live;
  long long cells = 0;
  for (int b = 0; b < nbox; b++) {
    const int32_t* in = boxes + (size_t)b * 6;
    const int32_t lo[3] = {std::max(in[0], 0), std::max(in[2], 0), std::max(in[4], 0)};
    const int32_t hi[3] = {std::min(in[1], nx - 1), std::min(in[3], ny - 1), std::min(in[5], nz - 1)};
    if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) continue;
    int32_t* c = &clipped[live.size() * 6];
    c[0] = lo[0]; c[1] = hi[0]; c[2] = lo[1]; c[3] = hi[1]; c[4] = lo[2]; c[5] = hi[2];
    cells += (long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    live.push_back(b);
  }
  std::memset(out, 0, sizeof(double) * 4 * (size_t)nbox);
  if (live.empty()) return LBM_OK;
  if (!h->cell_idx_valid) {
    ensure_host_geometry(h);
    std::vector<int32_t> idx((size_t)nx * ny * nz, -1);
    for (int p = 0; p < g.count; p++) {
      const int c = g.coor[g.ref_of[p]];
      const int i = c / (ny * nz), j = (c % (ny * nz)) / nz, k = c % nz;
      idx[i + (size_t)nx * (j + (size_t)ny * k)] = p;
    }
    if (h->cell_idx.bytes != idx.size() * sizeof(int32_t)) LBM_CUDA_TRY(h->cell_idx.alloc(idx.size() * sizeof(int32_t)));
    LBM_CUDA_TRY(cudaMemcpyAsync(h->cell_idx.p, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                 h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->cell_idx_valid = true;
  }
  const int nl = (int)live.size();
  const long long avg = cells / nl;
  const int chunks = (int)std::max<long long>(1, std::min<long long>(256, avg / 32768));
  DevBuf u, dboxes, partials, dout;
  LBM_CUDA_TRY(u.alloc((size_t)3 * g.npad * sizeof(double)));
  LBM_CUDA_TRY(dboxes.alloc((size_t)nl * 6 * sizeof(int32_t)));
  LBM_CUDA_TRY(partials.alloc((size_t)nl * chunks * 8 * sizeof(double)));
  LBM_CUDA_TRY(dout.alloc((size_t)nl * 4 * sizeof(double)));
  double r[8];
  if ((st = reduce_raw(h, r, nullptr, u.as<double>())) != LBM_OK) return st;
  LBM_CUDA_TRY(cudaMemcpyAsync(dboxes.p, clipped.data(), (size_t)nl * 6 * sizeof(int32_t), cudaMemcpyHostToDevice,
                               h->stream));
  LBM_CUDA_TRY(launch_box_sums(h->cell_idx.as<int32_t>(), u.as<double>(), g.npad, nx, ny, dboxes.as<int32_t>(), nl,
                               chunks, partials.as<double>(), dout.as<double>(), h->stream));
  std::vector<double> res((size_t)nl * 4);
  LBM_CUDA_TRY(cudaMemcpyAsync(res.data(), dout.p, res.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int l = 0; l < nl; l++)
    for (int i = 0; i < 4; i++) out[(size_t)live[l] * 4 + i] = res[(size_t)l * 4 + i];
  return LBM_OK;
}

// dp of the slab program's sub-volume permeabilities: whole-box length
// (SP:4844-4857, 4928-4941).
static double sp_dp(const lbm_handle* h) {
  if (h->prm.bc.in_bc == 0) return 0.0;
  const int dir = (h->prm.perdir >= 1 && h->prm.perdir <= 3) ? h->prm.perdir - 1 : 0;
  const int ext[3] = {h->geo.nx, h->geo.ny, h->geo.nz};
  const double c_s2 = h->lat.cs2, dx = h->lat.dx;
  return std::fabs(h->prm.bc.rho[2 * dir] - h->prm.bc.rho[2 * dir + 1]) * c_s2 / ext[dir] / dx;
}

lbm_status lbm_group_perm(lbm_handle* h, int ndiv, const int* n_sub, const int* size, const int* corner,
                          double* out) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (ndiv < 0 || (ndiv > 0 && (!n_sub || !size || !corner || !out))) return fail(LBM_ERR_ARG, "lbm_group_perm: bad argument");
  std::vector<int32_t> boxes;
  std::vector<int> vol;
  for (int d = 0; d < ndiv; d++) {
    if (n_sub[d] < 0 || size[d] <= 0) return fail(LBM_ERR_ARG, "lbm_group_perm: bad division");
    for (int a = 0; a < n_sub[d]; a++)
      for (int b = 0; b < n_sub[d]; b++)
        for (int c = 0; c < n_sub[d]; c++) {
          const int lo[3] = {corner[3 * d] + a * size[d], corner[3 * d + 1] + b * size[d], corner[3 * d + 2] + c * size[d]};
          for (int ax = 0; ax < 3; ax++) {
            boxes.push_back(lo[ax]);
            boxes.push_back(lo[ax] + size[d] - 1);
          }
          vol.push_back(size[d] * size[d] * size[d]);
        }
  }
  const int nbox = (int)vol.size();
  std::vector<double> sums((size_t)nbox * 4);
  if ((st = lbm_box_sums(h, nbox, boxes.data(), sums.data())) != LBM_OK) return st;
  const double dp = sp_dp(h), nu = h->prm.nu;
  const double gg[3] = {h->prm.gx, h->prm.gy, h->prm.gz};
  for (int b = 0; b < nbox; b++) {
    for (int i = 0; i < 3; i++) out[(size_t)b * 4 + i] = sums[(size_t)b * 4 + i] / (vol[b]) * (nu) / (gg[i] + dp);
    out[(size_t)b * 4 + 3] = sums[(size_t)b * 4 + 3] / vol[b];
  }
  return LBM_OK;
}

lbm_status lbm_local_perm(lbm_handle* h, double perm[3]) {
  lbm_status st = check_handle(h);
  if (st != LBM_OK) return st;
  if (!perm) return fail(LBM_ERR_ARG, "lbm_local_perm: null output");
  const Geometry& g = h->geo;
  const int x = g.nx >= 2 ? g.nx - 2 : 0;
  const int32_t box[6] = {x, x, 0, g.ny - 1, 0, g.nz - 1};
  double s[4];
  if ((st = lbm_box_sums(h, 1, box, s)) != LBM_OK) return st;
  const int* w = h->prm.window;
  const bool full = w[0] < 0 && w[1] < 0 && w[2] < 0 && w[3] < 0 && w[4] < 0 && w[5] < 0;
  const int lx = full ? g.nx : w[1] - w[0] + 1, ly = full ? g.ny : w[3] - w[2] + 1, lz = full ? g.nz : w[5] - w[4] + 1;
  const double dp = sp_dp(h), nu = h->prm.nu;
  perm[0] = s[0] / (ly * lz) * (nu) / (h->prm.gx + dp);
  perm[1] = s[1] / (lx * lz) * (nu) / (h->prm.gy + dp);
  perm[2] = s[2] / (lx * ly) * (nu) / (h->prm.gz + dp);
  return LBM_OK;
}

}  // extern "C"
