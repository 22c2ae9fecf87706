// Internal declarations shared by the host code and the CUDA kernels of
// liblbm.so.  Not part of the public ABI (include/lbm.h is).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "lbm.h"

namespace lbm {

constexpr int kQ = 19;

// ---------------------------------------------------------------- D3Q19 set
// Velocity set and opposite directions of the reference (SP3:167-180).
__host__ __device__ constexpr int cx(int q) {
  return (q == 1 || q == 7 || q == 9 || q == 15 || q == 17) ? 1
         : (q == 2 || q == 8 || q == 10 || q == 16 || q == 18) ? -1
                                                                : 0;
}
__host__ __device__ constexpr int cy(int q) {
  return (q == 3 || q == 7 || q == 8 || q == 11 || q == 13) ? 1
         : (q == 4 || q == 9 || q == 10 || q == 12 || q == 14) ? -1
                                                                 : 0;
}
__host__ __device__ constexpr int cz(int q) {
  return (q == 5 || q == 11 || q == 12 || q == 15 || q == 16) ? 1
         : (q == 6 || q == 13 || q == 14 || q == 17 || q == 18) ? -1
                                                                  : 0;
}
__host__ __device__ constexpr int opp(int q) {
  return q == 0 ? 0 : (q <= 6 ? (q % 2 ? q + 1 : q - 1) : (q <= 10 ? 17 - q : (q <= 14 ? 25 - q : 33 - q)));
}
__host__ __device__ constexpr double weight(int q) {
  return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// d'Humieres moment basis of the reference (SP3:64-83) as polynomials of the
// velocity components; row k, column q.
__host__ __device__ constexpr int mcoef(int k, int q) {
  const int x = cx(q), y = cy(q), z = cz(q);
  const int c2 = x * x + y * y + z * z;
  switch (k) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * c2 - 9) * x;
    case 5: return y;
    case 6: return (5 * c2 - 9) * y;
    case 7: return z;
    case 8: return (5 * c2 - 9) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (3 * c2 - 5) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3 * c2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    default: return (x * x - y * y) * z;
  }
}
// Squared norm of row k (rows are mutually orthogonal, so M^-1 = M^T diag(1/norm)).
__host__ __device__ constexpr int mnorm(int k) {
  int s = 0;
  for (int q = 0; q < kQ; q++) s += mcoef(k, q) * mcoef(k, q);
  return s;
}
// Opposite pairs (q, opp q) with q the first of the pair in index order.
__host__ __device__ constexpr int pair_q(int i) {
  return i == 0 ? 1 : i == 1 ? 3 : i == 2 ? 5 : i == 3 ? 7 : i == 4 ? 8 : i == 5 ? 11 : i == 6 ? 12 : i == 7 ? 15 : 16;
}
// even moments: symmetric under e -> -e; odd: antisymmetric.
__host__ __device__ constexpr bool even_moment(int k) {
  return !(k == 3 || k == 4 || k == 5 || k == 6 || k == 7 || k == 8 || k == 16 || k == 17 || k == 18);
}

// ---------------------------------------------------------------- constants
struct MrtConstants {
  double M[kQ][kQ];
  double MI[kQ][kQ];  // Gauss-Jordan inverse, bit-identical to the reference's
  double S[kQ];
  double s_v, s_o;
};
// Rates for a lattice of spacing dx and time step dt (the reference's init:
// lat_c = dx / dt, c_s2 = lat_c^2 / 3, tau = nu / (c_s2 dt) + 0.5); dx = dt = 1
// is the default lattice.
bool build_mrt_constants(double nu, MrtConstants* out, double dx = 1.0, double dt = 1.0);

// Self-defined lattice velocity (lattice_v with dx, dt; SP3:1286-1296,
// 1326-1330, 1382-1394, 1423-1500, 2414-2439): the discrete velocities are
// e lat_c, the equilibrium divides by c2 = lat_c^2 and c4 = c2^2, the Guo
// force by c_s2 and c_s2^2, the forcing enters the moments as dt F and the
// velocity as dt g / 2.  on = 0 is the default lattice (lat_c = dt = 1),
// for which the kernels keep their unit-lattice arithmetic.
struct Lattice {
  int on = 0;
  double c = 1.0;              // lat_c = dx / dt
  double ic = 1.0;             // 1 / lat_c
  double cs2 = 1.0 * 1.0 / 3;  // c_s^2 = lat_c^2 / 3
  double c2 = 1.0, c4 = 1.0;   // lat_c^2, lat_c^4 (feq)
  double dt = 1.0, dx = 1.0;
};
Lattice make_lattice(double dx, double dt);

// ---------------------------------------------------------------- geometry
struct Geometry {
  int nx = 0, ny = 0, nz = 0;
  int count = 0;                 // fluid nodes
  int npad = 0;                  // SoA stride (multiple of 256)
  double porosity = 0.0;         // over the permeability window
  std::vector<int32_t> coor;     // [count+1], ref id -> i*ny*nz + j*nz + k
  std::vector<int32_t> ref_of;   // [count], internal index -> ref id (1-based)
  std::vector<int32_t> int_of;   // [count+1], ref id -> internal index (row 0 = -1)
  std::vector<int32_t> src;      // [18][npad], pull sources (flat index q*npad + m)
  std::vector<uint8_t> in_window;// [count] internal order; empty = whole box
  int window_volume = 0;
};

// Fluid-node compaction in the reference order (SP3:1018-1071).
void compact_reference(const uint8_t* mask, int nx, int ny, int nz, Geometry* g);
// Internal ordering: fills ref_of / int_of for the requested curve.
void order_nodes(const uint8_t* mask, int ordering, Geometry* g);
// Pull table in internal order with halfway bounce-back resolved.
void build_pull_table(const uint8_t* mask, Geometry* g);
// Push table nei_loc (reference form) from the pull table.
void pull_to_push(const Geometry& g, int32_t* nei_loc);
void set_window(const int window[6], Geometry* g);

// ------------------------------------------------- pressure/velocity faces
// One boundary operation on the post-streaming populations F of a face node,
// in the reference's program order (boundary_pressure then
// boundary_velocity).  nb / nb4 are snapshot slots (internal index -
// snap_begin) of the nodes whose previous-step state the rule reads, -1 for
// none (the reference's row 0, zero).
enum BcKind : int8_t {
  kBcPressureRest = 0,    // F = f_eq(rho_b, 0)
  kBcPressureNbU = 1,     // F = f_eq(rho_b, u[nb])
  kBcPressureMoment = 2,  // F = MI (M f[nb] with m_0 = rho_b)
  kBcPressureNeq = 3,     // F = f_eq(rho_b, u[nb]) + f[nb4] - f_eq(rho[nb], u[nb])
  kBcVelocityEq = 4,      // F = f_eq(1, u_b)
  kBcVelocityNeq = 5,     // incoming q: F_q = f_eq(opp q; 1, u_b) - F_opp q + f_eq(q; 1, u_b)
  kBcVelocityNbRho = 6,   // F = f_eq(rho[nb], u_b)
};
struct BcOp {
  int8_t kind;
  int8_t face;  // INPUT.dat face index 0..5 = xp, xn, yp, yn, zp, zn (density / velocity of the rule)
  int8_t axis;  // kBcVelocityNeq: axis of the incoming test
  int8_t sign;  // kBcVelocityNeq: +1 -> q with e_axis < 0 are incoming, -1 -> e_axis > 0
  int32_t nb;
  int32_t nb4;
};
// Node classes after bc_partition, in internal order:
//   [0, snap_begin)          interior nodes (no boundary involvement)
//   [snap_begin, n_main)     nodes whose state a boundary rule reads
//   [n_main, count)          nodes a boundary rule writes (face nodes)
// The main step kernel runs over [0, n_main) and records the post-streaming
// state of [snap_begin, n_main); the boundary kernel runs over [n_main, count).
struct BcPlan {
  bool active = false;
  int n_main = 0, snap_begin = 0;
  std::vector<int32_t> op_off;  // [count - n_main + 1] CSR over boundary nodes
  std::vector<BcOp> ops;
};
bool bc_active(const lbm_boundary& bc);
// Reorders g (ref_of / int_of) into the three classes, keeping the order
// within each class, and builds the per-node operation lists.
void bc_partition(const uint8_t* mask, const lbm_boundary& bc, Geometry* g, BcPlan* plan);
// The same program without reordering: the written nodes (internal indices)
// with their operations (CSR, program order per node) and the nodes whose
// state the operations read; BcOp.nb / nb4 index snap_nodes (-1 = none).
struct BcLists {
  std::vector<int32_t> nodes, op_off, snap_nodes;
  std::vector<BcOp> ops;
};
void bc_node_lists(const lbm_boundary& bc, const Geometry& g, BcLists* out);

// Two pinned staging buffers for device -> pageable host copies; copies
// borrow them from a process-wide pool per device (transfer.cpp).
struct PinnedStage {
  static constexpr size_t kChunk = size_t(16) << 20;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  PinnedStage() = default;
  PinnedStage(const PinnedStage&) = delete;
  PinnedStage& operator=(const PinnedStage&) = delete;
  ~PinnedStage();
};
// Copies `bytes` from device memory `src` to host memory `dst` in order on
// `st` (a stream of the current device) and returns when the host copy is
// complete.
cudaError_t d2h_staged(void* dst, const void* src, size_t bytes, cudaStream_t st);
// Pins one stage for the current device if its pool has none yet (so that
// the process's first field read does not pay for it).
cudaError_t stage_pool_prime();

// Device memory of the solvers, from the current device's default memory
// pool with its release threshold raised: what a destroyed solver frees
// stays mapped in the process, and the next solver of a similar size takes
// it without new mappings.  dev_free first waits for the device to go idle,
// as cudaFree does, so that no launch in flight can still use the memory.
cudaError_t dev_alloc(void** p, size_t bytes);
void dev_free(void* p);
// Returns the memory freed solvers left in the pools to the driver.
cudaError_t dev_pool_trim();

// Mask and box of a single-phase handle (for solvers coupled to it).
const uint8_t* lbm_internal_mask(lbm_handle* h, int* nx, int* ny, int* nz);
extern "C" const uint8_t* lbm_cg_internal_mask(lbm_cg_handle* h, int* nx, int* ny, int* nz);

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
lbm_status fail(lbm_status s, const std::string& msg);

#define LBM_CUDA_TRY(expr)                                                               \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return ::lbm::fail(_e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,   \
                         std::string(#expr) + ": " + cudaGetErrorString(_e));            \
  } while (0)

// ---------------------------------------------------------------- kernels
// Storage kinds of the population arrays.
enum class Store { F64 = 0, F32 = 1, F16 = 2, F64D = 3 };

struct StepArgs {
  const void* src_pop;   // [19][npad] post-collision of the previous step
  void* dst_pop;         // [19][npad] this step's post-collision
  const int32_t* table;  // [18][npad]
  int n;                 // fluid nodes
  int npad;
  // macro input for a step that must use given rho/u (first step after init
  // or restart); null otherwise
  const void* rho_in;
  const void* u_in;      // [3][npad]
  // macro output of this step's pre-collision rho/u; null = not written
  void* rho_out;
  void* u_out;           // [3][npad]
  double gx, gy, gz;
  double s_v, s_o;
  double fp16_scale;
  // pressure/velocity faces: nodes [n_main, n) are left to the boundary
  // kernel; nodes [snap_begin, n_main) record their post-streaming state in
  // snap_dst ([23][nsnap] doubles: f_0..f_18, rho, ux, uy, uz; slot = p -
  // snap_begin).  Without faces n_main = n and snap_dst = null.
  int n_main;
  int snap_begin;
  int nsnap;
  double* snap_dst;
  // compact pull table (null = read `table`): per aligned warp of 32 nodes
  // and direction q a base node index ct_base[(q-1)*nwarps + w] (-1: the
  // warp reads `table` for q) and per node a 16-bit offset from it (0xFFFF:
  // halfway bounce-back, source opp(q)*npad + p); offsets of directions
  // 2i+1, 2i+2 share one 32-bit word, ct_off as [9][npad][2]
  const int32_t* ct_base;
  const uint16_t* ct_off;
  int nwarps;
  // lattice of the step.  The FP64 reference kernel takes g above as given
  // and does the reference's lattice arithmetic; the deviation-storage
  // kernels work in units of lat_c (g above is dt g / lat_c, the macro
  // arrays rho_in/u_in/u_out hold the velocity itself: read times 1/lat_c,
  // written times lat_c)
  Lattice lat;
};
cudaError_t launch_step(Store kind, const StepArgs& a, int block, cudaStream_t st);
// Builds the compact pull table from `table` ([18][npad], n fluid nodes);
// counts the (warp, direction) pairs left on the full table in *wide (device).
cudaError_t launch_compact_table(const int32_t* table, int n, int npad, int32_t* ct_base, uint16_t* ct_off,
                                 unsigned long long* wide, cudaStream_t st);

constexpr int kSnapRows = kQ + 4;  // per-step record of a node: f_0..f_18, rho, ux, uy, uz

// Boundary kernel: the face nodes [n_main, n) of one step (pull, rules, macro,
// record, collide) or, with bnd_f set, only the post-rule populations of the
// current state ([19][n - n_main] doubles) for reductions and exports.
struct BcArgs {
  StepArgs s;               // pops, table, macro in/out, rates, n_main, snap_begin, nsnap, snap_dst
  const double* snap_src;   // the previous step's record
  const int32_t* op_off;
  const BcOp* ops;
  const double* mi;         // [19*19] M^-1 (kBcPressureMoment)
  double face_rho[6];
  double face_u[6][3];
  double* bnd_f;            // finalize mode output, or null
};
cudaError_t launch_boundary(Store kind, const BcArgs& a, cudaStream_t st);

struct ReduceArgs {
  const void* pop;        // [19][npad] post-collision of the last step
  const int32_t* table;
  int n, npad;
  const void* rho_in;     // when the state is "given" (no step since set): use these
  const void* u_in;
  const void* u_prev;     // [3][npad] velocity one step earlier (null -> zero change)
  int last_p;             // internal index of the reference's last node (excluded from Error)
  const uint8_t* window;  // [n] or null
  double gx, gy, gz;
  double fp16_scale;
  double* rho_out;        // optional double[n] (internal order)
  double* u_out;          // optional double[3][npad]
  double* partials;       // [blocks][8]
  double* result;         // [8]
  int n_main;             // nodes [n_main, n) read their populations from bnd_f
  const double* bnd_f;    // [19][n - n_main] post-rule populations, or null
  Lattice lat;            // as StepArgs::lat (gx.. follow the same convention)
};
// result: t1, t2, t3, umax2, Qx, Qy, Qz, mass
cudaError_t launch_reduce(Store kind, const ReduceArgs& a, cudaStream_t st);
int reduce_blocks(int n);

// f[(count+1)*19] reference AoS <-> device storage
cudaError_t launch_export_pop(Store kind, const void* pop, const int32_t* table, const int32_t* ref_of,
                              int n, int npad, double fp16_scale, double* out, cudaStream_t st,
                              int n_main = 0, const double* bnd_f = nullptr);
cudaError_t launch_import_pop(Store kind, void* pop, const int32_t* table, const int32_t* ref_of, int n,
                              int npad, double fp16_scale, const double* in, cudaStream_t st);
// rho/u reference-layout doubles -> device macro arrays of the storage's type
cudaError_t launch_import_macro(Store kind, void* rho, void* u, const int32_t* ref_of, int n, int npad,
                                const double* rho_in, const double* u_in, cudaStream_t st);
cudaError_t launch_export_macro(const double* rho_int, const double* u_int, const int32_t* ref_of, int n,
                                int npad, double* rho_ref, double* u_ref, cudaStream_t st);
cudaError_t set_mi_constant(const double* mi361, cudaStream_t st);
// True when M^-1 has the zero / power-of-two pattern the bit-exact FP64
// kernel was compiled for (mi_pattern.h, generated from mrt.cpp).
bool mi_pattern_matches(const double* mi361);
// uniform post-streaming state f_q = feq[q] at every node, written through
// the inverse pull so the next step pulls exactly feq
cudaError_t launch_init_uniform(Store kind, void* pop, const int32_t* table, int n, int npad, double fp16_scale,
                                const double* feq19, cudaStream_t st);
cudaError_t launch_fill_macro(Store kind, void* rho, void* u, int n, int npad, double rho0, const double* u3,
                              cudaStream_t st);

size_t store_bytes(Store kind);

}  // namespace lbm
