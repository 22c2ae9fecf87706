// Host-side sparse indexing: fluid-node compaction, space-filling-curve
// orderings, pull neighbour table with halfway bounce-back, and the
// conversion back to the reference's push table.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "lbm_internal.h"

namespace lbm {

// Fluid ids in the reference order: k outer, j, i inner (x fastest), 1-based;
// coor[id] = i*ny*nz + j*nz + k (SP3:1018-1025, 1065-1071).
void compact_reference(const uint8_t* mask, int nx, int ny, int nz, Geometry* g) {
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  const long cells = (long)nx * ny * nz;
  long pores = 0;
  for (long c = 0; c < cells; c++) pores += (mask[c] == 0);
  g->count = (int)pores;
  g->coor.assign((size_t)pores + 1, 0);
  int id = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const uint8_t* row = mask + (size_t)nx * (j + (size_t)ny * k);
      for (int i = 0; i < nx; i++)
        if (row[i] == 0) g->coor[++id] = i * ny * nz + j * nz + k;
    }
  g->npad = ((g->count + 255) / 256) * 256;
  if (g->npad == 0) g->npad = 256;
  g->porosity = cells ? (double)pores / (double)cells : 0.0;
  g->window_volume = (int)cells;
}

static inline void cell_of(const Geometry& g, int id, int* i, int* j, int* k) {
  const int c = g.coor[id];
  *i = c / (g.ny * g.nz);
  *j = (c % (g.ny * g.nz)) / g.nz;
  *k = c % g.nz;
}

static inline uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

// 3-D Hilbert index by Skilling's transpose method ("Programming the Hilbert
// curve", AIP Conf. Proc. 707, 2004): axes -> transposed index -> interleave.
static uint64_t hilbert3(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Qb = M; Qb > 1; Qb >>= 1) {
    const uint32_t P = Qb - 1;
    for (int i = 0; i < 3; i++) {
      if (X[i] & Qb)
        X[0] ^= P;
      else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; i++) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Qb = M; Qb > 1; Qb >>= 1)
    if (X[2] & Qb) t ^= Qb - 1;
  for (int i = 0; i < 3; i++) X[i] ^= t;
  uint64_t h = 0;
  for (int b = bits - 1; b >= 0; b--)
    for (int i = 0; i < 3; i++) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

void order_nodes(const uint8_t* mask, int ordering, Geometry* g) {
  (void)mask;
  const int n = g->count;
  g->ref_of.resize(n);
  g->int_of.assign((size_t)n + 1, -1);
  if (ordering == LBM_ORDER_REFERENCE || n == 0) {
    for (int p = 0; p < n; p++) g->ref_of[p] = p + 1;
  } else {
    std::vector<uint64_t> key(n);
    int bits = 1;
    while ((1 << bits) < std::max(g->nx, std::max(g->ny, g->nz))) bits++;
    const int bx = 16, by = 4, bz = 4;
    const int nbx = (g->nx + bx - 1) / bx, nby = (g->ny + by - 1) / by;
    for (int id = 1; id <= n; id++) {
      int i, j, k;
      cell_of(*g, id, &i, &j, &k);
      uint64_t kk;
      if (ordering == LBM_ORDER_MORTON) {
        kk = spread3((uint64_t)i) | (spread3((uint64_t)j) << 1) | (spread3((uint64_t)k) << 2);
      } else if (ordering == LBM_ORDER_HILBERT) {
        kk = hilbert3((uint32_t)i, (uint32_t)j, (uint32_t)k, bits);
      } else {  // brick
        const uint64_t b = ((uint64_t)(k / bz) * nby + (uint64_t)(j / by)) * nbx + (uint64_t)(i / bx);
        kk = b * (uint64_t)(bx * by * bz) + (uint64_t)((k % bz) * (bx * by) + (j % by) * bx + (i % bx));
      }
      key[id - 1] = kk;
    }
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
    for (int p = 0; p < n; p++) g->ref_of[p] = idx[p] + 1;
  }
  for (int p = 0; p < n; p++) g->int_of[g->ref_of[p]] = p;
}

// Pull table: for node p and direction q >= 1 the post-streaming population
// f_q(p) is the post-collision value f*_q at the fluid cell p - e_q (periodic
// wrap on every axis, SP3:1128-1130); when that cell is solid it is the
// node's own f*_{opp q} (halfway bounce-back, SP3:1764-1771 where
// nei_loc == 0 writes F[ci][LR[mi]]).  Entries are flat indices into the
// [19][npad] population array.
void build_pull_table(const uint8_t* mask, Geometry* g) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, n = g->count, npad = g->npad;
  std::vector<int32_t> cell_id((size_t)nx * ny * nz, -1);  // x-fastest cell -> internal index
  for (int p = 0; p < n; p++) {
    int i, j, k;
    cell_of(*g, g->ref_of[p], &i, &j, &k);
    cell_id[i + (size_t)nx * (j + (size_t)ny * k)] = p;
  }
  g->src.assign((size_t)18 * npad, 0);
  for (int p = 0; p < n; p++) {
    int i, j, k;
    cell_of(*g, g->ref_of[p], &i, &j, &k);
    for (int q = 1; q < kQ; q++) {
      int ip = i - cx(q), jp = j - cy(q), kp = k - cz(q);
      if (ip < 0) ip = nx - 1;
      if (ip >= nx) ip = 0;
      if (jp < 0) jp = ny - 1;
      if (jp >= ny) jp = 0;
      if (kp < 0) kp = nz - 1;
      if (kp >= nz) kp = 0;
      const size_t c = ip + (size_t)nx * (jp + (size_t)ny * kp);
      int32_t s;
      if (mask[c] == 0)
        s = q * npad + cell_id[c];
      else
        s = opp(q) * npad + p;
      g->src[(size_t)(q - 1) * npad + p] = s;
    }
  }
  // padding lanes point at themselves in direction 0 (never launched)
  for (int q = 1; q < kQ; q++)
    for (int p = n; p < npad; p++) g->src[(size_t)(q - 1) * npad + p] = p;
}

// Inverse of build_pull_table: nei_loc[ref m][q] = ref id of m + e_q, or 0
// when that cell is solid (the reference's push form, SP3:1135-1140).
void pull_to_push(const Geometry& g, int32_t* nei) {
  const int n = g.count, npad = g.npad;
  std::memset(nei, 0, sizeof(int32_t) * (size_t)(n + 1) * kQ);
  for (int p = 0; p < n; p++) nei[(size_t)g.ref_of[p] * kQ + 0] = g.ref_of[p];
  for (int p = 0; p < n; p++)
    for (int q = 1; q < kQ; q++) {
      const int32_t s = g.src[(size_t)(q - 1) * npad + p];
      const int sq = s / npad, sm = s % npad;
      if (sq == q)  // streamed from node sm along +e_q: sm + e_q = p
        nei[(size_t)g.ref_of[sm] * kQ + q] = g.ref_of[p];
      else          // bounced: p + e_{opp q} is solid
        nei[(size_t)g.ref_of[p] * kQ + opp(q)] = 0;
    }
}

// Table rows of one pool instance: row q-1 holds, for each of its nodes p
// (internal order), the flat pool index of f_q's source: q*cap + begin + m for
// the fluid cell m = p - e_q, or opp(q)*cap + begin + p (bounce-back).
void fill_pool_rows(const uint8_t* mask, const Geometry& g, int64_t cap, int begin, int32_t* rows) {
  const int nx = g.nx, ny = g.ny, nz = g.nz, n = g.count;
  std::vector<int32_t> cell_id((size_t)nx * ny * nz, -1);
  for (int p = 0; p < n; p++) {
    int i, j, k;
    cell_of(g, g.ref_of[p], &i, &j, &k);
    cell_id[i + (size_t)nx * (j + (size_t)ny * k)] = p;
  }
  for (int p = 0; p < n; p++) {
    int i, j, k;
    cell_of(g, g.ref_of[p], &i, &j, &k);
    for (int q = 1; q < kQ; q++) {
      int ip = i - cx(q), jp = j - cy(q), kp = k - cz(q);
      ip = ip < 0 ? nx - 1 : (ip >= nx ? 0 : ip);
      jp = jp < 0 ? ny - 1 : (jp >= ny ? 0 : jp);
      kp = kp < 0 ? nz - 1 : (kp >= nz ? 0 : kp);
      const size_t c = ip + (size_t)nx * (jp + (size_t)ny * kp);
      const int64_t s = mask[c] == 0 ? (int64_t)q * cap + begin + cell_id[c] : (int64_t)opp(q) * cap + begin + p;
      rows[(size_t)(q - 1) * n + p] = (int32_t)s;
    }
  }
}

bool bc_active(const lbm_boundary& bc) {
  for (int s = 0; s < 6; s++)
    if (bc.pressure[s] == 1 || bc.velocity[s] == 1) return true;
  return false;
}

// The boundary program of one step, as boundary_pressure (SP3:2656-3116) and
// boundary_velocity (SP3:2450-2655) run it at one rank, flattened into
// per-node operation lists.  Face lists are the reference's (SP3:1164-1222):
// x faces k outer / j inner, y faces k outer / i inner, z faces j outer /
// i inner.  Kept as the reference has them:
//   - pressure Sub_BC 1, inward neighbour solid: the rest equilibrium of this
//     face's density goes to the i-th node of the y = ny-1 list (an index
//     past that list is outside the reference's array; it is dropped);
//   - pressure Sub_BC 3 takes f - f_eq from the -y neighbour on every face;
//   - velocity Sub_BC 2: x flags act on the z faces, z flags on the x faces.
namespace {

// One operation of the boundary program, nb / nb4 as reference ids (0 = none).
struct BcRaw {
  int32_t target;
  BcOp op;
};

std::vector<BcRaw> bc_program(const lbm_boundary& bc, const Geometry* g) {
  const int n = g->count;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  std::vector<int32_t> rid((size_t)nx * ny * nz, 0);  // x-fastest cell -> reference id, 0 = solid
  for (int id = 1; id <= n; id++) {
    int i, j, k;
    cell_of(*g, id, &i, &j, &k);
    rid[i + (size_t)nx * (j + (size_t)ny * k)] = id;
  }
  auto at = [&](int i, int j, int k) { return rid[i + (size_t)nx * (j + (size_t)ny * k)]; };
  // lists in slot order xn, xp, yn, yp, zn, zp
  std::vector<int32_t> list[6];
  for (int a = 0; a < nz; a++)
    for (int b = 0; b < ny; b++) {
      if (int32_t c = at(0, b, a)) list[0].push_back(c);
      if (int32_t c = at(nx - 1, b, a)) list[1].push_back(c);
    }
  for (int a = 0; a < nz; a++)
    for (int b = 0; b < nx; b++) {
      if (int32_t c = at(b, 0, a)) list[2].push_back(c);
      if (int32_t c = at(b, ny - 1, a)) list[3].push_back(c);
    }
  for (int a = 0; a < ny; a++)
    for (int b = 0; b < nx; b++) {
      if (int32_t c = at(b, a, 0)) list[4].push_back(c);
      if (int32_t c = at(b, a, nz - 1)) list[5].push_back(c);
    }
  // push neighbour id along direction q with periodic wrap (nei_loc), 0 if solid
  auto nei = [&](int32_t id, int q) {
    int i, j, k;
    cell_of(*g, id, &i, &j, &k);
    int ip = i + cx(q), jp = j + cy(q), kp = k + cz(q);
    ip = ip < 0 ? nx - 1 : (ip >= nx ? 0 : ip);
    jp = jp < 0 ? ny - 1 : (jp >= ny ? 0 : jp);
    kp = kp < 0 ? nz - 1 : (kp >= nz ? 0 : kp);
    return at(ip, jp, kp);
  };
  // INPUT face index (xp, xn, yp, yn, zp, zn) -> list slot, inward push direction
  static const int slot_of[6] = {1, 0, 3, 2, 5, 4};
  static const int dir_in[6] = {2, 1, 4, 3, 6, 5};
  std::vector<BcRaw> prog;
  auto emit = [&](int32_t target, int8_t kind, int face, int32_t nb, int32_t nb4, int axis = 0, int sign = 0) {
    prog.push_back(BcRaw{target, BcOp{kind, (int8_t)face, (int8_t)axis, (int8_t)sign, nb, nb4}});
  };
  bool any_pre = false, any_vel = false;
  for (int s = 0; s < 6; s++) {
    any_pre |= bc.pressure[s] == 1;
    any_vel |= bc.velocity[s] == 1;
  }
  const int sb = bc.sub_bc;
  if (any_pre && sb >= 0 && sb <= 3) {
    static const int order[6] = {2, 3, 0, 1, 4, 5};  // yp, yn, xp, xn, zp, zn
    for (int fc : order) {
      if (bc.pressure[fc] != 1) continue;
      const std::vector<int32_t>& L = list[slot_of[fc]];
      for (size_t i = 0; i < L.size(); i++) {
        const int32_t b = L[i], nb = nei(b, dir_in[fc]);
        if (sb == 0) {
          emit(b, kBcPressureRest, fc, 0, 0);
        } else if (nb == 0) {
          if (sb != 1)
            emit(b, kBcPressureRest, fc, 0, 0);
          else if (i < list[3].size())
            emit(list[3][i], kBcPressureRest, fc, 0, 0);
        } else if (sb == 1) {
          emit(b, kBcPressureNbU, fc, nb, 0);
        } else if (sb == 2) {
          emit(b, kBcPressureMoment, fc, nb, 0);
        } else {
          emit(b, kBcPressureNeq, fc, nb, nei(b, 4));
        }
      }
    }
  }
  if (any_vel) {
    if (sb == 0 || sb == 1) {
      static const int order[6] = {3, 2, 5, 4, 1, 0};  // yn, yp, zn, zp, xn, xp
      for (int fc : order)
        if (bc.velocity[fc] == 1)
          for (int32_t b : list[slot_of[fc]]) emit(b, kBcVelocityEq, fc, 0, 0);
    } else if (sb == 2) {
      static const int flag_of[6] = {2, 3, 0, 1, 4, 5};  // yp, yn, xp, xn, zp, zn flags
      static const int face_of[6] = {2, 3, 4, 5, 0, 1};  // ... drive yp, yn, zp, zn, xp, xn
      for (int oi = 0; oi < 6; oi++) {
        if (bc.velocity[flag_of[oi]] != 1) continue;
        const int fc = face_of[oi];
        for (int32_t b : list[slot_of[fc]]) emit(b, kBcVelocityNeq, fc, 0, 0, fc / 2, fc % 2 == 0 ? 1 : -1);
      }
    } else if (sb == 3) {
      static const int order[6] = {2, 3, 0, 1, 4, 5};  // yp, yn, xp, xn, zp, zn
      for (int fc : order)
        if (bc.velocity[fc] == 1)
          for (int32_t b : list[slot_of[fc]]) {
            const int32_t nb = nei(b, dir_in[fc]);
            if (nb != 0) emit(b, kBcVelocityNbRho, fc, nb, 0);
          }
    }
  }
  (void)n;
  return prog;
}

}  // namespace

void bc_partition(const uint8_t* mask, const lbm_boundary& bc, Geometry* g, BcPlan* plan) {
  (void)mask;
  *plan = BcPlan{};
  const int n = g->count;
  if (!bc_active(bc) || n == 0) {
    plan->n_main = plan->snap_begin = n;
    return;
  }
  plan->active = true;
  const std::vector<BcRaw> prog = bc_program(bc, g);
  // classes: 2 = written, 1 = read, 0 = neither
  std::vector<uint8_t> cls((size_t)n + 1, 0);
  for (const BcRaw& r : prog) cls[r.target] = 2;
  for (const BcRaw& r : prog) {
    if (r.op.nb > 0 && cls[r.op.nb] == 0) cls[r.op.nb] = 1;
    if (r.op.nb4 > 0 && cls[r.op.nb4] == 0) cls[r.op.nb4] = 1;
  }
  std::vector<int32_t> order;
  order.reserve(n);
  for (int c = 0; c < 3; c++)
    for (int p = 0; p < n; p++)
      if (cls[g->ref_of[p]] == c) order.push_back(g->ref_of[p]);
  int n0 = 0, n1 = 0;
  for (int id = 1; id <= n; id++) (cls[id] == 0 ? n0 : (cls[id] == 1 ? n1 : plan->n_main)) += 1;
  const int n2 = plan->n_main;
  plan->snap_begin = n0;
  plan->n_main = n0 + n1;
  g->ref_of = order;
  for (int p = 0; p < n; p++) g->int_of[g->ref_of[p]] = p;
  // per boundary node, its operations in program order
  const int nb_nodes = n2;
  plan->op_off.assign((size_t)nb_nodes + 1, 0);
  for (const BcRaw& r : prog) plan->op_off[g->int_of[r.target] - plan->n_main + 1]++;
  for (int i = 0; i < nb_nodes; i++) plan->op_off[i + 1] += plan->op_off[i];
  plan->ops.resize(prog.size());
  std::vector<int32_t> fill(plan->op_off.begin(), plan->op_off.end() - 1);
  auto slot = [&](int32_t id) { return id > 0 ? g->int_of[id] - plan->snap_begin : -1; };
  for (const BcRaw& r : prog) {
    BcOp op = r.op;
    op.nb = slot(r.op.nb);
    op.nb4 = slot(r.op.nb4);
    plan->ops[fill[g->int_of[r.target] - plan->n_main]++] = op;
  }
}

void bc_node_lists(const lbm_boundary& bc, const Geometry& g, BcLists* out) {
  *out = BcLists{};
  if (!bc_active(bc) || g.count == 0) return;
  const std::vector<BcRaw> prog = bc_program(bc, &g);
  // written nodes and read nodes, each in ascending internal index (the
  // face passes run a thread per listed node; with the colour-gradient
  // solver's node classes, bc_partition, these are consecutive runs).  Nodes
  // are independent (a rule writes its own node and reads the record), so
  // only each node's own operations keep their program order.
  std::vector<int32_t> face_of((size_t)g.count + 1, -1), snap_of((size_t)g.count + 1, -1);
  std::vector<int32_t> targets, reads;  // reference ids
  for (const BcRaw& r : prog) {
    if (face_of[r.target] < 0) {
      face_of[r.target] = 0;
      targets.push_back(r.target);
    }
    for (int32_t id : {r.op.nb, r.op.nb4})
      if (id > 0 && snap_of[id] < 0) {
        snap_of[id] = 0;
        reads.push_back(id);
      }
  }
  auto by_internal = [&](int32_t a, int32_t b) { return g.int_of[a] < g.int_of[b]; };
  std::sort(targets.begin(), targets.end(), by_internal);
  std::sort(reads.begin(), reads.end(), by_internal);
  for (size_t i = 0; i < targets.size(); i++) {
    face_of[targets[i]] = (int32_t)i;
    out->nodes.push_back(g.int_of[targets[i]]);
  }
  for (size_t i = 0; i < reads.size(); i++) {
    snap_of[reads[i]] = (int32_t)i;
    out->snap_nodes.push_back(g.int_of[reads[i]]);
  }
  const size_t nf = out->nodes.size();
  out->op_off.assign(nf + 1, 0);
  for (const BcRaw& r : prog) out->op_off[face_of[r.target] + 1]++;
  for (size_t i = 0; i < nf; i++) out->op_off[i + 1] += out->op_off[i];
  out->ops.resize(prog.size());
  std::vector<int32_t> fill(out->op_off.begin(), out->op_off.end() - 1);
  for (const BcRaw& r : prog) {
    BcOp op = r.op;
    op.nb = r.op.nb > 0 ? snap_of[r.op.nb] : -1;
    op.nb4 = r.op.nb4 > 0 ? snap_of[r.op.nb4] : -1;
    out->ops[fill[face_of[r.target]]++] = op;
  }
}

// Permeability window (per_xn..per_zp, SP3:1005-1020, 3581-3590).
void set_window(const int w[6], Geometry* g) {
  const bool full = (w[0] < 0 && w[1] < 0 && w[2] < 0 && w[3] < 0 && w[4] < 0 && w[5] < 0);
  if (full) {
    g->in_window.clear();
    g->window_volume = g->nx * g->ny * g->nz;
    return;
  }
  const int xn = w[0], xp = w[1], yn = w[2], yp = w[3], zn = w[4], zp = w[5];
  g->window_volume = (xp - xn + 1) * (yp - yn + 1) * (zp - zn + 1);
  g->in_window.assign(g->count, 0);
  long pores = 0;
  for (int p = 0; p < g->count; p++) {
    int i, j, k;
    cell_of(*g, g->ref_of[p], &i, &j, &k);
    const bool in = i >= xn && i <= xp && j >= yn && j <= yp && k >= zn && k <= zp;
    g->in_window[p] = in;
    pores += in;
  }
  g->porosity = g->window_volume > 0 ? (double)pores / (double)g->window_volume : 0.0;
}

}  // namespace lbm
