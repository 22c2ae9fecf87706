// Node pool shared by lbm_batch (a fixed set of solves) and lbm_server
// (continuous batching of a request stream).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "setup.h"

namespace lbm {

void compact_reference(const uint8_t* mask, int nx, int ny, int nz, Geometry* g);
void order_nodes(const uint8_t* mask, int ordering, Geometry* g);

namespace {

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  ~Buf() { release(); }
  void release() {
    if (p) lbm::dev_free(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b) {
    release();
    bytes = b;
    return b ? lbm::dev_alloc(&p, b) : cudaSuccess;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// A solve's host-side description and layout.
struct Job {
  long long id = -1;
  std::vector<uint8_t> mask;
  int nx = 0, ny = 0, nz = 0;
  double nu = 0.1, g[3] = {0, 0, 0};
  Geometry geo;  // compaction + node order (ref_of)
  bool built = false;
  double t_submit = 0, t_admit = 0;
};

// Host part of a solve's layout.  In the reference node order the numbering
// and the table are built on the device at admission, so the host only
// counts pores; other orders are built here.
void build_job(Job* j, int ordering) {
  if (ordering == LBM_ORDER_REFERENCE) {
    const size_t cells = (size_t)j->nx * j->ny * j->nz;
    long long pores = 0;
    const uint8_t* m = j->mask.data();
    for (size_t c = 0; c < cells; c++) pores += (m[c] == 0);
    j->geo = Geometry{};
    j->geo.nx = j->nx;
    j->geo.ny = j->ny;
    j->geo.nz = j->nz;
    j->geo.count = (int)pores;
    j->geo.porosity = (double)pores / (double)cells;
  } else {
    compact_reference(j->mask.data(), j->nx, j->ny, j->nz, &j->geo);
    order_nodes(j->mask.data(), ordering, &j->geo);
  }
  j->built = true;
}

void build_jobs_parallel(std::vector<Job*>& jobs, int ordering) {
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  std::atomic<size_t> next{0};
  for (unsigned t = 0; t < std::min<size_t>(hw, jobs.size()); t++)
    th.emplace_back([&] {
      for (size_t i = next++; i < jobs.size(); i = next++)
        if (!jobs[i]->built) build_job(jobs[i], ordering);
    });
  for (auto& t : th) t.join();
}

double rate_viscous(double nu) { return 1.0 / (nu / (1.0 / 3.0) + 0.5); }

}  // namespace

struct Pool {
  Store kind = Store::F32;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, done_ev = nullptr;
  cudaEvent_t chain_ev0 = nullptr, chain_ev1 = nullptr;  // device time of each chain
  // one record per chain: stepping nodes when it was launched, its steps and
  // its device time (the graph: list, steps, per-instance check)
  struct ChainRecord {
    long long stepping_nodes;
    int steps;
    float ms;
  };
  std::vector<ChainRecord> trace;
  int cap = 0, ntiles = 0, nslots = 0;
  int block = 256, grid = 0;
  int ordering = LBM_ORDER_REFERENCE;
  double fp16_scale = 1.0;
  Buf pop[2], table, tile_inst, inst, state, partials, active_tiles, n_active, work, slot_off;
  SetupScratch setup;
  std::vector<InstParams> h_inst;
  InstState* h_state = nullptr;  // pinned
  std::vector<int> h_tile_inst;
  std::map<int, int> free_tiles;  // first tile -> length
  std::vector<std::unique_ptr<Job>> slot_job;
  std::vector<int> slot_parity;  // buffer holding a finished slot's state
  int cur = 0;
  // chain graphs per step grid (the grid follows the stepping tile count,
  // rounded up to a power of two, so a few graphs cover every pool state)
  std::map<int, std::array<cudaGraphExec_t, 2>> graphs;
  int g_chain = 0;
  double g_tol = 0;
  long long g_max = 0;
  int g_block = 0;

  ~Pool() {
    drop_graphs();
    if (h_state) cudaFreeHost(h_state);
    for (cudaEvent_t e : {ev0, ev1, done_ev, chain_ev0, chain_ev1})
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  void drop_graphs() {
    for (auto& kv : graphs)
      for (auto& g : kv.second)
        if (g) cudaGraphExecDestroy(g);
    graphs.clear();
  }

  // Step grid of a chain: one block per stepping tile, rounded up to a power
  // of two (one captured graph per grid), at most the pool's full grid.
  int chain_grid() const {
    long long tiles = 0;
    for (int i = 0; i < nslots; i++)
      if (slot_job[i] && h_state[i].active) tiles += h_inst[i].tile_end - h_inst[i].tile_begin;
    tiles = std::max(1LL, tiles);
    long long g = 1;
    while (g < tiles) g <<= 1;
    return (int)std::min<long long>(g, grid);
  }

  lbm_status init(Store k, long long cap_nodes, int slots, int blk, int dev, int order, double f16) {
    kind = k;
    device = dev;
    block = (blk == 128 || blk == 512) ? blk : 256;
    ordering = order;
    fp16_scale = f16;
    const long long c = ((cap_nodes + kTile - 1) / kTile) * kTile;
    if (c <= 0 || c * kQ > (1LL << 31) - 1) return fail(LBM_ERR_ARG, "pool capacity out of range (int32 table)");
    cap = (int)c;
    ntiles = cap / kTile;
    nslots = slots;
    LBM_CUDA_TRY(cudaSetDevice(device));
    LBM_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    LBM_CUDA_TRY(cudaEventCreate(&ev0));
    LBM_CUDA_TRY(cudaEventCreate(&ev1));
    LBM_CUDA_TRY(cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming));
    LBM_CUDA_TRY(cudaEventCreate(&chain_ev0));
    LBM_CUDA_TRY(cudaEventCreate(&chain_ev1));
    const size_t s = store_bytes(kind);
    for (auto& b : pop) LBM_CUDA_TRY(b.alloc((size_t)kQ * cap * s));
    LBM_CUDA_TRY(table.alloc((size_t)18 * cap * sizeof(int32_t)));
    LBM_CUDA_TRY(tile_inst.alloc((size_t)ntiles * sizeof(int)));
    LBM_CUDA_TRY(inst.alloc((size_t)nslots * sizeof(InstParams)));
    LBM_CUDA_TRY(state.alloc((size_t)nslots * sizeof(InstState)));
    LBM_CUDA_TRY(partials.alloc((size_t)ntiles * 8 * sizeof(double)));
    LBM_CUDA_TRY(active_tiles.alloc((size_t)ntiles * sizeof(int)));
    LBM_CUDA_TRY(work.alloc((size_t)ntiles * sizeof(TileWork)));
    LBM_CUDA_TRY(slot_off.alloc((size_t)(nslots + 1) * sizeof(int)));
    LBM_CUDA_TRY(n_active.alloc(sizeof(int)));
    LBM_CUDA_TRY(cudaMemsetAsync(n_active.p, 0, sizeof(int), stream));
    LBM_CUDA_TRY(cudaMallocHost((void**)&h_state, (size_t)nslots * sizeof(InstState)));
    std::memset(h_state, 0, (size_t)nslots * sizeof(InstState));
    h_inst.assign(nslots, InstParams{});
    h_tile_inst.assign(ntiles, -1);
    slot_job.resize(nslots);
    slot_parity.assign(nslots, 0);
    free_tiles.clear();
    free_tiles[0] = ntiles;
    LBM_CUDA_TRY(cudaMemcpyAsync(tile_inst.p, h_tile_inst.data(), (size_t)ntiles * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(state.p, h_state, (size_t)nslots * sizeof(InstState), cudaMemcpyHostToDevice,
                                 stream));
    grid = batch_step_grid(ntiles, block);
    return LBM_OK;
  }

  int alloc_tiles(int n) {
    for (auto it = free_tiles.begin(); it != free_tiles.end(); ++it)
      if (it->second >= n) {
        const int b = it->first, len = it->second;
        free_tiles.erase(it);
        if (len > n) free_tiles[b + n] = len - n;
        return b;
      }
    return -1;
  }
  void free_range(int b, int n) {
    auto it = free_tiles.emplace(b, n).first;
    auto nx = std::next(it);
    if (nx != free_tiles.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_tiles.erase(nx);
    }
    if (it != free_tiles.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_tiles.erase(it);
      }
    }
  }
  int free_slot() const {
    for (int s = 0; s < nslots; s++)
      if (!slot_job[s]) return s;
    return -1;
  }

  InstParams params_of(const Job& j, int tile0) const {
    InstParams ip{};
    ip.begin = tile0 * kTile;
    ip.end = ip.begin + j.geo.count;
    ip.tile_begin = tile0;
    ip.tile_end = tile0 + (j.geo.count + kTile - 1) / kTile;
    const double sv = rate_viscous(j.nu);
    ip.s_v = (float)sv;
    ip.s_o = (float)(8 * (2 - sv) / (8 - sv));
    for (int d = 0; d < 3; d++) {
      ip.g[d] = (float)j.g[d];
      ip.u0[d] = 0.0f;
    }
    ip.fp16_scale = (float)fp16_scale;
    ip.volume = (double)j.nx * j.ny * j.nz;
    ip.porosity = j.geo.porosity;
    ip.nu = j.nu;
    return ip;
  }

  // table rows, tile ownership, constants, fresh state and the initial
  // populations of one solve placed at tile0
  lbm_status place(int slot, int tile0) {
    Job& j = *slot_job[slot];
    const InstParams ip = params_of(j, tile0);
    h_inst[slot] = ip;
    if (ordering == LBM_ORDER_REFERENCE) {
      lbm_status st = device_index_reference(j.mask.data(), j.nx, j.ny, j.nz, j.geo.count, table.as<int32_t>(), cap,
                                             ip.begin, nullptr, setup, stream);
      if (st != LBM_OK) return st;
    } else {
      std::vector<int32_t> rows((size_t)18 * j.geo.count);
      fill_pool_rows(j.mask.data(), j.geo, cap, ip.begin, rows.data());
      for (int q = 1; q < kQ; q++)
        LBM_CUDA_TRY(cudaMemcpyAsync(table.as<int32_t>() + (size_t)(q - 1) * cap + ip.begin,
                                     rows.data() + (size_t)(q - 1) * j.geo.count, sizeof(int32_t) * j.geo.count,
                                     cudaMemcpyHostToDevice, stream));
      LBM_CUDA_TRY(cudaStreamSynchronize(stream));  // rows is a host temporary
    }
    for (int t = ip.tile_begin; t < ip.tile_end; t++) h_tile_inst[t] = slot;
    LBM_CUDA_TRY(cudaMemcpyAsync(tile_inst.as<int>() + ip.tile_begin, h_tile_inst.data() + ip.tile_begin,
                                 sizeof(int) * (ip.tile_end - ip.tile_begin), cudaMemcpyHostToDevice, stream));
    LBM_CUDA_TRY(cudaMemcpyAsync(inst.as<InstParams>() + slot, &h_inst[slot], sizeof(InstParams),
                                 cudaMemcpyHostToDevice, stream));
    LBM_CUDA_TRY(launch_batch_init(kind, pop[cur].p, table.as<int32_t>(), cap, ip.begin, j.geo.count, ip, stream));
    InstState st{};
    st.active = 1;
    st.fresh = 1;
    h_state[slot] = st;
    LBM_CUDA_TRY(cudaMemcpyAsync(state.as<InstState>() + slot, &h_state[slot], sizeof(InstState),
                                 cudaMemcpyHostToDevice, stream));
    // the pinned h_state row is the copy source: wait before it can change
    LBM_CUDA_TRY(cudaStreamSynchronize(stream));
    return LBM_OK;
  }

  lbm_status unplace(int slot) {
    const InstParams& ip = h_inst[slot];
    for (int t = ip.tile_begin; t < ip.tile_end; t++) h_tile_inst[t] = -1;
    LBM_CUDA_TRY(cudaMemcpyAsync(tile_inst.as<int>() + ip.tile_begin, h_tile_inst.data() + ip.tile_begin,
                                 sizeof(int) * (ip.tile_end - ip.tile_begin), cudaMemcpyHostToDevice, stream));
    h_state[slot] = InstState{};
    LBM_CUDA_TRY(cudaMemcpyAsync(state.as<InstState>() + slot, &h_state[slot], sizeof(InstState),
                                 cudaMemcpyHostToDevice, stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(stream));
    free_range(ip.tile_begin, ip.tile_end - ip.tile_begin);
    slot_job[slot].reset();
    return LBM_OK;
  }

  BatchStepArgs step_args(int c) const {
    BatchStepArgs a{};
    a.src_pop = pop[c].p;
    a.dst_pop = pop[1 - c].p;
    a.table = table.as<int32_t>();
    a.cap = cap;
    a.ntiles = ntiles;
    a.tile_inst = tile_inst.as<int>();
    a.inst = inst.as<InstParams>();
    a.state = state.as<InstState>();
    a.active_tiles = active_tiles.as<int>();
    a.n_active = n_active.as<int>();
    a.work = work.as<TileWork>();
    return a;
  }
  BatchReduceArgs reduce_args(int c) const {
    BatchReduceArgs r{};
    r.pop = pop[c].p;
    r.table = table.as<int32_t>();
    r.cap = cap;
    r.ntiles = ntiles;
    r.tile_inst = tile_inst.as<int>();
    r.inst = inst.as<InstParams>();
    r.state = state.as<InstState>();
    r.nslots = nslots;
    r.tile_partials = partials.as<double>();
    r.active_tiles = active_tiles.as<int>();
    r.n_active = n_active.as<int>();
    r.work = work.as<TileWork>();
    r.slot_off = slot_off.as<int>();
    return r;
  }

  lbm_status capture(int c0, int chain, double tol, long long max_steps, int step_grid, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    LBM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    // the chain starts from the current set of stepping slots (admissions and
    // retirements happen between chains)
    cudaError_t err = launch_batch_list(reduce_args(c0), step_grid, block, stream);
    int c = c0;
    for (int s = 0; s < chain && err == cudaSuccess; s++) {
      err = launch_batch_step(kind, step_args(c), block, step_grid, s, stream);
      c = 1 - c;
    }
    if (err == cudaSuccess) err = launch_batch_check(kind, reduce_args(c), chain, tol, max_steps, stream);
    const cudaError_t end = cudaStreamEndCapture(stream, &g);
    if (err != cudaSuccess || end != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(LBM_ERR_CUDA, std::string("pool graph capture: ") + cudaGetErrorString(err ? err : end));
    }
    const cudaError_t inst_e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    LBM_CUDA_TRY(inst_e);
    return LBM_OK;
  }

  // Launches one chain (check_every steps + the check) and the read-back of
  // the slot states; returns without waiting.
  lbm_status launch_chain(int chain, double tol, long long max_steps) {
    if (chain != g_chain || tol != g_tol || max_steps != g_max || block != g_block) {
      drop_graphs();
      g_chain = chain;
      g_tol = tol;
      g_max = max_steps;
      g_block = block;
    }
    const int step_grid = chain_grid();
    auto it = graphs.find(step_grid);
    if (it == graphs.end()) it = graphs.emplace(step_grid, std::array<cudaGraphExec_t, 2>{nullptr, nullptr}).first;
    cudaGraphExec_t& ge = it->second[cur];
    if (!ge) {
      lbm_status st = capture(cur, chain, tol, max_steps, step_grid, &ge);
      if (st != LBM_OK) return st;
    }
    long long stepping = 0;
    for (int i = 0; i < nslots; i++)
      if (slot_job[i] && h_state[i].active) stepping += h_inst[i].end - h_inst[i].begin;
    trace.push_back({stepping, chain, -1.f});
    LBM_CUDA_TRY(cudaEventRecord(chain_ev0, stream));
    LBM_CUDA_TRY(cudaGraphLaunch(ge, stream));
    LBM_CUDA_TRY(cudaEventRecord(chain_ev1, stream));
    cur = (chain & 1) ? 1 - cur : cur;
    LBM_CUDA_TRY(cudaMemcpyAsync(h_state, state.p, (size_t)nslots * sizeof(InstState), cudaMemcpyDeviceToHost,
                                 stream));
    LBM_CUDA_TRY(cudaEventRecord(done_ev, stream));
    return LBM_OK;
  }
  lbm_status wait_chain() {
    LBM_CUDA_TRY(cudaEventSynchronize(done_ev));
    if (!trace.empty() && trace.back().ms < 0) {
      float ms = 0;
      LBM_CUDA_TRY(cudaEventElapsedTime(&ms, chain_ev0, chain_ev1));
      trace.back().ms = ms;
    }
    return LBM_OK;
  }

  lbm_solve_result result_of(int slot) const {
    lbm_solve_result r{};
    const InstState& s = h_state[slot];
    const InstParams& ip = h_inst[slot];
    r.steps = s.steps;
    r.status = s.done == 1 ? LBM_OK : (s.done == 3 ? LBM_ERR_NAN : LBM_ERR_NOT_CONVERGED);
    r.count = ip.end - ip.begin;
    const double g[3] = {ip.g[0], ip.g[1], ip.g[2]};
    for (int d = 0; d < 3; d++) r.perm[d] = s.q[d] / ip.volume * ip.nu / g[d];
    r.u_ave = s.uave;
    r.porosity = ip.porosity;
    r.mass = s.mass;
    return r;
  }

  lbm_status export_fields(int slot, double* rho, double* u) {
    const Job& j = *slot_job[slot];
    const InstParams& ip = h_inst[slot];
    const int n = j.geo.count;
    Buf ref, r, v;
    LBM_CUDA_TRY(ref.alloc(sizeof(int32_t) * n));
    LBM_CUDA_TRY(r.alloc(sizeof(double) * (n + 1)));
    LBM_CUDA_TRY(v.alloc(sizeof(double) * 3 * (n + 1)));
    std::vector<int32_t> iota;
    const int32_t* ref_src = j.geo.ref_of.data();
    if (j.geo.ref_of.empty()) {  // reference order: internal index p is reference id p + 1
      iota.resize(n);
      for (int p = 0; p < n; p++) iota[p] = p + 1;
      ref_src = iota.data();
    }
    LBM_CUDA_TRY(cudaMemcpyAsync(ref.p, ref_src, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
    LBM_CUDA_TRY(cudaMemsetAsync(r.p, 0, r.bytes, stream));
    LBM_CUDA_TRY(cudaMemsetAsync(v.p, 0, v.bytes, stream));
    LBM_CUDA_TRY(launch_batch_export_macro(kind, pop[slot_parity[slot]].p, table.as<int32_t>(), cap, ip.begin, n,
                                           ref.as<int32_t>(), ip, r.as<double>(), v.as<double>(), stream));
    if (rho) LBM_CUDA_TRY(cudaMemcpyAsync(rho, r.p, r.bytes, cudaMemcpyDeviceToHost, stream));
    if (u) LBM_CUDA_TRY(cudaMemcpyAsync(u, v.p, v.bytes, cudaMemcpyDeviceToHost, stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(stream));
    return LBM_OK;
  }
};

Store pool_store(int precision) { return precision == LBM_PREC_F16 ? Store::F16 : Store::F32; }

double auto_fp16_scale(const lbm_instance* inst, int n) {
  double target = 1e30;
  for (int i = 0; i < n; i++) {
    const double g = std::fmax(std::fabs(inst[i].gx), std::fmax(std::fabs(inst[i].gy), std::fabs(inst[i].gz)));
    if (g > 0) target = std::fmin(target, 10.0 * inst[i].nu / g);
  }
  if (target > 1e29) target = 1024.0;
  return std::fmin(std::fmax(std::exp2(std::round(std::log2(target))), 1.0), 16777216.0);
}

lbm_status check_instance(const lbm_instance& in) {
  if (!in.mask || in.nx <= 0 || in.ny <= 0 || in.nz <= 0) return fail(LBM_ERR_ARG, "instance: bad mask or size");
  if (!(in.nu > 0)) return fail(LBM_ERR_ARG, "instance: viscosity must be positive");
  return LBM_OK;
}

std::unique_ptr<Job> job_from(const lbm_instance& in) {
  auto j = std::make_unique<Job>();
  j->nx = in.nx;
  j->ny = in.ny;
  j->nz = in.nz;
  j->mask.assign(in.mask, in.mask + (size_t)in.nx * in.ny * in.nz);
  j->nu = in.nu;
  j->g[0] = in.gx;
  j->g[1] = in.gy;
  j->g[2] = in.gz;
  return j;
}

}  // namespace lbm

using namespace lbm;

struct lbm_batch {
  Pool pool;
  int n = 0;
  std::vector<int> first_tile;
  double last_ms = 0;
  long long node_steps = 0;
  std::vector<lbm_solve_result> results;
};

struct lbm_server {
  Pool pool;
  lbm_server_config cfg{};
  std::deque<std::unique_ptr<Job>> queue;
  std::vector<lbm_server_result> finished;
  long long next_id = 1;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  bool chain_in_flight = false;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

lbm_status batch_layout(lbm_batch* b) {
  Pool& P = b->pool;
  std::vector<Job*> jobs;
  for (int i = 0; i < b->n; i++) {
    P.slot_job[i]->built = false;
    jobs.push_back(P.slot_job[i].get());
  }
  build_jobs_parallel(jobs, P.ordering);
  for (int i = 0; i < b->n; i++) {
    lbm_status st = P.place(i, b->first_tile[i]);
    if (st != LBM_OK) return st;
    P.slot_parity[i] = 0;
  }
  P.drop_graphs();
  return LBM_OK;
}

lbm_status batch_reset(lbm_batch* b) {
  Pool& P = b->pool;
  P.cur = 0;
  for (int i = 0; i < b->n; i++) {
    lbm_status st = P.place(i, b->first_tile[i]);
    if (st != LBM_OK) return st;
    P.slot_parity[i] = 0;
  }
  return LBM_OK;
}

}  // namespace

extern "C" {

lbm_status lbm_batch_create(int n, const lbm_instance* inst, int precision, int ordering, int block, int device,
                            lbm_batch** out) {
  if (n <= 0 || !inst || !out) return fail(LBM_ERR_ARG, "lbm_batch_create: bad argument");
  *out = nullptr;
  if (precision != LBM_PREC_F32 && precision != LBM_PREC_F16)
    return fail(LBM_ERR_ARG, "lbm_batch_create: precision must be F32 or F16");
  for (int i = 0; i < n; i++) {
    lbm_status st = check_instance(inst[i]);
    if (st != LBM_OK) return st;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
  auto b = std::make_unique<lbm_batch>();
  b->n = n;
  std::vector<std::unique_ptr<Job>> jobs;
  std::vector<Job*> raw;
  for (int i = 0; i < n; i++) {
    jobs.push_back(job_from(inst[i]));
    raw.push_back(jobs.back().get());
  }
  const int ord = ordering == LBM_ORDER_AUTO ? LBM_ORDER_REFERENCE : ordering;
  build_jobs_parallel(raw, ord);
  long long tiles = 0;
  for (int i = 0; i < n; i++) {
    if (jobs[i]->geo.count == 0) return fail(LBM_ERR_ARG, "instance " + std::to_string(i) + " has no pore cells");
    b->first_tile.push_back((int)tiles);
    tiles += (jobs[i]->geo.count + kTile - 1) / kTile;
  }
  lbm_status st = b->pool.init(pool_store(precision), tiles * kTile, n, block, device, ord,
                               precision == LBM_PREC_F16 ? auto_fp16_scale(inst, n) : 1.0);
  if (st != LBM_OK) return st;
  for (int i = 0; i < n; i++) {
    const int t0 = b->pool.alloc_tiles((jobs[i]->geo.count + kTile - 1) / kTile);
    if (t0 != b->first_tile[i]) return fail(LBM_ERR_STATE, "pool layout mismatch");
    b->pool.slot_job[i] = std::move(jobs[i]);
    if ((st = b->pool.place(i, t0)) != LBM_OK) return st;
  }
  b->results.resize(n);
  *out = b.release();
  if (ordering == LBM_ORDER_AUTO || block == 0) {
    int o, bl;
    double ml;
    st = lbm_batch_autotune(*out, 20, &o, &bl, &ml);
    if (st != LBM_OK) {
      lbm_batch_destroy(*out);
      *out = nullptr;
      return st;
    }
  }
  return LBM_OK;
}

lbm_status lbm_batch_run(lbm_batch* b, double tol, int check_every, long long max_steps, lbm_solve_result* results) {
  if (!b || check_every <= 0 || !(tol > 0) || max_steps <= 0) return fail(LBM_ERR_ARG, "lbm_batch_run: bad argument");
  Pool& P = b->pool;
  LBM_CUDA_TRY(cudaSetDevice(P.device));
  LBM_CUDA_TRY(cudaEventRecord(P.ev0, P.stream));
  b->node_steps = 0;
  P.trace.clear();
  std::vector<long long> before(b->n);
  for (int i = 0; i < b->n; i++) before[i] = P.h_state[i].steps;
  for (;;) {
    int active = 0;
    for (int i = 0; i < b->n; i++) active += P.h_state[i].active;
    if (!active) break;
    std::vector<int> was_active(b->n);
    for (int i = 0; i < b->n; i++) was_active[i] = P.h_state[i].active;
    lbm_status st = P.launch_chain(check_every, tol, max_steps);
    if (st != LBM_OK) return st;
    if ((st = P.wait_chain()) != LBM_OK) return st;
    // a solve that stopped in this chain keeps its last state in the buffer
    // the chain ended on; later chains skip its tiles
    for (int i = 0; i < b->n; i++)
      if (was_active[i] && !P.h_state[i].active) P.slot_parity[i] = P.cur;
  }
  LBM_CUDA_TRY(cudaEventRecord(P.ev1, P.stream));
  LBM_CUDA_TRY(cudaEventSynchronize(P.ev1));
  float ms = 0;
  LBM_CUDA_TRY(cudaEventElapsedTime(&ms, P.ev0, P.ev1));
  b->last_ms = ms;
  for (int i = 0; i < b->n; i++) {
    b->results[i] = P.result_of(i);
    b->node_steps += (P.h_state[i].steps - before[i]) * (long long)b->results[i].count;
    if (results) results[i] = b->results[i];
  }
  return LBM_OK;
}

lbm_status lbm_batch_reset(lbm_batch* b) {
  if (!b) return fail(LBM_ERR_ARG, "null batch");
  LBM_CUDA_TRY(cudaSetDevice(b->pool.device));
  return batch_reset(b);
}

lbm_status lbm_batch_get_fields(lbm_batch* b, int i, double* rho, double* u) {
  if (!b || i < 0 || i >= b->n) return fail(LBM_ERR_ARG, "lbm_batch_get_fields: bad index");
  LBM_CUDA_TRY(cudaSetDevice(b->pool.device));
  return b->pool.export_fields(i, rho, u);
}

lbm_status lbm_batch_autotune(lbm_batch* b, int trial_steps, int* ordering_out, int* block_out, double* mlups_out) {
  if (!b) return fail(LBM_ERR_ARG, "null batch");
  Pool& P = b->pool;
  LBM_CUDA_TRY(cudaSetDevice(P.device));
  if (trial_steps <= 0) trial_steps = 20;
  long long nodes = 0;
  for (int i = 0; i < b->n; i++) nodes += P.slot_job[i]->geo.count;
  const int orders[2] = {LBM_ORDER_REFERENCE, LBM_ORDER_HILBERT};
  const int blocks[3] = {128, 256, 512};
  double best = -1;
  int best_o = P.ordering, best_b = P.block;
  lbm_status st;
  for (int o : orders) {
    P.ordering = o;
    if ((st = batch_layout(b)) != LBM_OK) return st;
    for (int bl : blocks) {
      P.block = bl;
      P.grid = batch_step_grid(P.ntiles, bl);
      if ((st = batch_reset(b)) != LBM_OK) return st;
      LBM_CUDA_TRY(launch_batch_list(P.reduce_args(P.cur), P.grid, P.block, P.stream));
      for (int s = 0; s < 2; s++) {  // warm-up
        LBM_CUDA_TRY(launch_batch_step(P.kind, P.step_args(P.cur), P.block, P.grid, s, P.stream));
        P.cur = 1 - P.cur;
      }
      LBM_CUDA_TRY(cudaEventRecord(P.ev0, P.stream));
      for (int s = 0; s < trial_steps; s++) {
        LBM_CUDA_TRY(launch_batch_step(P.kind, P.step_args(P.cur), P.block, P.grid, 1, P.stream));
        P.cur = 1 - P.cur;
      }
      LBM_CUDA_TRY(cudaEventRecord(P.ev1, P.stream));
      LBM_CUDA_TRY(cudaEventSynchronize(P.ev1));
      float ms = 0;
      LBM_CUDA_TRY(cudaEventElapsedTime(&ms, P.ev0, P.ev1));
      const double ml = (double)nodes * trial_steps / (ms * 1e3);
      if (ml > best) {
        best = ml;
        best_o = o;
        best_b = bl;
      }
    }
  }
  P.ordering = best_o;
  P.block = best_b;
  P.grid = batch_step_grid(P.ntiles, best_b);
  if ((st = batch_layout(b)) != LBM_OK) return st;
  if ((st = batch_reset(b)) != LBM_OK) return st;
  P.drop_graphs();
  if (ordering_out) *ordering_out = best_o;
  if (block_out) *block_out = best_b;
  if (mlups_out) *mlups_out = best;
  return LBM_OK;
}

lbm_status lbm_batch_trace(lbm_batch* b, double* out, int max_rows, int* n_rows) {
  if (!b || max_rows < 0 || (max_rows > 0 && !out)) return fail(LBM_ERR_ARG, "lbm_batch_trace: bad argument");
  const auto& t = b->pool.trace;
  const int n = (int)std::min<size_t>(t.size(), (size_t)max_rows);
  for (int i = 0; i < n; i++) {
    out[3 * i] = (double)t[i].stepping_nodes;
    out[3 * i + 1] = t[i].steps;
    out[3 * i + 2] = t[i].ms;
  }
  if (n_rows) *n_rows = (int)t.size();
  return LBM_OK;
}

lbm_status lbm_batch_info(lbm_batch* b, long long* total_nodes, double* last_run_ms, long long* node_steps) {
  if (!b) return fail(LBM_ERR_ARG, "null batch");
  if (total_nodes) {
    long long t = 0;
    for (int i = 0; i < b->n; i++) t += b->pool.slot_job[i]->geo.count;
    *total_nodes = t;
  }
  if (last_run_ms) *last_run_ms = b->last_ms;
  if (node_steps) *node_steps = b->node_steps;
  return LBM_OK;
}

void lbm_batch_destroy(lbm_batch* b) {
  if (!b) return;
  cudaSetDevice(b->pool.device);
  if (b->pool.stream) cudaStreamSynchronize(b->pool.stream);
  delete b;
}

// ------------------------------------------------------------------ server

void lbm_server_config_default(lbm_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->capacity_nodes = 64LL * 1024 * 1024;
  c->max_active = 256;
  c->precision = LBM_PREC_F32;
  c->ordering = LBM_ORDER_REFERENCE;
  c->block = 256;
  c->tol = 1e-6;
  c->check_every = 100;
  c->max_steps = 1000000;
  c->device = 0;
}

lbm_status lbm_server_create(const lbm_server_config* c, lbm_server** out) {
  if (!c || !out || c->max_active <= 0 || c->check_every <= 0 || !(c->tol > 0))
    return fail(LBM_ERR_ARG, "lbm_server_create: bad config");
  if (c->policy != LBM_SERVE_FIFO && c->policy != LBM_SERVE_SHORTEST_FIRST)
    return fail(LBM_ERR_ARG, "lbm_server_create: unknown admission policy");
  *out = nullptr;
  if (c->precision != LBM_PREC_F32 && c->precision != LBM_PREC_F16)
    return fail(LBM_ERR_ARG, "lbm_server_create: precision must be F32 or F16");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
  auto s = std::make_unique<lbm_server>();
  s->cfg = *c;
  const int ord = c->ordering == LBM_ORDER_AUTO ? LBM_ORDER_REFERENCE : c->ordering;
  lbm_status st = s->pool.init(pool_store(c->precision), c->capacity_nodes, c->max_active, c->block, c->device, ord,
                               c->precision == LBM_PREC_F16 ? 1048576.0 : 1.0);
  if (st != LBM_OK) return st;
  *out = s.release();
  return LBM_OK;
}

lbm_status lbm_server_submit(lbm_server* s, const lbm_instance* req, long long* request_id) {
  if (!s || !req) return fail(LBM_ERR_ARG, "lbm_server_submit: null argument");
  lbm_status st = check_instance(*req);
  if (st != LBM_OK) return st;
  long long pores = 0;
  const size_t cells = (size_t)req->nx * req->ny * req->nz;
  for (size_t i = 0; i < cells; i++) pores += req->mask[i] == 0;
  if (pores == 0) return fail(LBM_ERR_ARG, "request has no pore cells");
  if ((pores + kTile - 1) / kTile > s->pool.ntiles)
    return fail(LBM_ERR_ARG, "request needs more nodes than the whole pool holds");
  auto j = job_from(*req);
  j->id = s->next_id++;
  j->t_submit = s->now();
  if (request_id) *request_id = j->id;
  s->queue.push_back(std::move(j));
  return LBM_OK;
}

lbm_status lbm_server_pump(lbm_server* s, int* n_active, int* n_queued) {
  if (!s) return fail(LBM_ERR_ARG, "null server");
  Pool& P = s->pool;
  LBM_CUDA_TRY(cudaSetDevice(P.device));
  lbm_status st;
  int active = 0;
  for (int i = 0; i < P.nslots; i++) active += (P.slot_job[i] && P.h_state[i].active);
  // 1. resident solves advance one chain on the device ...
  if (active) {
    if ((st = P.launch_chain(s->cfg.check_every, s->cfg.tol, s->cfg.max_steps)) != LBM_OK) return st;
  }
  // 2. ... while the host builds the layouts of waiting requests
  {
    std::vector<Job*> todo;
    long long budget = (long long)P.cap;
    for (auto& j : s->queue) {
      if (budget <= 0) break;
      if (!j->built) todo.push_back(j.get());
      budget -= (long long)j->nx * j->ny * j->nz;
    }
    build_jobs_parallel(todo, P.ordering);
  }
  if (active) {
    if ((st = P.wait_chain()) != LBM_OK) return st;
    // 3. retire finished solves and free their nodes
    for (int i = 0; i < P.nslots; i++) {
      if (!P.slot_job[i] || P.h_state[i].active || !P.h_state[i].done) continue;
      lbm_server_result r{};
      r.request_id = P.slot_job[i]->id;
      r.result = P.result_of(i);
      r.t_submit = P.slot_job[i]->t_submit;
      r.t_admit = P.slot_job[i]->t_admit;
      r.t_done = s->now();
      s->finished.push_back(r);
      if ((st = P.unplace(i)) != LBM_OK) return st;
    }
  }
  // 4. admit waiting requests while slots, contiguous nodes and the
  //    saturation target allow
  long long resident = 0;
  for (int i = 0; i < P.nslots; i++)
    if (P.slot_job[i]) resident += P.slot_job[i]->geo.count;
  if (s->cfg.policy == LBM_SERVE_SHORTEST_FIRST) {
    // estimated work = cells x (extent along x)^2: the steps to the stop
    // test grow with the square of the length the flow develops over
    auto work = [](const std::unique_ptr<Job>& j) { return (double)j->nx * j->ny * j->nz * j->nx * (double)j->nx; };
    std::stable_sort(s->queue.begin(), s->queue.end(),
                     [&](const std::unique_ptr<Job>& a, const std::unique_ptr<Job>& b) { return work(a) < work(b); });
  }
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Job& j = **it;
    if (!j.built) build_job(&j, P.ordering);
    if (s->cfg.target_active_nodes > 0 && resident > 0 && resident + j.geo.count > s->cfg.target_active_nodes)
      break;  // in queue order: later requests wait too
    const int slot = P.free_slot();
    if (slot < 0) break;
    const int t0 = P.alloc_tiles((j.geo.count + kTile - 1) / kTile);
    if (t0 < 0) {
      ++it;  // skip ahead: a smaller request behind may fit
      continue;
    }
    j.t_admit = s->now();
    resident += j.geo.count;
    P.slot_job[slot] = std::move(*it);
    it = s->queue.erase(it);
    if ((st = P.place(slot, t0)) != LBM_OK) return st;
  }
  if (n_active) {
    int a = 0;
    for (int i = 0; i < P.nslots; i++) a += (P.slot_job[i] != nullptr);
    *n_active = a;
  }
  if (n_queued) *n_queued = (int)s->queue.size();
  return LBM_OK;
}

lbm_status lbm_server_poll(lbm_server* s, lbm_server_result* out, int max, int* n_out) {
  if (!s || (!out && max > 0)) return fail(LBM_ERR_ARG, "lbm_server_poll: bad argument");
  const int n = std::min<int>(max, (int)s->finished.size());
  for (int i = 0; i < n; i++) out[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + n);
  if (n_out) *n_out = n;
  return LBM_OK;
}

double lbm_server_now(lbm_server* s) { return s ? s->now() : 0.0; }

void lbm_server_destroy(lbm_server* s) {
  if (!s) return;
  cudaSetDevice(s->pool.device);
  if (s->pool.stream) cudaStreamSynchronize(s->pool.stream);
  delete s;
}

}  // extern "C"
