// C ABI of the D3Q7 solute solver (lbm_st7_*) and the flow -> solute
// velocity file of the reference.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "st7_api.h"

namespace lbm {
namespace {

struct Mem {
  void* p = nullptr;
  size_t bytes = 0;
  ~Mem() {
    if (p) lbm::dev_free(p);
  }
  cudaError_t alloc(size_t b) {
    if (p) lbm::dev_free(p);
    p = nullptr;
    bytes = b;
    return b ? lbm::dev_alloc(&p, b) : cudaSuccess;
  }
};

// Slab-solver ids at one rank run over pore cells with i outer, k fastest
// (SP:1168-1180), i.e. ascending coor = i*ny*nz + j*nz + k.  Returns, for each
// slab id s (0-based), the library's reference id (1-based).
std::vector<int32_t> slab_to_reference(const Geometry& g) {
  std::vector<int32_t> ids(g.count);
  std::iota(ids.begin(), ids.end(), 1);
  std::sort(ids.begin(), ids.end(), [&](int32_t a, int32_t b) { return g.coor[a] < g.coor[b]; });
  return ids;
}

}  // namespace

lbm_status read_st7_input_file(const char* path, lbm_st7_input* o);

}  // namespace lbm

using namespace lbm;

struct lbm_st7_handle {
  lbm_st7_params prm{};
  bool f64 = true;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Geometry geo;
  Mem g[2], table, u, c0, ref_of;
  int cur = 0;
  bool given = true;
  long long step = 0;
  double tau_s = 1.0;
  double c2 = 1.0, c4 = 1.0;  // lat_c^2, lat_c^4 (lattice_v)
  double last_ms = 0;
  int nq = 7;  // 7: D3Q7 solute program, 19: D3Q19 solute program
  ~lbm_st7_handle() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

St7Args st7_args(lbm_st7_handle* h, bool given) {
  St7Args a{};
  a.src = h->g[h->cur].p;
  a.dst = h->g[1 - h->cur].p;
  a.table = static_cast<const int32_t*>(h->table.p);
  a.u = h->u.p;
  a.c_given = given ? h->c0.p : nullptr;
  a.n = h->geo.count;
  a.npad = h->geo.npad;
  a.tau_s = h->tau_s;
  a.c2 = h->c2;
  a.c4 = h->c4;
  a.nq = h->nq;
  return a;
}

template <typename T>
std::vector<T> to_type(const std::vector<double>& v) {
  return std::vector<T>(v.begin(), v.end());
}

lbm_status upload_as(lbm_st7_handle* h, Mem& m, const std::vector<double>& v) {
  if (h->f64) {
    LBM_CUDA_TRY(cudaMemcpyAsync(m.p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<float> f = to_type<float>(v);
    LBM_CUDA_TRY(cudaMemcpyAsync(m.p, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice, h->stream));
    LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return LBM_OK;
}

}  // namespace

namespace {

lbm_status create_solute(const lbm_st7_params* p, const uint8_t* mask, int nx, int ny, int nz, const double* u_nodes,
                         const double* c0, int nq, lbm_st7_handle** out) {
  if (!p || !mask || !u_nodes || !c0 || !out || nx <= 0 || ny <= 0 || nz <= 0)
    return fail(LBM_ERR_ARG, "lbm_st7_create: bad argument");
  *out = nullptr;
  if (!(p->diffusivity > 0)) return fail(LBM_ERR_ARG, "lbm_st7_create: diffusivity must be positive");
  if (p->precision != LBM_PREC_F64 && p->precision != LBM_PREC_F32)
    return fail(LBM_ERR_ARG, "lbm_st7_create: precision must be F64 or F32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
  auto h = std::make_unique<lbm_st7_handle>();
  h->prm = *p;
  h->nq = nq;
  h->f64 = p->precision == LBM_PREC_F64;
  h->device = p->device;
  const double c_s2 = 1.0 * 1.0 / 3, dt = 1.0;
  h->tau_s = p->diffusivity / (c_s2 * dt) + 0.5;  // ST7:1262
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  LBM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev0));
  LBM_CUDA_TRY(cudaEventCreate(&h->ev1));
  Geometry& g = h->geo;
  compact_reference(mask, nx, ny, nz, &g);
  if (g.count == 0) return fail(LBM_ERR_ARG, "geometry has no pore cells");
  order_nodes(mask, LBM_ORDER_REFERENCE, &g);
  build_pull_table(mask, &g);
  const int n = g.count, npad = g.npad;
  const size_t s = h->f64 ? 8 : 4;
  const int rows = nq == kQ ? kQ : 6;  // D3Q7 keeps only directions 1..6
  for (auto& b : h->g) LBM_CUDA_TRY(b.alloc((size_t)rows * npad * s));
  LBM_CUDA_TRY(h->table.alloc((size_t)18 * npad * sizeof(int32_t)));
  LBM_CUDA_TRY(h->u.alloc((size_t)3 * npad * s));
  LBM_CUDA_TRY(h->c0.alloc((size_t)npad * s));
  LBM_CUDA_TRY(h->ref_of.alloc((size_t)n * sizeof(int32_t)));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->table.p, g.src.data(), sizeof(int32_t) * 18 * (size_t)npad, cudaMemcpyHostToDevice,
                               h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(h->ref_of.p, g.ref_of.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->stream));
  std::vector<double> uu((size_t)3 * npad, 0.0), cc((size_t)npad, 0.0);
  for (int x = 0; x < n; x++) {
    const int r = g.ref_of[x];
    for (int d = 0; d < 3; d++) uu[(size_t)d * npad + x] = u_nodes[(size_t)r * 3 + d];
    const int c = g.coor[r];
    const int i = c / (ny * nz), j = (c % (ny * nz)) / nz, k = c % nz;
    cc[x] = c0[i + (size_t)nx * (j + (size_t)ny * k)];
  }
  lbm_status st;
  if ((st = upload_as(h.get(), h->u, uu)) != LBM_OK) return st;
  if ((st = upload_as(h.get(), h->c0, cc)) != LBM_OK) return st;
  LBM_CUDA_TRY(cudaMemsetAsync(h->g[0].p, 0, h->g[0].bytes, h->stream));
  St7Args a = st7_args(h.get(), true);
  a.dst = h->g[0].p;  // the initial state is the pre-image of the first pull
  LBM_CUDA_TRY(st7_launch_init(h->f64, a, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = h.release();
  return LBM_OK;
}

lbm_status create_solute_from_flow(const lbm_st7_params* p, lbm_handle* flow, const double* c0, int nq,
                                   lbm_st7_handle** out) {
  if (!flow) return fail(LBM_ERR_ARG, "lbm_st7_create_from_flow: null flow handle");
  int count = 0;
  double por = 0;
  long long step = 0;
  lbm_status st = lbm_info(flow, &count, &por, &step);
  if (st != LBM_OK) return st;
  std::vector<double> u((size_t)(count + 1) * 3);
  if ((st = lbm_get_fields(flow, nullptr, u.data())) != LBM_OK) return st;
  int nx, ny, nz;
  const uint8_t* mask = lbm_internal_mask(flow, &nx, &ny, &nz);
  return create_solute(p, mask, nx, ny, nz, u.data(), c0, nq, out);
}

}  // namespace

extern "C" {

lbm_status lbm_st7_create(const lbm_st7_params* p, const uint8_t* mask, int nx, int ny, int nz, const double* u_nodes,
                          const double* c0, lbm_st7_handle** out) {
  return create_solute(p, mask, nx, ny, nz, u_nodes, c0, 7, out);
}

lbm_status lbm_st7_create_from_flow(const lbm_st7_params* p, lbm_handle* flow, const double* c0,
                                    lbm_st7_handle** out) {
  return create_solute_from_flow(p, flow, c0, 7, out);
}

lbm_status lbm_st19_create(const lbm_st7_params* p, const uint8_t* mask, int nx, int ny, int nz, const double* u_nodes,
                           const double* c0, lbm_st7_handle** out) {
  return create_solute(p, mask, nx, ny, nz, u_nodes, c0, kQ, out);
}

lbm_status lbm_st19_create_from_flow(const lbm_st7_params* p, lbm_handle* flow, const double* c0,
                                     lbm_st7_handle** out) {
  return create_solute_from_flow(p, flow, c0, kQ, out);
}

int lbm_st7_directions(lbm_st7_handle* h) { return h ? h->nq : 0; }

lbm_status lbm_st7_set_lattice(lbm_st7_handle* h, double dx, double dt) {
  if (!h) return fail(LBM_ERR_ARG, "null solute handle");
  if (!(dx > 0) || !(dt > 0)) return fail(LBM_ERR_ARG, "lbm_st7_set_lattice: dx and dt must be positive");
  // init with lattice_v (ST7:1259-1274; ST19 the same): lat_c = dx / dt,
  // c_s^2 = lat_c^2 / 3, tau_s = niu_s / (c_s^2 dt) + 1/2; the D3Q19
  // equilibrium divides by c2 = lat_c^2 and c4 = c2^2
  const double lat_c = dx / dt;
  const double c_s2 = lat_c * lat_c / 3;
  h->tau_s = h->prm.diffusivity / (c_s2 * dt) + 0.5;
  h->c2 = lat_c * lat_c;
  h->c4 = h->c2 * h->c2;
  return LBM_OK;
}

lbm_status lbm_st7_step(lbm_st7_handle* h, int nsteps) {
  if (!h || nsteps < 0) return fail(LBM_ERR_ARG, "lbm_st7_step: bad argument");
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  LBM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  for (int s = 0; s < nsteps; s++) {
    LBM_CUDA_TRY(st7_launch_step(h->f64, st7_args(h, h->given), h->stream));
    h->cur = 1 - h->cur;
    h->given = false;
  }
  LBM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  LBM_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0;
  LBM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_ms = ms;
  h->step += nsteps;
  return LBM_OK;
}

lbm_status lbm_st7_get_concentration(lbm_st7_handle* h, double* c) {
  if (!h || !c) return fail(LBM_ERR_ARG, "lbm_st7_get_concentration: bad argument");
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  const int n = h->geo.count;
  Mem out;
  LBM_CUDA_TRY(out.alloc(sizeof(double) * (size_t)h->geo.npad));
  LBM_CUDA_TRY(st7_launch_conc(h->f64, st7_args(h, h->given), static_cast<double*>(out.p), h->stream));
  std::vector<double> tmp(n);
  LBM_CUDA_TRY(cudaMemcpyAsync(tmp.data(), out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  c[0] = 0.0;
  for (int x = 0; x < n; x++) c[h->geo.ref_of[x]] = tmp[x];
  return LBM_OK;
}

lbm_status lbm_st7_get_populations(lbm_st7_handle* h, double* g) {
  if (!h || !g) return fail(LBM_ERR_ARG, "lbm_st7_get_populations: bad argument");
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  const int n = h->geo.count;
  Mem out;
  const size_t bytes = sizeof(double) * (size_t)(n + 1) * h->nq;
  LBM_CUDA_TRY(out.alloc(bytes));
  LBM_CUDA_TRY(cudaMemsetAsync(out.p, 0, bytes, h->stream));
  LBM_CUDA_TRY(st7_launch_export(h->f64, st7_args(h, false), static_cast<const int32_t*>(h->ref_of.p),
                                 static_cast<double*>(out.p), h->stream));
  LBM_CUDA_TRY(cudaMemcpyAsync(g, out.p, bytes, cudaMemcpyDeviceToHost, h->stream));
  LBM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

lbm_status lbm_st7_set_state(lbm_st7_handle* h, const double* g, const double* c) {
  if (!h || !g || !c) return fail(LBM_ERR_ARG, "lbm_st7_set_state: bad argument");
  LBM_CUDA_TRY(cudaSetDevice(h->device));
  const int n = h->geo.count, npad = h->geo.npad;
  Mem in;
  const size_t bytes = sizeof(double) * (size_t)(n + 1) * h->nq;
  LBM_CUDA_TRY(in.alloc(bytes));
  LBM_CUDA_TRY(cudaMemcpyAsync(in.p, g, bytes, cudaMemcpyHostToDevice, h->stream));
  St7Args a = st7_args(h, true);
  a.dst = h->g[h->cur].p;  // the buffer the next step pulls from
  LBM_CUDA_TRY(st7_launch_import(h->f64, a, static_cast<const int32_t*>(h->ref_of.p), static_cast<const double*>(in.p),
                                 h->stream));
  // the first step takes C as given, like the restored rho_r of the reference
  std::vector<double> cc((size_t)npad, 0.0);
  for (int x = 0; x < n; x++) cc[x] = c[h->geo.ref_of[x]];
  lbm_status st = upload_as(h, h->c0, cc);
  if (st != LBM_OK) return st;
  h->given = true;
  return LBM_OK;
}

lbm_status lbm_st7_info(lbm_st7_handle* h, int* count, long long* step, double* last_step_ms) {
  if (!h) return fail(LBM_ERR_ARG, "null st7 handle");
  if (count) *count = h->geo.count;
  if (step) *step = h->step;
  if (last_step_ms) *last_step_ms = h->last_ms;
  return LBM_OK;
}

void lbm_st7_destroy(lbm_st7_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
}

lbm_status lbm_write_velocity_for_solute_ordered(lbm_handle* flow, const char* path, int order) {
  if (!flow || !path) return fail(LBM_ERR_ARG, "lbm_write_velocity_for_solute: null argument");
  if (order != LBM_SOLUTE_ORDER_SLAB && order != LBM_SOLUTE_ORDER_XFAST)
    return fail(LBM_ERR_ARG, "lbm_write_velocity_for_solute: unknown record order");
  int count = 0;
  double por = 0;
  long long step = 0;
  lbm_status st = lbm_info(flow, &count, &por, &step);
  if (st != LBM_OK) return st;
  std::vector<double> u((size_t)(count + 1) * 3);
  if ((st = lbm_get_fields(flow, nullptr, u.data())) != LBM_OK) return st;
  std::vector<double> out((size_t)count * 3);
  if (order == LBM_SOLUTE_ORDER_XFAST) {
    // the library's ids are the x-fastest compaction: record s is id s+1
    std::copy(u.begin() + 3, u.end(), out.begin());
  } else {
    int nx, ny, nz;
    const uint8_t* mask = lbm_internal_mask(flow, &nx, &ny, &nz);
    Geometry g;
    compact_reference(mask, nx, ny, nz, &g);
    const std::vector<int32_t> slab = slab_to_reference(g);
    for (int s = 0; s < count; s++)
      for (int d = 0; d < 3; d++) out[(size_t)s * 3 + d] = u[(size_t)slab[s] * 3 + d];
  }
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(LBM_ERR_IO, std::string("cannot write ") + path);
  const size_t w = std::fwrite(out.data(), sizeof(double), out.size(), fp);
  std::fclose(fp);
  if (w != out.size()) return fail(LBM_ERR_IO, std::string("short write to ") + path);
  return LBM_OK;
}

lbm_status lbm_write_velocity_for_solute(lbm_handle* flow, const char* path) {
  return lbm_write_velocity_for_solute_ordered(flow, path, LBM_SOLUTE_ORDER_SLAB);
}

lbm_status lbm_read_velocity_for_solute_ordered(const char* path, const uint8_t* mask, int nx, int ny, int nz,
                                                int order, double* u_nodes) {
  if (!path || !mask || !u_nodes) return fail(LBM_ERR_ARG, "lbm_read_velocity_for_solute: null argument");
  if (order != LBM_SOLUTE_ORDER_SLAB && order != LBM_SOLUTE_ORDER_XFAST)
    return fail(LBM_ERR_ARG, "lbm_read_velocity_for_solute: unknown record order");
  Geometry g;
  compact_reference(mask, nx, ny, nz, &g);
  std::vector<double> in((size_t)g.count * 3);
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(LBM_ERR_IO, std::string("file open error on ") + path);
  const size_t r = std::fread(in.data(), sizeof(double), in.size(), fp);
  std::fclose(fp);
  if (r != in.size()) return fail(LBM_ERR_FORMAT, std::string(path) + ": shorter than Count*3 doubles");
  std::memset(u_nodes, 0, sizeof(double) * 3);
  if (order == LBM_SOLUTE_ORDER_XFAST) {
    std::copy(in.begin(), in.end(), u_nodes + 3);
    return LBM_OK;
  }
  const std::vector<int32_t> slab = slab_to_reference(g);
  for (int s = 0; s < g.count; s++)
    for (int d = 0; d < 3; d++) u_nodes[(size_t)slab[s] * 3 + d] = in[(size_t)s * 3 + d];
  return LBM_OK;
}

lbm_status lbm_read_st7_input(const char* path, lbm_st7_input* out) { return read_st7_input_file(path, out); }

// x-slab decomposition of the slab programs (ST7:951-975, the same steps in
// the single-phase slab program): rank r takes the x-planes
// [first_x[r], first_x[r+1]); the cut after rank r is the plane boundary
// whose cumulative pore count is nearest to (r+1)/nranks of all pores, the
// later plane on a tie.
lbm_status lbm_slab_partition(const uint8_t* mask, int nx, int ny, int nz, int nranks, int* first_x) {
  if (!mask || !first_x || nx <= 0 || ny <= 0 || nz <= 0 || nranks <= 0)
    return fail(LBM_ERR_ARG, "lbm_slab_partition: bad argument");
  std::vector<long long> plane(nx, 0);
  long long sum = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (mask[i + (size_t)nx * (j + (size_t)ny * k)] == 0) {
          plane[i]++;
          sum++;
        }
  const double ave = (double)sum / nranks;
  first_x[0] = 0;
  for (int r = 0; r < nranks - 1; r++) {
    long long pre = 0, aft = 0;
    int ni = 0;
    while (aft < ave * (r + 1)) {
      if (ni >= nx) return fail(LBM_ERR_ARG, "lbm_slab_partition: more ranks than x-planes with pores");
      pre = aft;
      aft += plane[ni];
      ni++;
    }
    first_x[r + 1] = ((double)(aft - ave * (r + 1)) > (double)(ave * (r + 1) - pre)) ? ni - 1 : ni;
  }
  first_x[nranks] = nx;
  for (int r = 0; r < nranks; r++)
    if (first_x[r + 1] < first_x[r]) return fail(LBM_ERR_ARG, "lbm_slab_partition: empty slab");
  return LBM_OK;
}

lbm_status lbm_read_velocity_for_solute(const char* path, const uint8_t* mask, int nx, int ny, int nz,
                                        double* u_nodes) {
  return lbm_read_velocity_for_solute_ordered(path, mask, nx, ny, nz, LBM_SOLUTE_ORDER_SLAB, u_nodes);
}

}  // extern "C"
