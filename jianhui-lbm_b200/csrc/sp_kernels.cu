// Single-phase fused collide + pull-stream kernels in deviation storage
// (FP32, FP16, FP64-fast) and the dispatch of every single-phase kernel.
//
// One thread owns one fluid node.  Per node and step it moves, from/to HBM:
//   18 x int32 table entries (coalesced), 19 pulled populations (gathered
//   through the table; neighbours are close in the node order), 19
//   post-collision populations (coalesced stores)
// = 2*19*s + 18*4 bytes, s = bytes per stored population.
#include "bc_kernels.cuh"

namespace lbm {

cudaError_t launch_step_f64(const StepArgs& a, int block, cudaStream_t st);
cudaError_t reduce_f64(const ReduceArgs& a, cudaStream_t st);
cudaError_t export_f64(const void*, const int32_t*, const int32_t*, int, int, double*, cudaStream_t, int,
                       const double*);
cudaError_t launch_boundary_f64(const BcArgs& a, cudaStream_t st);
cudaError_t import_f64(void*, const int32_t*, const int32_t*, int, int, const double*, cudaStream_t);
cudaError_t import_macro_f64(void*, void*, const int32_t*, int, int, const double*, const double*, cudaStream_t);

// Compact pull table: per aligned warp of 32 nodes and direction q one int32
// base node index (-1: the warp reads the int32 table for q) and per node a
// 16-bit offset from it (0xFFFF: halfway bounce-back, source opp(q)*npad +
// p), the offsets of directions 2i+1 and 2i+2 packed in one 32-bit word
// ([9][npad] words): 18*2 + 18*4/32 bytes of table per node instead of 72.
__device__ __forceinline__ size_t ct_off_index(int q, int p, int npad) {
  return (size_t)((q - 1) >> 1) * 2 * npad + 2 * (size_t)p + ((q - 1) & 1);
}

// One thread per (node, direction) row of 32 nodes: the warp's fluid sources
// in row q as a base plus 16-bit offsets, or -1 when they spread wider.
__global__ void __launch_bounds__(256) compact_table_kernel(const int32_t* __restrict__ table, int n, int npad,
                                                           int32_t* __restrict__ ct_base,
                                                           uint16_t* __restrict__ ct_off,
                                                           unsigned long long* __restrict__ wide) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;  // npad is a multiple of 256: whole warps
  const int q = blockIdx.y + 1;
  if (p >= npad) return;
  const int32_t e = table[(size_t)(q - 1) * npad + p];
  const bool live = p < n;
  const unsigned m = (unsigned)(e - q * npad);
  const bool fluid = live && m < (unsigned)npad;
  const bool bounce = live && e == opp(q) * npad + p;
  const unsigned lo = __reduce_min_sync(0xffffffffu, fluid ? m : 0xffffffffu);
  const unsigned hi = __reduce_max_sync(0xffffffffu, fluid ? m : 0u);
  const bool odd = __any_sync(0xffffffffu, live && !fluid && !bounce);
  const bool any = lo != 0xffffffffu;
  const bool too_wide = odd || (any && hi - lo > 0xFFFEu);
  const size_t w = p >> 5;
  if ((threadIdx.x & 31) == 0) {
    ct_base[(size_t)(q - 1) * (npad >> 5) + w] = too_wide ? -1 : (any ? (int32_t)lo : 0);
    if (too_wide) atomicAdd(wide, 1ull);
  }
  ct_off[ct_off_index(q, p, npad)] = (too_wide || !fluid) ? (uint16_t)0xFFFF : (uint16_t)(m - lo);
}

cudaError_t launch_compact_table(const int32_t* table, int n, int npad, int32_t* ct_base, uint16_t* ct_off,
                                 unsigned long long* wide, cudaStream_t st) {
  if (npad % 256 != 0) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(wide, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  compact_table_kernel<<<dim3(npad / 256, 18), 256, 0, st>>>(table, n, npad, ct_base, ct_off, wide);
  return cudaGetLastError();
}

// Resident blocks per SM asked of the register allocator: the FP32 step at
// 256 threads fits 5 blocks in 48 registers without spills (64 registers and
// 4 blocks otherwise): 209-211 against 214-216 us per step on the 256^3
// workload with the int32 table, 212 against 222-223 us with the compact one,
// in alternating runs on one box with the same results bit for bit.
constexpr int dev_min_blocks(Store k, int bs) { return (k == Store::F32 && bs == 256) ? 5 : 1; }

template <Store K, int BS, bool GIVEN, bool WRITE, bool CT>
__global__ void __launch_bounds__(BS, dev_min_blocks(K, BS)) step_dev_kernel(StepArgs a) {
  using T = typename Traits<K>::T;
  using A = typename Traits<K>::A;
  using Mac = typename Traits<K>::Mac;
  const int p = blockIdx.x * BS + threadIdx.x;
  // the block's warp bases of the compact table, read once into shared
  // memory; the offset words are loaded before the barrier so that their
  // latency overlaps the bases'
  __shared__ int32_t sbase[CT ? 18 : 1][CT ? BS / 32 : 1];
  uint32_t ow[CT ? 9 : 1];
  if (CT) {
    if (p < a.n_main) {
      const uint32_t* __restrict__ off = reinterpret_cast<const uint32_t*>(a.ct_off);
#pragma unroll
      for (int i = 0; i < 9; i++) ow[i] = __ldg(off + (size_t)i * a.npad + p);
    }
    for (int k = threadIdx.x; k < 18 * (BS / 32); k += BS) {
      const int qq = k / (BS / 32), w = k % (BS / 32);
      const int gw = blockIdx.x * (BS / 32) + w;
      sbase[qq][w] = gw < a.nwarps ? __ldg(a.ct_base + (size_t)qq * a.nwarps + gw) : -1;
    }
    __syncthreads();
  }
  if (p >= a.n_main) return;
  const T* __restrict__ src = static_cast<const T*>(a.src_pop);
  T* __restrict__ dst = static_cast<T*>(a.dst_pop);
  const float scale = (float)a.fp16_scale;
  const float inv_scale = (float)(1.0 / a.fp16_scale);

  A f[kQ];
  f[0] = load_pop<K>(src + p, inv_scale);
#pragma unroll
  if (CT) {
    const int wl = threadIdx.x >> 5;
#pragma unroll
    for (int q = 1; q < kQ; q++) {
      const int32_t b = sbase[q - 1][wl];
      const int o = ((q - 1) & 1) ? (int)(ow[(q - 1) >> 1] >> 16) : (int)(ow[(q - 1) >> 1] & 0xFFFFu);
      int32_t t = 0;
      if (b < 0) t = __ldg(a.table + (size_t)(q - 1) * a.npad + p);
      const int32_t c = o == 0xFFFF ? opp(q) * a.npad + p : q * a.npad + b + o;
      f[q] = load_pop<K>(src + (b < 0 ? t : c), inv_scale);
    }
  } else {
#pragma unroll
    for (int q = 1; q < kQ; q++) f[q] = load_pop<K>(src + __ldg(a.table + (size_t)(q - 1) * a.npad + p), inv_scale);
  }

  PairSplit<A> ps;
  split_pairs(f, ps);
  A drho, rho, ux, uy, uz;
  // velocities in units of lat_c (1 on the default lattice, where the
  // scalings below are exact)
  if (GIVEN) {
    const Mac* r = static_cast<const Mac*>(a.rho_in);
    const Mac* u = static_cast<const Mac*>(a.u_in);
    const A ic = A(a.lat.ic);
    rho = (A)r[p];
    drho = rho - A(1);
    ux = (A)u[p] * ic;
    uy = (A)u[a.npad + p] * ic;
    uz = (A)u[2 * a.npad + p] * ic;
  } else {
    macro_dev<A>(f, ps, A(0.5 * a.gx), A(0.5 * a.gy), A(0.5 * a.gz), drho, rho, ux, uy, uz);
  }
  if (WRITE) {
    const A c = A(a.lat.c);
    static_cast<Mac*>(a.rho_out)[p] = (Mac)rho;
    Mac* u = static_cast<Mac*>(a.u_out);
    u[p] = (Mac)(ux * c);
    u[a.npad + p] = (Mac)(uy * c);
    u[2 * a.npad + p] = (Mac)(uz * c);
  }
  if (a.snap_dst != nullptr && p >= a.snap_begin) {
    double full[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) full[q] = to_full<K>(f[q], q);
    snap_write(a.snap_dst, a.nsnap, p - a.snap_begin, full, rho, ux, uy, uz);
  }
  mrt_collide_dev<A>(f, ps, drho, rho, ux, uy, uz, A(a.gx), A(a.gy), A(a.gz), A(a.s_v), A(a.s_o));
#pragma unroll
  for (int q = 0; q < kQ; q++) store_pop<K>(dst + (size_t)q * a.npad + p, f[q], scale);
}

// Face nodes in deviation storage: the rules act on full populations in
// double, the macro step and collision are the step kernel's.
template <Store K, bool GIVEN, bool FINAL>
__global__ void __launch_bounds__(128) bc_dev_kernel(BcArgs a) {
  using T = typename Traits<K>::T;
  using A = typename Traits<K>::A;
  using Mac = typename Traits<K>::Mac;
  const int b = blockIdx.x * 128 + threadIdx.x;
  const int p = a.s.n_main + b;
  if (p >= a.s.n) return;
  const StepArgs& s = a.s;
  const T* __restrict__ src = static_cast<const T*>(s.src_pop);
  const float scale = (float)s.fp16_scale;
  const float inv_scale = (float)(1.0 / s.fp16_scale);
  double F[kQ];
  F[0] = to_full<K>(load_pop<K>(src + p, inv_scale), 0);
#pragma unroll
  for (int q = 1; q < kQ; q++)
    F[q] = to_full<K>(load_pop<K>(src + __ldg(s.table + (size_t)(q - 1) * s.npad + p), inv_scale), q);
  // the rules on the default lattice: velocities here are in units of lat_c
  if (!GIVEN) bc_apply(a, b, F, Lattice{});
  if (FINAL) {
    const size_t nb = (size_t)(s.n - s.n_main);
#pragma unroll
    for (int q = 0; q < kQ; q++) a.bnd_f[(size_t)q * nb + b] = F[q];
    return;
  }
  A f[kQ];
#pragma unroll
  for (int q = 0; q < kQ; q++) f[q] = from_full<K>(F[q], q);
  PairSplit<A> ps;
  split_pairs(f, ps);
  A drho, rho, ux, uy, uz;
  if (GIVEN) {
    const Mac* r = static_cast<const Mac*>(s.rho_in);
    const Mac* u = static_cast<const Mac*>(s.u_in);
    const A ic = A(s.lat.ic);
    rho = (A)r[p];
    drho = rho - A(1);
    ux = (A)u[p] * ic;
    uy = (A)u[s.npad + p] * ic;
    uz = (A)u[2 * s.npad + p] * ic;
  } else {
    macro_dev<A>(f, ps, A(0.5 * s.gx), A(0.5 * s.gy), A(0.5 * s.gz), drho, rho, ux, uy, uz);
  }
  if (s.rho_out != nullptr) {
    const A c = A(s.lat.c);
    static_cast<Mac*>(s.rho_out)[p] = (Mac)rho;
    Mac* u = static_cast<Mac*>(s.u_out);
    u[p] = (Mac)(ux * c);
    u[s.npad + p] = (Mac)(uy * c);
    u[2 * s.npad + p] = (Mac)(uz * c);
  }
  snap_write(s.snap_dst, s.nsnap, p - s.snap_begin, F, rho, ux, uy, uz);
  mrt_collide_dev<A>(f, ps, drho, rho, ux, uy, uz, A(s.gx), A(s.gy), A(s.gz), A(s.s_v), A(s.s_o));
  T* __restrict__ dst = static_cast<T*>(s.dst_pop);
#pragma unroll
  for (int q = 0; q < kQ; q++) store_pop<K>(dst + (size_t)q * s.npad + p, f[q], scale);
}

template <Store K>
static cudaError_t launch_bc_dev(const BcArgs& a, cudaStream_t st) {
  const int nb = a.s.n - a.s.n_main;
  if (nb <= 0) return cudaSuccess;
  const int grid = (nb + 127) / 128;
  if (a.bnd_f)
    bc_dev_kernel<K, false, true><<<grid, 128, 0, st>>>(a);
  else if (a.s.rho_in != nullptr)
    bc_dev_kernel<K, true, false><<<grid, 128, 0, st>>>(a);
  else
    bc_dev_kernel<K, false, false><<<grid, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_boundary(Store kind, const BcArgs& a, cudaStream_t st) {
  switch (kind) {
    case Store::F64: return launch_boundary_f64(a, st);
    case Store::F64D: return launch_bc_dev<Store::F64D>(a, st);
    case Store::F32: return launch_bc_dev<Store::F32>(a, st);
    case Store::F16: return launch_bc_dev<Store::F16>(a, st);
  }
  return cudaErrorInvalidValue;
}

template <Store K, int BS>
static cudaError_t launch_dev_bs(const StepArgs& a, cudaStream_t st) {
  const int grid = (a.n_main + BS - 1) / BS;
  if (grid == 0) return cudaSuccess;
  const bool given = a.rho_in != nullptr, write = a.rho_out != nullptr;
  if (a.ct_base != nullptr) {
    if (given && write)
      step_dev_kernel<K, BS, true, true, true><<<grid, BS, 0, st>>>(a);
    else if (given)
      step_dev_kernel<K, BS, true, false, true><<<grid, BS, 0, st>>>(a);
    else if (write)
      step_dev_kernel<K, BS, false, true, true><<<grid, BS, 0, st>>>(a);
    else
      step_dev_kernel<K, BS, false, false, true><<<grid, BS, 0, st>>>(a);
  } else {
    if (given && write)
      step_dev_kernel<K, BS, true, true, false><<<grid, BS, 0, st>>>(a);
    else if (given)
      step_dev_kernel<K, BS, true, false, false><<<grid, BS, 0, st>>>(a);
    else if (write)
      step_dev_kernel<K, BS, false, true, false><<<grid, BS, 0, st>>>(a);
    else
      step_dev_kernel<K, BS, false, false, false><<<grid, BS, 0, st>>>(a);
  }
  return cudaGetLastError();
}

template <Store K>
static cudaError_t launch_dev(const StepArgs& a, int block, cudaStream_t st) {
  switch (block) {
    case 64: return launch_dev_bs<K, 64>(a, st);
    case 128: return launch_dev_bs<K, 128>(a, st);
    case 512: return launch_dev_bs<K, 512>(a, st);
    default: return launch_dev_bs<K, 256>(a, st);
  }
}

cudaError_t launch_step(Store kind, const StepArgs& a, int block, cudaStream_t st) {
  switch (kind) {
    case Store::F64: return launch_step_f64(a, block, st);
    case Store::F64D: return launch_dev<Store::F64D>(a, block, st);
    case Store::F32: return launch_dev<Store::F32>(a, block, st);
    case Store::F16: return launch_dev<Store::F16>(a, block, st);
  }
  return cudaErrorInvalidValue;
}

int reduce_blocks(int n) {
  const int b = (n + kReduceThreads - 1) / kReduceThreads;
  return b < 1 ? 1 : (b > 148 * 4 ? 148 * 4 : b);
}

cudaError_t launch_reduce(Store kind, const ReduceArgs& a, cudaStream_t st) {
  switch (kind) {
    case Store::F64: return reduce_f64(a, st);
    case Store::F64D: return reduce_dispatch<Store::F64D>(a, st);
    case Store::F32: return reduce_dispatch<Store::F32>(a, st);
    case Store::F16: return reduce_dispatch<Store::F16>(a, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_export_pop(Store kind, const void* pop, const int32_t* table, const int32_t* ref_of, int n,
                              int npad, double fp16_scale, double* out, cudaStream_t st, int n_main,
                              const double* bnd_f) {
  switch (kind) {
    case Store::F64: return export_f64(pop, table, ref_of, n, npad, out, st, n_main, bnd_f);
    case Store::F64D:
      return export_dispatch<Store::F64D>(pop, table, ref_of, n, npad, fp16_scale, out, st, n_main, bnd_f);
    case Store::F32:
      return export_dispatch<Store::F32>(pop, table, ref_of, n, npad, fp16_scale, out, st, n_main, bnd_f);
    case Store::F16:
      return export_dispatch<Store::F16>(pop, table, ref_of, n, npad, fp16_scale, out, st, n_main, bnd_f);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_import_pop(Store kind, void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad,
                              double fp16_scale, const double* in, cudaStream_t st) {
  switch (kind) {
    case Store::F64: return import_f64(pop, table, ref_of, n, npad, in, st);
    case Store::F64D: return import_dispatch<Store::F64D>(pop, table, ref_of, n, npad, fp16_scale, in, st);
    case Store::F32: return import_dispatch<Store::F32>(pop, table, ref_of, n, npad, fp16_scale, in, st);
    case Store::F16: return import_dispatch<Store::F16>(pop, table, ref_of, n, npad, fp16_scale, in, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_import_macro(Store kind, void* rho, void* u, const int32_t* ref_of, int n, int npad,
                                const double* rho_in, const double* u_in, cudaStream_t st) {
  switch (kind) {
    case Store::F64: return import_macro_f64(rho, u, ref_of, n, npad, rho_in, u_in, st);
    case Store::F64D: return import_macro_dispatch<Store::F64D>(rho, u, ref_of, n, npad, rho_in, u_in, st);
    case Store::F32: return import_macro_dispatch<Store::F32>(rho, u, ref_of, n, npad, rho_in, u_in, st);
    case Store::F16: return import_macro_dispatch<Store::F16>(rho, u, ref_of, n, npad, rho_in, u_in, st);
  }
  return cudaErrorInvalidValue;
}

__global__ void export_macro_kernel(const double* __restrict__ rho_int, const double* __restrict__ u_int,
                                    const int32_t* __restrict__ ref_of, int n, int npad, double* __restrict__ rho_ref,
                                    double* __restrict__ u_ref) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int r = ref_of[p];
  if (rho_ref) rho_ref[r] = rho_int[p];
  if (u_ref) {
    u_ref[(size_t)r * 3 + 0] = u_int[p];
    u_ref[(size_t)r * 3 + 1] = u_int[npad + p];
    u_ref[(size_t)r * 3 + 2] = u_int[2 * npad + p];
  }
}

cudaError_t launch_export_macro(const double* rho_int, const double* u_int, const int32_t* ref_of, int n, int npad,
                                double* rho_ref, double* u_ref, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  export_macro_kernel<<<(n + 255) / 256, 256, 0, st>>>(rho_int, u_int, ref_of, n, npad, rho_ref, u_ref);
  return cudaGetLastError();
}

struct Feq19 {
  double v[kQ];
};

template <Store K>
__global__ void init_uniform_kernel(typename Traits<K>::T* __restrict__ pop, const int32_t* __restrict__ table, int n,
                                    int npad, float scale, Feq19 feq) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  store_pop<K>(pop + p, from_full<K>(feq.v[0], 0), scale);
#pragma unroll
  for (int q = 1; q < kQ; q++)
    store_pop<K>(pop + table[(size_t)(q - 1) * npad + p], from_full<K>(feq.v[q], q), scale);
}

template <typename Mac>
__global__ void fill_macro_kernel(Mac* __restrict__ rho, Mac* __restrict__ u, int n, int npad, double rho0,
                                  double ux, double uy, double uz) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  rho[p] = (Mac)rho0;
  u[p] = (Mac)ux;
  u[npad + p] = (Mac)uy;
  u[2 * npad + p] = (Mac)uz;
}

cudaError_t launch_init_uniform(Store kind, void* pop, const int32_t* table, int n, int npad, double fp16_scale,
                                const double* feq19, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  Feq19 f;
  for (int q = 0; q < kQ; q++) f.v[q] = feq19[q];
  const int g = (n + 255) / 256;
  const float sc = (float)fp16_scale;
  switch (kind) {
    case Store::F64: init_uniform_kernel<Store::F64><<<g, 256, 0, st>>>((double*)pop, table, n, npad, sc, f); break;
    case Store::F64D: init_uniform_kernel<Store::F64D><<<g, 256, 0, st>>>((double*)pop, table, n, npad, sc, f); break;
    case Store::F32: init_uniform_kernel<Store::F32><<<g, 256, 0, st>>>((float*)pop, table, n, npad, sc, f); break;
    case Store::F16: init_uniform_kernel<Store::F16><<<g, 256, 0, st>>>((__half*)pop, table, n, npad, sc, f); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_fill_macro(Store kind, void* rho, void* u, int n, int npad, double rho0, const double* u3,
                              cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int g = (n + 255) / 256;
  if (kind == Store::F64 || kind == Store::F64D)
    fill_macro_kernel<double><<<g, 256, 0, st>>>((double*)rho, (double*)u, n, npad, rho0, u3[0], u3[1], u3[2]);
  else
    fill_macro_kernel<float><<<g, 256, 0, st>>>((float*)rho, (float*)u, n, npad, rho0, u3[0], u3[1], u3[2]);
  return cudaGetLastError();
}

size_t store_bytes(Store kind) {
  switch (kind) {
    case Store::F64:
    case Store::F64D: return 8;
    case Store::F32: return 4;
    case Store::F16: return 2;
  }
  return 8;
}

}  // namespace lbm
