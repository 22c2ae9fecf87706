// Many independent single-phase solves in one node pool.
//
// Layout: every instance owns a contiguous, tile-aligned node range
// [begin, end) of one population pool pop[19][cap] and one pull table
// [18][cap] whose entries are flat indices q*cap + m into the same pool (an
// instance only ever pulls from its own range).  The pool is cut into tiles
// of kTile nodes; tile_inst[t] names the instance slot owning tile t (-1 =
// free).  At the start of every chain the list kernels compact the tiles of
// stepping slots into a work list (with each tile's constants); a step block
// takes one work item, the host launches at least one block per stepping
// item, and the captured CUDA graph of a chain only depends on the grid the
// host picks for the stepping tile count (one graph per power of two).
//
// Convergence is decided on the device: every chain of check_every steps ends
// with a per-tile sum of u, a per-instance sum of its tiles in fixed order
// (results do not depend on what else is in the pool), and an update that
// applies the reference's stop test |(u_ave_prev - u_ave)/u_ave_prev| < tol
// (SP:812-816, u_ave from Comput_Perm SP3:3634-3638) per instance.
#include "batch.h"
#include "kernels_common.cuh"

namespace lbm {

// Block b steps tile b of the work list (the stepping tiles in list order):
// kTile / BS passes of BS nodes, all on the one broadcast load of the tile's
// entry (the single-domain step waits on none).  The host launches at least
// as many blocks as there are stepping tiles (a power of two at or above
// their count, chain_grid), and the list kernels fill the entries past the
// stepping tiles with an empty node range, so a block needs no count of the
// stepping tiles: the blocks past the list read an empty entry and exit.
// FP32 at 256 threads: 5 resident blocks per SM in 48 registers without
// spills, as the single-domain step (16 sphere packs to the stop test:
// 0.427-0.429 against 0.430-0.432 s at 4 blocks, alternating runs).
template <Store K, int BS>
__global__ void __launch_bounds__(BS, (K == Store::F32 && BS == 256) ? 5 : 1)
    batch_step_kernel(BatchStepArgs a, int chain_step) {
  using T = typename Traits<K>::T;
  using A = typename Traits<K>::A;
  constexpr int kSub = kTile / BS;
  const T* __restrict__ src = static_cast<const T*>(a.src_pop);
  T* __restrict__ dst = static_cast<T*>(a.dst_pop);
  const size_t cap = (size_t)a.cap;
  const int i = blockIdx.x;
  if (i >= a.ntiles) return;
  const TileWork w = a.work[i];
  const float scale = w.fp16_scale, inv_scale = 1.0f / w.fp16_scale;
#pragma unroll 1
  for (int sub = 0; sub < kSub; sub++) {
    const int p = w.p0 + sub * BS + threadIdx.x;
    if (p >= w.end) return;
    A f[kQ];
    f[0] = load_pop<K>(src + p, inv_scale);
#pragma unroll
    for (int q = 1; q < kQ; q++) f[q] = load_pop<K>(src + __ldg(a.table + (size_t)(q - 1) * cap + p), inv_scale);
    PairSplit<A> ps;
    split_pairs(f, ps);
    A drho, rho, ux, uy, uz;
    if (chain_step == 0 && w.fresh) {
      rho = A(1);
      drho = A(0);
      ux = A(w.u0[0]);
      uy = A(w.u0[1]);
      uz = A(w.u0[2]);
    } else {
      macro_dev<A>(f, ps, A(0.5f * w.g[0]), A(0.5f * w.g[1]), A(0.5f * w.g[2]), drho, rho, ux, uy, uz);
    }
    mrt_collide_dev<A>(f, ps, drho, rho, ux, uy, uz, A(w.g[0]), A(w.g[1]), A(w.g[2]), A(w.s_v), A(w.s_o));
#pragma unroll
    for (int q = 0; q < kQ; q++) store_pop<K>(dst + (size_t)q * cap + p, f[q], scale);
  }
}

// Work list of a chain, in two launches whose cost follows the slots and the
// stepping tiles, not the pool size.  (1) One block: the stepping tile count
// of every slot, its exclusive scan into slot_off[0..nslots] (slot order) and
// n_active.  (2) Entry e of the list: the slot whose offset range holds e
// (binary search of slot_off), that slot's tile e - slot_off[s] with its
// constants; entries past the stepping tiles, up to the tiles the chain grid
// covers, get an empty node range (p0 = end = 0).
__device__ __forceinline__ int stepping_tiles(const BatchReduceArgs& a, int s) {
  return a.state[s].active ? a.inst[s].tile_end - a.inst[s].tile_begin : 0;
}

__global__ void __launch_bounds__(1024) batch_slot_scan_kernel(BatchReduceArgs a) {
  __shared__ int counts[1024];
  const int chunk = (a.nslots + 1023) / 1024;
  const int lo = min((int)threadIdx.x * chunk, a.nslots), hi = min(lo + chunk, a.nslots);
  int c = 0;
  for (int s = lo; s < hi; s++) c += stepping_tiles(a, s);
  counts[threadIdx.x] = c;
  __syncthreads();
  // inclusive scan (Hillis-Steele)
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = threadIdx.x >= off ? counts[threadIdx.x - off] : 0;
    __syncthreads();
    counts[threadIdx.x] += v;
    __syncthreads();
  }
  int w = counts[threadIdx.x] - c;
  for (int s = lo; s < hi; s++) {
    a.slot_off[s] = w;
    w += stepping_tiles(a, s);
  }
  if (threadIdx.x == 1023) {
    a.slot_off[a.nslots] = counts[1023];
    *a.n_active = counts[1023];
  }
}

__global__ void __launch_bounds__(256) batch_work_kernel(BatchReduceArgs a, int fill_to) {
  const int total = a.slot_off[a.nslots];
  const int n = max(total, fill_to);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    TileWork tw{};
    if (e < total) {
      // the last slot whose offset is <= e (slots without stepping tiles
      // share their offset with the next slot and are passed over)
      int lo = 0, hi = a.nslots - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.slot_off[mid] <= e)
          lo = mid;
        else
          hi = mid - 1;
      }
      const InstParams& ip = a.inst[lo];
      const int t = ip.tile_begin + (e - a.slot_off[lo]);
      tw.p0 = t * kTile;
      tw.end = ip.end;
      for (int d = 0; d < 3; d++) {
        tw.g[d] = ip.g[d];
        tw.u0[d] = ip.u0[d];
      }
      tw.s_v = ip.s_v;
      tw.s_o = ip.s_o;
      tw.fp16_scale = ip.fp16_scale;
      tw.fresh = a.state[lo].fresh;
      a.active_tiles[e] = t;
    }
    a.work[e] = tw;
  }
}

cudaError_t launch_batch_list(const BatchReduceArgs& a, int step_grid, int block, cudaStream_t st) {
  (void)block;
  const int fill_to = std::min(a.ntiles, step_grid);  // one block per tile
  batch_slot_scan_kernel<<<1, 1024, 0, st>>>(a);
  const int g = std::max(1, std::min((fill_to + 255) / 256, 4 * 148));
  batch_work_kernel<<<g, 256, 0, st>>>(a, fill_to);
  return cudaGetLastError();
}

// Sum of u (and rho) over one tile's post-streaming state.
template <Store K>
__device__ __forceinline__ void batch_tile_sum(const BatchReduceArgs& a, int t, const InstParams& ip, double* smem) {
  using T = typename Traits<K>::T;
  using A = typename Traits<K>::A;
  const T* __restrict__ pop = static_cast<const T*>(a.pop);
  const size_t cap = (size_t)a.cap;
  const float inv_scale = 1.0f / ip.fp16_scale;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int p = t * kTile + threadIdx.x;
  if (p < ip.end) {
    A f[kQ];
    f[0] = load_pop<K>(pop + p, inv_scale);
#pragma unroll
    for (int q = 1; q < kQ; q++) f[q] = load_pop<K>(pop + __ldg(a.table + (size_t)(q - 1) * cap + p), inv_scale);
    PairSplit<A> ps;
    split_pairs(f, ps);
    A drho, rho, ux, uy, uz;
    macro_dev<A>(f, ps, A(0.5f * ip.g[0]), A(0.5f * ip.g[1]), A(0.5f * ip.g[2]), drho, rho, ux, uy, uz);
    acc[4] = ux;
    acc[5] = uy;
    acc[6] = uz;
    acc[7] = rho;
  }
  block_reduce8(acc, a.tile_partials + (size_t)t * 8, smem);
}

// Persistent over the active tile list.
template <Store K>
__global__ void __launch_bounds__(kTile) batch_tile_sums_kernel(BatchReduceArgs a) {
  __shared__ double smem[8 * 32];
  const int na = *a.n_active;
  for (int i = blockIdx.x; i < na; i += gridDim.x) {
    const int t = a.active_tiles[i];
    const InstParams ip = a.inst[a.tile_inst[t]];
    batch_tile_sum<K>(a, t, ip, smem);
    __syncthreads();  // smem is reused by the next tile
  }
}

// One block per active slot: its tiles' partials in index order, then the
// stop test.  Deterministic: the sum order depends only on the instance.
__global__ void __launch_bounds__(256) batch_update_kernel(BatchReduceArgs a, int chain_len, double tol,
                                                           long long max_steps) {
  __shared__ double smem[8 * 32];
  __shared__ double tot[8];
  const int slot = blockIdx.x;
  if (slot >= a.nslots) return;
  InstState& st = a.state[slot];
  if (!st.active) return;
  const InstParams ip = a.inst[slot];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = ip.tile_begin + threadIdx.x; t < ip.tile_end; t += blockDim.x)
#pragma unroll
    for (int i = 4; i < 8; i++) acc[i] += a.tile_partials[(size_t)t * 8 + i];
  block_reduce8(acc, tot, smem);
  __syncthreads();
  if (threadIdx.x != 0) return;
  st.steps += chain_len;
  st.fresh = 0;
  const double V = ip.volume, phi = ip.porosity;
  double uave2 = 0.0;
  for (int d = 0; d < 3; d++) {
    st.q[d] = tot[4 + d];
    const double c = tot[4 + d] / (V * phi);
    uave2 += c * c;
  }
  st.mass = tot[7];
  const double uave = sqrt(uave2);
  const bool have_prev = st.checks > 0;
  const bool conv = have_prev && fabs((st.uave - uave) / st.uave) < tol;
  st.uave_prev = st.uave;
  st.uave = uave;
  st.checks += 1;
  if (!(uave == uave)) {
    st.active = 0;
    st.done = 3;  // non-finite
  } else if (conv) {
    st.active = 0;
    st.done = 1;
  } else if (st.steps >= max_steps) {
    st.active = 0;
    st.done = 2;
  }
}

// Post-streaming macro fields of one instance (reference layout, double).
template <Store K>
__global__ void batch_export_macro_kernel(const typename Traits<K>::T* __restrict__ pop, const int32_t* __restrict__ table,
                                          int cap, int begin, int n, const int32_t* __restrict__ ref_of,
                                          InstParams ip, double* __restrict__ rho_ref, double* __restrict__ u_ref) {
  using A = typename Traits<K>::A;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = begin + i;
  const float inv_scale = 1.0f / ip.fp16_scale;
  A f[kQ];
  f[0] = load_pop<K>(pop + p, inv_scale);
#pragma unroll
  for (int q = 1; q < kQ; q++) f[q] = load_pop<K>(pop + table[(size_t)(q - 1) * cap + p], inv_scale);
  PairSplit<A> ps;
  split_pairs(f, ps);
  A drho, rho, ux, uy, uz;
  macro_dev<A>(f, ps, A(0.5f * ip.g[0]), A(0.5f * ip.g[1]), A(0.5f * ip.g[2]), drho, rho, ux, uy, uz);
  const int r = ref_of[i];
  if (rho_ref) rho_ref[r] = rho;
  if (u_ref) {
    u_ref[(size_t)r * 3 + 0] = ux;
    u_ref[(size_t)r * 3 + 1] = uy;
    u_ref[(size_t)r * 3 + 2] = uz;
  }
}

// Uniform initial state feq(1, u0) of one instance's nodes, through the
// inverse pull (the table is a permutation of the instance's slots).
template <Store K>
__global__ void batch_init_kernel(typename Traits<K>::T* __restrict__ pop, const int32_t* __restrict__ table, int cap,
                                  int begin, int n, InstParams ip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = begin + i;
  const double u[3] = {ip.u0[0], ip.u0[1], ip.u0[2]};
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    const double eu = cx(q) * u[0] + cy(q) * u[1] + cz(q) * u[2];
    const double uv = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double feq = weight(q) * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
    const size_t dst = q == 0 ? (size_t)p : (size_t)table[(size_t)(q - 1) * cap + p];
    store_pop<K>(pop + dst, from_full<K>(feq, q), ip.fp16_scale);
  }
}

template <Store K>
static cudaError_t step_k(const BatchStepArgs& a, int block, int grid, int chain_step, cudaStream_t st) {
  switch (block) {
    case 128: batch_step_kernel<K, 128><<<grid, 128, 0, st>>>(a, chain_step); break;
    case 512: batch_step_kernel<K, 512><<<grid, 512, 0, st>>>(a, chain_step); break;
    default: batch_step_kernel<K, 256><<<grid, 256, 0, st>>>(a, chain_step); break;
  }
  return cudaGetLastError();
}

int batch_step_grid(int ntiles, int block) {
  // one block per tile of the whole pool; the chains of a partly stepping
  // pool launch a power of two at or above their stepping tile count
  // (chain_grid), the extra blocks find an empty entry and exit
  (void)block;
  return std::max(1, ntiles);
}

cudaError_t launch_batch_step(Store kind, const BatchStepArgs& a, int block, int grid, int chain_step,
                              cudaStream_t st) {
  if (kind == Store::F16) return step_k<Store::F16>(a, block, grid, chain_step, st);
  return step_k<Store::F32>(a, block, grid, chain_step, st);
}

cudaError_t launch_batch_check(Store kind, const BatchReduceArgs& a, int chain_len, double tol, long long max_steps,
                               cudaStream_t st) {
  if (a.ntiles > 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(a.ntiles, 2 * sms);
    if (kind == Store::F16)
      batch_tile_sums_kernel<Store::F16><<<grid, kTile, 0, st>>>(a);
    else
      batch_tile_sums_kernel<Store::F32><<<grid, kTile, 0, st>>>(a);
  }
  if (a.nslots > 0) batch_update_kernel<<<a.nslots, 256, 0, st>>>(a, chain_len, tol, max_steps);
  return cudaGetLastError();
}

cudaError_t launch_batch_export_macro(Store kind, const void* pop, const int32_t* table, int cap, int begin, int n,
                                      const int32_t* ref_of, const InstParams& ip, double* rho, double* u,
                                      cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int g = (n + 255) / 256;
  if (kind == Store::F16)
    batch_export_macro_kernel<Store::F16><<<g, 256, 0, st>>>((const __half*)pop, table, cap, begin, n, ref_of, ip, rho, u);
  else
    batch_export_macro_kernel<Store::F32><<<g, 256, 0, st>>>((const float*)pop, table, cap, begin, n, ref_of, ip, rho, u);
  return cudaGetLastError();
}

cudaError_t launch_batch_init(Store kind, void* pop, const int32_t* table, int cap, int begin, int n,
                              const InstParams& ip, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int g = (n + 255) / 256;
  if (kind == Store::F16)
    batch_init_kernel<Store::F16><<<g, 256, 0, st>>>((__half*)pop, table, cap, begin, n, ip);
  else
    batch_init_kernel<Store::F32><<<g, 256, 0, st>>>((float*)pop, table, cap, begin, n, ip);
  return cudaGetLastError();
}

}  // namespace lbm
