// Device code shared by the kernel translation units.
//
// Data layout in HBM (one solver instance):
//   pop   [19][npad]  post-collision populations of the last step, structure
//                     of arrays, one row per direction (storage type per Store)
//   table [18][npad]  int32 pull sources for q = 1..18: flat index into pop
//   rho   [npad], u [3][npad]  macro arrays (double for FP64 kinds, float else)
// A node p of step n pulls f_q(p) = pop[table[q-1][p]] (q >= 1) and
// pop[0*npad + p] (q = 0), relaxes in moment space and writes pop'[q][p].
#pragma once

#include <cuda_fp16.h>

#include "lbm_internal.h"

namespace lbm {

template <Store K>
struct Traits;
template <>
struct Traits<Store::F64> {
  using T = double;   // storage
  using A = double;   // arithmetic
  using Mac = double; // macro arrays
  static constexpr bool kDev = false;
};
template <>
struct Traits<Store::F64D> {
  using T = double;
  using A = double;
  using Mac = double;
  static constexpr bool kDev = true;
};
template <>
struct Traits<Store::F32> {
  using T = float;
  using A = float;
  using Mac = float;
  static constexpr bool kDev = true;
};
template <>
struct Traits<Store::F16> {
  using T = __half;
  using A = float;
  using Mac = float;
  static constexpr bool kDev = true;
};

// Read-only (non-coherent) loads: the source population array and the table
// are never written during a launch.
__device__ __forceinline__ double ldg_(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ldg_(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ldg_(const __half* p) {
  return __half2float(__ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(p))));
}

template <Store K>
__device__ __forceinline__ typename Traits<K>::A load_pop(const typename Traits<K>::T* p, float inv_scale) {
  if constexpr (K == Store::F16)
    return ldg_(p) * inv_scale;
  else
    return ldg_(p);
}
template <Store K>
__device__ __forceinline__ void store_pop(typename Traits<K>::T* p, typename Traits<K>::A v, float scale) {
  if constexpr (K == Store::F16)
    *p = __float2half_rn(v * scale);
  else
    *p = v;
}

// Storage value -> full population f_q as double (export path).
template <Store K>
__device__ __forceinline__ double to_full(typename Traits<K>::A v, int q) {
  if constexpr (Traits<K>::kDev)
    return (double)v + weight(q);
  else
    return (double)v;
}
template <Store K>
__device__ __forceinline__ typename Traits<K>::A from_full(double f, int q) {
  using A = typename Traits<K>::A;
  if constexpr (Traits<K>::kDev)
    return (A)(f - weight(q));
  else
    return (A)f;
}

// ----------------------------------------------------------------------------
// Reference-faithful FP64 macro step (comput_macro_variables, SP3:2414-2439):
// rho = ((0 + f0) + f1) + ... ; u_a = (sum e_a f + dt g_a / 2) / rho, summed in
// direction order.  Must be compiled without FMA contraction.
__device__ __forceinline__ void macro_faithful(const double (&f)[kQ], double hgx, double hgy, double hgz,
                                               double& rho, double& ux, double& uy, double& uz) {
  double r = f[0];
#pragma unroll
  for (int q = 1; q < kQ; q++) r = r + f[q];
  double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    if (cx(q) == 1) x = x + f[q];
    if (cx(q) == -1) x = x - f[q];
    if (cy(q) == 1) y = y + f[q];
    if (cy(q) == -1) y = y - f[q];
    if (cz(q) == 1) z = z + f[q];
    if (cz(q) == -1) z = z - f[q];
  }
  rho = r;
  ux = (x + hgx) / r;
  uy = (y + hgy) / r;
  uz = (z + hgz) / r;
}

// j = sum_q e_q lat_c f_q of a self-defined lattice (SP3:2421-2426 with
// elat = e lat_c): each product is rounded on its own, (-lat_c) f is exactly
// -(lat_c f), and the products of zero components add +-0.
__device__ __forceinline__ void lattice_momentum(const double (&f)[kQ], double c, double& jx, double& jy,
                                                 double& jz) {
  double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    if (cx(q) == 1) x = x + c * f[q];
    if (cx(q) == -1) x = x - c * f[q];
    if (cy(q) == 1) y = y + c * f[q];
    if (cy(q) == -1) y = y - c * f[q];
    if (cz(q) == 1) z = z + c * f[q];
    if (cz(q) == -1) z = z - c * f[q];
  }
  jx = x;
  jy = y;
  jz = z;
}

// macro_faithful on a self-defined lattice: u = (j + dt g / 2) / rho, the
// caller passing hg = dt g / 2 as the reference rounds it.
__device__ __forceinline__ void macro_faithful_lat(const double (&f)[kQ], double c, double hgx, double hgy,
                                                   double hgz, double& rho, double& ux, double& uy, double& uz) {
  double r = f[0];
#pragma unroll
  for (int q = 1; q < kQ; q++) r = r + f[q];
  double x, y, z;
  lattice_momentum(f, c, x, y, z);
  rho = r;
  ux = (x + hgx) / r;
  uy = (y + hgy) / r;
  uz = (z + hgz) / r;
}

// ----------------------------------------------------------------------------
// Deviation-form macro step: f = w + delta, rho = 1 + sum delta, j = sum e delta
// (sum w e = 0), u = (j + g/2) / rho.  s/d are the opposite-pair sums and
// differences the collision reuses.
template <typename A>
struct PairSplit {
  A s[9], d[9];
};

template <typename A>
__device__ __forceinline__ void split_pairs(const A (&f)[kQ], PairSplit<A>& ps) {
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const A a = f[pair_q(i)], b = f[opp(pair_q(i))];
    ps.s[i] = a + b;
    ps.d[i] = a - b;
  }
}

template <typename A>
__device__ __forceinline__ void macro_dev(const A (&f)[kQ], const PairSplit<A>& ps, A hgx, A hgy, A hgz,
                                          A& drho, A& rho, A& ux, A& uy, A& uz) {
  // pairwise order keeps the FP32 sum of small deviations well conditioned
  drho = f[0] + (((ps.s[0] + ps.s[1]) + ps.s[2]) + ((ps.s[3] + ps.s[4]) + (ps.s[5] + ps.s[6])) +
                 (ps.s[7] + ps.s[8]));
  A jx = A(0), jy = A(0), jz = A(0);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    if (cx(pair_q(i)) != 0) jx += A(cx(pair_q(i))) * ps.d[i];
    if (cy(pair_q(i)) != 0) jy += A(cy(pair_q(i))) * ps.d[i];
    if (cz(pair_q(i)) != 0) jz += A(cz(pair_q(i))) * ps.d[i];
  }
  rho = A(1) + drho;
  const A inv = A(1) / rho;
  ux = (jx + hgx) * inv;
  uy = (jy + hgy) * inv;
  uz = (jz + hgz) * inv;
}

// ----------------------------------------------------------------------------
// MRT collision with Guo forcing in moment space, deviation form.
//
// Same operator as the reference collision (SP3:1423-1779): m = M f,
// m* = m - S (m - m_eq) + (I - S/2) M G, f* = M^-1 m*, with
//   G_q = w_q [ (e_q - u).g / c_s^2 + (e_q.u)(e_q.g) / c_s^4 ]   (no rho factor)
//   f_eq = w rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u).
// Here m_eq and M G are their closed forms for this basis (derived from the
// definitions above and checked against M f_eq, M G numerically by the test
// suite), M f uses the even/odd split over opposite pairs, and M^-1 = M^T
// diag(1/|row|^2) because the rows of M are orthogonal.
// In/out: f holds deviations f - w on entry and post-collision deviations on exit.
template <typename A>
__device__ __forceinline__ void mrt_collide_dev(A (&f)[kQ], const PairSplit<A>& ps, A drho, A rho, A ux, A uy,
                                                A uz, A gx, A gy, A gz, A sv, A so) {
  A m[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    A acc = A(0);
    bool first = true;
    if (even_moment(k)) {
      if (mcoef(k, 0) != 0) {
        acc = A(mcoef(k, 0)) * f[0];
        first = false;
      }
#pragma unroll
      for (int i = 0; i < 9; i++)
        if (mcoef(k, pair_q(i)) != 0) {
          if (first) {
            acc = A(mcoef(k, pair_q(i))) * ps.s[i];
            first = false;
          } else {
            acc += A(mcoef(k, pair_q(i))) * ps.s[i];
          }
        }
    } else {
#pragma unroll
      for (int i = 0; i < 9; i++)
        if (mcoef(k, pair_q(i)) != 0) {
          if (first) {
            acc = A(mcoef(k, pair_q(i))) * ps.d[i];
            first = false;
          } else {
            acc += A(mcoef(k, pair_q(i))) * ps.d[i];
          }
        }
    }
    m[k] = acc;
  }

  const A usq = ux * ux + uy * uy + uz * uz;
  const A ug = ux * gx + uy * gy + uz * gz;
  const A hv = A(1) - A(0.5) * sv;
  const A ho = A(1) - A(0.5) * so;
  const A c23 = A(2.0 / 3.0);
  // a_k = [ -S_k (m_k - m_eq,k) + (1 - S_k/2) (M G)_k ] / |row k|^2
  A a[kQ];
  a[0] = A(0);
  a[1] = (-sv * (m[1] - (A(-11) * drho + A(19) * rho * usq)) + hv * A(38) * ug) * A(1.0 / mnorm(1));
  a[2] = (-sv * (m[2] - (A(3) * drho - A(5.5) * rho * usq)) - hv * A(11) * ug) * A(1.0 / mnorm(2));
  a[3] = gx * A(1.0 / mnorm(3));
  a[5] = gy * A(1.0 / mnorm(5));
  a[7] = gz * A(1.0 / mnorm(7));
  a[4] = (-so * (m[4] + c23 * rho * ux) - ho * c23 * gx) * A(1.0 / mnorm(4));
  a[6] = (-so * (m[6] + c23 * rho * uy) - ho * c23 * gy) * A(1.0 / mnorm(6));
  a[8] = (-so * (m[8] + c23 * rho * uz) - ho * c23 * gz) * A(1.0 / mnorm(8));
  const A p9 = rho * (A(2) * ux * ux - uy * uy - uz * uz);
  const A f9 = A(2) * (A(2) * ux * gx - uy * gy - uz * gz);
  a[9] = (-sv * (m[9] - p9) + hv * f9) * A(1.0 / mnorm(9));
  a[10] = (-sv * (m[10] + A(0.5) * p9) - hv * A(0.5) * f9) * A(1.0 / mnorm(10));
  const A p11 = rho * (uy * uy - uz * uz);
  const A f11 = A(2) * (uy * gy - uz * gz);
  a[11] = (-sv * (m[11] - p11) + hv * f11) * A(1.0 / mnorm(11));
  a[12] = (-sv * (m[12] + A(0.5) * p11) - hv * A(0.5) * f11) * A(1.0 / mnorm(12));
  a[13] = (-sv * (m[13] - rho * ux * uy) + hv * (ux * gy + uy * gx)) * A(1.0 / mnorm(13));
  a[14] = (-sv * (m[14] - rho * uy * uz) + hv * (uy * gz + uz * gy)) * A(1.0 / mnorm(14));
  a[15] = (-sv * (m[15] - rho * ux * uz) + hv * (ux * gz + uz * gx)) * A(1.0 / mnorm(15));
  a[16] = -so * m[16] * A(1.0 / mnorm(16));
  a[17] = -so * m[17] * A(1.0 / mnorm(17));
  a[18] = -so * m[18] * A(1.0 / mnorm(18));

  // f*_q = f_q + sum_k M_kq a_k, split into even/odd parts per opposite pair
  {
    A e0 = A(0);
#pragma unroll
    for (int k = 1; k < kQ; k++)
      if (even_moment(k) && mcoef(k, 0) != 0) e0 += A(mcoef(k, 0)) * a[k];
    f[0] += e0;
  }
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const int q = pair_q(i);
    A ev = A(0), od = A(0);
#pragma unroll
    for (int k = 1; k < kQ; k++) {
      if (mcoef(k, q) == 0) continue;
      if (even_moment(k))
        ev += A(mcoef(k, q)) * a[k];
      else
        od += A(mcoef(k, q)) * a[k];
    }
    f[q] += ev + od;
    f[opp(q)] += ev - od;
  }
}

// ----------------------------------------------------------------------------
// Block-level reduction of 8 accumulators: slot MAXSLOT (if any) is a max,
// the others sums; for the single-phase diagnostics the slots are
// (t1, t2, t3, umax^2, Qx, Qy, Qz, mass).  Deterministic for a fixed launch shape.
template <int MAXSLOT = 3>
__device__ __forceinline__ void block_reduce8(double (&v)[8], double* out, double* smem /*[8*32]*/) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const double o = __shfl_down_sync(0xffffffffu, v[i], off);
      v[i] = (i == MAXSLOT) ? fmax(v[i], o) : v[i] + o;
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < 8; i++) smem[warp * 8 + i] = v[i];
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (lane < nw) ? smem[lane * 8 + i] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const double o = __shfl_down_sync(0xffffffffu, v[i], off);
        v[i] = (i == MAXSLOT) ? fmax(v[i], o) : v[i] + o;
      }
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < 8; i++) out[i] = v[i];
  }
}

constexpr int kReduceThreads = 256;

// Second pass: one block sums the per-block partials in a fixed order.
__global__ void reduce_final_kernel(const double* __restrict__ partials, int nblocks, double* __restrict__ result);

// Diagnostic reduction over the current state (Error + Comput_Perm).
template <Store K>
__global__ void __launch_bounds__(kReduceThreads) reduce_kernel(ReduceArgs a) {
  using T = typename Traits<K>::T;
  using A = typename Traits<K>::A;
  using Mac = typename Traits<K>::Mac;
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const T* pop = static_cast<const T*>(a.pop);
  const float inv_scale = (float)(1.0 / a.fp16_scale);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
    double rho, ux, uy, uz;
    if (a.rho_in) {
      const Mac* r = static_cast<const Mac*>(a.rho_in);
      const Mac* u = static_cast<const Mac*>(a.u_in);
      rho = r[p];
      ux = u[p];
      uy = u[a.npad + p];
      uz = u[2 * a.npad + p];
    } else {
      A f[kQ];
      if (a.bnd_f != nullptr && p >= a.n_main) {
        // face node: populations after this state's boundary rules
        const size_t nb = (size_t)(a.n - a.n_main), b = (size_t)(p - a.n_main);
#pragma unroll
        for (int q = 0; q < kQ; q++) f[q] = from_full<K>(a.bnd_f[(size_t)q * nb + b], q);
      } else {
        f[0] = load_pop<K>(pop + p, inv_scale);
#pragma unroll
        for (int q = 1; q < kQ; q++)
          f[q] = load_pop<K>(pop + __ldg(a.table + (size_t)(q - 1) * a.npad + p), inv_scale);
      }
      if constexpr (K == Store::F64) {
        if (a.lat.on)
          macro_faithful_lat(f, a.lat.c, a.lat.dt * a.gx / 2, a.lat.dt * a.gy / 2, a.lat.dt * a.gz / 2, rho, ux,
                             uy, uz);
        else
          macro_faithful(f, a.gx / 2, a.gy / 2, a.gz / 2, rho, ux, uy, uz);
      } else {
        // units of lat_c (g is dt g / lat_c), scaled back to the velocity
        PairSplit<A> ps;
        split_pairs(f, ps);
        A drho, r, x, y, z;
        macro_dev<A>(f, ps, A(a.gx / 2), A(a.gy / 2), A(a.gz / 2), drho, r, x, y, z);
        rho = r;
        ux = (double)x * a.lat.c;
        uy = (double)y * a.lat.c;
        uz = (double)z * a.lat.c;
      }
    }
    if (a.rho_out) a.rho_out[p] = rho;
    if (a.u_out) {
      a.u_out[p] = ux;
      a.u_out[a.npad + p] = uy;
      a.u_out[2 * a.npad + p] = uz;
    }
    double px = ux, py = uy, pz = uz;
    if (a.u_prev) {
      const Mac* up = static_cast<const Mac*>(a.u_prev);
      px = up[p];
      py = up[a.npad + p];
      pz = up[2 * a.npad + p];
    }
    if (p != a.last_p) {
      const double u2 = ux * ux + uy * uy + uz * uz;
      acc[0] += (ux - px) * (ux - px) + (uy - py) * (uy - py) + (uz - pz) * (uz - pz);
      acc[1] += u2;
      acc[2] += sqrt(u2);
      acc[3] = fmax(acc[3], u2);
    }
    if (!a.window || a.window[p]) {
      acc[4] += ux;
      acc[5] += uy;
      acc[6] += uz;
    }
    acc[7] += rho;
  }
  block_reduce8(acc, a.partials + (size_t)blockIdx.x * 8, smem);
}

// Reference-layout export: out[ref_of[p]*19 + q] = f_q(p) (post-streaming, full f).
// Face nodes [n_main, n) take their populations from bnd_f when it is set.
template <Store K>
__global__ void export_pop_kernel(const typename Traits<K>::T* __restrict__ pop, const int32_t* __restrict__ table,
                                  const int32_t* __restrict__ ref_of, int n, int npad, float inv_scale,
                                  double* __restrict__ out, int n_main, const double* __restrict__ bnd_f) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  double* row = out + (size_t)ref_of[p] * kQ;
  if (bnd_f != nullptr && p >= n_main) {
    const size_t nb = (size_t)(n - n_main), b = (size_t)(p - n_main);
#pragma unroll
    for (int q = 0; q < kQ; q++) row[q] = bnd_f[(size_t)q * nb + b];
    return;
  }
  row[0] = to_full<K>(load_pop<K>(pop + p, inv_scale), 0);
#pragma unroll
  for (int q = 1; q < kQ; q++)
    row[q] = to_full<K>(load_pop<K>(pop + table[(size_t)(q - 1) * npad + p], inv_scale), q);
}

// Inverse of the pull: pop[table(q,p)] = f_q(p), so that the next step pulls
// exactly the given post-streaming populations.
template <Store K>
__global__ void import_pop_kernel(typename Traits<K>::T* __restrict__ pop, const int32_t* __restrict__ table,
                                  const int32_t* __restrict__ ref_of, int n, int npad, float scale,
                                  const double* __restrict__ in) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double* row = in + (size_t)ref_of[p] * kQ;
  store_pop<K>(pop + p, from_full<K>(row[0], 0), scale);
#pragma unroll
  for (int q = 1; q < kQ; q++) store_pop<K>(pop + table[(size_t)(q - 1) * npad + p], from_full<K>(row[q], q), scale);
}

template <Store K>
__global__ void import_macro_kernel(typename Traits<K>::Mac* __restrict__ rho, typename Traits<K>::Mac* __restrict__ u,
                                    const int32_t* __restrict__ ref_of, int n, int npad,
                                    const double* __restrict__ rho_in, const double* __restrict__ u_in) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int r = ref_of[p];
  rho[p] = rho_in[r];
  u[p] = u_in[(size_t)r * 3 + 0];
  u[npad + p] = u_in[(size_t)r * 3 + 1];
  u[2 * npad + p] = u_in[(size_t)r * 3 + 2];
}

template <Store K>
cudaError_t reduce_dispatch(const ReduceArgs& a, cudaStream_t st) {
  const int nb = reduce_blocks(a.n);
  reduce_kernel<K><<<nb, kReduceThreads, 0, st>>>(a);
  reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nb, a.result);
  return cudaGetLastError();
}

template <Store K>
cudaError_t export_dispatch(const void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad,
                            double fp16_scale, double* out, cudaStream_t st, int n_main = 0,
                            const double* bnd_f = nullptr) {
  if (n == 0) return cudaSuccess;
  export_pop_kernel<K><<<(n + 255) / 256, 256, 0, st>>>(static_cast<const typename Traits<K>::T*>(pop), table,
                                                        ref_of, n, npad, (float)(1.0 / fp16_scale), out, n_main,
                                                        bnd_f);
  return cudaGetLastError();
}

template <Store K>
cudaError_t import_dispatch(void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad,
                            double fp16_scale, const double* in, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  import_pop_kernel<K><<<(n + 255) / 256, 256, 0, st>>>(static_cast<typename Traits<K>::T*>(pop), table, ref_of, n,
                                                        npad, (float)fp16_scale, in);
  return cudaGetLastError();
}

template <Store K>
cudaError_t import_macro_dispatch(void* rho, void* u, const int32_t* ref_of, int n, int npad, const double* rho_in,
                                  const double* u_in, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  using Mac = typename Traits<K>::Mac;
  import_macro_kernel<K><<<(n + 255) / 256, 256, 0, st>>>(static_cast<Mac*>(rho), static_cast<Mac*>(u), ref_of, n,
                                                          npad, rho_in, u_in);
  return cudaGetLastError();
}

}  // namespace lbm
