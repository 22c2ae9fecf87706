// FP64 single-phase kernel that reproduces the reference collision bit for bit.
//
// This translation unit is compiled with -fmad=false: every a*b+c stays two
// correctly rounded operations, as in the reference built without FMA
// contraction, and every sum runs in the reference's index order.  The work
// per node is the reference's own sequence (SP3:1423-1779):
//   Guo force per direction, f_eq per direction, then per moment k
//   m_k = M_k . f, F_k = (1 - S_k/2) M_k . G, meq_k = M_k . f_eq,
//   m*_k = m_k - S_k (m_k - meq_k) + dt F_k;   f*_q = MI_q . m*
// with MI the Gauss-Jordan inverse the reference hard-codes.  Zero entries of
// M are skipped (adding a +-0 product never changes a running sum); all 361
// entries of MI are applied, so its round-off entries count as they do in the
// reference.  Streaming is a pull through the table instead of the
// reference's push through nei_loc, which moves values without arithmetic.
#include "bc_kernels.cuh"

namespace lbm {

__constant__ double c_MI[kQ * kQ];

cudaError_t set_mi_constant(const double* mi361, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_MI, mi361, sizeof(double) * kQ * kQ, 0, cudaMemcpyHostToDevice, st);
}

__device__ __forceinline__ double srate(int k, double sv, double so) {
  const bool conserved = (k == 0 || k == 3 || k == 5 || k == 7);
  const bool viscous = (k == 1 || k == 2 || (k >= 9 && k <= 15));
  return conserved ? 0.0 : (viscous ? sv : so);
}

// Collision of one node in the reference's operation order; writes the 19
// post-collision populations of node p.
__device__ __forceinline__ void collide_faithful(const double (&f)[kQ], double rho, double ux, double uy, double uz,
                                                 const StepArgs& a, int p) {
  double* __restrict__ dst = static_cast<double*>(a.dst_pop);
  const double c_s2 = 1.0 * 1.0 / 3;
  const double gx = a.gx, gy = a.gy, gz = a.gz;
  double guo[kQ], feq[kQ];
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    const double ex = cx(q), ey = cy(q), ez = cz(q);
    const double lm0 = ((ex - ux) * gx + (ey - uy) * gy + (ez - uz) * gz) / c_s2;
    const double lm1 = (ex * ux + ey * uy + ez * uz) * (ex * gx + ey * gy + ez * gz) / (c_s2 * c_s2);
    guo[q] = weight(q) * (lm0 + lm1);
    const double eu = ex * ux + ey * uy + ez * uz;
    const double uv = ux * ux + uy * uy + uz * uz;
    feq[q] = weight(q) * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
  }
  double ml[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    double m = 0.0, fh = 0.0, me = 0.0;
    bool first = true;
#pragma unroll
    for (int j = 0; j < kQ; j++) {
      const int c = mcoef(k, j);
      if (c == 0) continue;
      if (first) {
        m = (double)c * f[j];
        fh = (double)c * guo[j];
        me = (double)c * feq[j];
        first = false;
      } else {
        m = m + (double)c * f[j];
        fh = fh + (double)c * guo[j];
        me = me + (double)c * feq[j];
      }
    }
    const double S = srate(k, a.s_v, a.s_o);
    fh *= (1 - 0.5 * S);
    ml[k] = m - S * (m - me) + 1.0 * fh;
  }
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    double s = c_MI[q * kQ] * ml[0];
#pragma unroll
    for (int j = 1; j < kQ; j++) s = s + c_MI[q * kQ + j] * ml[j];
    dst[(size_t)q * a.npad + p] = s;
  }
}

__device__ __forceinline__ void pull_f64(const StepArgs& a, int p, double (&f)[kQ]) {
  const double* __restrict__ src = static_cast<const double*>(a.src_pop);
  f[0] = __ldg(src + p);
#pragma unroll
  for (int q = 1; q < kQ; q++) f[q] = __ldg(src + __ldg(a.table + (size_t)(q - 1) * a.npad + p));
}

__device__ __forceinline__ void macro_in_out(const StepArgs& a, int p, bool given, bool write, const double (&f)[kQ],
                                             double& rho, double& ux, double& uy, double& uz) {
  if (given) {
    const double* r = static_cast<const double*>(a.rho_in);
    const double* u = static_cast<const double*>(a.u_in);
    rho = r[p];
    ux = u[p];
    uy = u[a.npad + p];
    uz = u[2 * a.npad + p];
  } else {
    macro_faithful(f, a.gx / 2, a.gy / 2, a.gz / 2, rho, ux, uy, uz);
  }
  if (write) {
    static_cast<double*>(a.rho_out)[p] = rho;
    double* u = static_cast<double*>(a.u_out);
    u[p] = ux;
    u[a.npad + p] = uy;
    u[2 * a.npad + p] = uz;
  }
}

template <int BS, bool GIVEN, bool WRITE>
__global__ void __launch_bounds__(BS) step_f64_faithful(StepArgs a) {
  const int p = blockIdx.x * BS + threadIdx.x;
  if (p >= a.n_main) return;
  double f[kQ];
  pull_f64(a, p, f);
  double rho, ux, uy, uz;
  macro_in_out(a, p, GIVEN, WRITE, f, rho, ux, uy, uz);
  if (a.snap_dst != nullptr && p >= a.snap_begin) snap_write(a.snap_dst, a.nsnap, p - a.snap_begin, f, rho, ux, uy, uz);
  collide_faithful(f, rho, ux, uy, uz, a, p);
}

// Face nodes: pull, the boundary rules, macro step, record, collision.  With
// a.bnd_f set: only the populations after the rules (current state).
template <bool GIVEN, bool FINAL>
__global__ void __launch_bounds__(128) bc_f64_faithful(BcArgs a) {
  const int b = blockIdx.x * 128 + threadIdx.x;
  const int p = a.s.n_main + b;
  if (p >= a.s.n) return;
  double f[kQ];
  pull_f64(a.s, p, f);
  if (!GIVEN) bc_apply(a, b, f);
  if (FINAL) {
    const size_t nb = (size_t)(a.s.n - a.s.n_main);
#pragma unroll
    for (int q = 0; q < kQ; q++) a.bnd_f[(size_t)q * nb + b] = f[q];
    return;
  }
  double rho, ux, uy, uz;
  macro_in_out(a.s, p, GIVEN, a.s.rho_out != nullptr, f, rho, ux, uy, uz);
  snap_write(a.s.snap_dst, a.s.nsnap, p - a.s.snap_begin, f, rho, ux, uy, uz);
  collide_faithful(f, rho, ux, uy, uz, a.s, p);
}

cudaError_t launch_boundary_f64(const BcArgs& a, cudaStream_t st) {
  const int nb = a.s.n - a.s.n_main;
  if (nb <= 0) return cudaSuccess;
  const int grid = (nb + 127) / 128;
  const bool given = a.s.rho_in != nullptr;
  if (a.bnd_f)
    bc_f64_faithful<false, true><<<grid, 128, 0, st>>>(a);
  else if (given)
    bc_f64_faithful<true, false><<<grid, 128, 0, st>>>(a);
  else
    bc_f64_faithful<false, false><<<grid, 128, 0, st>>>(a);
  return cudaGetLastError();
}

// final pass of the diagnostics reduction (shared by all kinds)
__global__ void reduce_final_kernel(const double* __restrict__ partials, int nblocks, double* __restrict__ result) {
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] = (i == 3) ? fmax(acc[i], partials[(size_t)b * 8 + i]) : acc[i] + partials[(size_t)b * 8 + i];
  block_reduce8(acc, result, smem);
}

template <int BS>
static cudaError_t launch_f64_bs(const StepArgs& a, cudaStream_t st) {
  const int grid = (a.n_main + BS - 1) / BS;
  if (grid == 0) return cudaSuccess;
  const bool given = a.rho_in != nullptr, write = a.rho_out != nullptr;
  if (given && write)
    step_f64_faithful<BS, true, true><<<grid, BS, 0, st>>>(a);
  else if (given)
    step_f64_faithful<BS, true, false><<<grid, BS, 0, st>>>(a);
  else if (write)
    step_f64_faithful<BS, false, true><<<grid, BS, 0, st>>>(a);
  else
    step_f64_faithful<BS, false, false><<<grid, BS, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_step_f64(const StepArgs& a, int block, cudaStream_t st) {
  switch (block) {
    case 64: return launch_f64_bs<64>(a, st);
    case 128: return launch_f64_bs<128>(a, st);
    case 512: return launch_f64_bs<512>(a, st);
    default: return launch_f64_bs<256>(a, st);
  }
}

cudaError_t reduce_f64(const ReduceArgs& a, cudaStream_t st) { return reduce_dispatch<Store::F64>(a, st); }
cudaError_t export_f64(const void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad, double* out,
                       cudaStream_t st, int n_main, const double* bnd_f) {
  return export_dispatch<Store::F64>(pop, table, ref_of, n, npad, 1.0, out, st, n_main, bnd_f);
}
cudaError_t import_f64(void* pop, const int32_t* table, const int32_t* ref_of, int n, int npad, const double* in,
                       cudaStream_t st) {
  return import_dispatch<Store::F64>(pop, table, ref_of, n, npad, 1.0, in, st);
}
cudaError_t import_macro_f64(void* rho, void* u, const int32_t* ref_of, int n, int npad, const double* rho_in,
                             const double* u_in, cudaStream_t st) {
  return import_macro_dispatch<Store::F64>(rho, u, ref_of, n, npad, rho_in, u_in, st);
}

}  // namespace lbm
