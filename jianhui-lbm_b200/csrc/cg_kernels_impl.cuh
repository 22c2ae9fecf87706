// Kernel bodies of the colour-gradient model, templated on the arithmetic:
//   FAITHFUL = true : double, full populations, reference operation order
//                     (compile with -fmad=false), colour sums in the
//                     reference's push order (corder)
//   FAITHFUL = false: float, f stored as deviations f - w, FMA allowed
#pragma once

#include "cg_kernels.cuh"

namespace lbm {

template <bool FAITHFUL>
struct CgT;
template <>
struct CgT<true> {
  using T = double;
};
template <>
struct CgT<false> {
  using T = float;
};

// Colour pass: rho_r, rho_b, psi of every node from the pulled g_r, g_b.
template <bool FAITHFUL>
__global__ void __launch_bounds__(256) cg_colour_kernel(CgArgs a) {
  using T = typename CgT<FAITHFUL>::T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ gr = static_cast<const T*>(a.gr);
  const T* __restrict__ gb = static_cast<const T*>(a.gb);
  T rr = T(0), rb = T(0);
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    // FAITHFUL: contributions in the order the reference's scatter adds them
    const int q = FAITHFUL ? (int)__ldg(a.corder + (size_t)k * a.npad + x) : k;
    const size_t s = cg_slot(a.table, a.npad, x, q);
    rr = rr + __ldg(gr + s);
    rb = rb + __ldg(gb + s);
  }
  static_cast<T*>(a.rho_r)[x] = rr;
  static_cast<T*>(a.rho_b)[x] = rb;
  static_cast<T*>(a.psi)[x] = (rr - rb) / (rr + rb);
}

template <bool FAITHFUL>
__device__ __forceinline__ typename CgT<FAITHFUL>::T cg_mi(int q, int j);

// Collide pass.
template <bool FAITHFUL>
__global__ void __launch_bounds__(256) cg_collide_kernel(CgArgs a) {
  using T = typename CgT<FAITHFUL>::T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ fs = static_cast<const T*>(a.f_src);
  T* __restrict__ fd = static_cast<T*>(a.f_dst);
  const T* __restrict__ psi = static_cast<const T*>(a.psi);
  const size_t npad = (size_t)a.npad;

  // pulled post-streaming f in CG order (FP32: deviations f - w)
  T f[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) f[k] = __ldg(fs + cg_slot(a.table, a.npad, x, cg::row(k)));

  // rho, u (comput_macro_variables, CG3:3330-3352)
  T rho, ux, uy, uz, drho = T(0);
  if (a.given) {
    rho = T(1);
    ux = T(a.p.u0[0]);
    uy = T(a.p.u0[1]);
    uz = T(a.p.u0[2]);
  } else {
    T r = FAITHFUL ? f[0] : f[0];
#pragma unroll
    for (int k = 1; k < kQ; k++) r = r + f[k];
    T sx = T(0), sy = T(0), sz = T(0);
#pragma unroll
    for (int k = 0; k < kQ; k++) {
      if (cg::ex(k) == 1) sx = sx + f[k];
      if (cg::ex(k) == -1) sx = sx - f[k];
      if (cg::ey(k) == 1) sy = sy + f[k];
      if (cg::ey(k) == -1) sy = sy - f[k];
      if (cg::ez(k) == 1) sz = sz + f[k];
      if (cg::ez(k) == -1) sz = sz - f[k];
    }
    if (FAITHFUL) {
      rho = r;
    } else {
      drho = r;
      rho = T(1) + r;
    }
    ux = (sx + T(1.0 * a.p.gm[0]) / T(2)) / rho;
    uy = (sy + T(1.0 * a.p.gm[1]) / T(2)) / rho;
    uz = (sz + T(1.0 * a.p.gm[2]) / T(2)) / rho;
  }
  if (!FAITHFUL && a.given) drho = T(0);
  if (a.u_out) {
    T* uo = static_cast<T*>(a.u_out);
    uo[x] = ux;
    uo[(size_t)a.npad + x] = uy;
    uo[2 * (size_t)a.npad + x] = uz;
  }

  // colour gradient over x + e_t, solid neighbours at psi_solid (CG3:2684-2712)
  const T psi_x = psi[x];
  T C0 = T(0), C1 = T(0), C2 = T(0);
  int ind_S = 0;
#pragma unroll
  for (int t = 0; t < kQ; t++) {
    T pn;
    if (t == 0) {
      pn = psi_x;
    } else {
      const int q = opp(cg::row(t));  // pull row whose source is x + e_t
      const int32_t s = __ldg(a.table + (size_t)(q - 1) * npad + x);
      const int32_t lo = q * a.npad;
      if (s >= lo && s < lo + a.npad) {
        pn = psi[s - lo];
      } else {
        pn = T(a.p.psi_solid);
        ind_S = 1;
      }
    }
    const T c3w = T(3.0 / (1.0 * 1.0 * 1.0)) * T(weight(t));
    if (cg::ex(t) != 0) C0 = C0 + c3w * T(cg::ex(t)) * pn;
    if (cg::ey(t) != 0) C1 = C1 + c3w * T(cg::ey(t)) * pn;
    if (cg::ez(t) != 0) C2 = C2 + c3w * T(cg::ez(t)) * pn;
  }
  const T* __restrict__ rrp = static_cast<const T*>(a.rho_r);
  const T* __restrict__ rbp = static_cast<const T*>(a.rho_b);
  const T rr = rrp[x], rb = rbp[x];
  const T uu = ux * ux + uy * uy + uz * uz;
  if ((sqrt((rr - rb) * (rr - rb)) >= T(0.9)) && (ind_S == 1)) {
    C0 = T(0);
    C1 = T(0);
    C2 = T(0);
  }
  const T cc = sqrt(C0 * C0 + C1 * C1 + C2 * C2);
  T nx, ny, nz;
  if (cc > T(0)) {
    nx = C0 / cc;
    ny = C1 / cc;
    nz = C2 / cc;
  } else {
    nx = ny = nz = T(0);
  }

  // Guo force, zero outside the driven phase (CG3:2745-2825)
  const T gx = T(a.p.g[0]), gy = T(a.p.g[1]), gz = T(a.p.g[2]);
  const bool no_force = ((a.p.body_force_phase == 1) && (psi_x < T(a.p.flux_psi))) ||
                        ((a.p.body_force_phase == -1) && (psi_x > -T(a.p.flux_psi)));
  T guo[kQ];
  const T c_s2 = T(1.0 * 1.0 / 3);
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    if (no_force) {
      guo[q] = T(0);
    } else {
      const T e0 = T(cg::ex(q)), e1 = T(cg::ey(q)), e2 = T(cg::ez(q));
      const T lm0 = ((e0 - ux) * gx + (e1 - uy) * gy + (e2 - uz) * gz) / c_s2;
      const T lm1 = (e0 * ux + e1 * uy + e2 * uz) * (e0 * gx + e1 * gy + e2 * gz) / (c_s2 * c_s2);
      guo[q] = T(weight(q)) * (lm0 + lm1);
    }
  }

  // equilibrium moments with the surface-tension perturbation (CG3:2836-2851)
  const T cap = T(a.p.cap_a);
  T meq[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) meq[k] = T(0);
  meq[0] = FAITHFUL ? rho : drho;
  meq[3] = T(1.0) * ux;
  meq[5] = T(1.0) * uy;
  meq[7] = T(1.0) * uz;
  if (a.p.zero_sigma != nullptr && a.p.zero_sigma[x]) {
    // mixture-injection layer: the equilibrium moments without the surface
    // tension terms (CG3:2854-2867)
    meq[1] = T(1.0) * (ux * ux + uy * uy + uz * uz);
    meq[9] = T(1.0) * (T(2) * ux * ux - uy * uy - uz * uz);
    meq[11] = T(1.0) * (uy * uy - uz * uz);
    meq[13] = T(1.0) * ux * uy;
    meq[14] = T(1.0) * uy * uz;
    meq[15] = T(1.0) * ux * uz;
  } else {
    meq[1] = T(1.0) * (ux * ux + uy * uy + uz * uz) + cap * cc;
    meq[9] = T(1.0) * (T(2) * ux * ux - uy * uy - uz * uz) + T(0.5) * cap * cc * (T(2) * nx * nx - ny * ny - nz * nz);
    meq[11] = T(1.0) * (uy * uy - uz * uz) + T(0.5) * cap * cc * (ny * ny - nz * nz);
    meq[13] = T(1.0) * ux * uy + T(0.5) * cap * cc * (nx * ny);
    meq[14] = T(1.0) * uy * uz + T(0.5) * cap * cc * (ny * nz);
    meq[15] = T(1.0) * ux * uz + T(0.5) * cap * cc * (nx * nz);
  }

  // viscosity interpolation in psi (CG3:2862-2872)
  T s_v;
  if (psi_x > T(0)) {
    if (psi_x > T(a.p.delta))
      s_v = T(a.p.wl);
    else
      s_v = T(a.p.lg0) + T(a.p.l1) * psi_x + T(a.p.l2) * psi_x * psi_x;
  } else {
    if (psi_x < -T(a.p.delta))
      s_v = T(a.p.wg);
    else
      s_v = T(a.p.lg0) + T(a.p.g1) * psi_x + T(a.p.g2) * psi_x * psi_x;
  }
  const T s_o = T(8) * (T(2) - s_v) / (T(8) - s_v);

  T ml[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    T m = T(0), fh = T(0);
    bool first = true;
#pragma unroll
    for (int j = 0; j < kQ; j++) {
      const int c = cg::mcoef(k, j);
      if (c == 0) continue;
      if (first) {
        m = T(c) * f[j];
        fh = T(c) * guo[j];
        first = false;
      } else {
        m = m + T(c) * f[j];
        fh = fh + T(c) * guo[j];
      }
    }
    const bool cons = (k == 0 || k == 3 || k == 5 || k == 7);
    const bool visc = (k == 1 || k == 2 || (k >= 9 && k <= 15));
    const T S = cons ? T(0) : (visc ? s_v : s_o);
    fh *= (T(1) - T(0.5) * S);
    ml[k] = m - S * (m - meq[k]) + T(1.0) * fh;
  }
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    T s = cg_mi<FAITHFUL>(q, 0) * ml[0];
#pragma unroll
    for (int j = 1; j < kQ; j++) s = s + cg_mi<FAITHFUL>(q, j) * ml[j];
    fd[(size_t)cg::row(q) * npad + x] = s;
  }

  // equilibrium colour distributions and recolouring (CG3:3472-3505)
  T gr_[kQ], gb_[kQ];
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    const T eu = T(cg::ex(q)) * ux + T(cg::ey(q)) * uy + T(cg::ez(q)) * uz;
    const T E = T(1) + T(3) * eu / T(1.0) + T(4.5) * eu * eu / T(1.0) - T(1.5) * uu / T(1.0);
    gr_[q] = T(weight(q)) * rr * E;
    gb_[q] = T(weight(q)) * rb * E;
  }
  if (cc > T(0)) {
#pragma unroll
    for (int kk = 1; kk < kQ; kk += 2) {
      const T ef = T(cg::ex(kk)) * C0 + T(cg::ey(kk)) * C1 + T(cg::ez(kk)) * C2;
      T cp = gr_[kk] < gr_[kk + 1] ? gr_[kk] : gr_[kk + 1];
      cp = cp < gb_[kk] ? cp : gb_[kk];
      cp = cp < gb_[kk + 1] ? cp : gb_[kk + 1];
      cp *= ef / cc;
      gr_[kk] += cp;
      gr_[kk + 1] -= cp;
      gb_[kk] -= cp;
      gb_[kk + 1] += cp;
    }
  }
  T* __restrict__ grp = static_cast<T*>(a.gr);
  T* __restrict__ gbp = static_cast<T*>(a.gb);
#pragma unroll
  for (int q = 0; q < kQ; q++) {
    grp[(size_t)cg::row(q) * npad + x] = gr_[q];
    gbp[(size_t)cg::row(q) * npad + x] = gb_[q];
  }
}

template <bool FAITHFUL>
__global__ void __launch_bounds__(256) cg_reduce_kernel(CgReduceArgs a) {
  using T = typename CgT<FAITHFUL>::T;
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double acc2[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // Error (CG3:4683-4750) and saturation position sums
  const T* __restrict__ fs = static_cast<const T*>(a.f);
  const T* __restrict__ psi = static_cast<const T*>(a.psi);
  const T* __restrict__ up = static_cast<const T*>(a.u_prev);
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.n; x += gridDim.x * blockDim.x) {
    T rho, ux, uy, uz;
    if (a.given) {
      rho = T(1);
      ux = T(a.u0[0]);
      uy = T(a.u0[1]);
      uz = T(a.u0[2]);
    } else {
      T f[kQ];
#pragma unroll
      for (int k = 0; k < kQ; k++) f[k] = __ldg(fs + cg_slot(a.table, a.npad, x, cg::row(k)));
      T r = f[0];
#pragma unroll
      for (int k = 1; k < kQ; k++) r = r + f[k];
      T sx = T(0), sy = T(0), sz = T(0);
#pragma unroll
      for (int k = 0; k < kQ; k++) {
        if (cg::ex(k) == 1) sx = sx + f[k];
        if (cg::ex(k) == -1) sx = sx - f[k];
        if (cg::ey(k) == 1) sy = sy + f[k];
        if (cg::ey(k) == -1) sy = sy - f[k];
        if (cg::ez(k) == 1) sz = sz + f[k];
        if (cg::ez(k) == -1) sz = sz - f[k];
      }
      rho = FAITHFUL ? r : T(1) + r;
      ux = (sx + T(1.0 * a.g[0]) / T(2)) / rho;
      uy = (sy + T(1.0 * a.g[1]) / T(2)) / rho;
      uz = (sz + T(1.0 * a.g[2]) / T(2)) / rho;
    }
    if (a.rho_out) a.rho_out[x] = rho;
    if (a.u_out) {
      a.u_out[x] = ux;
      a.u_out[a.npad + x] = uy;
      a.u_out[2 * a.npad + x] = uz;
    }
    const double ps = psi[x];
    const double dx = ux, dy = uy, dz = uz;
    const bool in_win = a.win == nullptr || a.win[x] != 0;  // Comput_Perm's window (CG3:5156-5180)
    if (in_win && sqrt(dx * dx + dy * dy + dz * dz) < a.flux_umax) {
      if (ps >= a.flux_psi) {
        acc[0] += dx;
        acc[1] += dy;
        acc[2] += dz;
      }
      if (ps <= -a.flux_psi) {
        acc[4] += dx;
        acc[5] += dy;
        acc[6] += dz;
      }
    }
    if (in_win && ps >= 0) acc[3] += 1.0;  // Comput_Saturation counts psi >= 0 (CG3:5319)
    acc[7] += (double)rho;
    if (a.partials2) {
      double px = dx, py = dy, pz = dz;
      if (up) {
        px = up[x];
        py = up[(size_t)a.npad + x];
        pz = up[2 * (size_t)a.npad + x];
      }
      const double u2 = dx * dx + dy * dy + dz * dz;
      acc2[0] += (dx - px) * (dx - px) + (dy - py) * (dy - py) + (dz - pz) * (dz - pz);
      acc2[1] += u2;
      acc2[2] += sqrt(u2);
      acc2[3] = fmax(acc2[3], u2);
      if (a.axis && in_win) {
        const double sdir = (double)a.axis[x];
        if (ps >= 0)
          acc2[4] += ps * sdir;
        else
          acc2[5] += ps * sdir;
      }
    }
  }
  block_reduce8<-1>(acc, a.partials + (size_t)blockIdx.x * 8, smem);
  if (a.partials2) {
    __syncthreads();  // smem is reused
    block_reduce8<3>(acc2, a.partials2 + (size_t)blockIdx.x * 8, smem);
  }
}

// Fixed-order sum of the per-block partials (all slots are sums).
static __global__ void __launch_bounds__(1024) cg_reduce_final_kernel(const double* __restrict__ partials, int nblocks,
                                                              double* __restrict__ result) {
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] += partials[(size_t)b * 8 + i];
  block_reduce8<-1>(acc, result, smem);
}

}  // namespace lbm
