// Colour-gradient kernels in FP32: f stored as deviations f - w, FP32
// arithmetic, colour sums in direction order.
#include <cmath>

#include "cg_api.h"
#include "cg_kernels_impl.cuh"
#include "mi_pattern.h"

namespace lbm {

__constant__ float c_MIcg_f[kQ * kQ];

template <>
__device__ __forceinline__ float cg_mi<false>(int q, int j) {
  return c_MIcg_f[q * kQ + j];
}

// M^-1 split by parity.  Moments of even degree (rows kEven) depend only on
// f_0 and the pair sums s_i = f_{2i-1} + f_{2i}; odd ones (kOdd) only on the
// pair differences d_i = f_{2i-1} - f_{2i} (the CG order keeps opposite
// directions adjacent).  So f*_0 and h_i = (f*_{2i-1} + f*_{2i})/2 come from
// the even moments and g_i = (f*_{2i-1} - f*_{2i})/2 from the odd ones:
// 10x10 + 9x9 products instead of 19x19.
__host__ __device__ constexpr int kEven(int c) { return cg::even_moment(c); }  // 0, 1, 2, 9 .. 15
__host__ __device__ constexpr int kOdd(int c) { return cg::odd_moment(c); }    // 3 .. 8, 16, 17, 18
__constant__ float c_MIe[10 * 10];
__constant__ float c_MIo[9 * 9];

// The back-transform below skips the entries of the two blocks that the
// build-time pattern (mi_pattern.h, gen_mi_pattern.cpp) marks as zero; this
// checks that the inverse computed at run time has no larger entry there.
bool cg_block_pattern_matches(const double* mi) {
  for (int i = 0; i < 10; i++)
    for (int c = 0; c < 10; c++) {
      const int k = kEven(c);
      const double v = i == 0 ? mi[k] : 0.5 * (mi[(2 * i - 1) * kQ + k] + mi[(2 * i) * kQ + k]);
      if (!((cg_even_block_row(i) >> c) & 1u) && std::fabs(v) > 1e-12) return false;
    }
  for (int i = 1; i <= 9; i++)
    for (int c = 0; c < 9; c++) {
      const int k = kOdd(c);
      const double v = 0.5 * (mi[(2 * i - 1) * kQ + k] - mi[(2 * i) * kQ + k]);
      if (!((cg_odd_block_row(i - 1) >> c) & 1u) && std::fabs(v) > 1e-12) return false;
    }
  return true;
}

cudaError_t cg_set_mi_f32(const double* mi, cudaStream_t st) {
  float m[kQ * kQ], me[100], mo[81];
  for (int i = 0; i < kQ * kQ; i++) m[i] = (float)mi[i];
  for (int c = 0; c < 10; c++) me[c] = (float)mi[kEven(c)];
  for (int i = 1; i <= 9; i++) {
    for (int c = 0; c < 10; c++)
      me[i * 10 + c] = (float)(0.5 * (mi[(2 * i - 1) * kQ + kEven(c)] + mi[(2 * i) * kQ + kEven(c)]));
    for (int c = 0; c < 9; c++)
      mo[(i - 1) * 9 + c] = (float)(0.5 * (mi[(2 * i - 1) * kQ + kOdd(c)] - mi[(2 * i) * kQ + kOdd(c)]));
  }
  cudaError_t e = cudaMemcpyToSymbolAsync(c_MIcg_f, m, sizeof(m), 0, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_MIe, me, sizeof(me), 0, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_MIo, mo, sizeof(mo), 0, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);  // the arrays are host temporaries
}

// FP32 collide pass: the operator of the FP64 kernel (CG3:2684-3351) with
// the arithmetic arranged for the GPU: the 18 table entries are read once and
// serve both the population pull and the neighbour psi of the colour
// gradient; moments and the back-transform use the opposite-pair split, the
// Guo moments their closed forms; divisions by constants and repeated
// divisions become reciprocal multiplies.  The pass is bound by instruction
// latency rather than bytes, so it runs at 5 blocks of 256 per SM (48
// registers, 4 bytes spilled): 109.6 against 115.3 us per step on the 128^3
// cylinder workload at 4 blocks (64 registers); 6 blocks (40 registers, 48
// bytes spilled) gain nothing.
__global__ void __launch_bounds__(256, 5) cg_collide_fast_kernel(CgArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const float* __restrict__ fs = static_cast<const float*>(a.f_src);
  float* __restrict__ fd = static_cast<float*>(a.f_dst);
  const float* __restrict__ psi = static_cast<const float*>(a.psi);
  const int npad = a.npad;

  int32_t tb[kQ];  // tb[q] = pull source of storage row q (q >= 1)
  tb[0] = x;
#pragma unroll
  for (int q = 1; q < kQ; q++) tb[q] = __ldg(a.table + (size_t)(q - 1) * npad + x);

  // pulled deviations in CG order, pair sums / differences
  const float f0 = __ldg(fs + x);
  float sp[10], dp[10];
#pragma unroll
  for (int i = 1; i <= 9; i++) {
    const float fa = __ldg(fs + tb[cg::row(2 * i - 1)]), fb = __ldg(fs + tb[cg::row(2 * i)]);
    sp[i] = fa + fb;
    dp[i] = fa - fb;
  }

  // colour gradient (CG3:2684-2712): psi at x + e_t is the source node of
  // row opp(row(t)); the table entries are dead after this
  const float psi_x = psi[x];
  const float psi_s = (float)a.p.psi_solid;
  float C0 = 0.f, C1 = 0.f, C2 = 0.f;
  bool wall = false;
#pragma unroll
  for (int t = 1; t < kQ; t++) {
    const int q = opp(cg::row(t));
    // a pull from row q itself is a fluid neighbour; behind a wall the entry
    // points into the opposite row
    const uint32_t m = (uint32_t)(tb[q] - q * npad);
    float pn;
    if (m < (uint32_t)npad) {
      pn = psi[m];
    } else {
      pn = psi_s;
      wall = true;
    }
    const float c3w = (float)(3.0 * weight(t));
    if (cg::ex(t)) C0 += (c3w * (float)cg::ex(t)) * pn;
    if (cg::ey(t)) C1 += (c3w * (float)cg::ey(t)) * pn;
    if (cg::ez(t)) C2 += (c3w * (float)cg::ez(t)) * pn;
  }
  const float gx = (float)a.p.g[0], gy = (float)a.p.g[1], gz = (float)a.p.g[2];
  float drho, rho, ux, uy, uz;
  if (a.given) {
    drho = 0.f;
    rho = 1.f;
    ux = (float)a.p.u0[0];
    uy = (float)a.p.u0[1];
    uz = (float)a.p.u0[2];
  } else {
    float r = f0, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int i = 1; i <= 9; i++) {
      r += sp[i];
      if (cg::ex(2 * i - 1)) jx += (float)cg::ex(2 * i - 1) * dp[i];
      if (cg::ey(2 * i - 1)) jy += (float)cg::ey(2 * i - 1) * dp[i];
      if (cg::ez(2 * i - 1)) jz += (float)cg::ez(2 * i - 1) * dp[i];
    }
    drho = r;
    rho = 1.f + r;
    const float ir = 1.f / rho;
    ux = (jx + 0.5f * (float)a.p.gm[0]) * ir;
    uy = (jy + 0.5f * (float)a.p.gm[1]) * ir;
    uz = (jz + 0.5f * (float)a.p.gm[2]) * ir;
  }
  if (a.u_out) {
    float* uo = static_cast<float*>(a.u_out);
    uo[x] = ux;
    uo[(size_t)npad + x] = uy;
    uo[2 * (size_t)npad + x] = uz;
  }

  const float* __restrict__ rrp = static_cast<const float*>(a.rho_r);
  const float* __restrict__ rbp = static_cast<const float*>(a.rho_b);
  const float rr = rrp[x], rb = rbp[x];
  if (fabsf(rr - rb) >= 0.9f && wall) C0 = C1 = C2 = 0.f;
  const float cc = sqrtf(C0 * C0 + C1 * C1 + C2 * C2);
  const float icc = cc > 0.f ? 1.f / cc : 0.f;
  const float nx = C0 * icc, ny = C1 * icc, nz = C2 * icc;

  // Guo forcing moments M G (CG3:2745-2825, G_q = w_q [3 (e_q - u).g +
  // 9 (e_q.u)(e_q.g)]) in closed form for this basis: the lattice sums of
  // c_kq w_q e_q and c_kq w_q e_q e_q leave nine non-zero rows; zero where
  // the phase is not driven
  const bool no_force = ((a.p.body_force_phase == 1) && (psi_x < (float)a.p.flux_psi)) ||
                        ((a.p.body_force_phase == -1) && (psi_x > -(float)a.p.flux_psi));
  // (the undriven case scales the force by 0 so that the rows that are zero
  // for every node stay compile-time zeros)
  const float fg = no_force ? 0.f : 1.f;
  const float fx = fg * gx, fy = fg * gy, fz = fg * gz;
  float MG[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) MG[k] = 0.f;
  {
    const float xx = ux * fx, yy = uy * fy, zz = uz * fz;
    MG[1] = 2.f * (xx + yy + zz);
    MG[3] = fx;
    MG[5] = fy;
    MG[7] = fz;
    MG[9] = 4.f * xx - 2.f * yy - 2.f * zz;
    MG[11] = 2.f * yy - 2.f * zz;
    MG[13] = ux * fy + uy * fx;
    MG[14] = uy * fz + uz * fy;
    MG[15] = ux * fz + uz * fx;
  }

  // equilibrium moments with the surface-tension perturbation (CG3:2836-2851),
  // none in the zero-surface-tension layer of a mixture injection (CG3:2854-2867)
  const bool zero_sigma = a.p.zero_sigma != nullptr && a.p.zero_sigma[x];
  const float cap = zero_sigma ? 0.f : (float)a.p.cap_a;
  const float cc5 = 0.5f * cap * cc;
  float meq[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) meq[k] = 0.f;
  meq[0] = drho;
  meq[3] = ux;
  meq[5] = uy;
  meq[7] = uz;
  meq[1] = (ux * ux + uy * uy + uz * uz) + cap * cc;
  meq[9] = (2.f * ux * ux - uy * uy - uz * uz) + cc5 * (2.f * nx * nx - ny * ny - nz * nz);
  meq[11] = (uy * uy - uz * uz) + cc5 * (ny * ny - nz * nz);
  meq[13] = ux * uy + cc5 * (nx * ny);
  meq[14] = uy * uz + cc5 * (ny * nz);
  meq[15] = ux * uz + cc5 * (nx * nz);

  // viscosity interpolation in psi (CG3:2862-2872)
  float s_v;
  if (psi_x > 0.f)
    s_v = psi_x > (float)a.p.delta ? (float)a.p.wl : (float)a.p.lg0 + (float)a.p.l1 * psi_x + (float)a.p.l2 * psi_x * psi_x;
  else
    s_v = psi_x < -(float)a.p.delta ? (float)a.p.wg : (float)a.p.lg0 + (float)a.p.g1 * psi_x + (float)a.p.g2 * psi_x * psi_x;
  const float s_o = 8.f * (2.f - s_v) / (8.f - s_v);

  // relaxed moments m* = m - S (m - meq) + (1 - S/2) M G
  float ml[kQ];
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    const bool odd = (k >= 3 && k <= 8) || k >= 16;
    float m = odd ? 0.f : (float)cg::mcoef(k, 0) * f0;
#pragma unroll
    for (int i = 1; i <= 9; i++) {
      const int c = cg::mcoef(k, 2 * i - 1);
      if (c == 0) continue;
      m += (float)c * (odd ? dp[i] : sp[i]);
    }
    const bool cons = (k == 0 || k == 3 || k == 5 || k == 7);
    const bool visc = (k == 1 || k == 2 || (k >= 9 && k <= 15));
    const float S = cons ? 0.f : (visc ? s_v : s_o);
    ml[k] = m - S * (m - meq[k]) + (1.f - 0.5f * S) * MG[k];
  }

  // back-transform by parity blocks, without the blocks' zero entries (105
  // of 181 products remain)
  {
    float v = 0.f;
#pragma unroll
    for (int c = 0; c < 10; c++)
      if ((cg_even_block_row(0) >> c) & 1u) v += c_MIe[c] * ml[kEven(c)];
    fd[x] = v;
  }
#pragma unroll
  for (int i = 1; i <= 9; i++) {
    float h = 0.f, g = 0.f;
#pragma unroll
    for (int c = 0; c < 10; c++)
      if ((cg_even_block_row(i) >> c) & 1u) h += c_MIe[i * 10 + c] * ml[kEven(c)];
#pragma unroll
    for (int c = 0; c < 9; c++)
      if ((cg_odd_block_row(i - 1) >> c) & 1u) g += c_MIo[(i - 1) * 9 + c] * ml[kOdd(c)];
    fd[(size_t)cg::row(2 * i - 1) * npad + x] = h + g;
    fd[(size_t)cg::row(2 * i) * npad + x] = h - g;
  }

  // colour record of this node: the recoloured distributions it emits
  // (CG3:3472-3505) are a function of these eight values, and the next
  // colour pass recomputes each one where it is pulled instead of storing
  // 2 x 19 of them
  // two planes [2][npad] of float4: a warp's gathers of one plane read
  // 16 contiguous-ish bytes per node instead of half of every 32-byte record
  float4* __restrict__ rec = reinterpret_cast<float4*>(a.rec) + x;
  rec[0] = make_float4(rr, rb, ux, uy);
  rec[npad] = make_float4(uz, nx, ny, nz);
}

// FP32 colour pass (CG3:3472-3570 restated as a pull): rho_r(x), rho_b(x) =
// sums of the recoloured distributions arriving at x, each recomputed from
// the colour record of the node that emitted it.  Direction k of a node with
// record (r, b, u, n), k in the opposite pair (a, a+1) with a odd:
//   E_a = 1 + 3 e_a.u + 4.5 (e_a.u)^2 - 1.5 u.u,  E_{a+1} likewise with -e_a,
//   cp  = min(w r E_a, w r E_{a+1}, w b E_a, w b E_{a+1}) (e_a.n),
//   g_r,a = w r E_a + cp, g_r,a+1 = w r E_{a+1} - cp,
//   g_b,a = w b E_a - cp, g_b,a+1 = w b E_{a+1} + cp
// (n is the unit colour gradient, zero where the reference skips the
// recolouring).  The pull reads storage row q of x from node m = x - e_q, or,
// behind a wall, from x itself in the opposite direction (the other member
// of the same pair).
// The pass is bound by the latency of its 36 record gathers, not by their
// bytes: all 18 table entries are read first, then all 36 gathers are issued
// before any of them is used, at 64 registers (4 blocks of 256 per SM; 115
// against 127 us per step on the 128^3 cylinder workload with the gathers
// issued one direction at a time at 32 registers and full occupancy).
__global__ void __launch_bounds__(256, 4) cg_colour_fast_kernel(CgArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const float4* __restrict__ rec = reinterpret_cast<const float4*>(a.rec);
  const int npad = a.npad;
  int32_t src[kQ];
  bool first[kQ];
#pragma unroll
  for (int q = 1; q < kQ; q++) src[q] = __ldg(a.table + (size_t)(q - 1) * npad + x);
#pragma unroll
  for (int q = 1; q < kQ; q++) {
    const int k = cg::of_row(q);
    const int32_t lo = q * npad;
    const bool streamed = src[q] >= lo && src[q] < lo + npad;
    src[q] = streamed ? src[q] - lo : x;
    // member of the pair actually pulled: k itself when streamed, its opposite behind a wall
    first[q] = ((k % 2) != 0) == streamed;
  }
  float4 r0[kQ], r1[kQ];
  r0[0] = __ldg(rec + x);
  r1[0] = __ldg(rec + (size_t)npad + x);
#pragma unroll
  for (int q = 1; q < kQ; q++) {
    r0[q] = __ldg(rec + src[q]);
    r1[q] = __ldg(rec + (size_t)npad + src[q]);
  }
  float sr, sb;
  {
    const float uu = r0[0].z * r0[0].z + r0[0].w * r0[0].w + r1[0].x * r1[0].x;
    const float e0 = (float)weight(0) * (1.f - 1.5f * uu);
    sr = r0[0].x * e0;
    sb = r0[0].y * e0;
  }
#pragma unroll
  for (int q = 1; q < kQ; q++) {
    const int k = cg::of_row(q);
    const int ka = (k % 2) ? k : k - 1;  // first member of the pair
    const float ux = r0[q].z, uy = r0[q].w, uz = r1[q].x;
    const float eu = (float)cg::ex(ka) * ux + (float)cg::ey(ka) * uy + (float)cg::ez(ka) * uz;
    const float base = 1.f - 1.5f * (ux * ux + uy * uy + uz * uz) + 4.5f * eu * eu;
    const float Ea = base + 3.f * eu, Eb = base - 3.f * eu;
    const float w = (float)weight(ka);
    const float wr = w * r0[q].x, wb = w * r0[q].y;
    const float ra = wr * Ea, rb_ = wr * Eb, ba = wb * Ea, bb = wb * Eb;
    const float en = (float)cg::ex(ka) * r1[q].y + (float)cg::ey(ka) * r1[q].z + (float)cg::ez(ka) * r1[q].w;
    const float cp = fminf(fminf(ra, rb_), fminf(ba, bb)) * en;
    sr += first[q] ? ra + cp : rb_ - cp;
    sb += first[q] ? ba - cp : bb + cp;
  }
  static_cast<float*>(a.rho_r)[x] = sr;
  static_cast<float*>(a.rho_b)[x] = sb;
  static_cast<float*>(a.psi)[x] = (sr - sb) / (sr + sb);
}

cudaError_t cg_colour_f32(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_colour_fast_kernel<<<(a.n + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t cg_collide_f32(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_collide_fast_kernel<<<(a.n + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename T, bool DEV>
__global__ void cg_export_kernel(const T* __restrict__ f, const int32_t* __restrict__ table,
                                 const int32_t* __restrict__ ref_of, int n, int npad, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  double* row = out + (size_t)ref_of[x] * kQ;
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    const double v = (double)f[cg_slot(table, npad, x, cg::row(k))];
    row[k] = DEV ? v + weight(k) : v;
  }
}

cudaError_t cg_export_f(bool f64, const void* f, const int32_t* table, const int32_t* ref_of, int n, int npad,
                        double* out, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int g = (n + 255) / 256;
  if (f64)
    cg_export_kernel<double, false><<<g, 256, 0, st>>>((const double*)f, table, ref_of, n, npad, out);
  else
    cg_export_kernel<float, true><<<g, 256, 0, st>>>((const float*)f, table, ref_of, n, npad, out);
  return cudaGetLastError();
}

// Inverse of cg_export_kernel: each (node, direction) owns one pulled slot.
template <typename T, bool DEV>
__global__ void cg_import_kernel(T* __restrict__ f, const int32_t* __restrict__ table,
                                 const int32_t* __restrict__ ref_of, int n, int npad, const double* __restrict__ in) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  const double* row = in + (size_t)ref_of[x] * kQ;
#pragma unroll
  for (int k = 0; k < kQ; k++) f[cg_slot(table, npad, x, cg::row(k))] = (T)(DEV ? row[k] - weight(k) : row[k]);
}

cudaError_t cg_import_f(bool f64, void* f, const int32_t* table, const int32_t* ref_of, int n, int npad,
                        const double* in, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int g = (n + 255) / 256;
  if (f64)
    cg_import_kernel<double, false><<<g, 256, 0, st>>>((double*)f, table, ref_of, n, npad, in);
  else
    cg_import_kernel<float, true><<<g, 256, 0, st>>>((float*)f, table, ref_of, n, npad, in);
  return cudaGetLastError();
}

cudaError_t cg_reduce_f32(const CgReduceArgs& a, int nblocks, cudaStream_t st) {
  cg_reduce_kernel<false><<<nblocks, 256, 0, st>>>(a);
  cg_reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nblocks, a.result);
  if (a.partials2) reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials2, nblocks, a.result2);
  return cudaGetLastError();
}

}  // namespace lbm
