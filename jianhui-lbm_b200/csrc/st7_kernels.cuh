// D3Q7 solute step kernel, shared by the FP32 (st7_kernels.cu, FMA
// contraction allowed) and the FP64 (st7_faithful.cu, -fmad=false) builds.
//
// Reference: Single_Phase_3D/Solute_Transport_MPI_Software_Spars_6V.cpp
// ("ST7"): BGK relaxation towards C/6 (1 + 3 e.u) with tau_s (ST7:1464-1471),
// push streaming with halfway bounce-back (ST7:1475-1528) and C = sum of the
// six g (ST7:1619-1633).  Here g is pulled through rows 1..6 of the flow's
// pull table (a D3Q7 direction q is D3Q19 direction q, so a table entry
// q'*npad + m has q' in 1..6 and its row-6 storage index is entry - npad).
#pragma once

#include "cg_basis.h"
#include "st7_api.h"

namespace lbm {
namespace st7_detail {

template <typename T, bool GIVEN>
__global__ void __launch_bounds__(256) st7_step_kernel(St7Args a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  T* __restrict__ dst = static_cast<T*>(a.dst);
  const T* __restrict__ u = static_cast<const T*>(a.u);
  const size_t npad = (size_t)a.npad;
  T g[7];
  g[0] = T(0);
#pragma unroll
  for (int q = 1; q < 7; q++) g[q] = __ldg(src + (__ldg(a.table + (size_t)(q - 1) * npad + x) - npad));
  T C;
  if (GIVEN) {
    C = static_cast<const T*>(a.c_given)[x];
  } else {
    C = T(0);
#pragma unroll
    for (int q = 1; q < 7; q++) C = C + g[q];
  }
  if (a.c_out) static_cast<T*>(a.c_out)[x] = C;
  const T ux = u[x], uy = u[npad + x], uz = u[2 * npad + x];
  const T tau = T(a.tau_s);
#pragma unroll
  for (int q = 1; q < 7; q++) {
    const T eu = T(cx(q)) * ux + T(cy(q)) * uy + T(cz(q)) * uz;
    const T nv = g[q] - (g[q] - T(1.0 / 6.0) * C * (T(1) + T(3) * eu)) / tau;
    dst[(size_t)(q - 1) * npad + x] = nv;
  }
}

// D3Q19 solute step (the D3Q19 solute program, ST19:1346-1640): the same
// BGK update on the 19 directions of the flow lattice, towards
// w_q C (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u) (its equilibrium with
// c2 = c4 = lat_c^2 = 1), with C the sum of the 19 pulled g in the solute
// program's own direction order (ST19:121-127, 1636-1650: opposite directions
// adjacent, the colour-gradient order, storage row cg::row(k)).  g is stored
// as [19][npad] in the flow's row order, so a table entry q'*npad + m indexes
// it directly; each direction's update depends only on its vector.  e.u is
// summed over the non-zero components of e_q (a zero product only adds +-0).
template <int Q>
__device__ __forceinline__ double st19_edot(double ux, double uy, double uz) {
  double s = 0.0;
  bool first = true;
  if (cx(Q) != 0) {
    s = cx(Q) > 0 ? ux : -ux;
    first = false;
  }
  if (cy(Q) != 0) {
    s = first ? (cy(Q) > 0 ? uy : -uy) : (cy(Q) > 0 ? s + uy : s - uy);
    first = false;
  }
  if (cz(Q) != 0) s = first ? (cz(Q) > 0 ? uz : -uz) : (cz(Q) > 0 ? s + uz : s - uz);
  return s;
}

// UNIT: the default lattice (lat_c = 1), where the program's divisions by
// c2 = c4 = 1 are exact and left out; otherwise (lattice_v, ST19:1259-1268)
// 3 e.u / c2, 4.5 (e.u)^2 / c4 and 1.5 u.u / c2 as the program writes them.
template <typename T, bool GIVEN, bool UNIT>
__global__ void __launch_bounds__(256) st19_step_kernel(St7Args a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  T* __restrict__ dst = static_cast<T*>(a.dst);
  const T* __restrict__ u = static_cast<const T*>(a.u);
  const size_t npad = (size_t)a.npad;
  T g[kQ];
  g[0] = __ldg(src + x);
#pragma unroll
  for (int q = 1; q < kQ; q++) g[q] = __ldg(src + __ldg(a.table + (size_t)(q - 1) * npad + x));
  T C;
  if (GIVEN) {
    C = static_cast<const T*>(a.c_given)[x];
  } else {
    C = T(0);
#pragma unroll
    for (int k = 0; k < kQ; k++) C = C + g[cg::row(k)];
  }
  if (a.c_out) static_cast<T*>(a.c_out)[x] = C;
  const T ux = u[x], uy = u[npad + x], uz = u[2 * npad + x];
  const T uu = ux * ux + uy * uy + uz * uz;
  const T tau = T(a.tau_s);
  {
    const T eq = UNIT ? T(weight(0)) * C * (T(1) - T(1.5) * uu)
                      : T(weight(0)) * C * (T(1) + T(3) * T(0) / T(a.c2) + T(4.5) * T(0) * T(0) / T(a.c4) -
                                            T(1.5) * uu / T(a.c2));
    dst[x] = g[0] - (g[0] - eq) / tau;
  }
#pragma unroll
  for (int q = 1; q < kQ; q++) {
    T eu;
    if (q == 1) eu = (T)st19_edot<1>(ux, uy, uz);
    if (q == 2) eu = (T)st19_edot<2>(ux, uy, uz);
    if (q == 3) eu = (T)st19_edot<3>(ux, uy, uz);
    if (q == 4) eu = (T)st19_edot<4>(ux, uy, uz);
    if (q == 5) eu = (T)st19_edot<5>(ux, uy, uz);
    if (q == 6) eu = (T)st19_edot<6>(ux, uy, uz);
    if (q == 7) eu = (T)st19_edot<7>(ux, uy, uz);
    if (q == 8) eu = (T)st19_edot<8>(ux, uy, uz);
    if (q == 9) eu = (T)st19_edot<9>(ux, uy, uz);
    if (q == 10) eu = (T)st19_edot<10>(ux, uy, uz);
    if (q == 11) eu = (T)st19_edot<11>(ux, uy, uz);
    if (q == 12) eu = (T)st19_edot<12>(ux, uy, uz);
    if (q == 13) eu = (T)st19_edot<13>(ux, uy, uz);
    if (q == 14) eu = (T)st19_edot<14>(ux, uy, uz);
    if (q == 15) eu = (T)st19_edot<15>(ux, uy, uz);
    if (q == 16) eu = (T)st19_edot<16>(ux, uy, uz);
    if (q == 17) eu = (T)st19_edot<17>(ux, uy, uz);
    if (q == 18) eu = (T)st19_edot<18>(ux, uy, uz);
    const T eq = UNIT ? T(weight(q)) * C * (T(1) + T(3) * eu + T(4.5) * eu * eu - T(1.5) * uu)
                      : T(weight(q)) * C * (T(1) + T(3) * eu / T(a.c2) + T(4.5) * eu * eu / T(a.c4) -
                                            T(1.5) * uu / T(a.c2));
    dst[(size_t)q * npad + x] = g[q] - (g[q] - eq) / tau;
  }
}

template <typename T>
cudaError_t launch_step19(const St7Args& a, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  const bool unit = a.c2 == 1.0 && a.c4 == 1.0;
  if (a.c_given != nullptr)
    unit ? st19_step_kernel<T, true, true><<<g, 256, 0, st>>>(a) : st19_step_kernel<T, true, false><<<g, 256, 0, st>>>(a);
  else
    unit ? st19_step_kernel<T, false, true><<<g, 256, 0, st>>>(a)
         : st19_step_kernel<T, false, false><<<g, 256, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_step(const St7Args& a, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (a.c_given != nullptr)
    st7_step_kernel<T, true><<<g, 256, 0, st>>>(a);
  else
    st7_step_kernel<T, false><<<g, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace st7_detail
}  // namespace lbm
