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
