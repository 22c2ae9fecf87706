// D3Q7 solute (passive scalar) kernels on the single-phase sparse layout.
//
// Reference: Single_Phase_3D/Solute_Transport_MPI_Software_Spars_6V.cpp
// ("ST7"): six axis velocities e2 (ST7:130), BGK relaxation towards
// C/6 (1 + 3 e.u) with tau_s (ST7:1464-1471), push streaming with halfway
// bounce-back (ST7:1475-1528) and C = sum of the six g (ST7:1619-1633).
//
// Here: g is stored post-collision as six rows [6][npad] (directions 1..6,
// which are also directions 1..6 of the D3Q19 pull table), pulled through
// those six table rows: a table entry q'*npad + m of a D3Q7 direction has
// q' in 1..6, so the row-6 storage index is entry - npad.  One thread per
// node; 2*6*s + 6*4 + 3*s bytes per update.  Compiled with -fmad=false so
// the FP64 variant keeps the reference's arithmetic.
#include "st7_api.h"

namespace lbm {

namespace {

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

// C of every node from the pulled g (the macro step), internal order.
template <typename T>
__global__ void st7_conc_kernel(St7Args a, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  T C = T(0);
  if (a.c_given) {
    C = static_cast<const T*>(a.c_given)[x];
  } else {
#pragma unroll
    for (int q = 1; q < 7; q++) C = C + src[a.table[(size_t)(q - 1) * a.npad + x] - (size_t)a.npad];
  }
  out[x] = (double)C;
}

// Initial state g = C0/6 (1 + 3 e.u), written through the inverse pull.
// Initial populations g_k = C/6 (1 + 3 e_k.u) of `init` (ST7:1249-1327),
// which the reference evaluates before it reads the velocity file (ST7:472-
// 473), with the velocity array still zero: g_k = C/6.  Stored through the
// inverse pull so that the first step pulls exactly these values.
template <typename T>
__global__ void st7_init_kernel(St7Args a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T C = static_cast<const T*>(a.c_given)[x];
  const size_t npad = (size_t)a.npad;
  T* __restrict__ g = static_cast<T*>(a.dst);
  const T eu = T(0);
#pragma unroll
  for (int q = 1; q < 7; q++) {
    const size_t s = a.table[(size_t)(q - 1) * npad + x] - npad;
    g[s] = T(1.0 / 6.0) * C * (T(1) + T(3) * eu);
  }
}

// g as the next step pulls it, [(count+1)*7] in reference id order
// (column 0 unused), and its inverse.
template <typename T>
__global__ void st7_export_kernel(St7Args a, const int32_t* __restrict__ ref_of, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  const size_t npad = (size_t)a.npad;
  double* row = out + (size_t)ref_of[x] * 7;
  row[0] = 0.0;
#pragma unroll
  for (int q = 1; q < 7; q++) row[q] = (double)src[a.table[(size_t)(q - 1) * npad + x] - npad];
}

template <typename T>
__global__ void st7_import_kernel(St7Args a, const int32_t* __restrict__ ref_of, const double* __restrict__ in) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  T* __restrict__ dst = static_cast<T*>(a.dst);
  const size_t npad = (size_t)a.npad;
  const double* row = in + (size_t)ref_of[x] * 7;
#pragma unroll
  for (int q = 1; q < 7; q++) dst[a.table[(size_t)(q - 1) * npad + x] - npad] = (T)row[q];
}

}  // namespace

cudaError_t st7_launch_export(bool f64, const St7Args& a, const int32_t* ref_of, double* out, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (f64)
    st7_export_kernel<double><<<g, 256, 0, st>>>(a, ref_of, out);
  else
    st7_export_kernel<float><<<g, 256, 0, st>>>(a, ref_of, out);
  return cudaGetLastError();
}

cudaError_t st7_launch_import(bool f64, const St7Args& a, const int32_t* ref_of, const double* in, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (f64)
    st7_import_kernel<double><<<g, 256, 0, st>>>(a, ref_of, in);
  else
    st7_import_kernel<float><<<g, 256, 0, st>>>(a, ref_of, in);
  return cudaGetLastError();
}

cudaError_t st7_launch_step(bool f64, const St7Args& a, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  const bool given = a.c_given != nullptr;
  if (f64) {
    if (given)
      st7_step_kernel<double, true><<<g, 256, 0, st>>>(a);
    else
      st7_step_kernel<double, false><<<g, 256, 0, st>>>(a);
  } else {
    if (given)
      st7_step_kernel<float, true><<<g, 256, 0, st>>>(a);
    else
      st7_step_kernel<float, false><<<g, 256, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t st7_launch_conc(bool f64, const St7Args& a, double* out, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (f64)
    st7_conc_kernel<double><<<g, 256, 0, st>>>(a, out);
  else
    st7_conc_kernel<float><<<g, 256, 0, st>>>(a, out);
  return cudaGetLastError();
}

cudaError_t st7_launch_init(bool f64, const St7Args& a, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (f64)
    st7_init_kernel<double><<<g, 256, 0, st>>>(a);
  else
    st7_init_kernel<float><<<g, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace lbm
