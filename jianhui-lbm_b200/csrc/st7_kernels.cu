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
// node; 2*6*s + 6*4 + 3*s bytes per update.  The step kernel lives in
// st7_kernels.cuh; its FP64 instantiation is built in st7_faithful.cu with
// -fmad=false (the reference's unfused arithmetic), this file keeps FMA
// contraction for the FP32 path.
#include "st7_kernels.cuh"

namespace lbm {

namespace {

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

// D3Q19 (the solute program with 19 directions): g is [19][npad]; a node's
// pulled value of storage row q is g[x] for q = 0, else g[table[q-1][x]].
__device__ __forceinline__ size_t st19_slot(const St7Args& a, int x, int q) {
  return q == 0 ? (size_t)x : (size_t)a.table[(size_t)(q - 1) * a.npad + x];
}

// C = sum of the pulled g in the program's direction order (ST19:1636-1650).
template <typename T>
__global__ void st19_conc_kernel(St7Args a, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  T C = T(0);
  if (a.c_given) {
    C = static_cast<const T*>(a.c_given)[x];
  } else {
#pragma unroll
    for (int k = 0; k < kQ; k++) C = C + src[st19_slot(a, x, cg::row(k))];
  }
  out[x] = (double)C;
}

// Initial g_k = w_k C (1 + 3 e_k.u) of init (ST19:1300-1312) with the velocity
// not yet loaded (zero): w_k C, stored through the inverse pull.
template <typename T>
__global__ void st19_init_kernel(St7Args a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T C = static_cast<const T*>(a.c_given)[x];
  T* __restrict__ g = static_cast<T*>(a.dst);
#pragma unroll
  for (int q = 0; q < kQ; q++) g[st19_slot(a, x, q)] = T(weight(q)) * C * (T(1) + T(3) * T(0));
}

// g as the next step pulls it, [(count+1)*19] in reference id order and the
// program's direction order, and its inverse.
template <typename T>
__global__ void st19_export_kernel(St7Args a, const int32_t* __restrict__ ref_of, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  double* row = out + (size_t)ref_of[x] * kQ;
#pragma unroll
  for (int k = 0; k < kQ; k++) row[k] = (double)src[st19_slot(a, x, cg::row(k))];
}

template <typename T>
__global__ void st19_import_kernel(St7Args a, const int32_t* __restrict__ ref_of, const double* __restrict__ in) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.n) return;
  T* __restrict__ dst = static_cast<T*>(a.dst);
  const double* row = in + (size_t)ref_of[x] * kQ;
#pragma unroll
  for (int k = 0; k < kQ; k++) dst[st19_slot(a, x, cg::row(k))] = (T)row[k];
}

}  // namespace

cudaError_t st7_launch_export(bool f64, const St7Args& a, const int32_t* ref_of, double* out, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (a.nq == kQ) {
    if (f64)
      st19_export_kernel<double><<<g, 256, 0, st>>>(a, ref_of, out);
    else
      st19_export_kernel<float><<<g, 256, 0, st>>>(a, ref_of, out);
    return cudaGetLastError();
  }
  if (f64)
    st7_export_kernel<double><<<g, 256, 0, st>>>(a, ref_of, out);
  else
    st7_export_kernel<float><<<g, 256, 0, st>>>(a, ref_of, out);
  return cudaGetLastError();
}

cudaError_t st7_launch_import(bool f64, const St7Args& a, const int32_t* ref_of, const double* in, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (a.nq == kQ) {
    if (f64)
      st19_import_kernel<double><<<g, 256, 0, st>>>(a, ref_of, in);
    else
      st19_import_kernel<float><<<g, 256, 0, st>>>(a, ref_of, in);
    return cudaGetLastError();
  }
  if (f64)
    st7_import_kernel<double><<<g, 256, 0, st>>>(a, ref_of, in);
  else
    st7_import_kernel<float><<<g, 256, 0, st>>>(a, ref_of, in);
  return cudaGetLastError();
}

cudaError_t st7_launch_step(bool f64, const St7Args& a, cudaStream_t st) {
  if (a.nq == kQ) return f64 ? st19_launch_step_f64(a, st) : st7_detail::launch_step19<float>(a, st);
  return f64 ? st7_launch_step_f64(a, st) : st7_detail::launch_step<float>(a, st);
}

cudaError_t st7_launch_conc(bool f64, const St7Args& a, double* out, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (a.nq == kQ) {
    if (f64)
      st19_conc_kernel<double><<<g, 256, 0, st>>>(a, out);
    else
      st19_conc_kernel<float><<<g, 256, 0, st>>>(a, out);
    return cudaGetLastError();
  }
  if (f64)
    st7_conc_kernel<double><<<g, 256, 0, st>>>(a, out);
  else
    st7_conc_kernel<float><<<g, 256, 0, st>>>(a, out);
  return cudaGetLastError();
}

cudaError_t st7_launch_init(bool f64, const St7Args& a, cudaStream_t st) {
  if (a.n == 0) return cudaSuccess;
  const int g = (a.n + 255) / 256;
  if (a.nq == kQ) {
    if (f64)
      st19_init_kernel<double><<<g, 256, 0, st>>>(a);
    else
      st19_init_kernel<float><<<g, 256, 0, st>>>(a);
    return cudaGetLastError();
  }
  if (f64)
    st7_init_kernel<double><<<g, 256, 0, st>>>(a);
  else
    st7_init_kernel<float><<<g, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace lbm
