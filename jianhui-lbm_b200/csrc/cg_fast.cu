// Colour-gradient kernels in FP32: f stored as deviations f - w, FP32
// arithmetic, colour sums in direction order.
#include "cg_api.h"
#include "cg_kernels_impl.cuh"

namespace lbm {

__constant__ float c_MIcg_f[kQ * kQ];

template <>
__device__ __forceinline__ float cg_mi<false>(int q, int j) {
  return c_MIcg_f[q * kQ + j];
}

cudaError_t cg_set_mi_f32(const double* mi, cudaStream_t st) {
  float m[kQ * kQ];
  for (int i = 0; i < kQ * kQ; i++) m[i] = (float)mi[i];
  const cudaError_t e = cudaMemcpyToSymbolAsync(c_MIcg_f, m, sizeof(m), 0, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);  // m is a host temporary
}

cudaError_t cg_colour_f32(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_colour_kernel<false><<<(a.n + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t cg_collide_f32(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_collide_kernel<false><<<(a.n + 255) / 256, 256, 0, st>>>(a);
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

cudaError_t cg_reduce_f32(const CgReduceArgs& a, int nblocks, cudaStream_t st) {
  cg_reduce_kernel<false><<<nblocks, 256, 0, st>>>(a);
  cg_reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nblocks, a.result);
  return cudaGetLastError();
}

}  // namespace lbm
