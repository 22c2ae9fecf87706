// Colour-gradient kernels in FP64 with the reference's operation order
// (compiled with -fmad=false): populations, psi, rho_r, rho_b bit-identical
// to the reference colour-gradient solver.
#include "cg_api.h"
#include "cg_kernels_impl.cuh"

namespace lbm {

__constant__ double c_MIcg[kQ * kQ];

template <>
__device__ __forceinline__ double cg_mi<true>(int q, int j) {
  return c_MIcg[q * kQ + j];
}

cudaError_t cg_set_mi_f64(const double* mi, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_MIcg, mi, sizeof(double) * kQ * kQ, 0, cudaMemcpyHostToDevice, st);
}

cudaError_t cg_colour_f64(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_colour_kernel<true><<<(a.n + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t cg_collide_f64(const CgArgs& a, cudaStream_t st) {
  if (a.n > 0) cg_collide_kernel<true><<<(a.n + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// Constant-phase faces (in_psi_BC = 1 with psi_* = 1, CG3:3386-3620): after
// the colour pass every listed face node takes back its initial phase,
// rho_r = (psi0 + 1)/2 and rho_b = 1 - rho_r.
template <typename T>
__global__ void cg_phase_faces_kernel(const int32_t* __restrict__ nodes, const double* __restrict__ psi0, int nface,
                                      T* __restrict__ psi, T* __restrict__ rho_r, T* __restrict__ rho_b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nface) return;
  const int x = nodes[i];
  const double v = psi0[i];
  const double rr = (v * 1.0 + 1.0) / 2;
  psi[x] = (T)v;
  rho_r[x] = (T)rr;
  rho_b[x] = (T)(1.0 - rr);
}

cudaError_t cg_phase_faces(bool f64, const int32_t* nodes, const double* psi0, int nface, void* psi, void* rho_r,
                           void* rho_b, cudaStream_t st) {
  if (nface <= 0) return cudaSuccess;
  const int g = (nface + 255) / 256;
  if (f64)
    cg_phase_faces_kernel<double><<<g, 256, 0, st>>>(nodes, psi0, nface, (double*)psi, (double*)rho_r,
                                                     (double*)rho_b);
  else
    cg_phase_faces_kernel<float><<<g, 256, 0, st>>>(nodes, psi0, nface, (float*)psi, (float*)rho_r, (float*)rho_b);
  return cudaGetLastError();
}

cudaError_t cg_reduce_f64(const CgReduceArgs& a, int nblocks, cudaStream_t st) {
  cg_reduce_kernel<true><<<nblocks, 256, 0, st>>>(a);
  cg_reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nblocks, a.result);
  if (a.partials2) reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials2, nblocks, a.result2);
  return cudaGetLastError();
}

}  // namespace lbm
