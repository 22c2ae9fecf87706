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

cudaError_t cg_reduce_f64(const CgReduceArgs& a, int nblocks, cudaStream_t st) {
  cg_reduce_kernel<true><<<nblocks, 256, 0, st>>>(a);
  cg_reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nblocks, a.result);
  if (a.partials2) reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials2, nblocks, a.result2);
  return cudaGetLastError();
}

}  // namespace lbm
