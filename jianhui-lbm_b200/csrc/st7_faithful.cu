// FP64 solute steps: the D3Q7 and D3Q19 BGK updates in the reference's own
// arithmetic.
//
// Compiled with -fmad=false: every a*b+c of the relaxation
// g - (g - C/6 (1 + 3 e.u)) / tau_s (ST7:1464-1471) stays two correctly rounded
// operations, as in the reference program built without FMA contraction, so
// the concentration is bit-identical to it.
#include "st7_kernels.cuh"

namespace lbm {

cudaError_t st7_launch_step_f64(const St7Args& a, cudaStream_t st) {
  return st7_detail::launch_step<double>(a, st);
}

// The D3Q19 solute program's update in its own arithmetic (ST19:1475-1480).
cudaError_t st19_launch_step_f64(const St7Args& a, cudaStream_t st) {
  return st7_detail::launch_step19<double>(a, st);
}

}  // namespace lbm
