// FP64 solute step: the D3Q7 BGK update in the reference's own arithmetic.
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

}  // namespace lbm
