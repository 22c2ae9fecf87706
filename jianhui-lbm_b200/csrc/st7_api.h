// Host-visible structures and launchers of the D3Q7 solute kernels.
#pragma once

#include "lbm_internal.h"

namespace lbm {

struct St7Args {
  const void* src;        // [6][npad] post-collision g of the previous step
  void* dst;              // [6][npad]
  const int32_t* table;   // D3Q19 pull table [18][npad]; rows 0..5 used
  const void* u;          // [3][npad] advecting velocity
  const void* c_given;    // [npad] C for the first step after init, else null
  void* c_out;            // optional [npad]: C of this step's macro
  int n, npad;
  double tau_s;
  double c2, c4;          // lat_c^2 and lat_c^4 of the D3Q19 equilibrium (1 on the default lattice)
  int nq;                 // 7 (D3Q7, g as [6][npad]) or 19 (D3Q19, g as [19][npad])
};

cudaError_t st7_launch_step(bool f64, const St7Args& a, cudaStream_t st);
cudaError_t st7_launch_step_f64(const St7Args& a, cudaStream_t st);  // st7_faithful.cu, -fmad=false
cudaError_t st19_launch_step_f64(const St7Args& a, cudaStream_t st);  // st7_faithful.cu, -fmad=false
cudaError_t st7_launch_conc(bool f64, const St7Args& a, double* out, cudaStream_t st);
cudaError_t st7_launch_init(bool f64, const St7Args& a, cudaStream_t st);
// a.src: the state to export; a.dst: the buffer the next step pulls from
cudaError_t st7_launch_export(bool f64, const St7Args& a, const int32_t* ref_of, double* out, cudaStream_t st);
cudaError_t st7_launch_import(bool f64, const St7Args& a, const int32_t* ref_of, const double* in, cudaStream_t st);

}  // namespace lbm
