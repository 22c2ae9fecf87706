// Colour-gradient two-phase kernels (reference: MP_3D/Multi_Component_CG_MPI_SPARSE_Software_3DPartition.cpp,
// "CG3").  Included by cg_faithful.cu (FP64, no FMA contraction, reference
// operation order) and cg_fast.cu (FP32 deviation storage).
//
// Per step, two passes over the fluid nodes:
//   colour pass   rho_r(x) = sum of the recoloured red distributions pulled
//                 from the neighbours (the reference's scatter-add of g_r,
//                 CG3:3507-3570, restated as a pull), rho_b likewise,
//                 psi = (rho_r - rho_b)/(rho_r + rho_b)   (CG3:3343-3361)
//   collide pass  pull f; rho, u; colour gradient from psi at x + e_q
//                 (psi_solid at walls); Guo force masked by phase; MRT in
//                 the scaled CG basis with surface-tension terms in m_eq and
//                 psi-interpolated viscosity; equilibrium colour
//                 distributions and recolouring; write f*, g_r, g_b at x.
// Populations live in rows indexed by the single-phase direction order so
// the same pull table (halfway bounce-back resolved) serves f, g_r and g_b;
// the CG velocity order is used for all arithmetic.
#pragma once

#include "cg_api.h"
#include "cg_basis.h"
#include "kernels_common.cuh"

namespace lbm {

// flat index of node x's pulled slot for storage row q
__device__ __forceinline__ size_t cg_slot(const int32_t* __restrict__ table, int npad, int x, int q) {
  return q == 0 ? (size_t)x : (size_t)__ldg(table + (size_t)(q - 1) * npad + x);
}

}  // namespace lbm
