// Device side of the pressure/velocity faces (boundary_pressure SP3:2656-3116,
// boundary_velocity SP3:2450-2655), shared by the FP64 bit-exact translation
// unit (compiled with -fmad=false) and the deviation-storage one.
//
// The reference overwrites the post-streaming populations F of face nodes
// after streaming and before the macro step, from the previous step's f, rho,
// u of neighbouring nodes.  Here the step kernel leaves face nodes to
// bc_kernel, and every node a rule reads records its post-streaming state
// (after its own rules) and macro fields in a [23][nsnap] double array, ping-
// ponged with the populations; the next step's rules read that record.
#pragma once

#include "kernels_common.cuh"

namespace lbm {

// `feq` (SP3:1382-1394) in the reference's operation order: on the default
// lattice lat_c = c2 = c4 = 1, on a self-defined one (L.on) elat = e lat_c and
// the divisions by c2, c4.  The deviation-storage kernels pass the default
// lattice: their velocities are in units of lat_c, where the two agree.
__device__ __forceinline__ double bc_feq(int q, double rho, double ux, double uy, double uz, const Lattice& L) {
  const double uv = ux * ux + uy * uy + uz * uz;
  if (L.on) {
    const double ex = (double)cx(q) * L.c, ey = (double)cy(q) * L.c, ez = (double)cz(q) * L.c;
    const double eu = ex * ux + ey * uy + ez * uz;
    return weight(q) * rho * (1.0 + 3.0 * eu / L.c2 + 4.5 * eu * eu / L.c4 - 1.5 * uv / L.c2);
  }
  const double c2 = 1.0, c4 = 1.0;
  const double eu = (double)cx(q) * ux + (double)cy(q) * uy + (double)cz(q) * uz;
  return weight(q) * rho * (1.0 + 3.0 * eu / c2 + 4.5 * eu * eu / c4 - 1.5 * uv / c2);
}

__device__ __forceinline__ void snap_write(double* snap, int nsnap, int slot, const double (&f)[kQ], double rho,
                                           double ux, double uy, double uz) {
  const size_t ns = (size_t)nsnap, s = (size_t)slot;
#pragma unroll
  for (int q = 0; q < kQ; q++) snap[q * ns + s] = f[q];
  snap[kQ * ns + s] = rho;
  snap[(kQ + 1) * ns + s] = ux;
  snap[(kQ + 2) * ns + s] = uy;
  snap[(kQ + 3) * ns + s] = uz;
}

// The rules of face node b (index b = p - n_main) applied in program order to
// its post-streaming populations F, with the equilibria of lattice L.
__device__ __forceinline__ void bc_apply(const BcArgs& a, int b, double (&F)[kQ], const Lattice& L) {
  const double* __restrict__ S = a.snap_src;
  const size_t ns = (size_t)a.s.nsnap;
  const int o1 = a.op_off[b + 1];
  for (int o = a.op_off[b]; o < o1; o++) {
    const BcOp op = a.ops[o];
    const double rb = a.face_rho[op.face];
    const double ubx = a.face_u[op.face][0], uby = a.face_u[op.face][1], ubz = a.face_u[op.face][2];
    const size_t nb = (size_t)(op.nb < 0 ? 0 : op.nb);
    switch (op.kind) {
      case kBcPressureRest:
#pragma unroll
        for (int q = 0; q < kQ; q++) F[q] = bc_feq(q, rb, 0.0, 0.0, 0.0, L);
        break;
      case kBcPressureNbU: {
        const double ux = S[(kQ + 1) * ns + nb], uy = S[(kQ + 2) * ns + nb], uz = S[(kQ + 3) * ns + nb];
#pragma unroll
        for (int q = 0; q < kQ; q++) F[q] = bc_feq(q, rb, ux, uy, uz, L);
        break;
      }
      case kBcPressureMoment: {
        double fn[kQ], m[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) fn[q] = S[q * ns + nb];
#pragma unroll
        for (int i = 0; i < kQ; i++) {
          double acc = 0;
#pragma unroll
          for (int j = 0; j < kQ; j++) acc = acc + (double)mcoef(i, j) * fn[j];
          m[i] = acc;
        }
        m[0] = rb;
#pragma unroll
        for (int i = 0; i < kQ; i++) {
          double acc = 0;
#pragma unroll
          for (int j = 0; j < kQ; j++) acc = acc + a.mi[i * kQ + j] * m[j];
          F[i] = acc;
        }
        break;
      }
      case kBcPressureNeq: {
        const double ux = S[(kQ + 1) * ns + nb], uy = S[(kQ + 2) * ns + nb], uz = S[(kQ + 3) * ns + nb];
        const double rn = S[kQ * ns + nb];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
          const double f4 = op.nb4 >= 0 ? S[q * ns + (size_t)op.nb4] : 0.0;
          F[q] = bc_feq(q, rb, ux, uy, uz, L) + f4 - bc_feq(q, rn, ux, uy, uz, L);
        }
        break;
      }
      case kBcVelocityEq:
#pragma unroll
        for (int q = 0; q < kQ; q++) F[q] = bc_feq(q, 1.0, ubx, uby, ubz, L);
        break;
      case kBcVelocityNeq:
#pragma unroll
        for (int q = 0; q < kQ; q++) {
          const int e = op.axis == 0 ? cx(q) : (op.axis == 1 ? cy(q) : cz(q));
          if (op.sign > 0 ? e < 0 : e > 0)
            F[q] = bc_feq(opp(q), 1.0, ubx, uby, ubz, L) - F[opp(q)] + bc_feq(q, 1.0, ubx, uby, ubz, L);
        }
        break;
      case kBcVelocityNbRho: {
        const double rn = S[kQ * ns + nb];
#pragma unroll
        for (int q = 0; q < kQ; q++) F[q] = bc_feq(q, rn, ubx, uby, ubz, L);
        break;
      }
      default:
        break;
    }
  }
}

}  // namespace lbm
