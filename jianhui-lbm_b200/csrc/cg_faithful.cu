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

// Faces whose value copies another node's phase of this macro step (face
// flag 2): every value is read (the node's psi before any face rule, or a
// constant) before any face node is written, since a copied node may itself
// be a face node.
template <typename T>
__global__ void cg_phase_faces_gather_kernel(const int32_t* __restrict__ src, const double* __restrict__ val,
                                             int nface, const T* __restrict__ psi, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nface) return;
  const int s = src[i];
  out[i] = s >= 0 ? (double)psi[s] : val[i];
}

cudaError_t cg_phase_faces_gather(bool f64, const int32_t* src, const double* val, int nface, const void* psi,
                                  double* out, cudaStream_t st) {
  if (nface <= 0) return cudaSuccess;
  const int g = (nface + 255) / 256;
  if (f64)
    cg_phase_faces_gather_kernel<double><<<g, 256, 0, st>>>(src, val, nface, (const double*)psi, out);
  else
    cg_phase_faces_gather_kernel<float><<<g, 256, 0, st>>>(src, val, nface, (const float*)psi, out);
  return cudaGetLastError();
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

// ------------------------------------------------- pressure/velocity faces
// boundary_pressure (CG3:4221-4682) and boundary_velocity (CG3:4026-4220)
// act on the post-streaming populations F of the face nodes between
// collision and comput_macro_variables, reading f, rho and u of the previous
// macro step.  Both kernels work on full populations in double in the CG
// direction order with CG3's feq (CG3:2503-2540), M (CG3:63-83), MI and LR.

// feq of the colour-gradient program (CG3:2503-2540): the polynomial it
// computes first is overwritten; the value returned is row k of M^-1 applied
// to the equilibrium moments (rho, u, u u terms with rho_0 = 1), summed from
// j = 0 in the reference's order.
__device__ __forceinline__ double cg_feq(int k, double rho, double ux, double uy, double uz) {
  const double rho_0 = 1.0;
  double meq[kQ];
#pragma unroll
  for (int j = 0; j < kQ; j++) meq[j] = 0.0;
  meq[0] = rho;
  meq[3] = rho_0 * ux;
  meq[5] = rho_0 * uy;
  meq[7] = rho_0 * uz;
  meq[1] = rho_0 * (ux * ux + uy * uy + uz * uz);
  meq[9] = rho_0 * (2 * ux * ux - uy * uy - uz * uz);
  meq[11] = rho_0 * (uy * uy - uz * uz);
  meq[13] = rho_0 * ux * uy;
  meq[14] = rho_0 * uy * uz;
  meq[15] = rho_0 * ux * uz;
  double feq = 0.0;
#pragma unroll
  for (int j = 0; j < kQ; j++) feq = feq + c_MIcg[k * kQ + j] * meq[j];
  return feq;
}

__device__ __forceinline__ int cg_lr(int k) { return k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1); }

// F of node x (CG order, full populations) from its pulled slots.
template <typename T, bool DEV>
__device__ __forceinline__ void cg_pull_full(const T* __restrict__ f, const int32_t* __restrict__ table, int npad,
                                             int x, double (&F)[kQ]) {
#pragma unroll
  for (int k = 0; k < kQ; k++) {
    const double v = (double)f[cg_slot(table, npad, x, cg::row(k))];
    F[k] = DEV ? v + weight(k) : v;
  }
}

// Record pass: f, rho, u of every node a rule reads, as the macro step
// computes them (CG3:3330-3352; u with the pending macro step's force).
template <typename T, bool DEV>
__global__ void __launch_bounds__(128) cg_bc_record_kernel(CgBcArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nsnap) return;
  const int x = a.snap_nodes[i];
  double F[kQ];
  cg_pull_full<T, DEV>(static_cast<const T*>(a.f), a.table, a.npad, x, F);
  double rho, ux, uy, uz;
  if (a.given) {
    rho = 1.0;
    ux = a.u0[0];
    uy = a.u0[1];
    uz = a.u0[2];
  } else {
    double r = F[0];
#pragma unroll
    for (int k = 1; k < kQ; k++) r = r + F[k];
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
    for (int k = 0; k < kQ; k++) {
      if (cg::ex(k) == 1) sx = sx + F[k];
      if (cg::ex(k) == -1) sx = sx - F[k];
      if (cg::ey(k) == 1) sy = sy + F[k];
      if (cg::ey(k) == -1) sy = sy - F[k];
      if (cg::ez(k) == 1) sz = sz + F[k];
      if (cg::ez(k) == -1) sz = sz - F[k];
    }
    rho = r;
    ux = (sx + 1.0 * a.gm[0] / 2.0) / rho;
    uy = (sy + 1.0 * a.gm[1] / 2.0) / rho;
    uz = (sz + 1.0 * a.gm[2] / 2.0) / rho;
  }
  const size_t ns = (size_t)a.nsnap;
#pragma unroll
  for (int k = 0; k < kQ; k++) a.rec[k * ns + i] = F[k];
  a.rec[kQ * ns + i] = rho;
  a.rec[(kQ + 1) * ns + i] = ux;
  a.rec[(kQ + 2) * ns + i] = uy;
  a.rec[(kQ + 3) * ns + i] = uz;
}

// Face pass: the operations of each face node in program order on its pulled
// F, written back to the same slots (each (node, direction) owns one slot).
template <typename T, bool DEV>
__global__ void __launch_bounds__(128) cg_bc_faces_kernel(CgBcArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nface) return;
  const int x = a.nodes[b];
  T* __restrict__ f = static_cast<T*>(a.f);
  const double* __restrict__ S = a.rec;
  const size_t ns = (size_t)a.nsnap;
  // the first operation and the neighbour's recorded rho and u it reads are
  // loaded before the pull, so that their chain of loads (op_off -> ops ->
  // record) overlaps the node's (nodes -> table -> f) instead of following it
  const int o0 = a.op_off[b], o1 = a.op_off[b + 1];
  BcOp first{};
  double p_rn = 0.0, p_ux = 0.0, p_uy = 0.0, p_uz = 0.0;
  if (o0 < o1) {
    first = a.ops[o0];
    if (first.kind == kBcPressureNbU || first.kind == kBcPressureNeq || first.kind == kBcVelocityNbRho) {
      const size_t nb = (size_t)(first.nb < 0 ? 0 : first.nb);  // the rule's recorded neighbour
      p_rn = S[kQ * ns + nb];
      p_ux = S[(kQ + 1) * ns + nb];
      p_uy = S[(kQ + 2) * ns + nb];
      p_uz = S[(kQ + 3) * ns + nb];
    }
  }
  double F[kQ];
  cg_pull_full<T, DEV>(f, a.table, a.npad, x, F);
  for (int o = o0; o < o1; o++) {
    const bool pre = o == o0;
    const BcOp op = pre ? first : a.ops[o];
    const double rb = a.face_rho[op.face];
    const double ubx = a.face_u[op.face][0], uby = a.face_u[op.face][1], ubz = a.face_u[op.face][2];
    const size_t nb = (size_t)(op.nb < 0 ? 0 : op.nb);
    switch (op.kind) {
      case kBcPressureRest:
#pragma unroll
        for (int k = 0; k < kQ; k++) F[k] = cg_feq(k, rb, 0.0, 0.0, 0.0);
        break;
      case kBcPressureNbU: {
        const double ux = pre ? p_ux : S[(kQ + 1) * ns + nb], uy = pre ? p_uy : S[(kQ + 2) * ns + nb],
                     uz = pre ? p_uz : S[(kQ + 3) * ns + nb];
#pragma unroll
        for (int k = 0; k < kQ; k++) F[k] = cg_feq(k, rb, ux, uy, uz);
        break;
      }
      case kBcPressureMoment: {
        double m[kQ];
#pragma unroll
        for (int i = 0; i < kQ; i++) {
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < kQ; j++) acc = acc + (double)cg::mcoef(i, j) * S[j * ns + nb];
          m[i] = acc;
        }
        m[0] = rb;
#pragma unroll
        for (int i = 0; i < kQ; i++) {
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < kQ; j++) acc = acc + c_MIcg[i * kQ + j] * m[j];
          F[i] = acc;
        }
        break;
      }
      case kBcPressureNeq: {
        const double ux = pre ? p_ux : S[(kQ + 1) * ns + nb], uy = pre ? p_uy : S[(kQ + 2) * ns + nb],
                     uz = pre ? p_uz : S[(kQ + 3) * ns + nb];
        const double rn = pre ? p_rn : S[kQ * ns + nb];
#pragma unroll
        for (int k = 0; k < kQ; k++) {
          const double f4 = op.nb4 >= 0 ? S[k * ns + (size_t)op.nb4] : 0.0;
          F[k] = cg_feq(k, rb, ux, uy, uz) + f4 - cg_feq(k, rn, ux, uy, uz);
        }
        break;
      }
      case kBcVelocityEq:
#pragma unroll
        for (int k = 0; k < kQ; k++) F[k] = cg_feq(k, 1.0, ubx, uby, ubz);
        break;
      case kBcVelocityNeq:
#pragma unroll
        for (int k = 0; k < kQ; k++) {
          const int e = op.axis == 0 ? cg::ex(k) : (op.axis == 1 ? cg::ey(k) : cg::ez(k));
          if (op.sign > 0 ? e < 0 : e > 0)
            F[k] = cg_feq(cg_lr(k), 1.0, ubx, uby, ubz) - F[cg_lr(k)] + cg_feq(k, 1.0, ubx, uby, ubz);
        }
        break;
      case kBcVelocityNbRho: {
        const double rn = pre ? p_rn : S[kQ * ns + nb];
#pragma unroll
        for (int k = 0; k < kQ; k++) F[k] = cg_feq(k, rn, ubx, uby, ubz);
        break;
      }
      default:
        break;
    }
  }
#pragma unroll
  for (int k = 0; k < kQ; k++) f[cg_slot(a.table, a.npad, x, cg::row(k))] = (T)(DEV ? F[k] - weight(k) : F[k]);
}

cudaError_t cg_bc_record(bool f64, const CgBcArgs& a, cudaStream_t st) {
  if (a.nsnap <= 0) return cudaSuccess;
  const int g = (a.nsnap + 127) / 128;
  if (f64)
    cg_bc_record_kernel<double, false><<<g, 128, 0, st>>>(a);
  else
    cg_bc_record_kernel<float, true><<<g, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t cg_bc_faces(bool f64, const CgBcArgs& a, cudaStream_t st) {
  if (a.nface <= 0) return cudaSuccess;
  const int g = (a.nface + 127) / 128;
  if (f64)
    cg_bc_faces_kernel<double, false><<<g, 128, 0, st>>>(a);
  else
    cg_bc_faces_kernel<float, true><<<g, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t cg_reduce_f64(const CgReduceArgs& a, int nblocks, cudaStream_t st) {
  cg_reduce_kernel<true><<<nblocks, 256, 0, st>>>(a);
  cg_reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials, nblocks, a.result);
  if (a.partials2) reduce_final_kernel<<<1, 1024, 0, st>>>(a.partials2, nblocks, a.result2);
  return cudaGetLastError();
}

}  // namespace lbm
