// Sums of the velocity over axis-aligned boxes of cells: the flux sums of
// Comput_Perm's window (SP3:3559-3590), Comput_Grop_Perm's cubes
// (SP:4886-5091) and Comput_Perm_LOCAL's plane (SP:4831-4884).
//
// A dense cell -> internal node index map (-1 for solid) turns a box into a
// contiguous range of cell numbers per (y, z) row; each box is split into a
// fixed number of chunks, each chunk is one block that sums its cells in a
// fixed pattern and a fixed tree, and a final pass adds the chunks of a box in
// order: the result depends only on the box, not on timing.
#include "kernels_common.cuh"

namespace lbm {

namespace {

constexpr int kBoxThreads = 256;

struct BoxArgs {
  const int32_t* cell_idx;  // [nx*ny*nz] x fastest, -1 = solid
  const double* u;          // [3][npad] internal order
  const int32_t* boxes;     // [nbox][6] xn, xp, yn, yp, zn, zp (inclusive, inside the grid)
  int nbox, chunks, nx, ny, npad;
  double* partials;         // [nbox][chunks][8]
  double* out;              // [nbox][4]
};

__global__ void __launch_bounds__(kBoxThreads) box_chunk_kernel(BoxArgs a) {
  __shared__ double smem[8 * 32];
  const int box = blockIdx.y, chunk = blockIdx.x;
  const int32_t* bx = a.boxes + (size_t)box * 6;
  const long long lx = bx[1] - bx[0] + 1, ly = bx[3] - bx[2] + 1, lz = bx[5] - bx[4] + 1;
  const long long cells = lx * ly * lz;
  const long long per = (cells + a.chunks - 1) / a.chunks;
  const long long c0 = (long long)chunk * per, c1 = c0 + per < cells ? c0 + per : cells;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long c = c0 + threadIdx.x; c < c1; c += kBoxThreads) {
    const long long i = bx[0] + c % lx, j = bx[2] + (c / lx) % ly, k = bx[4] + c / (lx * ly);
    const int p = a.cell_idx[i + (long long)a.nx * (j + (long long)a.ny * k)];
    if (p >= 0) {
      v[0] += a.u[p];
      v[1] += a.u[(size_t)a.npad + p];
      v[2] += a.u[2 * (size_t)a.npad + p];
      v[3] += 1.0;
    }
  }
  block_reduce8<-1>(v, a.partials + ((size_t)box * a.chunks + chunk) * 8, smem);
}

__global__ void box_final_kernel(BoxArgs a) {
  const int box = blockIdx.x * blockDim.x + threadIdx.x;
  if (box >= a.nbox) return;
  double s[4] = {0, 0, 0, 0};
  for (int c = 0; c < a.chunks; c++)
    for (int i = 0; i < 4; i++) s[i] += a.partials[((size_t)box * a.chunks + c) * 8 + i];
  for (int i = 0; i < 4; i++) a.out[(size_t)box * 4 + i] = s[i];
}

}  // namespace

cudaError_t launch_box_sums(const int32_t* cell_idx, const double* u, int npad, int nx, int ny, const int32_t* boxes,
                            int nbox, int chunks, double* partials, double* out, cudaStream_t st) {
  if (nbox <= 0) return cudaSuccess;
  BoxArgs a{cell_idx, u, boxes, nbox, chunks, nx, ny, npad, partials, out};
  box_chunk_kernel<<<dim3(chunks, nbox), kBoxThreads, 0, st>>>(a);
  box_final_kernel<<<(nbox + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace lbm
