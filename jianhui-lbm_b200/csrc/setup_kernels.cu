// Device-side sparse indexing in the reference order: fluid-node compaction
// (SP3:1018-1071) by a prefix sum over the mask, and the pull table with
// halfway bounce-back (the pull form of nei_loc, SP3:1099-1151) by one thread
// per node.  Moves setup off the host: a 256^3 geometry is indexed in about a
// millisecond after its 16.8 MB mask is uploaded.
#include <cub/device/device_scan.cuh>

#include "setup.h"

namespace lbm {

namespace {

__global__ void pore_flags_kernel(const uint8_t* __restrict__ mask, long long cells, int32_t* __restrict__ flags) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells; c += (long long)gridDim.x * blockDim.x)
    flags[c] = mask[c] == 0;
}

// cell_id holds the exclusive prefix sum of pore flags on entry and the node
// id of each pore cell (-1 for solids) on exit; coor_x[id] = x-fastest cell.
__global__ void compact_kernel(const uint8_t* __restrict__ mask, long long cells, int32_t* __restrict__ cell_id,
                               int32_t* __restrict__ coor_x) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
       c += (long long)gridDim.x * blockDim.x) {
    if (mask[c] == 0)
      coor_x[cell_id[c]] = (int32_t)c;
    else
      cell_id[c] = -1;
  }
}

__global__ void pull_table_kernel(const int32_t* __restrict__ coor_x, const int32_t* __restrict__ cell_id, int n,
                                  int nx, int ny, int nz, int32_t* __restrict__ table, long long stride, int begin) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = coor_x[p];
  const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
#pragma unroll
  for (int q = 1; q < kQ; q++) {
    int ip = i - cx(q), jp = j - cy(q), kp = k - cz(q);
    ip = ip < 0 ? nx - 1 : (ip >= nx ? 0 : ip);
    jp = jp < 0 ? ny - 1 : (jp >= ny ? 0 : jp);
    kp = kp < 0 ? nz - 1 : (kp >= nz ? 0 : kp);
    const int m = cell_id[ip + nx * (jp + ny * kp)];
    const long long s = m >= 0 ? (long long)q * stride + begin + m : (long long)opp(q) * stride + begin + p;
    table[(size_t)(q - 1) * stride + begin + p] = (int32_t)s;
  }
}

__global__ void iota_kernel(int32_t* __restrict__ out, int n, int first) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = first + p;
}

// reference coor (i*ny*nz + j*nz + k) from the x-fastest cell index
__global__ void ref_coor_kernel(const int32_t* __restrict__ coor_x, int n, int nx, int ny, int nz,
                                int32_t* __restrict__ coor_ref) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = coor_x[p];
  const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
  coor_ref[p] = i * ny * nz + j * nz + k;
}

int grid_for(long long items) {
  const long long g = (items + 255) / 256;
  return (int)(g < 148 * 32 ? (g < 1 ? 1 : g) : 148 * 32);
}

}  // namespace

bool SetupScratch::borrow(void* base, size_t bytes, long long cells, int nodes) {
  if (!base || cells_cap || coor_cap || borrowed) return false;
  size_t tb = 0;
  if (cub::DeviceScan::ExclusiveSum(nullptr, tb, (int32_t*)nullptr, (int32_t*)nullptr, (int)cells) != cudaSuccess)
    return false;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t need = up(sizeof(int32_t) * (size_t)cells) + up((size_t)cells) + up(tb) +
                      up(sizeof(int32_t) * (size_t)std::max(nodes, 1));
  if (need > bytes) return false;
  char* p = static_cast<char*>(base);
  cell_id = reinterpret_cast<int32_t*>(p);
  p += up(sizeof(int32_t) * (size_t)cells);
  mask = reinterpret_cast<uint8_t*>(p);
  p += up((size_t)cells);
  temp = p;
  p += up(tb);
  coor_x = reinterpret_cast<int32_t*>(p);
  cells_cap = cells;
  coor_cap = nodes;
  temp_bytes = tb;
  borrowed = true;
  return true;
}

lbm_status SetupScratch::reserve(long long cells, int nodes) {
  if (borrowed) return (cells <= cells_cap && nodes <= coor_cap) ? LBM_OK : fail(LBM_ERR_STATE, "setup scratch too small");
  if (cells > cells_cap) {
    if (cell_id) cudaFree(cell_id);
    cell_id = nullptr;
    LBM_CUDA_TRY(cudaMalloc(&cell_id, sizeof(int32_t) * (size_t)cells));
    if (mask) cudaFree(mask);
    mask = nullptr;
    LBM_CUDA_TRY(cudaMalloc(&mask, (size_t)cells));
    size_t tb = 0;
    LBM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, cell_id, cell_id, (int)cells));
    if (tb > temp_bytes) {
      if (temp) cudaFree(temp);
      temp = nullptr;
      LBM_CUDA_TRY(cudaMalloc(&temp, tb));
      temp_bytes = tb;
    }
    cells_cap = cells;
  }
  if (nodes > coor_cap) {
    if (coor_x) cudaFree(coor_x);
    coor_x = nullptr;
    LBM_CUDA_TRY(cudaMalloc(&coor_x, sizeof(int32_t) * (size_t)nodes));
    coor_cap = nodes;
  }
  return LBM_OK;
}

void SetupScratch::release() {
  if (!borrowed)
    for (void* p : {(void*)cell_id, (void*)mask, temp, (void*)coor_x})
      if (p) cudaFree(p);
  borrowed = false;
  cell_id = nullptr;
  mask = nullptr;
  temp = nullptr;
  coor_x = nullptr;
  cells_cap = 0;
  coor_cap = 0;
  temp_bytes = 0;
}

lbm_status device_index_reference(const uint8_t* host_mask, int nx, int ny, int nz, int count, int32_t* table,
                                  long long stride, int begin, int32_t* ref_of_out, SetupScratch& s,
                                  cudaStream_t st) {
  const long long cells = (long long)nx * ny * nz;
  if (cells > (1LL << 31) - 1) return fail(LBM_ERR_ARG, "geometry exceeds 2^31 cells");
  lbm_status r = s.reserve(cells, count);
  if (r != LBM_OK) return r;
  LBM_CUDA_TRY(cudaMemcpyAsync(s.mask, host_mask, (size_t)cells, cudaMemcpyHostToDevice, st));
  pore_flags_kernel<<<grid_for(cells), 256, 0, st>>>(s.mask, cells, s.cell_id);
  size_t tb = s.temp_bytes;
  LBM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(s.temp, tb, s.cell_id, s.cell_id, (int)cells, st));
  compact_kernel<<<grid_for(cells), 256, 0, st>>>(s.mask, cells, s.cell_id, s.coor_x);
  if (count > 0) {
    pull_table_kernel<<<(count + 255) / 256, 256, 0, st>>>(s.coor_x, s.cell_id, count, nx, ny, nz, table, stride,
                                                          begin);
    if (ref_of_out) iota_kernel<<<(count + 255) / 256, 256, 0, st>>>(ref_of_out, count, 1);
  }
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

lbm_status device_ref_coor(int nx, int ny, int nz, int count, const SetupScratch& s, int32_t* d_out,
                           cudaStream_t st) {
  if (count > 0) ref_coor_kernel<<<(count + 255) / 256, 256, 0, st>>>(s.coor_x, count, nx, ny, nz, d_out);
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

}  // namespace lbm
