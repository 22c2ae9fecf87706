// Diagnostics reduction that allocates nothing (lbm_reduce_noalloc).
//
// For callers that own all device memory and may not allocate any: a host
// framework that hands its own arena or pool to every library it calls, code
// running inside a region where cudaMalloc is forbidden or would synchronise
// the device, or an embedding that must keep its memory footprint fixed.
// They pass their own device arrays in and a device buffer for the result;
// the only scratch the reduction needs -- one row of partial sums per tile
// of nodes -- is the file-scope array below, which every GPU that loads the
// library holds (512 KiB) until the process exits.
//
// Compiled with -fmad=false, like the bit-exact FP64 kernel, so the macro
// step and the per-node sums are the same operations as lbm_reduce's.
#include "kernels_common.cuh"

namespace lbm {

namespace {

constexpr int kTileThreads = 256;
constexpr int kNodesPerThread = 8;
constexpr int kTileNodes = kTileThreads * kNodesPerThread;  // 2048 nodes per tile
constexpr int kMaxTiles = 8192;                             // 16,777,216 nodes

// One row of 8 partial sums per tile.  Every launch writes the rows of all the
// tiles it uses before the final pass reads them, so nothing has to start at
// zero; the contents left by the previous call are simply overwritten.
static __device__ __align__(256) double g_tile_partials[kMaxTiles * 8];

__global__ void __launch_bounds__(kTileThreads)
    tile_reduce_kernel(const double* __restrict__ f, const double* __restrict__ u_prev, int n, int stride,
                       int skip_node, double hgx, double hgy, double hgz, double* __restrict__ partials) {
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int base = blockIdx.x * kTileNodes;
  for (int k = 0; k < kNodesPerThread; k++) {
    const int p = base + k * kTileThreads + threadIdx.x;
    if (p >= n) break;
    double fl[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) fl[q] = f[(size_t)q * stride + p];
    double rho, ux, uy, uz;
    macro_faithful(fl, hgx, hgy, hgz, rho, ux, uy, uz);
    double px = ux, py = uy, pz = uz;
    if (u_prev) {
      px = u_prev[p];
      py = u_prev[(size_t)stride + p];
      pz = u_prev[2 * (size_t)stride + p];
    }
    if (p != skip_node) {
      const double u2 = ux * ux + uy * uy + uz * uz;
      acc[0] += (ux - px) * (ux - px) + (uy - py) * (uy - py) + (uz - pz) * (uz - pz);
      acc[1] += u2;
      acc[2] += sqrt(u2);
      acc[3] = fmax(acc[3], u2);
    }
    acc[4] += ux;
    acc[5] += uy;
    acc[6] += uz;
    acc[7] += rho;
  }
  block_reduce8(acc, partials + (size_t)blockIdx.x * 8, smem);
}

__global__ void __launch_bounds__(1024)
    tile_final_kernel(const double* __restrict__ partials, int ntiles, double* __restrict__ result) {
  __shared__ double smem[8 * 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < ntiles; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < 8; i++)
      acc[i] = (i == 3) ? fmax(acc[i], partials[(size_t)b * 8 + i]) : acc[i] + partials[(size_t)b * 8 + i];
  block_reduce8(acc, result, smem);
}

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, never a device address, so every
// call looks the address up on the device that is current (the first lookup on
// a device also loads this library's kernels there).  The lookup allocates
// nothing and is cheap once the module is loaded; not caching it keeps the
// address valid after cudaDeviceReset recreates the device's context.
lbm_status scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(LBM_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_tile_partials);
  if (e != cudaSuccess)
    return fail(LBM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return LBM_OK;
}

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" LBM_API lbm_status lbm_reduce_noalloc(const double* f_dev, const double* u_prev_dev, int n, int stride,
                                                 int skip_node, double gx, double gy, double gz, double* result_dev,
                                                 void* stream) {
  if (!f_dev || !result_dev) return fail(LBM_ERR_ARG, "lbm_reduce_noalloc: null device pointer");
  if (n <= 0) return fail(LBM_ERR_ARG, "lbm_reduce_noalloc: n must be positive");
  if (n > kMaxTiles * kTileNodes)
    return fail(LBM_ERR_ARG, "lbm_reduce_noalloc: n = " + std::to_string(n) + " exceeds the " +
                                 std::to_string(kMaxTiles * kTileNodes) +
                                 "-node limit of its static scratch; use lbm_reduce on a handle instead");
  if (stride < n) return fail(LBM_ERR_ARG, "lbm_reduce_noalloc: stride must be >= n");
  double* scratch = nullptr;
  lbm_status st = scratch_address(&scratch);
  if (st != LBM_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int ntiles = (n + kTileNodes - 1) / kTileNodes;
  tile_reduce_kernel<<<ntiles, kTileThreads, 0, s>>>(f_dev, u_prev_dev, n, stride, skip_node, gx / 2, gy / 2, gz / 2,
                                                      scratch);
  tile_final_kernel<<<1, 1024, 0, s>>>(scratch, ntiles, result_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("lbm_reduce_noalloc launch: ") + cudaGetErrorString(e));
  return LBM_OK;
}
