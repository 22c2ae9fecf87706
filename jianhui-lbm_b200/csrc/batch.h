// Node-pool structures shared by the batch / server host code and kernels.
#pragma once

#include "lbm_internal.h"

namespace lbm {

constexpr int kTile = 512;  // nodes per tile; step block sizes 128/256/512 divide it

// Constants of one instance slot (written at admission).
struct InstParams {
  int begin, end;            // node range [begin, end) in the pool
  int tile_begin, tile_end;  // tile range
  float s_v, s_o;
  float g[3];
  float u0[3];
  float fp16_scale;
  double volume;             // nx*ny*nz (whole-box window)
  double porosity;
  double nu;
};

// Evolving per-slot state, updated on the device at every check.
struct InstState {
  double uave, uave_prev, mass;
  double q[3];
  long long steps;
  int checks;
  int active;  // stepping
  int fresh;   // admitted in this chain: first step takes rho = 1, u = u0
  int done;    // 0 running, 1 converged, 2 step cap, 3 non-finite
};

// One stepping tile of a chain, written by the list kernel so that a step
// block needs one broadcast load before its population gathers.
struct TileWork {
  int p0, end;  // first node of the tile; end of its instance's node range
  float g[3];
  float s_v, s_o;
  float fp16_scale;
  float u0[3];
  int fresh;    // first step of a newly admitted instance: rho = 1, u = u0
};

struct BatchStepArgs {
  const void* src_pop;
  void* dst_pop;
  const int32_t* table;
  int cap;     // pool nodes (row stride)
  int ntiles;  // cap / kTile
  const int* tile_inst;
  const InstParams* inst;
  const InstState* state;
  const int* active_tiles;  // tiles of stepping slots, slot by slot
  const int* n_active;      // its length (device scalar)
  const TileWork* work;     // [n_active] per stepping tile
};

struct BatchReduceArgs {
  const void* pop;
  const int32_t* table;
  int cap;
  int ntiles;
  const int* tile_inst;
  const InstParams* inst;
  InstState* state;
  int nslots;
  double* tile_partials;  // [ntiles][8]
  int* active_tiles;
  int* n_active;
  TileWork* work;
  int* slot_off;  // [nslots + 1] first list entry of each slot's stepping tiles
};

// Rebuilds the work list from the slot states: the stepping slots' tiles,
// then empty entries up to the tiles a step grid of step_grid blocks covers.
cudaError_t launch_batch_list(const BatchReduceArgs& a, int step_grid, int block, cudaStream_t st);

cudaError_t launch_batch_step(Store kind, const BatchStepArgs& a, int block, int grid, int chain_step,
                              cudaStream_t st);
cudaError_t launch_batch_check(Store kind, const BatchReduceArgs& a, int chain_len, double tol, long long max_steps,
                               cudaStream_t st);
cudaError_t launch_batch_export_macro(Store kind, const void* pop, const int32_t* table, int cap, int begin, int n,
                                      const int32_t* ref_of, const InstParams& ip, double* rho, double* u,
                                      cudaStream_t st);
cudaError_t launch_batch_init(Store kind, void* pop, const int32_t* table, int cap, int begin, int n,
                              const InstParams& ip, cudaStream_t st);
// Largest step grid of a pool: one block per tile of the pool (a block steps
// its tile in kTile / block passes).
int batch_step_grid(int ntiles, int block);

// The 18 table rows [18][g.count] of one instance placed at node `begin` of a
// pool with row stride `cap` (flat pool indices q*cap + begin + m).
void fill_pool_rows(const uint8_t* mask, const Geometry& g, int64_t cap, int begin, int32_t* rows);

}  // namespace lbm
