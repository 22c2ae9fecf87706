// Device-side indexing of a geometry (reference node order).
#pragma once

#include "lbm_internal.h"

namespace lbm {

// Reusable device scratch for indexing: the mask, a per-cell id array, the
// prefix-sum workspace and the node -> cell map of the last indexed geometry.
struct SetupScratch {
  uint8_t* mask = nullptr;
  int32_t* cell_id = nullptr;
  void* temp = nullptr;
  int32_t* coor_x = nullptr;  // node -> x-fastest cell index
  long long cells_cap = 0;
  int coor_cap = 0;
  size_t temp_bytes = 0;
  bool borrowed = false;  // the arrays live in a caller's buffer (see borrow)
  ~SetupScratch() { release(); }
  lbm_status reserve(long long cells, int nodes);
  // Places the arrays in [base, base + bytes) of a device buffer that is not
  // in use until the indexing has finished (a solver's second population
  // array), saving their allocation and release; false when they do not fit
  // (then reserve allocates them).
  bool borrow(void* base, size_t bytes, long long cells, int nodes);
  void release();
};

// Uploads the host mask, numbers its pore cells in x-fastest order (the
// reference order) and writes the 18 pull-table rows of those `count` nodes at
// table + (q-1)*stride + begin, with flat indices q*stride + begin + m.
// ref_of_out (optional) receives 1..count (internal index -> reference id).
lbm_status device_index_reference(const uint8_t* host_mask, int nx, int ny, int nz, int count, int32_t* table,
                                  long long stride, int begin, int32_t* ref_of_out, SetupScratch& s,
                                  cudaStream_t st);
// Reference coor (i*ny*nz + j*nz + k) of the last indexed geometry.
lbm_status device_ref_coor(int nx, int ny, int nz, int count, const SetupScratch& s, int32_t* d_out,
                           cudaStream_t st);

}  // namespace lbm
