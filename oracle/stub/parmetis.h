/*
 * ParMETIS stand-in used ONLY to compile the reference solvers as a one-rank
 * CPU oracle (test infrastructure).  With one rank every vertex belongs to
 * partition 0, which is what ParMETIS_V3_PartKway returns for nparts == 1.
 */
#ifndef ORACLE_STUB_PARMETIS_H
#define ORACLE_STUB_PARMETIS_H

#include "mpi.h"

typedef int idx_t;
typedef float real_t;

static inline int ParMETIS_V3_PartKway(idx_t* vtxdist, idx_t*, idx_t*, idx_t*, idx_t*,
                                       idx_t*, idx_t*, idx_t*, idx_t*, real_t*, real_t*,
                                       idx_t*, idx_t* edgecut, idx_t* part, MPI_Comm*) {
  const idx_t n = vtxdist[1] - vtxdist[0];
  for (idx_t i = 0; i < n; ++i) part[i] = 0;
  if (edgecut) *edgecut = 0;
  return 1;
}

#endif
