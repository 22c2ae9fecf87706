/*
 * Zero-filled array allocation for the reference programs run as oracles
 * (test infrastructure).  Some reference code reads an array before it writes
 * it: the solute program builds its initial populations from the velocity
 * array before it reads the velocity file (Solute_Transport_MPI_Software_
 * Spars_6V.cpp: init at :472 uses u, Backup_input_v at :473 fills it).  With
 * the C library's allocator those values are whatever the heap held; forced
 * to zero here (fresh pages are zero too) so the program is deterministic.
 * Included on the compiler command line (-include), the sources unchanged.
 */
#ifndef ORACLE_ZERO_HEAP_H
#define ORACLE_ZERO_HEAP_H
#include <cstdlib>
#include <new>

inline void* operator new[](std::size_t n) {
  void* p = std::calloc(n ? n : 1, 1);
  if (!p) throw std::bad_alloc();
  return p;
}
inline void operator delete[](void* p) noexcept { std::free(p); }
inline void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

#endif
