// Test infrastructure: a second build of the colour-gradient program whose
// clock-seeded random numbers (srand(time(0)+rank) before its random initial
// phase and at the start of every macro step, rand() % 10000 per draw) come
// from a fixed-seed generator, so that its random options can be pinned.
// The generator is the one the library documents for the same options:
// draw k after the last srand is the splitmix64 output (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", 2014) of the
// state seed + (k + 1) * 0x9E3779B97F4A7C15, shifted right by 33 bits (a
// 31-bit non-negative int, as rand() returns).  srand() only restarts the
// draw count: the seed is fixed here (LBM_FIXTURE_SEED), not taken from the
// clock.
#pragma once
#include <cstdint>
#include <cstdlib>

#ifndef LBM_FIXTURE_SEED
#define LBM_FIXTURE_SEED 20261203ULL
#endif

static uint64_t lbm_fixture_draws = 0;

static inline int lbm_fixture_rand() {
  uint64_t z = (uint64_t)LBM_FIXTURE_SEED + (lbm_fixture_draws + 1) * 0x9E3779B97F4A7C15ULL;
  lbm_fixture_draws++;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (int)(z >> 33);
}

static inline void lbm_fixture_srand(unsigned) { lbm_fixture_draws = 0; }

#define rand lbm_fixture_rand
#define srand lbm_fixture_srand
