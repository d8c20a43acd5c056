/*
 * orc_common.h — TEST INFRASTRUCTURE (the oracle), shared by the oracle
 * port (lbm_oracle.cpp) and the reference-codelet emulator (ref_poplar_emu.cpp).
 *
 * The seeded initial-condition perturbation and the channel inlet profile
 * are additions of this project (the reference has neither); they are
 * defined here once so that both CPU checkers and the GPU library produce
 * bit-identical initial states from integer hashing and exact double
 * arithmetic.  The GPU library restates the same formulas in its own code.
 */
#ifndef ORC_COMMON_H
#define ORC_COMMON_H
#include <stdint.h>

typedef struct orc_ext {
  int init_kind;      /* LBM_INIT_* of lbm_b200.h                        */
  int use_double;     /* 1: run the step in FP64 (the FP64 oracle)         */
  uint64_t seed;
  float noise_amp;
  int split;          /* >1: cut every decomposition tile into `split`     */
                      /* y-slabs (more host threads; results unchanged)    */
  int threads;        /* OpenMP threads, 0 = default                       */
} orc_ext;

static inline uint64_t orc_splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Uniform in [-1, 1) with 24 random bits; every operation is exact in
 * double, so the value is identical on any IEEE-754 machine. */
static inline double orc_unit_noise(uint64_t seed, uint64_t node, uint64_t comp) {
  uint64_t r = orc_splitmix64(seed * 0x9E3779B97F4A7C15ull + node * 4ull + comp);
  return (double)(r >> 40) * (1.0 / 16777216.0) * 2.0 - 1.0;
}

/* Parabolic inlet profile of the channel case,
 * u_x = u_max * 16 * eta(1-eta) * zeta(1-zeta), eta = y/(ny-1),
 * zeta = z/(nz-1) (zero on the wall nodes y,z in {0, n-1}). */
static inline float orc_inlet_profile(float umax, int y, int z, int ny, int nz) {
  double eta = (double)y / (double)(ny - 1);
  double zeta = (double)z / (double)(nz - 1);
  return (float)((double)umax * 16.0 * eta * (1.0 - eta) * zeta * (1.0 - zeta));
}

#endif
