// lbm_b200_compat.hpp — the reference's C++ host names over the C ABI of
// lbm_b200.h, so that the reference's callers (main.cpp and its kin) compile
// against this library with their own spelling.  Header-only, no state.
//
//   decomposition / set_move_decomp / slice_chunk  decomposition.cpp:17-161
//   inverseMRT(vector<vector<float>>&, ...)         inverseMRT.cpp:8
//   initialize / runSimulation                      initialize.cpp:23,
//                                                   runSimulation.cpp:22,
//                                                   kernel.cuh:16
// The Poplar versions of initialize/runSimulation take a Graph and Tensors
// that cannot cross a C ABI; here they take the domain handle that owns the
// device tensors.  Errors throw lbm_b200::Error (the reference calls exit()).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "lbm_b200.h"

namespace lbm_b200 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline int check(int rc) {
  if (rc < 0) throw Error(rc, lbm_last_error());
  return rc;
}

// RAII owner of one resident domain.
class Domain {
 public:
  explicit Domain(const Inputval& in, const lbm_options* opt = nullptr) {
    check(lbm_create(&in, opt, &d_));
  }
  ~Domain() {
    if (d_) lbm_destroy(d_);
  }
  Domain(const Domain&) = delete;
  Domain& operator=(const Domain&) = delete;
  lbm_domain* get() const { return d_; }

 private:
  lbm_domain* d_ = nullptr;
};

}  // namespace lbm_b200

inline int decomposition(Inputval* pinput, int Slice[][DIMENSION][2]) {
  return lbm_b200::check(lbm_decomposition(pinput, Slice));
}

inline int set_move_decomp(const int NTILE, const int Slice[][DIMENSION][2],
                           int Move[][DIRECTION_SIZE]) {
  return lbm_b200::check(lbm_set_move_decomp(NTILE, Slice, Move));
}

inline int slice_chunk(const unsigned tile, const int Slice[][DIMENSION][2], int* xs, int* xe,
                       int* ys, int* ye, int* zs, int* ze, int* chunk_nx, int* chunk_ny,
                       int* chunk_nz, int* chunk_len) {
  return lbm_slice_chunk(tile, Slice, xs, xe, ys, ye, zs, ze, chunk_nx, chunk_ny, chunk_nz,
                         chunk_len);
}

inline void inverseMRT(std::vector<std::vector<float>>& matori,
                       std::vector<std::vector<float>>& pInvMat) {
  float a[DIRECTION_SIZE * DIRECTION_SIZE], inv[DIRECTION_SIZE * DIRECTION_SIZE];
  for (int i = 0; i < DIRECTION_SIZE; ++i)
    for (int j = 0; j < DIRECTION_SIZE; ++j) a[i * DIRECTION_SIZE + j] = matori[i][j];
  lbm_b200::check(lbm_inverse_mrt(a, inv));
  pInvMat.assign(DIRECTION_SIZE, std::vector<float>(DIRECTION_SIZE));
  for (int i = 0; i < DIRECTION_SIZE; ++i)
    for (int j = 0; j < DIRECTION_SIZE; ++j) pInvMat[i][j] = inv[i * DIRECTION_SIZE + j];
}

// The Initialize program on the domain (node types, masks, equilibrium).
inline void initialize(Inputval* /*pinput*/, lbm_b200::Domain& d) {
  lbm_b200::check(lbm_initialize(d.get()));
}

// Repeat(maxitr, runSimulation program): pinput->maxitr fused steps.
inline void runSimulation(Inputval* pinput, lbm_b200::Domain& d) {
  lbm_b200::check(lbm_run_simulation(d.get(), pinput->maxitr));
}
