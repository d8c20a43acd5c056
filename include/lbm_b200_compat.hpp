// lbm_b200_compat.hpp — the reference's C++ host names over the C ABI of
// lbm_b200.h, so that the reference's callers (main.cpp, and kernel.cu's
// callers through kernel.cuh) compile against this library with their own
// spelling.  Header-only.
//
//   decomposition / set_move_decomp / slice_chunk  decomposition.cpp:17-161
//   inverseMRT(vector<vector<float>>&, ...)         inverseMRT.cpp:8
//   HostNodeData, DeviceNodeData, MRTMatrix,
//   LBMSolver                                       struct.h:8-76
//   initialize(Inputval*, LBMSolver*)               the icycle == 0 branch of
//                                                   kernel.cu:156-164 (and
//                                                   initialize.cpp:23)
//   runSimulation(Inputval*, LBMSolver*)            kernel.cuh:16, kernel.cu:18
//   saveFile(Inputval*, LBMSolver*, arIndex, type)  kernel.cuh:14, kernel.cu:699
//   initialize / runSimulation (Domain&)            initialize.cpp:23,
//                                                   runSimulation.cpp:22 +
//                                                   main.cpp:290-291 Repeat
// The Poplar programs take a Graph and Tensors, which cannot cross a C ABI;
// their overloads here take the domain handle that owns the device state.
// Errors throw lbm_b200::Error (the reference calls exit()).
//
// LBMSolver keeps the reference's member names.  The tables are filled at
// construction (main.cpp:87-146); m_pDomain (an addition) is the library
// handle, created by initialize / runSimulation and freed by the destructor
// (the reference never frees its device memory, main.cpp:29-33).
// m_DeviceNode points at the library's device arrays of the macroscopic
// state (lbm_device_fields) after each call; m_arF / m_arFTemp /
// m_nNodeType / m_nDirectionState stay NULL: the populations live in the
// library's private layout (read them with lbm_export_arF) and node types
// are computed in the kernels (lbm_get_node_info returns them).  m_HostNode
// is filled where kernel.cu fills it: the macroscopic fields and node types
// before each result file, the densities before each residual line.
#pragma once
#include <cmath>
#include <cstdio>
#include <filesystem>
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

#ifndef LBM_B200_NO_SOLVER_TYPES
// struct.h:8-28
typedef struct HostNodeData {
  std::vector<float> m_arF;
  std::vector<float> m_arFTemp;
  std::vector<float> m_dCurrDen;
  std::vector<float> m_dPrevDen;
  std::vector<float> m_dCurrVelx;
  std::vector<float> m_dCurrVely;
  std::vector<float> m_dCurrVelz;
  std::vector<float> m_dPrevVelx;
  std::vector<float> m_dPrevVely;
  std::vector<float> m_dPrevVelz;
  std::vector<int> m_nNodeType;
  std::vector<float> m_dTauEddy;
} HostNodeData;

// struct.h:30-50
typedef struct DeviceNodeData {
  float* m_arF;
  float* m_arFTemp;
  float* m_dCurrDen;
  float* m_dPrevDen;
  float* m_dCurrVelx;
  float* m_dCurrVely;
  float* m_dCurrVelz;
  float* m_dPrevVelx;
  float* m_dPrevVely;
  float* m_dPrevVelz;
  float* m_dTauEddy;
  int* m_nNodeType;
  int* m_nDirectionState;
} DeviceNodeData;

// struct.h:52-56
struct MRTMatrix {
  float m_MatMRT[DIRECTION_SIZE][DIRECTION_SIZE];
  float m_MatInv[DIRECTION_SIZE][DIRECTION_SIZE];
};

// struct.h:58-76 (m_pDomain added)
class LBMSolver {
 public:
  LBMSolver() {
    float dir[DIMENSION * DIRECTION_SIZE];
    lbm_d3q19_tables(dir, m_HostOppIndex, m_HostW, nullptr);
    for (int d = 0; d < DIMENSION; ++d)
      for (int q = 0; q < DIRECTION_SIZE; ++q) m_HostDirection[d][q] = dir[d * DIRECTION_SIZE + q];
    for (int q = 0; q < DIRECTION_SIZE; ++q) m_HostMove[q] = 0;
    m_DeviceNode = DeviceNodeData{};
  }
  virtual ~LBMSolver() {
    if (m_pDomain) lbm_destroy(m_pDomain);
  }
  LBMSolver(const LBMSolver&) = delete;
  LBMSolver& operator=(const LBMSolver&) = delete;

  float m_HostDirection[DIMENSION][DIRECTION_SIZE];
  int m_HostOppIndex[DIRECTION_SIZE];
  float m_HostW[DIRECTION_SIZE];
  int m_HostMove[DIRECTION_SIZE];
  HostNodeData m_HostNode;

  float* m_DeviceDirection = nullptr;
  int* m_DeviceOppIndex = nullptr;
  float* m_DeviceW = nullptr;
  int* m_DeviceMove = nullptr;
  MRTMatrix* m_DeviceMatrix = nullptr;
  DeviceNodeData m_DeviceNode;

  lbm_domain* m_pDomain = nullptr;  // the library handle
};
#endif  // LBM_B200_NO_SOLVER_TYPES

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

// ---------------------------------------------------------------------------
// Poplar spelling: the Initialize program and Repeat(maxitr, runSimulation)
// ---------------------------------------------------------------------------
inline void initialize(Inputval* /*pinput*/, lbm_b200::Domain& d) {
  lbm_b200::check(lbm_initialize(d.get()));
}

inline void runSimulation(Inputval* pinput, lbm_b200::Domain& d) {
  lbm_b200::check(lbm_run_simulation(d.get(), pinput->maxitr));
}

// ---------------------------------------------------------------------------
// kernel.cu spelling
// ---------------------------------------------------------------------------
#ifndef LBM_B200_NO_SOLVER_TYPES
namespace lbm_b200 {
inline void refresh_device_node(LBMSolver* s) {
  DeviceNodeData& n = s->m_DeviceNode;
  check(lbm_device_fields(s->m_pDomain, &n.m_dCurrDen, &n.m_dPrevDen, &n.m_dCurrVelx,
                          &n.m_dCurrVely, &n.m_dCurrVelz));
}
inline size_t nodes_of(const Inputval* in) { return (size_t)in->nx * in->ny * in->nz; }
}  // namespace lbm_b200

// The icycle == 0 iteration of kernel.cu:156-164: create the library's
// device state on first use and build the initial state (node types,
// direction masks, equilibrium populations; the Initialize compute set of
// initialize.cpp:23-98).  Leaves pinput->icycle at 1, the cycle the next
// runSimulation step starts from.
inline void initialize(Inputval* pinput, LBMSolver* psolver) {
  if (!psolver->m_pDomain) lbm_b200::check(lbm_create(pinput, nullptr, &psolver->m_pDomain));
  lbm_b200::check(lbm_initialize(psolver->m_pDomain));
  lbm_b200::refresh_device_node(psolver);
  pinput->icycle = 1;
}

// kernel.cu:699-1018: the result file of the current cycle from m_HostNode
// (filled by runSimulation before it calls this) as savetype (0 VTU as
// <SAVE_PATH>Output%06d.vtu with index icycle / nwrite, 1 result.csv and
// section.csv), into ./result/.  arIndex (the reference's cell list) is not
// needed: the writer builds the hexahedra itself.
inline void saveFile(Inputval* pinput, LBMSolver* psolver, std::vector<int> /*arIndex*/,
                     int savetype) {
  HostNodeData& h = psolver->m_HostNode;
  std::error_code ec;
  std::filesystem::create_directories("./result", ec);  // SAVE_PATH (common.h)
  if (savetype == LBM_SAVE_VTU) {
    char path[512];
    const int index = pinput->nwrite > 0 ? pinput->icycle / pinput->nwrite : 0;
    std::snprintf(path, sizeof(path), "./result/Output%06d.vtu", index);
    lbm_b200::check(lbm_write_vtu(path, pinput->nx, pinput->ny, pinput->nz, h.m_dCurrDen.data(),
                                  h.m_dCurrVelx.data(), h.m_dCurrVely.data(),
                                  h.m_dCurrVelz.data(), h.m_nNodeType.data()));
  } else {
    lbm_b200::check(lbm_write_csv("./result/result.csv", "./result/section.csv", pinput->nx,
                                  pinput->ny, pinput->nz, h.m_dCurrDen.data(),
                                  h.m_dCurrVelx.data(), h.m_dCurrVely.data(),
                                  h.m_dCurrVelz.data()));
  }
}

// kernel.cu:18-277: maxitr cycles from pinput->icycle; the cycle 0 builds
// the initial state (initialize above), every other cycle is one fused
// step.  After a cycle with icycle % nwrite == 0 the macroscopic fields and
// node types are read into m_HostNode and saveFile writes them (nwrite <= 0:
// no files); after a cycle with icycle % 100 == 0 the residual
// sum |PrevDen - CurrDen| is printed as "ITER=%d | ERROR=%.5e" and appended
// to iteration.dat.  Steps between those cycles run as one call.
inline void runSimulation(Inputval* pinput, LBMSolver* psolver) {
  const size_t n = lbm_b200::nodes_of(pinput);
  std::FILE* it = std::fopen("iteration.dat", "wt");
  if (it) std::fprintf(it, "%s\n", "iter, error");
  HostNodeData& h = psolver->m_HostNode;
  auto events = [&](int icycle) {
    if (pinput->nwrite > 0 && icycle % pinput->nwrite == 0) {
      h.m_dCurrDen.resize(n);
      h.m_dCurrVelx.resize(n);
      h.m_dCurrVely.resize(n);
      h.m_dCurrVelz.resize(n);
      h.m_nNodeType.resize(n);
      lbm_b200::check(lbm_get_macroscopic(psolver->m_pDomain, h.m_dCurrDen.data(),
                                          h.m_dCurrVelx.data(), h.m_dCurrVely.data(),
                                          h.m_dCurrVelz.data()));
      lbm_b200::check(lbm_get_node_info(psolver->m_pDomain, h.m_nNodeType.data(), nullptr));
      saveFile(pinput, psolver, std::vector<int>(), pinput->savetype);
    }
    if (icycle % 100 == 0) {
      double diag[8];
      lbm_b200::check(lbm_diagnostics(psolver->m_pDomain, diag));
      std::printf("ITER=%d | ERROR=%.5e\n", icycle, diag[4]);
      if (it) std::fprintf(it, "%d %.5e\n", icycle, diag[4]);
    }
  };
  int left = pinput->maxitr;
  try {
    while (left > 0) {
      const int c = pinput->icycle;
      if (c == 0) {
        initialize(pinput, psolver);  // icycle -> 1
        --left;
        events(0);
        continue;
      }
      // steps up to the next cycle with an event (or the end)
      int k = left;
      const int to100 = (100 - c % 100) % 100;
      if (to100 < k) k = to100;
      if (pinput->nwrite > 0) {
        const int tow = (pinput->nwrite - c % pinput->nwrite) % pinput->nwrite;
        if (tow < k) k = tow;
      }
      k += 1;  // the event cycle itself is stepped first
      if (k > left) k = left;
      if (!psolver->m_pDomain) lbm_b200::check(lbm_create(pinput, nullptr, &psolver->m_pDomain));
      lbm_b200::check(lbm_run_simulation(psolver->m_pDomain, k));
      pinput->icycle += k;
      left -= k;
      lbm_b200::refresh_device_node(psolver);
      events(pinput->icycle - 1);
    }
  } catch (...) {
    if (it) std::fclose(it);
    throw;
  }
  if (it) std::fclose(it);
}
#endif  // LBM_B200_NO_SOLVER_TYPES
