/*
 * ref_poplar_emu.cpp — TEST INFRASTRUCTURE ONLY (the oracle's reference leg).
 *
 * Runs the reference's OWN device code on the host: lbm_codelets.cpp is
 * compiled unmodified (through the shim/poplar/Vertex.hpp stand-in) from the
 * reference tree, together with its decomposition.cpp and inverseMRT.cpp.
 * This file is the project-written replacement for the Poplar graph runtime:
 * it restates the graph wiring of initialize.cpp:50-97 and
 * runSimulation.cpp:133-264 — for every compute set and every tile it gathers
 * the tensor slices the reference binds to the vertex fields into contiguous
 * buffers, calls Vertex::compute(), and scatters the written fields back, as
 * Poplar's exchange phase does.  Tiles of one compute set run in parallel
 * (OpenMP); they never write overlapping slices.
 *
 * The host tables of main.cpp:87-183 (Direction, OppIndex, arW, the MRT
 * matrix) are restated here because main.cpp needs the Poplar SDK.
 *
 * Built by oracle/Makefile into oracle/_ref/libpoplar_ref.so (git-ignored);
 * used by tests to pin the oracle port and to generate golden fixtures, and
 * by bench.py as the timed CPU baseline ("kind": "reference").
 * Only the cavity case with LES + MRT exists in the Poplar program (F7).
 */
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "struct.h"         /* reference: Inputval, common.h constants */
#include "lbm_codelets.cpp" /* reference: the six Vertex classes, unmodified */

#include "orc_common.h"

/* reference host functions (decomposition.cpp, inverseMRT.cpp) */
int decomposition(Inputval* pinput, int Slice[][DIMENSION][2]);
int set_move_decomp(const int NTILE, const int Slice[][DIMENSION][2], int Move[][DIRECTION_SIZE]);
int slice_chunk(const unsigned tile, const int Slice[][DIMENSION][2], int* xs, int* xe, int* ys,
                int* ye, int* zs, int* ze, int* chunk_nx, int* chunk_ny, int* chunk_nz,
                int* chunk_len);
void inverseMRT(std::vector<std::vector<float>>& matori, std::vector<std::vector<float>>& pInvMat);

namespace {

/* A dense host tensor with Poplar-style slicing (row-major, last dim fastest). */
template <class T>
struct Tensor4 {
  int d0 = 0, d1 = 0, d2 = 0, d3 = 1;
  std::vector<T> v;
  void alloc(int a, int b, int c, int d) {
    d0 = a;
    d1 = b;
    d2 = c;
    d3 = d;
    v.assign((size_t)a * b * c * d, T(0));
  }
  /* slice({a0,b0,c0},{a1,b1,c1}).flatten() copied out */
  void gather(int a0, int a1, int b0, int b1, int c0, int c1, std::vector<T>& out) const {
    out.resize((size_t)(a1 - a0) * (b1 - b0) * (c1 - c0) * d3);
    size_t k = 0;
    for (int a = a0; a < a1; ++a)
      for (int b = b0; b < b1; ++b) {
        const T* src = &v[(((size_t)a * d1 + b) * d2 + c0) * d3];
        size_t cnt = (size_t)(c1 - c0) * d3;
        std::memcpy(&out[k], src, cnt * sizeof(T));
        k += cnt;
      }
  }
  void scatter(int a0, int a1, int b0, int b1, int c0, int c1, const std::vector<T>& in) {
    size_t k = 0;
    for (int a = a0; a < a1; ++a)
      for (int b = b0; b < b1; ++b) {
        T* dst = &v[(((size_t)a * d1 + b) * d2 + c0) * d3];
        size_t cnt = (size_t)(c1 - c0) * d3;
        std::memcpy(dst, &in[k], cnt * sizeof(T));
        k += cnt;
      }
  }
};

template <class T>
void bind(poplar::Vector<T>& f, std::vector<T>& buf) {
  f.data = buf.data();
  f.count = (unsigned)buf.size();
}

struct Emu {
  Inputval in;
  orc_ext ext;
  int NX, NY, NZ;
  int ntile = 0;
  std::vector<std::array<int, 6>> tiles;  // xs xe ys ye zs ze
  std::vector<int> move;                  // [ntile][19]
  Tensor4<float> arF, arFTemp, CurrDen, PrevDen, CurrVelx, CurrVely, CurrVelz, TauEddy;
  Tensor4<int> NodeType, DirectionState;
  std::vector<float> Matrix, MatInv, Direction, arW;
  std::vector<int> OppIndex;
};

/* main.cpp:87-146 (restated) */
void host_tables(Emu& e) {
  static const int cx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  static const int cy[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
  static const int cz[19] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
  static const int op[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
  e.Direction.assign(3 * 19, 0.0f);
  e.arW.assign(19, 0.0f);
  e.OppIndex.assign(op, op + 19);
  for (int d = 0; d < 19; ++d) {
    e.Direction[XDIM * 19 + d] = (float)cx[d];
    e.Direction[YDIM * 19 + d] = (float)cy[d];
    e.Direction[ZDIM * 19 + d] = (float)cz[d];
    if (d == 0)
      e.arW[d] = 1.0f / 3.0f;
    else if (d > 0 && d < 7)
      e.arW[d] = 1.0f / 18.0f;
    else
      e.arW[d] = 1.0f / 36.0f;
  }
}

/* main.cpp:150-171 (restated) then the reference inverseMRT */
int mrt_tables(Emu& e) {
  static const float m[19][19] = {
      {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
      {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
      {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
      {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
      {0, 0, 0, 4, -4, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
      {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, 0, 0, -1, -1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
      {0, 0, 0, 2, 2, -2, -2, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1},
      {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 1, 1, -1, -1},
      {0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1}};
  std::vector<std::vector<float>> mat(19, std::vector<float>(19));
  std::vector<std::vector<float>> inv(19, std::vector<float>(19, 0.0f));
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) mat[i][j] = m[i][j];
  inverseMRT(mat, inv); /* reference */
  e.Matrix.resize(361);
  e.MatInv.resize(361);
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) {
      e.Matrix[i * 19 + j] = mat[i][j];
      e.MatInv[i * 19 + j] = inv[i][j];
    }
  return 0;
}

void run_initialize(Emu& e) {
  const int nt = (int)e.tiles.size();
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bDS, bNT;
    std::vector<float> bF, bD, bX, bY, bZ;
    e.DirectionState.gather(ys, ye, zs, ze, xs, xe, bDS);
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    e.CurrDen.gather(ys, ye, zs, ze, xs, xe, bD);
    e.CurrVelx.gather(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.gather(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.gather(ys, ye, zs, ze, xs, xe, bZ);
    Initialize v;
    bind(v.DirectionState.value, bDS);
    bind(v.nNodeType.value, bNT);
    bind(v.arF.value, bF);
    bind(v.CurrDen.value, bD);
    bind(v.CurrVelx.value, bX);
    bind(v.CurrVely.value, bY);
    bind(v.CurrVelz.value, bZ);
    bind(v.arW.value, e.arW);
    bind(v.Direction.value, e.Direction);
    v.RefDen.value = e.in.m_dRefDen;
    v.RefVelx.value = e.in.m_dRefVelx;
    v.RefVely.value = e.in.m_dRefVely;
    v.RefVelz.value = e.in.m_dRefVelz;
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.NX.value = e.in.nx;
    v.NY.value = e.in.ny;
    v.NZ.value = e.in.nz;
    v.PADX.value = xs;
    v.PADY.value = ys;
    v.PADZ.value = zs;
    v.compute();
    e.DirectionState.scatter(ys, ye, zs, ze, xs, xe, bDS);
    e.NodeType.scatter(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.scatter(ys, ye, zs, ze, xs, xe, bF);
    e.CurrDen.scatter(ys, ye, zs, ze, xs, xe, bD);
    e.CurrVelx.scatter(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.scatter(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.scatter(ys, ye, zs, ze, xs, xe, bZ);
  }
}

/* Seeded density perturbation (this project's addition; orc_common.h),
 * applied after the Initialize compute set with the codelet's feq formula. */
void perturb(Emu& e) {
  if (e.ext.init_kind != 1) return;
  const int nx = e.in.nx, ny = e.in.ny, nz = e.in.nz;
  for (int y = 0; y < ny; ++y)
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) {
        const long n = x + (long)nx * (z + (long)nz * y);
        if (e.NodeType.v[n] == NODE_STRUCT) continue;
        float den = (float)((double)e.in.m_dRefDen +
                            (double)e.ext.noise_amp * orc_unit_noise(e.ext.seed, (uint64_t)n, 0));
        float velx = e.CurrVelx.v[n], vely = e.CurrVely.v[n], velz = e.CurrVelz.v[n];
        for (int d = 0; d < 19; ++d) {
          float edotu = e.Direction[XDIM * 19 + d] * velx + e.Direction[YDIM * 19 + d] * vely +
                        e.Direction[ZDIM * 19 + d] * velz;
          float usquare = velx * velx + vely * vely + velz * velz;
          e.arF.v[d + n * 19] =
              e.arW[d] * den * (1.0f + 3.0f * edotu + 4.5f * edotu * edotu - 1.5f * usquare);
        }
        e.CurrDen.v[n] = den;
      }
}

void run_step(Emu& e) {
  const int nt = (int)e.tiles.size();
  /* ComputeTurbulence_LES (runSimulation.cpp:133-157) */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bNT;
    std::vector<float> bF, bD, bX, bY, bZ, bT;
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    e.CurrDen.gather(ys, ye, zs, ze, xs, xe, bD);
    e.CurrVelx.gather(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.gather(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.gather(ys, ye, zs, ze, xs, xe, bZ);
    e.TauEddy.gather(ys, ye, zs, ze, xs, xe, bT);
    ComputeTurbulence_LES v;
    bind(v.nNodeType.value, bNT);
    bind(v.arF.value, bF);
    bind(v.CurrDen.value, bD);
    bind(v.CurrVelx.value, bX);
    bind(v.CurrVely.value, bY);
    bind(v.CurrVelz.value, bZ);
    bind(v.dTauEddy.value, bT);
    bind(v.arW.value, e.arW);
    bind(v.Direction.value, e.Direction);
    v.dTau.value = e.in.m_dTau;
    v.dSmagorinsky.value = e.in.m_dSmagorinsky;
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.compute();
    e.TauEddy.scatter(ys, ye, zs, ze, xs, xe, bT);
  }
  /* Collision_MRT (runSimulation.cpp:159-188): arFTemp interior slice */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bNT;
    std::vector<float> bF, bFT, bD, bX, bY, bZ, bT;
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    e.arFTemp.gather(ys + 1, ye + 1, zs + 1, ze + 1, xs + 1, xe + 1, bFT);
    e.CurrDen.gather(ys, ye, zs, ze, xs, xe, bD);
    e.CurrVelx.gather(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.gather(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.gather(ys, ye, zs, ze, xs, xe, bZ);
    e.TauEddy.gather(ys, ye, zs, ze, xs, xe, bT);
    Collision_MRT v;
    bind(v.nNodeType.value, bNT);
    bind(v.arF.value, bF);
    bind(v.arFTemp.value, bFT);
    bind(v.CurrDen.value, bD);
    bind(v.CurrVelx.value, bX);
    bind(v.CurrVely.value, bY);
    bind(v.CurrVelz.value, bZ);
    bind(v.dTauEddy.value, bT);
    v.RefDen.value = e.in.m_dRefDen;
    v.dTau.value = e.in.m_dTau;
    v.dWeps.value = e.in.dWeps;
    v.dWepsj.value = e.in.dWepsj;
    v.dWXX.value = e.in.dWXX;
    bind(v.m_MatMRT.value, e.Matrix);
    bind(v.m_MatInv.value, e.MatInv);
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.compute();
    e.arFTemp.scatter(ys + 1, ye + 1, zs + 1, ze + 1, xs + 1, xe + 1, bFT);
  }
  /* Streaming (runSimulation.cpp:190-210): arFTemp slice with ghosts */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bNT, bDS, bMove(e.move.begin() + 19 * t, e.move.begin() + 19 * (t + 1));
    std::vector<float> bF, bFT;
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    e.arFTemp.gather(ys, ye + 2, zs, ze + 2, xs, xe + 2, bFT);
    e.DirectionState.gather(ys, ye, zs, ze, xs, xe, bDS);
    Streaming v;
    bind(v.nNodeType.value, bNT);
    bind(v.arF.value, bF);
    bind(v.arFTemp.value, bFT);
    bind(v.DirectionState.value, bDS);
    bind(v.Move.value, bMove);
    bind(v.nOppIndex.value, e.OppIndex);
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.compute();
    e.arF.scatter(ys, ye, zs, ze, xs, xe, bF);
  }
  /* BoundaryCavity (runSimulation.cpp:212-238) */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bNT, bDS;
    std::vector<float> bF, bFT;
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    e.arFTemp.gather(ys + 1, ye + 1, zs + 1, ze + 1, xs + 1, xe + 1, bFT);
    e.DirectionState.gather(ys, ye, zs, ze, xs, xe, bDS);
    BoundaryCavity v;
    bind(v.nNodeType.value, bNT);
    bind(v.arF.value, bF);
    bind(v.arFTemp.value, bFT);
    bind(v.arW.value, e.arW);
    bind(v.Direction.value, e.Direction);
    bind(v.DirectionState.value, bDS);
    bind(v.nOppIndex.value, e.OppIndex);
    v.RefDen.value = e.in.m_dRefDen;
    v.velx.value = e.in.m_dRefVelx;
    v.vely.value = e.in.m_dRefVely;
    v.velz.value = e.in.m_dRefVelz;
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.compute();
    e.arF.scatter(ys, ye, zs, ze, xs, xe, bF);
  }
  /* Macroscopic (runSimulation.cpp:240-261) */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < nt; ++t) {
    const int xs = e.tiles[t][0], xe = e.tiles[t][1], ys = e.tiles[t][2], ye = e.tiles[t][3],
              zs = e.tiles[t][4], ze = e.tiles[t][5];
    std::vector<int> bNT;
    std::vector<float> bF, bD, bP, bX, bY, bZ;
    e.NodeType.gather(ys, ye, zs, ze, xs, xe, bNT);
    e.CurrDen.gather(ys, ye, zs, ze, xs, xe, bD);
    e.PrevDen.gather(ys, ye, zs, ze, xs, xe, bP);
    e.CurrVelx.gather(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.gather(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.gather(ys, ye, zs, ze, xs, xe, bZ);
    e.arF.gather(ys, ye, zs, ze, xs, xe, bF);
    Macroscopic v;
    bind(v.nNodeType.value, bNT);
    bind(v.CurrDen.value, bD);
    bind(v.PrevDen.value, bP);
    bind(v.CurrVelx.value, bX);
    bind(v.CurrVely.value, bY);
    bind(v.CurrVelz.value, bZ);
    bind(v.arF.value, bF);
    bind(v.Direction.value, e.Direction);
    v.nx.value = xe - xs;
    v.ny.value = ye - ys;
    v.nz.value = ze - zs;
    v.length.value = (xe - xs) * (ye - ys) * (ze - zs);
    v.compute();
    e.CurrDen.scatter(ys, ye, zs, ze, xs, xe, bD);
    e.PrevDen.scatter(ys, ye, zs, ze, xs, xe, bP);
    e.CurrVelx.scatter(ys, ye, zs, ze, xs, xe, bX);
    e.CurrVely.scatter(ys, ye, zs, ze, xs, xe, bY);
    e.CurrVelz.scatter(ys, ye, zs, ze, xs, xe, bZ);
  }
}

}  // namespace

extern "C" {

void* ref_create(const Inputval* pin, const orc_ext* pext) {
  if (!pin || pin->casetype != CAVITY) return nullptr;
  if (pin->nx < 2 || pin->ny < 2 || pin->nz < 2) return nullptr;
  Emu* e = new Emu();
  e->in = *pin;
  if (pext)
    e->ext = *pext;
  else
    std::memset(&e->ext, 0, sizeof(e->ext));
#ifdef _OPENMP
  if (e->ext.threads > 0) omp_set_num_threads(e->ext.threads);
#endif
  e->NX = pin->nx;
  e->NY = pin->ny;
  e->NZ = pin->nz;
  host_tables(*e);
  mrt_tables(*e);
  static int Slice[TILE_NUM][DIMENSION][2];
  int nt = decomposition(&e->in, Slice); /* reference */
  /* optional y-split of every tile for more host threads (results unchanged) */
  static int Split[TILE_NUM][DIMENSION][2];
  int s = e->ext.split > 1 ? e->ext.split : 1;
  int ns = 0;
  for (int t = 0; t < nt; ++t) {
    int xs, xe, ys, ye, zs, ze, cnx, cny, cnz, clen;
    if (slice_chunk((unsigned)t, Slice, &xs, &xe, &ys, &ye, &zs, &ze, &cnx, &cny, &cnz, &clen))
      continue; /* reference: skip empty chunks */
    int h = ye - ys, k = s < h ? s : h;
    for (int i = 0; i < k && ns < TILE_NUM; ++i) {
      Split[ns][0][0] = xs;
      Split[ns][0][1] = xe;
      Split[ns][1][0] = ys + (h * i) / k;
      Split[ns][1][1] = ys + (h * (i + 1)) / k;
      Split[ns][2][0] = zs;
      Split[ns][2][1] = ze;
      ++ns;
    }
  }
  e->ntile = ns;
  e->move.assign((size_t)ns * 19, 0);
  set_move_decomp(ns, Split, (int(*)[DIRECTION_SIZE])e->move.data()); /* reference */
  for (int t = 0; t < ns; ++t)
    e->tiles.push_back({Split[t][0][0], Split[t][0][1], Split[t][1][0], Split[t][1][1],
                        Split[t][2][0], Split[t][2][1]});
  const int NX = e->NX, NY = e->NY, NZ = e->NZ;
  e->arF.alloc(NY, NZ, NX, 19);
  e->arFTemp.alloc(NY + 2, NZ + 2, NX + 2, 19);
  e->CurrDen.alloc(NY, NZ, NX, 1);
  e->PrevDen.alloc(NY, NZ, NX, 1);
  e->CurrVelx.alloc(NY, NZ, NX, 1);
  e->CurrVely.alloc(NY, NZ, NX, 1);
  e->CurrVelz.alloc(NY, NZ, NX, 1);
  e->TauEddy.alloc(NY, NZ, NX, 1);
  e->NodeType.alloc(NY, NZ, NX, 1);
  e->DirectionState.alloc(NY, NZ, NX, 1);
  run_initialize(*e);
  perturb(*e);
  return e;
}

int ref_step(void* h, int nsteps) {
  Emu* e = (Emu*)h;
  if (!e || nsteps < 0) return -1;
  for (int i = 0; i < nsteps; ++i) run_step(*e);
  return 0;
}

int ref_get(void* h, double* arF, double* den, double* vx, double* vy, double* vz, double* pden,
            double* te, int* nt, int* ds) {
  Emu* e = (Emu*)h;
  if (!e) return -1;
  const long N = (long)e->NX * e->NY * e->NZ;
  if (arF)
    for (long i = 0; i < N * 19; ++i) arF[i] = e->arF.v[i];
  for (long i = 0; i < N; ++i) {
    if (den) den[i] = e->CurrDen.v[i];
    if (vx) vx[i] = e->CurrVelx.v[i];
    if (vy) vy[i] = e->CurrVely.v[i];
    if (vz) vz[i] = e->CurrVelz.v[i];
    if (pden) pden[i] = e->PrevDen.v[i];
    if (te) te[i] = e->TauEddy.v[i];
    if (nt) nt[i] = e->NodeType.v[i];
    if (ds) ds[i] = e->DirectionState.v[i];
  }
  return 0;
}

void ref_destroy(void* h) { delete (Emu*)h; }

int ref_ntile(void* h) { return h ? ((Emu*)h)->ntile : -1; }

int ref_decomposition(const Inputval* pin, int Slice[][DIMENSION][2]) {
  Inputval c = *pin;
  return decomposition(&c, Slice);
}
int ref_set_move_decomp(int NTILE, const int Slice[][DIMENSION][2], int Move[][DIRECTION_SIZE]) {
  return set_move_decomp(NTILE, Slice, Move);
}
int ref_slice_chunk(unsigned tile, const int Slice[][DIMENSION][2], int* xs, int* xe, int* ys,
                    int* ye, int* zs, int* ze, int* cnx, int* cny, int* cnz, int* clen) {
  return slice_chunk(tile, Slice, xs, xe, ys, ye, zs, ze, cnx, cny, cnz, clen);
}
int ref_inverse_mrt(const float* mat, float* inv) {
  std::vector<std::vector<float>> a(19, std::vector<float>(19)), p(19, std::vector<float>(19, 0.f));
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) a[i][j] = mat[i * 19 + j];
  inverseMRT(a, p);
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) inv[i * 19 + j] = p[i][j];
  return 0;
}

}  // extern "C"
