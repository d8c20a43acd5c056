/*
 * lbm_oracle.cpp — TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU restatement of the reference D3Q19 time step, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * The product library never links, loads or calls this file.
 *
 * What it restates (reference file:line):
 *   tables               main.cpp:87-146, moment matrix main.cpp:149-171
 *   inverseMRT           inverseMRT.cpp:8-92 (Gauss-Jordan, same pivot rotation)
 *   decomposition        decomposition.cpp:10-161
 *   Initialize           lbm_codelets.cpp:111-242 (+ keSetNodeType kernel.cu:1046-1097)
 *   ComputeTurbulence_LES lbm_codelets.cpp:558-668
 *   Collision_MRT        lbm_codelets.cpp:409-550
 *   keCollision_SRT      kernel.cu:458-487 (FP64 literals kept, F11)
 *   Streaming            lbm_codelets.cpp:21-105 (pull), with the donor
 *                        STRUCT check of keStreaming kernel.cu:489-516
 *   BoundaryCavity       lbm_codelets.cpp:325-402
 *   keBoundaryInlet      kernel.cu:566-613
 *   keBoundaryOutlet     kernel.cu:615-657
 *   keBoundaryStruct     kernel.cu:659-697
 *   Macroscopic          lbm_codelets.cpp:248-318
 *   step order           runSimulation.cpp:263-264 / kernel.cu:166-199
 *
 * Layout is the Poplar one (F4): AoS, direction fastest, arF[ny][nz][nx][19]
 * and the ghost-padded arFTemp[ny+2][nz+2][nx+2][19].  Each compute set runs
 * tile by tile over the reference's 3x3x3 decomposition (OpenMP across tiles).
 *
 * Pinning: for the cavity MRT+LES step (the only one the Poplar codelets
 * implement) this restatement is compared bit for bit against the
 * reference's own lbm_codelets.cpp compiled here (oracle/_ref), and the
 * committed golden fixtures in tests/golden were produced by that build.
 * SRT, inlet, outlet and struct exist only in kernel.cu; they are pinned
 * against kernel.cu built from source and run on a B200.
 *
 * Build: oracle/Makefile (-O2 -ffp-contract=off so that no FMA contraction
 * changes the rounding relative to the reference build).
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/lbm_b200.h"
#include "orc_common.h"

namespace {

/* Direction vectors, main.cpp:87-105 (X, Y, Z components). */
const int kCx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int kCy[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int kCz[19] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
/* main.cpp:107-113 */
const int kOpp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
/* main.cpp:150-171 */
const int kM[19][19] = {
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

/* inverseMRT.cpp:8-92 restated on a flat row-major array.  The reference
 * rotates the pivot row to the end while |pivot| < 1e-9 (21-34); a singular
 * matrix would make that loop spin for ever, so here the rotation is
 * bounded and a singular matrix returns -1 instead of exit(0) (86-90). */
template <typename T>
int inverse_gj(const T* mat, T* inv) {
  const int n = 19;
  std::vector<std::vector<T>> a(n, std::vector<T>(n)), p(n, std::vector<T>(n, T(0)));
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) a[i][j] = mat[i * n + j];
  for (int i = 0; i < n; ++i) p[i][i] = T(1);
  for (int i = 0; i < n - 1; ++i) {
    int rot = 0;
    while (std::fabs((double)a[i][i]) < std::pow(10.0, -9.0)) {
      if (++rot > n - i) return -1;
      std::vector<T> ta = a[i], tp = p[i];
      for (int j = i; j < n - 1; ++j) {
        a[j] = a[j + 1];
        p[j] = p[j + 1];
      }
      a[n - 1] = ta;
      p[n - 1] = tp;
    }
    T inv_ii = a[i][i];
    for (int j = 0; j < n; ++j) {
      p[i][j] = p[i][j] / inv_ii;
      a[i][j] = a[i][j] / inv_ii;
    }
    std::vector<T> ta = a[i], tp = p[i];
    for (int j = i + 1; j < n; ++j) {
      T inv_ji = a[j][i];
      for (int k = 0; k < n; ++k) {
        p[j][k] = p[j][k] - tp[k] * inv_ji;
        a[j][k] = a[j][k] - ta[k] * inv_ji;
      }
    }
  }
  T inv_ee = a[n - 1][n - 1];
  for (int i = 0; i < n; ++i) {
    p[n - 1][i] = p[n - 1][i] / inv_ee;
    a[n - 1][i] = a[n - 1][i] / inv_ee;
  }
  for (int i = n - 1; i > 0; --i) {
    std::vector<T> ta = a[i], tp = p[i];
    for (int j = i - 1; j >= 0; --j) {
      T inv_ji = a[j][i];
      for (int k = 0; k < n; ++k) {
        p[j][k] = p[j][k] - tp[k] * inv_ji;
        a[j][k] = a[j][k] - ta[k] * inv_ji;
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    T s = T(0);
    for (int j = 0; j < n; ++j) s += std::fabs(a[i][j]);
    if ((double)s < std::pow(10.0, -10.0)) return -1;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) inv[i * n + j] = p[i][j];
  return 0;
}

struct Tile {
  int xs, xe, ys, ye, zs, ze;
};

/* decomposition.cpp:98-161 */
int decompose(const Inputval* in, int Slice[][DIMENSION][2]) {
  int tiles = 0;
  int chunk[3] = {in->nx / XDECOMP, in->ny / YDECOMP, in->nz / ZDECOMP};
  int st[3] = {0, 0, 0}, ed[3] = {0, 0, 0};
  const int ext[3] = {in->nx, in->ny, in->nz};
  const int dec[3] = {XDECOMP, YDECOMP, ZDECOMP};
  for (int i = 0; i < dec[0]; i++) {
    st[0] = i * chunk[0];
    ed[0] = (i == dec[0] - 1) ? ext[0] : (i + 1) * chunk[0];
    if (ed[0] > ext[0]) ed[0] = ext[0];
    for (int j = 0; j < dec[1]; j++) {
      st[1] = j * chunk[1];
      ed[1] = (j == dec[1] - 1) ? ext[1] : (j + 1) * chunk[1];
      if (ed[1] > ext[1]) ed[1] = ext[1];
      for (int k = 0; k < dec[2]; k++) {
        st[2] = k * chunk[2];
        ed[2] = (k == dec[2] - 1) ? ext[2] : (k + 1) * chunk[2];
        if (ed[2] > ext[2]) ed[2] = ext[2];
        for (int m = 0; m < DIMENSION; m++) {
          Slice[tiles][m][0] = st[m];
          Slice[tiles][m][1] = ed[m];
        }
        tiles++;
      }
    }
  }
  return tiles;
}

template <typename R>
struct Solver {
  Inputval in;
  orc_ext ext;
  int nx, ny, nz;
  long N;
  std::vector<R> arF, arFT, den, pden, vx, vy, vz, tau_e;
  std::vector<int> type, dstate;
  std::vector<float> inlet_u;  // [ny][nz], channel only
  R Dir[3 * 19], W[19];
  R Mat[19 * 19], Inv[19 * 19];
  std::vector<Tile> tiles;
  bool has_struct = false;
  std::vector<unsigned char> solid;  // [N] solid voxels (this project's general masks)

  long id(int x, int y, int z) const { return x + (long)nx * (z + (long)nz * y); }
  long pid(int x, int y, int z) const {
    return (x + 1) + (long)(nx + 2) * ((z + 1) + (long)(nz + 2) * (y + 1));
  }

  template <typename F>
  void for_tiles(F f) {
    const int nt = (int)tiles.size();
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < nt; ++t) {
      const Tile& T = tiles[t];
      for (int y = T.ys; y < T.ye; ++y)
        for (int z = T.zs; z < T.ze; ++z)
          for (int x = T.xs; x < T.xe; ++x) f(x, y, z);
    }
  }

  int setup(const Inputval* pin, const orc_ext* pext) {
    in = *pin;
    if (pext)
      ext = *pext;
    else
      std::memset(&ext, 0, sizeof(ext));
    nx = in.nx;
    ny = in.ny;
    nz = in.nz;
    if (nx < 2 || ny < 2 || nz < 2) return -1;
    N = (long)nx * ny * nz;
    const long NP = (long)(nx + 2) * (ny + 2) * (nz + 2);
    arF.assign(N * 19, R(0));
    arFT.assign(NP * 19, R(0));
    den.assign(N, R(0));
    pden.assign(N, R(0));
    vx.assign(N, R(0));
    vy.assign(N, R(0));
    vz.assign(N, R(0));
    tau_e.assign(N, R(0));
    type.assign(N, 0);
    dstate.assign(N, 0);
    for (int d = 0; d < 19; ++d) {
      Dir[XDIM * 19 + d] = R(kCx[d]);
      Dir[YDIM * 19 + d] = R(kCy[d]);
      Dir[ZDIM * 19 + d] = R(kCz[d]);
      /* main.cpp:141-146 (float division for the FP32 oracle) */
      if (d == 0)
        W[d] = R(1) / R(3);
      else if (d < 7)
        W[d] = R(1) / R(18);
      else
        W[d] = R(1) / R(36);
    }
    for (int i = 0; i < 19; ++i)
      for (int j = 0; j < 19; ++j) Mat[i * 19 + j] = R(kM[i][j]);
    if (inverse_gj<R>(Mat, Inv) != 0) return -2;

    static int Slice[TILE_NUM][DIMENSION][2];
    int nt;
#pragma omp critical(orc_slice)
    {
      nt = decompose(&in, Slice);
      tiles.clear();
      int split = ext.split > 1 ? ext.split : 1;
      for (int t = 0; t < nt; ++t) {
        Tile T{Slice[t][0][0], Slice[t][0][1], Slice[t][1][0], Slice[t][1][1], Slice[t][2][0],
               Slice[t][2][1]};
        /* slice_chunk (decomposition.cpp:66-94): empty chunks are skipped */
        if (T.xe - T.xs < 1 || T.ye - T.ys < 1 || T.ze - T.zs < 1) continue;
        int h = T.ye - T.ys;
        int s = split < h ? split : h;
        for (int k = 0; k < s; ++k) {
          Tile U = T;
          U.ys = T.ys + (h * k) / s;
          U.ye = T.ys + (h * (k + 1)) / s;
          if (U.ye > U.ys) tiles.push_back(U);
        }
      }
    }
    if (in.casetype == CHANNEL) {
      inlet_u.resize((size_t)ny * nz);
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z)
          inlet_u[(size_t)y * nz + z] = orc_inlet_profile(in.m_dRefVelx, y, z, ny, nz);
    }
    initialize();
    return 0;
  }

  /* keSetNodeType (kernel.cu:1046-1097) / Initialize codelet
   * (lbm_codelets.cpp:183-201); CHANNEL is this project's extension. */
  int node_type(int x, int y, int z) const {
    if (!solid.empty() && solid[id(x, y, z)]) return NODE_STRUCT;
    int t = NODE_FLUID;
    if (in.casetype == CAVITY) {
      if (y == 0) t = NODE_FIXEDWALL;
      if (y == ny - 1) t = NODE_MOVINGWALL;
      if ((x == 0 || x == nx - 1) || (z == 0 || z == nz - 1)) t = NODE_FIXEDWALL;
    } else if (in.casetype == POISEUILLE) {
      if (x == 0) t = NODE_INLET;
      if (x == nx - 1) t = NODE_OUTLET;
      if ((y - 25) * (y - 25) + (z - 25) * (z - 25) > 400) t = NODE_STRUCT;
    } else if (in.casetype == CHANNEL) {
      if (x == 0) t = NODE_INLET;
      if (x == nx - 1) t = NODE_OUTLET;
      if (y == 0 || y == ny - 1 || z == 0 || z == nz - 1) t = NODE_FIXEDWALL;
    }
    return t;
  }

  /* Initialize codelet, lbm_codelets.cpp:140-241 */
  void initialize() {
    has_struct = false;
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
          if (node_type(x, y, z) == NODE_STRUCT) has_struct = true;
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      int ds = 0;
      for (int d = 18; d > 0; --d) {
        int y1 = y + (int)Dir[YDIM * 19 + d];
        int z1 = z + (int)Dir[ZDIM * 19 + d];
        int x1 = x + (int)Dir[XDIM * 19 + d];
        if (x1 < nx && y1 < ny && z1 < nz && x1 >= 0 && y1 >= 0 && z1 >= 0)
          ds = (ds | 1) << 1;
        else
          ds = ds << 1;
      }
      dstate[n] = ds | 1;
      const int t = node_type(x, y, z);
      type[n] = t;
      if (t == NODE_STRUCT) return;
      R dn = R(in.m_dRefDen);
      R ux = R(0), uy = R(0), uz = R(0);
      if (t == NODE_MOVINGWALL) {
        ux = R(in.m_dRefVelx);
        uy = R(in.m_dRefVely);
        uz = R(in.m_dRefVelz);
      }
      /* Seeded perturbations (this project's addition; orc_common.h). */
      if (ext.init_kind == LBM_INIT_DENSITY_NOISE) {
        dn = R((float)((double)in.m_dRefDen +
                       (double)ext.noise_amp * orc_unit_noise(ext.seed, (uint64_t)n, 0)));
      } else if (ext.init_kind == LBM_INIT_CHANNEL &&
                 (t == NODE_FLUID || t == NODE_INLET || t == NODE_OUTLET)) {
        const double au = (double)ext.noise_amp * (double)in.m_dRefVelx;
        float prof = in.casetype == CHANNEL ? inlet_u[(size_t)y * nz + z] : 0.0f;
        ux = R((float)((double)prof + au * orc_unit_noise(ext.seed, (uint64_t)n, 0)));
        uy = R((float)(au * orc_unit_noise(ext.seed, (uint64_t)n, 1)));
        uz = R((float)(au * orc_unit_noise(ext.seed, (uint64_t)n, 2)));
      }
      for (int d = 0; d < 19; ++d) {
        R eu = Dir[XDIM * 19 + d] * ux + Dir[YDIM * 19 + d] * uy + Dir[ZDIM * 19 + d] * uz;
        R usq = ux * ux + uy * uy + uz * uz;
        arF[d + n * 19] = W[d] * dn * (R(1.0f) + R(3.0f) * eu + R(4.5f) * eu * eu - R(1.5f) * usq);
      }
      den[n] = dn;
      vx[n] = ux;
      vy[n] = uy;
      vz[n] = uz;
    });
  }

  /* ComputeTurbulence_LES codelet, lbm_codelets.cpp:558-668.  The
   * unqualified pow/sqrt of the codelet resolve to the C library's double
   * functions, so those parts are evaluated in double and rounded once. */
  void les() {
    const R tau = R(in.m_dTau), cs = R(in.m_dSmagorinsky);
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if (type[n] == NODE_STRUCT) return;
      R dn = den[n], ux = vx[n], uy = vy[n], uz = vz[n];
      R f[19];
      for (int d = 0; d < 19; ++d) f[d] = arF[d + n * 19];
      R usq = ux * ux + uy * uy + uz * uz;
      R p0[3] = {0, 0, 0}, p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0};
      for (int d = 0; d < 19; ++d) {
        R eu = Dir[XDIM * 19 + d] * ux + Dir[YDIM * 19 + d] * uy + Dir[ZDIM * 19 + d] * uz;
        R feq = W[d] * dn * (R(1.0f) + R(3.0f) * eu + R(4.5f) * eu * eu - R(1.5f) * usq);
        R d1 = Dir[XDIM * 19 + d], d2 = Dir[YDIM * 19 + d], d3 = Dir[ZDIM * 19 + d];
        R mul = f[d] - feq;
        R d11 = d1 * mul, d22 = d2 * mul, d33 = d3 * mul;
        p0[0] += d1 * d11;
        p0[1] += d1 * d22;
        p0[2] += d1 * d33;
        p1[0] += d2 * d11;
        p1[1] += d2 * d22;
        p1[2] += d2 * d33;
        p2[0] += d3 * d11;
        p2[1] += d3 * d22;
        p2[2] += d3 * d33;
      }
      R q = (p0[0] * p0[0] + p0[1] * p0[1] + p0[2] * p0[2]) +
            (p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]) +
            (p2[0] * p2[0] + p2[1] * p2[1] + p2[2] * p2[2]);
      const R c18 = R(18.0f) * R(1.41421356237f);
      R smag = (R)(0.5f * std::sqrt(std::pow((double)tau, 2.0) +
                                    c18 * std::pow((double)cs, 2.0) * std::sqrt((double)q) / dn));
      tau_e[n] = R(-0.5f) * tau + smag;
    });
  }

  /* Collision_MRT codelet, lbm_codelets.cpp:409-550 */
  void mrt() {
    const R rho0 = R(in.m_dRefDen), tau = R(in.m_dTau);
    const R weps = R(in.dWeps), wepsj = R(in.dWepsj), wxx = R(in.dWXX);
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if (type[n] == NODE_STRUCT) return;
      R dn = den[n];
      R te = tau_e[n];
      R j[3] = {dn * vx[n], dn * vy[n], dn * vz[n]};
      R f[19], ft[19], meq[19], s[19], m1[19];
      for (int d = 0; d < 19; ++d) f[d] = arF[d + n * 19];
      R jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
      meq[0] = dn;
      meq[1] = R(-11.0f) * dn + R(19.0f) / rho0 * jj;
      meq[2] = weps * dn + wepsj / rho0 * jj;
      meq[3] = j[0];
      meq[4] = R(-2.0f / 3.0f) * j[0];
      meq[5] = j[1];
      meq[6] = R(-2.0f / 3.0f) * j[1];
      meq[7] = j[2];
      meq[8] = R(-2.0f / 3.0f) * j[2];
      meq[9] = (R)(R(1.0f) / rho0 *
                   (2.0f * std::pow((double)j[0], 2.0) -
                    (std::pow((double)j[1], 2.0) + std::pow((double)j[2], 2.0))));
      meq[10] = wxx * meq[9];
      meq[11] = (R)(R(1.0f) / rho0 * (std::pow((double)j[1], 2.0) - std::pow((double)j[2], 2.0)));
      meq[12] = wxx * meq[11];
      meq[13] = j[0] * j[1] / rho0;
      meq[14] = j[1] * j[2] / rho0;
      meq[15] = j[2] * j[0] / rho0;
      meq[16] = meq[17] = meq[18] = R(0);
      const R sv = R(1.0f) / (tau + te);
      s[0] = R(0);
      s[1] = R(1.19f);
      s[2] = R(1.4f);
      s[3] = R(0);
      s[4] = R(1.2f);
      s[5] = R(0);
      s[6] = R(1.2f);
      s[7] = R(0);
      s[8] = R(1.2f);
      s[9] = sv;
      s[10] = R(1.4f);
      s[11] = sv;
      s[12] = R(1.4f);
      s[13] = s[14] = s[15] = sv;
      s[16] = s[17] = s[18] = R(1.98f);
      for (int i = 0; i < 19; ++i) {
        m1[i] = R(0);
        for (int k = 0; k < 19; ++k) m1[i] += Mat[k + i * 19] * f[k];
      }
      for (int i = 0; i < 19; ++i) ft[i] = s[i] * (m1[i] - meq[i]);
      for (int i = 0; i < 19; ++i) {
        m1[i] = R(0);
        for (int k = 0; k < 19; ++k) m1[i] += Inv[k + i * 19] * ft[k];
      }
      const long p = pid(x, y, z);
      for (int d = 0; d < 19; ++d) arFT[d + p * 19] = f[d] - m1[d];
    });
  }

  /* keCollision_SRT, kernel.cu:458-487.  The FP64 literals promote feq to
   * double before it is rounded to float (F11). */
  void srt() {
    const R tau = R(in.m_dTau);
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if (type[n] == NODE_STRUCT) return;
      R dn = den[n], ux = vx[n], uy = vy[n], uz = vz[n], te = tau_e[n];
      const long p = pid(x, y, z);
      for (int d = 0; d < 19; ++d) {
        R f = arF[d + n * 19];
        R eu = Dir[XDIM * 19 + d] * ux + Dir[YDIM * 19 + d] * uy + Dir[ZDIM * 19 + d] * uz;
        R usq = ux * ux + uy * uy + uz * uz;
        R feq = (R)((double)(W[d] * dn) * (1.0 + 3.0 * (double)eu + 4.5 * (double)eu * (double)eu -
                                           1.5 * (double)usq));
        arFT[d + p * 19] = f - (f - feq) / (tau + te);
      }
    });
  }

  /* Streaming codelet, lbm_codelets.cpp:21-105: arF[opp(d)](x) =
   * arFTemp[opp(d)](x + c_d) when bit d of DirectionState says x + c_d is
   * inside the domain.  When the geometry holds STRUCT nodes the donor is
   * also skipped if it is STRUCT, as keStreaming (kernel.cu:505-515) does. */
  void streaming() {
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if (type[n] == NODE_STRUCT) return;
      const int ds = dstate[n];
      for (int d = 0; d < 19; ++d) {
        if ((ds >> d) & 1) {
          int x1 = x + kCx[d], y1 = y + kCy[d], z1 = z + kCz[d];
          if (has_struct && type[id(x1, y1, z1)] == NODE_STRUCT) continue;
          const int o = kOpp[d];
          arF[o + n * 19] = arFT[o + pid(x1, y1, z1) * 19];
        }
      }
    });
  }

  /* BoundaryCavity codelet, lbm_codelets.cpp:325-402 */
  void boundary_cavity() {
    const R ux = R(in.m_dRefVelx), uy = R(in.m_dRefVely), uz = R(in.m_dRefVelz);
    const R rho0 = R(in.m_dRefDen);
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      const int t = type[n];
      if (t == NODE_FLUID) return;
      const int ds = dstate[n];
      const long p = pid(x, y, z);
      for (int d = 0; d < 19; ++d) {
        if (!((ds >> d) & 1)) {
          const int o = kOpp[d];
          const R ft = arFT[d + p * 19];
          if (t == NODE_FIXEDWALL) {
            arF[o + n * 19] = ft;
          } else if (t == NODE_MOVINGWALL) {
            R eu = Dir[XDIM * 19 + d] * ux + Dir[YDIM * 19 + d] * uy + Dir[ZDIM * 19 + d] * uz;
            arF[o + n * 19] = ft - R(6.0f) * W[d] * rho0 * eu;
          }
        }
      }
    });
  }

  /* keBoundaryStruct, kernel.cu:659-697 */
  void boundary_struct() {
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if ((type[n] & NODE_FLUID) == 0) return;
      const int ds = dstate[n];
      const long p = pid(x, y, z);
      for (int d = 0; d < 19; ++d) {
        if ((ds >> d) & 1) {
          if (type[id(x + kCx[d], y + kCy[d], z + kCz[d])] == NODE_STRUCT)
            arF[kOpp[d] + n * 19] = arFT[d + p * 19];
        }
      }
    });
  }

  /* keBoundaryInlet, kernel.cu:566-613 (uniform RefVel for POISEUILLE; the
   * CHANNEL case uses the parabolic profile at the node's (y, z)). */
  void boundary_inlet() {
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if ((type[n] & NODE_INLET) == 0) return;
      const int ds = dstate[n];
      const long p = pid(x, y, z);
      R ux = R(in.m_dRefVelx), uy = R(in.m_dRefVely), uz = R(in.m_dRefVelz);
      if (in.casetype == CHANNEL) {
        ux = R(inlet_u[(size_t)y * nz + z]);
        uy = uz = R(0);
      }
      for (int d = 0; d < 19; ++d) {
        if (!((ds >> d) & 1)) {
          const int o = kOpp[d];
          const R rin = den[id(x + 1, y, z)];
          R eu = Dir[XDIM * 19 + d] * ux + Dir[YDIM * 19 + d] * uy + Dir[ZDIM * 19 + d] * uz;
          arF[o + n * 19] =
              (R)((double)arFT[d + p * 19] - 6.0 * (double)W[d] * (double)rin * (double)eu);
        }
      }
    });
  }

  /* keBoundaryOutlet, kernel.cu:615-657 */
  void boundary_outlet() {
    const R rho0 = R(in.m_dRefDen);
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if ((type[n] & NODE_OUTLET) == 0) return;
      const int ds = dstate[n];
      const long p = pid(x, y, z);
      const long ni = id(x - 1, y, z);
      for (int d = 0; d < 19; ++d) {
        if (!((ds >> d) & 1)) {
          const int o = kOpp[d];
          R bx = (R)((double)vx[n] + 0.5 * (double)(vx[n] - vx[ni]));
          R by = (R)((double)vy[n] + 0.5 * (double)(vy[n] - vy[ni]));
          R bz = (R)((double)vz[n] + 0.5 * (double)(vz[n] - vz[ni]));
          R usq = bx * bx + by * by + bz * bz;
          R eu = Dir[XDIM * 19 + d] * bx + Dir[YDIM * 19 + d] * by + Dir[ZDIM * 19 + d] * bz;
          arF[o + n * 19] = (R)(-(double)arFT[d + p * 19] +
                                2.0 * (double)W[d] * (double)rho0 *
                                    (1.0 + 4.5 * ((double)eu * (double)eu) - 1.5 * (double)usq));
        }
      }
    });
  }

  /* Macroscopic codelet, lbm_codelets.cpp:248-318 */
  void macroscopic() {
    for_tiles([&](int x, int y, int z) {
      const long n = id(x, y, z);
      if (type[n] == NODE_STRUCT) return;
      R dn = R(0), ux = R(0), uy = R(0), uz = R(0);
      for (int d = 0; d < 19; ++d) {
        R f = arF[d + n * 19];
        dn += f;
        ux += f * Dir[XDIM * 19 + d];
        uy += f * Dir[YDIM * 19 + d];
        uz += f * Dir[ZDIM * 19 + d];
      }
      ux /= dn;
      uy /= dn;
      uz /= dn;
      pden[n] = den[n];
      den[n] = dn;
      vx[n] = ux;
      vy[n] = uy;
      vz[n] = uz;
    });
  }

  /* One step in the order of runSimulation.cpp:263-264 / kernel.cu:168-199 */
  void step() {
    if (in.bEnableLES) les();
    if (in.bEnableMRT)
      mrt();
    else
      srt();
    streaming();
    if (in.casetype == CAVITY) {
      boundary_cavity();
      if (has_struct) boundary_struct();  // solid mask: keBoundaryStruct's rule
    } else if (in.casetype == POISEUILLE) {
      boundary_struct();
      boundary_inlet();
      boundary_outlet();
    } else if (in.casetype == CHANNEL) {
      boundary_cavity();
      if (has_struct) boundary_struct();
      boundary_inlet();
      boundary_outlet();
    }
    macroscopic();
  }
};

struct Handle {
  int dbl;
  Solver<float>* sf;
  Solver<double>* sd;
};

template <typename R>
void get_fields(Solver<R>* s, double* arF, double* den, double* vx, double* vy, double* vz,
                double* pden, double* te, int* nt, int* ds) {
  const long N = s->N;
  if (arF)
    for (long i = 0; i < N * 19; ++i) arF[i] = (double)s->arF[i];
  for (long i = 0; i < N; ++i) {
    if (den) den[i] = (double)s->den[i];
    if (vx) vx[i] = (double)s->vx[i];
    if (vy) vy[i] = (double)s->vy[i];
    if (vz) vz[i] = (double)s->vz[i];
    if (pden) pden[i] = (double)s->pden[i];
    if (te) te[i] = (double)s->tau_e[i];
    if (nt) nt[i] = s->type[i];
    if (ds) ds[i] = s->dstate[i];
  }
}

/* Import: overwrite arF and recompute CurrDen/CurrVel with the Macroscopic
 * codelet (PrevDen takes the old density, as a step would). */
template <typename R>
void set_arF(Solver<R>* s, const double* arF) {
  for (long i = 0; i < s->N * 19; ++i) s->arF[i] = (R)arF[i];
  s->macroscopic();
}

/* Solid voxels mask[ny][nz][nx] (nonzero = STRUCT; NULL removes them):
 * the lbm_set_solid_mask counterpart.  Restarts from the initial state. */
template <typename R>
void set_solid(Solver<R>* s, const unsigned char* mask) {
  if (mask)
    s->solid.assign(mask, mask + s->N);
  else
    s->solid.clear();
  std::fill(s->arF.begin(), s->arF.end(), R(0));
  std::fill(s->arFT.begin(), s->arFT.end(), R(0));
  for (auto* v : {&s->den, &s->pden, &s->vx, &s->vy, &s->vz, &s->tau_e})
    std::fill(v->begin(), v->end(), R(0));
  s->initialize();
}

}  // namespace

extern "C" {

void* orc_create(const Inputval* in, const orc_ext* ext) {
  if (!in) return nullptr;
  Handle* h = new Handle();
  h->dbl = ext ? ext->use_double : 0;
  h->sf = nullptr;
  h->sd = nullptr;
#ifdef _OPENMP
  if (ext && ext->threads > 0) omp_set_num_threads(ext->threads);
#endif
  int rc;
  if (h->dbl) {
    h->sd = new Solver<double>();
    rc = h->sd->setup(in, ext);
  } else {
    h->sf = new Solver<float>();
    rc = h->sf->setup(in, ext);
  }
  if (rc != 0) {
    delete h->sf;
    delete h->sd;
    delete h;
    return nullptr;
  }
  return h;
}

int orc_set_solid(void* hp, const unsigned char* mask) {
  Handle* h = (Handle*)hp;
  if (!h) return -1;
  if (h->dbl)
    set_solid(h->sd, mask);
  else
    set_solid(h->sf, mask);
  return 0;
}

int orc_step(void* hp, int nsteps) {
  Handle* h = (Handle*)hp;
  if (!h || nsteps < 0) return -1;
  for (int i = 0; i < nsteps; ++i) {
    if (h->dbl)
      h->sd->step();
    else
      h->sf->step();
  }
  return 0;
}

int orc_get(void* hp, double* arF, double* den, double* vx, double* vy, double* vz, double* pden,
            double* te, int* nt, int* ds) {
  Handle* h = (Handle*)hp;
  if (!h) return -1;
  if (h->dbl)
    get_fields(h->sd, arF, den, vx, vy, vz, pden, te, nt, ds);
  else
    get_fields(h->sf, arF, den, vx, vy, vz, pden, te, nt, ds);
  return 0;
}

int orc_set_arF(void* hp, const double* arF) {
  Handle* h = (Handle*)hp;
  if (!h || !arF) return -1;
  if (h->dbl)
    set_arF(h->sd, arF);
  else
    set_arF(h->sf, arF);
  return 0;
}

void orc_destroy(void* hp) {
  Handle* h = (Handle*)hp;
  if (!h) return;
  delete h->sf;
  delete h->sd;
  delete h;
}

int orc_decomposition(const Inputval* in, int Slice[][DIMENSION][2]) {
  return decompose(in, Slice);
}

/* decomposition.cpp:10-15 and 17-62 */
int orc_set_move_decomp(int NTILE, const int Slice[][DIMENSION][2], int Move[][DIRECTION_SIZE]) {
  for (int t = 0; t < NTILE; ++t) {
    const int px = (Slice[t][0][1] - Slice[t][0][0]) + 2;
    const int pz = (Slice[t][2][1] - Slice[t][2][0]) + 2;
    const int slave = px * pz;
    for (int d = 0; d < 19; ++d)
      Move[t][d] = (kCx[d] + 1) + (kCy[d] + 1) * slave + (kCz[d] + 1) * px;
  }
  return 0;
}

/* decomposition.cpp:66-94 */
int orc_slice_chunk(unsigned tile, const int Slice[][DIMENSION][2], int* xs, int* xe, int* ys,
                    int* ye, int* zs, int* ze, int* cnx, int* cny, int* cnz, int* clen) {
  *xs = Slice[tile][0][0];
  *xe = Slice[tile][0][1];
  *ys = Slice[tile][1][0];
  *ye = Slice[tile][1][1];
  *zs = Slice[tile][2][0];
  *ze = Slice[tile][2][1];
  int dx = *xe - *xs, dy = *ye - *ys, dz = *ze - *zs;
  *cnx = dx;
  *cny = dy;
  *cnz = dz;
  *clen = dx * dy * dz;
  if (dx < 1 || dy < 1 || dz < 1) return 1;
  return 0;
}

int orc_inverse_mrt(const float* mat, float* inv) { return inverse_gj<float>(mat, inv); }

void orc_tables(float* dir, int* opp, float* w, float* M) {
  for (int d = 0; d < 19; ++d) {
    if (dir) {
      dir[XDIM * 19 + d] = (float)kCx[d];
      dir[YDIM * 19 + d] = (float)kCy[d];
      dir[ZDIM * 19 + d] = (float)kCz[d];
    }
    if (opp) opp[d] = kOpp[d];
    if (w) w[d] = d == 0 ? 1.0f / 3.0f : (d < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
  }
  if (M)
    for (int i = 0; i < 19; ++i)
      for (int j = 0; j < 19; ++j) M[i * 19 + j] = (float)kM[i][j];
}

/* Unit noise and inlet profile, exported so tests can check the GPU
 * library's restatement of the same formulas. */
double orc_noise(uint64_t seed, uint64_t node, uint64_t comp) {
  return orc_unit_noise(seed, node, comp);
}
float orc_profile(float umax, int y, int z, int ny, int nz) {
  return orc_inlet_profile(umax, y, z, ny, nz);
}

}  // extern "C"
