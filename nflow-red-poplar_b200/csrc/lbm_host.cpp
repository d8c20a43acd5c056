// lbm_host.cpp — host numerics of the drop-in surface (no GPU needed):
// decomposition / set_move_decomp / slice_chunk (decomposition.cpp:10-161),
// the Gauss-Jordan inverseMRT (inverseMRT.cpp:8-92), the D3Q19 tables of
// main.cpp:87-171, default options and the per-thread error message.
//
// Built with -ffp-contract=off so that lbm_inverse_mrt rounds exactly like
// the reference's FP32 inverseMRT.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_internal.h"

namespace {
thread_local std::string g_last_error;

const int kCx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int kCy[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int kCz[19] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
const int kOpp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
const signed char kM[19][19] = {
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
}  // namespace

namespace lbm {
int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
void clear_error() { g_last_error.clear(); }
}  // namespace lbm

extern "C" {

const char* lbm_last_error(void) { return g_last_error.c_str(); }

const char* lbm_version(void) { return "nflow-red-poplar_b200 0.1 (sm_100a)"; }

void lbm_default_options(lbm_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->storage = LBM_STORE_F32;
  opt->init_kind = LBM_INIT_REFERENCE;
  opt->seed = 1;
  opt->noise_amp = 0.0f;
  opt->store_scale = 0.0f;
  opt->stream_mode = LBM_STREAM_AB;
  opt->device = 0;
}

int lbm_decomposition(const Inputval* pinput, int Slice[][DIMENSION][2]) {
  if (!pinput || !Slice) return lbm::set_error(LBM_ERR_INVALID, "lbm_decomposition: NULL argument");
  if (pinput->nx < 1 || pinput->ny < 1 || pinput->nz < 1)
    return lbm::set_error(LBM_ERR_INVALID, "lbm_decomposition: non-positive extent");
  const int ext[3] = {pinput->nx, pinput->ny, pinput->nz};
  const int dec[3] = {XDECOMP, YDECOMP, ZDECOMP};
  int chunk[3];
  for (int m = 0; m < 3; ++m) chunk[m] = ext[m] / dec[m];
  int tiles = 0;
  int st[3], ed[3];
  for (int i = 0; i < dec[0]; ++i) {
    st[0] = i * chunk[0];
    ed[0] = (i == dec[0] - 1) ? ext[0] : (i + 1) * chunk[0];
    if (ed[0] > ext[0]) ed[0] = ext[0];
    for (int j = 0; j < dec[1]; ++j) {
      st[1] = j * chunk[1];
      ed[1] = (j == dec[1] - 1) ? ext[1] : (j + 1) * chunk[1];
      if (ed[1] > ext[1]) ed[1] = ext[1];
      for (int k = 0; k < dec[2]; ++k) {
        st[2] = k * chunk[2];
        ed[2] = (k == dec[2] - 1) ? ext[2] : (k + 1) * chunk[2];
        if (ed[2] > ext[2]) ed[2] = ext[2];
        for (int m = 0; m < DIMENSION; ++m) {
          Slice[tiles][m][0] = st[m];
          Slice[tiles][m][1] = ed[m];
        }
        ++tiles;
      }
    }
  }
  return tiles;
}

int lbm_set_move_decomp(int NTILE, const int Slice[][DIMENSION][2], int Move[][DIRECTION_SIZE]) {
  if (NTILE < 0 || (NTILE > 0 && (!Slice || !Move)))
    return lbm::set_error(LBM_ERR_INVALID, "lbm_set_move_decomp: bad argument");
  for (int t = 0; t < NTILE; ++t) {
    // padded chunk extents; neighbour (x,y,z) -> (x+1) + (y+1)*slave + (z+1)*px
    const int px = (Slice[t][0][1] - Slice[t][0][0]) + 2;
    const int pz = (Slice[t][2][1] - Slice[t][2][0]) + 2;
    const int slave = px * pz;
    for (int d = 0; d < DIRECTION_SIZE; ++d)
      Move[t][d] = (kCx[d] + 1) + (kCy[d] + 1) * slave + (kCz[d] + 1) * px;
  }
  return 0;
}

int lbm_slice_chunk(unsigned tile, const int Slice[][DIMENSION][2], int* xs, int* xe, int* ys,
                    int* ye, int* zs, int* ze, int* chunk_nx, int* chunk_ny, int* chunk_nz,
                    int* chunk_len) {
  if (!Slice || !xs || !xe || !ys || !ye || !zs || !ze || !chunk_nx || !chunk_ny || !chunk_nz ||
      !chunk_len)
    return lbm::set_error(LBM_ERR_INVALID, "lbm_slice_chunk: NULL argument");
  *xs = Slice[tile][0][0];
  *xe = Slice[tile][0][1];
  *ys = Slice[tile][1][0];
  *ye = Slice[tile][1][1];
  *zs = Slice[tile][2][0];
  *ze = Slice[tile][2][1];
  const int dx = *xe - *xs, dy = *ye - *ys, dz = *ze - *zs;
  *chunk_nx = dx;
  *chunk_ny = dy;
  *chunk_nz = dz;
  *chunk_len = dx * dy * dz;
  return (dx < 1 || dy < 1 || dz < 1) ? 1 : 0;
}

// Gauss-Jordan elimination in FP32 with the reference's pivot handling: a
// row whose pivot is below 1e-9 in magnitude is rotated to the bottom.  The
// rotation is bounded (the reference loops for ever on a singular matrix)
// and a singular matrix is reported, not exit()ed.
int lbm_inverse_mrt(const float* mat, float* inv) {
  if (!mat || !inv) return lbm::set_error(LBM_ERR_INVALID, "lbm_inverse_mrt: NULL argument");
  const int n = DIRECTION_SIZE;
  std::vector<std::vector<float>> a(n, std::vector<float>(n)), p(n, std::vector<float>(n, 0.0f));
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) a[i][j] = mat[i * n + j];
  for (int i = 0; i < n; ++i) p[i][i] = 1.0f;
  const double tiny = std::pow(10.0, -9.0);
  for (int i = 0; i < n - 1; ++i) {
    int rotations = 0;
    while (std::fabs(a[i][i]) < tiny) {
      if (++rotations > n - i)
        return lbm::set_error(LBM_ERR_SINGULAR, "lbm_inverse_mrt: singular matrix");
      std::vector<float> ra = a[i], rp = p[i];
      for (int j = i; j < n - 1; ++j) {
        a[j] = a[j + 1];
        p[j] = p[j + 1];
      }
      a[n - 1] = ra;
      p[n - 1] = rp;
    }
    const float piv = a[i][i];
    for (int j = 0; j < n; ++j) {
      p[i][j] = p[i][j] / piv;
      a[i][j] = a[i][j] / piv;
    }
    const std::vector<float> ra = a[i], rp = p[i];
    for (int j = i + 1; j < n; ++j) {
      const float fac = a[j][i];
      for (int k = 0; k < n; ++k) {
        p[j][k] = p[j][k] - rp[k] * fac;
        a[j][k] = a[j][k] - ra[k] * fac;
      }
    }
  }
  const float last = a[n - 1][n - 1];
  for (int i = 0; i < n; ++i) {
    p[n - 1][i] = p[n - 1][i] / last;
    a[n - 1][i] = a[n - 1][i] / last;
  }
  for (int i = n - 1; i > 0; --i) {
    const std::vector<float> ra = a[i], rp = p[i];
    for (int j = i - 1; j >= 0; --j) {
      const float fac = a[j][i];
      for (int k = 0; k < n; ++k) {
        p[j][k] = p[j][k] - rp[k] * fac;
        a[j][k] = a[j][k] - ra[k] * fac;
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    float s = 0.0f;
    for (int j = 0; j < n; ++j) s += std::fabs(a[i][j]);
    if (s < std::pow(10.0, -10.0))
      return lbm::set_error(LBM_ERR_SINGULAR, "lbm_inverse_mrt: singular matrix");
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) inv[i * n + j] = p[i][j];
  return LBM_OK;
}

void lbm_d3q19_tables(float* direction, int* opp, float* w, float* M) {
  for (int d = 0; d < DIRECTION_SIZE; ++d) {
    if (direction) {
      direction[XDIM * DIRECTION_SIZE + d] = (float)kCx[d];
      direction[YDIM * DIRECTION_SIZE + d] = (float)kCy[d];
      direction[ZDIM * DIRECTION_SIZE + d] = (float)kCz[d];
    }
    if (opp) opp[d] = kOpp[d];
    if (w) w[d] = d == 0 ? 1.0f / 3.0f : (d < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
  }
  if (M)
    for (int i = 0; i < DIRECTION_SIZE; ++i)
      for (int j = 0; j < DIRECTION_SIZE; ++j) M[i * DIRECTION_SIZE + j] = (float)kM[i][j];
}

}  // extern "C"
