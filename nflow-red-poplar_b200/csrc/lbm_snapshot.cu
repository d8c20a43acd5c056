// lbm_snapshot.cu — result files and the residual stop on a live domain.
//
// kernel.cu:203-228 copies CurrDen / CurrVel / NodeType to the host with
// blocking cudaMemcpy every nwrite steps and writes the file before the next
// step starts.  Here the state after the last step is first copied on the
// device (ordered on the handle's stream, a few hundred microseconds for
// 256^3), then to pinned host memory on a side stream, so stepping resumes
// at once and the transfer and the file writing (host threads) overlap the
// following steps.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lbm_domain.cuh"

using namespace lbm;

namespace {

int ensure_snapshot_buffers(lbm_domain* d) {
  if (d->snap_dev) return LBM_OK;
  const size_t n = (size_t)d->N;
  if (cudaMalloc(&d->snap_dev, 4 * n * sizeof(float)) != cudaSuccess) {
    d->snap_dev = nullptr;
    return set_error(LBM_ERR_OOM, "snapshot buffer of %zu bytes", 4 * n * sizeof(float));
  }
  if (cudaMallocHost(&d->snap_host, 4 * n * sizeof(float)) != cudaSuccess) {
    d->snap_host = nullptr;
    return set_error(LBM_ERR_OOM, "pinned snapshot buffer of %zu bytes", 4 * n * sizeof(float));
  }
  d->snap_type = new int[n];
  CK(cudaStreamCreateWithFlags(&d->snap_stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&d->snap_taken, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&d->snap_landed, cudaEventDisableTiming));
  // the geometry does not change: node types once, synchronously
  return lbm_get_node_info(d, d->snap_type, nullptr);
}

// checkpoint file: this header, then the ghost-padded AoS arF
// [ny+2][nz+2][nx+2][19] as float32 (the lbm_export_arF(padded = 1) view)
struct CheckpointHeader {
  char magic[8];          // "LBMCKPT1"
  int32_t nx, ny, nz, q;  // extents and populations
  int64_t step;           // steps done when saved
  int32_t storage;        // LBM_STORE_* of the saving domain (information only)
  int32_t casetype;
  int64_t reserved[3];
};
static_assert(sizeof(CheckpointHeader) == 64, "checkpoint header is 64 bytes");
constexpr char kCheckpointMagic[8] = {'L', 'B', 'M', 'C', 'K', 'P', 'T', '1'};

std::string join(const char* dir, const char* name) {
  std::string p = dir ? dir : "./result/";
  if (!p.empty() && p.back() != '/') p += '/';
  return p + name;
}

}  // namespace

extern "C" {

int lbm_snapshot(lbm_domain* d) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "no state");
  int rc = ensure_device(d);
  if (rc) return rc;
  if ((rc = ensure_snapshot_buffers(d))) return rc;
  // a previous snapshot may still be travelling to the host buffer
  CK(cudaStreamSynchronize(d->snap_stream));
  const size_t n = (size_t)d->N, nb = n * sizeof(float);
  const float* src[4] = {d->den[d->step & 1], d->ux, d->uy, d->uz};
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(d->snap_dev + i * n, src[i], nb, cudaMemcpyDeviceToDevice, d->stream));
  CK(cudaEventRecord(d->snap_taken, d->stream));
  CK(cudaStreamWaitEvent(d->snap_stream, d->snap_taken, 0));
  CK(cudaMemcpyAsync(d->snap_host, d->snap_dev, 4 * nb, cudaMemcpyDeviceToHost, d->snap_stream));
  CK(cudaEventRecord(d->snap_landed, d->snap_stream));
  d->snap_valid = true;
  return LBM_OK;
}

int lbm_save_snapshot(lbm_domain* d, int savetype, const char* dir, int index) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->snap_valid) return set_error(LBM_ERR_STATE, "no snapshot taken");
  if (savetype != LBM_SAVE_VTU && savetype != LBM_SAVE_CSV)
    return set_error(LBM_ERR_INVALID, "unknown savetype %d", savetype);
  if (index < 0) return set_error(LBM_ERR_INVALID, "negative file index");
  // the output directory is created if its parent exists (kernel.cu expects
  // ./result/ to be there and exits otherwise)
  const std::string dirname = join(dir, "");
  if (mkdir(dirname.c_str(), 0755) != 0 && errno != EEXIST)
    return set_error(LBM_ERR_IO, "cannot create %s: %s", dirname.c_str(), std::strerror(errno));
  CK(cudaSetDevice(d->opt.device));
  CK(cudaEventSynchronize(d->snap_landed));
  const size_t n = (size_t)d->N;
  const float* h = d->snap_host;
  const int nx = d->in.nx, ny = d->in.ny, nz = d->in.nz;
  if (savetype == LBM_SAVE_VTU) {
    char name[32];
    std::snprintf(name, sizeof(name), "Output%06d.vtu", index);
    return lbm_write_vtu(join(dir, name).c_str(), nx, ny, nz, h, h + n, h + 2 * n, h + 3 * n,
                         d->snap_type);
  }
  return lbm_write_csv(join(dir, "result.csv").c_str(), join(dir, "section.csv").c_str(), nx, ny,
                       nz, h, h + n, h + 2 * n, h + 3 * n);
}

int lbm_save_file(lbm_domain* d, int savetype, const char* dir, int index) {
  int rc = lbm_snapshot(d);
  if (rc) return rc;
  return lbm_save_snapshot(d, savetype, dir, index);
}

int lbm_save_checkpoint(lbm_domain* d, const char* path) {
  if (!d || !path) return set_error(LBM_ERR_INVALID, "NULL argument");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "no state");
  const size_t n = (size_t)(d->in.nx + 2) * (d->in.ny + 2) * (d->in.nz + 2) * Q;
  std::vector<float> arF(n);
  int rc = lbm_export_arF(d, arF.data(), 1);
  if (rc) return rc;
  CheckpointHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kCheckpointMagic, 8);
  h.nx = d->in.nx;
  h.ny = d->in.ny;
  h.nz = d->in.nz;
  h.q = Q;
  h.step = d->step;
  h.storage = d->opt.storage;
  h.casetype = d->in.casetype;
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(LBM_ERR_IO, "cannot open %s", path);
  const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
                  std::fwrite(arF.data(), sizeof(float), n, f) == n;
  if (std::fclose(f) != 0 || !ok) return set_error(LBM_ERR_IO, "cannot write %s", path);
  return LBM_OK;
}

int lbm_load_checkpoint(lbm_domain* d, const char* path, long long* step) {
  if (!d || !path) return set_error(LBM_ERR_INVALID, "NULL argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(LBM_ERR_IO, "cannot open %s", path);
  CheckpointHeader h;
  if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kCheckpointMagic, 8) != 0) {
    std::fclose(f);
    return set_error(LBM_ERR_INVALID, "%s is not a checkpoint file", path);
  }
  if (h.nx != d->in.nx || h.ny != d->in.ny || h.nz != d->in.nz || h.q != Q) {
    std::fclose(f);
    return set_error(LBM_ERR_INVALID, "checkpoint %s is %dx%dx%d, the domain %dx%dx%d", path,
                     h.nx, h.ny, h.nz, d->in.nx, d->in.ny, d->in.nz);
  }
  const size_t n = (size_t)(h.nx + 2) * (h.ny + 2) * (h.nz + 2) * Q;
  std::vector<float> arF(n);
  const bool ok = std::fread(arF.data(), sizeof(float), n, f) == n;
  std::fclose(f);
  if (!ok) return set_error(LBM_ERR_IO, "checkpoint %s is truncated", path);
  int rc = lbm_import_arF(d, arF.data(), 1);
  if (rc) return rc;
  if (step) *step = h.step;
  return LBM_OK;
}

int lbm_run_until_converged(lbm_domain* d, int max_steps, int check_every, double tol,
                            int* steps_taken, double* residual) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (max_steps < 0 || check_every < 1 || !(tol >= 0.0))
    return set_error(LBM_ERR_INVALID, "max_steps >= 0, check_every >= 1 and tol >= 0 required");
  int done = 0;
  double r = -1.0;
  if (steps_taken) *steps_taken = 0;
  while (done < max_steps) {
    const int k = check_every < max_steps - done ? check_every : max_steps - done;
    int rc = lbm_run_simulation(d, k);
    if (rc) return rc;
    done += k;
    if (steps_taken) *steps_taken = done;
    double diag[8];
    if ((rc = lbm_diagnostics(d, diag))) return rc;
    r = diag[4];
    if (residual) *residual = r;
    if (diag[7] > 0)
      return set_error(LBM_ERR_NOT_FINITE, "state went non-finite after %d steps", done);
    if (r <= tol) break;
  }
  return LBM_OK;
}

}  // extern "C"
