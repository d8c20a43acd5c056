// lbm_api.cu — the C ABI of include/lbm_b200.h for single domains: device
// memory ownership, the step loop (one fused kernel launch per step), the
// AoS<->SoA import/export of the reference's arF layouts and the FP64
// diagnostics.  No CPU fallback exists: every compute path is a CUDA kernel
// and a missing or unusable device is reported as an error.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "lbm_domain.cuh"

using namespace lbm;

// any non-finite value in n floats -> *flag = 1
namespace {
__global__ void k_check_finite(const float* __restrict__ p, long long n, int* flag) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride)
    if (!isfinite(p[i])) *flag = 1;
}

}  // namespace

namespace lbm {

__global__ void k_node_info(Geometry g, int* __restrict__ type, int* __restrict__ ds) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= g.nx) return;
  const long long n = x + (long long)g.nx * (z + (long long)g.nz * y);
  if (type) type[n] = node_type(g, x, y, z);
  if (ds) ds[n] = direction_state(g, x, y, z);
}

constexpr int kDiagThreads = 256;

// per block: [mass, mom x, mom y, mom z, L1 residual, kinetic energy,
// max |u|, non-finite count]; fixed grid and fixed reduction tree, so the
// result does not depend on scheduling.
__global__ void __launch_bounds__(kDiagThreads)
    k_diag_partial(const float* __restrict__ den, const float* __restrict__ den_prev,
                   const float* __restrict__ ux, const float* __restrict__ uy,
                   const float* __restrict__ uz, long long n, int has_prev,
                   double* __restrict__ partial) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const double r = den[i], a = ux[i], b = uy[i], c = uz[i];
    if (!(isfinite(r) && isfinite(a) && isfinite(b) && isfinite(c))) {
      v[7] += 1.0;
      continue;
    }
    v[0] += r;
    v[1] += r * a;
    v[2] += r * b;
    v[3] += r * c;
    if (has_prev) v[4] += fabs(r - (double)den_prev[i]);
    const double u2 = a * a + b * b + c * c;
    v[5] += 0.5 * r * u2;
    v[6] = fmax(v[6], sqrt(u2));
  }
  __shared__ double sh[8][kDiagThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 8; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = (k == 6) ? fmax(x, y) : x + y;
    }
    if (lane == 0) sh[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    double x = sh[k][0];
    for (int w = 1; w < kDiagThreads / 32; ++w) x = (k == 6) ? fmax(x, sh[k][w]) : x + sh[k][w];
    partial[blockIdx.x * 8 + k] = x;
  }
}

__global__ void k_diag_final(const double* __restrict__ partial, int nblocks,
                             double* __restrict__ out) {
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b)
      x = (k == 6) ? fmax(x, partial[b * 8 + k]) : x + partial[b * 8 + k];
    out[k] = x;
  }
}

}  // namespace lbm

extern "C" {

int lbm_estimate_bytes(const Inputval* pinput, const lbm_options* opt, size_t* bytes) {
  int rc = validate(pinput, opt);
  if (rc != LBM_OK) return rc;
  if (!bytes) return set_error(LBM_ERR_INVALID, "NULL bytes");
  *bytes = footprint(pinput, opt);
  return LBM_OK;
}

int lbm_create(const Inputval* pinput, const lbm_options* opt, lbm_domain** out) {
  if (!out) return set_error(LBM_ERR_INVALID, "NULL out");
  *out = nullptr;
  int rc = validate(pinput, opt);
  if (rc != LBM_OK) return rc;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return set_error(LBM_ERR_NO_DEVICE, "no CUDA device available (%s)",
                     e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
  lbm_domain* d = new (std::nothrow) lbm_domain();
  if (!d) return set_error(LBM_ERR_OOM, "host allocation failed");
  if (opt)
    d->opt = *opt;
  else
    lbm_default_options(&d->opt);
  if (d->opt.device < 0 || d->opt.device >= ndev) {
    delete d;
    return set_error(LBM_ERR_INVALID, "device %d out of range (%d devices)", d->opt.device, ndev);
  }
  auto fail = [&](int code) {
    free_all(d);
    delete d;
    return code;
  };
  if ((rc = ensure_device(d)) != LBM_OK) return fail(rc);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, d->opt.device) != cudaSuccess || prop.major < 10)
    return fail(set_error(LBM_ERR_NO_DEVICE, "device %d is not an sm_100 GPU", d->opt.device));
  domain_prepare(d, pinput, opt);
  auto alloc = [&](void** p, size_t b) -> int {
    cudaError_t ce = cudaMalloc(p, b);
    if (ce != cudaSuccess)
      return set_error(ce == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,
                       "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(ce));
    d->bytes += b;
    return LBM_OK;
  };
  // device words: [0] input check, [1] kernel error, [2..3] step counter
  if ((rc = domain_alloc_state(d, alloc)) || (rc = alloc((void**)&d->flag, 4 * sizeof(int))))
    return fail(rc);
  if (cudaMemset(d->flag, 0, 4 * sizeof(int)) != cudaSuccess)
    return fail(set_error(LBM_ERR_CUDA, "flag reset failed"));
  rc = storage_ops(d->opt.storage).tensor_maps(d, prop.multiProcessorCount);
  if (rc) return fail(rc);
  d->diag_blocks = 4 * prop.multiProcessorCount;
  if ((rc = alloc((void**)&d->partial, (size_t)d->diag_blocks * 8 * sizeof(double))) ||
      (rc = alloc((void**)&d->dout, 8 * sizeof(double))))
    return fail(rc);
  if (cudaStreamCreateWithFlags(&d->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess)
    return fail(set_error(LBM_ERR_CUDA, "stream/event creation failed"));
  d->stream = d->own;
  if ((rc = domain_upload_profile(d, d->stream))) return fail(rc);
  clear_error();
  *out = d;
  return LBM_OK;
}

int lbm_destroy(lbm_domain* d) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  cudaSetDevice(d->opt.device);
  if (d->stream) cudaStreamSynchronize(d->stream);
  free_all(d);
  delete d;
  return LBM_OK;
}

int lbm_set_stream(lbm_domain* d, void* s) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  d->stream = (cudaStream_t)s;  // NULL: the CUDA default stream
  return LBM_OK;
}

void* lbm_get_stream(lbm_domain* d) { return d ? (void*)d->stream : nullptr; }

int lbm_initialize(lbm_domain* d) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  int rc = ensure_device(d);
  if (rc) return rc;
  return domain_launch_init(d, d->stream);
}

}  // extern "C"

extern "C" {

int lbm_set_solid_mask(lbm_domain* d, const unsigned char* mask) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (d->pooled) return set_error(LBM_ERR_INVALID, "batch members take no solid mask");
  if (d->opt.stream_mode == LBM_STREAM_AA && mask)
    return set_error(LBM_ERR_INVALID, "solid masks need the pull (A/B) streaming");
  int rc = ensure_device(d);
  if (rc) return rc;
  if (mask) {
    if (!d->solid && cudaMalloc(&d->solid, (size_t)d->N) != cudaSuccess) {
      d->solid = nullptr;
      return set_error(LBM_ERR_OOM, "solid mask of %lld bytes", d->N);
    }
    CK(cudaMemcpyAsync(d->solid, mask, (size_t)d->N, cudaMemcpyHostToDevice, d->stream));
    d->g.solid = d->solid;
  } else {
    d->g.solid = nullptr;
  }
  // the step kernel and its captured graphs depend on the geometry
  for (int i = 0; i < 2; ++i)
    if (d->chunk[i]) {
      cudaGraphExecDestroy(d->chunk[i]);
      d->chunk[i] = nullptr;
    }
  return domain_launch_init(d, d->stream);
}

int lbm_run_simulation(lbm_domain* d, int nsteps) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "lbm_run_simulation before lbm_initialize");
  if (nsteps < 0) return set_error(LBM_ERR_INVALID, "nsteps=%d < 0", nsteps);
  if (nsteps == 0) return LBM_OK;
  int rc = ensure_device(d);
  if (rc) return rc;
  CK(cudaEventRecord(d->ev0, d->stream));
  if (d->opt.stream_mode == LBM_STREAM_AA) {
    rc = storage_ops(d->opt.storage).run_aa(d, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(d->ev1, d->stream));
    d->last_steps = nsteps;
    return LBM_OK;
  }
  rc = storage_ops(d->opt.storage).run_pull(d, nsteps);
  if (rc) return rc;
  CK(cudaEventRecord(d->ev1, d->stream));
  d->last_steps = nsteps;
  return LBM_OK;
}

int lbm_steps_done(const lbm_domain* d, long long* steps) {
  if (!d || !steps) return set_error(LBM_ERR_INVALID, "NULL argument");
  *steps = d->step;
  return LBM_OK;
}

int lbm_last_run_ms(lbm_domain* d, float* ms) {
  if (!d || !ms) return set_error(LBM_ERR_INVALID, "NULL argument");
  if (d->last_steps <= 0) return set_error(LBM_ERR_STATE, "no run recorded");
  int rc = ensure_device(d);
  if (rc) return rc;
  CK(cudaEventSynchronize(d->ev1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, d->ev0, d->ev1));
  *ms = t / (float)d->last_steps;
  return LBM_OK;
}

int lbm_import_arF(lbm_domain* d, const float* arF, int padded) {
  if (!d || !arF) return set_error(LBM_ERR_INVALID, "NULL argument");
  int rc = ensure_device(d);
  if (rc) return rc;
  const long long nodes =
      padded ? (long long)(d->g.nx + 2) * (d->g.ny + 2) * (d->g.nz + 2) : d->N;
  const size_t bytes = (size_t)nodes * Q * sizeof(float);
  if ((rc = ensure_staging(d, bytes))) return rc;
  CK(cudaMemcpyAsync(d->staging, arF, bytes, cudaMemcpyHostToDevice, d->stream));
  CK(cudaMemsetAsync(d->den[1], 0, (size_t)d->N * sizeof(float), d->stream));
  CK(cudaMemsetAsync(d->flag, 0, sizeof(int), d->stream));
  k_check_finite<<<4 * 148, 256, 0, d->stream>>>(d->staging, nodes * Q, d->flag);
  int hflag = 0;
  CK(cudaMemcpyAsync(&hflag, d->flag, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  if (hflag) {
    d->initialized = false;
    return set_error(LBM_ERR_NOT_FINITE, "lbm_import_arF: input holds NaN/Inf");
  }
  rc = storage_ops(d->opt.storage).import_staging(d, padded);
  if (rc) return rc;
  d->cur = 0;
  d->post_direct = true;
  CK(cudaMemsetAsync(d->flag + 2, 0, 2 * sizeof(int), d->stream));  // step counter
  d->aa_first = false;
  d->step = 0;
  d->initialized = true;
  d->last_steps = 0;
  return LBM_OK;
}

int lbm_export_arF(lbm_domain* d, float* arF, int padded) {
  if (!d || !arF) return set_error(LBM_ERR_INVALID, "NULL argument");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "lbm_export_arF before lbm_initialize");
  int rc = ensure_device(d);
  if (rc) return rc;
  const long long nodes =
      padded ? (long long)(d->g.nx + 2) * (d->g.ny + 2) * (d->g.nz + 2) : d->N;
  const size_t bytes = (size_t)nodes * Q * sizeof(float);
  if ((rc = ensure_staging(d, bytes))) return rc;
  if (padded) CK(cudaMemsetAsync(d->staging, 0, bytes, d->stream));
  rc = storage_ops(d->opt.storage).export_staging(d, padded);
  if (rc) return rc;
  CK(cudaMemcpyAsync(arF, d->staging, bytes, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return check_kernel_error(d);
}

int lbm_get_macroscopic(lbm_domain* d, float* den, float* velx, float* vely, float* velz) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "no state");
  int rc = ensure_device(d);
  if (rc) return rc;
  const size_t nb = (size_t)d->N * sizeof(float);
  if (den) CK(cudaMemcpyAsync(den, d->den[d->step & 1], nb, cudaMemcpyDeviceToHost, d->stream));
  if (velx) CK(cudaMemcpyAsync(velx, d->ux, nb, cudaMemcpyDeviceToHost, d->stream));
  if (vely) CK(cudaMemcpyAsync(vely, d->uy, nb, cudaMemcpyDeviceToHost, d->stream));
  if (velz) CK(cudaMemcpyAsync(velz, d->uz, nb, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return check_kernel_error(d);
}

int lbm_get_node_info(lbm_domain* d, int* node_type, int* direction_state) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  int rc = ensure_device(d);
  if (rc) return rc;
  const size_t nb = (size_t)d->N * sizeof(int);
  if ((rc = ensure_staging(d, 2 * nb))) return rc;
  int* t = (int*)d->staging;
  int* s = t + d->N;
  const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
  k_node_info<<<gr, b, 0, d->stream>>>(d->g, t, s);
  CK(cudaGetLastError());
  if (node_type) CK(cudaMemcpyAsync(node_type, t, nb, cudaMemcpyDeviceToHost, d->stream));
  if (direction_state)
    CK(cudaMemcpyAsync(direction_state, s, nb, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBM_OK;
}

int lbm_diagnostics(lbm_domain* d, double out[8]) {
  if (!d || !out) return set_error(LBM_ERR_INVALID, "NULL argument");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "no state");
  int rc = ensure_device(d);
  if (rc) return rc;
  if ((rc = ensure_diag_buffers(d))) return rc;
  const long long k = d->step;
  k_diag_partial<<<d->diag_blocks, kDiagThreads, 0, d->stream>>>(
      d->den[k & 1], d->den[(k + 1) & 1], d->ux, d->uy, d->uz, d->N, k > 0 ? 1 : 0, d->partial);
  k_diag_final<<<1, 32, 0, d->stream>>>(d->partial, d->diag_blocks, d->dout);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d->dout, 8 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBM_OK;
}

int lbm_sync(lbm_domain* d) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  int rc = ensure_device(d);
  if (rc) return rc;
  CK(cudaStreamSynchronize(d->stream));
  return check_kernel_error(d);
}

int lbm_device_bytes(const lbm_domain* d, size_t* bytes) {
  if (!d || !bytes) return set_error(LBM_ERR_INVALID, "NULL argument");
  *bytes = d->bytes;
  return LBM_OK;
}

int lbm_device_fields(lbm_domain* d, float** den, float** prev_den, float** velx, float** vely,
                      float** velz) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "domain not initialized");
  if (den) *den = d->den[d->step & 1];
  if (prev_den) *prev_den = d->den[(d->step + 1) & 1];
  if (velx) *velx = d->ux;
  if (vely) *vely = d->uy;
  if (velz) *velz = d->uz;
  return LBM_OK;
}

}  // extern "C"
