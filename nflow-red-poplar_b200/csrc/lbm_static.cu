// lbm_static.cu — the FP64 field diagnostics for callers that must not
// allocate device memory.
//
// lbm_diagnostics() reduces through a per-domain buffer of per-block partial
// sums that lbm_create() obtains from cudaMalloc.  Some callers cannot call
// cudaMalloc at the point where they want these numbers: code that runs under
// a fixed device-memory budget owned entirely by its own pool (a serving loop
// that has handed every byte to resident domains), code that must not
// synchronise the device (cudaMalloc/cudaFree may), or code whose device
// memory is managed by another runtime.  lbm_field_diagnostics_static() takes
// the fields as caller-owned device arrays and reduces them through a
// file-scope __device__ array instead, so it allocates nothing.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; two calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on it.  Nothing in it has to
// start at zero: every block writes all of its partial sums before the final
// pass reads them.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/lbm_b200.h"
#include "lbm_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 64;                 // nodes per thread
constexpr int kMaxBlocks = 4096;           // partial-sum slots in the scratch array
constexpr long long kNodesPerBlock = (long long)kThreads * kItems;
constexpr long long kMaxNodes = kMaxBlocks * kNodesPerBlock;  // 67,108,864 nodes
constexpr int kOutSlot = kMaxBlocks * 8;   // 8 result values after the partials

// [kMaxBlocks][8] partial sums, then the 8 results (264 KB per device)
__device__ __align__(256) double g_diag_scratch[kMaxBlocks * 8 + 8];

// Host code cannot pass g_diag_scratch to a kernel: in host code the name is
// a host-side stand-in, not a device address.  The device address is looked
// up once per device with cudaGetSymbolAddress.
std::mutex g_mu;
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};

int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return lbm::set_error(LBM_ERR_NO_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return lbm::set_error(LBM_ERR_INVALID, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_diag_scratch);
    if (e != cudaSuccess || !p)
      return lbm::set_error(LBM_ERR_CUDA, "cudaGetSymbolAddress(g_diag_scratch) failed: %s",
                            cudaGetErrorString(e));
    g_scratch_addr[dev] = (double*)p;
  }
  *out = g_scratch_addr[dev];
  return LBM_OK;
}

// per block: [mass, momentum x, y, z, L1 residual, kinetic energy, max |u|,
// non-finite count] over nodes [blockIdx.x * kNodesPerBlock, +kNodesPerBlock)
__global__ void __launch_bounds__(kThreads)
    k_static_partial(const float* __restrict__ den, const float* __restrict__ den_prev,
                     const float* __restrict__ ux, const float* __restrict__ uy,
                     const float* __restrict__ uz, long long n, double* __restrict__ scratch) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const long long base = blockIdx.x * kNodesPerBlock;
  for (int k = 0; k < kItems; ++k) {
    const long long i = base + (long long)k * kThreads + threadIdx.x;
    if (i >= n) break;
    const double r = den[i], a = ux[i], b = uy[i], c = uz[i];
    if (!(isfinite(r) && isfinite(a) && isfinite(b) && isfinite(c))) {
      v[7] += 1.0;
      continue;
    }
    v[0] += r;
    v[1] += r * a;
    v[2] += r * b;
    v[3] += r * c;
    if (den_prev) v[4] += fabs(r - (double)den_prev[i]);
    const double u2 = a * a + b * b + c * c;
    v[5] += 0.5 * r * u2;
    v[6] = fmax(v[6], sqrt(u2));
  }
  __shared__ double sh[8][kThreads / 32];
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
    for (int w = 1; w < kThreads / 32; ++w) x = (k == 6) ? fmax(x, sh[k][w]) : x + sh[k][w];
    scratch[blockIdx.x * 8 + k] = x;
  }
}

// the nblocks partial sums -> scratch[kOutSlot .. kOutSlot + 8), fixed order
__global__ void k_static_final(double* __restrict__ scratch, int nblocks) {
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b)
      x = (k == 6) ? fmax(x, scratch[b * 8 + k]) : x + scratch[b * 8 + k];
    scratch[kOutSlot + k] = x;
  }
}

}  // namespace

extern "C" {

int lbm_field_diagnostics_static(const float* den, const float* den_prev, const float* velx,
                                 const float* vely, const float* velz, long long n, double out[8],
                                 void* stream) {
  if (!den || !velx || !vely || !velz || !out)
    return lbm::set_error(LBM_ERR_INVALID, "lbm_field_diagnostics_static: NULL argument");
  if (n <= 0) return lbm::set_error(LBM_ERR_INVALID, "lbm_field_diagnostics_static: n <= 0");
  if (n > kMaxNodes)
    return lbm::set_error(LBM_ERR_INVALID,
                          "lbm_field_diagnostics_static: %lld nodes exceed the static scratch "
                          "capacity of %lld nodes",
                          n, kMaxNodes);
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nblocks = (int)((n + kNodesPerBlock - 1) / kNodesPerBlock);
  k_static_partial<<<nblocks, kThreads, 0, st>>>(den, den_prev, velx, vely, velz, n, scratch);
  k_static_final<<<1, 32, 0, st>>>(scratch, nblocks);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, scratch + kOutSlot, 8 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return lbm::set_error(LBM_ERR_CUDA, "lbm_field_diagnostics_static: %s", cudaGetErrorString(e));
  return LBM_OK;
}

}  // extern "C"
