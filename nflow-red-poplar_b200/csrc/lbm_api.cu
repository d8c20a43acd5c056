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

#include "lbm_internal.h"
#include "lbm_kernels.cuh"

using namespace lbm;

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return set_error(e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,      \
                       "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                         \
  } while (0)

struct lbm_domain {
  Inputval in;
  lbm_options opt;
  Geometry g;
  long long N = 0;    // nodes nx*ny*nz
  long long qs = 0;   // population stride in elements
  size_t elem = 4;    // bytes per stored population
  void* lat[2] = {nullptr, nullptr};
  int cur = 0;               // lattice holding f*_k
  bool post_direct = false;  // lat[cur^1] holds arF_k itself
  long long step = 0;
  bool initialized = false;
  float* den[2] = {nullptr, nullptr};  // rho_k in den[k&1], rho_{k-1} in den[(k-1)&1]
  float* ux = nullptr;
  float* uy = nullptr;
  float* uz = nullptr;
  float* inlet_u = nullptr;                // [ny*nz]
  float* prho[2] = {nullptr, nullptr};     // [ny*nz]
  float* pu[2] = {nullptr, nullptr};       // [2][3][ny*nz]
  float* staging = nullptr;                // AoS import/export buffer
  size_t staging_bytes = 0;
  int* flag = nullptr;                     // device error flag
  double* partial = nullptr;
  double* dout = nullptr;
  int diag_blocks = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int last_steps = 0;
  float scale = 1.f, inv_scale = 1.f;
  size_t bytes = 0;
  // CUDA graphs of kGraphSteps plain steps, one per starting lattice
  cudaGraphExec_t chunk[2] = {nullptr, nullptr};
  cudaStream_t capture = nullptr;
};

// steps per captured graph chunk (even, so that a chunk returns the lattices
// and the boundary planes to the parity it started from)
constexpr int kGraphSteps = 32;

namespace {

template <class T>
struct Tag {
  using type = T;
};

// call f(Tag<S>{}) with the storage type of the domain
template <class F>
int with_storage(int storage, F&& f) {
  switch (storage) {
    case LBM_STORE_F32: return f(Tag<float>{});
    case LBM_STORE_F64: return f(Tag<double>{});
    case LBM_STORE_F16_SHIFT: return f(Tag<__half>{});
    case LBM_STORE_BF16_SHIFT: return f(Tag<__nv_bfloat16>{});
  }
  return set_error(LBM_ERR_INVALID, "unknown storage %d", storage);
}

size_t storage_bytes(int storage) {
  switch (storage) {
    case LBM_STORE_F64: return 8;
    case LBM_STORE_F16_SHIFT:
    case LBM_STORE_BF16_SHIFT: return 2;
    default: return 4;
  }
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

int validate(const Inputval* in, const lbm_options* opt) {
  if (!in) return set_error(LBM_ERR_INVALID, "NULL Inputval");
  if (in->nx < 3 || in->ny < 3 || in->nz < 3)
    return set_error(LBM_ERR_INVALID, "domain %dx%dx%d too small (each extent must be >= 3)",
                     in->nx, in->ny, in->nz);
  if (in->ny > 65535 || in->nz > 65535)
    return set_error(LBM_ERR_INVALID, "ny and nz must be <= 65535");
  if (round_up(in->nx, 8) * (long long)in->ny * in->nz >= (1LL << 31) - 1024)
    return set_error(LBM_ERR_INVALID, "domain too large (px*ny*nz must be < 2^31)");
  if (in->casetype != CAVITY && in->casetype != CHANNEL)
    return set_error(LBM_ERR_INVALID,
                     "casetype %d not supported (CAVITY=1 and CHANNEL=2 are implemented)",
                     in->casetype);
  if (!(std::isfinite(in->m_dTau) && in->m_dTau > 0.0f))
    return set_error(LBM_ERR_INVALID, "relaxation time tau=%g must be positive", in->m_dTau);
  if (!(std::isfinite(in->m_dRefDen) && in->m_dRefDen > 0.0f))
    return set_error(LBM_ERR_INVALID, "RefDen=%g must be positive", in->m_dRefDen);
  if (!std::isfinite(in->m_dSmagorinsky) || !std::isfinite(in->m_dRefVelx) ||
      !std::isfinite(in->m_dRefVely) || !std::isfinite(in->m_dRefVelz) ||
      !std::isfinite(in->dWeps) || !std::isfinite(in->dWepsj) || !std::isfinite(in->dWXX))
    return set_error(LBM_ERR_NOT_FINITE, "non-finite parameter in Inputval");
  if (opt) {
    if (opt->storage < LBM_STORE_F32 || opt->storage > LBM_STORE_F64)
      return set_error(LBM_ERR_INVALID, "unknown storage %d", opt->storage);
    if (opt->init_kind < LBM_INIT_REFERENCE || opt->init_kind > LBM_INIT_CHANNEL)
      return set_error(LBM_ERR_INVALID, "unknown init_kind %d", opt->init_kind);
    if (opt->stream_mode != LBM_STREAM_AB)
      return set_error(LBM_ERR_INVALID, "stream_mode %d not supported", opt->stream_mode);
    if (!std::isfinite(opt->noise_amp) || !std::isfinite(opt->store_scale) ||
        opt->store_scale < 0.0f)
      return set_error(LBM_ERR_INVALID, "bad noise_amp/store_scale");
  }
  return LBM_OK;
}

struct Sizes {
  long long N, qs, P;
  int px;
};

// Extra elements between population planes (a multiple of 128); a non-zero
// value keeps the 19 streams of a node off power-of-two distances.
#ifndef LBM_PLANE_PAD
#define LBM_PLANE_PAD 0
#endif

Sizes sizes_of(const Inputval* in) {
  Sizes s;
  s.px = (int)round_up(in->nx, 8);
  s.N = (long long)in->nx * in->ny * in->nz;
  s.qs = round_up((long long)s.px * in->nz * in->ny, 128) + LBM_PLANE_PAD;
  s.P = (long long)in->ny * in->nz;
  return s;
}

size_t footprint(const Inputval* in, const lbm_options* opt) {
  const Sizes s = sizes_of(in);
  const size_t e = storage_bytes(opt ? opt->storage : LBM_STORE_F32);
  size_t b = 2 * (size_t)Q * s.qs * e;  // lattices
  b += 5 * (size_t)s.N * sizeof(float);  // den[2], ux, uy, uz
  b += 15 * (size_t)s.P * sizeof(float); // inlet profile + planes
  return b;
}

dim3 block_of(int nx) {
  int bx = (int)round_up(nx < 128 ? nx : 128, 32);
  return dim3(bx, 1, 1);
}
dim3 grid_of(const Geometry& g, dim3 b) {
  return dim3((g.nx + b.x - 1) / b.x, g.nz, g.ny);
}

template <class S>
StepArgs<S> make_args(const lbm_domain* d, const void* src, void* dst, long long k) {
  using R = RealOf<S>;
  StepArgs<S> a;
  std::memset(&a, 0, sizeof(a));
  a.src = (const S*)src;
  a.dst = (S*)dst;
  a.qs = d->qs;
  for (int q = 0; q < Q; ++q) {
    a.srcq[q] = src ? (const S*)src + q * d->qs : nullptr;
    a.dstq[q] = dst ? (S*)dst + q * d->qs : nullptr;
    a.off[q] = cx(q) + d->g.px * (cz(q) + d->g.nz * cy(q));
  }
  a.g = d->g;
  a.tau = R(d->in.m_dTau);
  const double cs = (double)d->in.m_dSmagorinsky;
  a.les_c = R((double)(18.0f * 1.41421356237f) * cs * cs);
  a.rho0 = R(d->in.m_dRefDen);
  a.ulx = R(d->in.m_dRefVelx);
  a.uly = R(d->in.m_dRefVely);
  a.ulz = R(d->in.m_dRefVelz);
  a.mp.rho0_inv = R(1) / R(d->in.m_dRefDen);
  a.mp.weps = R(d->in.dWeps);
  a.mp.wepsj = R(d->in.dWepsj);
  a.mp.wxx = R(d->in.dWXX);
  a.scale = d->scale;
  a.inv_scale = d->inv_scale;
  a.inlet_u = d->inlet_u;
  a.prho_in = d->prho[(k + 1) & 1];  // (k-1)&1
  a.prho_out = d->prho[k & 1];
  a.pu_in = d->pu[(k + 1) & 1];
  a.pu_out = d->pu[k & 1];
  return a;
}

// kernel selection by (collision, LES) at run time
template <class S, class F>
int with_model(const lbm_domain* d, F&& f) {
  const bool mrt = d->in.bEnableMRT, les = d->in.bEnableLES;
  if (mrt && les) return f(std::integral_constant<int, COLL_MRT>{}, std::true_type{});
  if (mrt) return f(std::integral_constant<int, COLL_MRT>{}, std::false_type{});
  if (les) return f(std::integral_constant<int, COLL_SRT>{}, std::true_type{});
  return f(std::integral_constant<int, COLL_SRT>{}, std::false_type{});
}

// the fused step kernel of the domain's storage: the packed two-node kernel
// for the FP32-arithmetic formats (unless the scalar one is requested),
// the scalar kernel for the FP64 build
template <class S, int COLL, bool LES>
void launch_step(const lbm_domain* d, const StepArgs<S>& a, cudaStream_t st) {
  if constexpr (!std::is_same<S, double>::value) {
    if (d->opt.kernel == LBM_KERNEL_PACKED) {
      const int pairs = (d->g.nx + 1) / 2;
      const dim3 b(64, 1, 1), gr((pairs + 63) / 64, d->g.nz, d->g.ny);
      k_step2<S, COLL, LES><<<gr, b, 0, st>>>(a);
      return;
    }
  }
  const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
  k_step<S, COLL, LES><<<gr, b, 0, st>>>(a);
}

int ensure_device(const lbm_domain* d) {
  CK(cudaSetDevice(d->opt.device));
  return LBM_OK;
}

int ensure_staging(lbm_domain* d, size_t bytes) {
  if (d->staging_bytes >= bytes) return LBM_OK;
  if (d->staging) {
    CK(cudaFree(d->staging));
    d->bytes -= d->staging_bytes;
    d->staging = nullptr;
    d->staging_bytes = 0;
  }
  CK(cudaMalloc(&d->staging, bytes));
  d->staging_bytes = bytes;
  d->bytes += bytes;
  return LBM_OK;
}

void free_all(lbm_domain* d) {
  for (int i = 0; i < 2; ++i) {
    if (d->lat[i]) cudaFree(d->lat[i]);
    if (d->den[i]) cudaFree(d->den[i]);
    if (d->prho[i]) cudaFree(d->prho[i]);
    if (d->pu[i]) cudaFree(d->pu[i]);
  }
  if (d->ux) cudaFree(d->ux);
  if (d->uy) cudaFree(d->uy);
  if (d->uz) cudaFree(d->uz);
  if (d->inlet_u) cudaFree(d->inlet_u);
  if (d->staging) cudaFree(d->staging);
  if (d->flag) cudaFree(d->flag);
  if (d->partial) cudaFree(d->partial);
  if (d->dout) cudaFree(d->dout);
  for (int i = 0; i < 2; ++i)
    if (d->chunk[i]) cudaGraphExecDestroy(d->chunk[i]);
  if (d->capture) cudaStreamDestroy(d->capture);
  if (d->ev0) cudaEventDestroy(d->ev0);
  if (d->ev1) cudaEventDestroy(d->ev1);
  if (d->own) cudaStreamDestroy(d->own);
}

// any non-finite value in n floats -> *flag = 1
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
  d->in = *pinput;
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
  const Sizes s = sizes_of(pinput);
  d->g.nx = pinput->nx;
  d->g.ny = pinput->ny;
  d->g.nz = pinput->nz;
  d->g.px = s.px;
  d->g.casetype = pinput->casetype;
  d->N = s.N;
  d->qs = s.qs;
  d->elem = storage_bytes(d->opt.storage);
  if (d->opt.storage == LBM_STORE_F16_SHIFT || d->opt.storage == LBM_STORE_BF16_SHIFT) {
    float sc = d->opt.store_scale;
    if (sc == 0.0f) sc = d->opt.storage == LBM_STORE_F16_SHIFT ? 1024.0f : 1.0f;
    d->scale = sc;
    d->inv_scale = 1.0f / sc;
  }
  const size_t lat_bytes = (size_t)Q * d->qs * d->elem;
  auto alloc = [&](void** p, size_t b) -> int {
    cudaError_t ce = cudaMalloc(p, b);
    if (ce != cudaSuccess)
      return set_error(ce == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,
                       "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(ce));
    d->bytes += b;
    return LBM_OK;
  };
  const size_t nb = (size_t)d->N * sizeof(float), pb = (size_t)s.P * sizeof(float);
  if ((rc = alloc(&d->lat[0], lat_bytes)) || (rc = alloc(&d->lat[1], lat_bytes)) ||
      (rc = alloc((void**)&d->den[0], nb)) || (rc = alloc((void**)&d->den[1], nb)) ||
      (rc = alloc((void**)&d->ux, nb)) || (rc = alloc((void**)&d->uy, nb)) ||
      (rc = alloc((void**)&d->uz, nb)) || (rc = alloc((void**)&d->inlet_u, pb)) ||
      (rc = alloc((void**)&d->prho[0], pb)) || (rc = alloc((void**)&d->prho[1], pb)) ||
      (rc = alloc((void**)&d->pu[0], 6 * pb)) || (rc = alloc((void**)&d->pu[1], 6 * pb)) ||
      (rc = alloc((void**)&d->flag, sizeof(int))))
    return fail(rc);
  d->diag_blocks = 4 * prop.multiProcessorCount;
  if ((rc = alloc((void**)&d->partial, (size_t)d->diag_blocks * 8 * sizeof(double))) ||
      (rc = alloc((void**)&d->dout, 8 * sizeof(double))))
    return fail(rc);
  if (cudaStreamCreateWithFlags(&d->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess)
    return fail(set_error(LBM_ERR_CUDA, "stream/event creation failed"));
  d->stream = d->own;
  // channel inlet profile u_x(y,z) = u_max 16 eta(1-eta) zeta(1-zeta)
  if (d->g.casetype == CHANNEL) {
    std::vector<float> prof((size_t)s.P);
    for (int y = 0; y < d->g.ny; ++y)
      for (int z = 0; z < d->g.nz; ++z) {
        const double eta = (double)y / (double)(d->g.ny - 1);
        const double zeta = (double)z / (double)(d->g.nz - 1);
        prof[(size_t)y * d->g.nz + z] = (float)((double)d->in.m_dRefVelx * 16.0 * eta *
                                                (1.0 - eta) * zeta * (1.0 - zeta));
      }
    if (cudaMemcpy(d->inlet_u, prof.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_error(LBM_ERR_CUDA, "inlet profile upload failed"));
  }
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
  InitParams ip;
  ip.kind = d->opt.init_kind;
  ip.seed = d->opt.seed;
  ip.noise_amp = d->opt.noise_amp;
  ip.rho0 = d->in.m_dRefDen;
  ip.ulx = d->in.m_dRefVelx;
  ip.uly = d->in.m_dRefVely;
  ip.ulz = d->in.m_dRefVelz;
  rc = with_storage(d->opt.storage, [&](auto tag) -> int {
    using S = typename decltype(tag)::type;
    return with_model<S>(d, [&](auto coll, auto les) -> int {
      StepArgs<S> a = make_args<S>(d, nullptr, d->lat[1], 0);
      a.den_out = d->den[0];
      a.ux_out = d->ux;
      a.uy_out = d->uy;
      a.uz_out = d->uz;
      const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
      k_init<S, decltype(coll)::value, decltype(les)::value>
          <<<gr, b, 0, d->stream>>>(a, (S*)d->lat[0], ip);
      CK(cudaGetLastError());
      return LBM_OK;
    });
  });
  if (rc) return rc;
  d->cur = 0;
  d->post_direct = true;
  d->step = 0;
  d->initialized = true;
  d->last_steps = 0;
  return LBM_OK;
}

int lbm_run_simulation(lbm_domain* d, int nsteps) {
  if (!d) return set_error(LBM_ERR_INVALID, "NULL domain");
  if (!d->initialized) return set_error(LBM_ERR_STATE, "lbm_run_simulation before lbm_initialize");
  if (nsteps < 0) return set_error(LBM_ERR_INVALID, "nsteps=%d < 0", nsteps);
  if (nsteps == 0) return LBM_OK;
  int rc = ensure_device(d);
  if (rc) return rc;
  CK(cudaEventRecord(d->ev0, d->stream));
  rc = with_storage(d->opt.storage, [&](auto tag) -> int {
    using S = typename decltype(tag)::type;
    return with_model<S>(d, [&](auto coll, auto les) -> int {
      constexpr int C = decltype(coll)::value;
      constexpr bool L = decltype(les)::value;
      // one plain step (no side outputs unless requested)
      auto step_args = [&](long long k, bool den, bool vel, int cur) {
        StepArgs<S> a = make_args<S>(d, d->lat[cur], d->lat[cur ^ 1], k);
        if (den) a.den_out = d->den[k & 1];
        if (vel) {
          a.ux_out = d->ux;
          a.uy_out = d->uy;
          a.uz_out = d->uz;
        }
        return a;
      };
      int plain = nsteps > 2 ? nsteps - 2 : 0;  // the last two steps write rho / u
      // whole graph chunks of kGraphSteps plain steps
      if (plain >= 2 * kGraphSteps) {
        cudaGraphExec_t& g = d->chunk[d->cur];
        if (!g) {
          if (!d->capture) CK(cudaStreamCreateWithFlags(&d->capture, cudaStreamNonBlocking));
          CK(cudaStreamBeginCapture(d->capture, cudaStreamCaptureModeThreadLocal));
          int cur = d->cur;
          long long k = d->step;
          for (int i = 0; i < kGraphSteps; ++i) {
            ++k;
            launch_step<S, C, L>(d, step_args(k, false, false, cur), d->capture);
            cur ^= 1;
          }
          cudaGraph_t graph;
          CK(cudaStreamEndCapture(d->capture, &graph));
          cudaError_t e = cudaGraphInstantiate(&g, graph, 0);
          cudaGraphDestroy(graph);
          if (e != cudaSuccess)
            return set_error(LBM_ERR_CUDA, "graph instantiation failed: %s",
                             cudaGetErrorString(e));
        }
        while (plain >= kGraphSteps) {
          CK(cudaGraphLaunch(g, d->stream));
          d->step += kGraphSteps;  // even: cur and plane parity unchanged
          plain -= kGraphSteps;
        }
      }
      const int rest = plain + (nsteps > 2 ? 2 : nsteps);
      for (int i = 0; i < rest; ++i) {
        const long long k = d->step + 1;
        launch_step<S, C, L>(d, step_args(k, i >= rest - 2, i == rest - 1, d->cur), d->stream);
        d->cur ^= 1;
        d->step = k;
      }
      d->post_direct = false;
      CK(cudaGetLastError());
      return LBM_OK;
    });
  });
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
  CK(cudaMemsetAsync(d->flag, 0, sizeof(int), d->stream));
  k_check_finite<<<4 * 148, 256, 0, d->stream>>>(d->staging, nodes * Q, d->flag);
  int hflag = 0;
  CK(cudaMemcpyAsync(&hflag, d->flag, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  if (hflag) {
    d->initialized = false;
    return set_error(LBM_ERR_NOT_FINITE, "lbm_import_arF: input holds NaN/Inf");
  }
  rc = with_storage(d->opt.storage, [&](auto tag) -> int {
    using S = typename decltype(tag)::type;
    return with_model<S>(d, [&](auto coll, auto les) -> int {
      StepArgs<S> a = make_args<S>(d, nullptr, d->lat[1], 0);
      a.den_out = d->den[0];
      a.ux_out = d->ux;
      a.uy_out = d->uy;
      a.uz_out = d->uz;
      const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
      k_import<S, decltype(coll)::value, decltype(les)::value>
          <<<gr, b, 0, d->stream>>>(a, d->staging, padded, (S*)d->lat[0]);
      CK(cudaGetLastError());
      return LBM_OK;
    });
  });
  if (rc) return rc;
  d->cur = 0;
  d->post_direct = true;
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
  rc = with_storage(d->opt.storage, [&](auto tag) -> int {
    using S = typename decltype(tag)::type;
    StepArgs<S> a = make_args<S>(d, d->lat[d->cur ^ 1], nullptr, d->step);
    const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
    k_export<S><<<gr, b, 0, d->stream>>>(a, d->staging, padded, d->post_direct ? 1 : 0);
    CK(cudaGetLastError());
    return LBM_OK;
  });
  if (rc) return rc;
  CK(cudaMemcpyAsync(arF, d->staging, bytes, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBM_OK;
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
  return LBM_OK;
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
  return LBM_OK;
}

int lbm_device_bytes(const lbm_domain* d, size_t* bytes) {
  if (!d || !bytes) return set_error(LBM_ERR_INVALID, "NULL argument");
  *bytes = d->bytes;
  return LBM_OK;
}

}  // extern "C"
