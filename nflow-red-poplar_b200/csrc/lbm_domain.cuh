// lbm_domain.cuh — internal state of one resident domain and the helpers
// shared by the single-domain C ABI (lbm_api.cu) and the batch engine
// (lbm_batch.cu): validation, sizes, buffer allocation, kernel-argument
// construction and launch selection.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "lbm_internal.h"
#include "lbm_kernels.cuh"
#include "lbm_tma.cuh"

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
  lbm::Geometry g;
  long long N = 0;    // nodes nx*ny*nz
  long long qs = 0;   // population stride in elements
  size_t elem = 4;    // bytes per stored population
  void* lat[2] = {nullptr, nullptr};
  int cur = 0;               // lattice holding f*_k
  bool post_direct = false;  // A/B: lat[cur^1] holds arF_k itself; AA: complete natural layout
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
  int* flag = nullptr;                     // device words: [0] input check, [1] kernel error
  CUtensorMap tmap[2];                     // TMA views of lat[0], lat[1] (16-bit / FP32)
  bool tmap_ok = false;
  int tma_grid = 0;                        // persistent CTAs of the TMA kernel
  double* partial = nullptr;
  double* dout = nullptr;
  int diag_blocks = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int last_steps = 0;
  float scale = 1.f, inv_scale = 1.f;
  size_t bytes = 0;
  bool pooled = false;  // buffers belong to a batch pool (lbm_batch), not freed here
  // CUDA graphs of kGraphSteps plain steps, one per starting lattice
  cudaGraphExec_t chunk[2] = {nullptr, nullptr};
  cudaStream_t capture = nullptr;
  // snapshot of the macroscopic state for the output writers
  // (lbm_snapshot / lbm_save_snapshot)
  float* snap_dev = nullptr;       // [4][N] rho, ux, uy, uz on the device
  float* snap_host = nullptr;      // [4][N] pinned host copy
  int* snap_type = nullptr;        // [N] node types (host)
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_taken = nullptr;   // device copy done (handle stream)
  cudaEvent_t snap_landed = nullptr;  // host copy done (side stream)
  bool snap_valid = false;
  unsigned char* solid = nullptr;  // [N] solid mask on the device (lbm_set_solid_mask)
  // AA streaming: cur is the layout of lat[0] (0 natural, 1 swapped);
  // aa_first: the next step is the first after the initial state
  bool aa_first = false;
  // channel on quad rows: the next AA step's inlet / outlet values
  // [2][5][ny*nz] (k_aa_xface_rules)
  float* xrule = nullptr;
};

// steps per captured graph chunk (even, so that a chunk returns the lattices
// and the boundary planes to the parity it started from)
constexpr int kGraphSteps = 32;

namespace lbm {

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

inline size_t storage_bytes(int storage) {
  switch (storage) {
    case LBM_STORE_F64: return 8;
    case LBM_STORE_F16_SHIFT:
    case LBM_STORE_BF16_SHIFT: return 2;
    default: return 4;
  }
}

inline long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// A 16-bit AA domain can be stored in quad rows (kRowsQuad): the word AA
// step needs rows of whole words without padding nodes (px == nx, a
// multiple of 8) and at least four words per row quarter.
inline bool aa_word_rows_fit(const Inputval* in, const lbm_options* opt) {
  return opt && (opt->storage == LBM_STORE_F16_SHIFT || opt->storage == LBM_STORE_BF16_SHIFT) &&
         opt->stream_mode == LBM_STREAM_AA && in->nx % 8 == 0 && in->nx >= 16;
}

inline int validate(const Inputval* in, const lbm_options* opt) {
  if (!in) return set_error(LBM_ERR_INVALID, "NULL Inputval");
  if (in->nx < 3 || in->ny < 3 || in->nz < 3)
    return set_error(LBM_ERR_INVALID, "domain %dx%dx%d too small (each extent must be >= 3)",
                     in->nx, in->ny, in->nz);
  if (in->ny > 65535 || in->nz > 65535)
    return set_error(LBM_ERR_INVALID, "ny and nz must be <= 65535");
  if (round_up(in->nx, 8) * (long long)in->ny * in->nz >= (1LL << 31) - 1024)
    return set_error(LBM_ERR_INVALID, "domain too large (px*ny*nz must be < 2^31)");
  if (in->casetype != CAVITY && in->casetype != CHANNEL && in->casetype != POISEUILLE)
    return set_error(LBM_ERR_INVALID,
                     "casetype %d not supported (POISEUILLE=0, CAVITY=1, CHANNEL=2)",
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
    if (opt->stream_mode != LBM_STREAM_AB && opt->stream_mode != LBM_STREAM_AA)
      return set_error(LBM_ERR_INVALID, "stream_mode %d not supported", opt->stream_mode);
    if (opt->stream_mode == LBM_STREAM_AA && in->casetype != CAVITY && in->casetype != CHANNEL)
      return set_error(LBM_ERR_INVALID,
                       "AA streaming is implemented for the cavity (casetype %d) and the channel "
                       "(casetype %d) only",
                       CAVITY, CHANNEL);
    if (opt->kernel < LBM_KERNEL_AUTO || opt->kernel > LBM_KERNEL_QUAD)
      return set_error(LBM_ERR_INVALID, "unknown kernel %d", opt->kernel);
    if (opt->kernel == LBM_KERNEL_QUAD && !aa_word_rows_fit(in, opt))
      return set_error(LBM_ERR_INVALID,
                       "the quad kernel is the 16-bit AA form: FP16/BF16 shifted storage with "
                       "LBM_STREAM_AA and nx a multiple of 8, at least 16 (nx = %d)",
                       in->nx);
    if (opt->kernel == LBM_KERNEL_PAIRED &&
        ((opt->storage != LBM_STORE_F16_SHIFT && opt->storage != LBM_STORE_BF16_SHIFT) ||
         opt->stream_mode != LBM_STREAM_AB))
      return set_error(LBM_ERR_INVALID,
                       "the paired kernel is the 16-bit pull (A/B) form: FP16/BF16 shifted "
                       "storage with LBM_STREAM_AB");
    if (opt->wait_test < 0 || (opt->wait_test > 0 && opt->kernel != LBM_KERNEL_TMA))
      return set_error(LBM_ERR_INVALID, "wait_test applies to the TMA kernel only");
    if (opt->rounding != LBM_ROUND_NEAREST && opt->rounding != LBM_ROUND_STOCHASTIC)
      return set_error(LBM_ERR_INVALID, "unknown rounding %d", opt->rounding);
    if (opt->rounding == LBM_ROUND_STOCHASTIC &&
        ((opt->storage != LBM_STORE_F16_SHIFT && opt->storage != LBM_STORE_BF16_SHIFT) ||
         (opt->stream_mode == LBM_STREAM_AB && opt->kernel != LBM_KERNEL_AUTO &&
          opt->kernel != LBM_KERNEL_PAIRED && opt->kernel != LBM_KERNEL_SCALAR) ||
         (opt->stream_mode == LBM_STREAM_AA &&
          ((opt->kernel != LBM_KERNEL_AUTO && opt->kernel != LBM_KERNEL_QUAD) ||
           !aa_word_rows_fit(in, opt)))))
      return set_error(LBM_ERR_INVALID,
                       "stochastic rounding needs FP16/BF16 shifted storage, with LBM_STREAM_AB "
                       "and kernel AUTO, PAIRED or SCALAR, or with LBM_STREAM_AA on quad rows "
                       "(kernel AUTO or QUAD, nx a multiple of 8, at least 16)");
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

inline Sizes sizes_of(const Inputval* in) {
  Sizes s;
  s.px = (int)round_up(in->nx, 8);
  s.N = (long long)in->nx * in->ny * in->nz;
  s.qs = round_up((long long)s.px * in->nz * in->ny, 128) + LBM_PLANE_PAD;
  s.P = (long long)in->ny * in->nz;
  return s;
}

inline size_t footprint(const Inputval* in, const lbm_options* opt) {
  const Sizes s = sizes_of(in);
  const size_t e = storage_bytes(opt ? opt->storage : LBM_STORE_F32);
  const int lattices = opt && opt->stream_mode == LBM_STREAM_AA ? 1 : 2;
  size_t b = lattices * (size_t)Q * s.qs * e;  // lattices
  b += 5 * (size_t)s.N * sizeof(float);  // den[2], ux, uy, uz
  b += 15 * (size_t)s.P * sizeof(float); // inlet profile + planes
  return b;
}

inline dim3 block_of(int nx) {
  int bx = (int)round_up(nx < 128 ? nx : 128, 32);
  return dim3(bx, 1, 1);
}
inline dim3 grid_of(const Geometry& g, dim3 b) {
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
    // paired / quad rows: a node one step away in x is two / four elements away
    a.off[q] = row_step(d->g.rows) * cx(q) + d->g.px * (cz(q) + d->g.nz * cy(q));
    a.srcq[q] = src ? (const S*)src + q * d->qs : nullptr;
    a.srcd[q] = src ? (const S*)src + (q * d->qs - a.off[q]) : nullptr;
    a.dstq[q] = dst ? (S*)dst + q * d->qs : nullptr;
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
  a.mp.e2c = kDev<S> ? R(3) - a.mp.weps : R(0);
  // step counter of the stochastic rounding: step k reads kctr[(k-1) & 1]
  // and writes kctr[k & 1] (d->flag[2..3])
  a.kctr = (unsigned*)(d->flag + 2);
  a.kpar = (int)((k - 1) & 1);
  a.sr = d->opt.rounding == LBM_ROUND_STOCHASTIC;
  a.sr_seed = (unsigned)(d->opt.seed * 0x9E3779B97F4A7C15ull >> 32);
  a.scale = d->scale;
  a.inv_scale = d->inv_scale;
  a.inlet_u = d->inlet_u;
  a.init_kind = d->opt.init_kind;
  a.noise_amp = d->opt.noise_amp;
  a.seed = d->opt.seed;
  a.prho_in = d->prho[(k + 1) & 1];  // (k-1)&1
  a.prho_out = d->prho[k & 1];
  a.pu_in = d->pu[(k + 1) & 1];
  a.pu_out = d->pu[k & 1];
  return a;
}

// Arguments of AA step k (one lattice, lat[0]) with the slot tables of its
// kind (k_aa_step):
//   local step:      srcd[q] = plane q,                 dstq[q] = plane opp q
//   neighbour step:  srcd[q] = plane opp q, minus off_q, dstq[q] = plane q, plus off_q
// den: the step writes rho of its input arF_{k-1}.
template <class S>
StepArgs<S> aa_args(const lbm_domain* d, long long k, bool den, int neighbor) {
  StepArgs<S> a = make_args<S>(d, d->lat[0], d->lat[0], k);
  S* lat = (S*)d->lat[0];
  for (int q = 0; q < Q; ++q) {
    if (!neighbor) {
      a.srcd[q] = lat + q * d->qs;
      a.dstq[q] = lat + opp(q) * d->qs;
    } else {
      a.srcd[q] = lat + (opp(q) * d->qs - a.off[q]);
      a.dstq[q] = lat + (q * d->qs + a.off[q]);
    }
  }
  if (den) a.den_out = d->den[(k - 1) & 1];
  a.aa_step = 1 + neighbor;
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
  if constexpr (kDev<S>) {
    if (d->g.rows == kRowsPaired) {
      // one thread per word, CTAs no wider than a row's words (px / 2)
      const dim3 bp = block_of(d->g.px / 2);
      const dim3 gr((d->g.px / 2 + bp.x - 1) / bp.x, d->g.nz, d->g.ny);
      if (paired_kernel_applies(d->g) && a.sr)
        k_step_paired<S, COLL, LES, true><<<gr, bp, 0, st>>>(a);
      else if (paired_kernel_applies(d->g))
        k_step_paired<S, COLL, LES, false><<<gr, bp, 0, st>>>(a);
      else if (a.sr)
        k_step_rows<S, COLL, LES, true><<<grid_of(d->g, block_of(d->g.nx)), block_of(d->g.nx),
                                          0, st>>>(a);
      else
        k_step_rows<S, COLL, LES, false><<<grid_of(d->g, block_of(d->g.nx)),
                                           block_of(d->g.nx), 0, st>>>(a);
      return;
    }
  }
  if constexpr (!std::is_same<S, double>::value) {
    if (has_struct(d->g)) {
      // struct geometry: the per-node kernel (its pull checks every donor)
    } else if (d->opt.kernel == LBM_KERNEL_PACKED) {
      const int pairs = (d->g.nx + 1) / 2;
      const dim3 b(64, 1, 1), gr((pairs + 63) / 64, d->g.nz, d->g.ny);
      k_step2<S, COLL, LES><<<gr, b, 0, st>>>(a);
      return;
    }
    else if (d->opt.kernel == LBM_KERNEL_TMA && d->tmap_ok) {
      using Cfg = TmaCfg<S>;
      const int which = (a.src == (const S*)d->lat[0]) ? 0 : 1;
      // the wait test withholds one tile and bounds every wait to ~1 ms
      const int stall = d->opt.wait_test > 0 ? d->opt.wait_test - 1 : -1;
      k_step_tma<S, COLL, LES><<<d->tma_grid, Cfg::THREADS, Cfg::SMEM, st>>>(
          a, d->tmap[which], d->flag + 1, stall, stall >= 0 ? 1000 : kWaitIters);
      return;
    }
  }
  const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
  if constexpr (kDev<S>) {
    if (a.sr) {
      k_step<S, COLL, LES, true><<<gr, b, 0, st>>>(a);
      return;
    }
  }
  k_step<S, COLL, LES, false><<<gr, b, 0, st>>>(a);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
typedef CUresult (*TensorMapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                      const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                      const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion,
                                      CUtensorMapFloatOOBfill);
inline TensorMapEncodeFn tensor_map_encoder() {
  static TensorMapEncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (TensorMapEncodeFn)p;
  }
  return fn;
}

// 4-D views (x, z, y, q) of both lattices with the TMA box of TmaCfg<S>,
// and the persistent grid of the TMA kernel.  Leaves tmap_ok false (the
// kernel option then falls back to the scalar kernel) for FP64 storage.
template <class S>
int domain_tensor_maps(lbm_domain* d, int sm_count) {
  if (d->opt.stream_mode == LBM_STREAM_AA || d->g.rows != kRowsPlain) {
    // the TMA kernel is a pull (A/B) kernel over plain rows
    d->tmap_ok = false;
    return LBM_OK;
  }
  if constexpr (std::is_same<S, double>::value) {
    d->tmap_ok = false;
    return LBM_OK;
  } else {
    using Cfg = TmaCfg<S>;
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc) return set_error(LBM_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    const CUtensorMapDataType dt = std::is_same<S, float>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : std::is_same<S, __half>::value
                                       ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                       : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const cuuint64_t es = sizeof(S);
    const cuuint64_t dims[4] = {(cuuint64_t)d->g.nx, (cuuint64_t)d->g.nz, (cuuint64_t)d->g.ny,
                                (cuuint64_t)Q};
    const cuuint64_t strides[3] = {(cuuint64_t)d->g.px * es,
                                   (cuuint64_t)d->g.px * d->g.nz * es, (cuuint64_t)d->qs * es};
    const cuuint32_t box[4] = {(cuuint32_t)Cfg::TXB, (cuuint32_t)Cfg::TZ, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int i = 0; i < 2; ++i) {
      CUresult r = enc(&d->tmap[i], dt, 4, d->lat[i], dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return set_error(LBM_ERR_CUDA, "tensor map encoding failed (%d)", (int)r);
    }
    int rc = with_model<S>(d, [&](auto coll, auto les) -> int {
      auto kern = k_step_tma<S, decltype(coll)::value, decltype(les)::value>;
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::THREADS, Cfg::SMEM));
      if (per_sm < 1) return set_error(LBM_ERR_CUDA, "TMA kernel does not fit an SM");
      const long long ntiles = (long long)((d->g.nx + Cfg::TX - 1) / Cfg::TX) *
                               ((d->g.nz + Cfg::TZ - 1) / Cfg::TZ) * d->g.ny;
      if (ntiles >= (1LL << 31)) return set_error(LBM_ERR_INVALID, "too many TMA tiles");
      d->tma_grid = (int)std::min<long long>(ntiles, (long long)per_sm * sm_count);
      return LBM_OK;
    });
    if (rc) return rc;
    d->tmap_ok = true;
    return LBM_OK;
  }
}

// LBM_ERR_TIMEOUT if a kernel of the domain reported a failed bounded wait
inline int check_kernel_error(lbm_domain* d) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, d->flag + 1, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  if (e) return set_error(LBM_ERR_TIMEOUT, "a step kernel gave up a bounded wait (code %d)", e);
  return LBM_OK;
}

inline int ensure_device(const lbm_domain* d) {
  CK(cudaSetDevice(d->opt.device));
  return LBM_OK;
}

inline int ensure_staging(lbm_domain* d, size_t bytes) {
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

inline void free_all(lbm_domain* d) {
  if (!d->pooled)
  for (int i = 0; i < 2; ++i) {
    if (d->lat[i]) cudaFree(d->lat[i]);
    if (d->den[i]) cudaFree(d->den[i]);
    if (d->prho[i]) cudaFree(d->prho[i]);
    if (d->pu[i]) cudaFree(d->pu[i]);
  }
  if (!d->pooled) {
    if (d->ux) cudaFree(d->ux);
    if (d->uy) cudaFree(d->uy);
    if (d->uz) cudaFree(d->uz);
    if (d->inlet_u) cudaFree(d->inlet_u);
  }
  if (d->solid) cudaFree(d->solid);
  if (d->snap_stream) cudaStreamSynchronize(d->snap_stream);
  if (d->snap_dev) cudaFree(d->snap_dev);
  if (d->snap_host) cudaFreeHost(d->snap_host);
  delete[] d->snap_type;
  if (d->snap_taken) cudaEventDestroy(d->snap_taken);
  if (d->snap_landed) cudaEventDestroy(d->snap_landed);
  if (d->snap_stream) cudaStreamDestroy(d->snap_stream);
  if (d->staging) cudaFree(d->staging);
  if (d->flag && !d->pooled) cudaFree(d->flag);  // batch members: from the pool
  if (d->partial) cudaFree(d->partial);
  if (d->dout) cudaFree(d->dout);
  if (d->xrule) cudaFree(d->xrule);
  for (int i = 0; i < 2; ++i)
    if (d->chunk[i]) cudaGraphExecDestroy(d->chunk[i]);
  if (d->capture) cudaStreamDestroy(d->capture);
  if (d->ev0) cudaEventDestroy(d->ev0);
  if (d->ev1) cudaEventDestroy(d->ev1);
  if (d->own) cudaStreamDestroy(d->own);
}


// Fill the geometry, sizes and storage scale of d from the case.
inline void domain_prepare(lbm_domain* d, const Inputval* pinput, const lbm_options* opt) {
  d->in = *pinput;
  if (opt)
    d->opt = *opt;
  else
    lbm_default_options(&d->opt);
  const Sizes s = sizes_of(pinput);
  d->g.nx = pinput->nx;
  d->g.ny = pinput->ny;
  d->g.nz = pinput->nz;
  d->g.px = s.px;
  d->g.casetype = pinput->casetype;
  d->g.solid = nullptr;
  // 16-bit pull (A/B) domains use paired rows and 16-bit AA domains quad
  // rows where they fit, unless another kernel is asked for
  const bool b16 =
      d->opt.storage == LBM_STORE_F16_SHIFT || d->opt.storage == LBM_STORE_BF16_SHIFT;
  d->g.rows = kRowsPlain;
  if (b16 && d->opt.stream_mode == LBM_STREAM_AB &&
      (d->opt.kernel == LBM_KERNEL_AUTO || d->opt.kernel == LBM_KERNEL_PAIRED))
    d->g.rows = kRowsPaired;
  if (aa_word_rows_fit(pinput, &d->opt) &&
      (d->opt.kernel == LBM_KERNEL_AUTO || d->opt.kernel == LBM_KERNEL_QUAD))
    d->g.rows = kRowsQuad;
  d->N = s.N;
  d->qs = s.qs;
  d->elem = storage_bytes(d->opt.storage);
  if (d->opt.storage == LBM_STORE_F16_SHIFT || d->opt.storage == LBM_STORE_BF16_SHIFT) {
    float sc = d->opt.store_scale;
    if (sc == 0.0f) sc = d->opt.storage == LBM_STORE_F16_SHIFT ? 1024.0f : 1.0f;
    d->scale = sc;
    d->inv_scale = 1.0f / sc;
  }
}

// Allocate the state buffers of d (lattices, macroscopic fields, boundary
// planes) through alloc(void** p, size_t bytes) -> status.
template <class Alloc>
int domain_alloc_state(lbm_domain* d, Alloc&& alloc) {
  const size_t lat_bytes = (size_t)Q * d->qs * d->elem;
  const size_t nb = (size_t)d->N * sizeof(float);
  const size_t pb = (size_t)d->g.ny * d->g.nz * sizeof(float);
  int rc;
  const bool aa = d->opt.stream_mode == LBM_STREAM_AA;  // one lattice, in place
  if ((rc = alloc(&d->lat[0], lat_bytes)) || (!aa && (rc = alloc(&d->lat[1], lat_bytes))) ||
      (rc = alloc((void**)&d->den[0], nb)) || (rc = alloc((void**)&d->den[1], nb)) ||
      (rc = alloc((void**)&d->ux, nb)) || (rc = alloc((void**)&d->uy, nb)) ||
      (rc = alloc((void**)&d->uz, nb)) || (rc = alloc((void**)&d->inlet_u, pb)) ||
      (rc = alloc((void**)&d->prho[0], pb)) || (rc = alloc((void**)&d->prho[1], pb)) ||
      (rc = alloc((void**)&d->pu[0], 6 * pb)) || (rc = alloc((void**)&d->pu[1], 6 * pb)))
    return rc;
  return LBM_OK;
}

// Bytes domain_alloc_state takes (each buffer rounded to 256 bytes).
inline size_t domain_state_bytes(const Inputval* in, const lbm_options* opt) {
  const Sizes s = sizes_of(in);
  auto r = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t e = storage_bytes(opt ? opt->storage : LBM_STORE_F32);
  const size_t nb = (size_t)s.N * sizeof(float), pb = (size_t)s.P * sizeof(float);
  const int lattices = opt && opt->stream_mode == LBM_STREAM_AA ? 1 : 2;
  return lattices * r((size_t)Q * s.qs * e) + 5 * r(nb) + 3 * r(pb) + 2 * r(6 * pb);
}

// Upload the channel inlet profile u_x(y,z) = u_max 16 eta(1-eta) zeta(1-zeta).
// u_x(y, z) of the channel inlet, on the device so that admission needs no
// host synchronisation; every operation is a correctly rounded double
// operation in the order of the host formula, so the values equal the host
// (and oracle) profile bit for bit
static __global__ void k_inlet_profile(float* __restrict__ prof, int ny, int nz, double umax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ny * nz) return;
  const int y = i / nz, z = i % nz;
  const double eta = __ddiv_rn((double)y, (double)(ny - 1));
  const double zeta = __ddiv_rn((double)z, (double)(nz - 1));
  double v = __dmul_rn(umax, 16.0);
  v = __dmul_rn(v, eta);
  v = __dmul_rn(v, __dsub_rn(1.0, eta));
  v = __dmul_rn(v, zeta);
  v = __dmul_rn(v, __dsub_rn(1.0, zeta));
  prof[i] = (float)v;
}

// Fill the channel inlet profile u_x(y,z) = u_max 16 eta(1-eta) zeta(1-zeta)
// (asynchronous on st).
inline int domain_upload_profile(lbm_domain* d, cudaStream_t st) {
  if (d->g.casetype != CHANNEL) return LBM_OK;
  const int n = d->g.ny * d->g.nz;
  k_inlet_profile<<<(n + 255) / 256, 256, 0, st>>>(d->inlet_u, d->g.ny, d->g.nz,
                                                   (double)d->in.m_dRefVelx);
  CK(cudaGetLastError());
  return LBM_OK;
}

// The diagnostics buffers of a domain (allocated on first use for batch
// members, whose admission allocates nothing outside the pool).
inline int ensure_diag_buffers(lbm_domain* d) {
  if (d->partial && d->dout) return LBM_OK;
  if (!d->partial && cudaMalloc((void**)&d->partial, (size_t)d->diag_blocks * 8 * sizeof(double)) !=
                         cudaSuccess) {
    d->partial = nullptr;
    return set_error(LBM_ERR_OOM, "diagnostics buffer");
  }
  if (!d->dout && cudaMalloc((void**)&d->dout, 8 * sizeof(double)) != cudaSuccess) {
    d->dout = nullptr;
    return set_error(LBM_ERR_OOM, "diagnostics buffer");
  }
  return LBM_OK;
}

// The storage-typed work of a single domain, one table per storage format,
// each built in its own translation unit (lbm_ops_impl.cuh).
struct StorageOps {
  int (*tensor_maps)(lbm_domain*, int sm_count);
  int (*launch_init)(lbm_domain*, cudaStream_t);
  int (*run_pull)(lbm_domain*, int nsteps);
  int (*run_aa)(lbm_domain*, int nsteps);
  int (*import_staging)(lbm_domain*, int padded);
  int (*export_staging)(lbm_domain*, int padded);
  int (*aa_macro)(lbm_domain*);  // rho, u of the AA state after step d->step
};
extern const StorageOps kOps_f32, kOps_f16, kOps_bf16, kOps_f64;
inline const StorageOps& storage_ops(int storage) {
  switch (storage) {
    case LBM_STORE_F16_SHIFT: return kOps_f16;
    case LBM_STORE_BF16_SHIFT: return kOps_bf16;
    case LBM_STORE_F64: return kOps_f64;
    default: return kOps_f32;
  }
}

// InitParams of the domain's initial condition.
inline InitParams init_params(const lbm_domain* d) {
  InitParams ip;
  ip.kind = d->opt.init_kind;
  ip.seed = d->opt.seed;
  ip.noise_amp = d->opt.noise_amp;
  ip.rho0 = d->in.m_dRefDen;
  ip.ulx = d->in.m_dRefVelx;
  ip.uly = d->in.m_dRefVely;
  ip.ulz = d->in.m_dRefVelz;
  return ip;
}

// Launch the initial-state kernel of d on st (pull form: post lattice
// lat[1], first collision into lat[0]; AA: arF_0 in lat[0]) and reset the
// step state.
inline int domain_launch_init(lbm_domain* d, cudaStream_t st) {
  const size_t nb = (size_t)d->N * sizeof(float);
  CK(cudaMemsetAsync(d->den[0], 0, nb, st));
  CK(cudaMemsetAsync(d->den[1], 0, nb, st));
  CK(cudaMemsetAsync(d->flag + 2, 0, 2 * sizeof(int), st));  // step counter
  int rc = storage_ops(d->opt.storage).launch_init(d, st);
  if (rc) return rc;
  d->cur = 0;
  d->post_direct = true;
  d->aa_first = d->opt.stream_mode == LBM_STREAM_AA;
  d->step = 0;
  d->initialized = true;
  d->last_steps = 0;
  return LBM_OK;
}

}  // namespace lbm
