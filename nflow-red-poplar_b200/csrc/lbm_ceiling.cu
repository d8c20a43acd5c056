// lbm_ceiling.cu — memory-pattern ceilings of the fused step.
//
// Each pattern performs exactly the global loads and stores of one lattice
// update of a step form (19 population loads and 19 stores per node, same
// addresses, same access widths, same thread mapping), with only a token
// amount of arithmetic (a sum of the loaded values folded into every store,
// so that nothing can be dropped by the compiler).  The rate a pattern
// reaches is therefore the ceiling of any step kernel with that memory
// pattern: a kernel with the full collision cannot be faster, and the gap
// between the two is the cost of its instructions and registers.
//
//   COPY            19 planes read and 19 written at the node itself,
//                   16-byte vectors per lane (streaming bound of 38 planes)
//   PULL            pull streaming: 19 loads from the donors x - c_q, one
//                   node per thread, one element per access (the k_step form)
//   PULL_PAIRED     16-bit only: rows stored as 32-bit words holding the
//                   nodes (w, w + px/2), two nodes per thread, every access a
//                   32-bit word; an x shift of the donor is a word shift
//   AA_LOCAL        AA local step: loads at the node, stores at the node into
//                   the opposite plane, one element per access, in place
//   AA_NEIGHBOR     AA neighbour step: loads of plane opp q at x - c_q,
//                   stores of plane q at x + c_q, one element per access
//   AA_LOCAL_V8     AA local step with 8-byte vectors per lane
//   AA_LOCAL_V16    AA local step with 16-byte vectors per lane
//   AA_PAIRED_LOCAL, AA_PAIRED_NEIGHBOR
//                   16-bit only: the AA steps over paired rows (32-bit words
//                   of the nodes (w, w + px/2)), two nodes per thread
//   PULL_QUAD, AA_QUAD_LOCAL, AA_QUAD_NEIGHBOR
//                   16-bit only: rows stored as 8-byte words holding the
//                   nodes (w, w + Q, w + 2Q, w + 3Q), Q = px/4, four nodes
//                   per thread; an x shift is a whole-word shift, so every
//                   access of both AA steps and of pull is an aligned vector
//
// Boxes of n^3 nodes, n a multiple of 32; shifted patterns visit the
// interior nodes only (every donor and destination then lies inside).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "../../include/lbm_b200.h"
#include "lbm_d3q19.cuh"
#include "lbm_internal.h"

namespace {

using lbm::cx;
using lbm::cy;
using lbm::cz;
using lbm::opp;
using lbm::Q;
using lbm::static_for;

// token arithmetic on one element
__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
template <class T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

struct Box {
  int n;
  long long qs;  // plane stride (elements)
};

__host__ __device__ __forceinline__ int off_of(int q, int n) {
  return cx(q) + n * (cz(q) + n * cy(q));
}

// pull: one node per thread, interior nodes
template <class T>
__global__ void __launch_bounds__(128) k_pull(const T* __restrict__ src, T* __restrict__ dst, Box b) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (x < 1 || x > b.n - 2 || z < 1 || z > b.n - 2 || y < 1 || y > b.n - 2) return;
  const int cell = x + b.n * (z + b.n * y);
  float v[Q], acc = 0.f;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    v[q] = to_f(src[q * b.qs + cell - off_of(q, b.n)]);
    acc += v[q];
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    dst[q * b.qs + cell] = from_f<T>(fmaf(v[q], 0.5f, acc * 1e-7f));
  });
}

// paired 16-bit rows: word w of a row holds nodes (w, w + n/2); interior
// words 1 .. n/2 - 2 of interior rows, so every donor word w - c_x exists
__global__ void __launch_bounds__(128)
    k_pull_paired(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, Box b) {
  const int H = b.n / 2;
  const int w = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (w < 1 || w > H - 2 || z < 1 || z > b.n - 2 || y < 1 || y > b.n - 2) return;
  const long long qw = b.qs / 2;  // plane stride in words
  const int cell = w + H * (z + b.n * y);
  float2 v[Q];
  float a0 = 0.f, a1 = 0.f;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int off = cx(q) + H * (cz(q) + b.n * cy(q));
    const uint32_t word = src[q * qw + cell - off];
    __half2 h;
    *reinterpret_cast<uint32_t*>(&h) = word;
    v[q] = __half22float2(h);
    a0 += v[q].x;
    a1 += v[q].y;
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const __half2 h = __floats2half2_rn(fmaf(v[q].x, 0.5f, a0 * 1e-7f), fmaf(v[q].y, 0.5f, a1 * 1e-7f));
    dst[q * qw + cell] = *reinterpret_cast<const uint32_t*>(&h);
  });
}

// AA local step, one element per access, all nodes, in place
template <class T>
__global__ void __launch_bounds__(128) k_aa_local(T* __restrict__ lat, Box b) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (x >= b.n) return;
  const long long cell = x + (long long)b.n * (z + (long long)b.n * y);
  float v[Q], acc = 0.f;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    v[q] = to_f(lat[q * b.qs + cell]);
    acc += v[q];
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    lat[opp(q) * b.qs + cell] = from_f<T>(fmaf(v[q], 0.5f, acc * 1e-7f));
  });
}

// AA neighbour step, interior nodes, in place: each thread reads and writes
// the same 19 slots (plane opp q at x - c_q, plane q at x + c_q... which is
// the slot (x - c_{opp q}) of plane opp(opp q)), so the update is race-free
template <class T>
__global__ void __launch_bounds__(128) k_aa_neighbor(T* __restrict__ lat, Box b) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (x < 1 || x > b.n - 2 || z < 1 || z > b.n - 2 || y < 1 || y > b.n - 2) return;
  const int cell = x + b.n * (z + b.n * y);
  float v[Q], acc = 0.f;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    v[q] = to_f(lat[opp(q) * b.qs + cell - off_of(q, b.n)]);
    acc += v[q];
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    lat[q * b.qs + cell + off_of(q, b.n)] = from_f<T>(fmaf(v[q], 0.5f, acc * 1e-7f));
  });
}

// AA local step with VB-byte vectors per lane (VB / sizeof(T) nodes per
// thread), all nodes, in place
template <class T, int VB>
__global__ void __launch_bounds__(128) k_aa_local_vec(T* __restrict__ lat, Box b) {
  constexpr int E = VB / (int)sizeof(T);  // elements per vector
  using Vec = typename std::conditional<VB == 16, uint4, uint2>::type;
  const int t = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (t * E >= b.n) return;
  const long long cell = (long long)t * E + (long long)b.n * (z + (long long)b.n * y);
  Vec v[Q];
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    v[q] = *reinterpret_cast<const Vec*>(lat + q * b.qs + cell);
    const T* el = reinterpret_cast<const T*>(&v[q]);
#pragma unroll
    for (int e = 0; e < E; ++e) acc[e] += to_f(el[e]);
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    Vec o;
    T* oe = reinterpret_cast<T*>(&o);
    const T* el = reinterpret_cast<const T*>(&v[q]);
#pragma unroll
    for (int e = 0; e < E; ++e) oe[e] = from_f<T>(fmaf(to_f(el[e]), 0.5f, acc[e] * 1e-7f));
    *reinterpret_cast<Vec*>(lat + opp(q) * b.qs + cell) = o;
  });
}

// 16-bit rows stored as words of NPW nodes (word w of a row holds the nodes
// w + k n/NPW, k < NPW): MODE 0 pull, 1 AA local, 2 AA neighbour; shifted
// modes visit the interior words 1 .. n/NPW - 2 of interior rows, so every
// shifted word lies inside the row
template <int NPW, int MODE>
__global__ void __launch_bounds__(128) k_words(const void* __restrict__ src_, void* __restrict__ dst_,
                                               Box b) {
  using W = typename std::conditional<NPW == 2, uint32_t,
                                      typename std::conditional<NPW == 4, uint2, uint4>::type>::type;
  constexpr int P = NPW / 2;  // 32-bit pieces per word
  const int NW = b.n / NPW;   // words per row
  const int w = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (MODE == 1) {
    if (w >= NW) return;
  } else if (w < 1 || w > NW - 2 || z < 1 || z > b.n - 2 || y < 1 || y > b.n - 2) {
    return;
  }
  const W* src = reinterpret_cast<const W*>(src_);
  W* dst = reinterpret_cast<W*>(MODE == 0 ? dst_ : const_cast<void*>(src_));
  const long long qw = b.qs / NPW;  // plane stride in words
  const long long cell = w + (long long)NW * (z + (long long)b.n * y);
  W v[Q];
  float2 acc[P];
#pragma unroll
  for (int p = 0; p < P; ++p) acc[p] = make_float2(0.f, 0.f);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int off = cx(q) + NW * (cz(q) + b.n * cy(q));
    if (MODE == 0) v[q] = src[q * qw + cell - off];
    if (MODE == 1) v[q] = src[q * qw + cell];
    if (MODE == 2) v[q] = src[opp(q) * qw + cell - off];
    const __half2* h = reinterpret_cast<const __half2*>(&v[q]);
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float2 f = __half22float2(h[p]);
      acc[p].x += f.x;
      acc[p].y += f.y;
    }
  });
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int off = cx(q) + NW * (cz(q) + b.n * cy(q));
    W o;
    __half2* oh = reinterpret_cast<__half2*>(&o);
    const __half2* h = reinterpret_cast<const __half2*>(&v[q]);
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float2 f = __half22float2(h[p]);
      oh[p] = __floats2half2_rn(fmaf(f.x, 0.5f, acc[p].x * 1e-7f), fmaf(f.y, 0.5f, acc[p].y * 1e-7f));
    }
    if (MODE == 0) dst[q * qw + cell] = o;
    if (MODE == 1) dst[opp(q) * qw + cell] = o;
    if (MODE == 2) dst[q * qw + cell + off] = o;
  });
}

// plain copy of 19 planes with 16-byte vectors, each plane streamed
// independently (the streaming bound of 19 + 19 planes)
template <class T>
__global__ void __launch_bounds__(128)
    k_copy(const T* __restrict__ src, T* __restrict__ dst, Box b) {
  constexpr int E = 16 / (int)sizeof(T);
  const int t = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, y = blockIdx.z;
  if (t * E >= b.n) return;
  const long long cell = (long long)t * E + (long long)b.n * (z + (long long)b.n * y);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    uint4 v = *reinterpret_cast<const uint4*>(src + q * b.qs + cell);
    T* e0 = reinterpret_cast<T*>(&v);
    e0[0] = from_f<T>(fmaf(to_f(e0[0]), 0.5f, 1e-7f));
    *reinterpret_cast<uint4*>(dst + q * b.qs + cell) = v;
  });
}

template <class T>
int launch(int pattern, void* a, void* b2, Box b, cudaStream_t st) {
  const dim3 blk(128), g1((b.n + 127) / 128, b.n, b.n);
  switch (pattern) {
    case LBM_PATTERN_COPY: {
      const int per = 16 / (int)sizeof(T);
      k_copy<T><<<dim3((b.n / per + 127) / 128, b.n, b.n), blk, 0, st>>>((const T*)a, (T*)b2, b);
      break;
    }
    case LBM_PATTERN_PULL: k_pull<T><<<g1, blk, 0, st>>>((const T*)a, (T*)b2, b); break;
    case LBM_PATTERN_PULL_PAIRED:
      k_pull_paired<<<dim3((b.n / 2 + 127) / 128, b.n, b.n), blk, 0, st>>>(
          (const uint32_t*)a, (uint32_t*)b2, b);
      break;
    case LBM_PATTERN_AA_LOCAL: k_aa_local<T><<<g1, blk, 0, st>>>((T*)a, b); break;
    case LBM_PATTERN_AA_NEIGHBOR: k_aa_neighbor<T><<<g1, blk, 0, st>>>((T*)a, b); break;
    case LBM_PATTERN_AA_LOCAL_V8: {
      const int per = 8 / (int)sizeof(T);
      k_aa_local_vec<T, 8><<<dim3((b.n / per + 127) / 128, b.n, b.n), blk, 0, st>>>((T*)a, b);
      break;
    }
    case LBM_PATTERN_AA_LOCAL_V16: {
      const int per = 16 / (int)sizeof(T);
      k_aa_local_vec<T, 16><<<dim3((b.n / per + 127) / 128, b.n, b.n), blk, 0, st>>>((T*)a, b);
      break;
    }
    case LBM_PATTERN_AA_PAIRED_LOCAL:
    case LBM_PATTERN_AA_PAIRED_NEIGHBOR:
    case LBM_PATTERN_PULL_QUAD:
    case LBM_PATTERN_AA_QUAD_LOCAL:
    case LBM_PATTERN_AA_QUAD_NEIGHBOR: {
      const int npw = pattern <= LBM_PATTERN_AA_PAIRED_NEIGHBOR ? 2 : 4;
      const dim3 gw((b.n / npw + 127) / 128, b.n, b.n);
      if (pattern == LBM_PATTERN_AA_PAIRED_LOCAL) k_words<2, 1><<<gw, blk, 0, st>>>(a, b2, b);
      if (pattern == LBM_PATTERN_AA_PAIRED_NEIGHBOR) k_words<2, 2><<<gw, blk, 0, st>>>(a, b2, b);
      if (pattern == LBM_PATTERN_PULL_QUAD) k_words<4, 0><<<gw, blk, 0, st>>>(a, b2, b);
      if (pattern == LBM_PATTERN_AA_QUAD_LOCAL) k_words<4, 1><<<gw, blk, 0, st>>>(a, b2, b);
      if (pattern == LBM_PATTERN_AA_QUAD_NEIGHBOR) k_words<4, 2><<<gw, blk, 0, st>>>(a, b2, b);
      break;
    }
  }
  return cudaGetLastError() == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

// nodes one launch of the pattern updates
long long nodes_of(int pattern, int n) {
  const long long i = n - 2;
  switch (pattern) {
    case LBM_PATTERN_PULL:
    case LBM_PATTERN_AA_NEIGHBOR: return i * i * i;
    case LBM_PATTERN_PULL_PAIRED:
    case LBM_PATTERN_AA_PAIRED_NEIGHBOR: return 2LL * (n / 2 - 2) * i * i;
    case LBM_PATTERN_PULL_QUAD:
    case LBM_PATTERN_AA_QUAD_NEIGHBOR: return 4LL * (n / 4 - 2) * i * i;
    default: return (long long)n * n * n;
  }
}

}  // namespace

extern "C" int lbm_pattern_ceiling(int pattern, int storage, int n, int iters, double* mlups,
                                   double* gbs) {
  if (!mlups || !gbs) return lbm::set_error(LBM_ERR_INVALID, "lbm_pattern_ceiling: NULL output");
  if (pattern < LBM_PATTERN_COPY || pattern > LBM_PATTERN_AA_QUAD_NEIGHBOR)
    return lbm::set_error(LBM_ERR_INVALID, "unknown pattern %d", pattern);
  if (storage != LBM_STORE_F32 && storage != LBM_STORE_F16_SHIFT)
    return lbm::set_error(LBM_ERR_INVALID, "patterns are timed for F32 and F16 storage only");
  if ((pattern == LBM_PATTERN_PULL_PAIRED || pattern >= LBM_PATTERN_AA_PAIRED_LOCAL) &&
      storage != LBM_STORE_F16_SHIFT)
    return lbm::set_error(LBM_ERR_INVALID, "the word patterns are 16-bit layouts");
  if (n < 32 || n > 512 || n % 32 || iters < 1 || iters > 100000)
    return lbm::set_error(LBM_ERR_INVALID, "n must be a multiple of 32 in [32, 512], iters >= 1");
  const size_t elem = storage == LBM_STORE_F32 ? 4 : 2;
  Box b;
  b.n = n;
  b.qs = (long long)n * n * n;
  const size_t bytes = (size_t)Q * b.qs * elem;
  void *a = nullptr, *c = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t st = nullptr;
  int rc = LBM_OK;
  float ms = 0.f;
  auto body = [&]() -> int {
    if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&c, bytes) != cudaSuccess)
      return lbm::set_error(LBM_ERR_OOM, "lbm_pattern_ceiling: %zu bytes", 2 * bytes);
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
      return lbm::set_error(LBM_ERR_CUDA, "lbm_pattern_ceiling: stream/event");
    // small finite values everywhere (the token arithmetic keeps them finite)
    if (cudaMemsetAsync(a, 0x11, bytes, st) != cudaSuccess ||
        cudaMemsetAsync(c, 0x11, bytes, st) != cudaSuccess)
      return lbm::set_error(LBM_ERR_CUDA, "lbm_pattern_ceiling: memset");
    auto one = [&](int i) {
      void* s = (i & 1) ? c : a;
      void* d = (i & 1) ? a : c;
      return storage == LBM_STORE_F32 ? launch<float>(pattern, s, d, b, st)
                                      : launch<__half>(pattern, s, d, b, st);
    };
    for (int i = 0; i < 3; ++i)
      if (one(i)) return lbm::set_error(LBM_ERR_CUDA, "lbm_pattern_ceiling: launch failed");
    cudaEventRecord(e0, st);
    for (int i = 0; i < iters; ++i)
      if (one(i)) return lbm::set_error(LBM_ERR_CUDA, "lbm_pattern_ceiling: launch failed");
    cudaEventRecord(e1, st);
    const cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess)
      return lbm::set_error(LBM_ERR_CUDA, "lbm_pattern_ceiling: %s", cudaGetErrorString(e));
    cudaEventElapsedTime(&ms, e0, e1);
    return LBM_OK;
  };
  rc = body();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (a) cudaFree(a);
  if (c) cudaFree(c);
  if (rc) return rc;
  const double per_launch_s = (double)ms / 1e3 / iters;
  const long long nodes = nodes_of(pattern, n);
  *mlups = (double)nodes / per_launch_s / 1e6;
  *gbs = 2.0 * Q * elem * (double)nodes / per_launch_s / 1e9;
  return LBM_OK;
}
