// lbm_batch_kernel.cuh — the persistent kernel of the batched form (see
// lbm_batch.cu) and the tables it reads.  Instantiated once per storage
// format in lbm_batch_f32.cu, lbm_batch_f16.cu and lbm_batch_bf16.cu (one
// translation unit each, built in parallel) and reached through the
// BatchKernels table of the format.
#pragma once

#include "lbm_domain.cuh"

namespace lbm {
namespace batch {

constexpr int kArgsBytes = 1024;  // one StepArgs<S> image, 16-byte multiple
static_assert(sizeof(StepArgs<float>) <= kArgsBytes, "StepArgs too large");
static_assert(sizeof(StepArgs<__half>) <= kArgsBytes, "StepArgs too large");
static_assert(sizeof(StepArgs<__nv_bfloat16>) <= kArgsBytes, "StepArgs too large");
// argument images per domain: lattice parity (2) x output kind (3: none,
// rho, rho + u)
constexpr int kImages = 6;

// per active domain, per chunk
struct SlotMeta {
  int image_base;    // index of the domain's first argument image
  int nx, nz;
  int active;        // steps the domain takes in this chunk
  unsigned long long mnx, mnz;  // ceil(2^64 / n): exact 32-bit division
  long long nodes;
  int cur0;          // lattice holding f* (AA: layout) at chunk start
  int entry0;        // AA: entry mode of the chunk's first step (k_aa_step)
};

// model: 0 SRT, 1 SRT+LES, 2 MRT, 3 MRT+LES; variant = (storage * 4 +
// model) * 2 + aa (aa: AA streaming).  A launch group is the domains of one
// variant; each step launches the group's kernel once.  Storage scales travel
// in the argument images.
constexpr int kGroups = 32;

// The domains of one group: meta[slot0 .. slot0 + nslots) and their tile
// prefix sums tile_off[off0 .. off0 + nslots] (tiles of the group's list).
struct GroupList {
  int nslots;
  int slot0;
  int off0;
  int pad;
  long long ntiles;
};

struct BatchTables {
  int tile;          // nodes per tile = block * npt
  int schedule;      // 0: contiguous tile range per CTA, 1: grid-stride
  GroupList v[kGroups];
  const SlotMeta* meta;
  const long long* tile_off;
  const unsigned char* images;   // [capacity * kImages][kArgsBytes]
};

__device__ __forceinline__ unsigned fastdiv(unsigned n, unsigned long long m) {
  return (unsigned)__umul64hi(m, (unsigned long long)n);
}

// the CTA's current domain, in shared memory: everything the tile loop
// needs besides the tile index itself, so that little stays live in
// registers across the node step
struct CurSlot {
  SlotMeta m;
  long long begin, end;  // the domain's tiles [begin, end) in the group list
  long long ntiles;      // tiles of the group
  int s;                 // slot index in the group, -1 before the first
  int ok;                // the domain takes step j
  int image;             // argument image in img[], -1 = none
  int fetch;             // image to copy into img[] on entry, -1 = none
};

// the nodes of local tile lt of the current domain
template <class S, int COLL, bool LES, bool AA>
__device__ __forceinline__ void batch_tile(const StepArgs<S>& a, const CurSlot& cur,
                                           unsigned lt, int npt, int j) {
  const unsigned base = lt * (unsigned)(blockDim.x * npt);
  for (int i = 0; i < npt; ++i) {
    const unsigned n = base + (unsigned)i * blockDim.x + threadIdx.x;
    if (n >= (unsigned)cur.m.nodes) break;
    const unsigned r = fastdiv(n, cur.m.mnx);
    const int x = (int)(n - r * (unsigned)cur.m.nx);
    const unsigned y = fastdiv(r, cur.m.mnz);
    const int z = (int)(r - y * (unsigned)cur.m.nz);
    if constexpr (AA)
      aa_step_node<S, COLL, LES>(a, x, (int)y, z, a.aa_step - 1,
                                 j == 0 ? cur.m.entry0 : kAAPending);
    else
      step_node<S, COLL, LES>(a, x, (int)y, z);
  }
}

// Make the slot holding tile t (at or after the current one) the CTA's
// current domain: meta, tile range and, when it takes step j, its argument
// image for launch j.  All threads of the CTA take the same path.
__device__ __forceinline__ void enter_slot(CurSlot& cur, unsigned char* img,
                                           const BatchTables* __restrict__ tab, int g, long long t,
                                           int j) {
  __syncthreads();  // every thread is done with the previous domain
  if (threadIdx.x == 0) {
    const GroupList& L = tab->v[g];
    const long long* off = tab->tile_off + L.off0;
    int lo = cur.s < 0 ? 0 : cur.s, hi = L.nslots;  // off[lo] <= t < off[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= t)
        lo = mid;
      else
        hi = mid;
    }
    const SlotMeta m = tab->meta[L.slot0 + lo];
    cur.m = m;
    cur.s = lo;
    cur.begin = off[lo];
    cur.end = off[lo + 1];
    cur.ok = j < m.active;
    const int image = m.image_base + ((m.cur0 + j) & 1) * 3 +
                      (j >= m.active - 1 ? 2 : (j >= m.active - 2 ? 1 : 0));
    cur.fetch = cur.ok && image != cur.image ? image : -1;
    if (cur.ok) cur.image = image;
  }
  __syncthreads();
  const int fetch = cur.fetch;
  if (fetch >= 0) {
    const int4* src = reinterpret_cast<const int4*>(tab->images + (size_t)fetch * kArgsBytes);
    int4* dst = reinterpret_cast<int4*>(img);
    for (int i = threadIdx.x; i < kArgsBytes / 16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
}

// One time step (launch j of a chunk) of every active domain of launch
// group g (one variant).  Schedule 0 gives CTA c the
// contiguous tiles [c*per, (c+1)*per) of the group's list; schedule 1 walks
// t = blockIdx.x, += gridDim.x.  Either way the CTA moves forward through the
// domains and reloads a domain's arguments only when it enters it.  The
// domain's arguments and meta stay in shared memory (uniform over the CTA).
// MINB (resident 256-thread CTAs the register budget must allow: 4 -> 64
// registers, 3 -> 80) trades occupancy against spills; the autotuner picks.
template <class S, int COLL, bool LES, int MINB, bool AA>
__global__ void __launch_bounds__(256, MINB) k_batch_step(const BatchTables* __restrict__ tab,
                                                          int g, int j, int npt) {
  __shared__ __align__(16) unsigned char img[kArgsBytes];
  __shared__ CurSlot cur;
  const StepArgs<S>& a = *reinterpret_cast<const StepArgs<S>*>(img);
  if (threadIdx.x == 0) {
    cur.s = -1;
    cur.image = -1;
    cur.end = 0;
    cur.ntiles = tab->v[g].ntiles;
  }
  __syncthreads();
  if (tab->schedule == 0) {
    const long long per = (cur.ntiles + gridDim.x - 1) / gridDim.x;
    const long long t0 = (long long)blockIdx.x * per;
    for (long long t = t0; t < min(t0 + per, cur.ntiles); ++t) {
      if (t >= cur.end) enter_slot(cur, img, tab, g, t, j);
      if (!cur.ok) {
        t = cur.end - 1;
        continue;
      }
      batch_tile<S, COLL, LES, AA>(a, cur, (unsigned)(t - cur.begin), npt, j);
    }
  } else {
    for (long long t = blockIdx.x; t < cur.ntiles; t += gridDim.x) {
      if (t >= cur.end) enter_slot(cur, img, tab, g, t, j);
      if (!cur.ok) continue;
      batch_tile<S, COLL, LES, AA>(a, cur, (unsigned)(t - cur.begin), npt, j);
    }
  }
}

// kernel of (model, register build, streaming): k[model][regs][aa];
// regs 0 -> the 64-register build, 1 -> the 80-register build
using BatchKernel = void (*)(const BatchTables*, int, int, int);
struct BatchKernels {
  BatchKernel k[4][2][2];
};

template <class S, int MINB, bool AA>
constexpr BatchKernel batch_kernel_of(int model) {
  return model == 0   ? k_batch_step<S, COLL_SRT, false, MINB, AA>
         : model == 1 ? k_batch_step<S, COLL_SRT, true, MINB, AA>
         : model == 2 ? k_batch_step<S, COLL_MRT, false, MINB, AA>
                      : k_batch_step<S, COLL_MRT, true, MINB, AA>;
}

template <class S>
BatchKernels make_batch_kernels() {
  BatchKernels t;
  for (int m = 0; m < 4; ++m) {
    t.k[m][0][0] = batch_kernel_of<S, 4, false>(m);
    t.k[m][1][0] = batch_kernel_of<S, 3, false>(m);
    t.k[m][0][1] = batch_kernel_of<S, 4, true>(m);
    t.k[m][1][1] = batch_kernel_of<S, 3, true>(m);
  }
  return t;
}

extern const BatchKernels kBatch_f32, kBatch_f16, kBatch_bf16;

}  // namespace batch
}  // namespace lbm
