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
  int nx, nz;        // items per row (nodes, or words of paired rows), rows per plane
  int active;        // steps the domain takes in this chunk
  unsigned long long mnx, mnz;  // ceil(2^64 / n): exact 32-bit division
  long long nodes;   // items: nodes, or words of paired rows
  int cur0;          // lattice holding f* (AA: layout) at chunk start
  int entry0;        // AA: entry mode of the chunk's first step (k_aa_step)
};

// model: 0 SRT, 1 SRT+LES, 2 MRT, 3 MRT+LES; mode: kModePull (plain rows,
// A/B), kModeAA (AA streaming), kModePaired (16-bit A/B in paired rows);
// variant = (storage * 4 + model) * 3 + mode.  A launch group is the
// domains of one variant; each step launches the group's kernel once.
// Storage scales travel in the argument images.
constexpr int kGroups = 32;
enum { kModePull = 0, kModeAA = 1, kModePaired = 2, kModes = 3 };

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
  int tile;          // nodes per tile = 32 * npt (a warp tile)
  int schedule;      // 0: contiguous tile range per warp, 1: warp-stride
  GroupList v[kGroups];
  const SlotMeta* meta;
  const long long* tile_off;
  const unsigned char* images;   // [capacity * kImages][kArgsBytes]
};

__device__ __forceinline__ unsigned fastdiv(unsigned n, unsigned long long m) {
  return (unsigned)__umul64hi(m, (unsigned long long)n);
}

// A warp's current domain, in shared memory (one per warp): everything the
// tile loop needs besides the tile index, so that little stays live in
// registers across the node step.
struct WarpSlot {
  SlotMeta m;
  unsigned begin, end;  // the domain's tiles [begin, end) in the group list
  int s;                // slot index in the group
  int ok;               // the domain takes step j
  int image;            // argument image held in the warp's img[], -1 = none
  int pad;
};

constexpr int kMaxWarps = 8;  // 256-thread CTAs at most

// Make the slot holding tile t (at or after the warp's current one) the
// warp's current domain: meta, tile range and, when it takes step j, its
// argument image for launch j, copied into the warp's own image.  Every
// lane of the warp takes the same path; no other warp is involved.
__device__ __forceinline__ void warp_enter(WarpSlot& cur, unsigned char* img,
                                           const BatchTables* __restrict__ tab, int g, unsigned t,
                                           int j) {
  const unsigned lane = threadIdx.x & 31u;
  __syncwarp();  // every lane is done with the previous domain's image
  int fetch = -1;
  if (lane == 0) {
    const GroupList& L = tab->v[g];
    const long long* off = tab->tile_off + L.off0;
    int lo = cur.s, hi = L.nslots;  // off[lo] <= t < off[hi]
    if (off[lo + 1] > (long long)t) {
      hi = lo + 1;
    } else {
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= (long long)t)
          lo = mid;
        else
          hi = mid;
      }
    }
    const SlotMeta m = tab->meta[L.slot0 + lo];
    cur.m = m;
    cur.s = lo;
    cur.begin = (unsigned)off[lo];
    cur.end = (unsigned)off[lo + 1];
    cur.ok = j < m.active;
    const int image = m.image_base + ((m.cur0 + j) & 1) * 3 +
                      (j >= m.active - 1 ? 2 : (j >= m.active - 2 ? 1 : 0));
    fetch = cur.ok && image != cur.image ? image : -1;
    if (cur.ok) cur.image = image;
  }
  fetch = __shfl_sync(0xffffffffu, fetch, 0);
  if (fetch >= 0) {
    const int4* src = reinterpret_cast<const int4*>(tab->images + (size_t)fetch * kArgsBytes);
    int4* dst = reinterpret_cast<int4*>(img);
    for (unsigned i = lane; i < kArgsBytes / 16; i += 32) dst[i] = src[i];
  }
  __syncwarp();
}

// One time step (launch j of a chunk) of every active domain of launch
// group g (one variant).  The unit of work is a warp tile: 32 x npt
// consecutive items of one domain (row-major, rows may wrap): nodes, or for
// members in paired rows (MODE kModePaired) the words of node pairs.  Each warp
// walks its own tiles: schedule 0, the contiguous range [w*per, (w+1)*per)
// of the group's list; schedule 1, t = w, += (warps in the grid).  A warp
// enters a domain (meta and argument image into its own shared memory)
// only when its next tile lies in another one, without waiting for the
// other warps of its CTA; the node step reads the arguments from there.
// Tile indices are 32-bit (the host keeps a group below 2^31 tiles).
// MINB (resident 256-thread CTAs the register budget must allow: 4 -> 64
// registers, 3 -> 80) trades occupancy against spills; the autotuner picks.
template <class S, int COLL, bool LES, int MINB, int MODE>
__global__ void __launch_bounds__(256, MINB) k_batch_step(const BatchTables* __restrict__ tab,
                                                          int g, int j, int npt) {
  __shared__ __align__(16) unsigned char img[kMaxWarps][kArgsBytes];
  __shared__ WarpSlot slots[kMaxWarps];
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const StepArgs<S>& a = *reinterpret_cast<const StepArgs<S>*>(img[warp]);
  WarpSlot& cur = slots[warp];
  const unsigned ntiles = (unsigned)tab->v[g].ntiles;
  const unsigned nw = gridDim.x * (blockDim.x >> 5);
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + warp;
  unsigned t, tend, stride;
  if (tab->schedule == 0) {
    const unsigned per = (ntiles + nw - 1) / nw;
    t = w * per;
    tend = min(t + per, ntiles);
    stride = 1;
  } else {
    t = w;
    tend = ntiles;
    stride = nw;
  }
  if (lane == 0) {
    cur.s = 0;
    cur.image = -1;
    cur.begin = 0;
    cur.end = 0;
    cur.ok = 0;
  }
  __syncwarp();
  const unsigned span = 32u * (unsigned)npt;
  for (; t < tend; t += stride) {
    if (t >= cur.end) warp_enter(cur, img[warp], tab, g, t, j);
    if (!cur.ok) {
      if (stride == 1) t = cur.end - 1;  // skip the domain
      continue;
    }
    const unsigned n0 = (t - cur.begin) * span;
    const unsigned nend = min(n0 + span, (unsigned)cur.m.nodes);
    for (unsigned n = n0 + lane; n < nend; n += 32u) {
      const unsigned r = fastdiv(n, cur.m.mnx);
      const int x = (int)(n - r * (unsigned)cur.m.nx);
      const unsigned y = fastdiv(r, cur.m.mnz);
      const int z = (int)(r - y * (unsigned)cur.m.nz);
      if constexpr (MODE == kModeAA)
        aa_step_node<S, COLL, LES>(a, x, (int)y, z, a.aa_step - 1,
                                   j == 0 ? cur.m.entry0 : kAAPending);
      else if constexpr (MODE == kModePaired)
        paired_word<S, COLL, LES, false>(a, x, (int)y, z);  // x: the word
      else
        step_node<S, COLL, LES>(a, x, (int)y, z);
    }
  }
}

// ------------------------------------------------------------------ //
// Schedule 2: flat grids with the arguments in the kernel parameter space.
// A launch steps one set of at most kFlatMax members of one variant by one
// time step: one CTA per 128 consecutive items (nodes, or words of paired
// rows) of a member, the member found by a loop over the set's CTA offsets
// that depends on blockIdx and parameters only, so it is the same for every
// thread, and the member's arguments read from the parameter space like
// those of a single-domain kernel.  Each set is a chain of launches in the
// chunk graph, independent of the other sets, so the sets' launches overlap
// on the GPU and fill each other's tails.  A set of one member launches the
// member's single-domain step kernel instead (its arguments are kernel
// parameters there as well).
// ------------------------------------------------------------------ //
constexpr int kFlatMax = 32;
constexpr int kFlatBlock = 128;

struct FlatMeta {
  int nx, nz;        // items per row, rows per plane
  unsigned items;    // items of the member
  int entry;         // AA: entry mode of this step (k_aa_step)
  unsigned long long mnx, mnz;
};

template <class S>
struct FlatSet {
  int n;                           // members of the set taking this step
  int pad[3];
  unsigned cta_off[kFlatMax + 1];  // CTAs of members [0, k): cta_off[k]
  FlatMeta meta[kFlatMax];
  StepArgs<S> args[kFlatMax];
};
static_assert(sizeof(FlatSet<float>) <= 32000, "kernel parameters are limited to 32 KB");
static_assert(sizeof(FlatSet<__half>) == sizeof(FlatSet<float>) &&
                  sizeof(FlatSet<__nv_bfloat16>) == sizeof(FlatSet<float>) &&
                  sizeof(StepArgs<__half>) == sizeof(StepArgs<float>) &&
                  sizeof(StepArgs<__nv_bfloat16>) == sizeof(StepArgs<float>),
              "the host fills every format's FlatSet through the FP32 layout");

template <class S, int COLL, bool LES, int MODE>
__global__ void __launch_bounds__(kFlatBlock, 8)
    k_batch_flat(const __grid_constant__ FlatSet<S> p) {
  int s = 0;
  for (int k = 1; k < p.n; ++k) s += blockIdx.x >= p.cta_off[k];
  const StepArgs<S>& a = p.args[s];
  const FlatMeta& m = p.meta[s];
  const unsigned n = (blockIdx.x - p.cta_off[s]) * (unsigned)kFlatBlock + threadIdx.x;
  if (n >= m.items) return;
  const unsigned r = fastdiv(n, m.mnx);
  const int x = (int)(n - r * (unsigned)m.nx);
  const unsigned y = fastdiv(r, m.mnz);
  const int z = (int)(r - y * (unsigned)m.nz);
  if constexpr (MODE == kModeAA)
    aa_step_node<S, COLL, LES>(a, x, (int)y, z, a.aa_step - 1, m.entry);
  else if constexpr (MODE == kModePaired)
    paired_word<S, COLL, LES, false>(a, x, (int)y, z);
  else
    step_node<S, COLL, LES>(a, x, (int)y, z);
}

// kernel of (model, register build, mode): k[model][regs][mode];
// regs 0 -> the 64-register build, 1 -> the 80-register build; the paired
// mode exists for the 16-bit formats only (nullptr for FP32)
using BatchKernel = void (*)(const BatchTables*, int, int, int);
struct BatchKernels {
  BatchKernel k[4][2][kModes];
  const void* flat[4][kModes];  // k_batch_flat<S, ...>: the FlatSet<S> of the format
  // the single-domain step kernels (a set of one member, schedule 2):
  // [model][mode][NB], NB the AA step kind (k_aa_step<.., NB>), 0 otherwise
  const void* single[4][kModes][2];
};

template <class S, int MINB, int MODE>
constexpr BatchKernel batch_kernel_of(int model) {
  return model == 0   ? k_batch_step<S, COLL_SRT, false, MINB, MODE>
         : model == 1 ? k_batch_step<S, COLL_SRT, true, MINB, MODE>
         : model == 2 ? k_batch_step<S, COLL_MRT, false, MINB, MODE>
                      : k_batch_step<S, COLL_MRT, true, MINB, MODE>;
}

template <class S, int MODE>
const void* flat_kernel_of(int model) {
  return model == 0   ? (const void*)k_batch_flat<S, COLL_SRT, false, MODE>
         : model == 1 ? (const void*)k_batch_flat<S, COLL_SRT, true, MODE>
         : model == 2 ? (const void*)k_batch_flat<S, COLL_MRT, false, MODE>
                      : (const void*)k_batch_flat<S, COLL_MRT, true, MODE>;
}

template <class S, int COLL, bool LES>
void set_single(BatchKernels& t, int m) {
  t.single[m][kModePull][0] = (const void*)k_step<S, COLL, LES, false>;
  t.single[m][kModePull][1] = nullptr;
  t.single[m][kModeAA][0] = (const void*)k_aa_step<S, COLL, LES, 0>;
  t.single[m][kModeAA][1] = (const void*)k_aa_step<S, COLL, LES, 1>;
  if constexpr (kDev<S>)
    t.single[m][kModePaired][0] = (const void*)k_step_paired<S, COLL, LES, false>;
  else
    t.single[m][kModePaired][0] = nullptr;
  t.single[m][kModePaired][1] = nullptr;
}

template <class S>
BatchKernels make_batch_kernels() {
  BatchKernels t;
  set_single<S, COLL_SRT, false>(t, 0);
  set_single<S, COLL_SRT, true>(t, 1);
  set_single<S, COLL_MRT, false>(t, 2);
  set_single<S, COLL_MRT, true>(t, 3);
  for (int m = 0; m < 4; ++m) {
    t.k[m][0][kModePull] = batch_kernel_of<S, 4, kModePull>(m);
    t.k[m][1][kModePull] = batch_kernel_of<S, 3, kModePull>(m);
    t.k[m][0][kModeAA] = batch_kernel_of<S, 4, kModeAA>(m);
    t.k[m][1][kModeAA] = batch_kernel_of<S, 3, kModeAA>(m);
    t.flat[m][kModePull] = flat_kernel_of<S, kModePull>(m);
    t.flat[m][kModeAA] = flat_kernel_of<S, kModeAA>(m);
    if constexpr (kDev<S>) {
      t.k[m][0][kModePaired] = batch_kernel_of<S, 4, kModePaired>(m);
      t.k[m][1][kModePaired] = batch_kernel_of<S, 3, kModePaired>(m);
      t.flat[m][kModePaired] = flat_kernel_of<S, kModePaired>(m);
    } else {
      t.k[m][0][kModePaired] = t.k[m][1][kModePaired] = nullptr;
      t.flat[m][kModePaired] = nullptr;
    }
  }
  return t;
}

extern const BatchKernels kBatch_f32, kBatch_f16, kBatch_bf16;

}  // namespace batch
}  // namespace lbm
