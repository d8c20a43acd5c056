// lbm_batch.cu — many independent domains of uneven size resident on one
// GPU and stepped together: one persistent kernel per time step over a tile
// work-list, step chunks captured as CUDA graphs, a device memory pool for
// admission by HBM budget, per-domain step targets (continuous batching) and
// an autotuner over the launch shape.
//
// Work-list.  Every active domain contributes ceil(nodes / tile) tiles, a
// tile (a warp tile) being 32*npt consecutive nodes in the domain's
// [y][z][x] order.  tile_off[] is the prefix sum over the active domains;
// each warp walks its own tiles (a contiguous range, or t = warp, += warps
// in the grid), finds a tile's domain by a search from its current one and
// copies that domain's kernel arguments into its own shared memory, with
// no barrier across the warps of a CTA.
// Each node then runs step_node<S, COLL, LES>() (aa_step_node for members
// with AA streaming) — the very function of the single-domain kernel — so a
// domain produces the same bits alone and in a batch, whatever else is
// resident (no cross-domain data, no atomics).  The kernels live in
// lbm_batch_kernel.cuh, one translation unit per storage format.
//
// Graphs.  All kernel inputs live in device tables, so the graph of a chunk
// (chunk_steps launches, launch j reading the tables) stays valid while the
// membership changes; only the tables are re-uploaded before each chunk.
#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "lbm_batch_kernel.cuh"

using namespace lbm;
using namespace lbm::batch;

namespace {

// variant -> kernel: variant = (storage * 4 + model) * kModes + mode
BatchKernel batch_kernel(int variant, int regs) {
  const int mode = variant % kModes, model = (variant / kModes) % 4,
            st = variant / (4 * kModes);
  const BatchKernels& t = st == 0 ? kBatch_f32 : (st == 1 ? kBatch_f16 : kBatch_bf16);
  return t.k[model][regs == 1 ? 1 : 0][mode];
}

// First-fit device pool with coalescing (offsets 256-byte aligned).
struct Pool {
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_;  // offset -> size
  std::map<size_t, size_t> used_;  // offset -> size
  void reset(char* b, size_t n) {
    base = b;
    size = n;
    free_.clear();
    used_.clear();
    if (n) free_[0] = n;
  }
  void* alloc(size_t n) {
    n = (n + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const size_t off = it->first, rest = it->second - n;
        free_.erase(it);
        if (rest) free_[off + n] = rest;
        used_[off] = n;
        return base + off;
      }
    }
    return nullptr;
  }
  void release(void* p) {
    if (!p) return;
    const size_t off = (size_t)((char*)p - base);
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t n = u->second;
    used_.erase(u);
    size_t start = off;
    auto nx = free_.lower_bound(off);
    if (nx != free_.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) {
        start = pv->first;
        n += pv->second;
        free_.erase(pv);
      }
    }
    nx = free_.lower_bound(off);
    if (nx != free_.end() && start + n == nx->first) {
      n += nx->second;
      free_.erase(nx);
    }
    free_[start] = n;
  }
  size_t used() const {
    size_t s = 0;
    for (auto& kv : used_) s += kv.second;
    return s;
  }
  size_t largest_free() const {
    size_t s = 0;
    for (auto& kv : free_) s = std::max(s, kv.second);
    return s;
  }
};

int model_of(const Inputval& in) { return (in.bEnableMRT ? 2 : 0) + (in.bEnableLES ? 1 : 0); }

int storage_index(int storage) {
  return storage == LBM_STORE_F16_SHIFT ? 1 : (storage == LBM_STORE_BF16_SHIFT ? 2 : 0);
}

}  // namespace

struct lbm_batch {
  lbm_batch_options opt;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t capture = nullptr;
  char* pool_mem = nullptr;
  Pool pool;
  struct Member {
    lbm_domain* d = nullptr;
    long long target = 0;
    int image_slot = 0;       // index in the image table
    long long issued = 0;     // steps issued so far
    long long done_chunk = -1;  // chunk whose completion makes the result final
    int last_active = 0;        // steps taken in the last chunk issued
    cudaEvent_t admitted = nullptr;  // initial state and images written (batch stream)
  };
  std::map<int, Member> members;
  int next_id = 1;
  int capacity = 0;               // image slots
  std::vector<int> free_images;
  // device tables and their pinned host images
  unsigned char* h_images = nullptr;  // pinned host copy of d_images (async uploads)
  cudaStream_t fetch = nullptr;       // results of finished members (lbm_batch_fetch)
  BatchTables* d_tab = nullptr;
  SlotMeta* d_meta = nullptr;
  long long* d_off = nullptr;
  unsigned char* d_images = nullptr;
  BatchTables* h_tab = nullptr;
  SlotMeta* h_meta = nullptr;
  long long* h_off = nullptr;
  cudaEvent_t tables_free = nullptr;  // previous table upload has been consumed
  // chunk graph
  cudaGraphExec_t graph = nullptr;
  int graph_block = 0, graph_npt = 0, graph_steps = 0, graph_sched = -1;
  std::vector<int> graph_groups;  // variant per launch group
  int graph_ctas = -1, graph_regs = -1;
  // completion tracking
  long long chunks_issued = 0;
  std::vector<std::pair<long long, cudaEvent_t>> chunk_events;
  std::vector<std::pair<long long, cudaGraphExec_t>> flat_execs;  // schedule 2, to release
  cudaGraphExec_t flat_cached = nullptr;  // schedule 2: the last chunk's graph
  long long flat_cached_chunk = 0;        // ... and the last chunk it ran
  std::vector<long long> flat_sig;        // ... and what it was built for
  long long chunks_completed = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long long last_lups = 0;
  int last_steps = 0;
};

namespace {

int chunk_steps(const lbm_batch* b) { return b->opt.chunk_steps > 0 ? b->opt.chunk_steps : 32; }

int launch_block(const lbm_batch* b) { return b->opt.block == 128 ? 128 : 256; }
int launch_npt(const lbm_batch* b) {
  return b->opt.nodes_per_thread > 0 ? b->opt.nodes_per_thread : 2;
}

// persistent grid of one variant's kernel: resident CTAs per SM x SMs
int launch_grid(lbm_batch* b, int variant, int block, int* grid) {
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel(variant, b->opt.regs),
                                                   block, 0));
  if (per_sm < 1) per_sm = 1;
  if (b->opt.ctas_per_sm > 0 && b->opt.ctas_per_sm < per_sm) per_sm = b->opt.ctas_per_sm;
  *grid = per_sm * b->sm_count;
  return LBM_OK;
}

int member_mode(const lbm_domain* d) {
  return d->opt.stream_mode == LBM_STREAM_AA ? kModeAA
                                             : (d->g.rows == kRowsPaired ? kModePaired : kModePull);
}

int member_variant(const lbm_domain* d) {
  return (storage_index(d->opt.storage) * 4 + model_of(d->in)) * kModes + member_mode(d);
}

// Launch groups (variants) of the members that still have steps to take,
// in a fixed order.
std::vector<int> pending_groups(const lbm_batch* b) {
  std::vector<int> gs;
  for (auto& kv : b->members)
    if (kv.second.issued < kv.second.target) {
      const int key = member_variant(kv.second.d);
      if (std::find(gs.begin(), gs.end(), key) == gs.end()) gs.push_back(key);
    }
  std::sort(gs.begin(), gs.end());
  return gs;
}

// (Re)capture the chunk graph: chunk_steps steps, each one launch per
// launch group, for the current launch shape.
int ensure_graph(lbm_batch* b, const std::vector<int>& groups) {
  const int block = launch_block(b), npt = launch_npt(b), steps = chunk_steps(b);
  const int sched = b->opt.schedule == 1 ? 1 : 0;
  if ((int)groups.size() > kGroups)
    return set_error(LBM_ERR_INVALID, "more than %d (model, storage, streaming) groups in a batch", kGroups);
  if (b->graph && b->graph_block == block && b->graph_npt == npt && b->graph_steps == steps &&
      b->graph_groups == groups && b->graph_sched == sched &&
      b->graph_ctas == b->opt.ctas_per_sm && b->graph_regs == b->opt.regs)
    return LBM_OK;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  std::vector<int> grids(groups.size());
  for (size_t g = 0; g < groups.size(); ++g) {
    int rc = launch_grid(b, groups[g], block, &grids[g]);
    if (rc) return rc;
  }
  CK(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
  for (int j = 0; j < steps; ++j)
    for (size_t g = 0; g < groups.size(); ++g)
      batch_kernel(groups[g], b->opt.regs)<<<grids[g], block, 0, b->capture>>>(b->d_tab, (int)g,
                                                                              j, npt);
  cudaGraph_t gr;
  CK(cudaStreamEndCapture(b->capture, &gr));
  cudaError_t e = cudaGraphInstantiate(&b->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess)
    return set_error(LBM_ERR_CUDA, "batch graph instantiation failed: %s", cudaGetErrorString(e));
  b->graph_block = block;
  b->graph_npt = npt;
  b->graph_steps = steps;
  b->graph_groups = groups;
  b->graph_sched = sched;
  b->graph_ctas = b->opt.ctas_per_sm;
  b->graph_regs = b->opt.regs;
  return LBM_OK;
}

// Argument images of a member: parity x {no output, rho, rho + u}.
int upload_images(lbm_batch* b, lbm_batch::Member& m) {
  lbm_domain* d = m.d;
  // the slot's pinned host image: its previous upload (an earlier member of
  // the slot) ran before that member's first chunk, long complete
  unsigned char* buf = b->h_images + (size_t)m.image_slot * kImages * kArgsBytes;
  std::memset(buf, 0, (size_t)kImages * kArgsBytes);
  int rc = with_storage(d->opt.storage, [&](auto tag) -> int {
    using S = typename decltype(tag)::type;
    if constexpr (std::is_same<S, double>::value) {
      return set_error(LBM_ERR_INVALID, "FP64 storage is not supported in batches");
    } else {
      const bool aa = d->opt.stream_mode == LBM_STREAM_AA;
      for (int par = 0; par < 2; ++par)
        for (int kind = 0; kind < 3; ++kind) {
          // a step starting from lattice (AA: layout) `par` has step number
          // of parity par^1; an AA step from layout par is a local (0) or a
          // neighbour (1) step and writes rho of its input
          StepArgs<S> a = aa ? aa_args<S>(d, par ^ 1, kind >= 1, par)
                             : make_args<S>(d, d->lat[par], d->lat[par ^ 1], par ^ 1);
          if (kind >= 1 && !aa) a.den_out = d->den[par ^ 1];
          if (kind == 2) {
            a.ux_out = d->ux;
            a.uy_out = d->uy;
            a.uz_out = d->uz;
          }
          std::memcpy(&buf[(size_t)(par * 3 + kind) * kArgsBytes], &a, sizeof(a));
        }
      return LBM_OK;
    }
  });
  if (rc) return rc;
  CK(cudaMemcpyAsync(b->d_images + (size_t)m.image_slot * kImages * kArgsBytes, buf,
                     (size_t)kImages * kArgsBytes, cudaMemcpyHostToDevice, b->stream));
  return LBM_OK;
}

int grow_images(lbm_batch* b) {
  const int cap = b->capacity ? b->capacity * 2 : 64;
  unsigned char* nimg = nullptr;
  unsigned char* himg = nullptr;
  SlotMeta *dm = nullptr, *hm = nullptr;
  long long *doff = nullptr, *hoff = nullptr;
  CK(cudaMalloc(&nimg, (size_t)cap * kImages * kArgsBytes));
  CK(cudaMallocHost(&himg, (size_t)cap * kImages * kArgsBytes));
  CK(cudaMalloc(&dm, (size_t)cap * sizeof(SlotMeta)));
  CK(cudaMalloc(&doff, (size_t)(cap + kGroups) * sizeof(long long)));
  CK(cudaMallocHost(&hm, (size_t)cap * sizeof(SlotMeta)));
  CK(cudaMallocHost(&hoff, (size_t)(cap + kGroups) * sizeof(long long)));
  CK(cudaStreamSynchronize(b->stream));
  if (b->d_images) {
    CK(cudaMemcpy(nimg, b->d_images, (size_t)b->capacity * kImages * kArgsBytes,
                  cudaMemcpyDeviceToDevice));
    std::memcpy(himg, b->h_images, (size_t)b->capacity * kImages * kArgsBytes);
    cudaFree(b->d_images);
    cudaFreeHost(b->h_images);
    cudaFree(b->d_meta);
    cudaFree(b->d_off);
    cudaFreeHost(b->h_meta);
    cudaFreeHost(b->h_off);
  }
  for (int i = cap - 1; i >= b->capacity; --i) b->free_images.push_back(i);
  b->d_images = nimg;
  b->h_images = himg;
  b->d_meta = dm;
  b->d_off = doff;
  b->h_meta = hm;
  b->h_off = hoff;
  b->capacity = cap;
  return LBM_OK;
}

void retire_completed(lbm_batch* b) {
  while (!b->chunk_events.empty()) {
    auto& ce = b->chunk_events.front();
    if (cudaEventQuery(ce.second) != cudaSuccess) break;
    b->chunks_completed = ce.first;
    cudaEventDestroy(ce.second);
    b->chunk_events.erase(b->chunk_events.begin());
  }
  while (!b->flat_execs.empty() && b->flat_execs.front().first <= b->chunks_completed) {
    cudaGraphExecDestroy(b->flat_execs.front().second);
    b->flat_execs.erase(b->flat_execs.begin());
  }
}

// After a chunk's launches: rho, u of the AA members, the completion event.
int finish_chunk(lbm_batch* b) {
  // AA members: rho, u of the state the chunk ends in (a single-domain AA
  // run ends the same way), before the chunk's completion event
  int rc;
  for (auto& kv : b->members) {
    lbm_domain* d = kv.second.d;
    if (d->opt.stream_mode == LBM_STREAM_AA && kv.second.last_active > 0 &&
        (rc = storage_ops(d->opt.storage).aa_macro(d)))
      return rc;
  }
  ++b->chunks_issued;
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, b->stream));
  b->chunk_events.push_back({b->chunks_issued, ev});
  return LBM_OK;
}

// Schedule 2.  A member of at least kOwnSetCtas CTAs (of 128 items) is a set
// of its own; the others are packed, per variant and in admission order,
// into sets of at most kFlatMax members and kSetCtas CTAs.  Each set is a
// chain of chunk_steps launches in a graph built for this chunk, with no
// edge between the chains.  Launch j of a set steps the members that take
// step j, with the argument image of their parity and output kind at that
// step: k_batch_flat, or the member's single-domain kernel when one member
// takes the step.
constexpr unsigned kOwnSetCtas = 2048;  // default of own_set_ctas
constexpr unsigned kSetCtas = 16384;

int issue_chunk_flat(lbm_batch* b, int steps_offered, long long* lups) {
  const int S = chunk_steps(b);
  *lups = 0;
  const std::vector<int> groups = pending_groups(b);
  if (groups.empty()) return LBM_OK;
  struct Item {
    lbm_batch::Member* m;
    int id, active, cur0, entry0, row_items;
    unsigned ctas;
  };
  long long updates = 0;
  const unsigned own = b->opt.own_set_ctas > 0 ? (unsigned)b->opt.own_set_ctas : kOwnSetCtas;
  for (auto& kv : b->members) kv.second.last_active = 0;
  std::vector<std::vector<Item>> sets;
  std::vector<int> set_variant;
  for (int v : groups) {
    std::vector<Item> cur;
    unsigned cur_ctas = 0;
    for (auto& kv : b->members) {
      lbm_batch::Member& m = kv.second;
      lbm_domain* d = m.d;
      const long long left = m.target - m.issued;
      if (left <= 0 || member_variant(d) != v) continue;
      Item it;
      it.m = &m;
      it.id = kv.first;
      it.active = (int)std::min<long long>(std::min(S, steps_offered), left);
      it.cur0 = d->cur;
      it.entry0 = d->aa_first ? kAAFromInit : (d->post_direct ? kAAComplete : kAAPending);
      it.row_items = d->g.rows == kRowsPaired ? d->g.px / 2 : d->g.nx;
      const long long items = (long long)it.row_items * d->g.nz * d->g.ny;
      it.ctas = (unsigned)((items + kFlatBlock - 1) / kFlatBlock);
      if (it.ctas >= own) {
        sets.push_back({it});  // a large member: a set of its own
        set_variant.push_back(v);
      } else {
        if (!cur.empty() && ((int)cur.size() == kFlatMax || cur_ctas + it.ctas > kSetCtas)) {
          sets.push_back(std::move(cur));
          set_variant.push_back(v);
          cur.clear();
          cur_ctas = 0;
        }
        cur.push_back(it);
        cur_ctas += it.ctas;
      }
      updates += d->N * it.active;
      // host bookkeeping of the steps this chunk takes
      d->step += it.active;
      d->cur ^= (it.active & 1);
      d->post_direct = false;
      d->aa_first = false;
      m.issued += it.active;
      m.last_active = it.active;
      if (m.issued >= m.target) m.done_chunk = b->chunks_issued + 1;
    }
    if (!cur.empty()) {
      sets.push_back(std::move(cur));
      set_variant.push_back(v);
    }
  }
  // The graph depends only on the sets, each member's identity, step
  // count, starting parity and entry mode (the arguments come from the
  // member's images, fixed at admission): in a steady state with an even
  // chunk the previous chunk's graph is launched again.
  std::vector<long long> sig;
  for (size_t k = 0; k < sets.size(); ++k) {
    sig.push_back(-1 - set_variant[k]);
    for (const Item& it : sets[k]) {
      sig.push_back(it.id);
      sig.push_back(((long long)it.active << 8) | (it.cur0 << 4) | it.entry0);
    }
  }
  if (b->flat_cached && sig == b->flat_sig) {
    CK(cudaGraphLaunch(b->flat_cached, b->stream));
    b->flat_cached_chunk = b->chunks_issued + 1;
    int rc = finish_chunk(b);
    if (rc) return rc;
    *lups = updates;
    return LBM_OK;
  }
  cudaGraph_t gr = nullptr;
  CK(cudaGraphCreate(&gr, 0));
  std::unique_ptr<FlatSet<float>> fs(new FlatSet<float>());
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k < sets.size() && e == cudaSuccess; ++k) {
    const int v = set_variant[k];
    const int mode = v % kModes, model = (v / kModes) % 4, st = v / (4 * kModes);
    const BatchKernels& t = st == 0 ? kBatch_f32 : (st == 1 ? kBatch_f16 : kBatch_bf16);
    cudaGraphNode_t prev = nullptr;
    for (int j = 0; j < S && e == cudaSuccess; ++j) {
      FlatSet<float>& p = *fs;
      p.n = 0;
      p.cta_off[0] = 0;
      const Item* only = nullptr;  // the member, when one takes step j
      for (const Item& it : sets[k]) {
        if (j >= it.active) continue;
        only = &it;
        const lbm_domain* d = it.m->d;
        const int kind = j >= it.active - 1 ? 2 : (j >= it.active - 2 ? 1 : 0);
        const int image = ((it.cur0 + j) & 1) * 3 + kind;
        std::memcpy(&p.args[p.n],
                    b->h_images + ((size_t)it.m->image_slot * kImages + image) * kArgsBytes,
                    sizeof(StepArgs<float>));
        FlatMeta& fm = p.meta[p.n];
        fm.nx = it.row_items;
        fm.nz = d->g.nz;
        fm.items = (unsigned)((long long)it.row_items * d->g.nz * d->g.ny);
        fm.entry = j == 0 ? it.entry0 : kAAPending;
        fm.mnx = ~0ull / (unsigned long long)it.row_items + 1;
        fm.mnz = ~0ull / (unsigned long long)d->g.nz + 1;
        p.cta_off[p.n + 1] = p.cta_off[p.n] + it.ctas;
        ++p.n;
      }
      if (p.n == 0) break;  // members only leave a set as j grows
      cudaKernelNodeParams kp;
      std::memset(&kp, 0, sizeof(kp));
      int entry = p.meta[0].entry;
      void* args[] = {fs.get(), &entry};
      kp.kernelParams = args;
      if (p.n == 1) {
        // one member: its single-domain kernel, launched as alone
        const lbm_domain* d = only->m->d;
        const int nb = mode == kModeAA ? p.args[0].aa_step - 1 : 0;
        kp.func = const_cast<void*>(t.single[model][mode][nb]);
        kp.blockDim = block_of(mode == kModePaired ? d->g.px / 2 : d->g.nx);
        kp.gridDim = dim3(((mode == kModePaired ? d->g.px / 2 : d->g.nx) + kp.blockDim.x - 1) /
                              kp.blockDim.x,
                          d->g.nz, d->g.ny);
        args[0] = &p.args[0];
      } else {
        kp.func = const_cast<void*>(t.flat[model][mode]);
        kp.gridDim = dim3(p.cta_off[p.n]);
        kp.blockDim = dim3(kFlatBlock);
      }
      cudaGraphNode_t node;
      e = cudaGraphAddKernelNode(&node, gr, prev ? &prev : nullptr, prev ? 1 : 0, &kp);
      prev = node;
    }
  }
  cudaGraphExec_t ex = nullptr;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess)
    return set_error(LBM_ERR_CUDA, "flat chunk graph: %s", cudaGetErrorString(e));
  e = cudaGraphLaunch(ex, b->stream);
  if (e != cudaSuccess) {
    cudaGraphExecDestroy(ex);
    return set_error(LBM_ERR_CUDA, "flat chunk launch: %s", cudaGetErrorString(e));
  }
  // the previous graph is released once its last chunk is complete
  // (retire_completed); this one is kept for the chunks that repeat it
  if (b->flat_cached) b->flat_execs.push_back({b->flat_cached_chunk, b->flat_cached});
  b->flat_cached = ex;
  b->flat_cached_chunk = b->chunks_issued + 1;
  b->flat_sig = std::move(sig);
  int rc = finish_chunk(b);
  if (rc) return rc;
  *lups = updates;
  return LBM_OK;
}

// Build and upload the tables of one chunk and launch its graph; returns
// the lattice updates.  Slots are grouped by variant.
int issue_chunk(lbm_batch* b, int steps_offered, long long* lups) {
  if (b->opt.schedule == 2) return issue_chunk_flat(b, steps_offered, lups);
  const int S = chunk_steps(b);
  *lups = 0;
  const std::vector<int> groups = pending_groups(b);
  if (groups.empty()) return LBM_OK;
  int rc = ensure_graph(b, groups);
  if (rc) return rc;
  const int tile = 32 * b->graph_npt;  // a warp tile
  CK(cudaEventSynchronize(b->tables_free));  // the pinned tables may be rewritten
  std::memset(b->h_tab->v, 0, sizeof(b->h_tab->v));
  int n = 0, noff = 0;
  long long updates = 0;
  for (auto& kv : b->members) kv.second.last_active = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    GroupList& L = b->h_tab->v[g];
    L.slot0 = n;
    L.off0 = noff;
    long long tiles = 0;
    for (auto& kv : b->members) {
      lbm_batch::Member& m = kv.second;
      lbm_domain* d = m.d;
      const long long left = m.target - m.issued;
      if (left <= 0 || member_variant(d) != groups[g]) continue;
      const int active = (int)std::min<long long>(std::min(S, steps_offered), left);
      SlotMeta& sm = b->h_meta[n];
      // items of a row: its nodes, or the words of a paired row
      const int row_items = d->g.rows == kRowsPaired ? d->g.px / 2 : d->g.nx;
      const long long items = (long long)row_items * d->g.nz * d->g.ny;
      sm.image_base = m.image_slot * kImages;
      sm.nx = row_items;
      sm.nz = d->g.nz;
      sm.mnx = ~0ull / (unsigned long long)row_items + 1;
      sm.mnz = ~0ull / (unsigned long long)d->g.nz + 1;
      sm.nodes = items;
      sm.active = active;
      sm.cur0 = d->cur;
      sm.entry0 = d->aa_first ? kAAFromInit : (d->post_direct ? kAAComplete : kAAPending);
      b->h_off[noff++] = tiles;
      tiles += (items + tile - 1) / tile;
      updates += d->N * active;
      // host bookkeeping of the steps this chunk takes
      d->step += active;
      d->cur ^= (active & 1);
      d->post_direct = false;
      d->aa_first = false;
      m.issued += active;
      m.last_active = active;
      if (m.issued >= m.target) m.done_chunk = b->chunks_issued + 1;
      ++n;
    }
    b->h_off[noff++] = tiles;
    L.nslots = n - L.slot0;
    L.ntiles = tiles;
  }
  b->h_tab->tile = tile;
  b->h_tab->schedule = b->graph_sched;
  b->h_tab->meta = b->d_meta;
  b->h_tab->tile_off = b->d_off;
  b->h_tab->images = b->d_images;
  CK(cudaMemcpyAsync(b->d_meta, b->h_meta, (size_t)n * sizeof(SlotMeta), cudaMemcpyHostToDevice,
                     b->stream));
  CK(cudaMemcpyAsync(b->d_off, b->h_off, (size_t)noff * sizeof(long long),
                     cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_tab, b->h_tab, sizeof(BatchTables), cudaMemcpyHostToDevice, b->stream));
  CK(cudaEventRecord(b->tables_free, b->stream));
  CK(cudaGraphLaunch(b->graph, b->stream));
  if ((rc = finish_chunk(b))) return rc;
  *lups = updates;
  return LBM_OK;
}

void destroy_member(lbm_batch* b, lbm_batch::Member& m) {
  lbm_domain* d = m.d;
  if (!d) return;
  void* bufs[] = {d->lat[0], d->lat[1],  d->den[0], d->den[1], d->ux,    d->uy,  d->uz,
                  d->inlet_u, d->prho[0], d->prho[1], d->pu[0], d->pu[1], d->flag};
  for (void* p : bufs) b->pool.release(p);
  d->stream = nullptr;  // the batch stream is not the domain's to destroy
  if (m.admitted) cudaEventDestroy(m.admitted);
  m.admitted = nullptr;
  free_all(d);
  delete d;
  m.d = nullptr;
  b->free_images.push_back(m.image_slot);
}

}  // namespace

namespace lbm {
// the stream every chunk of the batch runs on (the serving loop paces its
// chunk issue with events on it)
void* batch_stream(lbm_batch* b) { return b ? (void*)b->stream : nullptr; }
int batch_device(lbm_batch* b) { return b ? b->opt.device : 0; }
}  // namespace lbm

extern "C" {

void lbm_batch_default_options(lbm_batch_options* bo) {
  if (!bo) return;
  std::memset(bo, 0, sizeof(*bo));
  bo->hbm_budget = (size_t)8 << 30;
  bo->chunk_steps = 32;
  bo->block = 256;
  bo->nodes_per_thread = 2;
  bo->schedule = 2;  // flat grids: the fastest schedule on the mixes measured
}

int lbm_batch_domain_bytes(const Inputval* pinput, const lbm_options* opt, size_t* bytes) {
  int rc = validate(pinput, opt);
  if (rc) return rc;
  if (!bytes) return set_error(LBM_ERR_INVALID, "NULL bytes");
  *bytes = domain_state_bytes(pinput, opt);
  return LBM_OK;
}

int lbm_batch_create(const lbm_batch_options* bo, lbm_batch** out) {
  if (!out) return set_error(LBM_ERR_INVALID, "NULL out");
  *out = nullptr;
  lbm_batch_options o;
  if (bo)
    o = *bo;
  else
    lbm_batch_default_options(&o);
  if (o.chunk_steps < 0 || (o.chunk_steps & 1))
    return set_error(LBM_ERR_INVALID, "chunk_steps must be even");
  if (o.block != 0 && o.block != 128 && o.block != 256)
    return set_error(LBM_ERR_INVALID, "block must be 128 or 256");
  if (o.nodes_per_thread < 0 || o.nodes_per_thread > 16)
    return set_error(LBM_ERR_INVALID, "nodes_per_thread must be 1..16");
  if (o.schedule < 0 || o.schedule > 2)
    return set_error(LBM_ERR_INVALID, "schedule must be 0, 1 or 2");
  if (o.regs < 0 || o.regs > 1) return set_error(LBM_ERR_INVALID, "regs must be 0 or 1");
  if (o.own_set_ctas < 0) return set_error(LBM_ERR_INVALID, "own_set_ctas must be >= 0");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(LBM_ERR_NO_DEVICE, "no CUDA device available");
  if (o.device < 0 || o.device >= ndev) return set_error(LBM_ERR_INVALID, "bad device");
  CK(cudaSetDevice(o.device));
  lbm_batch* b = new lbm_batch();
  b->opt = o;
  auto fail = [&](int rc) {
    lbm_batch_destroy(b);
    return rc;
  };
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major < 10)
    return fail(set_error(LBM_ERR_NO_DEVICE, "device %d is not an sm_100 GPU", o.device));
  b->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->fetch, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->tables_free, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
    return fail(set_error(LBM_ERR_CUDA, "stream/event creation failed"));
  CK(cudaEventRecord(b->tables_free, b->stream));
  if (o.hbm_budget) {
    cudaError_t e = cudaMalloc(&b->pool_mem, o.hbm_budget);
    if (e != cudaSuccess)
      return fail(set_error(LBM_ERR_OOM, "pool of %zu bytes: %s", o.hbm_budget,
                            cudaGetErrorString(e)));
  }
  b->pool.reset(b->pool_mem, o.hbm_budget);
  int rc;
  if (cudaMalloc(&b->d_tab, sizeof(BatchTables)) != cudaSuccess ||
      cudaMallocHost(&b->h_tab, sizeof(BatchTables)) != cudaSuccess)
    return fail(set_error(LBM_ERR_OOM, "batch tables"));
  std::memset(b->h_tab, 0, sizeof(BatchTables));
  if ((rc = grow_images(b))) return fail(rc);
  *out = b;
  return LBM_OK;
}

int lbm_batch_destroy(lbm_batch* b) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  cudaSetDevice(b->opt.device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& kv : b->members) destroy_member(b, kv.second);
  b->members.clear();
  for (auto& ce : b->chunk_events) cudaEventDestroy(ce.second);
  for (auto& fe : b->flat_execs) cudaGraphExecDestroy(fe.second);
  if (b->flat_cached) cudaGraphExecDestroy(b->flat_cached);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_images) cudaFree(b->d_images);
  if (b->h_images) cudaFreeHost(b->h_images);
  if (b->fetch) cudaStreamDestroy(b->fetch);
  if (b->d_meta) cudaFree(b->d_meta);
  if (b->d_off) cudaFree(b->d_off);
  if (b->d_tab) cudaFree(b->d_tab);
  if (b->h_meta) cudaFreeHost(b->h_meta);
  if (b->h_off) cudaFreeHost(b->h_off);
  if (b->h_tab) cudaFreeHost(b->h_tab);
  if (b->pool_mem) cudaFree(b->pool_mem);
  if (b->tables_free) cudaEventDestroy(b->tables_free);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->capture) cudaStreamDestroy(b->capture);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return LBM_OK;
}

int lbm_batch_add(lbm_batch* b, const Inputval* pinput, const lbm_options* opt,
                  long long target_steps, int* id) {
  if (!b || !id) return set_error(LBM_ERR_INVALID, "NULL argument");
  int rc = validate(pinput, opt);
  if (rc) return rc;
  if (target_steps < 0) return set_error(LBM_ERR_INVALID, "negative step target");
  if (opt && opt->storage == LBM_STORE_F64)
    return set_error(LBM_ERR_INVALID, "FP64 storage is not supported in batches");
  if (opt && (opt->kernel == LBM_KERNEL_PACKED || opt->kernel == LBM_KERNEL_TMA ||
              opt->kernel == LBM_KERNEL_QUAD))
    return set_error(LBM_ERR_INVALID,
                     "batches step one node (or one paired word) per thread: kernel AUTO, "
                     "SCALAR or PAIRED");
  CK(cudaSetDevice(b->opt.device));
  if (b->free_images.empty() && (rc = grow_images(b))) return rc;
  lbm_domain* d = new lbm_domain();
  domain_prepare(d, pinput, opt);
  // 16-bit A/B members keep the paired rows of a single domain where the
  // paired step applies (no STRUCT nodes, nx large enough), else plain rows;
  // AA members keep plain rows (the batched AA step is per node)
  if (d->opt.stream_mode == LBM_STREAM_AA ||
      (d->g.rows == kRowsPaired && !paired_kernel_applies(d->g)))
    d->g.rows = kRowsPlain;
  d->opt.device = b->opt.device;
  d->pooled = true;
  d->stream = b->stream;
  std::vector<void*> taken;
  auto alloc = [&](void** p, size_t n) -> int {
    *p = b->pool.alloc(n);
    if (!*p) return LBM_ERR_BUDGET;
    taken.push_back(*p);
    d->bytes += (n + 255) / 256 * 256;
    return LBM_OK;
  };
  if ((rc = domain_alloc_state(d, alloc))) {
    for (void* p : taken) b->pool.release(p);
    delete d;
    return set_error(LBM_ERR_BUDGET, "domain of %zu bytes does not fit the pool (%zu free)",
                     domain_state_bytes(pinput, opt), b->pool.largest_free());
  }
  lbm_batch::Member m;
  m.d = d;
  m.target = target_steps;
  m.image_slot = b->free_images.back();
  b->free_images.pop_back();
  const int new_id = b->next_id++;
  b->members[new_id] = m;
  auto undo = [&](int code) {
    destroy_member(b, b->members[new_id]);
    b->members.erase(new_id);
    return code;
  };
  // admission allocates only from the pool and synchronises nothing: the
  // diagnostics / staging buffers of a member come from cudaMalloc on first
  // use (lbm_diagnostics, lbm_export_arF)
  d->diag_blocks = 4 * b->sm_count;
  if (opt && opt->rounding != LBM_ROUND_NEAREST)
    return undo(set_error(LBM_ERR_INVALID, "batch members round to nearest"));
  d->flag = (int*)b->pool.alloc(4 * sizeof(int));
  if (!d->flag) return undo(set_error(LBM_ERR_BUDGET, "pool full"));
  d->bytes += 256;
  if (cudaMemsetAsync(d->flag, 0, 4 * sizeof(int), b->stream) != cudaSuccess ||
      cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess)
    return undo(set_error(LBM_ERR_CUDA, "member set-up"));
  if ((rc = domain_upload_profile(d, b->stream)) || (rc = domain_launch_init(d, b->stream)) ||
      (rc = upload_images(b, b->members[new_id])))
    return undo(rc);
  // a member counts as finished only once its initial state exists on the
  // device: poll and fetch also wait for this event (a member with a step
  // target of 0 has no chunk of its own to wait for)
  if (cudaEventCreateWithFlags(&b->members[new_id].admitted, cudaEventDisableTiming) !=
          cudaSuccess ||
      cudaEventRecord(b->members[new_id].admitted, b->stream) != cudaSuccess)
    return undo(set_error(LBM_ERR_CUDA, "member admission event"));
  if (target_steps == 0) b->members[new_id].done_chunk = b->chunks_issued;
  *id = new_id;
  return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int steps) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  if (steps < 0) return set_error(LBM_ERR_INVALID, "negative steps");
  CK(cudaSetDevice(b->opt.device));
  // capture before the first event so that the timed span holds GPU work only
  const std::vector<int> groups = pending_groups(b);
  int rc = groups.empty() ? LBM_OK : ensure_graph(b, groups);
  if (rc) return rc;
  CK(cudaEventRecord(b->ev0, b->stream));
  long long total = 0;
  int left = steps;
  while (left > 0) {
    long long lups = 0;
    if ((rc = issue_chunk(b, left, &lups))) return rc;
    if (lups == 0) break;
    total += lups;
    left -= std::min(left, chunk_steps(b));
  }
  CK(cudaEventRecord(b->ev1, b->stream));
  b->last_lups = total;
  b->last_steps = steps - left;
  retire_completed(b);
  return LBM_OK;
}

int lbm_batch_last_step_ms(lbm_batch* b, float* ms, long long* lups) {
  if (!b || !ms) return set_error(LBM_ERR_INVALID, "NULL argument");
  CK(cudaEventSynchronize(b->ev1));
  float t = 0;
  CK(cudaEventElapsedTime(&t, b->ev0, b->ev1));
  *ms = b->last_steps > 0 ? t / b->last_steps : 0.0f;
  if (lups) *lups = b->last_lups;
  return LBM_OK;
}

int lbm_batch_poll(lbm_batch* b, int* ids, int max, int* n) {
  if (!b || !n || (max > 0 && !ids)) return set_error(LBM_ERR_INVALID, "NULL argument");
  retire_completed(b);
  int k = 0;
  for (auto& kv : b->members) {
    const lbm_batch::Member& m = kv.second;
    if (m.issued >= m.target && m.done_chunk <= b->chunks_completed &&
        (!m.admitted || cudaEventQuery(m.admitted) == cudaSuccess)) {
      if (k < max) ids[k] = kv.first;
      ++k;
    }
  }
  *n = std::min(k, max);
  return LBM_OK;
}

int lbm_batch_domain(lbm_batch* b, int id, lbm_domain** d) {
  if (!b || !d) return set_error(LBM_ERR_INVALID, "NULL argument");
  auto it = b->members.find(id);
  if (it == b->members.end()) return set_error(LBM_ERR_INVALID, "no member %d", id);
  *d = it->second.d;
  return LBM_OK;
}

int lbm_batch_remove(lbm_batch* b, int id) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  auto it = b->members.find(id);
  if (it == b->members.end()) return set_error(LBM_ERR_INVALID, "no member %d", id);
  CK(cudaSetDevice(b->opt.device));
  // a member still stepping is waited for; a finished one has no work in
  // flight (chunks issued after its last one do not reference it), and
  // anything that reuses its memory is queued behind those chunks
  retire_completed(b);
  if (it->second.issued < it->second.target || it->second.done_chunk > b->chunks_completed)
    CK(cudaStreamSynchronize(b->stream));
  destroy_member(b, it->second);
  b->members.erase(it);
  return LBM_OK;
}

int lbm_batch_fetch(lbm_batch* b, int id, float* den, float* velx, float* vely, float* velz) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  auto it = b->members.find(id);
  if (it == b->members.end()) return set_error(LBM_ERR_INVALID, "no member %d", id);
  const lbm_batch::Member& m = it->second;
  if (m.issued < m.target) return set_error(LBM_ERR_STATE, "member %d has not reached its target", id);
  CK(cudaSetDevice(b->opt.device));
  retire_completed(b);
  if (m.done_chunk > b->chunks_completed) {
    // wait for the member's last chunk only, not for the chunks behind it
    for (auto& ce : b->chunk_events)
      if (ce.first == m.done_chunk) {
        CK(cudaEventSynchronize(ce.second));
        break;
      }
  }
  // the fields exist once the member's initial state has been built (the
  // copies run on the fetch stream, not the batch stream)
  if (m.admitted) CK(cudaStreamWaitEvent(b->fetch, m.admitted, 0));
  lbm_domain* d = m.d;
  const size_t nb = (size_t)d->N * sizeof(float);
  float* outs[4] = {den, velx, vely, velz};
  const float* srcs[4] = {d->den[d->step & 1], d->ux, d->uy, d->uz};
  for (int i = 0; i < 4; ++i)
    if (outs[i]) CK(cudaMemcpyAsync(outs[i], srcs[i], nb, cudaMemcpyDeviceToHost, b->fetch));
  CK(cudaStreamSynchronize(b->fetch));
  return LBM_OK;
}

int lbm_batch_sync(lbm_batch* b) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  CK(cudaSetDevice(b->opt.device));
  CK(cudaStreamSynchronize(b->stream));
  retire_completed(b);
  return LBM_OK;
}

int lbm_batch_usage(lbm_batch* b, size_t* used, size_t* largest_free, int* ndomains) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  if (used) *used = b->pool.used();
  if (largest_free) *largest_free = b->pool.largest_free();
  if (ndomains) *ndomains = (int)b->members.size();
  return LBM_OK;
}

int lbm_batch_autotune(lbm_batch* b, int trial_steps, lbm_batch_options* chosen) {
  if (!b) return set_error(LBM_ERR_INVALID, "NULL batch");
  if (trial_steps <= 0) return set_error(LBM_ERR_INVALID, "trial_steps must be positive");
  // coordinate search: register build x schedule x block at 2 nodes per
  // thread and the flat grids, then (persistent schedules) nodes per thread,
  // then a cap of 2 CTAs per SM
  lbm_batch_options keep = b->opt, best_opt = b->opt;
  float best = 1e30f;
  bool done = false;
  auto trial = [&](const lbm_batch_options& o) -> int {
    b->opt = o;
    int rc = lbm_batch_step(b, trial_steps);
    float ms = 0;
    long long lups = 0;
    if (!rc) rc = lbm_batch_last_step_ms(b, &ms, &lups);
    if (rc) return rc;
    if (lups == 0) {  // nothing left to step
      done = true;
      return LBM_OK;
    }
    const float per_update = ms / (float)lups;
    if (per_update < best) {
      best = per_update;
      best_opt = o;
    }
    return LBM_OK;
  };
  std::vector<lbm_batch_options> stage;
  for (int regs : {0, 1})
    for (int sc : {0, 1})
      for (int blk : {128, 256}) {
        lbm_batch_options o = keep;
        o.regs = regs;
        o.schedule = sc;
        o.block = blk;
        o.nodes_per_thread = 2;
        o.ctas_per_sm = 0;
        stage.push_back(o);
      }
  for (int own : {512, 2048, 8192}) {
    lbm_batch_options o = keep;  // flat grids (launch shape fixed)
    o.schedule = 2;
    o.block = 128;
    o.nodes_per_thread = 2;
    o.regs = 0;
    o.ctas_per_sm = 0;
    o.own_set_ctas = own;
    stage.push_back(o);
  }
  for (int phase = 0; phase < 3 && !done; ++phase) {
    if (phase > 0 && best_opt.schedule == 2) break;  // nothing further to tune
    if (phase == 1) {
      stage.clear();
      for (int np : {1, 4, 8, 16}) {
        lbm_batch_options o = best_opt;
        o.nodes_per_thread = np;
        stage.push_back(o);
      }
    } else if (phase == 2) {
      stage.clear();
      lbm_batch_options o = best_opt;
      o.ctas_per_sm = 2;
      stage.push_back(o);
    }
    for (const lbm_batch_options& o : stage) {
      int rc = trial(o);
      if (rc) {
        b->opt = keep;
        return rc;
      }
      if (done) break;
    }
  }
  if (best >= 1e30f) {
    b->opt = keep;
    if (chosen) *chosen = keep;
    return LBM_OK;
  }
  b->opt = best_opt;
  if (chosen) *chosen = best_opt;
  return LBM_OK;
}

}  // extern "C"
