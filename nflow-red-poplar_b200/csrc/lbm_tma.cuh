// lbm_tma.cuh — the fused step with TMA-staged populations (sm_100a).
//
// Persistent CTAs: one producer warp and CONSUMER_WARPS consumer warps.  A
// tile is TX x TZ nodes of one y plane (x fastest).  For population q of a
// tile the producer issues one cp.async.bulk.tensor.4d load of the box of
// donors x - c_q into a shared-memory stage: the box starts at
// (x0 - HX, z0 - c_z, y - c_y, q) and is TX + 2 HX wide so that every x
// coordinate stays 16-byte aligned (HX = 16 bytes of elements) and the
// c_x = +-1 shifts are read from the halo; coordinates outside the domain
// are zero-filled by the TMA unit and belong to boundary nodes, which take
// the per-node boundary path.  Stages form a ring guarded by mbarriers
// (full: TMA bytes landed; empty: every consumer warp is done with it).
// Consumers take x-pairs, read their 19 populations from shared memory,
// evaluate the node arithmetic on packed FP32 lanes (F2) and store f*
// straight to global memory.  Rows on a y or z face of the box are all
// boundary nodes and their consumers take the per-node boundary path
// uniformly.  In the other rows the x-pairs at the two x faces are left to a
// boundary warp, which runs the per-node path (global loads) for those few
// nodes alongside the consumers instead of making half of the consumer warps
// diverge into it; it reads only the source lattice and writes only its own
// nodes, so it needs no barrier.
//
// The loads never occupy registers or load slots, so the memory
// parallelism is set by the stage count, not by occupancy: this is what
// lets the 16-bit storage formats run at their own bandwidth roofline.
//
// Every mbarrier wait is bounded; a wait that gives up writes a code into
// the domain's error word and the thread stops (the host reports
// LBM_ERR_TIMEOUT at its next synchronising call).  The producer issues
// loads only for stages the consumers will drain, so in normal operation
// the CTA (and its shared memory) outlives every load it issued.
#pragma once
#include <cuda.h>

#include "lbm_kernels.cuh"

namespace lbm {

template <class S>
struct TmaCfg {
  static constexpr int TX = 128;                       // tile nodes along x
  static constexpr int TZ = 8;                         // tile rows along z
  static constexpr int HX = 16 / (int)sizeof(S);       // 16-byte x halo
  static constexpr int TXB = TX + 2 * HX;              // box width
  static constexpr int BOX_BYTES = TXB * TZ * (int)sizeof(S);
  static constexpr int BOX_STRIDE = (BOX_BYTES + 127) / 128 * 128;
  static constexpr int STAGE_BYTES = Q * BOX_STRIDE;
  static constexpr int STAGES = sizeof(S) == 4 ? 2 : 4;
  static constexpr int CONSUMER_WARPS = TX / 2 * TZ / 32;  // one x-pair per thread
  // + one producer warp + one boundary warp
  static constexpr int THREADS = (CONSUMER_WARPS + 2) * 32;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 2 * STAGES * 8 + 128;
  static_assert(BOX_BYTES % 16 == 0, "TMA box row must be a multiple of 16 bytes");
  static_assert(TXB <= 256 && TZ <= 256, "TMA box dimension limit");
  static_assert(TZ * 4 <= 32, "the boundary warp covers 4 x-edge candidates per tile row");
};

// bounded mbarrier waits: try_wait suspends the thread for up to
// kSuspendNs per call (it returns as soon as the phase completes), and
// kWaitIters calls bound a wait to about a second
constexpr int kSuspendNs = 1000;
constexpr int kWaitIters = 1 << 20;
constexpr int kErrProducerWait = 1;
constexpr int kErrConsumerWait = 2;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int iters) {
  for (int i = 0; i < iters; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// a pair of populations from shared memory as packed FP32 (aligned: c_x = 0)
template <class S>
__device__ __forceinline__ F2 lds_pair(const S* p, int q, float inv_scale);
template <>
__device__ __forceinline__ F2 lds_pair<float>(const float* p, int, float) {
  return F2{*reinterpret_cast<const float2*>(p)};
}
template <>
__device__ __forceinline__ F2 lds_pair<__half>(const __half* p, int, float inv_scale) {
  const float2 h = __half22float2(*reinterpret_cast<const __half2*>(p));
  return F2{__fmul2_rn(h, make_float2(inv_scale, inv_scale))};
}
template <>
__device__ __forceinline__ F2 lds_pair<__nv_bfloat16>(const __nv_bfloat16* p, int,
                                                      float inv_scale) {
  const float2 h = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  return F2{__fmul2_rn(h, make_float2(inv_scale, inv_scale))};
}

// stall_tile >= 0 (the wait test of lbm_options.wait_test): the producer
// issues no copy for that tile and stops there, and every wait gives up after
// wait_iters tries; the copies it issued before are all drained by the
// consumers ahead of the withheld tile, so none is in flight when the
// consumers give up and the CTA exits.
template <class S, int COLL, bool LES>
__global__ void __launch_bounds__(TmaCfg<S>::THREADS, 1)
    k_step_tma(const __grid_constant__ StepArgs<S> a, const __grid_constant__ CUtensorMap src_map,
               int* __restrict__ err, int stall_tile, int wait_iters) {
  using C = TmaCfg<S>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // 128-byte aligned stage base, derived by pointer arithmetic on the
  // __shared__ array so that the compiler keeps the shared address space
  unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + C::STAGES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
  const int ntx = (nx + C::TX - 1) / C::TX, nzb = (nz + C::TZ - 1) / C::TZ;
  const int ntiles = ntx * nzb * ny;  // < 2^31 (checked when the domain is created)

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), C::CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  if (warp == C::CONSUMER_WARPS) {
    // ---------------- producer: one elected lane ----------------
    if (lane != 0) return;
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
      const int s = i % C::STAGES;
      const uint32_t ph = (uint32_t)(i / C::STAGES) & 1u;
      if (t == stall_tile) break;  // the wait test: this tile's copies are withheld
      if (!mbar_wait(smem_addr(&empty[s]), ph ^ 1u, wait_iters)) {
        atomicExch(err, kErrProducerWait);
        break;
      }
      const int xt = t % ntx;
      const int rest = t / ntx;
      const int zb = rest % nzb;
      const int y = rest / nzb;
      const int x0 = xt * C::TX, z0 = zb * C::TZ;
      const uint32_t bar = smem_addr(&full[s]);
      mbar_expect_tx(bar, (uint32_t)(Q * C::BOX_BYTES));
      unsigned char* stage = smem + s * C::STAGE_BYTES;
      static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        tma_load_4d(smem_addr(stage + q * C::BOX_STRIDE), &src_map, x0 - C::HX, z0 - cz(q),
                    y - cy(q), q, bar);
      });
    }
    return;
  }

  if (warp == C::CONSUMER_WARPS + 1) {
    // ---------------- boundary warp ----------------
    // lane = 4 * row + candidate; candidates x = 0, 1, nx-2, nx-1 of an
    // interior row, taken when no consumer pair covers them
    const int r = lane >> 2, c = lane & 3;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int xt = t % ntx;
      const int rest = t / ntx;
      const int zb = rest % nzb;
      const int y = rest / nzb;
      const int x0 = xt * C::TX, z = zb * C::TZ + r;
      if (r >= C::TZ || z >= nz || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) continue;
      const int x = c < 2 ? c : nx - 4 + c;
      if (x < x0 || x >= x0 + C::TX || x >= nx || (c >= 2 && x < 2)) continue;
      const int pair = x & ~1;
      if (pair >= 1 && pair + 1 <= nx - 2) continue;  // a consumer's interior pair
      step_node<S, COLL, LES>(a, x, y, z);
    }
    return;
  }

  // ---------------- consumers ----------------
  const int r = threadIdx.x / (C::TX / 2);
  const int xl = 2 * (threadIdx.x % (C::TX / 2));
  int i = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
    const int s = i % C::STAGES;
    const uint32_t ph = (uint32_t)(i / C::STAGES) & 1u;
    if (!mbar_wait(smem_addr(&full[s]), ph, wait_iters)) {
      atomicExch(err, kErrConsumerWait);
      return;
    }
    const int xt = t % ntx;
    const int rest = t / ntx;
    const int zb = rest % nzb;
    const int y = rest / nzb;
    const int x = xt * C::TX + xl, z = zb * C::TZ + r;
    if (x < nx && z < nz) {
      const bool two = x + 1 < nx;
      const bool face_row = y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
      const bool interior = !face_row && x >= 1 && x + 1 <= nx - 2;
      if (interior) {
        const S* stage = reinterpret_cast<const S*>(smem + s * C::STAGE_BYTES);
        const int cell = x + a.g.px * (z + nz * y);
        F2 f[Q];
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          const S* p = stage + q * (C::BOX_STRIDE / (int)sizeof(S)) + r * C::TXB + xl + C::HX -
                       cx(q);
          if constexpr (cx(q) == 0) {
            f[q] = lds_pair<S>(p, q, a.inv_scale);
          } else {
            f[q] = mk2(StoreTraits<S>::load(p, a.inv_scale),
                       StoreTraits<S>::load(p + 1, a.inv_scale));
          }
        });
        PairState<F2> ps;
        make_pairs<F2, kDev<S>>(f, ps);
        F2 ux, uy, uz;
        const F2 inv_rho = velocity<F2>(ps, ux, uy, uz);
        if (a.den_out || a.ux_out || a.g.casetype == CHANNEL) {
          write_macro<S>(a, x, y, z, ps.rho_full.v.x, ux.v.x, uy.v.x, uz.v.x);
          write_macro<S>(a, x + 1, y, z, ps.rho_full.v.y, ux.v.y, uy.v.y, uz.v.y);
        }
        collide_node<S, COLL, LES, true, F2>(f, ps, ux, uy, uz, inv_rho, a, [&](int q, F2 v) {
          st_pair<S>(a.dstq[q] + cell, v, q, a.scale);
        });
      } else if (face_row) {
        // a row of boundary nodes: the per-node path with the boundary rules
        step_node<S, COLL, LES>(a, x, y, z);
        if (two) step_node<S, COLL, LES>(a, x + 1, y, z);
      }
      // else: an x-face pair of an interior row, done by the boundary warp
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
  }
}

}  // namespace lbm
