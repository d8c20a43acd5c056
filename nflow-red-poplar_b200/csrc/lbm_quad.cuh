// lbm_quad.cuh — the 16-bit AA step over quad rows (kRowsQuad).
//
// Quad rows store the 8-byte word w of a row (0 <= w < D, D = px/4) as the
// nodes w, w + 2D, w + D, w + 3D in its four 16-bit slots: the low 32-bit
// half is the paired word (w, w + H) and the high half the paired word
// (w + D, w + D + H), H = px/2.  One thread takes one word, four nodes:
// both AA step kinds then touch every population as one aligned 8-byte
// word per thread (a warp moves 256 contiguous bytes per access), because
// a node one step away in x is one word away for all four nodes.  The node
// arithmetic runs twice, once per half, on F2 lanes (packed FP32) — the
// arithmetic of the paired pull step, which the 16-bit units compile
// without multiply-add contraction, so a node gets the same bits as from
// the per-node AA step over plain rows.
//
// Local step (natural -> swapped): word w of plane q in, word w of plane
// opp q out, all at the node.  Channels: the pending natural slots of the
// inlet (x = 0: slot 0 of word 0) and the outlet (x = nx - 1: slot 3 of word
// D - 1) take their open-face rules first, as in the per-node step.
//
// Neighbour step (swapped -> natural): population q of the four nodes is
// read from word w - c_x of the donor row in plane opp q and written to word
// w + c_x of the destination row in plane q.  The words that differ:
//   - seams: for word 0 with c_x = +1 the nodes x - 1 lie in word D - 1 one
//     slot down (kD - 1 = (D - 1) + (k - 1) D), and node 0's donor is outside
//     the box: the node's own slot (0, q), with the node's wall rule; for
//     word D - 1 with c_x = -1 likewise in word 0 one slot up, node nx - 1's
//     donor outside.  The stores mirror this: word 0 with c_x = -1 writes
//     three slots of word D - 1 (one 32-bit and one 16-bit store) and node
//     0's value into its own slot (0, opp q); word D - 1 with c_x = +1 writes
//     three slots of word 0 and node nx - 1's own slot.  Only these two
//     threads of a row branch, and only for the five populations with that
//     c_x.  Slot ownership makes the split stores race-free: in a neighbour
//     step every slot is read and written by one node only (x - c_p for slot
//     (x, p), or the node itself when that lies outside), so the slots of
//     word D - 1 that thread 0 writes are disjoint from the one that thread
//     D - 1 writes, and every whole-word store covers slots of its own four
//     nodes only (px == nx: no padding nodes).
//   - rows on a y or z face: a population whose donor row is outside reads
//     the node's own word of plane q and takes each node's wall rule; one
//     whose destination row is outside writes the node's own word of plane
//     opp q with each node's wall value (aa_wall).  The test is uniform along
//     the row.
// No word is read outside its plane's rows: a seam word is addressed in its
// own row, never one word past the row.
#pragma once
#include <type_traits>

#include "lbm_kernels.cuh"

namespace lbm {

// the word AA step applies to the domain's geometry (quad rows, no STRUCT
// nodes, px == nx: no padding nodes)
__host__ __device__ __forceinline__ bool aa_words_apply(const Geometry& g) {
  return g.rows == kRowsQuad && !has_struct(g) && g.px == g.nx && g.nx >= 16;
}

__device__ __forceinline__ uint2 ld_w8(const void* p) {
  return *reinterpret_cast<const uint2*>(p);
}
__device__ __forceinline__ void st_w8(void* p, uint2 v) { *reinterpret_cast<uint2*>(p) = v; }
__device__ __forceinline__ void st_w4(void* p, uint32_t v) {
  *reinterpret_cast<uint32_t*>(p) = v;
}
__device__ __forceinline__ void st_w2(void* p, uint32_t v) {
  *reinterpret_cast<unsigned short*>(p) = (unsigned short)v;
}

// Resident threads per SM the register budgets are sized for: the quad step
// (two F2 halves per thread, 128 registers) and the paired AA step (one F2
// half, 64 registers).
#ifndef LBM_QUAD_THREADS_PER_SM
#define LBM_QUAD_THREADS_PER_SM 512
#endif
#ifndef LBM_AA_PAIRED_THREADS_PER_SM
#define LBM_AA_PAIRED_THREADS_PER_SM 1024
#endif

// index of population q (c_x = +-1) among the five with its c_x
__host__ __device__ constexpr int xface_index(int q) {
  int j = 0;
  for (int p = 1; p < q; ++p) j += cx(p) == cx(q);
  return j;
}

// Channels on quad rows: after every AA step, the inlet / outlet values
// that the next step takes for the populations whose donor lies outside the
// box at the x faces of the interior rows: at x = 0 (inlet) the five with
// c_x = +1, at x = nx - 1 (outlet) the five with c_x = -1.  In both AA
// layouts the node's own slot (x, q) then holds f*_{opp q} (a pending
// natural slot after a neighbour step, the own slot after a local step), and
// the value is boundary_value of the node with the face planes the step
// just wrote: a = the next step's arguments.  The step kernels read the
// five values instead of evaluating the rule (FP64 arithmetic that only
// two threads of a row would run): the same FP32 values, so the same bits.
// grid = ceil(2 (ny - 2)(nz - 2) / 128) blocks of 128.
template <class S>
__global__ void __launch_bounds__(128) k_aa_xface_rules(const __grid_constant__ StepArgs<S> a,
                                                        float* __restrict__ out) {
  const int ni = (a.g.ny - 2) * (a.g.nz - 2);
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= 2 * ni) return;
  const int face = i >= ni, r = face ? i - ni : i;
  const int y = 1 + r / (a.g.nz - 2), z = 1 + r % (a.g.nz - 2);
  const int x = face ? a.g.nx - 1 : 0;
  const int P = a.g.ny * a.g.nz, yz = y * a.g.nz + z;
  const int t = node_type(a.g, x, y, z);
  const int cell = cell_of(a.g, x, y, z);
  static_for<1, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    if constexpr (cx(q) != 0) {
      if ((cx(q) == 1) == (face == 0)) {
        const RealOf<S> fo = ld(a.srcq[q] + cell, q, a.inv_scale);
        out[(face * 5 + xface_index(q)) * P + yz] = (float)boundary_value<S, q>(a, t, fo, y, z);
      }
    }
  });
}

// The wall rule of boundary_value (fixed wall: the value itself; moving
// wall: minus the lid term) for population q at a wall node of type t.
template <class S, int q>
__device__ __forceinline__ RealOf<S> wall_value(const StepArgs<S>& a, int t, RealOf<S> fo) {
  using R = RealOf<S>;
  if (t != NODE_MOVINGWALL) return fo;
  constexpr int d = opp(q);
  R eu = add_rn(add_rn(mul_rn(R(cx(d)), a.ulx), mul_rn(R(cy(d)), a.uly)), mul_rn(R(cz(d)), a.ulz));
  R term = mul_rn(mul_rn(mul_rn(R(6), weight<R>(d)), a.rho0), eu);
  return sub_rn(fo, term);
}

// a word of NH 32-bit halves (NH = 1: paired rows, 2: quad rows)
template <int NH>
using WordOf = typename std::conditional<NH == 1, uint32_t, uint2>::type;
template <int h>
__device__ __forceinline__ uint32_t& half_of(uint32_t& w) {
  return w;
}
template <int h>
__device__ __forceinline__ uint32_t& half_of(uint2& w) {
  return h ? w.y : w.x;
}
__device__ __forceinline__ uint32_t ld_word(const void* p, uint32_t*) {
  return *reinterpret_cast<const uint32_t*>(p);
}
__device__ __forceinline__ uint2 ld_word(const void* p, uint2*) { return ld_w8(p); }
__device__ __forceinline__ void st_word(void* p, uint32_t v) { st_w4(p, v); }
__device__ __forceinline__ void st_word(void* p, uint2 v) { st_w8(p, v); }

// One AA step (NB = 0 local, 1 neighbour) of the 2 NH nodes of word w of
// row (y, z), in paired rows (NH = 1: word w holds the nodes w, w + H) or
// quad rows (NH = 2: see above).  Slot tables as for the per-node AA step
// (aa_args with a.off[q] = 2 NH c_x + px (c_z + nz c_y)): local srcd[q] =
// plane q, dstq[q] = plane opp q; neighbour srcd[q] = plane opp q - off_q,
// dstq[q] = plane q + off_q; srcq[q] = plane q.  entry (local steps):
// kAAPending or kAAComplete (the first step after the initial state is the
// per-node step's).  In paired rows the seams are those of the pull step:
// node H - 1 (lo of word H - 1) and node H (hi of word 0) are x neighbours,
// node 0 is the lo of word 0 and node nx - 1 the hi of word H - 1.
// FACE (neighbour step): the row lies on a y or z face, so that some
// populations' donor or destination rows are outside the box; the rows off
// the faces are stepped by a launch without that code (FACE = false), the
// face rows by their own launch (k_aa_face_rows), which keeps each kernel's
// code short.
template <class S, int COLL, bool LES, bool SR, int NB, int NH, bool FACE>
__device__ __forceinline__ void aa_word(const StepArgs<S>& a, int w, int y, int z, int entry) {
  static_assert(kDev<S>, "paired and quad rows are 16-bit layouts");
  static_assert(NB || !FACE, "face rows matter to the neighbour step only");
  using W = WordOf<NH>;
  const int H = a.g.px >> 1, D = a.g.px >> 2;
  const int NW = a.g.px / (2 * NH);                    // words per row
  const int e = 2 * NH * w + a.g.px * (z + a.g.nz * y);  // slot 0 of the word
  const bool seam_lo = w == 0, seam_hi = w == NW - 1;
  // donor / destination row of population q inside the box (rows off a
  // face: always)
  auto row_in = [&](int dy, int dz) {
    if constexpr (!FACE) return true;
    return (unsigned)(y + dy) < (unsigned)a.g.ny && (unsigned)(z + dz) < (unsigned)a.g.nz;
  };
  W v[Q];
  if constexpr (!NB) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      v[q] = ld_word(a.srcd[q] + e, (W*)nullptr);
    });
  } else {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      if (row_in(-cy(q), -cz(q))) {
        // the donor word w - c_x, or across the seam the word at the other
        // end of the same donor row (px elements away)
        int adj = 0;
        if constexpr (cx(q) == 1) adj = seam_lo ? a.g.px : 0;
        if constexpr (cx(q) == -1) adj = seam_hi ? -a.g.px : 0;
        v[q] = ld_word(a.srcd[q] + (e + adj), (W*)nullptr);
      } else {
        v[q] = ld_word(a.srcq[q] + e, (W*)nullptr);  // own slots (x, q): f*_{opp q}
      }
    });
    if (seam_lo || seam_hi) {
      static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        if constexpr (cx(q) != 0) {
          if (((cx(q) == 1 && seam_lo) || (cx(q) == -1 && seam_hi)) &&
              row_in(-cy(q), -cz(q))) {
            const W X = v[q];
            const W own = ld_word(a.srcq[q] + e, (W*)nullptr);
            if constexpr (NH == 1) {
              if constexpr (cx(q) == 1)
                v[q] = __byte_perm(own, X, 0x5410);  // (own lo, node H - 1)
              else
                v[q] = __byte_perm(X, own, 0x7632);  // (node H, own hi)
            } else {
              if constexpr (cx(q) == 1) {
                // quarters (own k0, X k0, X k1, X k2) in slot order k0 k2 | k1 k3
                v[q].x = __byte_perm(own.x, X.y, 0x5410);
                v[q].y = X.x;
              } else {
                // quarters (X k1, X k2, X k3, own k3)
                v[q].x = X.y;
                v[q].y = __byte_perm(X.x, own.y, 0x7632);
              }
            }
          }
        }
      });
    }
  }
  if constexpr (SR) bump_step_counter<SR>(a);
  const uint32_t kstep = SR ? a.kctr[a.kpar] : 0u;
  // store of population q's word of results (slot order)
  auto store = [&](auto qc, W r) {
    constexpr int q = decltype(qc)::value;
    if constexpr (!NB) {
      st_word(a.dstq[q] + e, r);
    } else {
      if (!row_in(cy(q), cz(q))) {
        st_word(a.dst + (opp(q) * a.qs + e), r);  // own slots (x, opp q)
      } else if (cx(q) == -1 && seam_lo) {
        // the word across the seam is the last one of the destination row
        S* wd = a.dstq[q] + (e + a.g.px);
        if constexpr (NH == 1) {
          st_w2(wd, r >> 16);                               // node H -> H - 1
          st_w2(a.dst + (opp(q) * a.qs + e), r & 0xffffu);  // node 0: own slot
        } else {
          // its slots k0 k2 k1 <- results k1 k3 k2; quarter 0 (x = 0) to
          // its own slot
          st_w4(wd, r.y);
          st_w2(wd + 2, r.x >> 16);
          st_w2(a.dst + (opp(q) * a.qs + e), r.x & 0xffffu);
        }
      } else if (cx(q) == 1 && seam_hi) {
        // the word across the seam is the first one of the destination row
        S* wd = a.dstq[q] + (e - a.g.px);
        if constexpr (NH == 1) {
          st_w2(wd + 1, r & 0xffffu);                           // node H - 1 -> H
          st_w2(a.dst + (opp(q) * a.qs + e + 1), r >> 16);      // node nx - 1: own slot
        } else {
          // its slots k2 k1 k3 <- results k0 k1 k2; quarter 3 (x = nx - 1)
          // to its own slot
          st_w4(wd + 2, r.x);
          st_w2(wd + 1, r.y & 0xffffu);
          st_w2(a.dst + (opp(q) * a.qs + e + 3), r.y >> 16);
        }
      } else {
        st_word(a.dstq[q] + e, r);
      }
    }
  };
  // channels: the x-face lanes of this word take the values of
  // k_aa_xface_rules (node 0: lo lane of half 0 of word 0, c_x = +1
  // populations; node nx - 1: hi lane of the last half of the last word,
  // c_x = -1 populations)
  auto xface_lanes = [&](F2 (&f)[Q], int hb) {
    const int P = a.g.ny * a.g.nz, yz = y * a.g.nz + z;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      if constexpr (cx(q) == 1) {
        if (hb == 0 && seam_lo) f[q].v.x = a.xrule[xface_index(q) * P + yz];
      } else if constexpr (cx(q) == -1) {
        if (hb == NH - 1 && seam_hi) f[q].v.y = a.xrule[(5 + xface_index(q)) * P + yz];
      }
    });
  };
  // the halves, each a compile-time pass: half hb holds the nodes
  // (w + hb D, w + hb D + H); every pass but the last leaves its packed
  // results in its half of v[q], the last stores each population's word as
  // soon as its result is known
  auto pass = [&](auto hbc) {
    constexpr int hb = decltype(hbc)::value;
    const int xlo = w + hb * D, xhi = xlo + H;
    F2 f[Q];
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = unpack_pair<S>(half_of<hb>(v[q]), a.inv_scale);
    });
    [[maybe_unused]] int tlo = NODE_FLUID, thi = NODE_FLUID;
    if constexpr (NB) {
      // boundary rules of the donors outside the box.  Face rows: each
      // node's wall rule (rows on a y or z face hold walls only: the lid,
      // and fixed walls, which a channel's side faces keep over its inlet
      // and outlet; their x faces are fixed walls, whose rule is the value
      // itself).  Rows off the faces: the x faces (node 0, the lo lane of
      // the first half of word 0; node nx - 1, the hi lane of the last half
      // of the last word), whose rule is the value itself for the cavity's
      // fixed walls and, for the channel's inlet and outlet, the value
      // k_aa_xface_rules left for this step.
      if constexpr (FACE) {
        tlo = node_type(a.g, xlo, y, z);
        thi = node_type(a.g, xhi, y, z);
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          if (!row_in(-cy(q), -cz(q))) {
            f[q].v.x = wall_value<S, q>(a, tlo, f[q].v.x);
            f[q].v.y = wall_value<S, q>(a, thi, f[q].v.y);
          }
        });
      } else if (a.xrule && (seam_lo || seam_hi)) {
        xface_lanes(f, hb);
      }
    } else {
      // pending natural slots of the channel's inlet and outlet nodes: the
      // values k_aa_xface_rules left for this step
      if (entry == kAAPending && a.xrule && y > 0 && y < a.g.ny - 1 && z > 0 &&
          z < a.g.nz - 1 && (seam_lo || seam_hi))
        xface_lanes(f, hb);
    }
    PairState<F2> ps;
    make_pairs<F2, true>(f, ps);
    F2 ux, uy, uz;
    const F2 inv_rho = velocity<F2>(ps, ux, uy, uz);
    if (a.den_out || a.ux_out || a.g.casetype == CHANNEL) {
      write_macro<S>(a, xlo, y, z, ps.rho_full.v.x, ux.v.x, uy.v.x, uz.v.x);
      write_macro<S>(a, xhi, y, z, ps.rho_full.v.y, ux.v.y, uy.v.y, uz.v.y);
    }
    [[maybe_unused]] uint32_t h = 0u;
    if constexpr (SR) h = sr_hash((uint32_t)(xlo + H * (z + a.g.nz * y)), kstep, a.sr_seed);
    collide_node<S, COLL, LES, true, F2>(f, ps, ux, uy, uz, inv_rho, a, [&](auto qc, F2 r) {
      constexpr int q = decltype(qc)::value;
      if constexpr (FACE) {
        if (!row_in(cy(q), cz(q))) {
          // destination row outside: the wall value into the node's own slot
          r.v.x = aa_wall<S>(a, tlo, r.v.x, q);
          r.v.y = aa_wall<S>(a, thi, r.v.y, q);
        }
      }
      uint32_t p;
      if constexpr (SR)
        p = pack_pair_sr<S>(r, a.scale, sr_bits<q>(h));
      else
        p = pack_pair<S>(r, a.scale);
      if constexpr (hb < NH - 1) {
        half_of<hb>(v[q]) = p;
      } else {
        W out = v[q];
        half_of<hb>(out) = p;
        store(qc, out);
      }
    });
  };
  pass(std::integral_constant<int, 0>{});
  if constexpr (NH == 2) pass(std::integral_constant<int, 1>{});
}

// number of rows on a y or z face: 2 nz at y = 0 and y = ny - 1, then
// 2 (ny - 2) at z = 0 and z = nz - 1
__host__ __device__ __forceinline__ int aa_face_rows(const Geometry& g) {
  return 2 * g.nz + 2 * (g.ny - 2);
}

// Local step: grid = (ceil(NW / b), nz, ny), every row.  Neighbour step:
// grid = (ceil(NW / b), nz - 2, ny - 2 + FZ), FZ = ceil(aa_face_rows /
// (nz - 2)): the rows off the y and z faces, then the face rows in the
// trailing CTAs (a CTA-uniform branch into the code with the face rules,
// so the hot code of the interior rows stays short and the face rows fill
// the grid's tail).  NW = px / (2 NH) words per row, b = NW rounded up to a
// multiple of 32 and at most 128 threads, one word per thread.  In the
// neighbour step the two seam words of a row (0 and NW - 1) are taken by
// the row's first two threads, so only the row's first warp diverges into
// the seam code.
template <class S, int COLL, bool LES, bool SR, int NB, int NH>
__global__ void __launch_bounds__(128, (NH == 2 ? LBM_QUAD_THREADS_PER_SM
                                                : LBM_AA_PAIRED_THREADS_PER_SM) / 128)
    k_aa_words(const __grid_constant__ StepArgs<S> a, int entry) {
  const int NW = a.g.px / (2 * NH);
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= NW) return;
  if constexpr (!NB) {
    aa_word<S, COLL, LES, SR, 0, NH, false>(a, t, blockIdx.z, blockIdx.y, entry);  // y, z
  } else {
    const int w = t == 0 ? 0 : (t == 1 ? NW - 1 : t - 1);
    if ((int)blockIdx.z < a.g.ny - 2) {
      aa_word<S, COLL, LES, SR, 1, NH, false>(a, w, blockIdx.z + 1, blockIdx.y + 1, entry);
    } else {
      const int r = ((int)blockIdx.z - (a.g.ny - 2)) * (a.g.nz - 2) + (int)blockIdx.y;
      if (r >= aa_face_rows(a.g)) return;
      int y, z;
      if (r < 2 * a.g.nz) {
        y = r < a.g.nz ? 0 : a.g.ny - 1;
        z = r % a.g.nz;
      } else {
        const int r2 = r - 2 * a.g.nz;
        z = r2 < a.g.ny - 2 ? 0 : a.g.nz - 1;
        y = 1 + r2 % (a.g.ny - 2);
      }
      aa_word<S, COLL, LES, SR, 1, NH, true>(a, w, y, z, entry);
    }
  }
}

}  // namespace lbm
