// lbm_kernels.cuh — device kernels of the fused D3Q19 step.
//
// Storage: populations are SoA, pop[q * qstride + x + px*(z + nz*y)]
// (axis order [y][z][x] as the reference, x fastest, x pitch px padded to a
// multiple of 8 elements so every row starts 16-byte aligned).  Two
// lattices A/B: the kernel of step k pulls the post-collision populations
// f*_{k-1} from one lattice and writes f*_k into the other.
//
// One step = one launch of k_step, which per node
//   1. pulls f_k[q](x) = f*_{k-1}[q](x - c_q)              (Streaming,
//      lbm_codelets.cpp:57-76: arF[opp d](x) = arFTemp[opp d](x + c_d));
//   2. replaces every population whose donor x - c_q lies outside the
//      domain by the boundary rule of the node (BoundaryCavity
//      lbm_codelets.cpp:373-395, keBoundaryInlet kernel.cu:591-611,
//      keBoundaryOutlet kernel.cu:639-655), reading f*_{k-1} of the node
//      itself — the same values the reference reads from arFTemp;
//   3. forms rho, u (Macroscopic, lbm_codelets.cpp:287-312);
//   4. forms tau_eddy (ComputeTurbulence_LES) and collides (Collision_MRT
//      or keCollision_SRT) in registers, and stores f*_k.
// So one step reads 19 and writes 19 populations per node: the HBM
// roofline of 2*19*sizeof(storage) bytes per lattice update.
//
// The reference's step order LES -> collide -> stream -> BC -> macro is the
// same computation with the kernel boundary moved: what the reference holds
// in arF between steps (post-stream) is here reconstructed on demand from
// the other lattice (k_export), what it holds in arFTemp (post-collision)
// is the lattice this kernel writes.
#pragma once
#include <cstring>

#include "lbm_d3q19.cuh"
#include "../../include/lbm_b200.h"

namespace lbm {

template <class S>
using RealOf = typename StoreTraits<S>::R;
// the node arithmetic of storage S works on deviations g = f - w
template <class S>
constexpr bool kDev = StoreTraits<S>::dev;

// The collision of the 16-bit forms rebuilds f*_a, f*_abar from the pair
// sums (FROM_PAIRS in collide_node), in the per-node kernels as in the
// two-node kernels, so that a node gets the same bits from either.
template <class S>
constexpr bool kFromPairs = StoreTraits<S>::dev;

// internal value of population q from the population f, and back
template <class S, int q>
__device__ __forceinline__ RealOf<S> to_internal(RealOf<S> f) {
  if constexpr (kDev<S>) return f - weight<RealOf<S>>(q);
  else return f;
}
template <class S, int q>
__device__ __forceinline__ RealOf<S> to_population(RealOf<S> v) {
  if constexpr (kDev<S>) return v + weight<RealOf<S>>(q);
  else return v;
}

// round-to-nearest primitives that the compiler may not contract into FMA;
// used where the reference's own rounding sequence is reproduced
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Row layouts of the population planes (Geometry::rows).
//   kRowsPlain:  element x of a row holds node x.
//   kRowsPaired: 16-bit storage.  Element 2w of a row holds node w and
//                element 2w + 1 node w + px/2, so that the 32-bit word w
//                holds the node pair (w, w + px/2) and a donor one node away
//                in x is one word away for both nodes of the pair
//                (k_step_paired; AA form: k_aa_words).
//   kRowsQuad:   16-bit storage, AA form (px == nx, a multiple of 8).  With
//                D = px/4, the 8-byte word w of a row holds the nodes
//                w, w + 2D, w + D, w + 3D in its four 16-bit slots, so that
//                its low half is the paired word (w, w + px/2) and its high
//                half the paired word (w + D, w + D + px/2); a node one step
//                away in x is one word away for all four nodes (k_aa_words).
enum { kRowsPlain = 0, kRowsPaired = 1, kRowsQuad = 2 };

struct Geometry {
  int nx, ny, nz, px;
  int casetype;
  int rows;                    // kRows*
  const unsigned char* solid;  // [ny][nz][nx], nonzero = STRUCT; may be null
};

// element of node x within its row (any row layout)
__host__ __device__ __forceinline__ int row_slot(int x, int px, int rows) {
  if (rows == kRowsPlain) return x;
  if (rows == kRowsPaired) {
    const int h = px >> 1;
    return x < h ? 2 * x : 2 * (x - h) + 1;
  }
  const int d = px >> 2;
  const int k = x / d, w = x - k * d;  // quarter k of the row, word w
  return 4 * w + ((k & 1) << 1) + (k >> 1);
}
// in-plane element index of node (x, y, z)
__host__ __device__ __forceinline__ int cell_of(const Geometry& g, int x, int y, int z) {
  return row_slot(x, g.px, g.rows) + g.px * (z + g.nz * y);
}
// elements between x neighbours of a row layout
__host__ __device__ __forceinline__ int row_step(int rows) {
  return rows == kRowsPlain ? 1 : (rows == kRowsPaired ? 2 : 4);
}

// the geometry holds STRUCT nodes: POISEUILLE, or any case with a solid mask
__host__ __device__ __forceinline__ bool has_struct(const Geometry& g) {
  return g.casetype == POISEUILLE || g.solid != nullptr;
}

// node type of keSetNodeType (kernel.cu:1061-1097) / the Initialize codelet
// (lbm_codelets.cpp:183-201): CAVITY walls and lid; POISEUILLE inlet x=0,
// outlet x=nx-1, STRUCT outside the circle of radius 20 about (y,z)=(25,25);
// CHANNEL: inlet x=0, outlet x=nx-1, the four side faces are fixed walls and
// override inlet/outlet.  A solid mask makes its nodes STRUCT in any case.
__device__ __forceinline__ int node_type(const Geometry& g, int x, int y, int z) {
  if (g.solid && g.solid[x + (long long)g.nx * (z + (long long)g.nz * y)]) return NODE_STRUCT;
  int t = NODE_FLUID;
  if (g.casetype == CAVITY) {
    if (y == 0) t = NODE_FIXEDWALL;
    if (y == g.ny - 1) t = NODE_MOVINGWALL;
    if (x == 0 || x == g.nx - 1 || z == 0 || z == g.nz - 1) t = NODE_FIXEDWALL;
  } else if (g.casetype == POISEUILLE) {
    if (x == 0) t = NODE_INLET;
    if (x == g.nx - 1) t = NODE_OUTLET;
    if ((y - 25) * (y - 25) + (z - 25) * (z - 25) > 400) t = NODE_STRUCT;
  } else {  // CHANNEL
    if (x == 0) t = NODE_INLET;
    if (x == g.nx - 1) t = NODE_OUTLET;
    if (y == 0 || y == g.ny - 1 || z == 0 || z == g.nz - 1) t = NODE_FIXEDWALL;
  }
  return t;
}

// 19-bit inside mask of keInitialNodeDirection (kernel.cu:1027-1043):
// bit q set iff x + c_q lies inside the domain; bit 0 always set.
__device__ __forceinline__ int direction_state(const Geometry& g, int x, int y, int z) {
  int ds = 1;
  static_for<1, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int x1 = x + cx(q), y1 = y + cy(q), z1 = z + cz(q);
    if (x1 >= 0 && x1 < g.nx && y1 >= 0 && y1 < g.ny && z1 >= 0 && z1 < g.nz) ds |= 1 << q;
  });
  return ds;
}

template <class S>
struct StepArgs {
  using R = RealOf<S>;
  const S* __restrict__ src;  // f*_{k-1}
  S* __restrict__ dst;        // f*_k
  long long qs;               // population stride (elements)
  // hot-path addressing: plane of population q and the in-plane offset
  // c_x + c_z px + c_y px nz of its donor; node indices inside a plane are
  // 32-bit (px*nz*ny < 2^31 is checked when the domain is created)
  const S* srcq[Q];            // plane of population q
  const S* srcd[Q];            // srcq[q] - off[q]: the donor of a node is srcd[q][cell]
  S* dstq[Q];
  int off[Q];
  Geometry g;
  R tau, les_c, rho0;
  R ulx, uly, ulz;            // lid velocity (cavity)
  MrtParams<R> mp;
  float scale, inv_scale;     // shifted 16-bit storage
  const float* inlet_u;       // [ny*nz] channel inlet profile u_x(y,z)
  const float* prho_in;       // rho_{k-1} at x = 1        [ny*nz]
  float* prho_out;            // rho_k at x = 1
  const float* pu_in;         // u_{k-1} at x = nx-1, nx-2  [2][3][ny*nz]
  float* pu_out;              // u_k
  float* den_out;             // optional macroscopic outputs of arF_k
  float* ux_out;
  float* uy_out;
  float* uz_out;
  // initial condition (POISEUILLE: populations no rule ever writes keep
  // their initial value, as in the reference)
  int init_kind;
  float noise_amp;
  unsigned long long seed;
  // batched kernel: 0 pull step, 1 AA local step, 2 AA neighbour step
  int aa_step;
  // stochastic rounding of the 16-bit stores (paired kernel): step counter
  // pair (the step reads kctr[kpar], writes kctr[kpar ^ 1]) and seed
  unsigned* kctr;
  int kpar;
  int sr;
  unsigned sr_seed;
  // channel on quad rows: the inlet / outlet values this step takes for the
  // populations whose donor lies outside the box at x = 0 (c_x = +1) and
  // x = nx - 1 (c_x = -1), [2][5][ny*nz], computed after the step before
  // (k_aa_xface_rules)
  const float* xrule;
};

// internal value of a stored population
template <class S>
__device__ __forceinline__ RealOf<S> ld(const S* p, int, float inv_scale) {
  return StoreTraits<S>::load(p, inv_scale);
}

// Where the populations of a node live (cell = in-plane index of the node)
// and the storage scales of the shifted 16-bit forms (g = h * inv_scale on
// load, h = g * scale on store).  PlaneAddr takes the per-population plane pointers and
// scales of StepArgs, wherever the arguments are held: in the kernel
// parameter space (single-domain kernels) every pointer is a free operand;
// in shared memory (the batched kernel) each is one broadcast load, issued
// next to its use, so no per-population offset stays live in registers.
template <class S>
struct PlaneAddr {
  const StepArgs<S>& a;
  int cell;
  __device__ __forceinline__ PlaneAddr(const StepArgs<S>& args, int c) : a(args), cell(c) {}
  __device__ __forceinline__ const S* donor(int q) const { return a.srcd[q] + cell; }
  __device__ __forceinline__ const S* own(int q) const { return a.srcq[q] + cell; }
  __device__ __forceinline__ S* out(int q) const { return a.dstq[q] + cell; }
  __device__ __forceinline__ float inv_scale() const { return a.inv_scale; }
  __device__ __forceinline__ float scale() const { return a.scale; }
};

// The same per-node addressing for any row layout (a.g.rows): the
// donor x - c_q of population q is addressed through its own row slot.
// Used by the per-node kernels of paired domains (edge words, initial
// state, import, export); a donor outside the box is never formed.
template <class S>
struct RowAddr {
  const StepArgs<S>& a;
  int x, y, z;
  __device__ __forceinline__ RowAddr(const StepArgs<S>& args, int x_, int y_, int z_)
      : a(args), x(x_), y(y_), z(z_) {}
  __device__ __forceinline__ const S* donor(int q) const {
    return a.srcq[q] + cell_of(a.g, x - cx(q), y - cy(q), z - cz(q));
  }
  __device__ __forceinline__ const S* own(int q) const { return a.srcq[q] + cell_of(a.g, x, y, z); }
  __device__ __forceinline__ S* out(int q) const { return a.dstq[q] + cell_of(a.g, x, y, z); }
  __device__ __forceinline__ float inv_scale() const { return a.inv_scale; }
  __device__ __forceinline__ float scale() const { return a.scale; }
};

// Boundary value of population q at a node whose donor x - c_q is outside
// the domain.  d = opp(q) is the reference's "outside" direction; fo is
// f*_{k-1}[d] at the node itself (arFTemp[d](x) in the reference).
template <class S, int q>
__device__ __forceinline__ RealOf<S> boundary_value(const StepArgs<S>& a, int t, RealOf<S> fo,
                                                    int y, int z) {
  using R = RealOf<S>;
  constexpr int d = opp(q);
  if (t == NODE_FIXEDWALL) return fo;
  if (t == NODE_MOVINGWALL) {
    // BoundaryCavity: arF[opp d] = ftemp[d] - 6 w_d RefDen (c_d . u_lid)
    R eu = add_rn(add_rn(mul_rn(R(cx(d)), a.ulx), mul_rn(R(cy(d)), a.uly)),
                  mul_rn(R(cz(d)), a.ulz));
    R term = mul_rn(mul_rn(mul_rn(R(6), weight<R>(d)), a.rho0), eu);
    return sub_rn(fo, term);
  }
  const int yz = y * a.g.nz + z;
  if (t == NODE_INLET) {
    // keBoundaryInlet: ftemp[d] - 6.0 w_d rho(x+1) (c_d . u_in), FP64 literal;
    // u_in = RefVel (POISEUILLE) or the parabolic profile (CHANNEL)
    R eu;
    if (a.g.casetype == CHANNEL) {
      eu = mul_rn(R(cx(d)), R(a.inlet_u[yz]));
    } else {
      eu = add_rn(add_rn(mul_rn(R(cx(d)), a.ulx), mul_rn(R(cy(d)), a.uly)),
                  mul_rn(R(cz(d)), a.ulz));
    }
    const double v = (double)fo - 6.0 * (double)weight<R>(d) * (double)a.prho_in[yz] * (double)eu;
    return R(v);
  }
  if (t == NODE_OUTLET) {
    // keBoundaryOutlet: anti-bounce-back at RefDen with u extrapolated
    // from the node and its inner neighbour of the previous step
    const int P = a.g.ny * a.g.nz;
    const float* u0 = a.pu_in;          // x = nx-1
    const float* u1 = a.pu_in + 3 * P;  // x = nx-2
    const R bx = R((double)u0[yz] + 0.5 * (double)(u0[yz] - u1[yz]));
    const R by = R((double)u0[P + yz] + 0.5 * (double)(u0[P + yz] - u1[P + yz]));
    const R bz = R((double)u0[2 * P + yz] + 0.5 * (double)(u0[2 * P + yz] - u1[2 * P + yz]));
    const R usq = bx * bx + by * by + bz * bz;
    const R eu = R(cx(d)) * bx + R(cy(d)) * by + R(cz(d)) * bz;
    const double v = -(double)fo + 2.0 * (double)weight<R>(d) * (double)a.rho0 *
                                       (1.0 + 4.5 * ((double)eu * (double)eu) - 1.5 * (double)usq);
    // deviations: g_q = f_q - w = -(g_d + w) + X - w (w_q = w_d)
    if constexpr (kDev<S>) return R(v - 2.0 * (double)weight<R>(d));
    return R(v);
  }
  return fo;  // no rule for this node type: plain bounce-back
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// uniform in [-1, 1) from 24 hash bits; exact in double on any IEEE machine
__device__ __forceinline__ double unit_noise(uint64_t seed, uint64_t node, uint64_t comp) {
  const uint64_t r = splitmix64(seed * 0x9E3779B97F4A7C15ull + node * 4ull + comp);
  return __dadd_rn(__dmul_rn(__dmul_rn((double)(r >> 40), 1.0 / 16777216.0), 2.0), -1.0);
}

// Initial density / velocity of a node (Initialize codelet,
// lbm_codelets.cpp:207-235, plus the seeded perturbations of LBM_INIT_*).
struct InitState {
  float den, ux, uy, uz;
};
__device__ __forceinline__ InitState initial_state(const Geometry& g, int kind, uint64_t seed,
                                                   float amp, float rho0, float ulx, float uly,
                                                   float ulz, const float* inlet_u, int x, int y,
                                                   int z, int t) {
  const long long n = x + (long long)g.nx * (z + (long long)g.nz * y);
  InitState s{rho0, 0.f, 0.f, 0.f};
  if (t == NODE_MOVINGWALL) {
    s.ux = ulx;
    s.uy = uly;
    s.uz = ulz;
  }
  // separately rounded products and sums (no FMA), as in the CPU oracle
  if (kind == LBM_INIT_DENSITY_NOISE) {
    s.den = (float)__dadd_rn((double)rho0, __dmul_rn((double)amp, unit_noise(seed, (uint64_t)n, 0)));
  } else if (kind == LBM_INIT_CHANNEL &&
             (t == NODE_FLUID || t == NODE_INLET || t == NODE_OUTLET)) {
    const double au = __dmul_rn((double)amp, (double)ulx);
    const float prof = g.casetype == CHANNEL ? inlet_u[y * g.nz + z] : 0.0f;
    s.ux = (float)__dadd_rn((double)prof, __dmul_rn(au, unit_noise(seed, (uint64_t)n, 0)));
    s.uy = (float)__dmul_rn(au, unit_noise(seed, (uint64_t)n, 1));
    s.uz = (float)__dmul_rn(au, unit_noise(seed, (uint64_t)n, 2));
  }
  return s;
}

// feq of lbm_codelets.cpp:225-230 in the codelet's rounding order
template <class R, int q>
__device__ __forceinline__ R initial_feq(R rd, R ux, R uy, R uz) {
  const R eu = add_rn(add_rn(mul_rn(R(cx(q)), ux), mul_rn(R(cy(q)), uy)), mul_rn(R(cz(q)), uz));
  const R usq = add_rn(add_rn(mul_rn(ux, ux), mul_rn(uy, uy)), mul_rn(uz, uz));
  const R br = sub_rn(add_rn(add_rn(R(1), mul_rn(R(3), eu)), mul_rn(mul_rn(R(4.5), eu), eu)),
                      mul_rn(R(1.5), usq));
  return mul_rn(mul_rn(weight<R>(q), rd), br);
}

// Streaming + boundaries with STRUCT nodes (kernel.cu:489-516, 659-697,
// 566-657): a donor that is STRUCT does not stream (keStreaming skips it); a
// FLUID node takes half-way bounce-back from its own f*_{opp q}
// (keBoundaryStruct); donors outside the domain take the case's rule (in
// POISEUILLE only inlet/outlet nodes have one); every other population is
// never written in the reference and keeps its initial value.  POISEUILLE,
// and any case with a solid mask (the same rules on arbitrary voxels).
template <class S, class Addr>
__device__ __forceinline__ void pull_struct(RealOf<S> (&f)[Q], const StepArgs<S>& a, const Addr& ad,
                                            int x, int y, int z) {
  using R = RealOf<S>;
  const int t = node_type(a.g, x, y, z);
  const InitState is = initial_state(a.g, a.init_kind, a.seed, a.noise_amp, (float)a.rho0,
                                     (float)a.ulx, (float)a.uly, (float)a.ulz, a.inlet_u, x, y,
                                     z, t);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
    const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                        (unsigned)zs < (unsigned)a.g.nz;
    if (inside && node_type(a.g, xs, ys, zs) != NODE_STRUCT) {
      f[q] = ld(ad.donor(q), q, ad.inv_scale());
    } else if (inside && t == NODE_FLUID) {
      f[q] = ld(ad.own(opp(q)), opp(q), ad.inv_scale());
    } else if (!inside &&
               (a.g.casetype != POISEUILLE || t == NODE_INLET || t == NODE_OUTLET)) {
      const R fo = ld(ad.own(opp(q)), opp(q), ad.inv_scale());
      f[q] = boundary_value<S, q>(a, t, fo, y, z);
    } else {
      f[q] = to_internal<S, q>(initial_feq<R, q>(R(is.den), R(is.ux), R(is.uy), R(is.uz)));
    }
  });
}

// Steps 1-2: the post-stream, post-boundary populations f_k at (x,y,z);
// cell is the node's in-plane index.
template <class S, class Addr>
__device__ __forceinline__ void pull(RealOf<S> (&f)[Q], const StepArgs<S>& a, const Addr& ad, int x,
                                     int y, int z) {
  const bool edge = (x == 0) | (x == a.g.nx - 1) | (y == 0) | (y == a.g.ny - 1) | (z == 0) |
                    (z == a.g.nz - 1);
  if (has_struct(a.g)) {
    pull_struct<S>(f, a, ad, x, y, z);
  } else if (!edge) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = ld(ad.donor(q), q, ad.inv_scale());
    });
  } else {
    const int t = node_type(a.g, x, y, z);
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
      const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                          (unsigned)zs < (unsigned)a.g.nz;
      if (inside) {
        f[q] = ld(ad.donor(q), q, ad.inv_scale());
      } else {
        const RealOf<S> fo = ld(ad.own(opp(q)), opp(q), ad.inv_scale());
        f[q] = boundary_value<S, q>(a, t, fo, y, z);
      }
    });
  }
}

enum { COLL_SRT = 0, COLL_MRT = 1 };

// LES + collision of one node (or one F2 pair of nodes) in pair form.  ps
// holds the pair sums of f and the density / momentum the equilibrium is
// built from; u = j / rho.  emit(q, value) receives f*_q.
template <class S, int COLL, bool LES, bool FROM_PAIRS, class V, class Emit>
__device__ __forceinline__ void collide_node(const V (&f)[Q], const PairState<V>& ps, V ux, V uy,
                                             V uz, V inv_rho, const StepArgs<S>& a, Emit&& emit) {
  const V tau = bcast_param<V>(a.tau);
  V te = bc<V>(0);
  if constexpr (LES)
    te = les_tau_eddy_pairs<V>(ps, ux, uy, uz, inv_rho, tau, bcast_param<V>(a.les_c));
  const V inv = vrcp(tau + te);
  if constexpr (COLL == COLL_SRT)
    collide_srt_pairs<FROM_PAIRS, V, kDev<S>>(f, ps, ux, uy, uz, inv, emit);
  else
    collide_mrt_pairs<FROM_PAIRS, V, RealOf<S>, kDev<S>>(f, ps, inv, a.mp, emit);
}

// u = j * (1/rho); returns 1/rho
template <class V>
__device__ __forceinline__ V velocity(const PairState<V>& ps, V& ux, V& uy, V& uz) {
  const V inv = vrcp(ps.rho_full);
  ux = ps.jx * inv;
  uy = ps.jy * inv;
  uz = ps.jz * inv;
  return inv;
}

// Side outputs of the macroscopic state of arF_k.
template <class S>
__device__ __forceinline__ void write_macro(const StepArgs<S>& a, int x, int y, int z,
                                            RealOf<S> rho, RealOf<S> ux, RealOf<S> uy,
                                            RealOf<S> uz) {
  const long long n = x + (long long)a.g.nx * (z + (long long)a.g.nz * y);
  if (a.den_out) a.den_out[n] = (float)rho;
  if (a.ux_out) {
    a.ux_out[n] = (float)ux;
    a.uy_out[n] = (float)uy;
    a.uz_out[n] = (float)uz;
  }
  if (a.g.casetype == CHANNEL || a.g.casetype == POISEUILLE) {
    const int P = a.g.ny * a.g.nz, yz = y * a.g.nz + z;
    if (x == 1) a.prho_out[yz] = (float)rho;
    if (x == a.g.nx - 1) {
      a.pu_out[yz] = (float)ux;
      a.pu_out[P + yz] = (float)uy;
      a.pu_out[2 * P + yz] = (float)uz;
    }
    if (x == a.g.nx - 2) {
      a.pu_out[3 * P + yz] = (float)ux;
      a.pu_out[4 * P + yz] = (float)uy;
      a.pu_out[5 * P + yz] = (float)uz;
    }
  }
}

template <class S>
__device__ __forceinline__ void store_all(const StepArgs<S>& a, const RealOf<S> (&f)[Q],
                                          long long cell) {
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    StoreTraits<S>::store(a.dst + q * a.qs + cell, f[q], a.scale);
  });
}

// emit functor storing f*_q of one node into a lattice
template <class S>
struct StoreNode {
  S* base;
  long long qs;
  long long cell;
  float scale;
  __device__ __forceinline__ void operator()(int q, RealOf<S> v) const {
    StoreTraits<S>::store(base + q * qs + cell, v, scale);
  }
};

// Stochastic rounding (LBM_ROUND_STOCHASTIC).  cvt.rs rounds each FP32
// input to one of its two neighbouring 16-bit values, up with probability
// equal to the input's distance from the lower one in units of the spacing,
// using the caller's random bits (sm_100a).  The bits of a store are a hash
// of (pair word, step, seed, population), so a run is reproducible and a
// node gets the same bits whichever kernel stores it.  The pair word of node
// (x, y, z) is that of the paired rows, (x mod H) + H (z + nz y) with
// H = px / 2, and its half is x >= H, whatever the layout of the domain.
__device__ __forceinline__ uint32_t sr_hash(uint32_t word, uint32_t k, uint32_t seed) {
  uint32_t h = word * 0x9E3779B1u ^ (k * 0x85EBCA77u + seed);
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}
// bits of population q: h times an odd constant per q (a bijection of h,
// so each population's bits are uniform, and one multiply per store)
template <int q>
__device__ __forceinline__ uint32_t sr_bits(uint32_t h) {
  return h * (0x2C1B3C6Du + 2u * (uint32_t)q * 0x9E3779B9u);
}
__device__ __forceinline__ uint32_t sr_word(const Geometry& g, int x, int y, int z) {
  const int h = g.px >> 1;
  return (uint32_t)((x < h ? x : x - h) + h * (z + g.nz * y));
}

// Steps 3-6 of a node whose post-stream populations f are known:
// macroscopic, side outputs, LES, collision, store of f* (SR: stochastic
// rounding of the 16-bit stores, step number from a.kctr[a.kpar]).
template <class S, int COLL, bool LES, bool SR = false, class Addr>
__device__ __forceinline__ void finish_node(const RealOf<S> (&f)[Q], const StepArgs<S>& a,
                                            const Addr& ad, int x, int y, int z) {
  using R = RealOf<S>;
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  R ux, uy, uz;
  const R inv_rho = velocity<R>(ps, ux, uy, uz);
  write_macro<S>(a, x, y, z, ps.rho_full, ux, uy, uz);
  if constexpr (SR) {
    static_assert(kDev<S>, "stochastic rounding is a 16-bit store");
    const uint32_t h = sr_hash(sr_word(a.g, x, y, z), a.kctr[a.kpar], a.sr_seed);
    const int half = x >= (a.g.px >> 1);
    collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, inv_rho, a,
                                                 [&](auto qc, R v) {
      constexpr int q = decltype(qc)::value;
      StoreTraits<S>::store_sr(ad.out(q), v, ad.scale(), sr_bits<q>(h), half);
    });
  } else {
    collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, inv_rho, a,
                                                 [&](int q, R v) {
      StoreTraits<S>::store(ad.out(q), v, ad.scale());
    });
  }
}

// One fused step of the node (x, y, z): pull + boundary rules, macroscopic,
// LES, collision, store.  Shared by the single-domain and batched kernels,
// so a domain gets the same bits alone and in a batch (only where the
// arguments are held differs, not the arithmetic).
template <class S, int COLL, bool LES, bool SR = false, class Addr>
__device__ __forceinline__ void step_node_at(const StepArgs<S>& a, const Addr& ad, int x, int y,
                                             int z) {
  using R = RealOf<S>;
  // STRUCT nodes are never streamed, collided or measured (kernel.cu:294,
  // 323, 362, 464, 495, 1105)
  if (has_struct(a.g) && node_type(a.g, x, y, z) == NODE_STRUCT) return;
  R f[Q];
  pull<S>(f, a, ad, x, y, z);
  finish_node<S, COLL, LES, SR>(f, a, ad, x, y, z);
}

// stochastic rounding: the first thread of a step's grid leaves the next
// step number for the next step (the others read only kctr[kpar])
template <bool SR, class S>
__device__ __forceinline__ void bump_step_counter(const StepArgs<S>& a) {
  if constexpr (SR) {
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
      a.kctr[a.kpar ^ 1] = a.kctr[a.kpar] + 1;
  }
}
template <class S, int COLL, bool LES>
__device__ __forceinline__ void step_node(const StepArgs<S>& a, int x, int y, int z) {
  step_node_at<S, COLL, LES>(a, PlaneAddr<S>(a, x + a.g.px * (z + a.g.nz * y)), x, y, z);
}

// The fused step.  grid = (ceil(nx/blockDim.x), nz, ny), one thread per node.
template <class S, int COLL, bool LES, bool SR = false>
__global__ void __launch_bounds__(128) k_step(const __grid_constant__ StepArgs<S> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  bump_step_counter<SR>(a);
  if (x >= a.g.nx) return;
  step_node_at<S, COLL, LES, SR>(a, PlaneAddr<S>(a, x + a.g.px * (z + a.g.nz * y)), x, y, z);
}

// ------------------------------------------------------------------ //
// Initial state (Initialize codelet lbm_codelets.cpp:140-241 and the
// seeded perturbations of LBM_INIT_*): writes arF_0 into a.dst as plain
// post-stream populations (the "post" lattice) and collides it with the
// initial rho, u (as the reference's first step does with the CurrDen /
// CurrVel that Initialize stored) into post_collided.
// ------------------------------------------------------------------ //
struct InitParams {
  int kind;
  uint64_t seed;
  float noise_amp;
  float rho0, ulx, uly, ulz;  // RefDen, RefVel*
};

template <class S, int COLL, bool LES>
__global__ void __launch_bounds__(128)
    k_init(const __grid_constant__ StepArgs<S> a, S* __restrict__ collided, InitParams ip) {
  using R = RealOf<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= a.g.nx) return;
  const long long cell = cell_of(a.g, x, y, z);
  const int t = node_type(a.g, x, y, z);
  R f[Q];
  if (t == NODE_STRUCT) {
    // keInitialize leaves STRUCT nodes at the zeros of cudaMemset
    static_for<0, Q>([&](auto qc) { f[decltype(qc)::value] = R(0); });
    store_all<S>(a, f, cell);
    write_macro<S>(a, x, y, z, R(0), R(0), R(0), R(0));
    return;
  }
  const InitState is = initial_state(a.g, ip.kind, ip.seed, ip.noise_amp, ip.rho0, ip.ulx, ip.uly,
                                     ip.ulz, a.inlet_u, x, y, z, t);
  const R rd = R(is.den), ux = R(is.ux), uy = R(is.uy), uz = R(is.uz);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    f[q] = to_internal<S, q>(initial_feq<R, q>(rd, ux, uy, uz));
  });
  store_all<S>(a, f, cell);  // post-stream lattice
  write_macro<S>(a, x, y, z, rd, ux, uy, uz);
  if (!collided) return;  // AA streaming: the first step collides
  // the first step collides with the rho, u that Initialize stored
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  ps.rho = kDev<S> ? rd - R(1) : rd;
  ps.rho_full = rd;
  ps.jx = mul_rn(rd, ux);  // rounded products: the AA form repeats them exactly
  ps.jy = mul_rn(rd, uy);
  ps.jz = mul_rn(rd, uz);
  collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, vrcp(rd), a,
                                       StoreNode<S>{collided, a.qs, cell, a.scale});
}

// ------------------------------------------------------------------ //
// Import of host populations (AoS, direction fastest, optional ghost layer)
// into the post lattice, then macro + collision into `collided`.
// ------------------------------------------------------------------ //
template <class S, int COLL, bool LES>
__global__ void __launch_bounds__(128)
    k_import(const __grid_constant__ StepArgs<S> a, const float* __restrict__ aos, int padded,
             S* __restrict__ collided) {
  using R = RealOf<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= a.g.nx) return;
  const long long cell = cell_of(a.g, x, y, z);
  long long node;
  if (padded)
    node = (x + 1) + (long long)(a.g.nx + 2) * ((z + 1) + (long long)(a.g.nz + 2) * (y + 1));
  else
    node = x + (long long)a.g.nx * (z + (long long)a.g.nz * y);
  R f[Q];
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    f[q] = to_internal<S, q>(R(aos[q + node * Q]));
  });
  store_all<S>(a, f, cell);
  // re-read through the storage format so that the collided state starts
  // from exactly what the post lattice holds
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    f[q] = ld(a.dst + q * a.qs + cell, q, a.inv_scale);
  });
  if (has_struct(a.g) && node_type(a.g, x, y, z) == NODE_STRUCT) {
    write_macro<S>(a, x, y, z, R(0), R(0), R(0), R(0));
    return;
  }
  R ux, uy, uz;
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  if constexpr (kDev<S>) {
    velocity<R>(ps, ux, uy, uz);
    write_macro<S>(a, x, y, z, ps.rho_full, ux, uy, uz);
  } else {
    R rho;
    macroscopic<R>(f, rho, ux, uy, uz);  // CurrDen / CurrVel in the codelet's order
    write_macro<S>(a, x, y, z, rho, ux, uy, uz);
  }
  if (!collided) return;  // AA streaming: the next step collides
  const R inv_rho = velocity<R>(ps, ux, uy, uz);
  collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, inv_rho, a,
                                       StoreNode<S>{collided, a.qs, cell, a.scale});
}

// ------------------------------------------------------------------ //
// AA streaming (in place, one lattice), for the cavity geometry.
//
// Two layouts alternate.  "Natural": slot (x, q) holds the post-stream,
// post-boundary f_q(x) (arF).  A local step reads its node's natural
// slots, collides and writes f*_q into its own slot (x, opp q): the layout
// becomes "swapped", in which arF_q(x) = f*_q(x - c_q) sits in slot
// (x - c_q, opp q).  A neighbour step reads those slots, collides and writes
// f*_q(x) into (x + c_q, q), the natural slot of its destination: the
// layout is natural again.  Each neighbour-step thread reads and writes the
// same 19 slots, so the update is race-free in place.  Wall rules (on-node
// bounce-back with the lid term, lbm_codelets.cpp:373-395) act where a slot
// of the neighbour step lies outside the box: a donor x - c_q outside reads
// the node's own f*_{opp q} from (x, q); a destination x + c_q outside
// writes the wall value of population opp q into the node's natural slot
// (x, opp q).  Inlet and outlet rules (CHANNEL, kernel.cu:566-657) need the
// face densities / velocities of the step before, which the neighbour step
// is still computing when it writes: there the neighbour step writes the
// plain f*_q into (x, opp q) like a fixed wall, and the rule is applied
// when the natural slot is read (the next local step, the macroscopic and
// export kernels), with the face buffers of that step.  The natural layout
// is "complete" after the initial state and an import (every slot holds
// arF, rules applied) and "pending" after a neighbour step.  Same node
// arithmetic as the pull step; the two kernels agree to within a few FP32
// roundings (the compiler may fuse a multiply-add differently in each).
//
// Face buffers: AA step k reads arF_{k-1} and writes its rho / u into
// prho[k & 1] / pu[k & 1] (make_args with k); the rules for arF_{k-1} read
// those of step k-1.  Kernels that read the state after step s therefore
// take make_args with k = s + 1.
// ------------------------------------------------------------------ //

// arF of node (x, y, z) from the swapped layout (cell = cell_of the node)
template <class S>
__device__ __forceinline__ void aa_pull_swapped(RealOf<S> (&f)[Q], const StepArgs<S>& a, int x,
                                                int y, int z, int cell) {
  const bool edge = (x == 0) | (x == a.g.nx - 1) | (y == 0) | (y == a.g.ny - 1) | (z == 0) |
                    (z == a.g.nz - 1);
  if (a.g.rows != kRowsPlain) {
    // quad rows: x neighbours are not a fixed element offset apart
    const int t = edge ? node_type(a.g, x, y, z) : NODE_FLUID;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
      const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                          (unsigned)zs < (unsigned)a.g.nz;
      if (inside) {
        f[q] = ld(a.srcq[opp(q)] + cell_of(a.g, xs, ys, zs), q, a.inv_scale);
      } else {
        const RealOf<S> fo = ld(a.srcq[q] + cell, q, a.inv_scale);  // own f*_{opp q}
        f[q] = boundary_value<S, q>(a, t, fo, y, z);
      }
    });
    return;
  }
  if (!edge) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = ld(a.srcq[opp(q)] + (cell - a.off[q]), q, a.inv_scale);
    });
  } else {
    const int t = node_type(a.g, x, y, z);
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
      const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                          (unsigned)zs < (unsigned)a.g.nz;
      if (inside) {
        f[q] = ld(a.srcq[opp(q)] + (cell - a.off[q]), q, a.inv_scale);
      } else {
        const RealOf<S> fo = ld(a.srcq[q] + cell, q, a.inv_scale);  // own f*_{opp q}
        f[q] = boundary_value<S, q>(a, t, fo, y, z);
      }
    });
  }
}

// the wall value of population opp(d) at a node of type t from its f*_d:
// boundary_value<S, opp d> with a run-time d (cavity node types)
template <class S>
__device__ __forceinline__ RealOf<S> aa_wall(const StepArgs<S>& a, int t, RealOf<S> fo, int d) {
  using R = RealOf<S>;
  if (t != NODE_MOVINGWALL) return fo;
  R eu = add_rn(add_rn(mul_rn(R(cx(d)), a.ulx), mul_rn(R(cy(d)), a.uly)), mul_rn(R(cz(d)), a.ulz));
  R term = mul_rn(mul_rn(mul_rn(R(6), weight<R>(d)), a.rho0), eu);
  return sub_rn(fo, term);
}

// Inlet / outlet rules of a node of the natural layout whose slots are
// pending: each population whose donor x - c_q lies outside the box holds
// the node's own f*_{opp q} (see above); replace it by the boundary value.
template <class S>
__device__ __forceinline__ void aa_open_face_rules(RealOf<S> (&f)[Q], const StepArgs<S>& a, int x,
                                                   int y, int z) {
  if (a.g.casetype != CHANNEL) return;
  const int t = node_type(a.g, x, y, z);
  if (t != NODE_INLET && t != NODE_OUTLET) return;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
    const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                        (unsigned)zs < (unsigned)a.g.nz;
    if (!inside) f[q] = boundary_value<S, q>(a, t, f[q], y, z);
  });
}

// Slot addresses of an AA step, set per step in the kernel parameters so
// that an interior node needs one address operation per access:
//   local step:      a.srcd[q] = plane q,                 a.dstq[q] = plane opp q
//   neighbour step:  a.srcd[q] = plane opp q, minus off_q, a.dstq[q] = plane q, plus off_q
// (arF_q(x) is read at srcd[q] + cell, f*_q(x) written at dstq[q] + cell);
// a.srcq[q] stays the plain plane q, for the rules at the box faces.
template <class S>
struct AADst {
  const StepArgs<S>& a;
  int cell;
  __device__ __forceinline__ S* out(int q) const { return a.dstq[q] + cell; }
  __device__ __forceinline__ float scale() const { return a.scale; }
};

// The neighbour step of a node in a row that is not on a y or z face, for
// the warps that hold an x face of such rows.  Only the populations whose
// donor x - c_q or destination x + c_q leaves the box at x = 0 or x = nx-1
// differ from the interior form, and only in their slot: a donor outside is
// the node's own slot (x, q) (the wall rule of the node applied to it, which
// for the cavity's fixed walls is the value itself), a destination outside
// is the node's own slot (x, opp q) (the plain f*_q: x faces are fixed
// walls, inlets or outlets, whose rules are applied when the natural slot
// is read).  The slot is chosen per lane, so the warp does not diverge.
template <class S, int COLL, bool LES>
__device__ __forceinline__ void aa_neighbor_xface_node(const StepArgs<S>& a, int x, int y, int z,
                                                       int cell) {
  using R = RealOf<S>;
  const bool xlo = x == 0, xhi = x == a.g.nx - 1;
  R f[Q];
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const bool out = (cx(q) == 1 && xlo) || (cx(q) == -1 && xhi);
    f[q] = ld((out ? a.srcq[q] : a.srcd[q]) + cell, q, a.inv_scale);
  });
  if (a.g.casetype != CAVITY && (xlo || xhi)) {
    // inlet / outlet rules on the donors outside (the cavity's walls keep
    // the value)
    const int t = node_type(a.g, x, y, z);
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      if ((cx(q) == 1 && xlo) || (cx(q) == -1 && xhi))
        f[q] = boundary_value<S, q>(a, t, f[q], y, z);
    });
  }
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  R ux, uy, uz;
  const R inv_rho = velocity<R>(ps, ux, uy, uz);
  write_macro<S>(a, x, y, z, ps.rho_full, ux, uy, uz);
  collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, inv_rho, a, [&](auto qc, R v) {
    constexpr int q = decltype(qc)::value;
    const bool out = (cx(q) == -1 && xlo) || (cx(q) == 1 && xhi);
    StoreTraits<S>::store(out ? a.dst + (opp(q) * a.qs + cell) : a.dstq[q] + cell, v, a.scale);
  });
}

// One AA step of node (x, y, z) (shared by the single-domain and batched
// kernels); neighbor = 0: local step (natural -> swapped), 1: neighbour
// step (swapped -> natural).  entry (local steps): kAAPending, the natural
// slots are pending; kAAFromInit, the first step after the initial state,
// which collides with the rho, u that Initialize stored, as k_init does for
// the pull form; kAAComplete, the slots hold arF (after an import).
// a.src = a.dst = the lattice.
enum { kAAPending = 0, kAAFromInit = 1, kAAComplete = 2 };

//
// warp_row: the caller maps the lanes of a warp to the x-consecutive nodes
// x - lane .. x - lane + 31 of one row (the single-domain kernel), so that
// "this warp holds an x face" is known to every lane without a vote and a
// warp of an interior row that holds one takes the x-face form as a whole.
// Otherwise (the batched kernel, whose warps may span rows) each lane
// decides for itself.
template <class S, int COLL, bool LES, bool WARP_ROW = false>
__device__ __forceinline__ void aa_step_node(const StepArgs<S>& a, int x, int y, int z,
                                             int neighbor, int entry) {
  using R = RealOf<S>;
  // quad rows (16-bit storage) reach this per-node step only as a local
  // step, whose slots are all at the node
  const int cell = kDev<S> ? cell_of(a.g, x, y, z) : x + a.g.px * (z + a.g.nz * y);
  const bool face_row = (y == 0) | (y == a.g.ny - 1) | (z == 0) | (z == a.g.nz - 1);
  const bool xface = (x == 0) | (x == a.g.nx - 1);
  const bool edge = face_row | xface;
  bool xsel = xface;
  if constexpr (WARP_ROW) {
    const int x0 = x - (int)(threadIdx.x & 31u);  // the warp's first node
    xsel = x0 == 0 || (unsigned)(a.g.nx - 1 - x0) < 32u;
  }
  R f[Q];
  if (neighbor && !face_row && xsel) {
    aa_neighbor_xface_node<S, COLL, LES>(a, x, y, z, cell);
    return;
  }
  if (!neighbor || !edge) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = ld(a.srcd[q] + cell, q, a.inv_scale);
    });
    if (!neighbor && edge && entry == kAAPending) aa_open_face_rules<S>(f, a, x, y, z);
    const AADst<S> ad{a, cell};
    if (entry != kAAFromInit) {
      finish_node<S, COLL, LES>(f, a, ad, x, y, z);
    } else {
      const int t = node_type(a.g, x, y, z);
      const InitState is = initial_state(a.g, a.init_kind, a.seed, a.noise_amp, (float)a.rho0,
                                         (float)a.ulx, (float)a.uly, (float)a.ulz, a.inlet_u, x,
                                         y, z, t);
      const R rd = R(is.den), ux = R(is.ux), uy = R(is.uy), uz = R(is.uz);
      write_macro<S>(a, x, y, z, rd, ux, uy, uz);
      PairState<R> ps;
      make_pairs<R, kDev<S>>(f, ps);
      ps.rho = kDev<S> ? rd - R(1) : rd;
      ps.rho_full = rd;
      ps.jx = mul_rn(rd, ux);
      ps.jy = mul_rn(rd, uy);
      ps.jz = mul_rn(rd, uz);
      collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, vrcp(rd), a, [&](int q, R v) {
        StoreTraits<S>::store(ad.out(q), v, ad.scale());
      });
    }
    return;
  }
  // neighbour step at a box face: slots outside the box are the node's own
  const int t = node_type(a.g, x, y, z);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
    const bool inside = (unsigned)xs < (unsigned)a.g.nx && (unsigned)ys < (unsigned)a.g.ny &&
                        (unsigned)zs < (unsigned)a.g.nz;
    if (inside) {
      f[q] = ld(a.srcd[q] + cell, q, a.inv_scale);
    } else {
      const RealOf<S> fo = ld(a.srcq[q] + cell, q, a.inv_scale);  // own f*_{opp q}
      f[q] = boundary_value<S, q>(a, t, fo, y, z);
    }
  });
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  R ux, uy, uz;
  const R inv_rho = velocity<R>(ps, ux, uy, uz);
  write_macro<S>(a, x, y, z, ps.rho_full, ux, uy, uz);
  collide_node<S, COLL, LES, kFromPairs<S>, R>(f, ps, ux, uy, uz, inv_rho, a, [&](int q, R v) {
    const int xt = x + cx(q), yt = y + cy(q), zt = z + cz(q);
    const bool inside = (unsigned)xt < (unsigned)a.g.nx && (unsigned)yt < (unsigned)a.g.ny &&
                        (unsigned)zt < (unsigned)a.g.nz;
    if (inside)
      StoreTraits<S>::store(a.dstq[q] + cell, v, a.scale);
    else
      StoreTraits<S>::store(a.dst + (opp(q) * a.qs + cell), aa_wall<S>(a, t, v, q), a.scale);
  });
}

// One kernel per step kind (NB = neighbor): the local step, which has no
// box-face logic besides the open-face rules, fits 56 registers (9 CTAs of
// 128 per SM) without spills; the neighbour step keeps 64.
template <class S, int COLL, bool LES, int NB>
__global__ void __launch_bounds__(128, NB ? 8 : 9)
    k_aa_step(const __grid_constant__ StepArgs<S> a, int entry) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= a.g.nx) return;
  aa_step_node<S, COLL, LES, true>(a, x, y, z, NB, entry);
}

// rho and u of arF in the current AA layout, written through a.den_out /
// a.ux_out...: the same arithmetic as the step kernels' side outputs.
// layout: kAASwapped (after a local step), kAANaturalPending (after a
// neighbour step), kAANaturalComplete.
enum { kAANaturalComplete = 0, kAASwapped = 1, kAANaturalPending = 2 };

template <class S>
__global__ void __launch_bounds__(128) k_aa_macro(const __grid_constant__ StepArgs<S> a,
                                                  int layout) {
  using R = RealOf<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= a.g.nx) return;
  const int cell = cell_of(a.g, x, y, z);
  R f[Q];
  if (layout == kAASwapped) {
    aa_pull_swapped<S>(f, a, x, y, z, cell);
  } else {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = ld(a.srcq[q] + cell, q, a.inv_scale);
    });
    if (layout == kAANaturalPending) aa_open_face_rules<S>(f, a, x, y, z);
  }
  PairState<R> ps;
  make_pairs<R, kDev<S>>(f, ps);
  R ux, uy, uz;
  velocity<R>(ps, ux, uy, uz);
  write_macro<S>(a, x, y, z, ps.rho_full, ux, uy, uz);
}

enum { kExportPull = 0, kExportDirect = 1, kExportAASwapped = 2, kExportAANaturalPending = 3 };

// ------------------------------------------------------------------ //
// Export of arF_k into a device AoS buffer.  kExportDirect: a.src holds
// arF_k itself (right after initialize/import, or an AA lattice in the
// complete natural layout); kExportPull: a.src holds f*_{k-1} and arF_k is
// reconstructed by the same pull + boundary code as the step kernel; the
// AA modes read the lattice in the swapped or the pending natural layout.
// Padded output zeroes the ghost layer.
// ------------------------------------------------------------------ //
template <class S>
__global__ void __launch_bounds__(128)
    k_export(const __grid_constant__ StepArgs<S> a, float* __restrict__ aos, int padded,
             int mode) {
  using R = RealOf<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  if (x >= a.g.nx) return;
  const long long cell = cell_of(a.g, x, y, z);
  R f[Q];
  if (has_struct(a.g) && node_type(a.g, x, y, z) == NODE_STRUCT) {
    static_for<0, Q>([&](auto qc) { f[decltype(qc)::value] = R(0); });
  } else if (mode == kExportDirect || mode == kExportAANaturalPending) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = ld(a.src + q * a.qs + cell, q, a.inv_scale);
    });
    if (mode == kExportAANaturalPending) aa_open_face_rules<S>(f, a, x, y, z);
  } else if (mode == kExportAASwapped) {
    aa_pull_swapped<S>(f, a, x, y, z, (int)cell);
  } else if (a.g.rows != kRowsPlain) {
    pull<S>(f, a, RowAddr<S>(a, x, y, z), x, y, z);
  } else {
    pull<S>(f, a, PlaneAddr<S>(a, (int)cell), x, y, z);
  }
  long long node;
  if (padded)
    node = (x + 1) + (long long)(a.g.nx + 2) * ((z + 1) + (long long)(a.g.nz + 2) * (y + 1));
  else
    node = x + (long long)a.g.nx * (z + (long long)a.g.nz * y);
  const bool solid = has_struct(a.g) && node_type(a.g, x, y, z) == NODE_STRUCT;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    aos[q + node * Q] = solid ? 0.0f : (float)to_population<S, q>(f[q]);
  });
}

// ------------------------------------------------------------------ //
// Two nodes per thread: the pair (x0, x0+1), x0 even.  Populations with
// c_x = 0 are read as one aligned 2-element vector, the others as two
// scalars; all node arithmetic runs on F2 lanes (packed FP32), and the
// pair is stored as one vector per population.  A pair that touches the
// domain boundary takes the per-node boundary path and is packed after.
// ------------------------------------------------------------------ //
template <class S>
__device__ __forceinline__ F2 ld_pair(const S* p, int q, float inv_scale);
template <>
__device__ __forceinline__ F2 ld_pair<float>(const float* p, int, float) {
  return F2{*reinterpret_cast<const float2*>(p)};
}
template <>
__device__ __forceinline__ F2 ld_pair<__half>(const __half* p, int, float inv_scale) {
  const float2 h = __half22float2(*reinterpret_cast<const __half2*>(p));
  return F2{__fmul2_rn(h, make_float2(inv_scale, inv_scale))};
}
template <>
__device__ __forceinline__ F2 ld_pair<__nv_bfloat16>(const __nv_bfloat16* p, int,
                                                     float inv_scale) {
  const float2 h = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  return F2{__fmul2_rn(h, make_float2(inv_scale, inv_scale))};
}

template <class S>
__device__ __forceinline__ void st_pair(S* p, F2 v, int q, float scale);
template <>
__device__ __forceinline__ void st_pair<float>(float* p, F2 v, int, float) {
  *reinterpret_cast<float2*>(p) = v.v;
}
template <>
__device__ __forceinline__ void st_pair<__half>(__half* p, F2 v, int, float scale) {
  const float2 d = __fmul2_rn(v.v, make_float2(scale, scale));
  *reinterpret_cast<__half2*>(p) = __float22half2_rn(d);
}
template <>
__device__ __forceinline__ void st_pair<__nv_bfloat16>(__nv_bfloat16* p, F2 v, int,
                                                       float scale) {
  const float2 d = __fmul2_rn(v.v, make_float2(scale, scale));
  *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(d);
}

// minimum resident blocks per SM requested for the packed kernel (caps its
// registers per thread; 0 = no cap)
#ifndef LBM_PACKED_MIN_BLOCKS
#define LBM_PACKED_MIN_BLOCKS 0
#endif

template <class S, int COLL, bool LES>
__global__ void __launch_bounds__(64, LBM_PACKED_MIN_BLOCKS) k_step2(const __grid_constant__ StepArgs<S> a) {
  static_assert(std::is_same<RealOf<S>, float>::value, "packed kernel is FP32 arithmetic");
  const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int z = blockIdx.y, y = blockIdx.z;
  if (x0 >= a.g.nx) return;
  const int cell = x0 + a.g.px * (z + a.g.nz * y);
  const bool two = x0 + 1 < a.g.nx;
  const bool interior = x0 >= 1 && x0 + 1 <= a.g.nx - 2 && y >= 1 && y <= a.g.ny - 2 && z >= 1 &&
                        z <= a.g.nz - 2;
  F2 f[Q];
  if (interior) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const S* p = a.srcd[q] + cell;
      if constexpr (cx(q) == 0) {
        f[q] = ld_pair<S>(p, q, a.inv_scale);
      } else {
        f[q] = mk2(ld(p, q, a.inv_scale), ld(p + 1, q, a.inv_scale));
      }
    });
  } else {
    float fa[Q], fb[Q];
    pull<S>(fa, a, PlaneAddr<S>(a, cell), x0, y, z);
    if (two) {
      pull<S>(fb, a, PlaneAddr<S>(a, cell + 1), x0 + 1, y, z);
    } else {
      static_for<0, Q>([&](auto qc) { fb[decltype(qc)::value] = fa[decltype(qc)::value]; });
    }
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = mk2(fa[q], fb[q]);
    });
  }
  PairState<F2> ps;
  make_pairs<F2, kDev<S>>(f, ps);
  F2 ux, uy, uz;
  const F2 inv_rho = velocity<F2>(ps, ux, uy, uz);
  if (a.den_out || a.ux_out || a.g.casetype == CHANNEL) {
    write_macro<S>(a, x0, y, z, ps.rho_full.v.x, ux.v.x, uy.v.x, uz.v.x);
    if (two) write_macro<S>(a, x0 + 1, y, z, ps.rho_full.v.y, ux.v.y, uy.v.y, uz.v.y);
  }
  collide_node<S, COLL, LES, true, F2>(f, ps, ux, uy, uz, inv_rho, a, [&](int q, F2 v) {
    if (two)
      st_pair<S>(a.dstq[q] + cell, v, q, a.scale);
    else
      StoreTraits<S>::store(a.dstq[q] + cell, v.v.x, a.scale);
  });
}

// ------------------------------------------------------------------ //
// Paired rows: the 16-bit pull step with two nodes per thread and 32-bit
// accesses only.
//
// With paired rows (kRowsPaired), word w of a row holds the nodes (w, w + H),
// H = px / 2.  The donors x - c_q of both nodes of a pair then lie in one
// word of the donor row, shifted by c_x, so a thread loads one aligned
// 32-bit word per population for two nodes (a warp reads 128 contiguous
// bytes, as the FP32 kernel does for one node per thread), converts it with
// one packed conversion and runs the node arithmetic on F2 lanes (packed
// FP32: one instruction for both nodes).  Per pair: 19 word loads, 19 word
// stores, one F2 collision.
//
// k_step_paired takes every word.  A thread loads, for each population,
// the word beside its own (w - c_x) in the donor row, which holds the x
// donors of both lanes except in the special words:
//   - the seam: node H - 1 (lo of word H - 1) and node H (hi of word 0) are
//     x neighbours held in different words;
//   - x faces (x = 0, lo of word 0; x = nx - 1, a hi lane): the populations
//     whose donor lies outside take the node's boundary rule from the
//     node's own f*_{opp q};
// where the beside word (read past the row end: the neighbouring row's
// word, inside the allocation) is replaced lane by lane in a branch that
// only those threads take (two or three per row).  Rows on a y or z face
// take, for the populations whose donor row is outside, the wall rule of
// each lane's node (the test is uniform along the row).  Hi lanes past the
// last node (x >= nx when nx < px) compute on padding slots, which no real
// node reads and nothing exports.  The node types and rules are those of
// the per-node path, which steps the geometries with STRUCT nodes
// (k_step_rows); the 16-bit units are built without multiply-add
// contraction and both paths rebuild f* from the pair sums, so a node gets
// the same bits from either.
// ------------------------------------------------------------------ //
template <class S>
__device__ __forceinline__ F2 unpack_pair(uint32_t word, float inv_scale);
template <>
__device__ __forceinline__ F2 unpack_pair<__half>(uint32_t word, float inv_scale) {
  __half2 h;
  memcpy(&h, &word, 4);
  return F2{__fmul2_rn(__half22float2(h), make_float2(inv_scale, inv_scale))};
}
template <>
__device__ __forceinline__ F2 unpack_pair<__nv_bfloat16>(uint32_t word, float inv_scale) {
  __nv_bfloat162 h;
  memcpy(&h, &word, 4);
  return F2{__fmul2_rn(__bfloat1622float2(h), make_float2(inv_scale, inv_scale))};
}
template <class S>
__device__ __forceinline__ uint32_t pack_pair(F2 v, float scale);
template <>
__device__ __forceinline__ uint32_t pack_pair<__half>(F2 v, float scale) {
  const __half2 h = __float22half2_rn(__fmul2_rn(v.v, make_float2(scale, scale)));
  uint32_t word;
  memcpy(&word, &h, 4);
  return word;
}
template <>
__device__ __forceinline__ uint32_t pack_pair<__nv_bfloat16>(F2 v, float scale) {
  const __nv_bfloat162 h = __float22bfloat162_rn(__fmul2_rn(v.v, make_float2(scale, scale)));
  uint32_t word;
  memcpy(&word, &h, 4);
  return word;
}
template <class S>
__device__ __forceinline__ uint32_t pack_pair_sr(F2 v, float scale, uint32_t rbits);
template <>
__device__ __forceinline__ uint32_t pack_pair_sr<__half>(F2 v, float scale, uint32_t rbits) {
  const float2 x = __fmul2_rn(v.v, make_float2(scale, scale));
  uint32_t d;  // a (the hi lane) goes to the upper half, b (lo) to the lower
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(x.y), "f"(x.x), "r"(rbits));
  return d;
}
template <>
__device__ __forceinline__ uint32_t pack_pair_sr<__nv_bfloat16>(F2 v, float scale,
                                                               uint32_t rbits) {
  const float2 x = __fmul2_rn(v.v, make_float2(scale, scale));
  uint32_t d;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(x.y), "f"(x.x), "r"(rbits));
  return d;
}

// the paired step kernel applies to the domain (else: k_step_rows); nx >=
// 11 keeps both x faces out of each other's words and every hi lane's x + 1
// donor of a real node inside the row
__host__ __device__ __forceinline__ bool paired_kernel_applies(const Geometry& g) {
  return !has_struct(g) && (g.px >> 1) <= g.nx - 2;
}

// Resident threads per SM the register budget is sized for: 1024 (64
// registers per thread) measured fastest on the 256^3 cavity (55k MLUPS
// against 48k at 768 and 50k at 896; more warps hide more load latency,
// which outweighs the few spilled registers).
#ifndef LBM_PAIRED_THREADS_PER_SM
#define LBM_PAIRED_THREADS_PER_SM 1024
#endif

// grid = (ceil(H / b), nz, ny), b = H rounded up to a multiple of 32 and
// at most 128 threads, one word (two nodes) per thread; a.srcd[q] = plane q
// minus the donor offset 2 c_x + px (c_z + nz c_y)
#ifndef LBM_PAIRED_SR_THREADS_PER_SM
#define LBM_PAIRED_SR_THREADS_PER_SM 768
#endif
// One word w (0 <= w < px/2) of row (y, z): the step of its two nodes
// (shared by the single-domain and batched kernels).
template <class S, int COLL, bool LES, bool SR>
__device__ __forceinline__ void paired_word(const StepArgs<S>& a, int w, int y, int z) {
  static_assert(kDev<S>, "paired rows are a 16-bit layout");
  const int H = a.g.px >> 1;
  const int xh = w + H;                             // node of the hi lane
  const int e = 2 * w + a.g.px * (z + a.g.nz * y);  // the pair's word (lo slot)
  const bool face_row = y == 0 || y == a.g.ny - 1 || z == 0 || z == a.g.nz - 1;
  F2 f[Q];
  if (!face_row) {
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = unpack_pair<S>(*reinterpret_cast<const uint32_t*>(a.srcd[q] + e), a.inv_scale);
    });
  } else {
    const int t_lo = node_type(a.g, w, y, z);
    const int t_hi = xh < a.g.nx ? node_type(a.g, xh, y, z) : NODE_FLUID;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const bool inside = (unsigned)(y - cy(q)) < (unsigned)a.g.ny &&
                          (unsigned)(z - cz(q)) < (unsigned)a.g.nz;
      if (inside) {
        f[q] = unpack_pair<S>(*reinterpret_cast<const uint32_t*>(a.srcd[q] + e), a.inv_scale);
      } else {
        const F2 fo = unpack_pair<S>(*reinterpret_cast<const uint32_t*>(a.srcq[opp(q)] + e),
                                     a.inv_scale);
        f[q] = mk2(boundary_value<S, q>(a, t_lo, fo.v.x, y, z),
                   boundary_value<S, q>(a, t_hi, fo.v.y, y, z));
      }
    });
  }
  if (w == 0 || w == H - 1 || xh == a.g.nx - 1) {
    // the seam and the x faces (see above), lane by lane
    const int e0 = e - 2 * w;  // row start
    const int t_lo = node_type(a.g, w, y, z);
    const int t_hi = xh < a.g.nx ? node_type(a.g, xh, y, z) : NODE_FLUID;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      if constexpr (cx(q) != 0) {
        const bool inside = !face_row || ((unsigned)(y - cy(q)) < (unsigned)a.g.ny &&
                                          (unsigned)(z - cz(q)) < (unsigned)a.g.nz);
        if (inside) {
          const int ws = cx(q) == 1 ? H - 1 : 0;  // the word across the seam
          if ((cx(q) == 1 && w == 0) || (cx(q) == -1 && w == H - 1)) {
            const uint32_t sw =
                *reinterpret_cast<const uint32_t*>(a.srcd[q] + (e0 + 2 * ws + 2 * cx(q)));
            const F2 v = unpack_pair<S>(sw, a.inv_scale);
            if (cx(q) == 1)
              f[q].v.y = v.v.x;  // x = H takes node H - 1
            else
              f[q].v.x = v.v.y;  // x = H - 1 takes node H
          }
          const bool lo_out = cx(q) == 1 && w == 0;
          const bool hi_out = cx(q) == -1 && xh == a.g.nx - 1;
          if (lo_out || hi_out) {
            const F2 fo = unpack_pair<S>(*reinterpret_cast<const uint32_t*>(a.srcq[opp(q)] + e),
                                         a.inv_scale);
            if (lo_out) f[q].v.x = boundary_value<S, q>(a, t_lo, fo.v.x, y, z);
            if (hi_out) f[q].v.y = boundary_value<S, q>(a, t_hi, fo.v.y, y, z);
          }
        }
      }
    });
  }
  PairState<F2> ps;
  make_pairs<F2, true>(f, ps);
  F2 ux, uy, uz;
  const F2 inv_rho = velocity<F2>(ps, ux, uy, uz);
  if (a.den_out || a.ux_out || a.g.casetype == CHANNEL) {
    write_macro<S>(a, w, y, z, ps.rho_full.v.x, ux.v.x, uy.v.x, uz.v.x);
    if (xh < a.g.nx) write_macro<S>(a, xh, y, z, ps.rho_full.v.y, ux.v.y, uy.v.y, uz.v.y);
  }
  if constexpr (!SR) {
    collide_node<S, COLL, LES, true, F2>(f, ps, ux, uy, uz, inv_rho, a, [&](int q, F2 v) {
      *reinterpret_cast<uint32_t*>(a.dstq[q] + e) = pack_pair<S>(v, a.scale);
    });
  } else {
    // the step number: this step reads kctr[kpar] and leaves its successor
    // in kctr[kpar ^ 1] for the next step
    bump_step_counter<SR>(a);
    const uint32_t h = sr_hash((uint32_t)(e >> 1), a.kctr[a.kpar], a.sr_seed);
    collide_node<S, COLL, LES, true, F2>(f, ps, ux, uy, uz, inv_rho, a, [&](auto qc, F2 v) {
      constexpr int q = decltype(qc)::value;
      *reinterpret_cast<uint32_t*>(a.dstq[q] + e) = pack_pair_sr<S>(v, a.scale, sr_bits<q>(h));
    });
  }
}

template <class S, int COLL, bool LES, bool SR>
__global__ void __launch_bounds__(128, (SR ? LBM_PAIRED_SR_THREADS_PER_SM
                                           : LBM_PAIRED_THREADS_PER_SM) / 128)
    k_step_paired(const __grid_constant__ StepArgs<S> a) {
  const int w = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int z = blockIdx.y, y = blockIdx.z;
  if (w >= (a.g.px >> 1)) return;
  paired_word<S, COLL, LES, SR>(a, w, y, z);
}

// Paired domains the paired kernel does not apply to (STRUCT nodes, nx <
// 11): the per-node step over paired rows.  grid = (ceil(nx/128), nz, ny).
template <class S, int COLL, bool LES, bool SR = false>
__global__ void __launch_bounds__(128) k_step_rows(const __grid_constant__ StepArgs<S> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y, y = blockIdx.z;
  bump_step_counter<SR>(a);
  if (x >= a.g.nx) return;
  step_node_at<S, COLL, LES, SR>(a, RowAddr<S>(a, x, y, z), x, y, z);
}

// node type and inside mask per node, [ny][nz][nx]
__global__ void k_node_info(Geometry g, int* __restrict__ type, int* __restrict__ ds);

// Deterministic FP64 reductions of the macroscopic state:
// partial[b*8 + i] for block b, then k_diag_final sums blocks in order.
__global__ void k_diag_partial(const float* __restrict__ den, const float* __restrict__ den_prev,
                               const float* __restrict__ ux, const float* __restrict__ uy,
                               const float* __restrict__ uz, long long n, int has_prev,
                               double* __restrict__ partial);
__global__ void k_diag_final(const double* __restrict__ partial, int nblocks,
                             double* __restrict__ out);

}  // namespace lbm
