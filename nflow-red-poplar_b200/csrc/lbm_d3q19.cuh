// lbm_d3q19.cuh — D3Q19 lattice constants and the per-node arithmetic of
// the fused step (macroscopic moments, Smagorinsky LES, SRT and MRT
// collision), evaluated in registers with every lattice constant known at
// compile time.
//
// Velocity set, opposites and weights follow main.cpp:87-146 of the
// reference (direction ordering is part of the arF boundary format, so it is
// kept exactly).  The moment matrix is main.cpp:149-171.  Its rows are
// mutually orthogonal, so M^-1 = M^T diag(1/|row_k|^2): the back transform
// is a sparse transpose product, not the dense 19x19 product of
// Collision_MRT (lbm_codelets.cpp:508-532).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

namespace lbm {

constexpr int Q = 19;

__host__ __device__ constexpr int cx(int q) {
  constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  return t[q];
}
__host__ __device__ constexpr int cy(int q) {
  constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
  return t[q];
}
__host__ __device__ constexpr int cz(int q) {
  constexpr int t[19] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
  return t[q];
}
__host__ __device__ constexpr int opp(int q) {
  constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
  return t[q];
}
// weight class: 0 rest (1/3), 1 axis (1/18), 2 diagonal (1/36)
__host__ __device__ constexpr int wclass(int q) { return q == 0 ? 0 : (q < 7 ? 1 : 2); }

__host__ __device__ constexpr int mrt_m(int k, int j) {
  constexpr int t[19][19] = {
      {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
      {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
      {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
      {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
      {0, 0, 0, 4, -4, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
      {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, 0, 0, -1, -1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
      {0, 0, 0, 2, 2, -2, -2, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1},
      {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 1, 1, -1, -1},
      {0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1}};
  return t[k][j];
}
// |row k|^2 of the moment matrix
__host__ __device__ constexpr int mrt_norm2(int k) {
  int s = 0;
  for (int j = 0; j < 19; ++j) s += mrt_m(k, j) * mrt_m(k, j);
  return s;
}

template <int N>
using IC = std::integral_constant<int, N>;

// compile-time loop: f(std::integral_constant<int, I>) for I in [B, E)
template <int B, int E, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// ------------------------------------------------------------------ //
// Storage formats.  R is the arithmetic type (float, or double for the
// FP64 build).  The node arithmetic works on "internal" population values:
// the populations f themselves for FP32 / FP64, and the deviations
// g = f - w from the rest state for the shifted 16-bit formats, which hold
// g * scale.  Carrying g through the arithmetic (not only through the
// store) keeps every sum over populations a sum of small numbers: summed as
// f = w + g, the FP32 roundings of the sums follow the fixed bit patterns
// of the weights and add up to a systematic drift of the density (a mass
// gain of ~3e-7 per node and step was measured that way), which g avoids.
// ------------------------------------------------------------------ //
template <class S>
struct StoreTraits;
template <>
struct StoreTraits<float> {
  using R = float;
  static constexpr bool dev = false;  // internal value = f
  __device__ static __forceinline__ float from_raw(float h, float) { return h; }
  __device__ static __forceinline__ float load(const float* p, float) { return *p; }
  __device__ static __forceinline__ void store(float* p, float v, float) { *p = v; }
};
template <>
struct StoreTraits<double> {
  using R = double;
  static constexpr bool dev = false;
  __device__ static __forceinline__ double from_raw(double h, float) { return h; }
  __device__ static __forceinline__ double load(const double* p, float) { return *p; }
  __device__ static __forceinline__ void store(double* p, double v, float) { *p = v; }
};
template <>
struct StoreTraits<__half> {
  using R = float;
  static constexpr bool dev = true;  // internal value = f - w
  // g from the stored value h (exact: the scale is a power of two)
  __device__ static __forceinline__ float from_raw(__half h, float inv_scale) {
    return __half2float(h) * inv_scale;
  }
  __device__ static __forceinline__ float load(const __half* p, float inv_scale) {
    return from_raw(*p, inv_scale);
  }
  // h = g * scale, rounded once
  __device__ static __forceinline__ void store(__half* p, float g, float scale) {
    *p = __float2half_rn(g * scale);
  }
  // h = g * scale, rounded stochastically (cvt.rs, sm_100a) as the `half`
  // (0 lower, 1 upper) element of a 16x2 conversion with random bits rbits
  __device__ static __forceinline__ void store_sr(__half* p, float g, float scale,
                                                  uint32_t rbits, int half) {
    const float x = g * scale;
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;"
        : "=r"(d)
        : "f"(half ? x : 0.0f), "f"(half ? 0.0f : x), "r"(rbits));
    *reinterpret_cast<unsigned short*>(p) = (unsigned short)(half ? d >> 16 : d & 0xffffu);
  }
};
template <>
struct StoreTraits<__nv_bfloat16> {
  using R = float;
  static constexpr bool dev = true;
  __device__ static __forceinline__ float from_raw(__nv_bfloat16 h, float inv_scale) {
    return __bfloat162float(h) * inv_scale;
  }
  __device__ static __forceinline__ float load(const __nv_bfloat16* p, float inv_scale) {
    return from_raw(*p, inv_scale);
  }
  __device__ static __forceinline__ void store(__nv_bfloat16* p, float g, float scale) {
    *p = __float2bfloat16_rn(g * scale);
  }
  __device__ static __forceinline__ void store_sr(__nv_bfloat16* p, float g, float scale,
                                                  uint32_t rbits, int half) {
    const float x = g * scale;
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;"
        : "=r"(d)
        : "f"(half ? x : 0.0f), "f"(half ? 0.0f : x), "r"(rbits));
    *reinterpret_cast<unsigned short*>(p) = (unsigned short)(half ? d >> 16 : d & 0xffffu);
  }
};

template <class R>
__host__ __device__ constexpr R weight(int q) {
  return wclass(q) == 0 ? R(1) / R(3) : (wclass(q) == 1 ? R(1) / R(18) : R(1) / R(36));
}

// ------------------------------------------------------------------ //
// Arithmetic over "lanes": the node arithmetic below is written once for
// V = float (one node per thread), V = double (the FP64 build) and V = F2
// (two neighbouring nodes per thread in one register pair, evaluated with
// the sm_100 packed FP32 instructions: one FFMA2 / FADD2 / FMUL2 does the
// work of two scalar instructions).
// ------------------------------------------------------------------ //
struct F2 {
  float2 v;
};
__host__ __device__ __forceinline__ F2 mk2(float a, float b) {
  F2 r;
  r.v = make_float2(a, b);
  return r;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
// a - b as a + b*(-1): the product is exact, so this rounds like a subtraction
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  return F2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)};
}
__device__ __forceinline__ F2 operator-(F2 a) { return mk2(-a.v.x, -a.v.y); }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return mk2(a.v.x / b.v.x, a.v.y / b.v.y); }

__host__ __device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
__host__ __device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ F2 fma_(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }

// 1/x and sqrt(x) of the FP32 lanes with the single-instruction PTX
// approximations (rcp.approx: at most 1 ulp; sqrt.approx: relative error
// below 2^-23) — the node arithmetic needs 2 reciprocals and 2 square roots
// and is issue-bound; the FP64 build keeps the IEEE operations.
__host__ __device__ __forceinline__ float vrcp(float a) {
#ifdef __CUDA_ARCH__
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
#else
  return 1.0f / a;
#endif
}
__host__ __device__ __forceinline__ double vrcp(double a) { return 1.0 / a; }
__device__ __forceinline__ F2 vrcp(F2 a) { return mk2(vrcp(a.v.x), vrcp(a.v.y)); }

__host__ __device__ __forceinline__ float vsqrt(float a) {
#ifdef __CUDA_ARCH__
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
#else
  return sqrtf(a);
#endif
}
__host__ __device__ __forceinline__ double vsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ F2 vsqrt(F2 a) { return mk2(vsqrt(a.v.x), vsqrt(a.v.y)); }

// broadcast a compile-time constant to a lane value (rounded once to the
// lane's precision, like a float literal)
template <class V>
__host__ __device__ __forceinline__ V bc(double c);
template <>
__host__ __device__ __forceinline__ float bc<float>(double c) { return (float)c; }
template <>
__host__ __device__ __forceinline__ double bc<double>(double c) { return c; }
template <>
__host__ __device__ __forceinline__ F2 bc<F2>(double c) { return mk2((float)c, (float)c); }

// broadcast a run-time scalar parameter to a lane value
template <class V, class T>
__host__ __device__ __forceinline__ V bcast_param(T x) {
  if constexpr (std::is_same<V, F2>::value) return mk2((float)x, (float)x);
  else return (V)x;
}

// acc + c*x for a small integer c (exact for |c| == 1)
template <int C, class V>
__host__ __device__ __forceinline__ V acc_term(V acc, V x) {
  if constexpr (C == 1) return acc + x;
  else if constexpr (C == -1) return acc - x;
  else return fma_(bc<V>(C), x, acc);
}
template <int C, class V>
__host__ __device__ __forceinline__ V first_term(V x) {
  if constexpr (C == 1) return x;
  else if constexpr (C == -1) return -x;
  else return bc<V>(C) * x;
}

// ------------------------------------------------------------------ //
// Macroscopic moments of the Macroscopic codelet
// (lbm_codelets.cpp:287-306): rho = sum f, u = (sum c f) / rho, summed in
// direction order so that the result is bit-identical to the codelet
// (the skipped terms are exact zeros, the +-1 products are exact).
// ------------------------------------------------------------------ //
template <class V>
__device__ __forceinline__ void macroscopic(const V (&f)[Q], V& rho, V& ux, V& uy, V& uz) {
  V d = f[0], jx, jy, jz;
  static_for<1, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    d = d + f[q];
    // first non-zero term of each component: q = 1 (x), 5 (y), 3 (z)
    if constexpr (cx(q) != 0) {
      if constexpr (q == 1) jx = f[q];
      else jx = acc_term<cx(q)>(jx, f[q]);
    }
    if constexpr (cy(q) != 0) {
      if constexpr (q == 5) jy = f[q];
      else jy = acc_term<cy(q)>(jy, f[q]);
    }
    if constexpr (cz(q) != 0) {
      if constexpr (q == 3) jz = -f[q];
      else jz = acc_term<cz(q)>(jz, f[q]);
    }
  });
  rho = d;
  ux = jx / d;
  uy = jy / d;
  uz = jz / d;
}

// ------------------------------------------------------------------ //
// MRT collision of Collision_MRT (lbm_codelets.cpp:449-544):
//   m = M f;  dm_k = s_k (m_k - meq_k);  f* = f - M^-1 dm
// with the d'Humieres equilibrium moments of lbm_codelets.cpp:468-486 and
// the relaxation rates of lbm_codelets.cpp:488-506 (s9,11,13,14,15 =
// 1/(tau + tau_eddy)).  Conserved moments (k = 0,3,5,7) have s_k = 0 and
// are skipped; M^-1 = M^T diag(1/|row|^2).
// ------------------------------------------------------------------ //
template <class R>
struct MrtParams {
  R rho0_inv;  // 1/RefDen
  R weps, wepsj, wxx;
  // deviation arithmetic: M_2 . w - weps = 3 - weps, the part of the
  // epsilon moment's difference m_2 - meq_2 that the deviations g do not
  // carry (0 for the standard weps = 3, and 0 when the populations are f)
  R e2c;
};


// ------------------------------------------------------------------ //
// Opposite-pair form of the node arithmetic.  With s_p = f_a + f_abar and
// d_p = f_a - f_abar for the nine pairs (a, abar = opp(a)), every even
// moment row of M (symmetric under c -> -c: rho, e, eps, the stress rows
// 9-15) reads only s, every odd row (momentum, energy flux, 16-18) only d,
// and the back transform M^T dm splits into a part E_p common to a and abar
// and a part O_p of opposite sign.  This is the same linear algebra as
// collide_mrt above with about half the operations.
// ------------------------------------------------------------------ //
__host__ __device__ constexpr int pair_a(int p) {
  constexpr int t[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
  return t[p];
}

// rho is the sum of the internal values (the density for populations f,
// rho - 1 for deviations g, as sum w = 1); rho_full is the density itself.
// j = sum c f = sum c g (sum c w = 0).
template <class V>
struct PairState {
  V f0, s[9], d[9];
  V rho, jx, jy, jz;  // sum of the internal values and momentum sum c f
  V rho_full;
};

// DEV: f holds deviations g = f - w (16-bit shifted storage)
template <class V, bool DEV = false>
__host__ __device__ __forceinline__ void make_pairs(const V (&f)[Q], PairState<V>& ps) {
  ps.f0 = f[0];
  static_for<0, 9>([&](auto pc) {
    constexpr int p = decltype(pc)::value;
    ps.s[p] = f[pair_a(p)] + f[opp(pair_a(p))];
    ps.d[p] = f[pair_a(p)] - f[opp(pair_a(p))];
  });
  // rho = f0 + sum s; j_alpha = sum_p c_alpha(a_p) d_p
  V acc = ps.s[0] + ps.s[1];
  acc = acc + ps.s[2];
  V diag = ps.s[3] + ps.s[4];
  diag = diag + ps.s[5];
  diag = diag + ps.s[6];
  diag = diag + ps.s[7];
  diag = diag + ps.s[8];
  ps.rho = ps.f0 + (acc + diag);
  if constexpr (DEV)
    ps.rho_full = ps.rho + bc<V>(1);
  else
    ps.rho_full = ps.rho;
  V jx = ps.d[0] + ps.d[3];
  jx = jx - ps.d[4];
  jx = jx + ps.d[5];
  ps.jx = jx - ps.d[6];
  V jy = ps.d[2] + ps.d[5];
  jy = jy + ps.d[6];
  jy = jy + ps.d[7];
  ps.jy = jy + ps.d[8];
  V jz = ps.d[8] - ps.d[1];
  jz = jz - ps.d[3];
  jz = jz - ps.d[4];
  ps.jz = jz - ps.d[7];
}

// Smagorinsky tau_eddy from the pair sums (same closed form as les_tau_eddy)
template <class V>
__host__ __device__ __forceinline__ V les_tau_eddy_pairs(const PairState<V>& ps, V ux, V uy, V uz,
                                                         V inv_rho, V tau, V les_c) {
  const V* s = ps.s;
  V pxx = s[0] + s[3];
  pxx = pxx + s[4];
  pxx = pxx + s[5];
  pxx = pxx + s[6];
  V pyy = s[2] + s[5];
  pyy = pyy + s[6];
  pyy = pyy + s[7];
  pyy = pyy + s[8];
  V pzz = s[1] + s[3];
  pzz = pzz + s[4];
  pzz = pzz + s[7];
  pzz = pzz + s[8];
  const V pxy = s[5] - s[6];  // f11 - f12 - f13 + f14
  const V pxz = s[4] - s[3];  // -f7 + f8 + f9 - f10
  const V pyz = s[8] - s[7];  // -f15 + f16 + f17 - f18
  const V r3 = ps.rho * bc<V>(1.0 / 3.0);
  const V txx = pxx - fma_(ps.jx, ux, r3);
  const V tyy = pyy - fma_(ps.jy, uy, r3);
  const V tzz = pzz - fma_(ps.jz, uz, r3);
  const V txy = pxy - ps.jx * uy;
  const V txz = pxz - ps.jx * uz;
  const V tyz = pyz - ps.jy * uz;
  V off = txy * txy;
  off = fma_(txz, txz, off);
  off = fma_(tyz, tyz, off);
  V qq = txx * txx;
  qq = fma_(tyy, tyy, qq);
  qq = fma_(tzz, tzz, qq);
  qq = fma_(bc<V>(2), off, qq);
  return fma_(bc<V>(0.5), vsqrt(fma_(tau, tau, (les_c * vsqrt(qq)) * inv_rho)),
              bc<V>(-0.5) * tau);
}

// SRT in pair form: feq_a, feq_abar share w rho (1 - 1.5u^2 + 4.5 (c.u)^2)
// and differ in the sign of 3 w rho c.u.  emit(q, value) receives every
// post-collision population.  FROM_PAIRS: rebuild f_a, f_abar from s, d
// (f is not read after make_pairs, which shortens its register lifetime);
// otherwise f is updated in place.
template <bool FROM_PAIRS, class V, bool DEV = false, class Emit>
__host__ __device__ __forceinline__ void collide_srt_pairs(const V (&f)[Q], const PairState<V>& ps,
                                                           V ux, V uy, V uz, V inv_tau,
                                                           Emit&& emit) {
  V usq = ux * ux;
  usq = fma_(uy, uy, usq);
  usq = fma_(uz, uz, usq);
  // DEV: feq - w = w (rho_int + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)) with
  // rho_int = rho - 1, so that no term of size w is formed
  const V c0 = DEV ? bc<V>(-1.5) * usq : fma_(bc<V>(-1.5), usq, bc<V>(1));
  const V rho = ps.rho_full;
  if constexpr (DEV)
    emit(IC<0>{}, fma_(bc<V>(1.0 / 3.0) * fma_(rho, c0, ps.rho) - ps.f0, inv_tau, ps.f0));
  else
    emit(IC<0>{}, fma_((rho * bc<V>(1.0 / 3.0)) * c0 - ps.f0, inv_tau, ps.f0));
  const V wr1 = rho * bc<V>(1.0 / 18.0), wr2 = rho * bc<V>(1.0 / 36.0);
  static_for<0, 9>([&](auto pc) {
    constexpr int p = decltype(pc)::value;
    constexpr int a = pair_a(p), b = opp(a);
    V eu;
    bool first = true;
    if constexpr (cx(a) != 0) {
      eu = first_term<cx(a)>(ux);
      first = false;
    }
    if constexpr (cy(a) != 0) {
      if (first) eu = first_term<cy(a)>(uy);
      else eu = acc_term<cy(a)>(eu, uy);
      first = false;
    }
    if constexpr (cz(a) != 0) {
      if (first) eu = first_term<cz(a)>(uz);
      else eu = acc_term<cz(a)>(eu, uz);
    }
    const V wr = wclass(a) == 1 ? wr1 : wr2;
    V even;
    if constexpr (DEV)
      even = bc<V>(wclass(a) == 1 ? 1.0 / 18.0 : 1.0 / 36.0) *
             fma_(rho, fma_(bc<V>(4.5) * eu, eu, c0), ps.rho);
    else
      even = wr * fma_(bc<V>(4.5) * eu, eu, c0);
    const V odd = (bc<V>(3) * wr) * eu;
    if constexpr (FROM_PAIRS) {
      // s* = s + (2 even - s) inv,  d* = d + (2 odd - d) inv
      const V ss = fma_(fma_(bc<V>(2), even, -ps.s[p]), inv_tau, ps.s[p]);
      const V dd = fma_(fma_(bc<V>(2), odd, -ps.d[p]), inv_tau, ps.d[p]);
      emit(IC<a>{}, bc<V>(0.5) * (ss + dd));
      emit(IC<b>{}, bc<V>(0.5) * (ss - dd));
    } else {
      emit(IC<a>{}, fma_((even + odd) - f[a], inv_tau, f[a]));
      emit(IC<b>{}, fma_((even - odd) - f[b], inv_tau, f[b]));
    }
  });
}

// MRT in pair form (Collision_MRT, lbm_codelets.cpp:449-544), moments
// formed from s/d, relaxation dm'_k = s_k (m_k - meq_k) / |row_k|^2, back
// transform f_a -= E_p + O_p, f_abar -= E_p - O_p (or, FROM_PAIRS, the same
// rebuilt from s - 2E and d - 2O).  emit(q, value) receives the results.
// DEV: f, s, d hold deviations g = f - w and ps.rho = rho - 1; every
// equilibrium moment but meq_2 is then the same expression in ps.rho (the
// rest state's moments M w are (1, -11, 3, 0, ...) and meq_1 = -11 rho + ...
// is linear in rho), meq_2 adds the constant p.e2c.
template <bool FROM_PAIRS, class V, class R, bool DEV = false, class Emit>
__host__ __device__ __forceinline__ void collide_mrt_pairs(const V (&f)[Q], const PairState<V>& ps,
                                                           V s_nu, const MrtParams<R>& p,
                                                           Emit&& emit) {
  const V* s = ps.s;
  const V* d = ps.d;
  const V rho = ps.rho, jx = ps.jx, jy = ps.jy, jz = ps.jz;
  const V rho0_inv = bcast_param<V>(p.rho0_inv);
  // ---- moments (rows of main.cpp:150-171 expressed in s, d) ----
  const V A = (s[0] + s[1]) + s[2];                                  // axis pairs
  const V B = ((((s[3] + s[4]) + s[5]) + s[6]) + s[7]) + s[8];       // diagonal pairs
  const V m1 = fma_(bc<V>(-30), ps.f0, fma_(bc<V>(-11), A, bc<V>(8) * B));
  const V m2 = fma_(bc<V>(12), ps.f0, fma_(bc<V>(-4), A, B));
  const V G = ((s[3] + s[4]) + s[5]) + s[6];                          // x-diagonals
  const V H = s[7] + s[8];                                             // yz-diagonals
  const V s12 = s[1] + s[2];
  const V GmH = fma_(bc<V>(-2), H, G);
  const V m9 = fma_(bc<V>(2), s[0], GmH - s12);
  const V m10 = fma_(bc<V>(-4), s[0], fma_(bc<V>(2), s12, GmH));
  const V K = (s[5] + s[6]) - (s[3] + s[4]);
  const V m11 = (s[2] - s[1]) + K;
  const V m12 = fma_(bc<V>(2), s[1] - s[2], K);
  const V m13 = s[5] - s[6];
  const V m14 = s[8] - s[7];
  const V m15 = s[4] - s[3];
  const V m4 = fma_(bc<V>(-5), d[0], jx);
  const V m6 = fma_(bc<V>(-5), d[2], jy);
  const V m8 = fma_(bc<V>(5), d[1], jz);
  const V m16 = ((d[4] - d[3]) + d[5]) - d[6];
  const V m17 = ((d[7] - d[5]) - d[6]) + d[8];
  const V m18 = ((d[7] - d[3]) - d[4]) - d[8];
  // ---- equilibrium moments (lbm_codelets.cpp:468-486) ----
  V jj = jx * jx;
  jj = fma_(jy, jy, jj);
  jj = fma_(jz, jz, jj);
  const V jj0 = jj * rho0_inv;
  const V jyy = jy * jy, jzz = jz * jz;
  const V meq9 = rho0_inv * fma_(bc<V>(2) * jx, jx, -(jyy + jzz));
  const V meq11 = rho0_inv * (jyy - jzz);
  // ---- relaxed, pre-scaled differences dm'_k = s_k (m_k - meq_k)/|row|^2 ----
  const V e1 = bc<V>(1.19 / 2394.0) * (m1 - fma_(bc<V>(19), jj0, bc<V>(-11) * rho));
  V e2;
  if constexpr (DEV)
    e2 = bc<V>(1.4 / 252.0) *
         ((m2 - fma_(bcast_param<V>(p.wepsj), jj0, bcast_param<V>(p.weps) * rho)) +
          bcast_param<V>(p.e2c));
  else
    e2 = bc<V>(1.4 / 252.0) *
         (m2 - fma_(bcast_param<V>(p.wepsj), jj0, bcast_param<V>(p.weps) * rho));
  const V e4 = bc<V>(1.2 / 40.0) * fma_(bc<V>(2.0 / 3.0), jx, m4);
  const V e6 = bc<V>(1.2 / 40.0) * fma_(bc<V>(2.0 / 3.0), jy, m6);
  const V e8 = bc<V>(1.2 / 40.0) * fma_(bc<V>(2.0 / 3.0), jz, m8);
  const V e9 = (s_nu * bc<V>(1.0 / 36.0)) * (m9 - meq9);
  const V e10 = bc<V>(1.4 / 72.0) * (m10 - bcast_param<V>(p.wxx) * meq9);
  const V e11 = (s_nu * bc<V>(1.0 / 12.0)) * (m11 - meq11);
  const V e12 = bc<V>(1.4 / 24.0) * (m12 - bcast_param<V>(p.wxx) * meq11);
  const V snu4 = s_nu * bc<V>(1.0 / 4.0);
  const V e13 = snu4 * (m13 - (jx * jy) * rho0_inv);
  const V e14 = snu4 * (m14 - (jy * jz) * rho0_inv);
  const V e15 = snu4 * (m15 - (jz * jx) * rho0_inv);
  const V e16 = bc<V>(1.98 / 8.0) * m16;
  const V e17 = bc<V>(1.98 / 8.0) * m17;
  const V e18 = bc<V>(1.98 / 8.0) * m18;
  // ---- back transform, f -= M^T dm' ----
  emit(IC<0>{}, ps.f0 - fma_(bc<V>(-30), e1, bc<V>(12) * e2));
  const V eax = fma_(bc<V>(-11), e1, bc<V>(-4) * e2);  // rows 1,2 on axis directions
  const V edg = fma_(bc<V>(8), e1, e2);                 // rows 1,2 on diagonals
  const V g910 = e9 + e10;
  const V g1112 = e11 + e12;
  const V ax_yz = fma_(bc<V>(2), e10, eax - e9);       // -e9 + 2 e10 + eax (z and y axes)
  const V dxz = edg + (g910 - g1112);                   // x-z diagonals share
  const V dxy = edg + (g910 + g1112);                   // x-y diagonals share
  const V dyz = fma_(bc<V>(-2), g910, edg);             // y-z diagonals share
  V E[9], O[9];
  E[0] = fma_(bc<V>(2), e9, fma_(bc<V>(-4), e10, eax));  // a=1
  O[0] = bc<V>(-4) * e4;
  E[1] = fma_(bc<V>(2), e12, ax_yz - e11);                // a=3 (0,0,-1)
  O[1] = bc<V>(4) * e8;
  E[2] = fma_(bc<V>(-2), e12, ax_yz + e11);               // a=5 (0,1,0)
  O[2] = bc<V>(-4) * e6;
  E[3] = dxz - e15;                                       // a=7 (1,0,-1)
  O[3] = ((e4 - e8) - e16) - e18;
  E[4] = dxz + e15;                                       // a=8 (-1,0,-1)
  O[4] = ((e16 - e4) - e8) - e18;
  E[5] = dxy + e13;                                       // a=11 (1,1,0)
  O[5] = ((e4 + e6) + e16) - e17;
  E[6] = dxy - e13;                                       // a=12 (-1,1,0)
  O[6] = ((e6 - e4) - e16) - e17;
  E[7] = dyz - e14;                                       // a=15 (0,1,-1)
  O[7] = ((e6 - e8) + e17) + e18;
  E[8] = dyz + e14;                                       // a=16 (0,1,1)
  O[8] = ((e6 + e8) + e17) - e18;
  static_for<0, 9>([&](auto pc) {
    constexpr int q = decltype(pc)::value;
    constexpr int a = pair_a(q), b = opp(a);
    if constexpr (FROM_PAIRS) {
      const V ss = fma_(bc<V>(-2), E[q], s[q]);
      const V dd = fma_(bc<V>(-2), O[q], d[q]);
      emit(IC<a>{}, bc<V>(0.5) * (ss + dd));
      emit(IC<b>{}, bc<V>(0.5) * (ss - dd));
    } else {
      emit(IC<a>{}, f[a] - (E[q] + O[q]));
      emit(IC<b>{}, f[b] - (E[q] - O[q]));
    }
  });
}

}  // namespace lbm
