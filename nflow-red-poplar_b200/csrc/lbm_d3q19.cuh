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
// FP64 build).  Shifted 16-bit formats hold (f - w) * scale.
// ------------------------------------------------------------------ //
template <class S>
struct StoreTraits;
template <>
struct StoreTraits<float> {
  using R = float;
  static constexpr bool shifted = false;
  __device__ static __forceinline__ float load(const float* p, float, float) { return *p; }
  __device__ static __forceinline__ void store(float* p, float v, float, float) { *p = v; }
};
template <>
struct StoreTraits<double> {
  using R = double;
  static constexpr bool shifted = false;
  __device__ static __forceinline__ double load(const double* p, double, double) { return *p; }
  __device__ static __forceinline__ void store(double* p, double v, double, double) { *p = v; }
};
template <>
struct StoreTraits<__half> {
  using R = float;
  static constexpr bool shifted = true;
  __device__ static __forceinline__ float load(const __half* p, float w, float inv_scale) {
    return fmaf(__half2float(*p), inv_scale, w);
  }
  __device__ static __forceinline__ void store(__half* p, float v, float w, float scale) {
    *p = __float2half_rn((v - w) * scale);
  }
};
template <>
struct StoreTraits<__nv_bfloat16> {
  using R = float;
  static constexpr bool shifted = true;
  __device__ static __forceinline__ float load(const __nv_bfloat16* p, float w, float inv_scale) {
    return fmaf(__bfloat162float(*p), inv_scale, w);
  }
  __device__ static __forceinline__ void store(__nv_bfloat16* p, float v, float w, float scale) {
    *p = __float2bfloat16_rn((v - w) * scale);
  }
};

template <class R>
__host__ __device__ constexpr R weight(int q) {
  return wclass(q) == 0 ? R(1) / R(3) : (wclass(q) == 1 ? R(1) / R(18) : R(1) / R(36));
}

// ------------------------------------------------------------------ //
// Macroscopic moments of the Macroscopic codelet
// (lbm_codelets.cpp:287-306): rho = sum f, u = (sum c f) / rho, summed in
// direction order so that the result is bit-identical to the codelet
// (the skipped terms are exact zeros, the +-1 products are exact).
// ------------------------------------------------------------------ //
template <class R>
__device__ __forceinline__ void macroscopic(const R (&f)[Q], R& rho, R& ux, R& uy, R& uz) {
  R d = f[0], jx = R(0), jy = R(0), jz = R(0);
  static_for<1, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    d = d + f[q];
    // first non-zero term of each component: q = 1 (x), 5 (y), 3 (z)
    if constexpr (cx(q) != 0) {
      if constexpr (q == 1) jx = f[q];
      else jx = cx(q) > 0 ? jx + f[q] : jx - f[q];
    }
    if constexpr (cy(q) != 0) {
      if constexpr (q == 5) jy = f[q];
      else jy = cy(q) > 0 ? jy + f[q] : jy - f[q];
    }
    if constexpr (cz(q) != 0) {
      if constexpr (q == 3) jz = -f[q];
      else jz = cz(q) > 0 ? jz + f[q] : jz - f[q];
    }
  });
  rho = d;
  ux = jx / d;
  uy = jy / d;
  uz = jz / d;
}

// ------------------------------------------------------------------ //
// Smagorinsky eddy relaxation time (ComputeTurbulence_LES,
// lbm_codelets.cpp:611-662).  The non-equilibrium momentum flux
// Pi = sum c c (f - feq) is formed from the raw second moments and the
// closed-form second moment of the D3Q19 equilibrium,
// sum c_a c_b feq = rho/3 delta_ab + rho u_a u_b.
//   tau_eddy = -tau/2 + 1/2 sqrt(tau^2 + 18 sqrt(2) Cs^2 sqrt(Pi:Pi) / rho)
// les_c = 18*sqrt(2)*Cs^2 (host constant).
// ------------------------------------------------------------------ //
template <class R>
__device__ __forceinline__ R les_tau_eddy(const R (&f)[Q], R rho, R ux, R uy, R uz, R tau, R les_c) {
  R pxx = R(0), pyy = R(0), pzz = R(0), pxy = R(0), pxz = R(0), pyz = R(0);
  static_for<1, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    if constexpr (cx(q) != 0) pxx += f[q];
    if constexpr (cy(q) != 0) pyy += f[q];
    if constexpr (cz(q) != 0) pzz += f[q];
    if constexpr (cx(q) * cy(q) != 0) pxy += (cx(q) * cy(q) > 0 ? f[q] : -f[q]);
    if constexpr (cx(q) * cz(q) != 0) pxz += (cx(q) * cz(q) > 0 ? f[q] : -f[q]);
    if constexpr (cy(q) * cz(q) != 0) pyz += (cy(q) * cz(q) > 0 ? f[q] : -f[q]);
  });
  const R r3 = rho * (R(1) / R(3));
  const R txx = pxx - r3 - rho * ux * ux;
  const R tyy = pyy - r3 - rho * uy * uy;
  const R tzz = pzz - r3 - rho * uz * uz;
  const R txy = pxy - rho * ux * uy;
  const R txz = pxz - rho * ux * uz;
  const R tyz = pyz - rho * uy * uz;
  const R qq = txx * txx + tyy * tyy + tzz * tzz + R(2) * (txy * txy + txz * txz + tyz * tyz);
  return R(-0.5) * tau + R(0.5) * sqrt(tau * tau + les_c * sqrt(qq) / rho);
}

// ------------------------------------------------------------------ //
// SRT collision of keCollision_SRT (kernel.cu:479-486):
//   f* = f - (f - feq)/(tau + tau_eddy),
//   feq = w rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2)
// ------------------------------------------------------------------ //
template <class R>
__device__ __forceinline__ void collide_srt(R (&f)[Q], R rho, R ux, R uy, R uz, R inv_tau) {
  const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    R eu = R(0);
    if constexpr (cx(q) != 0) eu = (cx(q) > 0 ? ux : -ux);
    if constexpr (cy(q) != 0) eu = eu + (cy(q) > 0 ? uy : -uy);
    if constexpr (cz(q) != 0) eu = eu + (cz(q) > 0 ? uz : -uz);
    const R feq = weight<R>(q) * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - usq15);
    f[q] = f[q] - (f[q] - feq) * inv_tau;
  });
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
};

template <int K>
__host__ __device__ constexpr bool mrt_relaxed() {
  return !(K == 0 || K == 3 || K == 5 || K == 7);
}

template <class R>
__device__ __forceinline__ R mrt_rate(int k, R s_nu) {
  // compile-time k in callers; the switch folds away
  switch (k) {
    case 1: return R(1.19);
    case 2: return R(1.4);
    case 4: case 6: case 8: return R(1.2);
    case 10: case 12: return R(1.4);
    case 16: case 17: case 18: return R(1.98);
    default: return s_nu;  // 9, 11, 13, 14, 15
  }
}

template <class R>
__device__ __forceinline__ void collide_mrt(R (&f)[Q], R rho, R ux, R uy, R uz, R s_nu,
                                            const MrtParams<R>& p) {
  const R jx = rho * ux, jy = rho * uy, jz = rho * uz;
  const R jj = jx * jx + jy * jy + jz * jz;
  const R meq9 = p.rho0_inv * (R(2) * jx * jx - (jy * jy + jz * jz));
  const R meq11 = p.rho0_inv * (jy * jy - jz * jz);
  R dm[Q];
  static_for<1, Q>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if constexpr (mrt_relaxed<k>()) {
      R m = R(0);
      bool first = true;
      static_for<0, Q>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        constexpr int c = mrt_m(k, j);
        if constexpr (c != 0) {
          if (first) {
            m = (c == 1) ? f[j] : (c == -1 ? -f[j] : R(c) * f[j]);
            first = false;
          } else {
            m = (c == 1) ? m + f[j] : (c == -1 ? m - f[j] : m + R(c) * f[j]);
          }
        }
      });
      R meq;
      if constexpr (k == 1) meq = R(-11) * rho + R(19) * p.rho0_inv * jj;
      if constexpr (k == 2) meq = p.weps * rho + p.wepsj * p.rho0_inv * jj;
      if constexpr (k == 4) meq = R(-2.0 / 3.0) * jx;
      if constexpr (k == 6) meq = R(-2.0 / 3.0) * jy;
      if constexpr (k == 8) meq = R(-2.0 / 3.0) * jz;
      if constexpr (k == 9) meq = meq9;
      if constexpr (k == 10) meq = p.wxx * meq9;
      if constexpr (k == 11) meq = meq11;
      if constexpr (k == 12) meq = p.wxx * meq11;
      if constexpr (k == 13) meq = jx * jy * p.rho0_inv;
      if constexpr (k == 14) meq = jy * jz * p.rho0_inv;
      if constexpr (k == 15) meq = jz * jx * p.rho0_inv;
      if constexpr (k >= 16) meq = R(0);
      dm[k] = mrt_rate<R>(k, s_nu) * (R(1) / R(mrt_norm2(k))) * (m - meq);
    }
  });
  static_for<0, Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    R acc = R(0);
    bool first = true;
    static_for<1, Q>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      constexpr int c = mrt_m(k, i);
      if constexpr (mrt_relaxed<k>() && c != 0) {
        if (first) {
          acc = (c == 1) ? dm[k] : (c == -1 ? -dm[k] : R(c) * dm[k]);
          first = false;
        } else {
          acc = (c == 1) ? acc + dm[k] : (c == -1 ? acc - dm[k] : acc + R(c) * dm[k]);
        }
      }
    });
    f[i] = f[i] - acc;
  });
}

}  // namespace lbm
