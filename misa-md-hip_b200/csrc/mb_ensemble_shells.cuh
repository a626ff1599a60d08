// Split-mode pair loops with the BCC neighbour shells built into the code.
//
// The neighbour vectors of a BCC site in half-lattice units h = (hx, hy, hz) (all odd
// or all even) are the same for every site and every lattice constant; only their
// count depends on (cutoff + skin) / a0.  With the first MX_SHELLS shells fixed at
// compile time, every per-vector quantity is an immediate: the storage offset
// (dz * plane + dy * row + dx, with the plane and row strides in registers), the
// products C . e (C = -(a0 / 2) h), and the unrolled loop needs no stencil table.
// Per-shell scalars (rc^2 - R^2 and the split table index of R^2) stay runtime values.
#pragma once

#include <utility>

#include "mb_ensemble_kernel.cuh"

namespace mb {

struct HVec {
  int hx, hy, hz, n2;
};
struct BccShells {
  HVec v[112];
  int start[MX_SHELLS + 1];
  int n2[MX_SHELLS];
};

constexpr BccShells make_bcc_shells() {
  BccShells t{};
  const int n2s[MX_SHELLS] = {3, 4, 8, 11, 12, 16, 19, 20};
  int n = 0;
  for (int s = 0; s < MX_SHELLS; s++) {
    t.start[s] = n;
    t.n2[s] = n2s[s];
    for (int hz = -5; hz <= 5; hz++)
      for (int hy = -5; hy <= 5; hy++)
        for (int hx = -5; hx <= 5; hx++) {
          const bool same = ((hx - hy) % 2 == 0) && ((hx - hz) % 2 == 0);
          if (same && hx * hx + hy * hy + hz * hz == n2s[s]) t.v[n++] = HVec{hx, hy, hz, n2s[s]};
        }
  }
  t.start[MX_SHELLS] = n;
  return t;
}
constexpr BccShells kBcc = make_bcc_shells();
static_assert(kBcc.start[7] == 88 && kBcc.start[8] == 112, "BCC shells 1-7 hold 88 vectors, 1-8 112");

constexpr int shell_of(int k) {
  int s = 0;
  while (kBcc.start[s + 1] <= k) s++;
  return s;
}

template <int K0, int K1, class F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (K0 < K1) {
    f(std::integral_constant<int, K0>{});
    static_for<K0 + 1, K1>(f);
  }
}

// Storage of neighbour vector K: parity class and (dx, dy, dz) cells from the class base
// (sublattice-0 site: even vectors stay, odd ones start at the other array).
template <int K>
struct HStore {
  static constexpr HVec h = kBcc.v[K];
  static constexpr bool odd = (h.hx & 1) != 0;
  static constexpr int dx = odd ? (h.hx - 1) / 2 : h.hx / 2;
  static constexpr int dy = odd ? (h.hy - 1) / 2 : h.hy / 2;
  static constexpr int dz = odd ? (h.hz - 1) / 2 : h.hz / 2;
  static constexpr int sh = shell_of(K);
};

// h . e with the integer components of h as immediates (zero terms dropped).
template <int HX, int HY, int HZ>
__device__ __forceinline__ float hdot(float ex, float ey, float ez) {
  float acc;
  if constexpr (HX != 0) {
    acc = (float)HX * ex;
    if constexpr (HY != 0) acc = fmaf((float)HY, ey, acc);
    if constexpr (HZ != 0) acc = fmaf((float)HZ, ez, acc);
  } else if constexpr (HY != 0) {
    acc = (float)HY * ey;
    if constexpr (HZ != 0) acc = fmaf((float)HZ, ez, acc);
  } else {
    acc = (float)HZ * ez;
  }
  return acc;
}

struct MxSite {
  const float4 *be, *bo; // class bases: even vectors, odd vectors
  int pl, rw;
};

template <int K>
__device__ __forceinline__ float4 mxc_load(const MxSite &b) {
  using T = HStore<K>;
  const float4 *base = T::odd ? b.bo : b.be;
  return __ldg(base + (T::dz * b.pl + T::dy * b.rw) + T::dx);
}

// num = r^2 - R^2 = |e|^2 - a0 (h . e), e = u_i - u_j (ma0 = -a0).
template <int K>
__device__ __forceinline__ float mxc_num(float ma0, const float4 &u, const float4 &nb, float2 &exy, float &ez) {
  using T = HStore<K>;
  exy = __fadd2_rn(make_float2(u.x, u.y), make_float2(-nb.x, -nb.y));
  ez = u.z - nb.z;
  const float2 ee = __fmul2_rn(exy, exy);
  const float e2 = fmaf(ez, ez, ee.x + ee.y);
  return fmaf(ma0, hdot<T::h.hx, T::h.hy, T::h.hz>(exy.x, exy.y, ez), e2);
}

// Table interval and local coordinate of vector K's pair on grid G (0 density, 1 force).
template <int K, int G>
__device__ __forceinline__ int mxc_index(const MxShells &Q, float num, float &q) {
  constexpr int sh = HStore<K>::sh;
  const float tt = fmaf(num, Q.g[G].rds, Q.g[G].fr[sh]);
  const float fl = floorf(tt);
  q = tt - fl;
  return (int)fminf(fmaxf(fl + Q.g[G].kb[sh], 0.f), Q.g[G].mmax);
}

template <int K>
__device__ __forceinline__ float mxc_rho(const MxShells &Q, float ma0, const MxSite &b, const float4 &u,
                                         const float2 *tab) {
  const float4 nb = mxc_load<K>(b);
  float2 exy;
  float ez, q;
  const float num = mxc_num<K>(ma0, u, nb, exy, ez);
  const int m = mxc_index<K, 0>(Q, num, q);
  const float2 t = tab[m];
  const float v = fmaf(t.y, q, t.x);
  return num < Q.w[HStore<K>::sh] ? v : 0.f;
}

// {A, B} = {f'(r)/r, phi'(r)/r} interpolated between the knots of interval m.
__device__ __forceinline__ float2 mx_ab(const float2 *tab, int m, float q) {
  const float2 k0 = tab[m], k1 = tab[m + 1];
  return __ffma2_rn(__fadd2_rn(k1, make_float2(-k0.x, -k0.y)), make_float2(q, q), k0);
}

// fpair and pair vector d = C + e of vector K (fpair 0 beyond the cutoff).
template <int K, bool ENERGY>
__device__ __forceinline__ float mxc_force(const MxShells &Q, float ma0, const MxSite &b, const float4 &u,
                                           const float2 *tab, const float4 *ptab, float2 &dxy, float &dz, float &e) {
  using T = HStore<K>;
  const float4 nb = mxc_load<K>(b);
  float2 exy;
  float ez, q;
  const float num = mxc_num<K>(ma0, u, nb, exy, ez);
  const float ha = 0.5f * ma0;
  const int m = mxc_index<K, 1>(Q, num, q);
  const float2 ab = mx_ab(tab, m, q);
  const float fp = -fmaf(u.w + nb.w, ab.x, ab.y);
  const bool in = num < Q.w[T::sh];
  dxy = make_float2(T::h.hx ? fmaf(ha, (float)T::h.hx, exy.x) : exy.x,
                    T::h.hy ? fmaf(ha, (float)T::h.hy, exy.y) : exy.y);
  dz = T::h.hz ? fmaf(ha, (float)T::h.hz, ez) : ez;
  if (ENERGY) {
    const float4 p = __ldg(ptab + m);
    const float v = 0.5f * fmaf(fmaf(fmaf(p.w, q, p.z), q, p.y), q, p.x);
    e = in ? v : 0.f;
  }
  return in ? fp : 0.f;
}

} // namespace mb
