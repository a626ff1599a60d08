// Mixed-precision step as separate kernels (split mode).
//
// The persistent tile kernel (mb_ensemble.cu) keeps both passes, both spline tables
// and two TMA tile buffers resident, which caps it at 16 warps per SM.  Here the
// density pass and the force + velocity-Verlet pass are separate kernels, each holding
// only its own squared-distance table in shared memory and reading neighbour rows
// through L1, so each runs with 28-32 warps per SM.  Pair terms are FP32 (linear
// interpolation in s = r^2 of tables built from the FP64 spline, index from the small
// quantity r^2 - R^2) with two-sum accumulation; state and integration stay FP64.
// The kernels of one step (interstitial phases included) are captured into one CUDA
// graph by the ensemble host.  One large lattice is walked by bricks, many lattices by
// linear items (MxWalk).
#include <limits.h>

#include "mb_ensemble_kernel.cuh"
#include "mb_ensemble_pair.cuh"
#include "mb_ensemble_shells.cuh"

namespace mb {

#ifndef MX_RHO_THREADS
#define MX_RHO_THREADS 1024
#endif
#ifndef MX_FORCE_THREADS
#define MX_FORCE_THREADS 896 // 28 warps per SM at 72 registers; measured against 768 (80 registers,
                             // no spills) and 1024 (64, more spills): force pass 0.170 / 0.165 /
                             // 0.171 ns per atom on 128^3 cells
#endif
#define MX_SMEM_MAX (220 * 1024)

// n / d with m = floor((2^32 - 1) / d): multiply-high under-estimates by at most one.
__device__ __forceinline__ unsigned fdiv(unsigned n, unsigned d, unsigned m, unsigned &r) {
  unsigned q = __umulhi(n, m);
  r = n - q * d;
  if (r >= d) {
    q++;
    r -= d;
  }
  return q;
}

// Item it (0 .. W.bitems - 1) of brick `unit`: a row chunk of 32 sites, lane = x.
__device__ __forceinline__ bool mx_site(const LatDesc &d, const MxWalk &W, unsigned unit, unsigned it, int lane,
                                        int &s, int &cx, int &y, int &z, long long &i) {
  unsigned chunk, yb;
  const unsigned t = fdiv(unit, W.chunks, W.m_chunks, chunk);
  const unsigned zb = fdiv(t, W.nyb, W.m_nyb, yb);
  y = (int)(yb * W.by + it % W.by);
  s = (int)((it / W.by) & 1u);
  z = (int)(zb * W.bz + it / (2 * W.by));
  cx = (int)chunk * 32 + lane;
  if (cx >= d.bcx || y >= d.by || z >= d.bz) return false;
  i = (long long)s * d.E + ((long long)(z + 2) * d.ey + y + 2) * d.ecx + cx + 2;
  return true;
}

// ---------------------------------------------------------------- pair terms
// Geometry of one pair: e = u_i - u_j (displacements), d = C + e the pair vector and
// num = r^2 - R^2 = e . e + 2 C . e, exact to FP32 rounding of the small quantities.
// The table index is s / ds = R^2 / ds + num / ds: the large part is split on the
// host.  Entries are passed by value so that, in the unrolled loops, their fields
// are constant-bank operands of the arithmetic.
struct MxPair {
  float2 exy;
  float ez;
  float q;
  int m;
  bool in;
};

__device__ __forceinline__ MxPair mx_pair(const MxEntry E, float fr, float kb, float rds, float mmax,
                                          const float4 &u, const float4 &nb) {
  MxPair g;
  g.exy = __fadd2_rn(make_float2(u.x, u.y), make_float2(-nb.x, -nb.y));
  g.ez = u.z - nb.z;
  const float2 ee = __fmul2_rn(g.exy, g.exy);
  float num = fmaf(g.ez, g.ez, ee.x + ee.y);
  num = fmaf(E.t.x, g.exy.x, num);
  num = fmaf(E.t.y, g.exy.y, num);
  num = fmaf(E.t.z, g.ez, num);
  g.in = num < E.c.w;
  const float tt = fmaf(num, rds, fr);
  const float fl = floorf(tt);
  g.q = tt - fl;
  g.m = (int)fminf(fmaxf(fl + kb, 0.f), mmax);
  return g;
}

__device__ __forceinline__ float mx_rho_term(const MxEntry E, float rds, float mmax, const float4 &u,
                                             const float4 *base, const float2 *tab) {
  const float4 nb = __ldg(base + E.off);
  const MxPair g = mx_pair(E, E.t.w, E.kb, rds, mmax, u, nb);
  const float2 c = tab[g.m];
  const float v = fmaf(c.y, g.q, c.x);
  return g.in ? v : 0.f;
}

// Force term of one pair: fpair = -((df_i + df_j) A + B); returns fpair and the pair
// vector.
template <bool ENERGY>
__device__ __forceinline__ float mx_force_term(const MxEntry E, float rds, float mmax, const float4 &u,
                                               const float4 *base, const float2 *tab, const float4 *ptab,
                                               float2 &dxy, float &dz, float &e) {
  const float4 nb = __ldg(base + E.off);
  const MxPair g = mx_pair(E, E.fr_f, E.kb_f, rds, mmax, u, nb);
  const float2 ab = mx_ab(tab, g.m, g.q);
  const float fp = -fmaf(u.w + nb.w, ab.x, ab.y);
  dxy = make_float2(g.exy.x + E.c.x, g.exy.y + E.c.y);
  dz = g.ez + E.c.z;
  if (ENERGY) {
    const float4 p = __ldg(ptab + g.m);
    const float v = 0.5f * fmaf(fmaf(fmaf(p.w, g.q, p.z), g.q, p.y), g.q, p.x);
    e = g.in ? v : 0.f;
  }
  return g.in ? fp : 0.f;
}

// Site addressed by walk item `item` of this warp: brick walk (lattice `lat`) or linear
// walk (lattice found from item_first; `l`, `lo`, `hi` cache the current lattice).
struct MxAt {
  int l;
  unsigned lo, hi;
};

template <int WALK>
__device__ __forceinline__ bool mx_locate(const EnsParams &P, const MxWalk &W, int lat, unsigned item, int lane,
                                          MxAt &at, int &s, int &cx, int &y, int &z, long long &i) {
  if constexpr (WALK == 0) {
    at.l = lat;
    return mx_site(P.lats[lat], W, item / W.bitems, item % W.bitems, lane, s, cx, y, z, i);
  } else {
    if (item < at.lo || item >= at.hi) { // binary search of the owning lattice
      int a = 0, b = W.n_lats;
      while (b - a > 1) {
        const int m = (a + b) >> 1;
        if (__ldg(W.item_first + m) <= item)
          a = m;
        else
          b = m;
      }
      at.l = a;
      at.lo = __ldg(W.item_first + a);
      at.hi = __ldg(W.item_first + a + 1);
    }
    const LatDesc &d = P.lats[at.l];
    const unsigned plane_sites = (unsigned)(d.bcx * d.by), cpp = (plane_sites + 31u) / 32u;
    const unsigned j = item - at.lo;
    unsigned plane, chunk;
    if (W.lcb && plane_sites >= W.lmin) {
      // brick order (see MxWalk); the last z block and chunk block of a lattice are
      // shorter, so every item holds sites
      const unsigned per_zb = cpp * 2u * W.lbz, zb = j / per_zb, j1 = j - zb * per_zb;
      const unsigned nzp = 2u * min(W.lbz, (unsigned)d.bz - zb * W.lbz);
      const unsigned per_cb = W.lcb * nzp, cb = j1 / per_cb, j2 = j1 - cb * per_cb;
      const unsigned ncb = min(W.lcb, cpp - cb * W.lcb), p = j2 / ncb;
      plane = zb * 2u * W.lbz + p;
      chunk = cb * W.lcb + (j2 - p * ncb);
    } else {
      plane = j / cpp;
      chunk = j - plane * cpp;
    }
    const unsigned b = chunk * 32u + (unsigned)lane;
    if (b >= plane_sites) return false;
    s = (int)(plane & 1u);
    z = (int)(plane >> 1);
    y = (int)(b / (unsigned)d.bcx);
    cx = (int)(b - (unsigned)y * (unsigned)d.bcx);
    i = (long long)s * d.E + ((long long)(z + 2) * d.ey + y + 2) * d.ecx + cx + 2;
    return true;
  }
}

// Items of this block: bricks b, b + grid, ... (walk 0) or one contiguous range (walk 1).
template <int WALK>
__device__ __forceinline__ void mx_items(const MxWalk &W, unsigned &first, unsigned &count) {
  if constexpr (WALK == 0) {
    first = 0;
    count = 0;
  } else {
    const unsigned q = W.n_items / gridDim.x, r = W.n_items % gridDim.x;
    first = blockIdx.x * q + min(blockIdx.x, r);
    count = q + (blockIdx.x < r ? 1u : 0u);
  }
}

// Brick walk: the k-th item of this block (k = warp, warp + warps, ...) is item it of
// brick blockIdx.x + (k / W.bitems) * grid.  Returns the walk item or ~0u at the end.
template <int WALK>
__device__ __forceinline__ unsigned mx_next(const MxWalk &W, unsigned k, unsigned first, unsigned count) {
  if constexpr (WALK == 0) {
    const unsigned unit = blockIdx.x + (k / W.bitems) * gridDim.x;
    return unit < W.n_units ? unit * W.bitems + k % W.bitems : ~0u;
  } else {
    return k < count ? first + k : ~0u;
  }
}

// Strided views of lattice d for the built-in shells.
__device__ __forceinline__ MxSite mx_site_bases(const LatDesc &d, const float4 *u4, long long i, int s) {
  const long long E = d.E, d_odd = -2 * E + (long long)(d.ey + 1) * d.ecx + 1;
  return MxSite{u4 + i, u4 + i + E + (s ? d_odd : 0), d.ey * d.ecx, d.ecx};
}

// Density and df of one site; returns F(rho) for the energy.
// Site coordinates packed into one register across the pair loops: cx (11 bits),
// y (11), z (9), sublattice (1).
__device__ __forceinline__ unsigned mx_pack(int s, int cx, int y, int z) {
  return (unsigned)cx | ((unsigned)y << 11) | ((unsigned)z << 22) | ((unsigned)s << 31);
}
__device__ __forceinline__ void mx_unpack(unsigned p, int &s, int &cx, int &y, int &z) {
  cx = (int)(p & 2047u);
  y = (int)((p >> 11) & 2047u);
  z = (int)((p >> 22) & 511u);
  s = (int)(p >> 31);
}

// Margin (A^2) of the outer-entry masks over the pair test num < w: a pair the force
// pass finds inside the cutoff is in the mask whatever the FMA contraction of either
// pass.
#define MX_MASK_MARGIN 1e-3f

// near: bit k - 64 set when branch-walked built-in entry k (shells 7 and 8) is inside
// the cutoff (plus MX_MASK_MARGIN) for this site.
template <bool ENERGY, int FIXED>
__device__ __forceinline__ double mx_rho_site(const EnsParams &P, const MxStencil &S, const LatDesc &d,
                                              const float2 *s_f, float ma0, long long i, unsigned pos,
                                              unsigned long long &near) {
  const int s = (int)(pos >> 31);
  const int code = d.code[i];
  if (code < 0) return 0.0;
  const float4 *u4 = d.u4[d.cur];
  float4 *uw = d.u4[d.cur];
  const float4 u = __ldg(u4 + i);
  float rs = 0.f, rc = 0.f;
  if constexpr (FIXED) {
    const MxShells &Q = S.sh;
    const MxSite b = mx_site_bases(d, u4, i, s);
    constexpr int nbf = 64; // shells 1-6, walked without a branch; shells 7 (and 8) with one
    static_for<0, nbf / 2>([&](auto pc) {
      constexpr int k = 2 * decltype(pc)::value;
      two_sum(rs, rc, mxc_rho<k>(Q, ma0, b, u, s_f) + mxc_rho<k + 1>(Q, ma0, b, u, s_f));
    });
    static_for<nbf, kBcc.start[FIXED]>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      const float4 nb = mxc_load<k>(b);
      float2 exy;
      float ez, q;
      const float num = mxc_num<k>(ma0, u, nb, exy, ez);
      near |= (unsigned long long)(num < Q.w[HStore<k>::sh] + MX_MASK_MARGIN) << (k - nbf);
      if (num < Q.w[HStore<k>::sh]) {
        const int m = mxc_index<k, 0>(Q, num, q);
        const float2 t = s_f[m];
        two_sum(rs, rc, fmaf(t.y, q, t.x));
      }
    });
  } else {
    const float4 *be = u4 + i, *bo = u4 + i + (s ? S.d_odd : 0);
    const float rds = S.rds, mmax = (float)(S.n_rs - 1);
#pragma unroll
    for (int k = 0; k < MX_PAR_MAX; k += 2) {
      if (k >= S.n_odd) break;
      two_sum(rs, rc,
              mx_rho_term(S.odd[k], rds, mmax, u, bo, s_f) + mx_rho_term(S.odd[k + 1], rds, mmax, u, bo, s_f));
    }
#pragma unroll
    for (int k = 0; k < MX_PAR_MAX; k += 2) {
      if (k >= S.n_even) break;
      two_sum(rs, rc,
              mx_rho_term(S.even[k], rds, mmax, u, be, s_f) + mx_rho_term(S.even[k + 1], rds, mmax, u, be, s_f));
    }
    for (int k = 0; k < S.n_far; k++) {
      const MxEntry E = S.far[k];
      const float4 *bb = (E.odd & s) ? bo : be;
      const float4 nb = __ldg(bb + E.off);
      const MxPair g = mx_pair(E, E.t.w, E.kb, rds, mmax, u, nb);
      if (!g.in) continue;
      const float2 t = s_f[g.m];
      two_sum(rs, rc, fmaf(t.y, g.q, t.x));
    }
  }
  const double rho = (double)rs + (double)rc;
  d.rho[i] = (float)rho;
  if (code & MB_FLAG_ITL) return 0.0; // lattice part only: the interstitial items finish the site
  const double df = dF64(P.P, code & 0x3F, rho);
  reinterpret_cast<float *>(uw + i)[3] = (float)df;
  int sx, cx, y, z;
  mx_unpack(pos, sx, cx, y, z);
  const Geom g = lat_geom(d);
  for_images(g, sx, cx, y, z,
             [&](long long idx, double, double, double) { reinterpret_cast<float *>(uw + idx)[3] = (float)df; });
  return ENERGY ? F64(P.P, code & 0x3F, rho) : 0.0;
}

// Force + velocity-Verlet of one site; adds pair energy and kinetic energy.  Pair terms
// are added two at a time before one compensated add.
// outer: the branch-walked built-in entries (bit k - 64) that some site of this item has
// inside the cutoff at these positions (the density pass's masks); the others are not
// loaded.
template <bool ENERGY, int FIXED>
__device__ __forceinline__ void mx_force_site(const EnsParams &P, const MxStencil &S, const LatDesc &d,
                                              const float2 *s_ab, float ma0, long long i, unsigned pos,
                                              unsigned long long outer, double &e_pair, double &e_kin) {
  const int s = (int)(pos >> 31);
  const int code = d.code[i];
  if (code < 0) return;
  const float4 *u4 = d.u4[d.cur];
  float4 *un = d.u4[d.cur ^ 1];
  const float4 *ptab = P.P.ps32;
  const float4 u = __ldg(u4 + i);
  float2 fs = make_float2(0.f, 0.f), fc = fs;
  float zs = 0.f, zc = 0.f, ps = 0.f, pc = 0.f;
  auto add2 = [&](float2 d0, float z0, float f0, float e0, float2 d1, float z1, float f1, float e1) {
    two_sum2(fs, fc, __ffma2_rn(d1, make_float2(f1, f1), __fmul2_rn(d0, make_float2(f0, f0))));
    two_sum(zs, zc, fmaf(z1, f1, z0 * f0));
    if (ENERGY) two_sum(ps, pc, e0 + e1);
  };
  auto add1 = [&](float2 d0, float z0, float f0, float e0) {
    two_sum2(fs, fc, __fmul2_rn(d0, make_float2(f0, f0)));
    two_sum(zs, zc, z0 * f0);
    if (ENERGY) two_sum(ps, pc, e0);
  };
  if constexpr (FIXED) {
    const MxShells &Q = S.sh;
    const MxSite b = mx_site_bases(d, u4, i, s);
    constexpr int nbf = 64;
    static_for<0, nbf / 2>([&](auto pc2) {
      constexpr int k = 2 * decltype(pc2)::value;
      float2 d0, d1;
      float z0, z1, e0 = 0.f, e1 = 0.f;
      const float f0 = mxc_force<k, ENERGY>(Q, ma0, b, u, s_ab, ptab, d0, z0, e0);
      const float f1 = mxc_force<k + 1, ENERGY>(Q, ma0, b, u, s_ab, ptab, d1, z1, e1);
      add2(d0, z0, f0, e0, d1, z1, f1, e1);
    });
    static_for<nbf, kBcc.start[FIXED]>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      if ((outer >> (k - nbf)) & 1ull) {
        const float4 nb = mxc_load<k>(b);
        float2 exy;
        float ez;
        const float num = mxc_num<k>(ma0, u, nb, exy, ez);
        if (num < Q.w[HStore<k>::sh]) {
          float2 d0;
          float z0, e0 = 0.f;
          const float f0 = mxc_force<k, ENERGY>(Q, ma0, b, u, s_ab, ptab, d0, z0, e0);
          add1(d0, z0, f0, e0);
        }
      }
    });
  } else {
    const float4 *be = u4 + i, *bo = u4 + i + (s ? S.d_odd : 0);
    const float rds = S.rds_f, mmax = (float)(S.n_fs - 1);
    auto two = [&](const MxEntry E0, const MxEntry E1, const float4 *bb) {
      float2 d0, d1;
      float z0, z1, e0 = 0.f, e1 = 0.f;
      const float f0 = mx_force_term<ENERGY>(E0, rds, mmax, u, bb, s_ab, ptab, d0, z0, e0);
      const float f1 = mx_force_term<ENERGY>(E1, rds, mmax, u, bb, s_ab, ptab, d1, z1, e1);
      add2(d0, z0, f0, e0, d1, z1, f1, e1);
    };
#pragma unroll
    for (int k = 0; k < MX_PAR_MAX; k += 2) {
      if (k >= S.n_odd) break;
      two(S.odd[k], S.odd[k + 1], bo);
    }
#pragma unroll
    for (int k = 0; k < MX_PAR_MAX; k += 2) {
      if (k >= S.n_even) break;
      two(S.even[k], S.even[k + 1], be);
    }
    for (int k = 0; k < S.n_far; k++) {
      const MxEntry E = S.far[k];
      const float4 *bb = (E.odd & s) ? bo : be;
      const float4 nb = __ldg(bb + E.off);
      const MxPair g = mx_pair(E, E.fr_f, E.kb_f, rds, mmax, u, nb);
      if (!g.in) continue;
      float2 d0;
      float z0, e0 = 0.f;
      const float f0 = mx_force_term<ENERGY>(E, rds, mmax, u, bb, s_ab, ptab, d0, z0, e0);
      add1(d0, z0, f0, e0);
    }
  }
  const double fx = (double)fs.x + (double)fc.x;
  const double fy = (double)fs.y + (double)fc.y;
  const double fz = (double)zs + (double)zc;
  d.fx[i] = (float)fx;
  d.fy[i] = (float)fy;
  d.fz[i] = (float)fz;
  if (ENERGY) e_pair += (double)ps + (double)pc;
  if (code & MB_FLAG_ITL) return; // lattice part only: the interstitial items integrate the site
  double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
  if (d.primed) {
    vx += P.h * fx;
    vy += P.h * fy;
    vz += P.h * fz;
  }
  if (ENERGY) e_kin += 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
  vx += P.h * fx;
  vy += P.h * fy;
  vz += P.h * fz;
  const double nx = d.ux[i] + P.dt * vx, ny = d.uy[i] + P.dt * vy, nz = d.uz[i] + P.dt * vz;
  d.vx[i] = vx;
  d.vy[i] = vy;
  d.vz[i] = vz;
  d.ux[i] = nx;
  d.uy[i] = ny;
  d.uz[i] = nz;
  const float4 nu = make_float4((float)nx, (float)ny, (float)nz, 0.f);
  un[i] = nu;
  int sx, cx, y, z;
  mx_unpack(pos, sx, cx, y, z);
  ens_conv_check(P, d, sx, cx, y, z, nx, ny, nz);
  const Geom g = lat_geom(d);
  for_images(g, sx, cx, y, z, [&](long long idx, double, double, double) { un[idx] = nu; });
}

// Density pass.  FIXED: the built-in BCC shells (MxShells), else the runtime stencil
// (brick walk only).  Energy steps leave one {F(rho), 0} partial per walk item.
template <bool ENERGY, int FIXED, int WALK>
__global__ void __launch_bounds__(MX_RHO_THREADS, 1)
    k_mx_rho(const __grid_constant__ EnsParams P, const MxStencil S, int lat) {
  extern __shared__ float2 s_f[];
  for (int k = threadIdx.x; k < S.n_rs; k += blockDim.x) s_f[k] = P.P.fs32[k];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned nwarps = blockDim.x >> 5;
  const float ma0 = -S.sh.a0;
  unsigned first, count;
  mx_items<WALK>(S.walk, first, count);
  MxAt at{-1, 1u, 0u};
  for (unsigned k = threadIdx.x >> 5;; k += nwarps) {
    const unsigned item = mx_next<WALK>(S.walk, k, first, count);
    if (item == ~0u) break;
    int s = 0, cx = 0, y = 0, z = 0;
    long long i = 0;
    const bool ok = mx_locate<WALK>(P, S.walk, lat, item, lane, at, s, cx, y, z, i);
    const LatDesc &d = P.lats[at.l];
    double e = 0.0;
    unsigned long long near = 0;
    if (ok && lat_active(d)) e = mx_rho_site<ENERGY, FIXED>(P, S, d, s_f, ma0, i, mx_pack(s, cx, y, z), near);
    if (FIXED && P.outer) {
      const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)near);
      const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(near >> 32));
      if (lane == 0) P.outer[item] = make_uint2(lo, hi);
    }
    if (ENERGY) {
      e = warp_sum(e);
      if (lane == 0) P.epart[2 * (size_t)item] = e;
    }
  }
}

// Force + velocity-Verlet pass; energy steps add the pair energy to the item's partial
// and store its kinetic energy.
template <bool ENERGY, int FIXED, int WALK>
__global__ void __launch_bounds__(MX_FORCE_THREADS, 1)
    k_mx_force(const __grid_constant__ EnsParams P, const MxStencil S, int lat) {
  extern __shared__ float2 s_ab[];
  for (int k = threadIdx.x; k <= S.n_fs; k += blockDim.x) s_ab[k] = P.P.ab32[k];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned nwarps = blockDim.x >> 5;
  const float ma0 = -S.sh.a0;
  unsigned first, count;
  mx_items<WALK>(S.walk, first, count);
  MxAt at{-1, 1u, 0u};
  for (unsigned k = threadIdx.x >> 5;; k += nwarps) {
    const unsigned item = mx_next<WALK>(S.walk, k, first, count);
    if (item == ~0u) break;
    int s = 0, cx = 0, y = 0, z = 0;
    long long i = 0;
    const bool ok = mx_locate<WALK>(P, S.walk, lat, item, lane, at, s, cx, y, z, i);
    const LatDesc &d = P.lats[at.l];
    double ep = 0.0, ek = 0.0;
    unsigned long long outer = ~0ull;
    if (FIXED && P.outer) {
      const uint2 m2 = P.outer[item];
      outer = (unsigned long long)m2.x | ((unsigned long long)m2.y << 32);
    }
    if (ok && lat_active(d))
      mx_force_site<ENERGY, FIXED>(P, S, d, s_ab, ma0, i, mx_pack(s, cx, y, z), outer, ep, ek);
    if (ENERGY) {
      ep = warp_sum(ep);
      ek = warp_sum(ek);
      if (lane == 0) {
        P.epart[2 * (size_t)item] += ep;
        P.epart[2 * (size_t)item + 1] = ek;
      }
    }
  }
}

// Interstitial phases and step bookkeeping of split mode, one kernel each (the
// phases the persistent kernel separates with grid barriers).
__global__ void k_mx_itl_clear(const __grid_constant__ EnsParams P) {
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (lat_active(d)) itl_clear_flags(d);
  }
}

// Interstitial cell list of one lattice per CTA, from this step's positions: the counts
// of the previous build are cleared, (cell, index) keys sorted in shared memory, and each
// occupied cell gets its start and count.  The order (cell, index) does not depend on
// thread timing.
#define MX_BIN_THREADS 1024
__global__ void __launch_bounds__(MX_BIN_THREADS, 1) k_mx_itl_bin(const __grid_constant__ EnsParams P) {
  __shared__ long long key[MX_ICELL_MAX];
  const LatDesc &d = P.lats[P.itl_lats[blockIdx.x]];
  if (!lat_active(d) || !d.icount) return; // uniform per block
  const int tid = threadIdx.x, n = d.n_itl, cur = d.cur;
  const int nold = d.iflag[1];
  for (int k = tid; k < nold; k += blockDim.x) d.icount[d.icell_of[k]] = 0;
  __syncthreads();
  if (n > MX_ICELL_MAX) { // too many for the shared-memory sort: items walk the whole list
    if (tid == 0) {
      d.iflag[0] = 0;
      d.iflag[1] = 0;
    }
    return;
  }
  int n2 = 1;
  while (n2 < n) n2 <<= 1;
  for (int k = tid; k < n2; k += blockDim.x) {
    if (k < n) {
      int cx, cy, cz;
      itl_cell3(d, d.ipx[cur][k], d.ipy[cur][k], d.ipz[cur][k], cx, cy, cz);
      const int c = (cz * d.icn[1] + cy) * d.icn[0] + cx;
      d.icell_of[k] = c;
      key[k] = ((long long)c << 17) | (long long)k;
    } else {
      key[k] = LLONG_MAX;
    }
  }
  __syncthreads();
  if (n > 1) bitonic_sort(key, n2);
  for (int r = tid; r < n; r += blockDim.x) {
    const int c = (int)(key[r] >> 17);
    d.iitem[r] = (int)(key[r] & 0x1FFFF);
    if (r == 0 || (int)(key[r - 1] >> 17) != c) {
      int e = r + 1;
      while (e < n && (int)(key[e] >> 17) == c) e++;
      d.istart[c] = r;
      d.icount[c] = e - r;
    }
  }
  if (tid == 0) {
    d.iflag[0] = 1;
    d.iflag[1] = n;
  }
}

// The interstitial kernels run MX_ITL_THREADS threads per block; each warp keeps its list
// of in-reach window sites (window_compact) in shared memory.
#define MX_ITL_THREADS 256
__global__ void __launch_bounds__(MX_ITL_THREADS) k_mx_itl_mark(const __grid_constant__ EnsParams P) {
  __shared__ int s_list[MX_ITL_THREADS / 32][MB_WIN_LIST];
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (!lat_active(d)) continue;
    for (int it = gw; it < d.n_itl; it += warps) itl_mark_one(P, d, it, s_list[threadIdx.x >> 5]);
  }
}

template <bool FORCE, bool ENERGY>
__global__ void __launch_bounds__(MX_ITL_THREADS, 2) k_mx_itl_items(const __grid_constant__ EnsParams P) {
  __shared__ int s_list[MX_ITL_THREADS / 32][MB_WIN_LIST];
  itl_items<FORCE, ENERGY, true>(P, s_list[threadIdx.x >> 5]);
}

// Lattice <-> interstitial bookkeeping after the drift, one CTA per lattice that can
// hold interstitials (the FP64 path's k_convert64 does the same; see there): this
// step's candidates (box order) join the interstitial list and their sites become
// vacant in both float4 buffers; then interstitials within the recombination distance
// of a vacant site take it (lowest list index first) and the list is compacted in order.
#define MX_CONV_THREADS 1024
__global__ void __launch_bounds__(MX_CONV_THREADS, 1) k_mx_convert(const __grid_constant__ EnsParams P) {
  __shared__ long long key[MB_CAND_CAP];
  __shared__ unsigned removed[MB_CONV_ITL_MAX / 32];
  __shared__ int s_scan[MX_CONV_THREADS / 32];
  __shared__ int s_nclaim, s_base;
  LatDesc &d = const_cast<LatDesc &>(P.lats[P.itl_lats[blockIdx.x]]);
  if (!lat_active(d) || !d.cand) return; // uniform per block
  const int tid = threadIdx.x;
  const Geom g = lat_geom(d);
  const int c0 = d.cur, c1 = c0 ^ 1; // this step's buffer and the drifted one
  const int n0 = d.n_itl;
  const int nraw = *d.cand_n;
  const int nc = min(nraw, MB_CAND_CAP);
  int n2 = 1;
  while (n2 < nc) n2 <<= 1;
  for (int k = tid; k < n2; k += blockDim.x) key[k] = k < nc ? d.cand[k] : LLONG_MAX;
  __syncthreads();
  if (nc > 1) bitonic_sort(key, n2);
  const int nconv = min(nc, max(0, d.cap_itl - n0));
  const float4 vac = make_float4(ENS_VACANT, ENS_VACANT, ENS_VACANT, 0.f);
  for (int r = tid; r < nconv; r += blockDim.x) {
    const long long t = key[r];
    int s, cx, y, z;
    decode_box(g, t, s, cx, y, z);
    const long long i = ext_index(g, s, cx, y, z);
    const int k = n0 + r;
    double X, Y, Z;
    ideal_pos(s, cx, y, z, P.a0, X, Y, Z);
    const double ux = d.ux[i], uy = d.uy[i], uz = d.uz[i], vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
    d.ipx[c1][k] = X + ux;
    d.ipy[c1][k] = Y + uy;
    d.ipz[c1][k] = Z + uz;
    d.ipx[c0][k] = X + (ux - P.dt * vx); // the step's start (what a download reports)
    d.ipy[c0][k] = Y + (uy - P.dt * vy);
    d.ipz[c0][k] = Z + (uz - P.dt * vz);
    d.ivx[k] = vx;
    d.ivy[k] = vy;
    d.ivz[k] = vz;
    d.ifx[k] = (double)d.fx[i];
    d.ify[k] = (double)d.fy[i];
    d.ifz[k] = (double)d.fz[i];
    d.irho[k] = (double)d.rho[i];
    d.idf[k] = (double)d.u4[c0][i].w;
    d.itype[k] = (int8_t)(d.code[i] & 0x3F);
    d.iids[k] = d.ids[t];
    // vacant: far away in both float4 buffers (the pair loops reject vacancies by position)
    d.code[i] = -1;
    d.u4[c0][i] = vac;
    d.u4[c1][i] = vac;
    d.ux[i] = d.uy[i] = d.uz[i] = 0.0;
    d.vx[i] = d.vy[i] = d.vz[i] = 0.0;
    d.fx[i] = d.fy[i] = d.fz[i] = 0.f;
    for_images(g, s, cx, y, z, [&](long long idx, double, double, double) {
      d.code[idx] = -1;
      d.u4[c0][idx] = vac;
      d.u4[c1][idx] = vac;
    });
  }
  const int n1 = n0 + nconv;
  if (tid == 0) {
    d.conv_counters[0] += nconv;
    d.conv_counters[2] += nc - nconv;
    d.conv_counters[3] += nraw - nc;
    *d.cand_n = 0;
    s_nclaim = 0;
  }
  for (int w = tid; w < MB_CONV_ITL_MAX / 32; w += blockDim.x) removed[w] = 0u;
  __syncthreads();
  for (int k = tid; k < n1; k += blockDim.x) {
    const double qx = d.ipx[c1][k], qy = d.ipy[c1][k], qz = d.ipz[c1][k];
    double best = 1e300;
    long long gx = 0, gy = 0, gz = 0;
    int bs = 0;
    for (int sl = 0; sl < 2; sl++) {
      const double o = 0.5 * P.a0 * sl;
      const long long ax = llrint((qx - o) / P.a0), ay = llrint((qy - o) / P.a0), az = llrint((qz - o) / P.a0);
      const double X = 0.5 * P.a0 * (double)(2 * ax + sl), Y = P.a0 * ((double)ay + 0.5 * sl),
                   Z = P.a0 * ((double)az + 0.5 * sl);
      const double dd = (qx - X) * (qx - X) + (qy - Y) * (qy - Y) + (qz - Z) * (qz - Z);
      if (dd < best) {
        best = dd;
        gx = ax;
        gy = ay;
        gz = az;
        bs = sl;
      }
    }
    if (!(best < P.rec2)) continue;
    const int cx = pmod_int(gx, d.bcx), y = pmod_int(gy, d.by), z = pmod_int(gz, d.bz);
    if (d.code[ext_index(g, bs, cx, y, z)] >= 0) continue;
    const long long t = ((long long)z * d.by + y) * (2LL * d.bcx) + 2LL * cx + bs;
    const int slot = atomicAdd(&s_nclaim, 1);
    if (slot < MB_CAND_CAP) key[slot] = (t << 17) | (long long)k;
  }
  __syncthreads();
  const int ncl = min(s_nclaim, MB_CAND_CAP);
  n2 = 1;
  while (n2 < ncl) n2 <<= 1;
  for (int k = ncl + tid; k < n2; k += blockDim.x) key[k] = LLONG_MAX;
  __syncthreads();
  if (ncl > 1) bitonic_sort(key, n2);
  int nrec = 0;
  for (int r = tid; r < ncl; r += blockDim.x) {
    const long long t = key[r] >> 17;
    if (r > 0 && (key[r - 1] >> 17) == t) continue; // a lower list index took the site
    const int k = (int)(key[r] & 0x1FFFF);
    int s, cx, y, z;
    decode_box(g, t, s, cx, y, z);
    const long long i = ext_index(g, s, cx, y, z);
    double X, Y, Z;
    ideal_pos(s, cx, y, z, P.a0, X, Y, Z);
    const double ux = min_image(d.ipx[c1][k] - X, g.Lx, g.iLx), uy = min_image(d.ipy[c1][k] - Y, g.Ly, g.iLy),
                 uz = min_image(d.ipz[c1][k] - Z, g.Lz, g.iLz);
    const double pux = ux + (d.ipx[c0][k] - d.ipx[c1][k]), puy = uy + (d.ipy[c0][k] - d.ipy[c1][k]),
                 puz = uz + (d.ipz[c0][k] - d.ipz[c1][k]);
    const int8_t ty = d.itype[k];
    const float4 nu = make_float4((float)ux, (float)uy, (float)uz, 0.f);
    const float4 pu = make_float4((float)pux, (float)puy, (float)puz, (float)d.idf[k]);
    d.code[i] = ty;
    d.ux[i] = ux;
    d.uy[i] = uy;
    d.uz[i] = uz;
    d.vx[i] = d.ivx[k];
    d.vy[i] = d.ivy[k];
    d.vz[i] = d.ivz[k];
    d.fx[i] = (float)d.ifx[k];
    d.fy[i] = (float)d.ify[k];
    d.fz[i] = (float)d.ifz[k];
    d.rho[i] = (float)d.irho[k];
    d.u4[c1][i] = nu;
    d.u4[c0][i] = pu;
    d.ids[t] = d.iids[k];
    for_images(g, s, cx, y, z, [&](long long idx, double, double, double) {
      d.code[idx] = ty;
      d.u4[c1][idx] = nu;
      d.u4[c0][idx] = pu;
    });
    atomicOr(&removed[k >> 5], 1u << (k & 31));
    nrec++;
  }
  const double nrec_all = block_sum((double)nrec);
  if (tid == 0) {
    d.conv_counters[1] += (long long)nrec_all;
    s_base = 0;
  }
  __syncthreads();
  for (int q0 = 0; q0 < n1; q0 += blockDim.x) {
    const int k = q0 + tid;
    const bool keep = k < n1 && !((removed[k >> 5] >> (k & 31)) & 1u);
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) s_scan[wid] = __popc(ballot);
    __syncthreads();
    if (tid == 0) {
      int acc = s_base;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        const int c = s_scan[w];
        s_scan[w] = acc;
        acc += c;
      }
      s_base = acc;
    }
    __syncthreads();
    const int dst = s_scan[wid] + __popc(ballot & ((1u << lane) - 1u));
    double v[14];
    int8_t ty = 0;
    int64_t id = 0;
    if (keep) {
      v[0] = d.ipx[0][k], v[1] = d.ipy[0][k], v[2] = d.ipz[0][k], v[3] = d.ipx[1][k], v[4] = d.ipy[1][k];
      v[5] = d.ipz[1][k], v[6] = d.ivx[k], v[7] = d.ivy[k], v[8] = d.ivz[k], v[9] = d.ifx[k], v[10] = d.ify[k];
      v[11] = d.ifz[k], v[12] = d.irho[k], v[13] = d.idf[k];
      ty = d.itype[k];
      id = d.iids[k];
    }
    __syncthreads();
    if (keep && dst != k) {
      d.ipx[0][dst] = v[0], d.ipy[0][dst] = v[1], d.ipz[0][dst] = v[2], d.ipx[1][dst] = v[3], d.ipy[1][dst] = v[4];
      d.ipz[1][dst] = v[5], d.ivx[dst] = v[6], d.ivy[dst] = v[7], d.ivz[dst] = v[8], d.ifx[dst] = v[9];
      d.ify[dst] = v[10], d.ifz[dst] = v[11], d.irho[dst] = v[12], d.idf[dst] = v[13];
      d.itype[dst] = ty;
      d.iids[dst] = id;
    }
    __syncthreads();
  }
  if (tid == 0) d.n_itl = s_base;
}

__global__ void k_mx_bookkeeping(const __grid_constant__ EnsParams P) {
  for (int l = threadIdx.x; l < P.n_lats; l += blockDim.x) {
    LatDesc *d = const_cast<LatDesc *>(&P.lats[l]);
    if (!lat_active(*d)) continue;
    d->cur ^= 1;
    if (d->primed)
      d->steps_done++;
    else
      d->primed = 1;
  }
}

template <int FIXED, int WALK>
static int mx_set_attrs() {
  MB_CUDA(cudaFuncSetAttribute(k_mx_rho<false, FIXED, WALK>, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM_MAX));
  MB_CUDA(cudaFuncSetAttribute(k_mx_rho<true, FIXED, WALK>, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM_MAX));
  MB_CUDA(
      cudaFuncSetAttribute(k_mx_force<false, FIXED, WALK>, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM_MAX));
  MB_CUDA(cudaFuncSetAttribute(k_mx_force<true, FIXED, WALK>, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM_MAX));
  return MB_OK;
}

template <int FIXED, int WALK>
static void mx_pass(const EnsParams &P, const MxStencil &S, int lat, int energy, cudaStream_t s, int which,
                    size_t smem) {
  const int sms = device_sm_count();
  if (which == 0) {
    if (energy)
      k_mx_rho<true, FIXED, WALK><<<sms, MX_RHO_THREADS, smem, s>>>(P, S, lat);
    else
      k_mx_rho<false, FIXED, WALK><<<sms, MX_RHO_THREADS, smem, s>>>(P, S, lat);
  } else {
    if (energy)
      k_mx_force<true, FIXED, WALK><<<sms, MX_FORCE_THREADS, smem, s>>>(P, S, lat);
    else
      k_mx_force<false, FIXED, WALK><<<sms, MX_FORCE_THREADS, smem, s>>>(P, S, lat);
  }
}

static void mx_passes(const EnsParams &P, const MxStencil &S, int lat, int energy, cudaStream_t s, int which,
                      size_t smem) {
  if (S.walk.linear)
    S.fixed == 8 ? mx_pass<8, 1>(P, S, lat, energy, s, which, smem) : mx_pass<7, 1>(P, S, lat, energy, s, which, smem);
  else if (S.fixed == 8)
    mx_pass<8, 0>(P, S, lat, energy, s, which, smem);
  else if (S.fixed)
    mx_pass<7, 0>(P, S, lat, energy, s, which, smem);
  else
    mx_pass<0, 0>(P, S, lat, energy, s, which, smem);
}

// Per-lattice energies of an energy step: block l sums the partials of lattice l's items
// and adds its interstitial items.
__global__ void k_mx_energy(const LatDesc *lats, int n_lats, const unsigned *first, unsigned n_items,
                            const double *epart, double *out) {
  const int l = blockIdx.x;
  if (l >= n_lats) return;
  const unsigned a = first ? first[l] : 0u, b = first ? first[l + 1] : n_items;
  double pe = 0.0, ke = 0.0;
  for (unsigned t = a + threadIdx.x; t < b; t += blockDim.x) {
    pe += epart[2 * (size_t)t];
    ke += epart[2 * (size_t)t + 1];
  }
  pe = block_sum(pe);
  ke = block_sum(ke);
  if (threadIdx.x == 0) {
    out[2 * l] = pe + lats[l].e_itl[0];
    out[2 * l + 1] = ke + lats[l].e_itl[1];
  }
}

// One step of every active lattice.  ev (optional): events recorded around the density
// kernel (ev[0], ev[1]) and the force kernel (ev[2], ev[3]).  Energy steps also reduce
// the item partials into out[2 l], out[2 l + 1].
int mx_launch_step(const EnsParams &P, const MxStencil &S, int lat, int energy, cudaStream_t s, cudaEvent_t *ev,
                   double *out) {
  const int sms = device_sm_count();
  const size_t rho_smem = (size_t)S.n_rs * sizeof(float2), force_smem = (size_t)(S.n_fs + 1) * sizeof(float2);
  if (force_smem > MX_SMEM_MAX || rho_smem > MX_SMEM_MAX)
    return fail(MB_ERR_ARG, "squared-distance table larger than shared memory");
  if (S.walk.linear && !S.fixed) return fail(MB_ERR_STATE, "linear walk needs the built-in shells");
  static bool attr = false;
  if (!attr) {
    MB_TRY((mx_set_attrs<0, 0>()));
    MB_TRY((mx_set_attrs<7, 0>()));
    MB_TRY((mx_set_attrs<7, 1>()));
    MB_TRY((mx_set_attrs<8, 0>()));
    MB_TRY((mx_set_attrs<8, 1>()));
    attr = true;
  }
  const int itl_grid = 2 * sms;
  if (P.n_itl_lats > 0) {
    k_mx_itl_clear<<<itl_grid, 256, 0, s>>>(P);
    k_mx_itl_bin<<<P.n_itl_lats, MX_BIN_THREADS, 0, s>>>(P);
    k_mx_itl_mark<<<itl_grid, MX_ITL_THREADS, 0, s>>>(P);
  }
  if (ev) MB_CUDA(cudaEventRecord(ev[0], s));
  mx_passes(P, S, lat, energy, s, 0, rho_smem);
  if (ev) MB_CUDA(cudaEventRecord(ev[1], s));
  if (P.n_itl_lats > 0) {
    if (energy)
      k_mx_itl_items<false, true><<<itl_grid, MX_ITL_THREADS, 0, s>>>(P);
    else
      k_mx_itl_items<false, false><<<itl_grid, MX_ITL_THREADS, 0, s>>>(P);
  }
  if (ev) MB_CUDA(cudaEventRecord(ev[2], s));
  mx_passes(P, S, lat, energy, s, 1, force_smem);
  if (ev) MB_CUDA(cudaEventRecord(ev[3], s));
  if (P.n_itl_lats > 0) {
    if (energy)
      k_mx_itl_items<true, true><<<itl_grid, MX_ITL_THREADS, 0, s>>>(P);
    else
      k_mx_itl_items<true, false><<<itl_grid, MX_ITL_THREADS, 0, s>>>(P);
    if (P.conv2 > 0.0) k_mx_convert<<<P.n_itl_lats, MX_CONV_THREADS, 0, s>>>(P);
  }
  if (energy) {
    const int nl = S.walk.linear ? S.walk.n_lats : 1;
    k_mx_energy<<<nl, 256, 0, s>>>(S.walk.linear ? P.lats : P.lats + lat, nl,
                                   S.walk.linear ? S.walk.item_first : nullptr, S.walk.n_items, P.epart, out);
  }
  k_mx_bookkeeping<<<1, 128, 0, s>>>(P);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb
