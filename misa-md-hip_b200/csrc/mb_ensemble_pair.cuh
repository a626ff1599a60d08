// Per-pair FP32 arithmetic and interstitial items of the mixed-precision step,
// shared by the persistent tile kernel (mb_ensemble.cu) and the split kernels
// (mb_ensemble_split.cu, one lattice or many).
#pragma once

#include "mb_ensemble_kernel.cuh"

namespace mb {

// Spline knot and local coordinate of a pair from its deviation eps = r - R_k.
__device__ __forceinline__ void knot_of(const EnsParams &P, int s, int k, float eps, int &m, float &q) {
  const float2 kf = P.kf[s][k];
  const float t = kf.x + eps * P.rdr;
  const float fl = floorf(t);
  q = t - fl;
  m = min(max((int)(kf.y + fl), 0), P.P.nr - 2);
}

// Pair geometry shared by both passes (x and y in f32x2 lanes): returns false
// beyond the cutoff; on success r2 and the spline deviation numerator are set.
struct PairGeo {
  float2 dxy;
  float dz, r2, num;
};

// ALWAYS: also compute the numerator beyond the cutoff (branch-free walking).
template <bool ALWAYS>
__device__ __forceinline__ bool pair_geo(const EnsParams &P, const float4 &u, const float4 &nb, const float4 &C,
                                         PairGeo &g) {
  const float2 m1 = make_float2(-1.f, -1.f);
  const float2 exy = __ffma2_rn(make_float2(nb.x, nb.y), m1, make_float2(u.x, u.y)); // u - nb
  const float ez = u.z - nb.z;
  g.dxy = __fadd2_rn(make_float2(C.x, C.y), exy);
  g.dz = C.z + ez;
  const float2 sq = __fmul2_rn(g.dxy, g.dxy);
  g.r2 = sq.x + sq.y + g.dz * g.dz;
  const bool in = g.r2 < P.rc2f;
  if (!ALWAYS && !in) return false;
  const float2 pe = __fmul2_rn(__ffma2_rn(make_float2(2.f, 2.f), make_float2(C.x, C.y), exy), exy); // (2C + e) e
  g.num = pe.x + pe.y + (2.f * C.z + ez) * ez;
  return in;
}

// One density pair.  BF (branch-free): entries inside the cutoff for nearly every
// lane; the value is masked instead of branched around so iterations overlap.
template <bool BF>
__device__ __forceinline__ void rho_pair(const EnsParams &P, const float4 &u, const float4 &nb, const float4 &C, int s,
                                         int k, const float4 *s_fv, float &rs, float &rc) {
  PairGeo g;
  const bool in = pair_geo<BF>(P, u, nb, C, g);
  if (!BF && !in) return;
  const float r = g.r2 * rsqrtf(g.r2);
  int m;
  float q;
  knot_of(P, s, k, __fdividef(g.num, r + C.w), m, q);
  const float4 c = (m >= P.m_lo) ? s_fv[m - P.m_lo] : __ldg(&P.P.f_val32[m]);
  float v = ((c.w * q + c.z) * q + c.y) * q + c.x;
  if (BF) v = in ? v : 0.f;
  two_sum(rs, rc, v);
}

// Knuth two-sum on packed pairs of lanes (f32x2 instructions).
__device__ __forceinline__ void two_sum2(float2 &s, float2 &c, float2 x) {
  const float2 m1 = make_float2(-1.f, -1.f);
  const float2 t = __fadd2_rn(s, x);
  const float2 bp = __ffma2_rn(s, m1, t);                  // t - s
  const float2 sa = __ffma2_rn(__ffma2_rn(bp, m1, t), m1, s); // s - (t - bp)
  const float2 xb = __ffma2_rn(bp, m1, x);                  // x - bp
  c = __fadd2_rn(c, __fadd2_rn(sa, xb));
  s = t;
}

// One pair of the force pass: x and y components ride together in f32x2 lanes, and
// the derivative pieces of f and phi (stored as {f', phi'} pairs per knot) are
// evaluated by one packed Horner chain.
template <bool ENERGY, bool BF>
__device__ __forceinline__ void force_pair(const EnsParams &P, const float4 &u, const float4 &nb, const float4 &C,
                                           int s, int k, const float2 *s_fd, float2 &fxy_s, float2 &fxy_c, float &zs,
                                           float &zc, float &ps, float &pc) {
  PairGeo g;
  const bool in = pair_geo<BF>(P, u, nb, C, g);
  if (!BF && !in) return;
  const float r2 = g.r2, num = g.num, dz = g.dz;
  const float2 dxy = g.dxy;
  float rinv = rsqrtf(r2);
  rinv = rinv * (1.5f - 0.5f * r2 * rinv * rinv);
  const float r = r2 * rinv;
  int m;
  float q;
  knot_of(P, s, k, __fdividef(num, r + C.w), m, q);
  float2 c0, c1, c2;
  if (m >= P.m_lo) {
    const float2 *cp = s_fd + 3 * (m - P.m_lo);
    c0 = cp[0];
    c1 = cp[1];
    c2 = cp[2];
  } else {
    const float2 *cp = P.P.force32 + 3 * m;
    c0 = __ldg(cp);
    c1 = __ldg(cp + 1);
    c2 = __ldg(cp + 2);
  }
  const float2 qq = make_float2(q, q);
  const float2 dd = __ffma2_rn(__ffma2_rn(c2, qq, c1), qq, c0); // {f'(r), phi'(r)}
  float fpair = -((u.w + nb.w) * dd.x + dd.y) * rinv;
  if (BF) fpair = in ? fpair : 0.f;
  two_sum2(fxy_s, fxy_c, __fmul2_rn(dxy, make_float2(fpair, fpair)));
  two_sum(zs, zc, dz * fpair);
  if (ENERGY) {
    const float4 pv = __ldg(&P.P.phi_val32[m]);
    float e = 0.5f * (((pv.w * q + pv.z) * q + pv.y) * q + pv.x);
    if (BF) e = in ? e : 0.f;
    two_sum(ps, pc, e);
  }
}

// ------------------------------------------------------- interstitial items
// Sites flagged at the previous step of lattice d lose their flag (all CTAs share
// the old list); the count this step will fill starts at zero.  Counts alternate
// with the buffer parity: count[cur] is this step's list, count[cur ^ 1] the last.
__device__ __forceinline__ void itl_clear_flags(const LatDesc &d) {
  const int cur = d.cur;
  const int nold = min(d.flag_count[cur ^ 1], d.cap_flag);
  const int stride = gridDim.x * blockDim.x;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nold; k += stride) {
    const int idx = d.flag_list[k];
    d.code[idx] = (int8_t)(d.code[idx] & ~MB_FLAG_ITL);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.flag_count[cur] = 0;
}

// One warp flags the lattice sites within reach of interstitial `it`.  With
// `list` (this warp's MB_WIN_LIST entries of shared memory) the in-reach candidates are
// listed first and the lanes then flag only those.
__device__ __forceinline__ void itl_mark_one(const EnsParams &P, const LatDesc &d, int it, int *list = nullptr) {
  const Geom g = lat_geom(d);
  const int lane = threadIdx.x & 31;
  const int cur = d.cur;
  const double qx = d.ipx[cur][it], qy = d.ipy[cur][it], qz = d.ipz[cur][it];
  const Window w = make_window(qx, qy, qz, P.a0, P.reach);
  const int nlist = list ? window_compact(w, qx, qy, qz, P.a0, P.reach, list, MB_WIN_LIST) : -1;
  const int ncand = nlist >= 0 ? nlist : w.nx * w.ny * w.nz;
  for (int base = 0; base < ncand; base += 32) { // whole warp per round (warp_append)
    const int k = base + lane;
    long long idx = 0;
    bool fresh = false;
    double sx, sy, sz;
    if (k < ncand && window_site(g, w, nlist >= 0 ? list[k] : k, qx, qy, qz, P.a0, P.reach, idx, sx, sy, sz) &&
        d.code[idx] >= 0) {
      const uintptr_t addr = (uintptr_t)(d.code + idx);
      unsigned int *word = (unsigned int *)(addr & ~(uintptr_t)3);
      const unsigned int bit = (unsigned int)MB_FLAG_ITL << (8 * (addr & 3));
      fresh = !(atomicOr(word, bit) & bit);
    }
    // flag_count[2]: overflow, reported by the host
    warp_append(fresh, (int)idx, &d.flag_count[cur], d.flag_list, d.cap_flag, &d.flag_count[2]);
  }
}

// Coarse cell of a point of lattice d (wrapped into the box).
__device__ __forceinline__ void itl_cell3(const LatDesc &d, double x, double y, double z, int &cx, int &cy, int &cz) {
  const double fx = x / d.Lx - floor(x / d.Lx), fy = y / d.Ly - floor(y / d.Ly), fz = z / d.Lz - floor(z / d.Lz);
  cx = max(0, min((int)(fx * d.icn[0]), d.icn[0] - 1));
  cy = max(0, min((int)(fy * d.icn[1]), d.icn[1] - 1));
  cz = max(0, min((int)(fz * d.icn[2]), d.icn[2] - 1));
}

// Interstitial-pair part of an item: every interstitial within the 27 cells around the
// query point (the cells are at least cutoff + skin wide, so nothing in reach is left
// out), lane c walking cell c in list order; or the whole list when there is no cell
// list this step.  Each lane sums its own pairs in a fixed order.
template <bool CELLS, class Pair>
__device__ __forceinline__ void itl_pairs(const LatDesc &d, const Geom &g, int cur, double xi, double yi, double zi,
                                          int skip, int lane, Pair pair, bool with_df) {
  if (CELLS && d.icount && d.iflag[0]) {
    if (lane >= 27) return;
    int qx, qy, qz;
    itl_cell3(d, xi, yi, zi, qx, qy, qz);
    const int ox = lane % 3 - 1, oy = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
    const int cx = (qx + ox + d.icn[0]) % d.icn[0], cy = (qy + oy + d.icn[1]) % d.icn[1],
              cz = (qz + oz + d.icn[2]) % d.icn[2];
    const int c = (cz * d.icn[1] + cy) * d.icn[0] + cx;
    const int n = d.icount[c], s0 = d.istart[c];
    for (int j = s0; j < s0 + n; j++) {
      const int K = d.iitem[j];
      if (K == skip) continue;
      pair(min_image(xi - d.ipx[cur][K], g.Lx, g.iLx), min_image(yi - d.ipy[cur][K], g.Ly, g.iLy),
           min_image(zi - d.ipz[cur][K], g.Lz, g.iLz), d.itype[K], with_df ? d.idf[K] : 0.0);
    }
    return;
  }
  for (int K = lane; K < d.n_itl; K += 32) {
    if (K == skip) continue;
    pair(min_image(xi - d.ipx[cur][K], g.Lx, g.iLx), min_image(yi - d.ipy[cur][K], g.Ly, g.iLy),
         min_image(zi - d.ipz[cur][K], g.Lz, g.iLz), d.itype[K], with_df ? d.idf[K] : 0.0);
  }
}

// One FP64 pair of an interstitial item (atom of type ti, df dfi; partner of type tj, df
// dfj at pair vector d = own - partner): its density term into rho, or its force and pair
// energy into f and ep.  Pairs at or beyond the cutoff add nothing.
template <bool FORCE, bool ENERGY>
__device__ __forceinline__ void itl_pair(const EnsParams &P, int ti, double dfi, double dx, double dy, double dz,
                                         int tj, double dfj, double &rho, double &fx, double &fy, double &fz,
                                         double &ep) {
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (d2 >= P.rc2) return;
  const double rinv = rsqrt(d2);
  const double r = d2 * rinv;
  if (!FORCE) {
    rho += rho_of_r(P.P, tj, r);
  } else {
    double ph = 0.0;
    const double psip = pair_psip(P.P, ti, tj, r, dfi, dfj, ENERGY ? &ph : nullptr);
    const double fpair = -psip * rinv;
    fx += dx * fpair;
    fy += dy * fpair;
    fz += dz * fpair;
    if (ENERGY) ep += 0.5 * ph;
  }
}

// Last part of an item, on one lane, from its summed pairs: df (density pass), or force,
// velocity-Verlet, drift and ghost images (force pass), of a flagged site (i at s, cx, y,
// z) or of interstitial it.
template <bool FORCE, bool ENERGY>
__device__ __forceinline__ void itl_finish(const EnsParams &P, const LatDesc &d, const Geom &g, bool is_site,
                                           long long i, int s, int cx, int y, int z, int it, int ti, double xi,
                                           double yi, double zi, double rho, double fx, double fy, double fz,
                                           double ep) {
  const int cur = d.cur;
  if (!FORCE) {
    const double df = dF64(P.P, ti, rho);
    if (is_site) {
      float4 *uw = d.u4[cur];
      reinterpret_cast<float *>(uw + i)[3] = (float)df;
      d.rho[i] = (float)rho;
      for_images(g, s, cx, y, z,
                 [&](long long idx, double, double, double) { reinterpret_cast<float *>(uw + idx)[3] = (float)df; });
    } else {
      d.irho[it] = rho;
      d.idf[it] = df;
    }
    if (ENERGY) atomicAdd(&d.e_itl[0], F64(P.P, ti, rho));
    return;
  }
  double vx, vy, vz;
  if (is_site) {
    d.fx[i] = (float)fx;
    d.fy[i] = (float)fy;
    d.fz[i] = (float)fz;
    vx = d.vx[i];
    vy = d.vy[i];
    vz = d.vz[i];
  } else {
    d.ifx[it] = fx;
    d.ify[it] = fy;
    d.ifz[it] = fz;
    vx = d.ivx[it];
    vy = d.ivy[it];
    vz = d.ivz[it];
  }
  if (d.primed) {
    vx += P.h * fx;
    vy += P.h * fy;
    vz += P.h * fz;
  }
  if (ENERGY) {
    atomicAdd(&d.e_itl[0], ep);
    atomicAdd(&d.e_itl[1], 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E);
  }
  vx += P.h * fx;
  vy += P.h * fy;
  vz += P.h * fz;
  if (is_site) {
    d.vx[i] = vx;
    d.vy[i] = vy;
    d.vz[i] = vz;
    const double nx = d.ux[i] + P.dt * vx, ny = d.uy[i] + P.dt * vy, nz = d.uz[i] + P.dt * vz;
    d.ux[i] = nx;
    d.uy[i] = ny;
    d.uz[i] = nz;
    const float4 nu = make_float4((float)nx, (float)ny, (float)nz, 0.f);
    float4 *un = d.u4[cur ^ 1];
    un[i] = nu;
    ens_conv_check(P, d, s, cx, y, z, nx, ny, nz);
    for_images(g, s, cx, y, z, [&](long long idx, double, double, double) { un[idx] = nu; });
  } else {
    d.ivx[it] = vx;
    d.ivy[it] = vy;
    d.ivz[it] = vz;
    d.ipx[cur ^ 1][it] = xi + P.dt * vx;
    d.ipy[cur ^ 1][it] = yi + P.dt * vy;
    d.ipz[cur ^ 1][it] = zi + P.dt * vz;
  }
}

// Sum over the 8 lanes of a group (lanes 8g .. 8g + 7), in a fixed order.
__device__ __forceinline__ double group8_sum(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  return v;
}

// Pairs of interstitial it (position xi, yi, zi) with the lattice sites of its window,
// one warp, handed to pair (which sums them per lane).  With `list` (this warp's MB_WIN_LIST entries of shared
// memory) the in-reach sites are listed first and each lane then loads up to four of
// them at once; without it (or when more than MB_WIN_LIST sites are in reach) every
// candidate of the window is visited in rounds of 32.
template <class Pair>
__device__ __forceinline__ void itl_window_pairs(const EnsParams &P, const LatDesc &d, const Geom &g,
                                                 const float4 *u4, double xi, double yi, double zi, int *list,
                                                 bool with_df, Pair pair) {
  const int lane = threadIdx.x & 31;
  const Window win = make_window(xi, yi, zi, P.a0, P.reach);
  const int n = list ? window_compact(win, xi, yi, zi, P.a0, P.reach, list, MB_WIN_LIST) : -1;
  if (n >= 0) {
    for (int k0 = 0; k0 < n; k0 += 128) {
      long long j[4];
      double ox[4], oy[4], oz[4];
      bool ok[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int k = k0 + 32 * t + lane;
        j[t] = 0;
        ox[t] = oy[t] = oz[t] = 0.0;
        ok[t] = k < n && window_site_rel(g, win, list[k], xi, yi, zi, P.a0, P.reach, j[t], ox[t], oy[t], oz[t]);
      }
      int cj[4];
      float4 uj[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        cj[t] = ok[t] ? (int)d.code[j[t]] : -1;
        uj[t] = ok[t] ? u4[j[t]] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (cj[t] >= 0)
          pair(-(ox[t] + (double)uj[t].x), -(oy[t] + (double)uj[t].y), -(oz[t] + (double)uj[t].z), cj[t] & 0x3F,
               with_df ? (double)uj[t].w : 0.0);
    }
    return;
  }
  const int ncand = win.nx * win.ny * win.nz;
  for (int c = lane; c < ncand; c += 32) {
    long long j;
    double ox, oy, oz;
    if (!window_site_rel(g, win, c, xi, yi, zi, P.a0, P.reach, j, ox, oy, oz)) continue;
    const int cj = d.code[j];
    if (cj < 0) continue;
    const float4 uj = u4[j];
    pair(-(ox + (double)uj.x), -(oy + (double)uj.y), -(oz + (double)uj.z), cj & 0x3F, with_df ? (double)uj.w : 0.0);
  }
}

// Work of one warp on item w of lattice d: a flagged site (w < nflag) or an
// interstitial.  FORCE = false: density pass; true: force + integration pass.  A
// flagged site's lattice-pair part comes from the lattice kernels (rho / f of the site);
// its interstitial pairs, df, integration and ghost images are done here.  An
// interstitial's pairs (lattice window and other interstitials) are all done here, FP64.
// `list`: see itl_window_pairs.
template <bool FORCE, bool ENERGY, bool CELLS>
__device__ void itl_item(const EnsParams &P, const LatDesc &d, int w, int nflag, int *list = nullptr) {
  const int lane = threadIdx.x & 31;
  const Geom g = lat_geom(d);
  const int cur = d.cur;
  const float4 *u4 = d.u4[cur];
  const bool is_site = w < nflag;
  long long i = 0;
  int s = 0, cx = 0, y = 0, z = 0, it = 0, ti;
  double xi, yi, zi, dfi = 0.0;
  if (is_site) {
    i = d.flag_list[w];
    decode_ext(g, i, s, cx, y, z);
    ti = d.code[i] & 0x3F;
    double X, Y, Z;
    ideal_pos(s, cx, y, z, P.a0, X, Y, Z);
    xi = X + d.ux[i];
    yi = Y + d.uy[i];
    zi = Z + d.uz[i];
    if (FORCE) dfi = (double)u4[i].w;
  } else {
    it = w - nflag;
    ti = d.itype[it];
    xi = d.ipx[cur][it];
    yi = d.ipy[cur][it];
    zi = d.ipz[cur][it];
    if (FORCE) dfi = d.idf[it];
  }
  double acc0 = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, ep = 0.0;
  auto pair = [&](double dx, double dy, double dz, int tj, double dfj) {
    itl_pair<FORCE, ENERGY>(P, ti, dfi, dx, dy, dz, tj, dfj, acc0, fx, fy, fz, ep);
  };
  if (is_site) {
    // the lattice kernels summed this site's lattice pairs (FP32, compensated) into
    // rho / f; only the interstitial pairs are added here
    if (lane == 0) {
      if (FORCE) {
        fx = (double)d.fx[i];
        fy = (double)d.fy[i];
        fz = (double)d.fz[i];
      } else {
        acc0 = (double)d.rho[i];
      }
    }
  } else {
    itl_window_pairs(P, d, g, u4, xi, yi, zi, list, FORCE, pair);
  }
  itl_pairs<CELLS>(d, g, cur, xi, yi, zi, is_site ? -1 : it, lane, pair, FORCE);
  if (!FORCE) {
    acc0 = warp_sum(acc0);
  } else {
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    if (ENERGY) ep = warp_sum(ep);
  }
  if (lane == 0) itl_finish<FORCE, ENERGY>(P, d, g, is_site, i, s, cx, y, z, it, ti, xi, yi, zi, acc0, fx, fy, fz, ep);
}

// Flagged lattice site w of lattice d, worked by the 8-lane group of this lane (a warp
// works four sites at once; every lane of the warp takes part in the group sums, with a
// site or not): the lattice kernels summed its lattice pairs (FP32, compensated) into
// rho / f, the group adds its interstitial pairs in FP64 (lane l of the group walks cells
// l, l + 8, l + 16, l + 24 of the 27 around the site in the split kernels' cell list, or
// list entries l, l + 8, ... without one) and its first lane finishes the site.  A
// flagged site's item is a chain of dependent loads with little work, so four of them
// per warp keep four chains in flight.
template <bool FORCE, bool ENERGY>
__device__ void itl_site_group(const EnsParams &P, const LatDesc &d, int w, bool valid) {
  const int l8 = threadIdx.x & 7;
  const Geom g = lat_geom(d);
  const int cur = d.cur;
  long long i = 0;
  int s = 0, cx = 0, y = 0, z = 0, ti = 0;
  double xi = 0.0, yi = 0.0, zi = 0.0, dfi = 0.0;
  double acc0 = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, ep = 0.0;
  auto pair = [&](double dx, double dy, double dz, int tj, double dfj) {
    itl_pair<FORCE, ENERGY>(P, ti, dfi, dx, dy, dz, tj, dfj, acc0, fx, fy, fz, ep);
  };
  if (valid) {
    i = d.flag_list[w];
    decode_ext(g, i, s, cx, y, z);
    ti = d.code[i] & 0x3F;
    double X, Y, Z;
    ideal_pos(s, cx, y, z, P.a0, X, Y, Z);
    xi = X + d.ux[i];
    yi = Y + d.uy[i];
    zi = Z + d.uz[i];
    if (FORCE) dfi = (double)d.u4[cur][i].w;
    if (l8 == 0) {
      if (FORCE) {
        fx = (double)d.fx[i];
        fy = (double)d.fy[i];
        fz = (double)d.fz[i];
      } else {
        acc0 = (double)d.rho[i];
      }
    }
    if (d.icount && d.iflag[0]) {
      int qx, qy, qz;
      itl_cell3(d, xi, yi, zi, qx, qy, qz);
      for (int cc = l8; cc < 27; cc += 8) {
        const int ox = cc % 3 - 1, oy = (cc / 3) % 3 - 1, oz = cc / 9 - 1;
        const int ccx = (qx + ox + d.icn[0]) % d.icn[0], ccy = (qy + oy + d.icn[1]) % d.icn[1],
                  ccz = (qz + oz + d.icn[2]) % d.icn[2];
        const int c = (ccz * d.icn[1] + ccy) * d.icn[0] + ccx;
        const int n = d.icount[c], s0 = d.istart[c];
        for (int jj = s0; jj < s0 + n; jj++) {
          const int K = d.iitem[jj];
          pair(min_image(xi - d.ipx[cur][K], g.Lx, g.iLx), min_image(yi - d.ipy[cur][K], g.Ly, g.iLy),
               min_image(zi - d.ipz[cur][K], g.Lz, g.iLz), d.itype[K], FORCE ? d.idf[K] : 0.0);
        }
      }
    } else {
      for (int K = l8; K < d.n_itl; K += 8)
        pair(min_image(xi - d.ipx[cur][K], g.Lx, g.iLx), min_image(yi - d.ipy[cur][K], g.Ly, g.iLy),
             min_image(zi - d.ipz[cur][K], g.Lz, g.iLz), d.itype[K], FORCE ? d.idf[K] : 0.0);
    }
  }
  if (!FORCE) {
    acc0 = group8_sum(acc0);
  } else {
    fx = group8_sum(fx);
    fy = group8_sum(fy);
    fz = group8_sum(fz);
    if (ENERGY) ep = group8_sum(ep);
  }
  if (valid && l8 == 0)
    itl_finish<FORCE, ENERGY>(P, d, g, true, i, s, cx, y, z, 0, ti, xi, yi, zi, acc0, fx, fy, fz, ep);
}

// Items of every lattice that holds interstitials.  Split kernels (CELLS: their per-step
// interstitial cell list applies; `list`: this warp's window list): the interstitials
// first, one warp each, so that their window walks (the longest items) start at once,
// then the flagged sites four to a warp.  Persistent kernel: one item per warp, whole
// interstitial lists.
template <bool FORCE, bool ENERGY, bool CELLS = false>
__device__ void itl_items(const EnsParams &P, int *list = nullptr) {
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (!lat_active(d)) continue;
    const int nflag = min(d.flag_count[d.cur], d.cap_flag);
    if (CELLS) {
      const int n = d.n_itl + (nflag + 3) / 4;
      for (int w = gw; w < n; w += warps) {
        if (w < d.n_itl) {
          itl_item<FORCE, ENERGY, true>(P, d, nflag + w, nflag, list);
        } else {
          const int f = 4 * (w - d.n_itl) + (int)((threadIdx.x & 31) >> 3);
          itl_site_group<FORCE, ENERGY>(P, d, f, f < nflag);
        }
      }
    } else {
      const int n = nflag + d.n_itl;
      for (int w = gw; w < n; w += warps) itl_item<FORCE, ENERGY, false>(P, d, w, nflag);
    }
  }
}

} // namespace mb
