// Mixed-precision, multi-lattice EAM timestep (see mb_ensemble_kernel.cuh for the
// phase structure and the precision scheme).
#include <math.h>

#include "mb_ensemble_kernel.cuh"

namespace mb {

// ------------------------------------------------------------- tile phases
struct TileCtx {
  char *buf[2];
  uint64_t *bar;
  unsigned phase; // bit b: parity of the next completion of buffer b
};

__device__ __forceinline__ bool tile_live(const EnsParams &P, int t) {
  return lat_active(P.lats[P.tile_lat[t]]);
}

// Thread 0 issues the TMA load of tile t into buffer b.
__device__ __forceinline__ void issue_tile(const EnsParams &P, TileCtx &T, int t, int b) {
  const int l = P.tile_lat[t];
  const LatDesc &d = P.lats[l];
  const int *sh = P.shape_dims[d.shape];
  const int ti = P.tile_idx[t];
  const int tx = ti % d.ntx, ty = (ti / d.ntx) % d.nty, tz = ti / (d.ntx * d.nty);
  mbar_expect_tx(&T.bar[b], (unsigned)sh[3]);
  tma_load_5d(T.buf[b], &P.tmaps[2 * l + d.cur], 0, tx * sh[0], ty * sh[1], tz * sh[2], 0, &T.bar[b]);
}

// All threads wait for buffer b with a bounded poll.  If any thread gives up, the
// whole CTA raises err, drains the copy once more (bounded) and reports false.
__device__ __forceinline__ bool wait_tile(const EnsParams &P, TileCtx &T, int b) {
  __shared__ int s_timeout;
  if (threadIdx.x == 0) s_timeout = 0;
  __syncthreads();
  const unsigned par = (T.phase >> b) & 1u;
  unsigned spins = 0;
  bool ok = true;
  while (!mbar_try_wait(&T.bar[b], par)) {
    if (++spins > ENS_WAIT_SPINS) {
      ok = false;
      break;
    }
  }
  if (!ok) s_timeout = 1;
  __syncthreads();
  if (s_timeout) {
    if (threadIdx.x == 0) {
      atomicExch(P.err, 2);
      unsigned again = 0;
      while (!mbar_try_wait(&T.bar[b], par) && ++again < ENS_WAIT_SPINS) {
      }
    }
    __syncthreads();
    return false;
  }
  T.phase ^= 1u << b;
  return true;
}

// Site of thread `tid` inside a tile of shape sh, and its indices.
struct SiteRef {
  bool valid;
  int s, x, y, z;      // tile-local
  int o;               // shared-memory index (float4 units)
  long long i;         // global ext index
  int bcx, by, bz;     // box coordinates (cx per sublattice)
};

__device__ __forceinline__ SiteRef site_of(const LatDesc &d, const int *sh, int ti, int tid) {
  SiteRef r;
  const int TX = sh[0], TY = sh[1], TZ = sh[2];
  const int per = TX * TY * TZ;
  r.s = tid / per;
  const int rem = tid - r.s * per;
  r.x = rem % TX;
  r.y = (rem / TX) % TY;
  r.z = rem / (TX * TY);
  const int tx = ti % d.ntx, ty = (ti / d.ntx) % d.nty, tz = ti / (d.ntx * d.nty);
  r.bcx = tx * TX + r.x;
  r.by = ty * TY + r.y;
  r.bz = tz * TZ + r.z;
  r.valid = r.s < 2 && r.bcx < d.bcx && r.by < d.by && r.bz < d.bz;
  const int TXH = TX + 4, TYH = TY + 4, TZH = TZ + 4;
  r.o = ((r.s * TZH + r.z + 2) * TYH + r.y + 2) * TXH + r.x + 2;
  r.i = (long long)r.s * d.E + ((long long)(r.bz + 2) * d.ey + r.by + 2) * d.ecx + r.bcx + 2;
  return r;
}

// Spline knot and local coordinate of a pair from its deviation eps = r - R_k.
__device__ __forceinline__ void knot_of(const EnsParams &P, int s, int k, float eps, int &m, float &q) {
  const float t = P.fk[s][k] + eps * P.rdr;
  const float fl = floorf(t);
  m = P.mk[s][k] + (int)fl;
  q = t - fl;
  if (m > P.P.nr - 2) {
    m = P.P.nr - 2;
    q = 1.0f;
  }
  if (m < 0) {
    m = 0;
    q = 0.0f;
  }
}

template <bool ENERGY>
__device__ void rho_tiles(const EnsParams &P, TileCtx &T, const float4 *s_fv, double *e_acc) {
  int b = 0;
  int t = blockIdx.x;
  if (t < P.n_tiles && threadIdx.x == 0 && tile_live(P, t)) issue_tile(P, T, t, 0);
  for (; t < P.n_tiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    if (tn < P.n_tiles && threadIdx.x == 0 && tile_live(P, tn)) issue_tile(P, T, tn, b ^ 1);
    if (tile_live(P, t)) {
      if (!wait_tile(P, T, b)) return;
      const LatDesc &d = P.lats[P.tile_lat[t]];
      const int *sh = P.shape_dims[d.shape];
      const SiteRef me = site_of(d, sh, P.tile_idx[t], threadIdx.x);
      const float4 *tile = reinterpret_cast<const float4 *>(T.buf[b]);
      double e_site = 0.0;
      if (me.valid) {
        const int code = d.code[me.i];
        if (code >= 0 && !(code & MB_FLAG_ITL)) {
          const float4 u = tile[me.o];
          const int *soff = P.soff[d.shape][me.s];
          float rs = 0.f, rc = 0.f;
#pragma unroll 4
          for (int k = 0; k < P.n_st; k++) {
            const float4 nb = tile[me.o + soff[k]];
            const float4 C = P.ck[me.s][k];
            const float ex = u.x - nb.x, ey = u.y - nb.y, ez = u.z - nb.z;
            const float dx = C.x + ex, dy = C.y + ey, dz = C.z + ez;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < P.rc2f) {
              const float num = 2.f * (C.x * ex + C.y * ey + C.z * ez) + (ex * ex + ey * ey + ez * ez);
              const float r = r2 * rsqrtf(r2);
              const float eps = __fdividef(num, r + C.w);
              int m;
              float q;
              knot_of(P, me.s, k, eps, m, q);
              const float4 c = (m >= P.m_lo) ? s_fv[m - P.m_lo] : __ldg(&P.P.f_val32[m]);
              two_sum(rs, rc, ((c.w * q + c.z) * q + c.y) * q + c.x);
            }
          }
          const double rho = (double)rs + (double)rc;
          const double df = dF64(P.P, code & 0x3F, rho);
          float4 *u4 = d.u4[d.cur];
          reinterpret_cast<float *>(u4 + me.i)[3] = (float)df;
          d.rho[me.i] = (float)rho;
          const Geom g = lat_geom(d);
          for_images(g, me.s, me.bcx, me.by, me.bz,
                     [&](long long idx, double, double, double) { reinterpret_cast<float *>(u4 + idx)[3] = (float)df; });
          if (ENERGY) e_site = F64(P.P, code & 0x3F, rho);
        }
      }
      if (ENERGY) {
        const double tsum = block_sum(e_site);
        if (threadIdx.x == 0) P.epart[2 * t] = tsum;
      }
    } else if (ENERGY && threadIdx.x == 0) {
      P.epart[2 * t] = 0.0;
    }
    __syncthreads(); // buffer b is free again
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    b ^= 1;
  }
  (void)e_acc;
}

template <bool ENERGY>
__device__ void force_tiles(const EnsParams &P, TileCtx &T, const float2 *s_fd) {
  int b = 0;
  int t = blockIdx.x;
  if (t < P.n_tiles && threadIdx.x == 0 && tile_live(P, t)) issue_tile(P, T, t, 0);
  for (; t < P.n_tiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    if (tn < P.n_tiles && threadIdx.x == 0 && tile_live(P, tn)) issue_tile(P, T, tn, b ^ 1);
    if (tile_live(P, t)) {
      if (!wait_tile(P, T, b)) return;
      const LatDesc &d = P.lats[P.tile_lat[t]];
      const int *sh = P.shape_dims[d.shape];
      const SiteRef me = site_of(d, sh, P.tile_idx[t], threadIdx.x);
      const float4 *tile = reinterpret_cast<const float4 *>(T.buf[b]);
      double e_pair = 0.0, e_kin = 0.0;
      if (me.valid) {
        const int code = d.code[me.i];
        if (code >= 0 && !(code & MB_FLAG_ITL)) {
          const float4 u = tile[me.o];
          const int *soff = P.soff[d.shape][me.s];
          float xs = 0.f, xc = 0.f, ys = 0.f, yc = 0.f, zs = 0.f, zc = 0.f, ps = 0.f, pc = 0.f;
#pragma unroll 2
          for (int k = 0; k < P.n_st; k++) {
            const float4 nb = tile[me.o + soff[k]];
            const float4 C = P.ck[me.s][k];
            const float ex = u.x - nb.x, ey = u.y - nb.y, ez = u.z - nb.z;
            const float dx = C.x + ex, dy = C.y + ey, dz = C.z + ez;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < P.rc2f) {
              const float num = 2.f * (C.x * ex + C.y * ey + C.z * ez) + (ex * ex + ey * ey + ez * ez);
              float rinv = rsqrtf(r2);
              rinv = rinv * (1.5f - 0.5f * r2 * rinv * rinv);
              const float r = r2 * rinv;
              const float eps = __fdividef(num, r + C.w);
              int m;
              float q;
              knot_of(P, me.s, k, eps, m, q);
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
              const float fd = (c2.x * q + c1.x) * q + c0.x;
              const float pd = (c2.y * q + c1.y) * q + c0.y;
              const float fpair = -((u.w + nb.w) * fd + pd) * rinv;
              two_sum(xs, xc, dx * fpair);
              two_sum(ys, yc, dy * fpair);
              two_sum(zs, zc, dz * fpair);
              if (ENERGY) {
                const float4 pv = __ldg(&P.P.phi_val32[m]);
                two_sum(ps, pc, 0.5f * (((pv.w * q + pv.z) * q + pv.y) * q + pv.x));
              }
            }
          }
          const double fx = (double)xs + (double)xc, fy = (double)ys + (double)yc, fz = (double)zs + (double)zc;
          const long long i = me.i;
          d.fx[i] = (float)fx;
          d.fy[i] = (float)fy;
          d.fz[i] = (float)fz;
          double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
          if (d.primed) {
            vx += P.h * fx;
            vy += P.h * fy;
            vz += P.h * fz;
          }
          if (ENERGY) {
            e_kin = 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
            e_pair = (double)ps + (double)pc;
          }
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
          float4 *un = d.u4[d.cur ^ 1];
          un[i] = nu;
          const Geom g = lat_geom(d);
          for_images(g, me.s, me.bcx, me.by, me.bz, [&](long long idx, double, double, double) { un[idx] = nu; });
        }
      }
      if (ENERGY) {
        const double t1 = block_sum(e_pair);
        const double t2 = block_sum(e_kin);
        if (threadIdx.x == 0) {
          P.epart[2 * t] += t1;
          P.epart[2 * t + 1] = t2;
        }
      }
    } else if (ENERGY && threadIdx.x == 0) {
      P.epart[2 * t + 1] = 0.0;
    }
    __syncthreads();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    b ^= 1;
  }
}

// ------------------------------------------------------- interstitial items
__device__ __forceinline__ void itl_mark_lattice(const EnsParams &P, const LatDesc &d) {
  const int nold = min(d.flag_count[0], d.cap_flag);
  for (int k = threadIdx.x; k < nold; k += blockDim.x) {
    const int idx = d.flag_list[k];
    d.code[idx] = (int8_t)(d.code[idx] & ~MB_FLAG_ITL);
  }
  __syncthreads();
  if (threadIdx.x == 0) d.flag_count[0] = 0;
  __syncthreads();
  const Geom g = lat_geom(d);
  const int lane = threadIdx.x & 31;
  const int cur = d.cur;
  for (int it = threadIdx.x >> 5; it < d.n_itl; it += blockDim.x >> 5) {
    const double qx = d.ipx[cur][it], qy = d.ipy[cur][it], qz = d.ipz[cur][it];
    const Window w = make_window(qx, qy, qz, P.a0, P.reach);
    const int ncand = w.nx * w.ny * w.nz;
    for (int c = lane; c < ncand; c += 32) {
      long long idx;
      double sx, sy, sz;
      if (!window_site(g, w, c, qx, qy, qz, P.a0, P.reach, idx, sx, sy, sz)) continue;
      if (d.code[idx] < 0) continue;
      const uintptr_t addr = (uintptr_t)(d.code + idx);
      unsigned int *word = (unsigned int *)(addr & ~(uintptr_t)3);
      const unsigned int bit = (unsigned int)MB_FLAG_ITL << (8 * (addr & 3));
      const unsigned int old = atomicOr(word, bit);
      if (!(old & bit)) {
        const int slot = atomicAdd(&d.flag_count[0], 1);
        if (slot < d.cap_flag)
          d.flag_list[slot] = (int)idx;
        else
          d.flag_count[1] = 1;
      }
    }
  }
  __syncthreads();
}

// Work of one warp on item w of lattice d: a flagged site (w < nflag) or an
// interstitial.  FORCE = false: density pass; true: force + integration pass.
template <bool FORCE, bool ENERGY>
__device__ void itl_item(const EnsParams &P, const LatDesc &d, int w, int nflag) {
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
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 >= P.rc2) return;
    const double rinv = rsqrt(d2);
    const double r = d2 * rinv;
    if (!FORCE) {
      acc0 += rho_of_r(P.P, tj, r);
    } else {
      double ph = 0.0;
      const double psip = pair_psip(P.P, ti, tj, r, dfi, dfj, ENERGY ? &ph : nullptr);
      const double fpair = -psip * rinv;
      fx += dx * fpair;
      fy += dy * fpair;
      fz += dz * fpair;
      if (ENERGY) ep += 0.5 * ph;
    }
  };
  if (is_site) {
    for (int k = lane; k < P.n_st; k += 32) {
      const char4 e = P.sd[s][k];
      const long long j = i + (long long)e.x * d.E + ((long long)e.w * d.ey + e.z) * d.ecx + e.y;
      const int cj = d.code[j];
      if (cj < 0) continue;
      double xj, yj, zj;
      lat_pos(d, u4, j, P.a0, xj, yj, zj);
      pair(xi - xj, yi - yj, zi - zj, cj & 0x3F, FORCE ? (double)u4[j].w : 0.0);
    }
  } else {
    const Window win = make_window(xi, yi, zi, P.a0, P.reach);
    const int ncand = win.nx * win.ny * win.nz;
    for (int c = lane; c < ncand; c += 32) {
      long long j;
      double sx, sy, sz;
      if (!window_site(g, win, c, xi, yi, zi, P.a0, P.reach, j, sx, sy, sz)) continue;
      const int cj = d.code[j];
      if (cj < 0) continue;
      double xj, yj, zj;
      lat_pos(d, u4, j, P.a0, xj, yj, zj);
      pair(xi - (xj + sx), yi - (yj + sy), zi - (zj + sz), cj & 0x3F, FORCE ? (double)u4[j].w : 0.0);
    }
  }
  for (int K = lane; K < d.n_itl; K += 32) {
    if (!is_site && K == it) continue;
    pair(min_image(xi - d.ipx[cur][K], d.Lx), min_image(yi - d.ipy[cur][K], d.Ly), min_image(zi - d.ipz[cur][K], d.Lz),
         d.itype[K], FORCE ? d.idf[K] : 0.0);
  }
  if (!FORCE) {
    acc0 = warp_sum(acc0);
    if (lane == 0) {
      const double df = dF64(P.P, ti, acc0);
      if (is_site) {
        float4 *uw = d.u4[cur];
        reinterpret_cast<float *>(uw + i)[3] = (float)df;
        d.rho[i] = (float)acc0;
        for_images(g, s, cx, y, z,
                   [&](long long idx, double, double, double) { reinterpret_cast<float *>(uw + idx)[3] = (float)df; });
      } else {
        d.irho[it] = acc0;
        d.idf[it] = df;
      }
      if (ENERGY) atomicAdd(&d.e_itl[0], F64(P.P, ti, acc0));
    }
    return;
  }
  fx = warp_sum(fx);
  fy = warp_sum(fy);
  fz = warp_sum(fz);
  if (ENERGY) ep = warp_sum(ep);
  if (lane != 0) return;
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

template <bool FORCE, bool ENERGY>
__device__ void itl_items(const EnsParams &P) {
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (!lat_active(d)) continue;
    const int nflag = min(d.flag_count[0], d.cap_flag);
    const int n = nflag + d.n_itl;
    for (int w = gw; w < n; w += warps) itl_item<FORCE, ENERGY>(P, d, w, nflag);
  }
}

// ------------------------------------------------------------------ kernel
template <bool ENERGY>
__global__ void __launch_bounds__(ENS_THREADS, 1) k_ens_step(const __grid_constant__ EnsParams P) {
  extern __shared__ __align__(128) char smem[];
  float4 *s_fv = reinterpret_cast<float4 *>(smem);
  float2 *s_fd = reinterpret_cast<float2 *>(smem + (size_t)P.nsm * sizeof(float4));
  const size_t tab_bytes = ((size_t)P.nsm * (sizeof(float4) + 3 * sizeof(float2)) + 127) & ~(size_t)127;
  TileCtx T;
  T.buf[0] = smem + tab_bytes;
  T.buf[1] = smem + tab_bytes + ENS_TILE_MAX_BYTES;
  T.bar = reinterpret_cast<uint64_t *>(smem + tab_bytes + 2 * ENS_TILE_MAX_BYTES);
  T.phase = 0;
  for (int k = threadIdx.x; k < P.nsm; k += blockDim.x) {
    s_fv[k] = P.P.f_val32[P.m_lo + k];
    s_fd[3 * k + 0] = P.P.force32[3 * (P.m_lo + k) + 0];
    s_fd[3 * k + 1] = P.P.force32[3 * (P.m_lo + k) + 1];
    s_fd[3 * k + 2] = P.P.force32[3 * (P.m_lo + k) + 2];
  }
  if (threadIdx.x == 0) {
    mbar_init(&T.bar[0], 1);
    mbar_init(&T.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // A: interstitial flags (one CTA per lattice with interstitials)
  if (P.n_itl_lats > 0) {
    for (int q = blockIdx.x; q < P.n_itl_lats; q += gridDim.x) {
      const LatDesc &d = P.lats[P.itl_lats[q]];
      if (lat_active(d)) itl_mark_lattice(P, d);
    }
    if (!grid_sync(P.bar, P.err)) return;
  }
  // B: density over lattice tiles
  rho_tiles<ENERGY>(P, T, s_fv, nullptr);
  if (!grid_sync(P.bar, P.err)) return;
  // C: density of flagged sites and interstitials
  if (P.n_itl_lats > 0) {
    itl_items<false, ENERGY>(P);
    if (!grid_sync(P.bar, P.err)) return;
  }
  // D + E: forces and integration
  force_tiles<ENERGY>(P, T, s_fd);
  if (P.n_itl_lats > 0) itl_items<true, ENERGY>(P);
  if (!grid_sync(P.bar, P.err)) return;
  // F: step bookkeeping
  if (blockIdx.x == 0) {
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
}

// Per-lattice energy of the last energy step: tiles in order, then the
// interstitial items; out[2 l] = pe, out[2 l + 1] = ke.
__global__ void k_ens_energy(const LatDesc *lats, int n_lats, const int *tile_first, const double *epart, double *out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n_lats) return;
  double pe = 0.0, ke = 0.0;
  for (int t = tile_first[l]; t < tile_first[l + 1]; t++) {
    pe += epart[2 * t];
    ke += epart[2 * t + 1];
  }
  out[2 * l] = pe + lats[l].e_itl[0];
  out[2 * l + 1] = ke + lats[l].e_itl[1];
}

size_t ens_smem_bytes(int nsm) {
  const size_t tab = ((size_t)nsm * (sizeof(float4) + 3 * sizeof(float2)) + 127) & ~(size_t)127;
  return tab + 2 * ENS_TILE_MAX_BYTES + 2 * sizeof(uint64_t);
}

int ens_launch(const EnsParams &P, int grid, cudaStream_t s) {
  const size_t smem = ens_smem_bytes(P.nsm);
  static bool attr = false;
  if (!attr) {
    MB_CUDA(cudaFuncSetAttribute(k_ens_step<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MB_CUDA(cudaFuncSetAttribute(k_ens_step<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(ENS_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (P.energy)
    MB_CUDA(cudaLaunchKernelEx(&cfg, k_ens_step<true>, P));
  else
    MB_CUDA(cudaLaunchKernelEx(&cfg, k_ens_step<false>, P));
  return MB_OK;
}

int ens_max_grid(int nsm) {
  int per_sm = 0;
  const size_t smem = ens_smem_bytes(nsm);
  if (cudaFuncSetAttribute(k_ens_step<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_step<false>, ENS_THREADS, smem) != cudaSuccess)
    return 0;
  return per_sm * device_sm_count();
}

int ens_energy_launch(const LatDesc *lats, int n, const int *tile_first, const double *epart, double *out,
                      cudaStream_t s) {
  k_ens_energy<<<(n + 127) / 128, 128, 0, s>>>(lats, n, tile_first, epart, out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb
