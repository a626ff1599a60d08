// Mixed-precision, multi-lattice EAM timestep (see mb_ensemble_kernel.cuh for the
// phase structure and the precision scheme).
#include <math.h>

#include "mb_ensemble_kernel.cuh"

namespace mb {

// ------------------------------------------------------------- tile phases
// Pipeline: two tiles in flight.  Every warp waits for its tile's full mbarrier,
// computes one site per thread and releases the buffer (empty mbarrier, one arrival
// per warp); lane 0 of warp 0 then loads tile i + 2 into that buffer once all warps
// released it.  No CTA-wide barrier per tile (except the energy reduction on energy
// steps).  Every wait is bounded.
struct TileCtx {
  char *buf[2];
  uint64_t *full;   // [2] completed by the TMA transaction count
  uint64_t *empty;  // [2] completed by ENS_CONSUMERS / 32 warp arrivals
  unsigned fphase;  // consumer: parity of the next full completion, bit per buffer
  unsigned ephase;  // producer: parity of the next empty completion, bit per buffer
  unsigned used;    // producer: buffers that have held a tile already
};

__device__ __forceinline__ bool tile_live(const EnsParams &P, int t) { return lat_active(P.lats[P.tile_lat[t]]); }

// Thread issuing the TMA load of tile t into buffer b.
__device__ __forceinline__ void issue_tile(const EnsParams &P, TileCtx &T, int t, int b) {
  const int l = P.tile_lat[t];
  const LatDesc &d = P.lats[l];
  const unsigned org = P.tile_org[t];
  mbar_expect_tx(&T.full[b], (unsigned)P.shape_dims[d.shape][3]);
  tma_load_5d(T.buf[b], &P.tmaps[2 * l + d.cur], 0, (int)(org & 2047u), (int)((org >> 11) & 2047u), (int)(org >> 22),
              0, &T.full[b]);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait on an mbarrier phase; raises err (code) when it gives up.
__device__ __forceinline__ void bounded_wait(const EnsParams &P, uint64_t *bar, unsigned parity, int code) {
  unsigned spins = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++spins > ENS_WAIT_SPINS) {
      atomicExch(P.err, code);
      // a second bounded wait lets a copy still in flight land before anyone moves on
      unsigned again = 0;
      while (!mbar_try_wait(bar, parity) && ++again < ENS_WAIT_SPINS) {
      }
      return;
    }
  }
}

// Producer role, held by lane 0 of warp 0: keeps two live tiles in flight.  Tile
// i + 2 goes into the buffer of tile i once every warp has released that buffer;
// warp 0 therefore paces the CTA while the other warps run ahead by up to a tile.
struct Producer {
  int next; // next tile index to consider
  int nb;   // buffer of the next issue
};

__device__ __forceinline__ void producer_start(const EnsParams &P, TileCtx &T, Producer &pr) {
  pr.next = blockIdx.x;
  pr.nb = 0;
}

__device__ __forceinline__ void producer_issue(const EnsParams &P, TileCtx &T, Producer &pr) {
  while (pr.next < P.n_tiles && !tile_live(P, pr.next)) pr.next += gridDim.x;
  if (pr.next >= P.n_tiles) return;
  if (threadIdx.x == 0) {
    if (T.used & (1u << pr.nb)) {
      bounded_wait(P, &T.empty[pr.nb], (T.ephase >> pr.nb) & 1u, 3);
      T.ephase ^= 1u << pr.nb;
    }
    T.used |= 1u << pr.nb;
    issue_tile(P, T, pr.next, pr.nb);
  }
  pr.next += gridDim.x;
  pr.nb ^= 1;
}

// Site of consumer thread `tid` inside a tile of shape sh, and its indices.
struct SiteRef {
  bool valid;
  int s, x, y, z;      // tile-local
  int o;               // shared-memory index (float4 units)
  long long i;         // global ext index
  int bcx, by, bz;     // box coordinates (cx per sublattice)
};

__device__ __forceinline__ SiteRef site_of(const LatDesc &d, const int *sh, const int *lg, unsigned org, int tid) {
  SiteRef r;
  const int TX = sh[0], TY = sh[1], TZ = sh[2];
  r.s = tid >> lg[3];
  const int rem = tid & ((1 << lg[3]) - 1);
  r.x = rem & (TX - 1);
  r.y = (rem >> lg[0]) & (TY - 1);
  r.z = rem >> (lg[0] + lg[1]);
  r.bcx = (int)(org & 2047u) + r.x;
  r.by = (int)((org >> 11) & 2047u) + r.y;
  r.bz = (int)(org >> 22) + r.z;
  r.valid = r.s < 2 && r.bcx < d.bcx && r.by < d.by && r.bz < d.bz;
  const int TXH = TX + 4, TYH = TY + 4, TZH = TZ + 4;
  r.o = ((r.s * TZH + r.z + 2) * TYH + r.y + 2) * TXH + r.x + 2;
  r.i = (long long)r.s * d.E + ((long long)(r.bz + 2) * d.ey + r.by + 2) * d.ecx + r.bcx + 2;
  return r;
}

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

template <bool ENERGY>
__device__ void rho_tiles(const EnsParams &P, TileCtx &T, const float4 *s_fv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int b = 0;
  Producer pr;
  producer_start(P, T, pr);
  if (warp == 0) {
    producer_issue(P, T, pr);
    producer_issue(P, T, pr);
  }
  for (int t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
    if (!tile_live(P, t)) {
      if (ENERGY && threadIdx.x == 0) P.epart[2 * t] = 0.0;
      continue;
    }
    bounded_wait(P, &T.full[b], (T.fphase >> b) & 1u, 2);
    T.fphase ^= 1u << b;
    const LatDesc &d = P.lats[P.tile_lat[t]];
    const SiteRef me = site_of(d, P.shape_dims[d.shape], P.shape_log[d.shape], P.tile_org[t], threadIdx.x);
    const float4 *tile = reinterpret_cast<const float4 *>(T.buf[b]);
    double e_site = 0.0;
    int code = -1;
    if (me.valid) code = d.code[me.i];
    const bool work = me.valid && code >= 0 && !(code & MB_FLAG_ITL);
    float rs0 = 0.f, rc0 = 0.f, rs1 = 0.f, rc1 = 0.f;
    if (work) {
      const float4 u = tile[me.o];
      const int *soff = P.soff[d.shape][me.s];
      const int n = P.n_st, nn = P.n_near;
      const int s = me.s;
      int k = 0;
      float rs2 = 0.f, rc2 = 0.f, rs3 = 0.f, rc3 = 0.f;
      for (; k + 3 < nn; k += 4) {
        const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
        const float4 nb2 = tile[me.o + soff[k + 2]], nb3 = tile[me.o + soff[k + 3]];
        rho_pair<true>(P, u, nb0, P.ck[s][k], s, k, s_fv, rs0, rc0);
        rho_pair<true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fv, rs1, rc1);
        rho_pair<true>(P, u, nb2, P.ck[s][k + 2], s, k + 2, s_fv, rs2, rc2);
        rho_pair<true>(P, u, nb3, P.ck[s][k + 3], s, k + 3, s_fv, rs3, rc3);
      }
      two_sum(rs0, rc0, rs2);
      two_sum(rs1, rc1, rs3);
      rc0 += rc2;
      rc1 += rc3;
      for (; k + 1 < nn; k += 2) {
        const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
        rho_pair<true>(P, u, nb0, P.ck[s][k], s, k, s_fv, rs0, rc0);
        rho_pair<true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fv, rs1, rc1);
      }
      if (k < nn) {
        rho_pair<true>(P, u, tile[me.o + soff[k]], P.ck[s][k], s, k, s_fv, rs0, rc0);
        k++;
      }
      for (; k + 1 < n; k += 2) {
        const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
        rho_pair<false>(P, u, nb0, P.ck[s][k], s, k, s_fv, rs0, rc0);
        rho_pair<false>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fv, rs1, rc1);
      }
      if (k < n) rho_pair<false>(P, u, tile[me.o + soff[k]], P.ck[s][k], s, k, s_fv, rs0, rc0);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&T.empty[b]); // tile data no longer needed by this warp
    if (warp == 0) producer_issue(P, T, pr);  // tile i + 2 into this buffer
    if (work) {
      const double rho = ((double)rs0 + (double)rs1) + ((double)rc0 + (double)rc1);
      const double df = dF64(P.P, code & 0x3F, rho);
      float4 *u4 = d.u4[d.cur];
      reinterpret_cast<float *>(u4 + me.i)[3] = (float)df;
      d.rho[me.i] = (float)rho;
      const Geom g = lat_geom(d);
      for_images(g, me.s, me.bcx, me.by, me.bz,
                 [&](long long idx, double, double, double) { reinterpret_cast<float *>(u4 + idx)[3] = (float)df; });
      if (ENERGY) e_site = F64(P.P, code & 0x3F, rho);
    }
    if (ENERGY) {
      const double tsum = block_sum(e_site);
      if (threadIdx.x == 0) P.epart[2 * t] = tsum;
    }
    (void)warp;
    b ^= 1;
  }
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

template <bool ENERGY>
__device__ void force_tiles(const EnsParams &P, TileCtx &T, const float2 *s_fd) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int b = 0;
  Producer pr;
  producer_start(P, T, pr);
  if (warp == 0) {
    producer_issue(P, T, pr);
    producer_issue(P, T, pr);
  }
  for (int t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
    if (!tile_live(P, t)) {
      if (ENERGY && threadIdx.x == 0) P.epart[2 * t + 1] = 0.0;
      continue;
    }
    bounded_wait(P, &T.full[b], (T.fphase >> b) & 1u, 2);
    T.fphase ^= 1u << b;
    const LatDesc &d = P.lats[P.tile_lat[t]];
    const SiteRef me = site_of(d, P.shape_dims[d.shape], P.shape_log[d.shape], P.tile_org[t], threadIdx.x);
    const float4 *tile = reinterpret_cast<const float4 *>(T.buf[b]);
    double e_pair = 0.0, e_kin = 0.0;
    int code = -1;
    double vx = 0, vy = 0, vz = 0, ux = 0, uy = 0, uz = 0;
    if (me.valid) {
      code = d.code[me.i];
      // own-site master state, fetched early so its latency hides behind the pair loop
      vx = d.vx[me.i];
      vy = d.vy[me.i];
      vz = d.vz[me.i];
      ux = d.ux[me.i];
      uy = d.uy[me.i];
      uz = d.uz[me.i];
    }
    const bool work = me.valid && code >= 0 && !(code & MB_FLAG_ITL);
    float2 fs0 = make_float2(0.f, 0.f), fc0 = fs0, fs1 = fs0, fc1 = fs0;
    float zs0 = 0.f, zc0 = 0.f, ps0 = 0.f, pc0 = 0.f, zs1 = 0.f, zc1 = 0.f, ps1 = 0.f, pc1 = 0.f;
    if (work) {
      const float4 u = tile[me.o];
      const int *soff = P.soff[d.shape][me.s];
      const int n = P.n_st, nn = P.n_near;
      const int s = me.s;
      int k = 0;
      {
        float2 fs2 = make_float2(0.f, 0.f), fc2 = fs2, fs3 = fs2, fc3 = fs2;
        float zs2 = 0.f, zc2 = 0.f, ps2 = 0.f, pc2 = 0.f, zs3 = 0.f, zc3 = 0.f, ps3 = 0.f, pc3 = 0.f;
        for (; k + 3 < nn; k += 4) {
          const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
          const float4 nb2 = tile[me.o + soff[k + 2]], nb3 = tile[me.o + soff[k + 3]];
          force_pair<ENERGY, true>(P, u, nb0, P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
          force_pair<ENERGY, true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fd, fs1, fc1, zs1, zc1, ps1, pc1);
          force_pair<ENERGY, true>(P, u, nb2, P.ck[s][k + 2], s, k + 2, s_fd, fs2, fc2, zs2, zc2, ps2, pc2);
          force_pair<ENERGY, true>(P, u, nb3, P.ck[s][k + 3], s, k + 3, s_fd, fs3, fc3, zs3, zc3, ps3, pc3);
        }
        two_sum2(fs0, fc0, fs2);
        two_sum2(fs1, fc1, fs3);
        fc0 = __fadd2_rn(fc0, fc2);
        fc1 = __fadd2_rn(fc1, fc3);
        two_sum(zs0, zc0, zs2);
        two_sum(zs1, zc1, zs3);
        zc0 += zc2;
        zc1 += zc3;
        two_sum(ps0, pc0, ps2);
        two_sum(ps1, pc1, ps3);
        pc0 += pc2;
        pc1 += pc3;
      }
      for (; k + 1 < nn; k += 2) {
        const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
        force_pair<ENERGY, true>(P, u, nb0, P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
        force_pair<ENERGY, true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fd, fs1, fc1, zs1, zc1, ps1, pc1);
      }
      if (k < nn) {
        force_pair<ENERGY, true>(P, u, tile[me.o + soff[k]], P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
        k++;
      }
      for (; k + 1 < n; k += 2) {
        const float4 nb0 = tile[me.o + soff[k]], nb1 = tile[me.o + soff[k + 1]];
        force_pair<ENERGY, false>(P, u, nb0, P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
        force_pair<ENERGY, false>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fd, fs1, fc1, zs1, zc1, ps1, pc1);
      }
      if (k < n)
        force_pair<ENERGY, false>(P, u, tile[me.o + soff[k]], P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&T.empty[b]);
    if (warp == 0) producer_issue(P, T, pr);
    if (work) {
      const double fx = ((double)fs0.x + (double)fs1.x) + ((double)fc0.x + (double)fc1.x);
      const double fy = ((double)fs0.y + (double)fs1.y) + ((double)fc0.y + (double)fc1.y);
      const double fz = ((double)zs0 + (double)zs1) + ((double)zc0 + (double)zc1);
      const long long i = me.i;
      d.fx[i] = (float)fx;
      d.fy[i] = (float)fy;
      d.fz[i] = (float)fz;
      if (d.primed) {
        vx += P.h * fx;
        vy += P.h * fy;
        vz += P.h * fz;
      }
      if (ENERGY) {
        e_kin = 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
        e_pair = ((double)ps0 + (double)ps1) + ((double)pc0 + (double)pc1);
      }
      vx += P.h * fx;
      vy += P.h * fy;
      vz += P.h * fz;
      const double nx = ux + P.dt * vx, ny = uy + P.dt * vy, nz = uz + P.dt * vz;
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
    if (ENERGY) {
      const double t1 = block_sum(e_pair);
      const double t2 = block_sum(e_kin);
      if (threadIdx.x == 0) {
        P.epart[2 * t] += t1;
        P.epart[2 * t + 1] = t2;
      }
    }
    b ^= 1;
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

// Warp `w` of the grid flags the lattice sites within reach of interstitial w.
__device__ __forceinline__ void itl_mark_one(const EnsParams &P, const LatDesc &d, int it) {
  const Geom g = lat_geom(d);
  const int lane = threadIdx.x & 31;
  const int cur = d.cur;
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
      const int slot = atomicAdd(&d.flag_count[cur], 1);
      if (slot < d.cap_flag)
        d.flag_list[slot] = (int)idx;
      else
        d.flag_count[2] = 1; // overflow: reported by the host
    }
  }
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
    pair(min_image(xi - d.ipx[cur][K], g.Lx, g.iLx), min_image(yi - d.ipy[cur][K], g.Ly, g.iLy), min_image(zi - d.ipz[cur][K], g.Lz, g.iLz),
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
    const int nflag = min(d.flag_count[d.cur], d.cap_flag);
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
  T.full = reinterpret_cast<uint64_t *>(smem + tab_bytes + 2 * ENS_TILE_MAX_BYTES);
  T.empty = T.full + 2;
  T.fphase = T.ephase = T.used = 0;
  for (int k = threadIdx.x; k < P.nsm; k += blockDim.x) {
    s_fv[k] = P.P.f_val32[P.m_lo + k];
    s_fd[3 * k + 0] = P.P.force32[3 * (P.m_lo + k) + 0];
    s_fd[3 * k + 1] = P.P.force32[3 * (P.m_lo + k) + 1];
    s_fd[3 * k + 2] = P.P.force32[3 * (P.m_lo + k) + 2];
  }
  if (threadIdx.x == 0) {
    mbar_init(&T.full[0], 1);
    mbar_init(&T.full[1], 1);
    mbar_init(&T.empty[0], ENS_CONSUMERS / 32);
    mbar_init(&T.empty[1], ENS_CONSUMERS / 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // A: interstitial flags: clear the last step's, then flag this step's (all CTAs)
  if (P.n_itl_lats > 0) {
    for (int q = 0; q < P.n_itl_lats; q++) {
      const LatDesc &d = P.lats[P.itl_lats[q]];
      if (lat_active(d)) itl_clear_flags(d);
    }
    if (!grid_sync(P.bar, P.err)) return;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (int q = 0; q < P.n_itl_lats; q++) {
      const LatDesc &d = P.lats[P.itl_lats[q]];
      if (!lat_active(d)) continue;
      for (int it = gw; it < d.n_itl; it += warps) itl_mark_one(P, d, it);
    }
    if (!grid_sync(P.bar, P.err)) return;
  }
  // B: density over lattice tiles
  rho_tiles<ENERGY>(P, T, s_fv);
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
  return tab + 2 * ENS_TILE_MAX_BYTES + 4 * sizeof(uint64_t);
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
