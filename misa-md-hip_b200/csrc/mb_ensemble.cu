// Mixed-precision, multi-lattice EAM timestep (see mb_ensemble_kernel.cuh for the
// phase structure and the precision scheme).
#include <math.h>

#include "mb_ensemble_kernel.cuh"
#include "mb_ensemble_pair.cuh"

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
    const bool work = me.valid && code >= 0; // flagged sites: lattice part only (see itl_item)
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
    if (work && (code & MB_FLAG_ITL)) {
      d.rho[me.i] = (float)(((double)rs0 + (double)rs1) + ((double)rc0 + (double)rc1));
    } else if (work) {
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
    const bool work = me.valid && code >= 0; // flagged sites: lattice part only (see itl_item)
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
      if (ENERGY) e_pair = ((double)ps0 + (double)ps1) + ((double)pc0 + (double)pc1);
    }
    if (work && !(code & MB_FLAG_ITL)) { // flagged sites are integrated by the interstitial items
      const long long i = me.i;
      const double fx = ((double)fs0.x + (double)fs1.x) + ((double)fc0.x + (double)fc1.x);
      const double fy = ((double)fs0.y + (double)fs1.y) + ((double)fc0.y + (double)fc1.y);
      const double fz = ((double)zs0 + (double)zs1) + ((double)zc0 + (double)zc1);
      if (d.primed) {
        vx += P.h * fx;
        vy += P.h * fy;
        vz += P.h * fz;
      }
      if (ENERGY) e_kin = 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
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
    if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (int q = 0; q < P.n_itl_lats; q++) {
      const LatDesc &d = P.lats[P.itl_lats[q]];
      if (!lat_active(d)) continue;
      for (int it = gw; it < d.n_itl; it += warps) itl_mark_one(P, d, it);
    }
    if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
  }
  // B: density over lattice tiles
  rho_tiles<ENERGY>(P, T, s_fv);
  if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
  // C: density of flagged sites and interstitials
  if (P.n_itl_lats > 0) {
    itl_items<false, ENERGY>(P);
    if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
  }
  // D: forces and integration over lattice tiles (flagged sites: lattice part only)
  force_tiles<ENERGY>(P, T, s_fd);
  if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
  // E: forces and integration of flagged sites and interstitials
  if (P.n_itl_lats > 0) {
    itl_items<true, ENERGY>(P);
    if (!grid_sync(P.bar, P.err, P.bar_spins)) return;
  }
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
