// Plain FP64 EAM lattice kernels (the drop-in path).
//
// Reference semantics (misa-md-hip): one result per box site with type >= 0; the
// site walks the parity-selected stencil, skips vacant neighbours and pairs with
// r^2 >= rc^2; rho takes the NEIGHBOUR's density function and df = F'(rho) is
// fused after the sum (src/kernels/kernel_itl.hpp:69-105,
// src/kernels/kernel_pairs.hpp:21-32); the force is sum del * fpair with
// fpair = -(df_i f'_{t_j} + df_j f'_{t_i} + phi'_{t_i t_j}) / r, overwritten
// (src/kernels/kernel_pairs.hpp:39-60).
//
// B200 design:
//  * sublattice-split SoA: a warp is 32 consecutive sites of one sublattice row,
//    so every stencil entry is one contiguous, coalesced 256-byte row fetch per
//    coordinate, and the stencil offset is warp-uniform (read from the kernel's
//    parameter bank);
//  * vacant sites carry a far-away position, so the r^2 test rejects them with no
//    type fetch;
//  * the spline pieces of the hot function live in shared memory (loaded once per
//    persistent CTA): random per-lane knot gathers are served by shared-memory
//    banks instead of L1 tag lookups;
//  * sites near the domain faces write their periodic ghost images themselves
//    (no separate ghost-exchange pass), and the force pass closes the previous
//    velocity-Verlet step and drifts to the next positions (double-buffered).
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>

#include "mb_common.cuh"
#include "mb_device.cuh"

namespace mb {

__device__ __forceinline__ int itl_n(const Itl64 &I) { return I.nd ? *I.nd : I.n; }

// Box z layer of a point, wrapped into the periodic box (z-slab filters of the
// host-buffer step).
__device__ __forceinline__ int z_layer(const Geom &g, double a0, double z) {
  const double w = g.iLz > 0.0 ? z - g.Lz * floor(z * g.iLz) : z;
  const double c = floor(w / a0);
  return c < 0.0 ? 0 : (c >= (double)(g.bz - 1) ? g.bz - 1 : (int)c);
}

// Lists the box site of a drifted lattice atom that left its site (conversion on).
__device__ __forceinline__ void conv_check(const Geom &g, const StepParams &sp, int s, int cx, int y, int z, double nx,
                                           double ny, double nz) {
  if (!(sp.conv2 > 0.0)) return;
  double X, Y, Z;
  site_ideal(s, cx, y, z, sp.a0, X, Y, Z);
  const double ux = nx - X, uy = ny - Y, uz = nz - Z;
  if (ux * ux + uy * uy + uz * uz <= sp.conv2) return;
  const int slot = atomicAdd(sp.cand_n, 1);
  if (slot < MB_CAND_CAP) sp.cand[slot] = ((long long)z * g.by + y) * (2LL * g.bcx) + 2LL * cx + s;
}


#define MB_EPART_CAP 4096 // CTA partial sums per energy region
#ifndef MB_RHO_THREADS
#define MB_RHO_THREADS 1024  // 52 registers: a full SM of warps
#endif
#ifndef MB_FORCE_THREADS
#define MB_FORCE_THREADS 768 // up to 85 registers
#endif
#define MB_ITL_THREADS 256

int energy_partials_needed() { return 8 * MB_EPART_CAP; }

// Work items of the lattice passes: 32 consecutive sites (one x chunk) of one row.
// Rows walk (by == 0): chunk fastest, then y, sublattice, z; a z-slab of the box is a
// contiguous item range.  Brick walk (by > 0): the items of one brick (one chunk, by rows,
// bz planes, both sublattices: y fastest, then sublattice, then z) are consecutive, so the
// warps of a CTA work on neighbouring rows at once and share their neighbour rows in L1.
struct ItemWalk {
  int chunks;       // x chunks per row
  int by, bz;       // brick rows / planes (by == 0: rows walk)
  int nyb;          // bricks along y
};

__device__ __forceinline__ bool decode_item(const Geom &g, const ItemWalk &wk, long long w, int &chunk, int &y,
                                            int &s, int &z) {
  if (wk.by == 0) {
    long long t = w;
    chunk = (int)(t % wk.chunks);
    t /= wk.chunks;
    y = (int)(t % g.by);
    t /= g.by;
    s = (int)(t & 1);
    z = (int)(t >> 1);
    return true;
  }
  const int per = 2 * wk.by * wk.bz;
  const long long b = w / per;
  const int j = (int)(w - b * per);
  const int dy = j % wk.by, q = j / wk.by;
  s = q & 1;
  const int dz = q >> 1;
  chunk = (int)(b % wk.chunks);
  const long long r = b / wk.chunks;
  y = (int)(r % wk.nyb) * wk.by + dy;
  z = (int)(r / wk.nyb) * wk.bz + dz;
  return y < g.by && z < g.bz;
}

// Index of an item in rows-walk order, whatever walk a launch takes: the key of the
// per-item outer-entry masks, which the density pass writes and the force pass reads.
__device__ __forceinline__ long long item_id(const Geom &g, const ItemWalk &wk, int chunk, int y, int s, int z) {
  return ((long long)(2 * z + s) * g.by + y) * wk.chunks + chunk;
}

// -------------------------------------------------------------- rho pass
struct RhoArgs {
  Geom g;
  DevPot P;
  Lattice64 L;
  double rc2;
  double *e_partial;
  int skip_flagged;
  int m_lo;      // first knot kept in shared memory
  ItemWalk walk;
  long long w0, n_items; // items [w0, n_items): a z-slab of the box (z slowest) or every brick
  uint2 *outer;  // per item: bit b set when a lane has stencil entry n_near + b inside the cutoff (or null)
  double rc2m;   // the squared cutoff of those bits, a hair above rc2 (robust to the FMA contraction
                 // of either pass)
};

// One density term of a one-type lattice.  BF (branch-free): the stencil entry lies
// inside the cutoff at the ideal lattice, so nearly every lane needs the spline; the
// value is masked instead of branched around, which lets iterations overlap.
template <bool BF>
__device__ __forceinline__ double rho_term(const RhoArgs &a, const Lattice64 &L, const double2 *s_f2, long long j,
                                           double xi, double yi, double zi, bool *near = nullptr) {
  const double dx = xi - L.px[j], dy = yi - L.py[j], dz = zi - L.pz[j];
  const double d2 = dx * dx + dy * dy + dz * dz;
  const bool in = d2 < a.rc2;
  if (!BF) *near = d2 < a.rc2m;
  if (!BF && !in) return 0.0;
  const double r = d2 * rsqrt(d2);
  int m;
  double p;
  spl_locate_in(r, a.P.rdr, a.P.nr, m, p);
  double4 c;
  if (m >= a.m_lo) {
    const int k = m - a.m_lo, b = (k >> 2) & 1; // halves swapped on every other group of 4 knots
    const double2 lo = s_f2[2 * k + b], hi = s_f2[2 * k + (b ^ 1)];
    c = make_double4(lo.x, lo.y, hi.x, hi.y);
  } else {
    c = ldg4(&a.P.f_val[m]);
  }
  const double v = cubic(c, p);
  return (BF && !in) ? 0.0 : v;
}

// Density, df = F'(rho) and its ghost images of one lattice site (a lane of an item);
// returns the bits of the outer stencil entries (n_near + b) the site has inside the
// cutoff (one-type walk only).
template <bool ENERGY, bool ONE_TYPE>
__device__ __forceinline__ unsigned long long rho_site(const StencilSet &st, const RhoArgs &a, const double2 *s_f2,
                                                       int s, int cx, int y, int z, double &e_acc) {
  const Geom &g = a.g;
  const Lattice64 &L = a.L;
  const DevPot &P = a.P;
  const long long i = ext_index(g, s, cx, y, z);
  const int code = L.code[i];
  if (code < 0 || (a.skip_flagged && (code & MB_FLAG_ITL))) return 0;
  const int ti = code & 0x3F;
  const double xi = L.px[i], yi = L.py[i], zi = L.pz[i];
  const int *off = st.off[s];
  double rho = 0.0;
  unsigned long long near = 0;
  if (ONE_TYPE) {
    double r0 = 0.0, r1 = 0.0;
    int k = 0;
    for (; k + 1 < st.n_near; k += 2) {
      r0 += rho_term<true>(a, L, s_f2, i + off[k], xi, yi, zi);
      r1 += rho_term<true>(a, L, s_f2, i + off[k + 1], xi, yi, zi);
    }
    if (k < st.n_near) r0 += rho_term<true>(a, L, s_f2, i + off[k++], xi, yi, zi);
#pragma unroll 2
    for (; k < st.n; k++) {
      bool in;
      r1 += rho_term<false>(a, L, s_f2, i + off[k], xi, yi, zi, &in);
      near |= (unsigned long long)in << ((k - st.n_near) & 63);
    }
    rho = r0 + r1;
  } else {
#pragma unroll 4
    for (int k = 0; k < st.n; k++) {
      const long long j = i + off[k];
      const double dx = xi - L.px[j], dy = yi - L.py[j], dz = zi - L.pz[j];
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < a.rc2) {
        const double r = d2 * rsqrt(d2);
        int m;
        double p;
        spl_locate(r, P.rdr, P.nr, m, p);
        const int tj = L.code[j] & 0x3F;
        rho += cubic(ldg4(&P.f_val[(size_t)tj * P.nr + m]), p);
      }
    }
  }
  const double df = dF64(P, ti, rho);
  L.df[i] = df;
  if (L.rho) L.rho[i] = rho;
  if (g.images) for_images(g, s, cx, y, z, [&](long long idx, double, double, double) { L.df[idx] = df; });
  if (ENERGY) e_acc += F64(P, ti, rho);
  return near;
}

template <bool ENERGY, bool ONE_TYPE>
__global__ void __launch_bounds__(MB_RHO_THREADS, 1)
    k_rho64(const __grid_constant__ StencilSet st, const __grid_constant__ RhoArgs a) {
  // Spline pieces of knots m_lo.. as 16-byte halves; the halves of knot k trade places
  // when bit 2 of k is set.  A quarter-warp's 16-byte loads of one half then spread over
  // all 8 groups of 4 banks (by k mod 8) instead of 4 (k mod 4): fewer bank conflicts
  // for the random per-lane knots of a stencil entry.
  extern __shared__ double2 s_f2[];
  const DevPot &P = a.P;
  const int nsm = P.nr - a.m_lo;
  for (int k = threadIdx.x; k < nsm; k += blockDim.x) {
    const double4 v = P.f_val[a.m_lo + k];
    const int b = (k >> 2) & 1;
    s_f2[2 * k + b] = make_double2(v.x, v.y);
    s_f2[2 * k + (b ^ 1)] = make_double2(v.z, v.w);
  }
  __syncthreads();

  const Geom &g = a.g;
  const int lane = threadIdx.x & 31;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  double e_acc = 0.0;
  for (long long w = a.w0 + (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < a.n_items;
       w += wstride) {
    int chunk, y, s, z;
    if (!decode_item(g, a.walk, w, chunk, y, s, z)) continue; // the same for the whole warp
    const int cx = chunk * 32 + lane;
    unsigned long long near = 0; // outer stencil entries this lane has inside the cutoff
    if (cx < g.bcx) near = rho_site<ENERGY, ONE_TYPE>(st, a, s_f2, s, cx, y, z, e_acc);
    if (ONE_TYPE && a.outer) {
      const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)near);
      const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(near >> 32));
      if (lane == 0) a.outer[item_id(g, a.walk, chunk, y, s, z)] = make_uint2(lo, hi);
    }
  }
  if (ENERGY) {
    const double t = block_sum(e_acc);
    if (threadIdx.x == 0) a.e_partial[blockIdx.x] = t;
  }
}

// ------------------------------------------------------------ force pass
struct ForceArgs {
  Geom g;
  DevPot P;
  Lattice64 L;
  StepParams sp;
  double *e_pair;    // CTA partials of 1/2 sum phi
  double *e_kin;     // CTA partials of kinetic energy
  int skip_flagged;
  int m_lo;
  ItemWalk walk;
  long long w0, n_items; // items [w0, n_items)
  const uint2 *outer;    // per item: the outer stencil entries the density pass of these
                         // positions found inside the cutoff (or null: walk them all)
};

// One force term of a one-type lattice (see rho_term for BF).
template <bool ENERGY, bool BF>
__device__ __forceinline__ void force_term(const ForceArgs &a, const Lattice64 &L, const double2 *s_f1, long long j,
                                           double xi, double yi, double zi, double dfi, double &fx, double &fy,
                                           double &fz, double &ep) {
  const double dx = xi - L.px[j], dy = yi - L.py[j], dz = zi - L.pz[j];
  const double d2 = dx * dx + dy * dy + dz * dz;
  const bool in = d2 < a.sp.rc2;
  if (!BF && !in) return;
  const double rinv = rsqrt(d2);
  const double r = d2 * rinv;
  const double dfj = L.df[j];
  int m;
  double p;
  spl_locate_in(r, a.P.rdr, a.P.nr, m, p);
  double2 c0, c1, c2;
  if (m >= a.m_lo) {
    const double2 *q = s_f1 + (size_t)(m - a.m_lo) * 3;
    c0 = q[0];
    c1 = q[1];
    c2 = q[2];
  } else {
    const double2 *q = a.P.force1 + (size_t)m * 3;
    c0 = __ldg(q);
    c1 = __ldg(q + 1);
    c2 = __ldg(q + 2);
  }
  const double fp = (c2.x * p + c1.x) * p + c0.x;
  const double pp = (c2.y * p + c1.y) * p + c0.y;
  double fpair = -((dfi + dfj) * fp + pp) * rinv;
  if (BF && !in) fpair = 0.0;
  fx += dx * fpair;
  fy += dy * fpair;
  fz += dz * fpair;
  if (ENERGY) {
    const double e = 0.5 * cubic(ldg4(&a.P.phi_val[m]), p);
    ep += (BF && !in) ? 0.0 : e;
  }
}

template <bool ENERGY, bool ONE_TYPE>
__global__ void __launch_bounds__(MB_FORCE_THREADS, 1)
    k_force64(const __grid_constant__ StencilSet st, const __grid_constant__ ForceArgs a) {
  extern __shared__ double2 s_f1[]; // [knot][3]
  const DevPot &P = a.P;
  if (ONE_TYPE) {
    const int nsm = (P.nr - a.m_lo) * 3;
    for (int k = threadIdx.x; k < nsm; k += blockDim.x) s_f1[k] = P.force1[(size_t)a.m_lo * 3 + k];
    __syncthreads();
  }
  const Geom &g = a.g;
  const Lattice64 &L = a.L;
  const StepParams &sp = a.sp;
  const int lane = threadIdx.x & 31;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  double e_pair = 0.0, e_kin = 0.0;
  for (long long w = a.w0 + (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < a.n_items;
       w += wstride) {
    int chunk, y, s, z;
    if (!decode_item(g, a.walk, w, chunk, y, s, z)) continue;
    // outer entries (n_near + b) that no lane of this item has inside the cutoff are not
    // walked: they contribute nothing.  Without masks the same loop walks every outer
    // entry, so both give bitwise the same forces.
    const int n_outer = st.n - st.n_near;
    unsigned long long outer = n_outer >= 64 ? ~0ull : (1ull << n_outer) - 1;
    if (ONE_TYPE && a.outer) {
      const uint2 m2 = a.outer[item_id(g, a.walk, chunk, y, s, z)];
      outer = (unsigned long long)m2.x | ((unsigned long long)m2.y << 32);
    }
    const int cx = chunk * 32 + lane;
    if (cx >= g.bcx) continue;
    const long long i = ext_index(g, s, cx, y, z);
    const int code = L.code[i];
    if (code < 0 || (a.skip_flagged && (code & MB_FLAG_ITL))) continue;
    const int ti = code & 0x3F;
    const double xi = L.px[i], yi = L.py[i], zi = L.pz[i];
    const double dfi = L.df[i];
    const int *off = st.off[s];
    double fx = 0.0, fy = 0.0, fz = 0.0, ep = 0.0;
    if (ONE_TYPE) {
      double gx = 0.0, gy = 0.0, gz = 0.0, eq = 0.0;
      int k = 0;
      // four entries per trip (the two sums alternate as with two), so more neighbour
      // rows are in flight per warp: 1.547 -> 1.517 ms on 128^3 cells
      for (; k + 3 < st.n_near; k += 4) {
        force_term<ENERGY, true>(a, L, s_f1, i + off[k], xi, yi, zi, dfi, fx, fy, fz, ep);
        force_term<ENERGY, true>(a, L, s_f1, i + off[k + 1], xi, yi, zi, dfi, gx, gy, gz, eq);
        force_term<ENERGY, true>(a, L, s_f1, i + off[k + 2], xi, yi, zi, dfi, fx, fy, fz, ep);
        force_term<ENERGY, true>(a, L, s_f1, i + off[k + 3], xi, yi, zi, dfi, gx, gy, gz, eq);
      }
      for (; k + 1 < st.n_near; k += 2) {
        force_term<ENERGY, true>(a, L, s_f1, i + off[k], xi, yi, zi, dfi, fx, fy, fz, ep);
        force_term<ENERGY, true>(a, L, s_f1, i + off[k + 1], xi, yi, zi, dfi, gx, gy, gz, eq);
      }
      if (k < st.n_near) force_term<ENERGY, true>(a, L, s_f1, i + off[k++], xi, yi, zi, dfi, fx, fy, fz, ep);
      if (n_outer <= 64) {
        // set bits in ascending k, the order of the full walk, two per trip so that two
        // neighbour rows are in flight
        unsigned long long m = outer;
        while (m) {
          const int k1 = st.n_near + __ffsll((long long)m) - 1;
          m &= m - 1;
          if (m) {
            const int k2 = st.n_near + __ffsll((long long)m) - 1;
            m &= m - 1;
            force_term<ENERGY, false>(a, L, s_f1, i + off[k1], xi, yi, zi, dfi, gx, gy, gz, eq);
            force_term<ENERGY, false>(a, L, s_f1, i + off[k2], xi, yi, zi, dfi, gx, gy, gz, eq);
          } else {
            force_term<ENERGY, false>(a, L, s_f1, i + off[k1], xi, yi, zi, dfi, gx, gy, gz, eq);
          }
        }
      } else {
#pragma unroll 2
        for (; k < st.n; k++) force_term<ENERGY, false>(a, L, s_f1, i + off[k], xi, yi, zi, dfi, gx, gy, gz, eq);
      }
      fx += gx;
      fy += gy;
      fz += gz;
      ep += eq;
    } else {
#pragma unroll 4
      for (int k = 0; k < st.n; k++) {
        const long long j = i + off[k];
        const double dx = xi - L.px[j], dy = yi - L.py[j], dz = zi - L.pz[j];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < sp.rc2) {
          const double rinv = rsqrt(d2);
          const double r = d2 * rinv;
          const double dfj = L.df[j];
          const int tj = L.code[j] & 0x3F;
          double ph = 0.0;
          const double psip = pair_psip(P, ti, tj, r, dfi, dfj, ENERGY ? &ph : nullptr);
          if (ENERGY) ep += 0.5 * ph;
          const double fpair = -psip * rinv;
          fx += dx * fpair;
          fy += dy * fpair;
          fz += dz * fpair;
        }
      }
    }
    if (L.fx) {
      L.fx[i] = fx;
      L.fy[i] = fy;
      L.fz[i] = fz;
    }
    if (L.vx) {
      double vx = L.vx[i], vy = L.vy[i], vz = L.vz[i];
      if (sp.kick_pre) {
        vx += sp.h * fx;
        vy += sp.h * fy;
        vz += sp.h * fz;
      }
      if (ENERGY) e_kin += 0.5 * sp.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
      if (sp.drift) {
        vx += sp.h * fx;
        vy += sp.h * fy;
        vz += sp.h * fz;
        const double nx = xi + sp.dt * vx, ny = yi + sp.dt * vy, nz = zi + sp.dt * vz;
        L.nx[i] = nx;
        L.ny[i] = ny;
        L.nz[i] = nz;
        conv_check(g, sp, s, cx, y, z, nx, ny, nz);
        if (g.images)
          for_images(g, s, cx, y, z, [&](long long idx, double ox, double oy, double oz) {
            L.nx[idx] = nx + ox;
            L.ny[idx] = ny + oy;
            L.nz[idx] = nz + oz;
          });
      }
      L.vx[i] = vx;
      L.vy[i] = vy;
      L.vz[i] = vz;
    }
    if (ENERGY) e_pair += ep;
  }
  if (ENERGY) {
    const double t1 = block_sum(e_pair);
    if (threadIdx.x == 0) a.e_pair[blockIdx.x] = t1;
    const double t2 = block_sum(e_kin);
    if (threadIdx.x == 0) a.e_kin[blockIdx.x] = t2;
  }
}

// ----------------------------------------------------------- launchers
static int grid_for(long long warps_needed, int threads) {
  const long long ctas = (warps_needed * 32 + threads - 1) / threads;
  long long cap = device_sm_count();
  if (cap > MB_EPART_CAP) cap = MB_EPART_CAP;
  return (int)(ctas < cap ? (ctas > 0 ? ctas : 1) : cap);
}

static const int kSmemCap = 200 * 1024;

// The one-type kernels locate spline intervals without range clamps (spl_locate_in):
// every pair inside the cutoff must lie inside the r table, up to the rounding of its end
// (a pair that far out takes the last interval at p a few ulps past 1).
static bool cutoff_in_table(const DevPot &pot, double rc2) {
  const double end = (double)(pot.nr - 1) / pot.rdr;
  return rc2 <= end * end * (1.0 + 1e-12);
}

// Brick shapes (rows, planes) of the whole-box launches; {0, 0}: rows walk.  Measured on
// 128^3 cells: density pass 1.045 ms with rows, 1.013 with 2 x 8 bricks (its 32 warps
// take one brick); force pass 1.499 ms with rows, 1.52-1.57 with 3 x 4, 4 x 3, 2 x 6,
// 6 x 2 or 4 x 6 bricks.  The environment variables MB_RHO_BRICK / MB_FORCE_BRICK
// ("rows,planes") override them.
static int kRhoBrick[2] = {2, 8}, kForceBrick[2] = {0, 0};

static void brick_override(const char *name, int *shape) {
  const char *v = getenv(name);
  int by = 0, bz = 0;
  if (v && sscanf(v, "%d,%d", &by, &bz) == 2 && by >= 0 && bz >= 0 && by <= 64 && bz <= 64) {
    shape[0] = by;
    shape[1] = bz;
  }
}

static void set_walk(const Geom &g, int z0, int z1, const int *brick, ItemWalk &wk, long long &w0, long long &n1) {
  static bool read = false;
  if (!read) {
    brick_override("MB_RHO_BRICK", kRhoBrick);
    brick_override("MB_FORCE_BRICK", kForceBrick);
    read = true;
  }
  wk.chunks = (g.bcx + 31) / 32;
  const bool whole = z0 == 0 && z1 == g.bz;
  if (whole && brick[0] > 0 && brick[1] > 0) {
    wk.by = brick[0];
    wk.bz = brick[1];
    wk.nyb = (g.by + wk.by - 1) / wk.by;
    const long long nzb = (g.bz + wk.bz - 1) / wk.bz;
    w0 = 0;
    n1 = (long long)wk.chunks * wk.nyb * nzb * 2 * wk.by * wk.bz;
    return;
  }
  wk.by = wk.bz = wk.nyb = 0;
  w0 = (long long)wk.chunks * g.by * 2 * z0;
  n1 = (long long)wk.chunks * g.by * 2 * z1;
}

// Knots kept in shared memory: those at r >= 0.3 cutoff (lattice neighbours sit near
// 0.45 cutoff and beyond; closer pairs read the global table), within kSmemCap, so
// the rest of the SM's on-chip memory stays L1 for the neighbour rows.
static int smem_knots(const DevPot &pot, int bytes_per_knot) {
  int lo = (int)(0.3 * pot.cutoff * pot.rdr);
  if (lo < 0) lo = 0;
  if (lo > pot.nr - 2) lo = pot.nr - 2;
  int n = pot.nr - lo;
  if (n * bytes_per_knot > kSmemCap) n = kSmemCap / bytes_per_knot;
  return n;
}

// Per-item outer-entry masks fit in 64 bits.
static bool outer_masks_fit(const StencilSet &st) { return st.n - st.n_near <= 64; }

int launch_rho64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, double rc2,
                 double *e_partial, int energy, int skip_flagged, cudaStream_t s, int z0, int z1, uint2 *outer) {
  RhoArgs a;
  a.g = g;
  a.P = pot;
  a.L = L;
  a.rc2 = rc2;
  a.rc2m = rc2 * (1.0 + 1e-9);
  a.e_partial = e_partial;
  a.skip_flagged = skip_flagged;
  const bool one = pot.n_types == 1 && cutoff_in_table(pot, rc2);
  a.outer = one && outer_masks_fit(st) ? outer : nullptr;
  int nsm = smem_knots(pot, (int)sizeof(double4));
  if (!one) nsm = 0;
  a.m_lo = pot.nr - nsm;
  if (z1 < 0) z1 = g.bz;
  if (z0 < 0 || z0 >= z1 || z1 > g.bz) return z0 == z1 ? MB_OK : fail(MB_ERR_ARG, "z-slab outside the box");
  set_walk(g, z0, z1, kRhoBrick, a.walk, a.w0, a.n_items);
  const size_t smem = (size_t)nsm * sizeof(double4);
  const int grid = grid_for(a.n_items - a.w0, MB_RHO_THREADS);
  static bool attr_done = false;
  if (!attr_done) {
    MB_CUDA(cudaFuncSetAttribute(k_rho64<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
    MB_CUDA(cudaFuncSetAttribute(k_rho64<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
    attr_done = true;
  }
  if (one) {
    if (energy)
      k_rho64<true, true><<<grid, MB_RHO_THREADS, smem, s>>>(st, a);
    else
      k_rho64<false, true><<<grid, MB_RHO_THREADS, smem, s>>>(st, a);
  } else {
    if (energy)
      k_rho64<true, false><<<grid, MB_RHO_THREADS, 0, s>>>(st, a);
    else
      k_rho64<false, false><<<grid, MB_RHO_THREADS, 0, s>>>(st, a);
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_force64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const StepParams &sp,
                   double *e_partial, int energy, int skip_flagged, cudaStream_t s, int z0, int z1,
                   const uint2 *outer) {
  ForceArgs a;
  a.g = g;
  a.P = pot;
  a.L = L;
  a.sp = sp;
  a.e_pair = e_partial ? e_partial + MB_EPART_CAP : nullptr;
  a.e_kin = e_partial ? e_partial + 2 * MB_EPART_CAP : nullptr;
  a.skip_flagged = skip_flagged;
  const bool one = pot.n_types == 1 && cutoff_in_table(pot, sp.rc2);
  a.outer = one && outer_masks_fit(st) ? outer : nullptr;
  int nsm = smem_knots(pot, (int)(3 * sizeof(double2)));
  if (!one) nsm = 0;
  a.m_lo = pot.nr - nsm;
  if (z1 < 0) z1 = g.bz;
  if (z0 < 0 || z0 >= z1 || z1 > g.bz) return z0 == z1 ? MB_OK : fail(MB_ERR_ARG, "z-slab outside the box");
  set_walk(g, z0, z1, kForceBrick, a.walk, a.w0, a.n_items);
  const size_t smem = (size_t)nsm * 3 * sizeof(double2);
  const int grid = grid_for(a.n_items - a.w0, MB_FORCE_THREADS);
  static bool attr_done = false;
  if (!attr_done) {
    MB_CUDA(cudaFuncSetAttribute(k_force64<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
    MB_CUDA(cudaFuncSetAttribute(k_force64<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
    attr_done = true;
  }
  if (one) {
    if (energy)
      k_force64<true, true><<<grid, MB_FORCE_THREADS, smem, s>>>(st, a);
    else
      k_force64<false, true><<<grid, MB_FORCE_THREADS, smem, s>>>(st, a);
  } else {
    if (energy)
      k_force64<true, false><<<grid, MB_FORCE_THREADS, 0, s>>>(st, a);
    else
      k_force64<false, false><<<grid, MB_FORCE_THREADS, 0, s>>>(st, a);
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// ----------------------------------------------------- interstitial passes
// Lattice sites whose IDEAL position lies within reach of an interstitial are
// flagged (site code bit MB_FLAG_ITL) and skipped by the lattice passes; the
// warp-per-item kernels below recompute them in full (stencil + interstitials)
// together with the interstitials themselves.  Every pair with r < cutoff is thus
// seen from both sides as long as no lattice atom strays more than
// (reach - cutoff) from its site.

// Last step's flags come off (grid-stride over the old list) ...
__global__ void k_itl_clear(const Lattice64 L, const Itl64 I) {
  const int nold = min(I.flag_count[0], I.cap_flag);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nold; k += gridDim.x * blockDim.x) {
    const int idx = I.flag_list[k];
    L.code[idx] = (int8_t)(L.code[idx] & ~MB_FLAG_ITL);
  }
}

// ... then one warp per interstitial flags the sites within reach (the count was
// reset in between); only sites in box layers [z0, z1) when that is not the whole box.
// The in-reach sites of the window are listed first (window_compact), so the lanes then
// flag only those, several at once.
__global__ void __launch_bounds__(MB_ITL_THREADS)
    k_itl_mark(const Geom g, const Lattice64 L, const Itl64 I, int z0, int z1) {
  __shared__ int s_list[MB_ITL_THREADS / 32][MB_WIN_LIST];
  const bool all_z = z0 <= 0 && z1 >= g.bz;
  const int lane = threadIdx.x & 31;
  const int it = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  if (it >= itl_n(I)) return; // the same for the whole warp
  const double qx = I.px[it], qy = I.py[it], qz = I.pz[it];
  const Window w = make_window(qx, qy, qz, I.a0, I.reach);
  int *list = s_list[threadIdx.x >> 5];
  const int nlist = window_compact(w, qx, qy, qz, I.a0, I.reach, list, MB_WIN_LIST);
  const int ncand = nlist >= 0 ? nlist : w.nx * w.ny * w.nz;
  for (int base = 0; base < ncand; base += 32) { // whole warp per round (warp_append)
    const int k = base + lane;
    long long idx = 0;
    bool fresh = false;
    double sx, sy, sz;
    bool site = k < ncand && window_site(g, w, nlist >= 0 ? list[k] : k, qx, qy, qz, I.a0, I.reach, idx, sx, sy, sz);
    if (site && !all_z) {
      int ss, scx, sy_, sz_;
      decode_ext(g, idx, ss, scx, sy_, sz_);
      site = sz_ >= z0 && sz_ < z1;
    }
    if (site && L.code[idx] >= 0) {
      const uintptr_t addr = (uintptr_t)(L.code + idx);
      unsigned int *word = (unsigned int *)(addr & ~(uintptr_t)3);
      const unsigned int bit = (unsigned int)MB_FLAG_ITL << (8 * (addr & 3));
      fresh = !(atomicOr(word, bit) & bit);
    }
    // flag_count[1]: overflow, reported by the host
    warp_append(fresh, (int)idx, &I.flag_count[0], I.flag_list, I.cap_flag, &I.flag_count[1]);
  }
}

// Lattice sites of the window of interstitial q, one warp: pair(dx, dy, dz, type, df)
// for every occupied site in reach, d = q - (x_j + its periodic image shift), df only with
// DF.  The in-reach sites are listed first (window_compact, list: this warp's shared
// memory) and each lane then loads up to four of them at once: one round of dependent
// loads instead of one per 32 candidates.
template <bool DF, class Pair>
__device__ __forceinline__ void window_pairs64(const Geom &g, const Lattice64 &L, const Itl64 &I, double qx,
                                               double qy, double qz, int *list, Pair pair) {
  const int lane = threadIdx.x & 31;
  const Window win = make_window(qx, qy, qz, I.a0, I.reach);
  const int n = window_compact(win, qx, qy, qz, I.a0, I.reach, list, MB_WIN_LIST);
  if (n >= 0) {
    for (int k0 = 0; k0 < n; k0 += 128) {
      long long j[4];
      double sx[4], sy[4], sz[4];
      bool ok[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int k = k0 + 32 * t + lane;
        j[t] = 0;
        sx[t] = sy[t] = sz[t] = 0.0;
        ok[t] = k < n && window_site(g, win, list[k], qx, qy, qz, I.a0, I.reach, j[t], sx[t], sy[t], sz[t]);
      }
      int cj[4];
      double xj[4], yj[4], zj[4], dj[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        cj[t] = ok[t] ? (int)L.code[j[t]] : -1;
        xj[t] = ok[t] ? L.px[j[t]] : 0.0;
        yj[t] = ok[t] ? L.py[j[t]] : 0.0;
        zj[t] = ok[t] ? L.pz[j[t]] : 0.0;
        dj[t] = (DF && ok[t]) ? L.df[j[t]] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (cj[t] >= 0) pair(qx - (xj[t] + sx[t]), qy - (yj[t] + sy[t]), qz - (zj[t] + sz[t]), cj[t] & 0x3F, dj[t]);
    }
    return;
  }
  const int ncand = win.nx * win.ny * win.nz;
  for (int c = lane; c < ncand; c += 32) {
    long long j;
    double sx, sy, sz;
    if (!window_site(g, win, c, qx, qy, qz, I.a0, I.reach, j, sx, sy, sz)) continue;
    const int cj = L.code[j];
    if (cj < 0) continue;
    pair(qx - (L.px[j] + sx), qy - (L.py[j] + sy), qz - (L.pz[j] + sz), cj & 0x3F, DF ? L.df[j] : 0.0);
  }
}

// Items of the interstitial passes: the interstitials first (w < n_itl), so that their
// window walks (the longest items) start at once, then the flagged sites.
template <bool ENERGY>
__global__ void __launch_bounds__(MB_ITL_THREADS)
    k_itl_rho64(const __grid_constant__ StencilSet st, const Geom g, const DevPot P, const Lattice64 L, const Itl64 I,
                double rc2, double *e_partial, int z0, int z1) {
  const int lane = threadIdx.x & 31;
  const bool all_z = z0 <= 0 && z1 >= g.bz; // else only items in box layers [z0, z1)
  const int nflag = min(I.flag_count[0], I.cap_flag);
  const int n_itl = itl_n(I);
  const long long n_items = (long long)nflag + n_itl;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  __shared__ int s_list[MB_ITL_THREADS / 32][MB_WIN_LIST];
  int *list = s_list[threadIdx.x >> 5];
  double e_acc = 0.0;
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n_items; w += wstride) {
    if (w >= n_itl) {
      const long long i = I.flag_list[w - n_itl];
      int s, cx, y, z;
      decode_ext(g, i, s, cx, y, z);
      if (!all_z && (z < z0 || z >= z1)) continue;
      const int ti = L.code[i] & 0x3F;
      const double xi = L.px[i], yi = L.py[i], zi = L.pz[i];
      double rho = 0.0;
      for (int k = lane; k < st.n; k += 32) {
        const long long j = i + st.off[s][k];
        const double dx = xi - L.px[j], dy = yi - L.py[j], dz = zi - L.pz[j];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < rc2) rho += rho_of_r(P, L.code[j] & 0x3F, d2 * rsqrt(d2));
      }
      for (int K = lane; K < n_itl; K += 32) {
        const double dx = min_image(xi - I.px[K], g.Lx, g.iLx), dy = min_image(yi - I.py[K], g.Ly, g.iLy),
                     dz = min_image(zi - I.pz[K], g.Lz, g.iLz);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < rc2) rho += rho_of_r(P, I.type[K], d2 * rsqrt(d2));
      }
      rho = warp_sum(rho);
      if (lane == 0) {
        const double df = dF64(P, ti, rho);
        L.df[i] = df;
        if (L.rho) L.rho[i] = rho;
        if (g.images) for_images(g, s, cx, y, z, [&](long long idx, double, double, double) { L.df[idx] = df; });
        if (ENERGY) e_acc += F64(P, ti, rho);
      }
    } else {
      const int it = (int)w;
      const double qx = I.px[it], qy = I.py[it], qz = I.pz[it];
      if (!all_z) {
        const int lz = z_layer(g, I.a0, qz);
        if (lz < z0 || lz >= z1) continue;
      }
      double rho = 0.0;
      window_pairs64<false>(g, L, I, qx, qy, qz, list, [&](double dx, double dy, double dz, int tj, double) {
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < rc2) rho += rho_of_r(P, tj, d2 * rsqrt(d2));
      });
      for (int K = lane; K < n_itl; K += 32) {
        if (K == it) continue;
        const double dx = min_image(qx - I.px[K], g.Lx, g.iLx), dy = min_image(qy - I.py[K], g.Ly, g.iLy),
                     dz = min_image(qz - I.pz[K], g.Lz, g.iLz);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < rc2) rho += rho_of_r(P, I.type[K], d2 * rsqrt(d2));
      }
      rho = warp_sum(rho);
      if (lane == 0) {
        const int t = I.type[it];
        I.rho[it] = rho;
        I.df[it] = dF64(P, t, rho);
        if (ENERGY) e_acc += F64(P, t, rho);
      }
    }
  }
  if (ENERGY) {
    const double t = block_sum(e_acc);
    if (threadIdx.x == 0) e_partial[blockIdx.x] = t;
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(MB_ITL_THREADS)
    k_itl_force64(const __grid_constant__ StencilSet st, const Geom g, const DevPot P, const Lattice64 L,
                  const Itl64 I, const StepParams sp, double *e_pair, double *e_kin, int z0, int z1) {
  const int lane = threadIdx.x & 31;
  const bool all_z = z0 <= 0 && z1 >= g.bz; // else only items in box layers [z0, z1)
  const int nflag = min(I.flag_count[0], I.cap_flag);
  const int n_itl = itl_n(I);
  const long long n_items = (long long)nflag + n_itl;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  __shared__ int s_list[MB_ITL_THREADS / 32][MB_WIN_LIST];
  int *list = s_list[threadIdx.x >> 5];
  double ep_acc = 0.0, ek_acc = 0.0;
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n_items; w += wstride) {
    const bool is_site = w >= n_itl;
    long long i = 0;
    int s = 0, cx = 0, y = 0, z = 0, it = 0, ti;
    double xi, yi, zi, dfi;
    if (is_site) {
      i = I.flag_list[w - n_itl];
      decode_ext(g, i, s, cx, y, z);
      ti = L.code[i] & 0x3F;
      xi = L.px[i];
      yi = L.py[i];
      zi = L.pz[i];
      dfi = L.df[i];
    } else {
      it = (int)w;
      ti = I.type[it];
      xi = I.px[it];
      yi = I.py[it];
      zi = I.pz[it];
      dfi = I.df[it];
    }
    if (!all_z) {
      const int lz = is_site ? z : z_layer(g, I.a0, zi);
      if (lz < z0 || lz >= z1) continue;
    }
    double fx = 0.0, fy = 0.0, fz = 0.0, ep = 0.0;
    auto add_pair = [&](double dx, double dy, double dz, int tj, double dfj) {
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 >= sp.rc2) return;
      const double rinv = rsqrt(d2);
      double ph = 0.0;
      const double psip = pair_psip(P, ti, tj, d2 * rinv, dfi, dfj, ENERGY ? &ph : nullptr);
      const double fpair = -psip * rinv;
      fx += dx * fpair;
      fy += dy * fpair;
      fz += dz * fpair;
      if (ENERGY) ep += 0.5 * ph;
    };
    if (is_site) {
      for (int k = lane; k < st.n; k += 32) {
        const long long j = i + st.off[s][k];
        const int cj = L.code[j];
        if (cj < 0) continue;
        add_pair(xi - L.px[j], yi - L.py[j], zi - L.pz[j], cj & 0x3F, L.df[j]);
      }
    } else {
      window_pairs64<true>(g, L, I, xi, yi, zi, list, add_pair);
    }
    for (int K = lane; K < n_itl; K += 32) {
      if (!is_site && K == it) continue;
      add_pair(min_image(xi - I.px[K], g.Lx, g.iLx), min_image(yi - I.py[K], g.Ly, g.iLy), min_image(zi - I.pz[K], g.Lz, g.iLz),
               I.type[K], I.df[K]);
    }
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    if (ENERGY) ep = warp_sum(ep);
    if (lane == 0) {
      double *vxp = is_site ? L.vx : I.vx;
      const long long vi = is_site ? i : it;
      if (is_site) {
        if (L.fx) {
          L.fx[i] = fx;
          L.fy[i] = fy;
          L.fz[i] = fz;
        }
      } else {
        I.fx[it] = fx;
        I.fy[it] = fy;
        I.fz[it] = fz;
      }
      if (vxp) {
        double *vyp = is_site ? L.vy : I.vy, *vzp = is_site ? L.vz : I.vz;
        double vx = vxp[vi], vy = vyp[vi], vz = vzp[vi];
        if (sp.kick_pre) {
          vx += sp.h * fx;
          vy += sp.h * fy;
          vz += sp.h * fz;
        }
        if (ENERGY) ek_acc += 0.5 * sp.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
        if (sp.drift) {
          vx += sp.h * fx;
          vy += sp.h * fy;
          vz += sp.h * fz;
          const double nx = xi + sp.dt * vx, ny = yi + sp.dt * vy, nz = zi + sp.dt * vz;
          if (is_site) {
            L.nx[i] = nx;
            L.ny[i] = ny;
            L.nz[i] = nz;
            conv_check(g, sp, s, cx, y, z, nx, ny, nz);
            if (g.images)
              for_images(g, s, cx, y, z, [&](long long idx, double ox, double oy, double oz) {
                L.nx[idx] = nx + ox;
                L.ny[idx] = ny + oy;
                L.nz[idx] = nz + oz;
              });
          } else {
            I.nx[it] = nx;
            I.ny[it] = ny;
            I.nz[it] = nz;
          }
        }
        vxp[vi] = vx;
        vyp[vi] = vy;
        vzp[vi] = vz;
      }
      if (ENERGY) ep_acc += ep;
    }
  }
  if (ENERGY) {
    const double t1 = block_sum(ep_acc);
    if (threadIdx.x == 0) e_pair[blockIdx.x] = t1;
    const double t2 = block_sum(ek_acc);
    if (threadIdx.x == 0) e_kin[blockIdx.x] = t2;
  }
}

int launch_itl_mark64(const Geom &g, const Lattice64 &L, const Itl64 &I, cudaStream_t s) {
  int grid = (I.cap_flag + 255) / 256;
  if (grid > 4 * device_sm_count()) grid = 4 * device_sm_count();
  k_itl_clear<<<grid, 256, 0, s>>>(L, I);
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaMemsetAsync(I.flag_count, 0, sizeof(int), s));
  const int nmax = I.nd ? I.cap : I.n;
  if (nmax > 0)
    k_itl_mark<<<(nmax * 32 + MB_ITL_THREADS - 1) / MB_ITL_THREADS, MB_ITL_THREADS, 0, s>>>(g, L, I, 0, g.bz);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_itl_mark_slab64(const Geom &g, const Lattice64 &L, const Itl64 &I, int z0, int z1, cudaStream_t s) {
  const int nmax = I.nd ? I.cap : I.n;
  if (nmax > 0 && z0 < z1)
    k_itl_mark<<<(nmax * 32 + MB_ITL_THREADS - 1) / MB_ITL_THREADS, MB_ITL_THREADS, 0, s>>>(g, L, I, z0, z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

static int itl_grid(const Itl64 &I) {
  const long long warps = (long long)I.cap_flag + (I.nd ? I.cap : I.n);
  long long ctas = (warps * 32 + MB_ITL_THREADS - 1) / MB_ITL_THREADS;
  const long long cap = 4LL * device_sm_count();
  if (ctas > cap) ctas = cap;
  if (ctas > MB_EPART_CAP) ctas = MB_EPART_CAP;
  return (int)(ctas > 0 ? ctas : 1);
}

int launch_itl_rho64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const Itl64 &I,
                     double rc2, double *e_partial, int energy, cudaStream_t s, int z0, int z1) {
  if (!I.nd && I.n == 0) return MB_OK;
  if (z1 < 0) z1 = g.bz;
  const int grid = itl_grid(I);
  if (energy)
    k_itl_rho64<true><<<grid, MB_ITL_THREADS, 0, s>>>(st, g, pot, L, I, rc2, e_partial + 3 * MB_EPART_CAP, z0, z1);
  else
    k_itl_rho64<false><<<grid, MB_ITL_THREADS, 0, s>>>(st, g, pot, L, I, rc2, nullptr, z0, z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_itl_force64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const Itl64 &I,
                       const StepParams &sp, double *e_partial, int energy, cudaStream_t s, int z0, int z1) {
  if (!I.nd && I.n == 0) return MB_OK;
  if (z1 < 0) z1 = g.bz;
  const int grid = itl_grid(I);
  if (energy)
    k_itl_force64<true><<<grid, MB_ITL_THREADS, 0, s>>>(st, g, pot, L, I, sp, e_partial + 4 * MB_EPART_CAP,
                                                         e_partial + 5 * MB_EPART_CAP, z0, z1);
  else
    k_itl_force64<false><<<grid, MB_ITL_THREADS, 0, s>>>(st, g, pot, L, I, sp, nullptr, nullptr, z0, z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// ------------------------------------------ lattice <-> interstitial bookkeeping
// MISA-MD keeps atoms that have left their lattice site in its interstitial list (the
// plugin only sees type < 0 for such sites, src/kernels/kernel_itl.hpp:44).  After the
// drift of a step, one CTA
//   1. sorts this step's candidates (box index of sites whose atom is farther than the
//      conversion distance from the site) and appends their atoms to the interstitial
//      list in that order, vacating the sites (and their ghost images);
//   2. finds, for every interstitial, the nearest ideal site; one within the
//      recombination distance of a vacant site claims it, the lowest list index
//      winning a contested site;
//   3. moves each winner onto its site and compacts the list, keeping its order.
// Fixed orders (box index, list index) keep the result independent of thread timing.
#define MB_CONV_THREADS 1024

__global__ void __launch_bounds__(MB_CONV_THREADS, 1)
    k_convert64(const Geom g, const Lattice64 L, const Itl64 I, const StepParams sp, double rec2,
                int64_t *site_id, int *nd, long long *counters) {
  __shared__ long long key[MB_CAND_CAP];
  __shared__ unsigned removed[MB_CONV_ITL_MAX / 32];
  __shared__ int s_scan[MB_CONV_THREADS / 32];
  __shared__ int s_nclaim, s_base;
  const int tid = threadIdx.x;
  const int n0 = *nd;
  // 1. conversions in box order
  const int nraw = *sp.cand_n;
  const int nc = min(nraw, MB_CAND_CAP);
  int n2 = 1;
  while (n2 < nc) n2 <<= 1;
  for (int k = tid; k < n2; k += blockDim.x) key[k] = k < nc ? sp.cand[k] : LLONG_MAX;
  __syncthreads();
  if (nc > 1) bitonic_sort(key, n2);
  const int room = max(0, I.cap - n0);
  const int nconv = min(nc, room);
  for (int r = tid; r < nconv; r += blockDim.x) {
    const long long t = key[r];
    int s, cx, y, z;
    decode_box(g, t, s, cx, y, z);
    const long long i = ext_index(g, s, cx, y, z);
    const int k = n0 + r;
    I.nx[k] = L.nx[i];
    I.ny[k] = L.ny[i];
    I.nz[k] = L.nz[i];
    I.px[k] = L.px[i];
    I.py[k] = L.py[i];
    I.pz[k] = L.pz[i];
    I.vx[k] = L.vx[i];
    I.vy[k] = L.vy[i];
    I.vz[k] = L.vz[i];
    I.fx[k] = L.fx[i];
    I.fy[k] = L.fy[i];
    I.fz[k] = L.fz[i];
    I.rho[k] = L.rho ? L.rho[i] : 0.0;
    I.df[k] = L.df[i];
    I.type[k] = (int8_t)(L.code[i] & 0x3F);
    I.id[k] = site_id[t];
    // vacant: both position buffers far away (the pair loops reject vacancies by
    // position, and the buffer of this step comes back as the next step's drift target)
    L.code[i] = -1;
    L.nx[i] = L.ny[i] = L.nz[i] = MB_VACANT_POS;
    L.px[i] = L.py[i] = L.pz[i] = MB_VACANT_POS;
    L.vx[i] = L.vy[i] = L.vz[i] = 0.0;
    L.fx[i] = L.fy[i] = L.fz[i] = 0.0;
    for_images(g, s, cx, y, z, [&](long long idx, double, double, double) {
      L.code[idx] = -1;
      L.nx[idx] = L.ny[idx] = L.nz[idx] = MB_VACANT_POS;
      L.px[idx] = L.py[idx] = L.pz[idx] = MB_VACANT_POS;
    });
  }
  const int n1 = n0 + nconv;
  if (tid == 0) {
    counters[0] += nconv;
    counters[2] += nc - nconv;
    counters[3] += nraw - nc;
    *sp.cand_n = 0;
    s_nclaim = 0;
  }
  for (int w = tid; w < MB_CONV_ITL_MAX / 32; w += blockDim.x) removed[w] = 0u;
  __syncthreads(); // vacated sites visible to the claims below
  // 2. claims: nearest ideal site of every interstitial, when vacant and close enough
  for (int k = tid; k < n1; k += blockDim.x) {
    const double qx = I.nx[k], qy = I.ny[k], qz = I.nz[k];
    double best = 1e300;
    long long gx = 0, gy = 0, gz = 0;
    int bs = 0;
    for (int sl = 0; sl < 2; sl++) {
      const double o = 0.5 * sp.a0 * sl;
      const long long cx = llrint((qx - o) / sp.a0), cy = llrint((qy - o) / sp.a0), cz = llrint((qz - o) / sp.a0);
      const double X = 0.5 * sp.a0 * (double)(2 * cx + sl), Y = sp.a0 * ((double)cy + 0.5 * sl),
                   Z = sp.a0 * ((double)cz + 0.5 * sl);
      const double dd = (qx - X) * (qx - X) + (qy - Y) * (qy - Y) + (qz - Z) * (qz - Z);
      if (dd < best) {
        best = dd;
        gx = cx;
        gy = cy;
        gz = cz;
        bs = sl;
      }
    }
    if (!(best < rec2)) continue;
    const int cx = pmod_int(gx, g.bcx), y = pmod_int(gy, g.by), z = pmod_int(gz, g.bz);
    if (L.code[ext_index(g, bs, cx, y, z)] >= 0) continue;
    const long long t = ((long long)z * g.by + y) * (2LL * g.bcx) + 2LL * cx + bs;
    const int slot = atomicAdd(&s_nclaim, 1);
    if (slot < MB_CAND_CAP) key[slot] = (t << 17) | (long long)k; // k < 2^16 (MB_CONV_ITL_MAX)
  }
  __syncthreads();
  const int ncl = min(s_nclaim, MB_CAND_CAP);
  n2 = 1;
  while (n2 < ncl) n2 <<= 1;
  for (int k = ncl + tid; k < n2; k += blockDim.x) key[k] = LLONG_MAX;
  __syncthreads();
  if (ncl > 1) bitonic_sort(key, n2);
  // 3. winners move onto their sites
  int nrec = 0;
  for (int r = tid; r < ncl; r += blockDim.x) {
    const long long t = key[r] >> 17;
    if (r > 0 && (key[r - 1] >> 17) == t) continue; // a lower list index took the site
    const int k = (int)(key[r] & 0x1FFFF);
    int s, cx, y, z;
    decode_box(g, t, s, cx, y, z);
    const long long i = ext_index(g, s, cx, y, z);
    double X, Y, Z;
    site_ideal(s, cx, y, z, sp.a0, X, Y, Z);
    // displacement of the interstitial from the nearest image of the site
    const double ux = min_image(I.nx[k] - X, g.Lx, g.iLx), uy = min_image(I.ny[k] - Y, g.Ly, g.iLy),
                 uz = min_image(I.nz[k] - Z, g.Lz, g.iLz);
    const double nx = X + ux, ny = Y + uy, nz = Z + uz;
    // the previous positions too (the buffer a download reads), on the same image
    const double px = nx + (I.px[k] - I.nx[k]), py = ny + (I.py[k] - I.ny[k]), pz = nz + (I.pz[k] - I.nz[k]);
    const int8_t ty = I.type[k];
    L.code[i] = ty;
    L.nx[i] = nx;
    L.ny[i] = ny;
    L.nz[i] = nz;
    L.px[i] = px;
    L.py[i] = py;
    L.pz[i] = pz;
    L.vx[i] = I.vx[k];
    L.vy[i] = I.vy[k];
    L.vz[i] = I.vz[k];
    L.fx[i] = I.fx[k];
    L.fy[i] = I.fy[k];
    L.fz[i] = I.fz[k];
    L.df[i] = I.df[k];
    for_images(g, s, cx, y, z, [&](long long idx, double ox, double oy, double oz) {
      L.code[idx] = ty;
      L.nx[idx] = nx + ox;
      L.ny[idx] = ny + oy;
      L.nz[idx] = nz + oz;
      L.px[idx] = px + ox;
      L.py[idx] = py + oy;
      L.pz[idx] = pz + oz;
    });
    site_id[t] = I.id[k];
    atomicOr(&removed[k >> 5], 1u << (k & 31));
    nrec++;
  }
  const double nrec_all = block_sum((double)nrec); // exact for integer counts
  if (tid == 0) {
    counters[1] += (long long)nrec_all;
    s_base = 0;
  }
  __syncthreads();
  // 4. stable compaction of the list
  for (int c0 = 0; c0 < n1; c0 += blockDim.x) {
    const int k = c0 + tid;
    const bool keep = k < n1 && !((removed[k >> 5] >> (k & 31)) & 1u);
    // block exclusive scan of keep
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
      v[0] = I.px[k], v[1] = I.py[k], v[2] = I.pz[k], v[3] = I.nx[k], v[4] = I.ny[k], v[5] = I.nz[k];
      v[6] = I.vx[k], v[7] = I.vy[k], v[8] = I.vz[k], v[9] = I.fx[k], v[10] = I.fy[k], v[11] = I.fz[k];
      v[12] = I.rho[k], v[13] = I.df[k];
      ty = I.type[k];
      id = I.id[k];
    }
    __syncthreads(); // every read of this chunk before any write (dst <= k)
    if (keep && dst != k) {
      I.px[dst] = v[0], I.py[dst] = v[1], I.pz[dst] = v[2], I.nx[dst] = v[3], I.ny[dst] = v[4], I.nz[dst] = v[5];
      I.vx[dst] = v[6], I.vy[dst] = v[7], I.vz[dst] = v[8], I.fx[dst] = v[9], I.fy[dst] = v[10], I.fz[dst] = v[11];
      I.rho[dst] = v[12], I.df[dst] = v[13];
      I.type[dst] = ty;
      I.id[dst] = id;
    }
    __syncthreads();
  }
  if (tid == 0) *nd = s_base;
}

int launch_convert64(const Geom &g, const Lattice64 &L, const Itl64 &I, const StepParams &sp, double rec2,
                     int64_t *site_id, int *nd, long long *counters, cudaStream_t s) {
  if (!(sp.conv2 > 0.0)) return MB_OK;
  if (I.cap > MB_CONV_ITL_MAX) return fail(MB_ERR_ARG, "interstitial capacity above the conversion limit (65536)");
  k_convert64<<<1, MB_CONV_THREADS, 0, s>>>(g, L, I, sp, rec2, site_id, nd, counters);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// ------------------------------------------------ images / kick-drift
// Sites are numbered cx fastest, then y, sublattice, z: box layers [z0, z1) are the
// numbers [t0, t1) = [z0, z1) * 2 * by * bcx.
__global__ void k_images64(const Geom g, const Lattice64 L, int what, long long t0, long long t1) {
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    const int cx = (int)(t % g.bcx);
    long long r = t / g.bcx;
    const int y = (int)(r % g.by);
    r /= g.by;
    const int s = (int)(r & 1);
    const int z = (int)(r >> 1);
    const long long i = ext_index(g, s, cx, y, z);
    if (what & 1) {
      const double x0 = L.px[i], y0 = L.py[i], z0 = L.pz[i];
      const int8_t c = L.code[i];
      for_images(g, s, cx, y, z, [&](long long idx, double ox, double oy, double oz) {
        L.px[idx] = x0 + ox;
        L.py[idx] = y0 + oy;
        L.pz[idx] = z0 + oz;
        L.code[idx] = (int8_t)(c < 0 ? c : (c & 0x3F));
      });
    }
    if (what & 2) {
      const double d = L.df[i];
      for_images(g, s, cx, y, z, [&](long long idx, double, double, double) { L.df[idx] = d; });
    }
  }
}

int launch_images64(const Geom &g, const Lattice64 &L, int what, cudaStream_t s, int z0, int z1) {
  if (z1 < 0) z1 = g.bz;
  const long long layer = 2LL * g.bcx * g.by;
  const long long n = layer * (z1 - z0);
  if (n <= 0) return MB_OK;
  int grid = (int)((n + 255) / 256);
  if (grid > 8 * device_sm_count()) grid = 8 * device_sm_count();
  k_images64<<<grid, 256, 0, s>>>(g, L, what, layer * z0, layer * z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// First half of a velocity-Verlet step in place (used when the state arrives
// from the host each step): v += h f ; x += dt v, then refresh ghost images.
// Lattice sites [t0, t1) (numbered as in k_images64), then the interstitials when
// with_itl is set.
__global__ void k_kick_drift64(const Geom g, const Lattice64 L, const Itl64 I, const StepParams sp, long long t0,
                               long long t1, int with_itl) {
  const long long n = t1 - t0;
  const int n_itl = with_itl ? itl_n(I) : 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n + n_itl;
       q += (long long)gridDim.x * blockDim.x) {
    const long long t = t0 + q;
    if (q >= n) {
      const int it = (int)(q - n);
      I.vx[it] += sp.h * I.fx[it];
      I.vy[it] += sp.h * I.fy[it];
      I.vz[it] += sp.h * I.fz[it];
      I.px[it] += sp.dt * I.vx[it];
      I.py[it] += sp.dt * I.vy[it];
      I.pz[it] += sp.dt * I.vz[it];
      continue;
    }
    const int cx = (int)(t % g.bcx);
    long long r = t / g.bcx;
    const int y = (int)(r % g.by);
    r /= g.by;
    const int s = (int)(r & 1);
    const int z = (int)(r >> 1);
    const long long i = ext_index(g, s, cx, y, z);
    if (L.code[i] < 0) continue;
    const double vx = L.vx[i] + sp.h * L.fx[i], vy = L.vy[i] + sp.h * L.fy[i], vz = L.vz[i] + sp.h * L.fz[i];
    const double x0 = L.px[i] + sp.dt * vx, y0 = L.py[i] + sp.dt * vy, z0 = L.pz[i] + sp.dt * vz;
    L.vx[i] = vx;
    L.vy[i] = vy;
    L.vz[i] = vz;
    L.px[i] = x0;
    L.py[i] = y0;
    L.pz[i] = z0;
    for_images(g, s, cx, y, z, [&](long long idx, double ox, double oy, double oz) {
      L.px[idx] = x0 + ox;
      L.py[idx] = y0 + oy;
      L.pz[idx] = z0 + oz;
    });
  }
}

int launch_kick_drift64(const Geom &g, const Lattice64 &L, const Itl64 &I, const StepParams &sp, cudaStream_t s,
                        int z0, int z1, int with_itl) {
  if (z1 < 0) z1 = g.bz;
  const long long layer = 2LL * g.bcx * g.by;
  const long long n = layer * (z1 - z0) + (with_itl ? (I.nd ? I.cap : I.n) : 0);
  if (n <= 0) return MB_OK;
  int grid = (int)((n + 255) / 256);
  if (grid > 8 * device_sm_count()) grid = 8 * device_sm_count();
  k_kick_drift64<<<grid, 256, 0, s>>>(g, L, I, sp, layer * z0, layer * z1, with_itl);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// Sum of each energy region in a fixed order: out[0] = pe, out[1] = ke.
__global__ void k_reduce_energy(const double *part, double *out) {
  __shared__ double acc[2][256];
  double pe = 0.0, ke = 0.0;
  for (int k = threadIdx.x; k < MB_EPART_CAP; k += blockDim.x) {
    pe += part[0 * MB_EPART_CAP + k] + part[1 * MB_EPART_CAP + k] + part[3 * MB_EPART_CAP + k] +
          part[4 * MB_EPART_CAP + k];
    ke += part[2 * MB_EPART_CAP + k] + part[5 * MB_EPART_CAP + k];
  }
  acc[0][threadIdx.x] = pe;
  acc[1][threadIdx.x] = ke;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < 256; k++) {
      a += acc[0][k];
      b += acc[1][k];
    }
    out[0] = a;
    out[1] = b;
  }
}

int launch_reduce(const double *partials, int n, double *out, cudaStream_t s) {
  (void)n;
  k_reduce_energy<<<1, 256, 0, s>>>(partials, out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb
