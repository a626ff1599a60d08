// Mixed-precision, multi-lattice EAM timestep: device side.
//
// One persistent kernel advances every active lattice of an ensemble by one
// velocity-Verlet step.  Phases, separated by a grid barrier with a bounded spin:
//   A  interstitial bookkeeping: flag lattice sites within reach of an interstitial
//   B  rho / df over lattice tiles (FP32 pair + spline work, two-sum accumulation)
//   C  rho / df of flagged sites and interstitials (FP64, one warp per item)
//   D  force + velocity-Verlet over lattice tiles (FP32 pairs, FP64 integration)
//   E  force + velocity-Verlet of flagged sites and interstitials (FP64)
//   F  per-lattice step bookkeeping (buffer parity, step counters)
//
// Lattice state per site: FP64 displacement from the ideal BCC site (u64) and FP64
// velocity are the master copy; a float4 {u (FP32), df} array, ghost-extended by 2
// cells, is what the pair passes read.  A tile of 2 x (TX x TY x TZ) sites plus its
// 2-cell halo is staged into shared memory with one 5-D TMA load (float4 component,
// x, y, z, sublattice), double-buffered so the next tile streams in while the
// current one is computed.  Vacant sites carry a huge displacement so every r^2 test
// rejects them.
//
// Precision of the pair distance: FP32 cannot hold r to better than ~1e-7 A near
// 5 A, which alone gives force errors of ~2e-6 relative.  The spline index is
// therefore taken from eps = r - R_k, with R_k the ideal length of stencil entry k:
// eps = (2 C_k . d + d . d) / (r + R_k), d = u_i - u_j, is small and carries
// ~1e-8 A absolute precision; R_k / dr is split on the host into an integer knot and
// an FP32 fraction.
#pragma once

#include <cuda.h>

#include "mb_common.cuh"
#include "mb_device.cuh"

namespace mb {

#define ENS_CONSUMERS 512 // one site per thread per tile
#define ENS_THREADS 512
#define ENS_NSHAPE 4
#define ENS_MAX_ST 112
#define ENS_BAR_SPINS (1u << 25)
#define ENS_WAIT_SPINS (1u << 26)
#define ENS_VACANT 1.0e15f
#define ENS_TILE_MAX_BYTES 40960 // largest halo'd tile: 2 x 20 x 8 x 8 float4

struct LatDesc {
  int bcx, by, bz;       // box (cells along x per sublattice)
  int ecx, ey, ez;       // ghost-extended (box + 4)
  long long E;           // sites per sublattice array
  int ntx, nty, ntz;     // tiles along x, y, z
  int shape;             // tile shape id
  int n_itl, cap_flag;
  int cur;               // u4 buffer holding the current positions (flipped on the device)
  int primed;            // 1 once forces at the start positions exist
  long long steps_done, steps_target;
  double Lx, Ly, Lz;
  float4 *u4[2];         // {ux, uy, uz, df}, ghost-extended
  double *ux, *uy, *uz;  // FP64 displacement (master), ext-indexed
  double *vx, *vy, *vz;
  float *fx, *fy, *fz, *rho;
  int8_t *code;
  int *flag_list, *flag_count;
  double *ipx[2], *ipy[2], *ipz[2];
  double *ivx, *ivy, *ivz, *ifx, *ify, *ifz, *irho, *idf;
  int8_t *itype;
  double *e_itl; // [2] interstitial-item energy (pe, ke), accumulated atomically
  // lattice <-> interstitial conversion
  int cap_itl;
  int64_t *ids, *iids;   // atom ids of the box sites (box order) and of the interstitials
  long long *cand;       // [MB_CAND_CAP] box index of sites whose atom left them this step
  int *cand_n;
  long long *conv_counters; // [4] conversions, recombinations, refused, dropped
  // interstitial cell list (rebuilt at the start of every step): the box cut into
  // icn[0] x icn[1] x icn[2] cells of edge >= cutoff + skin (0: lattice too small, every
  // item walks the whole list); icount / istart per cell, iitem the list indices sorted by
  // (cell, index), icell_of the cell of each entry at the last build, iflag[0] = 1 when
  // the list is valid this step, iflag[1] = entries of the last build
  int icn[3];
  int *icount, *istart, *iitem, *icell_of, *iflag;
};
#define MX_ICELL_MAX 4096 // interstitials a cell list is built for (sorted in shared memory)

struct EnsParams {
  int n_st;                            // stencil entries, ordered by ideal distance
  int n_near;                          // entries whose ideal distance is inside the cutoff
  int soff[ENS_NSHAPE][2][ENS_MAX_ST]; // shared-memory offset (float4 units) of entry k, per shape / sublattice
  float4 ck[2][ENS_MAX_ST];            // ideal offset X_i - X_j (xyz) and its length (w)
  float2 kf[2][ENS_MAX_ST];            // {|C_k| / dr - floor(|C_k| / dr), floor(|C_k| / dr)}
  char4 sd[2][ENS_MAX_ST];             // target sublattice - own, dcx, dy, dz
  int shape_dims[ENS_NSHAPE][4];       // TX, TY, TZ, bytes
  int shape_log[ENS_NSHAPE][4];        // log2 TX, log2 TY, log2 TZ, log2 (TX TY TZ)
  DevPot P;
  float rdr, rc2f;
  int m_lo, nsm;
  double h, dt, mass, a0, rc2, reach;
  const LatDesc *lats;
  int n_lats;
  const int *tile_lat;
  const unsigned *tile_org; // tile origin: cx0 | y0 << 11 | z0 << 22 (box cells)
  int n_tiles;
  const CUtensorMap *tmaps; // [lattice][buffer]
  unsigned *bar;
  unsigned bar_spins; // polls a grid barrier makes before it gives up (ENS_BAR_SPINS by default)
  int *err;
  double *epart; // [tile][2]
  uint2 *outer;  // split kernels: per walk item, the branch-walked built-in stencil entries some site
                 // has inside the cutoff (written by the density pass, read by the force pass)
  const int *itl_lats;
  int n_itl_lats;
  int energy;
  double conv2, rec2; // conversion / recombination distances squared (conv2 = 0: off)
};

// Split mode stencil.  BCC is a Bravais lattice: both sublattices see the same ideal
// neighbour vectors, so the per-entry constants below serve every site.  Only the
// storage offset differs, and only for vectors that cross to the other sublattice
// (odd half-lattice components): a sublattice-1 site adds d_odd to their offset.
// Entries inside the cutoff (plus half the skin) are split by that parity into two
// lists walked without a per-pair branch, each padded to an even length; the rest
// are walked with a branch.
#define MX_PAR_MAX 40
struct MxEntry {
  float4 c;    // ideal X_i - X_j (xyz); w = rc^2 - R^2: the pair interacts when num < w
  float4 t;    // 2 (X_i - X_j) (xyz); w = frac(R^2 / ds) on the density grid
  float kb;    // floor(R^2 / ds) on the density grid
  float fr_f;  // frac / floor of R^2 / ds on the force grid
  float kb_f;
  int off;     // linear offset from a sublattice-0 site
  int odd;     // 1: crosses sublattices
  int pad_[3];
};

// Walks of the split kernels.  One large lattice: the box is cut into bricks of one x
// chunk (32 sites, one per lane) by MX_BY rows by MX_BZ planes by both sublattices; a
// block takes whole bricks (brick b, b + grid, ...) so the rows its warps read overlap
// and stay in L1.  Many lattices: every lattice's (z, sublattice) planes are cut into
// items of 32 consecutive sites (rows of small lattices share a warp) and each block
// walks one contiguous range of the concatenated items.
#define MX_BY 8
#define MX_BZ 8
#define MX_LCB 8      // linear walk, large lattices: bricks of 8 chunks ...
#define MX_LBZ 8      // ... by 8 z cells ...
#define MX_LMIN 4096  // ... for planes of at least 64 x 64 sites
struct MxWalk {
  int linear;                // 0: bricks of lattice `lat`; 1: linear items over every lattice
  unsigned chunks, m_chunks; // x chunks per row and floor((2^32 - 1) / chunks)
  unsigned by, bz, bitems;   // brick rows, planes and items (2 by bz; MX_BY, MX_BZ unless overridden)
  unsigned nyb, m_nyb;       // y bricks
  unsigned n_units;          // bricks
  // linear walk: item = 32 consecutive sites (a chunk) of one (z, sublattice) plane of a
  // lattice; lattice l owns items [item_first[l], item_first[l + 1]).  A lattice whose
  // (z, sublattice) planes hold at least lmin sites orders its items by bricks of lbz z
  // cells (both sublattices) by lcb chunks: z block, then chunk block, then plane, then
  // chunk, so that a block's warps share neighbour planes in L1 (10 planes of such a
  // lattice exceed it).  Smaller lattices go plane by plane, which measured faster for
  // them (lcb == 0: every lattice plane by plane).
  const unsigned *item_first;
  unsigned lcb, lbz, lmin;
  unsigned n_items; // every walk: items (energy partials)
  int n_lats;
};

// Split-mode stencil built into the kernel: the BCC neighbour shells up to |h|^2 = 19
// (7 shells, 88 vectors: cutoff + skin between the 7th and 8th shell, e.g. a0 = 2.855,
// rc = 5.6, skin = 0.7 for iron) or up to |h|^2 = 20 (8 shells, 112 vectors: between the
// 8th and 9th shell, e.g. skin 1.3).  Only per-shell and per-lattice scalars are runtime
// values.
#define MX_SHELLS 8
struct MxGrid {
  float rds, mmax;     // 1 / ds, last interval
  float fr[MX_SHELLS]; // frac(R^2 / ds)
  float kb[MX_SHELLS]; // floor(R^2 / ds)
};
struct MxShells {
  float w[MX_SHELLS];  // rc^2 - R^2
  MxGrid g[2];         // density grid, force grid
  float a0;
  int pl, rw;          // plane and row strides of the ghost-extended arrays
  long long E;         // sites per sublattice array
  long long d_odd;     // extra offset of odd entries for sublattice-1 sites
};

struct MxStencil {
  int n_odd, n_even, n_far;
  int d_odd;        // extra offset of odd entries for sublattice-1 sites
  int n_rs, n_fs;   // density / force table intervals
  float rds, rds_f; // 1 / ds of the density / force grid
  MxEntry odd[MX_PAR_MAX], even[MX_PAR_MAX], far[ENS_MAX_ST];
  MxWalk walk;
  int fixed;   // 7 or 8: the built-in shell stencil of that many shells applies (see MxShells); 0: runtime
  MxShells sh;
};

// ------------------------------------------------------------ primitives
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier (all CTAs co-resident: cooperative launch).  Gives up after
// `limit` polls, raising err; returns false once err is set.  Every CTA still arrives
// before it waits, so the barrier that gave up completes its count and the CTAs that
// return leave no tile copy in flight (barriers sit between the tile phases).
__device__ __forceinline__ bool grid_sync(unsigned *bar, int *err, unsigned limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned gen = ld_acquire_u32(bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == gridDim.x) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire_u32(bar + 1) == gen) {
        if (++spins > limit) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (ok && *(volatile int *)err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// 5-D tiled TMA load into this CTA's own shared memory from this GPU's memory: box
// {4, TX+4, TY+4, TZ+4, 2} of float32.
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_addr(dst)),
      "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

// Knuth two-sum: s + c carries the running sum with the rounding error of every add.
__device__ __forceinline__ void two_sum(float &s, float &c, float x) {
  const float t = s + x;
  const float bp = t - s;
  c += (s - (t - bp)) + (x - bp);
  s = t;
}

__device__ __forceinline__ Geom lat_geom(const LatDesc &d) {
  Geom g;
  g.ecx = d.ecx;
  g.ey = d.ey;
  g.ez = d.ez;
  g.gcx = 2;
  g.gy = 2;
  g.gz = 2;
  g.bcx = d.bcx;
  g.by = d.by;
  g.bz = d.bz;
  g.images = 1;
  g.zimg = 1;
  g.E = d.E;
  g.Lx = d.Lx;
  g.Ly = d.Ly;
  g.Lz = d.Lz;
  g.iLx = 1.0 / d.Lx;
  g.iLy = 1.0 / d.Ly;
  g.iLz = 1.0 / d.Lz;
  return g;
}

__device__ __forceinline__ bool lat_active(const LatDesc &d) { return !d.primed || d.steps_done < d.steps_target; }

// Lists box site (s, cx, y, z) of lattice d when its drifted atom (displacement u from
// the ideal site) lies farther than sqrt(conv2) from it (conversion on).
__device__ __forceinline__ void ens_conv_check(const EnsParams &P, const LatDesc &d, int s, int cx, int y, int z,
                                               double ux, double uy, double uz) {
  if (!(P.conv2 > 0.0) || !d.cand) return;
  if (ux * ux + uy * uy + uz * uz <= P.conv2) return;
  const int slot = atomicAdd(d.cand_n, 1);
  if (slot < MB_CAND_CAP) d.cand[slot] = ((long long)z * d.by + y) * (2LL * d.bcx) + 2LL * cx + s;
}

__device__ __forceinline__ void ideal_pos(int s, int cx, int y, int z, double a0, double &X, double &Y, double &Z) {
  const double h = 0.5 * s;
  X = 0.5 * a0 * (double)(2 * cx + s);
  Y = a0 * ((double)y + h);
  Z = a0 * ((double)z + h);
}

} // namespace mb
