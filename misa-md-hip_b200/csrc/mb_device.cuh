// Device helpers shared by the FP64 kernels and the mixed-precision ensemble kernel:
// spline evaluation, ghost-image enumeration, deterministic reductions and the
// interstitial window walk.
#pragma once

#include "mb_common.cuh"

namespace mb {

// ------------------------------------------------------------ spline helpers
__device__ __forceinline__ void spl_locate(double x, double rdx, int n, int &m, double &p) {
  const double pp = x * rdx;
  if (!(pp < (double)(n - 1))) {
    m = n - 2;
    p = 1.0;
    return;
  }
  int mm = (int)pp;
  mm = min(mm, n - 2);
  p = fmin(pp - (double)mm, 1.0);
  m = mm;
}
// spl_locate for x inside the table's range (x < (n - 1) / rdx, which every pair inside
// a cutoff within the table satisfies): the same m and p there; past the range m is
// clamped and p is meaningless, for terms the caller masks out.
__device__ __forceinline__ void spl_locate_in(double x, double rdx, int n, int &m, double &p) {
  const double pp = x * rdx;
  m = min((int)pp, n - 2);
  p = pp - (double)m;
}
__device__ __forceinline__ double cubic(const double4 c, double p) { return ((c.w * p + c.z) * p + c.y) * p + c.x; }
__device__ __forceinline__ double quad(const double4 d, double p) { return (d.z * p + d.y) * p + d.x; }
__device__ __forceinline__ int pair_idx(int a, int b, int nt) {
  if (a > b) {
    int t = a;
    a = b;
    b = t;
  }
  return a * nt - a * (a - 1) / 2 + (b - a);
}
__device__ __forceinline__ double dF64(const DevPot &P, int t, double rho) {
  int m;
  double p;
  spl_locate(rho, P.rdrho, P.nrho, m, p);
  return quad(ldg4(&P.F_der[(size_t)t * P.nrho + m]), p);
}
__device__ __forceinline__ double F64(const DevPot &P, int t, double rho) {
  if (rho > P.rho_max)
    return ldg4(&P.F_val[(size_t)t * P.nrho + P.nrho - 1]).x + dF64(P, t, rho) * (rho - P.rho_max);
  int m;
  double p;
  spl_locate(rho, P.rdrho, P.nrho, m, p);
  return cubic(ldg4(&P.F_val[(size_t)t * P.nrho + m]), p);
}
__device__ __forceinline__ double rho_of_r(const DevPot &P, int t, double r) {
  int m;
  double p;
  spl_locate(r, P.rdr, P.nr, m, p);
  return cubic(ldg4(&P.f_val[(size_t)t * P.nr + m]), p);
}
// fpair * r for a pair (general types, global tables)
__device__ __forceinline__ double pair_psip(const DevPot &P, int ti, int tj, double r, double dfi, double dfj,
                                            double *phi_out) {
  int m;
  double p;
  spl_locate(r, P.rdr, P.nr, m, p);
  const double fj = quad(ldg4(&P.f_der[(size_t)tj * P.nr + m]), p);
  const double fi = (ti == tj) ? fj : quad(ldg4(&P.f_der[(size_t)ti * P.nr + m]), p);
  const int q = pair_idx(ti, tj, P.n_types);
  const double ph = quad(ldg4(&P.phi_der[(size_t)q * P.nr + m]), p);
  if (phi_out) *phi_out = cubic(ldg4(&P.phi_val[(size_t)q * P.nr + m]), p);
  return dfi * fj + dfj * fi + ph;
}

// -------------------------------------------------------------- geometry
__device__ __forceinline__ long long ext_index(const Geom &g, int s, int cx, int y, int z) {
  return (long long)s * g.E + ((long long)(z + g.gz) * g.ey + (y + g.gy)) * g.ecx + (cx + g.gcx);
}
__device__ __forceinline__ void decode_ext(const Geom &g, long long i, int &s, int &cx, int &y, int &z) {
  s = (int)(i / g.E);
  long long r = i - (long long)s * g.E;
  const long long row = r / g.ecx;
  cx = (int)(r - row * g.ecx) - g.gcx;
  z = (int)(row / g.ey) - g.gz;
  y = (int)(row - (long long)(z + g.gz) * g.ey) - g.gy;
}

// Calls fn(ext_index, shift_x, shift_y, shift_z) for every periodic ghost image
// of box site (s, cx, y, z).  Requires box >= ghost in every dimension.
template <class Fn>
__device__ __forceinline__ void for_images(const Geom &g, int s, int cx, int y, int z, Fn fn) {
  const bool xo[3] = {true, cx >= g.bcx - g.gcx, cx < g.gcx};
  const bool yo[3] = {true, y >= g.by - g.gy, y < g.gy};
  const bool zo[3] = {true, g.zimg && z >= g.bz - g.gz, g.zimg && z < g.gz};
  if (!(xo[1] || xo[2] || yo[1] || yo[2] || zo[1] || zo[2])) return;
  const int xs[3] = {cx + g.gcx, cx + g.gcx - g.bcx, cx + g.gcx + g.bcx};
  const int ys[3] = {y + g.gy, y + g.gy - g.by, y + g.gy + g.by};
  const int zs[3] = {z + g.gz, z + g.gz - g.bz, z + g.gz + g.bz};
  const double sx[3] = {0.0, -g.Lx, g.Lx}, sy[3] = {0.0, -g.Ly, g.Ly}, sz[3] = {0.0, -g.Lz, g.Lz};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (!zo[c]) continue;
#pragma unroll
    for (int b = 0; b < 3; b++) {
      if (!yo[b]) continue;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        if (!xo[a] || (a == 0 && b == 0 && c == 0)) continue;
        const long long idx = (long long)s * g.E + ((long long)zs[c] * g.ey + ys[b]) * g.ecx + xs[a];
        fn(idx, sx[a], sy[b], sz[c]);
      }
    }
  }
}

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed shuffle tree, then warps in order); result in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
  return t;
}

struct Window {
  int gx0, gy0, gz0, nx, ny, nz;
};

__device__ __forceinline__ Window make_window(double qx, double qy, double qz, double a0, double R) {
  Window w;
  w.gx0 = (int)floor((qx - R) / (0.5 * a0));
  const int gx1 = (int)ceil((qx + R) / (0.5 * a0));
  w.gy0 = (int)floor((qy - R) / a0) - 1;
  const int gy1 = (int)ceil((qy + R) / a0);
  w.gz0 = (int)floor((qz - R) / a0) - 1;
  const int gz1 = (int)ceil((qz + R) / a0);
  w.nx = gx1 - w.gx0 + 1;
  w.ny = gy1 - w.gy0 + 1;
  w.nz = gz1 - w.gz0 + 1;
  return w;
}

__device__ __forceinline__ int pmod_i(int a, int b) {
  int r = a % b;
  return r < 0 ? r + b : r;
}

// Candidate c of window w: returns false when its ideal site is out of reach;
// otherwise the ext index of the box site and the periodic shift of the image.
__device__ __forceinline__ bool window_site(const Geom &g, const Window &w, int c, double qx, double qy, double qz,
                                            double a0, double R, long long &idx, double &sx, double &sy,
                                            double &sz) {
  const int ix = c % w.nx;
  const int rest = c / w.nx;
  const int iy = rest % w.ny;
  const int iz = rest / w.ny;
  const int gx = w.gx0 + ix, gy = w.gy0 + iy, gz = w.gz0 + iz;
  const double h = 0.5 * (double)(gx & 1);
  const double ox = 0.5 * a0 * gx - qx, oy = a0 * (gy + h) - qy, oz = a0 * (gz + h) - qz;
  if (ox * ox + oy * oy + oz * oz >= R * R) return false;
  const int bxd = 2 * g.bcx;
  const int bx = pmod_i(gx, bxd), by = pmod_i(gy, g.by), bz = pmod_i(gz, g.bz);
  sx = (double)((gx - bx) / bxd) * g.Lx;
  sy = (double)((gy - by) / g.by) * g.Ly;
  sz = (double)((gz - bz) / g.bz) * g.Lz;
  idx = ext_index(g, bx & 1, bx >> 1, by, bz);
  return true;
}

// The reach test of candidate c alone (the same arithmetic as window_site /
// window_site_rel, so the same candidates pass).
__device__ __forceinline__ bool window_in_reach(const Window &w, int c, double qx, double qy, double qz, double a0,
                                                double R) {
  const int ix = c % w.nx;
  const int rest = c / w.nx;
  const int iy = rest % w.ny;
  const int iz = rest / w.ny;
  const int gx = w.gx0 + ix, gy = w.gy0 + iy, gz = w.gz0 + iz;
  const double h = 0.5 * (double)(gx & 1);
  const double ox = 0.5 * a0 * gx - qx, oy = a0 * (gy + h) - qy, oz = a0 * (gz + h) - qz;
  return ox * ox + oy * oy + oz * oz < R * R;
}

// In-reach candidates of a window, listed by one warp in candidate order: list[k] for
// k < the returned count (list: this warp's cap entries of shared memory).  The reach
// test is cheap arithmetic and about 1 candidate in 8 passes (a sphere in its bounding
// box of sites), so the walk that follows loads only real sites, several per lane at
// once, instead of one dependent load chain per round of 32 candidates.  Returns -1
// when more than cap candidates pass (the caller then walks every candidate).
__device__ __forceinline__ int window_compact(const Window &w, double qx, double qy, double qz, double a0, double R,
                                              int *list, int cap) {
  const int lane = threadIdx.x & 31;
  const int ncand = w.nx * w.ny * w.nz;
  int n = 0;
  for (int base = 0; base < ncand; base += 32) {
    const int c = base + lane;
    const bool in = c < ncand && window_in_reach(w, c, qx, qy, qz, a0, R);
    const unsigned m = __ballot_sync(0xffffffffu, in);
    const int k = n + __popc(m & ((1u << lane) - 1u));
    if (in && k < cap) list[k] = c;
    n += __popc(m);
  }
  __syncwarp();
  return n <= cap ? n : -1;
}
#define MB_WIN_LIST 256 // compacted window entries per warp

// Appends this lane's entry (when `add`) to list[0 .. cap) with one atomicAdd on *count
// per warp instead of one per lane (many lanes appending at once would serialise on the
// counter); every lane of the warp must call it.  Entries past cap are dropped and
// *overflow is set.  The order of entries within a call follows the lanes.
__device__ __forceinline__ void warp_append(bool add, int value, int *count, int *list, int cap, int *overflow) {
  const unsigned m = __ballot_sync(0xffffffffu, add);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  int first = 0;
  if (lane == leader) first = atomicAdd(count, __popc(m));
  first = __shfl_sync(0xffffffffu, first, leader);
  if (!add) return;
  const int slot = first + __popc(m & ((1u << lane) - 1u));
  if (slot < cap)
    list[slot] = value;
  else
    *overflow = 1;
}

// Same candidate walk, returning the ideal image position relative to the query point
// (ox, oy, oz) instead of the periodic shift.
__device__ __forceinline__ bool window_site_rel(const Geom &g, const Window &w, int c, double qx, double qy,
                                                double qz, double a0, double R, long long &idx, double &ox,
                                                double &oy, double &oz) {
  const int ix = c % w.nx;
  const int rest = c / w.nx;
  const int iy = rest % w.ny;
  const int iz = rest / w.ny;
  const int gx = w.gx0 + ix, gy = w.gy0 + iy, gz = w.gz0 + iz;
  const double h = 0.5 * (double)(gx & 1);
  ox = 0.5 * a0 * gx - qx;
  oy = a0 * (gy + h) - qy;
  oz = a0 * (gz + h) - qz;
  if (ox * ox + oy * oy + oz * oz >= R * R) return false;
  const int bxd = 2 * g.bcx;
  const int bx = pmod_i(gx, bxd), by = pmod_i(gy, g.by), bz = pmod_i(gz, g.bz);
  idx = ext_index(g, bx & 1, bx >> 1, by, bz);
  return true;
}

__device__ __forceinline__ double min_image(double d, double L, double iL) { return d - L * rint(d * iL); }

// ------------------------------------------------- conversion helpers
// In-place ascending bitonic sort of n2 (a power of two) keys by the whole block.
__device__ __forceinline__ void bitonic_sort(long long *key, int n2) {
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < n2; t += blockDim.x) {
        const int p = t ^ j;
        if (p > t) {
          const bool up = (t & k) == 0;
          const long long a = key[t], b = key[p];
          if ((a > b) == up) {
            key[t] = b;
            key[p] = a;
          }
        }
      }
      __syncthreads();
    }
}

__device__ __forceinline__ void decode_box(const Geom &g, long long t, int &s, int &cx, int &y, int &z) {
  const long long bx = 2LL * g.bcx;
  const int xd = (int)(t % bx);
  const long long r = t / bx;
  y = (int)(r % g.by);
  z = (int)(r / g.by);
  s = xd & 1;
  cx = xd >> 1;
}

__device__ __forceinline__ int pmod_int(long long a, int b) {
  long long r = a % b;
  return (int)(r < 0 ? r + b : r);
}

} // namespace mb
