// Conversion between the host's AoS lattice records (mb_atom_element, the
// reference's _cuAtomElement, src/kernel_types.h:40-48) and the device's
// sublattice-split SoA arrays.
#include "mb_common.cuh"

namespace mb {

__device__ __forceinline__ long long split_index(const Geom &g, int ex, int ey, int ez) {
  // ex is a doubled column of the ghost-extended array
  return (long long)(ex & 1) * g.E + ((long long)ez * g.ey + ey) * g.ecx + (ex >> 1);
}

// Records [t0, t1) of the ext array (x fastest, then y, z: ext layers [t0, t1) / (ext_x * ext_y)).
__global__ void k_unpack_ext(const Geom g, const mb_atom_element *aos, int ext_x, int ext_y, int ext_z, Lattice64 L,
                             int with_df, int *bad_type, int n_types, long long t0, long long t1) {
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    const int ex = (int)(t % ext_x);
    const long long r = t / ext_x;
    const int ey = (int)(r % ext_y), ez = (int)(r / ext_y);
    const long long i = split_index(g, ex, ey, ez);
    const mb_atom_element &a = aos[t];
    int type = a.type;
    if (type >= n_types) { // no table for it: flagged, and kept out of the pair loops
      *bad_type = 1;
      type = -1;
    }
    const bool vac = type < 0;
    L.code[i] = (int8_t)(vac ? -1 : type);
    L.px[i] = vac ? MB_VACANT_POS : a.x[0];
    L.py[i] = vac ? MB_VACANT_POS : a.x[1];
    L.pz[i] = vac ? MB_VACANT_POS : a.x[2];
    if (with_df == 1) L.df[i] = a.df;
    if (with_df == 2 && L.rho) L.rho[i] = a.rho;
  }
}

// what: 1 rho+df, 2 force, 3 df only.  Only box sites with type >= 0 are written,
// as the reference's kernels do (src/kernels/kernel_itl.hpp:44,90-103).  Box sites
// [t0, t1) in box order (doubled x fastest, then y, z).
__global__ void k_pack_ext(const Geom g, mb_atom_element *aos, int ext_x, int ext_y, const Lattice64 L, int what,
                           int ghost_x, long long t0, long long t1) {
  const int bxd = 2 * g.bcx;
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % bxd);
    const long long r = t / bxd;
    const int by = (int)(r % g.by), bz = (int)(r / g.by);
    const int ex = bx + ghost_x, ey = by + g.gy, ez = bz + g.gz;
    const long long i = split_index(g, ex, ey, ez);
    if (L.code[i] < 0) continue;
    mb_atom_element &a = aos[((long long)ez * ext_y + ey) * ext_x + ex];
    if (what == 1) {
      a.rho = L.rho[i];
      a.df = L.df[i];
    } else if (what == 2) {
      a.f[0] = L.fx[i];
      a.f[1] = L.fy[i];
      a.f[2] = L.fz[i];
    } else {
      a.df = L.df[i];
    }
  }
}

// Box-order records (doubled x fastest, then y, z): records [t0, t1) are box layers
// [t0, t1) / (2 * bcx * by).
__global__ void k_unpack_box(const Geom g, const mb_atom_element *aos, Lattice64 L, int with_f, int *bad_type,
                             int64_t *ids, int n_types, long long t0, long long t1) {
  const int bxd = 2 * g.bcx;
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % bxd);
    const long long r = t / bxd;
    const int by = (int)(r % g.by), bz = (int)(r / g.by);
    const long long i = (long long)(bx & 1) * g.E + ((long long)(bz + g.gz) * g.ey + by + g.gy) * g.ecx +
                        (bx >> 1) + g.gcx;
    const mb_atom_element &a = aos[t];
    int type = a.type;
    if (type >= n_types) { // no table for it: flagged, and kept out of the pair loops
      *bad_type = 1;
      type = -1;
    }
    const bool vac = type < 0;
    L.code[i] = (int8_t)(vac ? -1 : type);
    L.px[i] = vac ? MB_VACANT_POS : a.x[0];
    L.py[i] = vac ? MB_VACANT_POS : a.x[1];
    L.pz[i] = vac ? MB_VACANT_POS : a.x[2];
    L.vx[i] = vac ? 0.0 : a.v[0];
    L.vy[i] = vac ? 0.0 : a.v[1];
    L.vz[i] = vac ? 0.0 : a.v[2];
    if (with_f) {
      L.fx[i] = vac ? 0.0 : a.f[0];
      L.fy[i] = vac ? 0.0 : a.f[1];
      L.fz[i] = vac ? 0.0 : a.f[2];
    }
    if (ids) ids[t] = a.id;
  }
}

// Box-order records of the synchronised state.  px/py/pz: positions of the
// step; unkick: v is stored half a step ahead and is brought back by h*f.
__global__ void k_pack_box(const Geom g, mb_atom_element *aos, const Lattice64 L, const double *px,
                           const double *py, const double *pz, double h, int unkick, const int64_t *ids, long long t0,
                           long long t1) {
  const int bxd = 2 * g.bcx;
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % bxd);
    const long long r = t / bxd;
    const int by = (int)(r % g.by), bz = (int)(r / g.by);
    const long long i = (long long)(bx & 1) * g.E + ((long long)(bz + g.gz) * g.ey + by + g.gy) * g.ecx +
                        (bx >> 1) + g.gcx;
    mb_atom_element a;
    const int c = L.code[i];
    a.id = ids ? ids[t] : t;
    a.type = c < 0 ? -1 : (c & 0x3F);
    a.pad_ = 0;
    if (c < 0) {
      for (int k = 0; k < 3; k++) a.x[k] = a.v[k] = a.f[k] = 0.0;
      a.rho = a.df = 0.0;
    } else {
      a.x[0] = px[i];
      a.x[1] = py[i];
      a.x[2] = pz[i];
      a.f[0] = L.fx[i];
      a.f[1] = L.fy[i];
      a.f[2] = L.fz[i];
      a.v[0] = L.vx[i] - (unkick ? h * a.f[0] : 0.0);
      a.v[1] = L.vy[i] - (unkick ? h * a.f[1] : 0.0);
      a.v[2] = L.vz[i] - (unkick ? h * a.f[2] : 0.0);
      a.rho = L.rho ? L.rho[i] : 0.0;
      a.df = L.df[i];
    }
    aos[t] = a;
  }
}

// calDf of the half-neighbour build (src/kernels/hip_kernels.hip.cpp:21-40).
__device__ __forceinline__ void spl_loc(double x, double rdx, int n, int &m, double &p) {
  const double pp = x * rdx;
  if (!(pp < (double)(n - 1))) {
    m = n - 2;
    p = 1.0;
    return;
  }
  int mm = min((int)pp, n - 2);
  p = fmin(pp - (double)mm, 1.0);
  m = mm;
}

__global__ void k_df_from_rho(const Geom g, const DevPot P, Lattice64 L) {
  const long long n = 2LL * g.bcx * g.by * g.bz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int cx = (int)(t % g.bcx);
    long long r = t / g.bcx;
    const int y = (int)(r % g.by);
    r /= g.by;
    const int s = (int)(r & 1), z = (int)(r >> 1);
    const long long i = (long long)s * g.E + ((long long)(z + g.gz) * g.ey + y + g.gy) * g.ecx + cx + g.gcx;
    const int c = L.code[i];
    if (c < 0) continue;
    int m;
    double p;
    spl_loc(L.rho[i], P.rdrho, P.nrho, m, p);
    const double4 d = ldg4(&P.F_der[(size_t)(c & 0x3F) * P.nrho + m]);
    L.df[i] = (d.z * p + d.y) * p + d.x;
  }
}

static int flat_grid(long long n) {
  long long g = (n + 255) / 256;
  const long long cap = 16LL * device_sm_count();
  if (g > cap) g = cap;
  return (int)(g > 0 ? g : 1);
}

int launch_unpack_ext(const Geom &g, const mb_atom_element *aos, int ext_x, int ext_y, int ext_z, Lattice64 L,
                      int with_df, int *bad_type, int n_types, cudaStream_t s, long long t0, long long t1) {
  const long long n = (long long)ext_x * ext_y * ext_z;
  if (t1 < 0 || t1 > n) t1 = n;
  if (t0 < 0) t0 = 0;
  if (t1 <= t0) return MB_OK;
  k_unpack_ext<<<flat_grid(t1 - t0), 256, 0, s>>>(g, aos, ext_x, ext_y, ext_z, L, with_df, bad_type, n_types, t0, t1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_pack_ext(const Geom &g, mb_atom_element *aos, int ext_x, int ext_y, const Lattice64 &L, int what,
                    cudaStream_t s, int z0, int z1) {
  if (z1 < 0) z1 = g.bz;
  const long long layer = 2LL * g.bcx * g.by;
  if (z1 <= z0) return MB_OK;
  k_pack_ext<<<flat_grid(layer * (z1 - z0)), 256, 0, s>>>(g, aos, ext_x, ext_y, L, what, 2 * g.gcx, layer * z0,
                                                           layer * z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_unpack_box_ids(const Geom &g, const mb_atom_element *aos, Lattice64 L, int with_f, int *bad_type,
                          int64_t *ids, int n_types, cudaStream_t s, int z0, int z1) {
  if (z1 < 0) z1 = g.bz;
  const long long layer = 2LL * g.bcx * g.by;
  if (z1 <= z0) return MB_OK;
  k_unpack_box<<<flat_grid(layer * (z1 - z0)), 256, 0, s>>>(g, aos, L, with_f, bad_type, ids, n_types, layer * z0,
                                                             layer * z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_unpack_box(const Geom &g, const mb_atom_element *aos, Lattice64 L, int with_f, int *bad_type,
                      int n_types, cudaStream_t s) {
  return launch_unpack_box_ids(g, aos, L, with_f, bad_type, nullptr, n_types, s);
}

int launch_pack_box_ids(const Geom &g, mb_atom_element *aos, const Lattice64 &L, const double *px, const double *py,
                        const double *pz, double h, int unkick, const int64_t *ids, cudaStream_t s, int z0, int z1) {
  if (z1 < 0) z1 = g.bz;
  const long long layer = 2LL * g.bcx * g.by;
  if (z1 <= z0) return MB_OK;
  k_pack_box<<<flat_grid(layer * (z1 - z0)), 256, 0, s>>>(g, aos, L, px, py, pz, h, unkick, ids, layer * z0,
                                                           layer * z1);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_pack_box(const Geom &g, mb_atom_element *aos, const Lattice64 &L, const double *px, const double *py,
                    const double *pz, double h, int unkick, cudaStream_t s) {
  return launch_pack_box_ids(g, aos, L, px, py, pz, h, unkick, nullptr, s);
}

int launch_df_from_rho(const Geom &g, const DevPot &pot, const Lattice64 &L, cudaStream_t s) {
  k_df_from_rho<<<flat_grid(2LL * g.bcx * g.by * g.bz), 256, 0, s>>>(g, pot, L);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb

// ------------------------------------------------------- z-slab halo layers
// A z-slab of a larger periodic lattice (one rank of a decomposed run) gets its z ghost
// layers from the neighbouring slabs.  A message is gz whole ext planes (both
// sublattices, x and y ghost columns included) of one field, ordered
// [component][sublattice][layer][y][x]: positions 3 components (double), df 1 (double),
// site codes 1 (int8).  side 0: my lowest gz box layers (for the slab below, its top
// ghost) / my bottom ghost layers; side 1: my highest gz box layers / my top ghost.
// Unpacked z positions get z_shift added (the periodic wrap between the last and the
// first slab).
namespace mb {

__global__ void k_halo(const Geom g, int what, int pack, int ez0, double *c0, double *c1, double *c2, int8_t *code,
                       void *buf, double z_shift) {
  const long long plane = (long long)g.ey * g.ecx;
  const long long per_s = plane * g.gz, n = 2 * per_s;
  const int ncomp = what == 1 ? 3 : 1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * ncomp;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / n);
    const long long r = t - (long long)c * n;
    const int s = (int)(r / per_s);
    const long long q = r - (long long)s * per_s; // layer-major inside the sublattice
    const long long idx = (long long)s * g.E + (long long)ez0 * plane + q;
    if (what == 3) {
      int8_t *b = static_cast<int8_t *>(buf);
      if (pack)
        b[r] = code[idx];
      else
        code[idx] = b[r];
    } else {
      double *col = c == 0 ? c0 : (c == 1 ? c1 : c2);
      double *b = static_cast<double *>(buf);
      if (pack)
        b[t] = col[idx];
      else
        col[idx] = c == 2 ? b[t] + z_shift : b[t];
    }
  }
}

long long halo_sites(const Geom &g) { return 2LL * g.gz * g.ey * g.ecx; }

int launch_halo(const Geom &g, int what, int pack, int side, double *c0, double *c1, double *c2, int8_t *code,
                void *buf, double z_shift, cudaStream_t s) {
  if (what < 1 || what > 3) return fail(MB_ERR_ARG, "halo field must be 1 (positions), 2 (df) or 3 (site codes)");
  if (side != 0 && side != 1) return fail(MB_ERR_ARG, "halo side must be 0 (below) or 1 (above)");
  if (!buf) return fail(MB_ERR_ARG, "null halo buffer");
  // ext z of the layers: packing reads box layers, unpacking fills ghost layers
  const int ez0 = pack ? (side == 0 ? g.gz : g.bz) : (side == 0 ? 0 : g.bz + g.gz);
  const long long n = halo_sites(g) * (what == 1 ? 3 : 1);
  long long grid = (n + 255) / 256;
  if (grid > 8LL * device_sm_count()) grid = 8LL * device_sm_count();
  k_halo<<<(int)(grid > 0 ? grid : 1), 256, 0, s>>>(g, what, pack, ez0, c0, c1, c2, code, buf,
                                                     what == 1 ? z_shift : 0.0);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb
