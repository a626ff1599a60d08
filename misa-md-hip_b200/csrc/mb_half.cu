// Half-neighbour (Newton's third law) passes of the drop-in hooks: the reference's
// USE_NEWTONS_THIRD_LOW build (src/md_hip_config.h:12; pair shares in
// src/kernels/kernel_pairs.hpp:21-32 and :39-60; half stencils taken at
// src/hip_arch_acc_imp.cpp:118-130; the df pass it enables at :183-205).
//
// The host hands over half stencils (one offset of each opposite pair).  Each pair
// (i, i + o) with i a box site belongs to the pass once and both atoms receive their
// share, ghost records included; the host adds a ghost record's shares to the atom it
// images (its reverse ghost communication).  Every ext record's rho (or f) is the sum
// of the shares it received, starting from zero.
//
// On the device each record gathers its shares instead of scattering them: it sums
// the pairs where it is the first atom (a box record, forward offsets of its parity)
// and those where it is the second (first atom self - o, a box site whose parity
// selects o).  The gather needs no atomics and its sums do not depend on thread
// order.  Records are read straight from the host's AoS layout (104-byte records,
// doubled-x linear index); the pair arithmetic is that of the full-neighbour FP64
// kernels.
#include <vector>

#include "mb_common.cuh"
#include "mb_device.cuh"

namespace mb {

struct HalfGeo {
  int ex, ey, ez;       // ext sizes (x doubled)
  int gx, gy, gz;       // ghost widths
  int bx, by, bz;       // box sizes
  long long start_x;    // global x index of the first box column (stencil parity)
  int n[2];             // half-stencil entries per parity
  int n_types;
};

__device__ __forceinline__ bool half_in_box(const HalfGeo &G, int x, int y, int z) {
  return x >= G.gx && x < G.gx + G.bx && y >= G.gy && y < G.gy + G.by && z >= G.gz && z < G.gz + G.bz;
}
__device__ __forceinline__ int half_parity(const HalfGeo &G, int x) {
  return (int)(((long long)(x - G.gx) + G.start_x) & 1LL);
}

struct HalfAtom {
  int type;
  double x, y, z, df;
};

__device__ __forceinline__ HalfAtom half_load(const mb_atom_element *aos, long long i, int n_types, int *bad) {
  const mb_atom_element &a = aos[i];
  HalfAtom h;
  h.type = a.type;
  if (h.type >= n_types) { // no table for it: flagged, and kept out of the sums
    *bad = 1;
    h.type = -1;
  }
  h.x = a.x[0];
  h.y = a.x[1];
  h.z = a.x[2];
  h.df = a.df;
  return h;
}

// Share of the pair (self, other) that self receives.
template <bool FORCE>
__device__ __forceinline__ void half_share(const DevPot &P, double rc2, const HalfAtom &s, const HalfAtom &o,
                                           double &ax, double &ay, double &az) {
  if (o.type < 0) return;
  const double dx = s.x - o.x, dy = s.y - o.y, dz = s.z - o.z;
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (d2 >= rc2) return;
  const double r = sqrt(d2);
  if constexpr (FORCE) {
    const double fp = -pair_psip(P, s.type, o.type, r, s.df, o.df, nullptr) / r;
    ax += dx * fp;
    ay += dy * fp;
    az += dz * fp;
  } else {
    ax += rho_of_r(P, o.type, r);
  }
}

template <bool FORCE>
__global__ void k_half64(mb_atom_element *aos, const HalfGeo G, const HalfOff *st, int cap, const DevPot P, double rc2,
                         int *bad) {
  const long long n = (long long)G.ex * G.ey * G.ez;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % G.ex);
    const long long r = t / G.ex;
    const int y = (int)(r % G.ey), z = (int)(r / G.ey);
    const HalfAtom s = half_load(aos, t, G.n_types, bad);
    double ax = 0.0, ay = 0.0, az = 0.0;
    if (s.type >= 0) {
      if (half_in_box(G, x, y, z)) { // first atom of the pairs along its own half stencil
        const int p = half_parity(G, x);
        for (int k = 0; k < G.n[p]; k++) {
          const HalfOff e = st[p * cap + k];
          half_share<FORCE>(P, rc2, s, half_load(aos, t + e.off, G.n_types, bad), ax, ay, az);
        }
      }
      for (int q = 0; q < 2; q++) // second atom of the pairs whose first atom is a box site
        for (int k = 0; k < G.n[q]; k++) {
          const HalfOff e = st[q * cap + k];
          const int xi = x - e.dx, yi = y - e.dy, zi = z - e.dz;
          if (!half_in_box(G, xi, yi, zi) || half_parity(G, xi) != q) continue;
          half_share<FORCE>(P, rc2, s, half_load(aos, t - e.off, G.n_types, bad), ax, ay, az);
        }
    }
    if constexpr (FORCE) {
      aos[t].f[0] = ax;
      aos[t].f[1] = ay;
      aos[t].f[2] = az;
    } else {
      aos[t].rho = ax;
    }
  }
}

// Decodes and checks the host's half stencils for the domain d.
int half_stencil_build(const mb_device_domain &d, const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                       std::vector<HalfOff> &out, int &cap) {
  const long long ex = d.ext_size_x, ey = d.ext_size_y, plane = ex * ey;
  cap = (int)std::max(n_even, n_odd);
  if (cap == 0) return fail(MB_ERR_ARG, "empty half stencil");
  out.assign(2 * (size_t)cap, HalfOff{});
  const int64_t *src[2] = {even, odd};
  const size_t cnt[2] = {n_even, n_odd};
  for (int p = 0; p < 2; p++)
    for (size_t k = 0; k < cnt[p]; k++) {
      const long long o = src[p][k];
      const long long dz = (o >= 0 ? o + plane / 2 : o - plane / 2) / plane;
      const long long rem = o - dz * plane;
      const long long dy = (rem >= 0 ? rem + ex / 2 : rem - ex / 2) / ex;
      const long long dx = rem - dy * ex;
      if (o == 0) return fail(MB_ERR_ARG, "half stencil holds the zero offset");
      if (llabs(dx) > d.ghost_size_x || llabs(dy) > d.ghost_size_y || llabs(dz) > d.ghost_size_z)
        return fail(MB_ERR_ARG, "half-stencil offset reaches beyond the ghost region");
      out[p * (size_t)cap + k] = HalfOff{o, (int)dx, (int)dy, (int)dz, 0};
    }
  // each pair once: the reverse of an offset must not be in the stencil of the
  // partner's parity
  for (int p = 0; p < 2; p++)
    for (size_t k = 0; k < cnt[p]; k++) {
      const HalfOff &e = out[p * (size_t)cap + k];
      const int q = (p + (int)(e.dx & 1)) & 1;
      for (size_t j = 0; j < cnt[q]; j++)
        if (out[q * (size_t)cap + j].off == -e.off)
          return fail(MB_ERR_ARG, "not a half stencil: an offset and its reverse are both present");
    }
  return MB_OK;
}

int launch_half64(bool force, mb_atom_element *aos, const mb_device_domain &d, const HalfOff *st, int cap,
                  const int n[2], const DevPot &P, double rc2, int *bad, cudaStream_t s) {
  HalfGeo G;
  G.ex = d.ext_size_x;
  G.ey = d.ext_size_y;
  G.ez = d.ext_size_z;
  G.gx = d.ghost_size_x;
  G.gy = d.ghost_size_y;
  G.gz = d.ghost_size_z;
  G.bx = d.box_size_x;
  G.by = d.box_size_y;
  G.bz = d.box_size_z;
  G.start_x = d.box_index_start_x;
  G.n[0] = n[0];
  G.n[1] = n[1];
  G.n_types = P.n_types;
  const long long total = (long long)G.ex * G.ey * G.ez;
  const int grid = (int)std::min<long long>((total + 255) / 256, 8LL * device_sm_count());
  if (force)
    k_half64<true><<<grid, 256, 0, s>>>(aos, G, st, cap, P, rc2, bad);
  else
    k_half64<false><<<grid, 256, 0, s>>>(aos, G, st, cap, P, rc2, bad);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

} // namespace mb
