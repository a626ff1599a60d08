// Shared declarations of the misa_b200 library (host + device).
//
// Device layout ("sublattice-split SoA"): the reference indexes a BCC lattice
// with x doubled, so neighbouring memory cells alternate between the two
// simple-cubic sublattices and every warp mixes two stencils
// (src/kernels/kernel_itl.hpp:82,86).  Here each sublattice s in {0,1} is its own
// ghost-extended (ecx, ey, ez) array, x fastest, so a warp always walks one
// stencil and every neighbour fetch is a contiguous 32-site row.  The site at
// doubled ext index ex lives in sublattice ex & 1, column ex >> 1.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "../../include/misa_b200.h"

#define MB_MAX_STENCIL 320       // per parity; the reference's full stencil is about 228
#define MB_FTM2V 9.64853321233e-3 // (eV/A)/amu -> A/fs^2
#define MB_MVV2E (1.0 / MB_FTM2V) // amu A^2/fs^2 -> eV
#define MB_VACANT_POS 1.0e30      // position given to vacant sites: every r^2 test rejects them
#define MB_FLAG_ITL 0x40          // site code bit: an interstitial is within reach

namespace mb {

// Read-only 32-byte load through the non-coherent path (two 16-byte halves).
__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// ----------------------------------------------------------------- tracing
// NVTX range around an entry point's work (shows in Nsight timelines; costs nothing
// when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
#define MB_RANGE(name) ::mb::NvtxRange mb_nvtx_range_(name)

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define MB_CUDA(call)                                                                                          \
  do {                                                                                                         \
    cudaError_t e_ = (call);                                                                                   \
    if (e_ != cudaSuccess) return ::mb::cuda_fail(e_, #call);                                                  \
  } while (0)

#define MB_TRY(call)                                                                                           \
  do {                                                                                                         \
    int rc_ = (call);                                                                                          \
    if (rc_ != MB_OK) return rc_;                                                                              \
  } while (0)

// ------------------------------------------------------------ potential
// Per-knot cubic pieces.  value(p) = ((c3 p + c2) p + s) p + y on [m, m+1];
// d/dx value = (d2 p + d1) p + d0 with d = (s, 2 c2, 3 c3) / dx.
struct DevPot {
  int n_types, nr, nrho;
  double rdr, rdrho, rho_max, cutoff;
  const double4 *f_val;   // [nt][nr]   {y, s, c2, c3}
  const double4 *f_der;   // [nt][nr]   {d0, d1, d2, 0}
  const double4 *F_val;   // [nt][nrho]
  const double4 *F_der;   // [nt][nrho]
  const double4 *phi_val; // [np][nr]
  const double4 *phi_der; // [np][nr]
  const double2 *force1;  // single type: [nr][3] {f d0, phi d0}, {f d1, phi d1}, {f d2, phi d2}
  // single precision copies for the mixed path
  const float4 *f_val32;   // [nt][nr]  {y, s, c2, c3}
  const float2 *force32;   // single type: [nr][3] {f d0, phi d0}, {f d1, phi d1}, {f d2, phi d2}
  const float4 *phi_val32; // single type: [nr]
  // single type, squared-distance form for the mixed split kernels, on uniform grids in
  // s = r^2, built from the FP64 r-spline and interpolated linearly.  Density: per
  // interval {value at s_j, rise over the interval}.
  // Force: per knot {A, B} = {f'(r) / r, phi'(r) / r} (knot pairs are read, which
  // halves the table against per-interval storage and allows a finer grid).
  // n_rs = n_fs = 0 when not built (several types).
  int n_rs;            // density intervals
  double ds_r;
  const float2 *fs32;  // [n_rs]
  int n_fs;            // force intervals
  double ds_f;
  const float2 *ab32;  // [n_fs + 1] knots
  const float4 *ps32;  // [n_fs] per interval cubic of phi in p (energy steps)
};

struct PotHost;
int pot_build(const mb_eam_tables *t, PotHost **out);
void pot_free(PotHost *p);
const DevPot &pot_dev(const PotHost *p);

// ------------------------------------------------------------- geometry
struct Geom {
  int ecx, ey, ez; // ext size per sublattice
  int gcx, gy, gz; // ghost widths (cells along x)
  int bcx, by, bz; // box size per sublattice
  int images;      // 1: sites write their periodic ghost images (device-resident mode)
  int zimg;        // with images: 1 also along z; 0 for a z-slab of a larger lattice, whose
                   // z ghost layers come from the neighbouring slabs
  long long E;     // sites per sublattice array
  double Lx, Ly, Lz;
  double iLx, iLy, iLz; // 1 / L (0 when there is no periodic box)
};

struct StencilSet {
  int n;                          // entries per parity (equal for both)
  int n_near;                     // leading entries inside the cutoff at the ideal lattice (0: unknown)
  int off[2][MB_MAX_STENCIL];     // [sublattice] split-layout linear offsets
};

// Convert reference-style doubled-x linear offsets to split-layout offsets.
// parity_of_sublattice[s] selects which reference stencil (0 even, 1 odd) the sites
// of sublattice s walk.
int stencil_from_linear(const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd, int ext_x, int ext_y,
                        const Geom &g, const int parity_of_sublattice[2], StencilSet *out);
// BCC stencil of every site with ideal distance < reach (doubled-x linear form,
// ordered dz, dy, dx ascending), for an ext array of ext_x x ext_y.
int stencil_generate(double a0, double reach, int ext_x, int ext_y, int64_t *even, int64_t *odd, int cap, int *n,
                     int *reach_x, int *reach_y, int *reach_z);
int stencil_sort_by_distance(double a0, double cutoff, int ext_x, int ext_y, int64_t *even, int64_t *odd, int n,
                             int *n_near);

// ------------------------------------------------------ kernel arguments
struct Lattice64 {
  double *px, *py, *pz; // positions (ext)
  int8_t *code;         // type, < 0 vacant, MB_FLAG_ITL marks sites near an interstitial
  double *df;           // F'(rho) (ext)
  double *rho;          // optional rho output (ext) or nullptr
  double *vx, *vy, *vz; // velocities (box sites used)
  double *fx, *fy, *fz; // forces (box sites used)
  double *nx, *ny, *nz; // positions written by the drift (ext) or nullptr
};

struct Itl64 {
  int n;                   // count, when nd is null (lists fixed by the host)
  const int *nd;           // device-resident count (lists that change on the device), or null
  int cap;                 // capacity of the list
  int cap_flag;
  double *px, *py, *pz;    // current positions
  double *nx, *ny, *nz;    // next positions
  double *vx, *vy, *vz, *fx, *fy, *fz, *rho, *df;
  int8_t *type;
  int64_t *id;
  int *flag_list;          // flagged box sites (ext index)
  int *flag_count;         // [0] this step, [1] overflow marker
  double a0, reach;        // window radius in A (cutoff + skin)
};

struct StepParams {
  double rc2;
  double h;      // 0.5 * dt * ftm2v / mass
  double dt;
  double mass;
  int kick_pre;  // 1: v += h f before the energy sample (closes the previous step)
  int drift;     // 1: v += h f ; x_next = x + dt v
  // lattice -> interstitial conversion (conv2 > 0): sites whose drifted atom lies
  // farther than sqrt(conv2) from the ideal site are listed in cand (box index)
  double a0, conv2;
  long long *cand;
  int *cand_n;
};
#define MB_CAND_CAP 2048     // conversion candidates handled per step
#define MB_CONV_ITL_MAX 65536 // interstitial capacity with conversion on

// Ideal position of box site (s, cx, y, z): x doubled = 2 cx + s.
__host__ __device__ __forceinline__ void site_ideal(int s, int cx, int y, int z, double a0, double &X, double &Y,
                                                    double &Z) {
  const double h = 0.5 * s;
  X = 0.5 * a0 * (double)(2 * cx + s);
  Y = a0 * ((double)y + h);
  Z = a0 * ((double)z + h);
}

// kernels (mb_kernels64.cu)
// [z0, z1): the box layers a launch covers (z1 < 0: up to the last layer).  The
// interstitial passes then take the flagged sites in those layers and the
// interstitials whose wrapped z lies in them.
// outer: per-item masks of the outer stencil entries (beyond the cutoff at the ideal
// lattice) that some site of the item has inside the cutoff, one uint2 per item of the
// box (items_per_box).  The density pass writes them; a force pass given them walks only
// those entries, so it must run on the positions of the density pass that wrote them
// (null: the force pass walks every entry).
int launch_rho64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, double rc2,
                 double *e_partial, int energy, int skip_flagged, cudaStream_t s, int z0 = 0, int z1 = -1,
                 uint2 *outer = nullptr);
int launch_force64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const StepParams &sp,
                   double *e_partial, int energy, int skip_flagged, cudaStream_t s, int z0 = 0, int z1 = -1,
                   const uint2 *outer = nullptr);
// Work items (32-site row chunks) of the whole box: the length of the outer masks.
inline long long items_per_box(const Geom &g) { return (long long)((g.bcx + 31) / 32) * g.by * 2 * g.bz; }
// Outer-entry masks on (default), or off when MB_OUTER_MASKS=0 (the force passes then walk
// every outer entry: the same results, kept for checking that); read when a sim is
// created or an ensemble's walk is rebuilt.
inline bool outer_masks_on() {
  const char *v = getenv("MB_OUTER_MASKS");
  return !(v && v[0] == '0');
}
int launch_itl_mark64(const Geom &g, const Lattice64 &L, const Itl64 &I, cudaStream_t s);
// Flags the sites of layers [z0, z1) near an interstitial, without clearing or
// resetting the list first.
int launch_itl_mark_slab64(const Geom &g, const Lattice64 &L, const Itl64 &I, int z0, int z1, cudaStream_t s);
int launch_itl_rho64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const Itl64 &I,
                     double rc2, double *e_partial, int energy, cudaStream_t s, int z0 = 0, int z1 = -1);
int launch_itl_force64(const Geom &g, const StencilSet &st, const DevPot &pot, const Lattice64 &L, const Itl64 &I,
                       const StepParams &sp, double *e_partial, int energy, cudaStream_t s, int z0 = 0, int z1 = -1);
int launch_images64(const Geom &g, const Lattice64 &L, int what, cudaStream_t s, int z0 = 0,
                    int z1 = -1); // what: 1 pos+code, 2 df
// Lattice <-> interstitial bookkeeping after a drift (one CTA): candidates of
// sp.cand become interstitials (box order), then interstitials within sqrt(rec2) of a
// vacant site take it (list order, first claim wins).  counters: [0] conversions,
// [1] recombinations, [2] refused conversions (list full), [3] dropped candidates.
int launch_convert64(const Geom &g, const Lattice64 &L, const Itl64 &I, const StepParams &sp, double rec2,
                     int64_t *site_id, int *nd, long long *counters, cudaStream_t s);
int launch_kick_drift64(const Geom &g, const Lattice64 &L, const Itl64 &I, const StepParams &sp, cudaStream_t s,
                        int z0 = 0, int z1 = -1, int with_itl = 1);
int launch_reduce(const double *partials, int n, double *out, cudaStream_t s);
int energy_partials_needed();

// AoS conversion (mb_layout.cu)
// Records whose type has no potential table (type >= n_types) raise *bad_type and
// are kept out of the passes as vacant sites.
// [t0, t1): ext records (t1 < 0: to the end); [z0, z1): box layers (z1 < 0: to the last).
int launch_unpack_ext(const Geom &g, const mb_atom_element *aos, int ext_x, int ext_y, int ext_z, Lattice64 L,
                      int with_df, int *bad_type, int n_types, cudaStream_t s, long long t0 = 0, long long t1 = -1);
int launch_pack_ext(const Geom &g, mb_atom_element *aos, int ext_x, int ext_y, const Lattice64 &L, int what,
                    cudaStream_t s, int z0 = 0, int z1 = -1); // what: 1 rho+df, 2 force, 3 df only
int launch_unpack_box(const Geom &g, const mb_atom_element *aos, Lattice64 L, int with_f, int *bad_type,
                      int n_types, cudaStream_t s);
int launch_pack_box(const Geom &g, mb_atom_element *aos, const Lattice64 &L, const double *px, const double *py,
                    const double *pz, double h, int unkick, cudaStream_t s);
int launch_unpack_box_ids(const Geom &g, const mb_atom_element *aos, Lattice64 L, int with_f, int *bad_type,
                          int64_t *ids, int n_types, cudaStream_t s, int z0 = 0, int z1 = -1);
int launch_pack_box_ids(const Geom &g, mb_atom_element *aos, const Lattice64 &L, const double *px, const double *py,
                        const double *pz, double h, int unkick, const int64_t *ids, cudaStream_t s, int z0 = 0,
                        int z1 = -1);
int launch_df_from_rho(const Geom &g, const DevPot &pot, const Lattice64 &L, cudaStream_t s);
// z-slab halo layers (mb_layout.cu): sites of one message, and the pack (box layers ->
// buf) / unpack (buf -> ghost layers, z positions + z_shift) of one field: what 1 positions
// (c0, c1, c2), 2 df (c0), 3 site codes.
long long halo_sites(const Geom &g);
int launch_halo(const Geom &g, int what, int pack, int side, double *c0, double *c1, double *c2, int8_t *code,
                void *buf, double z_shift, cudaStream_t s);

// Half-neighbour hook passes (mb_half.cu): a decoded half-stencil offset.
struct HalfOff {
  long long off; // linear offset in the host's ext array
  int dx, dy, dz, pad_;
};
int half_stencil_build(const mb_device_domain &d, const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                       std::vector<HalfOff> &out, int &cap);
int launch_half64(bool force, mb_atom_element *aos, const mb_device_domain &d, const HalfOff *st, int cap,
                  const int n[2], const DevPot &P, double rc2, int *bad, cudaStream_t s);

// ------------------------------------------------------------ utilities
int device_sm_count();

} // namespace mb
