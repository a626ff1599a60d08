// Ensemble of independent lattices advanced by the mixed-precision persistent
// kernel (mb_ensemble.cu): host side.  Lattices (slots) can be added and removed
// while others are mid-run, each with its own step target, which is what the
// serving loop builds continuous batching on.
#include <cudaTypedefs.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "mb_ensemble_kernel.cuh"

namespace mb {

size_t ens_smem_bytes(int nsm);
int ens_launch(const EnsParams &P, int grid, cudaStream_t s);
int ens_max_grid(int nsm);
int ens_energy_launch(const LatDesc *lats, int n, const int *tile_first, const double *epart, double *out,
                      cudaStream_t s);
int mx_launch_step(const EnsParams &P, const MxStencil &S, int lat, int energy, cudaStream_t s, cudaEvent_t *ev,
                   double *out);


static const int kShapes[ENS_NSHAPE][3] = {{16, 4, 4}, {8, 8, 4}, {8, 4, 8}, {4, 8, 8}};

static int shape_bytes(int k) { return 2 * (kShapes[k][0] + 4) * (kShapes[k][1] + 4) * (kShapes[k][2] + 4) * 16; }

// ------------------------------------------------------------ TMA encode
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

static int encode_tile_map(CUtensorMap *m, float4 *u4, int ecx, int ey, int ez, int shape) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(MB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[5] = {4, (cuuint64_t)ecx, (cuuint64_t)ey, (cuuint64_t)ez, 2};
  cuuint64_t strides[4] = {16, 16ull * ecx, 16ull * ecx * ey, 16ull * ecx * ey * ez};
  cuuint32_t box[5] = {4, (cuuint32_t)(kShapes[shape][0] + 4), (cuuint32_t)(kShapes[shape][1] + 4),
                       (cuuint32_t)(kShapes[shape][2] + 4), 2};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, (void *)u4, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return MB_OK;
}

// ------------------------------------------------------------ kernels
__global__ void k_ens_upload(LatDesc d, const mb_atom_element *aos, int64_t *ids, double a0, int *bad, int n_types) {
  const long long n = 2LL * d.bcx * d.by * d.bz;
  const int bxd = 2 * d.bcx;
  const Geom g = lat_geom(d);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % bxd);
    const long long r = t / bxd;
    const int by = (int)(r % d.by), bz = (int)(r / d.by);
    const int s = bx & 1, cx = bx >> 1;
    const long long i = (long long)s * d.E + ((long long)(bz + 2) * d.ey + by + 2) * d.ecx + cx + 2;
    const mb_atom_element &a = aos[t];
    int type = a.type;
    if (type >= n_types) { // no table for it: flagged, and kept out of the pair loops
      *bad = 1;
      type = -1;
    }
    const bool vac = type < 0;
    double X, Y, Z;
    ideal_pos(s, cx, by, bz, a0, X, Y, Z);
    const double ux = vac ? 0.0 : a.x[0] - X, uy = vac ? 0.0 : a.x[1] - Y, uz = vac ? 0.0 : a.x[2] - Z;
    d.code[i] = (int8_t)(vac ? -1 : type);
    d.ux[i] = ux;
    d.uy[i] = uy;
    d.uz[i] = uz;
    d.vx[i] = vac ? 0.0 : a.v[0];
    d.vy[i] = vac ? 0.0 : a.v[1];
    d.vz[i] = vac ? 0.0 : a.v[2];
    d.fx[i] = d.fy[i] = d.fz[i] = 0.f;
    d.rho[i] = 0.f;
    const float4 u = vac ? make_float4(ENS_VACANT, ENS_VACANT, ENS_VACANT, 0.f)
                         : make_float4((float)ux, (float)uy, (float)uz, 0.f);
    const int8_t c = (int8_t)(vac ? -1 : type);
    ids[t] = a.id;
    d.u4[0][i] = u;
    d.u4[1][i] = u;
    for_images(g, s, cx, by, bz, [&](long long idx, double, double, double) {
      d.u4[0][idx] = u;
      d.u4[1][idx] = u;
      d.code[idx] = c;
    });
  }
}

// Synchronised records of a lattice: positions and velocities are stored one drift /
// half kick ahead once primed and are brought back here.
__global__ void k_ens_pack(LatDesc d, mb_atom_element *aos, const int64_t *ids, double a0, double h, double dt) {
  const long long n = 2LL * d.bcx * d.by * d.bz;
  const int bxd = 2 * d.bcx;
  const float4 *u_df = d.u4[d.cur ^ 1];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % bxd);
    const long long r = t / bxd;
    const int by = (int)(r % d.by), bz = (int)(r / d.by);
    const int s = bx & 1, cx = bx >> 1;
    const long long i = (long long)s * d.E + ((long long)(bz + 2) * d.ey + by + 2) * d.ecx + cx + 2;
    mb_atom_element a;
    const int c = d.code[i];
    a.id = ids[t];
    a.type = c < 0 ? -1 : (c & 0x3F);
    a.pad_ = 0;
    if (c < 0) {
      for (int k = 0; k < 3; k++) a.x[k] = a.v[k] = a.f[k] = 0.0;
      a.rho = a.df = 0.0;
    } else {
      double X, Y, Z;
      ideal_pos(s, cx, by, bz, a0, X, Y, Z);
      const double f[3] = {(double)d.fx[i], (double)d.fy[i], (double)d.fz[i]};
      double v[3] = {d.vx[i], d.vy[i], d.vz[i]};
      double u[3] = {d.ux[i], d.uy[i], d.uz[i]};
      if (d.primed) {
        for (int k = 0; k < 3; k++) u[k] -= dt * v[k]; // undo the drift to the next step
        for (int k = 0; k < 3; k++) v[k] -= h * f[k];  // undo the half kick
      }
      a.x[0] = X + u[0];
      a.x[1] = Y + u[1];
      a.x[2] = Z + u[2];
      for (int k = 0; k < 3; k++) {
        a.v[k] = v[k];
        a.f[k] = f[k];
      }
      a.rho = (double)d.rho[i];
      a.df = d.primed ? (double)u_df[i].w : 0.0;
    }
    aos[t] = a;
  }
}

// ------------------------------------------------------------ host types
struct LatHost {
  bool used = false;
  LatDesc d{};
  int cells[3] = {0, 0, 0};
  int cap_itl = 0;
  void *block = nullptr; // every array of the lattice, one allocation
  size_t bytes = 0;
  int64_t *ids = nullptr;
  int64_t *iids = nullptr;
  std::vector<int64_t> host_iids;
  CUtensorMap tmap[2];
  std::vector<double> e_step, e_pe, e_ke;
  int policy_shape = -1;
};

} // namespace mb

struct mb_ensemble {
  mb_ensemble_config cfg{};
  mb::PotHost *pot = nullptr;
  mb::EnsParams P{};
  std::vector<mb::LatHost> slots;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[6] = {};
  // device work lists (rebuilt when slots change)
  mb::LatDesc *d_lats = nullptr;
  int *d_tile_lat = nullptr, *d_tile_idx = nullptr, *d_tile_first = nullptr, *d_itl_lats = nullptr;
  CUtensorMap *d_tmaps = nullptr;
  double *d_epart = nullptr, *d_eout = nullptr, *d_eitl = nullptr;
  unsigned *d_bar = nullptr;
  int *d_err = nullptr, *d_bad = nullptr;
  size_t cap_lats = 0, cap_tiles = 0;
  std::vector<int> order; // compact index -> slot
  std::vector<int> slot_pos; // slot -> compact index (-1 if absent)
  int n_tiles = 0;
  int grid = 0, max_grid = 0;
  bool dirty = true;
  bool synced_desc = true; // host copies of the dynamic descriptor fields are current
  cudaGraphExec_t graph = nullptr;
  bool graphs_ok = true;
  int policy = -1; // -1: size model per lattice; 0..3: one shape for all
  int mode = 0;  // 0: split kernels when the built-in shells apply, else persistent; 1: persistent; 2: split
  unsigned bar_spins = ENS_BAR_SPINS; // grid-barrier poll limit of the persistent kernel
  double conv_d = 0.0, rec_d = 0.0; // lattice <-> interstitial conversion (off while conv_d == 0)
  int split = 0; // kernels in use: 0 persistent, 1 split with the brick walk, 2 split with the linear walk
  unsigned *d_item_first = nullptr; // linear walk: first item of each lattice
  double *d_epart_items = nullptr;  // split: energy partials per walk item
  uint2 *d_outer_items = nullptr;   // split: outer-entry masks per walk item
  size_t cap_items = 0;
  int *d_icell = nullptr; // interstitial cell lists of every lattice (rebuilt each step)
  size_t cap_icell = 0;
  mb::MxStencil mxs{};
  size_t device_bytes = 0;
  size_t fixed_bytes = 0;
  long long launches = 0;
  std::mutex mu;
};

namespace mb {

static int edalloc(mb_ensemble *e, void **p, size_t bytes) {
  cudaError_t r = cudaMalloc(p, bytes);
  if (r != cudaSuccess) {
    *p = nullptr;
    return fail(MB_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                  cudaGetErrorString(r));
  }
  e->device_bytes += bytes;
  e->fixed_bytes += bytes;
  return MB_OK;
}

// Stencil tables of the tile kernel: every BCC site closer than reach, per sublattice.
static int ens_stencil(mb_ensemble *e) {
  const double a0 = e->cfg.lattice_const, reach = e->cfg.cutoff + e->cfg.stencil_skin;
  const int EX = 1 << 20, EY = 1 << 10;
  int64_t even[MB_MAX_STENCIL], odd[MB_MAX_STENCIL];
  int n = 0, rx, ry, rz;
  MB_TRY(stencil_generate(a0, reach, EX, EY, even, odd, MB_MAX_STENCIL, &n, &rx, &ry, &rz));
  if (n > ENS_MAX_ST) return fail(MB_ERR_ARG, "stencil longer than the tile kernel supports (cutoff + skin too large)");
  EnsParams &P = e->P;
  P.n_st = n;
  const double rdr = P.P.rdr;
  int n_near[2] = {0, 0};
  for (int s = 0; s < 2; s++) {
    const int64_t *src0 = s ? odd : even;
    // entries ordered by ideal distance: the ones inside the cutoff first (walked
    // without a per-pair branch), the outer shells after (mostly beyond the cutoff)
    std::vector<std::pair<double, int64_t>> ord;
    for (int k = 0; k < n; k++) {
      const long long o = src0[k];
      long long dz = (o >= 0 ? (o + (long long)EX * EY / 2) : (o - (long long)EX * EY / 2)) / ((long long)EX * EY);
      long long rem = o - dz * (long long)EX * EY;
      long long dy = (rem >= 0 ? rem + EX / 2 : rem - EX / 2) / EX;
      long long dx = rem - dy * EX;
      const int s2 = (int)((s + dx) & 1);
      const double ox = 0.5 * (double)dx, oy = (double)dy + 0.5 * (s2 - s), oz = (double)dz + 0.5 * (s2 - s);
      ord.push_back({a0 * sqrt(ox * ox + oy * oy + oz * oz), o});
    }
    std::stable_sort(ord.begin(), ord.end(),
                     [](const std::pair<double, int64_t> &x, const std::pair<double, int64_t> &y) {
                       return x.first < y.first;
                     });
    for (int k = 0; k < n; k++)
      if (ord[k].first < e->cfg.cutoff) n_near[s]++;
    for (int k = 0; k < n; k++) {
      const long long o = ord[k].second;
      long long dz = (o >= 0 ? (o + (long long)EX * EY / 2) : (o - (long long)EX * EY / 2)) / ((long long)EX * EY);
      long long rem = o - dz * (long long)EX * EY;
      long long dy = (rem >= 0 ? rem + EX / 2 : rem - EX / 2) / EX;
      long long dx = rem - dy * EX;
      const long long t = s + dx;
      const int s2 = (int)(t & 1);
      const long long dcx = (t - s2) / 2;
      if (llabs(dcx) > 2 || llabs(dy) > 2 || llabs(dz) > 2)
        return fail(MB_ERR_ARG, "stencil reaches beyond the 2-cell tile halo (cutoff + skin too large)");
      P.sd[s][k] = make_char4((signed char)(s2 - s), (signed char)dcx, (signed char)dy, (signed char)dz);
      // ideal X_i - X_j
      const double ox = 0.5 * (double)dx, oy = (double)dy + 0.5 * (s2 - s), oz = (double)dz + 0.5 * (s2 - s);
      const double cx = -a0 * ox, cy = -a0 * oy, cz = -a0 * oz;
      const double R = sqrt(cx * cx + cy * cy + cz * cz);
      P.ck[s][k] = make_float4((float)cx, (float)cy, (float)cz, (float)R);
      const double pk = R * rdr;
      const double mk = floor(pk);
      P.kf[s][k] = make_float2((float)(pk - mk), (float)mk);
      for (int sh = 0; sh < ENS_NSHAPE; sh++) {
        const int TXH = kShapes[sh][0] + 4, TYH = kShapes[sh][1] + 4, TZH = kShapes[sh][2] + 4;
        P.soff[sh][s][k] = (int)((s2 - s) * TXH * TYH * TZH + (dz * TYH + dy) * TXH + dcx);
      }
    }
  }
  if (n_near[0] != n_near[1]) return fail(MB_ERR_STATE, "even and odd stencils differ inside the cutoff");
  P.n_near = n_near[0];
  for (int sh = 0; sh < ENS_NSHAPE; sh++) {
    P.shape_dims[sh][0] = kShapes[sh][0];
    P.shape_dims[sh][1] = kShapes[sh][1];
    P.shape_dims[sh][2] = kShapes[sh][2];
    P.shape_dims[sh][3] = shape_bytes(sh);
    auto lg = [](int v) {
      int l = 0;
      while ((1 << l) < v) l++;
      return l;
    };
    P.shape_log[sh][0] = lg(kShapes[sh][0]);
    P.shape_log[sh][1] = lg(kShapes[sh][1]);
    P.shape_log[sh][2] = lg(kShapes[sh][2]);
    P.shape_log[sh][3] = P.shape_log[sh][0] + P.shape_log[sh][1] + P.shape_log[sh][2];
  }
  return MB_OK;
}

// Tile shape for a lattice: fewest padded sites, ties to the smaller halo.
static int model_shape(int bcx, int by, int bz) {
  int best = 0;
  double best_cost = 1e300;
  for (int k = 0; k < ENS_NSHAPE; k++) {
    const long long tiles = (long long)((bcx + kShapes[k][0] - 1) / kShapes[k][0]) *
                            ((by + kShapes[k][1] - 1) / kShapes[k][1]) * ((bz + kShapes[k][2] - 1) / kShapes[k][2]);
    const double cost = (double)tiles * (512.0 + 0.05 * (shape_bytes(k) / 16 - 512));
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = k;
    }
  }
  return best;
}

static size_t lattice_bytes(int cx, int cy, int cz, int cap_itl) {
  const size_t E = (size_t)(cx + 4) * (cy + 4) * (cz + 4), n = 2 * E, nb = 2 * (size_t)cx * cy * cz;
  auto a = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const int per = 2 * 4 * 64 + 64; // flagged sites per interstitial (upper bound of the window sphere)
  const size_t ci = (size_t)std::max(1, cap_itl);
  return 2 * a(n * 16) + 6 * a(n * 8) + 4 * a(n * 4) + a(n) + a(nb * 8) + a(ci * 8) * 16 + a(ci) +
         a((size_t)std::max(1, cap_itl * per) * 4) + a(16) + a(ci * 8) + a(MB_CAND_CAP * 8) + a(16) + a(32);
}

static int sync_desc(mb_ensemble *e) {
  // pull the device-updated fields (buffer parity, counters) back into the slots
  if (e->synced_desc || e->order.empty()) {
    e->synced_desc = true;
    return MB_OK;
  }
  std::vector<LatDesc> tmp(e->order.size());
  MB_CUDA(cudaMemcpyAsync(tmp.data(), e->d_lats, sizeof(LatDesc) * tmp.size(), cudaMemcpyDeviceToHost, e->stream));
  MB_CUDA(cudaStreamSynchronize(e->stream));
  for (size_t c = 0; c < e->order.size(); c++) {
    LatDesc &d = e->slots[e->order[c]].d;
    d.cur = tmp[c].cur;
    d.primed = tmp[c].primed;
    d.steps_done = tmp[c].steps_done;
    d.n_itl = tmp[c].n_itl; // conversions change it on the device
  }
  e->synced_desc = true;
  return MB_OK;
}

static void drop_graph(mb_ensemble *e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
}

// Rebuild descriptors, tile lists and tensor maps after slots or shapes change.
static const char *mx_stencil(const mb_ensemble *e, const LatDesc &d, MxStencil &S);

static int rebuild(mb_ensemble *e) {
  MB_TRY(sync_desc(e));
  drop_graph(e);
  e->order.clear();
  e->slot_pos.assign(e->slots.size(), -1);
  for (size_t s = 0; s < e->slots.size(); s++)
    if (e->slots[s].used) {
      e->slot_pos[s] = (int)e->order.size();
      e->order.push_back((int)s);
    }
  const int nl = (int)e->order.size();
  std::vector<LatDesc> descs(nl);
  std::vector<CUtensorMap> maps(2 * (size_t)std::max(1, nl));
  std::vector<int> tile_lat, tile_first(nl + 1, 0), itl_lats;
  std::vector<unsigned> tile_idx;
  for (int c = 0; c < nl; c++) {
    LatHost &L = e->slots[e->order[c]];
    const int shape = e->policy >= 0 ? e->policy : (L.policy_shape >= 0 ? L.policy_shape : model_shape(L.d.bcx, L.d.by, L.d.bz));
    L.d.shape = shape;
    L.d.ntx = (L.d.bcx + kShapes[shape][0] - 1) / kShapes[shape][0];
    L.d.nty = (L.d.by + kShapes[shape][1] - 1) / kShapes[shape][1];
    L.d.ntz = (L.d.bz + kShapes[shape][2] - 1) / kShapes[shape][2];
    for (int b = 0; b < 2; b++) MB_TRY(encode_tile_map(&L.tmap[b], L.d.u4[b], L.d.ecx, L.d.ey, L.d.ez, shape));
    maps[2 * c] = L.tmap[0];
    maps[2 * c + 1] = L.tmap[1];
    const int nt = L.d.ntx * L.d.nty * L.d.ntz;
    tile_first[c] = (int)tile_lat.size();
    for (int tz = 0; tz < L.d.ntz; tz++)
      for (int ty = 0; ty < L.d.nty; ty++)
        for (int tx = 0; tx < L.d.ntx; tx++) {
          tile_lat.push_back(c);
          tile_idx.push_back((unsigned)(tx * kShapes[shape][0]) | ((unsigned)(ty * kShapes[shape][1]) << 11) |
                             ((unsigned)(tz * kShapes[shape][2]) << 22));
        }
    (void)nt;
    if (L.d.n_itl > 0 || (e->conv_d > 0.0 && L.d.cap_itl > 0)) itl_lats.push_back(c);
    descs[c] = L.d;
  }
  tile_first[nl] = (int)tile_lat.size();
  e->n_tiles = (int)tile_lat.size();
  const size_t need_l = std::max(1, nl), need_t = std::max<size_t>(1, tile_lat.size());
  if (need_l > e->cap_lats) {
    const size_t C = std::max<size_t>({need_l, 2 * e->cap_lats, 16});
    void **arrs[] = {(void **)&e->d_lats, (void **)&e->d_tmaps,     (void **)&e->d_itl_lats,
                     (void **)&e->d_tile_first, (void **)&e->d_eout, (void **)&e->d_eitl,
                     (void **)&e->d_item_first};
    const size_t per[] = {sizeof(LatDesc), 2 * sizeof(CUtensorMap), sizeof(int), sizeof(int), 2 * sizeof(double),
                          2 * sizeof(double), sizeof(unsigned)};
    for (int a = 0; a < 7; a++) {
      if (*arrs[a]) {
        cudaFree(*arrs[a]);
        e->device_bytes -= (e->cap_lats + 1) * per[a];
        e->fixed_bytes -= (e->cap_lats + 1) * per[a];
      }
      *arrs[a] = nullptr;
      MB_TRY(edalloc(e, arrs[a], (C + 1) * per[a]));
    }
    e->cap_lats = C;
  }
  for (int c = 0; c < nl; c++) { // descriptors point into d_eitl
    e->slots[e->order[c]].d.e_itl = e->d_eitl + 2 * c;
    descs[c].e_itl = e->d_eitl + 2 * c;
  }
  // interstitial cell lists: cells of edge >= cutoff + skin, at least 3 per dimension
  // (27 distinct neighbour cells); lattices below that walk the whole list
  {
    const double reach = e->cfg.cutoff + e->cfg.stencil_skin;
    std::vector<size_t> off(nl, 0);
    size_t total = 0;
    for (int q : itl_lats) {
      LatDesc &d = e->slots[e->order[q]].d;
      const int n3[3] = {(int)(d.Lx / reach), (int)(d.Ly / reach), (int)(d.Lz / reach)};
      if (n3[0] < 3 || n3[1] < 3 || n3[2] < 3 || d.cap_itl < 1) continue;
      off[q] = total + 1; // 1-based: 0 = none
      total += 2 * (size_t)n3[0] * n3[1] * n3[2] + 2 * (size_t)d.cap_itl + 2;
    }
    if (total > e->cap_icell) {
      if (e->d_icell) {
        cudaFree(e->d_icell);
        e->device_bytes -= e->cap_icell * sizeof(int);
        e->fixed_bytes -= e->cap_icell * sizeof(int);
      }
      e->d_icell = nullptr;
      const size_t C = std::max(total, 2 * e->cap_icell);
      MB_TRY(edalloc(e, (void **)&e->d_icell, C * sizeof(int)));
      e->cap_icell = C;
    }
    if (total) MB_CUDA(cudaMemsetAsync(e->d_icell, 0, total * sizeof(int), e->stream));
    for (int c = 0; c < nl; c++) {
      LatDesc &d = e->slots[e->order[c]].d;
      d.icn[0] = d.icn[1] = d.icn[2] = 0;
      d.icount = d.istart = d.iitem = d.icell_of = d.iflag = nullptr;
      if (off[c]) {
        int *b = e->d_icell + (off[c] - 1);
        d.icn[0] = (int)(d.Lx / reach);
        d.icn[1] = (int)(d.Ly / reach);
        d.icn[2] = (int)(d.Lz / reach);
        const size_t nc = (size_t)d.icn[0] * d.icn[1] * d.icn[2];
        d.icount = b;
        d.istart = b + nc;
        d.iitem = b + 2 * nc;
        d.icell_of = b + 2 * nc + d.cap_itl;
        d.iflag = b + 2 * nc + 2 * (size_t)d.cap_itl;
      }
      descs[c].icn[0] = d.icn[0];
      descs[c].icn[1] = d.icn[1];
      descs[c].icn[2] = d.icn[2];
      descs[c].icount = d.icount;
      descs[c].istart = d.istart;
      descs[c].iitem = d.iitem;
      descs[c].icell_of = d.icell_of;
      descs[c].iflag = d.iflag;
    }
  }
  if (need_t > e->cap_tiles) {
    const size_t C = std::max<size_t>({need_t, 2 * e->cap_tiles, 256});
    void **arrs[] = {(void **)&e->d_tile_lat, (void **)&e->d_tile_idx, (void **)&e->d_epart};
    const size_t per[] = {sizeof(int), sizeof(int), 2 * sizeof(double)};
    for (int a = 0; a < 3; a++) {
      if (*arrs[a]) {
        cudaFree(*arrs[a]);
        e->device_bytes -= e->cap_tiles * per[a];
        e->fixed_bytes -= e->cap_tiles * per[a];
      }
      *arrs[a] = nullptr;
      MB_TRY(edalloc(e, arrs[a], C * per[a]));
    }
    e->cap_tiles = C;
  }
  if (nl > 0) {
    MB_CUDA(cudaMemcpyAsync(e->d_lats, descs.data(), sizeof(LatDesc) * nl, cudaMemcpyHostToDevice, e->stream));
    MB_CUDA(cudaMemcpyAsync(e->d_tmaps, maps.data(), sizeof(CUtensorMap) * 2 * nl, cudaMemcpyHostToDevice,
                            e->stream));
    MB_CUDA(cudaMemcpyAsync(e->d_tile_lat, tile_lat.data(), sizeof(int) * tile_lat.size(), cudaMemcpyHostToDevice,
                            e->stream));
    MB_CUDA(cudaMemcpyAsync(e->d_tile_idx, tile_idx.data(), sizeof(unsigned) * tile_idx.size(), cudaMemcpyHostToDevice,
                            e->stream));
    MB_CUDA(cudaMemcpyAsync(e->d_tile_first, tile_first.data(), sizeof(int) * (nl + 1), cudaMemcpyHostToDevice,
                            e->stream));
    if (!itl_lats.empty())
      MB_CUDA(cudaMemcpyAsync(e->d_itl_lats, itl_lats.data(), sizeof(int) * itl_lats.size(), cudaMemcpyHostToDevice,
                              e->stream));
    MB_CUDA(cudaStreamSynchronize(e->stream)); // host vectors go out of scope
  }
  EnsParams &P = e->P;
  P.lats = e->d_lats;
  P.n_lats = nl;
  P.tile_lat = e->d_tile_lat;
  P.tile_org = (const unsigned *)e->d_tile_idx;
  P.n_tiles = e->n_tiles;
  P.tmaps = e->d_tmaps;
  P.epart = e->d_epart;
  P.itl_lats = e->d_itl_lats;
  P.n_itl_lats = (int)itl_lats.size();
  P.bar = e->d_bar;
  P.bar_spins = e->bar_spins;
  P.err = e->d_err;
  e->grid = std::max(1, std::min(e->max_grid, e->n_tiles));
  // kernel structure: split kernels whenever their stencil applies (unless the
  // persistent kernel is asked for); one lattice at least a chunk wide walks bricks
  e->split = 0;
  if (nl >= 1 && e->mode != 1) {
    const char *why = mx_stencil(e, descs[0], e->mxs);
    for (int c = 0; c < nl && !why; c++)
      if (descs[c].bcx > 2047 || descs[c].by > 2047 || descs[c].bz > 511)
        why = "split kernels take lattices of at most 2047 x 2047 x 511 cells";
    if (!why && nl > 1 && !e->mxs.fixed) why = "split kernels over several lattices need the built-in BCC shells";
    if (why) {
      if (e->mode == 2) return fail(MB_ERR_UNSUPPORTED, why);
    } else {
      e->split = (nl == 1 && (descs[0].bcx >= 32 || !e->mxs.fixed)) ? 1 : 2;
    }
  }
  if (e->split) {
    MxWalk &W = e->mxs.walk;
    W.linear = e->split == 2;
    W.n_lats = nl;
    std::vector<unsigned> first(nl + 1, 0);
    unsigned long long n_items = 0;
    if (W.linear) {
      // brick order for lattices with large planes (MxWalk); the environment variable
      // MB_MX_LBRICK = "chunks,zcells,min_plane_sites" overrides it, for tuning ("0,0,0":
      // every lattice plane by plane)
      W.lcb = MX_LCB;
      W.lbz = MX_LBZ;
      W.lmin = MX_LMIN;
      if (const char *v = getenv("MB_MX_LBRICK")) {
        unsigned a = 0, b = 0, m = 0;
        if (sscanf(v, "%u,%u,%u", &a, &b, &m) == 3 && a <= 64 && b <= 64) {
          W.lcb = (a && b) ? a : 0;
          W.lbz = (a && b) ? b : 0;
          W.lmin = m;
        }
      }
      for (int c = 0; c < nl; c++) {
        const LatDesc &d = descs[c];
        first[c] = (unsigned)n_items;
        n_items += 2ull * d.bz * (((unsigned long long)d.bcx * d.by + 31) / 32);
      }
      first[nl] = (unsigned)n_items;
    } else {
      n_items = (unsigned long long)W.n_units * W.bitems;
    }
      if (n_items >= (1ull << 31)) return fail(MB_ERR_ARG, "too many sites for the 32-bit item walk");
    W.n_items = (unsigned)n_items;
    if (n_items > e->cap_items) {
      const size_t C = std::max<size_t>((size_t)n_items, 2 * e->cap_items);
      const size_t per = 2 * sizeof(double) + sizeof(uint2);
      if (e->d_epart_items) {
        cudaFree(e->d_epart_items);
        cudaFree(e->d_outer_items);
        e->device_bytes -= e->cap_items * per;
        e->fixed_bytes -= e->cap_items * per;
      }
      e->d_epart_items = nullptr;
      e->d_outer_items = nullptr;
      e->cap_items = 0;
      MB_TRY(edalloc(e, (void **)&e->d_epart_items, C * 2 * sizeof(double)));
      MB_TRY(edalloc(e, (void **)&e->d_outer_items, C * sizeof(uint2)));
      e->cap_items = C;
    }
    MB_CUDA(cudaMemcpyAsync(e->d_item_first, first.data(), sizeof(unsigned) * (nl + 1), cudaMemcpyHostToDevice,
                            e->stream));
    MB_CUDA(cudaStreamSynchronize(e->stream));
    W.item_first = e->d_item_first;
    P.epart = e->d_epart_items;
    P.outer = outer_masks_on() ? e->d_outer_items : nullptr;
  }
  e->dirty = false;
  return MB_OK;
}

// Split-mode stencil of lattice d (see MxStencil); returns why it cannot be built, or
// nullptr.  Neighbour vectors are enumerated in half-lattice units (hx, hy, hz), all
// of one parity, and ordered by length.
static const char *mx_stencil(const mb_ensemble *e, const LatDesc &d, MxStencil &S) {
  const DevPot &pp = e->P.P;
  if (pp.n_rs <= 0 || pp.n_fs <= 0) return "split kernels need the single-type squared-distance tables";
  const double a0 = e->cfg.lattice_const, rc = e->cfg.cutoff, reach = rc + e->cfg.stencil_skin;
  if (rc * rc > pp.ds_r * pp.n_rs * (1.0 + 1e-12) || rc * rc > pp.ds_f * pp.n_fs * (1.0 + 1e-12))
    return "cutoff beyond the potential table";
  const double h = 0.5 * a0;
  const int lim = (int)ceil(reach / h);
  struct V {
    double R;
    int hx, hy, hz;
  };
  std::vector<V> vs;
  for (int hz = -lim; hz <= lim; hz++)
    for (int hy = -lim; hy <= lim; hy++)
      for (int hx = -lim; hx <= lim; hx++) {
        if (!hx && !hy && !hz) continue;
        if (((hx ^ hy) & 1) || ((hx ^ hz) & 1)) continue;
        const double R = h * sqrt((double)(hx * hx + hy * hy + hz * hz));
        if (R < reach) vs.push_back({R, hx, hy, hz});
      }
  if ((int)vs.size() != e->P.n_st) return "split stencil differs from the lattice stencil";
  std::stable_sort(vs.begin(), vs.end(), [](const V &a, const V &b) { return a.R < b.R; });
  const long long E = d.E, ecx = d.ecx, ey = d.ey;
  const long long d_odd = -2 * E + (ey + 1) * ecx + 1;
  memset(&S, 0, sizeof(S));
  S.d_odd = (int)d_odd;
  S.n_rs = pp.n_rs;
  S.n_fs = pp.n_fs;
  S.rds = (float)(1.0 / pp.ds_r);
  S.rds_f = (float)(1.0 / pp.ds_f);
  const double bf_reach = rc + 0.5 * e->cfg.stencil_skin;
  for (const V &v : vs) {
    MxEntry E0;
    const bool odd = v.hx & 1;
    long long dcx, dy, dz;
    if (odd) {
      dcx = (v.hx - 1) / 2;
      dy = (v.hy - 1) / 2;
      dz = (v.hz - 1) / 2;
    } else {
      dcx = v.hx / 2;
      dy = v.hy / 2;
      dz = v.hz / 2;
    }
    // both sublattices' targets must stay inside the 2-cell ghost frame
    if (llabs(dcx) > 2 || llabs(dy) > 2 || llabs(dz) > 2 || (odd && (dcx + 1 > 2 || dy + 1 > 2 || dz + 1 > 2)))
      return "stencil reaches beyond the 2-cell ghost frame";
    E0.off = (int)((odd ? E : 0) + (dz * ey + dy) * ecx + dcx);
    E0.odd = odd ? 1 : 0;
    const double cx = -h * v.hx, cy = -h * v.hy, cz = -h * v.hz, R2 = v.R * v.R;
    E0.c = make_float4((float)cx, (float)cy, (float)cz, (float)(rc * rc - R2));
    const double x = R2 / pp.ds_r, fl = floor(x), xf = R2 / pp.ds_f, flf = floor(xf);
    E0.t = make_float4((float)(2 * cx), (float)(2 * cy), (float)(2 * cz), (float)(x - fl));
    E0.kb = (float)fl;
    E0.fr_f = (float)(xf - flf);
    E0.kb_f = (float)flf;
    E0.pad_[0] = E0.pad_[1] = E0.pad_[2] = 0;
    if (v.R < bf_reach && odd && S.n_odd < MX_PAR_MAX - 1)
      S.odd[S.n_odd++] = E0;
    else if (v.R < bf_reach && !odd && S.n_even < MX_PAR_MAX - 1)
      S.even[S.n_even++] = E0;
    else
      S.far[S.n_far++] = E0;
  }
  // pad each branch-free list to even length with an entry that never interacts
  auto pad = [](MxEntry *list, int &n) {
    if (n & 1) {
      list[n] = list[0];
      list[n].c.w = -3.0e38f;
      n++;
    }
  };
  if (S.n_odd == 0 || S.n_even == 0) return "split stencil has an empty branch-free class";
  pad(S.odd, S.n_odd);
  pad(S.even, S.n_even);
  // brick walk (shape MX_BY x MX_BZ; the environment variable MB_MX_BRICK = "rows,planes"
  // overrides it, for tuning)
  unsigned bby = MX_BY, bbz = MX_BZ;
  if (const char *v = getenv("MB_MX_BRICK")) {
    unsigned a = 0, b = 0;
    if (sscanf(v, "%u,%u", &a, &b) == 2 && a >= 1 && b >= 1 && a <= 32 && b <= 32) {
      bby = a;
      bbz = b;
    }
  }
  const unsigned chunks = (unsigned)((d.bcx + 31) / 32), nyb = (unsigned)((d.by + bby - 1) / bby),
                 nzb = (unsigned)((d.bz + bbz - 1) / bbz);
  const unsigned long long units = (unsigned long long)chunks * nyb * nzb;
  if (units * 2 * bby * bbz >= (1ull << 31)) return "lattice too large for the 32-bit brick walk";
  S.walk.by = bby;
  S.walk.bz = bbz;
  S.walk.bitems = 2 * bby * bbz;
  S.walk.chunks = chunks;
  S.walk.m_chunks = 0xFFFFFFFFu / chunks;
  S.walk.nyb = nyb;
  S.walk.m_nyb = 0xFFFFFFFFu / nyb;
  S.walk.n_units = (unsigned)units;
  // built-in shells: the stencil must be exactly BCC shells 1-7 (|h|^2 <= 19 < 20) or
  // 1-8 (|h|^2 <= 20 < 24)
  const double r7 = h * sqrt(19.0), r8 = h * sqrt(20.0), r9 = h * sqrt(24.0);
  const bool small = (long long)ey * ecx < (1ll << 31);
  S.fixed = (small && vs.size() == 88 && r7 < reach && reach <= r8)    ? 7
            : (small && vs.size() == 112 && r8 < reach && reach <= r9) ? 8
                                                                        : 0;
  const int n2s[MX_SHELLS] = {3, 4, 8, 11, 12, 16, 19, 20};
  MxShells &Q = S.sh;
  const double grid_ds[2] = {pp.ds_r, pp.ds_f};
  const int grid_n[2] = {pp.n_rs, pp.n_fs};
  for (int k = 0; k < MX_SHELLS; k++) Q.w[k] = (float)(rc * rc - h * h * n2s[k]);
  for (int gi = 0; gi < 2; gi++) {
    Q.g[gi].rds = (float)(1.0 / grid_ds[gi]);
    Q.g[gi].mmax = (float)(grid_n[gi] - 1);
    for (int k = 0; k < MX_SHELLS; k++) {
      const double x = h * h * n2s[k] / grid_ds[gi], fl = floor(x);
      Q.g[gi].fr[k] = (float)(x - fl);
      Q.g[gi].kb[k] = (float)fl;
    }
  }
  Q.a0 = (float)a0;
  Q.pl = (int)(ey * ecx);
  Q.rw = (int)ecx;
  Q.E = E;
  Q.d_odd = d_odd;
  return nullptr;
}

static int check_err(mb_ensemble *e) {
  int err = 0;
  MB_CUDA(cudaMemcpyAsync(&err, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  MB_CUDA(cudaStreamSynchronize(e->stream));
  if (err) {
    cudaMemsetAsync(e->d_err, 0, sizeof(int), e->stream);
    cudaMemsetAsync(e->d_bar, 0, 2 * sizeof(unsigned), e->stream);
    return fail(MB_ERR_TIMEOUT, err == 1 ? "a grid barrier of the ensemble step gave up waiting"
                                         : "a tile copy of the ensemble step gave up waiting");
  }
  return MB_OK;
}

// One launch (one step of every active lattice).
static int launch_step(mb_ensemble *e, int energy) {
  if (e->dirty) MB_TRY(rebuild(e));
  if (e->n_tiles == 0) return MB_OK;
  if (e->conv_d > 0.0 && !e->split)
    return fail(MB_ERR_UNSUPPORTED, "lattice <-> interstitial conversion runs with the split kernels only");
  e->synced_desc = false;
  EnsParams &P = e->P;
  if (energy) {
    MB_CUDA(cudaMemsetAsync(e->d_eitl, 0, sizeof(double) * 2 * e->order.size(), e->stream));
    P.energy = 1;
    if (e->split) {
      MB_TRY(mx_launch_step(P, e->mxs, 0, 1, e->stream, nullptr, e->d_eout));
    } else {
      MB_TRY(ens_launch(P, e->grid, e->stream));
      MB_TRY(ens_energy_launch(e->d_lats, (int)e->order.size(), e->d_tile_first, e->d_epart, e->d_eout, e->stream));
    }
    P.energy = 0;
    e->launches++;
    return MB_OK;
  }
  P.energy = 0;
  if (e->graphs_ok) {
    if (!e->graph) {
      cudaGraph_t g = nullptr;
      cudaError_t r = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
      if (r == cudaSuccess) {
        const int rc =
            e->split ? mx_launch_step(P, e->mxs, 0, 0, e->stream, nullptr, nullptr) : ens_launch(P, e->grid, e->stream);
        r = cudaStreamEndCapture(e->stream, &g);
        if (rc == MB_OK && r == cudaSuccess && g) {
          if (cudaGraphInstantiate(&e->graph, g, 0) != cudaSuccess) e->graph = nullptr;
        }
        if (g) cudaGraphDestroy(g);
      }
      cudaGetLastError();
      if (!e->graph) e->graphs_ok = false; // cooperative capture refused: launch directly
    }
    if (e->graph) {
      MB_CUDA(cudaGraphLaunch(e->graph, e->stream));
      e->launches++;
      return MB_OK;
    }
  }
  if (e->split)
    MB_TRY(mx_launch_step(P, e->mxs, 0, 0, e->stream, nullptr, nullptr));
  else
    MB_TRY(ens_launch(P, e->grid, e->stream));
  e->launches++;
  return MB_OK;
}

// Records energies of the lattices that took part in the last (energy) launch.
static int collect_energy(mb_ensemble *e, const std::vector<char> &was_active, const std::vector<long long> &step_of) {
  const size_t nl = e->order.size();
  std::vector<double> out(2 * nl);
  MB_CUDA(cudaMemcpyAsync(out.data(), e->d_eout, sizeof(double) * 2 * nl, cudaMemcpyDeviceToHost, e->stream));
  MB_CUDA(cudaStreamSynchronize(e->stream));
  for (size_t c = 0; c < nl; c++) {
    if (!was_active[c]) continue;
    LatHost &L = e->slots[e->order[c]];
    L.e_step.push_back((double)step_of[c]);
    L.e_pe.push_back(out[2 * c]);
    L.e_ke.push_back(out[2 * c + 1]);
  }
  return MB_OK;
}

static bool host_active(const LatDesc &d) { return !d.primed || d.steps_done < d.steps_target; }

// Launch until every lattice reached its target (or max_launches), recording
// energies every energy_every steps of each lattice.
static int advance(mb_ensemble *e, long long max_launches, int energy_every, long long *done) {
  long long n = 0;
  if (e->dirty) MB_TRY(rebuild(e));
  MB_TRY(sync_desc(e));
  // host mirror of the counters, advanced like the device does
  std::vector<LatDesc *> ds;
  for (int s : e->order) ds.push_back(&e->slots[s].d);
  while (n < max_launches) {
    bool any = false, energy = false;
    std::vector<char> act(ds.size(), 0);
    std::vector<long long> step_of(ds.size(), 0);
    for (size_t c = 0; c < ds.size(); c++) {
      if (!host_active(*ds[c])) continue;
      any = true;
      act[c] = 1;
      step_of[c] = ds[c]->primed ? ds[c]->steps_done + 1 : 0;
      if (energy_every > 0 && step_of[c] % energy_every == 0) energy = true;
    }
    if (!any) break;
    MB_TRY(launch_step(e, energy ? 1 : 0));
    if (energy) MB_TRY(collect_energy(e, act, step_of));
    for (size_t c = 0; c < ds.size(); c++) {
      if (!act[c]) continue;
      ds[c]->cur ^= 1;
      if (ds[c]->primed)
        ds[c]->steps_done++;
      else
        ds[c]->primed = 1;
    }
    n++;
  }
  // the mirror now matches what the device will hold, except the interstitial counts,
  // which conversions change on the device: then the next sync pulls them
  e->synced_desc = !(e->conv_d > 0.0);
  if (done) *done = n;
  return MB_OK;
}

static int push_targets(mb_ensemble *e) {
  // descriptors are small: re-upload after host-side changes of targets, with the
  // device-owned fields (parity, counters, interstitial counts) pulled back first
  MB_TRY(sync_desc(e));
  std::vector<LatDesc> descs;
  for (int s : e->order) descs.push_back(e->slots[s].d);
  if (!descs.empty())
    MB_CUDA(cudaMemcpyAsync(e->d_lats, descs.data(), sizeof(LatDesc) * descs.size(), cudaMemcpyHostToDevice,
                            e->stream));
  MB_CUDA(cudaStreamSynchronize(e->stream));
  return MB_OK;
}

static void free_slot(mb_ensemble *e, LatHost &L) {
  if (L.block) {
    cudaFree(L.block);
    e->device_bytes -= L.bytes;
  }
  L = LatHost();
}

} // namespace mb

using namespace mb;

extern "C" {

int mb_ensemble_create(const mb_ensemble_config *cfg, const mb_eam_tables *pot, mb_ensemble **out) {
  if (!cfg || !pot || !out) return fail(MB_ERR_ARG, "null argument");
  *out = nullptr;
  if (!(cfg->lattice_const > 0) || !(cfg->mass > 0) || !(cfg->dt > 0) || !(cfg->cutoff > 0) ||
      cfg->stencil_skin < 0)
    return fail(MB_ERR_ARG, "lattice_const, mass, dt, cutoff must be > 0 and skin >= 0");
  if (pot->n_types != 1) return fail(MB_ERR_UNSUPPORTED, "the mixed-precision tile kernel handles one atom type");
  mb_ensemble *e = new mb_ensemble();
  e->cfg = *cfg;
  int rc = pot_build(pot, &e->pot);
  if (rc != MB_OK) {
    delete e;
    return rc;
  }
  auto bail = [&](int code) {
    mb_ensemble_destroy(e);
    return code;
  };
  EnsParams &P = e->P;
  P.P = pot_dev(e->pot);
  P.rdr = (float)P.P.rdr;
  P.rc2f = (float)(cfg->cutoff * cfg->cutoff);
  P.rc2 = cfg->cutoff * cfg->cutoff;
  P.h = 0.5 * cfg->dt * MB_FTM2V / cfg->mass;
  P.dt = cfg->dt;
  P.mass = cfg->mass;
  P.a0 = cfg->lattice_const;
  P.reach = cfg->cutoff + cfg->stencil_skin;
  if ((rc = ens_stencil(e)) != MB_OK) return bail(rc);
  // shared-memory knots: as many of the last ones as fit beside two tile buffers
  const int budget = 232448 - 2048 - 2 * ENS_TILE_MAX_BYTES - 32;
  P.nsm = std::min(P.P.nr, budget / (int)(sizeof(float4) + 3 * sizeof(float2)));
  P.m_lo = P.P.nr - P.nsm;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MB_ERR_CUDA, "stream creation failed"));
  for (auto &ev : e->ev)
    if (cudaEventCreate(&ev) != cudaSuccess) return bail(fail(MB_ERR_CUDA, "event creation failed"));
  if ((rc = edalloc(e, (void **)&e->d_bar, 2 * sizeof(unsigned))) != MB_OK) return bail(rc);
  if ((rc = edalloc(e, (void **)&e->d_err, sizeof(int))) != MB_OK) return bail(rc);
  if ((rc = edalloc(e, (void **)&e->d_bad, sizeof(int))) != MB_OK) return bail(rc);
  cudaMemsetAsync(e->d_bar, 0, 2 * sizeof(unsigned), e->stream);
  cudaMemsetAsync(e->d_err, 0, sizeof(int), e->stream);
  e->max_grid = ens_max_grid(P.nsm);
  if (e->max_grid <= 0) return bail(fail(MB_ERR_CUDA, "the ensemble kernel cannot be resident (shared memory)"));
  if (cudaStreamSynchronize(e->stream) != cudaSuccess) return bail(fail(MB_ERR_CUDA, "sync failed"));
  *out = e;
  return MB_OK;
}

int mb_ensemble_destroy(mb_ensemble *e) {
  if (!e) return MB_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graph(e);
  for (auto &L : e->slots) free_slot(e, L);
  void *ptrs[] = {e->d_lats, e->d_tile_lat, e->d_tile_idx, e->d_tile_first, e->d_itl_lats, e->d_tmaps,
                  e->d_epart, e->d_eout, e->d_eitl, e->d_bar, e->d_err, e->d_bad, e->d_item_first,
                  e->d_epart_items, e->d_outer_items, e->d_icell};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &ev : e->ev)
    if (ev) cudaEventDestroy(ev);
  if (e->stream) cudaStreamDestroy(e->stream);
  pot_free(e->pot);
  delete e;
  return MB_OK;
}

int mb_ensemble_lattice_bytes(const mb_lattice_spec *spec, int64_t *bytes) {
  if (!spec || !bytes) return fail(MB_ERR_ARG, "null argument");
  *bytes = (int64_t)lattice_bytes(spec->cells_x, spec->cells_y, spec->cells_z, spec->max_interstitials);
  return MB_OK;
}

int mb_ensemble_add(mb_ensemble *e, const mb_lattice_spec *spec, const mb_atom_element *box,
                    const mb_atom_element *itl, int32_t n_itl, int64_t steps, int32_t *slot_out) {
  MB_RANGE("mb_ensemble_add");
  if (!e || !spec || !box || !slot_out) return fail(MB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  const int cx = spec->cells_x, cy = spec->cells_y, cz = spec->cells_z;
  if (cx < 2 || cy < 2 || cz < 2) return fail(MB_ERR_ARG, "lattice edges must be >= 2 cells");
  if (cx > 2000 || cy > 2000 || cz > 1000) return fail(MB_ERR_ARG, "lattice edges must be <= 2000 x 2000 x 1000 cells");
  const double reach = e->cfg.cutoff + e->cfg.stencil_skin, a0 = e->cfg.lattice_const;
  if (cx * a0 <= 2 * reach || cy * a0 <= 2 * reach || cz * a0 <= 2 * reach)
    return fail(MB_ERR_ARG, "box edge must exceed 2 * (cutoff + stencil_skin)");
  if (n_itl < 0 || n_itl > spec->max_interstitials) return fail(MB_ERR_ARG, "n_itl exceeds max_interstitials");
  if (n_itl > 0 && !itl) return fail(MB_ERR_ARG, "null interstitial array");
  if (steps < 0) return fail(MB_ERR_ARG, "steps < 0");
  for (int k = 0; k < n_itl; k++)
    if (itl[k].type != 0) return fail(MB_ERR_ARG, "interstitial type must be 0 (one-type potential)");
  const size_t bytes = lattice_bytes(cx, cy, cz, spec->max_interstitials);
  if (e->cfg.hbm_budget_bytes > 0 && e->device_bytes + bytes > (size_t)e->cfg.hbm_budget_bytes)
    return fail(MB_ERR_NOMEM, "HBM budget exceeded: " + std::to_string(e->device_bytes + bytes) + " > " +
                                  std::to_string(e->cfg.hbm_budget_bytes) + " bytes");
  if (e->cfg.max_lattices > 0) {
    int used = 0;
    for (auto &L : e->slots) used += L.used;
    if (used >= e->cfg.max_lattices) return fail(MB_ERR_NOMEM, "all lattice slots are in use");
  }
  MB_TRY(sync_desc(e));
  int slot = -1;
  for (size_t s = 0; s < e->slots.size(); s++)
    if (!e->slots[s].used) {
      slot = (int)s;
      break;
    }
  if (slot < 0) {
    slot = (int)e->slots.size();
    e->slots.emplace_back();
  }
  LatHost &L = e->slots[slot];
  void *block = nullptr;
  cudaError_t r = cudaMalloc(&block, bytes);
  if (r != cudaSuccess) return fail(MB_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(r));
  L.used = true;
  L.block = block;
  L.bytes = bytes;
  e->device_bytes += bytes;
  L.cells[0] = cx;
  L.cells[1] = cy;
  L.cells[2] = cz;
  L.cap_itl = spec->max_interstitials;
  LatDesc &d = L.d;
  d = LatDesc();
  d.bcx = cx;
  d.by = cy;
  d.bz = cz;
  d.ecx = cx + 4;
  d.ey = cy + 4;
  d.ez = cz + 4;
  d.E = (long long)d.ecx * d.ey * d.ez;
  d.Lx = cx * a0;
  d.Ly = cy * a0;
  d.Lz = cz * a0;
  d.n_itl = n_itl;
  d.steps_target = steps;
  const size_t n = 2 * (size_t)d.E, nb = 2 * (size_t)cx * cy * cz, ci = (size_t)std::max(1, L.cap_itl);
  const int per = 2 * 4 * 64 + 64;
  d.cap_flag = std::max(1, L.cap_itl * per);
  char *p = (char *)block;
  auto take = [&](size_t b) {
    char *q = p;
    p += (b + 255) & ~(size_t)255;
    return (void *)q;
  };
  d.u4[0] = (float4 *)take(n * 16);
  d.u4[1] = (float4 *)take(n * 16);
  d.ux = (double *)take(n * 8);
  d.uy = (double *)take(n * 8);
  d.uz = (double *)take(n * 8);
  d.vx = (double *)take(n * 8);
  d.vy = (double *)take(n * 8);
  d.vz = (double *)take(n * 8);
  d.fx = (float *)take(n * 4);
  d.fy = (float *)take(n * 4);
  d.fz = (float *)take(n * 4);
  d.rho = (float *)take(n * 4);
  d.code = (int8_t *)take(n);
  L.ids = (int64_t *)take(nb * 8);
  for (int b = 0; b < 2; b++) {
    d.ipx[b] = (double *)take(ci * 8);
    d.ipy[b] = (double *)take(ci * 8);
    d.ipz[b] = (double *)take(ci * 8);
  }
  d.ivx = (double *)take(ci * 8);
  d.ivy = (double *)take(ci * 8);
  d.ivz = (double *)take(ci * 8);
  d.ifx = (double *)take(ci * 8);
  d.ify = (double *)take(ci * 8);
  d.ifz = (double *)take(ci * 8);
  d.irho = (double *)take(ci * 8);
  d.idf = (double *)take(ci * 8);
  L.iids = (int64_t *)take(ci * 8);
  d.itype = (int8_t *)take(ci);
  d.flag_list = (int *)take((size_t)d.cap_flag * 4);
  d.flag_count = (int *)take(16); // [count parity 0, count parity 1, overflow, -]
  d.cand = (long long *)take(MB_CAND_CAP * 8);
  d.cand_n = (int *)take(16);
  d.conv_counters = (long long *)take(32);
  d.cap_itl = L.cap_itl;
  d.ids = L.ids;
  d.iids = L.iids;
  if ((size_t)(p - (char *)block) > bytes) return fail(MB_ERR_STATE, "lattice layout overflows its block");
  cudaStream_t s = e->stream;
  auto undo = [&](int code) {
    free_slot(e, L);
    return code;
  };
  if (cudaMemsetAsync(block, 0, bytes, s) != cudaSuccess) return undo(fail(MB_ERR_CUDA, "memset failed"));
  if (cudaMemsetAsync(d.code, 0xff, n, s) != cudaSuccess) return undo(fail(MB_ERR_CUDA, "memset failed"));
  mb_atom_element *stage = nullptr;
  if (cudaMalloc(&stage, nb * sizeof(mb_atom_element)) != cudaSuccess)
    return undo(fail(MB_ERR_NOMEM, "staging allocation failed"));
  cudaMemsetAsync(e->d_bad, 0, sizeof(int), s);
  cudaMemcpyAsync(stage, box, nb * sizeof(mb_atom_element), cudaMemcpyHostToDevice, s);
  int grid = (int)std::min<size_t>((nb + 255) / 256, 16 * (size_t)device_sm_count());
  k_ens_upload<<<grid, 256, 0, s>>>(d, stage, L.ids, a0, e->d_bad, e->P.P.n_types);
  if (n_itl > 0) {
    std::vector<double> buf(n_itl);
    std::vector<int8_t> t(n_itl, 0);
    L.host_iids.resize(n_itl);
    for (int k = 0; k < n_itl; k++) L.host_iids[k] = itl[k].id;
    auto put = [&](double *dst, int comp, int field) {
      for (int k = 0; k < n_itl; k++) buf[k] = field == 0 ? itl[k].x[comp] : itl[k].v[comp];
      cudaMemcpyAsync(dst, buf.data(), sizeof(double) * n_itl, cudaMemcpyHostToDevice, s);
      cudaStreamSynchronize(s);
    };
    put(d.ipx[0], 0, 0);
    put(d.ipy[0], 1, 0);
    put(d.ipz[0], 2, 0);
    put(d.ivx, 0, 1);
    put(d.ivy, 1, 1);
    put(d.ivz, 2, 1);
    cudaMemcpyAsync(d.itype, t.data(), n_itl, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(L.iids, L.host_iids.data(), sizeof(int64_t) * n_itl, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  }
  int bad = 0;
  cudaMemcpyAsync(&bad, e->d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaError_t er = cudaStreamSynchronize(s);
  cudaFree(stage);
  if (er != cudaSuccess) return undo(cuda_fail(er, "lattice upload"));
  if (bad) return undo(fail(MB_ERR_ARG, "atom type without a potential table"));
  d.cur = 0;
  d.primed = 0;
  d.steps_done = 0;
  e->dirty = true;
  *slot_out = slot;
  return MB_OK;
}

int mb_ensemble_remove(mb_ensemble *e, int32_t slot) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  MB_CUDA(cudaStreamSynchronize(e->stream));
  MB_TRY(sync_desc(e));
  free_slot(e, e->slots[slot]);
  e->dirty = true;
  return MB_OK;
}

int mb_ensemble_set_steps(mb_ensemble *e, int32_t slot, int64_t steps_target) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  if (steps_target < 0) return fail(MB_ERR_ARG, "steps_target < 0");
  MB_TRY(sync_desc(e));
  e->slots[slot].d.steps_target = steps_target;
  if (!e->dirty) MB_TRY(push_targets(e));
  return MB_OK;
}

int mb_ensemble_advance(mb_ensemble *e, int32_t max_launches, int32_t energy_every, int32_t *launches) {
  MB_RANGE("mb_ensemble_advance");
  if (!e || max_launches < 0 || energy_every < 0) return fail(MB_ERR_ARG, "bad arguments");
  std::lock_guard<std::mutex> lk(e->mu);
  long long n = 0;
  MB_TRY(advance(e, max_launches, energy_every, &n));
  if (launches) *launches = (int32_t)n;
  return MB_OK;
}

int mb_ensemble_run(mb_ensemble *e, int32_t nsteps, int32_t energy_every) {
  MB_RANGE("mb_ensemble_run");
  if (!e || nsteps < 0 || energy_every < 0) return fail(MB_ERR_ARG, "bad arguments");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  for (auto &L : e->slots)
    if (L.used) L.d.steps_target = L.d.steps_done + nsteps;
  if (e->dirty)
    MB_TRY(rebuild(e));
  else
    MB_TRY(push_targets(e));
  long long n = 0;
  MB_TRY(advance(e, (long long)nsteps + 1, energy_every, &n));
  return MB_OK;
}

int mb_ensemble_sync(mb_ensemble *e) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_CUDA(cudaStreamSynchronize(e->stream));
  MB_TRY(check_err(e));
  for (size_t c = 0; c < e->order.size(); c++) {
    const LatHost &L = e->slots[e->order[c]];
    if (L.d.n_itl > 0) {
      int fc[3];
      MB_CUDA(cudaMemcpy(fc, L.d.flag_count, sizeof(fc), cudaMemcpyDeviceToHost));
      if (fc[2]) return fail(MB_ERR_ARG, "interstitial flag list overflowed");
    }
  }
  return MB_OK;
}

int mb_ensemble_download(mb_ensemble *e, int32_t slot, mb_atom_element *box, mb_atom_element *itl, int32_t *n_itl) {
  if (!e || !box) return fail(MB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  MB_CUDA(cudaStreamSynchronize(e->stream));
  MB_TRY(check_err(e));
  MB_TRY(sync_desc(e));
  LatHost &L = e->slots[slot];
  const LatDesc &d = L.d;
  const size_t nb = 2 * (size_t)d.bcx * d.by * d.bz;
  mb_atom_element *stage = nullptr;
  MB_CUDA(cudaMalloc(&stage, nb * sizeof(mb_atom_element)));
  const int grid = (int)std::min<size_t>((nb + 255) / 256, 16 * (size_t)device_sm_count());
  k_ens_pack<<<grid, 256, 0, e->stream>>>(d, stage, L.ids, e->cfg.lattice_const, e->P.h, e->P.dt);
  cudaError_t r = cudaMemcpyAsync(box, stage, nb * sizeof(mb_atom_element), cudaMemcpyDeviceToHost, e->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
  cudaFree(stage);
  if (r != cudaSuccess) return cuda_fail(r, "lattice download");
  if (n_itl) *n_itl = d.n_itl;
  if (itl && d.n_itl > 0) {
    const int n = d.n_itl, c = d.primed ? (d.cur ^ 1) : d.cur;
    std::vector<double> x[3], v[3], f[3], rho(n), df(n);
    double *src_x[3] = {d.ipx[c], d.ipy[c], d.ipz[c]}, *src_v[3] = {d.ivx, d.ivy, d.ivz},
           *src_f[3] = {d.ifx, d.ify, d.ifz};
    for (int k = 0; k < 3; k++) {
      x[k].resize(n);
      v[k].resize(n);
      f[k].resize(n);
      MB_CUDA(cudaMemcpy(x[k].data(), src_x[k], sizeof(double) * n, cudaMemcpyDeviceToHost));
      MB_CUDA(cudaMemcpy(v[k].data(), src_v[k], sizeof(double) * n, cudaMemcpyDeviceToHost));
      MB_CUDA(cudaMemcpy(f[k].data(), src_f[k], sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    MB_CUDA(cudaMemcpy(rho.data(), d.irho, sizeof(double) * n, cudaMemcpyDeviceToHost));
    MB_CUDA(cudaMemcpy(df.data(), d.idf, sizeof(double) * n, cudaMemcpyDeviceToHost));
    std::vector<int64_t> ids(n);
    std::vector<int8_t> types(n);
    MB_CUDA(cudaMemcpy(ids.data(), d.iids, sizeof(int64_t) * n, cudaMemcpyDeviceToHost));
    MB_CUDA(cudaMemcpy(types.data(), d.itype, n, cudaMemcpyDeviceToHost));
    for (int q = 0; q < n; q++) {
      mb_atom_element &a = itl[q];
      a.id = ids[q];
      a.type = types[q];
      a.pad_ = 0;
      for (int k = 0; k < 3; k++) {
        a.x[k] = x[k][q];
        a.f[k] = f[k][q];
        a.v[k] = v[k][q] - (d.primed ? e->P.h * f[k][q] : 0.0);
      }
      a.rho = rho[q];
      a.df = df[q];
    }
  }
  return MB_OK;
}

int mb_ensemble_status(mb_ensemble *e, int32_t slot, int64_t *steps_done, int64_t *steps_target,
                       int64_t *device_bytes) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  MB_TRY(sync_desc(e));
  const LatHost &L = e->slots[slot];
  if (steps_done) *steps_done = L.d.steps_done;
  if (steps_target) *steps_target = L.d.steps_target;
  if (device_bytes) *device_bytes = (int64_t)L.bytes;
  return MB_OK;
}

int mb_ensemble_energies(mb_ensemble *e, int32_t slot, double *out, int32_t cap, int32_t *n) {
  if (!e || !n) return fail(MB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  const LatHost &L = e->slots[slot];
  const int m = (int)L.e_step.size();
  for (int k = 0; k < std::min(m, cap) && out; k++) {
    out[3 * k] = L.e_step[k];
    out[3 * k + 1] = L.e_pe[k];
    out[3 * k + 2] = L.e_ke[k];
  }
  *n = m;
  return MB_OK;
}

int mb_ensemble_clear_energies(mb_ensemble *e, int32_t slot) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  LatHost &L = e->slots[slot];
  L.e_step.clear();
  L.e_pe.clear();
  L.e_ke.clear();
  return MB_OK;
}

int mb_ensemble_time(mb_ensemble *e, int32_t nsteps, float *ms) {
  if (!e || !ms || nsteps <= 0) return fail(MB_ERR_ARG, "bad arguments");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  // every lattice stays active for the whole timed region: one spare step covers the
  // untimed priming launch below
  for (auto &L : e->slots)
    if (L.used) L.d.steps_target = L.d.steps_done + nsteps + 1;
  if (e->dirty)
    MB_TRY(rebuild(e));
  else
    MB_TRY(push_targets(e));
  bool unprimed = false;
  for (int s : e->order) unprimed |= !e->slots[s].d.primed;
  if (unprimed) {
    long long n = 0;
    MB_TRY(advance(e, 1, 0, &n));
  }
  MB_CUDA(cudaStreamSynchronize(e->stream));
  MB_CUDA(cudaEventRecord(e->ev[0], e->stream));
  long long n = 0;
  MB_TRY(advance(e, nsteps, 0, &n));
  MB_CUDA(cudaEventRecord(e->ev[1], e->stream));
  MB_CUDA(cudaEventSynchronize(e->ev[1]));
  MB_CUDA(cudaEventElapsedTime(ms, e->ev[0], e->ev[1]));
  MB_TRY(check_err(e));
  if (n != nsteps) return fail(MB_ERR_STATE, "timed launches ended early");
  return MB_OK;
}

int mb_ensemble_kernel_times(mb_ensemble *e, float *rho_ms, float *force_ms, int32_t *kernels_per_step) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  const int reps = 4;
  for (auto &L : e->slots)
    if (L.used) L.d.steps_target = L.d.steps_done + reps + 1;
  if (e->dirty)
    MB_TRY(rebuild(e));
  else
    MB_TRY(push_targets(e));
  if (e->n_tiles == 0) return fail(MB_ERR_STATE, "no lattices");
  bool unprimed = false;
  for (int s : e->order) unprimed |= !e->slots[s].d.primed;
  if (unprimed) {
    long long n = 0;
    MB_TRY(advance(e, 1, 0, &n));
  }
  float tr = 0.f, tf = 0.f;
  e->P.energy = 0;
  for (int k = 0; k < reps; k++) {
    if (e->split) {
      MB_TRY(mx_launch_step(e->P, e->mxs, 0, 0, e->stream, e->ev + 2, nullptr));
    } else {
      MB_CUDA(cudaEventRecord(e->ev[4], e->stream));
      MB_TRY(ens_launch(e->P, e->grid, e->stream));
      MB_CUDA(cudaEventRecord(e->ev[5], e->stream));
    }
    e->launches++;
    MB_CUDA(cudaStreamSynchronize(e->stream));
    float a = 0.f, b = 0.f;
    if (e->split) {
      MB_CUDA(cudaEventElapsedTime(&a, e->ev[2], e->ev[3]));
      MB_CUDA(cudaEventElapsedTime(&b, e->ev[4], e->ev[5]));
    } else {
      MB_CUDA(cudaEventElapsedTime(&b, e->ev[4], e->ev[5]));
    }
    tr += a;
    tf += b;
  }
  e->synced_desc = false;
  MB_TRY(check_err(e));
  if (rho_ms) *rho_ms = tr / reps;
  if (force_ms) *force_ms = tf / reps;
  if (kernels_per_step)
    *kernels_per_step =
        // split: rho, force, bookkeeping; with interstitials also clear, bin, mark and the
        // two item passes; with conversion the conversion kernel
        e->split ? (3 + (e->P.n_itl_lats > 0 ? 5 + (e->P.conv2 > 0.0 ? 1 : 0) : 0)) : 1;
  return MB_OK;
}

int mb_ensemble_set_policy(mb_ensemble *e, int32_t policy) {
  if (!e || policy < -1 || policy >= ENS_NSHAPE) return fail(MB_ERR_ARG, "policy must be -1..3");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  e->policy = policy;
  e->dirty = true;
  return MB_OK;
}

// Times every tile-shape policy on a snapshot of the ensemble and keeps the fastest;
// the lattices' state is restored afterwards, so tuning costs no simulation steps.
int mb_ensemble_autotune(mb_ensemble *e, int32_t steps, int32_t *policy, float *best_ms) {
  if (!e || steps <= 0) return fail(MB_ERR_ARG, "bad arguments");
  std::vector<std::pair<int, float>> results;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    MB_CUDA(cudaStreamSynchronize(e->stream));
    MB_TRY(sync_desc(e));
  }
  // snapshot every lattice block and descriptor
  std::vector<void *> snaps;
  std::vector<LatDesc> saved;
  size_t total = 0;
  for (auto &L : e->slots)
    if (L.used) total += L.bytes;
  void *snap = nullptr;
  if (cudaMalloc(&snap, std::max<size_t>(total, 256)) != cudaSuccess)
    return fail(MB_ERR_NOMEM, "no device memory for the autotune snapshot");
  size_t off = 0;
  for (auto &L : e->slots)
    if (L.used) {
      cudaMemcpyAsync((char *)snap + off, L.block, L.bytes, cudaMemcpyDeviceToDevice, e->stream);
      off += L.bytes;
      saved.push_back(L.d);
    }
  const int old_policy = e->policy, old_mode = e->mode;
  int rc = MB_OK;
  // candidates: the split kernels (encoded as policy ENS_NSHAPE), then every tile policy
  // of the persistent kernel; an explicit mode restricts the search to that kernel
  std::vector<std::pair<int, int>> cand; // (mode, policy)
  if (old_mode != 1) cand.push_back({2, old_policy});
  if (old_mode != 2)
    for (int pol = -1; pol < ENS_NSHAPE; pol++) cand.push_back({1, pol});
  for (size_t ci = 0; ci < cand.size() && rc == MB_OK; ci++) {
    rc = mb_ensemble_set_mode(e, cand[ci].first);
    if (rc == MB_OK) rc = mb_ensemble_set_policy(e, cand[ci].second);
    float ms = 0.f;
    if (rc == MB_OK) rc = mb_ensemble_time(e, steps, &ms);
    if (rc == MB_OK)
      results.push_back({cand[ci].first == 2 ? ENS_NSHAPE : cand[ci].second, ms});
    else if (cand[ci].first == 2 && rc == MB_ERR_UNSUPPORTED && old_mode == 0)
      rc = MB_OK; // split kernels do not apply here: tune the persistent kernel only
    // restore state for the next candidate
    std::lock_guard<std::mutex> lk(e->mu);
    cudaStreamSynchronize(e->stream);
    off = 0;
    size_t q = 0;
    for (auto &L : e->slots)
      if (L.used) {
        cudaMemcpyAsync(L.block, (char *)snap + off, L.bytes, cudaMemcpyDeviceToDevice, e->stream);
        off += L.bytes;
        const LatDesc &sd = saved[q++];
        L.d.cur = sd.cur;
        L.d.primed = sd.primed;
        L.d.steps_done = sd.steps_done;
        L.d.steps_target = sd.steps_target;
        L.d.n_itl = sd.n_itl; // the block copy restored the list itself
        L.e_step.clear();
        L.e_pe.clear();
        L.e_ke.clear();
      }
    cudaStreamSynchronize(e->stream);
    e->synced_desc = true;
    e->dirty = true;
  }
  cudaFree(snap);
  if (rc != MB_OK || results.empty()) {
    e->policy = old_policy;
    e->mode = old_mode;
    e->dirty = true;
    return rc != MB_OK ? rc : fail(MB_ERR_STATE, "no kernel could be timed");
  }
  auto best = std::min_element(results.begin(), results.end(),
                               [](const std::pair<int, float> &a, const std::pair<int, float> &b) {
                                 return a.second < b.second;
                               });
  if (best->first == ENS_NSHAPE) {
    MB_TRY(mb_ensemble_set_mode(e, old_mode == 0 ? 0 : 2));
    MB_TRY(mb_ensemble_set_policy(e, old_policy));
  } else {
    MB_TRY(mb_ensemble_set_mode(e, 1));
    MB_TRY(mb_ensemble_set_policy(e, best->first));
  }
  if (policy) *policy = best->first;
  if (best_ms) *best_ms = best->second;
  return MB_OK;
}

int mb_ensemble_info(mb_ensemble *e, int64_t *n_sites, int64_t *n_tiles, int64_t *device_bytes, int32_t *n_slots) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->dirty) MB_TRY(rebuild(e));
  int64_t ns = 0;
  int used = 0;
  for (auto &L : e->slots)
    if (L.used) {
      ns += 2LL * L.d.bcx * L.d.by * L.d.bz;
      used++;
    }
  if (n_sites) *n_sites = ns;
  if (n_tiles) *n_tiles = e->n_tiles;
  if (device_bytes) *device_bytes = (int64_t)e->device_bytes;
  if (n_slots) *n_slots = used;
  return MB_OK;
}

int mb_ensemble_set_mode(mb_ensemble *e, int32_t mode) {
  if (!e || mode < 0 || mode > 2) return fail(MB_ERR_ARG, "mode must be 0 (auto), 1 (persistent) or 2 (split)");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  e->mode = mode;
  e->dirty = true;
  return MB_OK;
}

int mb_ensemble_set_wait_limit(mb_ensemble *e, int64_t barrier_polls) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  if (barrier_polls > 0xFFFFFFFFLL) return fail(MB_ERR_ARG, "barrier_polls above 2^32 - 1");
  std::lock_guard<std::mutex> lk(e->mu);
  MB_TRY(sync_desc(e));
  e->bar_spins = barrier_polls < 0 ? ENS_BAR_SPINS : (unsigned)barrier_polls;
  e->P.bar_spins = e->bar_spins;
  drop_graph(e); // the captured launch holds the old limit
  return MB_OK;
}

int mb_ensemble_set_graphs(mb_ensemble *e, int enable) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  e->graphs_ok = enable != 0;
  drop_graph(e);
  return MB_OK;
}

int mb_ensemble_set_conversion(mb_ensemble *e, double convert_distance, double recombine_distance) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  if (convert_distance < 0 || recombine_distance < 0 || (convert_distance > 0 && recombine_distance >= convert_distance))
    return fail(MB_ERR_ARG, "need 0 <= recombine_distance < convert_distance (0 switches conversion off)");
  std::lock_guard<std::mutex> lk(e->mu);
  for (auto &L : e->slots)
    if (L.used && convert_distance > 0 && L.cap_itl > MB_CONV_ITL_MAX)
      return fail(MB_ERR_ARG, "max_interstitials above the conversion limit (65536)");
  MB_TRY(sync_desc(e));
  e->conv_d = convert_distance;
  e->rec_d = convert_distance > 0 ? recombine_distance : 0.0;
  e->P.conv2 = e->conv_d * e->conv_d;
  e->P.rec2 = e->rec_d * e->rec_d;
  e->dirty = true; // the interstitial lattice list and the captured step change
  return MB_OK;
}

int mb_ensemble_conversion_stats(mb_ensemble *e, int32_t slot, int64_t *counters, int32_t *n_itl) {
  if (!e) return fail(MB_ERR_ARG, "null ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= (int)e->slots.size() || !e->slots[slot].used) return fail(MB_ERR_ARG, "no such slot");
  MB_CUDA(cudaStreamSynchronize(e->stream));
  MB_TRY(sync_desc(e));
  const LatHost &L = e->slots[slot];
  long long c[4] = {0, 0, 0, 0};
  MB_CUDA(cudaMemcpy(c, L.d.conv_counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (counters)
    for (int k = 0; k < 4; k++) counters[k] = (int64_t)c[k];
  if (n_itl) *n_itl = L.d.n_itl;
  return MB_OK;
}

} // extern "C"
