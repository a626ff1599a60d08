// Drop-in plugin hooks: the misa-md-hip arch-acceleration interface
// (src/hip_arch_acc_imp.cpp:28-225, src/mem.cpp:14-32, src/cli.cpp:16-27) on the
// host's ghost-extended AoS lattice.
//
// The reference streams z-slabs of the AoS array through two device buffers
// with a fresh pair of streams per call (src/double-buffer/*).  Here the rho and
// force hooks stream the array in z-slabs too, on two long-lived copy streams: the
// ext layers slab k needs come in on one while the compute stream converts them to
// the split SoA layout, runs the pass over slab k's box layers and converts back, and
// slab k's box rows go out on the other while later slabs still come in.  The host
// fills the ghosts, so slab k depends on nothing after its own ext layers and the
// slabs need no particular thickness.  Same results (bitwise, for every slab count),
// same synchronous semantics, and none of the trailing-layer loss the reference's
// split has when box_z % batches != 0 (src/double-buffer/double_buffer.cpp:12,42-47):
// the layers are split evenly.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "mb_common.cuh"

#define MB_HOOK_SLAB_MAX 32

namespace mb {

struct HookCtx {
  bool env = false, domain = false, stencil = false, pot = false;
  int device = 0;
  unsigned int batches = 1;
  mb_device_domain dom{};
  Geom g{};
  StencilSet st{};
  std::vector<int64_t> even, odd;
  PotHost *potp = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // z-slab streaming of the rho and force hooks
  cudaStream_t cp_in = nullptr, cp_out = nullptr;
  cudaEvent_t ev_go = nullptr, ev_in[MB_HOOK_SLAB_MAX] = {}, ev_out[MB_HOOK_SLAB_MAX] = {};
  // device buffers sized for the ext lattice
  size_t n_ext = 0;
  mb_atom_element *aos = nullptr;
  double *px = nullptr, *py = nullptr, *pz = nullptr, *df = nullptr, *rho = nullptr, *fx = nullptr, *fy = nullptr,
         *fz = nullptr;
  int8_t *code = nullptr;
  int *bad = nullptr;
  float kernel_ms = 0.f, copy_ms = 0.f;
  // half-neighbour mode (the reference's USE_NEWTONS_THIRD_LOW build)
  bool half = false;
  HalfOff *d_half = nullptr;
  int half_cap = 0, half_n[2] = {0, 0};
};

static HookCtx g_ctx;
static std::mutex g_mu;

// Device address of the allocation-free rho pass's fixed scratch array, per device
// ordinal (looked up on first use; see mb_eam_rho_calc_noalloc).
#define MB_NOALLOC_MAX_DEVICES 64
static unsigned char *g_noalloc_dev[MB_NOALLOC_MAX_DEVICES] = {};

static void free_buffers(HookCtx &c) {
  void *ptrs[] = {c.aos, c.px, c.py, c.pz, c.df, c.rho, c.fx, c.fy, c.fz, c.code, c.bad};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  c.aos = nullptr;
  c.px = c.py = c.pz = c.df = c.rho = c.fx = c.fy = c.fz = nullptr;
  c.code = nullptr;
  c.bad = nullptr;
  c.n_ext = 0;
}

static int ensure_buffers(HookCtx &c) {
  const size_t n = (size_t)c.dom.ext_size_x * c.dom.ext_size_y * c.dom.ext_size_z;
  if (c.n_ext == n && c.aos) return MB_OK;
  free_buffers(c);
  MB_CUDA(cudaMalloc(&c.aos, n * sizeof(mb_atom_element)));
  double **dp[] = {&c.px, &c.py, &c.pz, &c.df, &c.rho, &c.fx, &c.fy, &c.fz};
  for (double **p : dp) MB_CUDA(cudaMalloc(p, n * sizeof(double)));
  MB_CUDA(cudaMalloc(&c.code, (n + 3) & ~(size_t)3));
  MB_CUDA(cudaMalloc(&c.bad, sizeof(int)));
  c.n_ext = n;
  return MB_OK;
}

static Lattice64 lattice_view(HookCtx &c) {
  Lattice64 L{};
  L.px = c.px;
  L.py = c.py;
  L.pz = c.pz;
  L.code = c.code;
  L.df = c.df;
  L.rho = c.rho;
  L.fx = c.fx;
  L.fy = c.fy;
  L.fz = c.fz;
  return L;
}

static void free_half(HookCtx &c) {
  if (c.d_half) cudaFree(c.d_half);
  c.d_half = nullptr;
  c.half_cap = 0;
  c.half_n[0] = c.half_n[1] = 0;
}

static int require_ready(const HookCtx &c) {
  if (!c.env) return fail(MB_ERR_STATE, "mb_env_init has not been called");
  if (!c.domain) return fail(MB_ERR_STATE, "mb_domain_init has not been called");
  if (!c.stencil) return fail(MB_ERR_STATE, "mb_nei_offset_init has not been called");
  if (!c.pot) return fail(MB_ERR_STATE, "mb_pot_init has not been called");
  return MB_OK;
}

// Slabs of a streamed hook pass: the -b/--batches count when the host set one above 1,
// else as many as give each slab at least 4 MiB of records, at most 16 (measured on
// 128^3 cells: 16 slabs 11.0 ms per pass, 32 slabs 11.4, 8 slabs 11.3, one piece 18.5);
// never more than one per box layer; 1 = one piece.
static int hook_slabs(const HookCtx &c) {
  const mb_device_domain &d = c.dom;
  if (d.ext_size_z != d.box_size_z + 2 * d.ghost_size_z) return 1;
  long long n = c.batches > 1 ? (long long)c.batches
                              : std::min<long long>(16, (long long)(c.n_ext * sizeof(mb_atom_element) / (4u << 20)));
  n = std::min<long long>(std::min<long long>(n, MB_HOOK_SLAB_MAX), d.box_size_z);
  return n < 2 ? 1 : (int)n;
}

// Copy the ext array in, convert, run `body` over box layers [z0, z1), convert back,
// copy the box rows out; in z-slabs when `sliced` and more than one slab is planned.
// kernel_ms / copy_ms: the span of the device work, and the rest of the call.
template <class Body>
static int run_hook(HookCtx &c, mb_atom_element *atoms, int with_df, int pack_what, bool sliced, Body body) {
  if (!atoms) return fail(MB_ERR_ARG, "null atoms array");
  MB_TRY(require_ready(c));
  MB_TRY(ensure_buffers(c));
  const mb_device_domain &d = c.dom;
  const size_t n = c.n_ext;
  const size_t ex = d.ext_size_x, ey = d.ext_size_y;
  auto row0 = [&](int z) { return (((size_t)d.ghost_size_z + z) * ey + d.ghost_size_y) * ex + d.ghost_size_x; };
  auto row1 = [&](int z) { return row0(z) + ((size_t)d.box_size_y - 1) * ex + d.box_size_x - 1; };
  cudaStream_t s = c.stream;
  const int n_types = pot_dev(c.potp).n_types;
  const int nsl = sliced ? hook_slabs(c) : 1;
  MB_CUDA(cudaMemsetAsync(c.bad, 0, sizeof(int), s));
  MB_CUDA(cudaEventRecord(c.ev[0], s));
  Lattice64 L = lattice_view(c);
  if (nsl == 1) {
    MB_CUDA(cudaMemcpyAsync(c.aos, atoms, n * sizeof(mb_atom_element), cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaEventRecord(c.ev[1], s));
    MB_TRY(launch_unpack_ext(c.g, c.aos, d.ext_size_x, d.ext_size_y, d.ext_size_z, L, with_df, c.bad, n_types, s));
    MB_TRY(body(L, s, 0, d.box_size_z));
    MB_TRY(launch_pack_ext(c.g, c.aos, d.ext_size_x, d.ext_size_y, L, pack_what, s));
    MB_CUDA(cudaEventRecord(c.ev[2], s));
    const size_t first = row0(0), last = row1(d.box_size_z - 1);
    MB_CUDA(cudaMemcpyAsync(atoms + first, c.aos + first, (last - first + 1) * sizeof(mb_atom_element),
                            cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaEventRecord(c.ev[3], s));
  } else {
    // slab k: box layers [zb[k], zb[k+1]); it reads ext layers [zb[k], zb[k+1] + 2 gz),
    // of which ext layers [E_k, zb[k+1] + 2 gz) arrive with it (E_0 = 0, E_k = zb[k] + 2 gz)
    int zb[MB_HOOK_SLAB_MAX + 1];
    for (int k = 0; k <= nsl; k++) zb[k] = (int)((long long)k * d.box_size_z / nsl);
    const size_t layer = ex * ey;
    auto e0 = [&](int k) { return k == 0 ? (size_t)0 : ((size_t)zb[k] + 2 * d.ghost_size_z) * layer; };
    auto e1 = [&](int k) { return ((size_t)zb[k + 1] + 2 * d.ghost_size_z) * layer; };
    MB_CUDA(cudaEventRecord(c.ev_go, s));
    MB_CUDA(cudaStreamWaitEvent(c.cp_in, c.ev_go, 0));
    for (int k = 0; k < nsl; k++) {
      MB_CUDA(cudaMemcpyAsync(c.aos + e0(k), atoms + e0(k), (e1(k) - e0(k)) * sizeof(mb_atom_element),
                              cudaMemcpyHostToDevice, c.cp_in));
      MB_CUDA(cudaEventRecord(c.ev_in[k], c.cp_in));
    }
    // one slab: wait for its layers, convert, compute, convert back, send its rows out
    auto slab = [&](int k) -> int {
      MB_CUDA(cudaStreamWaitEvent(s, c.ev_in[k], 0));
      if (k == 0) MB_CUDA(cudaEventRecord(c.ev[1], s));
      MB_TRY(launch_unpack_ext(c.g, c.aos, d.ext_size_x, d.ext_size_y, d.ext_size_z, L, with_df, c.bad, n_types, s,
                               (long long)e0(k), (long long)e1(k)));
      MB_TRY(body(L, s, zb[k], zb[k + 1]));
      MB_TRY(launch_pack_ext(c.g, c.aos, d.ext_size_x, d.ext_size_y, L, pack_what, s, zb[k], zb[k + 1]));
      MB_CUDA(cudaEventRecord(c.ev_out[k], s));
      MB_CUDA(cudaStreamWaitEvent(c.cp_out, c.ev_out[k], 0));
      const size_t first = row0(zb[k]), last = row1(zb[k + 1] - 1);
      MB_CUDA(cudaMemcpyAsync(atoms + first, c.aos + first, (last - first + 1) * sizeof(mb_atom_element),
                              cudaMemcpyDeviceToHost, c.cp_out));
      return MB_OK;
    };
    int rc = MB_OK;
    for (int k = 0; k < nsl && rc == MB_OK; k++) rc = slab(k);
    if (rc == MB_OK && cudaEventRecord(c.ev[2], s) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "cudaEventRecord");
    if (rc == MB_OK && cudaEventRecord(c.ev[3], c.cp_out) != cudaSuccess)
      rc = cuda_fail(cudaGetLastError(), "cudaEventRecord");
    // drain both copy streams, also after an error, so the caller's array is not in use
    const cudaError_t e_in = cudaStreamSynchronize(c.cp_in), e_out = cudaStreamSynchronize(c.cp_out);
    MB_TRY(rc);
    MB_CUDA(e_in);
    MB_CUDA(e_out);
  }
  int bad = 0;
  MB_CUDA(cudaMemcpyAsync(&bad, c.bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  float tot = 0, k = 0;
  cudaEventElapsedTime(&tot, c.ev[0], c.ev[3]);
  cudaEventElapsedTime(&k, c.ev[1], c.ev[2]);
  c.kernel_ms = k;
  c.copy_ms = tot - k;
  if (bad) return fail(MB_ERR_ARG, "atom type without a potential table (treated as vacant)");
  return MB_OK;
}

// Half-neighbour pass: the whole ext array goes in, every record's rho (or f) is
// rewritten with the shares it received, and the whole array comes back (ghost
// records carry the shares owed to atoms owned elsewhere).
static int run_half(HookCtx &c, mb_atom_element *atoms, bool force, double rc2) {
  if (!atoms) return fail(MB_ERR_ARG, "null atoms array");
  MB_TRY(require_ready(c));
  MB_TRY(ensure_buffers(c));
  const size_t n = c.n_ext;
  cudaStream_t s = c.stream;
  MB_CUDA(cudaMemsetAsync(c.bad, 0, sizeof(int), s));
  MB_CUDA(cudaEventRecord(c.ev[0], s));
  MB_CUDA(cudaMemcpyAsync(c.aos, atoms, n * sizeof(mb_atom_element), cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaEventRecord(c.ev[1], s));
  MB_TRY(launch_half64(force, c.aos, c.dom, c.d_half, c.half_cap, c.half_n, pot_dev(c.potp), rc2, c.bad, s));
  MB_CUDA(cudaEventRecord(c.ev[2], s));
  MB_CUDA(cudaMemcpyAsync(atoms, c.aos, n * sizeof(mb_atom_element), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaEventRecord(c.ev[3], s));
  int bad = 0;
  MB_CUDA(cudaMemcpyAsync(&bad, c.bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  float a = 0, b = 0, k = 0;
  cudaEventElapsedTime(&a, c.ev[0], c.ev[1]);
  cudaEventElapsedTime(&k, c.ev[1], c.ev[2]);
  cudaEventElapsedTime(&b, c.ev[2], c.ev[3]);
  c.kernel_ms = k;
  c.copy_ms = a + b;
  if (bad) return fail(MB_ERR_ARG, "atom type without a potential table (treated as vacant)");
  return MB_OK;
}

} // namespace mb

using namespace mb;

extern "C" {

int mb_env_init(int device) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  int n = 0;
  MB_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(MB_ERR_ARG, "device index out of range");
  MB_CUDA(cudaSetDevice(device));
  if (!c.stream) {
    MB_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    for (auto &e : c.ev) MB_CUDA(cudaEventCreate(&e));
    MB_CUDA(cudaStreamCreateWithFlags(&c.cp_in, cudaStreamNonBlocking));
    MB_CUDA(cudaStreamCreateWithFlags(&c.cp_out, cudaStreamNonBlocking));
    MB_CUDA(cudaEventCreateWithFlags(&c.ev_go, cudaEventDisableTiming));
    for (int k = 0; k < MB_HOOK_SLAB_MAX; k++) {
      MB_CUDA(cudaEventCreateWithFlags(&c.ev_in[k], cudaEventDisableTiming));
      MB_CUDA(cudaEventCreateWithFlags(&c.ev_out[k], cudaEventDisableTiming));
    }
  }
  c.device = device;
  c.env = true;
  return MB_OK;
}

int mb_env_clean(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (c.stream) cudaStreamSynchronize(c.stream);
  free_buffers(c);
  free_half(c);
  c.half = false;
  if (c.potp) pot_free(c.potp);
  c.potp = nullptr;
  for (auto &e : c.ev)
    if (e) cudaEventDestroy(e), e = nullptr;
  for (int k = 0; k < MB_HOOK_SLAB_MAX; k++) {
    if (c.ev_in[k]) cudaEventDestroy(c.ev_in[k]), c.ev_in[k] = nullptr;
    if (c.ev_out[k]) cudaEventDestroy(c.ev_out[k]), c.ev_out[k] = nullptr;
  }
  if (c.ev_go) cudaEventDestroy(c.ev_go), c.ev_go = nullptr;
  for (cudaStream_t *q : {&c.cp_in, &c.cp_out})
    if (*q) cudaStreamSynchronize(*q), cudaStreamDestroy(*q), *q = nullptr;
  if (c.stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
  c.env = c.domain = c.stencil = c.pot = false;
  for (auto &p : g_noalloc_dev) p = nullptr; // looked up again on the next call
  return MB_OK;
}

int mb_domain_init(const mb_device_domain *d) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!d) return fail(MB_ERR_ARG, "null domain");
  if (d->box_size_x <= 0 || d->box_size_y <= 0 || d->box_size_z <= 0) return fail(MB_ERR_ARG, "empty box");
  if (d->ghost_size_x < 0 || d->ghost_size_y < 0 || d->ghost_size_z < 0) return fail(MB_ERR_ARG, "negative ghost");
  if ((d->ghost_size_x & 1) || (d->box_size_x & 1))
    return fail(MB_ERR_ARG, "ghost_size_x and box_size_x are doubled BCC sizes and must be even");
  if (d->ext_size_x != d->box_size_x + 2 * d->ghost_size_x || d->ext_size_y != d->box_size_y + 2 * d->ghost_size_y ||
      d->ext_size_z != d->box_size_z + 2 * d->ghost_size_z)
    return fail(MB_ERR_ARG, "ext size must equal box + 2 * ghost");
  const long long next = (long long)d->ext_size_x * d->ext_size_y * d->ext_size_z;
  if (next / 2 > 0x3fffffffLL) return fail(MB_ERR_ARG, "lattice too large for 32-bit stencil offsets");
  c.dom = *d;
  Geom &g = c.g;
  g.ecx = d->ext_size_x / 2;
  g.ey = d->ext_size_y;
  g.ez = d->ext_size_z;
  g.gcx = d->ghost_size_x / 2;
  g.gy = d->ghost_size_y;
  g.gz = d->ghost_size_z;
  g.bcx = d->box_size_x / 2;
  g.by = d->box_size_y;
  g.bz = d->box_size_z;
  g.images = 0; // the host owns the ghost region in drop-in mode
  g.E = (long long)g.ecx * g.ey * g.ez;
  g.Lx = g.Ly = g.Lz = 0.0;
  g.iLx = g.iLy = g.iLz = 0.0;
  c.domain = true;
  // linear offsets are tied to the ext sizes they were made for: a new domain needs
  // mb_nei_offset_init again (the reference's init order: domain, then offsets)
  c.stencil = false;
  c.even.clear();
  c.odd.clear();
  free_half(c);
  return MB_OK;
}

int mb_set_half_neighbour(int enable) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!c.env) return fail(MB_ERR_STATE, "mb_env_init has not been called");
  const bool h = enable != 0;
  if (h != c.half) {
    // full and half stencils are different offset sets: the next pass needs
    // mb_nei_offset_init with the kind this mode takes
    c.half = h;
    c.stencil = false;
    c.even.clear();
    c.odd.clear();
    free_half(c);
  }
  return MB_OK;
}

int mb_nei_offset_init(const int64_t *nei_even, size_t n_even, const int64_t *nei_odd, size_t n_odd) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!c.domain) return fail(MB_ERR_STATE, "mb_domain_init must come before mb_nei_offset_init");
  if ((n_even && !nei_even) || (n_odd && !nei_odd)) return fail(MB_ERR_ARG, "null stencil");
  // sublattice s of the split layout holds doubled ext columns of parity s; with an
  // even ghost the global parity of its sites is (s + box_index_start_x) & 1
  // (the reference selects the stencil by (x + box_index_start_x) % 2,
  // src/kernels/kernel_itl.hpp:82).
  if (c.half) {
    std::vector<HalfOff> h;
    int cap = 0;
    MB_TRY(half_stencil_build(c.dom, nei_even, n_even, nei_odd, n_odd, h, cap));
    free_half(c);
    MB_CUDA(cudaMalloc(&c.d_half, h.size() * sizeof(HalfOff)));
    MB_CUDA(cudaMemcpy(c.d_half, h.data(), h.size() * sizeof(HalfOff), cudaMemcpyHostToDevice));
    c.half_cap = cap;
    c.half_n[0] = (int)n_even;
    c.half_n[1] = (int)n_odd;
    c.even.assign(nei_even, nei_even + n_even);
    c.odd.assign(nei_odd, nei_odd + n_odd);
    c.stencil = true;
    return MB_OK;
  }
  const int par[2] = {(int)(c.dom.box_index_start_x & 1), (int)((1 + c.dom.box_index_start_x) & 1)};
  StencilSet st;
  MB_TRY(stencil_from_linear(nei_even, n_even, nei_odd, n_odd, c.dom.ext_size_x, c.dom.ext_size_y, c.g, par, &st));
  c.st = st;
  c.even.assign(nei_even, nei_even + n_even);
  c.odd.assign(nei_odd, nei_odd + n_odd);
  c.stencil = true;
  return MB_OK;
}

int mb_pot_init(const mb_eam_tables *t) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!c.env) return fail(MB_ERR_STATE, "mb_env_init has not been called");
  PotHost *p = nullptr;
  MB_TRY(pot_build(t, &p));
  if (c.potp) pot_free(c.potp);
  c.potp = p;
  c.pot = true;
  return MB_OK;
}

int mb_eam_rho_calc(mb_atom_element *atoms, double cutoff_radius) {
  MB_RANGE("mb_eam_rho_calc");
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!(cutoff_radius > 0)) return fail(MB_ERR_ARG, "cutoff must be > 0");
  if (c.half) return run_half(c, atoms, false, cutoff_radius * cutoff_radius);
  return run_hook(c, atoms, 0, 1, true, [&](Lattice64 &L, cudaStream_t s, int z0, int z1) {
    return launch_rho64(c.g, c.st, pot_dev(c.potp), L, cutoff_radius * cutoff_radius, nullptr, 0, 0, s, z0, z1);
  });
}

int mb_eam_df_calc(mb_atom_element *atoms, double cutoff_radius) {
  MB_RANGE("mb_eam_df_calc");
  // Full-neighbour mode: df already came out of the rho pass
  // (src/hip_arch_acc_imp.cpp:184-186 returns at once).  Half-neighbour mode: the
  // host has added the ghost shares of rho to their owners; df = F'(rho) of the box
  // sites (calDf, src/kernels/hip_kernels.hip.cpp:21-40).
  (void)cutoff_radius;
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!c.half) return require_ready(c);
  return run_hook(c, atoms, 2, 3, false, [&](Lattice64 &L, cudaStream_t s, int, int) {
    return launch_df_from_rho(c.g, pot_dev(c.potp), L, s);
  });
}

int mb_eam_df_from_rho(mb_atom_element *atoms) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  return run_hook(c, atoms, 2, 3, false, [&](Lattice64 &L, cudaStream_t s, int, int) {
    return launch_df_from_rho(c.g, pot_dev(c.potp), L, s);
  });
}

int mb_eam_force_calc(mb_atom_element *atoms, double cutoff_radius) {
  MB_RANGE("mb_eam_force_calc");
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!(cutoff_radius > 0)) return fail(MB_ERR_ARG, "cutoff must be > 0");
  if (c.half) return run_half(c, atoms, true, cutoff_radius * cutoff_radius);
  return run_hook(c, atoms, 1, 2, true, [&](Lattice64 &L, cudaStream_t s, int z0, int z1) {
    StepParams sp{};
    sp.rc2 = cutoff_radius * cutoff_radius;
    Lattice64 Lf = L;
    Lf.vx = Lf.vy = Lf.vz = nullptr; // forces only, no integration in drop-in mode
    return launch_force64(c.g, c.st, pot_dev(c.potp), Lf, sp, nullptr, 0, 0, s, z0, z1);
  });
}

int mb_create_atoms_mem(void **atoms, size_t data_type_size, int64_t size_x, int64_t size_y, int64_t size_z,
                        int *allocated) {
  if (!atoms) return fail(MB_ERR_ARG, "null out pointer");
  if (allocated) *allocated = 0;
  if (size_x <= 0 || size_y <= 0 || size_z <= 0 || data_type_size == 0) return fail(MB_ERR_ARG, "empty allocation");
  const size_t bytes = (size_t)size_x * (size_t)size_y * (size_t)size_z * data_type_size;
  MB_CUDA(cudaHostAlloc(atoms, bytes, cudaHostAllocPortable));
  if (allocated) *allocated = 1;
  return MB_OK;
}

int mb_release_atoms_mem(void *atoms, int *released) {
  if (released) *released = 0;
  if (!atoms) return MB_OK;
  MB_CUDA(cudaFreeHost(atoms));
  if (released) *released = 1;
  return MB_OK;
}

int mb_cli_set_batches(unsigned int batches) {
  if (batches == 0) return fail(MB_ERR_ARG, "batches must be >= 1");
  g_ctx.batches = batches;
  return MB_OK;
}

unsigned int mb_cli_batches(void) { return g_ctx.batches; }

int mb_hook_last_timing(float *kernel_ms, float *copy_ms) {
  if (kernel_ms) *kernel_ms = g_ctx.kernel_ms;
  if (copy_ms) *copy_ms = g_ctx.copy_ms;
  return MB_OK;
}

} // extern "C"

// ------------------------------------------------------------------------
// Rho pass without any device allocation.
//
// Some hosts cannot let a plugin call cudaMalloc: a process whose device memory is
// already handed out by its own pool allocator (a plugin allocation would fail or
// fragment that pool), or a timestep loop that must not take the implicit device
// synchronisation cudaMalloc / cudaFree can cause.  For them the rho pass can run
// in a fixed scratch area that is part of the library image: a file-scope device
// array of MB_NOALLOC_SCRATCH_BYTES (16 MiB), held by every GPU that loads the
// library until the process exits.  It holds the device copy of the host's AoS
// lattice and the split-layout arrays the kernels work on (145 bytes per
// ghost-extended site), so lattices of up to about 115,000 ext sites fit (for
// example 30^3 unit cells with a (4, 2, 2) ghost); larger ones are refused.
//
// The array's name is only a host-side stand-in for the device symbol: host code
// must never pass it to a kernel.  The device address is fetched once per device
// with cudaGetSymbolAddress, on the first call made with that device current; that
// first call should therefore come before any stream capture.  Every call shares
// the one array and leaves its contents behind, so calls that overlap on the GPU
// (two host threads, two streams) race; this entry point serialises calls made
// through it, but nothing guards the array against a concurrent kernel elsewhere.
#define MB_NOALLOC_SCRATCH_BYTES (16u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[MB_NOALLOC_SCRATCH_BYTES];

namespace mb {

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Bytes of scratch one ext site needs (AoS copy + positions + code + df + rho),
// each array rounded up to 256 B, plus the error flag.
static size_t noalloc_bytes(size_t n) {
  return align256(n * sizeof(mb_atom_element)) + 5 * align256(n * sizeof(double)) + align256(n) + 256;
}

static size_t noalloc_max_sites() {
  size_t lo = 0, hi = MB_NOALLOC_SCRATCH_BYTES;
  while (lo < hi) {
    const size_t mid = (lo + hi + 1) / 2;
    if (noalloc_bytes(mid) <= MB_NOALLOC_SCRATCH_BYTES)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

} // namespace mb

extern "C" int mb_eam_rho_calc_noalloc(mb_atom_element *atoms, double cutoff_radius) {
  std::lock_guard<std::mutex> lk(g_mu);
  HookCtx &c = g_ctx;
  if (!atoms) return fail(MB_ERR_ARG, "null atoms array");
  if (!(cutoff_radius > 0)) return fail(MB_ERR_ARG, "cutoff must be > 0");
  MB_TRY(require_ready(c));
  if (c.half) return fail(MB_ERR_UNSUPPORTED, "mb_eam_rho_calc_noalloc runs the full-neighbour pass only");
  const mb_device_domain &d = c.dom;
  const size_t n = (size_t)d.ext_size_x * d.ext_size_y * d.ext_size_z;
  if (noalloc_bytes(n) > MB_NOALLOC_SCRATCH_BYTES)
    return fail(MB_ERR_ARG, "mb_eam_rho_calc_noalloc: the ghost-extended lattice has " + std::to_string(n) +
                                " sites; the fixed scratch of " + std::to_string(MB_NOALLOC_SCRATCH_BYTES) +
                                " bytes holds at most " + std::to_string(noalloc_max_sites()) +
                                " (use mb_eam_rho_calc for larger lattices)");
  // The hooks' stream lives on the device mb_env_init selected, and each GPU has its own
  // copy of the scratch array: the address must be the one of that device.
  int dev = 0;
  MB_CUDA(cudaGetDevice(&dev));
  if (dev != c.device)
    return fail(MB_ERR_STATE, "mb_eam_rho_calc_noalloc: the calling thread's current device (" + std::to_string(dev) +
                                  ") is not the device mb_env_init selected (" + std::to_string(c.device) + ")");
  if (dev < 0 || dev >= MB_NOALLOC_MAX_DEVICES) return fail(MB_ERR_ARG, "device ordinal beyond 63");
  if (!g_noalloc_dev[dev]) {
    void *p = nullptr;
    MB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_dev[dev] = (unsigned char *)p;
  }
  unsigned char *base = g_noalloc_dev[dev];
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    unsigned char *p = base + off;
    off += align256(bytes);
    return p;
  };
  mb_atom_element *aos = (mb_atom_element *)carve(n * sizeof(mb_atom_element));
  Lattice64 L{};
  L.px = (double *)carve(n * sizeof(double));
  L.py = (double *)carve(n * sizeof(double));
  L.pz = (double *)carve(n * sizeof(double));
  L.df = (double *)carve(n * sizeof(double));
  L.rho = (double *)carve(n * sizeof(double));
  L.code = (int8_t *)carve(n);
  int *bad = (int *)carve(sizeof(int));

  const size_t first = ((size_t)d.ghost_size_z * d.ext_size_y + d.ghost_size_y) * d.ext_size_x + d.ghost_size_x;
  const size_t last = ((size_t)(d.ghost_size_z + d.box_size_z - 1) * d.ext_size_y + d.ghost_size_y + d.box_size_y - 1) *
                          d.ext_size_x +
                      d.ghost_size_x + d.box_size_x - 1;
  cudaStream_t s = c.stream;
  MB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s)); // the flag must start at zero on every call
  MB_CUDA(cudaMemcpyAsync(aos, atoms, n * sizeof(mb_atom_element), cudaMemcpyHostToDevice, s));
  // From here the caller's array may be in use by a queued copy: every exit drains the
  // stream first, so the caller can free or reuse the array as soon as this returns.
  auto drained = [&](int rc) {
    const cudaError_t e = cudaStreamSynchronize(s);
    if (rc != MB_OK) return rc;
    return e == cudaSuccess ? MB_OK : cuda_fail(e, "cudaStreamSynchronize");
  };
  int rc = launch_unpack_ext(c.g, aos, d.ext_size_x, d.ext_size_y, d.ext_size_z, L, 0, bad, pot_dev(c.potp).n_types, s);
  if (rc == MB_OK) rc = launch_rho64(c.g, c.st, pot_dev(c.potp), L, cutoff_radius * cutoff_radius, nullptr, 0, 0, s);
  int flag = 0;
  if (rc == MB_OK && cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
  MB_TRY(drained(rc));
  // A record whose type has no potential table: refuse before anything is written back,
  // so the caller's array is left as it was.
  if (flag) return fail(MB_ERR_ARG, "atom type without a potential table (treated as vacant)");
  rc = launch_pack_ext(c.g, aos, d.ext_size_x, d.ext_size_y, L, 1, s);
  if (rc == MB_OK &&
      cudaMemcpyAsync(atoms + first, aos + first, (last - first + 1) * sizeof(mb_atom_element),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
  return drained(rc);
}
