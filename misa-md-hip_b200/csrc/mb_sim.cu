// Device-resident molecular dynamics on one lattice: the B200 replacement of the
// reference's per-pass host<->device streaming (src/double-buffer/*).
//
// State lives in HBM for the whole run.  One timestep is
//   mark sites near interstitials -> rho/df (lattice) -> rho/df (interstitial
//   items) -> force + velocity-Verlet (lattice) -> force + VV (interstitial items)
// where the force passes close step n (v += h f) and drift to step n+1 into the
// second position buffer, and every site near a face writes its own periodic ghost
// images.  The steady-state step pair is captured once into a CUDA graph.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mb_common.cuh"

#define MB_SLAB_MAX 32 // z-slabs of the pipelined host-buffer step

struct mb_sim {
  mb_sim_config cfg{};
  mb::PotHost *pot = nullptr;
  mb::Geom g{};
  mb::StencilSet st{};
  std::vector<int64_t> st_even, st_odd;
  int ext_x = 0, ext_y = 0, ext_z = 0;
  long long n_ext = 0, n_box = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  // lattice
  double *pos[2][3] = {};
  int8_t *code = nullptr;
  double *df = nullptr, *rho = nullptr, *v[3] = {}, *f[3] = {};
  int64_t *id = nullptr;
  // per-item masks of the outer stencil entries in the cutoff: written by each density
  // pass, read by the force pass at the same positions (outer_ok: the phase-wise steps of
  // a z-slab wrote them at the current positions)
  uint2 *outer = nullptr;
  bool outer_ok = false;
  // interstitials
  int n_itl = 0, cap_itl = 0, cap_flag = 0;
  double *ipos[2][3] = {}, *iv[3] = {}, *ifr[3] = {}, *irho = nullptr, *idf = nullptr;
  int8_t *itype = nullptr;
  int64_t *iid = nullptr;
  int *flag_list = nullptr, *flag_count = nullptr;
  int *d_nitl = nullptr; // device-resident interstitial count (conversions change it)
  // lattice <-> interstitial conversion (off while conv_d == 0)
  double conv_d = 0.0, rec_d = 0.0;
  long long *d_cand = nullptr, *d_conv_counters = nullptr; // counters[4]
  int *d_cand_n = nullptr;
  // energies
  double *epart = nullptr;
  double *eout = nullptr; // [cap_e][2]
  int cap_e = 0, n_e = 0;
  std::vector<int> e_steps;
  // staging
  mb_atom_element *stage = nullptr;
  size_t stage_n = 0;
  int *bad = nullptr;
  // state
  int cur = 0;
  bool primed = false;
  long long step = 0;
  bool use_graphs = true;
  cudaGraphExec_t graph = nullptr; // steady step pair starting at cur == 0
  size_t device_bytes = 0;
  float last_rho_ms = 0.f, last_force_ms = 0.f;
  // host-buffer step: z-slabs streamed in on cp_in and out on cp_out while the
  // compute stream works on the slabs that have arrived
  cudaStream_t cp_in = nullptr, cp_out = nullptr;
  cudaEvent_t ev_go = nullptr, ev_in[MB_SLAB_MAX] = {}, ev_out[MB_SLAB_MAX] = {};
  int host_slabs = 0; // 0: automatic (at least 4 MiB of records per slab), 1: one piece
  // z-slab of a larger periodic lattice (one rank of a decomposed run): box layers
  // [z_first, z_first + bz) of cells_z; z ghosts filled through mb_sim_halo_*
  bool slab = false;
  int z_first = 0;
  // mixed precision: the lattice lives in a one-slot ensemble (mb_ens_host.cu)
  mb_ensemble *ens = nullptr;
  int slot = -1;
};

namespace mb {

static int dalloc(mb_sim *s, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(MB_ERR_NOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                  " bytes failed: " + cudaGetErrorString(e));
  }
  s->device_bytes += bytes;
  return MB_OK;
}

Lattice64 sim_lattice(mb_sim *s, int which) {
  Lattice64 L{};
  L.px = s->pos[which][0];
  L.py = s->pos[which][1];
  L.pz = s->pos[which][2];
  L.nx = s->pos[which ^ 1][0];
  L.ny = s->pos[which ^ 1][1];
  L.nz = s->pos[which ^ 1][2];
  L.code = s->code;
  L.df = s->df;
  L.rho = s->rho;
  L.vx = s->v[0];
  L.vy = s->v[1];
  L.vz = s->v[2];
  L.fx = s->f[0];
  L.fy = s->f[1];
  L.fz = s->f[2];
  return L;
}

Itl64 sim_itl(mb_sim *s, int which) {
  Itl64 I{};
  I.n = s->n_itl;
  I.nd = s->d_nitl;
  I.cap = s->cap_itl;
  I.cap_flag = s->cap_flag;
  I.px = s->ipos[which][0];
  I.py = s->ipos[which][1];
  I.pz = s->ipos[which][2];
  I.nx = s->ipos[which ^ 1][0];
  I.ny = s->ipos[which ^ 1][1];
  I.nz = s->ipos[which ^ 1][2];
  I.vx = s->iv[0];
  I.vy = s->iv[1];
  I.vz = s->iv[2];
  I.fx = s->ifr[0];
  I.fy = s->ifr[1];
  I.fz = s->ifr[2];
  I.rho = s->irho;
  I.df = s->idf;
  I.type = s->itype;
  I.id = s->iid;
  I.flag_list = s->flag_list;
  I.flag_count = s->flag_count;
  I.a0 = s->cfg.lattice_const;
  I.reach = s->cfg.cutoff + s->cfg.stencil_skin;
  return I;
}

StepParams sim_params(const mb_sim *s, int kick_pre, int drift) {
  StepParams sp{};
  sp.rc2 = s->cfg.cutoff * s->cfg.cutoff;
  sp.h = 0.5 * s->cfg.dt * MB_FTM2V / s->cfg.mass;
  sp.dt = s->cfg.dt;
  sp.mass = s->cfg.mass;
  sp.kick_pre = kick_pre;
  sp.drift = drift;
  sp.a0 = s->cfg.lattice_const;
  if (drift && s->conv_d > 0.0) {
    sp.conv2 = s->conv_d * s->conv_d;
    sp.cand = s->d_cand;
    sp.cand_n = s->d_cand_n;
  }
  return sp;
}

// Interstitial passes run when the host placed interstitials or conversions may create
// them (the count itself lives on the device).
static bool itl_active(const mb_sim *s) { return s->n_itl > 0 || s->conv_d > 0.0; }

// One FP64 step at positions pos[cur] (forces, closing kick, drift to pos[cur^1]).
static int step64(mb_sim *s, int energy, int kick_pre, int drift, int timed) {
  const DevPot &P = pot_dev(s->pot);
  Lattice64 L = sim_lattice(s, s->cur);
  Itl64 I = sim_itl(s, s->cur);
  StepParams sp = sim_params(s, kick_pre, drift);
  double *ep = energy ? s->epart : nullptr;
  if (energy) MB_CUDA(cudaMemsetAsync(s->epart, 0, sizeof(double) * energy_partials_needed(), s->stream));
  const int itl = itl_active(s);
  if (itl) MB_TRY(launch_itl_mark64(s->g, L, I, s->stream));
  if (timed) MB_CUDA(cudaEventRecord(s->ev[4], s->stream));
  MB_TRY(launch_rho64(s->g, s->st, P, L, sp.rc2, ep, energy, itl, s->stream, 0, -1, s->outer));
  if (timed) MB_CUDA(cudaEventRecord(s->ev[5], s->stream));
  if (itl) MB_TRY(launch_itl_rho64(s->g, s->st, P, L, I, sp.rc2, ep, energy, s->stream));
  if (timed) MB_CUDA(cudaEventRecord(s->ev[6], s->stream));
  MB_TRY(launch_force64(s->g, s->st, P, L, sp, ep, energy, itl, s->stream, 0, -1, s->outer));
  if (timed) MB_CUDA(cudaEventRecord(s->ev[7], s->stream));
  if (itl) MB_TRY(launch_itl_force64(s->g, s->st, P, L, I, sp, ep, energy, s->stream));
  if (sp.conv2 > 0.0)
    MB_TRY(launch_convert64(s->g, L, I, sp, s->rec_d * s->rec_d, s->id, s->d_nitl, s->d_conv_counters, s->stream));
  return MB_OK;
}

static int record_energy(mb_sim *s) {
  if (s->n_e >= s->cap_e) {
    const int ncap = std::max(64, 2 * s->cap_e);
    double *nb = nullptr;
    MB_TRY(dalloc(s, (void **)&nb, sizeof(double) * 2 * ncap));
    if (s->eout) {
      MB_CUDA(cudaMemcpyAsync(nb, s->eout, sizeof(double) * 2 * s->cap_e, cudaMemcpyDeviceToDevice, s->stream));
      MB_CUDA(cudaStreamSynchronize(s->stream));
      cudaFree(s->eout);
      s->device_bytes -= sizeof(double) * 2 * s->cap_e;
    }
    s->eout = nb;
    s->cap_e = ncap;
  }
  MB_TRY(launch_reduce(s->epart, 0, s->eout + 2 * s->n_e, s->stream));
  s->e_steps.push_back((int)s->step);
  s->n_e++;
  return MB_OK;
}

static int do_step(mb_sim *s, int energy, int prime) {
  MB_TRY(step64(s, energy, prime ? 0 : 1, 1, 0));
  if (energy) MB_TRY(record_energy(s));
  s->cur ^= 1;
  return MB_OK;
}

static int prime(mb_sim *s, int energy) {
  if (s->primed) return MB_OK;
  // forces at x_0, v stays v_0 for the energy sample, then drift to x_1
  MB_TRY(do_step(s, energy, 1));
  s->primed = true;
  return MB_OK;
}

static void drop_graph(mb_sim *s) {
  if (s->graph) cudaGraphExecDestroy(s->graph);
  s->graph = nullptr;
}

static int build_graph(mb_sim *s) {
  if (s->graph) return MB_OK;
  if (s->cur != 0) return fail(MB_ERR_STATE, "graph capture must start at buffer 0");
  cudaGraph_t gr = nullptr;
  MB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = MB_OK;
  for (int k = 0; k < 2 && rc == MB_OK; k++) {
    rc = step64(s, 0, 1, 1, 0);
    s->cur ^= 1;
  }
  cudaError_t e = cudaStreamEndCapture(s->stream, &gr);
  if (rc != MB_OK) {
    if (gr) cudaGraphDestroy(gr);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&s->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) {
    s->graph = nullptr;
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  return MB_OK;
}

static int run_steps(mb_sim *s, int nsteps, int energy_every) {
  int k = 0;
  while (k < nsteps) {
    const long long next = s->step + 1;
    const bool e_here = energy_every > 0 && (next % energy_every == 0);
    const bool e_after = energy_every > 0 && ((next + 1) % energy_every == 0);
    if (s->use_graphs && s->cur == 0 && k + 2 <= nsteps && !e_here && !e_after) {
      MB_TRY(build_graph(s));
      MB_CUDA(cudaGraphLaunch(s->graph, s->stream));
      s->step += 2;
      k += 2;
      continue;
    }
    s->step = next;
    MB_TRY(do_step(s, e_here ? 1 : 0, 0));
    k++;
  }
  return MB_OK;
}

// ----------------------------------------------- mixed precision delegation
static int mixed_create(const mb_sim_config *cfg, const mb_eam_tables *pot, mb_sim **out) {
  mb_ensemble_config ec{};
  ec.lattice_const = cfg->lattice_const;
  ec.mass = cfg->mass;
  ec.dt = cfg->dt;
  ec.cutoff = cfg->cutoff;
  ec.stencil_skin = cfg->stencil_skin;
  ec.max_lattices = 1;
  mb_sim *s = new mb_sim();
  s->cfg = *cfg;
  s->n_box = 2LL * cfg->cells_x * cfg->cells_y * cfg->cells_z;
  const int rc = mb_ensemble_create(&ec, pot, &s->ens);
  if (rc != MB_OK) {
    delete s;
    return rc;
  }
  *out = s;
  return MB_OK;
}

static int mixed_upload(mb_sim *s, const mb_atom_element *box, const mb_atom_element *itl, int32_t n_itl) {
  if (s->slot >= 0) MB_TRY(mb_ensemble_remove(s->ens, s->slot));
  s->slot = -1;
  mb_lattice_spec spec{s->cfg.cells_x, s->cfg.cells_y, s->cfg.cells_z, s->cfg.max_interstitials};
  return mb_ensemble_add(s->ens, &spec, box, itl, n_itl, 0, &s->slot);
}

static int mixed_need_slot(mb_sim *s) {
  return s->slot >= 0 ? MB_OK : fail(MB_ERR_STATE, "mb_sim_upload has not been called");
}

} // namespace mb

using namespace mb;

extern "C" {

static int create_sim(const mb_sim_config *cfg, const mb_eam_tables *pot, int z_first, int z_count, mb_sim **out);

int mb_sim_create(const mb_sim_config *cfg, const mb_eam_tables *pot, mb_sim **out) {
  if (!cfg) return fail(MB_ERR_ARG, "null argument");
  return create_sim(cfg, pot, 0, cfg->cells_z, out);
}

int mb_sim_create_slab(const mb_sim_config *cfg, const mb_eam_tables *pot, int32_t z_first, int32_t z_count,
                       mb_sim **out) {
  if (!cfg) return fail(MB_ERR_ARG, "null argument");
  if (cfg->precision != MB_PREC_FP64) return fail(MB_ERR_UNSUPPORTED, "z-slab runs are FP64 only");
  if (cfg->max_interstitials != 0)
    return fail(MB_ERR_UNSUPPORTED, "z-slab runs take lattices without interstitials (max_interstitials = 0)");
  if (z_first < 0 || z_count < 1 || z_first + z_count > cfg->cells_z)
    return fail(MB_ERR_ARG, "the slab's cells [z_first, z_first + z_count) must lie inside [0, cells_z)");
  return create_sim(cfg, pot, z_first, z_count, out);
}

static int create_sim(const mb_sim_config *cfg, const mb_eam_tables *pot, int z_first, int z_count, mb_sim **out) {
  if (!cfg || !pot || !out) return fail(MB_ERR_ARG, "null argument");
  *out = nullptr;
  const bool slab = z_count != cfg->cells_z;
  if (cfg->cells_x < 1 || cfg->cells_y < 1 || cfg->cells_z < 1) return fail(MB_ERR_ARG, "cells must be >= 1");
  if (!(cfg->lattice_const > 0) || !(cfg->mass > 0) || !(cfg->dt > 0) || !(cfg->cutoff > 0) ||
      cfg->stencil_skin < 0)
    return fail(MB_ERR_ARG, "lattice_const, mass, dt, cutoff must be > 0 and skin >= 0");
  if (cfg->precision != MB_PREC_FP64 && cfg->precision != MB_PREC_MIXED)
    return fail(MB_ERR_ARG, "unknown precision");
  if (cfg->max_interstitials < 0) return fail(MB_ERR_ARG, "max_interstitials < 0");
  if (cfg->precision == MB_PREC_MIXED) {
    const double reach0 = cfg->cutoff + cfg->stencil_skin;
    if (cfg->cells_x * cfg->lattice_const <= 2 * reach0 || cfg->cells_y * cfg->lattice_const <= 2 * reach0 ||
        cfg->cells_z * cfg->lattice_const <= 2 * reach0)
      return fail(MB_ERR_ARG, "box edge must exceed 2 * (cutoff + stencil_skin)");
    return mixed_create(cfg, pot, out);
  }
  const double reach = cfg->cutoff + cfg->stencil_skin;
  // The box must hold more than two interaction spheres so periodic images are
  // unique (minimum image for interstitials, single-copy ghost images).
  if (cfg->cells_x * cfg->lattice_const <= 2 * reach || cfg->cells_y * cfg->lattice_const <= 2 * reach ||
      cfg->cells_z * cfg->lattice_const <= 2 * reach)
    return fail(MB_ERR_ARG, "box edge must exceed 2 * (cutoff + stencil_skin)");

  mb_sim *s = new mb_sim();
  s->cfg = *cfg;
  s->slab = slab;
  s->z_first = z_first;
  int rc = pot_build(pot, &s->pot);
  if (rc != MB_OK) {
    delete s;
    return rc;
  }
  if (pot->cutoff < cfg->cutoff * (1 - 1e-12)) {
    pot_free(s->pot);
    delete s;
    return fail(MB_ERR_ARG, "cutoff exceeds the tabulated range");
  }
  // stencil reach decides the ghost width
  int64_t even[MB_MAX_STENCIL], odd[MB_MAX_STENCIL];
  int n = 0, rx = 0, ry = 0, rz = 0;
  rc = stencil_generate(cfg->lattice_const, reach, 1 << 20, 1 << 10, even, odd, MB_MAX_STENCIL, &n, &rx, &ry, &rz);
  if (rc != MB_OK) {
    pot_free(s->pot);
    delete s;
    return rc;
  }
  Geom &g = s->g;
  g.bcx = cfg->cells_x;
  g.by = cfg->cells_y;
  g.bz = z_count;
  // a doubled-x reach rx spans floor((s + dx) / 2) columns of the split layout:
  // at most ceil(rx / 2) for either sublattice
  g.gcx = (rx + 1) / 2;
  g.gy = ry;
  g.gz = rz;
  if (g.bcx < g.gcx || g.by < g.gy || g.bz < g.gz) {
    pot_free(s->pot);
    delete s;
    return fail(MB_ERR_ARG, slab ? "a z-slab must be at least as thick as the ghost width (the stencil's z reach)"
                                  : "box smaller than the ghost width");
  }
  g.ecx = g.bcx + 2 * g.gcx;
  g.ey = g.by + 2 * g.gy;
  g.ez = g.bz + 2 * g.gz;
  g.E = (long long)g.ecx * g.ey * g.ez;
  g.images = 1;
  g.zimg = slab ? 0 : 1; // a slab's z ghost layers come from its neighbours (mb_sim_halo_*)
  g.Lx = cfg->cells_x * cfg->lattice_const;
  g.Ly = cfg->cells_y * cfg->lattice_const;
  g.Lz = cfg->cells_z * cfg->lattice_const;
  g.iLx = 1.0 / g.Lx;
  g.iLy = 1.0 / g.Ly;
  g.iLz = 1.0 / g.Lz;
  if (2 * g.E > 0x3fffffffLL) {
    pot_free(s->pot);
    delete s;
    return fail(MB_ERR_ARG, "lattice too large for 32-bit indices");
  }
  s->ext_x = 2 * g.ecx;
  s->ext_y = g.ey;
  s->ext_z = g.ez;
  s->n_ext = 2 * g.E;
  s->n_box = 2LL * g.bcx * g.by * g.bz;
  rc = stencil_generate(cfg->lattice_const, reach, s->ext_x, s->ext_y, even, odd, MB_MAX_STENCIL, &n, &rx, &ry, &rz);
  const int par[2] = {0, 1};
  int n_near = 0;
  if (rc == MB_OK && pot->n_types == 1)
    rc = stencil_sort_by_distance(cfg->lattice_const, cfg->cutoff, s->ext_x, s->ext_y, even, odd, n, &n_near);
  if (rc == MB_OK) rc = stencil_from_linear(even, n, odd, n, s->ext_x, s->ext_y, g, par, &s->st);
  s->st.n_near = n_near;
  if (rc != MB_OK) {
    pot_free(s->pot);
    delete s;
    return rc;
  }
  s->st_even.assign(even, even + n);
  s->st_odd.assign(odd, odd + n);

  auto cleanup = [&](int code) {
    mb_sim_destroy(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(MB_ERR_CUDA, "stream creation failed"));
  for (auto &e : s->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return cleanup(fail(MB_ERR_CUDA, "event creation failed"));
  const size_t ne = (size_t)s->n_ext;
  const bool fp64 = cfg->precision == MB_PREC_FP64;
  for (int b = 0; b < 2; b++)
    for (int c = 0; c < 3; c++)
      if ((rc = dalloc(s, (void **)&s->pos[b][c], ne * sizeof(double))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->code, (ne + 3) & ~(size_t)3)) != MB_OK) return cleanup(rc);
  if (fp64) {
    if ((rc = dalloc(s, (void **)&s->df, ne * sizeof(double))) != MB_OK) return cleanup(rc);
    if ((rc = dalloc(s, (void **)&s->rho, ne * sizeof(double))) != MB_OK) return cleanup(rc);
    if (outer_masks_on() &&
        (rc = dalloc(s, (void **)&s->outer, (size_t)items_per_box(s->g) * sizeof(uint2))) != MB_OK)
      return cleanup(rc);
  }
  for (int c = 0; c < 3; c++) {
    if ((rc = dalloc(s, (void **)&s->v[c], ne * sizeof(double))) != MB_OK) return cleanup(rc);
    if ((rc = dalloc(s, (void **)&s->f[c], ne * sizeof(double))) != MB_OK) return cleanup(rc);
  }
  if ((rc = dalloc(s, (void **)&s->id, (size_t)s->n_box * sizeof(int64_t))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->epart, sizeof(double) * energy_partials_needed())) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->bad, sizeof(int))) != MB_OK) return cleanup(rc);
  s->cap_itl = cfg->max_interstitials;
  const int ci = std::max(1, s->cap_itl);
  for (int b = 0; b < 2; b++)
    for (int c = 0; c < 3; c++)
      if ((rc = dalloc(s, (void **)&s->ipos[b][c], ci * sizeof(double))) != MB_OK) return cleanup(rc);
  for (int c = 0; c < 3; c++) {
    if ((rc = dalloc(s, (void **)&s->iv[c], ci * sizeof(double))) != MB_OK) return cleanup(rc);
    if ((rc = dalloc(s, (void **)&s->ifr[c], ci * sizeof(double))) != MB_OK) return cleanup(rc);
  }
  if ((rc = dalloc(s, (void **)&s->irho, ci * sizeof(double))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->idf, ci * sizeof(double))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->itype, ci)) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->iid, ci * sizeof(int64_t))) != MB_OK) return cleanup(rc);
  // sites in reach of one interstitial: the window sphere holds < 2 * (4/3 pi R^3) / (a0^3 / 2)
  const double R = reach;
  const int per = (int)(2.0 * 4.18879 * R * R * R / (0.5 * pow(cfg->lattice_const, 3))) + 64;
  s->cap_flag = std::max(1, s->cap_itl * per);
  if ((rc = dalloc(s, (void **)&s->flag_list, (size_t)s->cap_flag * sizeof(int))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->flag_count, 2 * sizeof(int))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->d_nitl, sizeof(int))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->d_cand, MB_CAND_CAP * sizeof(long long))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->d_cand_n, sizeof(int))) != MB_OK) return cleanup(rc);
  if ((rc = dalloc(s, (void **)&s->d_conv_counters, 4 * sizeof(long long))) != MB_OK) return cleanup(rc);
  if (cudaMemsetAsync(s->d_nitl, 0, sizeof(int), s->stream) != cudaSuccess ||
      cudaMemsetAsync(s->d_cand_n, 0, sizeof(int), s->stream) != cudaSuccess ||
      cudaMemsetAsync(s->d_conv_counters, 0, 4 * sizeof(long long), s->stream) != cudaSuccess)
    return cleanup(fail(MB_ERR_CUDA, "memset failed"));
  if (cudaMemsetAsync(s->flag_count, 0, 2 * sizeof(int), s->stream) != cudaSuccess)
    return cleanup(fail(MB_ERR_CUDA, "memset failed"));
  // vacant everywhere until an upload
  if (cudaMemsetAsync(s->code, 0xff, (ne + 3) & ~(size_t)3, s->stream) != cudaSuccess)
    return cleanup(fail(MB_ERR_CUDA, "memset failed"));
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return cleanup(fail(MB_ERR_CUDA, "sync failed"));
  *out = s;
  return MB_OK;
}

int mb_sim_destroy(mb_sim *s) {
  if (!s) return MB_OK;
  if (s->ens) {
    mb_ensemble_destroy(s->ens);
    delete s;
    return MB_OK;
  }
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  if (s->ens) mb_ensemble_destroy(s->ens);
  void *ptrs[] = {s->code, s->df, s->rho, s->outer, s->id, s->epart, s->eout, s->stage, s->bad, s->irho, s->idf, s->itype,
                  s->iid, s->flag_list, s->flag_count, s->d_nitl, s->d_cand, s->d_cand_n, s->d_conv_counters};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (int b = 0; b < 2; b++)
    for (int c = 0; c < 3; c++) {
      if (s->pos[b][c]) cudaFree(s->pos[b][c]);
      if (s->ipos[b][c]) cudaFree(s->ipos[b][c]);
    }
  for (int c = 0; c < 3; c++) {
    if (s->v[c]) cudaFree(s->v[c]);
    if (s->f[c]) cudaFree(s->f[c]);
    if (s->iv[c]) cudaFree(s->iv[c]);
    if (s->ifr[c]) cudaFree(s->ifr[c]);
  }
  for (auto &e : s->ev)
    if (e) cudaEventDestroy(e);
  for (int k = 0; k < MB_SLAB_MAX; k++) {
    if (s->ev_in[k]) cudaEventDestroy(s->ev_in[k]);
    if (s->ev_out[k]) cudaEventDestroy(s->ev_out[k]);
  }
  if (s->ev_go) cudaEventDestroy(s->ev_go);
  if (s->cp_in) {
    cudaStreamSynchronize(s->cp_in);
    cudaStreamDestroy(s->cp_in);
  }
  if (s->cp_out) {
    cudaStreamSynchronize(s->cp_out);
    cudaStreamDestroy(s->cp_out);
  }
  if (s->stream) cudaStreamDestroy(s->stream);
  pot_free(s->pot);
  delete s;
  return MB_OK;
}

static int ensure_stage(mb_sim *s, size_t n) {
  if (s->stage_n >= n) return MB_OK;
  if (s->stage) {
    cudaFree(s->stage);
    s->device_bytes -= s->stage_n * sizeof(mb_atom_element);
  }
  s->stage = nullptr;
  s->stage_n = 0;
  MB_TRY(dalloc(s, (void **)&s->stage, n * sizeof(mb_atom_element)));
  s->stage_n = n;
  return MB_OK;
}

static int upload_itl(mb_sim *s, const mb_atom_element *itl, int32_t n_itl, int with_f) {
  if (n_itl < 0 || n_itl > s->cap_itl) return fail(MB_ERR_ARG, "n_itl exceeds max_interstitials");
  if (n_itl > 0 && !itl) return fail(MB_ERR_ARG, "null interstitial array");
  s->n_itl = n_itl;
  MB_CUDA(cudaStreamSynchronize(s->stream));
  MB_CUDA(cudaMemcpy(s->d_nitl, &s->n_itl, sizeof(int), cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemsetAsync(s->d_cand_n, 0, sizeof(int), s->stream));
  if (n_itl == 0) return MB_OK;
  std::vector<double> buf((size_t)n_itl);
  std::vector<int8_t> t((size_t)n_itl);
  std::vector<int64_t> ids((size_t)n_itl);
  for (int k = 0; k < n_itl; k++) {
    if (itl[k].type < 0 || itl[k].type >= pot_dev(s->pot).n_types)
      return fail(MB_ERR_ARG, "interstitial type without a potential table");
    t[k] = (int8_t)itl[k].type;
    ids[k] = itl[k].id;
  }
  auto put = [&](double *dst, auto get) -> int {
    for (int k = 0; k < n_itl; k++) buf[k] = get(itl[k]);
    MB_CUDA(cudaMemcpyAsync(dst, buf.data(), sizeof(double) * n_itl, cudaMemcpyHostToDevice, s->stream));
    MB_CUDA(cudaStreamSynchronize(s->stream));
    return MB_OK;
  };
  for (int c = 0; c < 3; c++) {
    MB_TRY(put(s->ipos[s->cur][c], [c](const mb_atom_element &a) { return a.x[c]; }));
    MB_TRY(put(s->iv[c], [c](const mb_atom_element &a) { return a.v[c]; }));
    MB_TRY(put(s->ifr[c], [c, with_f](const mb_atom_element &a) { return with_f ? a.f[c] : 0.0; }));
  }
  MB_CUDA(cudaMemcpyAsync(s->itype, t.data(), n_itl, cudaMemcpyHostToDevice, s->stream));
  MB_CUDA(cudaMemcpyAsync(s->iid, ids.data(), sizeof(int64_t) * n_itl, cudaMemcpyHostToDevice, s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  return MB_OK;
}

static int download_itl(mb_sim *s, mb_atom_element *itl, int which, int unkick) {
  const int n = s->n_itl;
  if (n == 0) return MB_OK;
  std::vector<double> x[3], v[3], f[3], rho(n), df(n);
  std::vector<int8_t> t(n);
  std::vector<int64_t> ids(n);
  for (int c = 0; c < 3; c++) {
    x[c].resize(n);
    v[c].resize(n);
    f[c].resize(n);
    MB_CUDA(cudaMemcpyAsync(x[c].data(), s->ipos[which][c], sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    MB_CUDA(cudaMemcpyAsync(v[c].data(), s->iv[c], sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    MB_CUDA(cudaMemcpyAsync(f[c].data(), s->ifr[c], sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  }
  MB_CUDA(cudaMemcpyAsync(rho.data(), s->irho, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  MB_CUDA(cudaMemcpyAsync(df.data(), s->idf, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  MB_CUDA(cudaMemcpyAsync(t.data(), s->itype, n, cudaMemcpyDeviceToHost, s->stream));
  MB_CUDA(cudaMemcpyAsync(ids.data(), s->iid, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  const double h = sim_params(s, 0, 0).h;
  for (int k = 0; k < n; k++) {
    mb_atom_element &a = itl[k];
    a.id = ids[k];
    a.type = t[k];
    a.pad_ = 0;
    for (int c = 0; c < 3; c++) {
      a.x[c] = x[c][k];
      a.f[c] = f[c][k];
      a.v[c] = v[c][k] - (unkick ? h * f[c][k] : 0.0);
    }
    a.rho = rho[k];
    a.df = df[k];
  }
  return MB_OK;
}

int mb_sim_upload(mb_sim *s, const mb_atom_element *box_atoms, const mb_atom_element *itl, int32_t n_itl) {
  MB_RANGE("mb_sim_upload");
  if (s && s->ens) return box_atoms ? mixed_upload(s, box_atoms, itl, n_itl) : fail(MB_ERR_ARG, "null argument");
  if (!s || !box_atoms) return fail(MB_ERR_ARG, "null argument");
  MB_CUDA(cudaStreamSynchronize(s->stream));
  drop_graph(s);
  s->cur = 0;
  s->primed = false;
  s->step = 0;
  s->n_e = 0;
  s->e_steps.clear();
  s->outer_ok = false;
  MB_TRY(ensure_stage(s, (size_t)s->n_box));
  MB_CUDA(cudaMemcpyAsync(s->stage, box_atoms, (size_t)s->n_box * sizeof(mb_atom_element), cudaMemcpyHostToDevice,
                          s->stream));
  MB_CUDA(cudaMemsetAsync(s->bad, 0, sizeof(int), s->stream));
  // clear interstitial flags and any ghost codes, then load both position buffers
  MB_CUDA(cudaMemsetAsync(s->code, 0xff, ((size_t)s->n_ext + 3) & ~(size_t)3, s->stream));
  MB_CUDA(cudaMemsetAsync(s->flag_count, 0, 2 * sizeof(int), s->stream));
  for (int b = 0; b < 2; b++) {
    Lattice64 L = sim_lattice(s, b);
    MB_TRY(launch_unpack_box_ids(s->g, s->stage, L, 1, s->bad, s->id, pot_dev(s->pot).n_types, s->stream));
    MB_TRY(launch_images64(s->g, L, 1, s->stream));
  }
  int bad = 0;
  MB_CUDA(cudaMemcpyAsync(&bad, s->bad, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  if (bad) return fail(MB_ERR_ARG, "atom type without a potential table");
  MB_TRY(upload_itl(s, itl, n_itl, 1));
  return MB_OK;
}

int mb_sim_download(mb_sim *s, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t *n_itl) {
  MB_RANGE("mb_sim_download");
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_download(s->ens, s->slot, box_atoms, itl, n_itl);
  }
  if (!s || !box_atoms) return fail(MB_ERR_ARG, "null argument");
  MB_TRY(ensure_stage(s, (size_t)s->n_box));
  const int which = s->primed ? (s->cur ^ 1) : s->cur;
  const int unkick = s->primed ? 1 : 0;
  Lattice64 L = sim_lattice(s, s->cur);
  MB_TRY(launch_pack_box_ids(s->g, s->stage, L, s->pos[which][0], s->pos[which][1], s->pos[which][2],
                             sim_params(s, 0, 0).h, unkick, s->id, s->stream));
  MB_CUDA(cudaMemcpyAsync(box_atoms, s->stage, (size_t)s->n_box * sizeof(mb_atom_element), cudaMemcpyDeviceToHost,
                          s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  MB_CUDA(cudaMemcpy(&s->n_itl, s->d_nitl, sizeof(int), cudaMemcpyDeviceToHost));
  if (n_itl) *n_itl = s->n_itl;
  if (itl) MB_TRY(download_itl(s, itl, which, unkick));
  return MB_OK;
}

int mb_sim_run(mb_sim *s, int32_t nsteps, int32_t energy_every) {
  MB_RANGE("mb_sim_run");
  if (s && s->slab) return fail(MB_ERR_UNSUPPORTED, "a z-slab steps through mb_sim_slab_phase with halo exchanges");
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    MB_TRY(mb_ensemble_clear_energies(s->ens, s->slot));
    return mb_ensemble_run(s->ens, nsteps, energy_every);
  }
  if (!s || nsteps < 0) return fail(MB_ERR_ARG, "bad arguments");
  if (energy_every < 0) return fail(MB_ERR_ARG, "energy_every < 0");
  s->n_e = 0;
  s->e_steps.clear();
  if (!s->primed) {
    // step 0 energy sample rides on the priming pass
    MB_TRY(prime(s, energy_every > 0 ? 1 : 0));
  }
  MB_TRY(run_steps(s, nsteps, energy_every));
  return MB_OK;
}

int mb_sim_sync(mb_sim *s) {
  if (s && s->ens) return mb_ensemble_sync(s->ens);
  if (!s) return fail(MB_ERR_ARG, "null sim");
  MB_CUDA(cudaStreamSynchronize(s->stream));
  MB_CUDA(cudaMemcpy(&s->n_itl, s->d_nitl, sizeof(int), cudaMemcpyDeviceToHost));
  int fc[2] = {0, 0};
  if (itl_active(s)) {
    MB_CUDA(cudaMemcpy(fc, s->flag_count, sizeof(fc), cudaMemcpyDeviceToHost));
    if (fc[1]) return fail(MB_ERR_ARG, "interstitial flag list overflowed");
  }
  return MB_OK;
}

int mb_sim_energies(mb_sim *s, double *out, int32_t cap, int32_t *n) {
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_energies(s->ens, s->slot, out, cap, n);
  }
  if (!s || !n) return fail(MB_ERR_ARG, "null argument");
  MB_CUDA(cudaStreamSynchronize(s->stream));
  const int m = std::min(cap, s->n_e);
  std::vector<double> buf((size_t)2 * std::max(1, s->n_e));
  if (s->n_e > 0)
    MB_CUDA(cudaMemcpy(buf.data(), s->eout, sizeof(double) * 2 * s->n_e, cudaMemcpyDeviceToHost));
  for (int k = 0; k < m && out; k++) {
    out[3 * k + 0] = (double)s->e_steps[k];
    out[3 * k + 1] = buf[2 * k];
    out[3 * k + 2] = buf[2 * k + 1];
  }
  *n = s->n_e;
  return MB_OK;
}

int mb_sim_time_steps(mb_sim *s, int32_t nsteps, float *ms) {
  if (s && s->slab) return fail(MB_ERR_UNSUPPORTED, "a z-slab steps through mb_sim_slab_phase with halo exchanges");
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_time(s->ens, nsteps, ms);
  }
  if (!s || !ms || nsteps <= 0) return fail(MB_ERR_ARG, "bad arguments");
  if (!s->primed) MB_TRY(prime(s, 0));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  MB_CUDA(cudaEventRecord(s->ev[0], s->stream));
  MB_TRY(run_steps(s, nsteps, 0));
  MB_CUDA(cudaEventRecord(s->ev[1], s->stream));
  MB_CUDA(cudaEventSynchronize(s->ev[1]));
  MB_CUDA(cudaEventElapsedTime(ms, s->ev[0], s->ev[1]));
  return MB_OK;
}

int mb_sim_kernel_times(mb_sim *s, float *rho_ms, float *force_ms) {
  if (s && s->slab) return fail(MB_ERR_UNSUPPORTED, "a z-slab steps through mb_sim_slab_phase with halo exchanges");
  if (s && s->ens) { // split kernels: each pass timed; persistent kernel: the whole step
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_kernel_times(s->ens, rho_ms, force_ms, nullptr);
  }
  if (!s) return fail(MB_ERR_ARG, "null sim");
  if (!s->primed) MB_TRY(prime(s, 0));
  const int reps = 4;
  float tr = 0, tf = 0;
  for (int k = 0; k < reps; k++) {
    MB_TRY(step64(s, 0, 1, 1, 1));
    s->cur ^= 1;
    s->step++;
    MB_CUDA(cudaEventSynchronize(s->ev[7]));
    float a = 0, b = 0;
    MB_CUDA(cudaEventElapsedTime(&a, s->ev[4], s->ev[5]));
    MB_CUDA(cudaEventElapsedTime(&b, s->ev[6], s->ev[7]));
    tr += a;
    tf += b;
  }
  s->last_rho_ms = tr / reps;
  s->last_force_ms = tf / reps;
  if (rho_ms) *rho_ms = s->last_rho_ms;
  if (force_ms) *force_ms = s->last_force_ms;
  return MB_OK;
}

// Box layers [zb[k], zb[k+1]) of the host-buffer step's z-slabs.  Each slab is at
// least as thick as anything a site or an interstitial reaches (the stencil's ghost
// layers; interstitial windows of cutoff + skin, flagged sites within them), so the
// work on slab k reads only slabs k-1, k, k+1 (periodic in z).  An interstitial in box
// layer Z reaches sites of layers Z - ceil(R / a0) .. Z + ceil(R / a0) (sublattice-1
// sites sit half a layer up), hence ceil(R / a0) + 1 layers with a layer to spare.
// More slabs shorten the tail of the step (the periodic ring closes after the last
// slab arrives: two density and four force slabs and their copies out).  Automatic: as
// many as fit, with at least 4 MiB of records per slab (a slab's copy then outlasts the
// launches of its passes).  Fewer than 4 slabs: one piece.
static int slab_plan(const mb_sim *s, int *zb) {
  const int bz = s->g.bz;
  const double reach = s->cfg.cutoff + s->cfg.stencil_skin;
  const int rz = std::max(s->g.gz, (int)ceil(reach / s->cfg.lattice_const) + 1);
  const long long by_bytes = (long long)s->n_box * (long long)sizeof(mb_atom_element) / (4LL << 20);
  const int want = s->host_slabs > 0 ? s->host_slabs : (int)std::min<long long>(by_bytes, MB_SLAB_MAX);
  int n = std::min(std::min(want, bz / std::max(rz, 1)), MB_SLAB_MAX);
  if (n < 4) n = 1;
  for (int k = 0; k <= n; k++) zb[k] = (int)((long long)k * bz / n);
  return n;
}

static int ensure_pipe(mb_sim *s) {
  if (s->cp_in) return MB_OK;
  MB_CUDA(cudaStreamCreateWithFlags(&s->cp_in, cudaStreamNonBlocking));
  MB_CUDA(cudaStreamCreateWithFlags(&s->cp_out, cudaStreamNonBlocking));
  MB_CUDA(cudaEventCreateWithFlags(&s->ev_go, cudaEventDisableTiming));
  for (int k = 0; k < MB_SLAB_MAX; k++) {
    MB_CUDA(cudaEventCreateWithFlags(&s->ev_in[k], cudaEventDisableTiming));
    MB_CUDA(cudaEventCreateWithFlags(&s->ev_out[k], cudaEventDisableTiming));
  }
  return MB_OK;
}

// One step on the whole box: records in, then every pass, then records out.
static int step_host_whole(mb_sim *s, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t n_itl) {
  MB_CUDA(cudaMemcpyAsync(s->stage, box_atoms, (size_t)s->n_box * sizeof(mb_atom_element), cudaMemcpyHostToDevice,
                          s->stream));
  Lattice64 L = sim_lattice(s, 0);
  L.nx = L.ny = L.nz = nullptr;
  MB_TRY(launch_unpack_box_ids(s->g, s->stage, L, 1, s->bad, s->id, pot_dev(s->pot).n_types, s->stream));
  MB_TRY(launch_images64(s->g, L, 1, s->stream));
  MB_TRY(upload_itl(s, itl, n_itl, 1));
  Itl64 I = sim_itl(s, 0);
  StepParams sp = sim_params(s, 1, 0);
  MB_TRY(launch_kick_drift64(s->g, L, I, sp, s->stream));
  const DevPot &P = pot_dev(s->pot);
  const int it = s->n_itl > 0;
  if (it) MB_TRY(launch_itl_mark64(s->g, L, I, s->stream));
  MB_TRY(launch_rho64(s->g, s->st, P, L, sp.rc2, nullptr, 0, it, s->stream, 0, -1, s->outer));
  if (it) MB_TRY(launch_itl_rho64(s->g, s->st, P, L, I, sp.rc2, nullptr, 0, s->stream));
  MB_TRY(launch_force64(s->g, s->st, P, L, sp, nullptr, 0, it, s->stream, 0, -1, s->outer));
  if (it) MB_TRY(launch_itl_force64(s->g, s->st, P, L, I, sp, nullptr, 0, s->stream));
  MB_TRY(launch_pack_box_ids(s->g, s->stage, L, L.px, L.py, L.pz, sp.h, 0, s->id, s->stream));
  MB_CUDA(cudaMemcpyAsync(box_atoms, s->stage, (size_t)s->n_box * sizeof(mb_atom_element), cudaMemcpyDeviceToHost,
                          s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  if (itl) MB_TRY(download_itl(s, itl, 0, 0));
  return MB_OK;
}

// The same step streamed by z-slabs.  The records of slab k come in on cp_in; once
// they are there the compute stream unpacks, drifts and flags slab k, computes
// rho / df of slab k-1 >= 1 (its neighbours k-2..k have drifted) and the forces of
// slab k-2 >= 2 (the df of k-3..k-1 is there), whose records then go out on cp_out
// while later slabs still come in.  The periodic ring closes at the end: rho / df of
// slabs n-1 and 0, then the forces of slabs n-2, n-1, 0 and 1.
// Every site is computed by the same kernels in the same order as in one piece, so the
// records are bitwise the same.
static int step_host_slabs(mb_sim *s, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t n_itl, int n,
                           const int *zb) {
  MB_TRY(ensure_pipe(s));
  const Geom &g = s->g;
  const long long layer = 2LL * g.bcx * g.by; // records per box layer
  const size_t rec = sizeof(mb_atom_element);
  cudaStream_t cs = s->stream;
  // the slabs start travelling at once (the stage is free: the last call ended synced) ...
  MB_CUDA(cudaEventRecord(s->ev_go, cs));
  MB_CUDA(cudaStreamWaitEvent(s->cp_in, s->ev_go, 0));
  for (int k = 0; k < n; k++) {
    const long long r0 = zb[k] * layer, r1 = zb[k + 1] * layer;
    MB_CUDA(cudaMemcpyAsync(s->stage + r0, box_atoms + r0, (size_t)(r1 - r0) * rec, cudaMemcpyHostToDevice, s->cp_in));
    MB_CUDA(cudaEventRecord(s->ev_in[k], s->cp_in));
  }
  // ... while the interstitials go up on the compute stream
  const int urc = upload_itl(s, itl, n_itl, 1);
  if (urc != MB_OK) {
    cudaStreamSynchronize(s->cp_in); // the caller's records are not in use after a refusal
    return urc;
  }
  Lattice64 L = sim_lattice(s, 0);
  L.nx = L.ny = L.nz = nullptr;
  Itl64 I = sim_itl(s, 0);
  const StepParams sp = sim_params(s, 1, 0);
  const DevPot &P = pot_dev(s->pot);
  const int it = s->n_itl > 0;
  auto start = [&]() -> int { // interstitials drift first (their forces came with them); no site is flagged yet
    if (!it) return MB_OK;
    MB_CUDA(cudaMemsetAsync(s->flag_count, 0, sizeof(int), cs));
    return launch_kick_drift64(g, L, I, sp, cs, 0, 0, 1);
  };
  auto arrive = [&](int k) -> int {
    MB_CUDA(cudaStreamWaitEvent(cs, s->ev_in[k], 0));
    MB_TRY(launch_unpack_box_ids(g, s->stage, L, 1, s->bad, s->id, P.n_types, cs, zb[k], zb[k + 1]));
    MB_TRY(launch_images64(g, L, 1, cs, zb[k], zb[k + 1]));
    MB_TRY(launch_kick_drift64(g, L, I, sp, cs, zb[k], zb[k + 1], 0));
    if (it) MB_TRY(launch_itl_mark_slab64(g, L, I, zb[k], zb[k + 1], cs));
    return MB_OK;
  };
  auto rho = [&](int k) -> int {
    MB_TRY(launch_rho64(g, s->st, P, L, sp.rc2, nullptr, 0, it, cs, zb[k], zb[k + 1], s->outer));
    if (it) MB_TRY(launch_itl_rho64(g, s->st, P, L, I, sp.rc2, nullptr, 0, cs, zb[k], zb[k + 1]));
    return MB_OK;
  };
  auto force = [&](int k) -> int {
    MB_TRY(launch_force64(g, s->st, P, L, sp, nullptr, 0, it, cs, zb[k], zb[k + 1], s->outer));
    if (it) MB_TRY(launch_itl_force64(g, s->st, P, L, I, sp, nullptr, 0, cs, zb[k], zb[k + 1]));
    MB_TRY(launch_pack_box_ids(g, s->stage, L, L.px, L.py, L.pz, sp.h, 0, s->id, cs, zb[k], zb[k + 1]));
    MB_CUDA(cudaEventRecord(s->ev_out[k], cs));
    MB_CUDA(cudaStreamWaitEvent(s->cp_out, s->ev_out[k], 0));
    const long long r0 = zb[k] * layer, r1 = zb[k + 1] * layer;
    MB_CUDA(cudaMemcpyAsync(box_atoms + r0, s->stage + r0, (size_t)(r1 - r0) * rec, cudaMemcpyDeviceToHost, s->cp_out));
    return MB_OK;
  };
  int rc = start();
  for (int k = 0; k < n && rc == MB_OK; k++) {
    rc = arrive(k);
    if (rc == MB_OK && k >= 2) rc = rho(k - 1);
    if (rc == MB_OK && k >= 4) rc = force(k - 2);
  }
  const int tail_rho[2] = {n - 1, 0}, tail_force[4] = {n - 2, n - 1, 0, 1};
  for (int q = 0; q < 2 && rc == MB_OK; q++) rc = rho(tail_rho[q]);
  for (int q = 0; q < 4 && rc == MB_OK; q++) rc = force(tail_force[q]);
  // drain all three streams, also after an error, so the caller's buffer is not in use
  const cudaError_t e0 = cudaStreamSynchronize(s->cp_in), e1 = cudaStreamSynchronize(cs),
                    e2 = cudaStreamSynchronize(s->cp_out);
  MB_TRY(rc);
  MB_CUDA(e0);
  MB_CUDA(e1);
  MB_CUDA(e2);
  if (itl) MB_TRY(download_itl(s, itl, 0, 0));
  return MB_OK;
}

int mb_sim_step_host(mb_sim *s, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t n_itl) {
  MB_RANGE("mb_sim_step_host");
  if (s && s->slab) return fail(MB_ERR_UNSUPPORTED, "a z-slab steps through mb_sim_slab_phase with halo exchanges");
  if (!s || !box_atoms) return fail(MB_ERR_ARG, "null argument");
  if (s->cfg.precision != MB_PREC_FP64) return fail(MB_ERR_UNSUPPORTED, "host-buffer steps run the FP64 path");
  MB_TRY(ensure_stage(s, (size_t)s->n_box));
  drop_graph(s);
  s->cur = 0;
  s->primed = false;
  int zb[MB_SLAB_MAX + 1];
  const int n = slab_plan(s, zb);
  if (n == 1) return step_host_whole(s, box_atoms, itl, n_itl);
  return step_host_slabs(s, box_atoms, itl, n_itl, n, zb);
}

int mb_sim_set_host_slabs(mb_sim *s, int32_t n_slabs) {
  if (!s) return fail(MB_ERR_ARG, "null sim");
  if (n_slabs < 0 || n_slabs > MB_SLAB_MAX) return fail(MB_ERR_ARG, "n_slabs must lie in [0, 32]");
  s->host_slabs = n_slabs;
  return MB_OK;
}

int mb_sim_host_slabs(mb_sim *s, int32_t *n_slabs) {
  if (!s || !n_slabs) return fail(MB_ERR_ARG, "null argument");
  int zb[MB_SLAB_MAX + 1];
  *n_slabs = slab_plan(s, zb);
  return MB_OK;
}

int mb_sim_set_conversion(mb_sim *s, double convert_distance, double recombine_distance) {
  if (s && s->slab) return fail(MB_ERR_UNSUPPORTED, "a z-slab steps through mb_sim_slab_phase with halo exchanges");
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_set_conversion(s->ens, convert_distance, recombine_distance);
  }
  if (!s) return fail(MB_ERR_ARG, "null sim");
  if (convert_distance < 0 || recombine_distance < 0 || (convert_distance > 0 && recombine_distance >= convert_distance))
    return fail(MB_ERR_ARG, "need 0 <= recombine_distance < convert_distance (0 switches conversion off)");
  if (convert_distance > 0 && s->cap_itl > MB_CONV_ITL_MAX)
    return fail(MB_ERR_ARG, "max_interstitials above the conversion limit (65536)");
  if (convert_distance > 0 && s->cap_itl < 1) return fail(MB_ERR_ARG, "conversion needs max_interstitials > 0");
  MB_CUDA(cudaStreamSynchronize(s->stream));
  s->conv_d = convert_distance;
  s->rec_d = convert_distance > 0 ? recombine_distance : 0.0;
  drop_graph(s); // the captured step pair changes
  return MB_OK;
}

int mb_sim_conversion_stats(mb_sim *s, int64_t *counters, int32_t *n_itl) {
  if (s && s->ens) {
    MB_TRY(mixed_need_slot(s));
    return mb_ensemble_conversion_stats(s->ens, s->slot, counters, n_itl);
  }
  if (!s) return fail(MB_ERR_ARG, "null sim");
  MB_CUDA(cudaStreamSynchronize(s->stream));
  long long c[4] = {0, 0, 0, 0};
  MB_CUDA(cudaMemcpy(c, s->d_conv_counters, sizeof(c), cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(&s->n_itl, s->d_nitl, sizeof(int), cudaMemcpyDeviceToHost));
  if (counters)
    for (int k = 0; k < 4; k++) counters[k] = (int64_t)c[k];
  if (n_itl) *n_itl = s->n_itl;
  return MB_OK;
}

int mb_sim_info(mb_sim *s, int64_t *n_sites, int64_t *n_stencil, int64_t *device_bytes) {
  if (s && s->ens) {
    int32_t ns = 0;
    MB_TRY(mb_ensemble_info(s->ens, n_sites, nullptr, device_bytes, &ns));
    if (n_stencil) *n_stencil = -1;
    return MB_OK;
  }
  if (!s) return fail(MB_ERR_ARG, "null sim");
  if (n_sites) *n_sites = s->n_box;
  if (n_stencil) *n_stencil = s->st.n;
  if (device_bytes) *device_bytes = (int64_t)s->device_bytes;
  return MB_OK;
}

int mb_sim_set_graphs(mb_sim *s, int enable) {
  if (s && s->ens) return mb_ensemble_set_graphs(s->ens, enable);
  if (!s) return fail(MB_ERR_ARG, "null sim");
  s->use_graphs = enable != 0;
  if (!s->use_graphs) drop_graph(s);
  return MB_OK;
}

// ------------------------------------------------------------------ z-slab runs
// One rank's share of a lattice decomposed into z-slabs (mb_sim_create_slab): the host
// moves ghost layers between neighbouring slabs around each pass.

int mb_sim_halo_bytes(mb_sim *s, int32_t what, int64_t *bytes) {
  if (!s || !bytes || s->ens) return fail(MB_ERR_ARG, "bad arguments");
  if (what < 1 || what > 3) return fail(MB_ERR_ARG, "halo field must be 1 (positions), 2 (df) or 3 (site codes)");
  const long long n = halo_sites(s->g);
  *bytes = (int64_t)(what == 1 ? 3 * n * (long long)sizeof(double) : what == 2 ? n * (long long)sizeof(double) : n);
  return MB_OK;
}

static int halo(mb_sim *s, int what, int pack, int side, void *buf, double z_shift) {
  if (!s || s->ens) return fail(MB_ERR_ARG, "bad arguments");
  if (!s->slab) return fail(MB_ERR_STATE, "halo layers belong to z-slab runs (mb_sim_create_slab)");
  double *c0 = what == 1 ? s->pos[s->cur][0] : s->df, *c1 = s->pos[s->cur][1], *c2 = s->pos[s->cur][2];
  if (!pack && what != 2) s->outer_ok = false; // new ghost positions or codes: the masks are stale
  MB_TRY(launch_halo(s->g, what, pack, side, c0, c1, c2, s->code, buf, z_shift, s->stream));
  MB_CUDA(cudaStreamSynchronize(s->stream));
  return MB_OK;
}

int mb_sim_halo_pack(mb_sim *s, int32_t what, int32_t side, void *device_buf) {
  return halo(s, what, 1, side, device_buf, 0.0);
}

int mb_sim_halo_unpack(mb_sim *s, int32_t what, int32_t side, const void *device_buf, double z_shift) {
  return halo(s, what, 0, side, const_cast<void *>(device_buf), z_shift);
}

int mb_sim_slab_phase(mb_sim *s, int32_t phase, int32_t energy) {
  MB_RANGE("mb_sim_slab_phase");
  if (!s || s->ens) return fail(MB_ERR_ARG, "bad arguments");
  if (phase != 0 && phase != 1) return fail(MB_ERR_ARG, "phase must be 0 (rho) or 1 (force + integration)");
  if (s->n_itl > 0 || s->conv_d > 0.0)
    return fail(MB_ERR_UNSUPPORTED, "phase-wise steps take lattices without interstitials");
  const DevPot &P = pot_dev(s->pot);
  Lattice64 L = sim_lattice(s, s->cur);
  double *ep = energy ? s->epart : nullptr;
  if (phase == 0) {
    if (energy) MB_CUDA(cudaMemsetAsync(s->epart, 0, sizeof(double) * energy_partials_needed(), s->stream));
    MB_TRY(launch_rho64(s->g, s->st, P, L, s->cfg.cutoff * s->cfg.cutoff, ep, energy, 0, s->stream, 0, -1,
                        s->outer));
    s->outer_ok = true;
    return MB_OK;
  }
  // forces at pos[cur], closing kick of the previous step (once primed), drift to pos[cur ^ 1]
  const StepParams sp = sim_params(s, s->primed ? 1 : 0, 1);
  MB_TRY(launch_force64(s->g, s->st, P, L, sp, ep, energy, 0, s->stream, 0, -1, s->outer_ok ? s->outer : nullptr));
  s->outer_ok = false;
  const long long n = s->primed ? s->step + 1 : 0;
  s->step = n;
  if (energy) {
    if (s->n_e == 0) s->e_steps.clear();
    MB_TRY(record_energy(s));
  }
  s->primed = true;
  s->cur ^= 1;
  return MB_OK;
}

int mb_sim_clear_energies(mb_sim *s) {
  if (!s) return fail(MB_ERR_ARG, "null sim");
  if (s->ens) return mb_ensemble_clear_energies(s->ens, s->slot);
  s->n_e = 0;
  s->e_steps.clear();
  return MB_OK;
}

} // extern "C"
