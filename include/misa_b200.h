/*
 * misa_b200 — B200-native EAM hot path for MISA-MD, C ABI.
 *
 * Three layers, all plain C types (no torch, no C++ in the signatures):
 *   1. Drop-in hooks: the plugin interface of misa-md-hip, with the reference's
 *      argument meaning and synchronous semantics, on the host's own ghost-extended
 *      AoS lattice array.
 *   2. Device-resident molecular dynamics: one lattice (plus interstitials) kept in
 *      HBM, ghost wrap done on the device, velocity-Verlet fused into the force
 *      pass, FP64 or mixed precision.
 *   3. Ensembles and serving: many independent lattices advanced together.
 *
 * Every entry point returns MB_OK (0) or a positive MB_ERR_* code; the message of
 * the last failure on the calling thread is in mb_last_error().  Nothing aborts.
 */
#ifndef MISA_B200_H
#define MISA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MB_OK 0
#define MB_ERR_ARG 1         /* bad argument or size */
#define MB_ERR_CUDA 2        /* CUDA runtime failure (message has the CUDA error) */
#define MB_ERR_STATE 3       /* call order: e.g. a pass before mb_pot_init */
#define MB_ERR_NOMEM 4       /* device allocation refused / over budget */
#define MB_ERR_TIMEOUT 5     /* a bounded device wait gave up */
#define MB_ERR_UNSUPPORTED 6 /* valid request this build does not implement */

#define MB_PREC_FP64 0  /* plain FP64: the drop-in path */
#define MB_PREC_MIXED 1 /* FP32 pair/spline work, compensated FP32 sums, FP64 state */

const char *mb_last_error(void);
const char *mb_version(void);

/* ------------------------------------------------------------------ types */

/* One lattice site, byte-compatible with misa-md-hip's _cuAtomElement
 * (src/kernel_types.h:40-48), itself a copy of MISA-MD's AtomElement: 104 bytes.
 * type < 0 marks a vacancy / invalid site. */
typedef struct mb_atom_element {
  int64_t id;
  int32_t type;
  int32_t pad_;
  double x[3];
  double v[3];
  double f[3];
  double rho;
  double df;
} mb_atom_element;

/* Lattice geometry, field-for-field the reference's _hipDeviceDomain
 * (src/kernel_types.h:51-64).  Sizes along x are in the doubled BCC index
 * (two sites per unit cell).  ghost = local_low - ghost_low, ext = box + 2 ghost,
 * box_index_start = global index of the first box site. */
typedef struct mb_device_domain {
  int32_t ghost_size_x, ghost_size_y, ghost_size_z;
  int32_t box_size_x, box_size_y, box_size_z;
  int32_t ext_size_x, ext_size_y, ext_size_z;
  int32_t pad_;
  int64_t box_index_start_x, box_index_start_y, box_index_start_z;
} mb_device_domain;

/* Tabulated EAM potential.  Knots are uniformly spaced from 0: r_k = k*dr,
 * rho_k = k*drho.  f: n_types rows of nr electron-density values f_t(r);
 * F: n_types rows of nrho embedding energies F_t(rho); phi: n_types*(n_types+1)/2
 * rows of nr pair energies phi_ab(r) (not r*phi), packed upper triangle
 * (0,0),(0,1),..,(0,n-1),(1,1),...  Beyond the last rho knot F continues
 * linearly with its end slope; pairs at r >= cutoff do not interact. */
typedef struct mb_eam_tables {
  int32_t n_types; /* 1..3 (the reference uploads types {0,1,2}) */
  int32_t nr;
  int32_t nrho;
  int32_t pad_;
  double dr;
  double drho;
  double cutoff;
  const double *f;
  const double *F;
  const double *phi;
} mb_eam_tables;

/* ------------------------------------------------- 1. drop-in plugin hooks */

/* hip_env_init (src/hip_arch_acc_imp.cpp:28-40): select the device. */
int mb_env_init(int device);
/* hip_env_clean (src/hip_arch_acc_imp.cpp:42-45): frees every device buffer the
 * hooks own (the reference leaks them). */
int mb_env_clean(void);
/* hip_domain_init (src/hip_arch_acc_imp.cpp:47-99), taking the converted domain
 * instead of comm::BccDomain.  ghost_size_x and box_size_x must be even. */
int mb_domain_init(const mb_device_domain *domain);
/* hip_nei_offset_init (src/hip_arch_acc_imp.cpp:101-144): the even / odd x-parity
 * neighbour stencils as linear offsets into the ghost-extended array (what
 * NeighbourIndex::nei_even_offsets / nei_odd_offsets hold). */
int mb_nei_offset_init(const int64_t *nei_even, size_t n_even, const int64_t *nei_odd, size_t n_odd);
/* hip_pot_init (src/hip_arch_acc_imp.cpp:146-150): build and upload the spline tables. */
int mb_pot_init(const mb_eam_tables *tables);
/* hip_eam_rho_calc (src/hip_arch_acc_imp.cpp:163-181): for every box site with
 * type >= 0, rho = sum over the stencil of f_{t_j}(r) for r < cutoff, then
 * df = F'(rho) (fused, full-neighbour build).  atoms is the host's
 * ghost-extended AoS array (ghosts already filled); rho and df are written back.
 * The array travels in z-slabs (mb_cli_set_batches): later slabs come in while earlier
 * ones are computed and their box rows go back; page-locked memory from
 * mb_create_atoms_mem lets those copies run asynchronously. */
int mb_eam_rho_calc(mb_atom_element *atoms, double cutoff_radius);
/* hip_eam_df_calc (src/hip_arch_acc_imp.cpp:183-205): a no-op in the full-neighbour
 * build, exactly like the reference (df is produced by the rho pass); in
 * half-neighbour mode df = F'(rho) for every box site with type >= 0 (calDf). */
int mb_eam_df_calc(mb_atom_element *atoms, double cutoff_radius);
/* hip_eam_force_calc (src/hip_arch_acc_imp.cpp:207-225): f = sum del * fpair over
 * the stencil, overwriting f of every box site with type >= 0 (needs df of the
 * ghost sites filled by the host).  Streamed in z-slabs like mb_eam_rho_calc. */
int mb_eam_force_calc(mb_atom_element *atoms, double cutoff_radius);
/* The rho pass of mb_eam_rho_calc (same inputs, same results) for hosts that cannot
 * let a plugin allocate device memory: a process whose device memory is already
 * handed out by its own pool allocator, or a timestep loop that must not take the
 * implicit synchronisation cudaMalloc / cudaFree can cause.  No counterpart in the
 * reference.  It calls no cudaMalloc / cudaFree: its scratch is a fixed 16 MiB
 * device array inside the library, present on every GPU that loads the library
 * until exit, which limits the ghost-extended lattice to about 115,000 sites
 * (145 bytes each); larger lattices are refused with MB_ERR_ARG.  The calling
 * thread's current device must be the one mb_env_init selected (else MB_ERR_STATE).
 * The first call on a device (and the first after mb_env_clean) looks the array's
 * device address up (cudaGetSymbolAddress) and should come before any stream
 * capture.  A record whose type has no potential table is refused with MB_ERR_ARG
 * before anything is written back.  All calls share the array and it keeps the
 * previous call's contents; calls that overlap on the GPU race. */
int mb_eam_rho_calc_noalloc(mb_atom_element *atoms, double cutoff_radius);
/* The calDf kernel of the half-neighbour build (src/kernels/hip_kernels.hip.cpp:21-40):
 * df = F'(rho) for every box site with type >= 0. */
int mb_eam_df_from_rho(mb_atom_element *atoms);
/* The reference's USE_NEWTONS_THIRD_LOW build (src/md_hip_config.h:12), chosen at
 * run time: with enable != 0, mb_nei_offset_init takes half stencils (one offset of
 * each opposite pair, MISA-MD's nei_half_*_offsets, src/hip_arch_acc_imp.cpp:118-130)
 * and every pair (i, i + o) with i a box site is evaluated once, both atoms receiving
 * their share (src/kernels/kernel_pairs.hpp:21-32, 39-60).  mb_eam_rho_calc then
 * rewrites rho of every ext record, box and ghost, with the shares it received (no
 * df); the host adds ghost shares to their owners and calls mb_eam_df_calc;
 * mb_eam_force_calc rewrites f of every ext record the same way.  Switching modes
 * drops the stencil: mb_nei_offset_init must follow.  Default: full neighbour. */
int mb_set_half_neighbour(int enable);
/* hip_create_atoms_mem (src/mem.cpp:14-23): page-locked host allocation of
 * size_x*size_y*size_z elements; *allocated = 1 when this library allocated. */
int mb_create_atoms_mem(void **atoms, size_t data_type_size, int64_t size_x, int64_t size_y, int64_t size_z,
                        int *allocated);
/* hip_release_atoms_mem (src/mem.cpp:25-32). */
int mb_release_atoms_mem(void *atoms, int *released);
/* hip_cli_options / hip_cli_options_parse (src/cli.cpp:16-27): the -b/--batches
 * value, the number of z-slabs the rho and force hooks stream the array in (as the
 * reference's double buffer does, src/double-buffer/double_buffer.cpp:12-47, with the
 * layers split evenly; at most 32).  1, the reference's default, lets the library
 * choose (slabs of at least 4 MiB of records, at most 16).  The results are bitwise the
 * same for every count. */
int mb_cli_set_batches(unsigned int batches);
unsigned int mb_cli_batches(void);

/* Neighbour stencils in the reference's linear form for an ext array of
 * ext_x x ext_y: every BCC site whose ideal offset is shorter than reach (the role
 * MISA-MD's NeighbourIndex plays for hip_nei_offset_init).  Ordered dz, dy, dx
 * ascending; *n receives the length of each. */
int mb_stencil_linear(double lattice_const, double reach, int ext_x, int ext_y, int64_t *even, int64_t *odd, int cap,
                      int *n);
/* The 7 spline coefficients per knot the device tables are built from
 * (y, s, c2, c3, s/dx, 2 c2/dx, 3 c3/dx), for checking the table build on the host. */
int mb_spline_coeffs(const double *y, int n, double dx, double *coef7);

/* Timing of the last hook call (CUDA events): kernel_ms is the span of its device work
 * (from the first conversion to the last), copy_ms the rest of the call, i.e. the
 * copies that did not overlap it. */
int mb_hook_last_timing(float *kernel_ms, float *copy_ms);


/* ---------------------------------------- 2. device-resident simulation */

typedef struct mb_sim mb_sim;

typedef struct mb_sim_config {
  int32_t cells_x, cells_y, cells_z; /* unit cells; box = (2*cells_x, cells_y, cells_z) sites */
  int32_t precision;                 /* MB_PREC_FP64 or MB_PREC_MIXED */
  double lattice_const;              /* A */
  double mass;                       /* amu */
  double dt;                         /* fs */
  double cutoff;                     /* A */
  double stencil_skin;               /* A: stencil = sites with ideal distance < cutoff + skin */
  int32_t max_interstitials;
  int32_t pad_;
} mb_sim_config;

/* Per-site records in "box order": index ((z*box_y)+y)*box_x + x with x doubled. */
int mb_sim_create(const mb_sim_config *cfg, const mb_eam_tables *pot, mb_sim **out);
int mb_sim_destroy(mb_sim *sim);
/* Load positions, velocities and types (box order) plus an interstitial list.
 * Forces are (re)computed on the next run. */
int mb_sim_upload(mb_sim *sim, const mb_atom_element *box_atoms, const mb_atom_element *itl, int32_t n_itl);
/* Synchronised state at the current step: x, v, f, rho, df of every site. */
int mb_sim_download(mb_sim *sim, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t *n_itl);
/* Advance nsteps velocity-Verlet steps on the device (asynchronous on the sim's
 * stream).  energy_every > 0 records (pe, ke) every that many steps. */
int mb_sim_run(mb_sim *sim, int32_t nsteps, int32_t energy_every);
int mb_sim_sync(mb_sim *sim);
/* Energies recorded by the last run: n pairs (step, pe, ke) in eV. */
int mb_sim_energies(mb_sim *sim, double *out_step_pe_ke, int32_t cap, int32_t *n);
/* Device time of nsteps (CUDA events around the sim's stream), after one
 * untimed priming pass if needed. */
int mb_sim_time_steps(mb_sim *sim, int32_t nsteps, float *ms);
/* One full step through host buffers: upload box_atoms (x, v, f, type),
 * one velocity-Verlet step on the device, write x, v, f, rho, df back.  The
 * e2e form of the hot path: host<->device copies are part of every call.  The box is
 * streamed in z-slabs (box_atoms in box order, z slowest): records of later slabs
 * travel in while earlier ones are computed and earlier results travel out.  The
 * records are bitwise the same whatever the slab count.  Replaces the reference's
 * RhoDoubleBufferImp / ForceDoubleBufferImp streaming
 * (src/double-buffer/double_buffer.cpp:12-47) for a whole step. */
int mb_sim_step_host(mb_sim *sim, mb_atom_element *box_atoms, mb_atom_element *itl, int32_t n_itl);
/* Slabs of mb_sim_step_host: 0 automatic (as many as fit, at most 32, with at least
 * 4 MiB of records each), 1 one piece, else at most that many.  Each slab is at least
 * as thick as the stencil and the interstitial windows reach; fewer than 4 such slabs
 * run in one piece.  mb_sim_host_slabs reports the count a step takes. */
int mb_sim_set_host_slabs(mb_sim *sim, int32_t n_slabs);
int mb_sim_host_slabs(mb_sim *sim, int32_t *n_slabs);
/* Mean device milliseconds of the rho and force launches over 4 extra steps the sim
 * takes (mixed precision: as mb_ensemble_kernel_times). */
int mb_sim_kernel_times(mb_sim *sim, float *rho_ms, float *force_ms);
int mb_sim_info(mb_sim *sim, int64_t *n_sites, int64_t *n_stencil, int64_t *device_bytes);
/* CUDA graph capture of the steady-state step (on by default). */
int mb_sim_set_graphs(mb_sim *sim, int enable);
/* Lattice <-> interstitial bookkeeping of the device-resident run.  MISA-MD keeps atoms
 * that have left their lattice site in its interstitial list (the plugin only sees
 * type < 0 for such sites, src/kernels/kernel_itl.hpp:44).  With convert_distance > 0,
 * after every step an atom farther than convert_distance (A) from its lattice site
 * joins the end of the interstitial list (sites in box order) and its site becomes
 * vacant; then an interstitial (list order) within recombine_distance of a vacant site
 * takes that site and leaves the list.  0 switches it off (the default).  Needs
 * 0 < max_interstitials <= 65536; a conversion beyond the capacity is refused (the atom
 * stays on its site) and counted. */
int mb_sim_set_conversion(mb_sim *sim, double convert_distance, double recombine_distance);
/* counters[4]: conversions, recombinations, conversions refused (list full), candidates
 * dropped (more than 2048 in one step); *n_itl: the current interstitial count. */
int mb_sim_conversion_stats(mb_sim *sim, int64_t *counters, int32_t *n_itl);

/* ---- one lattice decomposed into z-slabs over several ranks (one GPU each)
 * The MISA-MD host splits its lattice over MPI ranks and exchanges ghost layers between
 * the passes: positions before rho, df before force (src/double-buffer/
 * rho_double_buffer_imp.h:38-39 holds "the lattice atoms array in current MPI process
 * (including ghost regions)").  A slab sim is one rank's share: box cells
 * [z_first, z_first + z_count) of cfg->cells_z (x and y whole and periodic), FP64, no
 * interstitials.  Its x / y ghost images are written on the device as in a whole-lattice
 * sim; its z ghost layers come from the neighbouring slabs through device buffers the
 * host moves (NCCL send / recv, a peer copy, ...):
 *   after mb_sim_upload: codes (what 3) once; every step: positions (what 1), phase 0
 *   (rho, df), df (what 2), phase 1 (forces, velocity-Verlet, drift).
 * z_count must be at least the ghost width (2 cells for cutoff + skin = 6.3 A at
 * a0 = 2.855 A).  Whole-lattice stepping (mb_sim_run, ...) is refused on a slab. */
int mb_sim_create_slab(const mb_sim_config *cfg, const mb_eam_tables *pot, int32_t z_first, int32_t z_count,
                       mb_sim **out);
/* Bytes of one halo message of field `what`: 1 positions (3 doubles per site), 2 df
 * (1 double), 3 site codes (1 byte); gz whole ext planes of both sublattices. */
int mb_sim_halo_bytes(mb_sim *sim, int32_t what, int64_t *bytes);
/* Copy this slab's lowest (side 0, for the slab below) or highest (side 1, for the slab
 * above) gz box layers of field `what` into device_buf; returns when the copy is done. */
int mb_sim_halo_pack(mb_sim *sim, int32_t what, int32_t side, void *device_buf);
/* Fill the bottom (side 0, from the slab below) or top (side 1, from the slab above) gz
 * ghost layers from device_buf; z positions get z_shift added (+-L_z across the periodic
 * wrap between the last and the first slab).  Returns when the copy is done. */
int mb_sim_halo_unpack(mb_sim *sim, int32_t what, int32_t side, const void *device_buf, double z_shift);
/* Half of a timestep of an FP64 sim without interstitials (a slab, or a whole lattice):
 * phase 0 rho / df at the current positions, phase 1 forces, the closing half kick of
 * the previous step and the drift to the next positions.  energy != 0 on both phases of
 * a step records this sim's (pe, ke) share of it (mb_sim_energies).  Asynchronous. */
int mb_sim_slab_phase(mb_sim *sim, int32_t phase, int32_t energy);
/* Drop the recorded energies (they otherwise accumulate across phase-wise steps). */
int mb_sim_clear_energies(mb_sim *sim);

/* ------------------------------------------- 3. ensembles and serving */

/* Many independent periodic lattices (slots) advanced together, one persistent
 * kernel launch per timestep, in mixed precision (FP32 pair and spline work with
 * compensated FP32 sums; FP64 positions, velocities, integration and energies).
 * Slots can be added and removed between launches while others are mid-run; each
 * has its own step target, after which it stops advancing. */
typedef struct mb_ensemble mb_ensemble;

typedef struct mb_ensemble_config {
  double lattice_const, mass, dt, cutoff, stencil_skin;
  int64_t hbm_budget_bytes; /* 0: unlimited; otherwise mb_ensemble_add refuses beyond it */
  int32_t max_lattices;     /* 0: unlimited */
  int32_t pad_;
} mb_ensemble_config;

typedef struct mb_lattice_spec {
  int32_t cells_x, cells_y, cells_z;
  int32_t max_interstitials;
} mb_lattice_spec;

int mb_ensemble_create(const mb_ensemble_config *cfg, const mb_eam_tables *pot, mb_ensemble **out);
int mb_ensemble_destroy(mb_ensemble *e);
/* Device bytes one lattice of this spec occupies (what admission budgets with). */
int mb_ensemble_lattice_bytes(const mb_lattice_spec *spec, int64_t *bytes);
/* Upload a lattice (box-order records + interstitials) into a free slot; it will
 * advance `steps` steps.  MB_ERR_NOMEM when the HBM budget or slot count is full. */
int mb_ensemble_add(mb_ensemble *e, const mb_lattice_spec *spec, const mb_atom_element *box,
                    const mb_atom_element *itl, int32_t n_itl, int64_t steps, int32_t *slot);
int mb_ensemble_remove(mb_ensemble *e, int32_t slot);
int mb_ensemble_set_steps(mb_ensemble *e, int32_t slot, int64_t steps_target);
/* Up to max_launches launches, stopping early once every slot reached its target;
 * energies are recorded at every multiple of energy_every of each slot's step. */
int mb_ensemble_advance(mb_ensemble *e, int32_t max_launches, int32_t energy_every, int32_t *launches);
/* Every slot advances nsteps more steps. */
int mb_ensemble_run(mb_ensemble *e, int32_t nsteps, int32_t energy_every);
int mb_ensemble_sync(mb_ensemble *e);
int mb_ensemble_download(mb_ensemble *e, int32_t slot, mb_atom_element *box, mb_atom_element *itl, int32_t *n_itl);
int mb_ensemble_status(mb_ensemble *e, int32_t slot, int64_t *steps_done, int64_t *steps_target,
                       int64_t *device_bytes);
/* Recorded (step, pe, ke) triples of a slot, eV. */
int mb_ensemble_energies(mb_ensemble *e, int32_t slot, double *out, int32_t cap, int32_t *n);
int mb_ensemble_clear_energies(mb_ensemble *e, int32_t slot);
/* Device time of nsteps launches of every slot (CUDA events; advances the state). */
int mb_ensemble_time(mb_ensemble *e, int32_t nsteps, float *ms);
/* Tile-shape policy: -1 picks a shape per lattice from its size, 0..3 one shape for all. */
int mb_ensemble_set_policy(mb_ensemble *e, int32_t policy);
/* Times the candidate kernels for `steps` launches each on a snapshot of the slots
 * (state restored afterwards) and keeps the fastest: the split kernels (reported as
 * *policy = 4; skipped when their stencil does not apply or mode 1 was set) and every
 * tile policy -1..3 of the persistent kernel (skipped when mode 2 was set). */
int mb_ensemble_autotune(mb_ensemble *e, int32_t steps, int32_t *policy, float *best_ms);
int mb_ensemble_info(mb_ensemble *e, int64_t *n_sites, int64_t *n_tiles, int64_t *device_bytes, int32_t *n_slots);
int mb_ensemble_set_graphs(mb_ensemble *e, int enable);
/* Polls a grid barrier of the persistent step kernel (mode 1) makes before it gives up:
 * the launch then ends early, the state of the lattices in flight is undefined, and the
 * next sync / download returns MB_ERR_TIMEOUT (the barrier is reset, so later launches run
 * normally).  Negative restores the default (2^25 polls, ~64 ns apart); 0 gives up at the
 * first poll that finds the barrier still closed.  For failure-detection tests. */
int mb_ensemble_set_wait_limit(mb_ensemble *e, int64_t barrier_polls);
/* Kernel structure: 0 (default) runs the separate density and force kernels ("split":
 * one CUDA graph of up to 8 launches per step, every lattice in each launch) whenever
 * their built-in BCC stencil applies and the persistent one-launch-per-step tile
 * kernel otherwise; 1 always the persistent kernel; 2 always split (MB_ERR_UNSUPPORTED
 * at the next launch if it cannot apply). */
int mb_ensemble_set_mode(mb_ensemble *e, int32_t mode);
/* mb_sim_set_conversion for every lattice of the ensemble (each within its own
 * max_interstitials). */
int mb_ensemble_set_conversion(mb_ensemble *e, double convert_distance, double recombine_distance);
int mb_ensemble_conversion_stats(mb_ensemble *e, int32_t slot, int64_t *counters, int32_t *n_itl);
/* Device time of one step's kernels, averaged over 4 extra steps every lattice takes
 * (CUDA events on the ensemble's stream): split kernels report the density pass in
 * *rho_ms and the force + integration pass in *force_ms; the persistent kernel
 * reports 0 and its whole launch.  *kernels_per_step: launches one step issues. */
int mb_ensemble_kernel_times(mb_ensemble *e, float *rho_ms, float *force_ms, int32_t *kernels_per_step);

#ifdef __cplusplus
}
#endif
#endif
