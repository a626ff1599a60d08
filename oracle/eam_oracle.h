/*
 * CPU oracle for the MISA-MD EAM lattice hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C, FP64 restatement of what the misa-md-hip plugin computes
 * (rho -> df = F'(rho) -> force) plus the host-side pieces of MISA-MD that the
 * plugin relies on but that are not vendored (periodic ghost fill, interstitial
 * contributions, velocity-Verlet, energy sums).  Only tests/, the smoke check
 * and the bench's CPU-baseline leg may load it, and only as the checker or the
 * timed CPU baseline — never as a code path of the product.
 *
 * PARITY UNPINNED against the reference itself: the plugin needs HIP, MPI, the
 * MISA-MD host and hip-potential v0.2.0, none of which can be built here, and
 * the reference ships no tests, golden vectors or fixtures.  The oracle is
 * pinned instead by analytic known answers (perfect-lattice density and
 * energy, zero force by symmetry), by finite differences (F = -dE/dx) and by
 * NVE energy conservation (tests/test_oracle.py).
 */
#ifndef MISA_B200_EAM_ORACLE_H
#define MISA_B200_EAM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same bytes as the reference's _cuAtomElement (src/kernel_types.h:40-48). */
typedef struct {
  int64_t id;
  int32_t type;
  int32_t pad_;
  double x[3];
  double v[3];
  double f[3];
  double rho;
  double df;
} orc_atom;

/* Field order of the reference's _hipDeviceDomain (src/kernel_types.h:51-64). */
typedef struct {
  int32_t ghost_size_x, ghost_size_y, ghost_size_z;
  int32_t box_size_x, box_size_y, box_size_z;
  int32_t ext_size_x, ext_size_y, ext_size_z;
  int32_t pad_;
  int64_t box_index_start_x, box_index_start_y, box_index_start_z;
} orc_domain;

typedef struct orc_pot orc_pot;

/* Tabulated-EAM spline of 7 coefficients per knot (see eam_oracle.c). */
void orc_spline_coeffs(const double *y, int n, double dx, double *coef7);

orc_pot *orc_pot_create(int n_types, int nr, double dr, int nrho, double drho, double cutoff, const double *f,
                        const double *F, const double *phi);
void orc_pot_destroy(orc_pot *p);
/* Coefficient table of one function: which 0=f(type a), 1=F(type a), 2=phi(pair a,b). */
const double *orc_pot_table(const orc_pot *p, int which, int a, int b);
double orc_rho_of_r(const orc_pot *p, int type, double r);
double orc_drho_of_r(const orc_pot *p, int type, double r);
double orc_phi_of_r(const orc_pot *p, int ta, int tb, double r);
double orc_dphi_of_r(const orc_pot *p, int ta, int tb, double r);
double orc_F_of_rho(const orc_pot *p, int type, double rho);
double orc_dF_of_rho(const orc_pot *p, int type, double rho);

/* Neighbour-offset stencils in the reference's linear form (even / odd x parity). */
int orc_stencil_build(const orc_domain *d, double a0, double reach, int64_t *even, int64_t *odd, int max_n);

/* Reference hook semantics on a host AoS lattice with ghosts already filled. */
void orc_rho_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                  const int64_t *odd, size_t n_odd, double cutoff);
void orc_df_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms);
void orc_force_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                    const int64_t *odd, size_t n_odd, double cutoff);

/* Half-neighbour (Newton's third law) passes of the reference's USE_NEWTONS_THIRD_LOW
 * build: each pair (i, i + o), i a box site and o from the half stencil, once; rho (f)
 * of every ext record, box and ghost, is the sum of the shares it received. */
void orc_rho_pass_half(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                       const int64_t *odd, size_t n_odd, double cutoff);
void orc_force_pass_half(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                         const int64_t *odd, size_t n_odd, double cutoff);

/* Single-rank periodic ghost fill.  mask bit 0: type+x, bit 1: df. */
void orc_ghost_fill(const orc_domain *d, orc_atom *atoms, const double box_len[3], int mask);

/* Full NVE velocity-Verlet with interstitials. */
typedef struct {
  double a0, mass, dt, cutoff;
  double itl_margin; /* index-window slack around interstitials, in A */
} orc_md_params;

typedef struct {
  double pe, ke; /* eV, whole system */
} orc_energy;

/* Compute rho/df/forces of lattice + interstitials at the current positions
 * (ghosts are refilled first).  Writes rho, df, f into atoms and itl. */
void orc_compute_forces(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl,
                        const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                        const orc_md_params *mp, orc_energy *e_out);

/* nsteps of velocity-Verlet; forces in atoms/itl must be current on entry.
 * energies (optional) receives nsteps+1 entries: before step 1 and after each step. */
void orc_md_run(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl,
                const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd, const orc_md_params *mp,
                int nsteps, orc_energy *energies);

/* Lattice <-> interstitial bookkeeping after a step (see eam_oracle.c): atoms farther
 * than d_conv from their site join the interstitial list (box order), interstitials
 * within d_rec of a vacant site take it (list order).  Returns the new count;
 * counters[3] accumulates conversions, recombinations, refused conversions. */
int orc_convert(const orc_domain *d, double a0, orc_atom *atoms, orc_atom *itl, int n_itl, int cap, double d_conv,
                double d_rec, int64_t *counters);

/* nsteps steps with orc_convert after every drift (before the new forces). */
int orc_md_run_convert(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl, int cap,
                       const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                       const orc_md_params *mp, int nsteps, double d_conv, double d_rec, int64_t *counters);

int orc_num_threads(void);
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
