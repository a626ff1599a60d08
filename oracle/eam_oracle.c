/*
 * CPU oracle for the MISA-MD EAM lattice hot path — TEST INFRASTRUCTURE ONLY.
 * Only tests/, the smoke check and the bench's CPU-baseline leg may load this
 * library, and only as the checker (or the timed CPU baseline).
 *
 * PARITY UNPINNED against the reference itself (it cannot be built here: HIP,
 * MPI, the MISA-MD host and hip-potential v0.2.0 are all absent, and it ships no
 * golden vectors).  Pinned by analytic known answers, finite differences and
 * NVE energy conservation in tests/test_oracle.py.
 *
 * What is restated, and from where (paths inside misa-md-hip):
 *   - site index map        src/kernels/kernel_itl.hpp:21-26 (x fastest, ghost offset)
 *   - parity-chosen stencil src/kernels/kernel_itl.hpp:82,86 ((x + box_index_start_x) % 2)
 *   - skip type < 0         src/kernels/kernel_itl.hpp:44, :53-55
 *   - cutoff test on r^2    src/kernels/kernel_pairs.hpp:23, :42
 *   - rho from the NEIGHBOUR's type, df fused after rho
 *                           src/kernels/kernel_pairs.hpp:26, src/kernels/kernel_itl.hpp:99-103
 *   - force = del * fpair(t_i, t_j, r^2, df_i, df_j), overwrite
 *                           src/kernels/kernel_pairs.hpp:48-54, src/kernels/kernel_itl.hpp:93-97
 *   - df pass               src/kernels/hip_kernels.hip.cpp:21-40
 * The spline arithmetic lives in hip-potential v0.2.0 (hip_pot::hipChargeDensity,
 * hipDEmbedEnergy, hipToForce; not vendored).  It is restated from the published
 * tabulated-EAM scheme used by MISA-MD's potential tables (the setfl/funcfl
 * cubic of XMD / LAMMPS pair_eam): knot slopes from a 4th-order central
 * difference (one-sided / 2nd-order at the two ends), a cubic Hermite piece per
 * interval, the index clamped to the last interval and the local coordinate to
 * [0,1]; beyond the rho table the embedding energy is extended linearly with the
 * end slope.  The ghost fill, interstitial terms, velocity-Verlet and energies are
 * the MISA-MD host's job (not vendored) and are restated from the EAM definition
 *   E = sum_i F_{t_i}(rho_i) + 1/2 sum_{i!=j} phi_{t_i t_j}(r_ij),
 *   rho_i = sum_{j!=i} f_{t_j}(r_ij).
 */
#include "eam_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_FTM2V 9.64853321233e-3 /* (eV/A)/amu -> A/fs^2 */
#define ORC_MVV2E (1.0 / ORC_FTM2V) /* amu A^2/fs^2 -> eV */

struct orc_pot {
  int n_types, nr, nrho;
  double dr, drho, rdr, rdrho, cutoff;
  double *f;   /* [n_types][nr][7] */
  double *F;   /* [n_types][nrho][7] */
  double *phi; /* [n_pairs][nr][7] */
};

/* Knot slopes and per-interval cubic.  coef7 per knot m:
 *   [0] y_m, [1] s_m, [2] c2_m, [3] c3_m   value(p) = ((c3 p + c2) p + s) p + y
 *   [4] s_m/dx, [5] 2 c2_m/dx, [6] 3 c3_m/dx   d/dx value = ([6] p + [5]) p + [4]
 */
void orc_spline_coeffs(const double *y, int n, double dx, double *c) {
  double *s = (double *)malloc(sizeof(double) * (size_t)n);
  s[0] = y[1] - y[0];
  s[1] = 0.5 * (y[2] - y[0]);
  s[n - 2] = 0.5 * (y[n - 1] - y[n - 3]);
  s[n - 1] = y[n - 1] - y[n - 2];
  for (int m = 2; m <= n - 3; m++) s[m] = ((y[m - 2] - y[m + 2]) + 8.0 * (y[m + 1] - y[m - 1])) / 12.0;
  for (int m = 0; m < n; m++) {
    double c2 = 0.0, c3 = 0.0;
    if (m < n - 1) {
      const double dy = y[m + 1] - y[m];
      c2 = 3.0 * dy - 2.0 * s[m] - s[m + 1];
      c3 = s[m] + s[m + 1] - 2.0 * dy;
    }
    double *k = c + 7 * (size_t)m;
    k[0] = y[m];
    k[1] = s[m];
    k[2] = c2;
    k[3] = c3;
    k[4] = s[m] / dx;
    k[5] = 2.0 * c2 / dx;
    k[6] = 3.0 * c3 / dx;
  }
  free(s);
}

static inline void spl_locate(double x, double rdx, int n, int *m, double *p) {
  const double pp = x * rdx;
  if (!(pp < (double)(n - 1))) {
    *m = n - 2;
    *p = 1.0;
    return;
  }
  int mm = (int)pp;
  if (mm > n - 2) mm = n - 2;
  double q = pp - (double)mm;
  if (q > 1.0) q = 1.0;
  *m = mm;
  *p = q;
}

static inline double spl_value(const double *tab, double x, double rdx, int n) {
  int m;
  double p;
  spl_locate(x, rdx, n, &m, &p);
  const double *k = tab + 7 * (size_t)m;
  return ((k[3] * p + k[2]) * p + k[1]) * p + k[0];
}

static inline double spl_deriv(const double *tab, double x, double rdx, int n) {
  int m;
  double p;
  spl_locate(x, rdx, n, &m, &p);
  const double *k = tab + 7 * (size_t)m;
  return (k[6] * p + k[5]) * p + k[4];
}

static inline int pair_index(int a, int b, int nt) {
  if (a > b) {
    int t = a;
    a = b;
    b = t;
  }
  /* packed upper triangle, row-major: (0,0),(0,1)..(0,nt-1),(1,1).. */
  return a * nt - a * (a - 1) / 2 + (b - a);
}

orc_pot *orc_pot_create(int n_types, int nr, double dr, int nrho, double drho, double cutoff, const double *f,
                        const double *F, const double *phi) {
  if (n_types < 1 || nr < 5 || nrho < 5) return NULL;
  orc_pot *p = (orc_pot *)calloc(1, sizeof(orc_pot));
  p->n_types = n_types;
  p->nr = nr;
  p->nrho = nrho;
  p->dr = dr;
  p->drho = drho;
  p->rdr = 1.0 / dr;
  p->rdrho = 1.0 / drho;
  p->cutoff = cutoff;
  const int np = n_types * (n_types + 1) / 2;
  p->f = (double *)malloc(sizeof(double) * 7 * (size_t)nr * n_types);
  p->F = (double *)malloc(sizeof(double) * 7 * (size_t)nrho * n_types);
  p->phi = (double *)malloc(sizeof(double) * 7 * (size_t)nr * np);
  for (int t = 0; t < n_types; t++) {
    orc_spline_coeffs(f + (size_t)t * nr, nr, dr, p->f + (size_t)t * nr * 7);
    orc_spline_coeffs(F + (size_t)t * nrho, nrho, drho, p->F + (size_t)t * nrho * 7);
  }
  for (int q = 0; q < np; q++) orc_spline_coeffs(phi + (size_t)q * nr, nr, dr, p->phi + (size_t)q * nr * 7);
  return p;
}

void orc_pot_destroy(orc_pot *p) {
  if (!p) return;
  free(p->f);
  free(p->F);
  free(p->phi);
  free(p);
}

const double *orc_pot_table(const orc_pot *p, int which, int a, int b) {
  if (which == 0) return p->f + (size_t)a * p->nr * 7;
  if (which == 1) return p->F + (size_t)a * p->nrho * 7;
  return p->phi + (size_t)pair_index(a, b, p->n_types) * p->nr * 7;
}

double orc_rho_of_r(const orc_pot *p, int t, double r) { return spl_value(orc_pot_table(p, 0, t, 0), r, p->rdr, p->nr); }
double orc_drho_of_r(const orc_pot *p, int t, double r) { return spl_deriv(orc_pot_table(p, 0, t, 0), r, p->rdr, p->nr); }
double orc_phi_of_r(const orc_pot *p, int a, int b, double r) {
  return spl_value(orc_pot_table(p, 2, a, b), r, p->rdr, p->nr);
}
double orc_dphi_of_r(const orc_pot *p, int a, int b, double r) {
  return spl_deriv(orc_pot_table(p, 2, a, b), r, p->rdr, p->nr);
}
double orc_dF_of_rho(const orc_pot *p, int t, double rho) {
  return spl_deriv(orc_pot_table(p, 1, t, 0), rho, p->rdrho, p->nrho);
}
/* Linear continuation past the last knot keeps E consistent with the clamped F'. */
double orc_F_of_rho(const orc_pot *p, int t, double rho) {
  const double *tab = orc_pot_table(p, 1, t, 0);
  const double rho_max = (double)(p->nrho - 1) * p->drho;
  if (rho > rho_max) {
    const double *k = tab + 7 * (size_t)(p->nrho - 1);
    return k[0] + orc_dF_of_rho(p, t, rho) * (rho - rho_max);
  }
  return spl_value(tab, rho, p->rdrho, p->nrho);
}

/* hipToForce restated: -(df_i f'_{t_j} + df_j f'_{t_i} + phi'_{t_i t_j}) / r */
static inline double pair_fpair(const orc_pot *p, int ti, int tj, double r, double dfi, double dfj) {
  const double fj = orc_drho_of_r(p, tj, r);
  const double fi = (ti == tj) ? fj : orc_drho_of_r(p, ti, r);
  const double ph = orc_dphi_of_r(p, ti, tj, r);
  return -(dfi * fj + dfj * fi + ph) / r;
}

/* ---------------------------------------------------------------- stencils */

/* Sites whose ideal BCC offset is in (0, reach), in the doubled-x linear form the
 * reference's kernels walk (src/hip_arch_acc_imp.cpp:101-144 receives them from
 * MISA-MD's NeighbourIndex).  Ideal site (gx, gy, gz) in units of a0:
 * (gx/2, gy + (gx&1)/2, gz + (gx&1)/2).  Ordered by dz, dy, dx ascending. */
int orc_stencil_build(const orc_domain *d, double a0, double reach, int64_t *even, int64_t *odd, int max_n) {
  const int cy = (int)ceil(reach / a0) + 1;
  const int cx = 2 * cy;
  int counts[2] = {0, 0};
  for (int par = 0; par < 2; par++) {
    int64_t *out = par ? odd : even;
    for (int dz = -cy; dz <= cy; dz++)
      for (int dy = -cy; dy <= cy; dy++)
        for (int dx = -cx; dx <= cx; dx++) {
          if (dx == 0 && dy == 0 && dz == 0) continue;
          const int npar = (par + dx) & 1;
          const double ox = 0.5 * dx;
          const double oy = dy + 0.5 * (npar - par);
          const double oz = dz + 0.5 * (npar - par);
          const double dist = a0 * sqrt(ox * ox + oy * oy + oz * oz);
          if (dist >= reach) continue;
          if (counts[par] >= max_n) return -1;
          out[counts[par]++] = ((int64_t)dz * d->ext_size_y + dy) * d->ext_size_x + dx;
        }
  }
  return counts[0] == counts[1] ? counts[0] : -2;
}

/* ------------------------------------------------------- reference passes */

/* Neumaier's compensated summation: *s + *c carries the sum of every x added. */
static inline void neumaier(double *s, double *c, double x) {
  const double t = *s + x;
  if (fabs(*s) >= fabs(x))
    *c += (*s - t) + x;
  else
    *c += (x - t) + *s;
  *s = t;
}

static inline int64_t site_linear(const orc_domain *d, int64_t x, int64_t y, int64_t z) {
  return ((z + d->ghost_size_z) * d->ext_size_y + y + d->ghost_size_y) * d->ext_size_x + x + d->ghost_size_x;
}

void orc_rho_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                  const int64_t *odd, size_t n_odd, double cutoff) {
  const double rc2 = cutoff * cutoff;
#pragma omp parallel for schedule(static) collapse(2)
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        const int64_t i = site_linear(d, x, y, z);
        orc_atom *a = atoms + i;
        if (a->type < 0) continue;
        const int ev = ((x + d->box_index_start_x) % 2) == 0;
        const int64_t *st = ev ? even : odd;
        const size_t ns = ev ? n_even : n_odd;
        double rho = 0.0;
        for (size_t k = 0; k < ns; k++) {
          const orc_atom *b = atoms + i + st[k];
          if (b->type < 0) continue;
          const double dx = a->x[0] - b->x[0], dy = a->x[1] - b->x[1], dz = a->x[2] - b->x[2];
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= rc2) continue;
          rho += orc_rho_of_r(p, b->type, sqrt(d2));
        }
        a->rho = rho;
        a->df = orc_dF_of_rho(p, a->type, rho);
      }
}

void orc_df_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms) {
#pragma omp parallel for schedule(static) collapse(2)
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        orc_atom *a = atoms + site_linear(d, x, y, z);
        if (a->type < 0) continue;
        a->df = orc_dF_of_rho(p, a->type, a->rho);
      }
}

void orc_force_pass(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                    const int64_t *odd, size_t n_odd, double cutoff) {
  const double rc2 = cutoff * cutoff;
#pragma omp parallel for schedule(static) collapse(2)
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        const int64_t i = site_linear(d, x, y, z);
        orc_atom *a = atoms + i;
        if (a->type < 0) continue;
        const int ev = ((x + d->box_index_start_x) % 2) == 0;
        const int64_t *st = ev ? even : odd;
        const size_t ns = ev ? n_even : n_odd;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (size_t k = 0; k < ns; k++) {
          const orc_atom *b = atoms + i + st[k];
          if (b->type < 0) continue;
          const double dx = a->x[0] - b->x[0], dy = a->x[1] - b->x[1], dz = a->x[2] - b->x[2];
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= rc2) continue;
          const double fp = pair_fpair(p, a->type, b->type, sqrt(d2), a->df, b->df);
          fx += dx * fp;
          fy += dy * fp;
          fz += dz * fp;
        }
        a->f[0] = fx;
        a->f[1] = fy;
        a->f[2] = fz;
      }
}

/* ------------------------------------------- half-neighbour (Newton) passes */

/* The reference's USE_NEWTONS_THIRD_LOW build (src/md_hip_config.h:12): the stencil
 * holds one offset of each opposite pair (src/hip_arch_acc_imp.cpp:118-130 takes
 * MISA-MD's nei_half_*_offsets), every pair (i, i + o) with i a box site is evaluated
 * once, and both atoms receive their share (src/kernels/kernel_pairs.hpp:21-32 for
 * rho, :39-60 for force).  Ghost records receive the shares of pairs whose partner is
 * owned elsewhere; the host adds them to their owners.  Every ext record's rho (or f)
 * starts from zero (the reference overwrites the current atom's sum at the end of its
 * loop, kernel_itl.hpp:90-97, which drops shares written to it earlier by other
 * threads; the sum here keeps every share).  Sequential on purpose: the scatter has
 * no races, and the order of the sum is fixed. */
void orc_rho_pass_half(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                       const int64_t *odd, size_t n_odd, double cutoff) {
  const double rc2 = cutoff * cutoff;
  const int64_t n = (int64_t)d->ext_size_x * d->ext_size_y * d->ext_size_z;
  for (int64_t i = 0; i < n; i++) atoms[i].rho = 0.0;
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        const int64_t i = site_linear(d, x, y, z);
        orc_atom *a = atoms + i;
        if (a->type < 0) continue;
        const int ev = ((x + d->box_index_start_x) % 2) == 0;
        const int64_t *st = ev ? even : odd;
        const size_t ns = ev ? n_even : n_odd;
        for (size_t k = 0; k < ns; k++) {
          orc_atom *b = atoms + i + st[k];
          if (b->type < 0) continue;
          const double dx = a->x[0] - b->x[0], dy = a->x[1] - b->x[1], dz = a->x[2] - b->x[2];
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= rc2) continue;
          const double r = sqrt(d2);
          a->rho += orc_rho_of_r(p, b->type, r);
          b->rho += orc_rho_of_r(p, a->type, r);
        }
      }
}

void orc_force_pass_half(const orc_pot *p, const orc_domain *d, orc_atom *atoms, const int64_t *even, size_t n_even,
                         const int64_t *odd, size_t n_odd, double cutoff) {
  const double rc2 = cutoff * cutoff;
  const int64_t n = (int64_t)d->ext_size_x * d->ext_size_y * d->ext_size_z;
  for (int64_t i = 0; i < n; i++) atoms[i].f[0] = atoms[i].f[1] = atoms[i].f[2] = 0.0;
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        const int64_t i = site_linear(d, x, y, z);
        orc_atom *a = atoms + i;
        if (a->type < 0) continue;
        const int ev = ((x + d->box_index_start_x) % 2) == 0;
        const int64_t *st = ev ? even : odd;
        const size_t ns = ev ? n_even : n_odd;
        for (size_t k = 0; k < ns; k++) {
          orc_atom *b = atoms + i + st[k];
          if (b->type < 0) continue;
          const double dx = a->x[0] - b->x[0], dy = a->x[1] - b->x[1], dz = a->x[2] - b->x[2];
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 >= rc2) continue;
          const double fp = pair_fpair(p, a->type, b->type, sqrt(d2), a->df, b->df);
          a->f[0] += dx * fp;
          a->f[1] += dy * fp;
          a->f[2] += dz * fp;
          b->f[0] -= dx * fp;
          b->f[1] -= dy * fp;
          b->f[2] -= dz * fp;
        }
      }
}

/* ------------------------------------------------------------ ghost fill */

static inline int64_t pmod(int64_t a, int64_t b) {
  int64_t r = a % b;
  return r < 0 ? r + b : r;
}

void orc_ghost_fill(const orc_domain *d, orc_atom *atoms, const double box_len[3], int mask) {
  const int64_t bx = d->box_size_x, by = d->box_size_y, bz = d->box_size_z;
#pragma omp parallel for schedule(static)
  for (int64_t ez = 0; ez < d->ext_size_z; ez++)
    for (int64_t ey = 0; ey < d->ext_size_y; ey++)
      for (int64_t ex = 0; ex < d->ext_size_x; ex++) {
        const int64_t x = ex - d->ghost_size_x, y = ey - d->ghost_size_y, z = ez - d->ghost_size_z;
        if (x >= 0 && x < bx && y >= 0 && y < by && z >= 0 && z < bz) continue;
        const int64_t sx = pmod(x, bx), sy = pmod(y, by), sz = pmod(z, bz);
        const orc_atom *s = atoms + site_linear(d, sx, sy, sz);
        orc_atom *g = atoms + (ez * d->ext_size_y + ey) * d->ext_size_x + ex;
        if (mask & 1) {
          g->type = s->type;
          g->id = s->id;
          g->x[0] = s->x[0] + (double)((x - sx) / bx) * box_len[0];
          g->x[1] = s->x[1] + (double)((y - sy) / by) * box_len[1];
          g->x[2] = s->x[2] + (double)((z - sz) / bz) * box_len[2];
        }
        if (mask & 2) g->df = s->df;
      }
}

/* ------------------------------------------------------------- full MD */

static inline double min_image(double dv, double L) { return dv - L * nearbyint(dv / L); }

typedef struct {
  int64_t box_i; /* linear index of the box site */
  double sx, sy, sz; /* periodic image shift */
} win_site;

/* Lattice sites whose ideal position lies within R of point q (periodic). */
static int itl_window(const orc_domain *d, double a0, const double *L, const double q[3], double R, win_site *out,
                      int max_out) {
  const int64_t bx = d->box_size_x, by = d->box_size_y, bz = d->box_size_z;
  const int64_t gx0 = (int64_t)floor((q[0] - R) / (0.5 * a0)), gx1 = (int64_t)ceil((q[0] + R) / (0.5 * a0));
  const int64_t gy0 = (int64_t)floor((q[1] - R) / a0) - 1, gy1 = (int64_t)ceil((q[1] + R) / a0);
  const int64_t gz0 = (int64_t)floor((q[2] - R) / a0) - 1, gz1 = (int64_t)ceil((q[2] + R) / a0);
  int n = 0;
  for (int64_t gz = gz0; gz <= gz1; gz++)
    for (int64_t gy = gy0; gy <= gy1; gy++)
      for (int64_t gx = gx0; gx <= gx1; gx++) {
        const double h = 0.5 * (double)(gx & 1);
        const double X = 0.5 * a0 * (double)gx, Y = a0 * ((double)gy + h), Z = a0 * ((double)gz + h);
        const double ox = X - q[0], oy = Y - q[1], oz = Z - q[2];
        if (ox * ox + oy * oy + oz * oz >= R * R) continue;
        const int64_t sx = pmod(gx, bx), sy = pmod(gy, by), sz = pmod(gz, bz);
        if (n >= max_out) return -1;
        out[n].box_i = site_linear(d, sx, sy, sz);
        out[n].sx = (double)((gx - sx) / bx) * L[0];
        out[n].sy = (double)((gy - sy) / by) * L[1];
        out[n].sz = (double)((gz - sz) / bz) * L[2];
        n++;
      }
  return n;
}

#define ORC_MAX_WIN 4096

void orc_compute_forces(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl,
                        const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                        const orc_md_params *mp, orc_energy *e_out) {
  const double a0 = mp->a0, rc = mp->cutoff, rc2 = rc * rc;
  const double L[3] = {0.5 * a0 * d->box_size_x, a0 * d->box_size_y, a0 * d->box_size_z};
  const double R = rc + mp->itl_margin;
  win_site *win = (win_site *)malloc(sizeof(win_site) * ORC_MAX_WIN);

  orc_ghost_fill(d, atoms, L, 1);
  orc_rho_pass(p, d, atoms, even, n_even, odd, n_odd, rc);

  /* interstitial density: scatter into lattice sites, gather into the interstitial */
  for (int I = 0; I < n_itl; I++) {
    orc_atom *a = itl + I;
    a->rho = 0.0;
  }
  for (int I = 0; I < n_itl; I++) {
    orc_atom *a = itl + I;
    const int nw = itl_window(d, a0, L, a->x, R, win, ORC_MAX_WIN);
    for (int w = 0; w < nw; w++) {
      orc_atom *b = atoms + win[w].box_i;
      if (b->type < 0) continue;
      const double dx = a->x[0] - (b->x[0] + win[w].sx), dy = a->x[1] - (b->x[1] + win[w].sy),
                   dz = a->x[2] - (b->x[2] + win[w].sz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 >= rc2) continue;
      const double r = sqrt(d2);
      a->rho += orc_rho_of_r(p, b->type, r);
      b->rho += orc_rho_of_r(p, a->type, r);
    }
    for (int K = 0; K < n_itl; K++) {
      if (K == I) continue;
      const orc_atom *b = itl + K;
      const double dx = min_image(a->x[0] - b->x[0], L[0]), dy = min_image(a->x[1] - b->x[1], L[1]),
                   dz = min_image(a->x[2] - b->x[2], L[2]);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 >= rc2) continue;
      a->rho += orc_rho_of_r(p, b->type, sqrt(d2));
    }
  }
  if (n_itl > 0) orc_df_pass(p, d, atoms);
  for (int I = 0; I < n_itl; I++) itl[I].df = orc_dF_of_rho(p, itl[I].type, itl[I].rho);
  orc_ghost_fill(d, atoms, L, 2);

  orc_force_pass(p, d, atoms, even, n_even, odd, n_odd, rc);
  for (int I = 0; I < n_itl; I++) itl[I].f[0] = itl[I].f[1] = itl[I].f[2] = 0.0;
  double pe_pair_itl = 0.0;
  for (int I = 0; I < n_itl; I++) {
    orc_atom *a = itl + I;
    const int nw = itl_window(d, a0, L, a->x, R, win, ORC_MAX_WIN);
    for (int w = 0; w < nw; w++) {
      orc_atom *b = atoms + win[w].box_i;
      if (b->type < 0) continue;
      const double dx = a->x[0] - (b->x[0] + win[w].sx), dy = a->x[1] - (b->x[1] + win[w].sy),
                   dz = a->x[2] - (b->x[2] + win[w].sz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 >= rc2) continue;
      const double r = sqrt(d2);
      const double fp = pair_fpair(p, a->type, b->type, r, a->df, b->df);
      a->f[0] += dx * fp;
      a->f[1] += dy * fp;
      a->f[2] += dz * fp;
      b->f[0] -= dx * fp;
      b->f[1] -= dy * fp;
      b->f[2] -= dz * fp;
      pe_pair_itl += orc_phi_of_r(p, a->type, b->type, r);
    }
    for (int K = 0; K < n_itl; K++) {
      if (K == I) continue;
      const orc_atom *b = itl + K;
      const double dx = min_image(a->x[0] - b->x[0], L[0]), dy = min_image(a->x[1] - b->x[1], L[1]),
                   dz = min_image(a->x[2] - b->x[2], L[2]);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 >= rc2) continue;
      const double r = sqrt(d2);
      const double fp = pair_fpair(p, a->type, b->type, r, a->df, b->df);
      a->f[0] += dx * fp;
      a->f[1] += dy * fp;
      a->f[2] += dz * fp;
      pe_pair_itl += 0.5 * orc_phi_of_r(p, a->type, b->type, r);
    }
  }
  free(win);

  if (e_out) {
    /* Energies are sums of millions of terms: each z layer is summed with Neumaier's
     * compensated summation, then the layers in order, so the totals carry about one
     * rounding of the result whatever the thread count (a plain OpenMP reduction leaves
     * ~1e-11 eV/atom of rounding at 4 M atoms). */
    const int64_t nzl = d->box_size_z;
    double *lay = (double *)calloc((size_t)(4 * nzl), sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < nzl; z++) {
      double sp = 0.0, cp = 0.0, sk = 0.0, ck = 0.0;
      for (int64_t y = 0; y < d->box_size_y; y++)
        for (int64_t x = 0; x < d->box_size_x; x++) {
          const int64_t i = site_linear(d, x, y, z);
          const orc_atom *a = atoms + i;
          if (a->type < 0) continue;
          double e = orc_F_of_rho(p, a->type, a->rho);
          const int ev = ((x + d->box_index_start_x) % 2) == 0;
          const int64_t *st = ev ? even : odd;
          const size_t ns = ev ? n_even : n_odd;
          for (size_t k = 0; k < ns; k++) {
            const orc_atom *b = atoms + i + st[k];
            if (b->type < 0) continue;
            const double dx = a->x[0] - b->x[0], dy = a->x[1] - b->x[1], dz = a->x[2] - b->x[2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 >= rc2) continue;
            e += 0.5 * orc_phi_of_r(p, a->type, b->type, sqrt(d2));
          }
          neumaier(&sp, &cp, e);
          neumaier(&sk, &ck, 0.5 * mp->mass * (a->v[0] * a->v[0] + a->v[1] * a->v[1] + a->v[2] * a->v[2]));
        }
      lay[4 * z + 0] = sp;
      lay[4 * z + 1] = cp;
      lay[4 * z + 2] = sk;
      lay[4 * z + 3] = ck;
    }
    double pe = 0.0, cpe = 0.0, ke = 0.0, cke = 0.0;
    for (int64_t z = 0; z < nzl; z++) {
      neumaier(&pe, &cpe, lay[4 * z + 0]);
      neumaier(&pe, &cpe, lay[4 * z + 1]);
      neumaier(&ke, &cke, lay[4 * z + 2]);
      neumaier(&ke, &cke, lay[4 * z + 3]);
    }
    free(lay);
    for (int I = 0; I < n_itl; I++) {
      const orc_atom *a = itl + I;
      neumaier(&pe, &cpe, orc_F_of_rho(p, a->type, a->rho));
      neumaier(&ke, &cke, 0.5 * mp->mass * (a->v[0] * a->v[0] + a->v[1] * a->v[1] + a->v[2] * a->v[2]));
    }
    pe += cpe;
    ke += cke;
    e_out->pe = pe + pe_pair_itl;
    e_out->ke = ke * ORC_MVV2E;
  }
}

/* ------------------------------------- lattice <-> interstitial bookkeeping */

static inline void box_ideal(int64_t x, int64_t y, int64_t z, double a0, double *X, double *Y, double *Z) {
  const double h = 0.5 * (double)(x & 1);
  *X = 0.5 * a0 * (double)x;
  *Y = a0 * ((double)y + h);
  *Z = a0 * ((double)z + h);
}

/* MISA-MD keeps atoms that have left their lattice site in its interstitial list (the
 * plugin only ever sees type < 0 for such sites, src/kernels/kernel_itl.hpp:44).  After a
 * step: every box site whose atom is farther than d_conv from the site's ideal position
 * (box order) moves to the end of the interstitial list and the site becomes vacant;
 * then every interstitial (list order) within d_rec of a vacant site's ideal position
 * takes that site (the first claim wins) and leaves the list, which keeps its order.
 * Returns the new count; counters[0] += conversions, [1] += recombinations, [2] += atoms
 * that could not be converted because the list was full (they stay on their site). */
int orc_convert(const orc_domain *d, double a0, orc_atom *atoms, orc_atom *itl, int n_itl, int cap, double d_conv,
                double d_rec, int64_t *counters) {
  const int64_t bx = d->box_size_x, by = d->box_size_y, bz = d->box_size_z;
  const double c2 = d_conv * d_conv, r2 = d_rec * d_rec;
  for (int64_t z = 0; z < bz; z++)
    for (int64_t y = 0; y < by; y++)
      for (int64_t x = 0; x < bx; x++) {
        orc_atom *a = atoms + site_linear(d, x, y, z);
        if (a->type < 0) continue;
        double X, Y, Z;
        box_ideal(x, y, z, a0, &X, &Y, &Z);
        const double ux = a->x[0] - X, uy = a->x[1] - Y, uz = a->x[2] - Z;
        if (ux * ux + uy * uy + uz * uz <= c2) continue;
        if (n_itl >= cap) {
          counters[2]++;
          continue;
        }
        itl[n_itl++] = *a;
        memset(a, 0, sizeof(*a));
        a->type = -1;
        a->x[0] = X;
        a->x[1] = Y;
        a->x[2] = Z;
        counters[0]++;
      }
  int keep = 0;
  for (int k = 0; k < n_itl; k++) {
    const orc_atom q = itl[k];
    /* nearest ideal site: the nearer of the two simple-cubic sublattices */
    int64_t bs[3] = {0, 0, 0};
    double best = 1e300, bu[3] = {0, 0, 0};
    for (int s = 0; s < 2; s++) {
      const double o = 0.5 * a0 * (double)s;
      const int64_t cx = (int64_t)nearbyint((q.x[0] - o) / a0), cy = (int64_t)nearbyint((q.x[1] - o) / a0),
                    cz = (int64_t)nearbyint((q.x[2] - o) / a0);
      double X, Y, Z;
      box_ideal(2 * cx + s, cy, cz, a0, &X, &Y, &Z);
      const double u[3] = {q.x[0] - X, q.x[1] - Y, q.x[2] - Z};
      const double dd = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
      if (dd < best) {
        best = dd;
        bs[0] = 2 * cx + s;
        bs[1] = cy;
        bs[2] = cz;
        bu[0] = u[0];
        bu[1] = u[1];
        bu[2] = u[2];
      }
    }
    const int64_t xb = pmod(bs[0], bx), yb = pmod(bs[1], by), zb = pmod(bs[2], bz);
    orc_atom *site = atoms + site_linear(d, xb, yb, zb);
    if (best < r2 && site->type < 0) {
      double X, Y, Z;
      box_ideal(xb, yb, zb, a0, &X, &Y, &Z);
      *site = q;
      site->x[0] = X + bu[0];
      site->x[1] = Y + bu[1];
      site->x[2] = Z + bu[2];
      counters[1]++;
      continue;
    }
    itl[keep++] = q;
  }
  return keep;
}

static void half_kick_and_drift(const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl, double h, double dt,
                                int drift) {
#pragma omp parallel for schedule(static) collapse(2)
  for (int64_t z = 0; z < d->box_size_z; z++)
    for (int64_t y = 0; y < d->box_size_y; y++)
      for (int64_t x = 0; x < d->box_size_x; x++) {
        orc_atom *a = atoms + site_linear(d, x, y, z);
        if (a->type < 0) continue;
        for (int c = 0; c < 3; c++) {
          a->v[c] += h * a->f[c];
          if (drift) a->x[c] += dt * a->v[c];
        }
      }
  for (int I = 0; I < n_itl; I++)
    for (int c = 0; c < 3; c++) {
      itl[I].v[c] += h * itl[I].f[c];
      if (drift) itl[I].x[c] += dt * itl[I].v[c];
    }
}

void orc_md_run(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl,
                const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd, const orc_md_params *mp,
                int nsteps, orc_energy *energies) {
  const double h = 0.5 * mp->dt * ORC_FTM2V / mp->mass;
  if (energies) orc_compute_forces(p, d, atoms, itl, n_itl, even, n_even, odd, n_odd, mp, &energies[0]);
  for (int s = 1; s <= nsteps; s++) {
    half_kick_and_drift(d, atoms, itl, n_itl, h, mp->dt, 1);
    orc_energy e;
    orc_compute_forces(p, d, atoms, itl, n_itl, even, n_even, odd, n_odd, mp, &e);
    half_kick_and_drift(d, atoms, itl, n_itl, h, mp->dt, 0);
    if (energies) {
      /* kinetic energy after the closing half kick */
      double ke = 0.0;
      for (int64_t z = 0; z < d->box_size_z; z++)
        for (int64_t y = 0; y < d->box_size_y; y++)
          for (int64_t x = 0; x < d->box_size_x; x++) {
            const orc_atom *a = atoms + site_linear(d, x, y, z);
            if (a->type < 0) continue;
            ke += 0.5 * mp->mass * (a->v[0] * a->v[0] + a->v[1] * a->v[1] + a->v[2] * a->v[2]);
          }
      for (int I = 0; I < n_itl; I++)
        ke += 0.5 * mp->mass * (itl[I].v[0] * itl[I].v[0] + itl[I].v[1] * itl[I].v[1] + itl[I].v[2] * itl[I].v[2]);
      energies[s].pe = e.pe;
      energies[s].ke = ke * ORC_MVV2E;
    }
  }
}

/* nsteps velocity-Verlet steps with the lattice <-> interstitial bookkeeping after
 * every drift, before the forces at the new positions: the order of the device-resident
 * run.  itl holds cap records, the first n_itl of them the list; returns the new count
 * (forces in atoms / itl must be current on entry). */
int orc_md_run_convert(const orc_pot *p, const orc_domain *d, orc_atom *atoms, orc_atom *itl, int n_itl, int cap,
                       const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd,
                       const orc_md_params *mp, int nsteps, double d_conv, double d_rec, int64_t *counters) {
  const double h = 0.5 * mp->dt * ORC_FTM2V / mp->mass;
  for (int s = 1; s <= nsteps; s++) {
    half_kick_and_drift(d, atoms, itl, n_itl, h, mp->dt, 1);
    n_itl = orc_convert(d, mp->a0, atoms, itl, n_itl, cap, d_conv, d_rec, counters);
    orc_compute_forces(p, d, atoms, itl, n_itl, even, n_even, odd, n_odd, mp, NULL);
    half_kick_and_drift(d, atoms, itl, n_itl, h, mp->dt, 0);
  }
  return n_itl;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
