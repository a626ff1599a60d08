// Potential tables: spline coefficients built on the host, packed for the device.
//
// The spline follows the tabulated-EAM scheme the reference delegates to
// hip-potential v0.2.0 (hip_pot::hipChargeDensity / hipDEmbedEnergy / hipToForce,
// called at src/kernels/kernel_pairs.hpp:26,48 and src/kernels/kernel_itl.hpp:101):
// knot slopes from a 4th-order central difference (one-sided and 2nd-order at the
// ends), one cubic Hermite piece per interval, index clamped to the last interval,
// local coordinate clamped to [0, 1].
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mb_common.cuh"

namespace mb {

struct PotHost {
  DevPot dev;
  void *blob = nullptr; // one device allocation holding every table
};

// c7 per knot: y, s, c2, c3, s/dx, 2 c2/dx, 3 c3/dx
static void knot_pieces(const double *y, int n, double dx, std::vector<double> &c7) {
  std::vector<double> s(n);
  s[0] = y[1] - y[0];
  s[1] = 0.5 * (y[2] - y[0]);
  s[n - 2] = 0.5 * (y[n - 1] - y[n - 3]);
  s[n - 1] = y[n - 1] - y[n - 2];
  for (int m = 2; m <= n - 3; m++) s[m] = ((y[m - 2] - y[m + 2]) + 8.0 * (y[m + 1] - y[m - 1])) / 12.0;
  c7.assign((size_t)n * 7, 0.0);
  for (int m = 0; m < n; m++) {
    double c2 = 0.0, c3 = 0.0;
    if (m < n - 1) {
      const double dy = y[m + 1] - y[m];
      c2 = 3.0 * dy - 2.0 * s[m] - s[m + 1];
      c3 = s[m] + s[m + 1] - 2.0 * dy;
    }
    double *k = &c7[(size_t)m * 7];
    k[0] = y[m];
    k[1] = s[m];
    k[2] = c2;
    k[3] = c3;
    k[4] = s[m] / dx;
    k[5] = 2.0 * c2 / dx;
    k[6] = 3.0 * c3 / dx;
  }
}

// FP64 spline value and derivative at x with the device's locate rule (index clamped to
// the last interval, local coordinate clamped to [0, 1]).
static void spl_eval(const std::vector<double> &c7, int n, double dx, double x, double &v, double &d) {
  const double rdx = 1.0 / dx, pp = x * rdx;
  int m;
  double p;
  if (!(pp < (double)(n - 1))) {
    m = n - 2;
    p = 1.0;
  } else {
    m = std::min((int)pp, n - 2);
    p = std::min(pp - (double)m, 1.0);
  }
  const double *k = &c7[(size_t)m * 7];
  v = ((k[3] * p + k[2]) * p + k[1]) * p + k[0];
  d = (k[6] * p + k[5]) * p + k[4];
}

// Cubic in p through (0, v0), (1/3, v1), (2/3, v2), (1, v3) (forward differences).
static void fit4(const double v[4], double c[4]) {
  const double d1 = v[1] - v[0], d2 = v[2] - 2.0 * v[1] + v[0], d3 = v[3] - 3.0 * v[2] + 3.0 * v[1] - v[0];
  c[0] = v[0];
  c[1] = 3.0 * (d1 - 0.5 * d2 + d3 / 3.0);
  c[2] = 4.5 * (d2 - d3);
  c[3] = 4.5 * d3;
}

// Squared-distance tables of one type (see DevPot::fs32), from the FP64 r-spline.
//  * density: one line per interval, the chord lowered by 2/3 of its midpoint gap (the
//    least-squares line of a locally quadratic function), so that the interpolation
//    error has zero mean and the density and embedding energy carry no bias;
//  * force: knot values of f'(r)/r and phi'(r)/r, linear in between, on a grid three
//    times finer than the density grid (force sums cancel, which amplifies relative
//    error): about 1e-7 of the force for a thermally disordered lattice;
//  * pair energy (energy steps only, read from global memory): a cubic per interval
//    through four exact points.
#ifndef MB_S_RHO_INTERVALS
#define MB_S_RHO_INTERVALS 8000
#endif
#ifndef MB_S_FORCE_INTERVALS
#define MB_S_FORCE_INTERVALS 24000
#endif
struct STables {
  std::vector<float2> fs, ab;
  std::vector<float4> ps;
  double ds_r = 0.0, ds_f = 0.0;
};
static void s_tables(const mb_eam_tables *t, STables &T) {
  std::vector<double> cf, cp;
  knot_pieces(t->f, t->nr, t->dr, cf);
  knot_pieces(t->phi, t->nr, t->dr, cp);
  const double rmax = std::min((double)(t->nr - 1) * t->dr, t->cutoff), smax = rmax * rmax;
  const double rfloor = 1e-3 * t->dr; // A and B stay finite at s = 0 (pairs never get there)
  const int nr_ = MB_S_RHO_INTERVALS, nf = MB_S_FORCE_INTERVALS;
  T.ds_r = smax / nr_;
  T.ds_f = smax / nf;
  auto fval = [&](const std::vector<double> &c, double s) {
    double v, dv;
    spl_eval(c, t->nr, t->dr, sqrt(s), v, dv);
    return v;
  };
  T.fs.resize(nr_);
  for (int j = 0; j < nr_; j++) {
    const double a = fval(cf, j * T.ds_r), b = fval(cf, (j + 1) * T.ds_r), mid = fval(cf, (j + 0.5) * T.ds_r);
    const double lift = (2.0 / 3.0) * (0.5 * (a + b) - mid);
    T.fs[j] = make_float2((float)(a - lift), (float)(b - a));
  }
  T.ab.resize(nf + 1);
  for (int j = 0; j <= nf; j++) {
    const double r = sqrt((double)j * T.ds_f), rr = std::max(r, rfloor);
    double f, fd, ph, phd;
    spl_eval(cf, t->nr, t->dr, r, f, fd);
    spl_eval(cp, t->nr, t->dr, r, ph, phd);
    T.ab[j] = make_float2((float)(fd / rr), (float)(phd / rr));
  }
  T.ps.resize(nf);
  for (int j = 0; j < nf; j++) {
    double v[4], c[4];
    for (int q = 0; q < 4; q++) v[q] = fval(cp, (j + q / 3.0) * T.ds_f);
    fit4(v, c);
    T.ps[j] = make_float4((float)c[0], (float)c[1], (float)c[2], (float)c[3]);
  }
}

int pot_build(const mb_eam_tables *t, PotHost **out) {
  if (!t || !out) return fail(MB_ERR_ARG, "null potential tables");
  if (t->n_types < 1 || t->n_types > 3) return fail(MB_ERR_ARG, "n_types must be 1..3");
  if (t->nr < 5 || t->nrho < 5) return fail(MB_ERR_ARG, "tables need at least 5 knots");
  if (!(t->dr > 0) || !(t->drho > 0) || !(t->cutoff > 0)) return fail(MB_ERR_ARG, "dr, drho, cutoff must be > 0");
  if (!t->f || !t->F || !t->phi) return fail(MB_ERR_ARG, "null table pointer");
  const int nt = t->n_types, nr = t->nr, nrho = t->nrho, np = nt * (nt + 1) / 2;

  std::vector<double4> f_val((size_t)nt * nr), f_der((size_t)nt * nr), F_val((size_t)nt * nrho),
      F_der((size_t)nt * nrho), phi_val((size_t)np * nr), phi_der((size_t)np * nr);
  std::vector<double2> force1((size_t)nr * 3);
  std::vector<float4> f_val32((size_t)nt * nr), phi_val32((size_t)nr);
  std::vector<float2> force32((size_t)nr * 3);
  std::vector<double> c7;
  auto split = [&](const std::vector<double> &c, std::vector<double4> &val, std::vector<double4> &der, size_t base,
                   int n) {
    for (int m = 0; m < n; m++) {
      const double *k = &c[(size_t)m * 7];
      val[base + m] = make_double4(k[0], k[1], k[2], k[3]);
      der[base + m] = make_double4(k[4], k[5], k[6], 0.0);
    }
  };
  for (int a = 0; a < nt; a++) {
    knot_pieces(t->f + (size_t)a * nr, nr, t->dr, c7);
    split(c7, f_val, f_der, (size_t)a * nr, nr);
    knot_pieces(t->F + (size_t)a * nrho, nrho, t->drho, c7);
    split(c7, F_val, F_der, (size_t)a * nrho, nrho);
  }
  for (int q = 0; q < np; q++) {
    knot_pieces(t->phi + (size_t)q * nr, nr, t->dr, c7);
    split(c7, phi_val, phi_der, (size_t)q * nr, nr);
  }
  for (int m = 0; m < nr; m++) {
    const double4 fd = f_der[m], pd = phi_der[m];
    force1[(size_t)m * 3 + 0] = make_double2(fd.x, pd.x);
    force1[(size_t)m * 3 + 1] = make_double2(fd.y, pd.y);
    force1[(size_t)m * 3 + 2] = make_double2(fd.z, pd.z);
    force32[(size_t)m * 3 + 0] = make_float2((float)fd.x, (float)pd.x);
    force32[(size_t)m * 3 + 1] = make_float2((float)fd.y, (float)pd.y);
    force32[(size_t)m * 3 + 2] = make_float2((float)fd.z, (float)pd.z);
    const double4 pv = phi_val[m];
    phi_val32[m] = make_float4((float)pv.x, (float)pv.y, (float)pv.z, (float)pv.w);
  }
  for (size_t i = 0; i < f_val.size(); i++) {
    const double4 v = f_val[i];
    f_val32[i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
  }

  STables st;
  if (nt == 1) s_tables(t, st);
  const std::vector<float2> &fs = st.fs, &ab = st.ab;
  const std::vector<float4> &ps = st.ps;

  size_t off = 0;
  auto reserve = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t o_fv = reserve(f_val.size() * sizeof(double4)), o_fd = reserve(f_der.size() * sizeof(double4)),
               o_Fv = reserve(F_val.size() * sizeof(double4)), o_Fd = reserve(F_der.size() * sizeof(double4)),
               o_pv = reserve(phi_val.size() * sizeof(double4)), o_pd = reserve(phi_der.size() * sizeof(double4)),
               o_f1 = reserve(force1.size() * sizeof(double2)), o_fv32 = reserve(f_val32.size() * sizeof(float4)),
               o_f32 = reserve(force32.size() * sizeof(float2)), o_pv32 = reserve(phi_val32.size() * sizeof(float4)),
               o_fs = reserve(fs.size() * sizeof(float2)), o_ab = reserve(ab.size() * sizeof(float2)),
               o_ps = reserve(ps.size() * sizeof(float4));
  PotHost *p = new PotHost();
  cudaError_t e = cudaMalloc(&p->blob, off);
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e, "cudaMalloc(potential tables)");
  }
  char *b = (char *)p->blob;
  std::vector<char> staging(off, 0);
  memcpy(&staging[o_fv], f_val.data(), f_val.size() * sizeof(double4));
  memcpy(&staging[o_fd], f_der.data(), f_der.size() * sizeof(double4));
  memcpy(&staging[o_Fv], F_val.data(), F_val.size() * sizeof(double4));
  memcpy(&staging[o_Fd], F_der.data(), F_der.size() * sizeof(double4));
  memcpy(&staging[o_pv], phi_val.data(), phi_val.size() * sizeof(double4));
  memcpy(&staging[o_pd], phi_der.data(), phi_der.size() * sizeof(double4));
  memcpy(&staging[o_f1], force1.data(), force1.size() * sizeof(double2));
  memcpy(&staging[o_fv32], f_val32.data(), f_val32.size() * sizeof(float4));
  memcpy(&staging[o_f32], force32.data(), force32.size() * sizeof(float2));
  memcpy(&staging[o_pv32], phi_val32.data(), phi_val32.size() * sizeof(float4));
  if (!fs.empty()) {
    memcpy(&staging[o_fs], fs.data(), fs.size() * sizeof(float2));
    memcpy(&staging[o_ab], ab.data(), ab.size() * sizeof(float2));
    memcpy(&staging[o_ps], ps.data(), ps.size() * sizeof(float4));
  }
  e = cudaMemcpy(p->blob, staging.data(), off, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p->blob);
    delete p;
    return cuda_fail(e, "cudaMemcpy(potential tables)");
  }
  DevPot &d = p->dev;
  d.n_types = nt;
  d.nr = nr;
  d.nrho = nrho;
  d.rdr = 1.0 / t->dr;
  d.rdrho = 1.0 / t->drho;
  d.rho_max = (double)(nrho - 1) * t->drho;
  d.cutoff = t->cutoff;
  d.f_val = (const double4 *)(b + o_fv);
  d.f_der = (const double4 *)(b + o_fd);
  d.F_val = (const double4 *)(b + o_Fv);
  d.F_der = (const double4 *)(b + o_Fd);
  d.phi_val = (const double4 *)(b + o_pv);
  d.phi_der = (const double4 *)(b + o_pd);
  d.force1 = (const double2 *)(b + o_f1);
  d.f_val32 = (const float4 *)(b + o_fv32);
  d.force32 = (const float2 *)(b + o_f32);
  d.phi_val32 = (const float4 *)(b + o_pv32);
  d.n_rs = (int)fs.size();
  d.ds_r = st.ds_r;
  d.fs32 = fs.empty() ? nullptr : (const float2 *)(b + o_fs);
  d.n_fs = (int)ps.size();
  d.ds_f = st.ds_f;
  d.ab32 = fs.empty() ? nullptr : (const float2 *)(b + o_ab);
  d.ps32 = fs.empty() ? nullptr : (const float4 *)(b + o_ps);
  *out = p;
  return MB_OK;
}

void pot_free(PotHost *p) {
  if (!p) return;
  if (p->blob) cudaFree(p->blob);
  delete p;
}

const DevPot &pot_dev(const PotHost *p) { return p->dev; }

} // namespace mb

// Host-side check of the table construction (no device needed): the 7 spline
// coefficients per knot of one row of knot values.
extern "C" int mb_spline_coeffs(const double *y, int n, double dx, double *coef7) {
  if (!y || !coef7 || n < 5 || !(dx > 0)) return mb::fail(MB_ERR_ARG, "mb_spline_coeffs: bad arguments");
  std::vector<double> c7;
  mb::knot_pieces(y, n, dx, c7);
  memcpy(coef7, c7.data(), sizeof(double) * 7 * (size_t)n);
  return MB_OK;
}
