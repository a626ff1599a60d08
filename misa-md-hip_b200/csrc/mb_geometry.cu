// Host-side geometry: stencil generation and conversion, error state.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "mb_common.cuh"

namespace mb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string("CUDA error '") + cudaGetErrorString(e) + "' in " + what;
  return MB_ERR_CUDA;
}

int device_sm_count() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

// Ideal BCC site (gx, gy, gz) with x doubled, in units of a0:
// (gx/2, gy + (gx&1)/2, gz + (gx&1)/2).
int stencil_generate(double a0, double reach, int ext_x, int ext_y, int64_t *even, int64_t *odd, int cap, int *n,
                     int *reach_x, int *reach_y, int *reach_z) {
  const int cy = (int)ceil(reach / a0) + 1;
  const int cx = 2 * cy;
  int cnt[2] = {0, 0};
  int rx = 0, ry = 0, rz = 0;
  for (int par = 0; par < 2; par++) {
    int64_t *out = par ? odd : even;
    for (int dz = -cy; dz <= cy; dz++)
      for (int dy = -cy; dy <= cy; dy++)
        for (int dx = -cx; dx <= cx; dx++) {
          if (dx == 0 && dy == 0 && dz == 0) continue;
          const int npar = (par + dx) & 1;
          const double ox = 0.5 * dx, oy = dy + 0.5 * (npar - par), oz = dz + 0.5 * (npar - par);
          if (a0 * sqrt(ox * ox + oy * oy + oz * oz) >= reach) continue;
          if (cnt[par] >= cap) return fail(MB_ERR_ARG, "stencil larger than MB_MAX_STENCIL");
          out[cnt[par]++] = ((int64_t)dz * ext_y + dy) * ext_x + dx;
          rx = dx < 0 ? (-dx > rx ? -dx : rx) : (dx > rx ? dx : rx);
          ry = dy < 0 ? (-dy > ry ? -dy : ry) : (dy > ry ? dy : ry);
          rz = dz < 0 ? (-dz > rz ? -dz : rz) : (dz > rz ? dz : rz);
        }
  }
  if (cnt[0] != cnt[1]) return fail(MB_ERR_ARG, "even/odd stencils differ in size");
  *n = cnt[0];
  *reach_x = rx;
  *reach_y = ry;
  *reach_z = rz;
  return MB_OK;
}

static inline long long round_div(long long a, long long b) {
  // nearest integer of a / b for b > 0
  return a >= 0 ? (a + b / 2) / b : -((-a + b / 2) / b);
}

int stencil_from_linear(const int64_t *even, size_t n_even, const int64_t *odd, size_t n_odd, int ext_x, int ext_y,
                        const Geom &g, const int parity_of_sublattice[2], StencilSet *out) {
  if (n_even != n_odd) return fail(MB_ERR_ARG, "even and odd stencils must have the same length");
  if (n_even > MB_MAX_STENCIL) return fail(MB_ERR_ARG, "stencil longer than MB_MAX_STENCIL");
  out->n = (int)n_even;
  out->n_near = 0;
  const long long plane = (long long)ext_x * ext_y;
  for (int s = 0; s < 2; s++) {
    const int64_t *src = parity_of_sublattice[s] ? odd : even;
    for (size_t k = 0; k < n_even; k++) {
      const long long o = src[k];
      const long long dz = round_div(o, plane);
      const long long rem = o - dz * plane;
      const long long dy = round_div(rem, ext_x);
      const long long dx = rem - dy * ext_x;
      if (2 * llabs(dx) >= ext_x || 2 * llabs(dy) >= ext_y)
        return fail(MB_ERR_ARG, "stencil offset does not decode inside the ghost-extended array");
      const long long t = s + dx;                       // target doubled column offset from column 2c+s
      const int s2 = (int)(t & 1);
      const long long dcx = (t - s2) / 2;               // floor division (t - s2 is even)
      if (llabs(dcx) > g.gcx || llabs(dy) > g.gy || llabs(dz) > g.gz)
        return fail(MB_ERR_ARG, "stencil reaches beyond the ghost region");
      const long long lin = (long long)(s2 - s) * g.E + (dz * g.ey + dy) * g.ecx + dcx;
      out->off[s][k] = (int)lin;
    }
  }
  return MB_OK;
}

// Reorders both parities' doubled-x linear stencils by ideal distance (stable) and
// returns how many lead entries lie inside `cutoff` (equal for both parities).
int stencil_sort_by_distance(double a0, double cutoff, int ext_x, int ext_y, int64_t *even, int64_t *odd, int n,
                             int *n_near) {
  const long long plane = (long long)ext_x * ext_y;
  int near[2] = {0, 0};
  for (int par = 0; par < 2; par++) {
    int64_t *src = par ? odd : even;
    std::vector<std::pair<double, int64_t>> ord;
    for (int k = 0; k < n; k++) {
      const long long o = src[k];
      const long long dz = round_div(o, plane), rem = o - dz * plane, dy = round_div(rem, ext_x),
                      dx = rem - dy * ext_x;
      const int npar = (int)((par + dx) & 1);
      const double ox = 0.5 * dx, oy = dy + 0.5 * (npar - par), oz = dz + 0.5 * (npar - par);
      const double R = a0 * sqrt(ox * ox + oy * oy + oz * oz);
      ord.push_back({R, o});
      if (R < cutoff) near[par]++;
    }
    std::stable_sort(ord.begin(), ord.end(), [](const std::pair<double, int64_t> &x,
                                                 const std::pair<double, int64_t> &y) { return x.first < y.first; });
    for (int k = 0; k < n; k++) src[k] = ord[k].second;
  }
  if (near[0] != near[1]) return fail(MB_ERR_STATE, "even and odd stencils differ inside the cutoff");
  *n_near = near[0];
  return MB_OK;
}

} // namespace mb

extern "C" const char *mb_last_error(void) { return mb::g_last_error.c_str(); }
extern "C" const char *mb_version(void) { return "misa_b200 0.1 (sm_100a)"; }

extern "C" int mb_stencil_linear(double a0, double reach, int ext_x, int ext_y, int64_t *even, int64_t *odd, int cap,
                                 int *n) {
  if (!even || !odd || !n || !(a0 > 0) || !(reach > 0) || ext_x <= 0 || ext_y <= 0)
    return mb::fail(MB_ERR_ARG, "mb_stencil_linear: bad arguments");
  int rx, ry, rz;
  return mb::stencil_generate(a0, reach, ext_x, ext_y, even, odd, cap, n, &rx, &ry, &rz);
}
