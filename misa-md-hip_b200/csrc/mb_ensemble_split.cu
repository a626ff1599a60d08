// Mixed-precision step of ONE large lattice as separate kernels (split mode).
//
// The persistent tile kernel (mb_ensemble.cu) keeps both passes, both spline tables
// and two TMA tile buffers resident, which caps it at 16 warps per SM.  A single
// large lattice does not need that: here the density pass and the force + velocity-
// Verlet pass are separate kernels, each holding only its own FP32 table in shared
// memory and reading neighbour rows through L1 (sublattice rows are contiguous), so
// each runs with 24-32 warps per SM.  The pair arithmetic (displacement-relative
// spline index, f32x2 lanes, two-sum accumulation) is the tile kernel's, so results
// agree with it to rounding of the summation order.  The kernels of one step are
// captured into one CUDA graph by the ensemble host.
#include "mb_ensemble_kernel.cuh"
#include "mb_ensemble_pair.cuh"

namespace mb {

#define MX_RHO_THREADS 1024
#define MX_FORCE_THREADS 768

// Rows of 32 sites along x: item w -> (chunk, y, s, z), as the FP64 kernels walk.
__device__ __forceinline__ bool mx_site(const LatDesc &d, int chunks, long long w, int lane, int &s, int &cx, int &y,
                                        int &z, long long &i) {
  long long t = w;
  const int chunk = (int)(t % chunks);
  t /= chunks;
  y = (int)(t % d.by);
  t /= d.by;
  s = (int)(t & 1);
  z = (int)(t >> 1);
  cx = chunk * 32 + lane;
  if (cx >= d.bcx) return false;
  i = (long long)s * d.E + ((long long)(z + 2) * d.ey + y + 2) * d.ecx + cx + 2;
  return true;
}

template <bool ENERGY>
__global__ void __launch_bounds__(MX_RHO_THREADS, 1)
    k_mx_rho(const __grid_constant__ EnsParams P, const __grid_constant__ MxStencil S, int lat) {
  extern __shared__ float4 s_fv[];
  for (int k = threadIdx.x; k < P.nsm; k += blockDim.x) s_fv[k] = P.P.f_val32[P.m_lo + k];
  __syncthreads();
  const LatDesc &d = P.lats[lat];
  const bool active = lat_active(d);
  const int lane = threadIdx.x & 31;
  const int chunks = (d.bcx + 31) / 32;
  const long long n_items = (long long)chunks * d.by * 2 * d.bz;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  const float4 *u4 = d.u4[d.cur];
  float4 *uw = d.u4[d.cur];
  double e_acc = 0.0;
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); active && w < n_items;
       w += wstride) {
    int s, cx, y, z;
    long long i;
    if (!mx_site(d, chunks, w, lane, s, cx, y, z, i)) continue;
    const int code = d.code[i];
    if (code < 0 || (code & MB_FLAG_ITL)) continue;
    const float4 u = __ldg(u4 + i);
    const int *off = S.off[s];
    float rs0 = 0.f, rc0 = 0.f, rs1 = 0.f, rc1 = 0.f;
    const int n = P.n_st, nn = P.n_near;
    int k = 0;
    for (; k + 1 < nn; k += 2) {
      const float4 nb0 = __ldg(u4 + i + off[k]), nb1 = __ldg(u4 + i + off[k + 1]);
      rho_pair<true>(P, u, nb0, P.ck[s][k], s, k, s_fv, rs0, rc0);
      rho_pair<true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fv, rs1, rc1);
    }
    if (k < nn) {
      rho_pair<true>(P, u, __ldg(u4 + i + off[k]), P.ck[s][k], s, k, s_fv, rs0, rc0);
      k++;
    }
    for (; k < n; k++) rho_pair<false>(P, u, __ldg(u4 + i + off[k]), P.ck[s][k], s, k, s_fv, rs1, rc1);
    const double rho = ((double)rs0 + (double)rs1) + ((double)rc0 + (double)rc1);
    const double df = dF64(P.P, code & 0x3F, rho);
    reinterpret_cast<float *>(uw + i)[3] = (float)df;
    d.rho[i] = (float)rho;
    const Geom g = lat_geom(d);
    for_images(g, s, cx, y, z,
               [&](long long idx, double, double, double) { reinterpret_cast<float *>(uw + idx)[3] = (float)df; });
    if (ENERGY) e_acc += F64(P.P, code & 0x3F, rho);
  }
  if (ENERGY) {
    const double t = block_sum(e_acc);
    if (threadIdx.x == 0) P.epart[2 * blockIdx.x] = t;
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(MX_FORCE_THREADS, 1)
    k_mx_force(const __grid_constant__ EnsParams P, const __grid_constant__ MxStencil S, int lat) {
  extern __shared__ float2 s_fd[];
  for (int k = threadIdx.x; k < 3 * P.nsm; k += blockDim.x) s_fd[k] = P.P.force32[3 * P.m_lo + k];
  __syncthreads();
  const LatDesc &d = P.lats[lat];
  const bool active = lat_active(d);
  const int lane = threadIdx.x & 31;
  const int chunks = (d.bcx + 31) / 32;
  const long long n_items = (long long)chunks * d.by * 2 * d.bz;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  const float4 *u4 = d.u4[d.cur];
  float4 *un = d.u4[d.cur ^ 1];
  double e_pair = 0.0, e_kin = 0.0;
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); active && w < n_items;
       w += wstride) {
    int s, cx, y, z;
    long long i;
    if (!mx_site(d, chunks, w, lane, s, cx, y, z, i)) continue;
    const int code = d.code[i];
    if (code < 0 || (code & MB_FLAG_ITL)) continue;
    const float4 u = __ldg(u4 + i);
    const int *off = S.off[s];
    float2 fs0 = make_float2(0.f, 0.f), fc0 = fs0, fs1 = fs0, fc1 = fs0;
    float zs0 = 0.f, zc0 = 0.f, ps0 = 0.f, pc0 = 0.f, zs1 = 0.f, zc1 = 0.f, ps1 = 0.f, pc1 = 0.f;
    const int n = P.n_st, nn = P.n_near;
    int k = 0;
    for (; k + 1 < nn; k += 2) {
      const float4 nb0 = __ldg(u4 + i + off[k]), nb1 = __ldg(u4 + i + off[k + 1]);
      force_pair<ENERGY, true>(P, u, nb0, P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
      force_pair<ENERGY, true>(P, u, nb1, P.ck[s][k + 1], s, k + 1, s_fd, fs1, fc1, zs1, zc1, ps1, pc1);
    }
    if (k < nn) {
      force_pair<ENERGY, true>(P, u, __ldg(u4 + i + off[k]), P.ck[s][k], s, k, s_fd, fs0, fc0, zs0, zc0, ps0, pc0);
      k++;
    }
    for (; k < n; k++)
      force_pair<ENERGY, false>(P, u, __ldg(u4 + i + off[k]), P.ck[s][k], s, k, s_fd, fs1, fc1, zs1, zc1, ps1, pc1);
    const double fx = ((double)fs0.x + (double)fs1.x) + ((double)fc0.x + (double)fc1.x);
    const double fy = ((double)fs0.y + (double)fs1.y) + ((double)fc0.y + (double)fc1.y);
    const double fz = ((double)zs0 + (double)zs1) + ((double)zc0 + (double)zc1);
    d.fx[i] = (float)fx;
    d.fy[i] = (float)fy;
    d.fz[i] = (float)fz;
    double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
    if (d.primed) {
      vx += P.h * fx;
      vy += P.h * fy;
      vz += P.h * fz;
    }
    if (ENERGY) {
      e_kin += 0.5 * P.mass * (vx * vx + vy * vy + vz * vz) * MB_MVV2E;
      e_pair += ((double)ps0 + (double)ps1) + ((double)pc0 + (double)pc1);
    }
    vx += P.h * fx;
    vy += P.h * fy;
    vz += P.h * fz;
    const double nx = d.ux[i] + P.dt * vx, ny = d.uy[i] + P.dt * vy, nz = d.uz[i] + P.dt * vz;
    d.vx[i] = vx;
    d.vy[i] = vy;
    d.vz[i] = vz;
    d.ux[i] = nx;
    d.uy[i] = ny;
    d.uz[i] = nz;
    const float4 nu = make_float4((float)nx, (float)ny, (float)nz, 0.f);
    un[i] = nu;
    const Geom g = lat_geom(d);
    for_images(g, s, cx, y, z, [&](long long idx, double, double, double) { un[idx] = nu; });
  }
  if (ENERGY) {
    const double t1 = block_sum(e_pair);
    const double t2 = block_sum(e_kin);
    if (threadIdx.x == 0) {
      P.epart[2 * blockIdx.x] += t1;
      P.epart[2 * blockIdx.x + 1] = t2;
    }
  }
}

// Interstitial phases and step bookkeeping of split mode, one kernel each (the
// phases the persistent kernel separates with grid barriers).
__global__ void k_mx_itl_clear(const __grid_constant__ EnsParams P) {
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (lat_active(d)) itl_clear_flags(d);
  }
}

__global__ void k_mx_itl_mark(const __grid_constant__ EnsParams P) {
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int q = 0; q < P.n_itl_lats; q++) {
    const LatDesc &d = P.lats[P.itl_lats[q]];
    if (!lat_active(d)) continue;
    for (int it = gw; it < d.n_itl; it += warps) itl_mark_one(P, d, it);
  }
}

template <bool FORCE, bool ENERGY>
__global__ void k_mx_itl_items(const __grid_constant__ EnsParams P) {
  itl_items<FORCE, ENERGY>(P);
}

__global__ void k_mx_bookkeeping(const __grid_constant__ EnsParams P) {
  for (int l = threadIdx.x; l < P.n_lats; l += blockDim.x) {
    LatDesc *d = const_cast<LatDesc *>(&P.lats[l]);
    if (!lat_active(*d)) continue;
    d->cur ^= 1;
    if (d->primed)
      d->steps_done++;
    else
      d->primed = 1;
  }
}

int mx_launch_step(const EnsParams &P, const MxStencil &S, int lat, int energy, cudaStream_t s) {
  const int sms = device_sm_count();
  const size_t rho_smem = (size_t)P.nsm * sizeof(float4), force_smem = (size_t)P.nsm * 3 * sizeof(float2);
  static bool attr = false;
  if (!attr) {
    MB_CUDA(cudaFuncSetAttribute(k_mx_rho<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    MB_CUDA(cudaFuncSetAttribute(k_mx_rho<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    MB_CUDA(cudaFuncSetAttribute(k_mx_force<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    MB_CUDA(cudaFuncSetAttribute(k_mx_force<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  const int itl_grid = 2 * sms;
  if (P.n_itl_lats > 0) {
    k_mx_itl_clear<<<itl_grid, 256, 0, s>>>(P);
    k_mx_itl_mark<<<itl_grid, 256, 0, s>>>(P);
  }
  if (energy)
    k_mx_rho<true><<<sms, MX_RHO_THREADS, rho_smem, s>>>(P, S, lat);
  else
    k_mx_rho<false><<<sms, MX_RHO_THREADS, rho_smem, s>>>(P, S, lat);
  if (P.n_itl_lats > 0) {
    if (energy)
      k_mx_itl_items<false, true><<<itl_grid, 256, 0, s>>>(P);
    else
      k_mx_itl_items<false, false><<<itl_grid, 256, 0, s>>>(P);
  }
  if (energy)
    k_mx_force<true><<<sms, MX_FORCE_THREADS, force_smem, s>>>(P, S, lat);
  else
    k_mx_force<false><<<sms, MX_FORCE_THREADS, force_smem, s>>>(P, S, lat);
  if (P.n_itl_lats > 0) {
    if (energy)
      k_mx_itl_items<true, true><<<itl_grid, 256, 0, s>>>(P);
    else
      k_mx_itl_items<true, false><<<itl_grid, 256, 0, s>>>(P);
  }
  k_mx_bookkeeping<<<1, 128, 0, s>>>(P);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// Energies of the split step: the per-CTA partials plus the interstitial items.
__global__ void k_mx_energy(const LatDesc *lats, int lat, const double *epart, int n_parts, double *out) {
  double pe = 0.0, ke = 0.0;
  for (int t = threadIdx.x; t < n_parts; t += blockDim.x) {
    pe += epart[2 * t];
    ke += epart[2 * t + 1];
  }
  pe = block_sum(pe);
  ke = block_sum(ke);
  if (threadIdx.x == 0) {
    out[0] = pe + lats[lat].e_itl[0];
    out[1] = ke + lats[lat].e_itl[1];
  }
}

int mx_energy_launch(const LatDesc *lats, int lat, const double *epart, double *out, cudaStream_t s) {
  k_mx_energy<<<1, 256, 0, s>>>(lats, lat, epart, device_sm_count(), out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mx_grid() { return device_sm_count(); }

} // namespace mb
