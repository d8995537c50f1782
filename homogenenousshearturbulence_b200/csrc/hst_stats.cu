// The statistics of outstats (src/hst_stats.f90:136-285) on the device:
// the box averages of the energy, the dissipation, the Reynolds stresses uv,
// vw, uw and the variances uu, vv, ww of the resident field, in FP64 with a
// fixed reduction order (the same result for the same field every time).
//
//   k_stats_moments  per Fourier column, the Parseval sums of the second
//                    moments with the y weights dyl (twice for ix > 0, the
//                    conjugate half), k^2 |u|^2 for the dissipation, and the
//                    mean-flow sums of the (0,0) column
//   k_stats_grad     per column, the weighted |dq/dy|^2 of one component
//                    (its compact derivative comes from the DY line solve)
//   k_stats_final    the block partials summed in order, the mean flow
//                    removed from the (0,0) variances, everything over ly
#include "hst_dev.cuh"
#include "hst_internal.h"

namespace hst {

constexpr int ST_WARPS = 8;  // warps a block; each walks whole columns

// sums of one warp, then of the block, in a fixed order; lane 0 of warp 0
// writes the block's NV partials
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* __restrict__ out) {
  __shared__ double part[ST_WARPS][NV];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) part[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int w = 0; w < ST_WARPS; ++w) t += part[w][k];
      out[(size_t)blockIdx.x * NV + k] = t;
    }
}

// partials: eps (k^2 |u|^2), uv, uu, vv, ww, vw, uw, mfx, mfz
__global__ void __launch_bounds__(32 * ST_WARPS) k_stats_moments(Geometry g, PhysScalars ps,
                                                                 const double2* __restrict__ V1,
                                                                 const double2* __restrict__ V2,
                                                                 const double2* __restrict__ V3,
                                                                 const double* __restrict__ dyl,
                                                                 double* __restrict__ partial) {
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int col = blockIdx.x * ST_WARPS + warp; col < g.ncol; col += gridDim.x * ST_WARPS) {
    const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
    const double al = ps.alfa0 * ix, be = ps.beta0 * iz, kk = al * al + be * be;
    const size_t cb = (size_t)col * g.rows + 2;
    for (int iy = lane; iy < g.ny; iy += 32) {
      const cxd u = V1[cb + iy], vv = V2[cb + iy], w = V3[cb + iy];
      const double d = dyl[iy];
      if (ix == 0 && iz == 0) {
        v[7] += u.x * d;
        v[8] += w.x * d;
        v[2] += d * (u.x * u.x + u.y * u.y);
        v[4] += d * (w.x * w.x + w.y * w.y);
        v[6] += d * (u.x * w.x + u.y * w.y);
        continue;
      }
      const double wt = ix == 0 ? d : 2.0 * d;
      const double pu = u.x * u.x + u.y * u.y, pv = vv.x * vv.x + vv.y * vv.y, pw = w.x * w.x + w.y * w.y;
      v[2] += wt * pu;
      v[3] += wt * pv;
      v[4] += wt * pw;
      v[1] += wt * (u.x * vv.x + u.y * vv.y);
      v[5] += wt * (w.x * vv.x + w.y * vv.y);
      v[6] += wt * (u.x * w.x + u.y * w.y);
      v[0] += wt * kk * (pu + pv + pw);
    }
  }
  block_sums<9>(v, partial);
}

// the weighted sum of |q|^2 over every column (q: the DY solve of one component)
__global__ void __launch_bounds__(32 * ST_WARPS) k_stats_grad(Geometry g, const double2* __restrict__ Q,
                                                              const double* __restrict__ dyl,
                                                              double* __restrict__ partial) {
  double v[1] = {0.0};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int col = blockIdx.x * ST_WARPS + warp; col < g.ncol; col += gridDim.x * ST_WARPS) {
    const int ix = col / g.nzT;
    const size_t cb = (size_t)col * g.rows + 2;
    for (int iy = lane; iy < g.ny; iy += 32) {
      const cxd q = Q[cb + iy];
      const double wt = ix == 0 ? dyl[iy] : 2.0 * dyl[iy];
      v[0] += wt * (q.x * q.x + q.y * q.y);
    }
  }
  block_sums<1>(v, partial);
}

// out: energy, dissipation, uv, vw, uu, vv, ww, uw (the order of the
// Runtimedata columns the reference writes)
__global__ void k_stats_final(int nblk, const double* __restrict__ pm, const double* __restrict__ pg, double ly_w,
                              double ni, double ly, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblk; ++b)
    for (int k = 0; k < 9; ++k) s[k] += pm[(size_t)b * 9 + k];
  double eps = s[0];
  for (int c = 0; c < 3; ++c)
    for (int b = 0; b < nblk; ++b) eps += pg[(size_t)c * nblk + b];
  double uu = s[2] - s[7] * s[7] / ly_w, ww = s[4] - s[8] * s[8] / ly_w, uw = s[6] - s[7] * s[8] / ly_w;
  const double vv = s[3], uv = s[1], vw = s[5];
  const double inv = 1.0 / ly;
  out[0] = 0.5 * (uu + vv + ww) * inv;
  out[1] = ni * eps * inv;
  out[2] = uv * inv;
  out[3] = vw * inv;
  out[4] = uu * inv;
  out[5] = vv * inv;
  out[6] = ww * inv;
  out[7] = uw * inv;
}

int stats_blocks(const Geometry& g, int nsm) {
  int b = 4 * (nsm > 0 ? nsm : 148);
  const int need = (g.ncol + ST_WARPS - 1) / ST_WARPS;
  return b < need ? b : need;
}

cudaError_t launch_stats_moments(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double* partial,
                                 cudaStream_t st) {
  k_stats_moments<<<stats_blocks(g, d.nsm), 32 * ST_WARPS, 0, st>>>(g, ps, d.F[0], d.F[1], d.F[2], d.dyl, partial);
  return cudaGetLastError();
}

cudaError_t launch_stats_grad(const Geometry& g, const DeviceState& d, int field, double* partial, cudaStream_t st) {
  k_stats_grad<<<stats_blocks(g, d.nsm), 32 * ST_WARPS, 0, st>>>(g, d.F[field], d.dyl, partial);
  return cudaGetLastError();
}

cudaError_t launch_stats_final(const Geometry& g, const DeviceState& d, const double* pm, const double* pg,
                               double ly_w, double ni, double ly, double* out, cudaStream_t st) {
  k_stats_final<<<1, 32, 0, st>>>(stats_blocks(g, d.nsm), pm, pg, ly_w, ni, ly, out);
  return cudaGetLastError();
}

}  // namespace hst
