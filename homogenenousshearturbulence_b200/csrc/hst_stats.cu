// The diagnostics of the resident field on the device: outstats and the
// pressure.  The statistics of outstats (src/hst_stats.f90:136-285):
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

// partials: eps (k^2 |u|^2), uv, uu, vv, ww, vw, uw, mfx, mfz, then q_out
// (the weighted |u|^2 of every column but the mean), ed and pd (the energy in
// the damped columns and its damping rate, gsoft = 1 for the soft damping);
// the Stokes layer is not part of the GPU substep, so no row is inside it and
// q_in, e_in are zero
constexpr int ST_NM = 12;
__global__ void __launch_bounds__(32 * ST_WARPS) k_stats_moments(Geometry g, PhysScalars ps,
                                                                 const double2* __restrict__ V1,
                                                                 const double2* __restrict__ V2,
                                                                 const double2* __restrict__ V3,
                                                                 const double* __restrict__ dyl,
                                                                 const double* __restrict__ gdamp, double gsoft,
                                                                 double* __restrict__ partial) {
  double v[ST_NM] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int col = blockIdx.x * ST_WARPS + warp; col < g.ncol; col += gridDim.x * ST_WARPS) {
    const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
    const double al = ps.alfa0 * ix, be = ps.beta0 * iz, kk = al * al + be * be;
    const double gd = gdamp[col];
    const size_t cb = (size_t)col * g.rows + 2;
    for (int iy = lane; iy < g.ny; iy += 32) {
      const cxd u = V1[cb + iy], vv = V2[cb + iy], w = V3[cb + iy];
      const double d = dyl[iy];
      if (ix == 0 && iz == 0) {
        v[7] += u.x * d;
        v[8] += w.x * d;
        if (gd > 0.0) {
          const double qc = d * ((u.x * u.x + u.y * u.y) + (w.x * w.x + w.y * w.y));
          v[10] += qc;
          v[11] += 2.0 * gsoft * gd * qc;
        }
        v[2] += d * (u.x * u.x + u.y * u.y);
        v[4] += d * (w.x * w.x + w.y * w.y);
        v[6] += d * (u.x * w.x + u.y * w.y);
        continue;
      }
      const double wt = ix == 0 ? d : 2.0 * d;
      const double pu = u.x * u.x + u.y * u.y, pv = vv.x * vv.x + vv.y * vv.y, pw = w.x * w.x + w.y * w.y;
      if (gd > 0.0) {
        const double qc = wt * (pu + pv + pw);
        v[10] += qc;
        v[11] += 2.0 * gsoft * gd * qc;
      }
      v[2] += wt * pu;
      v[3] += wt * pv;
      v[4] += wt * pw;
      v[1] += wt * (u.x * vv.x + u.y * vv.y);
      v[5] += wt * (w.x * vv.x + w.y * vv.y);
      v[6] += wt * (u.x * w.x + u.y * w.y);
      v[0] += wt * kk * (pu + pv + pw);
      v[9] += wt * (pu + pv + pw);
    }
  }
  block_sums<ST_NM>(v, partial);
}

// the column energies exz(iz, ix) = sum_y w |u|^2 (src/hst_stats.f90:225-240),
// one warp per column, lanes over rows, a fixed order
__global__ void __launch_bounds__(32 * ST_WARPS) k_stats_columns(Geometry g, const double2* __restrict__ V1,
                                                                 const double2* __restrict__ V2,
                                                                 const double2* __restrict__ V3,
                                                                 const double* __restrict__ dyl,
                                                                 double* __restrict__ exz) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * ST_WARPS + warp;
  if (col >= g.ncol) return;
  const int ix = col / g.nzT;
  const size_t cb = (size_t)col * g.rows + 2;
  double q = 0.0;
  for (int iy = lane; iy < g.ny; iy += 32) {
    const cxd u = V1[cb + iy], vv = V2[cb + iy], w = V3[cb + iy];
    const double wt = ix == 0 ? dyl[iy] : 2.0 * dyl[iy];
    q += wt * ((u.x * u.x + u.y * u.y) + (vv.x * vv.x + vv.y * vv.y) + (w.x * w.x + w.y * w.y));
  }
  for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  if (lane == 0) exz[col] = q;
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

// out[0..7]: energy, dissipation, uv, vw, uu, vv, ww, uw (the order of the
// Runtimedata columns the reference writes); out[8..23]: the reference's
// sums array before the box-mean correction (eps, uv, uu, vv, ww, vw, uw,
// mfx, mfz, q_in, q_out, e_in, e_out, ed, pd; ncol_damped is the host's)
__global__ void k_stats_final(int nblk, const double* __restrict__ pm, const double* __restrict__ pg, double ly_w,
                              double ni, double ly, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[ST_NM] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblk; ++b)
    for (int k = 0; k < ST_NM; ++k) s[k] += pm[(size_t)b * ST_NM + k];
  double eps = s[0];
  for (int c = 0; c < 3; ++c)
    for (int b = 0; b < nblk; ++b) eps += pg[(size_t)c * nblk + b];
  double* raw = out + 8;
  raw[0] = eps;
  for (int k = 1; k < 9; ++k) raw[k] = s[k];
  raw[9] = 0.0;    // q_in
  raw[10] = s[9];  // q_out
  raw[11] = 0.0;   // e_in
  raw[12] = eps;   // e_out
  raw[13] = s[10];
  raw[14] = s[11];
  raw[15] = 0.0;
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

// ------------------------------------------------------------ pressure ----
// compute_pressure (src/hst_pressure.f90:35-110): the Poisson right-hand
// side of one row from the six product spectra (their ghost rows the
// shear-periodic images, as in the right-hand-side kernel) and the
// mean-shear term -2 i (S alfa + S2 beta) D0 v; the (0,0) column holds
// -<vv>(y) itself.  One warp per column, lanes over rows.
template <typename QT>
__global__ void __launch_bounds__(32 * ST_WARPS) k_pressure_rhs(Geometry g, PhysScalars ps, double s2now, double sx,
                                                                double sz, const QT* __restrict__ Q,
                                                                const QT* __restrict__ Qg,
                                                                const double2* __restrict__ V2,
                                                                const double* __restrict__ der,
                                                                double2* __restrict__ R) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * ST_WARPS + warp;
  if (col >= g.ncol) return;
  const int ny = g.ny;
  const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
  const double al = ps.alfa0 * ix, be = ps.beta0 * iz;
  const cxd ph = cexpi(-(al * sx + be * sz));
  const size_t qs = (size_t)g.ncol * ny;
  const QT* Qc = Q + (size_t)col * ny;
  const double2* Vc = V2 + (size_t)col * g.rows + 2;
  const double cm = 2.0 * (ps.S * al + s2now * be);
  for (int r = lane; r < ny; r += 32) {
    cxd acc = mkc(0, 0);
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      cxd d0 = mkc(0, 0), d1 = mkc(0, 0), d2 = mkc(0, 0);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const int q = r + j - 2;
        cxd v;
        if (Qg && (q < 0 || q >= ny)) {  // the ghost rows' own spectra
          const QT qr = Qg[((size_t)p * g.ncol + col) * 4 + (q < 0 ? q + 2 : q - ny + 2)];
          v = mkc((double)qr.x, (double)qr.y);
        } else {
          const QT qr = Qc[(size_t)p * qs + (q < 0 ? q + ny : (q >= ny ? q - ny : q))];
          v = mkc((double)qr.x, (double)qr.y);
          if (q < 0) v = cmul(v, cconj(ph));
          if (q >= ny) v = cmul(v, ph);
        }
        const double e0 = derv(der, ny, r, 0, j - 2), e1 = derv(der, ny, r, 1, j - 2), e2 = derv(der, ny, r, 2, j - 2);
        d0 = mkc(d0.x + e0 * v.x, d0.y + e0 * v.y);
        d1 = mkc(d1.x + e1 * v.x, d1.y + e1 * v.y);
        d2 = mkc(d2.x + e2 * v.x, d2.y + e2 * v.y);
      }
      cxd term;
      if (p == 0) term = cscale(al * al, d0);                           // -(i alfa)^2 d0
      else if (p == 1) term = cneg(d2);                                 // -d2
      else if (p == 2) term = cscale(be * be, d0);                      // -(i beta)^2 d0
      else if (p == 3) term = mkc(2.0 * al * d1.y, -2.0 * al * d1.x);  // -2 i alfa d1
      else if (p == 4) term = mkc(2.0 * be * d1.y, -2.0 * be * d1.x);  // -2 i beta d1
      else term = cscale(2.0 * al * be, d0);                            // -2 (i alfa)(i beta) d0
      if (p == 0) {
        cxd v0 = mkc(0, 0);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          const double e0 = derv(der, ny, r, 0, j - 2);
          const cxd v = Vc[r + j - 2];
          v0 = mkc(v0.x + e0 * v.x, v0.y + e0 * v.y);
        }
        acc = mkc(term.x + cm * v0.y, term.y - cm * v0.x);  // term - 2 i (S alfa + S2 beta) v0
      } else {
        acc = cadd(acc, term);
      }
      if (ix == 0 && iz == 0 && p == 1) acc = mkc(-(double)Qc[qs + r].x, 0.0);
    }
    R[(size_t)col * g.rows + 2 + r] = acc;
  }
}

// the (0,0) mode: p = rhs, its y mean (weights dyl) removed, imaginary part zero
__global__ void k_pressure_mean(Geometry g, const double2* __restrict__ R, const double* __restrict__ dyl, double ly,
                                double2* __restrict__ P) {
  __shared__ double pmean;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int iy = 0; iy < g.ny; ++iy) s += R[2 + iy].x * dyl[iy];
    pmean = s / ly;
  }
  __syncthreads();
  for (int iy = threadIdx.x; iy < g.ny; iy += blockDim.x) P[2 + iy] = mkc(R[2 + iy].x - pmean, 0.0);
}

cudaError_t launch_pressure_rhs(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double s2now,
                                double sx, double sz, cudaStream_t st) {
  const int blocks = (g.ncol + ST_WARPS - 1) / ST_WARPS;
  if (g.mp)
    k_pressure_rhs<float2><<<blocks, 32 * ST_WARPS, 0, st>>>(g, ps, s2now, sx, sz, reinterpret_cast<const float2*>(d.Q),
                                                             reinterpret_cast<const float2*>(d.Qg), d.F[1], d.der,
                                                             d.F[5]);
  else
    k_pressure_rhs<double2><<<blocks, 32 * ST_WARPS, 0, st>>>(g, ps, s2now, sx, sz, d.Q, d.Qg, d.F[1], d.der, d.F[5]);
  return cudaGetLastError();
}

cudaError_t launch_pressure_mean(const Geometry& g, const DeviceState& d, double ly, int dst, cudaStream_t st) {
  // the (0,0) column is column nz (ix = 0, iz = 0)
  const size_t c00 = (size_t)g.nz * g.rows;
  k_pressure_mean<<<1, 256, 0, st>>>(g, d.F[5] + c00, d.dyl, ly, d.F[dst] + c00);
  return cudaGetLastError();
}

int stats_blocks(const Geometry& g, int nsm) {
  int b = 4 * (nsm > 0 ? nsm : 148);
  const int need = (g.ncol + ST_WARPS - 1) / ST_WARPS;
  return b < need ? b : need;
}

cudaError_t launch_stats_moments(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double gsoft,
                                 double* partial, cudaStream_t st) {
  k_stats_moments<<<stats_blocks(g, d.nsm), 32 * ST_WARPS, 0, st>>>(g, ps, d.F[0], d.F[1], d.F[2], d.dyl, d.gdamp,
                                                                     gsoft, partial);
  return cudaGetLastError();
}

cudaError_t launch_stats_columns(const Geometry& g, const DeviceState& d, double* exz, cudaStream_t st) {
  k_stats_columns<<<(g.ncol + ST_WARPS - 1) / ST_WARPS, 32 * ST_WARPS, 0, st>>>(g, d.F[0], d.F[1], d.F[2], d.dyl, exz);
  return cudaGetLastError();
}

int stats_partials() { return ST_NM; }

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
