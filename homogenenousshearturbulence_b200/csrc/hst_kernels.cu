// The kernels of the hst substep on sm_100a (FP64).
//
//   k_zinv    V (u, v, w) -> z-inverse transform on the padded z grid (Z)
//   k_xprod   Z -> x-inverse (c2r), the six velocity products times
//             1/(2 nxd nzd), the CFL maximum, x-forward (r2c) truncated to
//             the nx+1 retained modes (Pp)
//   k_zfwd    Pp -> z-forward transform truncated to the 2nz+1 modes (Q)
//   k_column  one warp group per Fourier column: the right-hand sides of
//             buildrhs_prepare and buildrhs, the hard damping mask, the
//             mean-shear phase shift (both forms), the D2V, ETA and DY line
//             solves, u and w, all ghost rows
//   k_line_solve, k_fill_ghosts: the single operations for the drop-in
//             interface and the tests
//
// Only the ny interior rows are transformed.  The products in the four
// ghost rows, which the reference transforms as well
// (src/hst_transforms.f90:3-6), are the shear-periodic images of the
// interior ones: the 3/2 rule makes the retained product modes exact, so the
// image of row k is row k times the wrap phase, which k_column applies when
// it reads them.
#include <cstdio>

#include "hst_dev.cuh"
#include "hst_fft.cuh"
#include "hst_internal.h"

namespace hst {

// --------------------------------------------------------------- k_zinv ----
// assemble_vvdz + IFT (src/hst_transforms.f90:33-54, src/hst_fft.f90:195-207)
// for a tile of Ty rows of one x mode of one component.
template <int PPT>
__global__ void k_zinv(Geometry g, const double2* __restrict__ V0, const double2* __restrict__ V1,
                       const double2* __restrict__ V2, double2* __restrict__ Z, const double2* __restrict__ twz) {
  extern __shared__ double2 sh[];
  const int yt = blockIdx.x, ix = blockIdx.y, c = blockIdx.z;
  const int Ty = g.Ty, NZ = g.nzd, nz = g.nz, nzT = g.nzT, LS = NZ + 1;
  const int nyT = g.ny / Ty;
  const double2* src = (c == 0 ? V0 : (c == 1 ? V1 : V2)) + (size_t)ix * nzT * g.rows + 2 + yt * Ty;
  for (int e = threadIdx.x; e < nzT * Ty; e += blockDim.x) {
    int izi = e / Ty, yi = e - izi * Ty;
    int iz = izi - nz;
    int kz = iz >= 0 ? iz : NZ + iz;
    sh[yi * LS + kz] = src[(size_t)izi * g.rows + yi];
  }
  for (int e = threadIdx.x; e < (NZ - nzT) * Ty; e += blockDim.x) {
    int k = e / Ty, yi = e - k * Ty;
    sh[yi * LS + nz + 1 + k] = mkc(0.0, 0.0);
  }
  __syncthreads();
  fft_lines<PPT>(sh, NZ, Ty, LS, twz, +1);
  double2* dst = Z + (((size_t)c * NZ) * nyT + yt) * g.nxB * Ty + (size_t)ix * Ty;
  for (int e = threadIdx.x; e < NZ * Ty; e += blockDim.x) {
    int kz = e / Ty, yi = e - kz * Ty;
    dst[(size_t)kz * nyT * g.nxB * Ty + yi] = sh[yi * LS + kz];
  }
}

// -------------------------------------------------------------- k_xprod ----
// to_x_points (zero padding + RFT), build_products for both groups,
// compute_cfl and HFT of the products (src/hst_transforms.f90:85-133,
// 163-179; src/hst_fft.f90:211-237) for one pair of rows at one z point.
// Two real lines are carried by one complex line: u + i v of each row and
// w0 + i w1 of the pair on the way in, (uu, vv), (ww, uv), (vw, uw) on the
// way out, separated by Hermitian symmetry.  The c2r reads only the real
// part of the kx = 0 mode, as FFTW's and cuFFT's c2r do.
template <int PPT>
__global__ void k_xprod(Geometry g, const double2* __restrict__ Z, double2* __restrict__ Pp,
                        const double2* __restrict__ twx, const double* __restrict__ dyl, PhysScalars ps, int want_cfl,
                        unsigned long long* __restrict__ cflmax) {
  extern __shared__ double2 sh[];
  const int NX = 2 * g.nxd, nx = g.nx, nxB = g.nxB, NZ = g.nzd, Ty = g.Ty;
  const int nyT = g.ny / Ty;
  const int y0 = 2 * blockIdx.x, kz = blockIdx.y;
  const int yt = y0 / Ty, yi0 = y0 - yt * Ty;
  cxd* A0 = sh;
  cxd* A1 = sh + NX;
  cxd* B = sh + 2 * NX;
  for (int k = threadIdx.x; k < NX; k += blockDim.x) {
    if (k > nx && k < NX - nx) {
      A0[k] = mkc(0, 0);
      A1[k] = mkc(0, 0);
      B[k] = mkc(0, 0);
    }
  }
  const size_t cs = (size_t)NZ * nyT * nxB * Ty;
  const size_t zb = ((size_t)kz * nyT + yt) * nxB * Ty + yi0;
  for (int ix = threadIdx.x; ix <= nx; ix += blockDim.x) {
    const size_t b = zb + (size_t)ix * Ty;
    cxd U0 = Z[b], U1 = Z[b + 1], W0v = Z[cs + b], W1v = Z[cs + b + 1], X0 = Z[2 * cs + b], X1 = Z[2 * cs + b + 1];
    // U: u modes, W*: v modes, X*: w modes
    if (ix == 0) {
      A0[0] = mkc(U0.x, W0v.x);
      A1[0] = mkc(U1.x, W1v.x);
      B[0] = mkc(X0.x, X1.x);
    } else {
      A0[ix] = mkc(U0.x - W0v.y, U0.y + W0v.x);
      A0[NX - ix] = mkc(U0.x + W0v.y, W0v.x - U0.y);
      A1[ix] = mkc(U1.x - W1v.y, U1.y + W1v.x);
      A1[NX - ix] = mkc(U1.x + W1v.y, W1v.x - U1.y);
      B[ix] = mkc(X0.x - X1.y, X0.y + X1.x);
      B[NX - ix] = mkc(X0.x + X1.y, X1.x - X0.y);
    }
  }
  __syncthreads();
  fft_lines<PPT>(sh, NX, 3, NX, twx, +1);
  double cm = 0.0;
  const double f = ps.factor;
  const double rdy0 = dyl[y0], rdy1 = dyl[y0 + 1];
  for (int x = threadIdx.x; x < NX; x += blockDim.x) {
    cxd a0 = A0[x], a1 = A1[x], b = B[x];
    double u0 = a0.x, v0 = a0.y, u1 = a1.x, v1 = a1.y, w0 = b.x, w1 = b.y;
    if (want_cfl) {
      double c0 = fabs(u0) / ps.dx + fabs(v0) / rdy0 + fabs(w0) / ps.dz;
      double c1 = fabs(u1) / ps.dx + fabs(v1) / rdy1 + fabs(w1) / ps.dz;
      cm = fmax(cm, fmax(c0, c1));
    }
    sh[0 * NX + x] = mkc(u0 * u0 * f, v0 * v0 * f);
    sh[1 * NX + x] = mkc(w0 * w0 * f, u0 * v0 * f);
    sh[2 * NX + x] = mkc(v0 * w0 * f, u0 * w0 * f);
    sh[3 * NX + x] = mkc(u1 * u1 * f, v1 * v1 * f);
    sh[4 * NX + x] = mkc(w1 * w1 * f, u1 * v1 * f);
    sh[5 * NX + x] = mkc(v1 * w1 * f, u1 * w1 * f);
  }
  if (want_cfl) {
    for (int o = 16; o > 0; o >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, o));
    if ((threadIdx.x & 31) == 0) atomicMax(cflmax, (unsigned long long)__double_as_longlong(cm));
  }
  __syncthreads();
  fft_lines<PPT>(sh, NX, 6, NX, twx, -1);
  for (int e = threadIdx.x; e < nxB * 3; e += blockDim.x) {
    int pl = e / nxB, ix = e - pl * nxB;
#pragma unroll
    for (int yy = 0; yy < 2; ++yy) {
      const cxd* L = sh + (pl + 3 * yy) * NX;
      cxd Zk = L[ix], Zm = L[ix == 0 ? 0 : NX - ix];
      cxd X = mkc(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y));
      cxd Y = mkc(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x));
      size_t o = ((size_t)kz * nyT + yt) * nxB * Ty + (size_t)ix * Ty + yi0 + yy;
      Pp[(size_t)(2 * pl) * cs + o] = X;
      Pp[(size_t)(2 * pl + 1) * cs + o] = Y;
    }
  }
}

// --------------------------------------------------------------- k_zfwd ----
// transpose_xTOz + FFT (src/hst_transforms.f90:135-139, src/hst_fft.f90:181-193)
// for a tile of Ty rows of one x mode of one product; keeps the 2nz+1
// retained z modes in the layout of a field without ghost rows.
template <int PPT>
__global__ void k_zfwd(Geometry g, const double2* __restrict__ Pp, double2* __restrict__ Q,
                       const double2* __restrict__ twz) {
  extern __shared__ double2 sh[];
  const int yt = blockIdx.x, ix = blockIdx.y, p = blockIdx.z;
  const int Ty = g.Ty, NZ = g.nzd, nz = g.nz, nzT = g.nzT, LS = NZ + 1;
  const int nyT = g.ny / Ty;
  const double2* src = Pp + (((size_t)p * NZ) * nyT + yt) * g.nxB * Ty + (size_t)ix * Ty;
  for (int e = threadIdx.x; e < NZ * Ty; e += blockDim.x) {
    int kz = e / Ty, yi = e - kz * Ty;
    sh[yi * LS + kz] = src[(size_t)kz * nyT * g.nxB * Ty + yi];
  }
  __syncthreads();
  fft_lines<PPT>(sh, NZ, Ty, LS, twz, -1);
  double2* dst = Q + ((size_t)p * g.ncol + (size_t)ix * nzT) * g.ny + yt * Ty;
  for (int e = threadIdx.x; e < nzT * Ty; e += blockDim.x) {
    int izi = e / Ty, yi = e - izi * Ty;
    int iz = izi - nz;
    int kz = iz >= 0 ? iz : NZ + iz;
    dst[(size_t)izi * g.ny + yi] = sh[yi * LS + kz];
  }
}

// ------------------------------------------------------------ k_column ----
struct ColumnArgs {
  Geometry g;
  PhysScalars ps;
  SubstepScalars sc;
  double2 *V1, *V2, *V3, *O1, *O2;
  const double2* Q;
  const double* der;
  const double* y;
  const double* gdamp;
};

__device__ __forceinline__ unsigned group_mask(int P) {
  if (P == 32) return 0xffffffffu;
  int lane = threadIdx.x & 31;
  return ((1u << P) - 1u) << ((lane / P) * P);
}

// a product spectrum at row q of its column, with the ghost images
__device__ __forceinline__ cxd q_at(const double2* __restrict__ Qc, int q, int ny, cxd ph) {
  if (q < 0) return cmul(Qc[q + ny], cconj(ph));
  if (q >= ny) return cmul(Qc[q - ny], ph);
  return Qc[q];
}

// write a line's interior and its four ghost rows (wrap_rows,
// src/hst_mpi.f90:340-355) into a field column; buf in LineGeom layout
template <int P>
__device__ __forceinline__ void store_with_ghosts(double2* __restrict__ col, const cxd* buf, const LineGeom& G, int ny,
                                                  cxd ph, int s, bool zero) {
  for (int r = s; r < ny; r += P) col[r + 2] = zero ? mkc(0, 0) : buf[G.at(r)];
  for (int k = s; k < 4; k += P) {
    // k = 0: row ny (row 0 ph), 1: row ny+1 (row 1 ph), 2: row -1 (row ny-1 conj), 3: row -2
    int srow = k == 0 ? 0 : (k == 1 ? 1 : (k == 2 ? ny - 1 : ny - 2));
    int drow = k == 0 ? ny : (k == 1 ? ny + 1 : (k == 2 ? -1 : -2));
    cxd v = zero ? mkc(0, 0) : buf[G.at(srow)];
    col[drow + 2] = cmul(v, k < 2 ? ph : cconj(ph));
  }
}

template <int P, bool EXACT, bool NONLIN>
__global__ void k_column(ColumnArgs a) {
  extern __shared__ double smem_d[];
  const Geometry& g = a.g;
  const int ny = g.ny, nz = g.nz, nzT = g.nzT;
  LineGeom G;
  G.n = ny;
  G.m = g.m;
  G.MS = g.MS;
  G.P = P;
  G.invm = (unsigned)((1u << 20) + g.m - 1) / (unsigned)g.m;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int col = blockIdx.x * groups + grp;
  if (col >= g.ncol) return;
  const unsigned gmask = group_mask(P);
  const int mi = g.m - 2;
  const int lineN = P * g.MS;
  const size_t per_group = (size_t)(EXACT ? 3 : 2) * lineN * 2 + (size_t)mi * 4 * P;  // doubles
  double* base = smem_d + per_group * grp;
  cxd* bufA = reinterpret_cast<cxd*>(base);
  cxd* bufB = bufA + lineN;
  cxd* bufC = bufB + lineN;  // EXACT only
  double* fac = base + (size_t)(EXACT ? 3 : 2) * lineN * 2;

  const int ix = col / nzT, iz = col - ix * nzT - nz;
  const bool c00 = (ix == 0 && iz == 0);
  const double al = a.ps.alfa0 * ix, be = a.ps.beta0 * iz;
  const double kk = al * al + be * be;
  const double ni = a.ps.ni;
  const SubstepScalars sc = a.sc;
  const double gcol = a.gdamp[col];
  const double gs = sc.gsoft * gcol;
  const bool masked = sc.damp_hard && gcol > 0.0;
  const size_t cb = (size_t)col * g.rows + 2;  // row 0 of the column
  const double2* __restrict__ V1c = a.V1 + cb;
  const double2* __restrict__ V2c = a.V2 + cb;
  const double2* __restrict__ V3c = a.V3 + cb;
  const double* __restrict__ der = a.der;
  const double kappa = sc.s2now * al - a.ps.S * be;  // (s2 i alfa - S i beta) / i
  const cxd ph_t = cexpi(-(al * sc.sx_t + be * sc.sz_t));

  // ---- right-hand sides, row by row (buildrhs_prepare :92-141, buildrhs :151-213)
  for (int r = s; r < ny; r += P) {
    double d0[5], d1[5], d2[5], d4[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      d0[j] = derv(der, ny, r, 0, j - 2);
      d1[j] = derv(der, ny, r, 1, j - 2);
      d2[j] = derv(der, ny, r, 2, j - 2);
      d4[j] = derv(der, ny, r, 3, j - 2);
    }
    // v equation
    cxd unkn = mkc(0, 0), impl = mkc(0, 0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      double helm = d2[j] - kk * d0[j];
      double biharm = d4[j] - 2.0 * kk * d2[j] + kk * kk * d0[j];
      cxd v = V2c[r + j - 2];
      unkn = mkc(unkn.x + helm * v.x, unkn.y + helm * v.y);
      double nb = ni * biharm;
      impl = mkc(impl.x + nb * v.x, impl.y + nb * v.y);
    }
    const size_t ro = (size_t)col * g.rows + 2 + r;
    cxd o2in = a.O2[ro];
    cxd r2 = mkc((sc.ode0 * unkn.x) / sc.deltat + impl.x - sc.ode2 * o2in.x - (sc.ode1 * gs) * unkn.x,
                 (sc.ode0 * unkn.y) / sc.deltat + impl.y - sc.ode2 * o2in.y - (sc.ode1 * gs) * unkn.y);
    cxd o2 = mkc(-gs * unkn.x, -gs * unkn.y);
    // eta equation (mean column: u, w packed)
    unkn = mkc(0, 0);
    impl = mkc(0, 0);
    cxd expl = mkc(0, 0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      double helm = d2[j] - kk * d0[j];
      cxd v1 = V1c[r + j - 2], v3 = V3c[r + j - 2], v2 = V2c[r + j - 2];
      cxd f;
      double w;
      if (c00) {
        f = mkc(v1.x, v3.x);
        w = ni * d2[j];
      } else {
        f = mkc(-be * v1.y + al * v3.y, be * v1.x - al * v3.x);
        w = ni * helm;
      }
      unkn = mkc(unkn.x + d0[j] * f.x, unkn.y + d0[j] * f.y);
      impl = mkc(impl.x + w * f.x, impl.y + w * f.y);
      double kd = kappa * d0[j];
      expl = mkc(expl.x - kd * v2.y, expl.y + kd * v2.x);
    }
    expl = mkc(expl.x - gs * unkn.x, expl.y - gs * unkn.y);
    cxd o1in = a.O1[ro];
    cxd r1 = mkc((sc.ode0 * unkn.x) / sc.deltat + impl.x - sc.ode2 * o1in.x + sc.ode1 * expl.x,
                 (sc.ode0 * unkn.y) / sc.deltat + impl.y - sc.ode2 * o1in.y + sc.ode1 * expl.y);
    cxd o1 = expl;
    if (NONLIN) {
#pragma unroll 1
      for (int p = 0; p < 6; ++p) {
        const double2* Qc = a.Q + ((size_t)p * g.ncol + col) * ny;
        cxd q0 = mkc(0, 0), q1 = mkc(0, 0), q2 = mkc(0, 0);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          cxd qv = q_at(Qc, r + j - 2, ny, ph_t);
          q0 = mkc(q0.x + d0[j] * qv.x, q0.y + d0[j] * qv.y);
          q1 = mkc(q1.x + d1[j] * qv.x, q1.y + d1[j] * qv.y);
          q2 = mkc(q2.x + d2[j] * qv.x, q2.y + d2[j] * qv.y);
        }
        cxd ru = mkc(0, 0), rw = mkc(0, 0), ex;
        switch (p) {
          case 0:  // uu
            ru = mkc(al * q0.y, -al * q0.x);
            ex = cscale(-(al * al), q1);
            break;
          case 1:  // vv
            ex = cscale(kk, q1);
            break;
          case 2:  // ww
            rw = mkc(be * q0.y, -be * q0.x);
            ex = cscale(-(be * be), q1);
            break;
          case 3:  // uv
            ru = cneg(q1);
            ex = mkc(-al * q2.y + -(al * kk) * q0.y, al * q2.x + (al * kk) * q0.x);
            break;
          case 4:  // vw
            rw = cneg(q1);
            ex = mkc(-be * q2.y + -(be * kk) * q0.y, be * q2.x + (be * kk) * q0.x);
            break;
          default:  // uw
            ru = mkc(be * q0.y, -be * q0.x);
            rw = mkc(al * q0.y, -al * q0.x);
            ex = cscale(-((2.0 * al) * be), q1);
            break;
        }
        r2 = mkc(r2.x + sc.ode1 * ex.x, r2.y + sc.ode1 * ex.y);
        o2 = cadd(o2, ex);
        cxd e;
        if (c00) e = mkc(ru.x, rw.x);
        else e = mkc(-be * ru.y + al * rw.y, be * ru.x - al * rw.x);
        r1 = mkc(r1.x + sc.ode1 * e.x, r1.y + sc.ode1 * e.y);
        o1 = cadd(o1, e);
      }
    }
    if (masked) {  // damping_mask (src/hst_damping.f90:119-133)
      r1 = r2 = o1 = o2 = mkc(0, 0);
    }
    if (!EXACT) {  // shear_shift, default form (src/hst_equations.f90:245-257)
      cxd f = cexpi(-(al * sc.dgx + be * sc.dgz) * a.y[r + 2]);
      r1 = cmul(r1, f);
      r2 = cmul(r2, f);
      o1 = cmul(o1, f);
      o2 = cmul(o2, f);
    }
    a.O1[ro] = o1;
    a.O2[ro] = o2;
    bufA[G.at(r)] = r1;
    bufB[G.at(r)] = r2;
  }
  __syncwarp(gmask);

  if (EXACT) {
    // shift_unweighted (src/hst_equations.f90:263-293) on rhs1, rhs2, old1,
    // old2: D0 solve with the wrap at t, node phase, ghost rows at t+dt_sub,
    // D0 stencil.  The scratch is this column of V1, dead here.
    const double th0 = al * sc.sx_t + be * sc.sz_t;
    const cxd ph1 = cexpi(-(al * sc.sx_n + be * sc.sz_n));
    double2* scr = a.V1 + (size_t)col * g.rows;
    for (int qi = 0; qi < 4; ++qi) {
      cxd* X = qi == 0 ? bufA : (qi == 1 ? bufB : bufC);
      double2* Og = qi == 2 ? a.O1 : a.O2;
      if (qi >= 2) {
        for (int r = s; r < ny; r += P) X[G.at(r)] = Og[(size_t)col * g.rows + 2 + r];
        __syncwarp(gmask);
      }
      group_solve<P>(K_D0, 0.0, ni, kk, th0, der, ny, G, X, fac, s, gmask);
      __syncwarp(gmask);
      for (int r = s; r < ny; r += P) {
        cxd v = cmul(X[G.at(r)], cexpi(-(al * sc.dgx + be * sc.dgz) * a.y[r + 2]));
        X[G.at(r)] = v;
      }
      __syncwarp(gmask);
      store_with_ghosts<P>(scr, X, G, ny, ph1, s, false);
      __syncwarp(gmask);
      for (int r = s; r < ny; r += P) {
        cxd acc = mkc(0, 0);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          double d0 = derv(der, ny, r, 0, j - 2);
          cxd v = scr[r + j];
          acc = mkc(acc.x + d0 * v.x, acc.y + d0 * v.y);
        }
        if (qi >= 2) Og[(size_t)col * g.rows + 2 + r] = acc;
        else X[G.at(r)] = acc;
      }
      __syncwarp(gmask);
    }
  }

  // ---- implicit solves (linsolve, src/hst_equations.f90:298-326)
  const double thn = al * sc.sx_n + be * sc.sz_n;
  const cxd phn = cexpi(-thn);
  group_solve<P>(K_D2V, sc.lambda, ni, kk, thn, der, ny, G, bufB, fac, s, gmask);
  __syncwarp(gmask);
  group_solve<P>(K_ETA, sc.lambda, ni, kk, thn, der, ny, G, bufA, fac, s, gmask);
  __syncwarp(gmask);
  double2* V2w = a.V2 + (size_t)col * g.rows;
  store_with_ghosts<P>(V2w, bufB, G, ny, phn, s, c00);
  __syncwarp(gmask);
  // D1 v through the ghost rows, then D0 (dv/dy) = D1 v (KIND_DY)
  for (int r = s; r < ny; r += P) {
    cxd acc = mkc(0, 0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      double d1 = derv(der, ny, r, 1, j - 2);
      cxd v = V2w[r + j];
      acc = mkc(acc.x + d1 * v.x, acc.y + d1 * v.y);
    }
    bufB[G.at(r)] = acc;
  }
  __syncwarp(gmask);
  group_solve<P>(K_DY, 0.0, ni, kk, thn, der, ny, G, bufB, fac, s, gmask);
  __syncwarp(gmask);
  // u, w from eta and dv/dy, into bufA (u) and bufB (w)
  for (int r = s; r < ny; r += P) {
    cxd eta = bufA[G.at(r)], dv = bufB[G.at(r)];
    cxd u, w;
    if (c00) {
      u = mkc(eta.x, 0.0);
      w = mkc(eta.y, 0.0);
    } else {
      // (i alfa dv - i beta eta) / k2, (i beta dv + i alfa eta) / k2
      u = mkc((-al * dv.y + be * eta.y) / kk, (al * dv.x - be * eta.x) / kk);
      w = mkc((-be * dv.y - al * eta.y) / kk, (be * dv.x + al * eta.x) / kk);
    }
    bufA[G.at(r)] = u;
    bufB[G.at(r)] = w;
  }
  __syncwarp(gmask);
  store_with_ghosts<P>(a.V1 + (size_t)col * g.rows, bufA, G, ny, phn, s, false);
  store_with_ghosts<P>(a.V3 + (size_t)col * g.rows, bufB, G, ny, phn, s, false);
}

// --------------------------------------------------------- k_line_solve ----
// line_solve (src/hst_linsolve.f90:147-233) for every Fourier column.
template <int P>
__global__ void k_line_solve(Geometry g, PhysScalars ps, int sys, double lambda, const double2* __restrict__ src,
                             double2* __restrict__ dst, double sx, double sz, const double* __restrict__ der) {
  extern __shared__ double smem_d[];
  const int ny = g.ny, nz = g.nz, nzT = g.nzT;
  LineGeom G;
  G.n = ny;
  G.m = g.m;
  G.MS = g.MS;
  G.P = P;
  G.invm = (unsigned)((1u << 20) + g.m - 1) / (unsigned)g.m;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int col = blockIdx.x * groups + grp;
  if (col >= g.ncol) return;
  const unsigned gmask = group_mask(P);
  const int mi = g.m - 2;
  const int lineN = P * g.MS;
  double* base = smem_d + ((size_t)lineN * 2 + (size_t)mi * 4 * P) * grp;
  cxd* buf = reinterpret_cast<cxd*>(base);
  double* fac = base + (size_t)lineN * 2;
  const int ix = col / nzT, iz = col - ix * nzT - nz;
  const double al = ps.alfa0 * ix, be = ps.beta0 * iz;
  const double kk = al * al + be * be;
  const double2* sc = src + (size_t)col * g.rows + 2;
  double2* dc = dst + (size_t)col * g.rows + 2;
  for (int r = s; r < ny; r += P) {
    cxd v;
    if (sys == K_DY) {
      v = mkc(0, 0);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        double d1 = derv(der, ny, r, 1, j - 2);
        cxd q = sc[r + j - 2];
        v = mkc(v.x + d1 * q.x, v.y + d1 * q.y);
      }
    } else {
      v = sc[r];
    }
    buf[G.at(r)] = v;
  }
  __syncwarp(gmask);
  group_solve<P>(sys, lambda, ps.ni, kk, al * sx + be * sz, der, ny, G, buf, fac, s, gmask);
  __syncwarp(gmask);
  const bool c00 = (ix == 0 && iz == 0);
  if (c00 && sys == K_POISSON) return;
  for (int r = s; r < ny; r += P) dc[r] = (c00 && sys == K_D2V) ? mkc(0, 0) : buf[G.at(r)];
}

// -------------------------------------------------------- k_fill_ghosts ----
__global__ void k_fill_ghosts(Geometry g, PhysScalars ps, double2* __restrict__ f, double sx, double sz) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.ncol) return;
  const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
  const cxd ph = cexpi(-(ps.alfa0 * ix * sx + ps.beta0 * iz * sz));
  double2* c = f + (size_t)col * g.rows + 2;
  const int ny = g.ny;
  c[ny] = cmul(c[0], ph);
  c[ny + 1] = cmul(c[1], ph);
  c[-1] = cmul(c[ny - 1], cconj(ph));
  c[-2] = cmul(c[ny - 2], cconj(ph));
}

// -------------------------------------------------------------- launchers ----
static int fft_threads(int points, int ppt) {
  int t = (points + ppt - 1) / ppt;
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

#define HST_PPT 8

cudaError_t launch_zinv(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  int T = fft_threads(g.nzd * g.Ty, HST_PPT);
  size_t smem = (size_t)g.Ty * (g.nzd + 1) * sizeof(double2);
  cudaFuncSetAttribute(k_zinv<HST_PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  dim3 grid(g.ny / g.Ty, g.nxB, 3);
  k_zinv<HST_PPT><<<grid, T, smem, st>>>(g, d.F[0], d.F[1], d.F[2], d.Z, d.twz);
  return cudaGetLastError();
}

cudaError_t launch_xprod(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int want_cfl,
                         cudaStream_t st) {
  int NX = 2 * g.nxd;
  int T = fft_threads(6 * NX, HST_PPT);
  size_t smem = (size_t)6 * NX * sizeof(double2);
  cudaFuncSetAttribute(k_xprod<HST_PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  dim3 grid(g.ny / 2, g.nzd);
  k_xprod<HST_PPT><<<grid, T, smem, st>>>(g, d.Z, d.Pp, d.twx, d.dyl, ph, want_cfl, d.cfl);
  return cudaGetLastError();
}

cudaError_t launch_zfwd(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  int T = fft_threads(g.nzd * g.Ty, HST_PPT);
  size_t smem = (size_t)g.Ty * (g.nzd + 1) * sizeof(double2);
  cudaFuncSetAttribute(k_zfwd<HST_PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  dim3 grid(g.ny / g.Ty, g.nxB, 6);
  k_zfwd<HST_PPT><<<grid, T, smem, st>>>(g, d.Pp, d.Q, d.twz);
  return cudaGetLastError();
}

size_t column_smem_bytes(const Geometry& g, int exact) {
  size_t lineN = (size_t)g.P * g.MS;
  return ((exact ? 3 : 2) * lineN * 2 + (size_t)(g.m - 2) * 4 * g.P) * sizeof(double);
}

template <int P, bool EXACT, bool NONLIN>
static cudaError_t launch_column_t(const ColumnArgs& a, cudaStream_t st) {
  const Geometry& g = a.g;
  int T = P >= 32 ? 32 : 64;
  if (T < P) T = P;
  int groups = T / P;
  size_t per = column_smem_bytes(g, EXACT);
  size_t smem = per * groups;
  cudaFuncSetAttribute(k_column<P, EXACT, NONLIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int blocks = (g.ncol + groups - 1) / groups;
  k_column<P, EXACT, NONLIN><<<blocks, T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int P>
static cudaError_t launch_column_p(const ColumnArgs& a, int exact, int nonlin, cudaStream_t st) {
  if (exact) return nonlin ? launch_column_t<P, true, true>(a, st) : launch_column_t<P, true, false>(a, st);
  return nonlin ? launch_column_t<P, false, true>(a, st) : launch_column_t<P, false, false>(a, st);
}

cudaError_t launch_column(const Geometry& g, const DeviceState& d, const PhysScalars& ph, const SubstepScalars& sc,
                          int exact, int nonlin, cudaStream_t st) {
  ColumnArgs a;
  a.g = g;
  a.ps = ph;
  a.sc = sc;
  a.V1 = d.F[0];
  a.V2 = d.F[1];
  a.V3 = d.F[2];
  a.O1 = d.F[3];
  a.O2 = d.F[4];
  a.Q = d.Q;
  a.der = d.der;
  a.y = d.y;
  a.gdamp = d.gdamp;
  switch (g.P) {
    case 2: return launch_column_p<2>(a, exact, nonlin, st);
    case 4: return launch_column_p<4>(a, exact, nonlin, st);
    case 8: return launch_column_p<8>(a, exact, nonlin, st);
    case 16: return launch_column_p<16>(a, exact, nonlin, st);
    case 32: return launch_column_p<32>(a, exact, nonlin, st);
  }
  return cudaErrorInvalidValue;
}

template <int P>
static cudaError_t launch_line_solve_t(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int sys,
                                       double lambda, int src, int dst, double sx, double sz, cudaStream_t st) {
  int T = P >= 32 ? 32 : 64;
  if (T < P) T = P;
  int groups = T / P;
  size_t per = ((size_t)P * g.MS * 2 + (size_t)(g.m - 2) * 4 * P) * sizeof(double);
  cudaFuncSetAttribute(k_line_solve<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int blocks = (g.ncol + groups - 1) / groups;
  k_line_solve<P><<<blocks, T, per * groups, st>>>(g, ph, sys, lambda, d.F[src], d.F[dst], sx, sz, d.der);
  return cudaGetLastError();
}

cudaError_t launch_line_solve(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int sys, double lambda,
                              int src, int dst, double sx, double sz, cudaStream_t st) {
  switch (g.P) {
    case 2: return launch_line_solve_t<2>(g, d, ph, sys, lambda, src, dst, sx, sz, st);
    case 4: return launch_line_solve_t<4>(g, d, ph, sys, lambda, src, dst, sx, sz, st);
    case 8: return launch_line_solve_t<8>(g, d, ph, sys, lambda, src, dst, sx, sz, st);
    case 16: return launch_line_solve_t<16>(g, d, ph, sys, lambda, src, dst, sx, sz, st);
    case 32: return launch_line_solve_t<32>(g, d, ph, sys, lambda, src, dst, sx, sz, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fill_ghosts(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int field, double sx,
                               double sz, cudaStream_t st) {
  int T = 128;
  k_fill_ghosts<<<(g.ncol + T - 1) / T, T, 0, st>>>(g, ph, d.F[field], sx, sz);
  return cudaGetLastError();
}

}  // namespace hst
