// The column kernels of the hst substep on sm_100a (FP64); the transforms
// (k_zinv, k_xprod, k_zfwd) are in hst_transforms.cu.
//
//   k_column     one warp group per Fourier column: the right-hand sides of
//                buildrhs_prepare and buildrhs, the hard damping mask, the
//                mean-shear phase shift (both forms), the D2V, ETA and DY
//                line solves, u and w, all ghost rows; or either half of it
//   k_rhs_tiled  the right-hand-side half as a streaming kernel fed by TMA
//                bulk copies
//   k_line_solve, k_fill_ghosts: the single operations for the drop-in
//                interface and the tests
//
// Only the ny interior rows are transformed.  The products in the four
// ghost rows, which the reference transforms as well
// (src/hst_transforms.f90:3-6), are the shear-periodic images of the
// interior ones: the 3/2 rule makes the retained product modes exact, so the
// image of row k is row k times the wrap phase, which the right-hand-side
// stage applies when it reads them.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "hst_dev.cuh"
#include "hst_internal.h"
#include "hst_rhs.cuh"

namespace hst {

// ------------------------------------------------------------ k_column ----
struct ColumnArgs {
  Geometry g;
  PhysScalars ps;
  SubstepScalars sc;
  double2 *V1, *V2, *V3, *O1, *O2, *R1, *R2;
  const double2* Q;
  const double2* Qg;  // the ghost rows' product spectra [6][ncol][4] (null: their wrap images)
  const double* der;
  const double* derS;
  const double* derU;  // the distinct rows of der (DerRows), or null
  const int* derI;
  int nderU;
  const double* d0tab;
  const double* y;
  const double* gdamp;
  int* err;   // set to 1 by a kernel whose bounded wait ran out
  int tiled;  // the right-hand sides through k_rhs_tiled
  const DeviceState* dstate;  // host side only: the launch's context state
  double* facg;               // global factor scratch of the persistent form (null: shared memory)
  int fac_groups;             // groups that scratch holds
};

__device__ __forceinline__ unsigned group_mask(int P) {
  if (P == 32) return 0xffffffffu;
  int lane = threadIdx.x & 31;
  return ((1u << P) - 1u) << ((lane / P) * P);
}

// a product spectrum at row q of its column, with the ghost images (or,
// with Qgc, the ghost rows' own transforms: rows -2, -1, ny, ny+1 there)
__device__ __forceinline__ cxd q_at(const double2* __restrict__ Qc, const double2* __restrict__ Qgc, int q, int ny,
                                    cxd ph) {
  if (q < 0) return Qgc ? Qgc[q + 2] : cmul(Qc[q + ny], cconj(ph));
  if (q >= ny) return Qgc ? Qgc[q - ny + 2] : cmul(Qc[q - ny], ph);
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

// MODE 0: everything in one kernel.  MODE 1: only the right-hand sides,
// streamed row by row (P = 32 lanes walk the rows of one column; no shared
// memory), written to RHS1/RHS2.  MODE 2: the rest, reading RHS1/RHS2.
// MODE 3 (EXACT only): the exact_shift shear shift of RHS1/2 and OLD1/2 in
// place and nothing else (the per-piece shear_shift).
enum { COL_FUSED = 0, COL_RHS = 1, COL_SOLVE = 2, COL_SHIFT = 3 };
// MODE 5, 6: the solves of MODE 2 in two passes of one line each (the v
// half, then the eta half with u and w), for the persistent form only
enum { COL_SOLVE_V = 5, COL_SOLVE_ETA = 6 };

// The work on one Fourier column (the body of k_column): bufA, bufB (bufC)
// the group's line buffers in shared memory, fac its factor scratch (the
// back-substitution factors of the D2V and ETA solves, (m-2) x 4 x P
// doubles, in shared or in global memory).
template <int P, bool EXACT, bool NONLIN, int MODE>
__device__ __forceinline__ void column_body(const ColumnArgs& a, int cg, int s, cxd* bufA, cxd* bufB, cxd* bufC,
                                            double* fac) {
  const Geometry& g = a.g;
  // cg: the column over all members (the fields' column index); col: the
  // Fourier column within its member
  const int mem = cg / g.ncol, col = cg - mem * g.ncol;
  const int ny = g.ny, nz = g.nz, nzT = g.nzT;
  LineGeom G;
  G.n = ny;
  G.m = g.m;
  G.MS = g.MS;
  G.P = P;
  G.invm = (unsigned)((1u << 20) + g.m - 1) / (unsigned)g.m;
  const unsigned gmask = group_mask(P);
  const int ix = col / nzT, iz = col - ix * nzT - nz;
  const bool c00 = (ix == 0 && iz == 0);
  const double al = a.ps.alfa0 * ix, be = a.ps.beta0 * iz;
  const double kk = al * al + be * be;
  const double ni = a.ps.ni;
  const SubstepScalars sc = a.sc;
  const size_t cb = (size_t)cg * g.rows + 2;  // row 0 of the column
  const double2* __restrict__ V1c = a.V1 + cb;
  const double2* __restrict__ V2c = a.V2 + cb;
  const double2* __restrict__ V3c = a.V3 + cb;
  const double* __restrict__ der = a.der;
  const SlabDer DS = {a.derS, g.m, P};

  // ---- right-hand sides, row by row (buildrhs_prepare :92-141, buildrhs :151-213)
  if (MODE == COL_FUSED || MODE == COL_RHS) {
    const ColConst cc = col_const(col, g, a.ps, sc, a.gdamp);
    const double2* Qc = a.Q + ((size_t)mem * 6 * g.ncol + col) * ny;
    const size_t qs = (size_t)g.ncol * ny;
#pragma unroll 1
    for (int r = s; r < ny; r += P) {
      auto tv = [&](int c, int j) -> cxd { return (c == 0 ? V1c : (c == 1 ? V2c : V3c))[r + j - 2]; };
      auto tq = [&](int p, int j) -> cxd {
        return q_at(Qc + p * qs, a.Qg ? a.Qg + (((size_t)mem * 6 + p) * g.ncol + col) * 4 : nullptr, r + j - 2, ny,
                    cc.ph_t);
      };
      const size_t ro = cb + r;
      cxd r1, r2, o1, o2;
      const double yr = a.y[r + 2];
      auto fsh = [&]() { return cexpi(-(cc.al * sc.dgx + cc.be * sc.dgz) * yr); };
      rhs_point<NONLIN, EXACT>(cc, sc, DerFull{der, ny}, ny, r, fsh, tv, tq, a.O1[ro], a.O2[ro], r1, r2, o1, o2);
      a.O1[ro] = o1;
      a.O2[ro] = o2;
      if (MODE == COL_RHS) {
        a.R1[ro] = r1;
        a.R2[ro] = r2;
      } else {
        bufA[G.at(r)] = r1;
        bufB[G.at(r)] = r2;
      }
    }
  }
  if (MODE == COL_RHS) return;

  // shift_unweighted (src/hst_equations.f90:263-293) on rhs1, rhs2, old1,
  // old2 (EXACT): D0 solve with the wrap at t, node phase, ghost rows at
  // t+dt_sub, D0 stencil.  The scratch is this column of V1 (and V3), dead
  // here.  The split stage shifts old1 and old2 as one pair of lines
  // (through bufA, bufB and back to OLD1, OLD2), then rhs1 and rhs2, so
  // that it holds two lines, not three; the pairs share the solves' table
  // loads and the phases.
  const double th0 = al * sc.sx_t + be * sc.sz_t;
  double2* scr = a.V1 + (size_t)cg * g.rows;
  if ((MODE == COL_SOLVE || MODE == COL_SHIFT) && EXACT) {
    const double gx = al * sc.dgx + be * sc.dgz;
    const cxd phs = cexpi(-(al * sc.sx_n + be * sc.sz_n));
    double2* scr2 = a.V3 + (size_t)cg * g.rows;
    cxd* const bufs[2] = {bufA, bufB};
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      const double2* s1 = pass == 0 ? a.O1 : a.R1;  // OLD1, OLD2 are written back below
      const double2* s2 = pass == 0 ? a.O2 : a.R2;
      for (int r = s; r < ny; r += P) {
        bufA[G.at(r)] = s1[cb + r];
        bufB[G.at(r)] = s2[cb + r];
      }
      __syncwarp(gmask);
      group_solve_d0<P, 2>(th0, a.d0tab, G, bufs, s, gmask);
      __syncwarp(gmask);
      // the node phase exp(-i gx y(r)); on a uniform grid by one product a
      // row from the lane's first row (rows s, s + P, ... are P dy apart)
      cxd e = cexpi(-gx * a.y[s + 2]);
      const cxd estep = sc.yuni ? cexpi(-gx * (sc.ytile * (P / 32.0))) : mkc(1.0, 0.0);
      for (int r = s; r < ny; r += P) {
        if (!sc.yuni && r != s) e = cexpi(-gx * a.y[r + 2]);
        bufA[G.at(r)] = cmul(bufA[G.at(r)], e);
        bufB[G.at(r)] = cmul(bufB[G.at(r)], e);
        e = cmul(e, estep);
      }
      __syncwarp(gmask);
      store_with_ghosts<P>(scr, bufA, G, ny, phs, s, false);
      store_with_ghosts<P>(scr2, bufB, G, ny, phs, s, false);
      __syncwarp(gmask);
      for (int r = s; r < ny; r += P) {
        cxd acc1 = mkc(0, 0), acc2 = mkc(0, 0);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          const double d0 = derv(der, ny, r, 0, j - 2);
          const cxd v1 = scr[r + j], v2 = scr2[r + j];
          acc1 = mkc(acc1.x + d0 * v1.x, acc1.y + d0 * v1.y);
          acc2 = mkc(acc2.x + d0 * v2.x, acc2.y + d0 * v2.y);
        }
        if (pass == 0) {
          a.O1[cb + r] = acc1;
          a.O2[cb + r] = acc2;
        } else if (MODE == COL_SHIFT) {
          a.R1[cb + r] = acc1;
          a.R2[cb + r] = acc2;
        } else {
          bufA[G.at(r)] = acc1;
          bufB[G.at(r)] = acc2;
        }
      }
      __syncwarp(gmask);
    }
  }
  if (MODE == COL_SHIFT) return;
  const int nseq = MODE == COL_SOLVE ? 1 : (EXACT ? 4 : 0);
#pragma unroll 1
  for (int k = (MODE == COL_SOLVE && EXACT) ? nseq : 0; k < nseq; ++k) {
    const int qi = MODE == COL_SOLVE ? -1 : k;
    if (qi < 0) {
      for (int r = s; r < ny; r += P) {
        bufA[G.at(r)] = a.R1[cb + r];
        bufB[G.at(r)] = a.R2[cb + r];
      }
      __syncwarp(gmask);
      continue;
    }
    cxd* X = qi == 0 ? bufA : (qi == 1 ? bufB : (MODE == COL_SOLVE ? bufA : bufC));
    double2* Og = qi == 2 ? a.O1 : a.O2;
    if (qi >= 2) {
      for (int r = s; r < ny; r += P) X[G.at(r)] = Og[cb + r];
      __syncwarp(gmask);
    }
    {
      cxd* const bufs[1] = {X};
      group_solve_d0<P, 1>(th0, a.d0tab, G, bufs, s, gmask);
    }
    __syncwarp(gmask);
    for (int r = s; r < ny; r += P) {
      cxd v = cmul(X[G.at(r)], cexpi(-(al * sc.dgx + be * sc.dgz) * a.y[r + 2]));
      X[G.at(r)] = v;
    }
    __syncwarp(gmask);
    store_with_ghosts<P>(scr, X, G, ny, cexpi(-(al * sc.sx_n + be * sc.sz_n)), s, false);
    __syncwarp(gmask);
    for (int r = s; r < ny; r += P) {
      cxd acc = mkc(0, 0);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        double d0 = derv(der, ny, r, 0, j - 2);
        cxd v = scr[r + j];
        acc = mkc(acc.x + d0 * v.x, acc.y + d0 * v.y);
      }
      if (qi >= 2) Og[cb + r] = acc;
      else X[G.at(r)] = acc;
    }
    __syncwarp(gmask);
  }

  // ---- implicit solves (linsolve, src/hst_equations.f90:298-326)
  const double thn = al * sc.sx_n + be * sc.sz_n;
  const cxd phn = cexpi(-thn);
  group_solve<P>(K_D2V, sc.lambda, ni, kk, thn, DS, G, bufB, fac, s, gmask);
  __syncwarp(gmask);
  group_solve<P>(K_ETA, sc.lambda, ni, kk, thn, DS, G, bufA, fac, s, gmask);
  __syncwarp(gmask);
  double2* V2w = a.V2 + (size_t)cg * g.rows;
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
  {
    cxd* const bufs[1] = {bufB};
    group_solve_d0<P, 1>(thn, a.d0tab, G, bufs, s, gmask);
  }
  __syncwarp(gmask);
  // u, w from eta and dv/dy, into bufA (u) and bufB (w)
  const double rkk = c00 ? 0.0 : 1.0 / kk;
  for (int r = s; r < ny; r += P) {
    cxd eta = bufA[G.at(r)], dv = bufB[G.at(r)];
    cxd u, w;
    if (c00) {
      u = mkc(eta.x, 0.0);
      w = mkc(eta.y, 0.0);
    } else {
      // (i alfa dv - i beta eta) / k2, (i beta dv + i alfa eta) / k2
      u = mkc((-al * dv.y + be * eta.y) * rkk, (al * dv.x - be * eta.x) * rkk);
      w = mkc((-be * dv.y - al * eta.y) * rkk, (be * dv.x + al * eta.x) * rkk);
    }
    bufA[G.at(r)] = u;
    bufB[G.at(r)] = w;
  }
  __syncwarp(gmask);
  store_with_ghosts<P>(a.V1 + (size_t)cg * g.rows, bufA, G, ny, phn, s, false);
  store_with_ghosts<P>(a.V3 + (size_t)cg * g.rows, bufB, G, ny, phn, s, false);
}

// The five-point stencil n (0: D0, 1: D1) of a line held slab by slab in
// shared memory, in place: lane s computes rows s m .. s m + m - 1 of its
// slab with a sliding window, the two rows beyond each end of the slab from
// the neighbouring lanes (by shuffle, taken before anything is written) and,
// across the box edge, the shear-periodic ghost images f(ny + k) = f(k) ph,
// f(-k) = f(ny - k) conj(ph) (wrap_rows, src/hst_mpi.f90:340-355).  The sum
// runs over j = -2..2 in order, as the reference's stencils do.
template <int P, class DST>
__device__ __forceinline__ void slab_stencil(int n, const DST& DS, cxd* sb, int m, int s, cxd ph, unsigned gmask) {
  const cxd f0 = sb[0], f1 = sb[1], l0 = sb[m - 2], l1 = sb[m - 1];
  const int up = (s + 1) & (P - 1), dn = (s - 1) & (P - 1);
  cxd a0 = shfl_c(gmask, f0, up, P), a1 = shfl_c(gmask, f1, up, P);  // rows s m + m, s m + m + 1
  cxd b0 = shfl_c(gmask, l0, dn, P), b1 = shfl_c(gmask, l1, dn, P);  // rows s m - 2, s m - 1
  if (s == P - 1) {
    a0 = cmul(a0, ph);
    a1 = cmul(a1, ph);
  }
  if (s == 0) {
    b0 = cmul(b0, cconj(ph));
    b1 = cmul(b1, cconj(ph));
  }
  cxd w0 = b0, w1 = b1, w2 = f0, w3 = f1, w4 = sb[2];
#pragma unroll 2
  for (int i = 0; i < m; ++i) {
    const double c0 = DS(s, i, n, 0), c1 = DS(s, i, n, 1), c2 = DS(s, i, n, 2), c3 = DS(s, i, n, 3),
                 c4 = DS(s, i, n, 4);
    cxd acc = mkc(0, 0);
    acc = mkc(acc.x + c0 * w0.x, acc.y + c0 * w0.y);
    acc = mkc(acc.x + c1 * w1.x, acc.y + c1 * w1.y);
    acc = mkc(acc.x + c2 * w2.x, acc.y + c2 * w2.y);
    acc = mkc(acc.x + c3 * w3.x, acc.y + c3 * w3.y);
    acc = mkc(acc.x + c4 * w4.x, acc.y + c4 * w4.y);
    const int nx = i + 3;
    const cxd nxt = nx < m ? sb[nx] : (nx == m ? a0 : a1);
    sb[i] = acc;
    w0 = w1;
    w1 = w2;
    w2 = w3;
    w3 = w4;
    w4 = nxt;
  }
}


// The solve stage on one column, for MODE COL_SOLVE (and COL_SHIFT: the
// exact_shift shift alone) with the lines and every intermediate in shared
// memory: no scratch column of V is written and read back.
//   EXACT: shift_unweighted (src/hst_equations.f90:263-293) of old1, old2,
//          rhs1, rhs2, one line at a time: D0 solve with the wrap at t
//          (factored table), node phase exp(-i gx y), D0 stencil with the
//          ghost images at t + dt_sub; old1, old2 back to OLD1, OLD2.
//   then linsolve (:298-326): D2V and ETA solves, v with its ghost rows to
//   V2, D1 stencil of v and the DY solve (table) in place, u and w, V1 and
//   V3 with their ghost rows.
// SHT (the shift alone): the D0 table and the D0 slice of der are read from
// the block's shared copies d0s and der0s instead of global memory
template <int P, bool EXACT, bool SHIFT_ONLY, bool SHT = false>
__device__ __forceinline__ void column_solve_body(const ColumnArgs& a, int cg, int s, cxd* bufA, cxd* bufB,
                                                  double* fac, const double* d0s = nullptr,
                                                  const double* der0s = nullptr) {
  static_assert(!SHT || SHIFT_ONLY, "shared tables for the shift alone");
  const Geometry& g = a.g;
  const int mem = cg / g.ncol, col = cg - mem * g.ncol;
  const int ny = g.ny, nz = g.nz, nzT = g.nzT, m = g.m;
  LineGeom G;
  G.n = ny;
  G.m = m;
  G.MS = g.MS;
  G.P = P;
  G.invm = (unsigned)((1u << 20) + m - 1) / (unsigned)m;
  const unsigned gmask = group_mask(P);
  const int ix = col / nzT, iz = col - ix * nzT - nz;
  const bool c00 = (ix == 0 && iz == 0);
  const double al = a.ps.alfa0 * ix, be = a.ps.beta0 * iz;
  const double kk = al * al + be * be;
  const SubstepScalars& sc = a.sc;
  const size_t cb = (size_t)cg * g.rows + 2;  // row 0 of the column
  const SlabDer DS = {a.derS, m, P};
  cxd* const sA = bufA + s * G.MS;  // this lane's slab
  cxd* const sB = bufB + s * G.MS;

  if (EXACT) {
    const double th0 = al * sc.sx_t + be * sc.sz_t;
    const double gx = al * sc.dgx + be * sc.dgz;
    const cxd phs = cexpi(-(al * sc.sx_n + be * sc.sz_n));
    // the node phase of the slab's first row; on a uniform grid the next
    // rows follow by one complex product each (dy = ly / ny apart)
    const cxd e0 = cexpi(-gx * a.y[s * m + 2]);
    const cxd estep = sc.yuni ? cexpi(-gx * (sc.ytile / 32.0)) : mkc(1.0, 0.0);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      // q = 0, 1: old1, old2 (back to OLD1, OLD2 through bufA); 2: rhs1
      // (kept in bufA); 3: rhs2 (kept in bufB; the shift alone stores each
      // line before it loads the next, all through bufA)
      cxd* X = q == 3 && !SHIFT_ONLY ? bufB : bufA;
      cxd* sX = q == 3 && !SHIFT_ONLY ? sB : sA;
      const double2* src = q == 0 ? a.O1 : (q == 1 ? a.O2 : (q == 2 ? a.R1 : a.R2));
      for (int r = s; r < ny; r += P) X[G.at(r)] = src[cb + r];
      __syncwarp(gmask);
      {
        cxd* const bufs[1] = {X};
        group_solve_d0<P, 1, SHT>(th0, SHT ? d0s : a.d0tab, G, bufs, s, gmask);
      }
      __syncwarp(gmask);
      cxd e = e0;
      for (int i = 0; i < m; ++i) {
        if (!sc.yuni && i > 0) e = cexpi(-gx * a.y[s * m + i + 2]);
        sX[i] = cmul(sX[i], e);
        e = cmul(e, estep);
      }
      __syncwarp(gmask);
      if constexpr (SHT)
        slab_stencil<P>(0, SlabDerT<true>{der0s, m, P}, sX, m, s, phs, gmask);
      else
        slab_stencil<P>(0, DS, sX, m, s, phs, gmask);
      __syncwarp(gmask);
      if (q < 2 || SHIFT_ONLY) {
        double2* dst = q == 0 ? a.O1 : (q == 1 ? a.O2 : (q == 2 ? a.R1 : a.R2));
        for (int r = s; r < ny; r += P) dst[cb + r] = X[G.at(r)];
        __syncwarp(gmask);
      }
    }
    if (SHIFT_ONLY) return;
  } else {
    for (int r = s; r < ny; r += P) {
      bufA[G.at(r)] = a.R1[cb + r];
      bufB[G.at(r)] = a.R2[cb + r];
    }
    __syncwarp(gmask);
  }

  // ---- implicit solves (linsolve, src/hst_equations.f90:298-326)
  const double thn = al * sc.sx_n + be * sc.sz_n;
  const cxd phn = cexpi(-thn);
  group_solve<P>(K_D2V, sc.lambda, a.ps.ni, kk, thn, DS, G, bufB, fac, s, gmask);
  __syncwarp(gmask);
  group_solve<P>(K_ETA, sc.lambda, a.ps.ni, kk, thn, DS, G, bufA, fac, s, gmask);
  __syncwarp(gmask);
  store_with_ghosts<P>(a.V2 + (size_t)cg * g.rows, bufB, G, ny, phn, s, c00);
  // D1 v through the ghost rows, then D0 (dv/dy) = D1 v (KIND_DY); the (0,0)
  // column's v is zero
  if (c00)
    for (int i = 0; i < m; ++i) sB[i] = mkc(0, 0);
  __syncwarp(gmask);
  slab_stencil<P>(1, DS, sB, m, s, phn, gmask);
  __syncwarp(gmask);
  {
    cxd* const bufs[1] = {bufB};
    group_solve_d0<P, 1>(thn, a.d0tab, G, bufs, s, gmask);
  }
  __syncwarp(gmask);
  // u, w from eta and dv/dy, into bufA (u) and bufB (w)
  const double rkk = c00 ? 0.0 : 1.0 / kk;
  for (int i = 0; i < m; ++i) {
    const cxd eta = sA[i], dv = sB[i];
    cxd u, w;
    if (c00) {
      u = mkc(eta.x, 0.0);
      w = mkc(eta.y, 0.0);
    } else {
      // (i alfa dv - i beta eta) / k2, (i beta dv + i alfa eta) / k2
      u = mkc((-al * dv.y + be * eta.y) * rkk, (al * dv.x - be * eta.x) * rkk);
      w = mkc((-be * dv.y - al * eta.y) * rkk, (be * dv.x + al * eta.x) * rkk);
    }
    sA[i] = u;
    sB[i] = w;
  }
  __syncwarp(gmask);
  store_with_ghosts<P>(a.V1 + (size_t)cg * g.rows, bufA, G, ny, phn, s, false);
  store_with_ghosts<P>(a.V3 + (size_t)cg * g.rows, bufB, G, ny, phn, s, false);
}

// One group of P lanes per Fourier column, every intermediate in shared
// memory, the factor scratch in shared memory after the lines (the fused
// stage, the streamed right-hand sides, and the solve stage when the context
// has no global factor scratch).
template <int P, bool EXACT, bool NONLIN, int MODE>
__global__ void k_column(ColumnArgs a) {
  extern __shared__ double smem_d[];
  const Geometry& g = a.g;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int col = blockIdx.x * groups + grp;  // over all members
  if (col >= g.ncol * g.nmem) return;
  const int mi = g.m - 2;
  const int lineN = P * g.MS;
  constexpr int NL = (EXACT && MODE == COL_FUSED) ? 3 : 2;  // lines held
  const size_t per_group = (size_t)NL * lineN * 2 + (size_t)mi * 4 * P;  // doubles
  double* base = smem_d + per_group * grp;
  cxd* bufA = reinterpret_cast<cxd*>(base);
  cxd* bufB = bufA + lineN;
  cxd* bufC = bufB + lineN;  // EXACT and COL_FUSED only
  column_body<P, EXACT, NONLIN, MODE>(a, col, s, bufA, bufB, bufC, base + (size_t)NL * lineN * 2);
}

// The solves of column_solve_body in two passes of one line each, so that a
// group holds one line of shared memory: HALF 0 solves D2V for v (V2 with
// its ghost rows), takes D1 v and solves DY for dv/dy, which it leaves in
// V1's interior rows; HALF 1 solves ETA, reads dv/dy back row by row and
// writes u over it (then u's ghost rows) and w (V3 with its ghost rows).
// The same operations in the same order as the one-pass form, so the same
// bits.
// SHT: der (its first nsl slices, D0 D1 D2 D4 in that order) read from the
// block's shared copy ders
template <int P, int HALF, bool SHT = false>
__device__ __forceinline__ void column_solve_half(const ColumnArgs& a, int cg, int s, cxd* buf, double* fac,
                                                  const double* ders = nullptr) {
  const Geometry& g = a.g;
  const int mem = cg / g.ncol, col = cg - mem * g.ncol;
  const int ny = g.ny, nz = g.nz, nzT = g.nzT, m = g.m;
  LineGeom G;
  G.n = ny;
  G.m = m;
  G.MS = g.MS;
  G.P = P;
  G.invm = (unsigned)((1u << 20) + m - 1) / (unsigned)m;
  const unsigned gmask = group_mask(P);
  const int ix = col / nzT, iz = col - ix * nzT - nz;
  const bool c00 = (ix == 0 && iz == 0);
  const double al = a.ps.alfa0 * ix, be = a.ps.beta0 * iz;
  const double kk = al * al + be * be;
  const SubstepScalars& sc = a.sc;
  const size_t cb = (size_t)cg * g.rows + 2;  // row 0 of the column
  const SlabDerT<SHT> DS = {SHT ? ders : a.derS, m, P};
  cxd* const sb = buf + s * G.MS;
  const double thn = al * sc.sx_n + be * sc.sz_n;
  const cxd phn = cexpi(-thn);
  double2* const v1 = a.V1 + (size_t)cg * g.rows;
  if (HALF == 0) {
    for (int r = s; r < ny; r += P) buf[G.at(r)] = a.R2[cb + r];
    __syncwarp(gmask);
    group_solve<P>(K_D2V, sc.lambda, a.ps.ni, kk, thn, DS, G, buf, fac, s, gmask);
    __syncwarp(gmask);
    store_with_ghosts<P>(a.V2 + (size_t)cg * g.rows, buf, G, ny, phn, s, c00);
    if (c00)
      for (int i = 0; i < m; ++i) sb[i] = mkc(0, 0);
    __syncwarp(gmask);
    slab_stencil<P>(1, DS, sb, m, s, phn, gmask);
    __syncwarp(gmask);
    {
      cxd* const bufs[1] = {buf};
      group_solve_d0<P, 1>(thn, a.d0tab, G, bufs, s, gmask);
    }
    __syncwarp(gmask);
    for (int r = s; r < ny; r += P) v1[r + 2] = buf[G.at(r)];
  } else {
    for (int r = s; r < ny; r += P) buf[G.at(r)] = a.R1[cb + r];
    __syncwarp(gmask);
    group_solve<P>(K_ETA, sc.lambda, a.ps.ni, kk, thn, DS, G, buf, fac, s, gmask);
    __syncwarp(gmask);
    const double rkk = c00 ? 0.0 : 1.0 / kk;
    // dv/dy eight rows at a time, every load issued before the first use
    for (int r0 = s; r0 < ny; r0 += 8 * P) {
      cxd dvb[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) dvb[k] = r0 + k * P < ny ? v1[r0 + k * P + 2] : mkc(0, 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int r = r0 + k * P;
        if (r >= ny) break;
        const cxd eta = buf[G.at(r)], dv = dvb[k];
        cxd u, w;
        if (c00) {
          u = mkc(eta.x, 0.0);
          w = mkc(eta.y, 0.0);
        } else {
          u = mkc((-al * dv.y + be * eta.y) * rkk, (al * dv.x - be * eta.x) * rkk);
          w = mkc((-be * dv.y - al * eta.y) * rkk, (be * dv.x + al * eta.x) * rkk);
        }
        v1[r + 2] = u;
        buf[G.at(r)] = w;
      }
    }
    // __syncwarp orders the lanes' global stores before the ghost-row reads
    __syncwarp(gmask);
    for (int k = s; k < 4; k += P) {
      const int srow = k == 0 ? 0 : (k == 1 ? 1 : (k == 2 ? ny - 1 : ny - 2));
      const int drow = k == 0 ? ny : (k == 1 ? ny + 1 : (k == 2 ? -1 : -2));
      v1[drow + 2] = cmul(v1[srow + 2], k < 2 ? phn : cconj(phn));
    }
    store_with_ghosts<P>(a.V3 + (size_t)cg * g.rows, buf, G, ny, phn, s, false);
  }
}

// lines of shared memory a group holds in the persistent kernels (PART 0:
// the solves, 1: the exact_shift shift alone, which takes its four lines
// one at a time through one, 2, 3: the two halves of the solves)
constexpr int solve_lines(int part) { return part == 0 ? 2 : 1; }

// The solve stage (PART 0; 1: the exact_shift shift alone; 2, 3: the halves
// of the solves) on a persistent grid: each group of P lanes walks the
// columns col, col + gridDim.x groups, ...; shared memory holds only the
// group's lines (solve_lines), and the group's factor scratch is its own
// slice of a.facg in global memory, rewritten column after column (so it
// stays in L2).  Fewer bytes of shared memory a warp let more warps share an
// SM.
template <int P, bool EXACT, int PART>
#ifndef COLSOLVE_MINB
#define COLSOLVE_MINB 8  // 128 registers: up to 16 single-warp blocks an SM
#endif
__global__ void __launch_bounds__(64, COLSOLVE_MINB) k_column_solve(ColumnArgs a) {
  extern __shared__ double smem_d[];
  const Geometry& g = a.g;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int lineN = P * g.MS;
  const size_t facn = (size_t)(g.m - 2) * 4 * P;
  const size_t per_group = (size_t)solve_lines(PART) * lineN * 2;  // doubles
  cxd* bufA = reinterpret_cast<cxd*>(smem_d + per_group * grp);
  cxd* bufB = bufA + lineN;
  const int slot = blockIdx.x * groups + grp;
  // the factor scratch: the group's slice of a.facg (the launcher runs this
  // kernel only when the context has one)
  if (a.facg == nullptr) return;
  double* fac = a.facg + (size_t)slot * facn;
  for (int col = slot; col < g.ncol * g.nmem; col += gridDim.x * groups)
    if constexpr (PART <= 1)
      column_solve_body<P, EXACT, PART == 1>(a, col, s, bufA, bufB, fac);
    else
      column_solve_half<P, PART - 2>(a, col, s, bufA, fac);
}

// The exact_shift shift alone with the D0 table and the D0 slice of der in
// shared memory, shared by the block's warps (one group of P = 32 lanes a
// warp, one line each): a persistent grid of one block an SM.
#ifndef HST_SHIFT_SHT
#define HST_SHIFT_SHT 1
#endif
#ifndef HST_HALF_SHT
#define HST_HALF_SHT 1
#endif
__host__ __device__ inline size_t shift_sht_tables(int m, int P) {
  return ((size_t)d0_fields(m, P) * P + (size_t)5 * m * P) * sizeof(double);
}
template <int P>
__global__ void __launch_bounds__(512, 1) k_column_shift_sht(ColumnArgs a) {
  extern __shared__ double smem_d[];
  const Geometry& g = a.g;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int ntab = d0_fields(g.m, P) * P, nder = 5 * g.m * P;
  double* const d0s = smem_d;
  double* const der0s = d0s + ntab;
  for (int i = threadIdx.x; i < ntab; i += blockDim.x) d0s[i] = a.d0tab[i];
  for (int i = threadIdx.x; i < nder; i += blockDim.x) der0s[i] = a.derS[i];
  __syncthreads();
  cxd* const bufA = reinterpret_cast<cxd*>(der0s + nder) + (size_t)grp * P * g.MS;
  for (int col = blockIdx.x * groups + grp; col < g.ncol * g.nmem; col += gridDim.x * groups)
    column_solve_body<P, true, true, true>(a, col, s, bufA, bufA, nullptr, d0s, der0s);
}

// The halves of the solves with der in shared memory (HALF 0 reads all four
// slices, HALF 1 the D0 and D2 slices, copied as the first three), shared
// by the block's warps, one group of P = 32 lanes and one line a warp: a
// persistent grid of one block an SM.
__host__ __device__ inline int half_der_slices(int half) { return half == 0 ? 4 : 3; }
template <int P, int HALF>
__global__ void __launch_bounds__(512, 1) k_column_half_sht(ColumnArgs a) {
  extern __shared__ double smem_d[];
  const Geometry& g = a.g;
  const int groups = blockDim.x / P;
  const int grp = threadIdx.x / P, s = threadIdx.x - grp * P;
  const int nder = half_der_slices(HALF) * 5 * g.m * P;
  double* const ders = smem_d;
  for (int i = threadIdx.x; i < nder; i += blockDim.x) ders[i] = a.derS[i];
  __syncthreads();
  if (a.facg == nullptr) return;
  cxd* const buf = reinterpret_cast<cxd*>(ders + nder) + (size_t)grp * P * g.MS;
  const int slot = blockIdx.x * groups + grp;
  double* const fac = a.facg + (size_t)slot * (g.m - 2) * 4 * P;
  for (int col = slot; col < g.ncol * g.nmem; col += gridDim.x * groups)
    column_solve_half<P, HALF, true>(a, col, s, buf, fac, ders);
}

// --------------------------------------------------------- k_line_solve ----
// line_solve (src/hst_linsolve.f90:147-233) for every Fourier column.
template <int P>
__global__ void k_line_solve(Geometry g, PhysScalars ps, int sys, double lambda, const double2* __restrict__ src,
                             double2* __restrict__ dst, double sx, double sz, const double* __restrict__ der,
                             const double* __restrict__ derS) {
  extern __shared__ double smem_d[];
  const SlabDer DS = {derS, g.m, P};
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
  group_solve<P>(sys, lambda, ps.ni, kk, al * sx + be * sz, DS, G, buf, fac, s, gmask);
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

// ----------------------------------------------------------- k_rhs_tiled ----
// The right-hand-side stage as a streaming kernel: one warp per Fourier
// column walks its rows in tiles of 32; the 36-row windows of the three
// velocity components and of the six product spectra, and the carried terms
// of each tile are fetched with TMA bulk copies into shared memory (two
// stages: the next tile is in flight while this one computes), so the warp
// issues a handful of copy instructions per tile instead of one load per
// stencil tap.  Needs ny a multiple of 32.
constexpr int RT_W = 36;                                 // window rows
constexpr int RT_STAGE = 3 * RT_W + 6 * RT_W + 2 * 32;  // double2 per stage: V[3][36], Q[6][36], old[2][32]
constexpr int RT_WARPS = 4;
#ifndef RT_MINB
#define RT_MINB 4  // 128 registers: four 4-warp blocks an SM (0.52 against 0.69 ms at 384^2 x 256)
#endif
constexpr int RT_WAIT_LIMIT = 1 << 22;

// QT: the complex type of the product spectra Q (float2 in the mixed-
// precision form: the window lands as FP32 and each value is widened to
// FP64 where it is read)
template <bool EXACT, bool NONLIN, typename QT>
__global__ void __launch_bounds__(32 * RT_WARPS, RT_MINB) k_rhs_tiled(ColumnArgs a, int* __restrict__ err) {
  extern __shared__ __align__(128) double2 smt[];
  __shared__ __align__(8) uint64_t bars[RT_WARPS][2];
  const Geometry& g = a.g;
  const int ny = g.ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cgl = blockIdx.x * RT_WARPS + warp;  // the column over all members
  if (cgl >= g.ncol * g.nmem) return;
  const int mem = cgl / g.ncol, col = cgl - mem * g.ncol;
  double2* st0 = smt + (size_t)warp * 2 * RT_STAGE;
  uint64_t* bar = bars[warp];
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncwarp();
  const int ntile = ny / 32;
  const size_t cbase = (size_t)cgl * g.rows;  // row -2 of the column
  const double2* Vg[3] = {a.V1, a.V2, a.V3};
  // lane 0 queues the copies of tile t into stage t & 1
  const QT* Qg = reinterpret_cast<const QT*>(a.Q);
  const QT* Qgg = reinterpret_cast<const QT*>(a.Qg);
  constexpr unsigned QE = sizeof(QT);
  auto issue = [&](int t) {
    const int stg = t & 1;
    double2* S = st0 + stg * RT_STAGE;
    const int r0 = t * 32;
    mbar_arrive_expect_tx(&bar[stg], (3 * RT_W + 2 * 32) * 16 + 6 * RT_W * QE);
#pragma unroll
    for (int c = 0; c < 3; ++c) bulk_g2s(S + c * RT_W, Vg[c] + cbase + r0, RT_W * 16, &bar[stg]);
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const QT* Qc = Qg + (((size_t)mem * 6 + p) * g.ncol + col) * ny;
      QT* D = reinterpret_cast<QT*>(S + 3 * RT_W) + p * RT_W;
      const int lo = r0 - 2, hi = r0 + 34;
      const int m0 = lo < 0 ? 0 : lo, m1 = hi > ny ? ny : hi;
      // the rows beyond the box: the wrapped interior rows (their phase is
      // applied in tq), or the ghost rows' own spectra
      const QT* Qgc = Qgg ? Qgg + (((size_t)mem * 6 + p) * g.ncol + col) * 4 : nullptr;
      if (lo < 0) bulk_g2s(D, Qgc ? Qgc : Qc + ny + lo, (unsigned)(-lo) * QE, &bar[stg]);
      bulk_g2s(D + (m0 - lo), Qc + m0, (unsigned)(m1 - m0) * QE, &bar[stg]);
      if (hi > ny) bulk_g2s(D + (ny - lo), Qgc ? Qgc + 2 : Qc, (unsigned)(hi - ny) * QE, &bar[stg]);
    }
    bulk_g2s(S + 9 * RT_W, a.O1 + cbase + 2 + r0, 32 * 16, &bar[stg]);
    bulk_g2s(S + 9 * RT_W + 32, a.O2 + cbase + 2 + r0, 32 * 16, &bar[stg]);
  };
  if (lane == 0) {
    issue(0);
    if (ntile > 1) issue(1);
  }
  const ColConst cc = col_const(col, g, a.ps, a.sc, a.gdamp);
  const SubstepScalars& sc = a.sc;
  typedef typename RealOf<QT>::T QR;
  const QT ph_q = QT{(QR)cc.ph_t.x, (QR)cc.ph_t.y};  // the ghost-row phase in the spectra's precision
  // the default-form shift factor of row t 32 + lane on a uniform grid:
  // exp(-i g y(lane)) times exp(-i g 32 dy)^t, one product a tile instead
  // of a sine and cosine a row (mixed precision only: in the FP64 form the
  // two extra live values cost this 128-register kernel more than the
  // sines save, 0.57 against 0.52 ms at 384^2 x 256)
  constexpr bool REC = !EXACT && sizeof(QT) == 8;
  cxd fbase = mkc(1.0, 0.0), fstep = mkc(1.0, 0.0);
  if (REC && sc.yuni) {
    const double gsh = cc.al * sc.dgx + cc.be * sc.dgz;
    fbase = cexpi(-gsh * a.y[lane + 2]);
    fstep = cexpi(-gsh * sc.ytile);
  }
  for (int t = 0; t < ntile; ++t) {
    const int stg = t & 1;
    if (!mbar_wait_bounded(&bar[stg], (t >> 1) & 1, RT_WAIT_LIMIT)) {
      // record the failure, give this warp's copies still in flight a
      // second bounded wait to land, and leave
      if (lane == 0) atomicExch(err, 1);
      mbar_wait_bounded(&bar[stg], (t >> 1) & 1, RT_WAIT_LIMIT);
      if (t + 1 < ntile) mbar_wait_bounded(&bar[stg ^ 1], ((t + 1) >> 1) & 1, RT_WAIT_LIMIT);
      return;
    }
    const double2* S = st0 + stg * RT_STAGE;
    const int r = t * 32 + lane;
    auto tv = [&](int c, int j) -> cxd { return S[c * RT_W + lane + j]; };
    const QT* SQ = reinterpret_cast<const QT*>(S + 3 * RT_W);
    auto tq = [&](int p, int j) -> QT {
      const QT q = SQ[p * RT_W + lane + j];
      const int row = r + j - 2;
      if (Qgg) return q;
      if (row < 0) return cmul(q, cconj(ph_q));
      if (row >= ny) return cmul(q, ph_q);
      return q;
    };
    cxd r1, r2, o1, o2;
    const double yr = a.y[r + 2];
    auto fsh = [&]() -> cxd {
      if (REC && sc.yuni) return fbase;
      return cexpi(-(cc.al * sc.dgx + cc.be * sc.dgz) * yr);
    };
    rhs_point<NONLIN, EXACT>(cc, sc, DerRows{a.derU, a.derI, a.nderU}, ny, r, fsh, tv, tq, S[9 * RT_W + lane],
                             S[9 * RT_W + 32 + lane], r1, r2, o1, o2);
    if (REC) fbase = cmul(fbase, fstep);
    const size_t ro = cbase + 2 + r;
    a.O1[ro] = o1;
    a.O2[ro] = o2;
    a.R1[ro] = r1;
    a.R2[ro] = r2;
    __syncwarp();
    if (lane == 0 && t + 2 < ntile) {
      fence_proxy_async();
      issue(t + 2);
    }
  }
}

// -------------------------------------------------------------- launchers ----
size_t column_lines_bytes(const Geometry& g) { return (size_t)2 * g.P * g.MS * sizeof(double2); }

size_t column_fac_doubles(const Geometry& g) { return (size_t)(g.m - 2) * 4 * g.P; }

size_t column_smem_bytes(const Geometry& g, int exact) {
  size_t lineN = (size_t)g.P * g.MS;
  return ((exact ? 3 : 2) * lineN * 2 + (size_t)(g.m - 2) * 4 * g.P) * sizeof(double);
}

template <int P, bool EXACT, bool NONLIN, int MODE>
static cudaError_t launch_column_t(const ColumnArgs& a, cudaStream_t st) {
  const Geometry& g = a.g;
  if (MODE == COL_RHS && g.ny % 32 == 0 && a.tiled) {  // TMA-staged tiles
    const size_t smem = (size_t)RT_WARPS * 2 * RT_STAGE * sizeof(double2);
    const int blocks = (g.ncol * g.nmem + RT_WARPS - 1) / RT_WARPS;
    if (g.mp) {
      smem_limit(*a.dstate, k_rhs_tiled<EXACT, NONLIN, float2>, (int)smem);
      k_rhs_tiled<EXACT, NONLIN, float2><<<blocks, 32 * RT_WARPS, smem, st>>>(a, a.err);
    } else {
      smem_limit(*a.dstate, k_rhs_tiled<EXACT, NONLIN, double2>, (int)smem);
      k_rhs_tiled<EXACT, NONLIN, double2><<<blocks, 32 * RT_WARPS, smem, st>>>(a, a.err);
    }
    return cudaGetLastError();
  }
  // the untiled and fused forms read FP64 product spectra only (the
  // linear right-hand sides read none)
  if (MODE != COL_SOLVE && MODE != COL_SHIFT && MODE != COL_SOLVE_V && MODE != COL_SOLVE_ETA && g.mp && NONLIN)
    return cudaErrorInvalidValue;
  if (MODE == COL_RHS) {  // one warp per column, four per block, no shared memory
    const int blocks = (g.ncol * g.nmem + 3) / 4;
    k_column<32, EXACT, NONLIN, COL_RHS><<<blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
  }
  // 32 or 64 threads, fewer groups when their shared memory would not fit
  // the solve stage runs persistent; its factor scratch is in global memory
  // when the context has one (HST_COLUMN_GFAC), else in shared memory
  // the persistent solve stage when the context keeps the factor scratch in
  // global memory, else the one-column-per-group kernel
  constexpr bool HALVES = MODE == COL_SOLVE_V || MODE == COL_SOLVE_ETA;
  constexpr int PART = MODE == COL_SHIFT ? 1 : MODE == COL_SOLVE_V ? 2 : MODE == COL_SOLVE_ETA ? 3 : 0;
  const bool gfac = (MODE == COL_SOLVE || (MODE == COL_SHIFT && EXACT) || HALVES) && a.facg != nullptr;
  if (HALVES && (!gfac || EXACT)) return cudaErrorInvalidValue;
  const size_t per = gfac ? column_lines_bytes(g) / 2 * solve_lines(PART) +
                               (a.facg ? 0 : column_fac_doubles(g) * sizeof(double))
                          : column_smem_bytes(g, EXACT && MODE == COL_FUSED);
  int groups = (P >= 32 ? 32 : 64) / P;
  if (groups < 1) groups = 1;
  while (groups > 1 && per * groups > 200 * 1024) groups >>= 1;
  if (per * groups > 200 * 1024) return cudaErrorInvalidValue;
  const int T = groups * P;
  size_t smem = per * groups;
  int blocks = (g.ncol * g.nmem + groups - 1) / groups;
  if constexpr (MODE == COL_SHIFT && EXACT && P == 32) {
    if (HST_SHIFT_SHT) {
      // warps a block: as many lines as fit beside the tables, at most 16
      const size_t tabs = shift_sht_tables(g.m, P), line = column_lines_bytes(g) / 2;
      const int W = (int)std::min<size_t>(16, (227 * 1024 - tabs) / line);
      if (W >= 4) {
        const size_t sm = tabs + (size_t)W * line;
        smem_limit(*a.dstate, k_column_shift_sht<P>, 227 * 1024);
        const int nsm = a.dstate->nsm > 0 ? a.dstate->nsm : 148;
        const int nb = std::min(nsm, (g.ncol * g.nmem + W - 1) / W);
        k_column_shift_sht<P><<<nb, 32 * W, sm, st>>>(a);
        return cudaGetLastError();
      }
    }
  }
  if constexpr ((MODE == COL_SOLVE_V || MODE == COL_SOLVE_ETA) && P == 32) {
    // the halves with der in shared memory (the factor scratch in global
    // memory): warps a block, as many lines as fit beside der, at most 16
    if (HST_HALF_SHT && gfac) {
      const int half = MODE == COL_SOLVE_V ? 0 : 1;
      const size_t tabs = (size_t)half_der_slices(half) * 5 * g.m * P * sizeof(double);
      const size_t line = column_lines_bytes(g) / 2;
      const int W = (int)std::min<size_t>(16, tabs < 227 * 1024 ? (227 * 1024 - tabs) / line : 0);
      const int nsm = a.dstate->nsm > 0 ? a.dstate->nsm : 148;
      if (W >= 4 && nsm * W <= a.fac_groups) {
        auto kh = half == 0 ? k_column_half_sht<P, 0> : k_column_half_sht<P, 1>;
        const size_t sm = tabs + (size_t)W * line;
        smem_limit(*a.dstate, kh, 227 * 1024);
        const int nb = std::min(nsm, (g.ncol * g.nmem + W - 1) / W);
        kh<<<nb, 32 * W, sm, st>>>(a);
        return cudaGetLastError();
      }
    }
  }
  if (gfac) {
    auto kern = k_column_solve<P, EXACT, PART>;
    smem_limit(*a.dstate, kern, 200 * 1024);
    // persistent: the blocks that are resident at once (at most 16 warps an
    // SM), and no more groups than the scratch has slices for
    int per_sm = blocks_per_sm(*a.dstate, kern, T, smem);
    per_sm = std::min(per_sm, std::max(1, 16 * 32 / T));
    const int nsm = a.dstate->nsm > 0 ? a.dstate->nsm : 148;
    blocks = std::min(blocks, per_sm * nsm);
    if (a.facg) blocks = std::min(blocks, a.fac_groups / groups);
    if (blocks < 1) return cudaErrorInvalidValue;
    kern<<<blocks, T, smem, st>>>(a);
    return cudaGetLastError();
  }
  if constexpr (HALVES) {
    return cudaErrorInvalidValue;
  } else {
    auto kern = k_column<P, EXACT, NONLIN, MODE>;
    smem_limit(*a.dstate, kern, 200 * 1024);
    kern<<<blocks, T, smem, st>>>(a);
    return cudaGetLastError();
  }
}

template <int P, bool EXACT, bool NONLIN>
static cudaError_t launch_column_m(const ColumnArgs& a, int part, cudaStream_t st) {
  if (part == COL_RHS) return launch_column_t<P, EXACT, NONLIN, COL_RHS>(a, st);
  if (part == COL_SOLVE) return launch_column_t<P, EXACT, NONLIN, COL_SOLVE>(a, st);
  if (part == COL_SHIFT) {
    if constexpr (EXACT && !NONLIN) return launch_column_t<P, true, false, COL_SHIFT>(a, st);
    return cudaErrorInvalidValue;
  }
  if (part == COL_SOLVE_V || part == COL_SOLVE_ETA) {
    if constexpr (!EXACT)
      return part == COL_SOLVE_V ? launch_column_t<P, false, NONLIN, COL_SOLVE_V>(a, st)
                                 : launch_column_t<P, false, NONLIN, COL_SOLVE_ETA>(a, st);
    return cudaErrorInvalidValue;
  }
  return launch_column_t<P, EXACT, NONLIN, COL_FUSED>(a, st);
}

template <int P>
static cudaError_t launch_column_p(const ColumnArgs& a, int exact, int nonlin, int part, cudaStream_t st) {
  if (exact)
    return nonlin ? launch_column_m<P, true, true>(a, part, st) : launch_column_m<P, true, false>(a, part, st);
  return nonlin ? launch_column_m<P, false, true>(a, part, st) : launch_column_m<P, false, false>(a, part, st);
}

cudaError_t launch_column(const Geometry& g, const DeviceState& d, const PhysScalars& ph, const SubstepScalars& sc,
                          int exact, int nonlin, int part, cudaStream_t st) {
  ColumnArgs a;
  a.g = g;
  a.ps = ph;
  a.sc = sc;
  a.V1 = d.F[0];
  a.V2 = d.F[1];
  a.V3 = d.F[2];
  a.O1 = d.F[3];
  a.O2 = d.F[4];
  a.R1 = d.F[5];
  a.R2 = d.F[6];
  a.Q = d.Q;
  a.Qg = d.Qg;
  a.der = d.der;
  a.derS = d.derS;
  a.derU = d.derU;
  a.derI = d.derI;
  a.nderU = d.nderU;
  a.d0tab = d.d0tab;
  a.y = d.y;
  a.gdamp = d.gdamp;
  a.err = d.err;
  a.dstate = &d;
  a.facg = d.facg;
  a.fac_groups = d.facg ? (int)std::min<size_t>(d.facg_doubles / column_fac_doubles(g), 1u << 30) : 0;
  if (a.fac_groups < 1) a.facg = nullptr;
  {
    const char* e = std::getenv("HST_RHS_TILED");
    a.tiled = !(e && std::atoi(e) == 0);
  }
  if (part == 4) {  // the right-hand-side stage, untiled (the per-piece prepare)
    a.tiled = 0;
    part = COL_RHS;
  }
  switch (g.P) {
    case 2: return launch_column_p<2>(a, exact, nonlin, part, st);
    case 4: return launch_column_p<4>(a, exact, nonlin, part, st);
    case 8: return launch_column_p<8>(a, exact, nonlin, part, st);
    case 16: return launch_column_p<16>(a, exact, nonlin, part, st);
    case 32: return launch_column_p<32>(a, exact, nonlin, part, st);
  }
  return cudaErrorInvalidValue;
}

// d0_factor of the group of P lanes: one warp, lanes 0..P-1
template <int P>
__global__ void k_d0_table(const double* __restrict__ derS, int m, double* __restrict__ tab) {
  const int s = threadIdx.x;
  if (s >= P) return;
  const SlabDer DS = {derS, m, P};
  d0_factor<P>(DS, m, s, group_mask(P), tab);
}

size_t d0_table_doubles(int ny) {
  // d0_fields(m, P) P = 9 (ny - 2P) + P (31 + 8 levels) <= 9 ny + 32 (31 + 8 4)
  return (size_t)9 * ny + 32 * (31 + 8 * 4);
}

cudaError_t launch_d0_table(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  if ((size_t)d0_fields(g.m, g.P) * g.P > d0_table_doubles(g.ny)) return cudaErrorInvalidValue;
  switch (g.P) {
    case 2: k_d0_table<2><<<1, 32, 0, st>>>(d.derS, g.m, d.d0tab); break;
    case 4: k_d0_table<4><<<1, 32, 0, st>>>(d.derS, g.m, d.d0tab); break;
    case 8: k_d0_table<8><<<1, 32, 0, st>>>(d.derS, g.m, d.d0tab); break;
    case 16: k_d0_table<16><<<1, 32, 0, st>>>(d.derS, g.m, d.d0tab); break;
    case 32: k_d0_table<32><<<1, 32, 0, st>>>(d.derS, g.m, d.d0tab); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int P>
static cudaError_t launch_line_solve_t(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int sys,
                                       double lambda, int src, int dst, double sx, double sz, cudaStream_t st) {
  size_t per = ((size_t)P * g.MS * 2 + (size_t)(g.m - 2) * 4 * P) * sizeof(double);
  int groups = (P >= 32 ? 32 : 64) / P;
  if (groups < 1) groups = 1;
  while (groups > 1 && per * groups > 200 * 1024) groups >>= 1;
  if (per * groups > 200 * 1024) return cudaErrorInvalidValue;
  const int T = groups * P;
  smem_limit(d, k_line_solve<P>, 200 * 1024);
  int blocks = (g.ncol + groups - 1) / groups;
  k_line_solve<P><<<blocks, T, per * groups, st>>>(g, ph, sys, lambda, d.F[src], d.F[dst], sx, sz, d.der, d.derS);
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
