// The right-hand sides of one row of one Fourier column:
// buildrhs_prepare (src/hst_equations.f90:92-141), buildrhs for both product
// groups (:151-213), the hard damping mask (src/hst_damping.f90:119-133) and
// the default mean-shear phase shift (src/hst_equations.f90:245-257).  The
// taps of the five-point stencils come through accessors, so the same
// arithmetic serves the kernels that read global memory and the one that
// reads tiles staged in shared memory.
#pragma once
#include "hst_dev.cuh"
#include "hst_internal.h"

namespace hst {

// what a column needs, uniform over its rows
struct ColConst {
  double al, be, kk, ni, S, gs, kappa;
  bool c00, masked;
  cxd ph_t;  // wrap phase at t: ghost images of the product rows
};

__device__ __forceinline__ ColConst col_const(int col, const Geometry& g, const PhysScalars& ps,
                                              const SubstepScalars& sc, const double* __restrict__ gdamp) {
  ColConst c;
  const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
  c.c00 = (ix == 0 && iz == 0);
  c.al = ps.alfa0 * ix;
  c.be = ps.beta0 * iz;
  c.kk = c.al * c.al + c.be * c.be;
  c.ni = ps.ni;
  c.S = ps.S;
  const double gcol = gdamp[col];
  c.gs = sc.gsoft * gcol;
  c.masked = sc.damp_hard && gcol > 0.0;
  c.kappa = sc.s2now * c.al - ps.S * c.be;  // (s2 i alfa - S i beta) / i
  c.ph_t = cexpi(-(c.al * sc.sx_t + c.be * sc.sz_t));
  return c;
}

// The terms of product p (0..5: uu, vv, ww, uv, vw, uw) of buildrhs
// (src/hst_equations.f90:167-209) from its D0, D1, D2 stencils q0, q1, q2,
// added to the right-hand sides r1 (eta), r2 (d2v) with weight ode2 = ODE(2)
// and to the carried terms o1, o2.
__device__ __forceinline__ void product_rhs(int p, const ColConst& c, double ode2, cxd q0, cxd q1, cxd q2, cxd& r1,
                                            cxd& r2, cxd& o1, cxd& o2) {
  const double al = c.al, be = c.be, kk = c.kk;
  cxd ru = mkc(0, 0), rw = mkc(0, 0), ex;
  if (p == 0) {  // uu
    ru = mkc(al * q0.y, -al * q0.x);
    ex = cscale(-(al * al), q1);
  } else if (p == 1) {  // vv
    ex = cscale(kk, q1);
  } else if (p == 2) {  // ww
    rw = mkc(be * q0.y, -be * q0.x);
    ex = cscale(-(be * be), q1);
  } else if (p == 3) {  // uv
    ru = cneg(q1);
    ex = mkc(-al * q2.y + -(al * kk) * q0.y, al * q2.x + (al * kk) * q0.x);
  } else if (p == 4) {  // vw
    rw = cneg(q1);
    ex = mkc(-be * q2.y + -(be * kk) * q0.y, be * q2.x + (be * kk) * q0.x);
  } else {  // uw
    ru = mkc(be * q0.y, -be * q0.x);
    rw = mkc(al * q0.y, -al * q0.x);
    ex = cscale(-((2.0 * al) * be), q1);
  }
  r2 = mkc(r2.x + ode2 * ex.x, r2.y + ode2 * ex.y);
  o2 = cadd(o2, ex);
  cxd e;
  if (c.c00) e = mkc(ru.x, rw.x);
  else e = mkc(-be * ru.y + al * rw.y, be * ru.x - al * rw.x);
  r1 = mkc(r1.x + ode2 * e.x, r1.y + ode2 * e.y);
  o1 = cadd(o1, e);
}

// TV(c, j): component c of V at row r + j - 2; TQ(p, j): product p at row
// r + j - 2 (ghost phase applied); fsh(): the default-form shift factor of
// row r, exp(-i (alfa dgx + beta dgz) y(r)), asked for last.  EXACT: no phase
// shift here (shift_unweighted follows in the solve kernel).  With FP32
// spectra ODE(1)/dt is sc.lambda (one product instead of a division a term:
// 0.50 against 0.52 ms at 384^2 x 256; the FP64 form keeps the division,
// which measured as fast).
template <bool NONLIN, bool EXACT, class TV, class TQ, class FS>
__device__ __forceinline__ void rhs_point(const ColConst& c, const SubstepScalars& sc, const double* __restrict__ der,
                                          int ny, int r, const FS& fsh, const TV& tv, const TQ& tq, cxd o1in, cxd o2in,
                                          cxd& r1, cxd& r2, cxd& o1, cxd& o2) {
  const double kk = c.kk, al = c.al, be = c.be, ni = c.ni, gs = c.gs;
  constexpr bool F32 = sizeof(decltype(tq(0, 0))) == 8;
  auto lam = [&](double u) { return F32 ? sc.lambda * u : (sc.ode0 * u) / sc.deltat; };
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
    cxd v = tv(1, j);
    unkn = mkc(unkn.x + helm * v.x, unkn.y + helm * v.y);
    double nb = ni * biharm;
    impl = mkc(impl.x + nb * v.x, impl.y + nb * v.y);
  }
  r2 = mkc(lam(unkn.x) + impl.x - sc.ode2 * o2in.x - (sc.ode1 * gs) * unkn.x,
           lam(unkn.y) + impl.y - sc.ode2 * o2in.y - (sc.ode1 * gs) * unkn.y);
  o2 = mkc(-gs * unkn.x, -gs * unkn.y);
  // eta equation (mean column: u, w packed)
  unkn = mkc(0, 0);
  impl = mkc(0, 0);
  cxd expl = mkc(0, 0);
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    double helm = d2[j] - kk * d0[j];
    cxd v1 = tv(0, j), v3 = tv(2, j), v2 = tv(1, j);
    cxd f;
    double w;
    if (c.c00) {
      f = mkc(v1.x, v3.x);
      w = ni * d2[j];
    } else {
      f = mkc(-be * v1.y + al * v3.y, be * v1.x - al * v3.x);
      w = ni * helm;
    }
    unkn = mkc(unkn.x + d0[j] * f.x, unkn.y + d0[j] * f.y);
    impl = mkc(impl.x + w * f.x, impl.y + w * f.y);
    double kd = c.kappa * d0[j];
    expl = mkc(expl.x - kd * v2.y, expl.y + kd * v2.x);
  }
  expl = mkc(expl.x - gs * unkn.x, expl.y - gs * unkn.y);
  r1 = mkc(lam(unkn.x) + impl.x - sc.ode2 * o1in.x + sc.ode1 * expl.x,
           lam(unkn.y) + impl.y - sc.ode2 * o1in.y + sc.ode1 * expl.y);
  o1 = expl;
  if (NONLIN) {
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      // the stencils of the product spectra in their own precision (FP32
      // in the mixed-precision form), the rest in FP64
      typedef decltype(tq(0, 0)) QV;
      typedef typename RealOf<QV>::T QR;
      QV a0 = QV{0, 0}, a1 = QV{0, 0}, a2 = QV{0, 0};
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const QV qv = tq(p, j);
        const QR e0 = (QR)d0[j], e1 = (QR)d1[j], e2 = (QR)d2[j];
        a0 = QV{a0.x + e0 * qv.x, a0.y + e0 * qv.y};
        a1 = QV{a1.x + e1 * qv.x, a1.y + e1 * qv.y};
        a2 = QV{a2.x + e2 * qv.x, a2.y + e2 * qv.y};
      }
      const cxd q0 = mkc(a0.x, a0.y), q1 = mkc(a1.x, a1.y), q2 = mkc(a2.x, a2.y);
      product_rhs(p, c, sc.ode1, q0, q1, q2, r1, r2, o1, o2);
    }
  }
  if (c.masked) {  // damping_mask
    r1 = r2 = o1 = o2 = mkc(0, 0);
  }
  if (!EXACT) {  // shear_shift, default form
    const cxd f = fsh();
    r1 = cmul(r1, f);
    r2 = cmul(r2, f);
    o1 = cmul(o1, f);
    o2 = cmul(o2, f);
  }
}

}  // namespace hst
