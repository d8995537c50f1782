// The right-hand sides of one row of one Fourier column:
// buildrhs_prepare (src/hst_equations.f90:92-141), buildrhs for both product
// groups (:151-213), the hard damping mask (src/hst_damping.f90:119-133) and
// the default mean-shear phase shift (src/hst_equations.f90:245-257).  The
// taps of the five-point stencils come through accessors, so the same
// arithmetic serves the kernels that read global memory and the one that
// reads tiles staged in shared memory.
#pragma once
#include <type_traits>

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
// and to the carried terms o1, o2.  CR: double2 (FP64), or float2 (the
// mixed-precision form, whose right-hand sides are accumulated in FP32).
template <typename CR>
__device__ __forceinline__ void product_rhs(int p, const ColConst& c, double ode2d, CR q0, CR q1, CR q2, CR& r1,
                                            CR& r2, CR& o1, CR& o2) {
  typedef typename RealOf<CR>::T R;
  const R al = (R)c.al, be = (R)c.be, kk = (R)c.kk, ode2 = (R)ode2d;
  CR ru = CR{0, 0}, rw = CR{0, 0}, ex;
  if (p == 0) {  // uu
    ru = CR{al * q0.y, -al * q0.x};
    ex = CR{-(al * al) * q1.x, -(al * al) * q1.y};
  } else if (p == 1) {  // vv
    ex = CR{kk * q1.x, kk * q1.y};
  } else if (p == 2) {  // ww
    rw = CR{be * q0.y, -be * q0.x};
    ex = CR{-(be * be) * q1.x, -(be * be) * q1.y};
  } else if (p == 3) {  // uv
    ru = CR{-q1.x, -q1.y};
    ex = CR{-al * q2.y + -(al * kk) * q0.y, al * q2.x + (al * kk) * q0.x};
  } else if (p == 4) {  // vw
    rw = CR{-q1.x, -q1.y};
    ex = CR{-be * q2.y + -(be * kk) * q0.y, be * q2.x + (be * kk) * q0.x};
  } else {  // uw
    ru = CR{be * q0.y, -be * q0.x};
    rw = CR{al * q0.y, -al * q0.x};
    ex = CR{-((R(2) * al) * be) * q1.x, -((R(2) * al) * be) * q1.y};
  }
  r2 = CR{r2.x + ode2 * ex.x, r2.y + ode2 * ex.y};
  o2 = CR{o2.x + ex.x, o2.y + ex.y};
  CR e;
  if (c.c00) e = CR{ru.x, rw.x};
  else e = CR{-be * ru.y + al * rw.y, be * ru.x - al * rw.x};
  r1 = CR{r1.x + ode2 * e.x, r1.y + ode2 * e.y};
  o1 = CR{o1.x + e.x, o1.y + e.y};
}

// TV(c, j): component c of V at row r + j - 2; TQ(p, j): product p at row
// r + j - 2 (ghost phase applied); fsh(): the default-form shift factor of
// row r, exp(-i (alfa dgx + beta dgz) y(r)), asked for last.  EXACT: no phase
// shift here (shift_unweighted follows in the solve kernel).
// Precision: with FP64 product spectra everything is FP64, in the
// reference's operation order.  With FP32 spectra (the mixed-precision form)
// the derivative right-hand sides are FP32 with FP32 accumulation -- the
// explicit half of the viscous terms, the mean-shear tilting, the damping,
// the carried terms and the six product terms (stencil weights formed in
// FP64 from der, k^2 and nu and rounded once, taps rounded to FP32) -- and
// one term stays FP64: ODE(1)/dt times the unknowns (D2 - k^2 D0) v and
// D0 eta, the Crank-Nicolson operator applied to the old state, which is
// larger than the rest by about 1/(nu k^2 dt) and sets the increment the
// FP64 solve resolves (all of it in FP32 measured 1.3e-5 relative L2 from
// the oracle after 30 substeps of 96^2 x 64 and 6.5e-5 at 768^2 x 512, over
// the 1e-5 bound).  The results are widened to FP64 for storage and for the
// default-form phase, which stays FP64.
#ifndef HST_MIXED_RHS_FP32
#define HST_MIXED_RHS_FP32 1  // 0: the mixed form's right-hand sides in FP64 but for the product stencils
#endif
template <bool NONLIN, bool EXACT, class TV, class TQ, class FS, class DA>
__device__ __forceinline__ void rhs_point(const ColConst& c, const SubstepScalars& sc, const DA& der, int ny, int r,
                                          const FS& fsh, const TV& tv, const TQ& tq, cxd o1in, cxd o2in, cxd& r1,
                                          cxd& r2, cxd& o1, cxd& o2) {
  const double kk = c.kk, al = c.al, be = c.be, ni = c.ni, gs = c.gs;
  constexpr bool F32 = sizeof(decltype(tq(0, 0))) == 8;
  double d0[5], d1[5], d2[5], d4[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    d0[j] = der(r, 0, j - 2);
    d1[j] = der(r, 1, j - 2);
    d2[j] = der(r, 2, j - 2);
    d4[j] = der(r, 3, j - 2);
  }
  if constexpr (!F32 || !HST_MIXED_RHS_FP32) {
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
    auto lam = [&](double u) { return F32 ? sc.lambda * u : (sc.ode0 * u) / sc.deltat; };
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
        // the product stencils in the spectra's own precision
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
        product_rhs<cxd>(p, c, sc.ode1, mkc(a0.x, a0.y), mkc(a1.x, a1.y), mkc(a2.x, a2.y), r1, r2, o1, o2);
      }
    }
  } else {
    // v equation: the unknown in FP64, the rest in FP32
    cxd unkn = mkc(0, 0);
    float2 impl = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double helm = d2[j] - kk * d0[j];
      const float nb = (float)(ni * (d4[j] - 2.0 * kk * d2[j] + kk * kk * d0[j]));
      const cxd v = tv(1, j);
      unkn = mkc(unkn.x + helm * v.x, unkn.y + helm * v.y);
      impl = make_float2(impl.x + nb * (float)v.x, impl.y + nb * (float)v.y);
    }
    const float o1gs = (float)(sc.ode1 * gs), gsf = (float)gs, ode2 = (float)sc.ode2, ode1 = (float)sc.ode1;
    const float2 u2 = make_float2((float)unkn.x, (float)unkn.y);
    float2 r2r = make_float2(impl.x - ode2 * (float)o2in.x - o1gs * u2.x, impl.y - ode2 * (float)o2in.y - o1gs * u2.y);
    float2 o2r = make_float2(-gsf * u2.x, -gsf * u2.y);
    const cxd lam2 = mkc(sc.lambda * unkn.x, sc.lambda * unkn.y);
    // eta equation (mean column: u, w packed)
    unkn = mkc(0, 0);
    impl = make_float2(0.f, 0.f);
    float2 expl = make_float2(0.f, 0.f);
    const float alf = (float)al, bef = (float)be;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const cxd v1 = tv(0, j), v3 = tv(2, j), v2 = tv(1, j);
      cxd f;
      float w;
      if (c.c00) {
        f = mkc(v1.x, v3.x);
        w = (float)(ni * d2[j]);
      } else {
        f = mkc(-be * v1.y + al * v3.y, be * v1.x - al * v3.x);
        w = (float)(ni * (d2[j] - kk * d0[j]));
      }
      unkn = mkc(unkn.x + d0[j] * f.x, unkn.y + d0[j] * f.y);
      impl = make_float2(impl.x + w * (float)f.x, impl.y + w * (float)f.y);
      const float kd = (float)(c.kappa * d0[j]);
      expl = make_float2(expl.x - kd * (float)v2.y, expl.y + kd * (float)v2.x);
    }
    (void)alf;
    (void)bef;
    const float2 u1 = make_float2((float)unkn.x, (float)unkn.y);
    expl = make_float2(expl.x - gsf * u1.x, expl.y - gsf * u1.y);
    float2 r1r = make_float2(impl.x - ode2 * (float)o1in.x + ode1 * expl.x, impl.y - ode2 * (float)o1in.y + ode1 * expl.y);
    float2 o1r = expl;
    const cxd lam1 = mkc(sc.lambda * unkn.x, sc.lambda * unkn.y);
    if (NONLIN) {
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f), a2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          const auto qv = tq(p, j);
          const float e0 = (float)d0[j], e1 = (float)d1[j], e2 = (float)d2[j];
          a0 = make_float2(a0.x + e0 * qv.x, a0.y + e0 * qv.y);
          a1 = make_float2(a1.x + e1 * qv.x, a1.y + e1 * qv.y);
          a2 = make_float2(a2.x + e2 * qv.x, a2.y + e2 * qv.y);
        }
        product_rhs<float2>(p, c, sc.ode1, a0, a1, a2, r1r, r2r, o1r, o2r);
      }
    }
    r1 = mkc(lam1.x + (double)r1r.x, lam1.y + (double)r1r.y);
    r2 = mkc(lam2.x + (double)r2r.x, lam2.y + (double)r2r.y);
    o1 = mkc(o1r.x, o1r.y);
    o2 = mkc(o2r.x, o2r.y);
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
