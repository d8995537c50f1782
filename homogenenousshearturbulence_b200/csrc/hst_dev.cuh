// Device building blocks of the hst substep on sm_100a: complex FP64
// arithmetic, the compact-stencil coefficients, the warp-group cyclic
// pentadiagonal line solver and the shared-memory Stockham FFT.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hst {

// ------------------------------------------------------------ complex ----
typedef double2 cxd;
__device__ __forceinline__ cxd mkc(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ cxd cadd(cxd a, cxd b) { return mkc(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cxd csub(cxd a, cxd b) { return mkc(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cxd cmul(cxd a, cxd b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cxd cscale(double s, cxd a) { return mkc(s * a.x, s * a.y); }
__device__ __forceinline__ cxd cconj(cxd a) { return mkc(a.x, -a.y); }
__device__ __forceinline__ cxd cneg(cxd a) { return mkc(-a.x, -a.y); }
// (0 + i b) * a
__device__ __forceinline__ cxd cmuli(double b, cxd a) { return mkc(-b * a.y, b * a.x); }
// a - s * b (s real)
__device__ __forceinline__ cxd cfms(cxd a, double s, cxd b) { return mkc(a.x - s * b.x, a.y - s * b.y); }
__device__ __forceinline__ cxd cdivr(cxd a, double d) { return mkc(a.x / d, a.y / d); }
// max that propagates NaN (fmax returns the other operand), as a positive
// quiet NaN
__device__ __forceinline__ double nan_max(double a, double b) {
  if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
  return fmax(a, b);
}
__device__ __forceinline__ cxd cexpi(double x) {
  double s, c;
  sincos(x, &s, &c);
  return mkc(c, s);
}
// complex division with range reduction (Smith)
__device__ __forceinline__ cxd cdiv(cxd a, cxd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return mkc((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.x * r + b.y;
    return mkc((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
// the same operations on complex64 (the transforms of the mixed-precision form)
typedef float2 cxf;
__device__ __forceinline__ cxf cadd(cxf a, cxf b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cxf csub(cxf a, cxf b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cxf cmul(cxf a, cxf b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cxf cscale(float s, cxf a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ cxf cconj(cxf a) { return make_float2(a.x, -a.y); }
// the real scalar type of a complex type
template <typename C>
struct RealOf;
template <>
struct RealOf<double2> {
  typedef double T;
};
template <>
struct RealOf<float2> {
  typedef float T;
};
__device__ __forceinline__ double shfl_d(unsigned mask, double v, int src, int width) {
  return __shfl_sync(mask, v, src, width);
}
__device__ __forceinline__ cxd shfl_c(unsigned mask, cxd v, int src, int width) {
  return mkc(__shfl_sync(mask, v.x, src, width), __shfl_sync(mask, v.y, src, width));
}

// ------------------------------------------- TMA bulk copies, mbarriers ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory, completion counted on
// bar (16-byte aligned addresses, size a multiple of 16; no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 4-D tiled tensor copy global -> this CTA's shared memory (no multicast);
// c0 is the innermost coordinate, in elements of the map's type
__device__ __forceinline__ void tma_load_4d(void* dst, const void* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
// 4-D tiled tensor copy shared -> global, completion tracked by bulk groups
__device__ __forceinline__ void tma_store_4d(const void* map, int c0, int c1, int c2, int c3, const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(map),
      "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// waits until the shared memory of every committed store has been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase `parity` of bar to complete, at most `limit` polls;
// false when the limit ran out (the caller records an error and returns).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// line-solve kinds (src/hst_linsolve.f90:83)
enum { K_D2V = 1, K_ETA = 2, K_POISSON = 3, K_D0 = 4, K_DY = 5 };

// der(iy, n, j), n = 0..3 (D0, D1, D2, D4), j = -2..2; Fortran order
// der(0:ny-1, 0:3, -2:2) as set up by src/hst_derivatives.f90:30-56.
__device__ __forceinline__ double derv(const double* __restrict__ der, int ny, int iy, int n, int j) {
  return __ldg(der + iy + ny * (n + 4 * (j + 2)));
}
// der(iy, n, j) through a table of its distinct rows: row iy of der is row
// idx[iy] of tab, stored coefficient-major (tab[(n + 4 (j + 2)) nu + u]) so
// that the lanes of a warp, whose rows map to a few distinct rows, read a
// few neighbouring words.  On a uniform grid ny rows have a few dozen
// distinct coefficient sets (rounding of the grid differences), so the
// table stays in L1 where der itself (20 ny doubles) does not.
struct DerRows {
  const double* __restrict__ tab;
  const int* __restrict__ idx;
  int nu;
  __device__ __forceinline__ double operator()(int iy, int n, int j) const {
    return __ldg(tab + (n + 4 * (j + 2)) * nu + __ldg(idx + iy));
  }
};
struct DerFull {
  const double* __restrict__ der;
  int ny;
  __device__ __forceinline__ double operator()(int iy, int n, int j) const { return derv(der, ny, iy, n, j); }
};

// The same table in slab-major order for a line-solve group of P lanes and
// m rows per lane: derS[((n*5 + j)*m + i)*P + s] = der(s*m + i, n, j - 2),
// so that the P lanes reading row i of their own slabs read consecutive
// addresses.
// SH: the table (or its first slices) copied into shared memory
template <bool SH = false>
struct SlabDerT {
  const double* __restrict__ p;
  int m, P;
  __device__ __forceinline__ double operator()(int s, int i, int n, int j) const {
    const double* q = p + ((size_t)((n * 5 + j) * m + i)) * P + s;
    if constexpr (SH)
      return *q;
    else
      return __ldg(q);
  }
};
typedef SlabDerT<false> SlabDer;

// The five band entries of row i of slab s of system `sys` before the wrap
// phase: coef, src/hst_linsolve.f90:236-252.
template <class DST>
__device__ __forceinline__ void row_coefs(int sys, double lambda, double ni, double kk, const DST& D, int s, int i,
                                          double a[5]) {
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    double d0 = D(s, i, 0, j);
    if (sys == K_D2V) {
      double d2 = D(s, i, 2, j), d4 = D(s, i, 3, j);
      a[j] = lambda * (d2 - kk * d0) - ni * (d4 - 2.0 * kk * d2 + kk * kk * d0);
    } else if (sys == K_ETA) {
      double d2 = D(s, i, 2, j);
      a[j] = lambda * d0 - ni * (d2 - kk * d0);
    } else if (sys == K_POISSON) {
      double d2 = D(s, i, 2, j);
      a[j] = d2 - kk * d0;
    } else {
      a[j] = d0;
    }
  }
}

// ------------------------------------------------ 2x2 block helpers ----
struct M2 {
  double a, b, c, d;  // [[a, b], [c, d]]
};
__device__ __forceinline__ M2 m2inv(M2 m) {
  double det = m.a * m.d - m.b * m.c;
  double r = 1.0 / det;
  M2 o = {m.d * r, -m.b * r, -m.c * r, m.a * r};
  return o;
}
__device__ __forceinline__ M2 m2mul(M2 x, M2 y) {
  M2 o = {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
  return o;
}
__device__ __forceinline__ M2 m2sub(M2 x, M2 y) {
  M2 o = {x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d};
  return o;
}
__device__ __forceinline__ M2 m2neg(M2 x) {
  M2 o = {-x.a, -x.b, -x.c, -x.d};
  return o;
}
struct V2c {
  cxd u, v;
};
__device__ __forceinline__ V2c m2vec(M2 m, V2c x) {
  V2c o = {mkc(m.a * x.u.x + m.b * x.v.x, m.a * x.u.y + m.b * x.v.y),
           mkc(m.c * x.u.x + m.d * x.v.x, m.c * x.u.y + m.d * x.v.y)};
  return o;
}
__device__ __forceinline__ V2c v2sub(V2c x, V2c y) {
  V2c o = {csub(x.u, y.u), csub(x.v, y.v)};
  return o;
}
__device__ __forceinline__ V2c v2scale(cxd s, V2c x) {
  V2c o = {cmul(s, x.u), cmul(s, x.v)};
  return o;
}
// complex 2x2
struct C2 {
  cxd a, b, c, d;
};
__device__ __forceinline__ C2 c2_from(M2 m) {
  C2 o = {mkc(m.a, 0), mkc(m.b, 0), mkc(m.c, 0), mkc(m.d, 0)};
  return o;
}
__device__ __forceinline__ C2 c2_axpby(M2 x, cxd s, M2 y, cxd t) {  // x s + y t
  C2 o = {cadd(cscale(x.a, s), cscale(y.a, t)), cadd(cscale(x.b, s), cscale(y.b, t)),
          cadd(cscale(x.c, s), cscale(y.c, t)), cadd(cscale(x.d, s), cscale(y.d, t))};
  return o;
}
__device__ __forceinline__ C2 c2mul_cr(C2 x, M2 y) {  // complex x real
  C2 o = {cadd(cscale(y.a, x.a), cscale(y.c, x.b)), cadd(cscale(y.b, x.a), cscale(y.d, x.b)),
          cadd(cscale(y.a, x.c), cscale(y.c, x.d)), cadd(cscale(y.b, x.c), cscale(y.d, x.d))};
  return o;
}
__device__ __forceinline__ C2 c2mul(C2 x, C2 y) {
  C2 o = {cadd(cmul(x.a, y.a), cmul(x.b, y.c)), cadd(cmul(x.a, y.b), cmul(x.b, y.d)),
          cadd(cmul(x.c, y.a), cmul(x.d, y.c)), cadd(cmul(x.c, y.b), cmul(x.d, y.d))};
  return o;
}
__device__ __forceinline__ V2c c2vec(C2 m, V2c x) {
  V2c o = {cadd(cmul(m.a, x.u), cmul(m.b, x.v)), cadd(cmul(m.c, x.u), cmul(m.d, x.v))};
  return o;
}
// solve m z = r for complex 2x2 m
__device__ __forceinline__ V2c c2solve(C2 m, V2c r) {
  cxd det = csub(cmul(m.a, m.d), cmul(m.b, m.c));
  cxd n1 = csub(cmul(m.d, r.u), cmul(m.b, r.v));
  cxd n2 = csub(cmul(m.a, r.v), cmul(m.c, r.u));
  V2c o = {cdiv(n1, det), cdiv(n2, det)};
  return o;
}
__device__ __forceinline__ M2 shfl_m2(unsigned mask, M2 m, int src, int w) {
  M2 o = {shfl_d(mask, m.a, src, w), shfl_d(mask, m.b, src, w), shfl_d(mask, m.c, src, w), shfl_d(mask, m.d, src, w)};
  return o;
}
__device__ __forceinline__ V2c shfl_v2(unsigned mask, V2c v, int src, int w) {
  V2c o = {shfl_c(mask, v.u, src, w), shfl_c(mask, v.v, src, w)};
  return o;
}
__device__ __forceinline__ C2 shfl_c2(unsigned mask, C2 m, int src, int w) {
  C2 o = {shfl_c(mask, m.a, src, w), shfl_c(mask, m.b, src, w), shfl_c(mask, m.c, src, w), shfl_c(mask, m.d, src, w)};
  return o;
}

// ------------------------------------------------- line buffer layout ----
// A line of n = P*m rows lives in shared memory slab by slab: slab s (the
// rows s*m .. s*m+m-1 owned by lane s of the group) starts at s*MS with
// MS = m rounded up to odd, so that the P lanes reading their own slab at
// the same offset hit different 16-byte bank groups.
struct LineGeom {
  int n, m, MS, P;
  unsigned invm;  // ceil(2^20 / m): r / m for r * m < 2^20
  __device__ __forceinline__ int slab(int r) const { return (int)(((unsigned)r * invm) >> 20); }
  __device__ __forceinline__ int at(int r) const {
    int s = slab(r);
    return s * MS + (r - s * m);
  }
};

// ------------------------------------------- the warp-group line solve ----
// One cyclic pentadiagonal system per line, solved by a group of P lanes
// (P a power of two, 2..32), lane s owning the slab of rows s*m..s*m+m-1.
// The algorithm is the reference's multi-slab bordering
// (src/hst_linsolve.f90:1-64, penta_forward :282-354, the reduced system of
// penta_backward :377-435) with every lane a slab: each lane factors its
// slab interior (real arithmetic, complex right-hand side) and writes the
// 28-value record; the 2P border unknowns then satisfy a block-cyclic
// tridiagonal system with 2x2 blocks.  Instead of dense Gaussian
// elimination over all slabs, that system is solved by parallel cyclic
// reduction across the lanes.  The wrap phase ph = exp(-i theta) enters only
// through the box edge; with b_s = mu^s c_s, mu = exp(-i theta/P), every
// block becomes real and the phase a uniform factor mu^(-1) (below) and mu
// (above), so the reduction runs on real 2x2 blocks with a complex
// right-hand side.  The back substitution then runs per slab
// (penta_backward :461-482).
//
// buf: the line (right-hand side in, solution out), in LineGeom layout.
// fac: per-lane factor scratch, (m-2) x 4 x P doubles.
// Rows of the right-hand side of KIND_DY must already hold D1 src.
template <int P, class DST = SlabDer>
__device__ void group_solve(int sys, double lambda, double ni, double kk, double theta, const DST& DS,
                            const LineGeom& G, cxd* buf, double* fac, int s, unsigned gmask) {
  const int m = G.m, mi = m - 2, MS = G.MS;
  cxd* sb = buf + s * MS;
  // ---- forward sweep of the slab interior (penta_forward)
  double u11 = 0, u12 = 0, p1 = 0, q1 = 0, u21 = 0, u22 = 0, p2 = 0, q2 = 0;
  double w1 = 0, w2 = 0, v1 = 0, v2 = 0, sp0 = 0, sq0 = 0, sp1 = 0, sq1 = 0;
  cxd x1 = mkc(0, 0), x2 = mkc(0, 0), sx0 = mkc(0, 0), sx1 = mkc(0, 0);
  for (int i = 0; i < mi; ++i) {
    double a[5];
    row_coefs(sys, lambda, ni, kk, DS, s, i, a);
    double p = 0, q = 0;
    if (i == 0) {
      p = a[0];
      q = a[1];
    }
    if (i == 1) q = a[0];
    cxd bx = sb[i];
    if (i >= 2) {
      double l = a[0];
      a[1] = a[1] - l * u21;
      a[2] = a[2] - l * u22;
      bx = cfms(bx, l, x2);
      p = p - l * p2;
      q = q - l * q2;
    }
    if (i >= 1) {
      double l = a[1];
      a[2] = a[2] - l * u11;
      a[3] = a[3] - l * u12;
      bx = cfms(bx, l, x1);
      p = p - l * p1;
      q = q - l * q1;
    }
    double rp = 1.0 / a[2];
    double t1 = a[3] * rp, t2 = a[4] * rp;
    bx = cscale(rp, bx);
    p = p * rp;
    q = q * rp;
    fac[(i * 4 + 0) * P + s] = t1;
    fac[(i * 4 + 1) * P + s] = t2;
    fac[(i * 4 + 2) * P + s] = p;
    fac[(i * 4 + 3) * P + s] = q;
    sb[i] = bx;
    double w = (i == 0) ? 1.0 : -(u11 * w1 + u22 * w2);
    double v = (i == 1) ? 1.0 : -(u11 * v1 + u22 * v2);
    sx0 = mkc(sx0.x + w * bx.x, sx0.y + w * bx.y);
    sp0 = sp0 + w * p;
    sq0 = sq0 + w * q;
    sx1 = mkc(sx1.x + v * bx.x, sx1.y + v * bx.y);
    sp1 = sp1 + v * p;
    sq1 = sq1 + v * q;
    w2 = w1;
    w1 = w;
    v2 = v1;
    v1 = v;
    u21 = u11;
    u22 = u12;
    x2 = x1;
    p2 = p1;
    q2 = q1;
    u11 = t1;
    u12 = t2;
    x1 = bx;
    p1 = p;
    q1 = q;
  }
  // the record of the slab (rec(1..28) of penta_forward)
  const cxd X0 = sx0;
  const double R3 = sp0, R4 = sq0, R5 = w2 * u22 + w1 * u11, R6 = w1 * u12;
  const cxd X1 = sx1;
  const double R9 = sp1, R10 = sq1, R11 = v2 * u22 + v1 * u11, R12 = v1 * u12;
  const cxd XM2 = csub(x2, cscale(u21, x1));
  const double R15 = p2 - u21 * p1, R16 = q2 - u21 * q1, R17 = u22 - u21 * u11, R18 = -u21 * u12;
  const cxd XM1 = x1;
  const double R21 = p1, R22 = q1, R23 = u11, R24 = u12;
  const cxd RB1 = sb[mi], RB2 = sb[mi + 1];
  // rows 0, 1 of the slab above (t = s+1)
  const int t = (s + 1) & (P - 1);
  const cxd TX0 = shfl_c(gmask, X0, t, P), TX1 = shfl_c(gmask, X1, t, P);
  const double T3 = shfl_d(gmask, R3, t, P), T4 = shfl_d(gmask, R4, t, P), T5 = shfl_d(gmask, R5, t, P),
               T6 = shfl_d(gmask, R6, t, P), T9 = shfl_d(gmask, R9, t, P), T10 = shfl_d(gmask, R10, t, P),
               T11 = shfl_d(gmask, R11, t, P), T12 = shfl_d(gmask, R12, t, P);
  // the two border rows of the slab (its rows mi, mi+1)
  double ab1[5], ab2[5];
  row_coefs(sys, lambda, ni, kk, DS, s, mi, ab1);
  row_coefs(sys, lambda, ni, kk, DS, s, mi + 1, ab2);
  const double c1m4 = ab1[0], c1m3 = ab1[1], d11 = ab1[2], d12 = ab1[3], c10 = ab1[4];
  const double c2m3 = ab2[0], d21 = ab2[1], d22 = ab2[2], c20 = ab2[3], c21 = ab2[4];
  // phases: ph = exp(-i theta) across the box edge; mu = ph^(1/P)
  const cxd ph = cexpi(-theta);
  const cxd mu = cexpi(-(theta / (double)P));
  // mu^s by binary powering (consistent with the squarings below)
  cxd mus = mkc(1.0, 0.0);
  {
    cxd b = mu;
    for (int e = s; e; e >>= 1) {
      if (e & 1) mus = cmul(mus, b);
      b = cmul(b, b);
    }
  }
  const cxd php = (s == P - 1) ? ph : mkc(1.0, 0.0);
  // block row s: L mu^-1 c_{s-1} + D c_s + U mu c_{s+1} = r mu^-s
  M2 L = {-(c1m4 * R15 + c1m3 * R21), -(c1m4 * R16 + c1m3 * R22), -(c2m3 * R21), -(c2m3 * R22)};
  M2 D = {d11 - (c1m4 * R17 + c1m3 * R23) - c10 * T3, d12 - (c1m4 * R18 + c1m3 * R24) - c10 * T4,
          d21 - c2m3 * R23 - (c20 * T3 + c21 * T9), d22 - c2m3 * R24 - (c20 * T4 + c21 * T10)};
  M2 U = {-(c10 * T5), -(c10 * T6), -(c20 * T5 + c21 * T11), -(c20 * T6 + c21 * T12)};
  V2c r;
  {
    cxd b1 = csub(csub(csub(RB1, cscale(c1m4, XM2)), cscale(c1m3, XM1)), cmul(cscale(c10, php), TX0));
    cxd b2 = csub(csub(RB2, cscale(c2m3, XM1)),
                  cmul(php, mkc(c20 * TX0.x + c21 * TX1.x, c20 * TX0.y + c21 * TX1.y)));
    V2c rr = {b1, b2};
    r = v2scale(cconj(mus), rr);
  }
  // parallel cyclic reduction: strides d = 1, 2, .., P/4
  cxd mud = mu;  // mu^d
  for (int d = 1; 2 * d < P; d <<= 1) {
    const int sm = (s - d) & (P - 1), sp = (s + d) & (P - 1);
    M2 Lm = shfl_m2(gmask, L, sm, P), Dm = shfl_m2(gmask, D, sm, P), Um = shfl_m2(gmask, U, sm, P);
    M2 Lp = shfl_m2(gmask, L, sp, P), Dp = shfl_m2(gmask, D, sp, P), Up = shfl_m2(gmask, U, sp, P);
    V2c rm = shfl_v2(gmask, r, sm, P), rpv = shfl_v2(gmask, r, sp, P);
    M2 A = m2mul(L, m2inv(Dm));
    M2 Gm = m2mul(U, m2inv(Dp));
    M2 Ln = m2neg(m2mul(A, Lm));
    M2 Un = m2neg(m2mul(Gm, Up));
    M2 Dn = m2sub(m2sub(D, m2mul(A, Um)), m2mul(Gm, Lp));
    V2c ta = v2scale(cconj(mud), m2vec(A, rm));
    V2c tg = v2scale(mud, m2vec(Gm, rpv));
    r = v2sub(v2sub(r, ta), tg);
    L = Ln;
    U = Un;
    D = Dn;
    mud = cmul(mud, mud);
  }
  // last level: c_{s-P/2} = c_{s+P/2}; pair with lane s ^ P/2
  V2c c;
  {
    C2 Mx = c2_axpby(L, cconj(mud), U, mud);
    const int q = s ^ (P >> 1);
    M2 Dq = shfl_m2(gmask, D, q, P);
    C2 Mq = shfl_c2(gmask, Mx, q, P);
    V2c rq = shfl_v2(gmask, r, q, P);
    C2 X = c2mul_cr(Mx, m2inv(Dq));
    C2 Sc = c2mul(X, Mq);
    C2 Dc = c2_from(D);
    Sc.a = csub(Dc.a, Sc.a);
    Sc.b = csub(Dc.b, Sc.b);
    Sc.c = csub(Dc.c, Sc.c);
    Sc.d = csub(Dc.d, Sc.d);
    V2c rhs = v2sub(r, c2vec(X, rq));
    c = c2solve(Sc, rhs);
  }
  // the border of this slab and of the slab below
  const cxd xb1 = cmul(mus, c.u), xb2 = cmul(mus, c.v);
  const int sb_ = (s - 1) & (P - 1);
  cxd yb1 = shfl_c(gmask, xb1, sb_, P), yb2 = shfl_c(gmask, xb2, sb_, P);
  if (s == 0) {
    yb1 = cmul(cconj(ph), yb1);
    yb2 = cmul(cconj(ph), yb2);
  }
  sb[mi] = xb1;
  sb[mi + 1] = xb2;
  // back substitution (penta_backward :467-482)
  cxd xk1 = xb1, xk2 = xb2;
  for (int i = mi - 1; i >= 0; --i) {
    double U1 = fac[(i * 4 + 0) * P + s], U2 = fac[(i * 4 + 1) * P + s];
    double B1 = fac[(i * 4 + 2) * P + s], B2 = fac[(i * 4 + 3) * P + s];
    cxd xr = sb[i];
    cxd xk = mkc(xr.x - B1 * yb1.x - B2 * yb2.x - U1 * xk1.x - U2 * xk2.x,
                 xr.y - B1 * yb1.y - B2 * yb2.y - U1 * xk1.y - U2 * xk2.y);
    sb[i] = xk;
    xk2 = xk1;
    xk1 = xk;
  }
}

// ------------------------------------- the D0 system, factored once ----
// The matrix of KIND_D0 and KIND_DY (the compact D0 operator) is the same
// for every Fourier column; only the wrap phase differs.  d0_factor runs the
// matrix half of group_solve once per context and keeps, per lane s of the
// group, every matrix quantity that the right-hand side meets: per interior
// row the two elimination multipliers, the pivot reciprocal, the record
// weights w, v and the back-substitution factors; the border-row
// coefficients; each reduction level's two 2x2 blocks; the blocks of the
// last level.  group_solve_d0 then runs only the right-hand-side half, the
// same operations in the same order as group_solve, so that the divisions,
// the block inverses and all matrix shuffles leave every column's
// dependency chain.  Field f of lane s sits at tab[f P + s].
__host__ __device__ constexpr int d0_levels(int P) {
  int n = 0;
  for (int d = 1; 2 * d < P; d <<= 1) ++n;
  return n;
}
__host__ __device__ constexpr int d0_fields(int m, int P) { return 9 * (m - 2) + 7 + 8 * d0_levels(P) + 24; }

template <int P>
__device__ void d0_factor(const SlabDer& DS, int m, int s, unsigned gmask, double* __restrict__ tab) {
  const int mi = m - 2;
  auto put = [&](int f, double v) { tab[(size_t)f * P + s] = v; };
  double u11 = 0, u12 = 0, p1 = 0, q1 = 0, u21 = 0, u22 = 0, p2 = 0, q2 = 0;
  double w1 = 0, w2 = 0, v1 = 0, v2 = 0, sp0 = 0, sq0 = 0, sp1 = 0, sq1 = 0;
  for (int i = 0; i < mi; ++i) {
    double a[5];
    row_coefs(K_D0, 0.0, 0.0, 0.0, DS, s, i, a);
    double p = 0, q = 0, l0 = 0, l1 = 0;
    if (i == 0) {
      p = a[0];
      q = a[1];
    }
    if (i == 1) q = a[0];
    if (i >= 2) {
      l0 = a[0];
      a[1] = a[1] - l0 * u21;
      a[2] = a[2] - l0 * u22;
      p = p - l0 * p2;
      q = q - l0 * q2;
    }
    if (i >= 1) {
      l1 = a[1];
      a[2] = a[2] - l1 * u11;
      a[3] = a[3] - l1 * u12;
      p = p - l1 * p1;
      q = q - l1 * q1;
    }
    const double rp = 1.0 / a[2];
    const double t1 = a[3] * rp, t2 = a[4] * rp;
    p = p * rp;
    q = q * rp;
    const double w = (i == 0) ? 1.0 : -(u11 * w1 + u22 * w2);
    const double v = (i == 1) ? 1.0 : -(u11 * v1 + u22 * v2);
    put(9 * i + 0, l0);
    put(9 * i + 1, l1);
    put(9 * i + 2, rp);
    put(9 * i + 3, w);
    put(9 * i + 4, v);
    put(9 * i + 5, t1);
    put(9 * i + 6, t2);
    put(9 * i + 7, p);
    put(9 * i + 8, q);
    sp0 = sp0 + w * p;
    sq0 = sq0 + w * q;
    sp1 = sp1 + v * p;
    sq1 = sq1 + v * q;
    w2 = w1;
    w1 = w;
    v2 = v1;
    v1 = v;
    u21 = u11;
    u22 = u12;
    p2 = p1;
    q2 = q1;
    u11 = t1;
    u12 = t2;
    p1 = p;
    q1 = q;
  }
  const double R3 = sp0, R4 = sq0, R5 = w2 * u22 + w1 * u11, R6 = w1 * u12;
  const double R9 = sp1, R10 = sq1, R11 = v2 * u22 + v1 * u11, R12 = v1 * u12;
  const double R15 = p2 - u21 * p1, R16 = q2 - u21 * q1, R17 = u22 - u21 * u11, R18 = -u21 * u12;
  const double R21 = p1, R22 = q1, R23 = u11, R24 = u12;
  const int t = (s + 1) & (P - 1);
  const double T3 = shfl_d(gmask, R3, t, P), T4 = shfl_d(gmask, R4, t, P), T5 = shfl_d(gmask, R5, t, P),
               T6 = shfl_d(gmask, R6, t, P), T9 = shfl_d(gmask, R9, t, P), T10 = shfl_d(gmask, R10, t, P),
               T11 = shfl_d(gmask, R11, t, P), T12 = shfl_d(gmask, R12, t, P);
  double ab1[5], ab2[5];
  row_coefs(K_D0, 0.0, 0.0, 0.0, DS, s, mi, ab1);
  row_coefs(K_D0, 0.0, 0.0, 0.0, DS, s, mi + 1, ab2);
  const double c1m4 = ab1[0], c1m3 = ab1[1], d11 = ab1[2], d12 = ab1[3], c10 = ab1[4];
  const double c2m3 = ab2[0], d21 = ab2[1], d22 = ab2[2], c20 = ab2[3], c21 = ab2[4];
  const int B = 9 * mi;
  put(B + 0, u21);
  put(B + 1, c1m4);
  put(B + 2, c1m3);
  put(B + 3, c10);
  put(B + 4, c2m3);
  put(B + 5, c20);
  put(B + 6, c21);
  M2 L = {-(c1m4 * R15 + c1m3 * R21), -(c1m4 * R16 + c1m3 * R22), -(c2m3 * R21), -(c2m3 * R22)};
  M2 D = {d11 - (c1m4 * R17 + c1m3 * R23) - c10 * T3, d12 - (c1m4 * R18 + c1m3 * R24) - c10 * T4,
          d21 - c2m3 * R23 - (c20 * T3 + c21 * T9), d22 - c2m3 * R24 - (c20 * T4 + c21 * T10)};
  M2 U = {-(c10 * T5), -(c10 * T6), -(c20 * T5 + c21 * T11), -(c20 * T6 + c21 * T12)};
  auto put2 = [&](int f, M2 x) {
    put(f, x.a);
    put(f + 1, x.b);
    put(f + 2, x.c);
    put(f + 3, x.d);
  };
  int f = B + 7;
  for (int d = 1; 2 * d < P; d <<= 1, f += 8) {
    const int sm = (s - d) & (P - 1), sp = (s + d) & (P - 1);
    M2 Lm = shfl_m2(gmask, L, sm, P), Dm = shfl_m2(gmask, D, sm, P), Um = shfl_m2(gmask, U, sm, P);
    M2 Lp = shfl_m2(gmask, L, sp, P), Dp = shfl_m2(gmask, D, sp, P), Up = shfl_m2(gmask, U, sp, P);
    M2 A = m2mul(L, m2inv(Dm));
    M2 Gm = m2mul(U, m2inv(Dp));
    M2 Ln = m2neg(m2mul(A, Lm));
    M2 Un = m2neg(m2mul(Gm, Up));
    M2 Dn = m2sub(m2sub(D, m2mul(A, Um)), m2mul(Gm, Lp));
    put2(f, A);
    put2(f + 4, Gm);
    L = Ln;
    U = Un;
    D = Dn;
  }
  const int q = s ^ (P >> 1);
  put2(f, L);
  put2(f + 4, U);
  put2(f + 8, shfl_m2(gmask, L, q, P));
  put2(f + 12, shfl_m2(gmask, U, q, P));
  put2(f + 16, m2inv(shfl_m2(gmask, D, q, P)));
  put2(f + 20, D);
}

// group_solve for the D0 matrix from the table of d0_factor, on NR lines
// at once (buf[k] each as group_solve's buf): the lines share every table
// load and run as independent dependency chains
template <int P, int NR, bool SH = false>
__device__ void group_solve_d0(double theta, const double* __restrict__ tab, const LineGeom& G, cxd* const* buf,
                               int s, unsigned gmask) {
  const int m = G.m, mi = m - 2, MS = G.MS;
  auto T = [&](int f) {
    if constexpr (SH)
      return tab[(size_t)f * P + s];
    else
      return __ldg(tab + (size_t)f * P + s);
  };
  auto T2 = [&](int f) { return M2{T(f), T(f + 1), T(f + 2), T(f + 3)}; };
  cxd* sb[NR];
  cxd x1[NR], x2[NR], sx0[NR], sx1[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    sb[k] = buf[k] + s * MS;
    x1[k] = x2[k] = sx0[k] = sx1[k] = mkc(0, 0);
  }
#pragma unroll 2
  for (int i = 0; i < mi; ++i) {
    const double l0 = T(9 * i + 0), l1 = T(9 * i + 1), rp = T(9 * i + 2), w = T(9 * i + 3), v = T(9 * i + 4);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      cxd bx = sb[k][i];
      if (i >= 2) bx = cfms(bx, l0, x2[k]);
      if (i >= 1) bx = cfms(bx, l1, x1[k]);
      bx = cscale(rp, bx);
      sb[k][i] = bx;
      sx0[k] = mkc(sx0[k].x + w * bx.x, sx0[k].y + w * bx.y);
      sx1[k] = mkc(sx1[k].x + v * bx.x, sx1[k].y + v * bx.y);
      x2[k] = x1[k];
      x1[k] = bx;
    }
  }
  const int B = 9 * mi;
  const double u21 = T(B);
  const double c1m4 = T(B + 1), c1m3 = T(B + 2), c10 = T(B + 3), c2m3 = T(B + 4), c20 = T(B + 5), c21 = T(B + 6);
  const int t = (s + 1) & (P - 1);
  const cxd ph = cexpi(-theta);
  const cxd mu = cexpi(-(theta / (double)P));
  cxd mus = mkc(1.0, 0.0);
  {
    cxd b = mu;
    for (int e = s; e; e >>= 1) {
      if (e & 1) mus = cmul(mus, b);
      b = cmul(b, b);
    }
  }
  const cxd php = (s == P - 1) ? ph : mkc(1.0, 0.0);
  V2c r[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const cxd XM2 = csub(x2[k], cscale(u21, x1[k]));
    const cxd XM1 = x1[k];
    const cxd RB1 = sb[k][mi], RB2 = sb[k][mi + 1];
    const cxd TX0 = shfl_c(gmask, sx0[k], t, P), TX1 = shfl_c(gmask, sx1[k], t, P);
    cxd b1 = csub(csub(csub(RB1, cscale(c1m4, XM2)), cscale(c1m3, XM1)), cmul(cscale(c10, php), TX0));
    cxd b2 = csub(csub(RB2, cscale(c2m3, XM1)),
                  cmul(php, mkc(c20 * TX0.x + c21 * TX1.x, c20 * TX0.y + c21 * TX1.y)));
    V2c rr = {b1, b2};
    r[k] = v2scale(cconj(mus), rr);
  }
  cxd mud = mu;
  int f = B + 7;
#pragma unroll
  for (int d = 1; 2 * d < P; d <<= 1, f += 8) {
    const int sm = (s - d) & (P - 1), sp = (s + d) & (P - 1);
    const M2 A = T2(f), Gm = T2(f + 4);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      V2c rm = shfl_v2(gmask, r[k], sm, P), rpv = shfl_v2(gmask, r[k], sp, P);
      V2c ta = v2scale(cconj(mud), m2vec(A, rm));
      V2c tg = v2scale(mud, m2vec(Gm, rpv));
      r[k] = v2sub(v2sub(r[k], ta), tg);
    }
    mud = cmul(mud, mud);
  }
  const C2 Mx = c2_axpby(T2(f), cconj(mud), T2(f + 4), mud);
  const C2 Mq = c2_axpby(T2(f + 8), cconj(mud), T2(f + 12), mud);
  const C2 X = c2mul_cr(Mx, T2(f + 16));
  C2 Sc = c2mul(X, Mq);
  {
    const C2 Dc = c2_from(T2(f + 20));
    Sc.a = csub(Dc.a, Sc.a);
    Sc.b = csub(Dc.b, Sc.b);
    Sc.c = csub(Dc.c, Sc.c);
    Sc.d = csub(Dc.d, Sc.d);
  }
  const int q = s ^ (P >> 1);
  const int sb_ = (s - 1) & (P - 1);
  cxd xk1[NR], xk2[NR], yb1[NR], yb2[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    V2c rq = shfl_v2(gmask, r[k], q, P);
    V2c rhs = v2sub(r[k], c2vec(X, rq));
    const V2c c = c2solve(Sc, rhs);
    const cxd xb1 = cmul(mus, c.u), xb2 = cmul(mus, c.v);
    yb1[k] = shfl_c(gmask, xb1, sb_, P);
    yb2[k] = shfl_c(gmask, xb2, sb_, P);
    if (s == 0) {
      yb1[k] = cmul(cconj(ph), yb1[k]);
      yb2[k] = cmul(cconj(ph), yb2[k]);
    }
    sb[k][mi] = xb1;
    sb[k][mi + 1] = xb2;
    xk1[k] = xb1;
    xk2[k] = xb2;
  }
#pragma unroll 2
  for (int i = mi - 1; i >= 0; --i) {
    const double U1 = T(9 * i + 5), U2 = T(9 * i + 6), B1 = T(9 * i + 7), B2 = T(9 * i + 8);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const cxd xr = sb[k][i];
      const cxd xk = mkc(xr.x - B1 * yb1[k].x - B2 * yb2[k].x - U1 * xk1[k].x - U2 * xk2[k].x,
                         xr.y - B1 * yb1[k].y - B2 * yb2[k].y - U1 * xk1[k].y - U2 * xk2[k].y);
      sb[k][i] = xk;
      xk2[k] = xk1[k];
      xk1[k] = xk;
    }
  }
}

}  // namespace hst
