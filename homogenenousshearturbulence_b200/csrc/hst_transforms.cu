// The transform kernels of the hst substep (FP64):
//
//   k_zinv   V (u, v, w) -> zero-padded z-inverse transform (Z)
//   k_xprod  Z -> x-inverse (c2r) of u, v, w; the six products times
//            1/(2 nxd nzd); the CFL maximum; x-forward (r2c) of the products
//            truncated to the nx+1 retained modes (Pp)
//   k_zfwd   Pp -> z-forward transform truncated to the 2nz+1 modes (Q)
//
// Together they are transform_to_physical + build_products (both groups) +
// products_to_spectral + compute_cfl of the reference
// (src/hst_transforms.f90:33-179, src/hst_fft.f90:181-237), with the local
// transposes (src/hst_mpi.f90:615-669) absorbed into the index maps.  Only
// the ny interior rows are transformed (see k_column for the ghost-row
// products).  Z and Pp are stored [component][y tile][kz][ix][Ty]: a block
// of k_zinv / k_zfwd (one x mode, one y tile, all kz) then spans a few
// huge pages instead of one page per kz.
#include <cmath>

#include "hst_dev.cuh"
#include "hst_fft.cuh"
#include "hst_internal.h"

namespace hst {

cudaError_t set_fft_constants() {
  double2 w[48];
  float2 wf[48];
  for (int k = 0; k < 48; ++k) {
    long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / 48.0L;
    w[k] = make_double2((double)cosl(a), (double)sinl(a));
    wf[k] = make_float2((float)cosl(a), (float)sinl(a));
  }
  cudaError_t e = cudaMemcpyToSymbol(c_w48, w, sizeof w);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_w48f, wf, sizeof wf);
  return e;
}

bool fft_length_ok(int n) { return plan_ok(n); }

#ifndef ZPAD16
#define ZPAD16 1  // 0: the 16- and 32-point z plans on unpadded lines
#endif
// The order of the z kernels' blocks: IXF = 1 runs the x modes of one y tile
// side by side (consecutive blocks read, or write, adjacent 64-byte runs of
// the [yt][kz][ix][Ty] tiles of Z and Pp), 0 the y tiles of one x mode.
// Measured at 768^2 x 512: the z-inverse 2.18 against 2.26 ms with 1 (1.75
// against 1.85 in FP32); the z-forward 4.82 against 4.68 ms (FP64) and 3.03
// against 3.14 ms (FP32), 0.327 against 0.302 ms at 384^2 x 256 (FP32).
#ifndef ZINV_IXF
#define ZINV_IXF 1
#endif
#ifndef ZFWD_IXF
#define ZFWD_IXF 0
#endif

// --------------------------------------------------------------- k_zinv ----
// assemble_vvdz + IFT (src/hst_transforms.f90:33-54, src/hst_fft.f90:195-207):
// line yi of the block is row y0 + yi of one x mode of one component; the
// z modes -nz..nz sit at padded index iz (iz >= 0) or nzd + iz.
// C: the complex type of the transforms (double2; float2 in the
// mixed-precision form, where V is read as FP64 and rounded once)
template <typename C>
__device__ __forceinline__ C to_c(double2 v) {
  typedef typename RealOf<C>::T T;
  return C{(T)v.x, (T)v.y};
}
template <typename C>
struct ZinvSrc {
  const double2* __restrict__ col;  // V + (ix nzT) rows + 2 + y0: row y0 of iz = -nz
  int rows, nz, NZ;
  int gap;  // the edge view: rows -2, -1 at 0, 1 and ny, ny+1 at gap + 2, gap + 3
  __device__ __forceinline__ C operator()(int yi, int kz) const {
    int iz;
    if (kz <= nz) iz = kz;
    else if (kz >= NZ - nz) iz = kz - NZ;
    else return C{0, 0};
    return to_c<C>(col[(size_t)(iz + nz) * rows + yi + (yi >= 2 ? gap : 0)]);
  }
};
template <typename C>
struct TileDst {  // one (component, y tile, x mode) z-line set of Z / Pp
  C* __restrict__ base;
  size_t zstride;
  __device__ __forceinline__ void operator()(int yi, int kz, C v) const { base[(size_t)kz * zstride + yi] = v; }
};
template <typename C>
struct TileSrc {
  const C* __restrict__ base;
  size_t zstride;
  __device__ __forceinline__ C operator()(int yi, int kz) const { return base[(size_t)kz * zstride + yi]; }
};

// the z kernels' compile-time plans keep their lines padded (ls_lines: one
// pad in 8 for the 8-point plans, in 16 for the 16- and 32-point plans),
// free of bank conflicts under the line-fastest mapping
// (FP64 16- and 32-point plans stay unpadded: at 384 points their eight
// rows a block are conflict-free anyway, and at 1536 the pad measured
// slower, 15.8 against 12.5 ms z-inverse and 27.0 against 23.6 ms
// z-forward, where in FP32 it gains, 12.2 against 13.2 and 15.6 against
// 17.8 ms)
template <int NT, int PPT, typename C>
__host__ __device__ constexpr bool z_padded() {
  return NT > 0 && (PPT <= 8 || (ZPAD16 && sizeof(C) == 8));
}
template <int NT, int PPT, typename C>
__host__ __device__ inline size_t z_smem(int nzd, int Ty) {
  const int ls = !z_padded<NT, PPT, C>() ? nzd + 1 : (PPT <= 8 ? ls_lines<C, 3>(nzd, Ty) : ls_lines<C, 4>(nzd, Ty));
  return (size_t)Ty * ls * sizeof(C);
}

template <int NT, int PPT, typename C>
__device__ __forceinline__ void zinv_body(const Geometry& g, const double2* __restrict__ V0,
                                          const double2* __restrict__ V1, const double2* __restrict__ V2,
                                          C* __restrict__ Z, const C* __restrict__ twz) {
  extern __shared__ double2 sh_d[];
  C* sh = reinterpret_cast<C*>(sh_d);
  const int yt = ZINV_IXF ? blockIdx.y : blockIdx.x, ix = ZINV_IXF ? blockIdx.x : blockIdx.y;
  const int c = blockIdx.z % 3, mem = blockIdx.z / 3;
  const int Ty = g.Ty, NZ = g.nzd, nyT = g.ny / Ty;
  const double2* V = (c == 0 ? V0 : (c == 1 ? V1 : V2)) + (size_t)mem * g.nf;
  Z += (size_t)mem * 3 * NZ * g.ny * g.nxB;
  const ZinvSrc<C> src = {V + (size_t)ix * g.nzT * g.rows + (g.edge_gap ? 0 : 2) + yt * Ty, g.rows, g.nz, NZ,
                          g.edge_gap};
  const TileDst<C> dst = {Z + (((size_t)c * nyT + yt) * NZ) * g.nxB * Ty + (size_t)ix * Ty, (size_t)g.nxB * Ty};
  fft_sel<NT, +1, PPT, false, false, false, z_padded<NT, PPT, C>()>(NZ, Ty, twz, sh, src, dst);
}
template <int NT, int PPT, typename C>
__global__ void __launch_bounds__(PPT <= 8 ? 512 : 256)
    k_zinv(Geometry g, const double2* __restrict__ V0, const double2* __restrict__ V1, const double2* __restrict__ V2,
           C* __restrict__ Z, const C* __restrict__ twz) {
  zinv_body<NT, PPT, C>(g, V0, V1, V2, Z, twz);
}
// the FP64 32-point plans (192 threads) held to two blocks an SM (1536
// points: 16.5 -> 12.5 ms at 1536^2 x 512; an explicit block minimum on
// the kernel above made the 384-point plan slower, 0.42 against 0.25 ms)
template <int NT>
__global__ void __launch_bounds__(192, 2) k_zinv_32(Geometry g, const double2* __restrict__ V0,
                                                    const double2* __restrict__ V1, const double2* __restrict__ V2,
                                                    double2* __restrict__ Z, const double2* __restrict__ twz) {
  zinv_body<NT, 32, double2>(g, V0, V1, V2, Z, twz);
}
// the FP32 1536-point plan (192 threads) held to three blocks an SM (an
// explicit block minimum on the kernel above made the 384-point plan slower)
__global__ void __launch_bounds__(192, 3) k_zinv_1536f(Geometry g, const double2* __restrict__ V0,
                                                       const double2* __restrict__ V1, const double2* __restrict__ V2,
                                                       float2* __restrict__ Z, const float2* __restrict__ twz) {
  zinv_body<1536, 32, float2>(g, V0, V1, V2, Z, twz);
}

// --------------------------------------------------------------- k_zfwd ----
// transpose_xTOz + FFT (src/hst_transforms.f90:135-139, src/hst_fft.f90:181-193)
// keeping the 2nz+1 retained modes, stored without ghost rows.
template <typename C>
struct ZfwdDst {
  C* __restrict__ base;  // Q + (p ncol + ix nzT) ny + y0
  int ny, nz, NZ;
  __device__ __forceinline__ void operator()(int yi, int k, C v) const {
    int iz;
    if (k <= nz) iz = k;
    else if (k >= NZ - nz) iz = k - NZ;
    else return;
    base[(size_t)(iz + nz) * ny + yi] = v;
  }
};

// (the explicit one-block minimum lets the compiler take 160 registers
// for the 16-point plans, which measured 0.46 against 0.50 ms at 384^2 x
// 256; the same on k_zinv measured slower; the 8-point plans are held to
// three blocks an SM: at 768^2 x 512 4.68 against 5.19 ms for two in FP64,
// where the kernel waits on its global loads, while the z-inverse measured
// slower held to two or three)
template <int NT, int PPT, typename C>
__global__ void __launch_bounds__(PPT <= 8 ? 384 : (PPT == 32 && NT > 0 ? 192 : 256),
                                  PPT <= 8 ? 3 : (PPT == 32 && NT > 0 ? 2 : 1))
    k_zfwd(Geometry g, const C* __restrict__ Pp, C* __restrict__ Q, const C* __restrict__ twz) {
  extern __shared__ double2 sh_d[];
  C* sh = reinterpret_cast<C*>(sh_d);
  const int yt = ZFWD_IXF ? blockIdx.y : blockIdx.x, ix = ZFWD_IXF ? blockIdx.x : blockIdx.y;
  const int p = blockIdx.z % 6, mem = blockIdx.z / 6;
  const int Ty = g.Ty, NZ = g.nzd, nyT = g.ny / Ty;
  Pp += (size_t)mem * 6 * NZ * g.ny * g.nxB;
  Q += (size_t)mem * 6 * g.ncol * g.ny;
  const TileSrc<C> src = {Pp + (((size_t)p * nyT + yt) * NZ) * g.nxB * Ty + (size_t)ix * Ty, (size_t)g.nxB * Ty};
  const ZfwdDst<C> dst = {Q + ((size_t)p * g.ncol + (size_t)ix * g.nzT) * g.ny + yt * Ty, g.ny, g.nz, NZ};
  fft_sel<NT, -1, PPT, false, false, false, z_padded<NT, PPT, C>()>(NZ, Ty, twz, sh, src, dst);
}

// -------------------------------------------------------------- k_xprod ----
// to_x_points (zero padding + RFT), build_products for both groups,
// compute_cfl and HFT of the products (src/hst_transforms.f90:85-133,
// 163-179; src/hst_fft.f90:211-237) for one pair of rows at one z point.
// Two real lines ride on one complex line: u + i v of each row and w0 + i w1
// of the pair on the way in; (uu, vv), (ww, uv), (vw, uw) of each row on
// the way out, separated by Hermitian symmetry.  The c2r reads only the
// real part of the kx = 0 mode, as FFTW's and cuFFT's c2r do.
template <typename C>
struct XinvSrc {
  const C* __restrict__ zb;  // Z tile of component 0 at (y tile, kz), + row offset in the tile
  size_t cs;                 // component stride of Z
  int Ty, nx, NX;
  __device__ __forceinline__ C operator()(int l, int k) const {
    const int m = k <= nx ? k : (k >= NX - nx ? NX - k : -1);
    if (m < 0) return C{0, 0};
    const C* p = zb + (size_t)m * Ty;
    C a, b;
    if (l == 0) {  // u(y0) + i v(y0)
      a = p[0];
      b = p[cs];
    } else if (l == 1) {  // u(y1) + i v(y1)
      a = p[1];
      b = p[cs + 1];
    } else {  // w(y0) + i w(y1)
      a = p[2 * cs];
      b = p[2 * cs + 1];
    }
    if (k == 0) return C{a.x, b.x};
    if (k <= nx) return C{a.x - b.y, a.y + b.x};
    return C{a.x + b.y, b.x - a.y};  // conj(a) + i conj(b)
  }
};
// The same from the block's staging copy of the tile, [comp 3][nxB][row 2]
// (landed by TMA)
template <typename C>
struct XinvSh {
  const C* s;
  int nxB, nx, NX;
  __device__ __forceinline__ C operator()(int l, int k) const {
    const int m = k <= nx ? k : (k >= NX - nx ? NX - k : -1);
    if (m < 0) return C{0, 0};
    C a, b;
    if (l == 0) {
      a = s[2 * m];
      b = s[2 * (nxB + m)];
    } else if (l == 1) {
      a = s[2 * m + 1];
      b = s[2 * (nxB + m) + 1];
    } else {
      a = s[2 * (2 * nxB + m)];
      b = s[2 * (2 * nxB + m) + 1];
    }
    if (k == 0) return C{a.x, b.x};
    if (k <= nx) return C{a.x - b.y, a.y + b.x};
    return C{a.x + b.y, b.x - a.y};
  }
};
// the products of row yy, pair pl (0: uu, vv; 1: ww, uv; 2: vw, uw) at x
template <typename LT, typename C>
struct ProdSrc {
  typedef typename RealOf<C>::T T;
  LT L;
  T f;
  __device__ __forceinline__ C operator()(int l, int x) const {
    const int yy = l >= 3 ? 1 : 0, pl = l - 3 * yy;
    const C a = L(yy, x), b = L(2, x);
    const T u = a.x, v = a.y, w = yy ? b.y : b.x;
    if (pl == 0) return C{u * u * f, v * v * f};
    if (pl == 1) return C{w * w * f, u * v * f};
    return C{v * w * f, u * w * f};
  }
};

#ifndef XPROD_MINB
#define XPROD_MINB 3
#endif
#ifndef XPROD_PP
#define XPROD_PP 1
#endif
#ifndef XPAD1536
#define XPAD1536 1
#endif
// line stride of the padded 1536-point x lines: 1728 + 3 (FP64) or + 11
// (FP32), the strides that a CPU count of the plan's shared accesses ranks
// best for three and six lines side by side
__host__ __device__ constexpr int xls_1536(int elem) { return elem == 16 ? 1731 : 1739; }
// launch bounds of k_xprod: 6 NX / PPT threads; the 8-point plan at 384
// is held to 72 registers so that three 288-thread blocks fit an SM, the
// FP32 32-point plan at 1536 to two blocks
constexpr int xprod_threads(int NT, int PPT) {
  return PPT <= 8 ? (NT == 384 ? 288 : (NT == 768 ? 576 : 640)) : (NT == 1536 ? 288 : 320);
}
#ifndef XPROD_MINB_768
#define XPROD_MINB_768 2
#endif
#ifndef XPROD_MINB_F32
#define XPROD_MINB_F32 4
#endif
constexpr int xprod_min_blocks(int NT, int PPT, int es) {
  return PPT <= 8 && NT == 384 ? (es == 8 ? XPROD_MINB_F32 : XPROD_MINB) : ((NT == 1536 || NT == 768) && es == 8 ? 2 : (NT == 768 && PPT <= 8 ? XPROD_MINB_768 : 1));
}

constexpr int XPROD_WAIT_LIMIT = 1 << 22;  // polls of the tile's TMA barrier before giving up

// shared layout of the TMA variant (double2 units): the six padded lines,
// then the staging tile (in: [3][nxB][2], out: [6][nxB][2]) rounded up to
// the next 128-byte address (tensor copies need 128-byte aligned shared
// addresses, and the dynamic shared base is only known to be 16-byte
// aligned), then the mbarrier and the tile flag
// the x kernel's padded line stride: at least ls_padded(NX), and 3 LS half
// a bank row modulo a bank row (S = 128 / elem elements), for the
// separation's alternating reads of lines pl and pl + 3
__host__ __device__ constexpr int ls_x(int NX, int elem) {
  const int S = 128 / elem, base = ls_padded(NX);
  return elem == 16 ? base + (((S / 2 - base) % S) + S) % S : base;
}
__host__ __device__ inline int xprod_stage_off(int NX, int elem) { return 6 * ls_x(NX, elem); }
__host__ __device__ inline size_t xprod_tma_smem(int NX, int nxB, size_t elem) {
  return ((size_t)xprod_stage_off(NX, (int)elem) + 12 * (size_t)nxB + 2) * elem + 128;
}
// At 768 points the staging tiles live inside the six lines instead (the
// tile in where lines 3..5 are, which the three inverse lines never touch;
// the tile out over the lines once they have been read), so that a block
// needs 6 padded lines of shared memory and two blocks share an SM
__host__ __device__ constexpr bool xprod_alias(int NT, int PPT) { return PPT <= 8 && NT == 768; }
__host__ __device__ inline size_t xprod_alias_smem(int NX, size_t elem) {
  return (size_t)6 * ls_x(NX, (int)elem) * elem + 128;
}

template <int NT, int PPT, typename C>
__global__ void __launch_bounds__(xprod_threads(NT, PPT), xprod_min_blocks(NT, PPT, (int)sizeof(C)))
    k_xprod(Geometry g, const C* __restrict__ Z, C* __restrict__ Pp, const C* __restrict__ twx,
            const double* __restrict__ dyl, PhysScalars ps, int want_cfl, unsigned long long* __restrict__ cflmax,
            const __grid_constant__ CUtensorMap tmZ, const __grid_constant__ CUtensorMap tmP, int* __restrict__ err) {
  typedef typename RealOf<C>::T T;
  extern __shared__ double2 sh_d[];
  C* sh = reinterpret_cast<C*>(sh_d);
  // 8-point plans: butterflies index-fastest over padded shared lines, the
  // tile in and out by TMA
  constexpr bool JF = (PPT <= 8 && NT > 0);
  // the 1536-point plan (butterflies line-fastest): lines padded one in
  // eight at the stride xls_1536 (fewer bank conflicts for both the three
  // inverse and the six forward lines)
  constexpr int XSH = (!JF && NT == 1536 && XPAD1536) ? 3 : 0;
  using LT = std::conditional_t<JF, ShLinesPT<C>, std::conditional_t<XSH != 0, ShLinesPT<C, 3>, ShLinesT<C>>>;
  const int NX = 2 * g.nxd, nx = g.nx, nxB = g.nxB, NZ = g.nzd, Ty = g.Ty;
  const int LS = JF ? ls_x(NX, (int)sizeof(C)) : (XSH ? xls_1536((int)sizeof(C)) : NX + 1);
  const int nyT = g.ny / Ty;
  const int y0 = 2 * blockIdx.x, kz = blockIdx.y % g.nzd, mem = blockIdx.y / g.nzd;
  Z += (size_t)mem * 3 * g.nzd * g.ny * g.nxB;
  Pp += (size_t)mem * 6 * g.nzd * g.ny * g.nxB;
  const int yt = y0 / Ty, yi0 = y0 - yt * Ty;
  const size_t cs = (size_t)NZ * nyT * nxB * Ty;
  const size_t tile = ((size_t)yt * NZ + kz) * nxB * Ty;
  const LT L = {sh, LS};
  constexpr bool ALIAS = xprod_alias(NT, PPT);
  auto align128 = [](C* q) { return q + ((128u - (smem_u32(q) & 127u)) & 127u) / sizeof(C); };
  C* stg = ALIAS ? sh + 3 * LS : sh + xprod_stage_off(NX, (int)sizeof(C));
  if constexpr (JF) stg = align128(stg);
  C* const stg_out = ALIAS ? align128(sh) : stg;
  __shared__ uint64_t bar_al;
  __shared__ int tile_ok_al;
  // u + i v of both rows and w0 + i w1 on the physical x grid
  if constexpr (JF) {
    uint64_t* bar = ALIAS ? &bar_al : reinterpret_cast<uint64_t*>(stg + 12 * nxB);
    int& tile_ok = ALIAS ? tile_ok_al : *reinterpret_cast<int*>(stg + 12 * nxB + 1);
    if ((smem_u32(stg) & 127u) != 0) {  // never taken: the staging tile is aligned above
      if (threadIdx.x == 0) atomicExch(err, 1);
      return;
    }
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
      mbar_arrive_expect_tx(bar, 3u * nxB * 2u * (unsigned)sizeof(C));
      tma_load_4d(stg, &tmZ, 2 * yi0, 0, yt * NZ + kz, 3 * mem, bar);
      bool ok = mbar_wait_bounded(bar, 0, XPROD_WAIT_LIMIT);
      if (!ok) {
        // record the failure and give the copy a second bounded wait
        // before the block (and its shared memory) goes away
        atomicExch(err, 1);
        mbar_wait_bounded(bar, 0, XPROD_WAIT_LIMIT);
      }
      tile_ok = ok;
    }
    __syncthreads();
    if (!tile_ok) return;
    // the three inverse lines ping-pong between lines 0..2 and 3..5 (the
    // tile in lies in 3..5 at 768 points, read by the first stage only)
    const XinvSh<C> xs = {stg, nxB, nx, NX};
    constexpr bool PP = XPROD_PP && Plan8<NT>::n == 3;
    fft_sel<NT, +1, PPT, false, true, JF, false, PP>(NX, 3, twx + NX, sh, xs, L, sh + 3 * LS, LS);
  } else {
    const XinvSrc<C> xs = {Z + tile + yi0, cs, Ty, nx, NX};
    fft_sel<NT, +1, PPT, false, true, JF, false, false, XSH>(NX, 3, twx, sh, xs, L, sh, LS);
  }
  __syncthreads();
  if (want_cfl) {
    double cm = 0.0;
    const double rdy0 = dyl[y0], rdy1 = dyl[y0 + 1];
    for (int x = threadIdx.x; x < NX; x += blockDim.x) {
      const C a0 = L(0, x), a1 = L(1, x), b = L(2, x);
      double c0 = fabs((double)a0.x) / ps.dx + fabs((double)a0.y) / rdy0 + fabs((double)b.x) / ps.dz;
      double c1 = fabs((double)a1.x) / ps.dx + fabs((double)a1.y) / rdy1 + fabs((double)b.y) / ps.dz;
      cm = nan_max(cm, nan_max(c0, c1));
    }
    for (int o = 16; o > 0; o >>= 1) cm = nan_max(cm, __shfl_xor_sync(0xffffffffu, cm, o));
    // a NaN keeps its bits: as an unsigned word it exceeds every finite
    // non-negative double and infinity, so it wins the maximum and the host
    // sees a non-finite CFL number
    if ((threadIdx.x & 31) == 0) atomicMax(cflmax, (unsigned long long)__double_as_longlong(cm));
  }
  // the six product lines, transformed forward in place
  const ProdSrc<LT, C> ps6 = {L, (T)ps.factor};
  fft_sel<NT, -1, PPT, true, true, JF, false, false, XSH>(NX, 6, JF ? twx + NX : twx, sh, ps6, L, sh, LS);
  __syncthreads();
  // separate the two real transforms of each line, keep kx = 0..nx.  In
  // FP64, with the tile out ([comp][ix][row]), item e is (row e & 1, mode
  // e >> 1), so that a warp's stores are consecutive; the lines' stride
  // (ls_x: 3 LS is half a bank row modulo a bank row) keeps the alternating
  // reads of lines pl and pl + 3 on distinct banks too (384^2 x 256: 1.151
  // -> 1.102 ms; in FP32 the same measured slower at 768 points, 7.66
  // against 7.29 ms, and the items stay (mode, both rows)).
  constexpr bool ALT = sizeof(C) == 16;
  if constexpr (ALIAS && !ALT) {
    // the tile out overlays the lines: every thread reads its (at most two,
    // as 3 nxB <= NX <= 2 blockDim) entries first, then writes
    C zk[2][2], zm[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e < nxB * 3) {
        const int pl = e / nxB, ix = e - pl * nxB;
#pragma unroll
        for (int yy = 0; yy < 2; ++yy) {
          zk[k][yy] = L(pl + 3 * yy, ix);
          zm[k][yy] = L(pl + 3 * yy, ix == 0 ? 0 : NX - ix);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e < nxB * 3) {
        const int pl = e / nxB, ix = e - pl * nxB;
#pragma unroll
        for (int yy = 0; yy < 2; ++yy) {
          const C Zk = zk[k][yy], Zm = zm[k][yy];
          const T h = T(0.5);
          stg_out[((2 * pl) * nxB + ix) * 2 + yy] = C{h * (Zk.x + Zm.x), h * (Zk.y - Zm.y)};
          stg_out[((2 * pl + 1) * nxB + ix) * 2 + yy] = C{h * (Zk.y + Zm.y), h * (Zm.x - Zk.x)};
        }
      }
    }
  } else if constexpr (ALIAS) {
    // the tile out overlays the lines: every thread reads its (at most
    // three, as 6 nxB <= 3 blockDim) entries first, then writes
    C zk[3], zm[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e < nxB * 6) {
        const int yy = e & 1, q = e >> 1, pl = q / nxB, ix = q - pl * nxB;
        zk[k] = L(pl + 3 * yy, ix);
        zm[k] = L(pl + 3 * yy, ix == 0 ? 0 : NX - ix);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e < nxB * 6) {
        const int yy = e & 1, q = e >> 1, pl = q / nxB, ix = q - pl * nxB;
        const C Zk = zk[k], Zm = zm[k];
        const T h = T(0.5);
        stg_out[((2 * pl) * nxB + ix) * 2 + yy] = C{h * (Zk.x + Zm.x), h * (Zk.y - Zm.y)};
        stg_out[((2 * pl + 1) * nxB + ix) * 2 + yy] = C{h * (Zk.y + Zm.y), h * (Zm.x - Zk.x)};
      }
    }
  } else if constexpr (JF && ALT) {
    for (int e = threadIdx.x; e < nxB * 6; e += blockDim.x) {
      const int yy = e & 1, q = e >> 1, pl = q / nxB, ix = q - pl * nxB;
      const int ln = pl + 3 * yy;
      const C Zk = L(ln, ix), Zm = L(ln, ix == 0 ? 0 : NX - ix);
      const T h = T(0.5);
      stg[((2 * pl) * nxB + ix) * 2 + yy] = C{h * (Zk.x + Zm.x), h * (Zk.y - Zm.y)};
      stg[((2 * pl + 1) * nxB + ix) * 2 + yy] = C{h * (Zk.y + Zm.y), h * (Zm.x - Zk.x)};
    }
  } else {
    for (int e = threadIdx.x; e < nxB * 3; e += blockDim.x) {
      int pl = e / nxB, ix = e - pl * nxB;
#pragma unroll
      for (int yy = 0; yy < 2; ++yy) {
        const int ln = pl + 3 * yy;
        const C Zk = L(ln, ix), Zm = L(ln, ix == 0 ? 0 : NX - ix);
        const T h = T(0.5);
        const C X = C{h * (Zk.x + Zm.x), h * (Zk.y - Zm.y)};
        const C Y = C{h * (Zk.y + Zm.y), h * (Zm.x - Zk.x)};
        if constexpr (JF) {
          stg[((2 * pl) * nxB + ix) * 2 + yy] = X;
          stg[((2 * pl + 1) * nxB + ix) * 2 + yy] = Y;
        } else {
          size_t o = tile + (size_t)ix * Ty + yi0 + yy;
          Pp[(size_t)(2 * pl) * cs + o] = X;
          Pp[(size_t)(2 * pl + 1) * cs + o] = Y;
        }
      }
    }
  }
  if constexpr (JF) {
    // the six spectra of both rows in one tensor store
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tma_store_4d(&tmP, 2 * yi0, 0, yt * NZ + kz, 6 * mem, stg_out);
      bulk_commit();
      bulk_wait_read_all();
    }
  }
}

// --------------------------------------- the reference-layout transforms ----
// FFT, IFT, RFT and HFT (src/hst_fft.f90:181-237) on the buffers of the
// per-piece path, which hold the reference's layouts: VVdz(nzd, nx+1,
// -2:ny+1, 3) and VVdx / VVdp(nxd+1, nzd, -2:ny+1, 3), the latter also seen as
// 2(nxd+1) reals a line (rVVdx, products).  A block loads LPB whole lines
// into shared memory, transforms them there with the runtime plan and
// writes them back over the same bytes (every line is read before any is
// written, so the in-place real <-> complex layouts are safe).  These serve
// the drop-in per-piece interface; the fused substep does not use them.
static int fft_threads(int points, int ppt);
struct PieceLines {
  double2* base;  // line l starts at base + l * stride (complex elements)
  size_t stride;
  int kind;       // 0: complex z line; 1: c2r x line (Hermitian, nxd+1 modes in); 2: r2c x line (reals in)
  int N;          // transform length
};
__device__ __forceinline__ double2 piece_load(const PieceLines& P, int l, int k) {
  const double2* b = P.base + (size_t)l * P.stride;
  if (P.kind == 0) return b[k];
  if (P.kind == 1) {
    const int h = P.N / 2;
    if (k <= h) return b[k];
    const double2 c = b[P.N - k];
    return make_double2(c.x, -c.y);
  }
  const double* r = reinterpret_cast<const double*>(b);
  return make_double2(r[k], 0.0);
}
template <int S>
__global__ void __launch_bounds__(256) k_piece_lines(PieceLines P, int nlines, int lpb, const double2* __restrict__ tw) {
  extern __shared__ double2 sh_d[];
  const int N = P.N, LS = N + 1;
  const int l0 = blockIdx.x * lpb;
  const int nl = min(lpb, nlines - l0);
  for (int e = threadIdx.x; e < lpb * N; e += blockDim.x) {
    const int l = e / N, k = e - l * N;
    sh_d[l * LS + k] = l < nl ? piece_load(P, l0 + l, k) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const ShLinesT<double2> L = {sh_d, LS};
  fft_global<S, 16, true, true>(N, lpb, tw, sh_d, L, L);
  __syncthreads();
  if (P.kind == 1) {  // real parts: 2(nxd+1) reals a line, the two past N zero
    for (int e = threadIdx.x; e < nl * (N + 2); e += blockDim.x) {
      const int l = e / (N + 2), k = e - l * (N + 2);
      double* r = reinterpret_cast<double*>(P.base + (size_t)(l0 + l) * P.stride);
      r[k] = k < N ? sh_d[l * LS + k].x : 0.0;
    }
  } else {
    const int nout = P.kind == 0 ? N : N / 2 + 1;
    for (int e = threadIdx.x; e < nl * nout; e += blockDim.x) {
      const int l = e / nout, k = e - l * nout;
      P.base[(size_t)(l0 + l) * P.stride + k] = sh_d[l * LS + k];
    }
  }
}

// kind 0/1/2 as PieceLines; S the transform's sign (+1 backward)
cudaError_t launch_piece_lines(const DeviceState& d, double2* base, size_t stride, int nlines, int N, int kind, int S,
                               const double2* tw, cudaStream_t st) {
  if (!plan_ok(N) || nlines <= 0) return cudaErrorInvalidValue;
  const PieceLines P = {base, stride, kind, N};
  const int lpb = N >= 1536 ? 1 : (N >= 768 ? 2 : 4);
  const int threads = fft_threads(lpb * N, 16);
  if (threads > 256) return cudaErrorInvalidValue;
  const size_t smem = (size_t)lpb * (N + 1) * sizeof(double2);
  const int blocks = (nlines + lpb - 1) / lpb;
  if (S > 0) {
    smem_limit(d, k_piece_lines<+1>, 220 * 1024);
    k_piece_lines<+1><<<blocks, threads, smem, st>>>(P, nlines, lpb, tw);
  } else {
    smem_limit(d, k_piece_lines<-1>, 220 * 1024);
    k_piece_lines<-1><<<blocks, threads, smem, st>>>(P, nlines, lpb, tw);
  }
  return cudaGetLastError();
}

// ------------------------------------------------------- staged twiddles ----
// The twiddles of the 8-point plan of N in stage order (see fft_stage_io):
// for each stage after the first, [r - 1][kk] = W_N^(kk r N/(Ns R)).
template <int N, typename C>
static int staged_twiddles_t(C* out) {
  using PL = Plan8<N>;
  const int rad[3] = {PL::r0, PL::r1, PL::r2};
  int n = 0, Ns = 1;
  for (int st = 0; st < PL::n; ++st) {
    const int R = rad[st];
    if (Ns > 1)
      for (int r = 1; r < R; ++r)
        for (int kk = 0; kk < Ns; ++kk) {
          const long e = (long)kk * r * (N / (Ns * R)) % N;
          long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)N;
          out[n].x = (typename RealOf<C>::T)cosl(a);
          out[n++].y = (typename RealOf<C>::T)sinl(a);
        }
    Ns *= R;
  }
  return n;
}

int staged_twiddles(int N, double2* out) {
  switch (N) {
    case 192: return staged_twiddles_t<192>(out);
    case 384: return staged_twiddles_t<384>(out);
    case 768: return staged_twiddles_t<768>(out);
  }
  return 0;
}
int staged_twiddles(int N, float2* out) {
  switch (N) {
    case 192: return staged_twiddles_t<192>(out);
    case 384: return staged_twiddles_t<384>(out);
    case 768: return staged_twiddles_t<768>(out);
  }
  return 0;
}

// ------------------------------------------------------------- TMA maps ----
// Z and Pp seen as 4-D f64 tensors: d0 = the 2 Ty doubles of one y tile
// (innermost), d1 = ix, d2 = (y tile, kz) as yt nzd + kz, d3 = component.
// The x kernel's box is {4 doubles (two rows), nxB, 1, comps}.
static bool xprod_uses_maps(const Geometry& g) {
  const int NX = 2 * g.nxd;
  return (g.pptx == 8 || g.mp) && (NX == 192 || NX == 384 || NX == 768) && g.nxB <= 256;
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

cudaError_t make_transform_maps(const Geometry& g, DeviceState& d) {
  d.maps = false;
  {
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 == cudaSuccess) e0 = cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e0 != cudaSuccess) return e0;
  }
  if (!xprod_uses_maps(g)) return cudaSuccess;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
  const EncodeTiled enc = reinterpret_cast<EncodeTiled>(fn);
  const int nyT = g.ny / g.Ty;
  for (int which = 0; which < 2; ++which) {
    const cuuint32_t comps = which == 0 ? 3 : 6;
    cuuint64_t dims[4] = {(cuuint64_t)2 * g.Ty, (cuuint64_t)g.nxB, (cuuint64_t)g.nzd * nyT, (cuuint64_t)comps * g.nmem};
    const cuuint64_t es = g.mp ? 8 : 16;  // bytes of one complex element
    cuuint64_t strides[3] = {es * g.Ty, es * g.Ty * g.nxB, es * g.Ty * g.nxB * g.nzd * nyT};
    cuuint32_t box[4] = {4, (cuuint32_t)g.nxB, 1, comps};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(which == 0 ? &d.tmZ : &d.tmPp, g.mp ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                     which == 0 ? (void*)d.Z : (void*)d.Pp, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    if (d.Zg) {  // the ghost rows' buffers: one tile of four rows
      cuuint64_t dg[4] = {8, (cuuint64_t)g.nxB, (cuuint64_t)g.nzd, (cuuint64_t)comps * g.nmem};
      cuuint64_t sg[3] = {es * 4, es * 4 * g.nxB, es * 4 * g.nxB * g.nzd};
      r = enc(which == 0 ? &d.tmZg : &d.tmPpg, g.mp ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
              which == 0 ? (void*)d.Zg : (void*)d.Ppg, dg, sg, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
  }
  d.maps = true;
  return cudaSuccess;
}

bool edge_rows_needed(const Geometry& g, bool s2_active) { return s2_active && g.nzd <= 3 * g.nz; }

// The view of the four ghost rows: the same transforms with ny = Ty = 4 on
// the edge buffers
static void edge_view(const Geometry& g, const DeviceState& d, Geometry& ge, DeviceState& de) {
  ge = g;
  ge.ny = 4;
  ge.Ty = 4;
  ge.edge_gap = g.ny;
  de = d;
  de.Z = d.Zg;
  de.Pp = d.Ppg;
  de.Q = d.Qg;
  de.tmZ = d.tmZg;
  de.tmPp = d.tmPpg;
}

// -------------------------------------------------------------- launchers ----
static int fft_threads(int points, int ppt) {
  int t = (points + ppt - 1) / ppt;
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

template <typename K>
static void big_smem(const DeviceState& d, K k) {
  smem_limit(d, k, 220 * 1024);
}

// Dispatch on the transform length: compile-time plans for the lengths the
// workloads use, with 8 points a thread (radix <= 12, P8) or 16 up to 384
// and 32 above (radix 16/24), the runtime plan otherwise.
#define HST_FFT_DISPATCH(N, PTS, P8, CALL)                  \
  do {                                                      \
    switch (N) {                                            \
      case 12: CALL(12, 16) break;                          \
      case 24: CALL(24, 16) break;                          \
      case 48: CALL(48, 16) break;                          \
      case 96: CALL(96, 16) break;                          \
      case 192:                                             \
        if (P8) CALL(192, 8) else CALL(192, 16) break;      \
      case 384:                                             \
        if (P8) CALL(384, 8) else CALL(384, 16) break;      \
      case 768:                                             \
        if (P8) CALL(768, 8) else CALL(768, 32) break;      \
      case 1536: CALL(1536, 32) break;                      \
      default:                                              \
        if ((PTS) <= 16 * 256) CALL(0, 16) else CALL(0, 32) \
        break;                                              \
    }                                                       \
  } while (0)

// The mixed-precision form compiles the transforms for the lengths its
// workloads use: 8 points a thread at 192, 384 and 768, 16 at 96, 32 (the
// radix 16, 16, 6 plan) at 1536.
#define HST_FFT_DISPATCH_MP(N, P16, CALL)          \
  do {                                             \
    switch (N) {                                   \
      case 96: CALL(96, 16) break;                 \
      case 192:                                    \
        if (P16) CALL(192, 16) else CALL(192, 8) break; \
      case 384:                                    \
        if (P16) CALL(384, 16) else CALL(384, 8) break; \
      case 768: CALL(768, 8) break;                \
      case 1536: CALL(1536, 32) break;             \
      default:                                     \
        return cudaErrorInvalidValue;              \
    }                                              \
  } while (0)

bool mp_length_ok(int n) { return n == 96 || n == 192 || n == 384 || n == 768 || n == 1536; }

static cudaError_t launch_zinv_main(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  const int pts = g.nzd * g.Ty;
  const dim3 grid(ZINV_IXF ? g.nxB : g.ny / g.Ty, ZINV_IXF ? g.ny / g.Ty : g.nxB, 3 * g.nmem);
  if (g.mp) {
    typedef float2 C;
    C* Z = reinterpret_cast<C*>(d.Z);
#define HST_ZINV(NT, PPT)                                                                                     \
  {                                                                                                           \
    const size_t smem = z_smem<NT, PPT, C>(g.nzd, g.Ty);                                                      \
    if (NT == 1536) {                                                                                         \
      big_smem(d, k_zinv_1536f);                                                                                 \
      k_zinv_1536f<<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.F[0], d.F[1], d.F[2], Z, d.twzf);          \
    } else {                                                                                                  \
      big_smem(d, k_zinv<NT, PPT, C>);                                                                           \
      k_zinv<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.F[0], d.F[1], d.F[2], Z, d.twzf);    \
    }                                                                                                         \
  }
    HST_FFT_DISPATCH_MP(g.nzd, g.pptz == 16, HST_ZINV);
#undef HST_ZINV
    return cudaGetLastError();
  }
  typedef double2 C;
#define HST_ZINV(NT, PPT)                                                                                     \
  {                                                                                                           \
    const size_t smem = z_smem<NT, PPT, C>(g.nzd, g.Ty);                                                      \
    if (PPT == 32 && NT > 0) {                                                                                \
      big_smem(d, k_zinv_32<NT>);                                                                             \
      k_zinv_32<NT><<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.F[0], d.F[1], d.F[2], d.Z, d.twz);        \
    } else {                                                                                                  \
      big_smem(d, k_zinv<NT, PPT, C>);                                                                        \
      k_zinv<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.F[0], d.F[1], d.F[2], d.Z, d.twz);   \
    }                                                                                                         \
  }
  HST_FFT_DISPATCH(g.nzd, pts, g.pptz == 8, HST_ZINV);
#undef HST_ZINV
  return cudaGetLastError();
}

static cudaError_t launch_zfwd_main(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  const int pts = g.nzd * g.Ty;
  const dim3 grid(ZFWD_IXF ? g.nxB : g.ny / g.Ty, ZFWD_IXF ? g.ny / g.Ty : g.nxB, 6 * g.nmem);
  if (g.mp) {
    typedef float2 C;
    const C* Pp = reinterpret_cast<const C*>(d.Pp);
    C* Q = reinterpret_cast<C*>(d.Q);
#define HST_ZFWD(NT, PPT)                                                                  \
  {                                                                                        \
    const size_t smem = z_smem<NT, PPT, C>(g.nzd, g.Ty);                                   \
    big_smem(d, k_zfwd<NT, PPT, C>);                                                          \
    k_zfwd<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, Pp, Q, d.twzf);       \
  }
    HST_FFT_DISPATCH_MP(g.nzd, g.pptz == 16, HST_ZFWD);
#undef HST_ZFWD
    return cudaGetLastError();
  }
  typedef double2 C;
#define HST_ZFWD(NT, PPT)                                                                  \
  {                                                                                        \
    const size_t smem = z_smem<NT, PPT, C>(g.nzd, g.Ty);                                   \
    big_smem(d, k_zfwd<NT, PPT, C>);                                                          \
    k_zfwd<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.Pp, d.Q, d.twz);    \
  }
  HST_FFT_DISPATCH(g.nzd, pts, g.pptz == 8, HST_ZFWD);
#undef HST_ZFWD
  return cudaGetLastError();
}

static cudaError_t launch_xprod_main(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int want_cfl,
                                     cudaStream_t st) {
  const int NX = 2 * g.nxd;
  const int pts = 6 * NX;
  if (xprod_uses_maps(g) != d.maps) return cudaErrorInvalidValue;
  const dim3 grid(g.ny / 2, g.nzd * g.nmem);
  if (g.mp) {
    typedef float2 C;
    const size_t lines = (size_t)6 * (NX == 1536 && XPAD1536 ? xls_1536(8) : NX + 1) * sizeof(C);
    const size_t smem = !xprod_uses_maps(g) ? lines
                        : (NX == 768 ? xprod_alias_smem(NX, sizeof(C)) : xprod_tma_smem(NX, g.nxB, sizeof(C)));
    const C* Z = reinterpret_cast<const C*>(d.Z);
    C* Pp = reinterpret_cast<C*>(d.Pp);
#define HST_XPROD(NT, PPT)                                                                                    \
  {                                                                                                           \
    big_smem(d, k_xprod<NT, PPT, C>);                                                                            \
    k_xprod<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, Z, Pp, d.twxf, d.dyl, ph, want_cfl,     \
                                                                    d.cfl, d.tmZ, d.tmPp, d.err);             \
  }
    HST_FFT_DISPATCH_MP(NX, false, HST_XPROD);
#undef HST_XPROD
    return cudaGetLastError();
  }
  typedef double2 C;
  const size_t lines = (size_t)6 * (NX == 1536 && XPAD1536 ? xls_1536(16) : NX + 1) * sizeof(C);
  const size_t smem = !xprod_uses_maps(g) ? lines
                      : (NX == 768 && g.pptx == 8 ? xprod_alias_smem(NX, sizeof(C))
                                                  : xprod_tma_smem(NX, g.nxB, sizeof(C)));
#define HST_XPROD(NT, PPT)                                                                                    \
  {                                                                                                           \
    big_smem(d, k_xprod<NT, PPT, C>);                                                                            \
    k_xprod<NT, PPT, C><<<grid, fft_threads(pts, PPT), smem, st>>>(g, d.Z, d.Pp, d.twx, d.dyl, ph, want_cfl,  \
                                                                    d.cfl, d.tmZ, d.tmPp, d.err);             \
  }
  HST_FFT_DISPATCH(NX, pts, g.pptx == 8, HST_XPROD);
#undef HST_XPROD
  return cudaGetLastError();
}

// each transform of the interior rows, then (when the context keeps them)
// of the four ghost rows; the ghost rows take no part in the CFL number
cudaError_t launch_zinv(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  cudaError_t e = launch_zinv_main(g, d, st);
  if (e != cudaSuccess || !d.Qg) return e;
  Geometry ge;
  DeviceState de;
  edge_view(g, d, ge, de);
  return launch_zinv_main(ge, de, st);
}
cudaError_t launch_xprod(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int want_cfl,
                         cudaStream_t st) {
  cudaError_t e = launch_xprod_main(g, d, ph, want_cfl, st);
  if (e != cudaSuccess || !d.Qg) return e;
  Geometry ge;
  DeviceState de;
  edge_view(g, d, ge, de);
  return launch_xprod_main(ge, de, ph, 0, st);
}
cudaError_t launch_zfwd(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  cudaError_t e = launch_zfwd_main(g, d, st);
  if (e != cudaSuccess || !d.Qg) return e;
  Geometry ge;
  DeviceState de;
  edge_view(g, d, ge, de);
  return launch_zfwd_main(ge, de, st);
}

}  // namespace hst
