// Stockham FFTs for the 3/2-dealiased x and z transforms.
//
// A block transforms nl lines of length N = 2^a 3^b.  Each radix-R stage
// is one pass: a thread gathers the R inputs of its butterflies into
// registers, applies the stage twiddles, computes a radix-R DFT in
// registers (R up to 24, built from radix-2/3/4 pieces), and scatters the
// outputs.  The first stage reads through a caller's loader (global memory,
// or a function of other lines) and the last stage writes through a
// caller's storer, so only the exchanges between stages go through shared
// memory: N = 384 is two stages (16 x 24) with one shared exchange, N = 768
// three stages.  Threads are mapped line-fastest so that global accesses of
// consecutive threads touch consecutive lines (the y rows, contiguous in
// memory); shared lines have an odd stride against bank conflicts.
// Stage twiddles come from W[e] = exp(-2 pi i e / N) in global memory, the
// twiddles inside a register DFT from a 48-entry table in constant memory
// (all threads read the same entry).  Both tables are computed on the host
// in extended precision.  Unnormalised both ways, like the reference's FFTW
// and cuFFT plans (src/hst_fft.f90:98-121): S = -1 forward, S = +1 backward.
#pragma once
#include <type_traits>

#include "hst_dev.cuh"

namespace hst {

#define HST_SQRT3_2 0.86602540378443864676

// exp(-2 pi i k / 48), k = 0..47, in both precisions (set per device by
// set_fft_constants; this header is included by one translation unit only)
__constant__ double2 c_w48[48];
__constant__ float2 c_w48f[48];
template <typename C>
__device__ __forceinline__ C w48(int i);
template <>
__device__ __forceinline__ double2 w48<double2>(int i) { return c_w48[i]; }
template <>
__device__ __forceinline__ float2 w48<float2>(int i) { return c_w48f[i]; }

template <int R, int S>
struct DFT;

template <int S>
struct DFT<2, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int S>
struct DFT<4, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]), a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
    C a3r = S < 0 ? C{a3.y, -a3.x} : C{-a3.y, a3.x};
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3r);
    v[3] = csub(a1, a3r);
  }
};
template <int S>
struct DFT<3, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    typedef typename RealOf<C>::T T;
    const T h = T(0.5), q = T(HST_SQRT3_2);
    C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    C m = C{v[0].x - h * t1.x, v[0].y - h * t1.y};
    C r = S < 0 ? C{q * t2.y, -q * t2.x} : C{-q * t2.y, q * t2.x};
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
};
// R = A B: B DFTs of size A on the elements b + B a, the twiddles
// W_R^(b ka), A DFTs of size B; output k = ka + A kb.
template <int A, int B, int S, typename C>
__device__ __forceinline__ void dft_ab(C* v) {
  C o[A * B];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    C t[A];
#pragma unroll
    for (int a = 0; a < A; ++a) t[a] = v[b + B * a];
    DFT<A, S>::run(t);
#pragma unroll
    for (int ka = 0; ka < A; ++ka) {
      if (b * ka == 0) {
        v[b + B * ka] = t[ka];
      } else {
        C w = w48<C>((b * ka * (48 / (A * B))) % 48);
        if (S > 0) w.y = -w.y;
        v[b + B * ka] = cmul(t[ka], w);
      }
    }
  }
#pragma unroll
  for (int ka = 0; ka < A; ++ka) {
    C t[B];
#pragma unroll
    for (int b = 0; b < B; ++b) t[b] = v[b + B * ka];
    DFT<B, S>::run(t);
#pragma unroll
    for (int kb = 0; kb < B; ++kb) o[ka + A * kb] = t[kb];
  }
#pragma unroll
  for (int k = 0; k < A * B; ++k) v[k] = o[k];
}
template <int S>
struct DFT<6, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) { dft_ab<3, 2, S>(v); }
};
template <int S>
struct DFT<8, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) { dft_ab<4, 2, S>(v); }
};
template <int S>
struct DFT<12, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) { dft_ab<4, 3, S>(v); }
};
template <int S>
struct DFT<16, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) { dft_ab<4, 4, S>(v); }
};
template <int S>
struct DFT<24, S> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) { dft_ab<8, 3, S>(v); }
};

// The runtime radix plan of N: radix-16 stages while more than 24 is left,
// then the rest in one stage (2, 3, 4, 6, 8, 12, 16 or 24).
struct FftPlan {
  int n;
  int r[4];
};
__host__ __device__ inline FftPlan make_plan(int N) {
  FftPlan p;
  p.n = 0;
  int m = N;
  while (m > 24 && m % 16 == 0 && p.n < 3) {
    p.r[p.n++] = 16;
    m /= 16;
  }
  if (m > 1) p.r[p.n++] = m;
  return p;
}
__host__ inline bool plan_ok(int N) {
  FftPlan p = make_plan(N);
  int prod = 1;
  for (int i = 0; i < p.n; ++i) {
    int r = p.r[i];
    if (!(r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 12 || r == 16 || r == 24)) return false;
    prod *= r;
  }
  return prod == N;
}

// Shared-memory line access (line stride LS)
template <typename C>
struct ShLinesT {
  C* p;
  int LS;
  __device__ __forceinline__ C operator()(int l, int i) const { return p[l * LS + i]; }
  __device__ __forceinline__ void operator()(int l, int i, C v) const { p[l * LS + i] = v; }
};
typedef ShLinesT<cxd> ShLines;
// The same with one pad element after every 8: with butterflies mapped
// index-fastest (JF) the radix-8/6/12 exchanges of the 8-point plans are
// then free of bank conflicts.  Line stride ls_padded(N).
// (SH: one pad element in 2^SH; 3 for the 8-point plans, 4 for the
// 16-point plans of the z kernels, whose first radix is 16)
template <typename C, int SH = 3>
struct ShLinesPT {
  C* p;
  int LS;
  __device__ __forceinline__ C operator()(int l, int i) const { return p[l * LS + i + (i >> SH)]; }
  __device__ __forceinline__ void operator()(int l, int i, C v) const { p[l * LS + i + (i >> SH)] = v; }
};
typedef ShLinesPT<cxd> ShLinesP;
__host__ __device__ constexpr int ls_padded(int N) { return N + N / 8 + 1; }
// The line stride of the same padded layout under the line-fastest mapping
// of the z kernels (butterfly b: line b % nl, index b / nl, so that the
// global loads and stores of nl adjacent rows coalesce): a wavefront's
// lanes cover nl lines times S/nl consecutive indices (S = 128 / sizeof(C)
// elements a bank row), and a stride of S/nl (mod S) with the pad in eight
// spreads them over distinct banks in every stage of the 8-point plans
// (nl in {2, 4, 8}).
template <typename C, int SH = 3>
__host__ __device__ inline int ls_lines(int N, int nl) {
  const int S = 128 / (int)sizeof(C);
  const int target = (S / nl) % S;
  const int base = N + (N >> SH);
  return base + ((target - base) % S + S) % S;
}

// One radix-R stage.  Butterfly b of the block: line l = b % nl, index
// j = b / nl.  Inputs ld(l, j + r N/R), outputs st(l, (j/Ns) Ns R + j%Ns + r Ns).
// SYNC: the stage reads and writes the same shared lines (all reads, then
// a barrier, then all writes).
// JF also selects the staged twiddle table: tw points at this stage's
// block [r - 1][kk] of W^(kk r N/(Ns R)), r = 1..R-1, kk = 0..Ns-1, so that
// a warp's twiddle loads are contiguous.
template <int R, int S, int PPT, bool SYNC, typename LD, typename ST, bool JF = false, typename C = cxd>
__device__ __forceinline__ void fft_stage_io(int N, int nl, int Ns, const C* __restrict__ tw, const LD& ld,
                                             const ST& st) {
  constexpr int MAXB = (PPT + R - 1) / R;
  const int nb = N / R;
  const int total = nb * nl;
  const int tstride = N / (Ns * R);
  C v[MAXB][R];
  int lj[MAXB];
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    int b = threadIdx.x + k * blockDim.x;
    lj[k] = -1;
    if (b < total) {
      int l = JF ? b / nb : b % nl, j = JF ? b % nb : b / nl;
      int kk = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        C x = ld(l, j + r * nb);
        if (r > 0 && kk > 0) {
          C w = JF ? __ldg(tw + (r - 1) * Ns + kk) : __ldg(tw + kk * r * tstride);
          if (S > 0) w.y = -w.y;
          x = cmul(x, w);
        }
        v[k][r] = x;
      }
      DFT<R, S>::run(v[k]);
      lj[k] = b;
    }
  }
  if (SYNC) __syncthreads();
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    if (lj[k] >= 0) {
      int l = JF ? lj[k] / nb : lj[k] % nl, j = JF ? lj[k] % nb : lj[k] / nl;
      int kk = j % Ns;
      int base = (j / Ns) * Ns * R + kk;
#pragma unroll
      for (int r = 0; r < R; ++r) st(l, base + r * Ns, v[k][r]);
    }
  }
}

template <int S, int PPT, bool SYNC, typename LD, typename ST, typename C>
__device__ __forceinline__ void fft_stage_r(int R, int N, int nl, int Ns, const C* __restrict__ tw, const LD& ld,
                                            const ST& st) {
  switch (R) {
    case 2: fft_stage_io<2, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 3: fft_stage_io<3, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 4: fft_stage_io<4, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 6: fft_stage_io<6, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 8: fft_stage_io<8, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 12: fft_stage_io<12, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 16: fft_stage_io<16, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    case 24: fft_stage_io<24, S, PPT, SYNC>(N, nl, Ns, tw, ld, st); break;
    default: break;
  }
}

// The whole transform of nl lines with the runtime plan: the first stage
// reads through src, the last writes through dst, the stages between
// exchange through `sh` (nl lines of stride N+1).  SRC_SH / DST_SH: src
// reads, dst writes the same shared buffer (the stage then synchronises
// between its reads and its writes).  Requires nl N <= PPT blockDim.x.
template <int S, int PPT, bool SRC_SH, bool DST_SH, typename LD, typename ST, typename C>
__device__ void fft_global(int N, int nl, const C* __restrict__ tw, C* sh, const LD& src, const ST& dst) {
  const FftPlan P = make_plan(N);
  const ShLinesT<C> L = {sh, N + 1};
  int Ns = 1;
  if (P.n == 1) {
    fft_stage_r<S, PPT, SRC_SH && DST_SH>(P.r[0], N, nl, Ns, tw, src, dst);
    return;
  }
  fft_stage_r<S, PPT, SRC_SH>(P.r[0], N, nl, Ns, tw, src, L);
  Ns *= P.r[0];
  __syncthreads();
  for (int s = 1; s + 1 < P.n; ++s) {
    fft_stage_r<S, PPT, true>(P.r[s], N, nl, Ns, tw, L, L);
    Ns *= P.r[s];
    __syncthreads();
  }
  fft_stage_r<S, PPT, DST_SH>(P.r[P.n - 1], N, nl, Ns, tw, L, dst);
}

// Compile-time plans of the lengths the configurations use (the 3/2-padded
// sizes 2^a 3 from 12 to 1536), so that each kernel instantiates only the
// radices it runs.
template <int N>
struct Plan {
  static constexpr int n = 0, r0 = 1, r1 = 1, r2 = 1;
};
template <> struct Plan<12> { static constexpr int n = 1, r0 = 12, r1 = 1, r2 = 1; };
template <> struct Plan<24> { static constexpr int n = 1, r0 = 24, r1 = 1, r2 = 1; };
template <> struct Plan<48> { static constexpr int n = 2, r0 = 16, r1 = 3, r2 = 1; };
template <> struct Plan<96> { static constexpr int n = 2, r0 = 16, r1 = 6, r2 = 1; };
template <> struct Plan<192> { static constexpr int n = 2, r0 = 16, r1 = 12, r2 = 1; };
template <> struct Plan<384> { static constexpr int n = 2, r0 = 16, r1 = 24, r2 = 1; };
template <> struct Plan<768> { static constexpr int n = 3, r0 = 16, r1 = 16, r2 = 3; };
template <> struct Plan<1536> { static constexpr int n = 3, r0 = 16, r1 = 16, r2 = 6; };

// Plans of at most radix 12 for 8 points a thread: more stages (one more
// shared exchange) for far fewer registers, hence more resident warps.
template <int N>
struct Plan8 {
  static constexpr int n = 0, r0 = 1, r1 = 1, r2 = 1;
};
template <> struct Plan8<12> { static constexpr int n = 1, r0 = 12, r1 = 1, r2 = 1; };
template <> struct Plan8<24> { static constexpr int n = 2, r0 = 4, r1 = 6, r2 = 1; };
template <> struct Plan8<48> { static constexpr int n = 2, r0 = 8, r1 = 6, r2 = 1; };
template <> struct Plan8<96> { static constexpr int n = 2, r0 = 8, r1 = 12, r2 = 1; };
template <> struct Plan8<192> { static constexpr int n = 3, r0 = 8, r1 = 4, r2 = 6; };
template <> struct Plan8<384> { static constexpr int n = 3, r0 = 8, r1 = 8, r2 = 6; };
template <> struct Plan8<768> { static constexpr int n = 3, r0 = 8, r1 = 8, r2 = 12; };

// PZ: the padded lines at stride ls_lines under the line-fastest mapping.
// PP (three-stage plans): the second stage writes a second set of nl lines
// at sh2 and the third reads them, so that neither stage reads and writes
// the same lines (two barriers fewer); src must not overlap the lines at sh
// and dst not those at sh2.
// XSH > 0: the caller's padded layout, one pad in 2^XSH at line stride lsx;
// with JF, lsx > 0 is the stride of the padded lines (at least ls_padded).
template <int N, int S, int PPT, bool SRC_SH, bool DST_SH, bool JF, bool PZ, bool PP, int XSH, typename LD,
          typename ST, typename C>
__device__ __forceinline__ void fft_fixed(int nl, const C* __restrict__ tw, C* sh, const LD& src, const ST& dst,
                                          C* sh2, int lsx) {
  using PL = std::conditional_t<(PPT <= 8), Plan8<N>, Plan<N>>;
  static_assert(PL::n > 0, "no compile-time plan for this length and points per thread");
  static_assert(!(JF && (PZ || XSH > 0)), "PZ and XSH are the line-fastest mapping's layouts");
  // the pad follows the plan's first radix (8 or 16), or the caller's
  constexpr int PSH = XSH > 0 ? XSH : (PPT <= 8 ? 3 : 4);
  using LT = std::conditional_t<JF, ShLinesPT<C>, std::conditional_t<(PZ || XSH > 0), ShLinesPT<C, PSH>, ShLinesT<C>>>;
  const LT L = {sh, JF ? (lsx > 0 ? lsx : ls_padded(N)) : (XSH > 0 ? lsx : (PZ ? ls_lines<C, PSH>(N, nl) : N + 1))};
  if constexpr (PL::n == 1) {
    fft_stage_io<PL::r0, S, PPT, SRC_SH && DST_SH, LD, ST, JF, C>(N, nl, 1, tw, src, dst);
  } else if constexpr (PL::n == 2) {
    fft_stage_io<PL::r0, S, PPT, SRC_SH, LD, LT, JF, C>(N, nl, 1, tw, src, L);
    __syncthreads();
    fft_stage_io<PL::r1, S, PPT, DST_SH, LT, ST, JF, C>(N, nl, PL::r0, tw, L, dst);
  } else {
    // staged table (JF): stage 2's block first, then stage 3's
    const C* tw3 = JF ? tw + (PL::r1 - 1) * PL::r0 : tw;
    fft_stage_io<PL::r0, S, PPT, SRC_SH, LD, LT, JF, C>(N, nl, 1, tw, src, L);
    __syncthreads();
    if constexpr (PP) {
      const LT L2 = {sh2, L.LS};
      fft_stage_io<PL::r1, S, PPT, false, LT, LT, JF, C>(N, nl, PL::r0, tw, L, L2);
      __syncthreads();
      fft_stage_io<PL::r2, S, PPT, false, LT, ST, JF, C>(N, nl, PL::r0 * PL::r1, tw3, L2, dst);
    } else {
      fft_stage_io<PL::r1, S, PPT, true, LT, LT, JF, C>(N, nl, PL::r0, tw, L, L);
      __syncthreads();
      fft_stage_io<PL::r2, S, PPT, DST_SH, LT, ST, JF, C>(N, nl, PL::r0 * PL::r1, tw3, L, dst);
    }
  }
}

// NT > 0: the compile-time plan of length NT; NT = 0: the runtime plan of N.
template <int NT, int S, int PPT, bool SRC_SH, bool DST_SH, bool JF = false, bool PZ = false, bool PP = false,
          int XSH = 0, typename LD, typename ST, typename C>
__device__ __forceinline__ void fft_sel(int N, int nl, const C* __restrict__ tw, C* sh, const LD& src,
                                        const ST& dst, C* sh2 = nullptr, int lsx = 0) {
  static_assert(!(PZ || PP || XSH > 0) || NT > 0, "PZ, PP and XSH need a compile-time plan");
  if constexpr (NT > 0) {
    fft_fixed<NT, S, PPT, SRC_SH, DST_SH, JF, PZ, PP, XSH>(nl, tw, sh, src, dst, sh2, lsx);
  } else {
    fft_global<S, PPT, SRC_SH, DST_SH>(N, nl, tw, sh, src, dst);
  }
}

}  // namespace hst
