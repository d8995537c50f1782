// Shared-memory Stockham FFT for the 3/2-dealiased x and z transforms.
//
// Several lines of length N (N = 2^a 3^b) sit in shared memory; all threads
// of the block cooperate on every radix stage: a thread loads the R inputs
// of its butterflies into registers, the block synchronises, and the
// outputs overwrite the same buffer (in place, so one copy of the lines is
// enough).  Twiddles come from a table W[e] = exp(-2 pi i e / N) computed on
// the host in extended precision.  Unnormalised in both directions, like
// the reference's FFTW / cuFFT plans (src/hst_fft.f90:98-121): sign -1 is
// the forward transform exp(-2 pi i j k / N), sign +1 the backward one.
#pragma once
#include "hst_dev.cuh"

namespace hst {

#define HST_SQRT3_2 0.86602540378443864676

template <int R>
__device__ __forceinline__ void butterfly(cxd* v, int sign) {
  if (R == 2) {
    cxd a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    cxd a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]), a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
    cxd a3r = sign < 0 ? mkc(a3.y, -a3.x) : mkc(-a3.y, a3.x);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3r);
    v[3] = csub(a1, a3r);
  } else if (R == 3) {
    cxd t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    cxd m = mkc(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    // (-i sign') sqrt(3)/2 t2, forward: -i
    cxd r = sign < 0 ? mkc(HST_SQRT3_2 * t2.y, -HST_SQRT3_2 * t2.x) : mkc(-HST_SQRT3_2 * t2.y, HST_SQRT3_2 * t2.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
}

// One radix-R Stockham stage on nl lines (line stride LS) of length N, where
// Ns is the product of the radices already applied.  MAXB bounds the
// butterflies per thread: nl*N/R <= MAXB*blockDim.x.
template <int R, int MAXB>
__device__ __forceinline__ void fft_stage(cxd* data, int N, int nl, int LS, int Ns, const cxd* __restrict__ tw,
                                          int sign) {
  const int nb = N / R;
  const int total = nb * nl;
  const int tstride = N / (Ns * R);
  cxd v[MAXB][R];
  int dst[MAXB];
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    int b = threadIdx.x + k * blockDim.x;
    dst[k] = -1;
    if (b < total) {
      int line = b / nb, j = b - line * nb;
      const cxd* L = data + line * LS;
      int kk = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        cxd x = L[j + r * nb];
        if (r > 0) {
          cxd w = __ldg(tw + kk * r * tstride);
          if (sign > 0) w.y = -w.y;
          x = cmul(x, w);
        }
        v[k][r] = x;
      }
      butterfly<R>(v[k], sign);
      dst[k] = line * LS + (j / Ns) * Ns * R + kk;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    if (dst[k] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) data[dst[k] + r * Ns] = v[k][r];
    }
  }
  __syncthreads();
}

// The radix plan of N = 4^a 2^b 3^c (b, c <= 1): radix-4 stages, then one
// radix-2, then one radix-3.  PPT bounds the points per thread.
template <int PPT>
__device__ void fft_lines(cxd* data, int N, int nl, int LS, const cxd* __restrict__ tw, int sign) {
  int n = N, Ns = 1;
  while (n % 4 == 0) {
    fft_stage<4, (PPT + 3) / 4>(data, N, nl, LS, Ns, tw, sign);
    n /= 4;
    Ns *= 4;
  }
  if (n % 2 == 0) {
    fft_stage<2, (PPT + 1) / 2>(data, N, nl, LS, Ns, tw, sign);
    n /= 2;
    Ns *= 2;
  }
  if (n % 3 == 0) {
    fft_stage<3, (PPT + 2) / 3>(data, N, nl, LS, Ns, tw, sign);
    n /= 3;
    Ns *= 3;
  }
}

}  // namespace hst
