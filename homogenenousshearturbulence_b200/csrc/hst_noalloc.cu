// hst_gpu_line_solve_noalloc: line_solve (src/hst_linsolve.f90:147-233) on
// fields the caller holds in its own device memory, without a context and
// without allocating anything.
//
// Who needs it: a caller that already keeps V, der and its work arrays on the
// device itself -- the reference's Fortran driver, whose OpenMP target data
// region maps those arrays (src/hst.f90:76) -- and that cannot let a library
// allocate next to them.  Creating an hst_ctx reserves the whole substep
// state (seven fields plus the transform buffers, gigabytes at production
// sizes) with cudaMalloc, which such a caller has no room for, and
// cudaMalloc/cudaFree also synchronise the device in the middle of the
// caller's queued work.  This entry point runs the same solve kernel as
// hst_gpu_line_solve and keeps its one piece of working memory, the
// slab-major copy of der that the solver groups read, in a fixed array in
// the module's static device memory.
//
// Limits and rules of use:
//   - ny <= HST_NOALLOC_MAX_NY (2048): the scratch holds 20 * 2048 doubles
//     (320 KiB per device); larger ny is rejected with HST_EARG.
//   - The scratch is one array per device.  Calls on the same device must
//     not overlap (on different streams or host threads): a later call's
//     table write races with an earlier call's solve.  Queue them on one
//     stream, or order them with events.
//   - Nothing in the scratch has to start at zero: every call first rewrites
//     each entry its solve reads.
//   - Every call looks up the scratch's device address with
//     cudaGetSymbolAddress on the current device (a table lookup, not an
//     allocation), so that the address is always the one of the context
//     current now: after cudaDeviceReset, or under another context made
//     current on the same device, the library's device code is loaded again
//     and the array may move.  The first call in a context may be the one
//     that loads that code: make it before any stream capture begins.
//   - Neither src nor der may overlap dst: the solve reads both while it
//     writes dst (HST_EARG otherwise).
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdlib>
#include <cstdio>

#include "hst_dev.cuh"
#include "hst_internal.h"

#define HST_NOALLOC_MAX_NY 2048

namespace {

// der(0:ny-1, 0:3, -2:2) reordered slab-major (the order of hst::SlabDer)
__device__ __align__(256) double g_line_der[20 * HST_NOALLOC_MAX_NY];

// out[((n*5 + j)*m + i)*P + s] = der(s*m + i, n, j - 2)
__global__ void k_slab_major(const double* __restrict__ der, double* __restrict__ out, int ny, int P, int m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 20 * ny) return;
  const int s = e % P;
  const int i = (e / P) % m;
  const int nj = e / (P * m);  // n * 5 + j
  const int n = nj / 5, j = nj - 5 * n;
  out[e] = der[(size_t)(s * m + i) + (size_t)ny * (n + 4 * j)];
}

int fail(char* msg, int len, int rc, const char* fmt, ...) {
  if (msg && len > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, (size_t)len, fmt, ap);
    va_end(ap);
  }
  return rc;
}

// lanes of a solver group: the rule of the context's default geometry (the
// widest power of two up to 32 that leaves at least 8 rows per lane, else 4;
// HST_LINE_LANES overrides), so the results are identical to those of a
// context that has not been autotuned; hst_gpu_autotune may give a context
// another group width, and the two then agree up to rounding
int line_lanes(int ny) {
  const char* env = std::getenv("HST_LINE_LANES");
  if (env) {
    int e = std::atoi(env);
    if (e >= 2 && e <= 32 && (e & (e - 1)) == 0 && ny % e == 0 && ny / e >= 4) return e;
  }
  for (int mmin : {8, 4})
    for (int c = 32; c >= 2; c >>= 1)
      if (ny % c == 0 && ny / c >= mmin) return c;
  return 0;
}

}  // namespace

extern "C" int hst_gpu_line_solve_noalloc(int nx, int ny, int nz, double alfa0, double beta0, double re, int sys,
                                          double lambda, const double* der, const double* src, double* dst,
                                          double shift_x, double shift_z, void* stream, char* msg, int msg_len) {
  if (msg && msg_len > 0) msg[0] = '\0';
  if (nx < 1 || nz < 1 || ny < 8 || ny % 2 != 0)
    return fail(msg, msg_len, HST_EARG, "need nx >= 1, nz >= 1 and ny >= 8 even (got %d, %d, %d)", nx, ny, nz);
  if (ny > HST_NOALLOC_MAX_NY)
    return fail(msg, msg_len, HST_EARG, "ny = %d exceeds the static scratch of this entry point (ny <= %d)", ny,
                HST_NOALLOC_MAX_NY);
  if (sys < hst::K_D2V || sys > hst::K_DY) return fail(msg, msg_len, HST_EARG, "unknown system kind %d", sys);
  if (!der || !src || !dst) return fail(msg, msg_len, HST_EARG, "null device pointer");
  if (((uintptr_t)src & 15) || ((uintptr_t)dst & 15) || ((uintptr_t)der & 7))
    return fail(msg, msg_len, HST_EARG, "src/dst must be 16-byte aligned, der 8-byte aligned");
  {
    // the solve reads src and der while it writes dst: neither may overlap it
    const size_t bytes = (size_t)(nx + 1) * (2 * nz + 1) * (ny + 4) * 16;
    const size_t dbytes = (size_t)20 * ny * sizeof(double);
    const uintptr_t a = (uintptr_t)src, b = (uintptr_t)dst, c = (uintptr_t)der;
    if (a < b + bytes && b < a + bytes) return fail(msg, msg_len, HST_EARG, "src and dst overlap");
    if (c < b + bytes && b < c + dbytes) return fail(msg, msg_len, HST_EARG, "der and dst overlap");
  }
  const int P = line_lanes(ny);
  if (!P) return fail(msg, msg_len, HST_EARG, "ny = %d: no solver group with at least 4 rows per lane", ny);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(msg, msg_len, HST_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  // the scratch's address in the context current now (see the header)
  double* scratch = nullptr;
  e = cudaGetSymbolAddress((void**)&scratch, g_line_der);
  if (e != cudaSuccess) return fail(msg, msg_len, HST_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));

  hst::Geometry g = {};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nxB = nx + 1;
  g.nzT = 2 * nz + 1;
  g.rows = ny + 4;
  g.ncol = g.nxB * g.nzT;
  g.nf = (long)g.ncol * g.rows;
  g.P = P;
  g.m = ny / P;
  g.MS = g.m | 1;
  hst::PhysScalars ps = {};
  ps.alfa0 = alfa0;
  ps.beta0 = beta0;
  ps.ni = 1.0 / re;
  hst::DeviceState d = {};
  d.F[0] = reinterpret_cast<double2*>(const_cast<double*>(src));
  d.F[1] = reinterpret_cast<double2*>(dst);
  d.der = const_cast<double*>(der);
  d.derS = scratch;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const int n = 20 * ny, T = 256;
  k_slab_major<<<(n + T - 1) / T, T, 0, st>>>(der, scratch, ny, P, g.m);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = hst::launch_line_solve(g, d, ps, sys, lambda, 0, 1, shift_x, shift_z, st);
  if (e != cudaSuccess) return fail(msg, msg_len, HST_ECUDA, "launch: %s", cudaGetErrorString(e));
  return HST_OK;
}
