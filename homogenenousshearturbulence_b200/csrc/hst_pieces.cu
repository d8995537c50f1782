// The substep one piece at a time, on buffers in the reference's layouts:
// the kernels behind hst_gpu_transform_to_physical, _build_products,
// _products_to_spectral, _vvdz_to_field, _buildrhs_prepare, _buildrhs,
// _damping_mask, _shear_shift and _linsolve.  A Fortran caller that runs the
// substep's pieces itself (the reference's test programs,
// tests/test_conservation.f90:56-82, or a driver that edits the products
// between the calls) gets the same buffers and the same effect of each call
// as the reference's module procedures.  The fused substep (hst_gpu_timestep)
// never uses them: there the pieces share passes over HBM.
//
// Layouts (complex128 unless said otherwise; r = iy + 2 the row with ghosts):
//   VVdz(nzd, nx+1, -2:ny+1, 3):  [m][r][ix][kz]
//   VVdx(nxd+1, nzd, -2:ny+1, 3): [m][r][kz][kx], also 2(nxd+1) reals a line (rVVdx)
//   VVdp: the layout of VVdx (the products, as reals)
#include "hst_dev.cuh"
#include "hst_internal.h"
#include "hst_rhs.cuh"

namespace hst {

namespace {

__device__ __forceinline__ size_t zidx(const Geometry& g, int m, int r, int ix, int kz) {
  return (((size_t)m * g.rows + r) * g.nxB + ix) * g.nzd + kz;
}
__device__ __forceinline__ size_t xidx(const Geometry& g, int m, int r, int kz) {  // line start, complex elements
  return (((size_t)m * g.rows + r) * g.nzd + kz) * (size_t)(g.nxd + 1);
}

// assemble_vvdz (src/hst_transforms.f90:33-54): V -> VVdz, every row
__global__ void k_assemble_vvdz(Geometry g, const double2* __restrict__ V0, const double2* __restrict__ V1,
                                const double2* __restrict__ V2, double2* __restrict__ Z) {
  const int r = blockIdx.y, m = blockIdx.z;
  const double2* V = m == 0 ? V0 : (m == 1 ? V1 : V2);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nxB * g.nzd; e += gridDim.x * blockDim.x) {
    const int ix = e / g.nzd, kz = e - ix * g.nzd;
    double2 v = make_double2(0.0, 0.0);
    int iz = 1 << 30;
    if (kz <= g.nz) iz = kz;
    else if (kz >= g.nzd - g.nz) iz = kz - g.nzd;
    if (iz != (1 << 30)) v = V[((size_t)ix * g.nzT + iz + g.nz) * g.rows + r];
    Z[zidx(g, m, r, ix, kz)] = v;
  }
}

// transpose_zTOx (src/hst_mpi.f90:751-761) and zero_vvdx_padding
// (src/hst_transforms.f90:58-72) of component m: VVdx(kx, kz) = VVdz(kz, kx)
// for kx <= nx, 0 for nx < kx <= nxd
__global__ void k_ztox(Geometry g, int m, const double2* __restrict__ Z, double2* __restrict__ X) {
  __shared__ double2 t[32][33];
  const int ix0 = blockIdx.x * 32, kz0 = blockIdx.y * 32, r = blockIdx.z;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int ix = ix0 + j, kz = kz0 + threadIdx.x;
    t[j][threadIdx.x] = (ix <= g.nx && kz < g.nzd) ? Z[zidx(g, m, r, ix, kz)] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kz = kz0 + j, ix = ix0 + threadIdx.x;
    if (kz < g.nzd && ix <= g.nxd) X[xidx(g, m, r, kz) + ix] = t[threadIdx.x][j];
  }
}

// transpose_xTOz (src/hst_mpi.f90:774-784) of component m: VVdz(kz, kx) =
// VVdp(kx, kz) for kx <= nx
__global__ void k_xtoz(Geometry g, int m, const double2* __restrict__ X, double2* __restrict__ Z) {
  __shared__ double2 t[32][33];
  const int ix0 = blockIdx.x * 32, kz0 = blockIdx.y * 32, r = blockIdx.z;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kz = kz0 + j, ix = ix0 + threadIdx.x;
    if (kz < g.nzd && ix <= g.nx) t[threadIdx.x][j] = X[xidx(g, m, r, kz) + ix];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int ix = ix0 + j, kz = kz0 + threadIdx.x;
    if (ix <= g.nx && kz < g.nzd) Z[zidx(g, m, r, ix, kz)] = t[j][threadIdx.x];
  }
}

// build_products(grp) (src/hst_transforms.f90:97-121): products(:, :, :, 1:3)
// from rVVdx(:, :, :, 1:3), every row, the 2 nxd physical points of a line
__global__ void k_build_products(Geometry g, int grp, double factor, const double2* __restrict__ X,
                                 double2* __restrict__ Pr) {
  const double* u = reinterpret_cast<const double*>(X);
  double* p = reinterpret_cast<double*>(Pr);
  const size_t line = 2 * (size_t)(g.nxd + 1), comp = line * g.nzd * g.rows;
  const int NX = 2 * g.nxd;
  const size_t n = (size_t)g.rows * g.nzd * NX;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t l = e / NX;
    const size_t o = l * line + (e - l * NX);
    const double a = u[o], b = u[o + comp], c = u[o + 2 * comp];
    if (grp == 1) {
      p[o] = a * a * factor;
      p[o + comp] = b * b * factor;
      p[o + 2 * comp] = c * c * factor;
    } else {
      p[o] = a * b * factor;
      p[o + comp] = b * c * factor;
      p[o + 2 * comp] = a * c * factor;
    }
  }
}

// vvdz_to_field (src/hst_transforms.f90:143-160): field(iy, iz, ix) =
// VVdz(izd(iz)+1, ix+1, iy, m), every row
__global__ void k_vvdz_to_field(Geometry g, int m, const double2* __restrict__ Z, double2* __restrict__ F) {
  const size_t n = (size_t)g.ncol * g.rows;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int col = (int)(e / g.rows), r = (int)(e - (size_t)col * g.rows);
    const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
    const int kz = iz >= 0 ? iz : g.nzd + iz;
    F[e] = Z[zidx(g, m, r, ix, kz)];
  }
}

// buildrhs(ODE, grp) (src/hst_equations.f90:151-213): the three products of
// group grp, which products_to_spectral has left in VVdz (every row), added
// to rhs and oldrhs; one warp per Fourier column, lanes over rows
__global__ void __launch_bounds__(256) k_buildrhs_group(Geometry g, PhysScalars ps, double ode2, int grp,
                                                        const double* __restrict__ der,
                                                        const double2* __restrict__ Z, double2* __restrict__ R1,
                                                        double2* __restrict__ R2, double2* __restrict__ O1,
                                                        double2* __restrict__ O2) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + warp;
  if (col >= g.ncol) return;
  const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
  const int kz = iz >= 0 ? iz : g.nzd + iz;
  ColConst c;
  c.al = ps.alfa0 * ix;
  c.be = ps.beta0 * iz;
  c.kk = c.al * c.al + c.be * c.be;
  c.c00 = (ix == 0 && iz == 0);
  const int ny = g.ny;
  const size_t cb = (size_t)col * g.rows + 2;
  for (int r = lane; r < ny; r += 32) {
    cxd r1 = R1[cb + r], r2 = R2[cb + r], o1 = O1[cb + r], o2 = O2[cb + r];
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      cxd q0 = mkc(0, 0), q1 = mkc(0, 0), q2 = mkc(0, 0);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const cxd v = Z[zidx(g, p, r + j, ix, kz)];  // row r + j - 2, stored at r + j
        const double e0 = derv(der, ny, r, 0, j - 2), e1 = derv(der, ny, r, 1, j - 2), e2 = derv(der, ny, r, 2, j - 2);
        q0 = mkc(q0.x + e0 * v.x, q0.y + e0 * v.y);
        q1 = mkc(q1.x + e1 * v.x, q1.y + e1 * v.y);
        q2 = mkc(q2.x + e2 * v.x, q2.y + e2 * v.y);
      }
      product_rhs(3 * (grp - 1) + p, c, ode2, q0, q1, q2, r1, r2, o1, o2);
    }
    R1[cb + r] = r1;
    R2[cb + r] = r2;
    O1[cb + r] = o1;
    O2[cb + r] = o2;
  }
}

// damping_mask (src/hst_damping.f90:119-133)
__global__ void k_damping_mask(Geometry g, const double* __restrict__ gdamp, double2* __restrict__ R1,
                               double2* __restrict__ R2, double2* __restrict__ O1, double2* __restrict__ O2) {
  const size_t n = (size_t)g.ncol * g.ny;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int col = (int)(e / g.ny), r = (int)(e - (size_t)col * g.ny);
    if (gdamp[col] > 0.0) {
      const size_t o = (size_t)col * g.rows + 2 + r;
      R1[o] = R2[o] = O1[o] = O2[o] = mkc(0, 0);
    }
  }
}

// shear_shift, default form (src/hst_equations.f90:245-257): rhs and oldrhs
// times the node phase exp(-i (alfa0 ix dgx + beta0 iz dgz) y(iy))
__global__ void k_shift_default(Geometry g, PhysScalars ps, double dgx, double dgz, const double* __restrict__ y,
                                double2* __restrict__ R1, double2* __restrict__ R2, double2* __restrict__ O1,
                                double2* __restrict__ O2) {
  const size_t n = (size_t)g.ncol * g.ny;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int col = (int)(e / g.ny), r = (int)(e - (size_t)col * g.ny);
    const int ix = col / g.nzT, iz = col - ix * g.nzT - g.nz;
    const cxd f = cexpi(-(ps.alfa0 * ix * dgx + ps.beta0 * iz * dgz) * y[r + 2]);
    const size_t o = (size_t)col * g.rows + 2 + r;
    R1[o] = cmul(R1[o], f);
    R2[o] = cmul(R2[o], f);
    O1[o] = cmul(O1[o], f);
    O2[o] = cmul(O2[o], f);
  }
}

int grid_of(size_t n, int T) {
  size_t b = (n + T - 1) / T;
  return (int)(b < 65535 * 16 ? b : 65535 * 16);
}

}  // namespace

cudaError_t launch_assemble_vvdz(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  const int T = 256;
  const dim3 grid((g.nxB * g.nzd + T - 1) / T, g.rows, 3);
  k_assemble_vvdz<<<grid, T, 0, st>>>(g, d.F[0], d.F[1], d.F[2], d.vvdz);
  return cudaGetLastError();
}

cudaError_t launch_transpose(const Geometry& g, const DeviceState& d, int to_x, int m, cudaStream_t st) {
  const dim3 block(32, 8);
  if (to_x) {
    const dim3 grid((g.nxd + 1 + 31) / 32, (g.nzd + 31) / 32, g.rows);
    k_ztox<<<grid, block, 0, st>>>(g, m, d.vvdz, d.vvdx);
  } else {
    const dim3 grid((g.nxB + 31) / 32, (g.nzd + 31) / 32, g.rows);
    k_xtoz<<<grid, block, 0, st>>>(g, m, d.vvdp, d.vvdz);
  }
  return cudaGetLastError();
}

cudaError_t launch_build_products(const Geometry& g, const DeviceState& d, const PhysScalars& ps, int grp,
                                  cudaStream_t st) {
  const int T = 256;
  k_build_products<<<grid_of((size_t)g.rows * g.nzd * 2 * g.nxd, T), T, 0, st>>>(g, grp, ps.factor, d.vvdx, d.vvdp);
  return cudaGetLastError();
}

cudaError_t launch_vvdz_to_field(const Geometry& g, const DeviceState& d, int m, int field, cudaStream_t st) {
  const int T = 256;
  k_vvdz_to_field<<<grid_of((size_t)g.ncol * g.rows, T), T, 0, st>>>(g, m, d.vvdz, d.F[field]);
  return cudaGetLastError();
}

cudaError_t launch_buildrhs_group(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double ode2,
                                  int grp, cudaStream_t st) {
  const int T = 256;
  k_buildrhs_group<<<(g.ncol + T / 32 - 1) / (T / 32), T, 0, st>>>(g, ps, ode2, grp, d.der, d.vvdz, d.F[5], d.F[6],
                                                                   d.F[3], d.F[4]);
  return cudaGetLastError();
}

cudaError_t launch_damping_mask(const Geometry& g, const DeviceState& d, cudaStream_t st) {
  const int T = 256;
  k_damping_mask<<<grid_of((size_t)g.ncol * g.ny, T), T, 0, st>>>(g, d.gdamp, d.F[5], d.F[6], d.F[3], d.F[4]);
  return cudaGetLastError();
}

cudaError_t launch_shift_default(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double dgx,
                                 double dgz, cudaStream_t st) {
  const int T = 256;
  k_shift_default<<<grid_of((size_t)g.ncol * g.ny, T), T, 0, st>>>(g, ps, dgx, dgz, d.y, d.F[5], d.F[6], d.F[3],
                                                                   d.F[4]);
  return cudaGetLastError();
}

}  // namespace hst
