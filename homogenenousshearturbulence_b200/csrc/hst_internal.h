// Internal interface between the C ABI (hst_capi.cu) and the kernels
// (hst_kernels.cu).  Not installed; the public interface is include/hst_gpu.h.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <unordered_map>
#include <unordered_set>

#include "../../include/hst_gpu.h"

namespace hst {

// Sizes and device pointers of one field: everything a launch needs.
struct Geometry {
  int nx, ny, nz;      // deck sizes
  int nxd, nzd;        // padded transform sizes (2 nxd physical x points, nzd z points)
  int nxB, nzT, rows;  // nx+1, 2nz+1, ny+4
  int ncol;            // nxB * nzT Fourier columns
  long nf;             // complex elements of one field (ncol * rows)
  int P, m, MS;        // line-solve group: P lanes, m rows per lane, slab stride
  int Ty;              // y tile of the transforms (divides ny)
  int pptx, pptz;      // FFT points per thread of the x and z transforms (8: the low-register plans)
  int mp;              // mixed precision: Z, Pp, Q and their transforms in FP32 (complex64)
  // 0, or (in the view of the four ghost rows that the edge transforms take)
  // ny: the z-inverse then reads rows -2, -1, ny, ny+1 of V
  int edge_gap;
  // members of an ensemble advanced together (1 for a single field): every
  // per-field buffer holds nmem members one after another (fields nf
  // elements a member, Z 3 ny nzd nxB, Pp 6 ny nzd nxB, Q 6 ncol ny), the
  // tables are shared, and the substep's kernels cover all members in one
  // launch each
  int nmem;
};

struct DeviceState {
  double2* F[7];        // V1 V2 V3 OLD1 OLD2 RHS1 RHS2, (iy fastest, ghost rows included)
  double2* Z;           // z-inverse of V: [3][nzd][ny/Ty][nxB][Ty]
  double2* Pp;          // x-forward of the products: [6][nzd][ny/Ty][nxB][Ty]
  double2* Q;           // spectral products: [6][ncol][ny]
  double* der;          // der(0:ny-1, 0:3, -2:2)
  double* derS;         // the same, slab-major for the line-solve groups (SlabDer)
  double* derU;         // der's distinct rows, coefficient-major (DerRows); nderU of them, 0: not used
  int* derI;            // the distinct row of each row
  int nderU;
  double* d0tab;        // the D0 matrix factored for the line-solve group (d0_factor)
  double* y;            // y(-2:ny+1)
  double* dyl;          // dyl(0:ny-1)
  double* gdamp;        // gdamp(-nz:nz, 0:nx)
  double2* twx;         // exp(-2 pi i e / (2 nxd)), then the staged table of the x kernel's 8-point plan
  double2* twz;         // exp(-2 pi i e / nzd)
  float2* twxf;         // the same tables in FP32 (mixed precision)
  float2* twzf;
  unsigned long long* cfl;  // running max (bits of a non-negative double)
  int* err;                 // set by a kernel whose bounded wait ran out
  // TMA maps of Z and Pp as 4-D f64 tensors {2 Ty, nxB, nzd ny/Ty, comps}
  // (set by make_transform_maps when the x kernel's 8-point plan uses them)
  CUtensorMap tmZ, tmPp;
  bool maps;
  // The products of the four ghost rows (-2, -1, ny, ny+1) transformed like
  // the interior ones (null when their shear-periodic images are exact):
  // Zg [3][nzd][nxB][4], Ppg [6][nzd][nxB][4], Qg [6][ncol][4], in the
  // transforms' precision, with their TMA maps
  double2 *Zg, *Ppg, *Qg;
  CUtensorMap tmZg, tmPpg;
  int nsm;        // SMs of the device
  double* stats;  // outstats scratch: block partials of the moments (stats_partials() a block),
                  // of the three gradients (one a block each), then the 24 results
  // the reference-layout buffers of the per-piece path (allocated by its
  // first call): VVdz [3][ny+4][nx+1][nzd], VVdx and VVdp [3][ny+4][nzd][nxd+1]
  double2 *vvdz, *vvdx, *vvdp;
  // kernels whose shared-memory limit has been raised in this context
  // (owned by the context; null: raise it at every launch)
  std::unordered_set<const void*>* configured;
  // resident blocks an SM of (kernel, threads, shared bytes) launches, asked
  // once (owned by the context; null: asked at every launch)
  std::unordered_map<uint64_t, int>* occupancy;
  // the column kernels' factor scratch in global memory (one slice per
  // resident solver group; null: the scratch stays in shared memory)
  double* facg;
  size_t facg_doubles;
};

// Resident blocks an SM of kernel k with T threads and `smem` dynamic
// shared bytes (cudaOccupancyMaxActiveBlocksPerMultiprocessor, cached).
template <typename K>
inline int blocks_per_sm(const DeviceState& d, K k, int T, size_t smem) {
  const uint64_t key = (uint64_t)(uintptr_t)reinterpret_cast<const void*>(k) * 1000003ull ^ ((uint64_t)T << 40) ^ smem;
  if (d.occupancy) {
    auto it = d.occupancy->find(key);
    if (it != d.occupancy->end()) return it->second;
  }
  int n = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, T, smem) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = 1;
  }
  if (d.occupancy) (*d.occupancy)[key] = n;
  return n;
}

// Raises kernel k's dynamic shared-memory limit to `bytes`, once per context
// (the attribute belongs to the function in the current context; setting it
// at every launch costs a driver call each time).
template <typename K>
inline cudaError_t smem_limit(const DeviceState& d, K k, int bytes) {
  const void* key = reinterpret_cast<const void*>(k);
  if (d.configured && d.configured->count(key)) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && d.configured) d.configured->insert(key);
  return e;
}

// Scalars of one substep of the column kernel.
struct SubstepScalars {
  double ode0, ode1, ode2, deltat, lambda;
  double s2now, gsoft;
  double dgx, dgz;
  double sx_t, sz_t;  // wrap displacements at t
  double sx_n, sz_n;  // at t + dt_sub
  int damp_hard;
  int yuni;      // the y grid is uniform (ystretch 0): y(r + 32) - y(r) = ytile
  double ytile;  // 32 ly / ny
};

struct PhysScalars {
  double alfa0, beta0, ni, S;
  double dx, dz, factor;
};

cudaError_t launch_zinv(const Geometry& g, const DeviceState& d, cudaStream_t st);
cudaError_t launch_xprod(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int want_cfl, cudaStream_t st);
cudaError_t launch_zfwd(const Geometry& g, const DeviceState& d, cudaStream_t st);
// part: 0 the fused column kernel, 1 its right-hand-side stage alone (row
// streaming, into RHS1/RHS2), 2 the rest (shift, solves, u, w) from RHS1/RHS2,
// 3 (exact only, nonlin 0) the exact_shift shift of RHS1/2, OLD1/2 alone,
// 4 the right-hand-side stage in its untiled FP64 form
cudaError_t launch_column(const Geometry& g, const DeviceState& d, const PhysScalars& ph, const SubstepScalars& sc,
                          int exact, int nonlin, int part, cudaStream_t st);
cudaError_t launch_line_solve(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int sys, double lambda,
                              int src, int dst, double sx, double sz, cudaStream_t st);
cudaError_t launch_fill_ghosts(const Geometry& g, const DeviceState& d, const PhysScalars& ph, int field, double sx,
                               double sz, cudaStream_t st);
size_t column_smem_bytes(const Geometry& g, int exact);
// the two line buffers of a solver group, and its factor scratch (doubles)
size_t column_lines_bytes(const Geometry& g);
size_t column_fac_doubles(const Geometry& g);
// the factored D0 matrix of the line-solve group (P, m of g) into d.d0tab,
// from d.derS; d0_table_doubles: the table's size for any group of ny rows
cudaError_t launch_d0_table(const Geometry& g, const DeviceState& d, cudaStream_t st);
size_t d0_table_doubles(int ny);
// outstats (src/hst_stats.f90:136-285): block count of the reductions and
// the three kernels (hst_stats.cu)
int stats_blocks(const Geometry& g, int nsm);
cudaError_t launch_stats_moments(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double gsoft,
                                 double* partial, cudaStream_t st);
// the column energies exz(-nz:nz, 0:nx) of outstats into exz (ncol doubles)
cudaError_t launch_stats_columns(const Geometry& g, const DeviceState& d, double* exz, cudaStream_t st);
// moment partials a reduction block writes
int stats_partials();
cudaError_t launch_stats_grad(const Geometry& g, const DeviceState& d, int field, double* partial, cudaStream_t st);
cudaError_t launch_stats_final(const Geometry& g, const DeviceState& d, const double* pm, const double* pg,
                               double ly_w, double ni, double ly, double* out, cudaStream_t st);
// compute_pressure (src/hst_pressure.f90:35-110): the right-hand side into
// RHS1 (after the transforms), and the (0,0) mode into dst (after the
// POISSON solve)
cudaError_t launch_pressure_rhs(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double s2now,
                                double sx, double sz, cudaStream_t st);
cudaError_t launch_pressure_mean(const Geometry& g, const DeviceState& d, double ly, int dst, cudaStream_t st);
// the per-piece path (hst_pieces.cu; the line transforms in hst_transforms.cu):
// kind 0 z line, 1 c2r x line, 2 r2c x line; S the sign of the exponent
cudaError_t launch_piece_lines(const DeviceState& d, double2* base, size_t stride, int nlines, int N, int kind, int S,
                               const double2* tw, cudaStream_t st);
cudaError_t launch_assemble_vvdz(const Geometry& g, const DeviceState& d, cudaStream_t st);
cudaError_t launch_transpose(const Geometry& g, const DeviceState& d, int to_x, int m, cudaStream_t st);
cudaError_t launch_build_products(const Geometry& g, const DeviceState& d, const PhysScalars& ps, int grp,
                                  cudaStream_t st);
cudaError_t launch_vvdz_to_field(const Geometry& g, const DeviceState& d, int m, int field, cudaStream_t st);
cudaError_t launch_buildrhs_group(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double ode2,
                                  int grp, cudaStream_t st);
cudaError_t launch_damping_mask(const Geometry& g, const DeviceState& d, cudaStream_t st);
cudaError_t launch_shift_default(const Geometry& g, const DeviceState& d, const PhysScalars& ps, double dgx,
                                 double dgz, cudaStream_t st);
// the ghost rows' products must be transformed themselves (not taken as the
// shear-periodic images of the interior rows): with a spanwise shift (S2) and
// nzd = 3 nz, the retained modes iz = +-nz alias product modes -+2nz, whose
// wrap phases differ
bool edge_rows_needed(const Geometry& g, bool s2_active);
// the TMA maps of Z and Pp for the x kernel (d.maps false when not used)
cudaError_t make_transform_maps(const Geometry& g, DeviceState& d);
// the stage-ordered twiddles of the 8-point plan of N into out (at most N
// entries); returns their number, 0 for a length without such a plan
int staged_twiddles(int N, double2* out);
int staged_twiddles(int N, float2* out);
// a transform length of the mixed-precision form
bool mp_length_ok(int n);
// the constant twiddles of the register DFTs, once per device
cudaError_t set_fft_constants();
// a transform length the FFT kernels support
bool fft_length_ok(int n);

}  // namespace hst
