/*
 * hst_gpu.h -- the C ABI of the B200 (sm_100a) implementation of the hst
 * RK3 (Rai-Moin) / Crank-Nicolson substep.
 *
 * It replaces, one GPU per process and the whole field resident on it, the
 * bodies of these Fortran module procedures of
 * davecats/homogenenousShearTurbulence (paths relative to that project):
 *   hst_equations   timestep, buildrhs_prepare, buildrhs, shear_shift, linsolve
 *                   (src/hst_equations.f90:45)
 *   hst_linsolve    line_solve, KIND_* (src/hst_linsolve.f90:79-83, 147-153)
 *   hst_transforms  transform_to_physical, build_products, products_to_spectral,
 *                   compute_cfl (src/hst_transforms.f90:27)
 *   hst_derivatives fill_ghosts, fill_ghosts_field, shear_shifts, s2_of,
 *                   s2_integral (src/hst_derivatives.f90:25-26)
 *   hst_fft         device_sync (src/hst_fft.f90:162)
 * The Fortran side (the hst.in deck, the Dati.cart files, the time loop)
 * stays as it is and calls these functions through an ISO_C_BINDING
 * interface block.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative HST_E* class;
 *     hst_gpu_last_error() holds the message.  The Fortran shim turns a
 *     non-zero status into `error stop`, as the reference's check()
 *     (src/hst_fft.f90:169-176) does.
 *   - Fields are complex128 (interleaved re, im) in the reference layout of
 *     one component of V: V(iy, iz, ix) with iy = -2..ny+1 fastest, then
 *     iz = -nz..nz, then ix = 0..nx (src/hst_params.f90:10-14, 101).
 *   - The context owns all device memory and one CUDA stream; host pointers
 *     are borrowed for the duration of a call.  Work is queued
 *     asynchronously; the host waits only in downloads, in the CFL read of
 *     hst_gpu_timestep and in hst_gpu_sync.  One host thread per context.
 */
#ifndef HST_GPU_H
#define HST_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HST_GPU_ABI_VERSION 3

/* status classes */
#define HST_OK 0
#define HST_EARG (-1)    /* bad argument or unsupported size */
#define HST_ENOMEM (-2)  /* device allocation refused */
#define HST_ECUDA (-3)   /* CUDA runtime error */
#define HST_ETIMEOUT (-4) /* a kernel's bounded wait ran out (the step's results are invalid) */
#define HST_EFINITE (-5) /* non-finite CFL (the field blew up) */

/* field ids: the three components of V, the carried explicit terms and the
 * right-hand sides (src/hst_params.f90:101-103) */
#define HST_V1 0
#define HST_V2 1
#define HST_V3 2
#define HST_OLD1 3
#define HST_OLD2 4
#define HST_RHS1 5
#define HST_RHS2 6

/* precision of the context (hst_gpu_params.precision) */
#define HST_PREC_FP64 0  /* everything in FP64: the drop-in */
#define HST_PREC_MIXED 1 /* the x-z transforms, the products and their spectra in FP32; the right-hand
                            sides, the shear shift, the line solves and u, w in FP64.  Needs 2 nxd and
                            nzd in {96, 192, 384, 768} and ny a multiple of 32.  No counterpart in the
                            reference, which is FP64 throughout. */

/* line-solve kinds, KIND_D2V .. KIND_DY (src/hst_linsolve.f90:83) */
#define HST_KIND_D2V 1
#define HST_KIND_ETA 2
#define HST_KIND_POISSON 3
#define HST_KIND_D0 4
#define HST_KIND_DY 5

/* What the context needs from the deck (the namelists of
 * src/hst_input.f90:19-23 and the derived quantities :92-102).  nxd, nzd <= 0: derived as the reference
 * does (fft_fit).  ystretch: the y grid of src/hst_setup.f90:80-89. */
typedef struct hst_gpu_params {
  int nx, ny, nz;
  int nxd, nzd;
  double alfa0, beta0, ly, ystretch;
  double re, S;
  int linear, exact_shift;
  double s2_mean, s2_amplitude, s2_period, s2_start;
  double damp_kpar, damp_kperp, damp_rate, damp_edge, damp_norm, damp_angle;
  int damp_hard, damp_mean, damp_follow;
  int device;    /* CUDA device ordinal */
  int precision; /* HST_PREC_FP64 or HST_PREC_MIXED */
} hst_gpu_params;

typedef struct hst_ctx hst_ctx;

/* ---------------------------------------------------------------- context */
/* Allocates the device state, builds the y grid, der, k2 and the damping
 * table on the host exactly as allocate_fields / setup_derivatives /
 * damping_setup do (src/hst_setup.f90:42-71, src/hst_derivatives.f90:30-56,
 * src/hst_damping.f90:68-78), uploads them.  The fields start at zero. */
int hst_gpu_create(const hst_gpu_params* p, hst_ctx** out);
/* An ensemble: nmem independent realisations of the same deck (same sizes,
 * physics, time step; their own initial fields) in one context, advanced
 * together -- hst_gpu_timestep / _timesteps run every member, each kernel
 * of the substep covering all members in one launch, and the CFL number is
 * the largest over the members.  The per-field device memory is nmem times
 * that of a single field; the tables are shared.  Every other entry point
 * (upload, download, fill_ghosts, line_solve, outstats, pressure, restart
 * files, the pieces, the asynchronous I/O) acts on the member chosen by
 * hst_gpu_select_member (member 0 at first).  hst_gpu_autotune refuses an
 * ensemble.  No counterpart in the reference, which runs one field a job. */
int hst_gpu_create_batch(const hst_gpu_params* p, int nmem, hst_ctx** out);
int hst_gpu_select_member(hst_ctx* ctx, int member);
int hst_gpu_members(const hst_ctx* ctx);
int hst_gpu_destroy(hst_ctx* ctx);
const char* hst_gpu_last_error(const hst_ctx* ctx);
/* Device bytes held by a context of these sizes (0 on bad sizes). */
double hst_gpu_device_bytes(const hst_gpu_params* p);

/* Replaces the derivative table der(0:ny-1, 0:3, -2:2) (Fortran order),
 * the grid y(-2:ny+1) and dyl(0:ny-1) by the caller's (a Fortran driver
 * passes its own module arrays, src/hst_params.f90:84-88).  Any pointer may
 * be NULL to keep the context's. */
int hst_gpu_set_tables(hst_ctx* ctx, const double* der, const double* y, const double* dyl);
/* Reads back the context's tables (same layouts). */
int hst_gpu_get_tables(const hst_ctx* ctx, double* der, double* y, double* dyl);

/* ----------------------------------------------------------------- fields */
/* replaces `!$omp target update to(V)` / `from(V)` (src/hst.f90:76,110,121,141) */
int hst_gpu_upload(hst_ctx* ctx, int field, const double* host);
int hst_gpu_download(hst_ctx* ctx, int field, double* host);

/* Asynchronous host I/O of the velocity components (field HST_V1..HST_V3),
 * for a driver that overlaps the two copy directions with each other and
 * with the solver.  No counterpart in the reference, whose target updates
 * (src/hst.f90:76,110,121,141) are synchronous.
 *   upload_async:   the host buffer (pinned: cudaHostAlloc / registered)
 *                   is copied on a copy-in stream into a device staging
 *                   copy of the component (which may overlap the work
 *                   queued so far), and from there into the field on the
 *                   solver's stream after all work queued so far; work
 *                   queued later sees the new field.  The buffer must not
 *                   change until hst_gpu_wait_io.  The first call per
 *                   component allocates its staging copy.
 *   download_async: the field as it is at this point of the queue (a
 *                   device snapshot, taken on the solver's stream) is copied
 *                   out on a copy-out stream; the host buffer is valid after
 *                   hst_gpu_wait_io.  The first call per component allocates
 *                   its snapshot.
 *   wait_io:        the host waits for every asynchronous copy; work queued
 *                   afterwards follows them. */
int hst_gpu_upload_async(hst_ctx* ctx, int field, const double* host);
int hst_gpu_download_async(hst_ctx* ctx, int field, double* host);
int hst_gpu_wait_io(hst_ctx* ctx);

/* ------------------------------------------------------------------- path */
/* timestep() (src/hst_equations.f90:56-87): three substeps; *time is
 * advanced as the reference advances it; *cfl receives the CFL number of
 * the third substep (compute_cfl, src/hst_transforms.f90:163-179). */
int hst_gpu_timestep(hst_ctx* ctx, double* time, double deltat, double* cfl);
/* timestep() n times in a row without reading the CFL (the host does not
 * wait); *time is advanced. */
int hst_gpu_timesteps(hst_ctx* ctx, int n, double* time, double deltat);

/* line_solve(sys, lambda, src, dst [, shift_x, shift_z])
 * (src/hst_linsolve.f90:147-233): has_shift = 0 uses the displacements of
 * `time` (shear_shifts, src/hst_derivatives.f90:123-128). */
int hst_gpu_line_solve(hst_ctx* ctx, int sys, double lambda, int src, int dst, int has_shift, double shift_x,
                       double shift_z, double time);
/* fill_ghosts_field(field, shift_x, shift_z) (src/hst_derivatives.f90:149-157) */
int hst_gpu_fill_ghosts(hst_ctx* ctx, int field, double shift_x, double shift_z);
/* fill_ghosts(c) at `time` (src/hst_derivatives.f90:134-145) */
int hst_gpu_fill_ghosts_at(hst_ctx* ctx, int field, double time);

/* transform_to_physical() + compute_cfl() (src/hst_transforms.f90:74-83,
 * 163-179): the CFL number of the current V. */
int hst_gpu_compute_cfl(hst_ctx* ctx, double* cfl);

/* outstats() (src/hst_stats.f90:136-285) of the resident field at `time`:
 * out[0..7] = energy <u_i u_i>/2, dissipation, uv, vw, uu, vv, ww, uw (box
 * averages, FP64, a fixed reduction order).  The dissipation's y part
 * comes from DY solves through HST_RHS1, which is overwritten. */
int hst_gpu_outstats(hst_ctx* ctx, double time, double* out);
/* The reductions of outstats as the reference leaves them in its `sums`
 * array (src/hst_stats.f90:242), before the box-mean correction and the
 * division by ly: sums[0..15] = eps, uv, uu, vv, ww, vw, uw, mfx, mfz, q_in,
 * q_out, e_in, e_out, ed, pd, ncol_damped (box-height integrals, rows
 * weighted by dyl; q_in and e_in are 0, as no row lies in a Stokes layer).
 * exz (may be NULL): the column energies exz(-nz:nz, 0:nx) = sum_y w |u|^2
 * of the 2-D spectrum (:225-240), (2nz+1)(nx+1) doubles, iz fastest, for the
 * caller's running average (spectrum_write, :110-134).  RHS1 is
 * overwritten. */
int hst_gpu_outstats_sums(hst_ctx* ctx, double time, double* sums, double* exz);

/* Tries the launch choices that keep every buffer's layout -- the lanes of
 * a line-solver group and the points a thread of the x and z FFT plans --
 * on this context's sizes (`steps` time steps of `deltat` each, after one
 * untimed step), keeps the fastest and restores the fields (V, OLD) and
 * the damping state.  A report of the candidates' times a step goes to
 * report[0:report_len) when report is not NULL.  It allocates a copy of
 * five fields while it runs.  No counterpart in the reference. */
int hst_gpu_autotune(hst_ctx* ctx, double deltat, int steps, char* report, int report_len);

/* compute_pressure (src/hst_pressure.f90:35-110) of the resident field at
 * `time` into field dst (HST_OLD1, HST_OLD2 or HST_RHS2; the reference's
 * write_pressure uses rhs(:,:,:,2)): the Poisson right-hand side from the
 * six products and the mean-shear term, the POISSON solve, the (0,0) mode
 * -<vv>(y) with zero mean.  RHS1 and the transform buffers are overwritten
 * (they are scratch between steps). */
int hst_gpu_pressure(hst_ctx* ctx, double time, int dst);

/* restart_write (src/hst_io.f90:240-315): the context's V in the reference's
 * CPL field file (Dati.cart) at `path`, with deltat, t_max, dt_field and
 * dt_save in its header text and the raw FP64 time, S, S2(time),
 * gamma_x = S time and gamma_y(time). */
int hst_gpu_write_restart(hst_ctx* ctx, const char* path, double time, double deltat, double t_max,
                          double dt_field, double dt_save);
/* restart_read (src/hst_io.f90:69-178) of a file of the same mesh: V, with
 * its ghost rows refilled at the file's time; *time (may be NULL) receives
 * that time. */
int hst_gpu_read_restart(hst_ctx* ctx, const char* path, double* time);

/* device_sync() (src/hst_fft.f90:162) */
int hst_gpu_sync(hst_ctx* ctx);

/* ------------------------------------------ the substep one piece at a time */
/* The module procedures a caller that runs the substep's pieces itself needs
 * (the reference's test programs do, e.g. tests/test_conservation.f90:56-82,
 * which edits the products between build_products and products_to_spectral).
 * They work on the transform buffers of hst_fft in the reference's layouts
 * (src/hst_fft.f90:39-46, 88-94), complex128, rows -2..ny+1 included:
 *   HST_BUF_VVDZ  VVdz(nzd, nx+1, -2:ny+1, 3)
 *   HST_BUF_VVDX  VVdx(nxd+1, nzd, -2:ny+1, 3), the same bytes as the reals
 *                 rVVdx(2(nxd+1), nzd, -2:ny+1, 3)
 *   HST_BUF_VVDP  VVdp(nxd+1, nzd, -2:ny+1, 3), the same bytes as the reals
 *                 products(2(nxd+1), nzd, -2:ny+1, 3)
 * The first call that needs them allocates the three buffers (at 768^2 x 512
 * about 15 GB) and zeroes them.  The fused hst_gpu_timestep does not use
 * them; its results agree with a substep run piece by piece to round-off.
 * Component arguments m are 1..3 as in the Fortran. */
#define HST_BUF_VVDZ 0
#define HST_BUF_VVDX 1
#define HST_BUF_VVDP 2
/* FFT, IFT, RFT, HFT (src/hst_fft.f90:181-237): z forward and backward on
 * VVdz(:,:,:,m) (complex, unnormalised); x complex-to-real VVdx(:,:,:,m) ->
 * rVVdx(:,:,:,m) (the imaginary parts of kx = 0 and nxd ignored, as FFTW's
 * c2r) and real-to-complex products(:,:,:,m) -> VVdp(:,:,:,m), in place */
#define HST_FFT_FFT 1
#define HST_FFT_IFT 2
#define HST_FFT_RFT 3
#define HST_FFT_HFT 4
int hst_gpu_fft(hst_ctx* ctx, int kind, int m);
/* the local layout changes of a one-rank run (src/hst_mpi.f90:751-784):
 * HST_Z_TO_X  VVdz(:,:,:,m) -> VVdx(:,:,:,m), x modes above nx zeroed
 *             (with zero_vvdx_padding, src/hst_transforms.f90:58-72)
 * HST_X_TO_Z  VVdp(:,:,:,m) -> VVdz(:,:,:,m), the x modes 0..nx */
#define HST_Z_TO_X 0
#define HST_X_TO_Z 1
int hst_gpu_transpose(hst_ctx* ctx, int dir, int m);
/* transform_to_physical() (src/hst_transforms.f90:74-83): V -> rVVdx(:,:,:,1:3),
 * every row */
int hst_gpu_transform_to_physical(hst_ctx* ctx);
/* build_products(g) (src/hst_transforms.f90:97-121), g = 1 (uu, vv, ww) or
 * 2 (uv, vw, uw), times 1/(2 nxd nzd), into products(:,:,:,1:3) */
int hst_gpu_build_products(hst_ctx* ctx, int g);
/* products_to_spectral() (src/hst_transforms.f90:125-139): products -> VVdz */
int hst_gpu_products_to_spectral(hst_ctx* ctx);
/* vvdz_to_field(field, m) (src/hst_transforms.f90:143-160) into a field */
int hst_gpu_vvdz_to_field(hst_ctx* ctx, int field, int m);
/* buildrhs_prepare(ODE) (src/hst_equations.f90:92-141) with the module
 * variables deltat and time passed: RHS1, RHS2, OLD1, OLD2 from V */
int hst_gpu_buildrhs_prepare(hst_ctx* ctx, const double* ODE, double deltat, double time);
/* buildrhs(ODE, g) (src/hst_equations.f90:151-213): the products of group g
 * that VVdz holds, added to RHS1/2 and OLD1/2 */
int hst_gpu_buildrhs(hst_ctx* ctx, const double* ODE, int g);
/* damping_update(time) and damping_mask() (src/hst_damping.f90:80-133);
 * no-ops when the deck has no (hard) damping */
int hst_gpu_damping_update(hst_ctx* ctx, double time);
int hst_gpu_damping_mask(hst_ctx* ctx);
/* shear_shift(dt_sub) at `time` (src/hst_equations.f90:226-293): RHS1/2 and
 * OLD1/2 to the frame of time + dt_sub; with exact_shift V1 (and V3) serve
 * as scratch, as V(:,:,:,1) does in the reference (V is dead there) */
int hst_gpu_shear_shift(hst_ctx* ctx, double dt_sub, double time);
/* linsolve(lambda) at `time` (the time after the shift,
 * src/hst_equations.f90:298-326): V from RHS1/2, every ghost row filled */
int hst_gpu_linsolve(hst_ctx* ctx, double lambda, double time);
/* one component of a buffer to / from the host (the reference layout) */
int hst_gpu_buffer_upload(hst_ctx* ctx, int buf, int m, const double* host);
int hst_gpu_buffer_download(hst_ctx* ctx, int buf, int m, double* host);
/* the device address and bytes of a whole buffer (3 components), for a
 * caller that works on it in place (on the context's stream) */
int hst_gpu_buffer_pointer(hst_ctx* ctx, int buf, void** dptr, size_t* bytes);

/* ------------------------------------------------ host address registry */
/* The Fortran shim passes its arrays (V(:,:,:,c), rhs(:,:,:,k), VVdz(:,:,:,m),
 * ...) by address; registering each array's base address once (from
 * allocate_fields and init_fft, src/hst_setup.f90:42-71, src/hst_fft.f90:88-94)
 * lets the calls below find the device copy, so the Fortran signatures stay
 * as they are.  Ids: the field ids above, or HST_ID_BUF(buf, m) for one
 * component of a buffer; `bytes` must be the size of that id.  No
 * counterpart in the reference, whose arrays are mapped by OpenMP. */
#define HST_ID_BUF(buf, m) (8 + 3 * (buf) + (m)-1)
int hst_gpu_register_host(hst_ctx* ctx, const void* host, size_t bytes, int id);
int hst_gpu_unregister_host(hst_ctx* ctx, const void* host);
/* the id registered at this base address, or HST_EARG */
int hst_gpu_host_id(const hst_ctx* ctx, const void* host);
/* `!$omp target update to(a)` / `from(a)` of a registered array */
int hst_gpu_upload_host(hst_ctx* ctx, const void* host);
int hst_gpu_download_host(hst_ctx* ctx, void* host);
/* line_solve, fill_ghosts_field and vvdz_to_field on registered fields,
 * as the Fortran call sites pass them (src/hst_linsolve.f90:147-153,
 * src/hst_derivatives.f90:149-157, src/hst_transforms.f90:143-160) */
int hst_gpu_line_solve_host(hst_ctx* ctx, int sys, double lambda, const void* src, void* dst, int has_shift,
                            double shift_x, double shift_z, double time);
int hst_gpu_fill_ghosts_host(hst_ctx* ctx, void* field, double shift_x, double shift_z);
int hst_gpu_vvdz_to_field_host(hst_ctx* ctx, void* field, int m);

/* ------------------------------------------------------ host-side scalars */
/* shear_shifts, s2_of, s2_integral (src/hst_derivatives.f90:85-128) for the
 * context's S and S2 law */
int hst_gpu_shear_shifts(const hst_ctx* ctx, double t, double* shift_x, double* shift_z);
double hst_gpu_s2_of(const hst_ctx* ctx, double t);
double hst_gpu_s2_integral(const hst_ctx* ctx, double t1, double t2);

/* Kernel classes of the accounting below */
#define HST_KC_ZINV 0       /* z-inverse transform of V */
#define HST_KC_XPROD 1      /* x transforms + products + CFL */
#define HST_KC_ZFWD 2       /* z-forward transform of the products */
#define HST_KC_COLUMN 3     /* the fused column kernel (right-hand sides, shift, solves, u, w) */
#define HST_KC_LINE_SOLVE 4 /* hst_gpu_line_solve */
#define HST_KC_GHOSTS 5     /* hst_gpu_fill_ghosts */
#define HST_KC_RHS 6        /* the right-hand sides streamed row by row (when the column stage is split) */
#define HST_KC_SHIFT 7      /* the exact_shift shear shift, when it runs as a kernel of its own */
#define HST_KC_N 8

/* Per-kernel device time: with profiling on, every launch is bracketed by
 * two CUDA events on the context's stream; hst_gpu_kernel_times waits for
 * the stream and returns, per class, the summed milliseconds and the number
 * of launches since the last reset (arrays of HST_KC_N; either may be NULL).
 * These have no counterpart in the reference, whose per-phase timer
 * (src/hst_timer.f90:35-53) synchronises the device instead. */
int hst_gpu_set_profiling(hst_ctx* ctx, int on);
int hst_gpu_kernel_times(hst_ctx* ctx, double* ms, long long* count);
int hst_gpu_reset_kernel_times(hst_ctx* ctx);

/* Kernel launches made since the context was created (for accounting). */
long long hst_gpu_launch_count(const hst_ctx* ctx);

/* The stream the context queues its work on (a cudaStream_t). */
void* hst_gpu_stream(const hst_ctx* ctx);

/* ----------------------------------------------- no context, no allocation */
/* line_solve(sys, lambda, src, dst, shift_x, shift_z) of hst_gpu_line_solve on
 * fields in the caller's own device memory: src and dst are device pointers
 * to one field each (the layout above, ghost rows included; src's ghosts
 * filled when sys is HST_KIND_DY), der a device pointer to der(0:ny-1, 0:3,
 * -2:2) in Fortran order; re gives ni = 1/re.  Queued on `stream` (a
 * cudaStream_t, NULL for the default stream) on the current device.  No
 * device memory is allocated: the working table lives in a static array of
 * the library, one per device, which limits ny to 2048 (larger ny returns
 * HST_EARG).  Calls on one device must not overlap in time (one stream, or
 * ordered by events).  Neither src nor der may overlap dst.  Every call looks
 * up the static array's address in the context current at that moment (a
 * lookup, not an allocation; a device reset may move the array); the first
 * call in a context may load the library's device code: make it before any
 * stream capture begins.  Results equal hst_gpu_line_solve's on a context
 * that has not been autotuned (hst_gpu_autotune may pick another solver
 * group width; the two then agree up to rounding).
 * Errors: a negative HST_E* class, with a message in msg[0:msg_len) when msg
 * is not NULL.  No counterpart in the reference, whose line_solve always
 * works on its module arrays (src/hst_linsolve.f90:147). */
int hst_gpu_line_solve_noalloc(int nx, int ny, int nz, double alfa0, double beta0, double re, int sys,
                               double lambda, const double* der, const double* src, double* dst, double shift_x,
                               double shift_z, void* stream, char* msg, int msg_len);

#ifdef __cplusplus
}
#endif
#endif
