/*
 * hst oracle: a CPU FP64 restatement of the hst RK3 (Rai-Moin) / Crank-Nicolson
 * substep and the set-up it needs.  TEST INFRASTRUCTURE ONLY: the parity tests,
 * the smoke check and the CPU-baseline leg of bench.py call it as the checker.
 * Nothing in the product links or runs it.
 *
 * Every function follows the reference's CPU path (gfortran + FFTW build of
 * davecats/homogenenousShearTurbulence), in the same operation order where
 * round-off matters; each definition in hst_oracle.cpp cites the file:line it
 * restates.  The FFT is the oracle's own unnormalised mixed-radix DFT with
 * FFTW's semantics (c2r reads only the real part of the k = 0 mode).
 *
 * Parity pin: tests/test_oracle_golden.py reproduces the reference's stored
 * regression fields tests/reference/small.fld, small_s2x.fld and
 * small_stokes.fld (50 steps each) at the reference's own 1e-10 tolerance.
 *
 * Field layout: the reference's V(iy, iz, ix) of one component, iy = -2..ny+1
 * fastest, then iz = -nz..nz, then ix = 0..nx; complex128 as (re, im) pairs.
 */
#ifndef HST_ORACLE_H
#define HST_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* The namelist deck (src/hst_input.f90:19-42 groups &mesh &physics
 * &time_control &init &damping).  Logicals are ints (0/1). */
typedef struct ora_params {
  int nx, ny, nz;
  double alfa0, beta0, ly, ystretch;
  double re, S;
  int linear, exact_shift;
  double s2_mean, s2_amplitude, s2_period, s2_start;
  double sl_amplitude, sl_period, sl_delta, sl_start;
  int sl_bodyforce, sl_ramp;
  double deltat, cflmax, t_max;
  long nstep;
  double time;
  int time_from_restart, restart_from_file;
  char restart_file[256];
  char initial_condition[32];
  double amplitude, kpeak;
  int seed;
  double tg_amplitude;
  int tg_mode;
  double damp_kpar, damp_kperp, damp_rate, damp_edge, damp_norm, damp_angle;
  int damp_hard, damp_mean, damp_follow;
} ora_params;

typedef struct ora_sim ora_sim;

/* field ids */
enum { ORA_V1 = 0, ORA_V2 = 1, ORA_V3 = 2, ORA_OLD1 = 3, ORA_OLD2 = 4, ORA_RHS1 = 5, ORA_RHS2 = 6 };
/* line-solve kinds (src/hst_linsolve.f90:83) */
enum { ORA_D2V = 1, ORA_ETA = 2, ORA_POISSON = 3, ORA_D0 = 4, ORA_DY = 5 };

void ora_default_params(ora_params* p);
int ora_read_deck(const char* path, ora_params* p); /* 0 ok, else error */

ora_sim* ora_create(const ora_params* p);
void ora_destroy(ora_sim* s);
void ora_set_threads(int n);

/* sizes */
int ora_nxd(const ora_sim* s);
int ora_nzd(const ora_sim* s);
long ora_field_size(const ora_sim* s); /* complex elements per field */

double* ora_field(ora_sim* s, int id); /* interleaved complex */
const double* ora_der(const ora_sim* s); /* der(0:ny-1, 0:3, -2:2), Fortran order */
const double* ora_y(const ora_sim* s);   /* y(-2:ny+1) */
const double* ora_dyl(const ora_sim* s); /* dyl(0:ny-1) */
double* ora_gdamp(ora_sim* s);           /* gdamp(-nz:nz, 0:nx) */
double* ora_products(ora_sim* s);        /* real view of VVdp: (2(nxd+1), nzd, ny+4, 3) */
double* ora_rvvdx(ora_sim* s);           /* real view of VVdx */
double* ora_vvdz(ora_sim* s);            /* complex VVdz(nzd, nx+1, ny+4, 3) */

double ora_get_time(const ora_sim* s);
void ora_set_time(ora_sim* s, double t);
double ora_get_deltat(const ora_sim* s);
void ora_set_deltat(ora_sim* s, double dt);
double ora_get_cfl(const ora_sim* s);
void ora_set_physics(ora_sim* s, double S, double ni, int linear);

void ora_generate_initial_field(ora_sim* s);
void ora_fill_ghosts(ora_sim* s, int id, double shift_x, double shift_z);
void ora_fill_ghosts_now(ora_sim* s, int id);
void ora_shear_shifts(const ora_sim* s, double t, double* sx, double* sz);
double ora_s2_of(const ora_sim* s, double t);
double ora_s2_integral(const ora_sim* s, double t1, double t2);

/* pieces of the substep (src/hst_equations.f90:45, src/hst_transforms.f90:27) */
void ora_transform_to_physical(ora_sim* s);
double ora_compute_cfl(ora_sim* s);
void ora_build_products(ora_sim* s, int g);
void ora_products_to_spectral(ora_sim* s);
void ora_vvdz_to_field(ora_sim* s, int m, double* out);
void ora_buildrhs_prepare(ora_sim* s, const double* ODE);
void ora_buildrhs(ora_sim* s, const double* ODE, int g);
void ora_shear_shift(ora_sim* s, double dt_sub);
void ora_linsolve(ora_sim* s, double lambda);
void ora_damping_update(ora_sim* s, double t);
void ora_damping_mask(ora_sim* s);
int ora_damping_active(const ora_sim* s);
void ora_line_solve(ora_sim* s, int sys, double lambda, int src, int dst, int has_shift, double sx, double sz);
void ora_timestep(ora_sim* s);
/* substep i = 0, 1, 2 of timestep */
void ora_substep(ora_sim* s, int i);
/* the time loop of src/hst.f90:49-133 without output: set-up (initial field
 * or restart), CFL, new_timestep, then up to max_steps steps */
void ora_start(ora_sim* s);
long ora_run(ora_sim* s, long max_steps);

/* statistics of src/hst_stats.f90:136-285: out = energy, diss, uv, vw, uu, vv, ww, uw
 * (box means, Runtimedata columns 10-13 and variances_runtime.dat) */
void ora_outstats(ora_sim* s, double* out);
/* outstats' 16 reduction sums before the mean correction and the column
 * energies exz(-nz:nz, 0:nx) (may be NULL) */
void ora_outstats_sums(ora_sim* s, double* sums, double* exz);
/* compute_pressure (src/hst_pressure.f90:35-110) into field dst; rhs1 is scratch */
void ora_compute_pressure(ora_sim* s, int dst);

/* CPL field files (src/hst_io.f90:240-315, 69-178) */
int ora_restart_write(ora_sim* s, const char* path);
int ora_restart_read(ora_sim* s, const char* path);

/* the keyed random number of src/hst_initial.f90:139-159 */
double ora_uniform_from_key(int seed, int component, int iy, int iz, int ix);

#ifdef __cplusplus
}
#endif
#endif
