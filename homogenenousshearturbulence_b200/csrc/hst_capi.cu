// The C ABI of include/hst_gpu.h: the context, its tables and the host-side
// sequencing of the substep.  Host arithmetic that feeds the device (grid,
// der, damping table, wrap displacements, S2 law, time) follows the
// reference's host code in the same operation order, so that a Fortran
// driver that passes its own tables and one that lets the context build them
// get the same numbers.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <new>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "hst_dev.cuh"
#include "hst_internal.h"

using hst::DeviceState;
using hst::Geometry;
using hst::PhysScalars;
using hst::SubstepScalars;

namespace {
const double PI = 3.141592653589793;
const double TWOPI = 6.283185307179586;

// x**n for a variable integer n, as gfortran evaluates it (binary powering)
double powi(double x, int m) {
  unsigned n = m < 0 ? -m : m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}
double fmodulo(double a, double p) {
  double r = std::fmod(a, p);
  if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r += p;
  return r;
}
int imodulo(int a, int p) {
  int r = a % p;
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  return r;
}
bool fft_fit(int n) {  // src/hst_input.f90:107-115
  if (n <= 0) return false;
  int j = n;
  while (j % 2 == 0) j /= 2;
  return j == 1 || j == 3;
}
double ymap(double xi, double ystretch) {  // src/hst_setup.f90:80-89
  if (ystretch <= 1.0e-10) return xi;
  if (xi <= 0.5) return 0.5 * std::tanh(2.0 * ystretch * xi) / std::tanh(ystretch);
  return 0.5 * (2.0 + std::tanh(2.0 * ystretch * (xi - 1.0)) / std::tanh(ystretch));
}
// dense 5x5 solve with partial pivoting (src/hst_derivatives.f90:59-79)
void solve5(const double Min[5][5], const double bin[5], double x[5]) {
  double M[5][5], b[5];
  std::memcpy(M, Min, sizeof M);
  std::memcpy(b, bin, sizeof b);
  for (int i = 0; i <= 4; ++i) {
    int p = i;
    double best = std::fabs(M[i][i]);
    for (int r = i + 1; r <= 4; ++r)
      if (std::fabs(M[r][i]) > best) {
        best = std::fabs(M[r][i]);
        p = r;
      }
    if (p != i) {
      for (int c = 0; c <= 4; ++c) std::swap(M[i][c], M[p][c]);
      std::swap(b[i], b[p]);
    }
    for (int j = i + 1; j <= 4; ++j) {
      double f = M[j][i] / M[i][i];
      for (int c = i; c <= 4; ++c) M[j][c] = M[j][c] - f * M[i][c];
      b[j] = b[j] - f * b[i];
    }
  }
  for (int i = 4; i >= 0; --i) {
    double s = 0.0;
    for (int c = i + 1; c <= 4; ++c) s = s + M[i][c] * x[c];
    x[i] = (b[i] - s) / M[i][i];
  }
}
// setup_derivatives (src/hst_derivatives.f90:30-56); y has the ghost rows
void setup_derivatives(int ny, const std::vector<double>& y, std::vector<double>& der) {
  der.assign((size_t)ny * 20, 0.0);
  for (int iy = 0; iy < ny; ++iy) {
    double dyj[5];
    for (int j = -2; j <= 2; ++j) dyj[j + 2] = y[iy + j + 2] - y[iy + 2];
    double M[5][5], t[5], d4[5], d0[5], d2[5], d1[5];
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) M[i][j] = powi(dyj[j], 4 - i);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    t[0] = 24.0;
    solve5(M, t, d4);
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) M[i][j] = (double)((5 - i) * (6 - i) * (7 - i) * (8 - i)) * powi(dyj[j], 4 - i);
    for (int i = 0; i <= 4; ++i) {
      double s = 0.0;
      for (int j = 0; j < 5; ++j) s = s + d4[j] * powi(dyj[j], 8 - i);
      t[i] = s;
    }
    solve5(M, t, d0);
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) M[i][j] = powi(dyj[j], 4 - i);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    for (int i = 0; i <= 2; ++i) {
      double s = 0.0;
      for (int j = 0; j < 5; ++j) s = s + d0[j] * (double)(4 - i) * (double)(3 - i) * powi(dyj[j], 2 - i);
      t[i] = s;
    }
    solve5(M, t, d2);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    for (int i = 0; i <= 3; ++i) {
      double s = 0.0;
      for (int j = 0; j < 5; ++j) s = s + d0[j] * (double)(4 - i) * powi(dyj[j], 3 - i);
      t[i] = s;
    }
    solve5(M, t, d1);
    const double* rows[4] = {d0, d1, d2, d4};
    for (int n = 0; n < 4; ++n)
      for (int j = 0; j < 5; ++j) der[(size_t)iy + (size_t)ny * (n + 4 * j)] = rows[n][j];
  }
}
}  // namespace

struct hst_ctx {
  hst_gpu_params p;
  Geometry g;
  DeviceState d;
  PhysScalars ps;
  double lx, lz;
  std::vector<double> y, dyl, der, gdamp;
  double theta_last;
  cudaStream_t stream;
  double* h_gdamp;                // pinned staging of gdamp uploads
  unsigned long long* h_cfl;      // pinned CFL read-back
  std::string err;
  // an ensemble of nmem members in one context (hst_gpu_create_batch): gb, db
  // the geometry and buffers of all members, which the substep runs on; g, d
  // the view of the selected member, which every other entry point uses
  int nmem = 1, member = 0;
  Geometry gb;
  DeviceState db;
  std::unordered_set<const void*> configured;  // kernels whose shared-memory limit is raised
  std::unordered_map<uint64_t, int> occupancy;  // resident blocks an SM, per launch shape
  long long launches;
  int device;
  // the column stage as two kernels (right-hand sides streamed row by row,
  // then the solves) or one; HST_COLUMN_FUSED=1 selects the single kernel
  bool column_split;
  // with exact_shift, the shift as a third kernel before the solves: on with
  // the persistent solve stage (slabs of 16 rows or more; 768^2 x 512: shift
  // 4.4 + solves 4.9 ms against 10.3 ms in one kernel), HST_SHIFT_SPLIT=0 / 1
  // forces it
  bool shift_split;
  bool solve_halves;  // the solve stage as two one-line passes
  // per-kernel-class CUDA-event accounting (hst_gpu_set_profiling)
  bool prof_on;
  std::vector<cudaEvent_t> ev;
  std::vector<int> ev_class;  // class of each recorded pair
  double prof_ms[HST_KC_N];
  long long prof_n[HST_KC_N];
  // asynchronous host I/O of V1..V3 (hst_gpu_upload_async and friends): a
  // copy-in and a copy-out stream; per component a device staging copy that
  // the copy-in stream fills while the solver still works on the previous
  // contents, and a device snapshot that the copy-out stream reads while the
  // solver goes on, each with the event that frees it again
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_main = nullptr, ev_in = nullptr, ev_stage = nullptr, ev_out = nullptr;
  double2* snap[3] = {nullptr, nullptr, nullptr};
  double2* stage[3] = {nullptr, nullptr, nullptr};
  // host address ranges registered by the caller (hst_gpu_register_host): a
  // Fortran array's base address -> field or buffer-component id
  struct HostRange {
    uintptr_t base;
    size_t bytes;
    int id;
  };
  std::vector<HostRange> host_ranges;
  cudaEvent_t ev_staged[3] = {nullptr, nullptr, nullptr};  // stage[c] copied into V (solver's stream)
  cudaEvent_t ev_read[3] = {nullptr, nullptr, nullptr};    // snap[c] copied to the host (copy-out stream)
  bool staged_used[3] = {false, false, false}, read_used[3] = {false, false, false};
};

// Runs `launch` (which queues one kernel on ctx->stream) between two events
// when profiling is on, and counts it.
template <typename F>
static cudaError_t timed(hst_ctx* c, int kc, F launch, int nlaunch = 1) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (c->prof_on) {
    size_t k = c->ev_class.size();
    while (c->ev.size() < 2 * (k + 1)) {
      cudaEvent_t e;
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
      c->ev.push_back(e);
    }
    a = c->ev[2 * k];
    b = c->ev[2 * k + 1];
    cudaEventRecord(a, c->stream);
  }
  cudaError_t r = launch();
  if (r != cudaSuccess) return r;
  c->launches += nlaunch;
  if (c->prof_on) {
    cudaEventRecord(b, c->stream);
    c->ev_class.push_back(kc);
  }
  return cudaSuccess;
}

static int fail(hst_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(b, sizeof b, fmt, ap);
    va_end(ap);
    c->err = b;
  }
  return code;
}
#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(ctx, HST_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// ------------------------------------------------------ host scalars ----
static double s2_of(const hst_gpu_params& p, double t) {  // src/hst_derivatives.f90:85-95
  if ((p.s2_amplitude == 0.0 && p.s2_mean == 0.0) || t < p.s2_start) return 0.0;
  if (p.s2_period > 0.0) return p.s2_mean + p.s2_amplitude * std::sin(TWOPI / p.s2_period * (t - p.s2_start));
  return p.s2_mean + p.s2_amplitude;
}
static double s2_integral(const hst_gpu_params& p, double t1, double t2) {  // :98-112
  if ((p.s2_amplitude == 0.0 && p.s2_mean == 0.0) || t2 <= p.s2_start) return 0.0;
  double a = std::max(t1, p.s2_start), b = t2;
  if (p.s2_period > 0.0) {
    double omega = TWOPI / p.s2_period;
    return p.s2_mean * (b - a) + p.s2_amplitude / omega * (std::cos(omega * (a - p.s2_start)) - std::cos(omega * (b - p.s2_start)));
  }
  return (p.s2_mean + p.s2_amplitude) * (b - a);
}
static void shear_shifts(const hst_ctx* c, double t, double* sx, double* sz) {  // :123-128
  *sx = fmodulo(c->p.S * t * c->p.ly, c->lx);
  *sz = fmodulo(s2_integral(c->p, c->p.s2_start, t) * c->p.ly, c->lz);
}
static bool damping_active(const hst_gpu_params& p) {  // src/hst_damping.f90:46-48
  return p.damp_kpar > 0.0 && p.damp_kperp > 0.0 && (p.damp_hard || p.damp_rate > 0.0);
}
// damping_update (src/hst_damping.f90:80-115); true when the table changed
static bool damping_update(hst_ctx* c, double t) {
  const hst_gpu_params& p = c->p;
  double theta = p.damp_follow ? std::atan2(s2_of(p, t), p.S) : p.damp_angle * PI / 180.0;
  if (theta == c->theta_last) return false;
  c->theta_last = theta;
  double cs = std::cos(theta), sn = std::sin(theta);
  for (int ix = 0; ix <= p.nx; ++ix) {
    double kx = p.alfa0 * ix;
    for (int iz = -p.nz; iz <= p.nz; ++iz) {
      double kz = p.beta0 * iz;
      double kpar = kx * cs + kz * sn, kperp = -kx * sn + kz * cs;
      double r = std::pow(std::pow(std::fabs(kpar) / p.damp_kpar, p.damp_norm) + std::pow(std::fabs(kperp) / p.damp_kperp, p.damp_norm),
                          1.0 / p.damp_norm);
      double g = 0.0;
      if (r < 1.0 - 1.0e-6) {
        if (p.damp_hard) g = 1.0;
        else if (r <= 1.0 - p.damp_edge) g = p.damp_rate;
        else {
          double x = (1.0 - r) / p.damp_edge;
          g = p.damp_rate * x * x * (3.0 - 2.0 * x);
        }
      }
      if (ix == 0 && iz == 0 && !p.damp_mean) g = 0.0;
      c->gdamp[(size_t)(iz + p.nz) + (size_t)(2 * p.nz + 1) * ix] = g;
    }
  }
  return true;
}

// ------------------------------------------------------ geometry ----
static int choose_geometry(const hst_gpu_params& p, Geometry& g, std::string& why) {
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.nxd = p.nxd;
  g.nzd = p.nzd;
  if (g.nxd <= 0) {
    g.nxd = 3 * (p.nx + 1) / 2;
    while (!fft_fit(g.nxd)) g.nxd++;
  }
  if (g.nzd <= 0) {
    g.nzd = 3 * p.nz;
    while (!fft_fit(g.nzd)) g.nzd++;
  }
  if (p.nx < 1 || p.nz < 1 || p.ny < 8) {
    why = "need nx >= 1, nz >= 1, ny >= 8";
    return HST_EARG;
  }
  if (!fft_fit(g.nxd) || !fft_fit(g.nzd) || 2 * g.nxd < 3 * (p.nx + 1) - 1 || g.nzd < 3 * p.nz) {
    why = "nxd, nzd must be 2^a 3^b (b <= 1) and satisfy the 3/2 rule";
    return HST_EARG;
  }
  if (p.ny % 2 != 0) {
    why = "ny must be even";
    return HST_EARG;
  }
  g.edge_gap = 0;
  g.nmem = 1;
  g.nxB = p.nx + 1;
  g.nzT = 2 * p.nz + 1;
  g.rows = p.ny + 4;
  g.ncol = g.nxB * g.nzT;
  g.nf = (long)g.ncol * g.rows;
  // line-solve group: P lanes of m rows; the widest group with m >= 8
  // (measured best at 384^2 x 256), else m >= 4
  int P = 0;
  const char* env = std::getenv("HST_LINE_LANES");
  if (env) {
    int e = std::atoi(env);
    if (e >= 2 && e <= 32 && (e & (e - 1)) == 0 && p.ny % e == 0 && p.ny / e >= 4) P = e;
  }
  for (int mmin : {8, 4}) {
    if (P) break;
    for (int c = 32; c >= 2; c >>= 1)
      if (p.ny % c == 0 && p.ny / c >= mmin) {
        P = c;
        break;
      }
  }
  if (!P) {
    why = "ny must be a multiple of 2 with at least 4 rows per lane";
    return HST_EARG;
  }
  g.P = P;
  g.m = p.ny / P;
  g.MS = g.m | 1;
  if (hst::column_smem_bytes(g, 1) > 200 * 1024) {
    why = "ny too large for one line-solver group's shared memory";
    return HST_EARG;
  }
  // FFT points per thread: 8 selects the low-register plans (lengths 192,
  // 384, 768; the x kernel then moves its tiles by TMA).  Measured at
  // 384^2 x 256: x 8 (1.31 against 2.41 ms), z 16 (0.26/0.50 against
  // 0.29/0.52 ms); at 768^2 x 512 the z kernels need 8 (2.4/4.9 against
  // 4.0/14.0 ms).  HST_FFT_PPT_X / HST_FFT_PPT_Z override.
  auto ppt_of = [](const char* name, int dflt) {
    const char* e = std::getenv(name);
    int v = e ? std::atoi(e) : dflt;
    return (v == 8 || v == 16) ? v : dflt;
  };
  g.pptx = ppt_of("HST_FFT_PPT_X", 8);
  g.pptz = ppt_of("HST_FFT_PPT_Z", g.nzd >= 768 ? 8 : 16);
  // mixed precision: the FP32 transforms of the lengths it compiles
  // (8 points a thread, 16 at 96) and the streamed right-hand sides
  g.mp = p.precision == HST_PREC_MIXED;
  if (p.precision != HST_PREC_FP64 && p.precision != HST_PREC_MIXED) {
    why = "precision must be HST_PREC_FP64 or HST_PREC_MIXED";
    return HST_EARG;
  }
  if (g.mp) {
    if (!hst::mp_length_ok(2 * g.nxd) || !hst::mp_length_ok(g.nzd) || p.ny % 32 != 0) {
      why = "mixed precision needs 2 nxd and nzd in {96, 192, 384, 768, 1536} and ny a multiple of 32";
      return HST_EARG;
    }
    g.pptx = 8;
    // 16 points a thread for the FP32 z transforms (zfwd 0.29 against 0.34 ms at 384)
    g.pptz = g.nzd == 768 ? 8 : ppt_of("HST_FFT_PPT_Z", 16);
  }
  // 1536 points: one plan in both precisions, 32 points a thread
  if (g.nzd == 1536) g.pptz = 32;
  // transform y tile (at most 512 threads for the 8-point z plans)
  g.Ty = 2;
  for (int t : {8, 4}) {
    // (the lines are padded, one element in eight for the 8-point plans, in
    // sixteen for the others: two blocks of up to 112 KB share an SM)
    const size_t line = g.pptz == 8 ? g.nzd + g.nzd / 8 + 8 : g.nzd + g.nzd / 16 + 8;
    if (p.ny % t == 0 && (size_t)t * line * 16 <= 112 * 1024 && (g.pptz != 8 || t * g.nzd / 8 <= 384)) {
      g.Ty = t;
      break;
    }
  }
  if (!hst::fft_length_ok(2 * g.nxd) || !hst::fft_length_ok(g.nzd) || g.Ty * g.nzd > 32 * 256 ||
      6 * 2 * g.nxd > 32 * 320) {
    why = "transform length not supported (2 nxd <= 1536, radices 2, 3, 4, 6, 8, 12, 16, 24)";
    return HST_EARG;
  }
  return HST_OK;
}

static double dev_bytes(const Geometry& g) {
  double nf = (double)g.nf;
  double z = 3.0 * g.nzd * g.ny * g.nxB, pp = 6.0 * g.nzd * g.ny * g.nxB, q = 6.0 * g.ncol * g.ny;
  return 16.0 * 7.0 * nf + (g.mp ? 8.0 : 16.0) * (z + pp + q) + 8.0 * (20.0 * g.ny + 2.0 * g.ny + 4 + g.ncol);
}

extern "C" double hst_gpu_device_bytes(const hst_gpu_params* p) {
  Geometry g;
  std::string why;
  if (!p || choose_geometry(*p, g, why) != HST_OK) return 0.0;
  return dev_bytes(g);
}

// der in the slab-major order of hst::SlabDer
static std::vector<double> slab_major(const std::vector<double>& der, int ny, int P, int m) {
  std::vector<double> o((size_t)20 * ny);
  for (int n = 0; n < 4; ++n)
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < m; ++i)
        for (int s = 0; s < P; ++s)
          o[((size_t)(n * 5 + j) * m + i) * P + s] = der[(size_t)(s * m + i) + (size_t)ny * (n + 4 * j)];
  return o;
}

// der's distinct rows (equal bits) coefficient-major, and each row's index
// among them, for hst::DerRows (nu <= ny: a stretched grid keeps them all)
static int der_rows(const std::vector<double>& der, int ny, std::vector<double>& tab, std::vector<int>& idx) {
  std::unordered_map<std::string, int> seen;
  std::vector<int> first;
  idx.assign(ny, 0);
  for (int r = 0; r < ny; ++r) {
    std::string key(20 * sizeof(double), '\0');
    for (int q = 0; q < 20; ++q) std::memcpy(&key[q * sizeof(double)], &der[(size_t)r + (size_t)ny * q], sizeof(double));
    auto it = seen.find(key);
    if (it == seen.end()) {
      it = seen.emplace(std::move(key), (int)first.size()).first;
      first.push_back(r);
    }
    idx[r] = it->second;
  }
  const int nu = (int)first.size();
  tab.assign((size_t)20 * nu, 0.0);
  for (int q = 0; q < 20; ++q)
    for (int u = 0; u < nu; ++u) tab[(size_t)q * nu + u] = der[(size_t)first[u] + (size_t)ny * q];
  return nu;
}
// uploads der's distinct-row table (stream-ordered after everything before)
static cudaError_t upload_der_rows(hst_ctx* ctx);

static std::vector<double2> twiddles(int n) {
  std::vector<double2> t(n);
  for (int k = 0; k < n; ++k) {
    long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
    t[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  return t;
}

static void free_device(hst_ctx* c) {
  if (c->nmem > 1) {
    // the per-member buffers belong to the base; the view only points into them
    DeviceState& d = c->d;
    for (int i = 0; i < 7; ++i) d.F[i] = c->db.F[i];
    d.Z = c->db.Z;
    d.Pp = c->db.Pp;
    d.Q = c->db.Q;
    d.Zg = c->db.Zg;
    d.Ppg = c->db.Ppg;
    d.Qg = c->db.Qg;
  }
  DeviceState& d = c->d;
  for (int i = 0; i < 7; ++i)
    if (d.F[i]) cudaFree(d.F[i]);
  void* ps[] = {d.Z,    d.Pp,   d.Q,    d.der,  d.derS,  d.d0tab, d.y,    d.dyl,  d.gdamp, d.twx, d.twz,
                d.twxf, d.twzf, d.cfl,  d.stats, d.vvdz, d.vvdx,  d.vvdp, d.Zg,   d.Ppg,  d.Qg,  d.derU, d.derI};
  for (void* q : ps)
    if (q) cudaFree(q);
  if (d.facg) cudaFree(d.facg);
  std::memset(&d, 0, sizeof d);
  d.configured = &c->configured;
  d.occupancy = &c->occupancy;
}

// The column kernels' factor scratch in global memory: one slice of
// (m-2) x 4 x P doubles per solver group that can be resident at once (at
// most 16 warps an SM), sized for the current group width.  It is used (and
// with it the persistent solve stage, k_column_solve) for slabs of 16 rows
// or more, where the scratch would otherwise take half a warp's shared memory
// (768^2 x 512: column 10.2 against 11.1 ms); at 8 rows a lane the one-column
// kernel with the scratch in shared memory measured faster (384^2 x 256:
// 0.54 against 0.75 ms).  HST_COLUMN_GFAC=1 / 0 forces either.
static cudaError_t ensure_facg(hst_ctx* ctx) {
  const Geometry& g = ctx->g;
  const char* e = std::getenv("HST_COLUMN_GFAC");
  const bool want = e ? std::atoi(e) == 1 : g.m >= 16;
  if (!want) {
    if (ctx->d.facg) {
      cudaError_t r = cudaStreamSynchronize(ctx->stream);
      if (r != cudaSuccess) return r;
      cudaFree(ctx->d.facg);
      ctx->d.facg = nullptr;
      ctx->d.facg_doubles = 0;
    }
    return cudaSuccess;
  }
  const int nsm = ctx->d.nsm > 0 ? ctx->d.nsm : 148;
  const size_t need = (size_t)nsm * 16 * (32 / std::min(g.P, 32)) * hst::column_fac_doubles(g);
  if (ctx->d.facg && ctx->d.facg_doubles >= need) return cudaSuccess;
  if (ctx->d.facg) {
    cudaError_t r = cudaStreamSynchronize(ctx->stream);
    if (r != cudaSuccess) return r;
    cudaFree(ctx->d.facg);
    ctx->d.facg = nullptr;
    ctx->d.facg_doubles = 0;
  }
  cudaError_t r = cudaMalloc((void**)&ctx->d.facg, need * sizeof(double));
  if (r != cudaSuccess) {
    cudaGetLastError();
    ctx->d.facg = nullptr;  // fall back to the scratch in shared memory
    return cudaSuccess;
  }
  ctx->d.facg_doubles = need;
  return cudaSuccess;
}

static int create_context(const hst_gpu_params* pin, int nmem, hst_ctx** out) {
  if (!pin || !out || nmem < 1 || nmem > 4096) return HST_EARG;
  *out = nullptr;
  hst_ctx* ctx = new (std::nothrow) hst_ctx();
  if (!ctx) return HST_ENOMEM;
  ctx->p = *pin;
  ctx->nmem = nmem;
  ctx->launches = 0;
  {
    const char* e = std::getenv("HST_COLUMN_FUSED");
    ctx->column_split = !(e && std::atoi(e) == 1);
    ctx->shift_split = false;  // decided once the geometry is known
    ctx->solve_halves = false;
  }
  ctx->prof_on = false;
  for (int k = 0; k < HST_KC_N; ++k) {
    ctx->prof_ms[k] = 0.0;
    ctx->prof_n[k] = 0;
  }
  ctx->stream = nullptr;
  ctx->h_gdamp = nullptr;
  ctx->h_cfl = nullptr;
  std::memset(&ctx->d, 0, sizeof ctx->d);
  ctx->d.configured = &ctx->configured;
  ctx->d.occupancy = &ctx->occupancy;
  std::string why;
  int rc = choose_geometry(*pin, ctx->g, why);
  if (rc != HST_OK) {
    std::fprintf(stderr, "hst_gpu_create: %s\n", why.c_str());
    delete ctx;
    return rc;
  }
  ctx->p.nxd = ctx->g.nxd;
  ctx->p.nzd = ctx->g.nzd;
  if (ctx->g.mp) {
    // the FP32 product spectra are read only by the streamed right-hand-side kernel
    const char* t = std::getenv("HST_RHS_TILED");
    if (!ctx->column_split || (t && std::atoi(t) == 0)) {
      std::fprintf(stderr, "hst_gpu_create: mixed precision needs the split column stage and the streamed "
                           "right-hand sides (HST_COLUMN_FUSED, HST_RHS_TILED unset)\n");
      delete ctx;
      return HST_EARG;
    }
  }
  const hst_gpu_params& p = ctx->p;
  const Geometry& g = ctx->g;
  ctx->device = p.device;
  // derived quantities (src/hst_input.f90:92-102)
  ctx->lx = 2.0 * PI / p.alfa0;
  ctx->lz = 2.0 * PI / p.beta0;
  ctx->ps.alfa0 = p.alfa0;
  ctx->ps.beta0 = p.beta0;
  ctx->ps.ni = 1.0 / p.re;
  ctx->ps.S = p.S;
  ctx->ps.dx = PI / (p.alfa0 * g.nxd);
  ctx->ps.dz = 2.0 * PI / (p.beta0 * g.nzd);
  ctx->ps.factor = 1.0 / (2.0 * g.nxd * g.nzd);
  // grid (src/hst_setup.f90:42-71)
  const int ny = p.ny;
  ctx->y.resize(ny + 4);
  for (int iy = -2; iy <= ny + 1; ++iy) {
    int mo = imodulo(iy, ny);
    ctx->y[iy + 2] = p.ly * ymap((double)mo / ny, p.ystretch) + p.ly * (double)((iy - mo) / ny);
  }
  ctx->dyl.resize(ny);
  for (int iy = 0; iy < ny; ++iy) ctx->dyl[iy] = 0.5 * (ctx->y[iy + 3] - ctx->y[iy + 1]);
  setup_derivatives(ny, ctx->y, ctx->der);
  ctx->gdamp.assign((size_t)g.ncol, 0.0);
  ctx->theta_last = -1.0e308;
  if (damping_active(p)) damping_update(ctx, 0.0);

  if (cudaSetDevice(p.device) != cudaSuccess) {
    std::fprintf(stderr, "hst_gpu_create: cannot select CUDA device %d\n", p.device);
    delete ctx;
    return HST_ECUDA;
  }
  auto alloc = [&](void** ptr, size_t bytes) -> bool {
    if (cudaMalloc(ptr, bytes) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return true;
  };
  DeviceState& d = ctx->d;
  bool ok = true;
  const size_t nm = (size_t)nmem;  // the per-field buffers hold every member
  for (int i = 0; i < 7 && ok; ++i) ok = alloc((void**)&d.F[i], sizeof(double2) * g.nf * nm);
  const size_t es = g.mp ? sizeof(float2) : sizeof(double2);  // the transforms' complex element
  ok = ok && alloc((void**)&d.Z, es * 3 * (size_t)g.nzd * g.ny * g.nxB * nm);
  ok = ok && alloc((void**)&d.Pp, es * 6 * (size_t)g.nzd * g.ny * g.nxB * nm);
  ok = ok && alloc((void**)&d.Q, es * 6 * (size_t)g.ncol * g.ny * nm);
  if (hst::edge_rows_needed(g, p.s2_amplitude != 0.0 || p.s2_mean != 0.0)) {
    ok = ok && alloc((void**)&d.Zg, es * 3 * (size_t)g.nzd * g.nxB * 4 * nm);
    ok = ok && alloc((void**)&d.Ppg, es * 6 * (size_t)g.nzd * g.nxB * 4 * nm);
    ok = ok && alloc((void**)&d.Qg, es * 6 * (size_t)g.ncol * 4 * nm);
  }
  ok = ok && alloc((void**)&d.der, sizeof(double) * 20 * (size_t)ny);
  ok = ok && alloc((void**)&d.derS, sizeof(double) * 20 * (size_t)ny);
  ok = ok && alloc((void**)&d.derU, sizeof(double) * 20 * (size_t)ny);
  ok = ok && alloc((void**)&d.derI, sizeof(int) * (size_t)ny);
  ok = ok && alloc((void**)&d.d0tab, sizeof(double) * hst::d0_table_doubles(ny));
  ok = ok && alloc((void**)&d.y, sizeof(double) * (ny + 4));
  ok = ok && alloc((void**)&d.dyl, sizeof(double) * ny);
  ok = ok && alloc((void**)&d.gdamp, sizeof(double) * g.ncol);
  ok = ok && alloc((void**)&d.twx, sizeof(double2) * 4 * g.nxd);
  ok = ok && alloc((void**)&d.twz, sizeof(double2) * g.nzd);
  ok = ok && alloc((void**)&d.twxf, sizeof(float2) * 4 * g.nxd);
  ok = ok && alloc((void**)&d.twzf, sizeof(float2) * g.nzd);
  // outstats scratch (sized for the largest reduction grid, 4 blocks an SM of up to 256 SMs)
  ok = ok && alloc((void**)&d.stats, sizeof(double) * ((hst::stats_partials() + 3) * 4 * 256 + 24));
  // two words: the CFL maximum and the bounded-wait error flag
  ok = ok && alloc((void**)&d.cfl, 2 * sizeof(unsigned long long));
  if (ok) d.err = reinterpret_cast<int*>(d.cfl + 1);
  if (!ok) {
    free_device(ctx);
    std::fprintf(stderr, "hst_gpu_create: device allocation of %.2f GB refused\n", dev_bytes(g) / 1e9);
    delete ctx;
    return HST_ENOMEM;
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost((void**)&ctx->h_gdamp, sizeof(double) * g.ncol) != cudaSuccess ||
      cudaMallocHost((void**)&ctx->h_cfl, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    free_device(ctx);
    delete ctx;
    return HST_ECUDA;
  }
  for (int i = 0; i < 7; ++i) cudaMemsetAsync(d.F[i], 0, sizeof(double2) * g.nf * nm, ctx->stream);
  cudaMemsetAsync(d.cfl, 0, 2 * sizeof(unsigned long long), ctx->stream);
  auto tx = twiddles(2 * g.nxd), tz = twiddles(g.nzd);
  cudaMemcpy(d.der, ctx->der.data(), sizeof(double) * 20 * ny, cudaMemcpyHostToDevice);
  cudaError_t etab;
  {
    auto ds = slab_major(ctx->der, ny, g.P, g.m);
    cudaMemcpy(d.derS, ds.data(), sizeof(double) * 20 * ny, cudaMemcpyHostToDevice);
    etab = hst::launch_d0_table(g, d, ctx->stream);
    if (etab == cudaSuccess) etab = upload_der_rows(ctx);
  }
  cudaMemcpy(d.y, ctx->y.data(), sizeof(double) * (ny + 4), cudaMemcpyHostToDevice);
  cudaMemcpy(d.dyl, ctx->dyl.data(), sizeof(double) * ny, cudaMemcpyHostToDevice);
  cudaMemcpy(d.gdamp, ctx->gdamp.data(), sizeof(double) * g.ncol, cudaMemcpyHostToDevice);
  tx.resize((size_t)4 * g.nxd, make_double2(0.0, 0.0));
  hst::staged_twiddles(2 * g.nxd, tx.data() + 2 * g.nxd);
  cudaMemcpy(d.twx, tx.data(), sizeof(double2) * tx.size(), cudaMemcpyHostToDevice);
  {
    // FP32 copies (rounded from the long double values)
    std::vector<float2> fx((size_t)4 * g.nxd, make_float2(0.f, 0.f)), fz(g.nzd);
    for (int k = 0; k < 2 * g.nxd; ++k) {
      long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)(2 * g.nxd);
      fx[k] = make_float2((float)cosl(a), (float)sinl(a));
    }
    hst::staged_twiddles(2 * g.nxd, fx.data() + 2 * g.nxd);
    for (int k = 0; k < g.nzd; ++k) {
      long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)g.nzd;
      fz[k] = make_float2((float)cosl(a), (float)sinl(a));
    }
    cudaMemcpy(d.twxf, fx.data(), sizeof(float2) * fx.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d.twzf, fz.data(), sizeof(float2) * fz.size(), cudaMemcpyHostToDevice);
  }
  cudaMemcpy(d.twz, tz.data(), sizeof(double2) * tz.size(), cudaMemcpyHostToDevice);
  cudaError_t e = etab;
  if (e == cudaSuccess) e = hst::set_fft_constants();
  // the base of all members (maps over nmem members), then member 0's view
  ctx->gb = g;
  ctx->gb.nmem = nmem;
  if (e == cudaSuccess) {
    ctx->db = d;
    e = hst::make_transform_maps(ctx->gb, ctx->db);
  }
  if (e == cudaSuccess) e = hst::make_transform_maps(g, d);
  if (e == cudaSuccess) e = ensure_facg(ctx);
  if (e == cudaSuccess) ctx->db.facg = d.facg, ctx->db.facg_doubles = d.facg_doubles;
  {
    const char* f = std::getenv("HST_SHIFT_SPLIT");
    ctx->shift_split = f ? std::atoi(f) == 1 : ctx->d.facg != nullptr;
    // the solves in two one-line passes (needs the global factor scratch)
    const char* h = std::getenv("HST_SOLVE_HALVES");
    ctx->solve_halves = ctx->d.facg != nullptr && (h ? std::atoi(h) == 1 : true);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "hst_gpu_create: %s\n", cudaGetErrorString(e));
    free_device(ctx);
    delete ctx;
    return HST_ECUDA;
  }
  *out = ctx;
  return HST_OK;
}

extern "C" int hst_gpu_create(const hst_gpu_params* p, hst_ctx** out) { return create_context(p, 1, out); }

extern "C" int hst_gpu_create_batch(const hst_gpu_params* p, int nmem, hst_ctx** out) {
  return create_context(p, nmem, out);
}

extern "C" int hst_gpu_members(const hst_ctx* ctx) { return ctx ? ctx->nmem : 0; }

// The view of member m: every per-field pointer offset to its slice of the
// base buffers, its own TMA maps
extern "C" int hst_gpu_select_member(hst_ctx* ctx, int m) {
  if (!ctx || m < 0 || m >= ctx->nmem) return fail(ctx, HST_EARG, "select_member: member %d of %d", m, ctx ? ctx->nmem : 0);
  if (m == ctx->member) return HST_OK;
  CK(cudaSetDevice(ctx->device));
  const Geometry& g = ctx->g;
  const DeviceState& b = ctx->db;
  DeviceState& d = ctx->d;
  const size_t mm = (size_t)m;
  for (int i = 0; i < 7; ++i) d.F[i] = b.F[i] + mm * g.nf;
  const size_t es = g.mp ? 1 : 2;  // complex elements of the transforms per double2 slot: FP32 ones pack two
  auto off = [&](double2* base, size_t elems) -> double2* {
    if (!base) return nullptr;
    return g.mp ? reinterpret_cast<double2*>(reinterpret_cast<float2*>(base) + mm * elems) : base + mm * elems;
  };
  (void)es;
  d.Z = off(b.Z, 3 * (size_t)g.nzd * g.ny * g.nxB);
  d.Pp = off(b.Pp, 6 * (size_t)g.nzd * g.ny * g.nxB);
  d.Q = off(b.Q, 6 * (size_t)g.ncol * g.ny);
  d.Zg = off(b.Zg, 3 * (size_t)g.nzd * g.nxB * 4);
  d.Ppg = off(b.Ppg, 6 * (size_t)g.nzd * g.nxB * 4);
  d.Qg = off(b.Qg, 6 * (size_t)g.ncol * 4);
  CK(cudaStreamSynchronize(ctx->stream));  // the maps are kernel arguments of work already queued
  CK(hst::make_transform_maps(g, d));
  ctx->member = m;
  return HST_OK;
}

extern "C" int hst_gpu_destroy(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (cudaStream_t q : {ctx->s_in, ctx->s_out})
    if (q) {
      cudaStreamSynchronize(q);
      cudaStreamDestroy(q);
    }
  for (cudaEvent_t e : {ctx->ev_main, ctx->ev_in, ctx->ev_stage, ctx->ev_out})
    if (e) cudaEventDestroy(e);
  for (int c = 0; c < 3; ++c) {
    if (ctx->ev_staged[c]) cudaEventDestroy(ctx->ev_staged[c]);
    if (ctx->ev_read[c]) cudaEventDestroy(ctx->ev_read[c]);
  }
  for (double2* q : ctx->snap)
    if (q) cudaFree(q);
  for (double2* q : ctx->stage)
    if (q) cudaFree(q);
  for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
  free_device(ctx);
  if (ctx->h_gdamp) cudaFreeHost(ctx->h_gdamp);
  if (ctx->h_cfl) cudaFreeHost(ctx->h_cfl);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return HST_OK;
}

static cudaError_t upload_der_rows(hst_ctx* ctx) {
  std::vector<double> tab;
  std::vector<int> idx;
  const int ny = ctx->p.ny;
  const int nu = der_rows(ctx->der, ny, tab, idx);
  // the kernels queued before may still read the previous table
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && nu > 0) e = cudaMemcpy(ctx->d.derU, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d.derI, idx.data(), sizeof(int) * ny, cudaMemcpyHostToDevice);
  ctx->d.nderU = e == cudaSuccess ? nu : 0;
  ctx->db.derU = ctx->d.derU;
  ctx->db.derI = ctx->d.derI;
  ctx->db.nderU = ctx->d.nderU;
  return e;
}

extern "C" const char* hst_gpu_last_error(const hst_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }
extern "C" long long hst_gpu_launch_count(const hst_ctx* ctx) { return ctx ? ctx->launches : 0; }
extern "C" void* hst_gpu_stream(const hst_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int hst_gpu_set_tables(hst_ctx* ctx, const double* der, const double* y, const double* dyl) {
  if (!ctx) return HST_EARG;
  const int ny = ctx->p.ny;
  CK(cudaSetDevice(ctx->device));
  if (der) {
    std::memcpy(ctx->der.data(), der, sizeof(double) * 20 * ny);
    CK(cudaMemcpy(ctx->d.der, ctx->der.data(), sizeof(double) * 20 * ny, cudaMemcpyHostToDevice));
    auto ds = slab_major(ctx->der, ny, ctx->g.P, ctx->g.m);
    CK(cudaMemcpy(ctx->d.derS, ds.data(), sizeof(double) * 20 * ny, cudaMemcpyHostToDevice));
    CK(hst::launch_d0_table(ctx->g, ctx->d, ctx->stream));
    CK(upload_der_rows(ctx));
  }
  if (y) {
    std::memcpy(ctx->y.data(), y, sizeof(double) * (ny + 4));
    CK(cudaMemcpyAsync(ctx->d.y, ctx->y.data(), sizeof(double) * (ny + 4), cudaMemcpyHostToDevice, ctx->stream));
  }
  if (dyl) {
    std::memcpy(ctx->dyl.data(), dyl, sizeof(double) * ny);
    CK(cudaMemcpyAsync(ctx->d.dyl, ctx->dyl.data(), sizeof(double) * ny, cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}

extern "C" int hst_gpu_get_tables(const hst_ctx* c, double* der, double* y, double* dyl) {
  if (!c) return HST_EARG;
  const int ny = c->p.ny;
  if (der) std::memcpy(der, c->der.data(), sizeof(double) * 20 * ny);
  if (y) std::memcpy(y, c->y.data(), sizeof(double) * (ny + 4));
  if (dyl) std::memcpy(dyl, c->dyl.data(), sizeof(double) * ny);
  return HST_OK;
}

extern "C" int hst_gpu_upload(hst_ctx* ctx, int field, const double* host) {
  if (!ctx || field < 0 || field > 6 || !host) return fail(ctx, HST_EARG, "upload: bad field %d", field);
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->d.F[field], host, sizeof(double2) * ctx->g.nf, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}

extern "C" int hst_gpu_download(hst_ctx* ctx, int field, double* host) {
  if (!ctx || field < 0 || field > 6 || !host) return fail(ctx, HST_EARG, "download: bad field %d", field);
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(host, ctx->d.F[field], sizeof(double2) * ctx->g.nf, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}

// ------------------------------------------------- asynchronous host I/O ----
static int ensure_io(hst_ctx* ctx) {
  if (ctx->s_in) return HST_OK;
  CK(cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&ctx->ev_main, &ctx->ev_in, &ctx->ev_stage, &ctx->ev_out})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (int c = 0; c < 3; ++c) {
    CK(cudaEventCreateWithFlags(&ctx->ev_staged[c], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_read[c], cudaEventDisableTiming));
  }
  return HST_OK;
}

extern "C" int hst_gpu_upload_async(hst_ctx* ctx, int field, const double* host) {
  if (!ctx || field < 0 || field > 2 || !host) return fail(ctx, HST_EARG, "upload_async: bad field %d", field);
  CK(cudaSetDevice(ctx->device));
  int rc = ensure_io(ctx);
  if (rc != HST_OK) return rc;
  const size_t bytes = sizeof(double2) * ctx->g.nf;
  if (!ctx->stage[field] && cudaMalloc((void**)&ctx->stage[field], bytes) != cudaSuccess) {
    cudaGetLastError();
    ctx->stage[field] = nullptr;
    return fail(ctx, HST_ENOMEM, "upload_async: staging copy of %.2f GB refused", bytes / 1e9);
  }
  // host -> staging copy on the copy-in stream, as soon as the solver's
  // stream has moved the previous upload of this component into V (so it
  // runs beside the work queued before this call); then staging -> V on
  // the solver's stream, after everything queued so far, before anything
  // queued later
  if (ctx->staged_used[field]) CK(cudaStreamWaitEvent(ctx->s_in, ctx->ev_staged[field], 0));
  CK(cudaMemcpyAsync(ctx->stage[field], host, bytes, cudaMemcpyHostToDevice, ctx->s_in));
  CK(cudaEventRecord(ctx->ev_in, ctx->s_in));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_in, 0));
  CK(cudaMemcpyAsync(ctx->d.F[field], ctx->stage[field], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaEventRecord(ctx->ev_staged[field], ctx->stream));
  ctx->staged_used[field] = true;
  return HST_OK;
}

extern "C" int hst_gpu_download_async(hst_ctx* ctx, int field, double* host) {
  if (!ctx || field < 0 || field > 2 || !host) return fail(ctx, HST_EARG, "download_async: bad field %d", field);
  CK(cudaSetDevice(ctx->device));
  int rc = ensure_io(ctx);
  if (rc != HST_OK) return rc;
  const size_t bytes = sizeof(double2) * ctx->g.nf;
  if (!ctx->snap[field] && cudaMalloc((void**)&ctx->snap[field], bytes) != cudaSuccess) {
    cudaGetLastError();
    ctx->snap[field] = nullptr;
    return fail(ctx, HST_ENOMEM, "download_async: snapshot of %.2f GB refused", bytes / 1e9);
  }
  // the snapshot may be overwritten once the previous copy-out of this
  // component has read it
  if (ctx->read_used[field]) CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_read[field], 0));
  CK(cudaMemcpyAsync(ctx->snap[field], ctx->d.F[field], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaEventRecord(ctx->ev_stage, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->s_out, ctx->ev_stage, 0));
  CK(cudaMemcpyAsync(host, ctx->snap[field], bytes, cudaMemcpyDeviceToHost, ctx->s_out));
  CK(cudaEventRecord(ctx->ev_read[field], ctx->s_out));
  ctx->read_used[field] = true;
  return HST_OK;
}

extern "C" int hst_gpu_wait_io(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->s_in) return HST_OK;
  // the solver's stream also waits for both copy streams, so that work
  // queued on it afterwards (or an event recorded there) follows the copies
  CK(cudaEventRecord(ctx->ev_in, ctx->s_in));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_in, 0));
  CK(cudaEventRecord(ctx->ev_out, ctx->s_out));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_out, 0));
  CK(cudaStreamSynchronize(ctx->s_in));
  CK(cudaStreamSynchronize(ctx->s_out));
  return HST_OK;
}

extern "C" int hst_gpu_sync(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}

extern "C" int hst_gpu_shear_shifts(const hst_ctx* c, double t, double* sx, double* sz) {
  if (!c || !sx || !sz) return HST_EARG;
  shear_shifts(c, t, sx, sz);
  return HST_OK;
}
extern "C" double hst_gpu_s2_of(const hst_ctx* c, double t) { return c ? s2_of(c->p, t) : 0.0; }
extern "C" double hst_gpu_s2_integral(const hst_ctx* c, double t1, double t2) {
  return c ? s2_integral(c->p, t1, t2) : 0.0;
}

extern "C" int hst_gpu_fill_ghosts(hst_ctx* ctx, int field, double sx, double sz) {
  if (!ctx || field < 0 || field > 6) return fail(ctx, HST_EARG, "fill_ghosts: bad field %d", field);
  CK(cudaSetDevice(ctx->device));
  CK(timed(ctx, HST_KC_GHOSTS, [&] { return hst::launch_fill_ghosts(ctx->g, ctx->d, ctx->ps, field, sx, sz, ctx->stream); }));
  return HST_OK;
}

extern "C" int hst_gpu_fill_ghosts_at(hst_ctx* ctx, int field, double time) {
  if (!ctx) return HST_EARG;
  double sx, sz;
  shear_shifts(ctx, time, &sx, &sz);
  return hst_gpu_fill_ghosts(ctx, field, sx, sz);
}

extern "C" int hst_gpu_line_solve(hst_ctx* ctx, int sys, double lambda, int src, int dst, int has_shift, double sx,
                                  double sz, double time) {
  if (!ctx || sys < 1 || sys > 5 || src < 0 || src > 6 || dst < 0 || dst > 6 || src == dst)
    return fail(ctx, HST_EARG, "line_solve: bad arguments (sys %d, src %d, dst %d)", sys, src, dst);
  if (!has_shift) shear_shifts(ctx, time, &sx, &sz);
  CK(cudaSetDevice(ctx->device));
  CK(timed(ctx, HST_KC_LINE_SOLVE,
           [&] { return hst::launch_line_solve(ctx->g, ctx->d, ctx->ps, sys, lambda, src, dst, sx, sz, ctx->stream); }));
  return HST_OK;
}

static int read_cfl(hst_ctx* ctx, double* cfl) {
  CK(cudaMemcpyAsync(ctx->h_cfl, ctx->d.cfl, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_cfl[1] != 0) {
    CK(cudaMemsetAsync(ctx->d.err, 0, sizeof(int), ctx->stream));
    return fail(ctx, HST_ETIMEOUT, "a kernel's bounded wait for its TMA copies ran out; the step is invalid");
  }
  unsigned long long b = *ctx->h_cfl;
  double v;
  std::memcpy(&v, &b, sizeof v);
  if (cfl) *cfl = v;
  if (!std::isfinite(v)) return fail(ctx, HST_EFINITE, "non-finite CFL number %g", v);
  return HST_OK;
}

extern "C" int hst_gpu_compute_cfl(hst_ctx* ctx, double* cfl) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->d.cfl, 0, sizeof(unsigned long long), ctx->stream));
  CK(timed(ctx, HST_KC_ZINV, [&] { return hst::launch_zinv(ctx->g, ctx->d, ctx->stream); }));
  CK(timed(ctx, HST_KC_XPROD, [&] { return hst::launch_xprod(ctx->g, ctx->d, ctx->ps, 1, ctx->stream); }));
  return read_cfl(ctx, cfl);
}

// outstats (src/hst_stats.f90:136-285) of the resident field at `time`:
// the three DY solves go through RHS1, which is scratch between steps (as
// the reference's rhs is).  res (24 doubles on the host): the 8 box averages,
// then the 16 sums of the reference's `sums` array; exz (ncol doubles, may
// be NULL): the column energies, computed into RHS1 after the solves.
static int outstats_all(hst_ctx* ctx, double time, double* res_h, double* exz_h) {
  CK(cudaSetDevice(ctx->device));
  const Geometry& g = ctx->g;
  const int nblk = hst::stats_blocks(g, ctx->d.nsm);
  if (nblk > 4 * 256) return fail(ctx, HST_EARG, "outstats: %d reduction blocks exceed the scratch", nblk);
  double* pm = ctx->d.stats;
  double* pg = pm + (size_t)hst::stats_partials() * nblk;
  double* res = pg + (size_t)3 * nblk;
  double sx, sz;
  shear_shifts(ctx, time, &sx, &sz);
  for (int c = 0; c < 3; ++c) {
    CK(timed(ctx, HST_KC_LINE_SOLVE, [&] {
      return hst::launch_line_solve(g, ctx->d, ctx->ps, hst::K_DY, 0.0, c, HST_RHS1, sx, sz, ctx->stream);
    }));
    CK(hst::launch_stats_grad(g, ctx->d, HST_RHS1, pg + (size_t)c * nblk, ctx->stream));
    ctx->launches++;
  }
  const double gsoft = (damping_active(ctx->p) && !ctx->p.damp_hard) ? 1.0 : 0.0;
  CK(hst::launch_stats_moments(g, ctx->d, ctx->ps, gsoft, pm, ctx->stream));
  double ly_w = 0.0;
  for (int iy = 0; iy < g.ny; ++iy) ly_w += ctx->dyl[iy];
  CK(hst::launch_stats_final(g, ctx->d, pm, pg, ly_w, ctx->ps.ni, ctx->p.ly, res, ctx->stream));
  ctx->launches += 2;
  double* exz_d = reinterpret_cast<double*>(ctx->d.F[HST_RHS1]);
  if (exz_h) {
    CK(hst::launch_stats_columns(g, ctx->d, exz_d, ctx->stream));
    ctx->launches++;
  }
  CK(cudaMemcpyAsync(res_h, res, 24 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (exz_h) CK(cudaMemcpyAsync(exz_h, exz_d, sizeof(double) * g.ncol, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // ncol_damped (src/hst_damping.f90:113): the columns of the current table
  int n = 0;
  if (damping_active(ctx->p))
    for (double v : ctx->gdamp) n += v > 0.0;
  res_h[8 + 15] = (double)n;
  return HST_OK;
}

extern "C" int hst_gpu_outstats(hst_ctx* ctx, double time, double* out) {
  if (!ctx || !out) return HST_EARG;
  double res[24];
  int rc = outstats_all(ctx, time, res, nullptr);
  if (rc != HST_OK) return rc;
  std::memcpy(out, res, 8 * sizeof(double));
  return HST_OK;
}

extern "C" int hst_gpu_outstats_sums(hst_ctx* ctx, double time, double* sums, double* exz) {
  if (!ctx || !sums) return HST_EARG;
  double res[24];
  int rc = outstats_all(ctx, time, res, exz);
  if (rc != HST_OK) return rc;
  std::memcpy(sums, res + 8, 16 * sizeof(double));
  return HST_OK;
}

// compute_pressure (src/hst_pressure.f90:35-110) of the resident field at
// `time` into field dst (RHS2 in the reference's write_pressure); the
// transform buffers and RHS1 are scratch
extern "C" int hst_gpu_pressure(hst_ctx* ctx, double time, int dst) {
  if (!ctx || dst < HST_OLD1 || dst > HST_RHS2 || dst == HST_RHS1)
    return fail(ctx, HST_EARG, "pressure: dst must be OLD1, OLD2 or RHS2 (got %d)", dst);
  CK(cudaSetDevice(ctx->device));
  const Geometry& g = ctx->g;
  double sx, sz;
  shear_shifts(ctx, time, &sx, &sz);
  CK(timed(ctx, HST_KC_ZINV, [&] { return hst::launch_zinv(g, ctx->d, ctx->stream); }));
  CK(timed(ctx, HST_KC_XPROD, [&] { return hst::launch_xprod(g, ctx->d, ctx->ps, 0, ctx->stream); }));
  CK(timed(ctx, HST_KC_ZFWD, [&] { return hst::launch_zfwd(g, ctx->d, ctx->stream); }));
  CK(hst::launch_pressure_rhs(g, ctx->d, ctx->ps, s2_of(ctx->p, time), sx, sz, ctx->stream));
  CK(timed(ctx, HST_KC_LINE_SOLVE, [&] {
    return hst::launch_line_solve(g, ctx->d, ctx->ps, hst::K_POISSON, 0.0, HST_RHS1, dst, sx, sz, ctx->stream);
  }));
  CK(hst::launch_pressure_mean(g, ctx->d, ctx->p.ly, dst, ctx->stream));
  ctx->launches += 2;
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}

static int queue_timestep(hst_ctx* ctx, double* time, double deltat);

// ------------------------------------------------------------ autotune ----
// Tries the launch choices that leave every buffer's layout unchanged -- the
// lanes of a line-solver group (P) and the points a thread of the x and z
// FFT plans -- on this context's own sizes, `steps` time steps each after
// one untimed step, keeps the fastest, and puts the fields and the time back
// as they were.  The report lists every candidate with its time a step.
extern "C" int hst_gpu_autotune(hst_ctx* ctx, double deltat, int steps, char* report, int report_len) {
  if (!ctx || steps < 1) return fail(ctx, HST_EARG, "autotune: bad arguments");
  if (ctx->nmem > 1) return fail(ctx, HST_EARG, "autotune: not for an ensemble context");
  CK(cudaSetDevice(ctx->device));
  Geometry& g = ctx->g;
  const Geometry g0 = g;
  std::string rep;
  // state to put back: V1..V3, OLD1, OLD2 (RHS1/2 and the transform buffers are scratch)
  std::vector<double2*> save(5, nullptr);
  auto release = [&] {
    for (double2* q : save)
      if (q) cudaFree(q);
  };
  const size_t fb = sizeof(double2) * g.nf;
  for (int i = 0; i < 5; ++i) {
    if (cudaMalloc((void**)&save[i], fb) != cudaSuccess) {
      cudaGetLastError();
      release();
      return fail(ctx, HST_ENOMEM, "autotune: no room for a copy of the state");
    }
    CK(cudaMemcpyAsync(save[i], ctx->d.F[i], fb, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  // the damping state the trial steps may move on
  const double theta0 = ctx->theta_last, time0 = 0.0;
  const std::vector<double> gdamp0 = ctx->gdamp;
  // candidates
  std::vector<int> lanes;
  for (int c = 32; c >= 4; c >>= 1) {
    Geometry t = g0;
    if (g0.ny % c != 0 || g0.ny / c < 4) continue;
    t.P = c;
    t.m = g0.ny / c;
    t.MS = t.m | 1;
    if (hst::column_smem_bytes(t, 1) <= 200 * 1024) lanes.push_back(c);
  }
  const int NX = 2 * g0.nxd;
  std::vector<int> px, pz;
  if (g0.mp) {
    px.push_back(8);
  } else {
    px.push_back(16);
    if (NX == 192 || NX == 384 || NX == 768) px.push_back(8);
  }
  for (int v : {16, 8}) {
    if (g0.mp && g0.nzd == 768 && v == 16) continue;
    if (v == 8 && !(g0.nzd == 192 || g0.nzd == 384 || g0.nzd == 768)) continue;
    if (v == 8 && g0.Ty * g0.nzd / 8 > 384) continue;
    if (v == 16 && g0.Ty * g0.nzd / 16 > 256) continue;
    pz.push_back(v);
  }
  if (pz.empty()) pz.push_back(g0.pptz);  // one plan only (1536 points)
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  Geometry gbest = g0;
  int rc = HST_OK;
  auto apply = [&](const Geometry& t) -> cudaError_t {
    g = t;
    auto ds = slab_major(ctx->der, g.ny, g.P, g.m);
    cudaError_t e = cudaMemcpy(ctx->d.derS, ds.data(), sizeof(double) * 20 * g.ny, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = hst::launch_d0_table(g, ctx->d, ctx->stream);
    if (e == cudaSuccess) e = hst::make_transform_maps(g, ctx->d);
    if (e == cudaSuccess) e = ensure_facg(ctx);
    return e;
  };
  for (int P : lanes)
    for (int a : px)
      for (int b : pz) {
        Geometry t = g0;
        t.P = P;
        t.m = g0.ny / P;
        t.MS = t.m | 1;
        t.pptx = a;
        t.pptz = b;
        if (apply(t) != cudaSuccess) continue;
        for (int i = 0; i < 5 && rc == HST_OK; ++i)
          if (cudaMemcpyAsync(ctx->d.F[i], save[i], fb, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
            rc = HST_ECUDA;
        double tt = time0;
        if (rc == HST_OK) rc = queue_timestep(ctx, &tt, deltat);
        if (rc == HST_OK && cudaEventRecord(e0, ctx->stream) != cudaSuccess) rc = HST_ECUDA;
        for (int k = 0; k < steps && rc == HST_OK; ++k) rc = queue_timestep(ctx, &tt, deltat);
        if (rc == HST_OK && cudaEventRecord(e1, ctx->stream) != cudaSuccess) rc = HST_ECUDA;
        if (rc == HST_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = HST_ECUDA;
        if (rc != HST_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double per = ms / steps;
        char line[128];
        std::snprintf(line, sizeof line, "P=%d x=%d z=%d: %.4f ms a step\n", P, a, b, per);
        rep += line;
        if (per < best) {
          best = per;
          gbest = t;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the winner, and the state as it was
  if (apply(rc == HST_OK ? gbest : g0) != cudaSuccess && rc == HST_OK) rc = HST_ECUDA;
  for (int i = 0; i < 5; ++i) cudaMemcpyAsync(ctx->d.F[i], save[i], fb, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  release();
  ctx->theta_last = theta0;
  if (ctx->gdamp != gdamp0) {
    ctx->gdamp = gdamp0;
    CK(cudaMemcpy(ctx->d.gdamp, ctx->gdamp.data(), sizeof(double) * g.ncol, cudaMemcpyHostToDevice));
  }
  if (rc != HST_OK) return rc;
  char line[128];
  std::snprintf(line, sizeof line, "chosen: P=%d x=%d z=%d\n", g.P, g.pptx, g.pptz);
  rep += line;
  if (report && report_len > 0) std::snprintf(report, (size_t)report_len, "%s", rep.c_str());
  return HST_OK;
}

// ---------------------------------------------------- restart files ----
// The CPL field file of restart_write / restart_read (src/hst_io.f90:69-178,
// 240-315): a text header (the mesh with the CPL names: its "ny" is nz and
// its "nz" is ny+1), raw FP64 time, S, S2, gamma_x, gamma_y, then
// V(-2..ny+1, -nz..nz, 0..nx) in CPL component order (u, w, v), components
// innermost; the file's ghost rows are plain copies of rows 0, 1 and
// ny-2, ny-1.
static std::string real_txt(double x) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17G", x);
  return b;
}

extern "C" int hst_gpu_write_restart(hst_ctx* ctx, const char* path, double time, double deltat, double t_max,
                                     double dt_field, double dt_save) {
  if (!ctx || !path) return HST_EARG;
  const hst_gpu_params& p = ctx->p;
  const Geometry& g = ctx->g;
  const int ny = g.ny, rows = g.rows;
  // the three components (FP64, the context's layout)
  std::vector<double2> V((size_t)3 * g.nf);
  for (int c = 0; c < 3; ++c) {
    int rc = hst_gpu_download(ctx, c, reinterpret_cast<double*>(V.data() + (size_t)c * g.nf));
    if (rc != HST_OK) return rc;
  }
  std::string h = "nx=" + std::to_string(p.nx) + " \tny=" + std::to_string(p.nz) + " \tnz=" + std::to_string(ny + 1) +
                  " \talpha0=" + real_txt(p.alfa0) + " \tbeta0=" + real_txt(p.beta0) +
                  " \thtcoeff=" + real_txt(p.ystretch > 0.0 ? p.ystretch : -1.0) + " \tRe=" + real_txt(p.re) +
                  " \tPr=0.71\n" + "deltat=" + real_txt(deltat) + " \tt_max=" + real_txt(t_max) +
                  " \tdt_field=" + real_txt(dt_field) + " \tdt_save=" + real_txt(dt_save) + "\n" +
                  "t_field=" + real_txt(time) + "\n" + "meanpx=0 \tmeanflowx=0 \tmeanpy=0 \tmeanflowy=0\n";
  auto raw = [&](const char* key, double v) {
    h += key;
    h += "=\n";
    h.append(reinterpret_cast<const char*>(&v), 8);
    h += "\n";
  };
  raw("time", time);
  raw("S", p.S);
  raw("S2", s2_of(p, time));
  raw("gamma_x", p.S * time);
  raw("gamma_y", s2_integral(p, p.s2_start, time));
  h += "Vfield=\n";
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(ctx, HST_EARG, "write_restart: cannot create %s", path);
  bool ok = std::fwrite(h.data(), 1, h.size(), fp) == h.size();
  static const int cpl[3] = {0, 2, 1};  // CPL (u, v, w) = (u, w, v) here
  std::vector<double2> line((size_t)rows * 3);
  for (int ix = 0; ix < g.nxB && ok; ++ix)
    for (int iz = 0; iz < g.nzT && ok; ++iz) {
      const size_t cb = ((size_t)ix * g.nzT + iz) * rows + 2;
      for (int r = -2; r <= ny + 1; ++r) {
        const int iy = r < 0 ? r + ny : (r >= ny ? r - ny : r);
        for (int k = 0; k < 3; ++k) line[(size_t)(r + 2) * 3 + k] = V[(size_t)cpl[k] * g.nf + cb + iy];
      }
      ok = std::fwrite(line.data(), sizeof(double2), line.size(), fp) == line.size();
    }
  ok = (std::fclose(fp) == 0) && ok;
  return ok ? HST_OK : fail(ctx, HST_EARG, "write_restart: short write to %s", path);
}

extern "C" int hst_gpu_read_restart(hst_ctx* ctx, const char* path, double* time) {
  if (!ctx || !path) return HST_EARG;
  const Geometry& g = ctx->g;
  const int ny = g.ny, rows = g.rows;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(ctx, HST_EARG, "read_restart: cannot open %s", path);
  std::vector<char> all;
  char b[1 << 16];
  size_t n;
  while ((n = std::fread(b, 1, sizeof b, fp)) > 0) all.insert(all.end(), b, b + n);
  std::fclose(fp);
  const std::string head(all.begin(), all.begin() + std::min<size_t>(all.size(), 4096));
  const size_t pv = head.find("Vfield=\n"), pt = head.find("time=\n");
  if (pv == std::string::npos || pt == std::string::npos) return fail(ctx, HST_EARG, "read_restart: %s has no CPL header", path);
  auto num = [&](const char* key) -> long {
    const size_t q = head.find(key);
    return q == std::string::npos ? -1 : std::strtol(head.c_str() + q + std::strlen(key), nullptr, 10);
  };
  if (num("nx=") != ctx->p.nx || num("ny=") != ctx->p.nz || num("nz=") != ny + 1)
    return fail(ctx, HST_EARG, "read_restart: %s holds another mesh (nx=%ld ny=%ld nz=%ld in CPL names)", path,
                num("nx="), num("ny="), num("nz="));
  double t;
  std::memcpy(&t, all.data() + pt + 6, 8);
  const size_t need = (size_t)g.nxB * g.nzT * rows * 3 * sizeof(double2);
  if (all.size() < pv + 8 + need) return fail(ctx, HST_EARG, "read_restart: %s is truncated", path);
  const char* data = all.data() + pv + 8;
  static const int cpl[3] = {0, 2, 1};
  std::vector<double2> V((size_t)g.nf);
  for (int k = 0; k < 3; ++k) {
    for (size_t col = 0; col < (size_t)g.ncol; ++col)
      for (int r = 0; r < rows; ++r)
        std::memcpy(&V[col * rows + r], data + ((col * rows + r) * 3 + k) * sizeof(double2), sizeof(double2));
    int rc = hst_gpu_upload(ctx, cpl[k], reinterpret_cast<const double*>(V.data()));
    if (rc == HST_OK) rc = hst_gpu_fill_ghosts_at(ctx, cpl[k], t);
    if (rc != HST_OK) return rc;
  }
  if (time) *time = t;
  return HST_OK;
}

// the solve stage of a substep whose right-hand sides (and exact_shift
// shift) are done: one kernel, or its two one-line halves
static cudaError_t solve_stage(hst_ctx* ctx, const hst::Geometry& G, const hst::DeviceState& D,
                               const hst::SubstepScalars& sc, int nonlin) {
  if (ctx->solve_halves)
    return timed(
        ctx, HST_KC_COLUMN,
        [&] {
          cudaError_t e = hst::launch_column(G, D, ctx->ps, sc, 0, nonlin, 5, ctx->stream);
          return e == cudaSuccess ? hst::launch_column(G, D, ctx->ps, sc, 0, nonlin, 6, ctx->stream) : e;
        },
        2);
  return timed(ctx, HST_KC_COLUMN, [&] { return hst::launch_column(G, D, ctx->ps, sc, 0, nonlin, 2, ctx->stream); });
}

// One time step (src/hst_equations.f90:56-87) queued on the stream.
static int queue_timestep(hst_ctx* ctx, double* time, double deltat) {
  static const double RK[3][3] = {{120.0 / 32.0, 2.0, 0.0}, {120.0 / 8.0, 50.0 / 8.0, 34.0 / 8.0},
                                  {120.0 / 20.0, 90.0 / 20.0, 50.0 / 20.0}};
  const hst_gpu_params& p = ctx->p;
  const bool damp = damping_active(p);
  // every member of an ensemble at once (the base buffers); the field itself otherwise
  const Geometry& G = ctx->nmem > 1 ? ctx->gb : ctx->g;
  const DeviceState& D = ctx->nmem > 1 ? ctx->db : ctx->d;
  for (int i = 0; i < 3; ++i) {
    const double* ODE = RK[i];
    const double t = *time;
    if (!p.linear || i == 2) {
      if (i == 2) CK(cudaMemsetAsync(D.cfl, 0, sizeof(unsigned long long), ctx->stream));
      CK(timed(ctx, HST_KC_ZINV, [&] { return hst::launch_zinv(G, D, ctx->stream); }));
      CK(timed(ctx, HST_KC_XPROD, [&] { return hst::launch_xprod(G, D, ctx->ps, i == 2, ctx->stream); }));
      if (!p.linear) CK(timed(ctx, HST_KC_ZFWD, [&] { return hst::launch_zfwd(G, D, ctx->stream); }));
    }
    if (damp && damping_update(ctx, t)) {
      // stream-ordered upload of the new table (the previous copy has been
      // consumed once the stream reaches it, so wait before refilling)
      CK(cudaStreamSynchronize(ctx->stream));
      std::memcpy(ctx->h_gdamp, ctx->gdamp.data(), sizeof(double) * ctx->g.ncol);
      CK(cudaMemcpyAsync(D.gdamp, ctx->h_gdamp, sizeof(double) * ctx->g.ncol, cudaMemcpyHostToDevice, ctx->stream));
    }
    SubstepScalars sc;
    sc.ode0 = ODE[0];
    sc.ode1 = ODE[1];
    sc.ode2 = ODE[2];
    sc.deltat = deltat;
    const double dt_sub = 2.0 / ODE[0] * deltat;
    sc.lambda = ODE[0] / deltat;
    sc.s2now = s2_of(p, t);
    sc.gsoft = (damp && !p.damp_hard) ? 1.0 : 0.0;
    sc.damp_hard = (p.damp_hard && damp) ? 1 : 0;
    sc.dgx = p.S * dt_sub;
    sc.dgz = s2_integral(p, t, t + dt_sub);
    sc.yuni = p.ystretch <= 1.0e-10 ? 1 : 0;
    sc.ytile = p.ly * 32.0 / p.ny;
    shear_shifts(ctx, t, &sc.sx_t, &sc.sz_t);
    shear_shifts(ctx, t + dt_sub, &sc.sx_n, &sc.sz_n);
    if (ctx->column_split) {
      CK(timed(ctx, HST_KC_RHS,
               [&] { return hst::launch_column(G, D, ctx->ps, sc, p.exact_shift, !p.linear, 1, ctx->stream); }));
      if (p.exact_shift && ctx->shift_split) {
        // the exact_shift shift as a kernel of its own (one line a group,
        // no factor scratch: more warps an SM), then the solves
        CK(timed(ctx, HST_KC_SHIFT,
                 [&] { return hst::launch_column(G, D, ctx->ps, sc, 1, 0, 3, ctx->stream); }));
        CK(solve_stage(ctx, G, D, sc, !p.linear));
      } else if (!p.exact_shift && ctx->solve_halves) {
        CK(solve_stage(ctx, G, D, sc, !p.linear));
      } else {
        CK(timed(ctx, HST_KC_COLUMN, [&] {
          return hst::launch_column(G, D, ctx->ps, sc, p.exact_shift, !p.linear, 2, ctx->stream);
        }));
      }
    } else {
      CK(timed(ctx, HST_KC_COLUMN,
               [&] { return hst::launch_column(G, D, ctx->ps, sc, p.exact_shift, !p.linear, 0, ctx->stream); }));
    }
    *time = t + dt_sub;
  }
  return HST_OK;
}

extern "C" int hst_gpu_timestep(hst_ctx* ctx, double* time, double deltat, double* cfl) {
  if (!ctx || !time) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  int rc = queue_timestep(ctx, time, deltat);
  if (rc != HST_OK) return rc;
  return read_cfl(ctx, cfl);
}

extern "C" int hst_gpu_timesteps(hst_ctx* ctx, int n, double* time, double deltat) {
  if (!ctx || !time || n < 0) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  for (int k = 0; k < n; ++k) {
    int rc = queue_timestep(ctx, time, deltat);
    if (rc != HST_OK) return rc;
  }
  return HST_OK;
}

extern "C" int hst_gpu_set_profiling(hst_ctx* ctx, int on) {
  if (!ctx) return HST_EARG;
  ctx->prof_on = on != 0;
  return HST_OK;
}

extern "C" int hst_gpu_kernel_times(hst_ctx* ctx, double* ms, long long* count) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  for (size_t k = 0; k < ctx->ev_class.size(); ++k) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->ev[2 * k], ctx->ev[2 * k + 1]));
    ctx->prof_ms[ctx->ev_class[k]] += t;
    ctx->prof_n[ctx->ev_class[k]] += 1;
  }
  ctx->ev_class.clear();
  for (int k = 0; k < HST_KC_N; ++k) {
    if (ms) ms[k] = ctx->prof_ms[k];
    if (count) count[k] = ctx->prof_n[k];
  }
  return HST_OK;
}

extern "C" int hst_gpu_reset_kernel_times(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->ev_class.clear();
  for (int k = 0; k < HST_KC_N; ++k) {
    ctx->prof_ms[k] = 0.0;
    ctx->prof_n[k] = 0;
  }
  return HST_OK;
}

// ------------------------------------------------- the substep in pieces ----
// The module procedures of hst_transforms, hst_fft and hst_equations one at
// a time, on buffers in the reference's layouts (hst_pieces.cu), for callers
// that run the substep's pieces themselves.  The buffers are allocated by the
// first call that needs them.
static size_t piece_comp_elems(const Geometry& g, int buf) {
  return buf == HST_BUF_VVDZ ? (size_t)g.rows * g.nxB * g.nzd : (size_t)g.rows * g.nzd * (g.nxd + 1);
}
static double2* piece_buf(hst_ctx* ctx, int buf) {
  return buf == HST_BUF_VVDZ ? ctx->d.vvdz : (buf == HST_BUF_VVDX ? ctx->d.vvdx : ctx->d.vvdp);
}

static int ensure_pieces(hst_ctx* ctx) {
  if (ctx->d.vvdz) return HST_OK;
  CK(cudaSetDevice(ctx->device));
  const Geometry& g = ctx->g;
  double2** bufs[3] = {&ctx->d.vvdz, &ctx->d.vvdx, &ctx->d.vvdp};
  for (int b = 0; b < 3; ++b) {
    const size_t bytes = sizeof(double2) * 3 * piece_comp_elems(g, b);
    if (cudaMalloc((void**)bufs[b], bytes) != cudaSuccess) {
      cudaGetLastError();
      for (int k = 0; k < 3; ++k)
        if (*bufs[k]) cudaFree(*bufs[k]);
      ctx->d.vvdz = ctx->d.vvdx = ctx->d.vvdp = nullptr;
      return fail(ctx, HST_ENOMEM, "the per-piece buffers (3 x %.2f GB) were refused",
                  3.0 * sizeof(double2) * piece_comp_elems(g, 1) / 1e9);
    }
    CK(cudaMemsetAsync(*bufs[b], 0, bytes, ctx->stream));
  }
  return HST_OK;
}

static int check_m(hst_ctx* ctx, int m, const char* what) {
  if (m < 1 || m > 3) return fail(ctx, HST_EARG, "%s: component m = %d, expected 1..3", what, m);
  return HST_OK;
}

extern "C" int hst_gpu_fft(hst_ctx* ctx, int kind, int m) {
  if (!ctx) return HST_EARG;
  int rc = check_m(ctx, m, "fft");
  if (rc == HST_OK) rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  const Geometry& g = ctx->g;
  const hst::DeviceState& d = ctx->d;
  const int c = m - 1;
  if (kind == HST_FFT_FFT || kind == HST_FFT_IFT) {
    const size_t ce = piece_comp_elems(g, HST_BUF_VVDZ);
    CK(hst::launch_piece_lines(d, d.vvdz + c * ce, g.nzd, g.rows * g.nxB, g.nzd, 0, kind == HST_FFT_IFT ? +1 : -1,
                               d.twz, ctx->stream));
  } else if (kind == HST_FFT_RFT) {
    const size_t ce = piece_comp_elems(g, HST_BUF_VVDX);
    CK(hst::launch_piece_lines(d, d.vvdx + c * ce, g.nxd + 1, g.rows * g.nzd, 2 * g.nxd, 1, +1, d.twx, ctx->stream));
  } else if (kind == HST_FFT_HFT) {
    const size_t ce = piece_comp_elems(g, HST_BUF_VVDP);
    CK(hst::launch_piece_lines(d, d.vvdp + c * ce, g.nxd + 1, g.rows * g.nzd, 2 * g.nxd, 2, -1, d.twx, ctx->stream));
  } else {
    return fail(ctx, HST_EARG, "fft: unknown kind %d", kind);
  }
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_transpose(hst_ctx* ctx, int dir, int m) {
  if (!ctx) return HST_EARG;
  int rc = check_m(ctx, m, "transpose");
  if (rc == HST_OK) rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  if (dir != HST_Z_TO_X && dir != HST_X_TO_Z) return fail(ctx, HST_EARG, "transpose: unknown direction %d", dir);
  CK(hst::launch_transpose(ctx->g, ctx->d, dir == HST_Z_TO_X, m - 1, ctx->stream));
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_transform_to_physical(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  int rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(hst::launch_assemble_vvdz(ctx->g, ctx->d, ctx->stream));
  ctx->launches++;
  for (int m = 1; m <= 3 && rc == HST_OK; ++m) {
    rc = hst_gpu_fft(ctx, HST_FFT_IFT, m);
    if (rc == HST_OK) rc = hst_gpu_transpose(ctx, HST_Z_TO_X, m);
    if (rc == HST_OK) rc = hst_gpu_fft(ctx, HST_FFT_RFT, m);
  }
  return rc;
}

extern "C" int hst_gpu_build_products(hst_ctx* ctx, int grp) {
  if (!ctx) return HST_EARG;
  if (grp != 1 && grp != 2) return fail(ctx, HST_EARG, "build_products: group %d, expected 1 or 2", grp);
  int rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(hst::launch_build_products(ctx->g, ctx->d, ctx->ps, grp, ctx->stream));
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_products_to_spectral(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  int rc = ensure_pieces(ctx);
  for (int m = 1; m <= 3 && rc == HST_OK; ++m) {
    rc = hst_gpu_fft(ctx, HST_FFT_HFT, m);
    if (rc == HST_OK) rc = hst_gpu_transpose(ctx, HST_X_TO_Z, m);
    if (rc == HST_OK) rc = hst_gpu_fft(ctx, HST_FFT_FFT, m);
  }
  return rc;
}

extern "C" int hst_gpu_vvdz_to_field(hst_ctx* ctx, int field, int m) {
  if (!ctx || field < 0 || field > 6) return fail(ctx, HST_EARG, "vvdz_to_field: bad field %d", field);
  int rc = check_m(ctx, m, "vvdz_to_field");
  if (rc == HST_OK) rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(hst::launch_vvdz_to_field(ctx->g, ctx->d, m - 1, field, ctx->stream));
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_buildrhs_prepare(hst_ctx* ctx, const double* ODE, double deltat, double time) {
  if (!ctx || !ODE || !(deltat > 0.0)) return fail(ctx, HST_EARG, "buildrhs_prepare: bad arguments");
  CK(cudaSetDevice(ctx->device));
  const hst_gpu_params& p = ctx->p;
  SubstepScalars sc = {};
  sc.ode0 = ODE[0];
  sc.ode1 = ODE[1];
  sc.ode2 = ODE[2];
  sc.deltat = deltat;
  sc.lambda = ODE[0] / deltat;
  sc.s2now = s2_of(p, time);
  sc.gsoft = (damping_active(p) && !p.damp_hard) ? 1.0 : 0.0;
  sc.damp_hard = 0;  // the mask is its own piece (hst_gpu_damping_mask)
  shear_shifts(ctx, time, &sc.sx_t, &sc.sz_t);
  CK(timed(ctx, HST_KC_RHS,
           [&] { return hst::launch_column(ctx->g, ctx->d, ctx->ps, sc, 1, 0, 4, ctx->stream); }));
  return HST_OK;
}

extern "C" int hst_gpu_buildrhs(hst_ctx* ctx, const double* ODE, int grp) {
  if (!ctx || !ODE || (grp != 1 && grp != 2)) return fail(ctx, HST_EARG, "buildrhs: bad arguments");
  int rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(hst::launch_buildrhs_group(ctx->g, ctx->d, ctx->ps, ODE[1], grp, ctx->stream));
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_damping_update(hst_ctx* ctx, double time) {
  if (!ctx) return HST_EARG;
  if (!damping_active(ctx->p) || !damping_update(ctx, time)) return HST_OK;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memcpy(ctx->h_gdamp, ctx->gdamp.data(), sizeof(double) * ctx->g.ncol);
  CK(cudaMemcpyAsync(ctx->d.gdamp, ctx->h_gdamp, sizeof(double) * ctx->g.ncol, cudaMemcpyHostToDevice, ctx->stream));
  return HST_OK;
}

extern "C" int hst_gpu_damping_mask(hst_ctx* ctx) {
  if (!ctx) return HST_EARG;
  if (!(ctx->p.damp_hard && damping_active(ctx->p))) return HST_OK;
  CK(cudaSetDevice(ctx->device));
  CK(hst::launch_damping_mask(ctx->g, ctx->d, ctx->stream));
  ctx->launches++;
  return HST_OK;
}

extern "C" int hst_gpu_shear_shift(hst_ctx* ctx, double dt_sub, double time) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  const hst_gpu_params& p = ctx->p;
  const double dgx = p.S * dt_sub, dgz = s2_integral(p, time, time + dt_sub);
  if (!p.exact_shift) {
    CK(hst::launch_shift_default(ctx->g, ctx->d, ctx->ps, dgx, dgz, ctx->stream));
    ctx->launches++;
    return HST_OK;
  }
  SubstepScalars sc = {};
  sc.dgx = dgx;
  sc.dgz = dgz;
  sc.yuni = p.ystretch <= 1.0e-10 ? 1 : 0;
  sc.ytile = p.ly * 32.0 / p.ny;
  shear_shifts(ctx, time, &sc.sx_t, &sc.sz_t);
  shear_shifts(ctx, time + dt_sub, &sc.sx_n, &sc.sz_n);
  CK(timed(ctx, HST_KC_COLUMN, [&] { return hst::launch_column(ctx->g, ctx->d, ctx->ps, sc, 1, 0, 3, ctx->stream); }));
  return HST_OK;
}

extern "C" int hst_gpu_linsolve(hst_ctx* ctx, double lambda, double time) {
  if (!ctx) return HST_EARG;
  CK(cudaSetDevice(ctx->device));
  SubstepScalars sc = {};
  sc.lambda = lambda;
  shear_shifts(ctx, time, &sc.sx_n, &sc.sz_n);
  CK(timed(ctx, HST_KC_COLUMN,
           [&] { return hst::launch_column(ctx->g, ctx->d, ctx->ps, sc, 0, !ctx->p.linear, 2, ctx->stream); }));
  return HST_OK;
}

extern "C" int hst_gpu_buffer_pointer(hst_ctx* ctx, int buf, void** dptr, size_t* bytes) {
  if (!ctx || buf < HST_BUF_VVDZ || buf > HST_BUF_VVDP || !dptr) return fail(ctx, HST_EARG, "buffer_pointer: bad buffer");
  int rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  *dptr = piece_buf(ctx, buf);
  if (bytes) *bytes = sizeof(double2) * 3 * piece_comp_elems(ctx->g, buf);
  return HST_OK;
}

static int buffer_copy(hst_ctx* ctx, int buf, int m, void* host, bool up) {
  if (!ctx || buf < HST_BUF_VVDZ || buf > HST_BUF_VVDP || !host) return fail(ctx, HST_EARG, "buffer copy: bad buffer");
  int rc = check_m(ctx, m, "buffer copy");
  if (rc == HST_OK) rc = ensure_pieces(ctx);
  if (rc != HST_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  const size_t ce = piece_comp_elems(ctx->g, buf);
  double2* dev = piece_buf(ctx, buf) + (size_t)(m - 1) * ce;
  if (up) CK(cudaMemcpyAsync(dev, host, sizeof(double2) * ce, cudaMemcpyHostToDevice, ctx->stream));
  else CK(cudaMemcpyAsync(host, dev, sizeof(double2) * ce, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HST_OK;
}
extern "C" int hst_gpu_buffer_upload(hst_ctx* ctx, int buf, int m, const double* host) {
  return buffer_copy(ctx, buf, m, const_cast<double*>(host), true);
}
extern "C" int hst_gpu_buffer_download(hst_ctx* ctx, int buf, int m, double* host) {
  return buffer_copy(ctx, buf, m, host, false);
}

// -------------------------------------------------- host address registry ----
static size_t id_bytes(const hst_ctx* ctx, int id) {
  if (id >= HST_V1 && id <= HST_RHS2) return sizeof(double2) * ctx->g.nf;
  if (id >= HST_ID_BUF(HST_BUF_VVDZ, 1) && id <= HST_ID_BUF(HST_BUF_VVDP, 3))
    return sizeof(double2) * piece_comp_elems(ctx->g, (id - HST_ID_BUF(0, 1)) / 3);
  return 0;
}

extern "C" int hst_gpu_register_host(hst_ctx* ctx, const void* host, size_t bytes, int id) {
  if (!ctx || !host) return HST_EARG;
  const size_t need = id_bytes(ctx, id);
  if (!need) return fail(ctx, HST_EARG, "register_host: unknown id %d", id);
  if (bytes != need)
    return fail(ctx, HST_EARG, "register_host: id %d holds %zu bytes, the host array %zu", id, need, bytes);
  const uintptr_t b = (uintptr_t)host;
  for (auto& r : ctx->host_ranges)
    if (b < r.base + r.bytes && r.base < b + bytes) {
      if (r.base == b && r.bytes == bytes) {  // the same array again: its id is replaced
        r.id = id;
        return HST_OK;
      }
      return fail(ctx, HST_EARG, "register_host: the array overlaps one registered as id %d", r.id);
    }
  ctx->host_ranges.push_back({b, bytes, id});
  return HST_OK;
}

extern "C" int hst_gpu_unregister_host(hst_ctx* ctx, const void* host) {
  if (!ctx) return HST_EARG;
  for (size_t k = 0; k < ctx->host_ranges.size(); ++k)
    if (ctx->host_ranges[k].base == (uintptr_t)host) {
      ctx->host_ranges.erase(ctx->host_ranges.begin() + (long)k);
      return HST_OK;
    }
  return fail(ctx, HST_EARG, "unregister_host: the address is not registered");
}

extern "C" int hst_gpu_host_id(const hst_ctx* ctx, const void* host) {
  if (!ctx) return HST_EARG;
  for (const auto& r : ctx->host_ranges)
    if (r.base == (uintptr_t)host) return r.id;
  return HST_EARG;
}

static int resolve(hst_ctx* ctx, const void* host, bool fields_only, const char* what) {
  const int id = hst_gpu_host_id(ctx, host);
  if (id < 0 || (fields_only && id > HST_RHS2))
    return fail(ctx, HST_EARG, "%s: the host array at %p is not registered%s", what, host,
                fields_only ? " as a field" : "");
  return id;
}

extern "C" int hst_gpu_upload_host(hst_ctx* ctx, const void* host) {
  if (!ctx) return HST_EARG;
  const int id = resolve(ctx, host, false, "upload_host");
  if (id < 0) return id;
  if (id <= HST_RHS2) return hst_gpu_upload(ctx, id, static_cast<const double*>(host));
  const int k = id - HST_ID_BUF(0, 1);
  return hst_gpu_buffer_upload(ctx, k / 3, k % 3 + 1, static_cast<const double*>(host));
}

extern "C" int hst_gpu_download_host(hst_ctx* ctx, void* host) {
  if (!ctx) return HST_EARG;
  const int id = resolve(ctx, host, false, "download_host");
  if (id < 0) return id;
  if (id <= HST_RHS2) return hst_gpu_download(ctx, id, static_cast<double*>(host));
  const int k = id - HST_ID_BUF(0, 1);
  return hst_gpu_buffer_download(ctx, k / 3, k % 3 + 1, static_cast<double*>(host));
}

extern "C" int hst_gpu_line_solve_host(hst_ctx* ctx, int sys, double lambda, const void* src, void* dst, int has_shift,
                                       double shift_x, double shift_z, double time) {
  if (!ctx) return HST_EARG;
  const int a = resolve(ctx, src, true, "line_solve_host src");
  if (a < 0) return a;
  const int b = resolve(ctx, dst, true, "line_solve_host dst");
  if (b < 0) return b;
  return hst_gpu_line_solve(ctx, sys, lambda, a, b, has_shift, shift_x, shift_z, time);
}

extern "C" int hst_gpu_fill_ghosts_host(hst_ctx* ctx, void* field, double shift_x, double shift_z) {
  if (!ctx) return HST_EARG;
  const int a = resolve(ctx, field, true, "fill_ghosts_host");
  if (a < 0) return a;
  return hst_gpu_fill_ghosts(ctx, a, shift_x, shift_z);
}

extern "C" int hst_gpu_vvdz_to_field_host(hst_ctx* ctx, void* field, int m) {
  if (!ctx) return HST_EARG;
  const int a = resolve(ctx, field, true, "vvdz_to_field_host");
  if (a < 0) return a;
  return hst_gpu_vvdz_to_field(ctx, a, m);
}
