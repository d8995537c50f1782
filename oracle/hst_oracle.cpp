// hst oracle: CPU FP64 restatement of the hst substep.  TEST INFRASTRUCTURE
// ONLY (the parity checker); see hst_oracle.h.  Citations are file:line in
// davecats/homogenenousShearTurbulence.
//
// Arithmetic follows the reference's gfortran build: no FMA contraction
// (compiled with -ffp-contract=off), complex multiplication by the textbook
// formula, integer powers by binary exponentiation (libgcc __powidf2, which
// gfortran calls for x**n with a variable n), left-to-right evaluation of
// products and sums as written in the Fortran.
#include "hst_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.141592653589793;
const double TWOPI = 6.283185307179586;

struct cx {
  double re, im;
};
inline cx C(double r, double i) { return cx{r, i}; }
inline cx operator+(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
inline cx operator-(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
inline cx operator-(cx a) { return C(-a.re, -a.im); }
inline cx operator*(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline cx operator*(double s, cx a) { return C(s * a.re, s * a.im); }
inline cx operator*(cx a, double s) { return C(a.re * s, a.im * s); }
inline cx operator/(cx a, double s) { return C(a.re / s, a.im / s); }
inline cx conj(cx a) { return C(a.re, -a.im); }
// complex division with range reduction (Smith), as gfortran's complex divide
inline cx cdiv(cx a, cx b) {
  if (std::fabs(b.re) >= std::fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return C((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  } else {
    double r = b.re / b.im, d = b.re * r + b.im;
    return C((a.re * r + a.im) / d, (a.im * r - a.re) / d);
  }
}
inline cx cexpi(double x) { return C(std::cos(x), std::sin(x)); }  // exp(dcmplx(0, x))

// x**n for a variable integer n: libgcc __powidf2 (binary exponentiation)
inline double powi(double x, int m) {
  unsigned n = m < 0 ? -m : m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

// Fortran MODULO for reals
inline double fmodulo(double a, double p) {
  double r = std::fmod(a, p);
  if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r += p;
  return r;
}
inline int imodulo(int a, int p) {
  int r = a % p;
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  return r;
}

// ---------------------------------------------------------------- FFT ----
// Unnormalised complex DFT, Stockham autosort, radices 4, 2, 3, 5.
// forward: exp(-2 pi i j k / N), backward: exp(+2 pi i j k / N) (FFTW's
// FFTW_FORWARD / FFTW_BACKWARD, src/hst_fft.f90:98-104).
struct FFTPlan {
  int N = 0;
  std::vector<int> radix;
  std::vector<cx> tw;  // exp(-2 pi i k / N)
  void init(int n) {
    N = n;
    radix.clear();
    int m = n;
    while (m % 4 == 0) { radix.push_back(4); m /= 4; }
    while (m % 2 == 0) { radix.push_back(2); m /= 2; }
    while (m % 3 == 0) { radix.push_back(3); m /= 3; }
    while (m % 5 == 0) { radix.push_back(5); m /= 5; }
    if (m != 1) { fprintf(stderr, "oracle FFT: unsupported length %d\n", n); abort(); }
    tw.resize(n);
    for (int k = 0; k < n; ++k) {
      long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
      tw[k] = C((double)cosl(a), (double)sinl(a));
    }
  }
  // in-place transform of data[0..N-1] (work: N scratch)
  void exec(cx* data, cx* work, int sign) const {
    cx* in = data;
    cx* out = work;
    int Ns = 1;
    const int L = N;
    for (int R : radix) {
      const int nb = L / R;
      const int tstride = L / (Ns * R);
      for (int j = 0; j < nb; ++j) {
        int k = j % Ns;
        cx v[5];
        for (int r = 0; r < R; ++r) {
          cx x = in[j + r * nb];
          int e = (k * r * tstride) % L;
          cx w = tw[e];
          if (sign > 0) w = conj(w);
          v[r] = (r == 0) ? x : x * w;
        }
        cx o[5];
        if (R == 2) {
          o[0] = v[0] + v[1];
          o[1] = v[0] - v[1];
        } else if (R == 4) {
          cx a0 = v[0] + v[2], a1 = v[0] - v[2], a2 = v[1] + v[3], a3 = v[1] - v[3];
          // multiply a3 by -i (forward) or +i (backward)
          cx a3r = sign < 0 ? C(a3.im, -a3.re) : C(-a3.im, a3.re);
          o[0] = a0 + a2;
          o[2] = a0 - a2;
          o[1] = a1 + a3r;
          o[3] = a1 - a3r;
        } else {
          for (int q = 0; q < R; ++q) {
            cx s = C(0, 0);
            for (int r = 0; r < R; ++r) {
              int e = ((q * r) % R) * (L / R);
              cx w = tw[e];
              if (sign > 0) w = conj(w);
              s = s + v[r] * w;
            }
            o[q] = s;
          }
        }
        int base = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; ++r) out[base + r * Ns] = o[r];
      }
      std::swap(in, out);
      Ns *= R;
    }
    if (in != data) std::memcpy(data, in, sizeof(cx) * N);
  }
};

}  // namespace

// ------------------------------------------------------------ the sim ----
struct ora_sim {
  ora_params p;
  // derived (src/hst_input.f90:94-102)
  int nx, ny, nz, nxd, nzd, nxB, nzT, rows;
  double ni, lx, lz, dx, dy, dz, factor, dt_fixed;
  double time, deltat, cfl;
  long istep;
  // grids (src/hst_setup.f90:42-71)
  std::vector<double> y, dyl, fy, der, k2, gdamp;
  std::vector<int> izd, inlayer;
  double theta_last;
  int ncol_damped = 0;  // damped columns (src/hst_damping.f90:42)
  // fields
  long nf;
  std::vector<cx> F[7];  // V1 V2 V3 old1 old2 rhs1 rhs2
  // transform buffers (src/hst_fft.f90:226-227)
  std::vector<cx> VVdz, VVdx, VVdp;
  FFTPlan pz, px;
  double RK[3][3];

  inline long fidx(int iy, int iz, int ix) const {
    return (long)(iy + 2) + (long)rows * ((long)(iz + nz) + (long)nzT * ix);
  }
  inline cx& f(int id, int iy, int iz, int ix) { return F[id][fidx(iy, iz, ix)]; }
  inline double D(int iy, int n, int j) const {  // der(iy, n, j)
    return der[(size_t)iy + (size_t)ny * ((size_t)n + 4 * (size_t)(j + 2))];
  }
  inline cx& vvdz(int k, int ix, int iy, int m) {  // VVdz(k+1, ix+1, iy, m+1), k 0-based
    return VVdz[(size_t)k + (size_t)nzd * ((size_t)ix + (size_t)nxB * ((size_t)(iy + 2) + (size_t)rows * m))];
  }
  inline cx* vvdx_line(int kz, int iy, int m) {  // VVdx(:, kz+1, iy, m+1)
    return &VVdx[(size_t)(nxd + 1) * ((size_t)kz + (size_t)nzd * ((size_t)(iy + 2) + (size_t)rows * m))];
  }
  inline cx* vvdp_line(int kz, int iy, int m) {
    return &VVdp[(size_t)(nxd + 1) * ((size_t)kz + (size_t)nzd * ((size_t)(iy + 2) + (size_t)rows * m))];
  }
};

extern "C" {

void ora_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void ora_default_params(ora_params* p) {
  // src/hst_input.f90:26-42
  std::memset(p, 0, sizeof(*p));
  p->nx = 63; p->ny = 128; p->nz = 63;
  p->ly = 2.0; p->alfa0 = 2.0 * PI / 3.0; p->beta0 = 2.0 * PI; p->ystretch = 0.0;
  p->re = 1000.0; p->S = 1.0; p->linear = 0; p->exact_shift = 0;
  p->sl_period = 1.0; p->sl_delta = 0.02; p->sl_bodyforce = 1;
  p->deltat = 0.0; p->cflmax = 1.0; p->t_max = 100.0; p->nstep = 1000000;
  p->time = 0.0; p->time_from_restart = 0;
  p->restart_from_file = 1;
  std::strcpy(p->restart_file, "Dati.cart.out");
  std::strcpy(p->initial_condition, "random");
  p->amplitude = 1.0e-3; p->seed = 1; p->kpeak = 4.0;
  p->damp_norm = 2.0; p->damp_follow = 1;
  p->tg_amplitude = 1.0; p->tg_mode = 1;
}

// ------------------------------------------------------ deck reader ----
// A reader for the namelist subset the decks use (src/hst_input.f90:19-23, 44-91).
static std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
static bool parse_bool(const std::string& v) {
  std::string s = lower(v);
  return s.find(".true.") != std::string::npos || s == "t" || s == ".t." || s == "true";
}
static double parse_real(const std::string& v) {
  std::string s = v;
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  return std::strtod(s.c_str(), nullptr);
}
static std::string parse_str(const std::string& v) {
  std::string s = v;
  size_t a = s.find_first_of("'\"");
  if (a == std::string::npos) return s;
  size_t b = s.find(s[a], a + 1);
  return s.substr(a + 1, b - a - 1);
}

int ora_read_deck(const char* path, ora_params* p) {
  ora_default_params(p);
  FILE* fp = std::fopen(path, "r");
  if (!fp) return 1;
  std::string text, line;
  char buf[4096];
  while (std::fgets(buf, sizeof buf, fp)) {
    line = buf;
    // strip comments (outside quotes)
    bool q = false;
    for (size_t i = 0; i < line.size(); ++i) {
      if (line[i] == '\'' || line[i] == '"') q = !q;
      if (line[i] == '!' && !q) { line = line.substr(0, i); break; }
    }
    text += line + "\n";
  }
  std::fclose(fp);
  // tokens key = value separated by commas/newlines inside &group ... /
  size_t pos = 0;
  while ((pos = text.find('&', pos)) != std::string::npos) {
    size_t end = text.find('/', pos);
    if (end == std::string::npos) break;
    std::string body = text.substr(pos + 1, end - pos - 1);
    // skip group name
    size_t sp = body.find_first_of(" \t\n");
    if (sp == std::string::npos) { pos = end + 1; continue; }
    body = body.substr(sp);
    // split on '=' : key before, value up to next comma that precedes a key
    std::vector<std::pair<std::string, std::string>> kv;
    size_t i = 0;
    while (i < body.size()) {
      size_t eq = body.find('=', i);
      if (eq == std::string::npos) break;
      std::string key = body.substr(i, eq - i);
      // key: last identifier
      size_t k0 = key.find_last_not_of(" \t\n,");
      if (k0 == std::string::npos) break;
      key = key.substr(0, k0 + 1);
      size_t k1 = key.find_last_of(" \t\n,");
      if (k1 != std::string::npos) key = key.substr(k1 + 1);
      // value: up to the next ',' or newline outside quotes
      size_t j = eq + 1;
      bool inq = false;
      while (j < body.size()) {
        char c = body[j];
        if (c == '\'' || c == '"') inq = !inq;
        if (!inq && (c == ',' || c == '\n')) break;
        ++j;
      }
      std::string val = body.substr(eq + 1, j - eq - 1);
      kv.push_back({lower(key), val});
      i = j + 1;
    }
    for (auto& e : kv) {
      const std::string& k = e.first;
      const std::string& v = e.second;
#define R_(name) else if (k == #name) p->name = parse_real(v);
#define I_(name) else if (k == #name) p->name = (int)std::lround(parse_real(v));
#define B_(name) else if (k == #name) p->name = parse_bool(v) ? 1 : 0;
      if (false) {}
      I_(nx) I_(ny) I_(nz) R_(alfa0) R_(beta0) R_(ly) R_(ystretch)
      R_(re) R_(S) B_(linear) B_(exact_shift) R_(s2_mean) R_(s2_amplitude) R_(s2_period) R_(s2_start)
      R_(sl_amplitude) R_(sl_period) R_(sl_delta) R_(sl_start) B_(sl_bodyforce) B_(sl_ramp)
      R_(deltat) R_(cflmax) R_(t_max) R_(time) B_(time_from_restart) B_(restart_from_file)
      R_(amplitude) R_(kpeak) I_(seed) R_(tg_amplitude) I_(tg_mode)
      R_(damp_kpar) R_(damp_kperp) R_(damp_rate) R_(damp_edge) R_(damp_norm) R_(damp_angle)
      B_(damp_hard) B_(damp_mean) B_(damp_follow)
      else if (k == "s") p->S = parse_real(v);
      else if (k == "nstep") p->nstep = std::lround(parse_real(v));
      else if (k == "restart_file") std::snprintf(p->restart_file, sizeof p->restart_file, "%s", parse_str(v).c_str());
      else if (k == "initial_condition") std::snprintf(p->initial_condition, sizeof p->initial_condition, "%s", parse_str(v).c_str());
#undef R_
#undef I_
#undef B_
    }
    pos = end + 1;
  }
  return 0;
}

// ----------------------------------------------------------- set-up ----
// fft_fit: src/hst_input.f90:107-115
static bool fft_fit(int n) {
  int j = n;
  while (j % 2 == 0) j /= 2;
  return j == 1 || j == 3;
}

// ymap: src/hst_setup.f90:80-89
static double ymap(double xi, double ystretch) {
  if (ystretch <= 1.0e-10) return xi;
  if (xi <= 0.5) return 0.5 * std::tanh(2.0 * ystretch * xi) / std::tanh(ystretch);
  return 0.5 * (2.0 + std::tanh(2.0 * ystretch * (xi - 1.0)) / std::tanh(ystretch));
}

// solve5: src/hst_derivatives.f90:59-79 (dense 5x5, partial pivoting)
static void solve5(const double Min[5][5], const double bin[5], double x[5]) {
  double M[5][5], b[5];
  std::memcpy(M, Min, sizeof M);
  std::memcpy(b, bin, sizeof b);
  for (int i = 0; i <= 4; ++i) {
    int p = i;
    double best = std::fabs(M[i][i]);
    for (int r = i + 1; r <= 4; ++r)
      if (std::fabs(M[r][i]) > best) { best = std::fabs(M[r][i]); p = r; }
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

// setup_derivatives: src/hst_derivatives.f90:30-56
static void setup_derivatives(ora_sim* s) {
  int ny = s->ny;
  s->der.assign((size_t)ny * 4 * 5, 0.0);
  auto Y = [&](int iy) { return s->y[iy + 2]; };
  auto setd = [&](int iy, int n, const double* v) {
    for (int j = 0; j < 5; ++j) s->der[(size_t)iy + (size_t)ny * ((size_t)n + 4 * (size_t)j)] = v[j];
  };
  for (int iy = 0; iy < ny; ++iy) {
    double dyj[5];
    for (int j = -2; j <= 2; ++j) dyj[j + 2] = Y(iy + j) - Y(iy);
    double M[5][5], t[5], d3[5], d0[5], d2[5], d1[5];
    // D4: exact fourth derivative of y^4
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) M[i][j] = powi(dyj[j], 4 - i);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    t[0] = 24.0;
    solve5(M, t, d3);
    // D0
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) {
        int c = (5 - i) * (6 - i) * (7 - i) * (8 - i);
        M[i][j] = (double)c * powi(dyj[j], 4 - i);
      }
    for (int i = 0; i <= 4; ++i) {
      double sm = 0.0;
      for (int j = 0; j < 5; ++j) sm = sm + d3[j] * powi(dyj[j], 8 - i);
      t[i] = sm;
    }
    solve5(M, t, d0);
    // D2 and D1 consistent with D0
    for (int i = 0; i <= 4; ++i)
      for (int j = 0; j <= 4; ++j) M[i][j] = powi(dyj[j], 4 - i);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    for (int i = 0; i <= 2; ++i) {
      double sm = 0.0;
      for (int j = 0; j < 5; ++j) sm = sm + d0[j] * (double)(4 - i) * (double)(3 - i) * powi(dyj[j], 2 - i);
      t[i] = sm;
    }
    solve5(M, t, d2);
    for (int i = 0; i < 5; ++i) t[i] = 0.0;
    for (int i = 0; i <= 3; ++i) {
      double sm = 0.0;
      for (int j = 0; j < 5; ++j) sm = sm + d0[j] * (double)(4 - i) * powi(dyj[j], 3 - i);
      t[i] = sm;
    }
    solve5(M, t, d1);
    setd(iy, 3, d3);
    setd(iy, 0, d0);
    setd(iy, 2, d2);
    setd(iy, 1, d1);
  }
}

// S2(t), its integral, gamma_y, the wrap displacements:
// src/hst_derivatives.f90:85-128
double ora_s2_of(const ora_sim* s, double t) {
  const ora_params& p = s->p;
  if ((p.s2_amplitude == 0.0 && p.s2_mean == 0.0) || t < p.s2_start) return 0.0;
  if (p.s2_period > 0.0) return p.s2_mean + p.s2_amplitude * std::sin(TWOPI / p.s2_period * (t - p.s2_start));
  return p.s2_mean + p.s2_amplitude;
}
double ora_s2_integral(const ora_sim* s, double t1, double t2) {
  const ora_params& p = s->p;
  if ((p.s2_amplitude == 0.0 && p.s2_mean == 0.0) || t2 <= p.s2_start) return 0.0;
  double a = std::max(t1, p.s2_start), b = t2;
  if (p.s2_period > 0.0) {
    double omega = TWOPI / p.s2_period;
    return p.s2_mean * (b - a) + p.s2_amplitude / omega * (std::cos(omega * (a - p.s2_start)) - std::cos(omega * (b - p.s2_start)));
  }
  return (p.s2_mean + p.s2_amplitude) * (b - a);
}
static double gamma_y_of(const ora_sim* s, double t) { return ora_s2_integral(s, s->p.s2_start, t); }
void ora_shear_shifts(const ora_sim* s, double t, double* sx, double* sz) {
  *sx = fmodulo(s->p.S * t * s->p.ly, s->lx);
  *sz = fmodulo(gamma_y_of(s, t) * s->p.ly, s->lz);
}

// damping: src/hst_damping.f90:46-133
int ora_damping_active(const ora_sim* s) {
  const ora_params& p = s->p;
  return p.damp_kpar > 0.0 && p.damp_kperp > 0.0 && (p.damp_hard || p.damp_rate > 0.0);
}
static double damping_soft_factor(const ora_sim* s) {
  return (ora_damping_active(s) && !s->p.damp_hard) ? 1.0 : 0.0;
}
static double damping_theta(const ora_sim* s, double t) {
  if (s->p.damp_follow) return std::atan2(ora_s2_of(s, t), s->p.S);
  return s->p.damp_angle * PI / 180.0;
}
void ora_damping_update(ora_sim* s, double t) {
  const ora_params& p = s->p;
  double theta = damping_theta(s, t);
  if (theta == s->theta_last) return;
  s->theta_last = theta;
  double c = std::cos(theta), sn = std::sin(theta);
  int n = 0;
  for (int ix = 0; ix <= s->nx; ++ix) {
    double kx = p.alfa0 * ix;
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      double kz = p.beta0 * iz;
      double kpar = kx * c + kz * sn;
      double kperp = -kx * sn + kz * c;
      double r = std::pow(std::pow(std::fabs(kpar) / p.damp_kpar, p.damp_norm) + std::pow(std::fabs(kperp) / p.damp_kperp, p.damp_norm), 1.0 / p.damp_norm);
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
      s->gdamp[(size_t)(iz + s->nz) + (size_t)s->nzT * ix] = g;
      if (g > 0.0) n = n + 1;
    }
  }
  s->ncol_damped = n;
}
void ora_damping_mask(ora_sim* s) {
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      if (s->gdamp[(size_t)(iz + s->nz) + (size_t)s->nzT * ix] > 0.0)
        for (int iy = 0; iy < s->ny; ++iy) {
          s->f(ORA_RHS1, iy, iz, ix) = C(0, 0);
          s->f(ORA_RHS2, iy, iz, ix) = C(0, 0);
          s->f(ORA_OLD1, iy, iz, ix) = C(0, 0);
          s->f(ORA_OLD2, iy, iz, ix) = C(0, 0);
        }
    }
}

// Stokes layer (src/hst_stokes.f90:181-261): kept only so that the
// stretched-grid golden field small_stokes.fld pins the oracle.
static bool stokes_active(const ora_sim* s) { return s->p.sl_amplitude != 0.0; }
static double sl_ramp(const ora_sim* s, double t) {
  const ora_params& p = s->p;
  if (t < p.sl_start) return 0.0;
  if (p.sl_ramp) {
    double tau = std::min((t - p.sl_start) / p.sl_period, 1.0);
    return 3.0 * (tau * tau) - 2.0 * (tau * tau * tau);
  }
  return 1.0;
}
static double stokes_profile(const ora_sim* s, double yy, double t) {
  const ora_params& p = s->p;
  double omega = TWOPI / p.sl_period;
  double e = (yy - 0.5 * p.ly) / p.sl_delta;
  double sv = std::sqrt(e * e + 0.1 * 0.1);
  return sl_ramp(s, t) * p.sl_amplitude * std::exp(-sv) * std::cos(omega * (t - p.sl_start) - sv);
}
static double stokes_force_at(const ora_sim* s, double yy, double t) {
  const ora_params& p = s->p;
  double omega = TWOPI / p.sl_period;
  double eta = yy - 0.5 * p.ly;
  double e = eta / p.sl_delta;
  double sv = std::sqrt(e * e + 0.1 * 0.1);
  double s1 = (eta / (p.sl_delta * p.sl_delta)) / sv;
  double s2 = (0.1 * 0.1 / (p.sl_delta * p.sl_delta)) / (sv * sv * sv);
  double theta = omega * (t - p.sl_start) - sv;
  return sl_ramp(s, t) * p.sl_amplitude * std::exp(-sv) *
         ((2.0 * s->ni * s1 * s1 - omega) * std::sin(theta) - s->ni * s2 * (std::sin(theta) - std::cos(theta)));
}
static void stokes_force(ora_sim* s, double t) {
  if (!(stokes_active(s) && s->p.sl_bodyforce)) return;
  int ny = s->ny;
  for (int iy = 0; iy < ny; ++iy) s->fy[iy + 2] = stokes_force_at(s, s->y[iy + 2], t);
  s->fy[0] = s->fy[ny - 2 + 2];
  s->fy[1] = s->fy[ny - 1 + 2];
  s->fy[ny + 2] = s->fy[2];
  s->fy[ny + 3] = s->fy[3];
}
static void stokes_apply(ora_sim* s) {
  if (!stokes_active(s)) return;
  bool whole = (!s->p.sl_bodyforce) || (s->time - s->p.sl_start <= 2.0 * s->p.sl_period);
  for (int iy = 0; iy < s->ny; ++iy)
    if (whole || iy == 0 || iy == s->ny - 1) s->f(ORA_V3, iy, 0, 0) = C(stokes_profile(s, s->y[iy + 2], s->time), 0.0);
}

ora_sim* ora_create(const ora_params* pin) {
  ora_sim* s = new ora_sim();
  s->p = *pin;
  const ora_params& p = s->p;
  s->nx = p.nx; s->ny = p.ny; s->nz = p.nz;
  // derived quantities: src/hst_input.f90:94-102
  s->ni = 1.0 / p.re;
  s->dt_fixed = p.deltat;
  s->lx = 2.0 * PI / p.alfa0;
  s->lz = 2.0 * PI / p.beta0;
  s->nxd = 3 * (p.nx + 1) / 2;
  while (!fft_fit(s->nxd)) s->nxd++;
  s->nzd = 3 * p.nz;
  while (!fft_fit(s->nzd)) s->nzd++;
  s->dx = PI / (p.alfa0 * s->nxd);
  s->dz = 2.0 * PI / (p.beta0 * s->nzd);
  s->dy = p.ly / p.ny;
  s->factor = 1.0 / (2.0 * s->nxd * s->nzd);
  s->nxB = p.nx + 1;
  s->nzT = 2 * p.nz + 1;
  s->rows = p.ny + 4;
  s->time = p.time;
  s->deltat = p.deltat;
  s->cfl = 0.0;
  s->istep = 0;
  s->theta_last = -1.0e308;
  // RK_rai: src/hst_params.f90:108-111, column i = substep
  double rk[9] = {120.0 / 32.0, 2.0, 0.0, 120.0 / 8.0, 50.0 / 8.0, 34.0 / 8.0, 120.0 / 20.0, 90.0 / 20.0, 50.0 / 20.0};
  for (int i = 0; i < 3; ++i)
    for (int r = 0; r < 3; ++r) s->RK[i][r] = rk[3 * i + r];
  // grids: src/hst_setup.f90:42-71
  int ny = p.ny;
  s->y.resize(ny + 4);
  for (int iy = -2; iy <= ny + 1; ++iy) {
    int mo = imodulo(iy, ny);
    s->y[iy + 2] = p.ly * ymap((double)mo / ny, p.ystretch) + p.ly * (double)((iy - mo) / ny);
  }
  s->dyl.resize(ny);
  for (int iy = 0; iy < ny; ++iy) s->dyl[iy] = 0.5 * (s->y[iy + 3] - s->y[iy + 1]);
  s->fy.assign(ny + 4, 0.0);
  s->inlayer.assign(ny, 0);
  s->izd.resize(s->nzT);
  for (int iz = -p.nz; iz <= p.nz; ++iz) s->izd[iz + p.nz] = iz >= 0 ? iz : s->nzd + iz;
  s->k2.resize((size_t)s->nzT * s->nxB);
  for (int ix = 0; ix <= p.nx; ++ix)
    for (int iz = -p.nz; iz <= p.nz; ++iz) {
      double a = p.alfa0 * ix, b = p.beta0 * iz;
      s->k2[(size_t)(iz + p.nz) + (size_t)s->nzT * ix] = a * a + b * b;
    }
  s->nf = (long)s->rows * s->nzT * s->nxB;
  for (int i = 0; i < 7; ++i) s->F[i].assign(s->nf, C(0, 0));
  s->VVdz.assign((size_t)s->nzd * s->nxB * s->rows * 3, C(0, 0));
  s->VVdx.assign((size_t)(s->nxd + 1) * s->nzd * s->rows * 3, C(0, 0));
  s->VVdp.assign((size_t)(s->nxd + 1) * s->nzd * s->rows * 3, C(0, 0));
  s->pz.init(s->nzd);
  s->px.init(2 * s->nxd);
  setup_derivatives(s);
  // damping_setup: src/hst_damping.f90:68-78
  s->gdamp.assign((size_t)s->nzT * s->nxB, 0.0);
  if (ora_damping_active(s)) ora_damping_update(s, s->time);
  // stokes_setup: src/hst_stokes.f90:222-231
  if (stokes_active(s))
    for (int iy = 0; iy < ny; ++iy)
      if (std::fabs(s->y[iy + 2] - 0.5 * p.ly) < 8.0 * p.sl_delta) s->inlayer[iy] = 1;
  return s;
}
void ora_destroy(ora_sim* s) { delete s; }

int ora_nxd(const ora_sim* s) { return s->nxd; }
int ora_nzd(const ora_sim* s) { return s->nzd; }
long ora_field_size(const ora_sim* s) { return s->nf; }
double* ora_field(ora_sim* s, int id) { return reinterpret_cast<double*>(s->F[id].data()); }
const double* ora_der(const ora_sim* s) { return s->der.data(); }
const double* ora_y(const ora_sim* s) { return s->y.data(); }
const double* ora_dyl(const ora_sim* s) { return s->dyl.data(); }
double* ora_gdamp(ora_sim* s) { return s->gdamp.data(); }
double* ora_products(ora_sim* s) { return reinterpret_cast<double*>(s->VVdp.data()); }
double* ora_rvvdx(ora_sim* s) { return reinterpret_cast<double*>(s->VVdx.data()); }
double* ora_vvdz(ora_sim* s) { return reinterpret_cast<double*>(s->VVdz.data()); }
double ora_get_time(const ora_sim* s) { return s->time; }
void ora_set_time(ora_sim* s, double t) { s->time = t; }
double ora_get_deltat(const ora_sim* s) { return s->deltat; }
void ora_set_deltat(ora_sim* s, double dt) { s->deltat = dt; }
double ora_get_cfl(const ora_sim* s) { return s->cfl; }
void ora_set_physics(ora_sim* s, double S, double ni, int linear) {
  s->p.S = S;
  s->ni = ni;
  s->p.linear = linear;
}

// ---------------------------------------------------- initial field ----
// uniform_from_key: src/hst_initial.f90:139-159
double ora_uniform_from_key(int seed, int component, int iy, int iz, int ix) {
  const int64_t MASK32 = 4294967295LL, MIX_A = 2146121005LL, MIX_B = 2032289749LL;
  int64_t h = (int64_t)seed;
  h = h + 2654435761LL * (int64_t)component;
  h = h + 2246822519LL * (int64_t)iy;
  h = h + 3266489917LL * (int64_t)iz;
  h = h + 668265263LL * (int64_t)ix;
  h = h & MASK32;
  h = h ^ (h >> 16);
  h = (h * MIX_A) & MASK32;
  h = h ^ (h >> 13);
  h = (h * MIX_B) & MASK32;
  h = h ^ (h >> 16);
  return (double)h * (1.0 / 4294967296.0);
}

// potential: src/hst_initial.f90:113-133
static void potential(const ora_sim* s, int ix, int iz, int m, cx a[3]) {
  int jz = iz, jm = m;
  bool mirror = false;
  if (ix == 0 && (iz < 0 || (iz == 0 && m < 0))) { jz = -iz; jm = -m; mirror = true; }
  for (int c = 1; c <= 3; ++c) {
    double r = ora_uniform_from_key(s->p.seed, c, jm, jz, ix);
    double phase = TWOPI * ora_uniform_from_key(s->p.seed, c + 3, jm, jz, ix);
    a[c - 1] = r * cexpi(phase);
    if (mirror) a[c - 1] = conj(a[c - 1]);
  }
}

// generate_initial_field: src/hst_initial.f90:27-67; Taylor-Green :76-108
void ora_generate_initial_field(ora_sim* s) {
  const ora_params& p = s->p;
  for (int c = 0; c < 3; ++c) s->F[c].assign(s->nf, C(0, 0));
  const cx I = C(0, 1);
  if (std::strncmp(p.initial_condition, "taylor_green", 12) == 0) {
    double ky = 2.0 * PI * p.tg_mode / p.ly;
    int ix = p.tg_mode;
    for (int iz = -p.tg_mode; iz <= p.tg_mode; iz += 2 * p.tg_mode)
      for (int iy = -2; iy <= s->ny + 1; ++iy) {
        s->f(0, iy, iz, ix) = (-I * p.tg_amplitude) * std::cos(ky * s->y[iy + 2]) / 4.0;
        s->f(1, iy, iz, ix) = C(-p.tg_amplitude * std::sin(ky * s->y[iy + 2]) / 4.0, 0.0);
      }
    return;
  }
  int mmax = s->ny / 3;
  for (int ix = 0; ix <= s->nx; ++ix) {
    double kx = p.alfa0 * ix;
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      double kz = p.beta0 * iz;
      if (ix == 0 && iz == 0) continue;
      for (int m = -mmax; m <= mmax; ++m) {
        double ky = 2.0 * PI * m / p.ly;
        double k = std::sqrt(kx * kx + ky * ky + kz * kz);
        if (k == 0.0) continue;
        double q = k / p.kpeak;
        double env = (q * q) * std::exp(1.0 - q * q);
        if (env < 1.0e-8) continue;
        cx a[3];
        potential(s, ix, iz, m, a);
        double sc = p.amplitude * env;
        for (int c = 0; c < 3; ++c) a[c] = sc * a[c];
        cx u[3];
        u[0] = I * (ky * a[2] - kz * a[1]);
        u[1] = I * (kz * a[0] - kx * a[2]);
        u[2] = I * (kx * a[1] - ky * a[0]);
        for (int iy = -2; iy <= s->ny + 1; ++iy) {
          cx ph = cexpi(ky * s->y[iy + 2]);
          for (int c = 0; c < 3; ++c) s->f(c, iy, iz, ix) = s->f(c, iy, iz, ix) + u[c] * ph;
        }
      }
    }
  }
}

// ----------------------------------------------------- ghost rows ----
// wrap_rows: src/hst_mpi.f90:340-355 (npy = 1)
void ora_fill_ghosts(ora_sim* s, int id, double shift_x, double shift_z) {
  int ny = s->ny;
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      cx ph = cexpi(-(s->p.alfa0 * ix * shift_x + s->p.beta0 * iz * shift_z));
      s->f(id, ny, iz, ix) = s->f(id, 0, iz, ix) * ph;
      s->f(id, ny + 1, iz, ix) = s->f(id, 1, iz, ix) * ph;
      s->f(id, -1, iz, ix) = s->f(id, ny - 1, iz, ix) * conj(ph);
      s->f(id, -2, iz, ix) = s->f(id, ny - 2, iz, ix) * conj(ph);
    }
}
// fill_ghosts: src/hst_derivatives.f90:134-145
void ora_fill_ghosts_now(ora_sim* s, int id) {
  double sx, sz;
  ora_shear_shifts(s, s->time, &sx, &sz);
  ora_fill_ghosts(s, id, sx, sz);
}

// ------------------------------------------------------ transforms ----
// assemble_vvdz + IFT + transpose + zero padding + RFT:
// src/hst_transforms.f90:33-90, src/hst_fft.f90:195-223
void ora_transform_to_physical(ora_sim* s) {
  const int nz = s->nz, nzd = s->nzd, nxd = s->nxd, rows = s->rows;
  // assemble_vvdz (:37-53)
#pragma omp parallel for collapse(2)
  for (int m = 0; m < 3; ++m)
    for (int iy = -2; iy <= s->ny + 1; ++iy)
      for (int ix = 0; ix <= s->nx; ++ix)
        for (int k = 1; k <= nzd; ++k) {
          cx v;
          if (k <= nz + 1) v = s->f(m, iy, k - 1, ix);
          else if (k <= nzd - nz) v = C(0, 0);
          else v = s->f(m, iy, k - nzd - 1, ix);
          s->vvdz(k - 1, ix, iy, m) = v;
        }
  // IFT(m): backward z transform in place
#pragma omp parallel
  {
    std::vector<cx> work(std::max(nzd, 2 * nxd));
    std::vector<cx> line(2 * nxd);
#pragma omp for collapse(2)
    for (int m = 0; m < 3; ++m)
      for (int iy = -2; iy <= s->ny + 1; ++iy)
        for (int ix = 0; ix <= s->nx; ++ix) s->pz.exec(&s->vvdz(0, ix, iy, m), work.data(), +1);
  }
  // transpose_zTOx (local), zero_vvdx_padding, RFT (c2r, FFTW semantics)
#pragma omp parallel
  {
    std::vector<cx> work(2 * nxd), line(2 * nxd);
#pragma omp for collapse(2)
    for (int m = 0; m < 3; ++m)
      for (int iy = -2; iy <= s->ny + 1; ++iy)
        for (int kz = 0; kz < nzd; ++kz) {
          cx* L = s->vvdx_line(kz, iy, m);
          for (int ix = 0; ix <= s->nx; ++ix) L[ix] = s->vvdz(kz, ix, iy, m);
          for (int ix = s->nx + 1; ix <= nxd; ++ix) L[ix] = C(0, 0);
          // c2r of length N = 2 nxd: Hermitian extension, imaginary parts of
          // the k = 0 and k = N/2 modes dropped
          const int N = 2 * nxd;
          line[0] = C(L[0].re, 0.0);
          line[nxd] = C(L[nxd].re, 0.0);
          for (int k = 1; k < nxd; ++k) {
            line[k] = L[k];
            line[N - k] = conj(L[k]);
          }
          s->px.exec(line.data(), work.data(), +1);
          double* r = reinterpret_cast<double*>(L);
          for (int j = 0; j < N; ++j) r[j] = line[j].re;
          r[N] = 0.0;
          r[N + 1] = 0.0;
        }
  }
  (void)rows;
}

// compute_cfl: src/hst_transforms.f90:163-179
double ora_compute_cfl(ora_sim* s) {
  const int nxd = s->nxd, nzd = s->nzd;
  double cfl = 0.0;
#pragma omp parallel for reduction(max : cfl)
  for (int iy = 0; iy < s->ny; ++iy)
    for (int kz = 0; kz < nzd; ++kz)
      for (int m = 0; m < 1; ++m) {
        const double* u = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 0));
        const double* v = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 1));
        const double* w = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 2));
        for (int j = 0; j < 2 * nxd; ++j) {
          double tmp = std::fabs(u[j]) / s->dx + std::fabs(v[j]) / s->dyl[iy] + std::fabs(w[j]) / s->dz;
          cfl = std::max(cfl, tmp);
        }
      }
  s->cfl = cfl;
  return cfl;
}

// build_products: src/hst_transforms.f90:97-121
void ora_build_products(ora_sim* s, int g) {
  const int nxd = s->nxd, nzd = s->nzd;
  const double factor = s->factor;
#pragma omp parallel for collapse(2)
  for (int iy = -2; iy <= s->ny + 1; ++iy)
    for (int kz = 0; kz < nzd; ++kz) {
      const double* U = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 0));
      const double* Vv = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 1));
      const double* W = reinterpret_cast<const double*>(s->vvdx_line(kz, iy, 2));
      double* P1 = reinterpret_cast<double*>(s->vvdp_line(kz, iy, 0));
      double* P2 = reinterpret_cast<double*>(s->vvdp_line(kz, iy, 1));
      double* P3 = reinterpret_cast<double*>(s->vvdp_line(kz, iy, 2));
      for (int k = 0; k < 2 * nxd; ++k) {
        double u = U[k], v = Vv[k], w = W[k];
        if (g == 1) {
          P1[k] = u * u * factor;
          P2[k] = v * v * factor;
          P3[k] = w * w * factor;
        } else {
          P1[k] = u * v * factor;
          P2[k] = v * w * factor;
          P3[k] = u * w * factor;
        }
      }
    }
}

// products_to_spectral: HFT (r2c) + transpose_xTOz + FFT (forward z):
// src/hst_transforms.f90:125-139, src/hst_fft.f90:181-193,225-237
void ora_products_to_spectral(ora_sim* s) {
  const int nxd = s->nxd, nzd = s->nzd;
#pragma omp parallel
  {
    std::vector<cx> work(std::max(nzd, 2 * nxd)), line(2 * nxd);
#pragma omp for collapse(2)
    for (int m = 0; m < 3; ++m)
      for (int iy = -2; iy <= s->ny + 1; ++iy)
        for (int kz = 0; kz < nzd; ++kz) {
          cx* L = s->vvdp_line(kz, iy, m);
          const double* r = reinterpret_cast<const double*>(L);
          const int N = 2 * nxd;
          for (int j = 0; j < N; ++j) line[j] = C(r[j], 0.0);
          s->px.exec(line.data(), work.data(), -1);
          for (int k = 0; k <= nxd; ++k) L[k] = line[k];
        }
#pragma omp for collapse(2)
    for (int m = 0; m < 3; ++m)
      for (int iy = -2; iy <= s->ny + 1; ++iy)
        for (int ix = 0; ix <= s->nx; ++ix) {
          for (int kz = 0; kz < nzd; ++kz) s->vvdz(kz, ix, iy, m) = s->vvdp_line(kz, iy, m)[ix];
          s->pz.exec(&s->vvdz(0, ix, iy, m), work.data(), -1);
        }
  }
}

// vvdz_to_field: src/hst_transforms.f90:142-157
void ora_vvdz_to_field(ora_sim* s, int m, double* outd) {
  cx* out = reinterpret_cast<cx*>(outd);
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iy = -2; iy <= s->ny + 1; ++iy)
      for (int iz = -s->nz; iz <= s->nz; ++iz) out[s->fidx(iy, iz, ix)] = s->vvdz(s->izd[iz + s->nz], ix, iy, m);
}

// ------------------------------------------------------- equations ----
// buildrhs_prepare: src/hst_equations.f90:92-141
void ora_buildrhs_prepare(ora_sim* s, const double* ODE) {
  const double s2now = ora_s2_of(s, s->time);
  const double gsoft = damping_soft_factor(s);
  stokes_force(s, s->time);
  const double ni = s->ni, S = s->p.S, deltat = s->deltat;
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      const size_t col = (size_t)(iz + s->nz) + (size_t)s->nzT * ix;
      const double kk = s->k2[col];
      const cx ialfa = C(0.0, ix * s->p.alfa0), ibeta = C(0.0, iz * s->p.beta0);
      for (int iy = 0; iy < s->ny; ++iy) {
        double g = gsoft * s->gdamp[col];
        cx unkn = C(0, 0), impl = C(0, 0), expl = C(0, 0);
        for (int j = -2; j <= 2; ++j) {
          double helm = s->D(iy, 2, j) - kk * s->D(iy, 0, j);
          double biharm = s->D(iy, 3, j) - 2.0 * kk * s->D(iy, 2, j) + kk * kk * s->D(iy, 0, j);
          unkn = unkn + helm * s->f(1, iy + j, iz, ix);
          impl = impl + (ni * biharm) * s->f(1, iy + j, iz, ix);
        }
        cx& r2 = s->f(ORA_RHS2, iy, iz, ix);
        cx& o2 = s->f(ORA_OLD2, iy, iz, ix);
        r2 = ((ODE[0] * unkn) / deltat + impl) - ODE[2] * o2 - (ODE[1] * g) * unkn;
        o2 = (-g) * unkn;
        unkn = C(0, 0);
        impl = C(0, 0);
        expl = C(0, 0);
        double force = 0.0;
        for (int j = -2; j <= 2; ++j) {
          double helm = s->D(iy, 2, j) - kk * s->D(iy, 0, j);
          if (ix == 0 && iz == 0) {
            cx f = C(s->f(0, iy + j, iz, ix).re, s->f(2, iy + j, iz, ix).re);
            unkn = unkn + s->D(iy, 0, j) * f;
            impl = impl + (ni * s->D(iy, 2, j)) * f;
            force = force + s->D(iy, 0, j) * s->fy[iy + j + 2];
          } else {
            cx f = ibeta * s->f(0, iy + j, iz, ix) - ialfa * s->f(2, iy + j, iz, ix);
            unkn = unkn + s->D(iy, 0, j) * f;
            impl = impl + (ni * helm) * f;
          }
          expl = expl + ((s2now * ialfa - S * ibeta) * s->D(iy, 0, j)) * s->f(1, iy + j, iz, ix);
        }
        if (ix == 0 && iz == 0) expl = expl + C(0.0, force);
        expl = expl - g * unkn;
        cx& r1 = s->f(ORA_RHS1, iy, iz, ix);
        cx& o1 = s->f(ORA_OLD1, iy, iz, ix);
        r1 = (((ODE[0] * unkn) / deltat + impl) - ODE[2] * o1) + ODE[1] * expl;
        o1 = expl;
      }
    }
}

// buildrhs: src/hst_equations.f90:151-213
void ora_buildrhs(ora_sim* s, const double* ODE, int g) {
  const bool no_mean_vw = stokes_active(s) && s->p.sl_bodyforce;
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      const size_t col = (size_t)(iz + s->nz) + (size_t)s->nzT * ix;
      const double kk = s->k2[col];
      const cx ialfa = C(0.0, ix * s->p.alfa0), ibeta = C(0.0, iz * s->p.beta0);
      const int kz = s->izd[iz + s->nz];
      for (int iy = 0; iy < s->ny; ++iy) {
        cx r1 = s->f(ORA_RHS1, iy, iz, ix), r2 = s->f(ORA_RHS2, iy, iz, ix);
        cx o1 = s->f(ORA_OLD1, iy, iz, ix), o2 = s->f(ORA_OLD2, iy, iz, ix);
        for (int p = 1; p <= 3; ++p) {
          int m = 3 * (g - 1) + p;
          cx d0 = C(0, 0), d1 = C(0, 0), d2 = C(0, 0);
          for (int j = -2; j <= 2; ++j) {
            cx q = s->vvdz(kz, ix, iy + j, p - 1);
            d0 = d0 + s->D(iy, 0, j) * q;
            d1 = d1 + s->D(iy, 1, j) * q;
            d2 = d2 + s->D(iy, 2, j) * q;
          }
          cx rhsu = C(0, 0), rhsw = C(0, 0), expl;
          switch (m) {
            case 1: rhsu = -(ialfa * d0); expl = (ialfa * ialfa) * d1; break;
            case 2: expl = kk * d1; break;
            case 3: rhsw = -(ibeta * d0); expl = (ibeta * ibeta) * d1; break;
            case 4: rhsu = -d1; expl = ialfa * d2 + (ialfa * kk) * d0; break;
            case 5:
              rhsw = -d1;
              if (no_mean_vw && ix == 0 && iz == 0) rhsw = C(0, 0);
              expl = ibeta * d2 + (ibeta * kk) * d0;
              break;
            default: rhsu = -(ibeta * d0); rhsw = -(ialfa * d0); expl = ((2.0 * ialfa) * ibeta) * d1; break;
          }
          r2 = r2 + ODE[1] * expl;
          o2 = o2 + expl;
          cx e;
          if (ix == 0 && iz == 0) e = C(rhsu.re, rhsw.re);
          else e = ibeta * rhsu - ialfa * rhsw;
          r1 = r1 + ODE[1] * e;
          o1 = o1 + e;
        }
        s->f(ORA_RHS1, iy, iz, ix) = r1;
        s->f(ORA_RHS2, iy, iz, ix) = r2;
        s->f(ORA_OLD1, iy, iz, ix) = o1;
        s->f(ORA_OLD2, iy, iz, ix) = o2;
      }
    }
}

// ----------------------------------------------------- line solver ----
// coef: src/hst_linsolve.f90:236-252
static inline double coef(const ora_sim* s, int sys, double lambda, double kk, int iy, int j) {
  const double ni = s->ni;
  switch (sys) {
    case ORA_D2V:
      return lambda * (s->D(iy, 2, j) - kk * s->D(iy, 0, j)) - ni * (s->D(iy, 3, j) - 2.0 * kk * s->D(iy, 2, j) + kk * kk * s->D(iy, 0, j));
    case ORA_ETA:
      return lambda * s->D(iy, 0, j) - ni * (s->D(iy, 2, j) - kk * s->D(iy, 0, j));
    case ORA_POISSON:
      return s->D(iy, 2, j) - kk * s->D(iy, 0, j);
    default:
      return s->D(iy, 0, j);
  }
}
// rhs_row: src/hst_linsolve.f90:257-271 (src points at row -2 of the line)
static inline cx rhs_row(const ora_sim* s, int sys, const cx* src, int iy) {
  if (sys == ORA_DY) {
    cx r = C(0, 0);
    for (int j = -2; j <= 2; ++j) r = r + s->D(iy, 1, j) * src[iy + j + 2];
    return r;
  }
  return src[iy + 2];
}

// One line: penta_forward (src/hst_linsolve.f90:282-354) and
// penta_backward (:359-483) with one slab (npy = 1).
static void solve_line(const ora_sim* s, int sys, double lambda, double kk, cx ph, const cx* src, cx* dst,
                       std::vector<double>& U1, std::vector<double>& U2, std::vector<double>& B1,
                       std::vector<double>& B2, std::vector<cx>& XR) {
  const int m = s->ny, mi = m - 2;
  double rec[29];
  {
    double u11 = 0, u12 = 0, p1 = 0, q1 = 0, u21 = 0, u22 = 0, p2 = 0, q2 = 0;
    cx x1 = C(0, 0), x2 = C(0, 0);
    double w1 = 0, w2 = 0, v1 = 0, v2 = 0;
    cx sx0 = C(0, 0), sx1 = C(0, 0);
    double sp0 = 0, sq0 = 0, sp1 = 0, sq1 = 0;
    for (int i = 0; i < mi; ++i) {
      double a[5];
      for (int j = -2; j <= 2; ++j) a[j + 2] = coef(s, sys, lambda, kk, i, j);
      double p = 0, q = 0;
      if (i == 0) { p = a[0]; q = a[1]; }
      if (i == 1) q = a[0];
      cx bx = rhs_row(s, sys, src, i);
      if (i >= 2) {
        double l = a[0];
        a[1] = a[1] - l * u21;
        a[2] = a[2] - l * u22;
        bx = bx - l * x2;
        p = p - l * p2;
        q = q - l * q2;
      }
      if (i >= 1) {
        double l = a[1];
        a[2] = a[2] - l * u11;
        a[3] = a[3] - l * u12;
        bx = bx - l * x1;
        p = p - l * p1;
        q = q - l * q1;
      }
      double rp = 1.0 / a[2];
      double t1 = a[3] * rp, t2 = a[4] * rp;
      bx = bx * rp;
      p = p * rp;
      q = q * rp;
      U1[i] = t1; U2[i] = t2; B1[i] = p; B2[i] = q; XR[i] = bx;
      double w = -(u11 * w1 + u22 * w2);
      if (i == 0) w = 1.0;
      double v = -(u11 * v1 + u22 * v2);
      if (i == 1) v = 1.0;
      sx0 = sx0 + w * bx; sp0 = sp0 + w * p; sq0 = sq0 + w * q;
      sx1 = sx1 + v * bx; sp1 = sp1 + v * p; sq1 = sq1 + v * q;
      w2 = w1; w1 = w; v2 = v1; v1 = v;
      u21 = u11; u22 = u12; x2 = x1; p2 = p1; q2 = q1;
      u11 = t1; u12 = t2; x1 = bx; p1 = p; q1 = q;
    }
    rec[1] = sx0.re; rec[2] = sx0.im; rec[3] = sp0; rec[4] = sq0;
    rec[5] = w2 * u22 + w1 * u11; rec[6] = w1 * u12;
    rec[7] = sx1.re; rec[8] = sx1.im; rec[9] = sp1; rec[10] = sq1;
    rec[11] = v2 * u22 + v1 * u11; rec[12] = v1 * u12;
    cx bx = x2 - u21 * x1;
    rec[13] = bx.re; rec[14] = bx.im; rec[15] = p2 - u21 * p1; rec[16] = q2 - u21 * q1;
    rec[17] = u22 - u21 * u11; rec[18] = -u21 * u12;
    rec[19] = x1.re; rec[20] = x1.im; rec[21] = p1; rec[22] = q1;
    rec[23] = u11; rec[24] = u12;
    bx = rhs_row(s, sys, src, m - 2);
    rec[25] = bx.re; rec[26] = bx.im;
    bx = rhs_row(s, sys, src, m - 1);
    rec[27] = bx.re; rec[28] = bx.im;
  }
  // reduced 2x2 system (nslab = 1: s = t = 0, all blocks accumulate)
  cx A[3][3], b[3];
  for (int r = 1; r <= 2; ++r) {
    b[r] = C(0, 0);
    for (int c = 1; c <= 2; ++c) A[r][c] = C(0, 0);
  }
  {
    const cx cph = conj(ph), php = ph;
    const int ga = m - 2;
    double c1m4 = coef(s, sys, lambda, kk, ga, -2), c1m3 = coef(s, sys, lambda, kk, ga, -1);
    double d11 = coef(s, sys, lambda, kk, ga, 0), d12 = coef(s, sys, lambda, kk, ga, 1);
    double c10 = coef(s, sys, lambda, kk, ga, 2);
    double c2m3 = coef(s, sys, lambda, kk, ga + 1, -2), d21 = coef(s, sys, lambda, kk, ga + 1, -1);
    double d22 = coef(s, sys, lambda, kk, ga + 1, 0), c20 = coef(s, sys, lambda, kk, ga + 1, 1);
    double c21 = coef(s, sys, lambda, kk, ga + 1, 2);
    int r = 1;
    cx xm2 = C(rec[13], rec[14]), xm1 = C(rec[19], rec[20]);
    cx x0 = C(rec[1], rec[2]);
    b[r] = ((C(rec[25], rec[26]) - c1m4 * xm2) - c1m3 * xm1) - (c10 * php) * x0;
    A[r][1] = A[r][1] - cph * (c1m4 * rec[15] + c1m3 * rec[21]);
    A[r][2] = A[r][2] - cph * (c1m4 * rec[16] + c1m3 * rec[22]);
    A[r][1] = A[r][1] + C(d11, 0.0) - C(c1m4 * rec[17] + c1m3 * rec[23], 0.0);
    A[r][2] = A[r][2] + C(d12, 0.0) - C(c1m4 * rec[18] + c1m3 * rec[24], 0.0);
    cx f = c10 * php;
    f = f * conj(ph);  // t == 0
    A[r][1] = A[r][1] - f * rec[3];
    A[r][2] = A[r][2] - f * rec[4];
    A[r][1] = A[r][1] - (c10 * php) * rec[5];
    A[r][2] = A[r][2] - (c10 * php) * rec[6];
    r = 2;
    cx xx1 = C(rec[7], rec[8]);
    b[r] = (C(rec[27], rec[28]) - c2m3 * xm1) - php * (c20 * x0 + c21 * xx1);
    A[r][1] = A[r][1] - (cph * c2m3) * rec[21];
    A[r][2] = A[r][2] - (cph * c2m3) * rec[22];
    A[r][1] = A[r][1] + C(d21, 0.0) - C(c2m3 * rec[23], 0.0);
    A[r][2] = A[r][2] + C(d22, 0.0) - C(c2m3 * rec[24], 0.0);
    f = php;
    f = f * conj(ph);
    A[r][1] = A[r][1] - f * (c20 * rec[3] + c21 * rec[9]);
    A[r][2] = A[r][2] - f * (c20 * rec[4] + c21 * rec[10]);
    A[r][1] = A[r][1] - php * (c20 * rec[5] + c21 * rec[11]);
    A[r][2] = A[r][2] - php * (c20 * rec[6] + c21 * rec[12]);
  }
  // Gaussian elimination without pivoting, back substitution (:437-453)
  {
    cx piv = cdiv(C(1.0, 0.0), A[1][1]);
    cx f = A[2][1] * piv;
    A[2][2] = A[2][2] - f * A[1][2];
    b[2] = b[2] - f * b[1];
    b[2] = cdiv(b[2], A[2][2]);
    cx g = b[1] - A[1][2] * b[2];
    b[1] = cdiv(g, A[1][1]);
  }
  cx xb1 = b[1], xb2 = b[2];
  dst[m - 2 + 2] = xb1;
  dst[m - 1 + 2] = xb2;
  cx yb1 = conj(ph) * b[1], yb2 = conj(ph) * b[2];
  cx xk1 = xb1, xk2 = xb2;
  for (int i = m - 3; i >= 0; --i) {
    cx xk = (((XR[i] - B1[i] * yb1) - B2[i] * yb2) - U1[i] * xk1) - U2[i] * xk2;
    dst[i + 2] = xk;
    xk2 = xk1;
    xk1 = xk;
  }
}

// line_solve: src/hst_linsolve.f90:147-233
void ora_line_solve(ora_sim* s, int sys, double lambda, int src, int dst, int has_shift, double sx, double sz) {
  if (!has_shift) ora_shear_shifts(s, s->time, &sx, &sz);
  const int ny = s->ny;
#pragma omp parallel
  {
    std::vector<double> U1(ny), U2(ny), B1(ny), B2(ny);
    std::vector<cx> XR(ny);
#pragma omp for
    for (int ix = 0; ix <= s->nx; ++ix)
      for (int iz = -s->nz; iz <= s->nz; ++iz) {
        cx* d = &s->F[dst][s->fidx(-2, iz, ix)];
        if (ix == 0 && iz == 0 && sys == ORA_D2V) {
          for (int iy = 0; iy < ny; ++iy) d[iy + 2] = C(0, 0);
          continue;
        }
        if (ix == 0 && iz == 0 && sys == ORA_POISSON) continue;
        const double kk = s->k2[(size_t)(iz + s->nz) + (size_t)s->nzT * ix];
        cx ph = cexpi(-(s->p.alfa0 * ix * sx + s->p.beta0 * iz * sz));
        solve_line(s, sys, lambda, kk, ph, &s->F[src][s->fidx(-2, iz, ix)], d, U1, U2, B1, B2, XR);
      }
  }
}

// shear_shift + shift_unweighted: src/hst_equations.f90:226-293
static void shift_unweighted(ora_sim* s, int q, double dgx, double dgz, double sx0, double sz0, double sx1, double sz1) {
  ora_line_solve(s, ORA_D0, 0.0, q, ORA_V1, 1, sx0, sz0);
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz)
      for (int iy = 0; iy < s->ny; ++iy)
        s->f(ORA_V1, iy, iz, ix) = s->f(ORA_V1, iy, iz, ix) * cexpi(-(s->p.alfa0 * ix * dgx + s->p.beta0 * iz * dgz) * s->y[iy + 2]);
  ora_fill_ghosts(s, ORA_V1, sx1, sz1);
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz)
      for (int iy = 0; iy < s->ny; ++iy) {
        cx acc = C(0, 0);
        for (int j = -2; j <= 2; ++j) acc = acc + s->D(iy, 0, j) * s->f(ORA_V1, iy + j, iz, ix);
        s->f(q, iy, iz, ix) = acc;
      }
}
void ora_shear_shift(ora_sim* s, double dt_sub) {
  double dgx = s->p.S * dt_sub;
  double dgz = ora_s2_integral(s, s->time, s->time + dt_sub);
  if (s->p.exact_shift) {
    double sx0, sz0, sx1, sz1;
    ora_shear_shifts(s, s->time, &sx0, &sz0);
    ora_shear_shifts(s, s->time + dt_sub, &sx1, &sz1);
    shift_unweighted(s, ORA_RHS1, dgx, dgz, sx0, sz0, sx1, sz1);
    shift_unweighted(s, ORA_RHS2, dgx, dgz, sx0, sz0, sx1, sz1);
    shift_unweighted(s, ORA_OLD1, dgx, dgz, sx0, sz0, sx1, sz1);
    shift_unweighted(s, ORA_OLD2, dgx, dgz, sx0, sz0, sx1, sz1);
    return;
  }
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz)
      for (int iy = 0; iy < s->ny; ++iy) {
        cx f = cexpi(-(s->p.alfa0 * ix * dgx + s->p.beta0 * iz * dgz) * s->y[iy + 2]);
        s->f(ORA_RHS1, iy, iz, ix) = s->f(ORA_RHS1, iy, iz, ix) * f;
        s->f(ORA_RHS2, iy, iz, ix) = s->f(ORA_RHS2, iy, iz, ix) * f;
        s->f(ORA_OLD1, iy, iz, ix) = s->f(ORA_OLD1, iy, iz, ix) * f;
        s->f(ORA_OLD2, iy, iz, ix) = s->f(ORA_OLD2, iy, iz, ix) * f;
      }
}

// linsolve: src/hst_equations.f90:298-326
void ora_linsolve(ora_sim* s, double lambda) {
  ora_line_solve(s, ORA_D2V, lambda, ORA_RHS2, ORA_V2, 0, 0, 0);
  ora_line_solve(s, ORA_ETA, lambda, ORA_RHS1, ORA_V1, 0, 0, 0);
  ora_fill_ghosts_now(s, ORA_V2);
  ora_line_solve(s, ORA_DY, 0.0, ORA_V2, ORA_V3, 0, 0, 0);
#pragma omp parallel for
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      const double kk = s->k2[(size_t)(iz + s->nz) + (size_t)s->nzT * ix];
      const cx ialfa = C(0.0, ix * s->p.alfa0), ibeta = C(0.0, iz * s->p.beta0);
      for (int iy = 0; iy < s->ny; ++iy) {
        cx& u = s->f(0, iy, iz, ix);
        cx& w = s->f(2, iy, iz, ix);
        if (ix == 0 && iz == 0) {
          cx temp = u;
          u = C(temp.re, 0.0);
          w = C(temp.im, 0.0);
        } else {
          cx temp = (ialfa * w - ibeta * u) / kk;
          w = (ibeta * w + ialfa * u) / kk;
          u = temp;
        }
      }
    }
  ora_fill_ghosts_now(s, ORA_V1);
  ora_fill_ghosts_now(s, ORA_V3);
}

// substep i (0, 1, 2) of timestep: one pass of the loop body of
// src/hst_equations.f90:58-86
void ora_substep(ora_sim* s, int i) {
  {
    const double* ODE = s->RK[i];
    if (!s->p.linear || i == 2) ora_transform_to_physical(s);
    if (i == 2) ora_compute_cfl(s);
    if (ora_damping_active(s)) ora_damping_update(s, s->time);
    ora_buildrhs_prepare(s, ODE);
    if (!s->p.linear) {
      for (int g = 1; g <= 2; ++g) {
        ora_build_products(s, g);
        ora_products_to_spectral(s);
        ora_buildrhs(s, ODE, g);
      }
    }
    if (s->p.damp_hard && ora_damping_active(s)) ora_damping_mask(s);
    double dt_sub = 2.0 / ODE[0] * s->deltat;
    ora_shear_shift(s, dt_sub);
    s->time = s->time + dt_sub;
    ora_linsolve(s, ODE[0] / s->deltat);
    if (stokes_active(s)) {
      stokes_apply(s);
      ora_fill_ghosts_now(s, ORA_V3);
    }
  }
}

// timestep: src/hst_equations.f90:56-87
void ora_timestep(ora_sim* s) {
  for (int i = 0; i < 3; ++i) ora_substep(s, i);
}

// new_timestep: src/hst.f90:163-169 (one rank)
static void new_timestep(ora_sim* s) {
  if (s->p.cflmax > 0.0 && s->cfl > 0.0) s->deltat = s->p.cflmax / s->cfl;
  if (s->dt_fixed > 0.0) s->deltat = std::min(s->deltat, s->dt_fixed);
  if (s->dt_fixed > 0.0 && s->p.cflmax <= 0.0) s->deltat = s->dt_fixed;
}

// set-up part of program hst: src/hst.f90:70-88
void ora_start(ora_sim* s) {
  bool loaded = false;
  if (s->p.restart_from_file) loaded = (ora_restart_read(s, s->p.restart_file) == 0);
  if (!loaded) ora_generate_initial_field(s);
  stokes_apply(s);
  for (int m = 0; m < 3; ++m) ora_fill_ghosts_now(s, m);
  if (s->deltat == 0.0) s->deltat = 1.0;
  ora_transform_to_physical(s);
  ora_compute_cfl(s);
  new_timestep(s);
}

// the time loop: src/hst.f90:98-133 (no output)
long ora_run(ora_sim* s, long max_steps) {
  long n = 0;
  while (s->time < s->p.t_max - 0.5 * s->deltat && s->istep < s->p.nstep && n < max_steps) {
    s->istep++;
    n++;
    ora_timestep(s);
    new_timestep(s);
  }
  return n;
}

// The reductions of outstats (src/hst_stats.f90:136-243) as the reference
// leaves them in its `sums` array before the box-mean correction:
// sums = [eps, uv, uu, vv, ww, vw, uw, mfx, mfz, q_in, q_out, e_in, e_out,
// ed, pd, ncol_damped] (box-height integrals over rows weighted by dyl), and
// the column energies exz(-nz:nz, 0:nx) = sum_y w |u|^2 (:225-240).
void ora_outstats_sums(ora_sim* s, double* sums, double* exz) {
  const int nx = s->nx, nz = s->nz, ny = s->ny;
  const int inc00 = stokes_active(s) ? 0 : 1;
  const double gsoft = damping_soft_factor(s);
  const int NV = 15;
  std::vector<double> part((size_t)(nx + 1) * NV, 0.0);
#pragma omp parallel for
  for (int ix = 0; ix <= nx; ++ix) {
    double v[15] = {0};  // eps uv uu vv ww vw uw mfx mfz q_in q_out e_in e_out ed pd
    for (int iz = -nz; iz <= nz; ++iz) {
      const size_t col = (size_t)(iz + nz) + (size_t)s->nzT * ix;
      const double kk = s->k2[col], gd = s->gdamp[col];
      for (int iy = 0; iy < ny; ++iy) {
        cx cu = s->f(0, iy, iz, ix), cv = s->f(1, iy, iz, ix), cw = s->f(2, iy, iz, ix);
        if (ix == 0 && iz == 0) {
          v[7] = v[7] + cu.re * s->dyl[iy];
          v[8] = v[8] + cw.re * s->dyl[iy];
          if (gd > 0.0) {
            double qc = s->dyl[iy] * (cu * conj(cu) + cw * conj(cw)).re;
            v[13] = v[13] + qc;
            v[14] = v[14] + 2.0 * gsoft * gd * qc;
          }
          if (inc00 == 1) {
            v[2] = v[2] + s->dyl[iy] * (cu * conj(cu)).re;
            v[4] = v[4] + s->dyl[iy] * (cw * conj(cw)).re;
            v[6] = v[6] + s->dyl[iy] * (cu * conj(cw)).re;
          }
          continue;
        }
        double w = 2.0 * s->dyl[iy];
        if (ix == 0) w = s->dyl[iy];
        const double q = (cu * conj(cu) + cv * conj(cv) + cw * conj(cw)).re;
        if (gd > 0.0) {
          double qc = w * q;
          v[13] = v[13] + qc;
          v[14] = v[14] + 2.0 * gsoft * gd * qc;
        }
        v[2] = v[2] + w * (cu * conj(cu)).re;
        v[3] = v[3] + w * (cv * conj(cv)).re;
        v[4] = v[4] + w * (cw * conj(cw)).re;
        v[1] = v[1] + w * (cu * conj(cv)).re;
        v[5] = v[5] + w * (cw * conj(cv)).re;
        v[6] = v[6] + w * (cu * conj(cw)).re;
        v[0] = v[0] + w * kk * q;
        if (s->inlayer[iy] == 1) {
          v[9] = v[9] + w * q;
          v[11] = v[11] + w * kk * q;
        } else {
          v[10] = v[10] + w * q;
          v[12] = v[12] + w * kk * q;
        }
      }
    }
    for (int k = 0; k < NV; ++k) part[(size_t)ix * NV + k] = v[k];
  }
  for (int k = 0; k < 16; ++k) sums[k] = 0.0;
  for (int ix = 0; ix <= nx; ++ix)
    for (int k = 0; k < NV; ++k) sums[k] += part[(size_t)ix * NV + k];
  // y derivatives of the three components into rhs1 (:198-223)
  for (int c = 0; c < 3; ++c) {
    ora_line_solve(s, ORA_DY, 0.0, c, ORA_RHS1, 0, 0, 0);
    std::vector<double> gp((size_t)(nx + 1) * 3, 0.0);
#pragma omp parallel for
    for (int ix = 0; ix <= nx; ++ix) {
      double grad = 0, g_in = 0, g_out = 0;
      for (int iz = -nz; iz <= nz; ++iz)
        for (int iy = 0; iy < ny; ++iy) {
          if (ix == 0 && iz == 0 && inc00 == 0) continue;
          double w = 2.0 * s->dyl[iy];
          if (ix == 0) w = s->dyl[iy];
          cx dq = s->f(ORA_RHS1, iy, iz, ix);
          const double q = (dq * conj(dq)).re;
          grad = grad + w * q;
          if (s->inlayer[iy] == 1) g_in = g_in + w * q;
          else g_out = g_out + w * q;
        }
      gp[(size_t)ix * 3] = grad;
      gp[(size_t)ix * 3 + 1] = g_in;
      gp[(size_t)ix * 3 + 2] = g_out;
    }
    for (int ix = 0; ix <= nx; ++ix) {
      sums[0] += gp[(size_t)ix * 3];
      sums[11] += gp[(size_t)ix * 3 + 1];
      sums[12] += gp[(size_t)ix * 3 + 2];
    }
  }
  sums[15] = (double)(ora_damping_active(s) ? s->ncol_damped : 0);
  // column energies
  if (exz) {
#pragma omp parallel for
    for (int ix = 0; ix <= nx; ++ix)
      for (int iz = -nz; iz <= nz; ++iz) {
        double qc = 0.0;
        for (int iy = 0; iy < ny; ++iy) {
          cx cu = s->f(0, iy, iz, ix), cv = s->f(1, iy, iz, ix), cw = s->f(2, iy, iz, ix);
          double w = 2.0 * s->dyl[iy];
          if (ix == 0) w = s->dyl[iy];
          qc = qc + w * (cu * conj(cu) + cv * conj(cv) + cw * conj(cw)).re;
        }
        exz[(size_t)(iz + nz) + (size_t)s->nzT * ix] = qc;
      }
  }
}

// outstats: src/hst_stats.f90:136-285 (energy, dissipation, uv, vw, normal stresses)
void ora_outstats(ora_sim* s, double* out) {
  const int nx = s->nx, nz = s->nz, ny = s->ny;
  const bool inc00 = !stokes_active(s);
  std::vector<double> part((size_t)(nx + 1) * 10, 0.0);
#pragma omp parallel for
  for (int ix = 0; ix <= nx; ++ix) {
    double eps = 0, uv = 0, uu = 0, vv = 0, ww = 0, vw = 0, uw = 0, mfx = 0, mfz = 0;
    for (int iz = -nz; iz <= nz; ++iz) {
      const double kk = s->k2[(size_t)(iz + nz) + (size_t)s->nzT * ix];
      for (int iy = 0; iy < ny; ++iy) {
        cx cu = s->f(0, iy, iz, ix), cv = s->f(1, iy, iz, ix), cw = s->f(2, iy, iz, ix);
        if (ix == 0 && iz == 0) {
          mfx = mfx + cu.re * s->dyl[iy];
          mfz = mfz + cw.re * s->dyl[iy];
          if (inc00) {
            uu = uu + s->dyl[iy] * (cu * conj(cu)).re;
            ww = ww + s->dyl[iy] * (cw * conj(cw)).re;
            uw = uw + s->dyl[iy] * (cu * conj(cw)).re;
          }
          continue;
        }
        double w = 2.0 * s->dyl[iy];
        if (ix == 0) w = s->dyl[iy];
        uu = uu + w * (cu * conj(cu)).re;
        vv = vv + w * (cv * conj(cv)).re;
        ww = ww + w * (cw * conj(cw)).re;
        uv = uv + w * (cu * conj(cv)).re;
        vw = vw + w * (cw * conj(cv)).re;
        uw = uw + w * (cu * conj(cw)).re;
        eps = eps + w * kk * (cu * conj(cu) + cv * conj(cv) + cw * conj(cw)).re;
      }
    }
    double* pp = &part[(size_t)ix * 10];
    pp[0] = eps; pp[1] = uv; pp[2] = uu; pp[3] = vv; pp[4] = ww; pp[5] = vw; pp[6] = uw; pp[7] = mfx; pp[8] = mfz;
  }
  double sums[10] = {0};
  for (int ix = 0; ix <= nx; ++ix)
    for (int k = 0; k < 9; ++k) sums[k] += part[(size_t)ix * 10 + k];
  // dissipation from the three compact y derivatives (KIND_DY into rhs1)
  for (int c = 0; c < 3; ++c) {
    ora_line_solve(s, ORA_DY, 0.0, c, ORA_RHS1, 0, 0, 0);
    std::vector<double> gp(nx + 1, 0.0);
#pragma omp parallel for
    for (int ix = 0; ix <= nx; ++ix) {
      double grad = 0;
      for (int iz = -nz; iz <= nz; ++iz)
        for (int iy = 0; iy < ny; ++iy) {
          if (ix == 0 && iz == 0 && !inc00) continue;
          double w = 2.0 * s->dyl[iy];
          if (ix == 0) w = s->dyl[iy];
          cx dq = s->f(ORA_RHS1, iy, iz, ix);
          grad = grad + w * (dq * conj(dq)).re;
        }
      gp[ix] = grad;
    }
    for (int ix = 0; ix <= nx; ++ix) sums[0] += gp[ix];
  }
  double eps = sums[0], uv = sums[1], uu = sums[2], vv = sums[3], ww = sums[4], vw = sums[5], uw = sums[6];
  double mfx = sums[7], mfz = sums[8];
  if (inc00) {
    double ly_w = 0.0;
    for (int iy = 0; iy < ny; ++iy) ly_w += s->dyl[iy];
    uu = uu - mfx * mfx / ly_w;
    ww = ww - mfz * mfz / ly_w;
    uw = uw - mfx * mfz / ly_w;
  }
  double q2 = uu + vv + ww;
  double inv_ly = 1.0 / s->p.ly;
  out[0] = 0.5 * q2 * inv_ly;
  out[1] = s->ni * eps * inv_ly;
  out[2] = uv * inv_ly;
  out[3] = vw * inv_ly;
  out[4] = uu * inv_ly;
  out[5] = vv * inv_ly;
  out[6] = ww * inv_ly;
  out[7] = uw * inv_ly;
}

// ------------------------------------------------------------ pressure ----
// compute_pressure: src/hst_pressure.f90:35-110.  The right-hand side of
// the pressure Poisson equation from the six product spectra (both groups)
// and the mean-shear term, into rhs1; the POISSON solve into dst; the (0,0)
// mode is -<vv> itself with its y mean removed.
void ora_compute_pressure(ora_sim* s, int dst) {
  const double s2now = ora_s2_of(s, s->time);
  const double S = s->p.S;
  ora_transform_to_physical(s);
  for (int g = 1; g <= 2; ++g) {
    ora_build_products(s, g);
    ora_products_to_spectral(s);
#pragma omp parallel for
    for (int ix = 0; ix <= s->nx; ++ix)
      for (int iz = -s->nz; iz <= s->nz; ++iz) {
        const cx ialfa = C(0.0, ix * s->p.alfa0), ibeta = C(0.0, iz * s->p.beta0);
        const int kz = s->izd[iz + s->nz];
        for (int iy = 0; iy < s->ny; ++iy) {
          cx r = s->f(ORA_RHS1, iy, iz, ix);
          for (int p = 1; p <= 3; ++p) {
            const int m = 3 * (g - 1) + p;
            cx d0 = C(0, 0), d1 = C(0, 0), d2 = C(0, 0);
            for (int j = -2; j <= 2; ++j) {
              cx q = s->vvdz(kz, ix, iy + j, p - 1);
              d0 = d0 + s->D(iy, 0, j) * q;
              d1 = d1 + s->D(iy, 1, j) * q;
              d2 = d2 + s->D(iy, 2, j) * q;
            }
            cx term;
            switch (m) {
              case 1: term = -((ialfa * ialfa) * d0); break;
              case 2: term = -d2; break;
              case 3: term = -((ibeta * ibeta) * d0); break;
              case 4: term = -((2.0 * ialfa) * d1); break;
              case 5: term = -((2.0 * ibeta) * d1); break;
              default: term = -(((2.0 * ialfa) * ibeta) * d0); break;
            }
            if (m == 1) {
              cx v0 = C(0, 0);
              for (int j = -2; j <= 2; ++j) v0 = v0 + s->D(iy, 0, j) * s->f(ORA_V2, iy + j, iz, ix);
              r = term - (2.0 * (S * ialfa + s2now * ibeta)) * v0;
            } else {
              r = r + term;
            }
            if (ix == 0 && iz == 0 && m == 2) r = C(-s->vvdz(0, 0, iy, p - 1).re, 0.0);
          }
          s->f(ORA_RHS1, iy, iz, ix) = r;
        }
      }
  }
  ora_line_solve(s, ORA_POISSON, 0.0, ORA_RHS1, dst, 0, 0, 0);
  double pmean = 0.0;
  for (int iy = 0; iy < s->ny; ++iy) {
    s->f(dst, iy, 0, 0) = s->f(ORA_RHS1, iy, 0, 0);
    pmean = pmean + s->f(dst, iy, 0, 0).re * s->dyl[iy];
  }
  pmean = pmean / s->p.ly;
  for (int iy = 0; iy < s->ny; ++iy) s->f(dst, iy, 0, 0) = C(s->f(dst, iy, 0, 0).re - pmean, 0.0);
}

// -------------------------------------------------------- field files ----
// restart_write / write_cpl: src/hst_io.f90:240-315.  Header as io.cpl
// writes it; the array (0..nx, -nz..nz, -2..ny+1) of CPL (u, v, w) =
// our (u, w, v), C order with the components innermost; ghost rows are
// plain periodic copies.
static std::string fmt_r(double x) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17G", x);
  return b;
}
int ora_restart_write(ora_sim* s, const char* path) {
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return 1;
  const ora_params& p = s->p;
  std::string h = "nx=" + std::to_string(s->nx) + " \tny=" + std::to_string(s->nz) + " \tnz=" + std::to_string(s->ny + 1) +
                  " \talpha0=" + fmt_r(p.alfa0) + " \tbeta0=" + fmt_r(p.beta0) + " \thtcoeff=" + fmt_r(p.ystretch > 0 ? p.ystretch : -1.0) +
                  " \tRe=" + fmt_r(p.re) + " \tPr=0.71\n" + "deltat=" + fmt_r(s->deltat) + " \tt_max=" + fmt_r(p.t_max) +
                  " \tdt_field=" + fmt_r(1e9) + " \tdt_save=" + fmt_r(1e9) + "\n" + "t_field=" + fmt_r(s->time) + "\n" +
                  "meanpx=0 \tmeanflowx=0 \tmeanpy=0 \tmeanflowy=0\n";
  std::fwrite(h.data(), 1, h.size(), fp);
  auto raw = [&](const char* key, double v) {
    std::fputs(key, fp);
    std::fputs("=\n", fp);
    std::fwrite(&v, 8, 1, fp);
    std::fputc('\n', fp);
  };
  raw("time", s->time);
  raw("S", p.S);
  raw("S2", ora_s2_of(s, s->time));
  raw("gamma_x", p.S * s->time);
  raw("gamma_y", gamma_y_of(s, s->time));
  std::fputs("Vfield=\n", fp);
  const int order[3] = {0, 2, 1};
  const int ny = s->ny;
  std::vector<cx> buf((size_t)(ny + 4) * 3);
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz) {
      for (int r = -2; r <= ny + 1; ++r) {
        int iy = r < 0 ? r + ny : (r >= ny ? r - ny : r);  // periodic copies
        for (int c = 0; c < 3; ++c) buf[(size_t)(r + 2) * 3 + c] = s->f(order[c], iy, iz, ix);
      }
      std::fwrite(buf.data(), sizeof(cx), buf.size(), fp);
    }
  std::fclose(fp);
  return 0;
}
// restart_read: src/hst_io.f90:69-178 (same mesh; no remap)
int ora_restart_read(ora_sim* s, const char* path) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return 1;
  std::vector<char> all;
  char b[65536];
  size_t n;
  while ((n = std::fread(b, 1, sizeof b, fp)) > 0) all.insert(all.end(), b, b + n);
  std::fclose(fp);
  std::string head(all.begin(), all.begin() + std::min<size_t>(all.size(), 4096));
  size_t pv = head.find("Vfield=\n");
  if (pv == std::string::npos) return 2;
  auto hv = [&](const char* key) -> double {
    size_t q = head.find(key);
    if (q == std::string::npos) return -1e308;
    return std::strtod(head.c_str() + q + std::strlen(key), nullptr);
  };
  int r_nx = (int)hv("nx="), r_ny = (int)hv("ny="), r_nz = (int)hv("nz=");
  if (r_nx != s->nx || r_ny != s->nz || r_nz - 1 != s->ny) return 3;
  size_t pt = head.find("time=\n");
  double r_time;
  std::memcpy(&r_time, all.data() + pt + 6, 8);
  if (s->p.time_from_restart) s->time = r_time;
  const char* data = all.data() + pv + 8;
  size_t need = (size_t)(s->nx + 1) * s->nzT * (s->ny + 4) * 3 * sizeof(cx);
  if (all.size() < pv + 8 + need) return 4;
  const int order[3] = {0, 2, 1};
  const int ny = s->ny;
  for (int ix = 0; ix <= s->nx; ++ix)
    for (int iz = -s->nz; iz <= s->nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int c = 0; c < 3; ++c) {
          size_t off = ((((size_t)ix * s->nzT + (iz + s->nz)) * (ny + 4) + (iy + 2)) * 3 + c) * sizeof(cx);
          std::memcpy(&s->f(order[c], iy, iz, ix), data + off, sizeof(cx));
        }
  return 0;
}

}  // extern "C"
