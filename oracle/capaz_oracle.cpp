// capaz_oracle.cpp — CPU restatement of the reference time step (the oracle).
//
// TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg load this library, and only as the parity reference or the timed
// CPU baseline.  The product (capaz_b200/) never calls it.
//
// What it follows, stage by stage, in the reference's own operation order so
// that IEEE-754 double arithmetic reproduces the reference bit for bit:
//   S_calculation          cpu.cpp:28-36, 171-182
//   ro_P_Xi_calculation    cpu.cpp:3-15, 143-169; two-phase.cpp:4-23;
//                          three-phase.cpp:11-240
//   u_calculation          cpu.cpp:17-26, 185-207, 266-314, 346-477
//   roS_calculation (NR)   cpu.cpp:52-65, 236-314, 619-731
//   P_S_calculation        cpu.cpp:80-89; two-phase.cpp:25-56;
//                          three-phase.cpp:286-339 with gauss.cpp:6-92
//   boundary_conditions    cpu.cpp:91-141; two-phase.cpp:59-111;
//                          three-phase.cpp:345-427; main.cpp:255-267
//   data_initialization    two-phase.cpp:113-172; three-phase.cpp:429-500
// Loops run over cells in parallel (OpenMP): every stage writes only its own
// cell and reads values of the previous stage, and on grids with nx, ny >= 3
// and nz == 1 or nz >= 3 each boundary cell reads an interior cell, so the
// result does not depend on the loop order.
//
// Extensions (neutral values reproduce the reference exactly; parity of the
// non-neutral values is unpinned by the reference):
//   - per-cell permeability K[cell] in Xi (CAPAZ_FLAG_PERCELL_K), as the
//     Buckley-Leverett module does (b-l.cpp:65-66);
//   - top-face pressure P_atm + P_top_offset in Border_P;
//   - two-phase background initial S_n (S_n_background) off the source window;
//   - per-cell porosity m at initialisation;
//   - three-phase top source limited to the SOURCE window
//     (CAPAZ_FLAG_SOURCE_WINDOW), as the two-phase rule is.
#include <math.h>
#include <omp.h>

#include <cmath>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../include/capaz_b200.h"

namespace {

struct Grid {
  int nx, ny, nz;
  long sx, sy, sz, n;
  Grid(const capaz_params* p) : nx(p->nx), ny(p->ny), nz(p->nz) {
    sx = 1;
    sy = nx;
    sz = (long)nx * ny;
    n = sz * nz;
  }
  long at(int i, int j, int k) const { return i + (long)j * sy + (long)k * sz; }
  // Cells where roS and Newton run (cpu.cpp:621, two-phase.cpp:27).
  bool interior(int i, int j, int k) const {
    return (((i != 0) && (i != nx - 1)) || (nx < 2)) && (j != 0) && (j != ny - 1) &&
           (((k != 0) && (k != nz - 1)) || (nz < 2));
  }
  // set_boundary_basic_coordinate, CPU form (cpu.cpp:107-141).
  long basic(int i, int j, int k) const {
    int i1 = i, j1 = j, k1 = k;
    if ((i == 0) && (nx > 2)) i1++;
    if ((i == nx - 1) && (nx > 2)) i1--;
    if (j == 0) j1++;
    if (j == ny - 1) j1--;
    if ((k == 0) && (nz > 2)) k1++;
    if ((k == nz - 1) && (nz > 2)) k1--;
    return at(i1, j1, k1);
  }
};

// Dual numbers (value, derivative) for the forward-mode (tangent-linear)
// reference gradient: every operation carries its first derivative along one
// direction.  Branches (upwind choices, |x|) follow the value, as the
// forward step does.
using std::fabs;
using std::pow;

struct Dual {
  double v, d;
  Dual(double x = 0.) : v(x), d(0.) {}
  Dual(double x, double y) : v(x), d(y) {}
};
inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) {
  return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v));
}
inline bool operator!(const Dual& a) { return !a.v; }
inline Dual fabs(const Dual& a) { return a.v < 0 ? -a : a; }
inline Dual pow(const Dual& a, double e) {
  const double r = std::pow(a.v, e);
  return Dual(r, (a.d == 0.) ? 0. : e * std::pow(a.v, e - 1.) * a.d);
}
inline double value(double x) { return x; }
inline double value(const Dual& x) { return x.v; }

// right_difference / left_difference / central_difference (cpu.cpp:185-314).
template <class T>
inline T rdiff(const T* a, long l, long s, double h) { return (a[l + s] - a[l]) / h; }
template <class T>
inline T ldiff(const T* a, long l, long s, double h) { return (a[l] - a[l - s]) / h; }
inline double cdiff(const double* a, long l, long s, double h) { return (a[l + s] - a[l - s]) / (2. * h); }

// directed_difference (cpu.cpp:236-264): first-order upwind flux difference.
template <class T>
inline T directed(T x1, T x2, const T* Xi, const T* ro, long l, long s, double h) {
  return (((x2 + fabs(x2)) / 2. - (x1 - fabs(x1)) / 2.) * (-1.) * Xi[l] * ro[l] -
          (x1 + fabs(x1)) / 2. * (-1.) * Xi[l - s] * ro[l - s] +
          (x2 - fabs(x2)) / 2. * (-1.) * Xi[l + s] * ro[l + s]) /
         h;
}

// reverse_matrix: Gauss-Jordan inverse that pivots only when |pivot| < 1e-8
// (gauss.cpp:6-92).  Returns 0, -1 (singular) or -2 (bad arguments).
int reverse_matrix(double* a, int n) {
  if (a == NULL || n < 2) return -2;
  const double e = 1E-8;
  const int n1 = n * 2;
  double matr[2 * 8 * 8];
  double row[2 * 8];
  if (n > 8) return -2;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) matr[j + n1 * i] = a[j + n * i];
  for (int i = 0; i < n; i++)
    for (int j = n; j < n1; j++) matr[j + n1 * i] = (j == n + i) ? 1 : 0;
  for (int k = 0; k < n; k++) {
    double f = matr[k + n1 * k];
    if (fabs(f) < e) {
      int det_flag = 0;
      for (int i = k + 1; i < n; i++) {
        if (matr[k + n1 * i] > e) {
          det_flag = 1;
          for (int j = 0; j < n1; j++) {
            row[j] = matr[j + n1 * k];
            matr[j + n1 * k] = matr[j + n1 * i];
            matr[j + n1 * i] = row[j];
          }
          f = matr[k + n1 * k];
        }
      }
      if (det_flag == 0) return -1;
    }
    for (int j = 0; j < n1; j++) matr[j + n1 * k] /= f;
    for (int i = 0; i < n; i++)
      if (i != k) {
        double f1 = matr[k + n1 * i];
        for (int j = 0; j < n1; j++) matr[j + n1 * i] -= (matr[j + n1 * k] * f1);
      }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) a[j + n * i] = matr[j + n + n1 * i];
  return 0;
}

// ---------------------------------------------------------------------------
// Three-phase constitutive relations, CPU form (three-phase.cpp:11-186).  The
// CPU capillary pressures and their derivatives are identically zero
// (three-phase.cpp:25,32,39,47,58,80,103,125).
inline double k_w3(double S_w_e, double A) {
  double k_w = 0;
  if (S_w_e >= 1e-3) k_w = pow(S_w_e, 0.5) * pow(1. - pow(1. - pow(S_w_e, A / (A - 1.)), (A - 1.) / A), 2.);
  return k_w;
}
inline double k_g3(double S_g_e, double A) {
  double k_g = 0;
  if (S_g_e >= 1e-3) k_g = pow(S_g_e, 0.5) * pow(1. - pow(1. - S_g_e, A / (A - 1.)), 2. * (A - 1.) / A);
  return k_g;
}
inline double k_n3(double S_w_e, double S_n_e, double A) {
  double k_n = 0;
  double S_g_e = 1. - S_w_e - S_n_e;
  if (S_n_e >= 1e-3) {
    double k_n_w = pow(1. - S_w_e, 0.5) * pow(1. - pow(S_w_e, A / (A - 1.)), 2. * (A - 1.) / A);
    double k_n_g = pow(S_n_e, 0.5) * pow(1. - pow(1. - pow(S_n_e, A / (A - 1.)), (A - 1.) / A), 2.);
    k_n = S_n_e * k_n_w * k_n_g / (1 - S_w_e) / (1 - S_g_e);
  }
  return k_n;
}

template <class T>
struct WorkT {
  std::vector<T> S_w, S_g, P_n, P_g, ro_w, ro_n, ro_g, Xi_w, Xi_n, Xi_g;
  std::vector<T> roS_w, roS_n, roS_g, roS_w_old, roS_n_old, roS_g_old;
  // Three-phase: P_n, P_g as u_calculation sees them (after ro_P_Xi), kept
  // when keep_u_pressures is set.
  bool keep_u_pressures = false;
  std::vector<double> Pn_u, Pg_u;
};
using Work = WorkT<double>;

// |I - NX/2| <= SOURCE and |K - NZ/2| <= SOURCE in global indices (a z-slab
// of a decomposed grid has its own plane 0 at global index z_offset).
inline bool in_window(const capaz_params* p, int i, int k) {
  const int nzg = p->nz_global > 0 ? p->nz_global : p->nz;
  const int kg = k + p->z_offset;
  return (i >= p->nx / 2 - p->source) && (i <= p->nx / 2 + p->source) && (kg >= nzg / 2 - p->source) &&
         (kg <= nzg / 2 + p->source);
}

template <class T>
inline T Kc(const capaz_params* p, const T* K, long l) {
  return ((p->flags & CAPAZ_FLAG_PERCELL_K) && K) ? K[l] : T(p->K0);
}

// ---------------------------------------------------------------------------
// Two-phase step.
template <class T>
void step2(const capaz_params* p, const Grid& g, T* P_w, T* S_n, const T* m, const T* K, WorkT<T>& w) {
  const double lam = p->lambda, S_wr = p->S_wr;
  const double e_kw = (2. + 3. * lam) / lam, e_kn = (2. + lam) / lam, e_pk = -1. / lam;
  T *S_w = w.S_w.data(), *P_n = w.P_n.data(), *ro_w = w.ro_w.data(), *ro_n = w.ro_n.data();
  T *Xi_w = w.Xi_w.data(), *Xi_n = w.Xi_n.data();
  T *roS_w = w.roS_w.data(), *roS_n = w.roS_n.data();
  T *roS_w_old = w.roS_w_old.data(), *roS_n_old = w.roS_n_old.data();

  // S_calculation (all cells).
#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) S_w[l] = 1. - S_n[l];

  // ro_P_Xi_calculation (all cells are active on one rank).
#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) {
    T S_e = (1. - S_n[l] - S_wr) / (1. - S_wr);
    T k_w = pow(S_e, e_kw);
    T k_n = (1. - S_e) * (1. - S_e) * (1 - pow(S_e, e_kn));
    T P_k = p->P_d * pow((1. - S_n[l] - S_wr) / (1. - S_wr), e_pk);
    P_n[l] = P_w[l] + P_k;
    Xi_w[l] = -1. * Kc(p, K, l) * k_w / p->mu_w;
    Xi_n[l] = -1. * Kc(p, K, l) * k_n / p->mu_n;
    ro_w[l] = p->ro0_w * (1. + (p->beta_w) * (P_w[l] - p->P_atm));
    ro_n[l] = p->ro0_n * (1. + (p->beta_n) * (P_n[l] - p->P_atm));
  }

  // roS_calculation, NR form (assign_roS_nr).
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        if (!m[l]) continue;
        const double q_w = 0., q_n = 0.;  // wells_q (two-phase.cpp:187-192)
        roS_w[l] = ro_w[l] * (1. - S_n[l]);
        roS_n[l] = ro_n[l] * S_n[l];
        T x1, x2, fx_w, fy_w, fz_w, fx_n, fy_n, fz_n;
        if (g.nz < 2) {
          fz_w = 0.;
          fz_n = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_w, l, g.sz, p->hz);
          fz_w = directed(x1, x2, Xi_w, ro_w, l, g.sz, p->hz);
          x2 = -1. * rdiff(P_n, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_n, l, g.sz, p->hz);
          fz_n = directed(x1, x2, Xi_n, ro_n, l, g.sz, p->hz);
        }
        if (g.nx < 2) {
          fx_w = 0.;
          fx_n = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_w, l, g.sx, p->hx);
          fx_w = directed(x1, x2, Xi_w, ro_w, l, g.sx, p->hx);
          x2 = -1. * rdiff(P_n, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_n, l, g.sx, p->hx);
          fx_n = directed(x1, x2, Xi_n, ro_n, l, g.sx, p->hx);
        }
        x2 = -1. * rdiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        x1 = -1. * ldiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        fy_w = directed(x1, x2, Xi_w, ro_w, l, g.sy, p->hy);
        x2 = -1. * rdiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        x1 = -1. * ldiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        fy_n = directed(x1, x2, Xi_n, ro_n, l, g.sy, p->hy);
        T A1 = roS_w[l] - (p->dt / m[l]) * (-q_w + fx_w + fy_w + fz_w);
        T A2 = roS_n[l] - (p->dt / m[l]) * (-q_n + fx_n + fy_n + fz_n);
        roS_w_old[l] = roS_w[l];
        roS_n_old[l] = roS_n[l];
        roS_w[l] = A1;
        roS_n[l] = A2;
      }

  // P_S_calculation (Newton, two-phase.cpp:25-56).
  const double P_d = p->P_d;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        T Pw = P_w[l], Sn = S_n[l];
        for (int it = 1; it <= p->newton_iterations; it++) {
          T S_e = (1 - Sn - S_wr) / (1 - S_wr);
          T P_k = P_d * pow(S_e, (-1.) / lam);
          T AAA = pow(S_e, (((-1.) / lam) - 1.));
          T F1 = p->ro0_w * (1. + (p->beta_w) * (Pw - p->P_atm)) * (1. - Sn) - roS_w[l];
          T F2 = p->ro0_n * (1. + (p->beta_n) * (Pw + P_k - p->P_atm)) * Sn - roS_n[l];
          T PkS = AAA * (P_d) / (lam * (1 - S_wr));
          T F1P = p->ro0_w * (p->beta_w) * (1 - Sn);
          T F2P = p->ro0_n * (p->beta_n) * Sn;
          T F1S = (-1) * (p->ro0_w) * (1 + (p->beta_w) * (Pw - p->P_atm));
          T F2S = p->ro0_n * (1 + (p->beta_n) * (Pw + P_k - p->P_atm + (Sn * PkS)));
          T det = F1P * F2S - F1S * F2P;
          T nPw = Pw - (1 / det) * (F2S * F1 - F1S * F2);
          T nSn = Sn - (1 / det) * (F1P * F2 - F2P * F1);
          Pw = nPw;
          Sn = nSn;
        }
        P_w[l] = Pw;
        S_n[l] = Sn;
      }

  // boundary_conditions: Border_S then Border_P per boundary cell.
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        bool bnd = (i == 0) || (i == g.nx - 1) || (j == 0) || (j == g.ny - 1) ||
                   (((k == 0) || (k == g.nz - 1)) && (g.nz >= 2));
        if (!bnd) continue;
        long l1 = g.basic(i, j, k);
        long l = g.at(i, j, k);
        if ((j != 0) || (p->source <= 0)) S_n[l] = S_n[l1];
        if ((j == 0) && (p->source > 0)) S_n[l] = in_window(p, i, k) ? T(p->S_n_gr) : S_n[l1];
        if ((j != 0) && (j != g.ny - 1)) {
          P_w[l] = P_w[l1];
        } else if (j == 0) {
          P_w[l] = T(p->P_atm + p->P_top_offset);
        } else {
          T ro_g_dy = (ro_n[l1] * S_n[l1] + ro_w[l1] * (1 - S_n[l1])) * (m[l1]) * (p->g_const) * (p->hy);
          P_w[l] = P_w[l1] + ro_g_dy;
        }
      }
}

// ---------------------------------------------------------------------------
// Buckley-Leverett task (B_L build: Backley-Leverett/b-l.cpp with cpu.cpp).

// assing_k (b-l.cpp:5-55), the "IPM" relative permeabilities of S_w.
inline void bl_relperm(double S_w, double* k_w, double* k_n) {
  const double S_sv = 0.1, S_zv = 0.8, S_1 = 0.70324;
  if ((S_sv <= S_w) && (S_w <= S_zv))
    *k_n = ((S_zv - S_w) / (S_zv - S_sv)) * ((S_zv - S_w) / (S_zv - S_sv));
  else if ((0 <= S_w) && (S_w <= S_sv))
    *k_n = 1.;
  else
    *k_n = 0.;
  if ((S_sv <= S_w) && (S_w <= S_1))
    *k_w = ((S_w - S_sv) / (S_zv - S_sv)) * ((S_w - S_sv) / (S_zv - S_sv));
  else if ((0 <= S_w) && (S_w <= S_sv))
    *k_w = 0.;
  else if ((S_1 <= S_w) && (S_w <= S_zv))
    *k_w = 0.8 * pow((S_w - S_sv) / (S_zv - S_sv), 0.5);
  else
    *k_w = 1.;
}

// is_injection_well / is_output_well (b-l.cpp:221-237): two 2x2 corners of
// every z-plane.
inline bool bl_injection(const Grid& g, int i, int j) {
  return ((i == 1) && (j == 1)) || ((i == 0) && (j == 0)) || ((i == 1) && (j == 0)) || ((i == 0) && (j == 1));
}
inline bool bl_output(const Grid& g, int i, int j) {
  return ((i == g.nx - 2) && (j == g.ny - 2)) || ((i == g.nx - 1) && (j == g.ny - 1)) ||
         ((i == g.nx - 1) && (j == g.ny - 2)) || ((i == g.nx - 2) && (j == g.ny - 1));
}

// data_initialization (b-l.cpp:173-219): S_n = BACKGROUND_Sn, P_w from
// BACKGROUND_Pw at the top down each column, the weight taken with the
// reference densities and the cell's own S_n and m.
void init_bl(const capaz_params* p, const Grid& g, const double* m, double* P_w, double* S_n) {
  for (int i = 0; i < g.nx; i++)
    for (int j = 0; j < g.ny; j++)
      for (int k = 0; k < g.nz; k++) {
        long l = g.at(i, j, k);
        S_n[l] = p->background_Sn;
        double ro_g_dy = (p->ro0_n * S_n[l] + p->ro0_w * (1 - S_n[l])) * (m[l]) * (p->g_const) * (p->hy);
        if (j == 0) P_w[l] = p->background_Pw;
        else P_w[l] = P_w[l - g.sy] + ro_g_dy;
      }
}

void step_bl(const capaz_params* p, const Grid& g, double* P_w, double* S_n, const double* m, const double* K,
             Work& w) {
  double *S_w = w.S_w.data(), *P_n = w.P_n.data(), *ro_w = w.ro_w.data(), *ro_n = w.ro_n.data();
  double *Xi_w = w.Xi_w.data(), *Xi_n = w.Xi_n.data();
  double *roS_w = w.roS_w.data(), *roS_n = w.roS_n.data();
  double *roS_w_old = w.roS_w_old.data(), *roS_n_old = w.roS_n_old.data();

#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) S_w[l] = 1. - S_n[l];

  // assign_P_Xi (b-l.cpp:57-72) and assign_ro (cpu.cpp).
#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) {
    double k_w = 0., k_n = 0.;
    bl_relperm(1. - S_n[l], &k_w, &k_n);
    P_n[l] = P_w[l];
    Xi_w[l] = -1. * Kc(p, K, l) * k_w / p->mu_w;
    Xi_n[l] = -1. * Kc(p, K, l) * k_n / p->mu_n;
    ro_w[l] = p->ro0_w * (1. + (p->beta_w) * (P_w[l] - p->P_atm));
    ro_n[l] = p->ro0_n * (1. + (p->beta_n) * (P_n[l] - p->P_atm));
  }

  // assign_roS_nr (cpu.cpp:619-731) with wells_q (b-l.cpp:239-262).
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        if (!m[l]) continue;
        double q_w = 0., q_n = 0.;
        if (bl_injection(g, i, j)) {
          q_w = p->Q;
          q_n = 0.;
        }
        if (bl_output(g, i, j)) {
          double k_w = 0., k_n = 0.;
          bl_relperm(1. - S_n[l], &k_w, &k_n);
          double F_bl = (k_w / p->mu_w) / (k_w / p->mu_w + k_n / p->mu_n);
          q_w = -1. * p->Q * F_bl;
          q_n = -1. * p->Q * (1. - F_bl);
        }
        roS_w[l] = ro_w[l] * (1. - S_n[l]);
        roS_n[l] = ro_n[l] * S_n[l];
        double x1, x2, fx_w, fy_w, fz_w, fx_n, fy_n, fz_n;
        if (g.nz < 2) {
          fz_w = 0.;
          fz_n = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_w, l, g.sz, p->hz);
          fz_w = directed(x1, x2, Xi_w, ro_w, l, g.sz, p->hz);
          x2 = -1. * rdiff(P_n, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_n, l, g.sz, p->hz);
          fz_n = directed(x1, x2, Xi_n, ro_n, l, g.sz, p->hz);
        }
        if (g.nx < 2) {
          fx_w = 0.;
          fx_n = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_w, l, g.sx, p->hx);
          fx_w = directed(x1, x2, Xi_w, ro_w, l, g.sx, p->hx);
          x2 = -1. * rdiff(P_n, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_n, l, g.sx, p->hx);
          fx_n = directed(x1, x2, Xi_n, ro_n, l, g.sx, p->hx);
        }
        x2 = -1. * rdiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        x1 = -1. * ldiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        fy_w = directed(x1, x2, Xi_w, ro_w, l, g.sy, p->hy);
        x2 = -1. * rdiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        x1 = -1. * ldiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        fy_n = directed(x1, x2, Xi_n, ro_n, l, g.sy, p->hy);
        double A1 = roS_w[l] - (p->dt / m[l]) * (-q_w + fx_w + fy_w + fz_w);
        double A2 = roS_n[l] - (p->dt / m[l]) * (-q_n + fx_n + fy_n + fz_n);
        roS_w_old[l] = roS_w[l];
        roS_n_old[l] = roS_n[l];
        roS_w[l] = A1;
        roS_n[l] = A2;
      }

  // Newton (b-l.cpp:74-102): no capillary pressure.
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        double Pw = P_w[l], Sn = S_n[l];
        for (int it = 1; it <= p->newton_iterations; it++) {
          double F1 = p->ro0_w * (1. + (p->beta_w) * (Pw - p->P_atm)) * (1. - Sn) - roS_w[l];
          double F2 = p->ro0_n * (1. + (p->beta_n) * (Pw - p->P_atm)) * Sn - roS_n[l];
          double F1P = p->ro0_w * (p->beta_w) * (1 - Sn);
          double F2P = p->ro0_n * (p->beta_n) * Sn;
          double F1S = (-1) * (p->ro0_w) * (1 + (p->beta_w) * (Pw - p->P_atm));
          double F2S = p->ro0_n * (1 + (p->beta_n) * (Pw - p->P_atm));
          double det = F1P * F2S - F1S * F2P;
          double nPw = Pw - (1. / det) * (F2S * F1 - F1S * F2);
          double nSn = Sn - (1. / det) * (F1P * F2 - F2P * F1);
          Pw = nPw;
          Sn = nSn;
        }
        P_w[l] = Pw;
        S_n[l] = Sn;
      }

  // boundary_conditions: Border_S and Border_P (b-l.cpp:104-171) on every
  // cell (interior cells are their own basic coordinate), then the wells'
  // pressures.
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        long l1 = g.basic(i, j, k);
        long l = g.at(i, j, k);
        S_n[l] = S_n[l1];
        if ((j != 0) && (j != g.ny - 1)) {
          P_w[l] = P_w[l1];
        } else {
          double ro_g_dy = (p->ro0_n * S_n[l] + p->ro0_w * (1 - S_n[l])) * (m[l]) * (p->g_const) * (p->hy);
          P_w[l] = P_w[l1] + ro_g_dy;
        }
        if (bl_injection(g, i, j)) P_w[l] = p->injwell_Pw;
        if (bl_output(g, i, j)) P_w[l] = p->outwell_Pw;
      }
}

// roS_calculation of the three-phase task, NR form (cpu.cpp:619-731 with
// wells_q three-phase.cpp:529-550, all rates zero): the conserved updates
// roS_p and roS_p_old on interior cells from the ro_P_Xi arrays.
void roS3(const capaz_params* p, const Grid& g, const double* P_w, const double* S_w, const double* S_n,
          const double* P_n, const double* P_g, const double* m, Work& w) {
  double *ro_w = w.ro_w.data(), *ro_n = w.ro_n.data(), *ro_g = w.ro_g.data();
  double *Xi_w = w.Xi_w.data(), *Xi_n = w.Xi_n.data(), *Xi_g = w.Xi_g.data();
  double *roS_w = w.roS_w.data(), *roS_n = w.roS_n.data(), *roS_g = w.roS_g.data();
  double *roS_w_old = w.roS_w_old.data(), *roS_n_old = w.roS_n_old.data(), *roS_g_old = w.roS_g_old.data();
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        if (!m[l]) continue;
        const double q_w = 0., q_n = 0., q_g = 0.;  // wells_q (three-phase.cpp:529-550)
        roS_w[l] = ro_w[l] * S_w[l];
        roS_g[l] = ro_g[l] * (1. - S_w[l] - S_n[l]);
        roS_n[l] = ro_n[l] * S_n[l];
        double x1, x2, fx_w, fy_w, fz_w, fx_n, fy_n, fz_n, fx_g, fy_g, fz_g;
        if (g.nz < 2) {
          fz_w = fz_n = fz_g = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_w, l, g.sz, p->hz);
          fz_w = directed(x1, x2, Xi_w, ro_w, l, g.sz, p->hz);
          x2 = -1. * rdiff(P_n, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_n, l, g.sz, p->hz);
          fz_n = directed(x1, x2, Xi_n, ro_n, l, g.sz, p->hz);
          x2 = -1. * rdiff(P_g, l, g.sz, p->hz);
          x1 = -1. * ldiff(P_g, l, g.sz, p->hz);
          fz_g = directed(x1, x2, Xi_g, ro_g, l, g.sz, p->hz);
        }
        if (g.nx < 2) {
          fx_w = fx_n = fx_g = 0.;
        } else {
          x2 = -1. * rdiff(P_w, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_w, l, g.sx, p->hx);
          fx_w = directed(x1, x2, Xi_w, ro_w, l, g.sx, p->hx);
          x2 = -1. * rdiff(P_n, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_n, l, g.sx, p->hx);
          fx_n = directed(x1, x2, Xi_n, ro_n, l, g.sx, p->hx);
          x2 = -1. * rdiff(P_g, l, g.sx, p->hx);
          x1 = -1. * ldiff(P_g, l, g.sx, p->hx);
          fx_g = directed(x1, x2, Xi_g, ro_g, l, g.sx, p->hx);
        }
        x2 = -1. * rdiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        x1 = -1. * ldiff(P_w, l, g.sy, p->hy) + p->g_const * (ro_w[l]);
        fy_w = directed(x1, x2, Xi_w, ro_w, l, g.sy, p->hy);
        x2 = -1. * rdiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        x1 = -1. * ldiff(P_n, l, g.sy, p->hy) + p->g_const * (ro_n[l]);
        fy_n = directed(x1, x2, Xi_n, ro_n, l, g.sy, p->hy);
        double A1 = roS_w[l] - (p->dt / m[l]) * (-q_w + fx_w + fy_w + fz_w);
        double A2 = roS_n[l] - (p->dt / m[l]) * (-q_n + fx_n + fy_n + fz_n);
        roS_w_old[l] = roS_w[l];
        roS_n_old[l] = roS_n[l];
        roS_w[l] = A1;
        roS_n[l] = A2;
        x2 = -1. * rdiff(P_g, l, g.sy, p->hy) + p->g_const * (ro_g[l]);
        x1 = -1. * ldiff(P_g, l, g.sy, p->hy) + p->g_const * (ro_g[l]);
        fy_g = directed(x1, x2, Xi_g, ro_g, l, g.sy, p->hy);
        double A3 = roS_g[l] - (p->dt / m[l]) * (q_g + fx_g + fy_g + fz_g);
        roS_g_old[l] = roS_g[l];
        roS_g[l] = A3;
      }

}

// Border_P of the three-phase task (three-phase.cpp:362-427) for boundary cell
// l with basic coordinate l1, capillary pressures zero.
void border_P3(const capaz_params* p, int j, int ny, double* P_w, double* P_n, double* P_g, long l, long l1) {
  const double Pk_nw = 0, Pk_gn = 0;
  if ((j != 0) && (j != ny - 1)) {
    P_w[l] = P_w[l1];
    P_n[l] = P_w[l1] + Pk_nw;
    P_g[l] = P_w[l1] + Pk_nw + Pk_gn;
  } else if (j == 0) {
    P_w[l] = (P_w[l1] - (p->ro0_w) * (p->g_const) * (p->hy) * (1. - (p->beta_w) * (p->P_atm))) /
             (1. + (p->beta_w) * (p->ro0_w) * (p->g_const) * (p->hy));
    P_n[l] = (P_w[l1] + Pk_nw - (p->ro0_n) * (p->g_const) * (p->hy) * (1. - (p->beta_n) * (p->P_atm))) /
             (1. + (p->beta_n) * (p->ro0_n) * (p->g_const) * (p->hy));
    P_g[l] = (P_w[l1] + Pk_nw + Pk_gn) / (1. + (p->ro0_g) * (p->g_const) * (p->hy) / (p->P_atm));
  } else {
    P_w[l] = (P_w[l1] + (p->ro0_w) * (p->g_const) * (p->hy) * (1. - (p->beta_w) * (p->P_atm))) /
             (1. - (p->beta_w) * (p->ro0_w) * (p->g_const) * (p->hy));
    P_n[l] = (P_w[l1] + Pk_nw + (p->ro0_n) * (p->g_const) * (p->hy) * (1. - (p->beta_n) * (p->P_atm))) /
             (1. - (p->beta_n) * (p->ro0_n) * (p->g_const) * (p->hy));
    P_g[l] = (P_w[l1] + Pk_nw + Pk_gn) / (1. - (p->ro0_g) * (p->g_const) * (p->hy) / (p->P_atm));
  }
}

// ---------------------------------------------------------------------------
// Three-phase step (CPU physics).
void step3(const capaz_params* p, const Grid& g, double* P_w, double* S_w, double* S_n, double* P_n,
           double* P_g, const double* m, const double* K, Work& w) {
  const double A = p->lambda;
  const double den = 1. - p->S_wr - p->S_nr - p->S_gr;
  double *S_g = w.S_g.data(), *ro_w = w.ro_w.data(), *ro_n = w.ro_n.data(), *ro_g = w.ro_g.data();
  double *Xi_w = w.Xi_w.data(), *Xi_n = w.Xi_n.data(), *Xi_g = w.Xi_g.data();
  double *roS_w = w.roS_w.data(), *roS_n = w.roS_n.data(), *roS_g = w.roS_g.data();
  double *roS_w_old = w.roS_w_old.data(), *roS_n_old = w.roS_n_old.data(), *roS_g_old = w.roS_g_old.data();

  // S_calculation (all cells).
#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) S_g[l] = 1. - S_w[l] - S_n[l];

  // ro_P_Xi_calculation: Xi and rho on all cells, P_n and P_g on interior
  // cells only (three-phase.cpp:225-235).
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        long l = g.at(i, j, k);
        double S_w_e = (S_w[l] - p->S_wr) / den;
        double S_n_e = (S_n[l] - p->S_nr) / den;
        double S_g_e = 1. - S_w_e - S_n_e;
        double k_w = k_w3(S_w_e, A), k_g = k_g3(S_g_e, A), k_n = k_n3(S_w_e, S_n_e, A);
        double Kl = Kc(p, K, l);
        Xi_w[l] = (-1.) * Kl * k_w / p->mu_w;
        Xi_n[l] = (-1.) * Kl * k_n / p->mu_n;
        Xi_g[l] = (-1.) * Kl * k_g / p->mu_g;
        if (g.interior(i, j, k)) {
          const double Pk_nw = 0, Pk_gn = 0;
          P_n[l] = P_w[l] + Pk_nw;
          P_g[l] = P_w[l] + Pk_nw + Pk_gn;
        }
        ro_w[l] = p->ro0_w * (1. + (p->beta_w) * (P_w[l] - p->P_atm));
        ro_n[l] = p->ro0_n * (1. + (p->beta_n) * (P_n[l] - p->P_atm));
        ro_g[l] = p->ro0_g * P_g[l] / p->P_atm;
      }
  if (w.keep_u_pressures) {
    w.Pn_u.assign(P_n, P_n + g.n);
    w.Pg_u.assign(P_g, P_g + g.n);
  }

  roS3(p, g, P_w, S_w, S_n, P_n, P_g, m, w);

  // P_S_calculation: 3x3 Newton (three-phase.cpp:286-339).
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        double Pw = P_w[l], Sw = S_w[l], Sn = S_n[l];
        for (int it = 1; it <= p->newton_iterations; it++) {
          const double Pk_nw = 0, Pk_gn = 0, PkSw = 0, PkSn = 0;
          double Sg = 1. - Sw - Sn;
          double F1 = p->ro0_w * (1. + (p->beta_w) * (Pw - p->P_atm)) * Sw - roS_w[l];
          double F2 = p->ro0_n * (1. + (p->beta_n) * (Pw + Pk_nw - p->P_atm)) * Sn - roS_n[l];
          double F3 = p->ro0_g * (Pw + Pk_nw + Pk_gn) / p->P_atm * Sg - roS_g[l];
          double dF[9];
          dF[0] = p->ro0_w * p->beta_w * Sw;
          dF[3] = p->ro0_n * p->beta_n * Sn;
          dF[6] = p->ro0_g * Sg / p->P_atm;
          dF[1] = p->ro0_w * (1 + p->beta_w * (Pw - p->P_atm));
          dF[4] = p->ro0_n * (1. + (p->beta_n) * PkSw) * Sn;
          dF[7] = (-1) * p->ro0_g * (Pw + Pk_nw + Pk_gn - Sg * (PkSn + PkSw)) / p->P_atm;
          dF[2] = 0;
          dF[5] = p->ro0_n * (1. + p->beta_n * (Pw + Pk_nw - p->P_atm));
          dF[8] = (-1) * p->ro0_g * (Pw + Pk_nw + Pk_gn - Sg * PkSn) / p->P_atm;
          reverse_matrix(dF, 3);
          double nPw = Pw - (dF[0] * F1 + dF[1] * F2 + dF[2] * F3);
          double nSw = Sw - (dF[3] * F1 + dF[4] * F2 + dF[5] * F3);
          double nSn = Sn - (dF[6] * F1 + dF[7] * F2 + dF[8] * F3);
          Pw = nPw;
          Sw = nSw;
          Sn = nSn;
        }
        P_w[l] = Pw;
        S_w[l] = Sw;
        S_n[l] = Sn;
      }

  // boundary_conditions (three-phase.cpp:345-427).
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        bool bnd = (((i == 0) || (i == g.nx - 1)) && (g.nx >= 2)) || (j == 0) || (j == g.ny - 1) ||
                   (((k == 0) || (k == g.nz - 1)) && (g.nz >= 2));
        if (!bnd) continue;
        long l1 = g.basic(i, j, k);
        long l = g.at(i, j, k);
        // With CAPAZ_FLAG_SOURCE_WINDOW (extension) only the SOURCE window of
        // the top face is a source; without it, the whole face, as written.
        const bool src = (j == 0) && (p->source > 0) &&
                         (!(p->flags & CAPAZ_FLAG_SOURCE_WINDOW) || in_window(p, i, k));
        if (!src) {
          S_w[l] = S_w[l1];
          S_n[l] = S_n[l1];
        } else {
          S_w[l] = p->S_w_gr;
          S_n[l] = p->S_n_gr;
        }
        border_P3(p, j, g.ny, P_w, P_n, P_g, l, l1);
      }
}

// ---------------------------------------------------------------------------
// Three-phase step with the energy equation (THREE_PHASE + ENERGY build).
// Constants are energy.cpp:1-30's globals (T_0 also assign_ro's local,
// cpu.cpp:120-123); temperatures of the initial state and of the top and
// bottom rows are three-phase.cpp:487 and energy.cpp:404-411.
namespace en {
const double T_0 = 273., ro_r = 2000.;
const double lambda0_w = 0.553, lambda0_n = 0.14, lambda0_g = 0.0237, lambda0_r = 1.;
const double lambdaA_w = 3E-3, lambdaA_n = 1E-3, lambdaA_g = 0.82;
const double c0_w = 4.194E3, c0_n = 1.7E3, c0_g = 1E3, c0_r = 0.8E3;
const double C_w = 1.15, C_w2 = 0.015, C_n = 3.4, C_g = 0.119, C_r = 0.75;
const double alfa_w = 1.32E-7, alfa_n = 9.2E-7;
const double T_init = 285., T_top = 400., T_bottom = 273.;

// Specific heats (energy.cpp:33-51) and enthalpies (energy.cpp:84-140).
inline double c_w(double T) { return c0_w - C_w * (T - T_0) + C_w2 * (T - T_0) * (T - T_0); }
inline double c_n(double T) { return c0_n + C_n * (T - T_0); }
inline double c_g(double T) { return c0_g + C_g * (T - T_0); }
inline double c_r(double T) { return c0_r + C_r * (T - T_0); }
inline double H_w(const capaz_params* p, double T) {
  return (p->P_atm / p->ro0_w) + (T - T_0) * (c0_w - (T - T_0) * (C_w / 2 + C_w2 * (T - T_0) / 3));
}
inline double H_n(const capaz_params* p, double T) { return (p->P_atm / p->ro0_n) + (T - T_0) * (c0_n + C_n * (T - T_0) / 2); }
inline double H_g(const capaz_params* p, double T) { return (p->P_atm / p->ro0_g) + (T - T_0) * (c0_g + C_g * (T - T_0) / 2); }
inline double H_r(const capaz_params* p, double T) { return (p->P_atm / ro_r) + (T - T_0) * (c0_r + C_r * (T - T_0) / 2); }
// Effective heat conductivity (energy.cpp:54-81).
inline double lam_eff(double m, double Sw, double Sn, double Sg, double T) {
  return m * (Sw * (lambda0_w * (1 - lambdaA_w * (T - T_0))) + Sn * (lambda0_n * (1 - lambdaA_n * (T - T_0))) +
              Sg * (lambda0_g * pow((T / T_0), lambdaA_g))) +
         (1. - m) * lambda0_r;
}
// Densities of (P, T) and their derivatives (energy.cpp:143-228).
inline double ro_w(const capaz_params* p, double P, double T) {
  return p->ro0_w * (1. + (p->beta_w) * (P - p->P_atm) - alfa_w * (T - T_0));
}
inline double ro_n(const capaz_params* p, double P, double T) {
  return p->ro0_n * (1. + (p->beta_n) * (P - p->P_atm) - alfa_n * (T - T_0));
}
inline double ro_g(const capaz_params* p, double P, double T) { return p->ro0_g * (P / p->P_atm) * (T_0 / T); }
}  // namespace en

void velocities(const capaz_params* p, const Grid& g, const double* P, const double* Xi, const double* ro,
                double* ux, double* uy, double* uz);

struct WorkE {
  std::vector<double> H_w, H_n, H_g, H_r, E, E_new, lam;
  std::vector<double> ux_w, uy_w, uz_w, ux_n, uy_n, uz_n, ux_g, uy_g, uz_g;
};

// One step of the energy build's time_step_function (main.cpp:93-108):
// S, ro/P/Xi (temperature-dependent viscosities three-phase.cpp:210-215 and
// densities cpu.cpp:118-127), u, roS (as three-phase), H and E at the current
// state (cpu.cpp:38-49), E_new (cpu.cpp:67-77, energy.cpp:232-343), the 5x5
// Newton in (S_w, S_n, S_g, P_w, T) (energy.cpp:348-462) and the boundary
// rules (three-phase.cpp:345-427, energy.cpp:396-418).
void step3e(const capaz_params* p, const Grid& g, double* P_w, double* S_w, double* S_n, double* P_n, double* P_g,
            double* T, const double* m, const double* K, Work& w, WorkE& e) {
  using namespace en;
  const double A = p->lambda;
  const double den = 1. - p->S_wr - p->S_nr - p->S_gr;
  double *S_g = w.S_g.data(), *rw = w.ro_w.data(), *rn = w.ro_n.data(), *rg = w.ro_g.data();
  double *Xi_w = w.Xi_w.data(), *Xi_n = w.Xi_n.data(), *Xi_g = w.Xi_g.data();
  double *roS_w = w.roS_w.data(), *roS_n = w.roS_n.data(), *roS_g = w.roS_g.data();

#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) S_g[l] = 1. - S_w[l] - S_n[l];

#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        long l = g.at(i, j, k);
        double S_w_e = (S_w[l] - p->S_wr) / den;
        double S_n_e = (S_n[l] - p->S_nr) / den;
        double S_g_e = 1. - S_w_e - S_n_e;
        double k_w = k_w3(S_w_e, A), k_g = k_g3(S_g_e, A), k_n = k_n3(S_w_e, S_n_e, A);
        double mu_w = 1. / (29.21 * T[l] - 7506.64);
        double mu_n = 7.256E-10 * exp(4141.9 / T[l]);
        double mu_g = 1.717E-5 * pow((T[l] / 273.), 0.683);
        double Kl = Kc(p, K, l);
        Xi_w[l] = (-1.) * Kl * k_w / mu_w;
        Xi_n[l] = (-1.) * Kl * k_n / mu_n;
        Xi_g[l] = (-1.) * Kl * k_g / mu_g;
        if (g.interior(i, j, k)) {
          const double Pk_nw = 0, Pk_gn = 0;
          P_n[l] = P_w[l] + Pk_nw;
          P_g[l] = P_w[l] + Pk_nw + Pk_gn;
        }
        rw[l] = ro_w(p, P_w[l], T[l]);
        rn[l] = ro_n(p, P_n[l], T[l]);
        rg[l] = ro_g(p, P_g[l], T[l]);
      }

  velocities(p, g, P_w, Xi_w, rw, e.ux_w.data(), e.uy_w.data(), e.uz_w.data());
  velocities(p, g, P_n, Xi_n, rn, e.ux_n.data(), e.uy_n.data(), e.uz_n.data());
  velocities(p, g, P_g, Xi_g, rg, e.ux_g.data(), e.uy_g.data(), e.uz_g.data());

  roS3(p, g, P_w, S_w, S_n, P_n, P_g, m, w);

  // H_E_current_calculation (all cells).
  double *Hw = e.H_w.data(), *Hn = e.H_n.data(), *Hg = e.H_g.data(), *Hr = e.H_r.data();
  double *E = e.E.data(), *E_new = e.E_new.data(), *lam = e.lam.data();
#pragma omp parallel for schedule(static)
  for (long l = 0; l < g.n; l++) {
    Hw[l] = H_w(p, T[l]);
    Hn[l] = H_n(p, T[l]);
    Hg[l] = H_g(p, T[l]);
    Hr[l] = H_r(p, T[l]);
    E[l] = (m[l] * (S_w[l] * (rw[l] * Hw[l] - P_w[l]) + S_n[l] * (rn[l] * Hn[l] - P_n[l]) +
                    S_g[l] * (rg[l] * Hg[l] - P_g[l])) +
            (1. - m[l]) * (ro_r * Hr[l] - P_w[l]));
    lam[l] = lam_eff(m[l], S_w[l], S_n[l], S_g[l], T[l]);
  }

  // E_calculation: E_new = E + dt (T_flow + Q_hw + Q_hr - E_flow) on
  // interior cells; the z term of T_flow replaces the sum, the z term of
  // E_flow takes the y velocities (energy.cpp:256-261, 302-311, as written).
  const double *uxw = e.ux_w.data(), *uyw = e.uy_w.data(), *uxn = e.ux_n.data(), *uyn = e.uy_n.data();
  const double *uxg = e.ux_g.data(), *uyg = e.uy_g.data();
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        double Tf = 0;
        if (g.nx > 2)
          Tf += (lam[l + 1] * T[l + 1] - 2 * lam[l] * T[l] + lam[l - 1] * T[l - 1]) / ((p->hx) * (p->hx));
        if (g.ny > 2)
          Tf += (lam[l + g.sy] * T[l + g.sy] - 2 * lam[l] * T[l] + lam[l - g.sy] * T[l - g.sy]) / ((p->hy) * (p->hy));
        if (g.nz > 2)
          Tf = (lam[l + g.sz] * T[l + g.sz] - 2 * lam[l] * T[l] + lam[l - g.sz] * T[l - g.sz]) / ((p->hz) * (p->hz));
        auto flux = [&](long s, const double* uw, const double* un, const double* ug, double h) {
          return (rw[l + s] * Hw[l + s] * uw[l + s] - rw[l - s] * Hw[l - s] * uw[l - s] +
                  rn[l + s] * Hn[l + s] * un[l + s] - rn[l - s] * Hn[l - s] * un[l - s] +
                  rg[l + s] * Hg[l + s] * ug[l + s] - rg[l - s] * Hg[l - s] * ug[l - s]) /
                 (2. * h);
        };
        double Ef = 0;
        if (g.nx > 2) Ef += flux(g.sx, uxw, uxn, uxg, p->hx);
        if (g.ny > 2) Ef += flux(g.sy, uyw, uyn, uyg, p->hy);
        if (g.nz > 2) Ef += flux(g.sz, uyw, uyn, uyg, p->hz);
        const double Q_hw = 0, Q_hr = 0;
        E_new[l] = E[l] + (p->dt) * (Tf + Q_hw + Q_hr - Ef);
      }

  // P_S_calculation: the 5x5 Newton with reverse_matrix and
  // mult_matrix_vector (gauss.cpp:6-104); rows F0..F4, columns
  // d/d(S_w, S_n, S_g, P, T).  reverse_matrix leaves dF as it is when it
  // finds no pivot, and the reference uses dF all the same.
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        if (!g.interior(i, j, k)) continue;
        long l = g.at(i, j, k);
        const int n = 5;
        const double ml = m[l];
        for (int it = 1; it <= p->newton_iterations; it++) {
          const double P = P_w[l], Tl = T[l], Sw = S_w[l], Sn = S_n[l], Sg = S_g[l];
          double F[5], dF[25], c[5];
          F[0] = Sg + Sw + Sn - 1.;
          F[1] = ro_w(p, P, Tl) * Sw - roS_w[l];
          F[2] = ro_n(p, P, Tl) * Sn - roS_n[l];
          F[3] = ro_g(p, P, Tl) * Sg - roS_g[l];
          F[4] = ml * (Sw * (ro_w(p, P, Tl) * Hw[l] - P) + Sn * (ro_n(p, P, Tl) * Hn[l] - P) +
                       Sg * (ro_g(p, P, Tl) * Hg[l] - P)) +
                 (1. - ml) * (ro_r * Hr[l] - P) - E_new[l];
          const double dwP = p->ro0_w * (p->beta_w), dwT = (-1) * p->ro0_w * alfa_w;
          const double dnP = p->ro0_n * (p->beta_n), dnT = (-1) * p->ro0_n * alfa_n;
          const double dgP = (p->ro0_g / p->P_atm) * (T_0 / Tl);
          const double dgT = p->ro0_g * (P / p->P_atm) * (-1) * (T_0 / Tl) / Tl;
          dF[0] = 1.;
          dF[1] = 1.;
          dF[2] = 1.;
          dF[3] = 0.;
          dF[4] = 0.;
          dF[0 + n] = ro_w(p, P, Tl);
          dF[1 + n] = 0.;
          dF[2 + n] = 0.;
          dF[3 + n] = dwP * Sw;
          dF[4 + n] = dwT * Sw;
          dF[0 + n * 2] = 0.;
          dF[1 + n * 2] = ro_n(p, P, Tl);
          dF[2 + n * 2] = 0.;
          dF[3 + n * 2] = dnP * Sn;
          dF[4 + n * 2] = dnT * Sn;
          dF[0 + n * 3] = 0.;
          dF[1 + n * 3] = 0.;
          dF[2 + n * 3] = ro_g(p, P, Tl);
          dF[3 + n * 3] = dgP * Sg;
          dF[4 + n * 3] = dgT * Sg;
          dF[0 + n * 4] = ml * (ro_w(p, P, Tl) * Hw[l] - P);
          dF[1 + n * 4] = ml * (ro_n(p, P, Tl) * Hn[l] - P);
          dF[2 + n * 4] = ml * (ro_g(p, P, Tl) * Hg[l] - P);
          dF[3 + n * 4] = ml * (Sw * (dwP * Hw[l] - 1.) + Sn * (dnP * Hn[l] - 1.) + Sg * (dgP * Hg[l] - 1.)) +
                          (1. - ml) * (-1);
          dF[4 + n * 4] = ml * (Sw * (dwT * Hw[l] + ro_w(p, P, Tl) * c_w(Tl)) +
                                Sn * (dnT * Hn[l] + ro_n(p, P, Tl) * c_n(Tl)) +
                                Sg * (dgT * Hg[l] + ro_g(p, P, Tl) * c_g(Tl))) +
                          (1. - ml) * ro_r * c_r(Tl);
          reverse_matrix(dF, n);
          for (int a = 0; a < n; a++) {
            c[a] = 0;
            for (int b = 0; b < n; b++) c[a] += dF[b + n * a] * F[b];
          }
          S_w[l] = Sw - c[0];
          S_n[l] = Sn - c[1];
          S_g[l] = Sg - c[2];
          P_w[l] = P - c[3];
          T[l] = Tl - c[4];
          Hw[l] = H_w(p, T[l]);
          Hn[l] = H_n(p, T[l]);
          Hg[l] = H_g(p, T[l]);
          Hr[l] = H_r(p, T[l]);
        }
        E[l] = E_new[l];
      }

  // boundary_conditions: Border_S, Border_P (three-phase), Border_T.
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        bool bnd = (((i == 0) || (i == g.nx - 1)) && (g.nx >= 2)) || (j == 0) || (j == g.ny - 1) ||
                   (((k == 0) || (k == g.nz - 1)) && (g.nz >= 2));
        if (!bnd) continue;
        long l1 = g.basic(i, j, k);
        long l = g.at(i, j, k);
        const bool src = (j == 0) && (p->source > 0) &&
                         (!(p->flags & CAPAZ_FLAG_SOURCE_WINDOW) || in_window(p, i, k));
        if (!src) {
          S_w[l] = S_w[l1];
          S_n[l] = S_n[l1];
        } else {
          S_w[l] = p->S_w_gr;
          S_n[l] = p->S_n_gr;
        }
        border_P3(p, j, g.ny, P_w, P_n, P_g, l, l1);
        if (j == 0) T[l] = T_top;
        else if (j == g.ny - 1) T[l] = T_bottom;
        else T[l] = T[l1];
      }
}

// u_calculation (cpu.cpp:346-477) for one phase, from the start-of-step arrays.
void velocities(const capaz_params* p, const Grid& g, const double* P, const double* Xi, const double* ro,
                double* ux, double* uy, double* uz) {
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++)
      for (int i = 0; i < g.nx; i++) {
        long l = g.at(i, j, k);
        if (p->nx > 2) {
          if (i == 0) ux[l] = Xi[l] * rdiff(P, l, g.sx, p->hx);
          else if (i == g.nx - 1) ux[l] = Xi[l] * ldiff(P, l, g.sx, p->hx);
          else ux[l] = Xi[l] * cdiff(P, l, g.sx, p->hx);
        } else {
          ux[l] = 0.;
        }
        if (p->ny > 2) {
          if (j == 0) uy[l] = Xi[l] * (rdiff(P, l, g.sy, p->hy) - ro[l] * (p->g_const));
          else if (j == g.ny - 1) uy[l] = Xi[l] * (ldiff(P, l, g.sy, p->hy) - ro[l] * (p->g_const));
          else uy[l] = Xi[l] * (cdiff(P, l, g.sy, p->hy) - ro[l] * (p->g_const));
        } else {
          uy[l] = 0.;
        }
        if (p->nz > 2) {
          if (k == 0) uz[l] = Xi[l] * rdiff(P, l, g.sz, p->hz);
          else if (k == g.nz - 1) uz[l] = Xi[l] * ldiff(P, l, g.sz, p->hz);
          else uz[l] = Xi[l] * cdiff(P, l, g.sz, p->hz);
        } else {
          uz[l] = 0.;
        }
      }
}

// Two-phase data_initialization (two-phase.cu:6-65 as the GPU build runs
// it): S_n from the injection window, P_w hydrostatic down each column with
// the porosity inside the weight (P[j] = P[j-1] + rho_eff(j-1) m(j-1) g hy).
template <class T>
void init2(const capaz_params* p, const Grid& g, const T* m, T* P_w, T* S_n) {
  std::vector<T> ro_w(g.n), ro_n(g.n);
  for (int i = 0; i < g.nx; i++)
    for (int j = 0; j < g.ny; j++)
      for (int k = 0; k < g.nz; k++) {
        long l = g.at(i, j, k);
        if ((j == 0) && in_window(p, i, k)) S_n[l] = p->S_n_gr;
        else S_n[l] = p->S_n_background;
        if (j == 0) {
          P_w[l] = p->P_atm;
        } else {
          long u = l - g.sy;
          T ro_g_dy = (ro_n[u] * S_n[u] + ro_w[u] * (1 - S_n[u])) * (m[u]) * (p->g_const) * (p->hy);
          P_w[l] = P_w[u] + ro_g_dy;
        }
        ro_w[l] = p->ro0_w * (1. + (p->beta_w) * (P_w[l] - p->P_atm));
        ro_n[l] = p->ro0_n * (1. + (p->beta_n) * (P_w[l] - p->P_atm));
      }
}

int check_grid(const capaz_params* p) {
  if (!p) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (p->phases != 2 && p->phases != 3) return CAPAZ_ERR_INVALID_ARGUMENT;
  // nx == 1 is the reference's three-phase column case (Three-phase/defines.ini).
  const bool nx_ok = p->nx >= 3 || (p->phases == 3 && p->nx == 1);
  if (!nx_ok || p->ny < 3 || p->nz < 1 || p->nz == 2) return CAPAZ_ERR_UNSUPPORTED_GRID;
  return CAPAZ_OK;
}

}  // namespace

extern "C" {

// Gauss-Jordan inverse of gauss.cpp:6-92 (row-major n x n, in place).
int oracle_reverse_matrix(double* a, int n) { return reverse_matrix(a, n); }

// data_initialization.  `m` (in/out): if m_in is non-NULL it gives the
// porosity per cell, else M_0 is written everywhere.  Two-phase writes P_w,
// S_n; three-phase also S_w, P_n, P_g.
int oracle_init(const capaz_params* p, const double* m_in, double* m, double* P_w, double* S_w,
                double* S_n, double* P_n, double* P_g) {
  int rc = check_grid(p);
  if (rc) return rc;
  Grid g(p);
  if (p->phases == 2) {
    for (long l = 0; l < g.n; l++) m[l] = m_in ? m_in[l] : p->porosity;
    if (p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT) init_bl(p, g, m, P_w, S_n);
    else init2(p, g, m, P_w, S_n);
  } else {
    for (long l = 0; l < g.n; l++) {
      m[l] = m_in ? m_in[l] : p->porosity;
      S_w[l] = p->S_w_init;
      S_n[l] = p->S_n_init;
      P_w[l] = p->P_atm;
      P_n[l] = p->P_atm;
      P_g[l] = p->P_atm;
    }
  }
  return CAPAZ_OK;
}

// Advances nsteps.  Two-phase: P_w, S_n in/out (S_w, P_n, P_g may be NULL).
// Three-phase: P_w, S_w, S_n, P_n, P_g in/out.  K may be NULL (uniform K0).
// `derived`, if non-NULL, is an array of CAPAZ_FIELD_COUNT pointers (entries
// may be NULL) that receive the derived fields of the LAST step, as the
// reference's arrays hold them after time_step_function returns.
// `diag`, if non-NULL, receives the diagnostics of the last step.
int oracle_step(const capaz_params* p, int nsteps, double* P_w, double* S_w, double* S_n, double* P_n,
                double* P_g, const double* m, const double* K, double** derived, capaz_diag* diag,
                int nthreads) {
  int rc = check_grid(p);
  if (rc) return rc;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Grid g(p);
  Work w;
  const long n = g.n;
  w.S_w.assign(n, 0.);
  w.P_n.assign(n, 0.);
  w.ro_w.assign(n, 0.);
  w.ro_n.assign(n, 0.);
  w.Xi_w.assign(n, 0.);
  w.Xi_n.assign(n, 0.);
  w.roS_w.assign(n, 0.);
  w.roS_n.assign(n, 0.);
  w.roS_w_old.assign(n, 0.);
  w.roS_n_old.assign(n, 0.);
  if (p->phases == 3) {
    w.S_g.assign(n, 0.);
    w.ro_g.assign(n, 0.);
    w.Xi_g.assign(n, 0.);
    w.roS_g.assign(n, 0.);
    w.roS_g_old.assign(n, 0.);
  }
  // Keep the start-of-step state of the last step for the velocities.
  std::vector<double> Pw0;
  for (int s = 0; s < nsteps; s++) {
    bool last = (s == nsteps - 1);
    if (last && derived) {
      Pw0.assign(P_w, P_w + n);
      w.keep_u_pressures = (p->phases == 3);
    }
    if (p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT) step_bl(p, g, P_w, S_n, m, K, w);
    else if (p->phases == 2) step2(p, g, P_w, S_n, m, K, w);
    else step3(p, g, P_w, S_w, S_n, P_n, P_g, m, K, w);
  }
  if (derived && nsteps > 0) {
    auto put = [&](int f, const std::vector<double>& v) {
      if (derived[f] && !v.empty()) memcpy(derived[f], v.data(), sizeof(double) * n);
    };
    if (p->phases == 2) {
      put(CAPAZ_FIELD_S_W, w.S_w);
      put(CAPAZ_FIELD_P_N, w.P_n);
    } else {
      put(CAPAZ_FIELD_S_G, w.S_g);
      put(CAPAZ_FIELD_RO_G, w.ro_g);
      put(CAPAZ_FIELD_XI_G, w.Xi_g);
      put(CAPAZ_FIELD_ROS_G, w.roS_g);
      put(CAPAZ_FIELD_ROS_G_OLD, w.roS_g_old);
    }
    put(CAPAZ_FIELD_RO_W, w.ro_w);
    put(CAPAZ_FIELD_RO_N, w.ro_n);
    put(CAPAZ_FIELD_XI_W, w.Xi_w);
    put(CAPAZ_FIELD_XI_N, w.Xi_n);
    put(CAPAZ_FIELD_ROS_W, w.roS_w);
    put(CAPAZ_FIELD_ROS_N, w.roS_n);
    put(CAPAZ_FIELD_ROS_W_OLD, w.roS_w_old);
    put(CAPAZ_FIELD_ROS_N_OLD, w.roS_n_old);
    // Velocities from the start-of-step pressures (P_n for two-phase is the
    // start-of-step value held in w.P_n).
    std::vector<double> tx(n), ty(n), tz(n);
    auto vel = [&](const double* P, const std::vector<double>& Xi, const std::vector<double>& ro, int fx) {
      velocities(p, g, P, Xi.data(), ro.data(), tx.data(), ty.data(), tz.data());
      put(fx, tx);
      put(fx + 1, ty);
      put(fx + 2, tz);
    };
    vel(Pw0.data(), w.Xi_w, w.ro_w, CAPAZ_FIELD_UX_W);
    if (p->phases == 2) {
      vel(w.P_n.data(), w.Xi_n, w.ro_n, CAPAZ_FIELD_UX_N);
    } else {
      vel(w.Pn_u.data(), w.Xi_n, w.ro_n, CAPAZ_FIELD_UX_N);
      vel(w.Pg_u.data(), w.Xi_g, w.ro_g, CAPAZ_FIELD_UX_G);
    }
  }
  if (diag) {
    // Diagnostics of the final state, summed per k-plane then over planes in
    // order (deterministic for any thread count).
    memset(diag, 0, sizeof *diag);
    const double V = p->hx * p->hy * p->hz;
    std::vector<double> pm(3 * (size_t)g.nz, 0.), pr(g.nz, 0.), pnf(g.nz, 0.);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g.nz; k++) {
      double s0 = 0, s1 = 0, s2 = 0, r = 0, nf = 0;
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) {
          if (!g.interior(i, j, k)) continue;
          long l = g.at(i, j, k);
          double Pw = P_w[l], Sn = S_n[l];
          double rw = p->ro0_w * (1. + (p->beta_w) * (Pw - p->P_atm));
          if (p->phases == 2) {
            double S_e = (1 - Sn - p->S_wr) / (1 - p->S_wr);
            double Pk = (p->P_d != 0. && p->model != CAPAZ_MODEL_BUCKLEY_LEVERETT)
                            ? p->P_d * pow(S_e, (-1.) / p->lambda) : 0.;
            double rn = p->ro0_n * (1. + (p->beta_n) * (Pw + Pk - p->P_atm));
            double F1 = rw * (1. - Sn) - w.roS_w[l];
            double F2 = rn * Sn - w.roS_n[l];
            s0 += m[l] * rw * (1. - Sn) * V;
            s1 += m[l] * rn * Sn * V;
            double rr = fmax(fabs(F1) / p->ro0_w, fabs(F2) / p->ro0_n);
            if (!(rr <= r)) r = rr;
            if (!isfinite(Pw) || !isfinite(Sn)) nf += 1;
          } else {
            double Sw = S_w[l], Sg = 1. - Sw - Sn;
            double rn = p->ro0_n * (1. + (p->beta_n) * (Pw - p->P_atm));
            double rg = p->ro0_g * Pw / p->P_atm;
            double F1 = rw * Sw - w.roS_w[l];
            double F2 = rn * Sn - w.roS_n[l];
            double F3 = rg * Sg - w.roS_g[l];
            s0 += m[l] * rw * Sw * V;
            s1 += m[l] * rn * Sn * V;
            s2 += m[l] * rg * Sg * V;
            double rr = fmax(fmax(fabs(F1) / p->ro0_w, fabs(F2) / p->ro0_n), fabs(F3) / p->ro0_g);
            if (!(rr <= r)) r = rr;
            if (!isfinite(Pw) || !isfinite(Sn) || !isfinite(Sw)) nf += 1;
          }
        }
      pm[3 * k] = s0;
      pm[3 * k + 1] = s1;
      pm[3 * k + 2] = s2;
      pr[k] = r;
      pnf[k] = nf;
    }
    for (int k = 0; k < g.nz; k++) {
      diag->mass[0] += pm[3 * k];
      diag->mass[1] += pm[3 * k + 1];
      diag->mass[2] += pm[3 * k + 2];
      if (!(pr[k] <= diag->max_residual)) diag->max_residual = pr[k];
      diag->nonfinite_cells += pnf[k];
    }
  }
  return CAPAZ_OK;
}

// Energy model (CAPAZ_MODEL_ENERGY): the initial temperature of
// data_initialization (three-phase.cpp:485-490) on every cell.
int oracle_init_temperature(const capaz_params* p, double* T) {
  int rc = check_grid(p);
  if (rc) return rc;
  Grid g(p);
  for (long l = 0; l < g.n; l++) T[l] = en::T_init;
  return CAPAZ_OK;
}

// Energy model: advances nsteps; P_w, S_w, S_n, P_n, P_g, T in/out.
// `derived` as for oracle_step: the reference's other arrays after the last
// step (S_g, rho, Xi, u, roS, roS_old, H, E, E_new).
int oracle_step_energy(const capaz_params* p, int nsteps, double* P_w, double* S_w, double* S_n, double* P_n,
                       double* P_g, double* T, const double* m, const double* K, double** derived, int nthreads) {
  int rc = check_grid(p);
  if (rc) return rc;
  if (p->phases != 3) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Grid g(p);
  const long n = g.n;
  Work w;
  WorkE e;
  for (auto* v : {&w.S_g, &w.ro_w, &w.ro_n, &w.ro_g, &w.Xi_w, &w.Xi_n, &w.Xi_g, &w.roS_w, &w.roS_n, &w.roS_g,
                  &w.roS_w_old, &w.roS_n_old, &w.roS_g_old})
    v->assign(n, 0.);
  for (auto* v : {&e.H_w, &e.H_n, &e.H_g, &e.H_r, &e.E, &e.E_new, &e.lam, &e.ux_w, &e.uy_w, &e.uz_w, &e.ux_n,
                  &e.uy_n, &e.uz_n, &e.ux_g, &e.uy_g, &e.uz_g})
    v->assign(n, 0.);
  for (int s = 0; s < nsteps; s++) step3e(p, g, P_w, S_w, S_n, P_n, P_g, T, m, K, w, e);
  if (derived && nsteps > 0) {
    auto put = [&](int f, const std::vector<double>& v) {
      if (derived[f]) memcpy(derived[f], v.data(), sizeof(double) * n);
    };
    put(CAPAZ_FIELD_S_G, w.S_g);
    put(CAPAZ_FIELD_RO_W, w.ro_w);
    put(CAPAZ_FIELD_RO_N, w.ro_n);
    put(CAPAZ_FIELD_RO_G, w.ro_g);
    put(CAPAZ_FIELD_XI_W, w.Xi_w);
    put(CAPAZ_FIELD_XI_N, w.Xi_n);
    put(CAPAZ_FIELD_XI_G, w.Xi_g);
    put(CAPAZ_FIELD_UX_W, e.ux_w);
    put(CAPAZ_FIELD_UY_W, e.uy_w);
    put(CAPAZ_FIELD_UZ_W, e.uz_w);
    put(CAPAZ_FIELD_UX_N, e.ux_n);
    put(CAPAZ_FIELD_UY_N, e.uy_n);
    put(CAPAZ_FIELD_UZ_N, e.uz_n);
    put(CAPAZ_FIELD_UX_G, e.ux_g);
    put(CAPAZ_FIELD_UY_G, e.uy_g);
    put(CAPAZ_FIELD_UZ_G, e.uz_g);
    put(CAPAZ_FIELD_ROS_W, w.roS_w);
    put(CAPAZ_FIELD_ROS_N, w.roS_n);
    put(CAPAZ_FIELD_ROS_G, w.roS_g);
    put(CAPAZ_FIELD_ROS_W_OLD, w.roS_w_old);
    put(CAPAZ_FIELD_ROS_N_OLD, w.roS_n_old);
    put(CAPAZ_FIELD_ROS_G_OLD, w.roS_g_old);
    put(CAPAZ_FIELD_H_W, e.H_w);
    put(CAPAZ_FIELD_H_N, e.H_n);
    put(CAPAZ_FIELD_H_G, e.H_g);
    put(CAPAZ_FIELD_H_R, e.H_r);
    put(CAPAZ_FIELD_E, e.E);
    put(CAPAZ_FIELD_E_NEW, e.E_new);
  }
  return CAPAZ_OK;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

// Forward-mode (tangent-linear) derivative of the observation misfit
//   J = sum over t = every, 2*every, ... <= nsteps, o < nobs of
//       ((1 - S_n(t, obs[o])) - data[(t/every - 1)*nobs + o])^2
// along the direction (dlnK, dm) of (ln K, porosity), through nsteps
// two-phase steps (the two-phase step above, instantiated on dual numbers:
// the Newton iterations are differentiated as unrolled).  With init_from_m
// the initial state is data_initialization's, a function of m; otherwise
// (P0, S0) is the initial state and does not depend on the parameters.
// dlnK / dm may be NULL (zero).  Per-cell K is used (the K array).
int oracle_tangent(const capaz_params* p_in, int nsteps, const double* m, const double* K, const double* dlnK,
                   const double* dm, int init_from_m, const double* P0, const double* S0, const long* obs,
                   int nobs, int every, const double* data, double* J, double* dJ, int nthreads) {
  int rc = check_grid(p_in);
  if (rc) return rc;
  if (p_in->phases != 2 || every < 1 || nsteps < 0 || !m || !K) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (!init_from_m && (!P0 || !S0)) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  capaz_params pp = *p_in;
  pp.flags |= CAPAZ_FLAG_PERCELL_K;
  const capaz_params* p = &pp;
  Grid g(p);
  const long n = g.n;
  std::vector<Dual> md(n), Kd(n), P(n), S(n);
  for (long l = 0; l < n; l++) {
    md[l] = Dual(m[l], dm ? dm[l] : 0.);
    Kd[l] = Dual(K[l], dlnK ? K[l] * dlnK[l] : 0.);
  }
  if (init_from_m) {
    init2(p, g, md.data(), P.data(), S.data());
  } else {
    for (long l = 0; l < n; l++) {
      P[l] = Dual(P0[l]);
      S[l] = Dual(S0[l]);
    }
  }
  WorkT<Dual> w;
  for (auto* v : {&w.S_w, &w.P_n, &w.ro_w, &w.ro_n, &w.Xi_w, &w.Xi_n, &w.roS_w, &w.roS_n, &w.roS_w_old,
                  &w.roS_n_old})
    v->assign(n, Dual(0.));
  Dual acc(0.);
  for (int t = 1; t <= nsteps; t++) {
    step2(p, g, P.data(), S.data(), md.data(), Kd.data(), w);
    if (t % every == 0) {
      const double* d = data ? data + (size_t)(t / every - 1) * nobs : nullptr;
      for (int o = 0; o < nobs; o++) {
        Dual r = (1. - S[obs[o]]) - (d ? d[o] : 0.);
        acc = acc + r * r;
      }
    }
  }
  if (J) *J = acc.v;
  if (dJ) *dJ = acc.d;
  return CAPAZ_OK;
}

}  // extern "C"
