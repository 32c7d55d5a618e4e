// Device functions shared by the three-phase steps (step3_fp64.cu, the
// plain three-phase model; step3e.cu, three-phase with the energy equation).
#pragma once

#include <math.h>

namespace capaz {
namespace phys3 {

// Relative permeabilities, three-phase.cpp:146-186.  With a2 (A == 2 and
// CAPAZ_FLAG_POW_PRODUCTS) the exponents A/(A-1) = 2, (A-1)/A = 1/2 and
// 2(A-1)/A = 1 are taken as products and square roots.
__device__ __forceinline__ double k_w3(double S_w_e, double A, bool a2 = false) {
  double k_w = 0;
  if (S_w_e >= 1e-3) {
    if (a2) {
      const double t = 1. - sqrt(1. - S_w_e * S_w_e);
      k_w = sqrt(S_w_e) * (t * t);
    } else {
      k_w = pow(S_w_e, 0.5) * pow(1. - pow(1. - pow(S_w_e, A / (A - 1.)), (A - 1.) / A), 2.);
    }
  }
  return k_w;
}
__device__ __forceinline__ double k_g3(double S_g_e, double A, bool a2 = false) {
  double k_g = 0;
  if (S_g_e >= 1e-3) {
    if (a2) {
      const double u = 1. - S_g_e;
      k_g = sqrt(S_g_e) * (1. - u * u);
    } else {
      k_g = pow(S_g_e, 0.5) * pow(1. - pow(1. - S_g_e, A / (A - 1.)), 2. * (A - 1.) / A);
    }
  }
  return k_g;
}
__device__ __forceinline__ double k_n3(double S_w_e, double S_n_e, double A, bool a2 = false) {
  double k_n = 0;
  double S_g_e = 1. - S_w_e - S_n_e;
  if (S_n_e >= 1e-3) {
    double k_n_w, k_n_g;
    if (a2) {
      k_n_w = sqrt(1. - S_w_e) * (1. - S_w_e * S_w_e);
      const double t = 1. - sqrt(1. - S_n_e * S_n_e);
      k_n_g = sqrt(S_n_e) * (t * t);
    } else {
      k_n_w = pow(1. - S_w_e, 0.5) * pow(1. - pow(S_w_e, A / (A - 1.)), 2. * (A - 1.) / A);
      k_n_g = pow(S_n_e, 0.5) * pow(1. - pow(1. - pow(S_n_e, A / (A - 1.)), (A - 1.) / A), 2.);
    }
    k_n = S_n_e * k_n_w * k_n_g / (1 - S_w_e) / (1 - S_g_e);
  }
  return k_n;
}

__device__ __forceinline__ double directed(double x1, double x2, double Xc, double rc, double Xm, double rm,
                                           double Xp, double rp, double h) {
  return (((x2 + fabs(x2)) / 2. - (x1 - fabs(x1)) / 2.) * (-1.) * Xc * rc -
          (x1 + fabs(x1)) / 2. * (-1.) * Xm * rm + (x2 - fabs(x2)) / 2. * (-1.) * Xp * rp) /
         h;
}

// reverse_matrix (gauss.cpp:6-92) for an N x N row-major matrix: Gauss-Jordan
// on [a | I] that looks for another pivot row only when |pivot| < 1e-8,
// taking the last row below with entry > 1e-8.  Returns false where the
// reference reports a zero determinant (it then leaves `a` unchanged).
// RCP: scale the pivot row by the pivot's reciprocal (one division per row
// instead of 2N; each entry within an ulp of the reference's quotient).
template <int N, bool RCP = false>
__device__ __forceinline__ bool reverse_matrix(double* a) {
  const double e = 1E-8;
  double matr[N][2 * N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      matr[i][j] = a[j + N * i];
      matr[i][j + N] = (j == i) ? 1 : 0;
    }
#pragma unroll
  for (int k = 0; k < N; k++) {
    double f = matr[k][k];
    if (fabs(f) < e) {
      int det_flag = 0;
#pragma unroll
      for (int i = k + 1; i < N; i++) {
        if (matr[i][k] > e) {
          det_flag = 1;
#pragma unroll
          for (int j = 0; j < 2 * N; j++) {
            double row = matr[k][j];
            matr[k][j] = matr[i][j];
            matr[i][j] = row;
          }
          f = matr[k][k];
        }
      }
      if (det_flag == 0) return false;
    }
    if (RCP) {
      const double r = 1. / f;
#pragma unroll
      for (int j = 0; j < 2 * N; j++) matr[k][j] *= r;
    } else {
#pragma unroll
      for (int j = 0; j < 2 * N; j++) matr[k][j] /= f;
    }
#pragma unroll
    for (int i = 0; i < N; i++)
      if (i != k) {
        double f1 = matr[i][k];
#pragma unroll
        for (int j = 0; j < 2 * N; j++) matr[i][j] -= (matr[k][j] * f1);
      }
  }
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) a[j + N * i] = matr[i][j + N];
  return true;
}

// x = a^-1 F by Gauss-Jordan on [a | F] with reverse_matrix's pivot rule
// (another pivot row only when |pivot| < 1e-8: the last row below with entry
// > 1e-8) and the pivot row scaled by the pivot's reciprocal.  The left block
// goes through exactly the operations reverse_matrix applies to it, so the
// pivot decisions are the same; the right-hand side replaces the identity
// block, which saves the product with the inverse (the result differs from
// inverse-times-F by rounding only).  Returns false, leaving x unset, where
// reverse_matrix finds no pivot.
template <int N>
__device__ __forceinline__ bool solve_gj(const double* a, const double* F, double* x) {
  const double e = 1E-8;
  double matr[N][N + 1];
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int j = 0; j < N; j++) matr[i][j] = a[j + N * i];
    matr[i][N] = F[i];
  }
#pragma unroll
  for (int k = 0; k < N; k++) {
    double f = matr[k][k];
    if (fabs(f) < e) {
      int det_flag = 0;
#pragma unroll
      for (int i = k + 1; i < N; i++) {
        if (matr[i][k] > e) {
          det_flag = 1;
#pragma unroll
          for (int j = 0; j <= N; j++) {
            double row = matr[k][j];
            matr[k][j] = matr[i][j];
            matr[i][j] = row;
          }
          f = matr[k][k];
        }
      }
      if (det_flag == 0) return false;
    }
    const double r = 1. / f;
#pragma unroll
    for (int j = 0; j <= N; j++) matr[k][j] *= r;
#pragma unroll
    for (int i = 0; i < N; i++)
      if (i != k) {
        double f1 = matr[i][k];
#pragma unroll
        for (int j = 0; j <= N; j++) matr[i][j] -= (matr[k][j] * f1);
      }
  }
#pragma unroll
  for (int i = 0; i < N; i++) x[i] = matr[i][N];
  return true;
}

}  // namespace phys3
}  // namespace capaz
