// Three-phase step with the energy equation (the reference's THREE_PHASE +
// ENERGY build: energy.cpp with the three-phase module and cpu.cpp), FP64,
// in the reference's operation order (compiled with -fmad=false).
//
// The build has no GPU code in the reference (energy.cpp is CPU only).  Its
// time step adds a fifth unknown, the temperature T, and two stages:
//   H_E_current_calculation  enthalpies H_p(T) and the internal energy E of
//                            every cell at the current state (cpu.cpp:38-49)
//   E_calculation            E_new = E + dt (T_flow - E_flow) on interior
//                            cells: heat conduction with the effective
//                            conductivity and advected enthalpy with central
//                            differences of rho H u (energy.cpp:232-343;
//                            the z term of T_flow replaces the sum and the z
//                            term of E_flow takes the y velocities, as written)
// and replaces the 3x3 Newton by a 5x5 one in (S_w, S_n, S_g, P_w, T) with
// the reference's Gauss-Jordan inverse (energy.cpp:348-462); viscosities
// and densities depend on T (three-phase.cpp:210-215, cpu.cpp:118-127); the
// top and bottom rows hold fixed temperatures (Border_T, energy.cpp:396-418).
//
// The advected-enthalpy term reads velocities of the neighbours, which are
// central differences of their neighbours' pressures: the stencil reaches two
// cells.  The step is therefore five launches over per-cell arrays, the
// reference's own arrays (they are also what the derived fields return):
//   1 derive     S_g, Xi, P_n and P_g (interior), rho, H, E, conductivity
//   2 velocity   u of the three phases on every cell
//   3 balance    roS and roS_old of the three phases, E_new (interior)
//   4 newton     the 5x5 Newton in place (interior, own cell only)
//   5 boundary   Border_S, Border_P, Border_T
// Each launch reads only values no other thread of the same launch writes,
// so the state is updated in place, as the reference updates it.
#include <math.h>

#include "capaz_internal.h"
#include "phys3.cuh"

namespace capaz {
namespace {

using phys3::directed;

// energy.cpp:1-30 (T_0 also assign_ro's local, cpu.cpp:120-123).
constexpr double T_0 = 273., ro_r = 2000.;
constexpr double lambda0_w = 0.553, lambda0_n = 0.14, lambda0_g = 0.0237, lambda0_r = 1.;
constexpr double lambdaA_w = 3E-3, lambdaA_n = 1E-3, lambdaA_g = 0.82;
constexpr double c0_w = 4.194E3, c0_n = 1.7E3, c0_g = 1E3, c0_r = 0.8E3;
constexpr double C_w = 1.15, C_w2 = 0.015, C_n = 3.4, C_g = 0.119, C_r = 0.75;
constexpr double alfa_w = 1.32E-7, alfa_n = 9.2E-7;
constexpr double T_top = 400., T_bottom = 273.;  // Border_T, energy.cpp:404-411

__device__ __forceinline__ double c_w(double T) { return c0_w - C_w * (T - T_0) + C_w2 * (T - T_0) * (T - T_0); }
__device__ __forceinline__ double c_n(double T) { return c0_n + C_n * (T - T_0); }
__device__ __forceinline__ double c_g(double T) { return c0_g + C_g * (T - T_0); }
__device__ __forceinline__ double c_r(double T) { return c0_r + C_r * (T - T_0); }
__device__ __forceinline__ double H_w(const Step3Const& c, double T) {
  return (c.P_atm / c.ro0_w) + (T - T_0) * (c0_w - (T - T_0) * (C_w / 2 + C_w2 * (T - T_0) / 3));
}
__device__ __forceinline__ double H_n(const Step3Const& c, double T) {
  return (c.P_atm / c.ro0_n) + (T - T_0) * (c0_n + C_n * (T - T_0) / 2);
}
__device__ __forceinline__ double H_g(const Step3Const& c, double T) {
  return (c.P_atm / c.ro0_g) + (T - T_0) * (c0_g + C_g * (T - T_0) / 2);
}
__device__ __forceinline__ double H_r(const Step3Const& c, double T) {
  return (c.P_atm / ro_r) + (T - T_0) * (c0_r + C_r * (T - T_0) / 2);
}
__device__ __forceinline__ double ro_w(const Step3Const& c, double P, double T) {
  return c.ro0_w * (1. + (c.beta_w) * (P - c.P_atm) - alfa_w * (T - T_0));
}
__device__ __forceinline__ double ro_n(const Step3Const& c, double P, double T) {
  return c.ro0_n * (1. + (c.beta_n) * (P - c.P_atm) - alfa_n * (T - T_0));
}
__device__ __forceinline__ double ro_g(const Step3Const& c, double P, double T) {
  return c.ro0_g * (P / c.P_atm) * (T_0 / T);
}

__device__ __forceinline__ bool interior3e(const Step3Const& c, int i, int j, int k) {
  return (((i != 0) && (i != c.nx - 1)) || (c.nx < 2)) && (j != 0) && (j != c.ny - 1) &&
         (((k != 0) && (k != c.nz - 1)) || (c.nz < 2));
}

struct Cell {
  int i, j, k;
};
__device__ __forceinline__ Cell cell_of(const Step3Const& c, long long l) {
  return Cell{(int)(l % c.nx), (int)((l / c.nx) % c.ny), (int)(l / c.sz)};
}

// 1: S_calculation, ro_P_Xi_calculation, H_E_current_calculation and the
// effective conductivity (energy.cpp:54-81) of every cell.
// Four CTAs of 256 threads per SM (64 registers).
__global__ void __launch_bounds__(256, 4)
    energy_derive_kernel(const Step3Const c, EnergyState st, const double* __restrict__ m,
                         const double* __restrict__ K, double* __restrict__ w) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const Cell q = cell_of(c, l);
  const long long n = c.ncell;
  const double Sw = st.Sw[l], Sn = st.Sn[l], T = st.T[l], Pw = st.Pw[l], ml = m[l];
  const double Sg = 1. - Sw - Sn;
  const double den = 1. - c.S_wr - c.S_nr - c.S_gr;
  const double S_w_e = (Sw - c.S_wr) / den;
  const double S_n_e = (Sn - c.S_nr) / den;
  const double S_g_e = 1. - S_w_e - S_n_e;
  const double k_w = phys3::k_w3(S_w_e, c.A), k_g = phys3::k_g3(S_g_e, c.A), k_n = phys3::k_n3(S_w_e, S_n_e, c.A);
  const double mu_w = 1. / (29.21 * T - 7506.64);
  const double mu_n = 7.256E-10 * exp(4141.9 / T);
  const double mu_g = 1.717E-5 * pow((T / 273.), 0.683);
  const double Kl = K ? K[l] : c.K0;
  double Pn, Pg;
  if (interior3e(c, q.i, q.j, q.k)) {
    const double Pk_nw = 0, Pk_gn = 0;
    Pn = Pw + Pk_nw;
    Pg = Pw + Pk_nw + Pk_gn;
    st.Pn[l] = Pn;
    st.Pg[l] = Pg;
  } else {
    Pn = st.Pn[l];
    Pg = st.Pg[l];
  }
  const double rw = ro_w(c, Pw, T), rn = ro_n(c, Pn, T), rg = ro_g(c, Pg, T);
  const double Hw = H_w(c, T), Hn = H_n(c, T), Hg = H_g(c, T), Hr = H_r(c, T);
  w[EW_SG * n + l] = Sg;
  w[EW_XI_W * n + l] = (-1.) * Kl * k_w / mu_w;
  w[EW_XI_N * n + l] = (-1.) * Kl * k_n / mu_n;
  w[EW_XI_G * n + l] = (-1.) * Kl * k_g / mu_g;
  w[EW_RO_W * n + l] = rw;
  w[EW_RO_N * n + l] = rn;
  w[EW_RO_G * n + l] = rg;
  w[EW_H_W * n + l] = Hw;
  w[EW_H_N * n + l] = Hn;
  w[EW_H_G * n + l] = Hg;
  w[EW_H_R * n + l] = Hr;
  w[EW_E * n + l] = (ml * (Sw * (rw * Hw - Pw) + Sn * (rn * Hn - Pn) + Sg * (rg * Hg - Pg)) +
                     (1. - ml) * (ro_r * Hr - Pw));
  w[EW_LAM * n + l] = ml * (Sw * (lambda0_w * (1 - lambdaA_w * (T - T_0))) +
                            Sn * (lambda0_n * (1 - lambdaA_n * (T - T_0))) +
                            Sg * (lambda0_g * pow((T / T_0), lambdaA_g))) +
                      (1. - ml) * lambda0_r;
}

// 2: u_calculation (cpu.cpp:346-477) of the three phases on every cell:
// central differences, one-sided at the ends, gravity on y.
__global__ void energy_velocity_kernel(const Step3Const c, EnergyState st, double* __restrict__ w) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const Cell q = cell_of(c, l);
  const long long n = c.ncell;
  const double* P3[3] = {st.Pw, st.Pn, st.Pg};
#pragma unroll
  for (int ph = 0; ph < 3; ph++) {
    const double* P = P3[ph];
    const double Xi = w[(EW_XI_W + ph) * n + l], ro = w[(EW_RO_W + ph) * n + l];
    double ux = 0., uy = 0., uz = 0.;
    if (c.nx > 2) {
      if (q.i == 0) ux = Xi * ((P[l + 1] - P[l]) / c.hx);
      else if (q.i == c.nx - 1) ux = Xi * ((P[l] - P[l - 1]) / c.hx);
      else ux = Xi * ((P[l + 1] - P[l - 1]) / (2. * c.hx));
    }
    if (c.ny > 2) {
      if (q.j == 0) uy = Xi * ((P[l + c.sy] - P[l]) / c.hy - ro * (c.g));
      else if (q.j == c.ny - 1) uy = Xi * ((P[l] - P[l - c.sy]) / c.hy - ro * (c.g));
      else uy = Xi * ((P[l + c.sy] - P[l - c.sy]) / (2. * c.hy) - ro * (c.g));
    }
    if (c.nz > 2) {
      if (q.k == 0) uz = Xi * ((P[l + c.sz] - P[l]) / c.hz);
      else if (q.k == c.nz - 1) uz = Xi * ((P[l] - P[l - c.sz]) / c.hz);
      else uz = Xi * ((P[l + c.sz] - P[l - c.sz]) / (2. * c.hz));
    }
    w[(EW_UX_W + 3 * ph) * n + l] = ux;
    w[(EW_UX_W + 3 * ph + 1) * n + l] = uy;
    w[(EW_UX_W + 3 * ph + 2) * n + l] = uz;
  }
}

// 3: roS_calculation (NR form, cpu.cpp:619-731, rates zero) and
// E_calculation on interior cells.
// Three CTAs of 256 threads per SM (85 registers).
__global__ void __launch_bounds__(256, 3)
    energy_balance_kernel(const Step3Const c, EnergyState st, const double* __restrict__ m,
                          double* __restrict__ w) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const Cell q = cell_of(c, l);
  if (!interior3e(c, q.i, q.j, q.k)) return;
  const long long n = c.ncell;
  const double* Xi_w = w + EW_XI_W * n;
  const double* Xi_n = w + EW_XI_N * n;
  const double* Xi_g = w + EW_XI_G * n;
  const double* rw = w + EW_RO_W * n;
  const double* rn = w + EW_RO_N * n;
  const double* rg = w + EW_RO_G * n;
  const double ml = m[l];
  if (ml) {
    const double q_w = 0., q_n = 0., q_g = 0.;  // wells_q (three-phase.cpp:529-550)
    const double Sw = st.Sw[l], Sn = st.Sn[l];
    const double roS_w = rw[l] * Sw;
    const double roS_g = rg[l] * (1. - Sw - Sn);
    const double roS_n = rn[l] * Sn;
    auto face = [&](const double* P, const double* Xi, const double* ro, long long s, double h, double grav) {
      const double x2 = -1. * ((P[l + s] - P[l]) / h) + grav;
      const double x1 = -1. * ((P[l] - P[l - s]) / h) + grav;
      return directed(x1, x2, Xi[l], ro[l], Xi[l - s], ro[l - s], Xi[l + s], ro[l + s], h);
    };
    // The reference adds g rho on y only; on x and z the force is -dP/h alone.
    auto face0 = [&](const double* P, const double* Xi, const double* ro, long long s, double h) {
      const double x2 = -1. * ((P[l + s] - P[l]) / h);
      const double x1 = -1. * ((P[l] - P[l - s]) / h);
      return directed(x1, x2, Xi[l], ro[l], Xi[l - s], ro[l - s], Xi[l + s], ro[l + s], h);
    };
    double fx_w = 0., fx_n = 0., fx_g = 0., fz_w = 0., fz_n = 0., fz_g = 0.;
    if (c.nz >= 2) {
      fz_w = face0(st.Pw, Xi_w, rw, c.sz, c.hz);
      fz_n = face0(st.Pn, Xi_n, rn, c.sz, c.hz);
      fz_g = face0(st.Pg, Xi_g, rg, c.sz, c.hz);
    }
    if (c.nx >= 2) {
      fx_w = face0(st.Pw, Xi_w, rw, 1, c.hx);
      fx_n = face0(st.Pn, Xi_n, rn, 1, c.hx);
      fx_g = face0(st.Pg, Xi_g, rg, 1, c.hx);
    }
    const double fy_w = face(st.Pw, Xi_w, rw, c.sy, c.hy, c.g * (rw[l]));
    const double fy_n = face(st.Pn, Xi_n, rn, c.sy, c.hy, c.g * (rn[l]));
    const double fy_g = face(st.Pg, Xi_g, rg, c.sy, c.hy, c.g * (rg[l]));
    w[EW_ROS_W * n + l] = roS_w - (c.dt / ml) * (-q_w + fx_w + fy_w + fz_w);
    w[EW_ROS_N * n + l] = roS_n - (c.dt / ml) * (-q_n + fx_n + fy_n + fz_n);
    w[EW_ROS_G * n + l] = roS_g - (c.dt / ml) * (q_g + fx_g + fy_g + fz_g);
    w[EW_ROS_W_OLD * n + l] = roS_w;
    w[EW_ROS_N_OLD * n + l] = roS_n;
    w[EW_ROS_G_OLD * n + l] = roS_g;
  }
  // E_new = E + dt (T_flow + Q_hw + Q_hr - E_flow).
  const double* lam = w + EW_LAM * n;
  const double* T = st.T;
  double Tf = 0;
  if (c.nx > 2) Tf += (lam[l + 1] * T[l + 1] - 2 * lam[l] * T[l] + lam[l - 1] * T[l - 1]) / ((c.hx) * (c.hx));
  if (c.ny > 2)
    Tf += (lam[l + c.sy] * T[l + c.sy] - 2 * lam[l] * T[l] + lam[l - c.sy] * T[l - c.sy]) / ((c.hy) * (c.hy));
  if (c.nz > 2)
    Tf = (lam[l + c.sz] * T[l + c.sz] - 2 * lam[l] * T[l] + lam[l - c.sz] * T[l - c.sz]) / ((c.hz) * (c.hz));
  const double* Hw = w + EW_H_W * n;
  const double* Hn = w + EW_H_N * n;
  const double* Hg = w + EW_H_G * n;
  auto flux = [&](long long s, int ax, double h) {
    const double* uw = w + (EW_UX_W + ax) * n;
    const double* un = w + (EW_UX_W + 3 + ax) * n;
    const double* ug = w + (EW_UX_W + 6 + ax) * n;
    return (rw[l + s] * Hw[l + s] * uw[l + s] - rw[l - s] * Hw[l - s] * uw[l - s] +
            rn[l + s] * Hn[l + s] * un[l + s] - rn[l - s] * Hn[l - s] * un[l - s] +
            rg[l + s] * Hg[l + s] * ug[l + s] - rg[l - s] * Hg[l - s] * ug[l - s]) /
           (2. * h);
  };
  double Ef = 0;
  if (c.nx > 2) Ef += flux(1, 0, c.hx);
  if (c.ny > 2) Ef += flux(c.sy, 1, c.hy);
  if (c.nz > 2) Ef += flux(c.sz, 1, c.hz);  // the y velocities, as energy.cpp:302-311 writes it
  const double Q_hw = 0, Q_hr = 0;
  w[EW_E_NEW * n + l] = w[EW_E * n + l] + (c.dt) * (Tf + Q_hw + Q_hr - Ef);
}

// 4: P_S_calculation, the 5x5 Newton of energy.cpp:348-462 on one interior
// cell in place.  reverse_matrix leaves dF as it is when it finds no pivot,
// and the reference uses dF all the same.
// Three CTAs of 256 threads per SM (85 registers, some spills to L1): the
// resident warps pay for the spills.
__global__ void __launch_bounds__(256, 3)
    energy_newton_kernel(const Step3Const c, EnergyState st, const double* __restrict__ m, double* __restrict__ w,
                         unsigned int* __restrict__ err) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const Cell q = cell_of(c, l);
  if (!interior3e(c, q.i, q.j, q.k)) return;
  const long long n = c.ncell;
  constexpr int N = 5;
  const double ml = m[l];
  const double rSw = w[EW_ROS_W * n + l], rSn = w[EW_ROS_N * n + l], rSg = w[EW_ROS_G * n + l];
  const double E_new = w[EW_E_NEW * n + l];
  double Sw = st.Sw[l], Sn = st.Sn[l], Sg = w[EW_SG * n + l], P = st.Pw[l], T = st.T[l];
  double Hw = w[EW_H_W * n + l], Hn = w[EW_H_N * n + l], Hg = w[EW_H_G * n + l], Hr = w[EW_H_R * n + l];
  for (int it = 1; it <= c.iters; it++) {
    double F[N], dF[N * N];
    F[0] = Sg + Sw + Sn - 1.;
    F[1] = ro_w(c, P, T) * Sw - rSw;
    F[2] = ro_n(c, P, T) * Sn - rSn;
    F[3] = ro_g(c, P, T) * Sg - rSg;
    F[4] = ml * (Sw * (ro_w(c, P, T) * Hw - P) + Sn * (ro_n(c, P, T) * Hn - P) + Sg * (ro_g(c, P, T) * Hg - P)) +
           (1. - ml) * (ro_r * Hr - P) - E_new;
    const double dwP = c.ro0_w * (c.beta_w), dwT = (-1) * c.ro0_w * alfa_w;
    const double dnP = c.ro0_n * (c.beta_n), dnT = (-1) * c.ro0_n * alfa_n;
    const double dgP = (c.ro0_g / c.P_atm) * (T_0 / T);
    const double dgT = c.ro0_g * (P / c.P_atm) * (-1) * (T_0 / T) / T;
    dF[0] = 1.;
    dF[1] = 1.;
    dF[2] = 1.;
    dF[3] = 0.;
    dF[4] = 0.;
    dF[0 + N] = ro_w(c, P, T);
    dF[1 + N] = 0.;
    dF[2 + N] = 0.;
    dF[3 + N] = dwP * Sw;
    dF[4 + N] = dwT * Sw;
    dF[0 + N * 2] = 0.;
    dF[1 + N * 2] = ro_n(c, P, T);
    dF[2 + N * 2] = 0.;
    dF[3 + N * 2] = dnP * Sn;
    dF[4 + N * 2] = dnT * Sn;
    dF[0 + N * 3] = 0.;
    dF[1 + N * 3] = 0.;
    dF[2 + N * 3] = ro_g(c, P, T);
    dF[3 + N * 3] = dgP * Sg;
    dF[4 + N * 3] = dgT * Sg;
    dF[0 + N * 4] = ml * (ro_w(c, P, T) * Hw - P);
    dF[1 + N * 4] = ml * (ro_n(c, P, T) * Hn - P);
    dF[2 + N * 4] = ml * (ro_g(c, P, T) * Hg - P);
    dF[3 + N * 4] = ml * (Sw * (dwP * Hw - 1.) + Sn * (dnP * Hn - 1.) + Sg * (dgP * Hg - 1.)) + (1. - ml) * (-1);
    dF[4 + N * 4] = ml * (Sw * (dwT * Hw + ro_w(c, P, T) * c_w(T)) + Sn * (dnT * Hn + ro_n(c, P, T) * c_n(T)) +
                          Sg * (dgT * Hg + ro_g(c, P, T) * c_g(T))) +
                    (1. - ml) * ro_r * c_r(T);
    // corr = dF^-1 F (energy.cpp inverts dF with reverse_matrix and
    // multiplies); where no pivot is found the reference multiplies by dF
    // itself, which reverse_matrix left unchanged.
    double corr[N];
    if (!phys3::solve_gj<N>(dF, F, corr)) {
#pragma unroll
      for (int a = 0; a < N; a++) {
        corr[a] = 0;
#pragma unroll
        for (int b = 0; b < N; b++) corr[a] += dF[b + N * a] * F[b];
      }
    }
    Sw = Sw - corr[0];
    Sn = Sn - corr[1];
    Sg = Sg - corr[2];
    P = P - corr[3];
    T = T - corr[4];
    Hw = H_w(c, T);
    Hn = H_n(c, T);
    Hg = H_g(c, T);
    Hr = H_r(c, T);
  }
  st.Sw[l] = Sw;
  st.Sn[l] = Sn;
  st.Pw[l] = P;
  st.T[l] = T;
  w[EW_SG * n + l] = Sg;
  w[EW_H_W * n + l] = Hw;
  w[EW_H_N * n + l] = Hn;
  w[EW_H_G * n + l] = Hg;
  w[EW_H_R * n + l] = Hr;
  w[EW_E * n + l] = E_new;
  if (!(isfinite(Sw) && isfinite(Sn) && isfinite(P) && isfinite(T))) atomicOr(err, 1u);
}

// 5: boundary_conditions: Border_S and Border_P of three-phase.cpp:345-427
// and Border_T, from the basic coordinate (cpu.cpp:107-141), an interior
// cell on the grids the context accepts.
__global__ void energy_boundary_kernel(const Step3Const c, EnergyState st) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const Cell q = cell_of(c, l);
  const bool bnd = (((q.i == 0) || (q.i == c.nx - 1)) && (c.nx >= 2)) || (q.j == 0) || (q.j == c.ny - 1) ||
                   (((q.k == 0) || (q.k == c.nz - 1)) && (c.nz >= 2));
  if (!bnd) return;
  int i1 = q.i, j1 = q.j, k1 = q.k;
  if ((q.i == 0) && (c.nx > 2)) i1++;
  if ((q.i == c.nx - 1) && (c.nx > 2)) i1--;
  if (q.j == 0) j1++;
  if (q.j == c.ny - 1) j1--;
  if ((q.k == 0) && (c.nz > 2)) k1++;
  if ((q.k == c.nz - 1) && (c.nz > 2)) k1--;
  const long long l1 = i1 + j1 * c.sy + (long long)k1 * c.sz;
  const bool win = (q.i >= c.nx / 2 - c.source) && (q.i <= c.nx / 2 + c.source) && (q.k >= c.win_k0) &&
                   (q.k <= c.win_k1);
  const bool src = (q.j == 0) && (c.source > 0) && (!c.source_window || win);
  if (!src) {
    st.Sw[l] = st.Sw[l1];
    st.Sn[l] = st.Sn[l1];
  } else {
    st.Sw[l] = c.S_w_gr;
    st.Sn[l] = c.S_n_gr;
  }
  const double Pk_nw = 0, Pk_gn = 0;
  const double P1 = st.Pw[l1];
  if ((q.j != 0) && (q.j != c.ny - 1)) {
    st.Pw[l] = P1;
    st.Pn[l] = P1 + Pk_nw;
    st.Pg[l] = P1 + Pk_nw + Pk_gn;
  } else if (q.j == 0) {
    st.Pw[l] = (P1 - (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
               (1. + (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
    st.Pn[l] = (P1 + Pk_nw - (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
               (1. + (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
    st.Pg[l] = (P1 + Pk_nw + Pk_gn) / (1. + (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
  } else {
    st.Pw[l] = (P1 + (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
               (1. - (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
    st.Pn[l] = (P1 + Pk_nw + (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
               (1. - (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
    st.Pg[l] = (P1 + Pk_nw + Pk_gn) / (1. - (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
  }
  if (q.j == 0) st.T[l] = T_top;
  else if (q.j == c.ny - 1) st.T[l] = T_bottom;
  else st.T[l] = st.T[l1];
}

}  // namespace

cudaError_t launch_step3_energy(const Step3Const& c, const EnergyState& st, const double* m, const double* K,
                                double* work, unsigned int* err, cudaStream_t s) {
  const unsigned nb = (unsigned)((c.ncell + 255) / 256);
  energy_derive_kernel<<<nb, 256, 0, s>>>(c, st, m, K, work);
  energy_velocity_kernel<<<nb, 256, 0, s>>>(c, st, work);
  energy_balance_kernel<<<nb, 256, 0, s>>>(c, st, m, work);
  energy_newton_kernel<<<nb, 256, 0, s>>>(c, st, m, work, err);
  energy_boundary_kernel<<<nb, 256, 0, s>>>(c, st);
  return cudaGetLastError();
}

}  // namespace capaz
