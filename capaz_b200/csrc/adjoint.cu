// Discrete adjoint of the two-phase FP64 step: gradient of an observation
// misfit with respect to ln K and porosity, per cell.
//
// Forward map of one step (the reference's time_step_function, two-phase,
// cpu.cpp / two-phase.cpp as restated by the FP64 step kernel), x = (P_w, S_n):
//   interior c:  A_p(c) = roS_p(x_c) - dt/m_c * sum_d (F_right - F_left)/h_d
//                F_right = x2 * M(upwind), x2 = -(P_+ - P_c)/h (+ g rho_c on y),
//                F_left  = x1 * M(upwind), x1 = -(P_c - P_-)/h (+ g rho_c on y),
//                M_p = K k_p(S) / mu_p * rho_p  (= -Xi_p * rho_p),
//                y'_c = Newton(A(c))  solves  G(y') = roS(y') - A = 0,
//   boundary b:  copies of the basic-coordinate cell's new value, the top row
//                P = const (and S = const in the injection window), the
//                bottom row P_b = P'_l1 + (rho_n S'_l1 + rho_w (1-S'_l1)) m g hy
//                with start-of-step densities (cpu.cpp:143-183).
// The transpose of one step is two gathers, so no atomics are needed:
//   phase 1 (interior c): lambda_hat(c) = lambda'(c) + the adjoints of the
//            boundary cells whose basic coordinate is c; Newton transposed by
//            the implicit-function theorem at the final iterate,
//            Abar(c) = J(y'_c)^-T lambda_hat(c);
//   phase 2 (every cell q): the adjoint of q's start-of-step (P, S) and the
//            ln K / porosity gradient increments from every A(c) whose stencil
//            reads q (c = q and its six neighbours), plus the bottom-row
//            start-of-step density terms.
// Upwind switches take the branch of the forward values (x >= 0 upwinds from
// the lower-index side, the branch the |x| form differentiates to at 0).
// Time stepping is checkpointed: the forward saves the state every K steps,
// the backward recomputes each segment's states from its checkpoint and
// sweeps it in reverse.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "capaz_ctx.h"
#include "capaz_internal.h"

using namespace capaz;

namespace {

struct AdjConst {
  int nx, ny, nz, planar, source, win_k0, win_k1;
  long long sy, sz, n;
  double hx, hy, hz, dt, g, P_atm, ro0_w, ro0_n, beta_w, beta_n, mu_w, mu_n, S_wr, P_d, lambda;
  double e_kw, e_kn, e_pk;
};

AdjConst make_adj_const(const capaz_params& p) {
  AdjConst c;
  c.nx = p.nx;
  c.ny = p.ny;
  c.nz = p.nz;
  c.planar = p.nz < 2;
  c.source = p.source;
  window_k(p, &c.win_k0, &c.win_k1);
  c.sy = p.nx;
  c.sz = (long long)p.nx * p.ny;
  c.n = c.sz * p.nz;
  c.hx = p.hx;
  c.hy = p.hy;
  c.hz = p.hz;
  c.dt = p.dt;
  c.g = p.g_const;
  c.P_atm = p.P_atm;
  c.ro0_w = p.ro0_w;
  c.ro0_n = p.ro0_n;
  c.beta_w = p.beta_w;
  c.beta_n = p.beta_n;
  c.mu_w = p.mu_w;
  c.mu_n = p.mu_n;
  c.S_wr = p.S_wr;
  c.P_d = p.P_d;
  c.lambda = p.lambda;
  c.e_kw = (2. + 3. * p.lambda) / p.lambda;
  c.e_kn = (2. + p.lambda) / p.lambda;
  c.e_pk = -1. / p.lambda;
  return c;
}

__device__ __forceinline__ bool is_interior(const AdjConst& c, int i, int j, int k) {
  return i > 0 && i < c.nx - 1 && j > 0 && j < c.ny - 1 && (c.planar || (k > 0 && k < c.nz - 1));
}

__device__ __forceinline__ bool in_window(const AdjConst& c, int i, int k) {
  return (i >= c.nx / 2 - c.source) && (i <= c.nx / 2 + c.source) && (k >= c.win_k0) && (k <= c.win_k1);
}

// Constitutive relations and their S-derivatives (two-phase.cpp:11-23,
// Brooks-Corey / Burdine).
struct Props {
  double Pn, dPk, rw, rn, kw, kn, dkw, dkn;
};

template <bool PD0>
__device__ __forceinline__ Props props(const AdjConst& c, double P, double S) {
  Props r;
  const double inv = 1. / (1. - c.S_wr);
  const double Se = (1. - S - c.S_wr) * inv;
  const double pw = pow(Se, c.e_kw - 1.);
  const double pn = pow(Se, c.e_kn - 1.);
  r.kw = pw * Se;
  const double om = 1. - Se;
  r.kn = om * om * (1. - pn * Se);
  // d/dS = -inv * d/dSe
  r.dkw = -inv * c.e_kw * pw;
  r.dkn = -inv * (-2. * om * (1. - pn * Se) - om * om * c.e_kn * pn);
  if (PD0) {
    r.Pn = P;
    r.dPk = 0.;
  } else {
    const double pk1 = pow(Se, c.e_pk - 1.);
    r.Pn = P + c.P_d * pk1 * Se;
    r.dPk = c.P_d * pk1 * inv / c.lambda;
  }
  r.rw = c.ro0_w * (1. + c.beta_w * (P - c.P_atm));
  r.rn = c.ro0_n * (1. + c.beta_n * (r.Pn - c.P_atm));
  return r;
}

// Start-of-step mobilities times densities of every cell, and P_n.
template <bool PD0>
__global__ void adj_props_kernel(const AdjConst c, const double* __restrict__ P, const double* __restrict__ S,
                                 const double* __restrict__ K, double* __restrict__ Mw, double* __restrict__ Mn,
                                 double* __restrict__ Pn) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.n) return;
  const Props r = props<PD0>(c, P[l], S[l]);
  const double Kl = K[l];
  Mw[l] = Kl * r.kw / c.mu_w * r.rw;
  Mn[l] = Kl * r.kn / c.mu_n * r.rn;
  if (!PD0) Pn[l] = r.Pn;
}

// Boundary cells whose basic coordinate (cpu.cpp:107-141) is interior cell
// (i, j, k): per axis the cell's own coordinate, plus the adjacent boundary
// coordinate when the cell is next to that face.
__device__ __forceinline__ int axis_options(int x, int nx, bool active, int* opt) {
  int q = 0;
  opt[q++] = x;
  if (active) {
    if (x == 1) opt[q++] = 0;
    if (x == nx - 2) opt[q++] = nx - 1;
  }
  return q;
}

// Phase 1: Abar(c) = J(y'_c)^-T (lambda'(c) + boundary copies of c).
template <bool PD0>
__global__ void adj_phase1_kernel(const AdjConst c, const double* __restrict__ lamP, const double* __restrict__ lamS,
                                  const double* __restrict__ Pnew, const double* __restrict__ Snew,
                                  const double* __restrict__ Pold, const double* __restrict__ Sold,
                                  const double* __restrict__ m, double* __restrict__ Aw, double* __restrict__ An) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.n) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  if (!is_interior(c, i, j, k)) return;
  double hP = lamP[l], hS = lamS[l];
  const double S1 = Snew[l], P1 = Pnew[l];
  int oi[3], oj[3], ok[3];
  const int ni = axis_options(i, c.nx, true, oi);
  const int nj = axis_options(j, c.ny, true, oj);
  const int nk = axis_options(k, c.nz, !c.planar, ok);
  if (ni * nj * nk > 1) {
    double drho = 0.;
    bool have_rho = false;
    for (int a = 0; a < ni; a++)
      for (int b = 0; b < nj; b++)
        for (int d = 0; d < nk; d++) {
          if (a == 0 && b == 0 && d == 0) continue;
          const int ib = oi[a], jb = oj[b], kb = ok[d];
          const long long lb = ib + jb * c.sy + kb * c.sz;
          const bool s_const = (jb == 0) && (c.source > 0) && in_window(c, ib, kb);
          if (!s_const) hS += lamS[lb];
          if (jb == 0) continue;  // top-row pressure is a constant
          const double lp = lamP[lb];
          hP += lp;
          if (jb == c.ny - 1) {
            if (!have_rho) {
              const Props r0 = props<PD0>(c, Pold[l], Sold[l]);
              drho = (r0.rn - r0.rw) * m[l] * c.g * c.hy;
              have_rho = true;
            }
            hS += lp * drho;
          }
        }
  }
  // Jacobian of G(P, S) = (rho_w(P)(1-S), rho_n(P + P_k(S)) S) at the final
  // iterate; solve J^T Abar = lambda_hat.
  const Props r1 = props<PD0>(c, P1, S1);
  const double J11 = c.ro0_w * c.beta_w * (1. - S1);
  const double J12 = -r1.rw;
  const double J21 = c.ro0_n * c.beta_n * S1;
  const double J22 = r1.rn + c.ro0_n * c.beta_n * S1 * r1.dPk;
  const double det = J11 * J22 - J12 * J21;
  Aw[l] = (J22 * hP - J21 * hS) / det;
  An[l] = (J11 * hS - J12 * hP) / det;
}

// Phase 2: adjoint of the start-of-step state of every cell and the
// gradient increments.  Abar is read only at interior cells.
template <bool PD0>
// Three CTAs per SM (85 registers, some spills): 6 % faster than two.
__global__ void __launch_bounds__(256, 3) adj_phase2_kernel(
    const AdjConst c, const double* __restrict__ P, const double* __restrict__ S, const double* __restrict__ K,
    const double* __restrict__ m, const double* __restrict__ Mw, const double* __restrict__ Mn,
    const double* __restrict__ PnArr, const double* __restrict__ Aw, const double* __restrict__ An,
    const double* __restrict__ lamP_next, const double* __restrict__ Snew, double* __restrict__ lamP_out,
    double* __restrict__ lamS_out, double* __restrict__ gK, double* __restrict__ gm) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.n) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  const double Pq = P[l], Sq = S[l], Kq = K[l], mq = m[l];
  const Props r = props<PD0>(c, Pq, Sq);
  const double Mwq = Kq * r.kw / c.mu_w * r.rw, Mnq = Kq * r.kn / c.mu_n * r.rn;
  const double Pnq = r.Pn;
  double lP = 0., lS = 0., Pnb = 0., Mwb = 0., Mnb = 0., rwb = 0., rnb = 0., gmq = 0.;
  const bool inq = is_interior(c, i, j, k);

  const int naxes = c.planar ? 2 : 3;
  for (int ax = 0; ax < naxes; ax++) {
    const long long s = ax == 0 ? 1 : (ax == 1 ? c.sy : c.sz);
    const double h = ax == 0 ? c.hx : (ax == 1 ? c.hy : c.hz);
    const int x = ax == 0 ? i : (ax == 1 ? j : k);
    const int nxa = ax == 0 ? c.nx : (ax == 1 ? c.ny : c.nz);
    const double gw = ax == 1 ? c.g : 0.;
    // Neighbour centre above (c = q + s): the face is its left face.
    if (x + 1 < nxa) {
      const long long lc = l + s;
      const int ic = ax == 0 ? i + 1 : i, jc = ax == 1 ? j + 1 : j, kc = ax == 2 ? k + 1 : k;
      if (is_interior(c, ic, jc, kc)) {
        const double Pc = P[lc];
        const double Pnc = PD0 ? Pc : PnArr[lc];
        const double coef = c.dt / (m[lc] * h);
        const double rwc = c.ro0_w * (1. + c.beta_w * (Pc - c.P_atm));
        const double rnc = c.ro0_n * (1. + c.beta_n * (Pnc - c.P_atm));
        {  // water
          const double x1 = -(Pc - Pq) / h + gw * rwc;
          const double w = coef * Aw[lc];
          const bool up = x1 >= 0.;
          lP += w * (up ? Mwq : Mw[lc]) / h;
          if (up) Mwb += w * x1;
        }
        {  // non-wetting
          const double x1 = -(Pnc - Pnq) / h + gw * rnc;
          const double w = coef * An[lc];
          const bool up = x1 >= 0.;
          Pnb += w * (up ? Mnq : Mn[lc]) / h;
          if (up) Mnb += w * x1;
        }
      }
    }
    // Neighbour centre below (c = q - s): the face is its right face.
    if (x - 1 >= 0) {
      const long long lc = l - s;
      const int ic = ax == 0 ? i - 1 : i, jc = ax == 1 ? j - 1 : j, kc = ax == 2 ? k - 1 : k;
      if (is_interior(c, ic, jc, kc)) {
        const double Pc = P[lc];
        const double Pnc = PD0 ? Pc : PnArr[lc];
        const double coef = -c.dt / (m[lc] * h);
        const double rwc = c.ro0_w * (1. + c.beta_w * (Pc - c.P_atm));
        const double rnc = c.ro0_n * (1. + c.beta_n * (Pnc - c.P_atm));
        {
          const double x2 = -(Pq - Pc) / h + gw * rwc;
          const double w = coef * Aw[lc];
          const bool up = x2 >= 0.;
          lP -= w * (up ? Mw[lc] : Mwq) / h;
          if (!up) Mwb += w * x2;
        }
        {
          const double x2 = -(Pnq - Pnc) / h + gw * rnc;
          const double w = coef * An[lc];
          const bool up = x2 >= 0.;
          Pnb -= w * (up ? Mn[lc] : Mnq) / h;
          if (!up) Mnb += w * x2;
        }
      }
    }
    // Own centre.
    if (inq) {
      const double Pp = P[l + s], Pm = P[l - s];
      const double Pnp = PD0 ? Pp : PnArr[l + s], Pnm = PD0 ? Pm : PnArr[l - s];
      const double coef = -c.dt / (mq * h);
      double fw, fn;
      {
        const double x2 = -(Pp - Pq) / h + gw * r.rw, x1 = -(Pq - Pm) / h + gw * r.rw;
        const double Mr = x2 >= 0. ? Mwq : Mw[l + s], Ml = x1 >= 0. ? Mw[l - s] : Mwq;
        fw = (x2 * Mr - x1 * Ml) / h;
        const double w = coef * Aw[l];
        lP += w * (Mr + Ml) / h;
        rwb += w * gw * (Mr - Ml);
        Mwb += w * ((x2 >= 0. ? x2 : 0.) - (x1 < 0. ? x1 : 0.));
      }
      {
        const double x2 = -(Pnp - Pnq) / h + gw * r.rn, x1 = -(Pnq - Pnm) / h + gw * r.rn;
        const double Mr = x2 >= 0. ? Mnq : Mn[l + s], Ml = x1 >= 0. ? Mn[l - s] : Mnq;
        fn = (x2 * Mr - x1 * Ml) / h;
        const double w = coef * An[l];
        Pnb += w * (Mr + Ml) / h;
        rnb += w * gw * (Mr - Ml);
        Mnb += w * ((x2 >= 0. ? x2 : 0.) - (x1 < 0. ? x1 : 0.));
      }
      // dA/dm = dt/m^2 * sum_d f
      gmq += (c.dt / (mq * mq)) * (Aw[l] * fw + An[l] * fn);
    }
  }
  if (inq) {
    // roS_w = rho_w(P)(1-S), roS_n = rho_n(P_n) S.
    const double aw = Aw[l], an = An[l];
    lP += aw * c.ro0_w * c.beta_w * (1. - Sq);
    lS -= aw * r.rw;
    Pnb += an * c.ro0_n * c.beta_n * Sq;
    lS += an * r.rn;
    // Bottom-row boundary cells fed by this cell: start-of-step densities
    // and porosity in P_b = P'_q + (rho_n S'_q + rho_w (1 - S'_q)) m_q g hy.
    if (j == c.ny - 2) {
      int oi[3], ok[3];
      const int ni = axis_options(i, c.nx, true, oi);
      const int nk = axis_options(k, c.nz, !c.planar, ok);
      double lb = 0.;
      for (int a = 0; a < ni; a++)
        for (int d = 0; d < nk; d++) lb += lamP_next[oi[a] + (c.ny - 1) * c.sy + ok[d] * c.sz];
      if (lb != 0.) {
        const double S1 = Snew[l];
        const double ghy = c.g * c.hy;
        rwb += lb * (1. - S1) * mq * ghy;
        rnb += lb * S1 * mq * ghy;
        gmq += lb * (r.rn * S1 + r.rw * (1. - S1)) * ghy;
      }
    }
  }
  // Mobility and density adjoints back to (P, S, ln K).
  const double Kw = Kq / c.mu_w, Kn = Kq / c.mu_n;
  lP += (Mwb * Kw * r.kw + rwb) * c.ro0_w * c.beta_w;
  lS += Mwb * Kw * r.dkw * r.rw;
  Pnb += (Mnb * Kn * r.kn + rnb) * c.ro0_n * c.beta_n;
  lS += Mnb * Kn * r.dkn * r.rn;
  lP += Pnb;
  if (!PD0) lS += Pnb * r.dPk;
  lamP_out[l] = lP;
  lamS_out[l] = lS;
  gK[l] += Mwb * Mwq + Mnb * Mnq;
  gm[l] += gmq;
}

// Two-phase data_initialization on the device, one thread per (i, k)
// column, in the host restatement's operation order.
__global__ void init2_columns_kernel(const AdjConst c, double S_n_gr, double S_n_bg, const double* __restrict__ m,
                                     double* __restrict__ P, double* __restrict__ S) {
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)c.nx * c.nz) return;
  const int i = (int)(col % c.nx), k = (int)(col / c.nx);
  double Pu = 0., Su = 0., rwu = 0., rnu = 0., mu = 0.;
  for (int j = 0; j < c.ny; j++) {
    const long long l = i + j * c.sy + k * c.sz;
    const double Sl = ((j == 0) && in_window(c, i, k)) ? S_n_gr : S_n_bg;
    double Pl;
    if (j == 0) {
      Pl = c.P_atm;
    } else {
      const double ro_g_dy = (rnu * Su + rwu * (1 - Su)) * (mu) * (c.g) * (c.hy);
      Pl = Pu + ro_g_dy;
    }
    P[l] = Pl;
    S[l] = Sl;
    rwu = c.ro0_w * (1. + (c.beta_w) * (Pl - c.P_atm));
    rnu = c.ro0_n * (1. + (c.beta_n) * (Pl - c.P_atm));
    Pu = Pl;
    Su = Sl;
    mu = m[l];
  }
}

// Transpose of init2_columns_kernel with respect to m (S does not depend on
// the parameters): gm += (dP0/dm)^T lambda0_P.
__global__ void init2_adjoint_kernel(const AdjConst c, const double* __restrict__ P0, const double* __restrict__ S0,
                                     const double* __restrict__ m, const double* __restrict__ lamP0,
                                     double* __restrict__ gm) {
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)c.nx * c.nz) return;
  const int i = (int)(col % c.nx), k = (int)(col / c.nx);
  double carry = 0.;
  const double ghy = c.g * c.hy;
  for (int j = c.ny - 1; j >= 1; j--) {
    const long long l = i + j * c.sy + k * c.sz, u = l - c.sy;
    const double Pbar = lamP0[l] + carry;
    const double Pu = P0[u], Su = S0[u], mu = m[u];
    const double rw = c.ro0_w * (1. + c.beta_w * (Pu - c.P_atm));
    const double rn = c.ro0_n * (1. + c.beta_n * (Pu - c.P_atm));
    gm[u] += Pbar * (rn * Su + rw * (1. - Su)) * ghy;
    carry = Pbar * (1. + (c.ro0_n * c.beta_n * Su + c.ro0_w * c.beta_w * (1. - Su)) * mu * ghy);
  }
}

// Residuals at the observed cells and their squared sum (fixed order).
__global__ void obs_residual_kernel(const double* __restrict__ S, const long long* __restrict__ obs, int nobs,
                                    const double* __restrict__ data, double* __restrict__ resid,
                                    double* __restrict__ part) {
  __shared__ double red[256];
  double acc = 0.;
  for (int o = threadIdx.x; o < nobs; o += blockDim.x) {
    const double r = (1. - S[obs[o]]) - data[o];
    resid[o] = r;
    acc += r * r;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *part = red[0];
}

// dJ/dS_n at the observed cells: -2 r (S_w = 1 - S_n).  Cells are distinct.
__global__ void obs_source_kernel(const long long* __restrict__ obs, int nobs, const double* __restrict__ resid,
                                  double* __restrict__ lamS) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < nobs) lamS[obs[o]] -= 2. * resid[o];
}

unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

struct capaz_adjoint {
  capaz_ctx* ctx = nullptr;
  int nsteps = 0, every_cp = 0, nobs = 0, obs_every = 0, nobs_t = 0, flags = 0;
  long long n = 0;
  bool forward_done = false;
  double dt_fwd = 0.;
  long long* obs = nullptr;
  double* data = nullptr;   // nobs_t x nobs
  double* resid = nullptr;  // nobs_t x nobs
  double* parts = nullptr;  // nobs_t
  std::vector<double*> cp;  // checkpoints: P then S, 2n each
  double* seg = nullptr;    // (every_cp + 1) states, 2n each
  double* lam[2] = {nullptr, nullptr};  // P then S, 2n each
  double* Abar = nullptr;   // Aw then An, 2n
  double* props = nullptr;  // Mw, Mn, Pn: 3n
  double* grad = nullptr;   // gK then gm, 2n

  int fail(int code, const char* msg) {
    ctx->last_error = msg;
    return code;
  }
  int fail_cuda(cudaError_t e, const char* what) {
    cudaGetLastError();
    ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? CAPAZ_ERR_OUT_OF_MEMORY : CAPAZ_ERR_CUDA;
  }
  void release() {
    cudaSetDevice(ctx->device);
    for (double* q : cp) cudaFree(q);
    cp.clear();
    void* bufs[] = {obs, data, resid, parts, seg, lam[0], lam[1], Abar, props, grad};
    for (void* q : bufs) cudaFree(q);
    obs = nullptr;
    data = resid = parts = seg = Abar = props = grad = nullptr;
    lam[0] = lam[1] = nullptr;
  }
  int transpose_step(const double* Pold, const double* Sold, const double* Pnew, const double* Snew, int src,
                     cudaStream_t s);
  int forward(double* misfit, cudaStream_t s);
  int backward(double* gK, double* gm, bool on_device, cudaStream_t s);
};

#define ADJ_TRY(call, what)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return fail_cuda(e_, what); \
  } while (0)

int capaz_adjoint::transpose_step(const double* Pold, const double* Sold, const double* Pnew, const double* Snew,
                                  int src, cudaStream_t s) {
  const AdjConst c = make_adj_const(ctx->p);
  const bool pd0 = ctx->p.P_d == 0.;
  const int bs = 256;
  const unsigned nb = blocks_for(n, bs);
  double *Mw = props, *Mn = props + n, *Pn = props + 2 * n;
  double *lP = lam[src], *lS = lam[src] + n, *oP = lam[src ^ 1], *oS = lam[src ^ 1] + n;
  const double* K = (const double*)ctx->K;
  const double* m = (const double*)ctx->m;
  if (pd0) {
    adj_props_kernel<true><<<nb, bs, 0, s>>>(c, Pold, Sold, K, Mw, Mn, Pn);
    adj_phase1_kernel<true><<<nb, bs, 0, s>>>(c, lP, lS, Pnew, Snew, Pold, Sold, m, Abar, Abar + n);
    adj_phase2_kernel<true><<<nb, bs, 0, s>>>(c, Pold, Sold, K, m, Mw, Mn, Pn, Abar, Abar + n, lP, Snew, oP, oS,
                                              grad, grad + n);
  } else {
    adj_props_kernel<false><<<nb, bs, 0, s>>>(c, Pold, Sold, K, Mw, Mn, Pn);
    adj_phase1_kernel<false><<<nb, bs, 0, s>>>(c, lP, lS, Pnew, Snew, Pold, Sold, m, Abar, Abar + n);
    adj_phase2_kernel<false><<<nb, bs, 0, s>>>(c, Pold, Sold, K, m, Mw, Mn, Pn, Abar, Abar + n, lP, Snew, oP, oS,
                                               grad, grad + n);
  }
  ctx->launches += 3;
  ADJ_TRY(cudaGetLastError(), "adjoint step launch");
  return CAPAZ_OK;
}

int capaz_adjoint::forward(double* misfit, cudaStream_t s) {
  ADJ_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  const AdjConst c = make_adj_const(ctx->p);
  double* P = (double*)ctx->state[ctx->cur][0];
  double* S = (double*)ctx->state[ctx->cur][1];
  if (flags & CAPAZ_ADJ_INIT_FROM_M) {
    init2_columns_kernel<<<blocks_for((long long)c.nx * c.nz, 128), 128, 0, s>>>(
        c, ctx->p.S_n_gr, ctx->p.S_n_background, (const double*)ctx->m, P, S);
    ctx->launches++;
    ADJ_TRY(cudaGetLastError(), "init launch");
  }
  const size_t fb = sizeof(double) * n;
  for (int t = 0; t <= nsteps; t++) {
    if (t > 0) {
      int st = ctx->step(1, s);
      if (st) return st;
      P = (double*)ctx->state[ctx->cur][0];
      S = (double*)ctx->state[ctx->cur][1];
      if (t % obs_every == 0) {
        const int ti = t / obs_every - 1;
        obs_residual_kernel<<<1, 256, 0, s>>>(S, obs, nobs, data + (size_t)ti * nobs, resid + (size_t)ti * nobs,
                                              parts + ti);
        ctx->launches++;
        ADJ_TRY(cudaGetLastError(), "observation launch");
      }
    }
    if (t % every_cp == 0 && t < nsteps) {
      double* q = cp[t / every_cp];
      ADJ_TRY(cudaMemcpyAsync(q, P, fb, cudaMemcpyDeviceToDevice, s), "checkpoint copy");
      ADJ_TRY(cudaMemcpyAsync(q + n, S, fb, cudaMemcpyDeviceToDevice, s), "checkpoint copy");
    }
  }
  std::vector<double> h(nobs_t > 0 ? nobs_t : 1, 0.);
  if (nobs_t > 0) ADJ_TRY(cudaMemcpyAsync(h.data(), parts, sizeof(double) * nobs_t, cudaMemcpyDeviceToHost, s), "misfit");
  ADJ_TRY(cudaStreamSynchronize(s), "forward");
  double J = 0.;
  for (int q = 0; q < nobs_t; q++) J += h[q];
  if (misfit) *misfit = J;
  dt_fwd = ctx->p.dt;
  forward_done = true;
  return ctx->check_flag();
}

int capaz_adjoint::backward(double* gK_out, double* gm_out, bool on_device, cudaStream_t s) {
  ADJ_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!forward_done) return fail(CAPAZ_ERR_BAD_STATE, "capaz_backward: run capaz_forward_checkpointed first");
  if (ctx->p.dt != dt_fwd) return fail(CAPAZ_ERR_BAD_STATE, "capaz_backward: dt changed since the forward pass");
  const size_t fb = sizeof(double) * n;
  ADJ_TRY(cudaMemsetAsync(lam[0], 0, 2 * fb, s), "memset");
  ADJ_TRY(cudaMemsetAsync(grad, 0, 2 * fb, s), "memset");
  const Step2Const c2 = make_step2_const(ctx->p);
  const double* K = (const double*)ctx->K;
  const double* m = (const double*)ctx->m;
  int src = 0;
  const int nseg = (nsteps + every_cp - 1) / every_cp;
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int t0 = sg * every_cp, t1 = std::min(nsteps, t0 + every_cp);
    // Recompute the segment's states from its checkpoint.
    ADJ_TRY(cudaMemcpyAsync(seg, cp[sg], 2 * fb, cudaMemcpyDeviceToDevice, s), "restore checkpoint");
    for (int t = t0 + 1; t <= t1; t++) {
      double* in = seg + (size_t)2 * n * (t - 1 - t0);
      double* out = seg + (size_t)2 * n * (t - t0);
      int nl = 0;
      ADJ_TRY(launch_step2_fp64(c2, in, in + n, out, out + n, m, K, true, nullptr, ctx->err_flag, s, &nl),
              "recompute launch");
      ctx->launches += nl;
    }
    for (int t = t1; t > t0; t--) {
      if (t % obs_every == 0) {
        const int ti = t / obs_every - 1;
        obs_source_kernel<<<blocks_for(nobs, 256), 256, 0, s>>>(obs, nobs, resid + (size_t)ti * nobs,
                                                                lam[src] + n);
        ctx->launches++;
        ADJ_TRY(cudaGetLastError(), "observation source launch");
      }
      const double* xo = seg + (size_t)2 * n * (t - 1 - t0);
      const double* xn = seg + (size_t)2 * n * (t - t0);
      int st = transpose_step(xo, xo + n, xn, xn + n, src, s);
      if (st) return st;
      src ^= 1;
    }
  }
  if (flags & CAPAZ_ADJ_INIT_FROM_M) {
    const AdjConst c = make_adj_const(ctx->p);
    init2_adjoint_kernel<<<blocks_for((long long)c.nx * c.nz, 128), 128, 0, s>>>(c, cp[0], cp[0] + n, m, lam[src],
                                                                                 grad + n);
    ctx->launches++;
    ADJ_TRY(cudaGetLastError(), "init adjoint launch");
  }
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (gK_out) ADJ_TRY(cudaMemcpyAsync(gK_out, grad, fb, kind, s), "gradient copy");
  if (gm_out) ADJ_TRY(cudaMemcpyAsync(gm_out, grad + n, fb, kind, s), "gradient copy");
  if (!on_device) ADJ_TRY(cudaStreamSynchronize(s), "backward");
  return ctx->check_flag();
}

extern "C" {

capaz_adjoint* capaz_adjoint_create(capaz_ctx* ctx, int nsteps, int checkpoint_every, const long long* obs_cells,
                                    int nobs, int obs_every, int flags, int* status) {
  auto ret = [&](int st, const char* msg) -> capaz_adjoint* {
    if (status) *status = st;
    if (msg) {
      if (ctx) ctx->last_error = msg;
      set_create_error(msg);
    }
    return nullptr;
  };
  if (!ctx) return ret(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_adjoint_create: null context");
  const capaz_params& p = ctx->p;
  if (p.phases != 2 || p.form != CAPAZ_FORM_FP64 || p.model != CAPAZ_MODEL_DEFAULT)
    return ret(CAPAZ_ERR_UNSUPPORTED, "capaz_adjoint_create: the adjoint covers the two-phase task, FP64 form");
  if (!(p.flags & CAPAZ_FLAG_PERCELL_K))
    return ret(CAPAZ_ERR_UNSUPPORTED, "capaz_adjoint_create: needs CAPAZ_FLAG_PERCELL_K (gradient per cell)");
  if (nsteps < 1 || checkpoint_every < 1 || obs_every < 1 || nobs < 0 || (nobs > 0 && !obs_cells) ||
      (flags & ~CAPAZ_ADJ_INIT_FROM_M))
    return ret(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_adjoint_create: bad nsteps/checkpoint_every/obs arguments");
  const long long n = ctx->n;
  std::vector<long long> sorted(obs_cells, obs_cells + nobs);
  std::sort(sorted.begin(), sorted.end());
  for (int o = 0; o < nobs; o++) {
    if (sorted[o] < 0 || sorted[o] >= n) return ret(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_adjoint_create: obs cell out of range");
    if (o > 0 && sorted[o] == sorted[o - 1])
      return ret(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_adjoint_create: observed cells must be distinct");
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ret(CAPAZ_ERR_CUDA, "capaz_adjoint_create: cudaSetDevice");
  capaz_adjoint* a = new capaz_adjoint;
  a->ctx = ctx;
  a->nsteps = nsteps;
  a->every_cp = std::min(checkpoint_every, nsteps);
  a->nobs = nobs;
  a->obs_every = obs_every;
  a->nobs_t = nsteps / obs_every;
  a->flags = flags;
  a->n = n;
  const size_t fb = sizeof(double) * n;
  const int ncp = (nsteps + a->every_cp - 1) / a->every_cp;
  bool ok = true;
  auto alloc = [&](void** q, size_t bytes) {
    if (ok && cudaMalloc(q, bytes ? bytes : 8) != cudaSuccess) ok = false;
  };
  const size_t od = sizeof(double) * (size_t)std::max(1, nobs) * std::max(1, a->nobs_t);
  alloc((void**)&a->obs, sizeof(long long) * std::max(1, nobs));
  alloc((void**)&a->data, od);
  alloc((void**)&a->resid, od);
  alloc((void**)&a->parts, sizeof(double) * std::max(1, a->nobs_t));
  a->cp.assign(ncp, nullptr);
  for (int q = 0; q < ncp; q++) alloc((void**)&a->cp[q], 2 * fb);
  alloc((void**)&a->seg, 2 * fb * (size_t)(a->every_cp + 1));
  alloc((void**)&a->lam[0], 2 * fb);
  alloc((void**)&a->lam[1], 2 * fb);
  alloc((void**)&a->Abar, 2 * fb);
  alloc((void**)&a->props, 3 * fb);
  alloc((void**)&a->grad, 2 * fb);
  if (ok && nobs > 0) ok = cudaMemcpy(a->obs, obs_cells, sizeof(long long) * nobs, cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) ok = cudaMemset(a->data, 0, od) == cudaSuccess;
  if (ok) ok = cudaMemset(a->Abar, 0, 2 * fb) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    a->release();
    delete a;
    return ret(CAPAZ_ERR_OUT_OF_MEMORY, "capaz_adjoint_create: device allocation failed");
  }
  if (status) *status = CAPAZ_OK;
  return a;
}

int capaz_adjoint_destroy(capaz_adjoint* a) {
  if (!a) return CAPAZ_ERR_INVALID_ARGUMENT;
  a->release();
  delete a;
  return CAPAZ_OK;
}

int capaz_adjoint_set_observations(capaz_adjoint* a, const double* data, int on_device, void* stream) {
  if (!a || !data) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(a->ctx->device) != cudaSuccess) return a->fail(CAPAZ_ERR_CUDA, "cudaSetDevice");
  const size_t bytes = sizeof(double) * (size_t)a->nobs * a->nobs_t;
  if (bytes == 0) return CAPAZ_OK;
  cudaStream_t s = (cudaStream_t)stream;
  {
    cudaError_t e = cudaMemcpyAsync(a->data, data, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return a->fail_cuda(e, "capaz_adjoint_set_observations");
  }
  a->forward_done = false;
  return CAPAZ_OK;
}

int capaz_forward_checkpointed(capaz_adjoint* a, double* misfit, void* stream) {
  if (!a) return CAPAZ_ERR_INVALID_ARGUMENT;
  return a->forward(misfit, (cudaStream_t)stream);
}

int capaz_backward(capaz_adjoint* a, double* grad_lnK, double* grad_m, int dst_on_device, void* stream) {
  if (!a) return CAPAZ_ERR_INVALID_ARGUMENT;
  return a->backward(grad_lnK, grad_m, dst_on_device != 0, (cudaStream_t)stream);
}

}  // extern "C"
