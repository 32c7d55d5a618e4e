// Buckley-Leverett task (the reference's B_L build: Backley-Leverett/b-l.cpp
// with cpu.cpp), FP64, in the reference's operation order (compiled with
// -fmad=false like the other reference-exact kernels).
//
// Physics against the two-phase task: piecewise relative permeabilities of
// S_w (assing_k, b-l.cpp:5-55), no capillary pressure (P_n = P_w), per-cell K
// from the permeability file, an injection and a production well in
// opposite corners of every z-plane (wells_q, b-l.cpp:239-262: the injection
// well adds Q of water, the production well removes Q split by the
// fractional flow), and boundary rules of its own (b-l.cpp:104-171): every
// boundary cell copies S_n from its basic coordinate; rows j = 0 and
// j = NY-1 add the weight (rho0_n S_n + rho0_w (1 - S_n)) m g hy of the cell
// itself to the basic cell's P_w; the 2x2 corner blocks hold the wells'
// pressures (interior well cells included).
//
// Two launches per step: the interior update (flux difference, wells,
// Newton) writes the interior of the output state; the boundary kernel then
// writes every boundary cell and the wells' pressures.  The task's grids are
// small (the reference runs 100 x 100), so the interior kernel evaluates the
// six neighbours' constitutive relations itself instead of staging planes.
#include <math.h>

#include "capaz_internal.h"

namespace capaz {
namespace {

__device__ __forceinline__ void bl_relperm(double S_w, double& k_w, double& k_n) {
  const double S_sv = 0.1, S_zv = 0.8, S_1 = 0.70324;
  if ((S_sv <= S_w) && (S_w <= S_zv))
    k_n = ((S_zv - S_w) / (S_zv - S_sv)) * ((S_zv - S_w) / (S_zv - S_sv));
  else if ((0 <= S_w) && (S_w <= S_sv))
    k_n = 1.;
  else
    k_n = 0.;
  if ((S_sv <= S_w) && (S_w <= S_1))
    k_w = ((S_w - S_sv) / (S_zv - S_sv)) * ((S_w - S_sv) / (S_zv - S_sv));
  else if ((0 <= S_w) && (S_w <= S_sv))
    k_w = 0.;
  else if ((S_1 <= S_w) && (S_w <= S_zv))
    k_w = 0.8 * pow((S_w - S_sv) / (S_zv - S_sv), 0.5);
  else
    k_w = 1.;
}

// assign_P_Xi (b-l.cpp:57-72) and assign_ro (cpu.cpp) of one cell.
__device__ __forceinline__ void bl_derive(const BLConst& b, double Pw, double Sn, double K, double& rw, double& rn,
                                          double& Xw, double& Xn) {
  double k_w = 0., k_n = 0.;
  bl_relperm(1. - Sn, k_w, k_n);
  Xw = -1. * K * k_w / b.c.mu_w;
  Xn = -1. * K * k_n / b.c.mu_n;
  rw = b.c.ro0_w * (1. + (b.c.beta_w) * (Pw - b.c.P_atm));
  rn = b.c.ro0_n * (1. + (b.c.beta_n) * (Pw - b.c.P_atm));
}

__device__ __forceinline__ void bl_derive_at(const BLConst& b, const double* Pw, const double* Sn, const double* K,
                                             bool percell, long long l, double& rw, double& rn, double& Xw,
                                             double& Xn) {
  bl_derive(b, Pw[l], Sn[l], percell ? K[l] : b.c.K0, rw, rn, Xw, Xn);
}

// directed_difference (cpu.cpp:236-264).
__device__ __forceinline__ double bl_directed(double x1, double x2, double Xc, double rc, double Xm, double rm,
                                              double Xp, double rp, double h) {
  return (((x2 + fabs(x2)) / 2. - (x1 - fabs(x1)) / 2.) * (-1.) * Xc * rc -
          (x1 + fabs(x1)) / 2. * (-1.) * Xm * rm + (x2 - fabs(x2)) / 2. * (-1.) * Xp * rp) /
         h;
}

__device__ __forceinline__ bool bl_injection(int i, int j) {
  return ((i == 1) && (j == 1)) || ((i == 0) && (j == 0)) || ((i == 1) && (j == 0)) || ((i == 0) && (j == 1));
}
__device__ __forceinline__ bool bl_output(const Step2Const& c, int i, int j) {
  return ((i == c.nx - 2) && (j == c.ny - 2)) || ((i == c.nx - 1) && (j == c.ny - 1)) ||
         ((i == c.nx - 1) && (j == c.ny - 2)) || ((i == c.nx - 2) && (j == c.ny - 1));
}

// wells_q (b-l.cpp:239-262) at cell (i, j) with saturation Sn.
__device__ __forceinline__ void bl_wells(const BLConst& b, int i, int j, double Sn, double& q_w, double& q_n) {
  q_w = 0.;
  q_n = 0.;
  if (bl_injection(i, j)) {
    q_w = b.Q;
    q_n = 0.;
  }
  if (bl_output(b.c, i, j)) {
    double k_w = 0., k_n = 0.;
    bl_relperm(1. - Sn, k_w, k_n);
    const double F_bl = (k_w / b.c.mu_w) / (k_w / b.c.mu_w + k_n / b.c.mu_n);
    q_w = -1. * b.Q * F_bl;
    q_n = -1. * b.Q * (1. - F_bl);
  }
}

__device__ __forceinline__ bool bl_interior(const Step2Const& c, int i, int j, int k) {
  return (i != 0) && (i != c.nx - 1) && (j != 0) && (j != c.ny - 1) && (((k != 0) && (k != c.nz - 1)) || (c.nz < 2));
}

// The flux difference of one phase at interior cell l (assign_roS_nr,
// cpu.cpp:619-731): axes z, x, y in the reference's order, gravity on y.
__device__ __forceinline__ void bl_fluxes(const BLConst& b, const double* Pw, const double* Sn, const double* K,
                                          bool percell, long long l, double rw, double rn, double Xw, double Xn,
                                          double f_w[3], double f_n[3]) {
  const Step2Const& c = b.c;
  for (int axis = 0; axis < 3; axis++) {
    f_w[axis] = 0.;
    f_n[axis] = 0.;
    if (axis == 2 && c.nz < 2) continue;
    const long long s = axis == 0 ? 1 : axis == 1 ? c.sy : c.sz;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    double rmw, rmn, Xmw, Xmn, rpw, rpn, Xpw, Xpn;
    bl_derive_at(b, Pw, Sn, K, percell, l - s, rmw, rmn, Xmw, Xmn);
    bl_derive_at(b, Pw, Sn, K, percell, l + s, rpw, rpn, Xpw, Xpn);
    const double Pc = Pw[l], Pm = Pw[l - s], Pp = Pw[l + s];
    // P_n = P_w: both phases see the same pressure differences.
    double x2 = -1. * ((Pp - Pc) / h), x1 = -1. * ((Pc - Pm) / h);
    double x2w = x2, x1w = x1, x2n = x2, x1n = x1;
    if (axis == 1) {
      x2w = x2 + c.g * (rw);
      x1w = x1 + c.g * (rw);
      x2n = x2 + c.g * (rn);
      x1n = x1 + c.g * (rn);
    }
    f_w[axis] = bl_directed(x1w, x2w, Xw, rw, Xmw, rmw, Xpw, rpw, h);
    f_n[axis] = bl_directed(x1n, x2n, Xn, rn, Xmn, rmn, Xpn, rpn, h);
  }
}

// Four CTAs of 256 threads per SM (64 registers).
__global__ void __launch_bounds__(256, 4) step_bl_interior_kernel(const BLConst b, const double* __restrict__ Pw, const double* __restrict__ Sn,
                                        double* __restrict__ Pw_out, double* __restrict__ Sn_out,
                                        const double* __restrict__ m, const double* __restrict__ K, bool percell,
                                        unsigned int* __restrict__ err) {
  const Step2Const& c = b.c;
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  if (!bl_interior(c, i, j, k)) return;
  const double mc = m[l];  // > 0 on every cell (checked when m is set)
  double P = Pw[l], S = Sn[l];
  double rw, rn, Xw, Xn;
  bl_derive_at(b, Pw, Sn, K, percell, l, rw, rn, Xw, Xn);
  double q_w, q_n;
  bl_wells(b, i, j, S, q_w, q_n);
  const double roS_w = rw * (1. - S), roS_n = rn * S;
  double f_w[3], f_n[3];
  bl_fluxes(b, Pw, Sn, K, percell, l, rw, rn, Xw, Xn, f_w, f_n);
  // A = roS - dt/m (-q + fx + fy + fz)
  const double A1 = roS_w - (c.dt / mc) * (-q_w + f_w[0] + f_w[1] + f_w[2]);
  const double A2 = roS_n - (c.dt / mc) * (-q_n + f_n[0] + f_n[1] + f_n[2]);
  // Newton (b-l.cpp:74-102).
  for (int w = 1; w <= c.iters; w++) {
    const double F1 = c.ro0_w * (1. + (c.beta_w) * (P - c.P_atm)) * (1. - S) - A1;
    const double F2 = c.ro0_n * (1. + (c.beta_n) * (P - c.P_atm)) * S - A2;
    const double F1P = c.ro0_w * (c.beta_w) * (1 - S);
    const double F2P = c.ro0_n * (c.beta_n) * S;
    const double F1S = (-1) * (c.ro0_w) * (1 + (c.beta_w) * (P - c.P_atm));
    const double F2S = c.ro0_n * (1 + (c.beta_n) * (P - c.P_atm));
    const double det = F1P * F2S - F1S * F2P;
    const double nP = P - (1. / det) * (F2S * F1 - F1S * F2);
    const double nS = S - (1. / det) * (F1P * F2 - F2P * F1);
    const bool fixed = same_bits(nP, P) && same_bits(nS, S);
    P = nP;
    S = nS;
    if (fixed) break;  // the remaining iterations would repeat this one
  }
  Pw_out[l] = P;
  Sn_out[l] = S;
  if (!(isfinite(P) && isfinite(S))) atomicOr(err, 1u);
  // The wells hold their pressures (b-l.cpp:165-170) on interior cells too.
  if (bl_injection(i, j)) Pw_out[l] = b.injwell_Pw;
  if (bl_output(c, i, j)) Pw_out[l] = b.outwell_Pw;
}

// The same interior update with the x and y neighbours' derived values
// staged in shared memory: a CTA takes a TX x TY tile of one z-plane, every
// window cell (halo included) is derived once, and the stencil reads the
// window; z neighbours (3-D grids) are derived in place as above.  The values
// and the operation order are those of step_bl_interior_kernel.
__global__ void __launch_bounds__(NTHREADS, 4)
    step_bl_tile_kernel(const BLConst b, const double* __restrict__ Pw, const double* __restrict__ Sn,
                        double* __restrict__ Pw_out, double* __restrict__ Sn_out, const double* __restrict__ m,
                        const double* __restrict__ K, bool percell, unsigned int* __restrict__ err) {
  __shared__ double sP[PC], srw[PC], srn[PC], sXw[PC], sXn[PC];
  const Step2Const& c = b.c;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
  const int k = c.nz < 2 ? 0 : 1 + (int)blockIdx.z;
  const long long kz = (long long)k * c.sz;
  for (int q = tid; q < PC; q += NTHREADS) {
    const int gi = i0 - 1 + q % PX, gj = j0 - 1 + q / PX;
    if (gi < c.nx && gj < c.ny) {
      const long long lq = gi + gj * c.sy + kz;
      sP[q] = Pw[lq];
      bl_derive_at(b, Pw, Sn, K, percell, lq, srw[q], srn[q], sXw[q], sXn[q]);
    }
  }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  if (i > c.nx - 2 || j > c.ny - 2) return;
  const int q = (ty + 1) * PX + (tx + 1);
  const long long l = i + j * c.sy + kz;
  const double mc = m[l];  // > 0 on every cell (checked when m is set)
  double P = sP[q], S = Sn[l];
  const double rw = srw[q], rn = srn[q], Xw = sXw[q], Xn = sXn[q];
  double q_w, q_n;
  bl_wells(b, i, j, S, q_w, q_n);
  const double roS_w = rw * (1. - S), roS_n = rn * S;
  double f_w[3], f_n[3];
  for (int axis = 0; axis < 3; axis++) {
    f_w[axis] = 0.;
    f_n[axis] = 0.;
    if (axis == 2 && c.nz < 2) continue;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    double rmw, rmn, Xmw, Xmn, rpw, rpn, Xpw, Xpn, Pm, Pp;
    if (axis < 2) {
      const int a = axis == 0 ? q - 1 : q - PX, bq = axis == 0 ? q + 1 : q + PX;
      rmw = srw[a], rmn = srn[a], Xmw = sXw[a], Xmn = sXn[a], Pm = sP[a];
      rpw = srw[bq], rpn = srn[bq], Xpw = sXw[bq], Xpn = sXn[bq], Pp = sP[bq];
    } else {
      bl_derive_at(b, Pw, Sn, K, percell, l - c.sz, rmw, rmn, Xmw, Xmn);
      bl_derive_at(b, Pw, Sn, K, percell, l + c.sz, rpw, rpn, Xpw, Xpn);
      Pm = Pw[l - c.sz];
      Pp = Pw[l + c.sz];
    }
    const double Pc = P;
    double x2 = -1. * ((Pp - Pc) / h), x1 = -1. * ((Pc - Pm) / h);
    double x2w = x2, x1w = x1, x2n = x2, x1n = x1;
    if (axis == 1) {
      x2w = x2 + c.g * (rw);
      x1w = x1 + c.g * (rw);
      x2n = x2 + c.g * (rn);
      x1n = x1 + c.g * (rn);
    }
    f_w[axis] = bl_directed(x1w, x2w, Xw, rw, Xmw, rmw, Xpw, rpw, h);
    f_n[axis] = bl_directed(x1n, x2n, Xn, rn, Xmn, rmn, Xpn, rpn, h);
  }
  const double A1 = roS_w - (c.dt / mc) * (-q_w + f_w[0] + f_w[1] + f_w[2]);
  const double A2 = roS_n - (c.dt / mc) * (-q_n + f_n[0] + f_n[1] + f_n[2]);
  for (int w = 1; w <= c.iters; w++) {
    const double F1 = c.ro0_w * (1. + (c.beta_w) * (P - c.P_atm)) * (1. - S) - A1;
    const double F2 = c.ro0_n * (1. + (c.beta_n) * (P - c.P_atm)) * S - A2;
    const double F1P = c.ro0_w * (c.beta_w) * (1 - S);
    const double F2P = c.ro0_n * (c.beta_n) * S;
    const double F1S = (-1) * (c.ro0_w) * (1 + (c.beta_w) * (P - c.P_atm));
    const double F2S = c.ro0_n * (1 + (c.beta_n) * (P - c.P_atm));
    const double det = F1P * F2S - F1S * F2P;
    const double nP = P - (1. / det) * (F2S * F1 - F1S * F2);
    const double nS = S - (1. / det) * (F1P * F2 - F2P * F1);
    const bool fixed = same_bits(nP, P) && same_bits(nS, S);
    P = nP;
    S = nS;
    if (fixed) break;  // the remaining iterations would repeat this one
  }
  Pw_out[l] = P;
  Sn_out[l] = S;
  if (!(isfinite(P) && isfinite(S))) atomicOr(err, 1u);
  if (bl_injection(i, j)) Pw_out[l] = b.injwell_Pw;
  if (bl_output(c, i, j)) Pw_out[l] = b.outwell_Pw;
}

// Border_S and Border_P (b-l.cpp:104-171), then the wells' pressures, on the
// boundary cells: one thread per cell q of the grid's shell (faces, then
// edges and corners, as boundary_cells counts them).  Interior cells are
// their own basic coordinate; the interior update has already given the
// interior well cells their wells' pressures.  Every boundary cell whose
// basic coordinate is an interior well cell is itself a well cell, so no
// thread reads a value another thread of this launch writes, and none reads
// a well pressure it keeps.
__global__ void step_bl_boundary_kernel(const BLConst b, double* __restrict__ Pw_out, double* __restrict__ Sn_out,
                                        const double* __restrict__ m, int nbound) {
  const Step2Const& c = b.c;
  int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (q >= nbound) return;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  int i, j, k;
  if (nz == 1) {
    k = 0;
    if (q < 2 * nx) {
      j = q < nx ? 0 : ny - 1;
      i = q % nx;
    } else {
      q -= 2 * nx;
      i = q < ny - 2 ? 0 : nx - 1;
      j = 1 + q % (ny - 2);
    }
  } else {
    const int A = nx * nz, B = (ny - 2) * nz, C = (nx - 2) * (ny - 2);
    if (q < 2 * A) {
      j = q < A ? 0 : ny - 1;
      q %= A;
      i = q % nx;
      k = q / nx;
    } else if ((q -= 2 * A) < 2 * B) {
      i = q < B ? 0 : nx - 1;
      q %= B;
      j = 1 + q % (ny - 2);
      k = q / (ny - 2);
    } else {
      q -= 2 * B;
      k = q < C ? 0 : nz - 1;
      q %= C;
      i = 1 + q % (nx - 2);
      j = 1 + q / (nx - 2);
    }
  }
  const long long l = i + j * c.sy + (long long)k * c.sz;
  const bool inj = bl_injection(i, j), out = bl_output(c, i, j);
  int i1 = i, j1 = j, k1 = k;
  if ((i == 0) && (c.nx > 2)) i1++;
  if ((i == c.nx - 1) && (c.nx > 2)) i1--;
  if (j == 0) j1++;
  if (j == c.ny - 1) j1--;
  if ((k == 0) && (c.nz > 2)) k1++;
  if ((k == c.nz - 1) && (c.nz > 2)) k1--;
  const long long l1 = i1 + j1 * c.sy + (long long)k1 * c.sz;
  const double S = Sn_out[l1];
  Sn_out[l] = S;
  double P;
  if ((j != 0) && (j != c.ny - 1)) {
    P = Pw_out[l1];
  } else {
    const double ro_g_dy = (c.ro0_n * S + c.ro0_w * (1 - S)) * (m[l]) * (c.g) * (c.hy);
    P = Pw_out[l1] + ro_g_dy;
  }
  if (inj) P = b.injwell_Pw;
  if (out) P = b.outwell_Pw;
  Pw_out[l] = P;
}

// Per-cell arrays the reference keeps, from a state (as its arrays hold them
// after time_step_function: derived from the start-of-step state).
__global__ void derived_bl_kernel(const BLConst b, int field, const double* __restrict__ Pw,
                                  const double* __restrict__ Sn, const double* __restrict__ m,
                                  const double* __restrict__ K, bool percell, double* __restrict__ out) {
  const Step2Const& c = b.c;
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  double rw, rn, Xw, Xn;
  bl_derive_at(b, Pw, Sn, K, percell, l, rw, rn, Xw, Xn);
  switch (field) {
    case CAPAZ_FIELD_S_W: out[l] = 1. - Sn[l]; return;
    case CAPAZ_FIELD_P_N: out[l] = Pw[l]; return;
    case CAPAZ_FIELD_RO_W: out[l] = rw; return;
    case CAPAZ_FIELD_RO_N: out[l] = rn; return;
    case CAPAZ_FIELD_XI_W: out[l] = Xw; return;
    case CAPAZ_FIELD_XI_N: out[l] = Xn; return;
    default: break;
  }
  if (field >= CAPAZ_FIELD_UX_W && field <= CAPAZ_FIELD_UZ_N) {
    // assign_u (cpu.cpp:346-477): central differences, one-sided at the ends.
    const bool wph = field <= CAPAZ_FIELD_UZ_W;
    const int axis = (field - CAPAZ_FIELD_UX_W) % 3;
    const long long s = axis == 0 ? 1 : axis == 1 ? c.sy : c.sz;
    const int idx = axis == 0 ? i : axis == 1 ? j : k;
    const int N = axis == 0 ? c.nx : axis == 1 ? c.ny : c.nz;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    if (N <= 2) {
      out[l] = 0.;
      return;
    }
    const double Pc = Pw[l];
    const double Pm = idx > 0 ? Pw[l - s] : 0., Pp = idx < N - 1 ? Pw[l + s] : 0.;
    const double Xc = wph ? Xw : Xn, ro = wph ? rw : rn;
    double d;
    if (idx == 0) d = (Pp - Pc) / h;
    else if (idx == N - 1) d = (Pc - Pm) / h;
    else d = (Pp - Pm) / (2. * h);
    out[l] = axis == 1 ? Xc * (d - ro * (c.g)) : Xc * d;
    return;
  }
  if (!bl_interior(c, i, j, k)) {
    out[l] = 0.;
    return;
  }
  const double S = Sn[l];
  if (field == CAPAZ_FIELD_ROS_W_OLD) {
    out[l] = rw * (1. - S);
    return;
  }
  if (field == CAPAZ_FIELD_ROS_N_OLD) {
    out[l] = rn * S;
    return;
  }
  double q_w, q_n, f_w[3], f_n[3];
  bl_wells(b, i, j, S, q_w, q_n);
  bl_fluxes(b, Pw, Sn, K, percell, l, rw, rn, Xw, Xn, f_w, f_n);
  if (field == CAPAZ_FIELD_ROS_W)
    out[l] = rw * (1. - S) - (c.dt / m[l]) * (-q_w + f_w[0] + f_w[1] + f_w[2]);
  else
    out[l] = rn * S - (c.dt / m[l]) * (-q_n + f_n[0] + f_n[1] + f_n[2]);
}

unsigned bl_blocks(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t launch_step_bl(const BLConst& b, const double* Pw_in, const double* Sn_in, double* Pw_out, double* Sn_out,
                           const double* m, const double* K, bool percell_k, unsigned int* err, cudaStream_t s) {
  const unsigned nb = bl_blocks(b.c.ncell);
  const Step2Const& c = b.c;
  const dim3 tiles((unsigned)((c.nx - 2 + TX - 1) / TX), (unsigned)((c.ny - 2 + TY - 1) / TY),
                   (unsigned)(c.nz < 2 ? 1 : c.nz - 2));
  if (tiles.y <= 65535u && tiles.z <= 65535u)
    step_bl_tile_kernel<<<tiles, dim3(TX, TY), 0, s>>>(b, Pw_in, Sn_in, Pw_out, Sn_out, m, K, percell_k, err);
  else  // beyond the grid's y/z block limits: one thread per cell
    step_bl_interior_kernel<<<nb, 256, 0, s>>>(b, Pw_in, Sn_in, Pw_out, Sn_out, m, K, percell_k, err);
  const int nbound = boundary_cells(c.nx, c.ny, c.nz);
  step_bl_boundary_kernel<<<(unsigned)((nbound + 255) / 256), 256, 0, s>>>(b, Pw_out, Sn_out, m, nbound);
  return cudaGetLastError();
}

cudaError_t launch_derived_bl(const BLConst& b, int field, const double* Pw, const double* Sn, const double* m,
                              const double* K, bool percell_k, double* out, cudaStream_t s) {
  derived_bl_kernel<<<bl_blocks(b.c.ncell), 256, 0, s>>>(b, field, Pw, Sn, m, K, percell_k, out);
  return cudaGetLastError();
}

}  // namespace capaz
