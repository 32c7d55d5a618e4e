// Fused three-phase (water / NAPL / gas) time step, FP64 ("plain" form).
//
// One launch performs the reference CPU three-phase time step:
//   S_calculation       S_g = 1 - S_w - S_n                (cpu.cpp:171-182)
//   ro_P_Xi_calculation relative permeabilities of three-phase.cpp:146-186,
//                       Xi on every cell, P_n = P_g = P_w on interior cells
//                       (capillary pressures are zero in the CPU model,
//                       three-phase.cpp:23-143), rho_w, rho_n, ideal-gas rho_g
//                       (cpu.cpp:158-160)
//   roS_calculation     upwind flux difference for the three phases
//                       (cpu.cpp:619-731)
//   P_S_calculation     `ITERATIONS` Newton iterations on (P_w, S_w, S_n) with
//                       the Jacobian of three-phase.cpp:307-323 inverted by
//                       the Gauss-Jordan elimination of gauss.cpp:6-92
//   boundary_conditions Border_S / Border_P of three-phase.cpp:345-427
// Storage: P_w, S_w, S_n on all cells; P_n, P_g are state only on boundary
// cells (interior values are P_w, recomputed).  Ping-pong buffers as in the
// two-phase step.  Compiled with -fmad=false, reference operation order.
#include <math.h>

#include "capaz_internal.h"
#include "phys3.cuh"

namespace capaz {
namespace {

using phys3::directed;
using phys3::k_g3;
using phys3::k_n3;
using phys3::k_w3;

struct Plane3 {
  double Pw[PC], Pn[PC], Pg[PC], ro_w[PC], ro_n[PC], ro_g[PC], Xi_w[PC], Xi_n[PC], Xi_g[PC];
};
constexpr size_t kSmem3 = 3 * sizeof(Plane3);

__device__ __forceinline__ bool interior3(const Step3Const& c, int i, int j, int k) {
  return (((i != 0) && (i != c.nx - 1)) || (c.nx < 2)) && (j != 0) && (j != c.ny - 1) &&
         (((k != 0) && (k != c.nz - 1)) || (c.nz < 2));
}

struct D3 {
  double Pw, Pn, Pg, ro_w, ro_n, ro_g, Xi_w, Xi_n, Xi_g;
};

// ro_P_Xi for one cell (three-phase.cpp:198-240, cpu.cpp:158-160).
__device__ __forceinline__ D3 derive3(const Step3Const& c, double Pw, double Sw, double Sn, double Pn_st,
                                     double Pg_st, double K, bool inter) {
  D3 o;
  const double den = 1. - c.S_wr - c.S_nr - c.S_gr;
  double S_w_e = (Sw - c.S_wr) / den;
  double S_n_e = (Sn - c.S_nr) / den;
  double S_g_e = 1. - S_w_e - S_n_e;
  double k_w = k_w3(S_w_e, c.A, c.a2), k_g = k_g3(S_g_e, c.A, c.a2), k_n = k_n3(S_w_e, S_n_e, c.A, c.a2);
  o.Xi_w = (-1.) * K * k_w / c.mu_w;
  o.Xi_n = (-1.) * K * k_n / c.mu_n;
  o.Xi_g = (-1.) * K * k_g / c.mu_g;
  o.Pw = Pw;
  if (inter) {
    const double Pk_nw = 0, Pk_gn = 0;
    o.Pn = Pw + Pk_nw;
    o.Pg = Pw + Pk_nw + Pk_gn;
  } else {
    o.Pn = Pn_st;
    o.Pg = Pg_st;
  }
  o.ro_w = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm));
  o.ro_n = c.ro0_n * (1. + (c.beta_n) * (o.Pn - c.P_atm));
  o.ro_g = c.ro0_g * o.Pg / c.P_atm;
  return o;
}

__device__ __forceinline__ bool in_window3(const Step3Const& c, int i, int k) {
  return (i >= c.nx / 2 - c.source) && (i <= c.nx / 2 + c.source) && (k >= c.win_k0) && (k <= c.win_k1);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Three CTAs per SM (3 x 73 KB of plane ring, 85 registers): the FP64
// pipeline needs the resident warps more than the registers.
template <bool UNIK, bool PLANAR, bool DIAG>
__global__ void __launch_bounds__(NTHREADS, 3)
    step3_fp64_kernel(const Step3Const c, Step3Buffers in, Step3Buffers out, const double* __restrict__ m,
                      const double* __restrict__ K, double* __restrict__ diag_partials,
                      unsigned int* __restrict__ err_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Plane3* ring = reinterpret_cast<Plane3*>(smem_raw);
  const int tid = threadIdx.x + TX * threadIdx.y;
  const int tile = blockIdx.x;
  const int ti = tile % c.tiles_x, tj = tile / c.tiles_x;
  const int i0 = c.i_lo + ti * TX, j0 = 1 + tj * TY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const bool active = (i <= c.i_hi) && (j <= c.ny - 2);
  const int cidx = (threadIdx.y + 1) * PX + (threadIdx.x + 1);
  int kb, ke;
  if (PLANAR) {
    kb = 0;
    ke = 1;
  } else {
    kb = 1 + blockIdx.y * c.zchunk;
    ke = min(kb + c.zchunk, c.nz - 1);
  }

  auto fill = [&](int k) {
    Plane3& P = ring[k % 3];
    for (int q = tid; q < PC; q += NTHREADS) {
      int gi = i0 - 1 + q % PX, gj = j0 - 1 + q / PX;
      if (gi >= 0 && gi < c.nx && gj < c.ny) {
        long long l = gi + gj * c.sy + (long long)k * c.sz;
        double Kl = UNIK ? c.K0 : K[l];
        D3 d = derive3(c, in.Pw[l], in.Sw[l], in.Sn[l], in.Pn[l], in.Pg[l], Kl, interior3(c, gi, gj, k));
        P.Pw[q] = d.Pw;
        P.Pn[q] = d.Pn;
        P.Pg[q] = d.Pg;
        P.ro_w[q] = d.ro_w;
        P.ro_n[q] = d.ro_n;
        P.ro_g[q] = d.ro_g;
        P.Xi_w[q] = d.Xi_w;
        P.Xi_n[q] = d.Xi_n;
        P.Xi_g[q] = d.Xi_g;
      }
    }
  };

  double acc[3] = {0., 0., 0.}, rmax = 0., nonfinite = 0.;
  if (!PLANAR) fill(kb - 1);
  fill(kb);
  for (int k = kb; k < ke; k++) {
    if (!PLANAR) fill(k + 1);
    __syncthreads();
    if (active) {
      const Plane3& C = ring[k % 3];
      const long long l = i + j * c.sy + (long long)k * c.sz;
      const double mc = m[l];
      const double Sw0 = in.Sw[l], Sn0 = in.Sn[l];
      const double q_w = 0., q_n = 0., q_g = 0.;  // wells_q (three-phase.cpp:529-550)
      const double roS_w = C.ro_w[cidx] * Sw0;
      const double roS_g = C.ro_g[cidx] * (1. - Sw0 - Sn0);
      const double roS_n = C.ro_n[cidx] * Sn0;
      double f[3][3];  // [phase][axis x,y,z]
      const double* Pp[3] = {C.Pw, C.Pn, C.Pg};
      const double* Rp[3] = {C.ro_w, C.ro_n, C.ro_g};
      const double* Xp[3] = {C.Xi_w, C.Xi_n, C.Xi_g};
#pragma unroll
      for (int ph = 0; ph < 3; ph++) {
        const double Pc = Pp[ph][cidx], rc = Rp[ph][cidx], Xc = Xp[ph][cidx];
        double x1, x2;
        if (PLANAR) {
          f[ph][2] = 0.;
        } else {
          const Plane3& M = ring[(k + 2) % 3];
          const Plane3& Q = ring[(k + 1) % 3];
          const double* PM[3] = {M.Pw, M.Pn, M.Pg};
          const double* PQ[3] = {Q.Pw, Q.Pn, Q.Pg};
          const double* RM[3] = {M.ro_w, M.ro_n, M.ro_g};
          const double* RQ[3] = {Q.ro_w, Q.ro_n, Q.ro_g};
          const double* XM[3] = {M.Xi_w, M.Xi_n, M.Xi_g};
          const double* XQ[3] = {Q.Xi_w, Q.Xi_n, Q.Xi_g};
          x2 = -1. * ((PQ[ph][cidx] - Pc) / c.hz);
          x1 = -1. * ((Pc - PM[ph][cidx]) / c.hz);
          f[ph][2] = directed(x1, x2, Xc, rc, XM[ph][cidx], RM[ph][cidx], XQ[ph][cidx], RQ[ph][cidx], c.hz);
        }
        if (c.nx < 2) {
          f[ph][0] = 0.;
        } else {
          const int a = cidx - 1, b = cidx + 1;
          x2 = -1. * ((Pp[ph][b] - Pc) / c.hx);
          x1 = -1. * ((Pc - Pp[ph][a]) / c.hx);
          f[ph][0] = directed(x1, x2, Xc, rc, Xp[ph][a], Rp[ph][a], Xp[ph][b], Rp[ph][b], c.hx);
        }
        {
          const int a = cidx - PX, b = cidx + PX;
          x2 = -1. * ((Pp[ph][b] - Pc) / c.hy) + c.g * (rc);
          x1 = -1. * ((Pc - Pp[ph][a]) / c.hy) + c.g * (rc);
          f[ph][1] = directed(x1, x2, Xc, rc, Xp[ph][a], Rp[ph][a], Xp[ph][b], Rp[ph][b], c.hy);
        }
      }
      const double dtm = c.dt / mc;
      const double A1 = roS_w - dtm * (-q_w + f[0][0] + f[0][1] + f[0][2]);
      const double A2 = roS_n - dtm * (-q_n + f[1][0] + f[1][1] + f[1][2]);
      const double A3 = roS_g - dtm * (q_g + f[2][0] + f[2][1] + f[2][2]);

      // Newton (three-phase.cpp:294-333).
      double Pw = C.Pw[cidx], Sw = Sw0, Sn = Sn0;
      double F1 = 0, F2 = 0, F3 = 0;
      for (int w = 1; w <= c.iters; w++) {
        const double Pk_nw = 0, Pk_gn = 0, PkSw = 0, PkSn = 0;
        double Sg = 1. - Sw - Sn;
        F1 = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm)) * Sw - A1;
        F2 = c.ro0_n * (1. + (c.beta_n) * (Pw + Pk_nw - c.P_atm)) * Sn - A2;
        F3 = c.ro0_g * (Pw + Pk_nw + Pk_gn) / c.P_atm * Sg - A3;
        double dF[9];
        dF[0] = c.ro0_w * c.beta_w * Sw;
        dF[3] = c.ro0_n * c.beta_n * Sn;
        dF[6] = c.ro0_g * Sg / c.P_atm;
        dF[1] = c.ro0_w * (1 + c.beta_w * (Pw - c.P_atm));
        dF[4] = c.ro0_n * (1. + (c.beta_n) * PkSw) * Sn;
        dF[7] = (-1) * c.ro0_g * (Pw + Pk_nw + Pk_gn - Sg * (PkSn + PkSw)) / c.P_atm;
        dF[2] = 0;
        dF[5] = c.ro0_n * (1. + c.beta_n * (Pw + Pk_nw - c.P_atm));
        dF[8] = (-1) * c.ro0_g * (Pw + Pk_nw + Pk_gn - Sg * PkSn) / c.P_atm;
        phys3::reverse_matrix<3>(dF);
        double nPw = Pw - (dF[0] * F1 + dF[1] * F2 + dF[2] * F3);
        double nSw = Sw - (dF[3] * F1 + dF[4] * F2 + dF[5] * F3);
        double nSn = Sn - (dF[6] * F1 + dF[7] * F2 + dF[8] * F3);
        Pw = nPw;
        Sw = nSw;
        Sn = nSn;
      }
      out.Pw[l] = Pw;
      out.Sw[l] = Sw;
      out.Sn[l] = Sn;
      const bool finite = isfinite(Pw) && isfinite(Sw) && isfinite(Sn);
      if (!finite) atomicOr(err_flag, 1u);

      // Border_S / Border_P for the boundary cells mapped onto (i, j, k).
      const bool xb = c.nx >= 3;
      const bool edge = (xb && (i == 1 || i == c.nx - 2)) || (j == 1) || (j == c.ny - 2) ||
                        (!PLANAR && ((k == 1) || (k == c.nz - 2)));
      if (edge) {
        int xs[3], ys[3], zs[3], nxs = 0, nys = 0, nzs = 0;
        xs[nxs++] = i;
        if (xb && i == 1) xs[nxs++] = 0;
        if (xb && i == c.nx - 2) xs[nxs++] = c.nx - 1;
        ys[nys++] = j;
        if (j == 1) ys[nys++] = 0;
        if (j == c.ny - 2) ys[nys++] = c.ny - 1;
        zs[nzs++] = k;
        if (!PLANAR) {
          if (k == 1) zs[nzs++] = 0;
          if (k == c.nz - 2) zs[nzs++] = c.nz - 1;
        }
        const double Pk_nw = 0, Pk_gn = 0;
        for (int qa = 0; qa < nxs; qa++)
          for (int qb = 0; qb < nys; qb++)
            for (int qd = 0; qd < nzs; qd++) {
              if (qa == 0 && qb == 0 && qd == 0) continue;
              const int bj = ys[qb], bi = xs[qa], bk = zs[qd];
              const long long lb = bi + bj * c.sy + (long long)bk * c.sz;
              double sw = Sw, sn = Sn;
              if ((bj == 0) && (c.source > 0) && (!c.source_window || in_window3(c, bi, bk))) {
                sw = c.S_w_gr;
                sn = c.S_n_gr;
              }
              double pw, pn, pg;
              if ((bj != 0) && (bj != c.ny - 1)) {
                pw = Pw;
                pn = Pw + Pk_nw;
                pg = Pw + Pk_nw + Pk_gn;
              } else if (bj == 0) {
                pw = (Pw - (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
                     (1. + (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
                pn = (Pw + Pk_nw - (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
                     (1. + (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
                pg = (Pw + Pk_nw + Pk_gn) / (1. + (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
              } else {
                pw = (Pw + (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
                     (1. - (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
                pn = (Pw + Pk_nw + (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
                     (1. - (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
                pg = (Pw + Pk_nw + Pk_gn) / (1. - (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
              }
              out.Sw[lb] = sw;
              out.Sn[lb] = sn;
              out.Pw[lb] = pw;
              out.Pn[lb] = pn;
              out.Pg[lb] = pg;
            }
      }
      if (DIAG) {
        const double Sg = 1. - Sw - Sn;
        const double rw = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm));
        const double rn = c.ro0_n * (1. + (c.beta_n) * (Pw - c.P_atm));
        const double rg = c.ro0_g * Pw / c.P_atm;
        acc[0] += mc * rw * Sw * c.vol;
        acc[1] += mc * rn * Sn * c.vol;
        acc[2] += mc * rg * Sg * c.vol;
        const double G1 = rw * Sw - A1, G2 = rn * Sn - A2, G3 = rg * Sg - A3;
        const double r = fmax(fmax(fabs(G1) / c.ro0_w, fabs(G2) / c.ro0_n), fabs(G3) / c.ro0_g);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    }
    __syncthreads();
  }

  if (DIAG) {
    __shared__ double red[NTHREADS / 32][5];
    const int lane = tid & 31, wid = tid >> 5;
    double v[5] = {warp_sum(acc[0]), warp_sum(acc[1]), warp_sum(acc[2]), warp_max(rmax), warp_sum(nonfinite)};
    if (lane == 0)
      for (int q = 0; q < 5; q++) red[wid][q] = v[q];
    __syncthreads();
    if (tid == 0) {
      double t[5] = {0, 0, 0, 0, 0};
      for (int w = 0; w < NTHREADS / 32; w++) {
        t[0] += red[w][0];
        t[1] += red[w][1];
        t[2] += red[w][2];
        t[3] = fmax(t[3], red[w][3]);
        t[4] += red[w][4];
      }
      double* o = diag_partials + (size_t)DIAG_STRIDE * (blockIdx.x + (size_t)gridDim.x * blockIdx.y);
      for (int q = 0; q < 5; q++) o[q] = t[q];
    }
  }
}

template <bool UNIK, bool PLANAR, bool DIAG>
cudaError_t launch_t(const Step3Const& c, const Step3Buffers& in, const Step3Buffers& out, const double* m,
                     const double* K, double* diag, unsigned int* err, cudaStream_t s) {
  auto kern = step3_fp64_kernel<UNIK, PLANAR, DIAG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem3);
  if (e != cudaSuccess) return e;
  dim3 grid(c.tiles_x * c.tiles_y, c.nzchunks);
  kern<<<grid, dim3(TX, TY), kSmem3, s>>>(c, in, out, m, K, diag, err);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_step3_fp64(const Step3Const& c, const Step3Buffers& in, const Step3Buffers& out, const double* m,
                              const double* K, double* diag, unsigned int* err, cudaStream_t s) {
  const bool unik = K == nullptr, planar = c.nz == 1, dg = diag != nullptr;
  if (unik) {
    if (planar) return dg ? launch_t<true, true, true>(c, in, out, m, K, diag, err, s) : launch_t<true, true, false>(c, in, out, m, K, diag, err, s);
    return dg ? launch_t<true, false, true>(c, in, out, m, K, diag, err, s) : launch_t<true, false, false>(c, in, out, m, K, diag, err, s);
  }
  if (planar) return dg ? launch_t<false, true, true>(c, in, out, m, K, diag, err, s) : launch_t<false, true, false>(c, in, out, m, K, diag, err, s);
  return dg ? launch_t<false, false, true>(c, in, out, m, K, diag, err, s) : launch_t<false, false, false>(c, in, out, m, K, diag, err, s);
}

// ---------------------------------------------------------------------------
// Derived fields of a three-phase state (not on the hot path).
namespace {
__global__ void derived3_kernel(const Step3Const c, int field, Step3Buffers st, const double* __restrict__ m,
                                const double* __restrict__ K, double* __restrict__ out) {
  long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  auto at = [&](long long q, int qi, int qj, int qk) {
    return derive3(c, st.Pw[q], st.Sw[q], st.Sn[q], st.Pn[q], st.Pg[q], K ? K[q] : c.K0, interior3(c, qi, qj, qk));
  };
  const D3 d = at(l, i, j, k);
  switch (field) {
    case CAPAZ_FIELD_S_G: out[l] = 1. - st.Sw[l] - st.Sn[l]; return;
    case CAPAZ_FIELD_RO_W: out[l] = d.ro_w; return;
    case CAPAZ_FIELD_RO_N: out[l] = d.ro_n; return;
    case CAPAZ_FIELD_RO_G: out[l] = d.ro_g; return;
    case CAPAZ_FIELD_XI_W: out[l] = d.Xi_w; return;
    case CAPAZ_FIELD_XI_N: out[l] = d.Xi_n; return;
    case CAPAZ_FIELD_XI_G: out[l] = d.Xi_g; return;
    default: break;
  }
  if (field >= CAPAZ_FIELD_UX_W && field <= CAPAZ_FIELD_UZ_G) {
    const int ph = (field - CAPAZ_FIELD_UX_W) / 3, axis = (field - CAPAZ_FIELD_UX_W) % 3;
    const long long s = axis == 0 ? 1 : axis == 1 ? c.sy : c.sz;
    const int idx = axis == 0 ? i : axis == 1 ? j : k;
    const int N = axis == 0 ? c.nx : axis == 1 ? c.ny : c.nz;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    if (N <= 2) {
      out[l] = 0.;
      return;
    }
    auto Pof = [&](const D3& x) { return ph == 0 ? x.Pw : ph == 1 ? x.Pn : x.Pg; };
    const double Xc = ph == 0 ? d.Xi_w : ph == 1 ? d.Xi_n : d.Xi_g;
    const double rc = ph == 0 ? d.ro_w : ph == 1 ? d.ro_n : d.ro_g;
    const double Pc = Pof(d);
    double Pm = 0., Pp = 0.;
    if (idx > 0) Pm = Pof(at(l - s, i - (axis == 0), j - (axis == 1), k - (axis == 2)));
    if (idx < N - 1) Pp = Pof(at(l + s, i + (axis == 0), j + (axis == 1), k + (axis == 2)));
    double dd;
    if (idx == 0) dd = (Pp - Pc) / h;
    else if (idx == N - 1) dd = (Pc - Pm) / h;
    else dd = (Pp - Pm) / (2. * h);
    out[l] = (axis == 1) ? Xc * (dd - rc * (c.g)) : Xc * dd;
    return;
  }
  if (!interior3(c, i, j, k)) {
    out[l] = 0.;
    return;
  }
  const double Sw = st.Sw[l], Sn = st.Sn[l];
  if (field == CAPAZ_FIELD_ROS_W_OLD) { out[l] = d.ro_w * Sw; return; }
  if (field == CAPAZ_FIELD_ROS_N_OLD) { out[l] = d.ro_n * Sn; return; }
  if (field == CAPAZ_FIELD_ROS_G_OLD) { out[l] = d.ro_g * (1. - Sw - Sn); return; }
  const int ph = field == CAPAZ_FIELD_ROS_W ? 0 : field == CAPAZ_FIELD_ROS_N ? 1 : 2;
  auto Pof = [&](const D3& x) { return ph == 0 ? x.Pw : ph == 1 ? x.Pn : x.Pg; };
  auto Xof = [&](const D3& x) { return ph == 0 ? x.Xi_w : ph == 1 ? x.Xi_n : x.Xi_g; };
  auto Rof = [&](const D3& x) { return ph == 0 ? x.ro_w : ph == 1 ? x.ro_n : x.ro_g; };
  double f[3] = {0., 0., 0.};
  for (int axis = 0; axis < 3; axis++) {
    if (axis == 0 && c.nx < 2) continue;
    if (axis == 2 && c.nz < 2) continue;
    const long long s = axis == 0 ? 1 : axis == 1 ? c.sy : c.sz;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    const D3 dm = at(l - s, i - (axis == 0), j - (axis == 1), k - (axis == 2));
    const D3 dp = at(l + s, i + (axis == 0), j + (axis == 1), k + (axis == 2));
    double x2 = -1. * ((Pof(dp) - Pof(d)) / h), x1 = -1. * ((Pof(d) - Pof(dm)) / h);
    if (axis == 1) {
      x2 = x2 + c.g * (Rof(d));
      x1 = x1 + c.g * (Rof(d));
    }
    f[axis] = directed(x1, x2, Xof(d), Rof(d), Xof(dm), Rof(dm), Xof(dp), Rof(dp), h);
  }
  const double roS = ph == 0 ? d.ro_w * Sw : ph == 1 ? d.ro_n * Sn : d.ro_g * (1. - Sw - Sn);
  const double q0 = ph == 2 ? 0. : -0.;
  out[l] = roS - (c.dt / m[l]) * (q0 + f[0] + f[1] + f[2]);
}

// P_n / P_g as the reference's arrays hold them after a step: interior cells
// carry the start-of-step P_w (ro_P_Xi_calculation), boundary cells the value
// of the step's Border_P.
__global__ void compose3_kernel(const Step3Const c, const double* __restrict__ Pw_start,
                                const double* __restrict__ bnd_now, double* __restrict__ out) {
  long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  out[l] = interior3(c, i, j, k) ? Pw_start[l] + 0. : bnd_now[l];
}
}  // namespace

cudaError_t launch_derived3_fp64(const Step3Const& c, int field, const Step3Buffers& st, const double* m,
                                 const double* K, double* out, cudaStream_t s) {
  const int bs = 128;
  derived3_kernel<<<(unsigned)((c.ncell + bs - 1) / bs), bs, 0, s>>>(c, field, st, m, K, out);
  return cudaGetLastError();
}

cudaError_t launch_compose3(const Step3Const& c, const double* Pw_start, const double* bnd_now, double* out,
                            cudaStream_t s) {
  const int bs = 256;
  compose3_kernel<<<(unsigned)((c.ncell + bs - 1) / bs), bs, 0, s>>>(c, Pw_start, bnd_now, out);
  return cudaGetLastError();
}

}  // namespace capaz
