// Three-phase precision form: FP32 storage and stencil, FP64 Newton.
//
// The state is stored as FP32 deviations from a reference state: pressures
// P_w, P_n, P_g from the per-row reference pressure P_ref(j) (the row means
// of P_w when it was set), saturations S_w, S_n from their grid means.  One
// launch per step, tiled as the FP64 three-phase step (32 x 8 columns per
// CTA marching along z); the raw state of each plane's window is copied into
// shared memory with cp.async two planes ahead, and the derived planes live
// in a 4-slot ring, so one barrier per plane suffices:
//   - every cell of the plane window is derived in FP32: effective
//     saturations, the reference CPU relative permeabilities
//     (three-phase.cpp:146-186; square roots when A = 2), densities from the
//     per-row reference densities plus the linear pressure term, and the
//     mobility-densities M_p = K k_p rho_p / mu_p (= -Xi_p rho_p);
//   - the upwind flux difference of each phase (cpu.cpp:236-264 in select
//     form) is formed per axis as out - in, the three axis terms Kahan-summed
//     in FP32; d(rho S)_p = -dt/m div F_p goes to FP64;
//   - one Newton step in FP64 from the stored state solves the bilinear
//     increment equations rho_p(P + dP)(S_p + dS_p) - rho_p(P) S_p =
//     d(rho S)_p for (dP, dS_w, dS_n) (S_g = 1 - S_w - S_n) up to the dP dS
//     terms, with the 3x3 Jacobian solved by Cramer's rule and a refined
//     FP32-seeded reciprocal; the new deviations are rounded to FP32 once;
//   - boundary cells (Border_S, Border_P of three-phase.cpp:345-427) are
//     written by the thread of their basic-coordinate cell in FP64 from its
//     new state, as in the FP64 step.
// Diagnostics (mass per phase, the reference Newton functions' residual at
// the result, non-finite cells) are evaluated in FP64.
#include <math.h>
#include <stdint.h>

#include "capaz_internal.h"
#include "phys3f.cuh"

namespace capaz {
namespace {

// Derived values of one window cell: pressure deviations of the three
// phases and their mobility-densities.
struct Plane3F {
  float p[3][PC];
  float M[3][PC];
};
// Raw state of one plane of the window, copied from global memory ahead of
// its derive with cp.async (each thread copies and derives its own cells).
struct Raw3F {
  float pw[PC], sw[PC], sn[PC], K[PC], pn[PC], pg[PC];
};
constexpr int NRING = 4;  // derived planes: k-1, k, k+1 read while k+2 is derived
struct Smem3F {
  Plane3F ring[NRING];
  Raw3F raw[2];
};
constexpr size_t kSmem3F = sizeof(Smem3F);

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ bool interior3f(const Step3FConst& c, int i, int j, int k) {
  return (((i != 0) && (i != c.nx - 1)) || (c.nx < 2)) && (j != 0) && (j != c.ny - 1) &&
         (((k != 0) && (k != c.nz - 1)) || (c.nz < 2));
}
__device__ __forceinline__ bool in_window3f(const Step3FConst& c, int i, int k) {
  return (i >= c.nx / 2 - c.source) && (i <= c.nx / 2 + c.source) && (k >= c.win_k0) && (k <= c.win_k1);
}

__device__ __forceinline__ float face(float x1, float x2, float Mc, float Mm, float Mp) {
  return x2 * (x2 > 0.f ? Mc : Mp) - x1 * (x1 > 0.f ? Mm : Mc);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool UNIK, bool PLANAR, bool DIAG, bool A2>
__global__ void __launch_bounds__(NTHREADS, 2)
    step3_fp32c_kernel(const Step3FConst c, const Step3FArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem3F& sm = *reinterpret_cast<Smem3F*>(smem_raw);
  Plane3F* ring = sm.ring;
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
  const float den_inv = c.inv_den;
  static_assert(PC <= 2 * NTHREADS, "a thread derives at most two window cells per plane");

  // The (at most two) window cells this thread derives in every plane:
  // window index, grid offset in the plane, row, and whether the cell lies on
  // the grid and on an x/y boundary (whose P_n, P_g are stored state).
  int wq[2], wrow[2];
  long long woff[2];
  bool won[2], wbnd[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int q = tid + h * NTHREADS;
    const int gi = i0 - 1 + q % PX, gj = j0 - 1 + q / PX;
    wq[h] = q;
    won[h] = q < PC && gi >= 0 && gi < c.nx && gj < c.ny;
    wrow[h] = won[h] ? gj : 0;
    woff[h] = won[h] ? gi + gj * c.sy : 0;
    wbnd[h] = !((((gi != 0) && (gi != c.nx - 1)) || (c.nx < 2)) && (gj != 0) && (gj != c.ny - 1));
  }

  auto kbnd_of = [&](int k) { return !(((k != 0) && (k != c.nz - 1)) || (c.nz < 2)); };
  // Start copying the raw state of plane k's window cells of this thread
  // into raw stage b (one commit group per plane).
  auto issue = [&](int k, int b) {
    Raw3F& R = sm.raw[b];
    const bool kbnd = kbnd_of(k);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (won[h]) {
        const int q = wq[h];
        const long long l = woff[h] + (long long)k * c.sz;
        cp_async4(&R.pw[q], a.p_w + l);
        cp_async4(&R.sw[q], a.s_w + l);
        cp_async4(&R.sn[q], a.s_n + l);
        if (!UNIK) cp_async4(&R.K[q], a.K + l);
        if (wbnd[h] || kbnd) {
          cp_async4(&R.pn[q], a.p_n + l);
          cp_async4(&R.pg[q], a.p_g + l);
        }
      }
    }
    cp_async_commit();
  };
  // Derive plane k of the window from raw stage b into its ring slot.
  auto fill = [&](int k, int b) {
    Plane3F& P = ring[k % NRING];
    const Raw3F& R = sm.raw[b];
    const bool kbnd = kbnd_of(k);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (won[h]) {
        const int q = wq[h], gj = wrow[h];
        const float pw = R.pw[q];
        float pn = pw, pg = pw;  // interior: P_n = P_g = P_w (capillary pressures zero)
        if (wbnd[h] || kbnd) {
          pn = R.pn[q];
          pg = R.pg[q];
        }
        const float Sw = c.S_ref_w_f + R.sw[q], Sn = c.S_ref_n_f + R.sn[q];
        const float S_w_e = (Sw - c.S_wr_f) * den_inv, S_n_e = (Sn - c.S_nr_f) * den_inv;
        float k_w, k_n, k_g;
        relperm3f<A2>(c, S_w_e, S_n_e, k_w, k_n, k_g);
        const float Kl = UNIK ? c.K0_f : R.K[q];
        const float4 r = a.rowF[gj];  // rho_p(P_ref(j)) for w, n, g
        P.p[0][q] = pw;
        P.p[1][q] = pn;
        P.p[2][q] = pg;
        P.M[0][q] = Kl * k_w * fmaf(c.aw_f, pw, r.x) * c.inv_mu_w_f;
        P.M[1][q] = Kl * k_n * fmaf(c.an_f, pn, r.y) * c.inv_mu_n_f;
        P.M[2][q] = Kl * k_g * fmaf(c.bg_f, pg, r.z) * c.inv_mu_g_f;
      }
    }
  };

  double acc[3] = {0., 0., 0.}, rmax = 0., nonfinite = 0.;
  // Pipeline: the raw copy of plane k+2 is in flight while plane k+1 is
  // derived and plane k updated; plane k+1 goes into a ring slot that no
  // thread still reads (the update of k-1 read k-2..k), so one barrier per
  // plane suffices.  Raw stage of plane q: (q - kb + 1) & 1.
  if (PLANAR) {
    issue(kb, 0);
    cp_async_wait<0>();
    fill(kb, 0);
  } else {
    issue(kb - 1, 0);
    issue(kb, 1);
    cp_async_wait<1>();
    fill(kb - 1, 0);
    if (kb + 1 <= ke) issue(kb + 1, 0);
    else cp_async_commit();  // keep one group per plane
    cp_async_wait<1>();
    fill(kb, 1);
  }
  for (int k = kb; k < ke; k++) {
    if (!PLANAR) {
      const int b1 = (k + 1 - kb + 1) & 1;  // stage of plane k+1
      if (k + 2 <= ke) issue(k + 2, b1 ^ 1);
      else cp_async_commit();
      cp_async_wait<1>();
      fill(k + 1, b1);
    }
    __syncthreads();
    if (active) {
      const Plane3F& C = ring[k % NRING];
      const long long l = i + j * c.sy + (long long)k * c.sz;
      const float mc = a.m[l];
      const float sw0 = a.s_w[l], sn0 = a.s_n[l];
      const float4 row = a.rowF[j];
      const float dn = a.rowF[j - 1].w, dp = row.w;  // P_ref(j) - P_ref(j-1), P_ref(j+1) - P_ref(j)
      const float rho_row[3] = {row.x, row.y, row.z};
      const float slope[3] = {c.aw_f, c.an_f, c.bg_f};
      float div[3];
#pragma unroll
      for (int ph = 0; ph < 3; ph++) {
        const float pc = C.p[ph][cidx], Mc = C.M[ph][cidx];
        // x
        float fx = 0.f;
        if (c.nx >= 2) {
          const float pa = C.p[ph][cidx - 1], pb = C.p[ph][cidx + 1];
          fx = face((pa - pc) * c.inv_hx2_f, (pc - pb) * c.inv_hx2_f, Mc, C.M[ph][cidx - 1], C.M[ph][cidx + 1]);
        }
        // y (vertical, gravity g rho of the centre cell)
        const float gr = c.g_inv_hy_f * fmaf(slope[ph], pc, rho_row[ph]);
        const float y1 = fmaf(C.p[ph][cidx - PX] - pc, c.inv_hy2_f, -dn * c.inv_hy2_f) + gr;
        const float y2 = fmaf(pc - C.p[ph][cidx + PX], c.inv_hy2_f, -dp * c.inv_hy2_f) + gr;
        const float fy = face(y1, y2, Mc, C.M[ph][cidx - PX], C.M[ph][cidx + PX]);
        // Kahan sum of the axis terms
        float s = fx + fy;
        float comp = (s - fx) - fy;
        if (!PLANAR) {
          const Plane3F& Mz = ring[(k - 1) % NRING];
          const Plane3F& Qz = ring[(k + 1) % NRING];
          const float fz = face((Mz.p[ph][cidx] - pc) * c.inv_hz2_f, (pc - Qz.p[ph][cidx]) * c.inv_hz2_f, Mc,
                                Mz.M[ph][cidx], Qz.M[ph][cidx]);
          const float y = fz - comp;
          const float t = s + y;
          comp = (t - s) - y;
          s = t;
        }
        div[ph] = s - comp;
      }
      // Conserved increments d(rho S)_p = -dt/m div F_p, then Newton in FP64.
      const float dtm = __fdividef(c.dt_f, mc);
      const double dAw = (double)(-dtm * div[0]), dAn = (double)(-dtm * div[1]), dAg = (double)(-dtm * div[2]);
      const double prel = a.Pref[j] - c.P_atm;
      const double pw0 = (double)C.p[0][cidx];
      const double P = a.Pref[j] + pw0;
      const double Sw = c.S_ref_w + (double)sw0, Sn = c.S_ref_n + (double)sn0, Sg = 1. - Sw - Sn;
      const double rw = fma(c.aw, prel + pw0, c.ro0_w), rn = fma(c.an, prel + pw0, c.ro0_n);
      // One Newton step from the stored state (zero increments): the
      // Jacobian solve of the bilinear system, exact up to the dP dS terms
      // (relative size |dS| / S of the increments).  Jacobian in
      // (dP, dS_w, dS_n), with a13 = a22 = 0 and a33 = a32:
      //   [aw Sw   rw       0  ]
      //   [an Sn   0        rn ]
      //   [bg Sg  -bg P   -bg P]
      // and right-hand side (dAw, dAn, dAg).
      double dP, dSw, dSn;
      {
        const double a11 = c.aw * Sw, a12 = rw;
        const double a21 = c.an * Sn, a23 = rn;
        const double a31 = c.bg * Sg, a32 = -c.bg * P;
        const double c11 = -a23 * a32, c12 = a23 * a31 - a21 * a32, c13 = a21 * a32;
        const double det = a11 * c11 + a12 * c12;
        double inv = (double)__frcp_rn((float)det);  // FP32 seed, one Newton-Raphson step: 2^-46
        inv = inv * fma(-det, inv, 2.0);
        dP = (dAw * c11 + a12 * (a23 * dAg - dAn * a32)) * inv;
        dSw = (a11 * (dAn * a32 - a23 * dAg) + dAw * c12) * inv;
        dSn = (a12 * (dAn * a31 - a21 * dAg) + dAw * c13 - a11 * dAn * a32) * inv;
      }
      const double Pn1 = P + dP, Swn = Sw + dSw, Snn = Sn + dSn;
      a.o_pw[l] = (float)(pw0 + dP);
      a.o_sw[l] = (float)((double)sw0 + dSw);
      a.o_sn[l] = (float)((double)sn0 + dSn);
      const bool finite = isfinite(Pn1) && isfinite(Swn) && isfinite(Snn);
      if (!finite) atomicOr(a.err, 1u);

      // Border_S / Border_P for the boundary cells mapped onto (i, j, k).
      const bool xb = c.nx >= 3;
      const bool edge = (xb && (i == 1 || i == c.nx - 2)) || (j == 1) || (j == c.ny - 2) ||
                        (!PLANAR && ((k == 1) || (k == c.nz - 2)));
      if (edge) {
        // Candidate coordinates per axis: the cell's own, then the boundary
        // planes it is the basic coordinate of (-1: none).  Fixed-size,
        // fully unrolled loops keep these in registers.
        const int xs[3] = {i, (xb && i == 1) ? 0 : -1, (xb && i == c.nx - 2) ? c.nx - 1 : -1};
        const int ys[3] = {j, (j == 1) ? 0 : -1, (j == c.ny - 2) ? c.ny - 1 : -1};
        const int zs[3] = {k, (!PLANAR && k == 1) ? 0 : -1, (!PLANAR && k == c.nz - 2) ? c.nz - 1 : -1};
#pragma unroll
        for (int qa = 0; qa < 3; qa++)
#pragma unroll
          for (int qb = 0; qb < 3; qb++)
#pragma unroll
            for (int qd = 0; qd < 3; qd++) {
              if (qa == 0 && qb == 0 && qd == 0) continue;
              if (xs[qa] < 0 || ys[qb] < 0 || zs[qd] < 0) continue;
              const int bj = ys[qb], bi = xs[qa], bk = zs[qd];
              const long long lb = bi + bj * c.sy + (long long)bk * c.sz;
              double sw = Swn, sn = Snn;
              if ((bj == 0) && (c.source > 0) && (!c.source_window || in_window3f(c, bi, bk))) {
                sw = c.S_w_gr;
                sn = c.S_n_gr;
              }
              double pw, pn, pg;
              if ((bj != 0) && (bj != c.ny - 1)) {
                pw = pn = pg = Pn1;
              } else if (bj == 0) {
                pw = (Pn1 - (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
                     (1. + (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
                pn = (Pn1 - (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
                     (1. + (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
                pg = Pn1 / (1. + (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
              } else {
                pw = (Pn1 + (c.ro0_w) * (c.g) * (c.hy) * (1. - (c.beta_w) * (c.P_atm))) /
                     (1. - (c.beta_w) * (c.ro0_w) * (c.g) * (c.hy));
                pn = (Pn1 + (c.ro0_n) * (c.g) * (c.hy) * (1. - (c.beta_n) * (c.P_atm))) /
                     (1. - (c.beta_n) * (c.ro0_n) * (c.g) * (c.hy));
                pg = Pn1 / (1. - (c.ro0_g) * (c.g) * (c.hy) / (c.P_atm));
              }
              const double pr = a.Pref[bj];
              a.o_sw[lb] = (float)(sw - c.S_ref_w);
              a.o_sn[lb] = (float)(sn - c.S_ref_n);
              a.o_pw[lb] = (float)(pw - pr);
              a.o_pn[lb] = (float)(pn - pr);
              a.o_pg[lb] = (float)(pg - pr);
            }
      }
      if (DIAG) {
        const double Sgn = 1. - Swn - Snn;
        const double rw1 = c.ro0_w * (1. + (c.beta_w) * (Pn1 - c.P_atm));
        const double rn1 = c.ro0_n * (1. + (c.beta_n) * (Pn1 - c.P_atm));
        const double rg1 = c.ro0_g * Pn1 / c.P_atm;
        const double vm = (double)mc * c.vol;
        acc[0] += vm * rw1 * Swn;
        acc[1] += vm * rn1 * Snn;
        acc[2] += vm * rg1 * Sgn;
        // the reference's Newton functions F_p = rho_p S_p - roS_p at the result
        const double G1 = rw1 * Swn - (rw * Sw + dAw);
        const double G2 = rn1 * Snn - (rn * Sn + dAn);
        const double G3 = rg1 * Sgn - (c.ro0_g * P / c.P_atm * Sg + dAg);
        const double r = fmax(fmax(fabs(G1) / c.ro0_w, fabs(G2) / c.ro0_n), fabs(G3) / c.ro0_g);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    }
  }
  cp_async_wait<0>();

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
      double* o = a.diag + (size_t)DIAG_STRIDE * (blockIdx.x + (size_t)gridDim.x * blockIdx.y);
      for (int q = 0; q < 5; q++) o[q] = t[q];
    }
  }
}

template <bool UNIK, bool PLANAR, bool DIAG, bool A2>
cudaError_t launch_t(const Step3FConst& c, const Step3FArgs& a, cudaStream_t s) {
  auto kern = step3_fp32c_kernel<UNIK, PLANAR, DIAG, A2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem3F);
  if (e != cudaSuccess) return e;
  dim3 grid(c.tiles_x * c.tiles_y, c.nzchunks);
  kern<<<grid, dim3(TX, TY), kSmem3F, s>>>(c, a);
  return cudaGetLastError();
}

template <bool UNIK, bool PLANAR, bool DIAG>
cudaError_t launch_a(const Step3FConst& c, const Step3FArgs& a, cudaStream_t s) {
  return c.a2 ? launch_t<UNIK, PLANAR, DIAG, true>(c, a, s) : launch_t<UNIK, PLANAR, DIAG, false>(c, a, s);
}

template <bool UNIK, bool PLANAR>
cudaError_t launch_d(const Step3FConst& c, const Step3FArgs& a, cudaStream_t s) {
  return a.diag ? launch_a<UNIK, PLANAR, true>(c, a, s) : launch_a<UNIK, PLANAR, false>(c, a, s);
}

__global__ void row_tables3_kernel(const double* __restrict__ Pref, int ny, double P_atm, double ro0_w, double ro0_n,
                                   double ro0_g, double aw, double an, float4* __restrict__ rowF) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny) return;
  const double prel = Pref[j] - P_atm;
  const double dnext = (j + 1 < ny) ? (Pref[j + 1] - Pref[j]) : 0.;
  rowF[j] = make_float4((float)(ro0_w + aw * prel), (float)(ro0_n + an * prel), (float)(ro0_g * Pref[j] / P_atm),
                        (float)dnext);
}

}  // namespace

cudaError_t launch_step3_fp32c(const Step3FConst& c, const Step3FArgs& a, cudaStream_t s) {
  const bool unik = a.K == nullptr, planar = c.nz == 1;
  if (unik) return planar ? launch_d<true, true>(c, a, s) : launch_d<true, false>(c, a, s);
  return planar ? launch_d<false, true>(c, a, s) : launch_d<false, false>(c, a, s);
}

cudaError_t launch_row_tables3(const double* Pref, int ny, const Step3FConst& c, float4* rowF, cudaStream_t s) {
  row_tables3_kernel<<<(ny + 127) / 128, 128, 0, s>>>(Pref, ny, c.P_atm, c.ro0_w, c.ro0_n, c.ro0_g, c.aw, c.an, rowF);
  return cudaGetLastError();
}

}  // namespace capaz
