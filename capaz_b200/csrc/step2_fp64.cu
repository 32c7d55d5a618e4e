// Fused two-phase time step, FP64 ("plain" form).
//
// One launch performs the reference's whole time_step_function
// (main.cpp:93-108) on one rank:
//   S_calculation      -> S_w = 1 - S_n is never stored (used in registers)
//   ro_P_Xi_calculation-> P_n, Xi_w, Xi_n, rho_w, rho_n per cell, computed once
//                         per plane window in shared memory, halo included
//                         (two-phase.cpp:4-23, cpu.cpp:143-169)
//   u_calculation      -> not needed by the NR update; materialised on request
//   roS_calculation    -> upwind 7-point flux difference (cpu.cpp:619-731)
//   P_S_calculation    -> 2x2 Newton in registers (two-phase.cpp:25-56)
//   boundary_conditions-> each interior cell next to the boundary writes the
//                         boundary cells whose basic coordinate it is
//                         (cpu.cpp:107-141, two-phase.cpp:59-111)
// State is ping-ponged: the step reads (P_w, S_n) from one buffer pair and
// writes every cell of the other, so a cell's state makes one HBM round trip
// per step and nothing else is stored.
//
// Arithmetic: this file is compiled with -fmad=false and every expression
// keeps the reference's operation order, so each add, multiply and divide is
// the same IEEE-754 double operation the reference CPU build performs.  The
// only difference from the CPU build is pow (CUDA's vs the host libm's).
//
// Layout: tile of TX x TY interior columns per CTA (one thread each), marching
// a chunk of z-planes; a ring of three plane windows ((TX+2) x (TY+2), one-cell
// halo) of the derived quantities lives in shared memory.
#include <math.h>

#include "capaz_internal.h"
#include "diag_reduce.cuh"

namespace capaz {
namespace {

// The neighbours' derived values (the cell's own S_n comes from global
// memory): 6 fields, 49 KB for the ring, so that four CTAs fit an SM.
struct Plane2 {
  double Pw[PC], Pn[PC], ro_w[PC], ro_n[PC], Xi_w[PC], Xi_n[PC];
};
constexpr size_t kSmem2 = 3 * sizeof(Plane2);

// ro_P_Xi for one cell (two-phase.cpp:8-17; cpu.cpp:164-165).
template <bool PD0>
__device__ __forceinline__ void derive2(const Step2Const& c, double Pw, double Sn, double K, double& Pn,
                                        double& ro_w, double& ro_n, double& Xi_w, double& Xi_n) {
  double S_e = (1. - Sn - c.S_wr) / (1. - c.S_wr);
  double k_w, k_n;
  if (c.lam2) {
    // lambda == 2: S_e^4 and S_e^2 as products (CAPAZ_FLAG_POW_PRODUCTS).
    const double e2 = S_e * S_e;
    k_w = e2 * e2;
    k_n = (1. - S_e) * (1. - S_e) * (1 - e2);
  } else {
    k_w = pow(S_e, c.e_kw);
    k_n = (1. - S_e) * (1. - S_e) * (1 - pow(S_e, c.e_kn));
  }
  double P_k;
  if (PD0 && S_e >= c.se_fast_min) {
    P_k = 0.;  // P_d == 0 and pow finite: P_d*pow(...) is +0 exactly
  } else {
    P_k = c.P_d * pow((1. - Sn - c.S_wr) / (1. - c.S_wr), c.e_pk);
  }
  Pn = Pw + P_k;
  Xi_w = -1. * K * k_w / c.mu_w;
  Xi_n = -1. * K * k_n / c.mu_n;
  ro_w = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm));
  ro_n = c.ro0_n * (1. + (c.beta_n) * (Pn - c.P_atm));
}

// directed_difference (cpu.cpp:236-264) with the neighbour values passed in.
__device__ __forceinline__ double directed(double x1, double x2, double Xc, double rc, double Xm, double rm,
                                           double Xp, double rp, double h) {
  return (((x2 + fabs(x2)) / 2. - (x1 - fabs(x1)) / 2.) * (-1.) * Xc * rc -
          (x1 + fabs(x1)) / 2. * (-1.) * Xm * rm + (x2 - fabs(x2)) / 2. * (-1.) * Xp * rp) /
         h;
}

// Newton for one interior cell (two-phase.cpp:33-50), state in registers.
template <bool PD0>
__device__ __forceinline__ void newton2(const Step2Const& c, double roS_w, double roS_n, double& Pw,
                                        double& Sn) {
  for (int w = 1; w <= c.iters; w++) {
    double P_k, PkS;
    // P_d == 0: P_k and PkS are +0 whenever S_e is above the threshold;
    // the numerator alone decides that in all but a sliver next to it.
    if (PD0 && (1 - Sn - c.S_wr) > c.se_fast_num) {
      P_k = 0.;
      PkS = 0.;
    } else if (double S_e = (1 - Sn - c.S_wr) / (1 - c.S_wr); PD0 && S_e >= c.se_fast_min) {
      P_k = 0.;
      PkS = 0.;
    } else {
      P_k = c.P_d * pow(S_e, c.e_pk);
      double AAA = pow(S_e, c.e_aaa);
      PkS = AAA * (c.P_d) / (c.lambda * (1 - c.S_wr));
    }
    double F1 = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm)) * (1. - Sn) - roS_w;
    double F2 = c.ro0_n * (1. + (c.beta_n) * (Pw + P_k - c.P_atm)) * Sn - roS_n;
    double F1P = c.ro0_w * (c.beta_w) * (1 - Sn);
    double F2P = c.ro0_n * (c.beta_n) * Sn;
    double F1S = (-1) * (c.ro0_w) * (1 + (c.beta_w) * (Pw - c.P_atm));
    double F2S = c.ro0_n * (1 + (c.beta_n) * (Pw + P_k - c.P_atm + (Sn * PkS)));
    double det = F1P * F2S - F1S * F2P;
    double nPw = Pw - (1 / det) * (F2S * F1 - F1S * F2);
    double nSn = Sn - (1 / det) * (F1P * F2 - F2P * F1);
    Pw = nPw;
    Sn = nSn;
  }
}

// Newton residual at the final iterate, for the diagnostics.
template <bool PD0>
__device__ __forceinline__ double residual2(const Step2Const& c, double roS_w, double roS_n, double Pw,
                                            double Sn) {
  double S_e = (1 - Sn - c.S_wr) / (1 - c.S_wr);
  double P_k = (c.P_d != 0.) ? c.P_d * pow(S_e, c.e_pk) : 0.;
  double rw = c.ro0_w * (1. + (c.beta_w) * (Pw - c.P_atm));
  double rn = c.ro0_n * (1. + (c.beta_n) * (Pw + P_k - c.P_atm));
  double F1 = rw * (1. - Sn) - roS_w;
  double F2 = rn * Sn - roS_n;
  return fmax(fabs(F1) / c.ro0_w, fabs(F2) / c.ro0_n);
}

__device__ __forceinline__ bool in_window(const Step2Const& c, int i, int k) {
  return (i >= c.nx / 2 - c.source) && (i <= c.nx / 2 + c.source) && (k >= c.win_k0) && (k <= c.win_k1);
}

// Border_S + Border_P for every boundary cell whose basic coordinate is the
// interior cell (i, j, k); values from that cell's new state and its
// start-of-step densities (ro_eff_gdy, main.cpp:263-264).
template <bool PLANAR>
__device__ __forceinline__ void write_boundary2(const Step2Const& c, int i, int j, int k, double Pw,
                                                double Sn, double ro_w, double ro_n, double m,
                                                double* __restrict__ Pw_out, double* __restrict__ Sn_out) {
  int xs[3], ys[3], zs[3];
  int nxs = 0, nys = 0, nzs = 0;
  xs[nxs++] = i;
  if (i == 1) xs[nxs++] = 0;
  if (i == c.nx - 2) xs[nxs++] = c.nx - 1;
  ys[nys++] = j;
  if (j == 1) ys[nys++] = 0;
  if (j == c.ny - 2) ys[nys++] = c.ny - 1;
  zs[nzs++] = k;
  if (!PLANAR) {
    if (k == 1) zs[nzs++] = 0;
    if (k == c.nz - 2) zs[nzs++] = c.nz - 1;
  }
  if (nxs == 1 && nys == 1 && nzs == 1) return;
  double ro_g_dy = (ro_n * Sn + ro_w * (1 - Sn)) * (m) * (c.g) * (c.hy);
  for (int a = 0; a < nxs; a++)
    for (int b = 0; b < nys; b++)
      for (int d = 0; d < nzs; d++) {
        if (a == 0 && b == 0 && d == 0) continue;
        int bi = xs[a], bj = ys[b], bk = zs[d];
        long long l = bi + bj * c.sy + bk * c.sz;
        double s = Sn;
        if ((bj == 0) && (c.source > 0) && in_window(c, bi, bk)) s = c.S_n_gr;
        double p;
        if ((bj != 0) && (bj != c.ny - 1)) p = Pw;
        else if (bj == 0) p = c.P_atm + c.P_top;
        else p = Pw + ro_g_dy;
        Sn_out[l] = s;
        Pw_out[l] = p;
      }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One work item: the TX x TY column tile `tile` over z-chunk `zc`.  Called
// by every thread of the CTA (it contains barriers).
template <bool UNIK, bool PD0, bool PLANAR, bool DIAG>
__device__ __forceinline__ void fp64_tile(const Step2Const& c, const double* __restrict__ Pw_in,
                                          const double* __restrict__ Sn_in, double* __restrict__ Pw_out,
                                          double* __restrict__ Sn_out, const double* __restrict__ m,
                                          const double* __restrict__ K, unsigned int* __restrict__ err_flag,
                                          int tile, int zc, Plane2* ring, double* diag_slot) {
  const int tid = threadIdx.x + TX * threadIdx.y;
  const int ti = tile % c.tiles_x, tj = tile / c.tiles_x;
  const int i0 = 1 + ti * TX, j0 = 1 + tj * TY;  // first interior cell of the tile
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const bool active = (i <= c.nx - 2) && (j <= c.ny - 2);
  const int cidx = (threadIdx.y + 1) * PX + (threadIdx.x + 1);

  int kb, ke;  // interior planes [kb, ke) owned by this CTA
  if (PLANAR) {
    kb = 0;
    ke = 1;
  } else {
    kb = 1 + zc * c.zchunk;
    ke = min(kb + c.zchunk, c.nz - 1);
  }

  // Fill the plane window of plane k into ring slot k % 3.
  auto fill = [&](int k) {
    Plane2& P = ring[k % 3];
    for (int q = tid; q < PC; q += NTHREADS) {
      int gi = i0 - 1 + q % PX, gj = j0 - 1 + q / PX;
      if (gi < c.nx && gj < c.ny) {
        long long l = gi + gj * c.sy + (long long)k * c.sz;
        double Pw = Pw_in[l], Sn = Sn_in[l];
        double Kl = UNIK ? c.K0 : K[l];
        double Pn, ro_w, ro_n, Xi_w, Xi_n;
        derive2<PD0>(c, Pw, Sn, Kl, Pn, ro_w, ro_n, Xi_w, Xi_n);
        P.Pw[q] = Pw;
        P.Pn[q] = Pn;
        P.ro_w[q] = ro_w;
        P.ro_n[q] = ro_n;
        P.Xi_w[q] = Xi_w;
        P.Xi_n[q] = Xi_n;
      }
    }
  };

  double acc_w = 0., acc_n = 0., rmax = 0., nonfinite = 0.;

  if (!PLANAR) fill(kb - 1);
  fill(kb);
  for (int k = kb; k < ke; k++) {
    if (!PLANAR) fill(k + 1);
    __syncthreads();
    if (active) {
      const Plane2& C = ring[k % 3];
      const long long l = i + j * c.sy + (long long)k * c.sz;
      const double mc = m[l];
      const double Pw = C.Pw[cidx], Pn = C.Pn[cidx], Sn = Sn_in[l];
      const double rw = C.ro_w[cidx], rn = C.ro_n[cidx];
      const double q_w = 0., q_n = 0.;  // wells_q (two-phase.cpp:187-192)
      const double roS_w = rw * (1. - Sn);
      const double roS_n = rn * Sn;
      double x1, x2, fx_w, fy_w, fz_w, fx_n, fy_n, fz_n;
      if (PLANAR) {
        fz_w = 0.;
        fz_n = 0.;
      } else {
        const Plane2& M = ring[(k + 2) % 3];  // k - 1
        const Plane2& Q = ring[(k + 1) % 3];  // k + 1
        x2 = -1. * ((Q.Pw[cidx] - Pw) / c.hz);
        x1 = -1. * ((Pw - M.Pw[cidx]) / c.hz);
        fz_w = directed(x1, x2, C.Xi_w[cidx], rw, M.Xi_w[cidx], M.ro_w[cidx], Q.Xi_w[cidx], Q.ro_w[cidx], c.hz);
        x2 = -1. * ((Q.Pn[cidx] - Pn) / c.hz);
        x1 = -1. * ((Pn - M.Pn[cidx]) / c.hz);
        fz_n = directed(x1, x2, C.Xi_n[cidx], rn, M.Xi_n[cidx], M.ro_n[cidx], Q.Xi_n[cidx], Q.ro_n[cidx], c.hz);
      }
      {
        const int a = cidx - 1, b = cidx + 1;
        x2 = -1. * ((C.Pw[b] - Pw) / c.hx);
        x1 = -1. * ((Pw - C.Pw[a]) / c.hx);
        fx_w = directed(x1, x2, C.Xi_w[cidx], rw, C.Xi_w[a], C.ro_w[a], C.Xi_w[b], C.ro_w[b], c.hx);
        x2 = -1. * ((C.Pn[b] - Pn) / c.hx);
        x1 = -1. * ((Pn - C.Pn[a]) / c.hx);
        fx_n = directed(x1, x2, C.Xi_n[cidx], rn, C.Xi_n[a], C.ro_n[a], C.Xi_n[b], C.ro_n[b], c.hx);
      }
      {
        const int a = cidx - PX, b = cidx + PX;
        x2 = -1. * ((C.Pw[b] - Pw) / c.hy) + c.g * (rw);
        x1 = -1. * ((Pw - C.Pw[a]) / c.hy) + c.g * (rw);
        fy_w = directed(x1, x2, C.Xi_w[cidx], rw, C.Xi_w[a], C.ro_w[a], C.Xi_w[b], C.ro_w[b], c.hy);
        x2 = -1. * ((C.Pn[b] - Pn) / c.hy) + c.g * (rn);
        x1 = -1. * ((Pn - C.Pn[a]) / c.hy) + c.g * (rn);
        fy_n = directed(x1, x2, C.Xi_n[cidx], rn, C.Xi_n[a], C.ro_n[a], C.Xi_n[b], C.ro_n[b], c.hy);
      }
      const double A1 = roS_w - (c.dt / mc) * (-q_w + fx_w + fy_w + fz_w);
      const double A2 = roS_n - (c.dt / mc) * (-q_n + fx_n + fy_n + fz_n);
      double nPw = Pw, nSn = Sn;
      newton2<PD0>(c, A1, A2, nPw, nSn);
      Pw_out[l] = nPw;
      Sn_out[l] = nSn;
      const bool edge = (i == 1) || (i == c.nx - 2) || (j == 1) || (j == c.ny - 2) ||
                        (!PLANAR && ((k == 1) || (k == c.nz - 2)));
      if (edge) write_boundary2<PLANAR>(c, i, j, k, nPw, nSn, rw, rn, mc, Pw_out, Sn_out);
      const bool finite = isfinite(nPw) && isfinite(nSn);
      if (!finite) atomicOr(err_flag, 1u);
      if (DIAG) {
        double S_e = (1 - nSn - c.S_wr) / (1 - c.S_wr);
        double P_k = (c.P_d != 0.) ? c.P_d * pow(S_e, c.e_pk) : 0.;
        double rw1 = c.ro0_w * (1. + (c.beta_w) * (nPw - c.P_atm));
        double rn1 = c.ro0_n * (1. + (c.beta_n) * (nPw + P_k - c.P_atm));
        acc_w += mc * rw1 * (1. - nSn) * c.vol;
        acc_n += mc * rn1 * nSn * c.vol;
        double r = residual2<PD0>(c, A1, A2, nPw, nSn);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    }
    __syncthreads();
  }

  if (DIAG) {
    // Warp shuffles, then one value per warp through shared memory.
    __shared__ double red[NTHREADS / 32][4];
    const int lane = tid & 31, wid = tid >> 5;
    double s0 = warp_sum(acc_w), s1 = warp_sum(acc_n), r = warp_max(rmax), nf = warp_sum(nonfinite);
    if (lane == 0) {
      red[wid][0] = s0;
      red[wid][1] = s1;
      red[wid][2] = r;
      red[wid][3] = nf;
    }
    __syncthreads();
    if (tid == 0) {
      double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
      for (int w = 0; w < NTHREADS / 32; w++) {
        t0 += red[w][0];
        t1 += red[w][1];
        t2 = fmax(t2, red[w][2]);
        t3 += red[w][3];
      }
      diag_slot[0] = t0;
      diag_slot[1] = t1;
      diag_slot[2] = 0.;
      diag_slot[3] = t2;
      diag_slot[4] = t3;
    }
    __syncthreads();
  }
}

template <bool UNIK, bool PD0, bool PLANAR, bool DIAG>
__global__ void __launch_bounds__(NTHREADS, 4)
    step2_fp64_kernel(const Step2Const c, const double* __restrict__ Pw_in, const double* __restrict__ Sn_in,
                      double* __restrict__ Pw_out, double* __restrict__ Sn_out, const double* __restrict__ m,
                      const double* __restrict__ K, double* __restrict__ diag_partials,
                      unsigned int* __restrict__ err_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Plane2* ring = reinterpret_cast<Plane2*>(smem_raw);
  double* slot = DIAG ? diag_partials + (size_t)DIAG_STRIDE * (blockIdx.x + (size_t)gridDim.x * blockIdx.y) : nullptr;
  fp64_tile<UNIK, PD0, PLANAR, DIAG>(c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, err_flag, blockIdx.x, blockIdx.y, ring,
                                     slot);
}

// Batched persistent kernel: CTAs take (instance, tile, z-chunk) work items
// from a shared counter until the list is exhausted, so instances of uneven
// size share one launch.  All instances have the same flags (K per cell,
// P_d == 0); planar and 3-D instances may be mixed.
template <bool UNIK, bool PD0>
__global__ void __launch_bounds__(NTHREADS, 4)
    step2_fp64_batch_kernel(const Inst64* __restrict__ insts, const int4* __restrict__ items, int nitems, int parity,
                            unsigned int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Plane2* ring = reinterpret_cast<Plane2*>(smem_raw);
  __shared__ int w_sh;
  for (;;) {
    if (threadIdx.x == 0 && threadIdx.y == 0) w_sh = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int w = w_sh;
    __syncthreads();
    if (w >= nitems) break;
    const int4 it = items[w];
    const Inst64& I = insts[it.x];
    const Step2Const& c = I.c;
    const int src = parity, dst = parity ^ 1;
    if (c.nz == 1)
      fp64_tile<UNIK, PD0, true, false>(c, I.Pw[src], I.Sn[src], I.Pw[dst], I.Sn[dst], I.m, I.K, I.err, it.y, it.z,
                                        ring, nullptr);
    else
      fp64_tile<UNIK, PD0, false, false>(c, I.Pw[src], I.Sn[src], I.Pw[dst], I.Sn[dst], I.m, I.K, I.err, it.y, it.z,
                                         ring, nullptr);
  }
}

// Sums the per-block partials in block order (deterministic) into out[5].
__global__ void diag_finalize_kernel(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  __shared__ double red[4][DIAG_STRIDE];
  // Launched as a programmatic dependent of the step's last kernel: wait for
  // it (a no-op for an ordinary launch).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  diag_reduce_block<4>(partials, nblocks, out, red);  // 128 threads
}

template <bool UNIK, bool PD0, bool PLANAR, bool DIAG>
cudaError_t launch_t(const Step2Const& c, const double* Pw_in, const double* Sn_in, double* Pw_out,
                     double* Sn_out, const double* m, const double* K, double* diag, unsigned int* err,
                     cudaStream_t s) {
  auto kern = step2_fp64_kernel<UNIK, PD0, PLANAR, DIAG>;
  static bool attr_set = false;  // per instantiation, per process
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem2);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  dim3 grid(c.tiles_x * c.tiles_y, c.nzchunks);
  kern<<<grid, dim3(TX, TY), kSmem2, s>>>(c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, diag, err);
  return cudaGetLastError();
}

template <bool UNIK, bool PD0, bool PLANAR>
cudaError_t launch_d(bool diag_on, const Step2Const& c, const double* a, const double* b, double* d,
                     double* e, const double* m, const double* K, double* diag, unsigned int* err,
                     cudaStream_t s) {
  return diag_on ? launch_t<UNIK, PD0, PLANAR, true>(c, a, b, d, e, m, K, diag, err, s)
                 : launch_t<UNIK, PD0, PLANAR, false>(c, a, b, d, e, m, K, diag, err, s);
}
template <bool UNIK, bool PD0>
cudaError_t launch_p(bool planar, bool diag_on, const Step2Const& c, const double* a, const double* b,
                     double* d, double* e, const double* m, const double* K, double* diag,
                     unsigned int* err, cudaStream_t s) {
  return planar ? launch_d<UNIK, PD0, true>(diag_on, c, a, b, d, e, m, K, diag, err, s)
                : launch_d<UNIK, PD0, false>(diag_on, c, a, b, d, e, m, K, diag, err, s);
}

// ---------------------------------------------------------------------------
// Derived fields of a start-of-step state (not on the hot path): one thread
// per cell, direct loads, the same device functions as the fused step.
template <bool PD0>
__device__ void derive_at(const Step2Const& c, const double* Pw, const double* Sn, const double* K,
                          bool percell, long long l, double& Pn, double& rw, double& rn, double& Xw, double& Xn) {
  derive2<PD0>(c, Pw[l], Sn[l], percell ? K[l] : c.K0, Pn, rw, rn, Xw, Xn);
}

template <bool PD0>
__global__ void derived2_kernel(const Step2Const c, int field, const double* __restrict__ Pw,
                                const double* __restrict__ Sn, const double* __restrict__ m,
                                const double* __restrict__ K, bool percell, double* __restrict__ out) {
  long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= c.ncell) return;
  const int i = (int)(l % c.nx), j = (int)((l / c.nx) % c.ny), k = (int)(l / c.sz);
  double Pn, rw, rn, Xw, Xn;
  derive_at<PD0>(c, Pw, Sn, K, percell, l, Pn, rw, rn, Xw, Xn);
  switch (field) {
    case CAPAZ_FIELD_S_W: out[l] = 1. - Sn[l]; return;
    case CAPAZ_FIELD_P_N: out[l] = Pn; return;
    case CAPAZ_FIELD_RO_W: out[l] = rw; return;
    case CAPAZ_FIELD_RO_N: out[l] = rn; return;
    case CAPAZ_FIELD_XI_W: out[l] = Xw; return;
    case CAPAZ_FIELD_XI_N: out[l] = Xn; return;
    default: break;
  }
  // Velocities (cpu.cpp:346-477): central differences, one-sided at the ends.
  if (field >= CAPAZ_FIELD_UX_W && field <= CAPAZ_FIELD_UZ_N) {
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
    double Pc, Pm = 0., Pp = 0., Xc, ro;
    double t0, t1, t2, t3;
    if (wph) {
      Pc = Pw[l];
      Xc = Xw;
      ro = rw;
      if (idx > 0) Pm = Pw[l - s];
      if (idx < N - 1) Pp = Pw[l + s];
    } else {
      Pc = Pn;
      Xc = Xn;
      ro = rn;
      if (idx > 0) derive_at<PD0>(c, Pw, Sn, K, percell, l - s, Pm, t0, t1, t2, t3);
      if (idx < N - 1) derive_at<PD0>(c, Pw, Sn, K, percell, l + s, Pp, t0, t1, t2, t3);
    }
    double d;
    if (idx == 0) d = (Pp - Pc) / h;
    else if (idx == N - 1) d = (Pc - Pm) / h;
    else d = (Pp - Pm) / (2. * h);
    if (axis == 1) out[l] = Xc * (d - ro * (c.g));
    else out[l] = Xc * d;
    return;
  }
  // roS (after the flux update) and roS_old: interior cells only; other
  // cells are not written by the reference and read as 0 here.
  const bool inter = (i != 0) && (i != c.nx - 1) && (j != 0) && (j != c.ny - 1) &&
                     (((k != 0) && (k != c.nz - 1)) || (c.nz < 2));
  if (!inter) {
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
  const bool wph = field == CAPAZ_FIELD_ROS_W;
  const double Pc = wph ? Pw[l] : Pn, Xc = wph ? Xw : Xn, rc = wph ? rw : rn;
  double f[3] = {0., 0., 0.};
  for (int axis = 0; axis < 3; axis++) {
    if (axis == 2 && c.nz < 2) continue;
    const long long s = axis == 0 ? 1 : axis == 1 ? c.sy : c.sz;
    const double h = axis == 0 ? c.hx : axis == 1 ? c.hy : c.hz;
    double Pm, rm_w, rm_n, Xm_w, Xm_n, Pp, rp_w, rp_n, Xp_w, Xp_n;
    derive_at<PD0>(c, Pw, Sn, K, percell, l - s, Pm, rm_w, rm_n, Xm_w, Xm_n);
    derive_at<PD0>(c, Pw, Sn, K, percell, l + s, Pp, rp_w, rp_n, Xp_w, Xp_n);
    if (wph) {
      Pm = Pw[l - s];
      Pp = Pw[l + s];
    }
    double x2 = -1. * ((Pp - Pc) / h), x1 = -1. * ((Pc - Pm) / h);
    if (axis == 1) {
      x2 = x2 + c.g * (rc);
      x1 = x1 + c.g * (rc);
    }
    f[axis] = wph ? directed(x1, x2, Xc, rc, Xm_w, rm_w, Xp_w, rp_w, h)
                  : directed(x1, x2, Xc, rc, Xm_n, rm_n, Xp_n, rp_n, h);
  }
  const double roS = wph ? rw * (1. - S) : rn * S;
  out[l] = roS - (c.dt / m[l]) * (-0. + f[0] + f[1] + f[2]);
}

}  // namespace

int step2_grid_blocks(const Step2Const& c) { return c.tiles_x * c.tiles_y * c.nzchunks; }

cudaError_t launch_step2_fp64(const Step2Const& c, const double* Pw_in, const double* Sn_in, double* Pw_out,
                              double* Sn_out, const double* m, const double* K, bool percell_k,
                              double* diag_partials, unsigned int* err_flag, cudaStream_t s, int* nlaunch) {
  const bool planar = c.nz == 1;
  const bool pd0 = (c.P_d == 0.) && (c.se_fast_min > 0.);
  const bool diag_on = diag_partials != nullptr;
  cudaError_t e;
  if (!percell_k)
    e = pd0 ? launch_p<true, true>(planar, diag_on, c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, diag_partials, err_flag, s)
            : launch_p<true, false>(planar, diag_on, c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, diag_partials, err_flag, s);
  else
    e = pd0 ? launch_p<false, true>(planar, diag_on, c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, diag_partials, err_flag, s)
            : launch_p<false, false>(planar, diag_on, c, Pw_in, Sn_in, Pw_out, Sn_out, m, K, diag_partials, err_flag, s);
  if (nlaunch) *nlaunch += 1;
  return e;
}

cudaError_t launch_step2_fp64_batch(const Inst64* insts, const int4* items, int nitems, int parity, bool unik, bool pd0,
                                    unsigned int* counter, int grid, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
#define CAPAZ_BATCH64(U, P)                                                                               \
  do {                                                                                                    \
    auto kern = step2_fp64_batch_kernel<U, P>;                                                            \
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem2);            \
    if (e != cudaSuccess) return e;                                                                       \
    kern<<<grid, dim3(TX, TY), kSmem2, s>>>(insts, items, nitems, parity, counter);                       \
  } while (0)
  if (unik) {
    if (pd0) CAPAZ_BATCH64(true, true);
    else CAPAZ_BATCH64(true, false);
  } else {
    if (pd0) CAPAZ_BATCH64(false, true);
    else CAPAZ_BATCH64(false, false);
  }
#undef CAPAZ_BATCH64
  return cudaGetLastError();
}

int step2_fp64_batch_grid(int device) {
  int sms = 148, per = 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp64_batch_kernel<false, true>, NTHREADS, kSmem2);
  if (per < 1) per = 1;
  return sms * per;
}

// One block launched with programmatic stream serialisation: its launch
// overlaps the tail of the kernel before it, which it waits for on entry.
template <typename... Params, typename... Args>
static cudaError_t launch_single_dependent(void (*kernel)(Params...), int threads, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

cudaError_t launch_diag_finalize(const double* partials, int nblocks, double* out, cudaStream_t s) {
  return launch_single_dependent(diag_finalize_kernel, 128, s, partials, nblocks, out);
}

// Copies the reduced diagnostics into mapped pinned host memory: the kernel's
// stores reach the host without a copy-engine transfer, and the event recorded
// after it tells the host when they have landed.
__global__ void diag_publish_kernel(const double* __restrict__ d, double* __restrict__ host_mapped) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (threadIdx.x < DIAG_STRIDE) host_mapped[threadIdx.x] = d[threadIdx.x];
  __threadfence_system();
}

cudaError_t launch_diag_publish(const double* d, double* host_mapped, cudaStream_t s) {
  return launch_single_dependent(diag_publish_kernel, 32, s, d, host_mapped);
}

cudaError_t launch_derived2_fp64(const Step2Const& c, int field, const double* Pw, const double* Sn,
                                 const double* m, const double* K, bool percell_k, double* out, cudaStream_t s) {
  const long long n = c.ncell;
  const int bs = 256;
  const unsigned nb = (unsigned)((n + bs - 1) / bs);
  const bool pd0 = (c.P_d == 0.) && (c.se_fast_min > 0.);
  if (pd0) derived2_kernel<true><<<nb, bs, 0, s>>>(c, field, Pw, Sn, m, K, percell_k, out);
  else derived2_kernel<false><<<nb, bs, 0, s>>>(c, field, Pw, Sn, m, K, percell_k, out);
  return cudaGetLastError();
}

}  // namespace capaz
