// Fused two-phase time step, precision form (CAPAZ_FORM_FP32C).
//
// The same step as step2_fp64.cu (flux stencil of cpu.cpp:619-731, Newton of
// two-phase.cpp:25-56, boundary rules of two-phase.cpp:59-111) with:
//   - storage: FP32 P_w, S_n, m, K (24 bytes of HBM traffic per cell-step
//     with per-cell K).  P_w and S_n are stored as FP32 deviations from a
//     reference state, P_w - P_ref(j) and S_n - S_ref, where P_ref(j) is a
//     per-row pressure profile and S_ref a constant fixed when the state is
//     loaded.  With compressibility 1e-9 1/Pa the stable time step is so short
//     that S changes by 1e-9..1e-8 per step, below half an FP32 ulp of S
//     itself (3e-8 at 0.85): stored as plain FP32 those increments would be
//     rounded away every step.  The deviations keep them.
//   - stencil: FP32 arithmetic; the face terms of the flux divergence are
//     summed with compensation (Neumaier's variant of Kahan summation), so
//     the in/out cancellation of nearly balanced faces keeps FP32 accuracy.
//   - Newton: FP64, in delta form on (dP, dS) about the stored state with the
//     conserved target rho*S + d(rho S), d(rho S) = -dt/m div F, so rho*S
//     never round-trips through FP32; two iterations (the system is bilinear
//     in the unknowns without capillary pressure and starts within one step's
//     change of the solution).
//   - diagnostics (mass balance, Newton residual): FP64.
// Tiling: TX x TY columns per CTA marching a z-chunk; each thread keeps its
// own column's k-1 / k / k+1 values in registers, and a 3-slot ring of plane
// windows (one-cell halo) in shared memory serves the x/y neighbours with
// one barrier per plane.
#include <math.h>

#include "capaz_internal.h"

namespace capaz {
namespace {

struct PlaneF {
  float p[PC];   // pressure deviation, water phase
  float pn[PC];  // pressure deviation, NAPL phase (p + P_k)
  float Mw[PC];  // -Xi_w*rho_w = K k_w rho_w / mu_w >= 0
  float Mn[PC];
};

__device__ __forceinline__ float ipowf(float x, int n) {
  float r = 1.f, b = x;
  while (n > 0) {
    if (n & 1) r *= b;
    b *= b;
    n >>= 1;
  }
  return r;
}

struct Cell {
  float p, pn, s, Mw, Mn, rho_w, rho_n;
};

// ro_P_Xi in FP32 (two-phase.cpp:8-17; cpu.cpp:164-165) for one cell.
template <bool PD0, bool INTPOW>
__device__ __forceinline__ Cell derive32(const Step2FConst& c, float p, float s, float K, float prel) {
  Cell o;
  const float S = c.S_ref_f + s;
  const float S_e = (c.one_m_swr_f - S) * c.inv_one_m_swr_f;
  float k_w, k_n;
  if (INTPOW) {
    k_w = ipowf(S_e, c.n_kw);
    k_n = (1.f - S_e) * (1.f - S_e) * (1.f - ipowf(S_e, c.n_kn));
  } else {
    k_w = powf(S_e, c.e_kw_f);
    k_n = (1.f - S_e) * (1.f - S_e) * (1.f - powf(S_e, c.e_kn_f));
  }
  float pk = 0.f;
  if (!PD0) pk = c.P_d_f * powf(S_e, c.e_pk_f);
  o.p = p;
  o.s = s;
  o.pn = p + pk;
  o.rho_w = c.ro0_w_f * (1.f + c.beta_w_f * (prel + p));
  o.rho_n = c.ro0_n_f * (1.f + c.beta_n_f * (prel + p + pk));
  o.Mw = K * k_w * c.inv_mu_w_f * o.rho_w;
  o.Mn = K * k_n * c.inv_mu_n_f * o.rho_n;
  return o;
}

// Neumaier-compensated accumulation.
struct CSum {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
};

// Upwind face terms of one axis (cpu.cpp:236-264 with M = -Xi*rho):
//   [max(x2,0) + max(-x1,0)] M_c - max(x1,0) M_minus + min(x2,0) M_plus, / h.
__device__ __forceinline__ void axis_terms(CSum& acc, float x1, float x2, float Mc, float Mm, float Mp, float inv_h) {
  acc.add((fmaxf(x2, 0.f) + fmaxf(-x1, 0.f)) * Mc * inv_h);
  acc.add(-fmaxf(x1, 0.f) * Mm * inv_h);
  acc.add(fminf(x2, 0.f) * Mp * inv_h);
}

__device__ __forceinline__ bool in_window(const Step2FConst& c, int i, int k) {
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

// One work item: the TX x TY column tile `tile` of the grid over z-chunk
// `zc`.  Called by every thread of the CTA (it contains barriers).
template <bool UNIK, bool PD0, bool INTPOW, bool PLANAR, bool DIAG>
__device__ __forceinline__ void fp32c_tile(const Step2FConst& c, const Step2FArgs& A, int tile, int zc,
                                           PlaneF* ring, double* diag_slot) {
  const float* __restrict__ p_in = A.p_in;
  const float* __restrict__ s_in = A.s_in;
  float* __restrict__ p_out = A.p_out;
  float* __restrict__ s_out = A.s_out;
  const float* __restrict__ m = A.m;
  const float* __restrict__ K = A.K;
  const double* __restrict__ Pref = A.Pref;
  const float* __restrict__ PrelF = A.PrelF;
  const float* __restrict__ dPrefF = A.dPrefF;
  unsigned int* __restrict__ err_flag = A.err;
  const int tid = threadIdx.x + TX * threadIdx.y;
  const int ti = tile % c.tiles_x, tj = tile / c.tiles_x;
  const int i0 = 1 + ti * TX, j0 = 1 + tj * TY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const bool active = (i <= c.nx - 2) && (j <= c.ny - 2);
  const int cidx = (threadIdx.y + 1) * PX + (threadIdx.x + 1);

  int kb, ke;
  if (PLANAR) {
    kb = 0;
    ke = 1;
  } else {
    kb = 1 + zc * c.zchunk;
    ke = min(kb + c.zchunk, c.nz - 1);
  }

  // Fill the plane window of plane k (halo and own cell) into ring[k % 3];
  // returns the own cell's values.
  auto fill = [&](int k) -> Cell {
    PlaneF& P = ring[k % 3];
    Cell own;
    own.p = own.pn = own.s = own.Mw = own.Mn = own.rho_w = own.rho_n = 0.f;
    for (int q = tid; q < PC; q += NTHREADS) {
      // q < NTHREADS: own cell of thread q (mapped to its window slot);
      // q >= NTHREADS: one of the halo cells.
      int slot;
      if (q < NTHREADS) {
        slot = (q / TX + 1) * PX + (q % TX + 1);
      } else {
        int h = q - NTHREADS;  // 0 .. 2*PX + 2*TY - 1
        if (h < PX) slot = h;                                   // top row
        else if (h < 2 * PX) slot = (PY - 1) * PX + (h - PX);   // bottom row
        else if (h < 2 * PX + TY) slot = (h - 2 * PX + 1) * PX; // left column
        else slot = (h - 2 * PX - TY + 1) * PX + (PX - 1);      // right column
      }
      const int gi = i0 - 1 + slot % PX, gj = j0 - 1 + slot / PX;
      if (gi < c.nx && gj < c.ny) {
        const long long l = gi + gj * c.sy + (long long)k * c.sz;
        const float Kl = UNIK ? c.K0_f : K[l];
        Cell v = derive32<PD0, INTPOW>(c, p_in[l], s_in[l], Kl, PrelF[gj]);
        P.p[slot] = v.p;
        P.pn[slot] = v.pn;
        P.Mw[slot] = v.Mw;
        P.Mn[slot] = v.Mn;
        if (q < NTHREADS) own = v;
      }
    }
    return own;
  };

  double acc_w = 0., acc_n = 0., rmax = 0., nonfinite = 0.;
  Cell cm, cc, cp;  // own column at k-1, k, k+1
  if (!PLANAR) cm = fill(kb - 1);
  cc = fill(kb);
  for (int k = kb; k < ke; k++) {
    if (!PLANAR) cp = fill(k + 1);
    __syncthreads();
    if (active) {
      const PlaneF& C = ring[k % 3];
      const long long l = i + j * c.sy + (long long)k * c.sz;
      const float mc = m[l];
      const float s0 = cc.s;
      const float gw = c.g_f * cc.rho_w, gn = c.g_f * cc.rho_n;
      CSum dw, dn;
      {  // x
        const int a = cidx - 1, b = cidx + 1;
        axis_terms(dw, -(cc.p - C.p[a]) * c.inv_hx_f, -(C.p[b] - cc.p) * c.inv_hx_f, cc.Mw, C.Mw[a], C.Mw[b], c.inv_hx_f);
        axis_terms(dn, -(cc.pn - C.pn[a]) * c.inv_hx_f, -(C.pn[b] - cc.pn) * c.inv_hx_f, cc.Mn, C.Mn[a], C.Mn[b], c.inv_hx_f);
      }
      {  // y (vertical): P(j+1) - P(j) = dPref(j) + p(j+1) - p(j)
        const int a = cidx - PX, b = cidx + PX;
        const float dup = dPrefF[j], ddn = dPrefF[j - 1];
        const float x2w = -((dup + (C.p[b] - cc.p)) * c.inv_hy_f) + gw;
        const float x1w = -((ddn + (cc.p - C.p[a])) * c.inv_hy_f) + gw;
        axis_terms(dw, x1w, x2w, cc.Mw, C.Mw[a], C.Mw[b], c.inv_hy_f);
        const float x2n = -((dup + (C.pn[b] - cc.pn)) * c.inv_hy_f) + gn;
        const float x1n = -((ddn + (cc.pn - C.pn[a])) * c.inv_hy_f) + gn;
        axis_terms(dn, x1n, x2n, cc.Mn, C.Mn[a], C.Mn[b], c.inv_hy_f);
      }
      if (!PLANAR) {  // z
        axis_terms(dw, -(cc.p - cm.p) * c.inv_hz_f, -(cp.p - cc.p) * c.inv_hz_f, cc.Mw, cm.Mw, cp.Mw, c.inv_hz_f);
        axis_terms(dn, -(cc.pn - cm.pn) * c.inv_hz_f, -(cp.pn - cc.pn) * c.inv_hz_f, cc.Mn, cm.Mn, cp.Mn, c.inv_hz_f);
      }
      // Conserved increments d(rho S) = -dt/m * div F, in FP64.
      const double dtm = c.dt / (double)mc;
      const double Aw = -dtm * ((double)dw.s + (double)dw.c);
      const double An = -dtm * ((double)dn.s + (double)dn.c);

      // FP64 delta-form Newton about the stored state (two-phase.cpp:25-56).
      const double S = c.S_ref + (double)s0;
      const double prel = (Pref[j] - c.P_atm) + (double)cc.p;
      double Pk0 = 0.;
      if (!PD0) Pk0 = c.P_d * pow((1. - S - c.S_wr) / (1. - c.S_wr), c.e_pk);
      const double rw = c.ro0_w * (1. + c.beta_w * prel);
      const double rn = c.ro0_n * (1. + c.beta_n * (prel + Pk0));
      const double a = c.ro0_w * c.beta_w, b = c.ro0_n * c.beta_n;
      double dP = 0., dS = 0., F1 = 0., F2 = 0.;
      for (int it = 0; it <= c.iters; it++) {
        double Pk1 = 0., dPk = 0.;
        if (!PD0) {
          const double Se1 = (1. - (S + dS) - c.S_wr) / (1. - c.S_wr);
          Pk1 = c.P_d * pow(Se1, c.e_pk);
          dPk = -Pk1 * c.e_pk / (Se1 * (1. - c.S_wr));  // dP_k/dS
        }
        F1 = -rw * dS + a * dP * (1. - S - dS) - Aw;
        F2 = rn * dS + b * (dP + (Pk1 - Pk0)) * (S + dS) - An;
        if (it == c.iters) break;  // last pass only evaluates the residual
        const double J11 = a * (1. - S - dS), J12 = -rw - a * dP;
        const double J21 = b * (S + dS), J22 = rn + b * (dP + (Pk1 - Pk0)) + b * dPk * (S + dS);
        const double det = J11 * J22 - J12 * J21;
        const double inv = 1. / det;
        dP -= (J22 * F1 - J12 * F2) * inv;
        dS -= (J11 * F2 - J21 * F1) * inv;
      }
      const float p1 = (float)((double)cc.p + dP);
      const float s1 = (float)((double)s0 + dS);
      p_out[l] = p1;
      s_out[l] = s1;
      const bool finite = isfinite(p1) && isfinite(s1);
      if (!finite) atomicOr(err_flag, 1u);

      // Boundary cells whose basic coordinate is (i, j, k) (cpu.cpp:107-141).
      const bool edge = (i == 1) || (i == c.nx - 2) || (j == 1) || (j == c.ny - 2) ||
                        (!PLANAR && ((k == 1) || (k == c.nz - 2)));
      if (edge) {
        const double Snew = c.S_ref + (double)s1;
        const double Pnew = Pref[j] + (double)p1;
        const double ro_g_dy = (rn * Snew + rw * (1 - Snew)) * (double)mc * c.g * c.hy;
        int xs[3], ys[3], zs[3], nxs = 0, nys = 0, nzs = 0;
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
        for (int qa = 0; qa < nxs; qa++)
          for (int qb = 0; qb < nys; qb++)
            for (int qd = 0; qd < nzs; qd++) {
              if (qa == 0 && qb == 0 && qd == 0) continue;
              const int bi = xs[qa], bj = ys[qb], bk = zs[qd];
              const long long lb = bi + bj * c.sy + (long long)bk * c.sz;
              float sb = s1;
              if ((bj == 0) && (c.source > 0) && in_window(c, bi, bk)) sb = (float)(c.S_n_gr - c.S_ref);
              float pb;
              if ((bj != 0) && (bj != c.ny - 1)) pb = p1;
              else if (bj == 0) pb = (float)((c.P_atm + c.P_top) - Pref[0]);
              else pb = (float)(Pnew + ro_g_dy - Pref[c.ny - 1]);
              s_out[lb] = sb;
              p_out[lb] = pb;
            }
      }
      if (DIAG) {
        const double S1 = c.S_ref + (double)s1;
        const double P1rel = (Pref[j] - c.P_atm) + (double)p1;
        const double rw1 = c.ro0_w * (1. + c.beta_w * P1rel);
        double Pk1 = 0.;
        if (!PD0) Pk1 = c.P_d * pow((1. - S1 - c.S_wr) / (1. - c.S_wr), c.e_pk);
        const double rn1 = c.ro0_n * (1. + c.beta_n * (P1rel + Pk1));
        acc_w += (double)mc * rw1 * (1. - S1) * c.vol;
        acc_n += (double)mc * rn1 * S1 * c.vol;
        const double r = fmax(fabs(F1) / c.ro0_w, fabs(F2) / c.ro0_n);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    }
    cm = cc;
    cc = cp;
    // The next fill writes ring[(k+2) % 3], last read in iteration k-1,
    // which every thread finished before this iteration's barrier.
  }
  if (DIAG) {
    __syncthreads();
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
  }
  // The caller may start another work item on this CTA: every thread must be
  // done with the plane ring first.
  __syncthreads();
}

template <bool UNIK, bool PD0, bool INTPOW, bool PLANAR, bool DIAG>
__global__ void __launch_bounds__(NTHREADS) step2_fp32c_kernel(const Step2FConst c, const Step2FArgs a) {
  __shared__ PlaneF ring[3];
  double* slot = DIAG ? a.diag + (size_t)DIAG_STRIDE * (blockIdx.x + (size_t)gridDim.x * blockIdx.y) : nullptr;
  fp32c_tile<UNIK, PD0, INTPOW, PLANAR, DIAG>(c, a, blockIdx.x, blockIdx.y, ring, slot);
}

// Batched persistent kernel (see step2_fp64_batch_kernel).
template <bool UNIK, bool PD0, bool INTPOW>
__global__ void __launch_bounds__(NTHREADS)
    step2_fp32c_batch_kernel(const InstF* __restrict__ insts, const int4* __restrict__ items, int nitems, int parity,
                             unsigned int* __restrict__ counter) {
  __shared__ PlaneF ring[3];
  __shared__ int w_sh;
  for (;;) {
    if (threadIdx.x == 0 && threadIdx.y == 0) w_sh = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int w = w_sh;
    __syncthreads();
    if (w >= nitems) break;
    const int4 it = items[w];
    const InstF& I = insts[it.x];
    if (I.c.nz == 1)
      fp32c_tile<UNIK, PD0, INTPOW, true, false>(I.c, I.a[parity], it.y, it.z, ring, nullptr);
    else
      fp32c_tile<UNIK, PD0, INTPOW, false, false>(I.c, I.a[parity], it.y, it.z, ring, nullptr);
  }
}

template <bool UNIK, bool PD0, bool INTPOW, bool PLANAR, bool DIAG>
cudaError_t launch_t(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s) {
  dim3 grid(c.tiles_x * c.tiles_y, c.nzchunks);
  step2_fp32c_kernel<UNIK, PD0, INTPOW, PLANAR, DIAG><<<grid, dim3(TX, TY), 0, s>>>(c, a);
  return cudaGetLastError();
}
template <bool UNIK, bool PD0, bool INTPOW, bool PLANAR>
cudaError_t launch_d(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s) {
  return a.diag ? launch_t<UNIK, PD0, INTPOW, PLANAR, true>(c, a, s) : launch_t<UNIK, PD0, INTPOW, PLANAR, false>(c, a, s);
}
template <bool UNIK, bool PD0, bool INTPOW>
cudaError_t launch_p(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s) {
  return c.nz == 1 ? launch_d<UNIK, PD0, INTPOW, true>(c, a, s) : launch_d<UNIK, PD0, INTPOW, false>(c, a, s);
}
template <bool UNIK, bool PD0>
cudaError_t launch_i(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s) {
  return c.intpow ? launch_p<UNIK, PD0, true>(c, a, s) : launch_p<UNIK, PD0, false>(c, a, s);
}

}  // namespace

cudaError_t launch_step2_fp32c_batch(const InstF* insts, const int4* items, int nitems, int parity, bool unik,
                                     bool pd0, bool intpow, unsigned int* counter, int grid, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
#define CAPAZ_BATCH32(U, P, I) step2_fp32c_batch_kernel<U, P, I><<<grid, dim3(TX, TY), 0, s>>>(insts, items, nitems, parity, counter)
  if (unik) {
    if (pd0) { if (intpow) CAPAZ_BATCH32(true, true, true); else CAPAZ_BATCH32(true, true, false); }
    else { if (intpow) CAPAZ_BATCH32(true, false, true); else CAPAZ_BATCH32(true, false, false); }
  } else {
    if (pd0) { if (intpow) CAPAZ_BATCH32(false, true, true); else CAPAZ_BATCH32(false, true, false); }
    else { if (intpow) CAPAZ_BATCH32(false, false, true); else CAPAZ_BATCH32(false, false, false); }
  }
#undef CAPAZ_BATCH32
  return cudaGetLastError();
}

int step2_fp32c_batch_grid(int device) {
  int sms = 148, per = 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_batch_kernel<false, true, true>, NTHREADS, 0);
  if (per < 1) per = 1;
  return sms * per;
}

cudaError_t launch_step2_fp32c(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s) {
  const bool unik = a.K == nullptr;
  const bool pd0 = c.P_d == 0.;
  if (unik) return pd0 ? launch_i<true, true>(c, a, s) : launch_i<true, false>(c, a, s);
  return pd0 ? launch_i<false, true>(c, a, s) : launch_i<false, false>(c, a, s);
}

// ---------------------------------------------------------------------------
// Decoding of the stored deviations to FP64 fields (not on the hot path).
__global__ void decode2_kernel(const float* __restrict__ p, const float* __restrict__ s,
                               const double* __restrict__ Pref, double S_ref, int nx, int ny, long long n,
                               double* __restrict__ P, double* __restrict__ S) {
  long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int j = (int)((l / nx) % ny);
  P[l] = Pref[j] + (double)p[l];
  S[l] = S_ref + (double)s[l];
}

cudaError_t launch_decode2(const float* p, const float* s, const double* Pref, double S_ref, int nx, int ny,
                           long long n, double* P, double* S, cudaStream_t st) {
  const int bs = 256;
  decode2_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, st>>>(p, s, Pref, S_ref, nx, ny, n, P, S);
  return cudaGetLastError();
}

__global__ void widen_kernel(const float* __restrict__ a, long long n, double* __restrict__ out) {
  long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l < n) out[l] = (double)a[l];
}

cudaError_t launch_widen(const float* a, long long n, double* out, cudaStream_t st) {
  const int bs = 256;
  widen_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, st>>>(a, n, out);
  return cudaGetLastError();
}

}  // namespace capaz
