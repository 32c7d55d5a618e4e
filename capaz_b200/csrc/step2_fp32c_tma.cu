// Two-phase precision-form step with TMA-staged z-planes (sm_100a).
//
// Same arithmetic model as step2_fp32c.cu (FP32 deviation storage, FP32
// stencil with Kahan-compensated divergence, FP64 delta-form Newton), laid out
// for Blackwell's memory system:
//   - persistent CTAs take (instance, tile, z-chunk) work items from a global
//     counter, so one launch covers one grid or a whole ensemble of uneven
//     grids without tail waves;
//   - one elected thread streams the raw planes (p, s, K, m) of the tile's
//     window (a 36 x 10 box at x = 32*ti, a 128-byte-aligned start) into a
//     4-stage shared-memory ring with cp.async.bulk.tensor (TMA, 3-D tensor
//     maps, no multicast) completing on mbarriers, 4 planes ahead of use;
//   - every thread derives its own cell (and the halo threads one more cell)
//     from the staged plane into a 4-slot ring of derived planes, keeps its
//     own column's k-1/k/k+1 values in registers, and computes the upwind
//     fluxes of the centre plane: one barrier per plane.
// Waits on mbarriers are bounded; a wait that runs out sets bit 2 of the
// error flag and the CTA carries on with whatever the stage holds, so the
// kernel always finishes and the host reports the error.
#include <cuda.h>
#include <math.h>
#include <stdint.h>

#include "capaz_internal.h"

namespace capaz {
namespace {

constexpr int BXW = 36;   // TMA box width (floats): 144 bytes, a multiple of 16
constexpr int BYW = 10;   // TMA box height: TY + 2
constexpr int NST = 4;    // raw-plane stages in flight
constexpr int RAWN = 384; // floats reserved per array per stage (1536 B, 128-B multiple)
constexpr unsigned long long WAIT_LIMIT = 1ull << 22;  // try_wait polls before giving up

struct alignas(128) RawStage {
  float p[RAWN], s[RAWN], K[RAWN], m[RAWN];
};
struct DerPlane {
  float p[PC], pn[PC], Mw[PC], Mn[PC];
};

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

struct OwnCell {
  float p, pn, s, m, Mw, Mn, rho_w, rho_n;
};

// ro_P_Xi in FP32 for one cell (two-phase.cpp:8-17).  LAM2: lambda == 2,
// k_w = S_e^4, k_n = (1-S_e)^2 (1-S_e^2) exactly as the exponents say.
template <bool PD0, bool LAM2>
__device__ __forceinline__ OwnCell derive(const Step2FConst& c, float p, float s, float K, float m, float prel) {
  OwnCell o;
  const float S = c.S_ref_f + s;
  const float S_e = (c.one_m_swr_f - S) * c.inv_one_m_swr_f;
  float k_w, k_n;
  if (LAM2) {
    const float e2 = S_e * S_e;
    k_w = e2 * e2;
    k_n = (1.f - S_e) * (1.f - S_e) * (1.f - e2);
  } else {
    k_w = powf(S_e, c.e_kw_f);
    k_n = (1.f - S_e) * (1.f - S_e) * (1.f - powf(S_e, c.e_kn_f));
  }
  float pk = 0.f;
  if (!PD0) pk = c.P_d_f * powf(S_e, c.e_pk_f);
  o.p = p;
  o.pn = p + pk;
  o.s = s;
  o.m = m;
  o.rho_w = c.ro0_w_f * (1.f + c.beta_w_f * (prel + p));
  o.rho_n = c.ro0_n_f * (1.f + c.beta_n_f * (prel + p + pk));
  o.Mw = K * k_w * c.inv_mu_w_f * o.rho_w;
  o.Mn = K * k_n * c.inv_mu_n_f * o.rho_n;
  return o;
}

// Kahan summation (4 flops per term).
struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Upwind flux difference of one axis (cpu.cpp:236-264 in select form):
//   outflow through the + face  x2 * (x2 > 0 ? M_c : M_+),
//   inflow through the - face   x1 * (x1 > 0 ? M_- : M_c).
__device__ __forceinline__ void axis(Kahan& acc, float x1, float x2, float Mc, float Mm, float Mp, float inv_h) {
  acc.add(x2 * (x2 > 0.f ? Mc : Mp) * inv_h);
  acc.add(-(x1 * (x1 > 0.f ? Mm : Mc)) * inv_h);
}

__device__ __forceinline__ bool in_window(const Step2FConst& c, int i, int k) {
  return (i >= c.nx / 2 - c.source) && (i <= c.nx / 2 + c.source) && (k >= c.nz / 2 - c.source) &&
         (k <= c.nz / 2 + c.source);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool UNIK, bool PD0, bool LAM2, bool DIAG>
__global__ void __launch_bounds__(NTHREADS, 3)
    step2_fp32c_tma_kernel(const InstT* __restrict__ insts, const int4* __restrict__ items, int nitems, int parity,
                           unsigned int* __restrict__ counter, double* __restrict__ diag_partials) {
  __shared__ RawStage raw[NST];
  __shared__ DerPlane der[4];
  __shared__ __align__(8) uint64_t bar[NST];
  __shared__ int w_sh;
  __shared__ float rowPrelF[BYW], rowDPrefF[BYW];
  __shared__ double rowPrelD[BYW], rowPrefD[BYW];

  const int tid = threadIdx.x + TX * threadIdx.y;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (tid == 0) {
    for (int q = 0; q < NST; q++) mbar_init(&bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;  // bit q: parity of the next completion of stage q

  // Window slot handled by this thread: its own cell, and for tid < 84 one
  // halo cell of the (TX+2) x (TY+2) window.
  const int own_slot = (ty + 1) * PX + (tx + 1);
  int halo_slot = -1;
  if (tid < PC - NTHREADS) {
    const int h = tid;
    if (h < PX) halo_slot = h;
    else if (h < 2 * PX) halo_slot = (PY - 1) * PX + (h - PX);
    else if (h < 2 * PX + TY) halo_slot = (h - 2 * PX + 1) * PX;
    else halo_slot = (h - 2 * PX - TY + 1) * PX + (PX - 1);
  }
  const int own_raw = (ty + 1) * BXW + (tx + 1);
  const int halo_raw = halo_slot >= 0 ? (halo_slot / PX) * BXW + (halo_slot % PX) : 0;
  const int halo_row = halo_slot >= 0 ? halo_slot / PX : 0;

  double acc_w = 0., acc_n = 0., rmax = 0., nonfinite = 0.;

  for (;;) {
    if (tid == 0) w_sh = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int w = w_sh;
    if (w >= nitems) break;
    const int4 it = items[w];
    const InstT& I = insts[it.x];
    const Step2FConst& c = I.c;
    const Step2FArgs& A = I.a[parity];
    const CUtensorMap* mp = &I.map_p[parity];
    const CUtensorMap* ms = &I.map_s[parity];
    const CUtensorMap* mK = &I.map_K;
    const CUtensorMap* mm = &I.map_m;
    const int tile = it.y, zc = it.z;
    const int ti = tile % c.tiles_x, tj = tile / c.tiles_x;
    const int i0 = 1 + ti * TX, j0 = 1 + tj * TY;
    const int x0 = i0 - 1;  // == 32 * ti: 128-byte aligned TMA start
    const int i = i0 + tx, j = j0 + ty;
    const bool active = (i <= c.nx - 2) && (j <= c.ny - 2);
    const bool planar = c.nz == 1;
    const int kb = planar ? 0 : 1 + zc * c.zchunk;
    const int ke = planar ? 0 : min(kb + c.zchunk, c.nz - 1);  // last plane loaded
    const int pb = planar ? 0 : kb - 1;                         // first plane loaded
    const uint32_t stage_bytes = (UNIK ? 3u : 4u) * (uint32_t)(BXW * BYW * sizeof(float));

    if (tid < BYW) {
      const int gj = min(j0 - 1 + tid, c.ny - 1);
      rowPrelF[tid] = A.PrelF[gj];
      rowDPrefF[tid] = A.dPrefF[gj];
      rowPrefD[tid] = A.Pref[gj];
      rowPrelD[tid] = A.Pref[gj] - c.P_atm;
    }
    if (tid == 0) {
      for (int q = 0; q < NST && pb + q <= ke; q++) {
        const int pl = pb + q;
        mbar_expect_tx(&bar[q], stage_bytes);
        tma_load_3d(raw[q].p, mp, x0, j0 - 1, pl, &bar[q]);
        tma_load_3d(raw[q].s, ms, x0, j0 - 1, pl, &bar[q]);
        if (!UNIK) tma_load_3d(raw[q].K, mK, x0, j0 - 1, pl, &bar[q]);
        tma_load_3d(raw[q].m, mm, x0, j0 - 1, pl, &bar[q]);
      }
    }
    __syncthreads();

    OwnCell cm, cc, cp;  // own column at p-2, p-1, p
    for (int pl = pb; pl <= ke; pl++) {
      const int st = (pl - pb) % NST;
      {  // wait for the plane (bounded)
        const uint32_t par = (phase >> st) & 1u;
        unsigned long long tries = 0;
        while (!mbar_try_wait(&bar[st], par)) {
          if (++tries > WAIT_LIMIT) {
            atomicOr(A.err, 2u);
            break;
          }
        }
        phase ^= (1u << st);
      }
      // Derived quantities of plane pl into der[pl & 3].
      const RawStage& R = raw[st];
      DerPlane& D = der[pl & 3];
      {
        const float Kv = UNIK ? c.K0_f : R.K[own_raw];
        OwnCell v = derive<PD0, LAM2>(c, R.p[own_raw], R.s[own_raw], Kv, R.m[own_raw], rowPrelF[ty + 1]);
        D.p[own_slot] = v.p;
        D.pn[own_slot] = v.pn;
        D.Mw[own_slot] = v.Mw;
        D.Mn[own_slot] = v.Mn;
        cm = cc;
        cc = cp;
        cp = v;
      }
      if (halo_slot >= 0) {
        const float Kv = UNIK ? c.K0_f : R.K[halo_raw];
        OwnCell v = derive<PD0, LAM2>(c, R.p[halo_raw], R.s[halo_raw], Kv, R.m[halo_raw], rowPrelF[halo_row]);
        D.p[halo_slot] = v.p;
        D.pn[halo_slot] = v.pn;
        D.Mw[halo_slot] = v.Mw;
        D.Mn[halo_slot] = v.Mn;
      }
      __syncthreads();
      // Stage st is consumed by every thread: refill it four planes ahead.
      if (tid == 0 && pl + NST <= ke) {
        fence_proxy_async();
        const int nxt = pl + NST;
        mbar_expect_tx(&bar[st], stage_bytes);
        tma_load_3d(raw[st].p, mp, x0, j0 - 1, nxt, &bar[st]);
        tma_load_3d(raw[st].s, ms, x0, j0 - 1, nxt, &bar[st]);
        if (!UNIK) tma_load_3d(raw[st].K, mK, x0, j0 - 1, nxt, &bar[st]);
        tma_load_3d(raw[st].m, mm, x0, j0 - 1, nxt, &bar[st]);
      }
      // Centre plane: pl - 1 (3-D) or pl (planar).
      if (!planar && pl < kb + 1) continue;
      const int k = planar ? pl : pl - 1;
      if (!active) continue;
      const OwnCell& C0 = planar ? cp : cc;
      const DerPlane& C = der[k & 3];
      const int cidx = own_slot;
      const float gw = c.g_f * C0.rho_w, gn = c.g_f * C0.rho_n;
      Kahan dw, dn;
      {  // x
        const int a = cidx - 1, b = cidx + 1;
        axis(dw, -(C0.p - C.p[a]) * c.inv_hx_f, -(C.p[b] - C0.p) * c.inv_hx_f, C0.Mw, C.Mw[a], C.Mw[b], c.inv_hx_f);
        axis(dn, -(C0.pn - C.pn[a]) * c.inv_hx_f, -(C.pn[b] - C0.pn) * c.inv_hx_f, C0.Mn, C.Mn[a], C.Mn[b],
             c.inv_hx_f);
      }
      {  // y (vertical): P(j+1) - P(j) = dPref(j) + p(j+1) - p(j)
        const int a = cidx - PX, b = cidx + PX;
        const float dup = rowDPrefF[ty + 1], ddn = rowDPrefF[ty];
        axis(dw, -((ddn + (C0.p - C.p[a])) * c.inv_hy_f) + gw, -((dup + (C.p[b] - C0.p)) * c.inv_hy_f) + gw, C0.Mw,
             C.Mw[a], C.Mw[b], c.inv_hy_f);
        axis(dn, -((ddn + (C0.pn - C.pn[a])) * c.inv_hy_f) + gn, -((dup + (C.pn[b] - C0.pn)) * c.inv_hy_f) + gn,
             C0.Mn, C.Mn[a], C.Mn[b], c.inv_hy_f);
      }
      if (!planar) {  // z, from the registers of the own column
        axis(dw, -(cc.p - cm.p) * c.inv_hz_f, -(cp.p - cc.p) * c.inv_hz_f, cc.Mw, cm.Mw, cp.Mw, c.inv_hz_f);
        axis(dn, -(cc.pn - cm.pn) * c.inv_hz_f, -(cp.pn - cc.pn) * c.inv_hz_f, cc.Mn, cm.Mn, cp.Mn, c.inv_hz_f);
      }
      const double dtm = c.dt / (double)C0.m;
      const double Aw = -dtm * dw.value();
      const double An = -dtm * dn.value();

      // FP64 delta-form Newton about the stored state (two-phase.cpp:25-56).
      const double S = c.S_ref + (double)C0.s;
      const double prel = rowPrelD[ty + 1] + (double)C0.p;
      double Pk0 = 0.;
      if (!PD0) Pk0 = c.P_d * pow((1. - S - c.S_wr) / (1. - c.S_wr), c.e_pk);
      const double rw = c.ro0_w * (1. + c.beta_w * prel);
      const double rn = c.ro0_n * (1. + c.beta_n * (prel + Pk0));
      const double aw = c.ro0_w * c.beta_w, bn = c.ro0_n * c.beta_n;
      double dP = 0., dS = 0., F1 = 0., F2 = 0.;
      const int nit = DIAG ? c.iters + 1 : c.iters;
      for (int itn = 0; itn < nit; itn++) {
        double Pk1 = 0., dPk = 0.;
        if (!PD0) {
          const double Se1 = (1. - (S + dS) - c.S_wr) / (1. - c.S_wr);
          Pk1 = c.P_d * pow(Se1, c.e_pk);
          dPk = -Pk1 * c.e_pk / (Se1 * (1. - c.S_wr));
        }
        F1 = -rw * dS + aw * dP * (1. - S - dS) - Aw;
        F2 = rn * dS + bn * (dP + (Pk1 - Pk0)) * (S + dS) - An;
        if (itn == c.iters) break;  // diagnostics: residual at the final iterate
        const double J11 = aw * (1. - S - dS), J12 = -rw - aw * dP;
        const double J21 = bn * (S + dS), J22 = rn + bn * (dP + (Pk1 - Pk0)) + bn * dPk * (S + dS);
        const double inv = 1. / (J11 * J22 - J12 * J21);
        dP -= (J22 * F1 - J12 * F2) * inv;
        dS -= (J11 * F2 - J21 * F1) * inv;
      }
      const float p1 = (float)((double)C0.p + dP);
      const float s1 = (float)((double)C0.s + dS);
      const long long l = i + j * c.sy + (long long)k * c.sz;
      A.p_out[l] = p1;
      A.s_out[l] = s1;
      const bool finite = isfinite(p1) && isfinite(s1);
      if (!finite) atomicOr(A.err, 1u);

      const bool edge = (i == 1) || (i == c.nx - 2) || (j == 1) || (j == c.ny - 2) ||
                        (!planar && ((k == 1) || (k == c.nz - 2)));
      if (edge) {
        const double Snew = c.S_ref + (double)s1;
        const double Pnew = rowPrefD[ty + 1] + (double)p1;
        const double ro_g_dy = (rn * Snew + rw * (1 - Snew)) * (double)C0.m * c.g * c.hy;
        int xs[3], ys[3], zs[3], nxs = 0, nys = 0, nzs = 0;
        xs[nxs++] = i;
        if (i == 1) xs[nxs++] = 0;
        if (i == c.nx - 2) xs[nxs++] = c.nx - 1;
        ys[nys++] = j;
        if (j == 1) ys[nys++] = 0;
        if (j == c.ny - 2) ys[nys++] = c.ny - 1;
        zs[nzs++] = k;
        if (!planar) {
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
              float pbv;
              if ((bj != 0) && (bj != c.ny - 1)) pbv = p1;
              else if (bj == 0) pbv = (float)((c.P_atm + c.P_top) - A.Pref[0]);
              else pbv = (float)(Pnew + ro_g_dy - A.Pref[c.ny - 1]);
              A.s_out[lb] = sb;
              A.p_out[lb] = pbv;
            }
      }
      if (DIAG) {
        const double S1 = c.S_ref + (double)s1;
        const double P1rel = rowPrelD[ty + 1] + (double)p1;
        double Pk1 = 0.;
        if (!PD0) Pk1 = c.P_d * pow((1. - S1 - c.S_wr) / (1. - c.S_wr), c.e_pk);
        const double rw1 = c.ro0_w * (1. + c.beta_w * P1rel);
        const double rn1 = c.ro0_n * (1. + c.beta_n * (P1rel + Pk1));
        acc_w += (double)C0.m * rw1 * (1. - S1) * c.vol;
        acc_n += (double)C0.m * rn1 * S1 * c.vol;
        const double r = fmax(fabs(F1) / c.ro0_w, fabs(F2) / c.ro0_n);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    }
    __syncthreads();  // the next item's loads reuse the stages and rows
  }

  if (DIAG) {
    __shared__ double red[NTHREADS / 32][4];
    const int lane = tid & 31, wid = tid >> 5;
    const double s0 = warp_sum(acc_w), s1 = warp_sum(acc_n), r = warp_max(rmax), nf = warp_sum(nonfinite);
    if (lane == 0) {
      red[wid][0] = s0;
      red[wid][1] = s1;
      red[wid][2] = r;
      red[wid][3] = nf;
    }
    __syncthreads();
    if (tid == 0) {
      double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
      for (int q = 0; q < NTHREADS / 32; q++) {
        t0 += red[q][0];
        t1 += red[q][1];
        t2 = fmax(t2, red[q][2]);
        t3 += red[q][3];
      }
      double* out = diag_partials + (size_t)DIAG_STRIDE * blockIdx.x;
      out[0] = t0;
      out[1] = t1;
      out[2] = 0.;
      out[3] = t2;
      out[4] = t3;
    }
  }
}

template <bool UNIK, bool PD0, bool LAM2, bool DIAG>
int occupancy_t() {
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_tma_kernel<UNIK, PD0, LAM2, DIAG>, NTHREADS, 0);
  return per;
}

}  // namespace

cudaError_t launch_step2_fp32c_tma(const InstT* insts, const int4* items, int nitems, int parity, const TmaFlags& f,
                                   unsigned int* counter, double* diag_partials, int grid, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
  const bool dg = diag_partials != nullptr;
#define CAPAZ_TMA_LAUNCH(U, P, L, D) \
  step2_fp32c_tma_kernel<U, P, L, D><<<grid, dim3(TX, TY), 0, s>>>(insts, items, nitems, parity, counter, diag_partials)
#define CAPAZ_TMA_D(U, P, L) \
  do {                       \
    if (dg) CAPAZ_TMA_LAUNCH(U, P, L, true); else CAPAZ_TMA_LAUNCH(U, P, L, false); \
  } while (0)
#define CAPAZ_TMA_L(U, P) \
  do {                    \
    if (f.lam2) CAPAZ_TMA_D(U, P, true); else CAPAZ_TMA_D(U, P, false); \
  } while (0)
  if (f.unik) {
    if (f.pd0) CAPAZ_TMA_L(true, true); else CAPAZ_TMA_L(true, false);
  } else {
    if (f.pd0) CAPAZ_TMA_L(false, true); else CAPAZ_TMA_L(false, false);
  }
#undef CAPAZ_TMA_L
#undef CAPAZ_TMA_D
#undef CAPAZ_TMA_LAUNCH
  return cudaGetLastError();
}

int step2_fp32c_tma_grid(int device, const TmaFlags& f) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int per = f.unik ? (f.pd0 ? occupancy_t<true, true, true, true>() : occupancy_t<true, false, true, true>())
                   : (f.pd0 ? occupancy_t<false, true, true, true>() : occupancy_t<false, false, true, true>());
  if (per < 1) per = 1;
  return sms * per;
}

// Builds the 3-D tensor map of one float32 field of an nx x ny x nz grid
// with the 36 x 10 x 1 box of the kernel.  nx must be a multiple of 4 (row
// pitch a multiple of 16 bytes).
int encode_field_map(CUtensorMap* map, const float* base, int nx, int ny, int nz) {
  typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !ptr)
      return -1;
    fn = (EncodeFn)ptr;
  }
  if (nx % 4 != 0) return -2;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
  const cuuint32_t box[3] = {(cuuint32_t)BXW, (cuuint32_t)BYW, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

}  // namespace capaz
