// Two-phase precision-form step with TMA-staged z-planes (sm_100a).
//
// Same model as step2_fp32c.cu (FP32 deviation storage, FP32 stencil with
// Kahan-compensated divergence, FP64 delta-form Newton), specialised for the
// configuration the workloads use (no capillary pressure, P_d = 0, so
// P_n = P_w; Brooks-Corey index lambda = 2, so k_w = S_e^4 and
// k_n = (1-S_e)^2 (1-S_e^2)), and laid out for Blackwell:
//   - persistent CTAs take (instance, tile, z-chunk) work items from a global
//     counter, so one launch covers one grid or a whole ensemble of uneven
//     grids without tail waves;
//   - a tile is 32 x 16 cells; each of the 256 threads owns two cells of a
//     column (rows ty and ty + 8), which halves the per-cell share of the
//     plane loop's fixed work and brings the halo down to 96 cells per 512;
//   - one elected thread streams the raw planes (p, s, K, m) of the tile's
//     window (a 36 x 18 box at x = 32*ti, a 128-byte-aligned start) into a
//     3-stage shared-memory ring with cp.async.bulk.tensor (TMA, 3-D tensor
//     maps, no multicast) completing on mbarriers;
//   - every thread derives its cells (three warps one halo cell more; the
//     window's corners are never read) into a 3-slot ring of derived planes,
//     (p, M_w, M_n) packed as float4, and reads the centre plane and its
//     -z / +z neighbours from the ring: one barrier per plane, and few enough
//     registers for three CTAs per SM;
//   - physics constants are kernel parameters (constant-bank operands);
//     per-row quantities (rho at the row's reference pressure, the scaled
//     reference-pressure step) come from small per-instance tables.
// Arithmetic per face (cpu.cpp:236-264 in select form): the driving force
// x = -dP/h (+ g rho_c on the vertical axis) is evaluated once for both
// phases; outflow through the + face is x2 * M(upwind), inflow through the
// - face x1 * M(upwind); the in/out difference of an axis is formed first
// (exact when the two nearly cancel, by Sterbenz's lemma) and the three axis
// terms are Kahan-summed, both phases at once in packed f32x2 arithmetic.
// d(rho S) = -dt/m * div goes to FP64, where one Newton step with the
// Jacobian at the stored state solves the bilinear system for (dP, dS).
// Boundary cells are written by a second, small kernel over the boundary
// shell after the sweep, which keeps the sweep free of per-cell face tests.
// Waits on mbarriers are bounded; a wait that runs out sets bit 1 of the
// error flag and the CTA carries on, so the kernel always finishes.
#include <cuda.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "capaz_internal.h"
#include "diag_reduce.cuh"

namespace capaz {
namespace {

constexpr int TYK = TMA_TY;        // thread rows of a CTA
constexpr int NTK = TX * TYK;      // threads of a CTA
constexpr int TYT = TMA_TILE_Y;    // tile height: each thread row owns two cell rows (ty, ty + TYK)
constexpr int WX = TX + 2;         // derived-plane window: tile plus a one-cell halo
constexpr int WY = TYT + 2;
constexpr int WCELLS = WX * WY;
constexpr int NHALO = 2 * TX + 2 * TYT;  // halo cells derived by threads 0..NHALO-1 (no corners)
constexpr int BXW = 36;            // TMA box width (floats): 144 bytes, a multiple of 16
constexpr int BYW = WY;            // TMA box height
constexpr int NST = 3;             // planes in flight (raw stages and derived slots)
constexpr int RAWN = (BXW * BYW + 31) / 32 * 32;  // floats reserved per array per stage (128-B multiple)
static_assert(BXW * BYW <= RAWN, "raw stage too small");
static_assert(NHALO <= NTK && 2 * TYT <= 32, "halo cells exceed the block");
constexpr unsigned long long WAIT_LIMIT = 1ull << 22;  // try_wait polls before giving up

struct alignas(128) RawStage {
  float p[RAWN], s[RAWN], K[RAWN], m[RAWN];
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
// Programmatic dependent launch: wait until the grids this launch depends on
// have completed and their memory is visible (a no-op for an ordinary launch).
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Derived values of one cell: pressure deviation and the two phases'
// mobility-density M = K k_r rho / mu (= -Xi * rho of the reference).
struct Der {
  float p, Mw, Mn;
};
// The centre cell also needs its saturation deviation, porosity and
// densities.
struct Ctr {
  float s, m, rw, rn;
};

__device__ __forceinline__ void derive(const PhysF& f, float c1, float Aw, float An, float p, float s, float K,
                                       Der& d) {
  // Aw, An: rho_p / mu_p at the row's reference pressure; rho_p(P) / mu_p is
  // linear in the pressure deviation p.
  const float S_e = (c1 - s) * f.inv_one_m_swr;
  const float e2 = S_e * S_e;
  const float om = 1.f - S_e;
  const float kw = e2 * e2;
  const float kn = om * om * (1.f - e2);
  d.p = p;
  d.Mw = K * kw * fmaf(f.cw_mu, p, Aw);
  d.Mn = K * kn * fmaf(f.cn_mu, p, An);
}

// In/out difference of one axis for one phase: x1, x2 are the scaled driving
// forces on the - and + faces (positive towards +).
__device__ __forceinline__ float face_diff(float x1, float x2, float Mc, float Mm, float Mp) {
  const float out = x2 * (x2 > 0.f ? Mc : Mp);
  const float in = x1 * (x1 > 0.f ? Mm : Mc);
  return out - in;
}

// Two FP32 values in one 64-bit register pair for sm_100's packed f32x2
// arithmetic: every lane is an ordinary round-to-nearest FP32 operation, one
// instruction for both phases.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pack2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void unpack2(f32x2 r, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Kahan sum of three terms of both phases at once, the first term taken as
// the start.
struct Kahan2 {
  f32x2 s, c;
  __device__ __forceinline__ explicit Kahan2(f32x2 a) : s(a), c(0ull) {}
  __device__ __forceinline__ void add(f32x2 x) {
    const f32x2 y = sub2(x, c);
    const f32x2 t = add2(s, y);
    c = sub2(sub2(t, s), y);
    s = t;
  }
  __device__ __forceinline__ f32x2 sum() const { return sub2(s, c); }
};

__device__ __forceinline__ double rcp64(double x) {
  // FP32 seed refined by one Newton-Raphson step r <- r (2 - x r), which
  // squares the relative error: 2^-23 -> 2^-46, far below the FP32 storage
  // of the result.
  double r = (double)__frcp_rn((float)x);
  r = r * fma(-x, r, 2.0);
  return r;
}

__device__ __forceinline__ bool in_window(const InstT* I, int i, int k) {
  return (i >= I->nx / 2 - I->source) && (i <= I->nx / 2 + I->source) && (k >= I->win_k0) && (k <= I->win_k1);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Shared memory of one CTA (dynamic, 62 KB: three CTAs per SM).
struct Smem {
  RawStage raw[NST];
  float4 der[NST][WCELLS];  // (p, M_w, M_n, -) of the window, one slot per plane in flight
  uint64_t bar[NST];
  float4 rowF[WY];          // (rho_w/mu_w, rho_n/mu_n at the row's P_ref, dP_ref/hy^2 to the next row, -)
  double rowPrel[WY];       // P_ref - P_atm
  double rowPref[WY];
  double red[NTK / 32][4];  // diagnostics reduction
  int w_sh;
};
constexpr size_t kSmemBytes = sizeof(Smem);

#ifndef CAPAZ_TMA_MIN_BLOCKS
#define CAPAZ_TMA_MIN_BLOCKS 3
#endif
template <bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
__global__ void __launch_bounds__(NTK, CAPAZ_TMA_MIN_BLOCKS)
    step2_fp32c_tma_kernel(const __grid_constant__ PhysF f, const InstT* __restrict__ insts,
                           const int4* __restrict__ items, int nitems, int parity, unsigned int* __restrict__ counter,
                           double* __restrict__ diag_partials) {
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_bytes);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + TX * ty;
  if (tid == 0) {
    for (int q = 0; q < NST; q++) mbar_init(&sm.bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;  // bit q: parity of the next completion of stage q

  // The thread's two cells are tile rows ty and ty + TYK (window rows +1).
  const int ownA = (ty + 1) * WX + (tx + 1), ownB = ownA + TYK * WX;
  const int rawA = (ty + 1) * BXW + (tx + 1), rawB = rawA + TYK * BXW;
  // Halo cells of the 7-point stencil (the window's corners are never read):
  // warp 0 the row above the tile, warp 1 the row below, warp 2 the columns
  // left (lanes 0-15) and right (lanes 16-31).
  int halo_slot = -1, halo_raw = 0, halo_row = 0;
  if (tid < NHALO) {
    const int wq = tid >> 5, lane = tid & 31;
    int hx, hy;
    if (wq == 0) hx = lane + 1, hy = 0;
    else if (wq == 1) hx = lane + 1, hy = WY - 1;
    else if (lane < TYT) hx = 0, hy = lane + 1;
    else hx = WX - 1, hy = lane - TYT + 1;
    halo_slot = hy * WX + hx;
    halo_raw = hy * BXW + hx;
    halo_row = hy;
  }

  double acc_w = 0., acc_n = 0., nonfinite = 0.;
  float rmax = 0.f;
  // Diagnostics: masses summed without the cell volume (applied once per
  // CTA), residuals scaled by 1/rho_0.
  const float iro0w_f = DIAG ? (float)(1. / f.ro0_w) : 0.f, iro0n_f = DIAG ? (float)(1. / f.ro0_n) : 0.f;
  const float aw_ro0w_f = DIAG ? (float)(f.aw / f.ro0_w) : 0.f, bn_ro0n_f = DIAG ? (float)(f.bn / f.ro0_n) : 0.f;
  // Everything above overlaps the previous kernel's tail; the work counter and
  // the state are touched only after it has completed.
  grid_dependency_wait();

  for (;;) {
    if (tid == 0) sm.w_sh = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int w = sm.w_sh;
    if (w >= nitems) {
      // No work left for this CTA: the boundary kernel may be scheduled (it
      // waits for the whole sweep with griddepcontrol.wait).
      asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
      break;
    }
    const int4 it = items[w];
    const InstT* __restrict__ I = insts + it.x;
    const int nx = I->nx, ny = I->ny, nz = I->nz;
    const int sy32 = (int)I->sy, sz32 = (int)I->sz;  // instances hold < 2^31 cells
    const float c1 = I->c1_f;
    const float dt_f = I->dt_f;
    const double S_ref = I->S_ref;
    const Step2FArgs& A = I->a[parity];
    float* __restrict__ p_out = A.p_out;
    float* __restrict__ s_out = A.s_out;
    unsigned int* __restrict__ err = A.err;
    const int tile = it.y, zc = it.z;
    const int ti = tile % I->tiles_x, tj = tile / I->tiles_x;
    const int i0 = 1 + ti * TX, j0 = 1 + tj * TYT;
    const int x0 = i0 - 1;  // == 32 * ti: 128-byte aligned TMA start
    const int i = i0 + tx, jA = j0 + ty, jB = jA + TYK;
    const bool activeA = (i <= nx - 2) && (jA <= ny - 2);
    const bool activeB = (i <= nx - 2) && (jB <= ny - 2);
    const int lA0 = i + jA * sy32;
    bool bad = false;
    const int kb = PLANAR ? 0 : 1 + zc * I->zchunk;
    const int ke = PLANAR ? 0 : min(kb + I->zchunk, nz - 1);  // last plane loaded
    const int pb = PLANAR ? 0 : kb - 1;                         // first plane loaded
    const uint32_t stage_bytes = (UNIK ? 3u : 4u) * (uint32_t)(BXW * BYW * sizeof(float));

    if (tid < WY) {
      const int gj = min(j0 - 1 + tid, ny - 1);
      sm.rowF[tid] = I->rowF[gj];
      sm.rowPrel[tid] = I->Pref[gj] - f.P_atm;
      sm.rowPref[tid] = I->Pref[gj];
    }
    if (tid == 0) {
      for (int q = 0; q < NST && pb + q <= ke; q++) {
        const int pl = pb + q;
        mbar_expect_tx(&sm.bar[q], stage_bytes);
        tma_load_3d(sm.raw[q].p, &I->map_p[parity], x0, j0 - 1, pl, &sm.bar[q]);
        tma_load_3d(sm.raw[q].s, &I->map_s[parity], x0, j0 - 1, pl, &sm.bar[q]);
        if (!UNIK) tma_load_3d(sm.raw[q].K, &I->map_K, x0, j0 - 1, pl, &sm.bar[q]);
        tma_load_3d(sm.raw[q].m, &I->map_m, x0, j0 - 1, pl, &sm.bar[q]);
      }
    }
    __syncthreads();
    const float4 rowA = sm.rowF[ty + 1], rowB = sm.rowF[ty + TYK + 1];
    const float dnA = sm.rowF[ty].z, dnB = sm.rowF[ty + TYK].z;

    // The centre-plane update of one cell: D holds the centre plane, Dm / Dp
    // the planes below and above it; sc, mc are the cell's saturation
    // deviation and porosity.
    auto update = [&](const float4* __restrict__ D, const float4* __restrict__ Dm, const float4* __restrict__ Dp,
                      int own, float4 row, float dPs_dn, int wrow, float sc, float mc, int l, bool active) {
      const float4 c4 = D[own];
      const Der C0{c4.x, c4.y, c4.z};
      f32x2 D2;  // (div F_w, div F_n)
      {
        const float4 a = D[own - 1], b = D[own + 1];
        // Forces: pressure differences of neighbours (exact when they are
        // close), scaled by 1/h^2 unless the spacing is 1.
        const float x1 = UNITH ? a.x - C0.p : (a.x - C0.p) * f.inv_hx2;
        const float x2 = UNITH ? C0.p - b.x : (C0.p - b.x) * f.inv_hx2;
        const bool u1 = x1 > 0.f, u2 = x2 > 0.f;
        const float dxw = x2 * (u2 ? C0.Mw : b.y) - x1 * (u1 ? a.y : C0.Mw);
        const float dxn = x2 * (u2 ? C0.Mn : b.z) - x1 * (u1 ? a.z : C0.Mn);
        // y (vertical, gravity): P(j+1) - P(j) = dP_ref(j) + p(j+1) - p(j)
        const float4 ya = D[own - WX], yb = D[own + WX];
        const float gw = f.g_mu_w * fmaf(f.cw_mu, C0.p, row.x), gn = f.g_mu_n * fmaf(f.cn_mu, C0.p, row.y);
        const float y1 = UNITH ? (ya.x - C0.p) - dPs_dn : fmaf(ya.x - C0.p, f.inv_hy2, -dPs_dn);
        const float y2 = UNITH ? (C0.p - yb.x) - row.z : fmaf(C0.p - yb.x, f.inv_hy2, -row.z);
        const float dyw = face_diff(y1 + gw, y2 + gw, C0.Mw, ya.y, yb.y);
        const float dyn = face_diff(y1 + gn, y2 + gn, C0.Mn, ya.z, yb.z);
        Kahan2 k(pack2(dxw, dxn));
        k.add(pack2(dyw, dyn));
        if (!PLANAR) {
          const float4 m4 = Dm[own], p4 = Dp[own];
          const Der m1{m4.x, m4.y, m4.z}, p1{p4.x, p4.y, p4.z};
          const float z1 = UNITH ? m1.p - C0.p : (m1.p - C0.p) * f.inv_hz2;
          const float z2 = UNITH ? C0.p - p1.p : (C0.p - p1.p) * f.inv_hz2;
          const bool v1 = z1 > 0.f, v2 = z2 > 0.f;
          k.add(pack2(z2 * (v2 ? C0.Mw : p1.Mw) - z1 * (v1 ? m1.Mw : C0.Mw),
                      z2 * (v2 ? C0.Mn : p1.Mn) - z1 * (v1 ? m1.Mn : C0.Mn)));
        }
        D2 = k.sum();
      }
      // Conserved increments d(rho S) = -dt/m * div F (FP32), Newton in FP64.
      const float dtm = __fdividef(dt_f, mc);
      float Awf, Anf;
      unpack2(mul2(pack2(-dtm, -dtm), D2), Awf, Anf);
      const double Aw = (double)Awf;
      const double An = (double)Anf;
      const double S = S_ref + (double)sc;
      const double prel = sm.rowPrel[wrow];
      const double pr = prel + (double)C0.p;
      const double rw = fma(f.aw, pr, f.ro0_w);
      const double rn = fma(f.bn, pr, f.ro0_n);
      const double J11 = f.aw * (1. - S), J21 = f.bn * S;
      const double det = fma(J11, rn, rw * J21);  // J11 J22 - J12 J21, J12 = -rw, J22 = rn
      const double inv = rcp64(det);
      // One Newton step from the stored state: the Jacobian solve of the
      // bilinear system, exact up to the dP*dS terms (relative size
      // |dS| / S ~ 1e-8 of the increments).
      const double dP = (rn * Aw + rw * An) * inv;
      const double dS = (J11 * An - J21 * Aw) * inv;
      float rf = 0.f;
      if (DIAG) {
        // The reference's Newton functions at (dP, dS),
        //   F1 = (rw + a_w dP)(1 - S - dS) - rw (1 - S) - Aw,
        //   F2 = (rn + b_n dP)(S + dS) - rn S - An,
        // are, for the solve above, exactly F1 = Aw e - a_w dP dS and
        // F2 = An e + b_n dP dS with e = det * inv - 1 (the linear part
        // leaves Aw e, An e).  Written so they have no cancellation left;
        // FP32 holds their size (~1e-14 of Aw) to 1e-7, and they are
        // reported scaled by 1/rho_0.
        const float e = (float)fma(det, inv, -1.);
        const float q = (float)(dP * dS);
        const float F1 = fmaf(Awf * iro0w_f, e, -aw_ro0w_f * q);
        const float F2 = fmaf(Anf * iro0n_f, e, bn_ro0n_f * q);
        rf = fmaxf(fabsf(F1), fabsf(F2));
      }
      const float pn = (float)((double)C0.p + dP);
      const float snew = (float)((double)sc + dS);
      // Cells beyond the grid's interior (partial tiles) compute on the
      // window's fill values and store nothing.
      if (active) {
        p_out[l] = pn;
        s_out[l] = snew;
      }
      const bool finite = isfinite(pn) && isfinite(snew);
      bad |= active && !finite;
      if (DIAG && active) {
        const double md = (double)mc;
        const double mS1 = md * (S_ref + (double)snew);  // m S_n; m (1 - S_n) = m - m S_n
        const double P1rel = prel + (double)pn;
        acc_w = fma(md - mS1, fma(f.aw, P1rel, f.ro0_w), acc_w);
        acc_n = fma(mS1, fma(f.bn, P1rel, f.ro0_n), acc_n);
        if (!(rf <= rmax)) rmax = rf;
        if (!finite) nonfinite += 1.;
      }
    };

    // The sweep: plane pl is derived into ring slot u = (pl - pb) mod 3 while
    // the centre plane pl - 1 is updated from the slots of pl - 2, pl - 1, pl.
    // Unrolled by three so that every slot index is a compile-time constant.
    float sA0 = 0.f, mA0 = 0.f, sB0 = 0.f, mB0 = 0.f;  // centre plane's s, m of the two cells
    auto plane = [&](auto U, int pl) {
      constexpr int u = decltype(U)::value;
      {  // wait for the plane (bounded)
        const uint32_t par = (phase >> u) & 1u;
        unsigned long long tries = 0;
        while (!mbar_try_wait(&sm.bar[u], par)) {
          if (++tries > WAIT_LIMIT) {
            atomicOr(err, 2u);
            break;
          }
        }
        phase ^= (1u << u);
      }
      const RawStage& R = sm.raw[u];
      float4* __restrict__ D = sm.der[u];
      float sA1, mA1, sB1, mB1;
      {
        Der dA, dB;
        sA1 = R.s[rawA];
        sB1 = R.s[rawB];
        mA1 = R.m[rawA];
        mB1 = R.m[rawB];
        derive(f, c1, rowA.x, rowA.y, R.p[rawA], sA1, UNIK ? f.K0 : R.K[rawA], dA);
        derive(f, c1, rowB.x, rowB.y, R.p[rawB], sB1, UNIK ? f.K0 : R.K[rawB], dB);
        D[ownA] = make_float4(dA.p, dA.Mw, dA.Mn, 0.f);
        D[ownB] = make_float4(dB.p, dB.Mw, dB.Mn, 0.f);
      }
      if (halo_slot >= 0) {
        const float4 rh = sm.rowF[halo_row];
        Der h;
        derive(f, c1, rh.x, rh.y, R.p[halo_raw], R.s[halo_raw], UNIK ? f.K0 : R.K[halo_raw], h);
        D[halo_slot] = make_float4(h.p, h.Mw, h.Mn, 0.f);
      }
      __syncthreads();
      // Stage u has been read by every thread: refill it three planes ahead.
      if (tid == 0 && pl + NST <= ke) {
        fence_proxy_async();
        const int nxt = pl + NST;
        mbar_expect_tx(&sm.bar[u], stage_bytes);
        tma_load_3d(sm.raw[u].p, &I->map_p[parity], x0, j0 - 1, nxt, &sm.bar[u]);
        tma_load_3d(sm.raw[u].s, &I->map_s[parity], x0, j0 - 1, nxt, &sm.bar[u]);
        if (!UNIK) tma_load_3d(sm.raw[u].K, &I->map_K, x0, j0 - 1, nxt, &sm.bar[u]);
        tma_load_3d(sm.raw[u].m, &I->map_m, x0, j0 - 1, nxt, &sm.bar[u]);
      }
      if (PLANAR) {
        const int lA = lA0, lB = lA0 + TYK * sy32;
        update(D, D, D, ownA, rowA, dnA, ty + 1, sA1, mA1, lA, activeA);
        update(D, D, D, ownB, rowB, dnB, ty + TYK + 1, sB1, mB1, lB, activeB);
      } else if (pl >= pb + 2) {
        constexpr int uc = (u + 2) % NST, um = (u + 1) % NST;
        const int k = pl - 1;
        const int lA = lA0 + k * sz32, lB = lA + TYK * sy32;
        update(sm.der[uc], sm.der[um], D, ownA, rowA, dnA, ty + 1, sA0, mA0, lA, activeA);
        update(sm.der[uc], sm.der[um], D, ownB, rowB, dnB, ty + TYK + 1, sB0, mB0, lB, activeB);
      }
      sA0 = sA1;
      mA0 = mA1;
      sB0 = sB1;
      mB0 = mB1;
    };
    for (int base = pb; base <= ke; base += NST) {
      plane(std::integral_constant<int, 0>{}, base);
      if (base + 1 > ke) break;
      plane(std::integral_constant<int, 1>{}, base + 1);
      if (base + 2 > ke) break;
      plane(std::integral_constant<int, 2>{}, base + 2);
    }
    if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) atomicOr(err, 1u);
    __syncthreads();  // the next item's loads reuse the stages and rows
  }

  if (DIAG) {
    double(*red)[4] = sm.red;
    const int lane = tid & 31, wid = tid >> 5;
    const double s0 = warp_sum(acc_w), s1 = warp_sum(acc_n), r = warp_max((double)rmax), nf = warp_sum(nonfinite);
    if (lane == 0) {
      red[wid][0] = s0;
      red[wid][1] = s1;
      red[wid][2] = r;
      red[wid][3] = nf;
    }
    __syncthreads();
    if (tid == 0) {
      double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
      for (int q = 0; q < NTK / 32; q++) {
        t0 += red[q][0];
        t1 += red[q][1];
        t2 = fmax(t2, red[q][2]);
        t3 += red[q][3];
      }
      double* out = diag_partials + (size_t)DIAG_STRIDE * blockIdx.x;
      out[0] = t0 * f.vol;
      out[1] = t1 * f.vol;
      out[2] = 0.;
      out[3] = t2;
      out[4] = t3;
    }
  }
}

// Boundary cells after the sweep (boundary_conditions, two-phase.cpp:59-111):
// each takes the new state of its basic-coordinate cell (cpu.cpp:107-141),
// an interior cell; the top row holds P_atm (+ the top offset) and, inside
// the injection window, S_n_gr; the bottom row adds the weight
// (rho_n S_n + rho_w (1 - S_n)) m g hy of the basic cell with its new S_n and
// start-of-step densities (Border_P, main.cpp:255-267).  One thread per
// boundary cell; items are (instance, first cell) blocks of BOUND_BLOCK.
// With diagnostics, block 0 also reduces the sweep's per-CTA partials into
// diag_out (they are complete once the sweep is), so the step needs no
// separate reduction launch.
__global__ void __launch_bounds__(BOUND_BLOCK)
    boundary_fp32c_kernel(const __grid_constant__ PhysF f, const InstT* __restrict__ insts,
                          const int2* __restrict__ bitems, int parity, unsigned int* __restrict__ counter,
                          const double* __restrict__ diag_partials, int nparts, double* __restrict__ diag_out) {
  grid_dependency_wait();  // the sweep's interior values and its use of the counter
  // The sweep before this launch has taken all its work items: rearm its
  // work counter for the next step.
  if (blockIdx.x == 0 && threadIdx.x == 0) *counter = 0u;
  if (diag_out != nullptr && blockIdx.x == 0) {
    __shared__ double red[BOUND_BLOCK / 32][DIAG_STRIDE];
    diag_reduce_block<BOUND_BLOCK / 32>(diag_partials, nparts, diag_out, red);
  }
  const int2 it = bitems[blockIdx.x];
  const InstT* __restrict__ I = insts + it.x;
  const int q0 = it.y + (int)threadIdx.x;
  if (q0 >= I->nbound) return;
  const int nx = I->nx, ny = I->ny, nz = I->nz;
  int q = q0, i, j, k;
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
  const int i1 = min(max(i, 1), nx - 2), j1 = min(max(j, 1), ny - 2);
  const int k1 = nz == 1 ? 0 : min(max(k, 1), nz - 2);
  const long long sy = I->sy, sz = I->sz;
  const long long lb = i + j * sy + (long long)k * sz, l1 = i1 + j1 * sy + (long long)k1 * sz;
  const Step2FArgs& A = I->a[parity];
  const float s1 = A.s_out[l1];
  float sb = s1;
  if ((j == 0) && (I->source > 0) && in_window(I, i, k)) sb = I->sgr_dev_f;
  float pb;
  if ((j != 0) && (j != ny - 1)) {
    pb = A.p_out[l1];
  } else if (j == 0) {
    pb = (float)((f.P_atm + f.P_top) - I->Pref[0]);
  } else {
    const double prel = I->Pref[j1] - f.P_atm;
    const double pr = prel + (double)A.p_in[l1];  // start-of-step pressure of the basic cell
    const double rw = fma(f.aw, pr, f.ro0_w), rn = fma(f.bn, pr, f.ro0_n);
    const double Snew = I->S_ref + (double)s1;
    const double Pnew = (prel + f.P_atm) + (double)A.p_out[l1];
    const double ro_g_dy = (rn * Snew + rw * (1 - Snew)) * (double)A.m[l1] * f.g * f.hy;
    pb = (float)(Pnew + ro_g_dy - I->Pref[ny - 1]);
  }
  A.s_out[lb] = sb;
  A.p_out[lb] = pb;
}

// Launches with programmatic stream serialisation: the kernel may start
// while the previous kernel in the stream finishes, and waits for it with
// griddepcontrol.wait before touching what that kernel writes.
template <typename... Params, typename... Args>
cudaError_t launch_dependent(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Opts the kernel into its dynamic shared memory, once per device.
template <bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
cudaError_t prepare_t() {
  static unsigned long long done = 0;  // bit d: set on device d
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(step2_fp32c_tma_kernel<UNIK, DIAG, PLANAR, UNITH>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  if (e == cudaSuccess) __atomic_fetch_or(&done, bit, __ATOMIC_ACQ_REL);
  return e;
}

template <bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
cudaError_t launch_t(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                     unsigned int* counter, double* diag_partials, int grid, cudaStream_t s) {
  cudaError_t e = prepare_t<UNIK, DIAG, PLANAR, UNITH>();
  if (e != cudaSuccess) return e;
  return launch_dependent(step2_fp32c_tma_kernel<UNIK, DIAG, PLANAR, UNITH>, dim3(grid), dim3(TX, TYK), kSmemBytes,
                          s, f, insts, items, nitems, parity, counter, diag_partials);
}

template <bool UNIK, bool DIAG, bool PLANAR>
cudaError_t launch_h(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                     unsigned int* counter, double* diag_partials, int grid, cudaStream_t s) {
  // Unit spacing (the workloads' h = 1 m): forces are plain differences.
  const bool unith = f.inv_hx2 == 1.f && f.inv_hy2 == 1.f && f.inv_hz2 == 1.f;
  return unith ? launch_t<UNIK, DIAG, PLANAR, true>(f, insts, items, nitems, parity, counter, diag_partials, grid, s)
               : launch_t<UNIK, DIAG, PLANAR, false>(f, insts, items, nitems, parity, counter, diag_partials, grid, s);
}

template <bool UNIK, bool DIAG>
cudaError_t launch_p(bool planar, const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                     unsigned int* counter, double* diag_partials, int grid, cudaStream_t s) {
  return planar ? launch_h<UNIK, DIAG, true>(f, insts, items, nitems, parity, counter, diag_partials, grid, s)
                : launch_h<UNIK, DIAG, false>(f, insts, items, nitems, parity, counter, diag_partials, grid, s);
}

}  // namespace

cudaError_t launch_step2_fp32c_tma(const PhysF& f, const InstT* insts, const int4* items, int nitems,
                                   const int2* bitems, int nbitems, int parity, bool unik, bool planar,
                                   unsigned int* counter, double* diag_partials, int grid, cudaStream_t s,
                                   double* diag_out) {
  // `counter` is zero on entry: zeroed at allocation and rearmed by every
  // boundary launch.
  cudaError_t e;
  if (unik)
    e = diag_partials ? launch_p<true, true>(planar, f, insts, items, nitems, parity, counter, diag_partials, grid, s)
                      : launch_p<true, false>(planar, f, insts, items, nitems, parity, counter, nullptr, grid, s);
  else
    e = diag_partials ? launch_p<false, true>(planar, f, insts, items, nitems, parity, counter, diag_partials, grid, s)
                      : launch_p<false, false>(planar, f, insts, items, nitems, parity, counter, nullptr, grid, s);
  if (e != cudaSuccess) return e;
  return launch_dependent(boundary_fp32c_kernel, dim3(nbitems), dim3(BOUND_BLOCK), 0, s, f, insts, bitems, parity,
                          counter, (const double*)diag_partials, grid, diag_partials ? diag_out : nullptr);
}

int step2_fp32c_tma_grid(int device, bool unik) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int per = 0;
  if (unik) {
    prepare_t<true, true, false, false>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_tma_kernel<true, true, false, false>, NTK,
                                                  kSmemBytes);
  } else {
    prepare_t<false, true, false, false>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_tma_kernel<false, true, false, false>, NTK,
                                                  kSmemBytes);
  }
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
