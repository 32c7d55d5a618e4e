// Two-phase precision-form step with TMA-staged z-planes (sm_100a).
//
// Same model as step2_fp32c.cu (FP32 deviation storage, FP32 stencil with
// Kahan-compensated divergence, FP64 delta-form Newton), specialised for the
// configuration the workloads use (no capillary pressure, P_d = 0, so
// P_n = P_w; Brooks-Corey index lambda = 2, so k_w = S_e^4 and
// k_n = (1-S_e)^2 (1-S_e^2)), and laid out for Blackwell:
//   - persistent CTAs take (instance, tile, z-range) work items, the first
//     one by their index and the rest from a global counter, so one launch
//     covers one grid or a whole ensemble of uneven grids; a grid's z-ranges
//     are sized so its items fill the grid of CTAs in as few rounds as
//     possible;
//   - a tile is 32 x 16 cells, a CTA four warps; each thread owns a column
//     segment of four cells and keeps their derived values in registers
//     across planes, so only the x neighbours and the segment ends go
//     through shared memory (the sweep kernel's comment has the details);
//   - the raw planes (p, s, K, m) of the tile's window (a 36 x 18 box at
//     x = 32*ti, a 128-byte-aligned start) stream into a three-stage ring
//     with cp.async.bulk.tensor (TMA, 3-D tensor maps, no multicast)
//     completing on mbarriers, issued by a thread of the warp that derives no
//     halo cells;
//   - at most 128 registers (the launch bound) and 52 KB of shared memory:
//     four CTAs per SM;
//   - physics constants are kernel parameters (constant-bank operands);
//     per-row quantities (rho at the row's reference pressure, the scaled
//     reference-pressure step) come from small per-instance tables.
// Arithmetic per face (cpu.cpp:236-264 in select form): the driving force
// x = -dP/h (+ g rho_c on the vertical axis) is evaluated once for both
// phases; outflow through the + face is x2 * M(upwind), inflow through the
// - face x1 * M(upwind); the out - in term of an axis is one fused
// multiply-add and the three axis terms are Kahan-summed, both phases at once
// in packed f32x2 arithmetic.  d(rho S) = -dt/m * div goes to FP64, where one
// Newton step with the Jacobian at the stored state solves the bilinear
// system for (dP, dS).  Boundary cells are written by a second, small kernel
// over the boundary shell after the sweep, which keeps the sweep free of
// per-cell face tests.
// Waits on mbarriers are bounded (about a second of SM clocks).  A wait that
// runs out in any thread stops the whole CTA: the per-plane barrier votes on
// it, the CTA sets bit 1 of the error flag, waits (bounded again) for the
// copies it still has in flight, and leaves its work list; no stage is
// consumed or re-armed after a timeout, so the kernel always finishes.
#include <cuda.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "capaz_internal.h"
#include "diag_reduce.cuh"

namespace capaz {
namespace {

constexpr int WX = TX + 2;         // derived-plane window: tile plus a one-cell halo
constexpr int BXW = 36;            // TMA box width (floats): 144 bytes, a multiple of 16
constexpr long long WAIT_CYCLES = 2000000000ll;  // bounded waits give up after ~1 s of SM clocks

// Geometry of a tile of TYT interior rows (TMA_TILE_SHAPES): the window with
// its halo, the raw TMA box, the CTA (one warp per four rows) and the CTAs
// that fit an SM.
template <int TYT_>
struct Tile {
  static constexpr int TYT = TYT_;
  static constexpr int WY = TYT + 2;
  static constexpr int WCELLS = WX * WY;
  static constexpr int NHALO = 2 * TX + 2 * TYT;  // halo cells derived by threads 0..NHALO-1 (no corners)
  static constexpr int BYW = WY;                  // TMA box height
  static constexpr int RAWN = (BXW * BYW + 31) / 32 * 32;  // floats per array per stage (128-B multiple)
  static constexpr int R = 4;                     // cells per thread
  static constexpr int NW = TYT / R;              // warps per CTA
  static constexpr int NT = TX * NW;              // threads per CTA
  static constexpr int MINB = TYT <= 16 ? 4 : 2;  // CTAs per SM the launch bounds aim for
};

template <int RAWN_>
struct alignas(128) RawStage {
  float p[RAWN_], s[RAWN_], K[RAWN_], m[RAWN_];
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
// Waits for the completion of phase `par` of a stage barrier; false if it
// has not completed after WAIT_CYCLES.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t par) {
  if (mbar_try_wait(bar, par)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, par))
    if (clock64() - t0 > WAIT_CYCLES) return false;
  return true;
}
__device__ __forceinline__ void st_global(float* p, float v) {
  asm volatile("st.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
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
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Kahan sum of three terms of both phases at once, the first term taken as
// the start.
struct Kahan2 {
  f32x2 s, c;
  __device__ __forceinline__ explicit Kahan2(f32x2 a) : s(a), c(0ull) {}
  // The first two terms: the compensation starts at the rounding of a + b.
  __device__ __forceinline__ Kahan2(f32x2 a, f32x2 b) : s(add2(a, b)), c(sub2(sub2(s, a), b)) {}
  __device__ __forceinline__ void add(f32x2 x) {
    const f32x2 y = sub2(x, c);
    const f32x2 t = add2(s, y);
    c = sub2(sub2(t, s), y);
    s = t;
  }
  __device__ __forceinline__ f32x2 sum() const { return sub2(s, c); }
};

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

// The sweep.  A CTA of four warps covers a 32 x 16 tile of interior cells
// (a 34 x 18 window with its halo); thread (tx, ty) owns the column segment of
// four cells at x = tx, rows 4 ty .. 4 ty + 3.  Per z-plane, one elected
// thread of the warp without halo work streams the raw window (p, s, K, m)
// into a three-stage ring with cp.async.bulk.tensor (3-D tensor maps, no
// multicast) completing on mbarriers; every thread derives its four cells
// (three warps also one halo cell each) into registers and into the plane's
// shared derived slot, as the pair (p, p) and the pair (M_w, M_n) with
// M = K k_r rho / mu.  In the same barrier interval it updates its cells of
// the plane below: the x neighbours and the segment's two end neighbours
// come from that plane's slot (complete since the previous barrier), the
// vertical neighbours inside the segment and both z neighbours from
// registers, and s and m from that plane's raw stage, which is refilled only
// after the barrier that ends the update.  The -z inflow of each cell is the
// +z outflow it computed on the plane below (the same product), carried in
// registers.  One barrier per plane separates a slot's update reads from its
// next writes (two derived slots alternate) and a raw stage's last reads from
// its refill (three stages: the centre plane's, this plane's, and the next
// one in flight).  Both phases run in packed f32x2 arithmetic: a face's
// pressure difference is a (dp, dp) pair, the selected upwind mobilities a
// (M_w, M_n) pair, the out - in term of an axis one multiply and one fused
// multiply-add; on the vertical axis the phases' gravity terms are one pair
// (g rho_p / hy at the centre, minus the reference profile's step, per row).
// The three axis terms are Kahan-summed per phase.  The FP64 Newton takes the
// densities from the row's reference densities plus the stored pressure
// deviation, and its reciprocal from the hardware double-precision estimate
// refined by one Newton-Raphson step, with or without diagnostics, so a step
// with diagnostics gives the same state as one without.  The plane loop
// is unrolled by two so the register roles of consecutive planes swap
// without copies.  The rows' constant pairs are read from shared memory where
// they are used, which leaves the registers to the four cells.
constexpr int RC_NRAW = 3;  // raw planes: the centre (k - 1, its s and m), k (derived), k + 1 (in flight)
constexpr int RC_NDER = 2;  // derived planes: k - 1 (read), k (written)
template <int TYT>
struct SmemRC {
  using TL = Tile<TYT>;
  RawStage<TL::RAWN> raw[RC_NRAW];
  ulonglong2 der[RC_NDER][TL::WCELLS];
  uint64_t bar[RC_NRAW];
  float4 rowF[TL::WY];
  float2 rowAR[TL::WY];
  float4 rowG[TL::WY];
  double2 rowR[TL::WY];
  double red[TL::NW][DIAG_STRIDE];
  int w_sh;
};

template <int TYT, bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
__global__ void __launch_bounds__(Tile<TYT>::NT, Tile<TYT>::MINB)
    step2_fp32c_tma_kernel(const __grid_constant__ PhysF f, const InstT* __restrict__ insts,
                          const int4* __restrict__ items, int nitems, int parity, unsigned int* __restrict__ counters,
                          double* __restrict__ diag_partials, double* __restrict__ diag_out,
                          double* __restrict__ diag_host) {
  using TL = Tile<TYT>;
  constexpr int WY = TL::WY, NHALO = TL::NHALO, BYW = TL::BYW, RC_R = TL::R, RC_TY = TL::NW, RC_NT = TL::NT;
  static_assert(NHALO <= RC_NT - 32, "a warp without halo work issues the copies");
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  SmemRC<TYT>& sm = *reinterpret_cast<SmemRC<TYT>*>(smem_bytes);
  constexpr int ISS = RC_NT - 32;  // issuer: the first thread of the last warp, which derives no halo cells

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + TX * ty;
  if (tid == ISS) {
    for (int q = 0; q < RC_NRAW; q++) mbar_init(&sm.bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;
  uint32_t armed = 0;
  bool stopped = false;

  const int own0 = (RC_R * ty + 1) * WX + (tx + 1);   // window index of the segment's first cell
  const int raw0 = (RC_R * ty + 1) * BXW + (tx + 1);
  int halo_slot = -1, halo_raw = 0, halo_row = 0;
  if (tid < NHALO) {
    // Halo cells of the 7-point stencil (the window's corners are never
    // read): the row above the tile, the row below, the left column, the
    // right column.
    int hx, hy;
    if (tid < TX) hx = tid + 1, hy = 0;
    else if (tid < 2 * TX) hx = tid - TX + 1, hy = WY - 1;
    else if (tid < 2 * TX + TYT) hx = 0, hy = tid - 2 * TX + 1;
    else hx = WX - 1, hy = tid - 2 * TX - TYT + 1;
    halo_slot = hy * WX + hx;
    halo_raw = hy * BXW + hx;
    halo_row = hy;
  }
  const f32x2 CR = pack2(f.cw_mu, f.cn_mu);
  const f32x2 CG = pack2(f.g_mu_w * f.cw_mu, f.g_mu_n * f.cn_mu);
  const f32x2 HX2 = pack2(f.inv_hx2, f.inv_hx2), HY2 = pack2(f.inv_hy2, f.inv_hy2), HZ2 = pack2(f.inv_hz2, f.inv_hz2);

  double acc_w = 0., acc_n = 0., nonfinite = 0.;
  float rmax = 0.f;
  const float iro0w_f = DIAG ? (float)(1. / f.ro0_w) : 0.f, iro0n_f = DIAG ? (float)(1. / f.ro0_n) : 0.f;
  const float aw_ro0w_f = DIAG ? (float)(f.aw / f.ro0_w) : 0.f, bn_ro0n_f = DIAG ? (float)(f.bn / f.ro0_n) : 0.f;
  // counters[parity]: this launch's work items; counters[2 + parity]: its
  // CTAs that have finished.  The launch before this one used the other
  // parity's pair and has completed once griddepcontrol.wait returns, so
  // this launch rearms them for the next.
  // The first item of a CTA is its own index, the others come from the
  // counter.  The work list and the instance records are written by the host
  // only, so the first item's are read before waiting for the previous
  // kernel; everything a kernel writes (state, media, row tables, counters)
  // is touched after the wait.
  unsigned int* counter = counters + parity;
  bool waited = false;
  auto wait_previous = [&]() {
    grid_dependency_wait();
    waited = true;
    if (blockIdx.x == 0 && tid == 0) {
      counters[parity ^ 1] = 0u;
      counters[2 + (parity ^ 1)] = 0u;
    }
  };
  int w = blockIdx.x;

  for (;;) {
    if (w >= nitems) {
      if (!waited) wait_previous();
      asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
      break;
    }
    const int4 it = items[w];
    const InstT* __restrict__ I = insts + it.x;
    const int nx = I->nx, ny = I->ny;
    const int sy32 = (int)I->sy, sz32 = (int)I->sz;
    const float c1s = I->c1_f * f.inv_one_m_swr;  // S_e = c1s - s / (1 - S_wr)
    const float dt_f = I->dt_f;
    const double S_ref = I->S_ref;
    const double aw1 = f.aw * (1. - S_ref), bnS = f.bn * S_ref;  // J11, J21 at s = 0
    const Step2FArgs& A = I->a[parity];
    float* __restrict__ p_out = A.p_out;
    float* __restrict__ s_out = A.s_out;
    unsigned int* __restrict__ err = A.err;
    if (!waited) wait_previous();
    const int tile = it.y;  // it.z, it.w: first centre plane, last plane loaded (centres it.z .. it.w - 1)
    const int ti = tile % I->tiles_x, tj = tile / I->tiles_x;
    const int i0 = 1 + ti * TX, j0 = 1 + tj * TYT;
    const int x0 = i0 - 1;
    const int i = i0 + tx, jS = j0 + RC_R * ty;  // the segment's first row
    unsigned active = 0;
#pragma unroll
    for (int r = 0; r < RC_R; r++)
      if (i <= nx - 2 && jS + r <= ny - 2) active |= 1u << r;
    const int l0 = i + jS * sy32;
    bool bad = false;
    float chk = 0.f;  // sum of |p| + |s| of the written cells (non-diagnostic steps)
    const int kb = PLANAR ? 0 : it.z;
    const int ke = PLANAR ? 0 : it.w;
    const int pb = PLANAR ? 0 : kb - 1;
    const uint32_t stage_bytes = (UNIK ? 3u : 4u) * (uint32_t)(BXW * BYW * sizeof(float)) + I->test_tx_extra;

    if (tid < WY) {
      const int gj = min(j0 - 1 + tid, ny - 1);
      const double prel = I->Pref[gj] - f.P_atm;
      sm.rowF[tid] = I->rowF[gj];
      sm.rowR[tid] = make_double2(fma(f.aw, prel, f.ro0_w), fma(f.bn, prel, f.ro0_n));
    }
    auto issue = [&](int q, int pl) {
      mbar_expect_tx(&sm.bar[q], stage_bytes);
      armed |= 1u << q;
      tma_load_3d(sm.raw[q].p, &I->map_p[parity], x0, j0 - 1, pl, &sm.bar[q]);
      tma_load_3d(sm.raw[q].s, &I->map_s[parity], x0, j0 - 1, pl, &sm.bar[q]);
      if (!UNIK) tma_load_3d(sm.raw[q].K, &I->map_K, x0, j0 - 1, pl, &sm.bar[q]);
      tma_load_3d(sm.raw[q].m, &I->map_m, x0, j0 - 1, pl, &sm.bar[q]);
    };
    if (tid == ISS)
      for (int q = 0; q < RC_NRAW && pb + q <= ke; q++) issue(q, pb + q);
    int qs = 0;  // raw stage of the plane being derived
    __syncthreads();
    // Row pairs of the window's rows (the own rows 1 .. TYT are used): the
    // reference densities over mu, and the vertical gravity terms of the
    // faces below and above.
    if (tid >= 1 && tid < WY) {
      const float4 rw = sm.rowF[tid];
      const float dn = sm.rowF[tid - 1].z;
      const float gw = f.g_mu_w * rw.x, gn = f.g_mu_n * rw.y;
      sm.rowAR[tid] = make_float2(rw.x, rw.y);
      sm.rowG[tid] = make_float4(gw - dn, gn - dn, gw - rw.z, gn - rw.z);
    }
    __syncthreads();
    auto AR = [&](int r) { const float2 v = sm.rowAR[RC_R * ty + 1 + r]; return pack2(v.x, v.y); };
    auto G1 = [&](int r) { const float4 v = sm.rowG[RC_R * ty + 1 + r]; return pack2(v.x, v.y); };
    auto G2 = [&](int r) { const float4 v = sm.rowG[RC_R * ty + 1 + r]; return pack2(v.z, v.w); };

    auto derive_cell = [&](f32x2 ARr, float p, float sv, float K) -> ulonglong2 {
      const float S_e = fmaf(-sv, f.inv_one_m_swr, c1s);
      const float e2 = S_e * S_e;
      const float om = 1.f - S_e;
      const float kw = e2 * e2;
      const float kn = om * om * (1.f - e2);
      const f32x2 PP = pack2(p, p);
      const f32x2 MM = mul2(pack2(K * kw, K * kn), fma2(CR, PP, ARr));
      return make_ulonglong2(PP, MM);
    };
    auto xaxis = [&](ulonglong2 c, ulonglong2 a, ulonglong2 b) -> f32x2 {
      f32x2 X2 = sub2(c.x, b.x), N1 = sub2(c.x, a.x);
      if (!UNITH) {
        X2 = mul2(X2, HX2);
        N1 = mul2(N1, HX2);
      }
      float x2, n1, t;
      unpack2(X2, x2, t);
      unpack2(N1, n1, t);
      const f32x2 S2 = x2 > 0.f ? c.y : b.y;
      const f32x2 S1 = n1 < 0.f ? a.y : c.y;
      return fma2(N1, S1, mul2(X2, S2));
    };
    auto zflux = [&](ulonglong2 c, ulonglong2 b) -> f32x2 {
      f32x2 X2 = sub2(c.x, b.x);
      if (!UNITH) X2 = mul2(X2, HZ2);
      float x2, t;
      unpack2(X2, x2, t);
      return mul2(X2, x2 > 0.f ? c.y : b.y);
    };
    auto yaxis = [&](ulonglong2 c, ulonglong2 ya, ulonglong2 yb, f32x2 g1, f32x2 g2) -> f32x2 {
      f32x2 E2 = sub2(c.x, yb.x), E1 = sub2(c.x, ya.x);
      if (!UNITH) {
        E2 = mul2(E2, HY2);
        E1 = mul2(E1, HY2);
      }
      const f32x2 Y2 = add2(E2, fma2(CG, c.x, g2));
      const f32x2 N1 = sub2(E1, fma2(CG, c.x, g1));
      float y2w, y2n, n1w, n1n, cw, cn, bw, bn_, aw_, an_;
      unpack2(Y2, y2w, y2n);
      unpack2(N1, n1w, n1n);
      unpack2(c.y, cw, cn);
      unpack2(yb.y, bw, bn_);
      unpack2(ya.y, aw_, an_);
      const f32x2 S2 = pack2(y2w > 0.f ? cw : bw, y2n > 0.f ? cn : bn_);
      const f32x2 S1 = pack2(n1w < 0.f ? aw_ : cw, n1n < 0.f ? an_ : cn);
      return fma2(N1, S1, mul2(Y2, S2));
    };
    // The Newton recovery of one cell from its flux difference pair D2.
    auto finish = [&](ulonglong2 c, f32x2 D2, int r, float sc, float mc, int l, bool act) {
      float pc, t0;
      unpack2(c.x, pc, t0);
      const float dtm = __fdividef(dt_f, mc);
      float Awf, Anf;
      unpack2(mul2(pack2(-dtm, -dtm), D2), Awf, Anf);
      const double Aw = (double)Awf, An = (double)Anf;
      const double pd = (double)pc, sd = (double)sc;
      const double2 rr = sm.rowR[RC_R * ty + 1 + r];
      const double rw = fma(f.aw, pd, rr.x);
      const double rn = fma(f.bn, pd, rr.y);
      const double J11 = fma(-f.aw, sd, aw1), J21 = fma(f.bn, sd, bnS);
      const double det = fma(J11, rn, rw * J21);
      double inv;
      asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(inv) : "d"(det));
      inv = fma(inv, fma(-det, inv, 1.), inv);
      const double dP = fma(rn, Aw, rw * An) * inv;
      const double dS = fma(J11, An, -(J21 * Aw)) * inv;
      const float pn = (float)(pd + dP);
      const float snew = (float)(sd + dS);
      if (act) {
        st_global(p_out + l, pn);
        st_global(s_out + l, snew);
      }
      if (!DIAG) {
        if (act) chk += fabsf(pn) + fabsf(snew);  // not finite (or beyond FLT_MAX) once any term is
      } else {
        // Diagnostics of the written cells: the phase masses of the new state
        // in FP64, at the unrounded new (P, S), within an FP32 rounding of
        // the stored values; the Newton residual; the non-finite count.
        if (act) {
          const bool fin = fabsf(pn) + fabsf(snew) <= 3.0e38f;
          bad |= !fin;
          const double md = (double)mc;
          const double P1 = pd + dP;
          const double mS1 = md * ((S_ref + sd) + dS);
          acc_w = fma(md - mS1, fma(f.aw, P1, rr.x), acc_w);
          acc_n = fma(mS1, fma(f.bn, P1, rr.y), acc_n);
          const float e = (float)fma(det, inv, -1.);
          const float q = (float)(dP * dS);
          const float F1 = fmaf(Awf * iro0w_f, e, -aw_ro0w_f * q);
          const float F2 = fmaf(Anf * iro0n_f, e, bn_ro0n_f * q);
          const float rf = fmaxf(fabsf(F1), fabsf(F2));
          if (!(rf <= rmax)) rmax = rf;
          if (!fin) nonfinite += 1.;
        }
      }
    };

    // Derived cells of two consecutive planes in registers: planes pb, pb + 2,
    // ... in X0, the others in X1 (the loop is unrolled by two, so the
    // centre and next-plane roles swap without copies).
    ulonglong2 X0[RC_R], X1[RC_R];
    f32x2 Zin[RC_R];                     // -z inflow pairs of the centre cells
    auto plane = [&](auto T, int pl) -> bool {
      constexpr int t = decltype(T)::value;  // (pl - pb) mod 2: plane pl's derived slot
      ulonglong2(&N)[RC_R] = t ? X1 : X0;
      ulonglong2(&C)[RC_R] = t ? X0 : X1;
      ulonglong2* const Dw = sm.der[t];      // plane pl
      ulonglong2* const Dr = sm.der[t ^ 1];  // plane pl - 1
      const int qc = qs == 0 ? RC_NRAW - 1 : qs - 1;  // raw stage of plane pl - 1
      const bool landed = mbar_wait_bounded(&sm.bar[qs], (phase >> qs) & 1u);
      if (landed) {
        phase ^= (1u << qs);
        armed &= ~(1u << qs);
      }
      const auto& R = sm.raw[qs];
      const auto& RC = sm.raw[qc];
      {
#pragma unroll
        for (int r = 0; r < RC_R; r++) {
          const int ri = raw0 + r * BXW;
          N[r] = derive_cell(AR(r), R.p[ri], R.s[ri], UNIK ? f.K0 : R.K[ri]);
          Dw[own0 + r * WX] = N[r];
        }
        if (halo_slot >= 0) {
          const float4 rh = sm.rowF[halo_row];
          Dw[halo_slot] = derive_cell(pack2(rh.x, rh.y), R.p[halo_raw], R.s[halo_raw], UNIK ? f.K0 : R.K[halo_raw]);
        }
      }
      // The update of the centre plane pl - 1 before the barrier: its slot
      // was written before the previous barrier, this plane's own cells are
      // in registers, so the derive and the update overlap.  A thread whose
      // wait ran out stores nothing.
      if (!PLANAR) {
        if (pl == pb + 1) {
#pragma unroll
          for (int r = 0; r < RC_R; r++) Zin[r] = zflux(C[r], N[r]);  // inflow of plane kb through its -z face
        } else if (pl >= pb + 2) {
          // x and segment-end neighbours from the centre plane's slot, the
          // rest from registers, s and m from its raw stage.
          const int lk = l0 + (pl - 1) * sz32;
#pragma unroll
          for (int r = 0; r < RC_R; r++) {
            const int o = own0 + r * WX;
            const ulonglong2 c = C[r];
            const ulonglong2 ya = r == 0 ? Dr[o - WX] : C[r - 1];
            const ulonglong2 yb = r == RC_R - 1 ? Dr[o + WX] : C[r + 1];
            Kahan2 k(xaxis(c, Dr[o - 1], Dr[o + 1]), yaxis(c, ya, yb, G1(r), G2(r)));
            const f32x2 out = zflux(c, N[r]);
            k.add(sub2(out, Zin[r]));
            Zin[r] = out;
            finish(c, k.sum(), r, RC.s[raw0 + r * BXW], RC.m[raw0 + r * BXW], lk + r * sy32,
                   landed && ((active >> r) & 1u));
          }
        }
      }
      if (__syncthreads_or(!landed)) {
        if (tid == ISS) {
          atomicOr(err, 2u);
          for (int qq = 0; qq < RC_NRAW; qq++)
            if (armed & (1u << qq)) mbar_wait_bounded(&sm.bar[qq], (phase >> qq) & 1u);
        }
        __syncthreads();
        return true;
      }
      // Plane pl - 1's stage is free once every thread has updated it.
      if (tid == ISS && pl > pb && pl + RC_NRAW - 1 <= ke) {
        fence_proxy_async();
        issue(qc, pl + RC_NRAW - 1);
      }
      if (PLANAR) {
#pragma unroll
        for (int r = 0; r < RC_R; r++) {
          const int o = own0 + r * WX;
          const ulonglong2 c = N[r];
          const ulonglong2 ya = r == 0 ? Dw[o - WX] : N[r - 1];
          const ulonglong2 yb = r == RC_R - 1 ? Dw[o + WX] : N[r + 1];
          Kahan2 k(xaxis(c, Dw[o - 1], Dw[o + 1]), yaxis(c, ya, yb, G1(r), G2(r)));
          finish(c, k.sum(), r, R.s[raw0 + r * BXW], R.m[raw0 + r * BXW], l0 + r * sy32, (active >> r) & 1u);
        }
      }
      qs = qs == RC_NRAW - 1 ? 0 : qs + 1;
      return false;
    };
    for (int base = pb; base <= ke; base += 2) {
      if (plane(std::integral_constant<int, 0>{}, base)) { stopped = true; break; }
      if (base + 1 > ke) break;
      if (plane(std::integral_constant<int, 1>{}, base + 1)) { stopped = true; break; }
    }
    if (stopped) break;
    if (!DIAG) bad = !(chk <= 3.0e38f);
    if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) atomicOr(err, 1u);
    if (tid == 0) sm.w_sh = (int)gridDim.x + (int)atomicAdd(counter, 1u);
    __syncthreads();  // the next item's loads reuse the stages, slots and rows
    w = sm.w_sh;
  }

  if (DIAG) {
    // Per-CTA partials, then the last CTA to finish reduces them in index
    // order (deterministic) into diag_out.
    double(*red)[DIAG_STRIDE] = sm.red;
    const int lane = tid & 31, wid = tid >> 5;
    const double s0 = warp_sum(acc_w), s1 = warp_sum(acc_n), rr = warp_max((double)rmax), nf = warp_sum(nonfinite);
    if (lane == 0) {
      red[wid][0] = s0;
      red[wid][1] = s1;
      red[wid][2] = rr;
      red[wid][3] = nf;
    }
    __syncthreads();
    if (tid == 0) {
      double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
      for (int qq = 0; qq < RC_TY; qq++) {
        t0 += red[qq][0];
        t1 += red[qq][1];
        t2 = fmax(t2, red[qq][2]);
        t3 += red[qq][3];
      }
      double* out = diag_partials + (size_t)DIAG_STRIDE * blockIdx.x;
      out[0] = t0 * f.vol;
      out[1] = t1 * f.vol;
      out[2] = 0.;
      out[3] = t2;
      out[4] = t3;
      __threadfence();
      sm.w_sh = (atomicAdd(counters + 2 + parity, 1u) == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (sm.w_sh) {
      __threadfence();
      const int nparts = gridDim.x;
      const int per = (nparts + RC_NT - 1) / RC_NT;
      const int b0 = tid * per, b1 = min(nparts, b0 + per);
      double v[DIAG_STRIDE] = {0., 0., 0., 0., 0.};
      for (int b = b0; b < b1; b++) {
        const volatile double* q = diag_partials + (size_t)DIAG_STRIDE * b;
        v[0] += q[0];
        v[1] += q[1];
        v[2] += q[2];
        v[3] = fmax(v[3], q[3]);
        v[4] += q[4];
      }
      for (int o = 1; o < 32; o <<= 1) {
        double t[DIAG_STRIDE];
#pragma unroll
        for (int e = 0; e < DIAG_STRIDE; e++) t[e] = __shfl_down_sync(0xffffffffu, v[e], o);
        if ((lane & (2 * o - 1)) == 0) {
          v[0] += t[0];
          v[1] += t[1];
          v[2] += t[2];
          v[3] = fmax(v[3], t[3]);
          v[4] += t[4];
        }
      }
      if (lane == 0)
        for (int e = 0; e < DIAG_STRIDE; e++) red[wid][e] = v[e];
      __syncthreads();
      if (tid == 0) {
        double t[DIAG_STRIDE] = {0., 0., 0., 0., 0.};
        for (int qq = 0; qq < RC_TY; qq++) {
          t[0] += red[qq][0];
          t[1] += red[qq][1];
          t[2] += red[qq][2];
          t[3] = fmax(t[3], red[qq][3]);
          t[4] += red[qq][4];
        }
        for (int e = 0; e < DIAG_STRIDE; e++) diag_out[e] = t[e];
        if (diag_host) {
          // Published into mapped pinned host memory as well: the host reads
          // it after an event recorded behind this step, with no further launch.
          for (int e = 0; e < DIAG_STRIDE; e++) diag_host[e] = t[e];
          __threadfence_system();
        }
      }
    }
  }
}

// Boundary cells after the sweep (boundary_conditions, two-phase.cpp:59-111):
// each takes the new state of its basic-coordinate cell (cpu.cpp:107-141),
// an interior cell; the top row holds P_atm (+ the top offset) and, inside
// the injection window, S_n_gr; the bottom row adds the weight
// (rho_n S_n + rho_w (1 - S_n)) m g hy of the basic cell with its new S_n and
// start-of-step densities (Border_P, main.cpp:255-267).  One thread per
// boundary cell; items are (instance, first cell) blocks of BOUND_BLOCK.  A
// z-slab's halo planes (its planes 0 and nz - 1 when a neighbour owns them)
// are left to the halo exchange.
__global__ void __launch_bounds__(BOUND_BLOCK)
    boundary_fp32c_kernel(const __grid_constant__ PhysF f, const InstT* __restrict__ insts,
                          const int2* __restrict__ bitems, int parity) {
  // The work lists and instance records are not written by the sweep: the
  // cell's position is worked out before waiting for the sweep's values, and
  // the next step's sweep may be scheduled as soon as every block is here
  // (it waits for this kernel's completion before reading the state).
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
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
  if ((k == 0 && I->halo_lo) || (k == nz - 1 && I->halo_hi)) return;
  const int i1 = min(max(i, 1), nx - 2), j1 = min(max(j, 1), ny - 2);
  const int k1 = nz == 1 ? 0 : min(max(k, 1), nz - 2);
  const long long sy = I->sy, sz = I->sz;
  const long long lb = i + j * sy + (long long)k * sz, l1 = i1 + j1 * sy + (long long)k1 * sz;
  const Step2FArgs& A = I->a[parity];
  float* __restrict__ const s_out = A.s_out;
  float* __restrict__ const p_out = A.p_out;
  grid_dependency_wait();  // the sweep's interior values
  const float s1 = s_out[l1];
  float sb = s1;
  if ((j == 0) && (I->source > 0) && in_window(I, i, k)) sb = I->sgr_dev_f;
  float pb;
  if ((j != 0) && (j != ny - 1)) {
    pb = p_out[l1];
  } else if (j == 0) {
    pb = (float)((f.P_atm + f.P_top) - I->Pref[0]);
  } else {
    const double prel = I->Pref[j1] - f.P_atm;
    const double pr = prel + (double)A.p_in[l1];  // start-of-step pressure of the basic cell
    const double rw = fma(f.aw, pr, f.ro0_w), rn = fma(f.bn, pr, f.ro0_n);
    const double Snew = I->S_ref + (double)s1;
    const double Pnew = (prel + f.P_atm) + (double)p_out[l1];
    const double ro_g_dy = (rn * Snew + rw * (1 - Snew)) * (double)A.m[l1] * f.g * f.hy;
    pb = (float)(Pnew + ro_g_dy - I->Pref[ny - 1]);
  }
  s_out[lb] = sb;
  p_out[lb] = pb;
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
template <int TYT, bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
cudaError_t prepare_t() {
  static unsigned long long done = 0;  // bit d: set on device d
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(step2_fp32c_tma_kernel<TYT, UNIK, DIAG, PLANAR, UNITH>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemRC<TYT>));
  if (e == cudaSuccess) __atomic_fetch_or(&done, bit, __ATOMIC_ACQ_REL);
  return e;
}

template <int TYT, bool UNIK, bool DIAG, bool PLANAR, bool UNITH>
cudaError_t launch_t(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                     unsigned int* counter, double* diag_partials, int grid, cudaStream_t s, double* diag_out,
                     double* diag_host) {
  cudaError_t e = prepare_t<TYT, UNIK, DIAG, PLANAR, UNITH>();
  if (e != cudaSuccess) return e;
  return launch_dependent(step2_fp32c_tma_kernel<TYT, UNIK, DIAG, PLANAR, UNITH>, dim3(grid),
                          dim3(TX, Tile<TYT>::NW), sizeof(SmemRC<TYT>), s, f, insts, items, nitems, parity, counter,
                          diag_partials, diag_out, diag_host);
}

template <int TYT, bool UNIK, bool DIAG, bool PLANAR>
cudaError_t launch_h(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                     unsigned int* counter, double* diag_partials, int grid, cudaStream_t s, double* diag_out,
                     double* diag_host) {
  // Unit spacing (the workloads' h = 1 m): forces are plain differences.
  const bool unith = f.inv_hx2 == 1.f && f.inv_hy2 == 1.f && f.inv_hz2 == 1.f;
  return unith ? launch_t<TYT, UNIK, DIAG, PLANAR, true>(f, insts, items, nitems, parity, counter, diag_partials,
                                                          grid, s, diag_out, diag_host)
               : launch_t<TYT, UNIK, DIAG, PLANAR, false>(f, insts, items, nitems, parity, counter, diag_partials,
                                                           grid, s, diag_out, diag_host);
}

template <int TYT>
cudaError_t launch_shape(bool unik, bool planar, const PhysF& f, const InstT* insts, const int4* items, int nitems,
                         int parity, unsigned int* counter, double* diag_partials, int grid, cudaStream_t s,
                         double* diag_out, double* diag_host) {
  const bool d = diag_partials != nullptr;
#define CAPAZ_LH(U, D, P) launch_h<TYT, U, D, P>(f, insts, items, nitems, parity, counter, d ? diag_partials : nullptr, \
                                                 grid, s, d ? diag_out : nullptr, d ? diag_host : nullptr)
  if (unik) {
    if (d) return planar ? CAPAZ_LH(true, true, true) : CAPAZ_LH(true, true, false);
    return planar ? CAPAZ_LH(true, false, true) : CAPAZ_LH(true, false, false);
  }
  if (d) return planar ? CAPAZ_LH(false, true, true) : CAPAZ_LH(false, true, false);
  return planar ? CAPAZ_LH(false, false, true) : CAPAZ_LH(false, false, false);
#undef CAPAZ_LH
}

template <int TYT>
int grid_shape(int device, bool unik) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int per = 0;
  if (unik) {
    prepare_t<TYT, true, true, false, false>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_tma_kernel<TYT, true, true, false, false>,
                                                  Tile<TYT>::NT, sizeof(SmemRC<TYT>));
  } else {
    prepare_t<TYT, false, true, false, false>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step2_fp32c_tma_kernel<TYT, false, true, false, false>,
                                                  Tile<TYT>::NT, sizeof(SmemRC<TYT>));
  }
  if (per < 1) per = 1;
  return sms * per;
}

}  // namespace

bool tma_tile_supported(int tile_y) { return tile_y == 16 || tile_y == 32; }

cudaError_t launch_step2_fp32c_tma(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                                   bool unik, bool planar, unsigned int* counters, double* diag_partials, int grid,
                                   cudaStream_t s, double* diag_out, int tile_y, double* diag_host) {
  // counters[0..3] are zero at allocation; every launch rearms the pair of
  // the other parity (see the kernel).
  if (tile_y == 32)
    return launch_shape<32>(unik, planar, f, insts, items, nitems, parity, counters, diag_partials, grid, s, diag_out,
                            diag_host);
  if (tile_y == 16)
    return launch_shape<16>(unik, planar, f, insts, items, nitems, parity, counters, diag_partials, grid, s, diag_out,
                            diag_host);
  return cudaErrorInvalidValue;
}

cudaError_t launch_boundary_fp32c(const PhysF& f, const InstT* insts, const int2* bitems, int nbitems, int parity,
                                  cudaStream_t s) {
  return launch_dependent(boundary_fp32c_kernel, dim3(nbitems), dim3(BOUND_BLOCK), 0, s, f, insts, bitems, parity);
}

int step2_fp32c_tma_grid(int device, bool unik, int tile_y) {
  return tile_y == 32 ? grid_shape<32>(device, unik) : grid_shape<16>(device, unik);
}

// Builds the 3-D tensor map of one float32 field of an nx x ny x nz grid
// with the kernel's 36 x (tile_y + 2) x 1 box.  nx must be a multiple of 4
// (row pitch a multiple of 16 bytes).
int encode_field_map(CUtensorMap* map, const float* base, int nx, int ny, int nz, int tile_y) {
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
  const cuuint32_t box[3] = {(cuuint32_t)BXW, (cuuint32_t)(tile_y + 2), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

}  // namespace capaz
