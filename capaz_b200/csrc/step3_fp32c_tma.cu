// Three-phase precision-form step with TMA-staged z-planes (sm_100a).
//
// The model of step3_fp32c.cu (FP32 deviation storage of P_w, S_w, S_n; FP32
// stencil with Kahan-compensated per-phase divergence; one FP64 Newton step
// on the bilinear increment equations with the 3x3 Jacobian solved by
// Cramer's rule), laid out as the two-phase TMA sweep for grids whose x
// extent is a multiple of 4:
//   - persistent CTAs of 256 threads take (tile, z-chunk) items from a
//     counter; a tile is 32 x 16 interior cells and each thread owns two
//     cells of a column (rows ty and ty + 8);
//   - one thread of a warp without halo work streams the raw window of each
//     plane (P_w, S_w, S_n, K, m deviations; a 36 x 18 box at x = 32*ti)
//     into a three-stage ring with cp.async.bulk.tensor (3-D tensor maps in
//     the kernel's parameters, no multicast) completing on mbarriers with
//     bounded waits;
//   - every thread derives its cells (three warps one halo cell more) into a
//     three-slot ring: (p_w, M_w, M_n, M_g) with M_p = K k_p rho_p / mu_p, and
//     (p_n, p_g), which differ from p_w only on the grid's top and bottom
//     rows (three-phase.cpp:345-427 with zero capillary pressures) and are
//     read there from the stored state;
//   - the update of the plane below, in the same barrier interval as the
//     derive: it reads the centre and its x and y neighbours from the centre
//     plane's slot (complete since the previous barrier), its z neighbours'
//     own cells from the slots of the planes around it, and the centre's
//     s and m from its raw stage, which is refilled (with the plane two ahead)
//     only after the barrier that ends the update: one barrier per plane;
//   - boundary cells are written after the sweep by a kernel over the
//     boundary shell (Border_S, Border_P), from the new state of each cell's
//     basic-coordinate cell; that kernel also rearms the work counter.
// The relative permeabilities are the reference CPU ones (three-phase.cpp:
// 146-186) in FP32, by products and square roots when A = 2.
#include <cuda.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "capaz_internal.h"
#include "phys3f.cuh"

namespace capaz {
namespace {

constexpr int Y3 = 8;                     // thread rows; each owns rows ty and ty + Y3 of the tile
constexpr int NT3 = TX * Y3;              // threads per CTA
constexpr int T3 = 2 * Y3;                // tile rows
constexpr int WX3 = TX + 2, WY3 = T3 + 2, WC3 = WX3 * WY3;
constexpr int BX3 = 36;                   // TMA box width (floats): 144 bytes
constexpr int RAW3 = (BX3 * WY3 + 31) / 32 * 32;
constexpr int NST3 = 3;                   // raw stages and derived slots
constexpr int NH3 = 2 * TX + 2 * T3;      // halo cells (the window's corners are never read)
constexpr int ISS3 = NT3 - 32;            // issuer: first thread of the last warp (no halo work)
static_assert(NH3 <= ISS3, "the issuing warp must not derive halo cells");
constexpr long long WAIT3 = 2000000000ll;  // bounded waits give up after ~1 s of SM clocks

struct alignas(128) Raw3T {
  float pw[RAW3], sw[RAW3], sn[RAW3], K[RAW3], m[RAW3];
};
struct Smem3T {
  Raw3T raw[NST3];
  float4 der[NST3][WC3];  // (p_w, M_w, M_n, M_g)
  float2 png[NST3][WC3];  // (p_n, p_g)
  uint64_t bar[NST3];
  float4 rowF[WY3];       // rho_w, rho_n, rho_g at P_ref(j); P_ref(j+1) - P_ref(j)
  double rowPref[WY3];
  double red[NT3 / 32][5];
  int w_sh;
};
constexpr size_t kSmem3T = sizeof(Smem3T);

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t par) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(par)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t par) {
  if (bar_try(b, par)) return true;
  const long long t0 = clock64();
  while (!bar_try(b, par))
    if (clock64() - t0 > WAIT3) return false;
  return true;
}
__device__ __forceinline__ void tma3(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(su32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(su32(b))
      : "memory");
}
__device__ __forceinline__ float face3(float x1, float x2, float Mc, float Mm, float Mp) {
  return x2 * (x2 > 0.f ? Mc : Mp) - x1 * (x1 > 0.f ? Mm : Mc);
}
__device__ __forceinline__ double wsum3(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax3(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool UNIK, bool DIAG, bool PLANAR, bool A2, bool UNITH>
__global__ void __launch_bounds__(NT3, 2)
    step3_fp32c_tma_kernel(const __grid_constant__ Step3FConst c, const __grid_constant__ Step3TArgs a) {
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  Smem3T& sm = *reinterpret_cast<Smem3T*>(smem_bytes);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + TX * ty;
  if (tid == ISS3) {
    for (int q = 0; q < NST3; q++) bar_init(&sm.bar[q]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0, armed = 0;
  bool stopped = false;

  const int ownA = (ty + 1) * WX3 + (tx + 1), ownB = ownA + Y3 * WX3;
  const int rawA = (ty + 1) * BX3 + (tx + 1), rawB = rawA + Y3 * BX3;
  int hslot = -1, hraw = 0, hx = 0, hy = 0;
  if (tid < NH3) {
    if (tid < TX) hx = tid + 1, hy = 0;
    else if (tid < 2 * TX) hx = tid - TX + 1, hy = WY3 - 1;
    else if (tid < 2 * TX + T3) hx = 0, hy = tid - 2 * TX + 1;
    else hx = WX3 - 1, hy = tid - 2 * TX - T3 + 1;
    hslot = hy * WX3 + hx;
    hraw = hy * BX3 + hx;
  }
  const int ntiles = c.tiles_x * c.tiles_y;
  const int nitems = ntiles * c.nzchunks;
  const uint32_t stage_bytes = (UNIK ? 4u : 5u) * (uint32_t)(BX3 * WY3 * sizeof(float));
  double acc[3] = {0., 0., 0.}, rmax = 0., nonfinite = 0.;
  // Launched with programmatic stream serialisation: the previous kernel
  // (the boundary kernel, which rearms the counter) has completed and its
  // writes are visible once this returns.
  asm volatile("griddepcontrol.wait;" ::: "memory");

  for (;;) {
    if (tid == 0) sm.w_sh = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int w = sm.w_sh;
    if (w >= nitems) {
      asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
      break;
    }
    const int tile = w % ntiles, zc = w / ntiles;
    const int ti = tile % c.tiles_x, tj = tile / c.tiles_x;
    const int i0 = 1 + ti * TX, j0 = 1 + tj * T3, x0 = i0 - 1;
    const int i = i0 + tx, jA = j0 + ty, jB = jA + Y3;
    const bool actA = (i <= c.nx - 2) && (jA <= c.ny - 2), actB = (i <= c.nx - 2) && (jB <= c.ny - 2);
    const int kb = PLANAR ? 0 : 1 + (int)((long long)zc * (c.nz - 2) / c.nzchunks);
    const int ke = PLANAR ? 0 : 1 + (int)((long long)(zc + 1) * (c.nz - 2) / c.nzchunks);
    const int pb = PLANAR ? 0 : kb - 1;
    bool bad = false;
    float chk = 0.f;  // sum of |p_w| + |s_w| + |s_n| of the written cells (non-diagnostic steps)
    if (tid < WY3) {
      const int gj = min(j0 - 1 + tid, c.ny - 1);
      sm.rowF[tid] = a.rowF[gj];
      sm.rowPref[tid] = a.Pref[gj];
    }
    auto issue = [&](int q, int pl) {
      bar_expect(&sm.bar[q], stage_bytes);
      armed |= 1u << q;
      tma3(sm.raw[q].pw, &a.map_pw, x0, j0 - 1, pl, &sm.bar[q]);
      tma3(sm.raw[q].sw, &a.map_sw, x0, j0 - 1, pl, &sm.bar[q]);
      tma3(sm.raw[q].sn, &a.map_sn, x0, j0 - 1, pl, &sm.bar[q]);
      if (!UNIK) tma3(sm.raw[q].K, &a.map_K, x0, j0 - 1, pl, &sm.bar[q]);
      tma3(sm.raw[q].m, &a.map_m, x0, j0 - 1, pl, &sm.bar[q]);
    };
    if (tid == ISS3)
      for (int q = 0; q < NST3 && pb + q <= ke; q++) issue(q, pb + q);
    __syncthreads();
    // Rows of the grid with their own P_n, P_g (the top and bottom boundary
    // rows): the own rows can be one only in a tile that runs past the grid.
    const bool bA = jA == c.ny - 1, bB = jB == c.ny - 1;
    const int gh_i = i0 - 1 + hx, gh_j = j0 - 1 + hy;
    const bool bH = hslot >= 0 && gh_i < c.nx && (gh_j == 0 || gh_j == c.ny - 1);

    // Derives one window cell of plane pl (raw index r, window index o,
    // window row wr) into the slot.
    auto derive = [&](const Raw3T& R, float4* D, float2* G, int r, int o, int wr, bool brow, int gi, int gj,
                      int pl) {
      const float pw = R.pw[r];
      float pn = pw, pg = pw;
      if (brow) {
        const long long l = gi + gj * c.sy + (long long)pl * c.sz;
        pn = a.p_n[l];
        pg = a.p_g[l];
      }
      const float Sw = c.S_ref_w_f + R.sw[r], Sn = c.S_ref_n_f + R.sn[r];
      const float S_w_e = (Sw - c.S_wr_f) * c.inv_den, S_n_e = (Sn - c.S_nr_f) * c.inv_den;
      float k_w, k_n, k_g;
      relperm3f<A2>(c, S_w_e, S_n_e, k_w, k_n, k_g);
      const float Kl = UNIK ? c.K0_f : R.K[r];
      const float4 rf = sm.rowF[wr];
      D[o] = make_float4(pw, Kl * k_w * fmaf(c.aw_f, pw, rf.x) * c.inv_mu_w_f,
                         Kl * k_n * fmaf(c.an_f, pn, rf.y) * c.inv_mu_n_f, Kl * k_g * fmaf(c.bg_f, pg, rf.z) * c.inv_mu_g_f);
      G[o] = make_float2(pn, pg);
    };

    // Update of one interior cell of the centre plane k (slots Dc, Dm, Dp).
    auto update = [&](const float4* Dc, const float2* Gc, const float4* Dm, const float4* Dp, int own, int wr,
                      float sw0, float sn0, float mc, long long l, bool act, int j) {
      const float4 cc = Dc[own], xa = Dc[own - 1], xb = Dc[own + 1], ya = Dc[own - WX3], yb = Dc[own + WX3];
      const float2 yaN = Gc[own - WX3], ybN = Gc[own + WX3];
      const float pc = cc.x;  // interior: p_n = p_g = p_w
      const float4 row = sm.rowF[wr];
      // Unit spacing (the workloads' h = 1 m): the 1/h^2 factors drop out.
      const float ihx = UNITH ? 1.f : c.inv_hx2_f, ihy = UNITH ? 1.f : c.inv_hy2_f, ihz = UNITH ? 1.f : c.inv_hz2_f;
      const float dn = sm.rowF[wr - 1].w * ihy, dp = row.w * ihy;
      const float x1 = (xa.x - pc) * ihx, x2 = (pc - xb.x) * ihx;
      float z1 = 0.f, z2 = 0.f;
      float4 zm, zp;
      if (!PLANAR) {
        zm = Dm[own];
        zp = Dp[own];
        z1 = (zm.x - pc) * ihz;
        z2 = (pc - zp.x) * ihz;
      }
      const float pa[3] = {ya.x, yaN.x, yaN.y}, pbv[3] = {yb.x, ybN.x, ybN.y};
      const float Mc[3] = {cc.y, cc.z, cc.w}, Ma[3] = {xa.y, xa.z, xa.w}, Mb[3] = {xb.y, xb.z, xb.w};
      const float My1[3] = {ya.y, ya.z, ya.w}, My2[3] = {yb.y, yb.z, yb.w};
      const float slope[3] = {c.aw_f, c.an_f, c.bg_f}, rho[3] = {row.x, row.y, row.z};
      float div[3];
#pragma unroll
      for (int ph = 0; ph < 3; ph++) {
        const float fx = face3(x1, x2, Mc[ph], Ma[ph], Mb[ph]);
        const float gr = c.g_inv_hy_f * fmaf(slope[ph], pc, rho[ph]);
        const float y1 = fmaf(pa[ph] - pc, ihy, -dn) + gr;
        const float y2 = fmaf(pc - pbv[ph], ihy, -dp) + gr;
        const float fy = face3(y1, y2, Mc[ph], My1[ph], My2[ph]);
        float s = fx + fy;
        float comp = (s - fx) - fy;
        if (!PLANAR) {
          const float Mzm[3] = {zm.y, zm.z, zm.w}, Mzp[3] = {zp.y, zp.z, zp.w};
          const float fz = face3(z1, z2, Mc[ph], Mzm[ph], Mzp[ph]);
          const float yk = fz - comp;
          const float t = s + yk;
          comp = (t - s) - yk;
          s = t;
        }
        div[ph] = s - comp;
      }
      // d(rho S)_p = -dt/m div F_p, then one Newton step in FP64 from the
      // stored state: the Jacobian in (dP, dS_w, dS_n), with a13 = a22 = 0
      // and a33 = a32, solved by Cramer's rule.
      const float dtm = __fdividef(c.dt_f, mc);
      const double dAw = (double)(-dtm * div[0]), dAn = (double)(-dtm * div[1]), dAg = (double)(-dtm * div[2]);
      const double Pref = sm.rowPref[wr];
      const double pw0 = (double)pc;
      const double P = Pref + pw0, prel = Pref - c.P_atm;
      const double Sw = c.S_ref_w + (double)sw0, Sn = c.S_ref_n + (double)sn0, Sg = 1. - Sw - Sn;
      const double rw = fma(c.aw, prel + pw0, c.ro0_w), rn = fma(c.an, prel + pw0, c.ro0_n);
      const double a11 = c.aw * Sw, a12 = rw;
      const double a21 = c.an * Sn, a23 = rn;
      const double a31 = c.bg * Sg, a32 = -c.bg * P;
      const double c11 = -a23 * a32, c12 = a23 * a31 - a21 * a32, c13 = a21 * a32;
      const double det = a11 * c11 + a12 * c12;
      double inv;
      asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(inv) : "d"(det));
      inv = fma(inv, fma(-det, inv, 1.), inv);  // Newton-Raphson steps on the hardware estimate
      inv = fma(inv, fma(-det, inv, 1.), inv);
      const double dP = (dAw * c11 + a12 * (a23 * dAg - dAn * a32)) * inv;
      const double dSw = (a11 * (dAn * a32 - a23 * dAg) + dAw * c12) * inv;
      const double dSn = (a12 * (dAn * a31 - a21 * dAg) + dAw * c13 - a11 * dAn * a32) * inv;
      const double Pn1 = P + dP, Swn = Sw + dSw, Snn = Sn + dSn;
      const float pwf = (float)(pw0 + dP), swf = (float)((double)sw0 + dSw), snf = (float)((double)sn0 + dSn);
      if (act) {
        a.o_pw[l] = pwf;
        a.o_sw[l] = swf;
        a.o_sn[l] = snf;
      }
      bool finite = true;
      if (DIAG) {
        finite = isfinite(Pn1) && isfinite(Swn) && isfinite(Snn);
        bad |= act && !finite;
      } else if (act) {
        chk += fabsf(pwf) + fabsf(swf) + fabsf(snf);  // not finite (or beyond FLT_MAX) once any term is
      }
      if (DIAG && act) {
        const double Sgn = 1. - Swn - Snn;
        const double rw1 = c.ro0_w * (1. + (c.beta_w) * (Pn1 - c.P_atm));
        const double rn1 = c.ro0_n * (1. + (c.beta_n) * (Pn1 - c.P_atm));
        const double rg1 = c.ro0_g * Pn1 / c.P_atm;
        const double vm = (double)mc * c.vol;
        acc[0] += vm * rw1 * Swn;
        acc[1] += vm * rn1 * Snn;
        acc[2] += vm * rg1 * Sgn;
        const double G1 = rw1 * Swn - (rw * Sw + dAw);
        const double G2 = rn1 * Snn - (rn * Sn + dAn);
        const double G3 = rg1 * Sgn - (c.ro0_g * P / c.P_atm * Sg + dAg);
        const double r = fmax(fmax(fabs(G1) / c.ro0_w, fabs(G2) / c.ro0_n), fabs(G3) / c.ro0_g);
        if (!(r <= rmax)) rmax = r;
        if (!finite) nonfinite += 1.;
      }
    };

    // Plane pl: derive into slot u, then update the centre plane pl - 1
    // (slot and raw stage uc, its s and m read there) before the barrier; the
    // stage of plane pl - 1 is refilled with plane pl + 2 after it.
    auto plane = [&](auto U, int pl) -> bool {
      constexpr int u = decltype(U)::value;
      constexpr int uc = (u + 2) % NST3, um = (u + 1) % NST3;  // planes pl - 1 and pl - 2
      const bool landed = bar_wait(&sm.bar[u], (phase >> u) & 1u);
      if (landed) {
        phase ^= 1u << u;
        armed &= ~(1u << u);
      }
      const Raw3T& R = sm.raw[u];
      float4* D = sm.der[u];
      float2* G = sm.png[u];
      derive(R, D, G, rawA, ownA, ty + 1, bA, i, jA, pl);
      derive(R, D, G, rawB, ownB, ty + Y3 + 1, bB, i, jB, pl);
      if (hslot >= 0) derive(R, D, G, hraw, hslot, hy, bH, gh_i, gh_j, pl);
      if (!PLANAR && pl >= pb + 2) {
        const Raw3T& RC = sm.raw[uc];
        const long long lk = i + (long long)(pl - 1) * c.sz;
        update(sm.der[uc], sm.png[uc], sm.der[um], D, ownA, ty + 1, RC.sw[rawA], RC.sn[rawA], RC.m[rawA],
               lk + (long long)jA * c.sy, landed && actA, jA);
        update(sm.der[uc], sm.png[uc], sm.der[um], D, ownB, ty + Y3 + 1, RC.sw[rawB], RC.sn[rawB], RC.m[rawB],
               lk + (long long)jB * c.sy, landed && actB, jB);
      }
      if (__syncthreads_or(!landed)) {
        if (tid == ISS3) {
          atomicOr(a.err, 2u);
          for (int q = 0; q < NST3; q++)
            if (armed & (1u << q)) bar_wait(&sm.bar[q], (phase >> q) & 1u);
        }
        __syncthreads();
        return true;
      }
      if (tid == ISS3 && pl > pb && pl + NST3 - 1 <= ke) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(uc, pl + NST3 - 1);
      }
      if (PLANAR) {
        update(D, G, D, D, ownA, ty + 1, R.sw[rawA], R.sn[rawA], R.m[rawA], i + (long long)jA * c.sy, actA, jA);
        update(D, G, D, D, ownB, ty + Y3 + 1, R.sw[rawB], R.sn[rawB], R.m[rawB], i + (long long)jB * c.sy, actB, jB);
      }
      return false;
    };
    for (int base = pb; base <= ke; base += NST3) {
      if (plane(std::integral_constant<int, 0>{}, base)) { stopped = true; break; }
      if (base + 1 > ke) break;
      if (plane(std::integral_constant<int, 1>{}, base + 1)) { stopped = true; break; }
      if (base + 2 > ke) break;
      if (plane(std::integral_constant<int, 2>{}, base + 2)) { stopped = true; break; }
    }
    if (stopped) break;
    if (!DIAG) bad = !(chk <= 3.0e38f);
    if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0) atomicOr(a.err, 1u);
    __syncthreads();  // the next item reuses the stages, slots and rows
  }

  if (DIAG) {
    const int lane = tid & 31, wid = tid >> 5;
    const double v[5] = {wsum3(acc[0]), wsum3(acc[1]), wsum3(acc[2]), wmax3(rmax), wsum3(nonfinite)};
    if (lane == 0)
      for (int q = 0; q < 5; q++) sm.red[wid][q] = v[q];
    __syncthreads();
    if (tid == 0) {
      double t[5] = {0, 0, 0, 0, 0};
      for (int q = 0; q < NT3 / 32; q++) {
        t[0] += sm.red[q][0];
        t[1] += sm.red[q][1];
        t[2] += sm.red[q][2];
        t[3] = fmax(t[3], sm.red[q][3]);
        t[4] += sm.red[q][4];
      }
      double* o = a.diag + (size_t)DIAG_STRIDE * blockIdx.x;
      for (int q = 0; q < 5; q++) o[q] = t[q];
    }
  }
}

// Boundary cells after the sweep (boundary_conditions, three-phase.cpp:
// 345-427): each takes the new state of its basic-coordinate cell
// (cpu.cpp:107-141), an interior cell.  Saturations are copied, except on
// the top row inside the source window (S_w_gr, S_n_gr); pressures are
// copied on the sides, and on the top and bottom rows are the basic cell's
// P extrapolated by one row of each phase's hydrostatic weight (the FP64
// step's expressions).  Block 0 rearms the sweep's work counter.
__global__ void __launch_bounds__(256) boundary3_kernel(const __grid_constant__ Step3FConst c,
                                                         const __grid_constant__ Step3TArgs a, int nbound) {
  // The next sweep may be scheduled once every block is here (it waits for
  // this kernel's completion); the cell's position is worked out before
  // waiting for the sweep's values.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int q0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (q0 >= nbound) return;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
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
  const long long lb = i + j * c.sy + (long long)k * c.sz, l1 = i1 + j1 * c.sy + (long long)k1 * c.sz;
  asm volatile("griddepcontrol.wait;" ::: "memory");  // the sweep's interior values
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.counter = 0u;
  const double Pn1 = a.Pref[j1] + (double)a.o_pw[l1];
  double sw = c.S_ref_w + (double)a.o_sw[l1], sn = c.S_ref_n + (double)a.o_sn[l1];
  if ((j == 0) && (c.source > 0) &&
      (!c.source_window || ((i >= nx / 2 - c.source) && (i <= nx / 2 + c.source) && (k >= c.win_k0) &&
                            (k <= c.win_k1)))) {
    sw = c.S_w_gr;
    sn = c.S_n_gr;
  }
  double pw, pn, pg;
  if ((j != 0) && (j != ny - 1)) {
    pw = pn = pg = Pn1;
  } else if (j == 0) {
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
  const double pr = a.Pref[j];
  a.o_sw[lb] = (float)(sw - c.S_ref_w);
  a.o_sn[lb] = (float)(sn - c.S_ref_n);
  a.o_pw[lb] = (float)(pw - pr);
  a.o_pn[lb] = (float)(pn - pr);
  a.o_pg[lb] = (float)(pg - pr);
}

// Launches with programmatic stream serialisation: the kernel may start
// while the previous kernel in the stream finishes, and waits for it with
// griddepcontrol.wait before touching what that kernel writes.
template <typename... Params, typename... Args>
cudaError_t launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
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

template <bool UNIK, bool DIAG, bool PLANAR, bool A2, bool UNITH>
cudaError_t launch_t3(const Step3FConst& c, const Step3TArgs& a, int grid, cudaStream_t s) {
  auto kern = step3_fp32c_tma_kernel<UNIK, DIAG, PLANAR, A2, UNITH>;
  static unsigned long long done = 0;  // bit d: shared memory opted in on device d
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit)) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem3T);
    if (e != cudaSuccess) return e;
    __atomic_fetch_or(&done, bit, __ATOMIC_ACQ_REL);
  }
  return launch_pdl(kern, dim3(grid), dim3(TX, Y3), kSmem3T, s, c, a);
}

template <bool UNIK, bool DIAG, bool PLANAR, bool A2>
cudaError_t launch_h3(const Step3FConst& c, const Step3TArgs& a, int grid, cudaStream_t s) {
  const bool unith = c.inv_hx2_f == 1.f && c.inv_hy2_f == 1.f && c.inv_hz2_f == 1.f;
  return unith ? launch_t3<UNIK, DIAG, PLANAR, A2, true>(c, a, grid, s)
               : launch_t3<UNIK, DIAG, PLANAR, A2, false>(c, a, grid, s);
}

template <bool UNIK, bool DIAG>
cudaError_t launch_pa(bool planar, bool a2, const Step3FConst& c, const Step3TArgs& a, int grid, cudaStream_t s) {
  if (planar) return a2 ? launch_h3<UNIK, DIAG, true, true>(c, a, grid, s) : launch_h3<UNIK, DIAG, true, false>(c, a, grid, s);
  return a2 ? launch_h3<UNIK, DIAG, false, true>(c, a, grid, s) : launch_h3<UNIK, DIAG, false, false>(c, a, grid, s);
}

}  // namespace

int step3_fp32c_tma_tiles_y(int ny) { return (ny - 2 + T3 - 1) / T3; }

int step3_fp32c_tma_grid(int device) {
  int sms = 148, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  auto kern = step3_fp32c_tma_kernel<false, true, false, true, false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem3T) != cudaSuccess) {
    cudaGetLastError();
    return sms;
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, NT3, kSmem3T);
  return sms * (per < 1 ? 1 : per);
}

cudaError_t launch_step3_fp32c_tma(const Step3FConst& c, const Step3TArgs& a, int grid, int nbound, cudaStream_t s) {
  // `counter` is zero on entry: zeroed at allocation and rearmed by every
  // boundary launch.
  const bool unik = a.K == nullptr, planar = c.nz == 1, a2 = c.a2 != 0, diag = a.diag != nullptr;
  cudaError_t e = unik ? (diag ? launch_pa<true, true>(planar, a2, c, a, grid, s)
                               : launch_pa<true, false>(planar, a2, c, a, grid, s))
                       : (diag ? launch_pa<false, true>(planar, a2, c, a, grid, s)
                               : launch_pa<false, false>(planar, a2, c, a, grid, s));
  if (e != cudaSuccess) return e;
  return launch_pdl(boundary3_kernel, dim3((nbound + 255) / 256), dim3(256), 0, s, c, a, nbound);
}

}  // namespace capaz
