// Internal declarations shared by the kernels and the C-ABI layer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/capaz_b200.h"

namespace capaz {

#ifdef __CUDACC__
// True when a and b have the same bits.  A Newton iteration that returns its
// input bit for bit has reached a fixed point: every later iteration repeats
// it, so stopping there gives exactly the result of the full iteration count.
__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
#endif

// Message returned by capaz_last_error(NULL) (calls without a context).
void set_create_error(const char* msg);

// Output tile of the fused sweep: TX x TY interior cells per z-plane, one
// thread per column, marching along z with a 3-plane ring in shared memory.
constexpr int TX = 32;
constexpr int TY = 8;
constexpr int PX = TX + 2;   // plane window with a one-cell halo
constexpr int PY = TY + 2;
constexpr int PC = PX * PY;  // 340 cells per plane window
constexpr int NTHREADS = TX * TY;

// Per-step constants of the two-phase FP64 step, passed by value.  Every
// derived constant is computed on the host with the same expression the
// reference evaluates inline, so its double value is identical.
// Injection window in z, in local plane indices: k in [win_k0, win_k1]
// (|k_global - NZ_global/2| <= SOURCE).
inline void window_k(const capaz_params& p, int* k0, int* k1) {
  const int nzg = p.nz_global > 0 ? p.nz_global : p.nz;
  *k0 = nzg / 2 - p.source - p.z_offset;
  *k1 = nzg / 2 + p.source - p.z_offset;
}

struct Step2Const {
  int nx, ny, nz;
  int source, iters, win_k0, win_k1;
  int tiles_x, tiles_y, zchunk, nzchunks;
  long long sy, sz, ncell;
  double hx, hy, hz, dt, g, P_atm, P_top;
  double ro0_w, ro0_n, beta_w, beta_n, mu_w, mu_n;
  double S_wr, lambda, P_d, K0, S_n_gr;
  double e_kw;        // (2. + 3.*lambda)/lambda   two-phase.cpp:11
  double e_kn;        // (2. + lambda)/lambda      two-phase.cpp:12
  double e_pk;        // -1./lambda                two-phase.cpp:13, 36
  double e_aaa;       // (-1./lambda) - 1.         two-phase.cpp:37
  double se_fast_min; // S_e at or above which P_d*pow(S_e, e) == +0 exactly
  double se_fast_num; // 1 - S_n - S_wr above which S_e >= se_fast_min without dividing
  double vol;         // hx*hy*hz (diagnostics)
  int lam2;           // CAPAZ_FLAG_POW_PRODUCTS with lambda == 2: relperms by products
};

// Constants of the two-phase precision-form step (step2_fp32c.cu).
struct Step2FConst {
  int nx, ny, nz;
  int source, iters, win_k0, win_k1;
  int tiles_x, tiles_y, zchunk, nzchunks;
  int intpow, n_kw, n_kn;  // relative-permeability exponents are small integers
  long long sy, sz;
  float S_ref_f, one_m_swr_f, inv_one_m_swr_f, e_kw_f, e_kn_f, e_pk_f, P_d_f;
  float ro0_w_f, ro0_n_f, beta_w_f, beta_n_f, inv_mu_w_f, inv_mu_n_f, K0_f, g_f;
  float inv_hx_f, inv_hy_f, inv_hz_f;
  double S_ref, dt, P_atm, P_top, P_d, S_wr, e_pk, ro0_w, ro0_n, beta_w, beta_n, g, hy, S_n_gr, vol;
};

struct Step2FArgs {
  const float *p_in, *s_in;
  float *p_out, *s_out;
  const float *m, *K;  // K == nullptr: uniform K0
  const double* Pref;  // per-row reference pressure (ny)
  const float* PrelF;  // Pref - P_atm (ny), FP32
  const float* dPrefF; // Pref[j+1] - Pref[j] (ny), FP32
  double* diag;        // per-block partials or nullptr
  unsigned int* err;
};

cudaError_t launch_step2_fp32c(const Step2FConst& c, const Step2FArgs& a, cudaStream_t s);
cudaError_t launch_decode2(const float* p, const float* s, const double* Pref, double S_ref, int nx, int ny,
                           long long n, double* P, double* S, cudaStream_t st);
cudaError_t launch_widen(const float* a, long long n, double* out, cudaStream_t st);

// Constants of the three-phase FP64 step (step3_fp64.cu).
struct Step3Const {
  int nx, ny, nz, source, iters, source_window, win_k0, win_k1;
  int tiles_x, tiles_y, zchunk, nzchunks, i_lo, i_hi;
  long long sy, sz, ncell;
  double hx, hy, hz, dt, g, P_atm;
  double ro0_w, ro0_n, ro0_g, beta_w, beta_n, mu_w, mu_n, mu_g;
  double S_wr, S_nr, S_gr, A, K0, S_w_gr, S_n_gr, vol;
  int a2;  // CAPAZ_FLAG_POW_PRODUCTS with A == 2: relperms by products and sqrt
};
struct Step3Buffers {
  double *Pw, *Sw, *Sn, *Pn, *Pg;
};
cudaError_t launch_step3_fp64(const Step3Const& c, const Step3Buffers& in, const Step3Buffers& out, const double* m,
                              const double* K, double* diag, unsigned int* err, cudaStream_t s);
cudaError_t launch_derived3_fp64(const Step3Const& c, int field, const Step3Buffers& st, const double* m,
                                 const double* K, double* out, cudaStream_t s);
cudaError_t launch_compose3(const Step3Const& c, const double* Pw_start, const double* bnd_now, double* out,
                            cudaStream_t s);

// Three-phase precision form (step3_fp32c.cu): FP32 deviations of P_w, P_n,
// P_g from the per-row reference pressure and of S_w, S_n from their means.
struct Step3FConst {
  int nx, ny, nz, source, source_window, win_k0, win_k1;
  int tiles_x, tiles_y, zchunk, nzchunks, i_lo, i_hi, a2;
  long long sy, sz;
  float S_ref_w_f, S_ref_n_f, S_wr_f, S_nr_f, inv_den, K0_f, aw_f, an_f, bg_f;
  float inv_mu_w_f, inv_mu_n_f, inv_mu_g_f, inv_hx2_f, inv_hy2_f, inv_hz2_f, g_inv_hy_f, dt_f, e1, e2, e3;
  double S_ref_w, S_ref_n, P_atm, aw, an, bg, ro0_w, ro0_n, ro0_g, beta_w, beta_n, g, hy, S_w_gr, S_n_gr, vol;
};
struct Step3FArgs {
  const float *p_w, *s_w, *s_n, *p_n, *p_g;
  float *o_pw, *o_sw, *o_sn, *o_pn, *o_pg;
  const float *m, *K;   // K == nullptr: uniform K0
  const float4* rowF;   // ny: rho_w, rho_n, rho_g at P_ref(j), P_ref(j+1) - P_ref(j)
  const double* Pref;   // ny
  double* diag;         // per-block partials or nullptr
  unsigned int* err;
};
cudaError_t launch_step3_fp32c(const Step3FConst& c, const Step3FArgs& a, cudaStream_t s);
// The same step with TMA-staged planes (step3_fp32c_tma.cu), for nx a
// multiple of 4 (nx >= 4): a persistent sweep over the interior cells
// (32 x 16 tiles, c.tiles_y from step3_fp32c_tma_tiles_y) and a kernel over
// the boundary shell, which rearms the work counter.
struct Step3TArgs {
  CUtensorMap map_pw, map_sw, map_sn, map_K, map_m;  // input P_w, S_w, S_n deviations, K, m (36 x 18 boxes)
  const float *p_n, *p_g;                            // input P_n, P_g deviations (read on the top and bottom rows)
  float *o_pw, *o_sw, *o_sn, *o_pn, *o_pg;
  const float* K;                                    // nullptr: uniform K0
  const float4* rowF;                                // as in Step3FArgs
  const double* Pref;
  double* diag;                                      // per-CTA partials or nullptr
  unsigned int* err;
  unsigned int* counter;                             // work counter, zero between launches
};
int step3_fp32c_tma_tiles_y(int ny);
int step3_fp32c_tma_grid(int device);
cudaError_t launch_step3_fp32c_tma(const Step3FConst& c, const Step3TArgs& a, int grid, int nbound, cudaStream_t s);
cudaError_t launch_row_tables3(const double* Pref, int ny, const Step3FConst& c, float4* rowF, cudaStream_t s);

// Batched (ensemble) steps: one persistent launch over (instance, tile,
// z-chunk) work items.  State pointers per ping-pong parity.
struct Inst64 {
  Step2Const c;
  double* Pw[2];
  double* Sn[2];
  const double* m;
  const double* K;
  unsigned int* err;
};
struct InstF {
  Step2FConst c;
  Step2FArgs a[2];  // a[parity]: reads buffer parity, writes parity ^ 1
};
cudaError_t launch_step2_fp64_batch(const Inst64* insts, const int4* items, int nitems, int parity, bool unik, bool pd0,
                                    unsigned int* counter, int grid, cudaStream_t s);
cudaError_t launch_step2_fp32c_batch(const InstF* insts, const int4* items, int nitems, int parity, bool unik,
                                     bool pd0, bool intpow, unsigned int* counter, int grid, cudaStream_t s);
int step2_fp64_batch_grid(int device);
int step2_fp32c_batch_grid(int device);

// TMA-staged precision-form step (step2_fp32c_tma.cu), for P_d = 0 and
// lambda = 2.  Physics constants shared by every instance of a launch are a
// kernel parameter; per-instance geometry, dt, S_ref and tensor maps live
// in one descriptor per instance in global memory.
struct PhysF {
  float inv_one_m_swr, ro0w_bw, ro0n_bn, inv_mu_w, inv_mu_n, K0, inv_hx2, inv_hy2, inv_hz2, g_inv_hy;
  // rho_p / mu_p is formed directly: (rho_0p beta_p / mu_p) p + rho_p(P_ref)/mu_p
  // (per-row table); the gravity force g rho_p / hy is then (g mu_p / hy) times it.
  float cw_mu, cn_mu, g_mu_w, g_mu_n;
  int iters;
  double ro0_w, ro0_n, aw, bn, P_atm, P_top, g, hy, vol, mu_w, mu_n;
};
struct alignas(128) InstT {
  CUtensorMap map_p[2], map_s[2], map_K, map_m;
  int nx, ny, nz, tiles_x, tiles_y, zchunk, nzchunks, source, win_k0, win_k1;
  long long sy, sz;
  float c1_f;       // 1 - S_wr - S_ref
  float dt_f;
  float sgr_dev_f;  // S_n_gr - S_ref (stored deviation of the source saturation)
  int nbound;       // boundary cells (written by the boundary kernel after the sweep)
  int halo_lo, halo_hi;  // planes 0 / nz-1 are z-slab halo planes: the boundary kernel leaves them
  int tile_y;       // rows of a tile (the tensor maps' box is 36 x (tile_y + 2))
  // Bytes each raw stage announces beyond what its copies bring: 0, except
  // under CAPAZ_FLAG_TEST_WAIT_TIMEOUT, where it makes the first bounded
  // wait of every CTA run out (a test of the timeout path; nothing faults).
  unsigned int test_tx_extra;
  double S_ref, dt;
  const float4* rowF;  // ny: (rho_w/mu_w, rho_n/mu_n at P_ref(j), (P_ref(j+1)-P_ref(j))/hy^2, 0)
  const double* Pref;  // ny
  Step2FArgs a[2];     // a[parity]: state pointers and the error flag
};
// Tiles of the TMA-staged precision step: TX x tile_y interior cells, one
// warp per four rows; tile_y is 16 (four warps, four CTAs per SM) or 32
// (eight warps, two CTAs per SM).  TMA_TILE_Y is the default.
constexpr int TMA_TILE_Y = 16;
bool tma_tile_supported(int tile_y);
// All instances of one launch are planar (nz == 1) or all three-dimensional.
// A step is the sweep over the interior cells (work items: instance, tile,
// first centre plane, last plane loaded) and then the boundary kernel over
// every instance's boundary shell (bitems: (instance, first boundary cell)
// blocks of BOUND_BLOCK).  counters: four zeroed words (work items and
// finished CTAs per state parity) that the sweeps rearm themselves.  With
// diag_partials, the sweep writes per-CTA diagnostics partials (grid of
// them) and its last CTA reduces them into diag_out, and also into diag_host
// (the device view of mapped pinned host memory) when that is not null.
constexpr int BOUND_BLOCK = 256;
constexpr int SWEEP_COUNTERS = 4;
cudaError_t launch_step2_fp32c_tma(const PhysF& f, const InstT* insts, const int4* items, int nitems, int parity,
                                   bool unik, bool planar, unsigned int* counters, double* diag_partials, int grid,
                                   cudaStream_t s, double* diag_out, int tile_y, double* diag_host = nullptr);
cudaError_t launch_boundary_fp32c(const PhysF& f, const InstT* insts, const int2* bitems, int nbitems, int parity,
                                  cudaStream_t s);
// Boundary cells of an nx x ny x nz grid (faces, edges, corners; nz == 1: the
// four sides of the plane).
inline int boundary_cells(int nx, int ny, int nz) {
  if (nz == 1) return 2 * nx + 2 * (ny - 2);
  return 2 * nx * nz + 2 * (ny - 2) * nz + 2 * (nx - 2) * (ny - 2);
}
int step2_fp32c_tma_grid(int device, bool unik, int tile_y);
int encode_field_map(CUtensorMap* map, const float* base, int nx, int ny, int nz, int tile_y);
cudaError_t launch_row_tables(const double* Pref, int ny, const PhysF& f, float4* rowF, cudaStream_t s);

// Field preparation (fields.cu).
cudaError_t launch_first_invalid(const double* a, long long n, unsigned long long* first, cudaStream_t s);
cudaError_t launch_encode_pressure(const double* P, int nx, int ny, int nz, double P_atm, double* Pref, float* PrelF,
                                   float* dPrefF, float* out, cudaStream_t s);
cudaError_t launch_encode_saturation(const double* S, long long n, double* part, double* S_ref, float* out,
                                     cudaStream_t s);
cudaError_t launch_narrow(const double* a, long long n, float* out, cudaStream_t s);
cudaError_t launch_encode_pressure_rel(const double* P, const double* Pref, int nx, int ny, long long n, float* out,
                                       cudaStream_t s);
cudaError_t launch_decode_pressure(const float* p, const double* Pref, int nx, int ny, long long n, double* out,
                                   cudaStream_t s);
// Tables of a given per-row reference (P_ref - P_atm, P_ref(j+1) - P_ref(j))
// and saturation deviations from a given reference value.
cudaError_t launch_pref_tables(const double* Pref, int ny, double P_atm, float* PrelF, float* dPrefF, cudaStream_t s);
cudaError_t launch_encode_saturation_ref(const double* S, long long n, const double* S_ref, float* out,
                                         cudaStream_t s);

// Per-block partial diagnostics: mass[3], max residual, non-finite count.
constexpr int DIAG_STRIDE = 5;

// Launchers (kernels_fp64.cu).  Return cudaError_t of the launch.
cudaError_t launch_step2_fp64(const Step2Const& c, const double* Pw_in, const double* Sn_in,
                              double* Pw_out, double* Sn_out, const double* m, const double* K,
                              bool percell_k, double* diag_partials, unsigned int* err_flag,
                              cudaStream_t s, int* nlaunch);
cudaError_t launch_diag_finalize(const double* partials, int nblocks, double* out, cudaStream_t s);
cudaError_t launch_diag_publish(const double* d, double* host_mapped, cudaStream_t s);
// Derived field `field` of the start-of-step state (Pw, Sn) into out.
cudaError_t launch_derived2_fp64(const Step2Const& c, int field, const double* Pw, const double* Sn,
                                 const double* m, const double* K, bool percell_k, double* out,
                                 cudaStream_t s);
int step2_grid_blocks(const Step2Const& c);

// Three-phase with the energy equation (step3e.cu).  The state is updated in
// place; `work` holds EW_COUNT arrays of ncell doubles, the reference's other
// per-cell arrays as they stand after the last step.
struct EnergyState {
  double *Pw, *Sn, *Sw, *Pn, *Pg, *T;
};
enum EnergyWork {
  EW_SG, EW_RO_W, EW_RO_N, EW_RO_G, EW_XI_W, EW_XI_N, EW_XI_G,
  EW_UX_W, EW_UY_W, EW_UZ_W, EW_UX_N, EW_UY_N, EW_UZ_N, EW_UX_G, EW_UY_G, EW_UZ_G,
  EW_ROS_W, EW_ROS_N, EW_ROS_G, EW_ROS_W_OLD, EW_ROS_N_OLD, EW_ROS_G_OLD,
  EW_H_W, EW_H_N, EW_H_G, EW_H_R, EW_E, EW_E_NEW, EW_LAM, EW_COUNT
};
constexpr double ENERGY_T_INIT = 285.;  // data_initialization, three-phase.cpp:487
cudaError_t launch_step3_energy(const Step3Const& c, const EnergyState& st, const double* m, const double* K,
                                double* work, unsigned int* err, cudaStream_t s);

// Buckley-Leverett task (step_bl.cu): the two-phase constants plus the
// wells' rate and pressures.
struct BLConst {
  Step2Const c;
  double Q, injwell_Pw, outwell_Pw;
};
cudaError_t launch_step_bl(const BLConst& b, const double* Pw_in, const double* Sn_in, double* Pw_out, double* Sn_out,
                           const double* m, const double* K, bool percell_k, unsigned int* err, cudaStream_t s);
cudaError_t launch_derived_bl(const BLConst& b, int field, const double* Pw, const double* Sn, const double* m,
                              const double* K, bool percell_k, double* out, cudaStream_t s);

}  // namespace capaz
