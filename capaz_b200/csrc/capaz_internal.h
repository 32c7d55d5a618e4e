// Internal declarations shared by the kernels and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/capaz_b200.h"

namespace capaz {

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
struct Step2Const {
  int nx, ny, nz;
  int source, iters;
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
  double vol;         // hx*hy*hz (diagnostics)
};

// Per-block partial diagnostics: mass[3], max residual, non-finite count.
constexpr int DIAG_STRIDE = 5;

// Launchers (kernels_fp64.cu).  Return cudaError_t of the launch.
cudaError_t launch_step2_fp64(const Step2Const& c, const double* Pw_in, const double* Sn_in,
                              double* Pw_out, double* Sn_out, const double* m, const double* K,
                              bool percell_k, double* diag_partials, unsigned int* err_flag,
                              cudaStream_t s, int* nlaunch);
cudaError_t launch_diag_finalize(const double* partials, int nblocks, double* out, cudaStream_t s);
// Derived field `field` of the start-of-step state (Pw, Sn) into out.
cudaError_t launch_derived2_fp64(const Step2Const& c, int field, const double* Pw, const double* Sn,
                                 const double* m, const double* K, bool percell_k, double* out,
                                 cudaStream_t s);
int step2_grid_blocks(const Step2Const& c);

}  // namespace capaz
