// Step dispatch and derived-field materialisation for a context.
#include "capaz_ctx.h"
#include "capaz_internal.h"

using namespace capaz;

int capaz_ctx::step(int nsteps, cudaStream_t s) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  if (nsteps == 0) return CAPAZ_OK;
  const bool diag = (p.flags & CAPAZ_FLAG_DIAGNOSTICS) != 0;
  if (p.phases == 2 && p.form == CAPAZ_FORM_FP64) {
    const Step2Const c = make_step2_const(p);
    if (diag && !diag_partials) {
      diag_blocks = step2_grid_blocks(c);
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    const bool percell = (p.flags & CAPAZ_FLAG_PERCELL_K) != 0;
    for (int t = 0; t < nsteps; t++) {
      const int nxt = cur ^ 1;
      int nl = 0;
      const bool last = (t == nsteps - 1);
      e = launch_step2_fp64(c, (const double*)state[cur][0], (const double*)state[cur][1],
                            (double*)state[nxt][0], (double*)state[nxt][1], (const double*)m,
                            (const double*)K, percell, (diag && last) ? diag_partials : nullptr, err_flag,
                            s, &nl);
      launches += nl;
      if (e != cudaSuccess) return fail_cuda(e, "step2_fp64 launch");
      cur = nxt;
      steps_done++;
    }
    if (diag) {
      e = launch_diag_finalize(diag_partials, diag_blocks, diag_out, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "diag finalize launch");
    }
    return CAPAZ_OK;
  }
  return fail_msg(CAPAZ_ERR_UNSUPPORTED, "this phase/form combination is not built yet");
}

int capaz_ctx::derived(int field, cudaStream_t s, bool from_current) {
  int st = ensure_scratch();
  if (st) return st;
  // Start-of-step state of the last step (the current state before any step).
  const int src = (steps_done > 0 && !from_current) ? (cur ^ 1) : cur;
  if (p.phases == 2 && p.form == CAPAZ_FORM_FP64) {
    const Step2Const c = make_step2_const(p);
    const bool percell = (p.flags & CAPAZ_FLAG_PERCELL_K) != 0;
    switch (field) {
      case CAPAZ_FIELD_S_G: case CAPAZ_FIELD_RO_G: case CAPAZ_FIELD_XI_G: case CAPAZ_FIELD_UX_G:
      case CAPAZ_FIELD_UY_G: case CAPAZ_FIELD_UZ_G: case CAPAZ_FIELD_ROS_G: case CAPAZ_FIELD_ROS_G_OLD:
      case CAPAZ_FIELD_P_G:
        return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "gas fields exist in three-phase only");
      default: break;
    }
    cudaError_t e = launch_derived2_fp64(c, field, (const double*)state[src][0], (const double*)state[src][1],
                                         (const double*)m, (const double*)K, percell, scratch, s);
    launches++;
    if (e != cudaSuccess) return fail_cuda(e, "derived launch");
    return CAPAZ_OK;
  }
  return fail_msg(CAPAZ_ERR_UNSUPPORTED, "derived fields for this phase/form are not built yet");
}
