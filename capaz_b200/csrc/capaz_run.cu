// Step dispatch and derived-field materialisation for a context.
#include <string.h>

#include <algorithm>
#include <vector>

#include "capaz_ctx.h"
#include "capaz_internal.h"

using namespace capaz;

// The number of z-chunks of the interior planes for a persistent sweep over
// ntiles tiles with gmax resident CTAs: the one that minimises the estimated
// span, the rounds of items per CTA (rounded up) times the planes an item
// loads (its chunk and two halo planes).  Chunks shorter than four planes
// derive more halo planes than they update and are not considered.  Chunk zc
// covers the centre planes 1 + zc*interior/n .. 1 + (zc+1)*interior/n - 1.
static int balanced_zchunks(long long ntiles, int interior, int gmax) {
  int best = 1;
  long long best_cost = -1;
  for (int nc = 1; nc <= interior; nc++) {
    const int len = (interior + nc - 1) / nc;
    if (nc > 1 && len < 4) break;
    const long long cost = ((ntiles * nc + gmax - 1) / gmax) * (len + 2);
    if (best_cost < 0 || cost < best_cost) best_cost = cost, best = nc;
  }
  return best;
}

int capaz_ctx::step(int nsteps, cudaStream_t s) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  if (nsteps == 0) return CAPAZ_OK;
  const bool diag = (p.flags & CAPAZ_FLAG_DIAGNOSTICS) != 0;
  if (p.model == CAPAZ_MODEL_ENERGY) {
    const Step3Const c = make_step3_const(p);
    const EnergyState st{(double*)state[cur][0], (double*)state[cur][1], (double*)state[cur][2],
                         (double*)state[cur][3], (double*)state[cur][4], (double*)state[cur][5]};
    const double* Kp = (p.flags & CAPAZ_FLAG_PERCELL_K) ? (const double*)K : nullptr;
    for (int t = 0; t < nsteps; t++) {
      e = launch_step3_energy(c, st, (const double*)m, Kp, ework, err_flag, s);
      launches += 5;
      if (e != cudaSuccess) return fail_cuda(e, "step3_energy launch");
      steps_done++;
    }
    return CAPAZ_OK;
  }
  if (p.model == CAPAZ_MODEL_BUCKLEY_LEVERETT) {
    const BLConst b = make_bl_const(p);
    const bool percell = (p.flags & CAPAZ_FLAG_PERCELL_K) != 0;
    for (int t = 0; t < nsteps; t++) {
      const int nxt = cur ^ 1;
      e = launch_step_bl(b, (const double*)state[cur][0], (const double*)state[cur][1], (double*)state[nxt][0],
                         (double*)state[nxt][1], (const double*)m, (const double*)K, percell, err_flag, s);
      launches += 2;
      if (e != cudaSuccess) return fail_cuda(e, "step_bl launch");
      cur = nxt;
      steps_done++;
    }
    return CAPAZ_OK;
  }
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
  if (tma_applies()) {
    int st = tma_prepare();
    if (st) return st;
    if (counters_dirty) {
      // Split steps advanced the state without this path's launches: its
      // per-parity counters are rezeroed instead of rearmed.
      e = cudaMemsetAsync(tma_counter, 0, sizeof(unsigned int) * SWEEP_COUNTERS, s);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counters)");
      counters_dirty = false;
    }
    const PhysF f = make_physf(p);
    const bool unik = !(p.flags & CAPAZ_FLAG_PERCELL_K);
    if (diag && !diag_partials) {
      diag_blocks = tma_grid;
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    for (int t = 0; t < nsteps; t++) {
      const bool last = t == nsteps - 1;
      // With diagnostics, the last step's boundary kernel also reduces the
      // sweep's partials into diag_out.
      double* const pub = (diag && last) ? publish_to : nullptr;
      e = launch_step2_fp32c_tma(f, tma_inst, tma_items, tma_nitems, cur, unik, p.nz == 1, tma_counter,
                                 (diag && last) ? diag_partials : nullptr, tma_grid, s, diag_out, tma_tile_y, pub);
      if (pub) published = true;
      if (e == cudaSuccess) e = launch_boundary_fp32c(f, tma_inst, tma_bitems, tma_nbitems, cur, s);
      launches += 2;
      if (e != cudaSuccess) return fail_cuda(e, "step2_fp32c_tma launch");
      cur ^= 1;
      steps_done++;
    }
    return CAPAZ_OK;
  }
  if (p.phases == 2 && p.form == CAPAZ_FORM_FP32C) {
    const Step2FConst c = make_step2f_const(p, S_ref);
    if (diag && !diag_partials) {
      diag_blocks = c.tiles_x * c.tiles_y * c.nzchunks;
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    for (int t = 0; t < nsteps; t++) {
      const int nxt = cur ^ 1;
      Step2FArgs a;
      a.p_in = (const float*)state[cur][0];
      a.s_in = (const float*)state[cur][1];
      a.p_out = (float*)state[nxt][0];
      a.s_out = (float*)state[nxt][1];
      a.m = (const float*)m;
      a.K = (p.flags & CAPAZ_FLAG_PERCELL_K) ? (const float*)K : nullptr;
      a.Pref = Pref;
      a.PrelF = PrelF;
      a.dPrefF = dPrefF;
      a.diag = (diag && t == nsteps - 1) ? diag_partials : nullptr;
      a.err = err_flag;
      e = launch_step2_fp32c(c, a, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "step2_fp32c launch");
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
  if (p.phases == 3 && p.form == CAPAZ_FORM_FP64) {
    const Step3Const c = make_step3_const(p);
    if (diag && !diag_partials) {
      diag_blocks = c.tiles_x * c.tiles_y * c.nzchunks;
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    const double* Kp = (p.flags & CAPAZ_FLAG_PERCELL_K) ? (const double*)K : nullptr;
    for (int t = 0; t < nsteps; t++) {
      const int nxt = cur ^ 1;
      Step3Buffers in{(double*)state[cur][0], (double*)state[cur][2], (double*)state[cur][1], (double*)state[cur][3],
                      (double*)state[cur][4]};
      Step3Buffers out{(double*)state[nxt][0], (double*)state[nxt][2], (double*)state[nxt][1],
                       (double*)state[nxt][3], (double*)state[nxt][4]};
      e = launch_step3_fp64(c, in, out, (const double*)m, Kp, (diag && t == nsteps - 1) ? diag_partials : nullptr,
                            err_flag, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "step3_fp64 launch");
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
  if (p.phases == 3 && p.form == CAPAZ_FORM_FP32C && p.nx % 4 == 0 && p.nx >= 4 && !(p.flags & CAPAZ_FLAG_NO_TMA)) {
    Step3FConst c = make_step3f_const(p, S_ref_w, S_ref);
    c.tiles_y = step3_fp32c_tma_tiles_y(p.ny);
    const int g3 = step3_fp32c_tma_grid(device);
    if (g3 <= 0) return fail_msg(CAPAZ_ERR_CUDA, "no resident CTA for the three-phase sweep");
    if (p.nz > 1) {
      c.nzchunks = balanced_zchunks((long long)c.tiles_x * c.tiles_y, p.nz - 2, g3);
      c.zchunk = (p.nz - 2 + c.nzchunks - 1) / c.nzchunks;
    }
    if (!t3_ready) {
      const int ty = 16;
      for (int b = 0; b < 2; b++) {
        Step3TArgs& a = t3a[b];
        memset(&a, 0, sizeof a);
        if (encode_field_map(&a.map_pw, (const float*)state[b][0], p.nx, p.ny, p.nz, ty) ||
            encode_field_map(&a.map_sw, (const float*)state[b][2], p.nx, p.ny, p.nz, ty) ||
            encode_field_map(&a.map_sn, (const float*)state[b][1], p.nx, p.ny, p.nz, ty) ||
            encode_field_map(&a.map_m, (const float*)m, p.nx, p.ny, p.nz, ty))
          return fail_msg(CAPAZ_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        if (p.flags & CAPAZ_FLAG_PERCELL_K) {
          if (encode_field_map(&a.map_K, (const float*)K, p.nx, p.ny, p.nz, ty))
            return fail_msg(CAPAZ_ERR_CUDA, "cuTensorMapEncodeTiled failed (K)");
          a.K = (const float*)K;
        } else {
          a.map_K = a.map_m;  // unused (uniform K)
          a.K = nullptr;
        }
        a.p_n = (const float*)state[b][3];
        a.p_g = (const float*)state[b][4];
        a.o_pw = (float*)state[b ^ 1][0];
        a.o_sn = (float*)state[b ^ 1][1];
        a.o_sw = (float*)state[b ^ 1][2];
        a.o_pn = (float*)state[b ^ 1][3];
        a.o_pg = (float*)state[b ^ 1][4];
        a.rowF = rowF;
        a.Pref = Pref;
        a.err = err_flag;
      }
      if (!t3_counter) {
        e = cudaMalloc(&t3_counter, sizeof(unsigned int));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(counter)");
        e = cudaMemset(t3_counter, 0, sizeof(unsigned int));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMemset(counter)");
      }
      t3a[0].counter = t3a[1].counter = t3_counter;
      t3_grid = std::min(c.tiles_x * c.tiles_y * c.nzchunks, g3);
      t3_ready = true;
    }
    if (diag && !diag_partials) {
      diag_blocks = t3_grid;
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    const int nbound = boundary_cells(p.nx, p.ny, p.nz);
    for (int t = 0; t < nsteps; t++) {
      Step3TArgs a = t3a[cur];
      a.diag = (diag && t == nsteps - 1) ? diag_partials : nullptr;
      e = launch_step3_fp32c_tma(c, a, t3_grid, nbound, s);
      launches += 2;
      if (e != cudaSuccess) return fail_cuda(e, "step3_fp32c_tma launch");
      cur ^= 1;
      steps_done++;
    }
    if (diag) {
      e = launch_diag_finalize(diag_partials, t3_grid, diag_out, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "diag finalize launch");
    }
    return CAPAZ_OK;
  }
  if (p.phases == 3 && p.form == CAPAZ_FORM_FP32C) {
    const Step3FConst c = make_step3f_const(p, S_ref_w, S_ref);
    if (diag && !diag_partials) {
      diag_blocks = c.tiles_x * c.tiles_y * c.nzchunks;
      e = cudaMalloc(&diag_partials, sizeof(double) * DIAG_STRIDE * diag_blocks);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(diag)");
    }
    for (int t = 0; t < nsteps; t++) {
      const int nxt = cur ^ 1;
      Step3FArgs a;
      a.p_w = (const float*)state[cur][0];
      a.s_n = (const float*)state[cur][1];
      a.s_w = (const float*)state[cur][2];
      a.p_n = (const float*)state[cur][3];
      a.p_g = (const float*)state[cur][4];
      a.o_pw = (float*)state[nxt][0];
      a.o_sn = (float*)state[nxt][1];
      a.o_sw = (float*)state[nxt][2];
      a.o_pn = (float*)state[nxt][3];
      a.o_pg = (float*)state[nxt][4];
      a.m = (const float*)m;
      a.K = (p.flags & CAPAZ_FLAG_PERCELL_K) ? (const float*)K : nullptr;
      a.rowF = rowF;
      a.Pref = Pref;
      a.diag = (diag && t == nsteps - 1) ? diag_partials : nullptr;
      a.err = err_flag;
      e = launch_step3_fp32c(c, a, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "step3_fp32c launch");
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
  if (p.model == CAPAZ_MODEL_ENERGY) {
    // The reference's arrays as the last step left them (zero before the
    // first step); P_n, P_g are state arrays of this model.
    int slot = -1;
    switch (field) {
      case CAPAZ_FIELD_S_G: slot = EW_SG; break;
      case CAPAZ_FIELD_RO_W: slot = EW_RO_W; break;
      case CAPAZ_FIELD_RO_N: slot = EW_RO_N; break;
      case CAPAZ_FIELD_RO_G: slot = EW_RO_G; break;
      case CAPAZ_FIELD_XI_W: slot = EW_XI_W; break;
      case CAPAZ_FIELD_XI_N: slot = EW_XI_N; break;
      case CAPAZ_FIELD_XI_G: slot = EW_XI_G; break;
      case CAPAZ_FIELD_ROS_W: slot = EW_ROS_W; break;
      case CAPAZ_FIELD_ROS_N: slot = EW_ROS_N; break;
      case CAPAZ_FIELD_ROS_G: slot = EW_ROS_G; break;
      case CAPAZ_FIELD_ROS_W_OLD: slot = EW_ROS_W_OLD; break;
      case CAPAZ_FIELD_ROS_N_OLD: slot = EW_ROS_N_OLD; break;
      case CAPAZ_FIELD_ROS_G_OLD: slot = EW_ROS_G_OLD; break;
      case CAPAZ_FIELD_H_W: slot = EW_H_W; break;
      case CAPAZ_FIELD_H_N: slot = EW_H_N; break;
      case CAPAZ_FIELD_H_G: slot = EW_H_G; break;
      case CAPAZ_FIELD_H_R: slot = EW_H_R; break;
      case CAPAZ_FIELD_E: slot = EW_E; break;
      case CAPAZ_FIELD_E_NEW: slot = EW_E_NEW; break;
      default:
        if (field >= CAPAZ_FIELD_UX_W && field <= CAPAZ_FIELD_UZ_G) slot = EW_UX_W + (field - CAPAZ_FIELD_UX_W);
        break;
    }
    const void* from = slot >= 0 ? (const void*)(ework + (size_t)slot * n)
                                 : (field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G)
                                       ? state[cur][state_slot(field)]
                                       : nullptr;
    if (!from) return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "field not kept by the energy model");
    cudaError_t e = cudaMemcpyAsync(scratch, from, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return fail_cuda(e, "derived copy");
    return CAPAZ_OK;
  }
  if (field >= CAPAZ_FIELD_T) return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "energy fields exist in the energy model only");
  if (p.model == CAPAZ_MODEL_BUCKLEY_LEVERETT) {
    if (field == CAPAZ_FIELD_S_G || field == CAPAZ_FIELD_RO_G || field == CAPAZ_FIELD_XI_G ||
        field == CAPAZ_FIELD_UX_G || field == CAPAZ_FIELD_UY_G || field == CAPAZ_FIELD_UZ_G ||
        field == CAPAZ_FIELD_ROS_G || field == CAPAZ_FIELD_ROS_G_OLD || field == CAPAZ_FIELD_P_G)
      return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "gas fields exist in three-phase only");
    cudaError_t e = launch_derived_bl(make_bl_const(p), field, (const double*)state[src][0],
                                      (const double*)state[src][1], (const double*)m, (const double*)K,
                                      (p.flags & CAPAZ_FLAG_PERCELL_K) != 0, scratch, s);
    launches++;
    if (e != cudaSuccess) return fail_cuda(e, "derived launch");
    return CAPAZ_OK;
  }
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
  if (p.phases == 2 && p.form == CAPAZ_FORM_FP32C) {
    // Decode the chosen state to FP64 and evaluate the FP64 derived kernel.
    st = decode_all(src, s);
    if (st) return st;
    const Step2Const c = make_step2_const(p);
    const bool percell = (p.flags & CAPAZ_FLAG_PERCELL_K) != 0;
    cudaError_t e = launch_derived2_fp64(c, field, wide[0], wide[1], wide[2], wide[3], percell, scratch, s);
    launches++;
    if (e != cudaSuccess) return fail_cuda(e, "derived launch");
    return CAPAZ_OK;
  }
  if (p.phases == 3 && p.form == CAPAZ_FORM_FP64) {
    const Step3Const c = make_step3_const(p);
    const double* Kp = (p.flags & CAPAZ_FLAG_PERCELL_K) ? (const double*)K : nullptr;
    Step3Buffers stb{(double*)state[src][0], (double*)state[src][2], (double*)state[src][1], (double*)state[src][3],
                     (double*)state[src][4]};
    if (field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G) {
      // The reference's P_n, P_g arrays after a step: start-of-step P_w on
      // interior cells, this step's Border_P values on boundary cells.
      const int slot = field == CAPAZ_FIELD_P_N ? 3 : 4;
      cudaError_t e = launch_compose3(c, (const double*)state[src][0], (const double*)state[cur][slot], scratch, s);
      launches++;
      if (e != cudaSuccess) return fail_cuda(e, "compose launch");
      return CAPAZ_OK;
    }
    if (field == CAPAZ_FIELD_S_W || field == CAPAZ_FIELD_P_W || field == CAPAZ_FIELD_S_N)
      return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "state field");
    cudaError_t e = launch_derived3_fp64(c, field, stb, (const double*)m, Kp, scratch, s);
    launches++;
    if (e != cudaSuccess) return fail_cuda(e, "derived launch");
    return CAPAZ_OK;
  }
  if (p.phases == 3 && p.form == CAPAZ_FORM_FP32C) {
    // Decode to FP64 and evaluate the FP64 three-phase derived kernels.
    const Step3Const c = make_step3_const(p);
    if (field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G) {
      // Start-of-step P_w on interior cells, current Border_P values elsewhere.
      if (!stage) {
        cudaError_t e = cudaMalloc(&stage, n * sizeof(double));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(stage)");
      }
      cudaError_t e = launch_decode_pressure((const float*)state[src][0], Pref, p.nx, p.ny, n, stage, s);
      if (e != cudaSuccess) return fail_cuda(e, "decode launch");
      st = decode_all(cur, s);
      if (st) return st;
      e = launch_compose3(c, stage, wide[field == CAPAZ_FIELD_P_N ? 5 : 6], scratch, s);
      launches += 2;
      if (e != cudaSuccess) return fail_cuda(e, "compose launch");
      return CAPAZ_OK;
    }
    if (field == CAPAZ_FIELD_S_W || field == CAPAZ_FIELD_P_W || field == CAPAZ_FIELD_S_N)
      return fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "state field");
    st = decode_all(src, s);
    if (st) return st;
    const double* Kp = (p.flags & CAPAZ_FLAG_PERCELL_K) ? wide[3] : nullptr;
    Step3Buffers stb{wide[0], wide[4], wide[1], wide[5], wide[6]};
    cudaError_t e = launch_derived3_fp64(c, field, stb, wide[2], Kp, scratch, s);
    launches++;
    if (e != cudaSuccess) return fail_cuda(e, "derived launch");
    return CAPAZ_OK;
  }
  return fail_msg(CAPAZ_ERR_UNSUPPORTED, "derived fields for this phase/form are not built yet");
}

// One time step as two sweeps: the edge planes (1 and nz - 2, with their
// boundary cells) on `edge`, the interior planes (2 .. nz - 3) on
// `interior`.  Each stream first waits for everything queued on the other,
// so the caller's exchange of the previous step's planes on `edge` is done
// before this step reads them.  The new state becomes current at once; its
// edge planes are complete in `edge` order and can be sent while the
// interior sweep runs.
int capaz_ctx::step_split(cudaStream_t edge, cudaStream_t interior) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  if (!tma_applies() || p.nz < 4 || (p.flags & CAPAZ_FLAG_DIAGNOSTICS))
    return fail_msg(CAPAZ_ERR_UNSUPPORTED,
                    "split steps need the two-phase precision form with the TMA sweep (nx a multiple of 4, ny and "
                    "nz at least 4) and no diagnostics");
  int st = tma_prepare();
  if (st) return st;
  const bool unik = !(p.flags & CAPAZ_FLAG_PERCELL_K);
  if (!split_items || split_tile_y != tma_tile_y) {
    const int ty = tma_tile_y;
    const int ntiles = ((p.nx - 2 + TX - 1) / TX) * ((p.ny - 2 + ty - 1) / ty);
    std::vector<int4> items;
    for (int t = 0; t < ntiles; t++) items.push_back(make_int4(0, t, 1, 2));
    if (p.nz - 2 > 1)
      for (int t = 0; t < ntiles; t++) items.push_back(make_int4(0, t, p.nz - 2, p.nz - 1));
    split_nedge = (int)items.size();
    const int full = step2_fp32c_tma_grid(device, unik, ty);
    const int inner = p.nz - 4;  // centre planes 2 .. nz - 3
    if (inner > 0) {
      const int nc = balanced_zchunks(ntiles, inner, full);
      for (int zc = 0; zc < nc; zc++)
        for (int t = 0; t < ntiles; t++)
          items.push_back(make_int4(0, t, 2 + (int)((long long)zc * inner / nc),
                                    2 + (int)((long long)(zc + 1) * inner / nc)));
    }
    split_nint = (int)items.size() - split_nedge;
    if (split_items) cudaFree(split_items);
    split_items = nullptr;
    e = cudaMalloc(&split_items, sizeof(int4) * items.size());
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(split items)");
    e = cudaMemcpy(split_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpy(split items)");
    split_grid_e = std::min(split_nedge, full);
    split_grid_i = std::min(std::max(split_nint, 1), full);
    split_tile_y = ty;
    if (!split_counters) {
      e = cudaMalloc(&split_counters, sizeof(unsigned int) * 2 * SWEEP_COUNTERS);
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(split counters)");
    }
    for (auto& ev : split_ev)
      if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
  }
  // Join the two streams.
  if ((e = cudaEventRecord(split_ev[0], edge)) != cudaSuccess ||
      (e = cudaEventRecord(split_ev[1], interior)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(edge, split_ev[1], 0)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(interior, split_ev[0], 0)) != cudaSuccess)
    return fail_cuda(e, "stream join");
  // Counters are rezeroed every split step (the two sweeps do not alternate
  // with each other the way consecutive single launches do).
  if ((e = cudaMemsetAsync(split_counters, 0, sizeof(unsigned int) * SWEEP_COUNTERS, edge)) != cudaSuccess ||
      (e = cudaMemsetAsync(split_counters + SWEEP_COUNTERS, 0, sizeof(unsigned int) * SWEEP_COUNTERS, interior)) !=
          cudaSuccess)
    return fail_cuda(e, "cudaMemsetAsync(split counters)");
  const PhysF f = make_physf(p);
  e = launch_step2_fp32c_tma(f, tma_inst, split_items, split_nedge, cur, unik, false, split_counters, nullptr,
                             split_grid_e, edge, nullptr, tma_tile_y);
  if (e != cudaSuccess) return fail_cuda(e, "edge sweep launch");
  launches++;
  if (split_nint > 0) {
    e = launch_step2_fp32c_tma(f, tma_inst, split_items + split_nedge, split_nint, cur, unik, false,
                               split_counters + SWEEP_COUNTERS, nullptr, split_grid_i, interior, nullptr, tma_tile_y);
    if (e != cudaSuccess) return fail_cuda(e, "interior sweep launch");
    launches++;
  }
  // The boundary cells (of every plane but the halo planes) after both
  // sweeps, on the interior stream.
  if ((e = cudaEventRecord(split_ev[0], edge)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(interior, split_ev[0], 0)) != cudaSuccess)
    return fail_cuda(e, "stream join");
  e = launch_boundary_fp32c(f, tma_inst, tma_bitems, tma_nbitems, cur, interior);
  if (e != cudaSuccess) return fail_cuda(e, "boundary launch");
  launches++;
  cur ^= 1;
  steps_done++;
  counters_dirty = true;
  return CAPAZ_OK;
}

bool capaz_ctx::tma_applies() const {
  // The sweep writes each boundary cell from its basic cell with at most one
  // face per axis: grids at least four cells thick (or planar in z).
  return p.phases == 2 && p.form == CAPAZ_FORM_FP32C && p.nx % 4 == 0 && p.P_d == 0. && p.lambda == 2.0 &&
         p.ny >= 4 && (p.nz == 1 || p.nz >= 4) && !(p.flags & CAPAZ_FLAG_NO_TMA);
}

// Builds (or refreshes) the device descriptor of the TMA-staged precision
// step: tensor maps of both state buffers and of K and m, the geometry, dt
// and S_ref, and the work-item list.
int capaz_ctx::tma_prepare() {
  if (tma_ready && tma_dt == p.dt && tma_S_ref == S_ref && tma_built_tile_y == tma_tile_y) return CAPAZ_OK;
  const int ty = tma_tile_y;
  InstT h;
  memset(&h, 0, sizeof h);
  const Step2Const d = make_step2_const(p);
  h.nx = p.nx;
  h.ny = p.ny;
  h.nz = p.nz;
  h.tiles_x = d.tiles_x;
  h.tiles_y = (p.ny - 2 + ty - 1) / ty;
  h.tile_y = ty;
  h.source = p.source;
  window_k(p, &h.win_k0, &h.win_k1);
  h.sy = d.sy;
  h.sz = d.sz;
  // z-chunks that fill the persistent grid (balanced_zchunks).
  const int gmax = step2_fp32c_tma_grid(device, !(p.flags & CAPAZ_FLAG_PERCELL_K), ty);
  if (gmax <= 0) return fail_msg(CAPAZ_ERR_CUDA, "no resident CTA for the precision sweep");
  if (p.nz > 1) {
    h.nzchunks = balanced_zchunks((long long)h.tiles_x * h.tiles_y, p.nz - 2, gmax);
    h.zchunk = (p.nz - 2 + h.nzchunks - 1) / h.nzchunks;
  } else {
    h.zchunk = 1;
    h.nzchunks = 1;
  }
  h.c1_f = (float)(1. - p.S_wr - S_ref);
  h.dt_f = (float)p.dt;
  h.sgr_dev_f = (float)(p.S_n_gr - S_ref);
  h.nbound = boundary_cells(p.nx, p.ny, p.nz);
  h.halo_lo = p.z_offset > 0;
  h.halo_hi = p.nz_global > 0 && p.z_offset + p.nz < p.nz_global;
  h.test_tx_extra = (p.flags & CAPAZ_FLAG_TEST_WAIT_TIMEOUT) ? 16u : 0u;
  h.S_ref = S_ref;
  h.dt = p.dt;
  h.rowF = rowF;
  h.Pref = Pref;
  for (int b = 0; b < 2; b++) {
    if (encode_field_map(&h.map_p[b], (const float*)state[b][0], p.nx, p.ny, p.nz, ty) ||
        encode_field_map(&h.map_s[b], (const float*)state[b][1], p.nx, p.ny, p.nz, ty))
      return fail_msg(CAPAZ_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  }
  if (encode_field_map(&h.map_m, (const float*)m, p.nx, p.ny, p.nz, ty))
    return fail_msg(CAPAZ_ERR_CUDA, "cuTensorMapEncodeTiled failed (m)");
  if (K && encode_field_map(&h.map_K, (const float*)K, p.nx, p.ny, p.nz, ty))
    return fail_msg(CAPAZ_ERR_CUDA, "cuTensorMapEncodeTiled failed (K)");
  if (!K) h.map_K = h.map_m;  // unused (uniform K)
  for (int b = 0; b < 2; b++) {
    Step2FArgs& a = h.a[b];
    a.p_in = (const float*)state[b][0];
    a.s_in = (const float*)state[b][1];
    a.p_out = (float*)state[b ^ 1][0];
    a.s_out = (float*)state[b ^ 1][1];
    a.m = (const float*)m;
    a.K = (const float*)K;
    a.Pref = Pref;
    a.PrelF = PrelF;
    a.dPrefF = dPrefF;
    a.diag = nullptr;
    a.err = err_flag;
  }
  cudaError_t e;
  if (tma_ready) {
    // A step launched earlier may still read the old descriptor.
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail_cuda(e, "cudaDeviceSynchronize");
  }
  if (!tma_inst) {
    e = cudaMalloc(&tma_inst, sizeof(InstT));
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(tma)");
    e = cudaMalloc(&tma_counter, sizeof(unsigned int) * SWEEP_COUNTERS);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(tma)");
    e = cudaMemset(tma_counter, 0, sizeof(unsigned int) * SWEEP_COUNTERS);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemset(tma)");
  }
  e = cudaMemcpy(tma_inst, &h, sizeof h, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpy(tma descriptor)");
  if (!tma_items || tma_built_tile_y != ty) {
    // Items ordered z-chunk-major: CTAs that run together work on the same
    // z range, so the halos of neighbouring tiles meet in L2.
    const int ntiles = h.tiles_x * h.tiles_y;
    std::vector<int4> items;
    const long long interior = std::max(p.nz - 2, 1);
    for (int zc = 0; zc < h.nzchunks; zc++)
      for (int t = 0; t < ntiles; t++) {
        const int kb = p.nz == 1 ? 0 : 1 + (int)(zc * interior / h.nzchunks);
        const int ke = p.nz == 1 ? 0 : 1 + (int)((zc + 1) * interior / h.nzchunks);
        items.push_back(make_int4(0, t, kb, ke));
      }
    if (tma_items && (int)items.size() > tma_nitems) {
      cudaFree(tma_items);
      tma_items = nullptr;
    }
    tma_nitems = (int)items.size();
    if (!tma_items) {
      e = cudaMalloc(&tma_items, sizeof(int4) * items.size());
      if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(items)");
    }
    e = cudaMemcpy(tma_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpy(items)");
    tma_grid = std::min(tma_nitems, gmax);
    if (diag_partials && diag_blocks < tma_grid) {
      // The diagnostics partials are sized for the previous grid.
      cudaFree(diag_partials);
      diag_partials = nullptr;
    }
  }
  if (!tma_bitems) {
    std::vector<int2> bitems;
    for (int q = 0; q < h.nbound; q += BOUND_BLOCK) bitems.push_back(make_int2(0, q));
    tma_nbitems = (int)bitems.size();
    e = cudaMalloc(&tma_bitems, sizeof(int2) * bitems.size());
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc(items)");
    e = cudaMemcpy(tma_bitems, bitems.data(), sizeof(int2) * bitems.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpy(items)");
  }
  tma_dt = p.dt;
  tma_S_ref = S_ref;
  tma_built_tile_y = ty;
  tma_ready = true;
  return CAPAZ_OK;
}
