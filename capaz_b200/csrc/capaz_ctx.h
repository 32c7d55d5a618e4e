// The context behind the opaque capaz_ctx handle of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "capaz_internal.h"

struct capaz_ctx {
  capaz_params p;
  int device = 0;
  long long n = 0;
  // State ping-pong buffers: state[buffer][slot], slots P_w, S_n, S_w, P_n,
  // P_g (the last three for three-phase only), T (energy model).  `cur`
  // holds the current state; after a step the other buffer holds the
  // start-of-step state, from which derived fields are materialised.  The
  // energy model steps buffer `cur` in place and keeps the reference's other
  // arrays of the last step in `ework` (EW_COUNT fields).
  void* state[2][6] = {{nullptr}};
  double* ework = nullptr;
  int cur = 0;
  long long steps_done = 0;
  void* m = nullptr;
  void* K = nullptr;
  unsigned int* err_flag = nullptr;  // set by kernels on non-finite results
  double* diag_partials = nullptr;   // per-block diagnostics
  int diag_blocks = 0;
  double* diag_out = nullptr;        // reduced diagnostics (DIAG_STRIDE)
  // Pinned host ring of diagnostics copies: CAPAZ_DIAG_SLOTS posted slots and
  // one more for capaz_read_diag; an event marks each slot's copy.
  double* diag_host = nullptr;      // mapped: diag_host_dev is its device view
  double* diag_host_dev = nullptr;
  cudaEvent_t diag_ev[CAPAZ_DIAG_SLOTS + 1] = {};
  bool diag_posted[CAPAZ_DIAG_SLOTS + 1] = {};
  // Set by step_post_diag for the next step() call: where the last step's
  // sweep also writes its reduced diagnostics (mapped pinned memory), and
  // whether it did.
  double* publish_to = nullptr;
  bool published = false;
  double* scratch = nullptr;         // one float64 field, derived fields
  void* host_stage = nullptr;
  // Precision form: state stored as FP32 deviations from P_ref(j) and S_ref.
  double* Pref = nullptr;    // ny
  float* PrelF = nullptr;    // ny: Pref - P_atm
  float* dPrefF = nullptr;   // ny: Pref[j+1] - Pref[j]
  double S_ref = 0.;    // S_n reference
  double S_ref_w = 0.;  // S_w reference (three-phase)
  // FP64 decode scratch: P_w, S_n, m, K, then S_w, P_n, P_g (three-phase).
  double* wide[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // TMA path of the precision form.
  capaz::InstT* tma_inst = nullptr;  // device descriptor
  int4* tma_items = nullptr;
  int tma_nitems = 0;
  unsigned int* tma_counter = nullptr;  // SWEEP_COUNTERS words
  int2* tma_bitems = nullptr;  // boundary-kernel blocks
  int tma_nbitems = 0;
  double tma_dt = 0., tma_S_ref = 0.;  // values baked into the descriptor
  float4* rowF = nullptr;              // per-row tables (precision form)
  bool tma_applies() const;
  int tma_grid = 0;
  // TMA path of the three-phase precision form: arguments per state parity.
  // A reference state fixed by capaz_set_reference: P_w and S_n are then
  // encoded against it instead of their own means.
  bool ref_locked = false;
  // capaz_step_split: work items of the edge planes (1, nz-2) then of the
  // interior planes, their counters (SWEEP_COUNTERS words each), events.
  int4* split_items = nullptr;
  int split_nedge = 0, split_nint = 0, split_tile_y = 0, split_grid_e = 0, split_grid_i = 0;
  unsigned int* split_counters = nullptr;
  cudaEvent_t split_ev[2] = {nullptr, nullptr};
  bool counters_dirty = false;  // a split step ran: rezero the single-launch counters
  int step_split(cudaStream_t edge, cudaStream_t interior);
  capaz::Step3TArgs t3a[2];
  bool t3_ready = false;
  unsigned int* t3_counter = nullptr;
  int t3_grid = 0;
  int tma_tile_y = capaz::TMA_TILE_Y;  // rows of a sweep tile (16 or 32)
  int tma_built_tile_y = 0;            // the tile the descriptor and item list were built for
  bool tma_ready = false;
  int tma_prepare();
  double* stage = nullptr;           // float64 staging of set_field
  unsigned long long* first_bad = nullptr;  // validation result
  double* sum_parts = nullptr;       // 1024 partial sums (S_ref)
  double* S_ref_dev = nullptr;
  long long launches = 0;
  bool defaults_unchecked = false;   // set while allocate() stores the defaults
  std::string last_error;

  static int state_slot(int field) {
    switch (field) {
      case CAPAZ_FIELD_P_W: return 0;
      case CAPAZ_FIELD_S_N: return 1;
      case CAPAZ_FIELD_S_W: return 2;
      case CAPAZ_FIELD_P_N: return 3;
      case CAPAZ_FIELD_P_G: return 4;
      case CAPAZ_FIELD_T: return 5;
      default: return -1;
    }
  }

  int allocate();
  void release();
  int ensure_scratch();
  int set_field(int field, const void* src, bool on_device, cudaStream_t s);
  int get_field(int field, void* dst, bool on_device, cudaStream_t s);
  // Materialises derived `field` into scratch from the start-of-step state
  // (from_current == false; the current state before any step) or from the
  // current state.
  int derived(int field, cudaStream_t s, bool from_current = false);
  int init_state(cudaStream_t s);
  int get_derived(int field, bool from_current, void* dst, bool on_device, cudaStream_t s);
  int step(int nsteps, cudaStream_t s);
  int read_diag(capaz_diag* out, cudaStream_t s);
  int post_diag(int slot, cudaStream_t s);
  int step_post_diag(int nsteps, int slot, cudaStream_t s);
  int wait_diag(int slot, capaz_diag* out);
  int check_flag();
  // Precision form: FP64 view of (P_w, S_n, m, K) of state buffer b.
  int decode_all(int b, cudaStream_t s);
  int sync();
  int fail_cuda(cudaError_t e, const char* what);
  int fail_msg(int code, const char* msg);
};

namespace capaz {
Step2Const make_step2_const(const capaz_params& p);
BLConst make_bl_const(const capaz_params& p);
Step2FConst make_step2f_const(const capaz_params& p, double S_ref);
Step3Const make_step3_const(const capaz_params& p);
Step3FConst make_step3f_const(const capaz_params& p, double S_ref_w, double S_ref_n);
PhysF make_physf(const capaz_params& p);
void reference_init_host(const capaz_params& p, const double* m, double* Pw, double* Sw, double* Sn, double* Pn,
                         double* Pg);
}
