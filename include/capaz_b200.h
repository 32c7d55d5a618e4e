/*
 * capaz_b200.h — C ABI of the Blackwell (sm_100a) implementation of the CAPAZ
 * multiphase-filtration time step.
 *
 * The reference runs one time step as a sequence of stage functions
 * (main.cpp:93-108, declared in defines.h:186-194): S_calculation,
 * ro_P_Xi_calculation, u_calculation, roS_calculation, P_S_calculation and
 * boundary_conditions, each a separate kernel over separately stored arrays
 * (gpu.cu:243-650).  Here the whole step is one fused sweep over the grid:
 * a cell's state (P_w, S_n[, S_w]) makes one HBM round trip per step and every
 * derived quantity (S_w, P_n, rho, Xi, u, roS) lives in registers or shared
 * memory.  Derived fields are materialised on request from the retained
 * previous state (capaz_get_field), so nothing the reference stores is lost.
 *
 * Conventions shared with the reference:
 *   - axes follow the reference: x = i, y = j (vertical; j = 0 is the top
 *     face, gravity acts along +j), z = k (main.cpp:255-267, cpu.cpp:699-705);
 *   - arrays are structure-of-arrays with index i + j*nx + k*nx*ny
 *     (main.cpp:695), float64 at the boundary of this ABI;
 *   - one rank: every cell is active (no_communication.cpp:3-8).
 *
 * Every entry point returns a status code (CAPAZ_OK == 0).  Nothing here
 * calls exit() or throws across the ABI; the reference instead prints and
 * exits (shared_test.cpp:23-33).  A context is not shared between threads.
 */
#ifndef CAPAZ_B200_H
#define CAPAZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CAPAZ_ABI_VERSION 6

/* ---- status codes ------------------------------------------------------ */
enum capaz_status {
  CAPAZ_OK = 0,
  CAPAZ_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad field id, bad value   */
  CAPAZ_ERR_UNSUPPORTED_GRID = 2, /* nx,ny < 3, nz == 2, or too large        */
  CAPAZ_ERR_CUDA = 3,             /* a CUDA runtime call failed              */
  CAPAZ_ERR_OUT_OF_MEMORY = 4,
  CAPAZ_ERR_NO_DEVICE = 5,
  CAPAZ_ERR_NONFINITE = 6,        /* a step produced NaN/Inf (device flag)   */
  CAPAZ_ERR_BAD_STATE = 7,        /* input state outside the model's domain  */
  CAPAZ_ERR_INI = 8,              /* defines.ini could not be read / parsed  */
  CAPAZ_ERR_UNSUPPORTED = 9       /* valid request this build does not do    */
};

/* ---- model / numerical form -------------------------------------------- */
enum capaz_form {
  /* FP64 storage and arithmetic, the reference's operation order, no FMA
   * contraction: matches the reference CPU step (cpu.cpp + two-phase.cpp /
   * three-phase.cpp) to the last bit except where libm and CUDA pow differ. */
  CAPAZ_FORM_FP64 = 0,
  /* FP32 storage of P, S, m, K; FP32 stencil with compensated (Kahan)
   * accumulation of the flux divergence; FP64 delta-form Newton and FP64
   * mass balance. */
  CAPAZ_FORM_FP32C = 1
};

/* Flags (capaz_params.flags). */
#define CAPAZ_FLAG_PERCELL_K 0x1u /* Xi uses K[cell] instead of K0 (extension) */
#define CAPAZ_FLAG_DIAGNOSTICS 0x2u /* reduce mass balance + max residual each step */
/* Three-phase: the top-face source covers only the SOURCE window around the
 * face centre (the two-phase rule, two-phase.cpp:71-77) instead of the whole
 * face (three-phase.cpp:358-362).  Extension. */
#define CAPAZ_FLAG_SOURCE_WINDOW 0x4u
/* Precision form: use the plain-load kernel even where the TMA-staged one
 * applies (nx a multiple of 4).  For comparisons and tests. */
#define CAPAZ_FLAG_NO_TMA 0x8u
/* Test only.  The TMA-staged precision sweep announces 16 bytes more per
 * plane than its copies bring, so every CTA's first bounded wait runs out
 * (about a second): the CTA stops its work, waits (bounded) for its copies
 * in flight and exits, and the step reports CAPAZ_ERR_CUDA.  Exercises the
 * timeout path without a fault or a hang. */
#define CAPAZ_FLAG_TEST_WAIT_TIMEOUT 0x10u
/* FP64 forms with Brooks-Corey index lambda == 2 (two-phase: k_w = S_e^4,
 * k_n = (1-S_e)^2 (1-S_e^2); three-phase with A == 2: the square roots and
 * squares of three-phase.cpp:146-186): the relative permeabilities by
 * products and sqrt instead of pow.  Each value is within a few ulps of the
 * pow form; P and S stay within 1e-12 of the reference (measured).  Ignored
 * for other lambda and in the precision form (which always uses products). */
#define CAPAZ_FLAG_POW_PRODUCTS 0x20u

/*
 * Physical and numerical parameters: the subset of the reference's `consts`
 * (defines.h:79-113) that the time step reads, plus the extensions listed at
 * the end.  Units are SI, as in defines.ini.  Only media 0 is used, as in the
 * reference (two-phase.cpp:6).
 */
typedef struct capaz_params {
  int32_t nx, ny, nz;        /* NX, NY, NZ                                    */
  int32_t phases;            /* 2 (TWO_PHASE) or 3 (THREE_PHASE)              */
  int32_t form;              /* enum capaz_form                               */
  int32_t newton_iterations; /* ITERATIONS                                    */
  int32_t source;            /* SOURCE: half-width of the top source window   */
  uint32_t flags;            /* CAPAZ_FLAG_*                                  */
  double hx, hy, hz, dt;     /* HX, HY, HZ, DT                                */
  double beta_w, beta_n, beta_g; /* BETA_W, BETA_N, BETA_G                    */
  double ro0_w, ro0_n, ro0_g;    /* RO_W, RO_N, RO_G                          */
  double mu_w, mu_n, mu_g;       /* MU_W, MU_N, MU_G                          */
  double g_const, P_atm;     /* G_CONST, P_ATM                                */
  double lambda;             /* LAMBDA_0                                      */
  double S_wr, S_nr, S_gr;   /* S_WR_0, S_NR_0, S_GR_0                        */
  double P_d;                /* P_D_0 (two-phase entry pressure)              */
  double S_n_gr, S_w_gr;     /* S_N_GR, S_W_GR: saturations on the source     */
  double S_w_init, S_n_init; /* S_W_INIT, S_N_INIT (three-phase initial state) */
  double porosity;           /* M_0: porosity used by capaz_init_state        */
  double K0;                 /* K_0: permeability when K is uniform           */
  double timeX;              /* TIMEX (informational)                         */
  /* ---- extensions (neutral values reproduce the reference exactly) ---- */
  double P_top_offset;       /* top-face P_w = P_atm + P_top_offset (0)       */
  double S_n_background;     /* two-phase initial S_n off the source (0)      */
  /* A z-slab of a larger grid (multi-GPU decomposition): the global index of
   * local plane 0 and the global NZ, which place the injection window
   * |k - NZ/2| <= SOURCE in global coordinates.  0, 0: the whole grid. */
  int32_t z_offset;
  int32_t nz_global;
  /* ---- model selection and the Buckley-Leverett task (B_L build,
   * Backley-Leverett/b-l.cpp); read from defines.ini as Q, BACKGROUND_Pw,
   * BACKGROUND_Sn, INJECTION_WELL_Pw, OUTPUT_WELL_Pw (main.cpp:1436-1480) ---- */
  int32_t model;             /* enum capaz_model                              */
  int32_t pad_;
  double Q;                  /* Q: well rate                                  */
  double background_Pw;      /* BACKGROUND_Pw: P_w of the top row at t = 0    */
  double background_Sn;      /* BACKGROUND_Sn: initial S_n                    */
  double injwell_Pw;         /* INJECTION_WELL_Pw                             */
  double outwell_Pw;         /* OUTPUT_WELL_Pw                                */
  double reserved[1];
} capaz_params;

/* Physics of the step (capaz_params.model). */
enum capaz_model {
  CAPAZ_MODEL_DEFAULT = 0, /* two-phase (two-phase.cpp) or three-phase (three-phase.cpp) by `phases` */
  /* Buckley-Leverett task (Backley-Leverett/b-l.cpp): two phases, piecewise
   * relative permeabilities, per-cell K, an injection and a production well
   * in opposite corners of every z-plane; FP64 form only. */
  CAPAZ_MODEL_BUCKLEY_LEVERETT = 1,
  /* Three-phase with the energy equation (THREE_PHASE + ENERGY build:
   * energy.cpp): temperature as a fifth unknown of a 5x5 Newton per cell,
   * temperature-dependent densities and viscosities, heat conduction and
   * advected enthalpy; FP64 form only. */
  CAPAZ_MODEL_ENERGY = 2
};

/* Field identifiers for capaz_set_field / capaz_get_field. */
enum capaz_field {
  /* state (read-write) */
  CAPAZ_FIELD_P_W = 0,
  CAPAZ_FIELD_S_N = 1,
  CAPAZ_FIELD_S_W = 2,  /* state for three-phase; derived (1 - S_n) for two */
  CAPAZ_FIELD_M = 3,    /* porosity per cell                                */
  CAPAZ_FIELD_K = 4,    /* permeability per cell (CAPAZ_FLAG_PERCELL_K)     */
  CAPAZ_FIELD_P_N = 5,  /* derived; three-phase: state on boundary cells    */
  CAPAZ_FIELD_P_G = 6,  /* derived; three-phase: state on boundary cells    */
  /* derived at the start of the last step (read-only), as the reference's
   * arrays hold them after time_step_function returns */
  CAPAZ_FIELD_S_G = 7,
  CAPAZ_FIELD_RO_W = 8,
  CAPAZ_FIELD_RO_N = 9,
  CAPAZ_FIELD_RO_G = 10,
  CAPAZ_FIELD_XI_W = 11,
  CAPAZ_FIELD_XI_N = 12,
  CAPAZ_FIELD_XI_G = 13,
  CAPAZ_FIELD_UX_W = 14, CAPAZ_FIELD_UY_W = 15, CAPAZ_FIELD_UZ_W = 16,
  CAPAZ_FIELD_UX_N = 17, CAPAZ_FIELD_UY_N = 18, CAPAZ_FIELD_UZ_N = 19,
  CAPAZ_FIELD_UX_G = 20, CAPAZ_FIELD_UY_G = 21, CAPAZ_FIELD_UZ_G = 22,
  CAPAZ_FIELD_ROS_W = 23,     /* conserved update before Newton (interior)  */
  CAPAZ_FIELD_ROS_N = 24,
  CAPAZ_FIELD_ROS_G = 25,
  CAPAZ_FIELD_ROS_W_OLD = 26, /* rho*S at the start of the step (interior)  */
  CAPAZ_FIELD_ROS_N_OLD = 27,
  CAPAZ_FIELD_ROS_G_OLD = 28,
  /* energy model (CAPAZ_MODEL_ENERGY) */
  CAPAZ_FIELD_T = 29,      /* temperature (state)                          */
  CAPAZ_FIELD_H_W = 30,    /* enthalpies of the phases and of the rock     */
  CAPAZ_FIELD_H_N = 31,
  CAPAZ_FIELD_H_G = 32,
  CAPAZ_FIELD_H_R = 33,
  CAPAZ_FIELD_E = 34,      /* internal energy per unit volume              */
  CAPAZ_FIELD_E_NEW = 35,  /* energy balance of the step (interior)        */
  CAPAZ_FIELD_COUNT = 36
};

/* Per-step diagnostics (CAPAZ_FLAG_DIAGNOSTICS), reduced on the device with
 * warp shuffles over the interior cells after the step:
 *   mass[p]      = sum over interior cells of m * rho_p(P) * S_p * hx*hy*hz
 *   max_residual = max over interior cells of the Newton residual at the
 *                  final iterate, max_p |F_p| / ro0_p (F_p = rho_p(P) S_p -
 *                  roS_p, the reference's Newton functions) — a saturation-
 *                  equivalent, dimensionless residual;
 *   nonfinite_cells = interior cells whose new P or S is NaN/Inf.
 * The two-phase precision form's tiled sweep (nx a multiple of 4) takes one
 * linearised Newton step and evaluates F_p through the exact identities
 * F_w = A_w e - a_w dP dS, F_n = A_n e + b_n dP dS (e = det * inv - 1 of its
 * solve), to 1e-7 relative. */
typedef struct capaz_diag {
  double mass[3];
  double max_residual;
  double nonfinite_cells;
} capaz_diag;

typedef struct capaz_ctx capaz_ctx;

/* Library / parameters ----------------------------------------------------- */
int capaz_abi_version(void);
/* sizeof(capaz_params) and sizeof(capaz_diag) as compiled into the library,
 * so bindings in other languages can check their struct layouts. */
size_t capaz_params_size(void);
size_t capaz_diag_size(void);
/* Fills the reference's Two-phase/defines.ini defaults for the fields it sets
 * (used where a defines.ini omits a key) and the neutral extension values. */
int capaz_params_default(capaz_params* p);
/* Parses a defines.ini the way read_defines does (main.cpp:1280-1639):
 * "KEY=value" lines, '#' comment lines, the value ending at the first space.
 * Keys not in the file keep their value in *p. */
int capaz_params_from_ini(const char* path, capaz_params* p);
/* Checks a parameter set; returns CAPAZ_OK or the reason it is rejected. */
int capaz_params_validate(const capaz_params* p);

/* Context ------------------------------------------------------------------ */
/* Creates a context on CUDA device `device` and allocates all device memory
 * the step needs (state ping-pong buffers, m, K, derived-field scratch on
 * demand).  On failure returns NULL and writes the reason to *status. */
capaz_ctx* capaz_create(const capaz_params* p, int device, int* status);
int capaz_destroy(capaz_ctx* ctx);
int capaz_get_params(const capaz_ctx* ctx, capaz_params* out);
/* Message for the last error on this context (static storage). */
const char* capaz_last_error(const capaz_ctx* ctx);

/* Host <-> device (float64 host arrays of nx*ny*nz values).  `stream` is a
 * cudaStream_t or NULL for the legacy default stream.  set_field validates the
 * state it receives: m must be > 0 and finite, K > 0 and finite. */
int capaz_set_field(capaz_ctx* ctx, int field, const double* host, void* stream);
int capaz_get_field(capaz_ctx* ctx, int field, double* host, void* stream);
/* Derived fields of an explicitly chosen state: CAPAZ_STATE_STEP_START is
 * the state at the start of the last step (what capaz_get_field uses after
 * a step), CAPAZ_STATE_CURRENT the current state (what the reference's
 * arrays hold between its stage calls, before the Newton stage runs).
 * `dst` is host memory unless dst_on_device is non-zero. */
enum capaz_state_sel { CAPAZ_STATE_STEP_START = 0, CAPAZ_STATE_CURRENT = 1 };
int capaz_get_derived(capaz_ctx* ctx, int field, int state_sel, void* dst, int dst_on_device, void* stream);
/* Device-resident variants: `dev` is a device pointer of the context's device
 * holding nx*ny*nz values: float64 for capaz_set_field_device (either form;
 * the precision form encodes them); float64 for capaz_get_field_device,
 * except m and K of CAPAZ_FORM_FP32C, which come as their float32 storage. */
int capaz_set_field_device(capaz_ctx* ctx, int field, const void* dev, void* stream);
int capaz_get_field_device(capaz_ctx* ctx, int field, void* dev, void* stream);

/* The reference's initial state (two-phase.cpp:113-172, three-phase.cpp:
 * 438-500), computed on the host with the porosity already set in the
 * context (CAPAZ_FIELD_M; M_0 everywhere if never set) and uploaded. */
int capaz_init_state(capaz_ctx* ctx, void* stream);
/* The same initial state on host arrays of nx*ny*nz values, no device
 * involved.  m: in/out — if m_given is 0 it is filled with M_0, else read.
 * Two-phase writes P_w, S_n (S_w, P_n, P_g may be NULL); three-phase writes
 * P_w, S_w, S_n, P_n, P_g. */
int capaz_reference_init(const capaz_params* p, double* m, int m_given, double* P_w, double* S_w,
                         double* S_n, double* P_n, double* P_g);

/* Advances `nsteps` time steps on `stream`; t is not used by the scheme
 * (the reference's roS_calculation ignores it in the NR form).  With
 * CAPAZ_FLAG_DIAGNOSTICS the diagnostics of the last step are kept on the
 * device; capaz_read_diag copies them out (synchronising on `stream`). */
int capaz_step(capaz_ctx* ctx, int nsteps, void* stream);
int capaz_read_diag(capaz_ctx* ctx, capaz_diag* out, void* stream);
/* Pipelined diagnostics.  capaz_post_diag enqueues on `stream` the copy of the
 * last step's diagnostics into slot `slot` (0 <= slot < CAPAZ_DIAG_SLOTS) of a
 * pinned host ring owned by the context and returns without waiting;
 * capaz_wait_diag waits for that slot's copy and returns it.  Posting after
 * step i and waiting for step i - 1 keeps step i queued on the device while
 * the host reads.  Waiting on a slot with no copy posted since its last wait
 * is CAPAZ_ERR_INVALID_ARGUMENT. */
#define CAPAZ_DIAG_SLOTS 4
int capaz_post_diag(capaz_ctx* ctx, int slot, void* stream);
int capaz_wait_diag(capaz_ctx* ctx, int slot, capaz_diag* out);
/* capaz_step followed by capaz_post_diag(slot) in one call (needs
 * CAPAZ_FLAG_DIAGNOSTICS).  In the precision form's TMA-staged sweep the last
 * step writes its reduced diagnostics straight into the ring slot, which saves
 * the copy launch; elsewhere it is the two calls.  capaz_wait_diag(slot)
 * returns them. */
int capaz_step_post_diag(capaz_ctx* ctx, int nsteps, int slot, void* stream);
/* Sets dt for the following steps (a per-step parameter in the reference:
 * consts.dt); host value, no device traffic beyond the kernel argument. */
int capaz_set_dt(capaz_ctx* ctx, double dt);
/* Precision form with the TMA-staged sweep: rows of the sweep's tile, 16
 * (default; four warps per CTA, four CTAs per SM) or 32 (eight warps, two
 * CTAs per SM).  The result does not depend on it.  CAPAZ_ERR_UNSUPPORTED
 * for other values. */
int capaz_set_sweep_tile(capaz_ctx* ctx, int tile_y);

/* ---- ensembles ----------------------------------------------------------
 * A batch steps `count` independent two-phase instances of uneven grid
 * sizes (each with its own parameters, dt, m, K and state) with ONE
 * persistent kernel launch per step: CTAs take (instance, tile, z-chunk)
 * work items from a shared counter.  All instances must share phases (2),
 * form, flags, and the relative-permeability / capillary class (lambda == 2
 * or not, P_d == 0 or not); precision-form batches need nx % 4 == 0.
 * Steps are replayed from a captured CUDA graph.  Fields are read and
 * written through each instance's context (capaz_batch_instance), which the
 * batch owns.  There is no counterpart in the reference (one problem per
 * run, main.cpp:7-79). */
typedef struct capaz_batch capaz_batch;
capaz_batch* capaz_batch_create(const capaz_params* params, int count, int device, int* status);
int capaz_batch_destroy(capaz_batch* b);
capaz_ctx* capaz_batch_instance(capaz_batch* b, int index);
int capaz_batch_step(capaz_batch* b, int nsteps, void* stream);
/* Times candidate launch shapes (z-chunk depth, CTAs per SM and, for the
 * precision form, the sweep's tile: 32 x 16 or 32 x 32 cells) on the batch's
 * own data for a few steps each, keeps the fastest, and restores every
 * instance's state afterwards.  Writes the choice to zchunk / ctas_per_sm
 * (either may be NULL; capaz_batch_get_tuning also returns the tile). */
int capaz_batch_autotune(capaz_batch* b, void* stream, int* zchunk, int* ctas_per_sm);
/* The batch's launch shape: z-chunk depth, CTAs per SM (0: as many as fit)
 * and the precision form's tile rows (16 or 32; 0 for FP64 batches). */
int capaz_batch_get_tuning(const capaz_batch* b, int* zchunk, int* ctas_per_sm, int* tile_y);
/* Sets the launch shape directly (tile_y is ignored for FP64 batches);
 * CAPAZ_ERR_UNSUPPORTED for a tile other than 16 or 32 rows. */
int capaz_batch_set_tuning(capaz_batch* b, int zchunk, int ctas_per_sm, int tile_y);
int64_t capaz_batch_launch_count(const capaz_batch* b);

/* Number of kernels the library launched on this context so far. */
int64_t capaz_launch_count(const capaz_ctx* ctx);
/* Synchronises the context's device and reports any pending CUDA error. */
int capaz_sync(capaz_ctx* ctx);

/* ---- z-slab decomposition (multi-GPU) -----------------------------------
 * One z-plane k of a state field of the current state as float64 in device
 * memory (nx*ny values, index i + j*nx); the precision form decodes /
 * encodes with the context's reference state.  A slab of a decomposed grid
 * (capaz_params.z_offset / nz_global) exchanges its first and last owned
 * planes with its neighbours after every step and writes theirs into its
 * halo planes (P_S_exchange, mpi.cpp:113-294, once per step). */
int capaz_get_plane(capaz_ctx* ctx, int field, int k, double* dst_device, void* stream);
int capaz_set_plane(capaz_ctx* ctx, int field, int k, const double* src_device, void* stream);
/* The same plane in its stored representation, device to device: float64 in
 * the FP64 form, the float32 deviation from the reference state in the
 * precision form (nx*ny values either way).  Slabs whose contexts share one
 * reference state (capaz_set_reference) exchange these bytes unchanged:
 * half the bytes of the float64 planes, and the slabs then step exactly like
 * the undivided grid. */
int capaz_get_plane_raw(capaz_ctx* ctx, int field, int k, void* dst_device, void* stream);
int capaz_set_plane_raw(capaz_ctx* ctx, int field, int k, const void* src_device, void* stream);
/* Two-phase precision form: the reference state (per-row reference pressure,
 * ny values, and reference S_n) against which P_w and S_n are stored.
 * capaz_set_reference fixes it: the current state is re-encoded, and later
 * P_w and S_n (capaz_set_field, capaz_init_state) are encoded against it
 * instead of their own means.  CAPAZ_ERR_UNSUPPORTED for other forms. */
int capaz_get_reference(capaz_ctx* ctx, double* Pref_host, double* S_ref);
int capaz_set_reference(capaz_ctx* ctx, const double* Pref_host, double S_ref);
/* One time step as two sweeps so that a slab's halo exchange overlaps the
 * interior: the edge planes (1 and nz-2, with their boundary cells) on
 * edge_stream, the interior planes on interior_stream.  Each stream first
 * waits for the work queued on the other, so an exchange queued on
 * edge_stream after the previous call has landed before this step reads it.
 * On return the new state is current: its edge planes are final in
 * edge_stream order (read them with capaz_get_plane_raw there and write the
 * received halo planes with capaz_set_plane_raw there), the interior in
 * interior_stream order.  Synchronise both streams (or capaz_sync) before
 * reading whole fields.  Two-phase precision form with the TMA-staged sweep
 * (nx a multiple of 4), nz >= 3, no diagnostics (CAPAZ_ERR_UNSUPPORTED
 * otherwise).  The exchange the reference does with MPI after its stages
 * (mpi.cpp:113-241) becomes one exchange per step that the interior sweep
 * hides. */
int capaz_step_split(capaz_ctx* ctx, void* edge_stream, void* interior_stream);

/* ---- heterogeneous media -------------------------------------------------
 * capaz_read_permeability_file: the permeability file of load_permeability
 * (main.cpp:918-1032, LOAD_K_FROM_FILE): a header "Nx Ny" (nz == 1) or
 * "Nx Ny Nz" that must equal the grid (the reference only warns), then Ny
 * rows of Nx blank-separated values v; K = 1e-10 exp(v) in every z layer.
 * Host only (no context); K receives nx*ny*nz values.  Errors through
 * capaz_last_error(NULL).  capaz_load_permeability reads the file into the
 * context's per-cell K (needs CAPAZ_FLAG_PERCELL_K).
 * capaz_generate_media (no counterpart in the reference): a seeded Gaussian
 * field G with covariance exp(-r/ell) (r in cells) by the randomisation
 * method with `nmodes` Fourier modes, generated on the device; sets
 * K = K_mean exp(sigma G) and porosity = clip(phi0 + dphi G, 0.1, 0.4). */
int capaz_read_permeability_file(const char* path, int nx, int ny, int nz, double* K);
int capaz_load_permeability(capaz_ctx* ctx, const char* path);
int capaz_generate_media(capaz_ctx* ctx, unsigned long long seed, double sigma, double ell, double K_mean,
                         double phi0, double dphi, int nmodes);

/* ---- output and checkpoint files (the reference's formats) --------------
 * capaz_write_plot: the Tecplot point file print_plots writes
 * (main.cpp:549-781), <dir>/S=%012.4f.dat with the reference's header and
 * rows (i outer, j, k; y flipped), `t` the file's time; creates `dir`.
 * Velocities are those of the last step (zero before the first step, as the
 * reference's arrays are).  capaz_save / capaz_restore: save.dat of
 * save/restore (main.cpp:1035-1145): int32 time counter, then nx*ny*nz
 * float64 each of [S_w], P_w, S_n, roS_w_old, roS_n_old, [roS_g_old], m
 * ([..]: three-phase).  Restore reads exactly those sizes (the reference's
 * restore reads locNy*locNy planes) and loads m and the state; three-phase
 * P_n and P_g are set to P_w (the CPU model has no capillary pressure). */
int capaz_write_plot(capaz_ctx* ctx, const char* dir, double t);
int capaz_save(capaz_ctx* ctx, const char* path, int time_counter);
int capaz_restore(capaz_ctx* ctx, const char* path, int* time_counter);

/* ---- differentiation ------------------------------------------------------
 * Discrete adjoint of the two-phase FP64 step (CAPAZ_FORM_FP64 with
 * CAPAZ_FLAG_PERCELL_K).  The misfit is
 *   J = sum over t = obs_every, 2*obs_every, ... <= nsteps and o < nobs of
 *       ((1 - S_n(t, obs_cells[o])) - data[(t/obs_every - 1)*nobs + o])^2,
 * i.e. squared differences of the wetting saturation at the observed cells
 * (flat indices i + j*nx + k*nx*ny, distinct) every obs_every steps.
 * capaz_forward_checkpointed runs nsteps steps of the context (from its
 * current state, or with CAPAZ_ADJ_INIT_FROM_M from data_initialization's
 * state for the context's porosity, which makes that state a function of m),
 * saving the state every checkpoint_every steps; the context is left at
 * step nsteps.  capaz_backward recomputes each checkpoint segment and sweeps
 * it in reverse, giving dJ/d(ln K) and dJ/dm per cell (nx*ny*nz float64 each,
 * host or device destinations; either may be NULL).  The Newton recovery is
 * transposed through the implicit-function theorem at its final iterate.
 * Memory: (ceil(nsteps/checkpoint_every) + checkpoint_every + 12) * 8 bytes
 * per cell, plus the observations. */
#define CAPAZ_ADJ_INIT_FROM_M 0x1
typedef struct capaz_adjoint capaz_adjoint;
capaz_adjoint* capaz_adjoint_create(capaz_ctx* ctx, int nsteps, int checkpoint_every, const long long* obs_cells,
                                    int nobs, int obs_every, int flags, int* status);
int capaz_adjoint_destroy(capaz_adjoint* a);
/* data: (nsteps/obs_every) x nobs float64, zero until set. */
int capaz_adjoint_set_observations(capaz_adjoint* a, const double* data, int on_device, void* stream);
int capaz_forward_checkpointed(capaz_adjoint* a, double* misfit, void* stream);
int capaz_backward(capaz_adjoint* a, double* grad_lnK, double* grad_m, int dst_on_device, void* stream);

/* ---- allocation-free mass balance ----------------------------------------
 * No counterpart in the reference.  Sums, over the interior cells of a
 * two-phase FP64 state held in caller-owned device memory (nz*ny*nx doubles
 * each, the layout of the context fields), the quantities of
 * CAPAZ_FLAG_DIAGNOSTICS: out[0..4] (device memory, the capaz_diag layout)
 * receive mass_w, mass_n, 0, 0 and the count of cells whose P or S is not
 * finite.  All scratch is a fixed device array of the library, so no call
 * allocates memory.  Every call made outside stream capture looks up the
 * scratch address in the current context's copy of the library (a lookup,
 * no allocation); a call on a capturing stream reuses the address of the
 * device's last uncaptured call, so make the first call on a device (with
 * that device current) before any stream capture.  Models other than
 * CAPAZ_MODEL_DEFAULT and CAPAZ_MODEL_BUCKLEY_LEVERETT are rejected with
 * CAPAZ_ERR_UNSUPPORTED; grids with (ny-2)*max(nz-2,1) >
 * CAPAZ_NOALLOC_MAX_ROWS with CAPAZ_ERR_UNSUPPORTED_GRID.  Calls that overlap on one
 * device (other streams or host threads) share the scratch and race: order
 * them.  Errors are reported through capaz_last_error(NULL). */
#define CAPAZ_NOALLOC_MAX_ROWS 131072
int capaz_mass_noalloc(const capaz_params* p, const double* P_w, const double* S_n, const double* m,
                       double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CAPAZ_B200_H */
