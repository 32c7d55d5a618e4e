/*
 * capaz_refabi.h — link-level drop-in for the reference's GPU backend:
 * libcapaz_dropin_2ph.so for the two-phase build, libcapaz_dropin_3ph.so
 * (this header with CAPAZ_REFABI_THREE_PHASE defined) for the three-phase
 * build.
 *
 * The reference's host program (main.cpp + no_communication.cpp +
 * shared_test.cpp + gauss.cpp, built with -D TWO_PHASE or -D THREE_PHASE)
 * links one
 * architecture backend: cpu.cpp or the CUDA object gpu.o (sh/run.sh:98-112,
 * 165).  This library exports, with C++ linkage and the reference's
 * signatures (defines.h:115-207), every symbol the host program takes from
 * that backend, so it links in place of gpu.o.  Each stage function runs on
 * the C ABI of include/capaz_b200.h; the whole step is one fused kernel.
 *
 * The two structs below must have the reference's member order and types
 * (defines.h:65-76 and 79-113 with TWO_PHASE or THREE_PHASE defined, ENERGY
 * undefined) so that structs passed by value between the reference's
 * objects and this library agree byte for byte: sizeof(ptr_Arrays) == 160,
 * sizeof(consts) == 384 (two-phase), 232 and 488 (three-phase) on x86-64.
 *
 * Semantics, compared with the reference's gpu.cu:
 *   - device_initialization creates the context (device = rank % devices,
 *     gpu.cu:770-771) from the constants in `def`, which are fixed from then
 *     on, as the reference's __constant__ copy is (gpu.cu:792-795).
 *   - The Dev arrays returned by device_memory_allocation are real device
 *     arrays of locNx*locNy*locNz doubles; the state itself lives in the
 *     context.  load_data_to_device / load_data_to_host move values between
 *     host, those arrays and the context, so a host program that touches
 *     device data only through them, as the reference's does, sees the
 *     reference's values.
 *   - The stages of time_step_function (main.cpp:93-108) are accepted in the
 *     reference's order; P_S_calculation launches the fused step (flux,
 *     Newton and boundary update together) and boundary_conditions closes
 *     it.  A stage called out of that order is an error.
 *   - Derived arrays (S_w, P_n, ro, Xi, u, roS, roS_old) are computed when
 *     downloaded, from the state the reference's array would reflect.
 *   - K: the two-phase physics uses K_0 from defines.ini (two-phase.cpp:16-17),
 *     not the K array, exactly as the reference does.
 *   - Errors print "Error: ..." and exit(1), as print_error does
 *     (shared_test.cpp:23-33).  One rank only: the halo pack/unpack
 *     functions report an error if called.
 */
#ifndef CAPAZ_REFABI_H
#define CAPAZ_REFABI_H
/* Three-phase (libcapaz_dropin_3ph.so): the CPU model's physics, capillary
 * pressures zero and K_0 throughout (three-phase.cpp), the whole top face a
 * source when SOURCE > 0, as the reference's CPU backend computes it; the
 * reference's GPU three-phase code differs from its CPU code, and the CPU
 * code is the one followed. */

/* defines.h:65-76. */
struct ptr_Arrays_tag {
  double *S_n, *S_w, *P_w, *P_n, *ro_w, *ro_n, *ux_w, *uy_w, *uz_w, *ux_n, *uy_n, *uz_n, *Xi_w, *Xi_n, *roS_w,
      *roS_w_old, *roS_n, *roS_n_old;
  double *m, *K;
#ifdef CAPAZ_REFABI_THREE_PHASE
  double *S_g, *P_g, *ro_g, *ux_g, *uy_g, *uz_g, *Xi_g, *roS_g, *roS_g_old;
#endif
};
typedef struct ptr_Arrays_tag ptr_Arrays;

/* defines.h:79-113. */
struct consts_tag {
  double upscale_l, upscale_t;
  double lambda[2];
  double S_wr[2];
  double porosity[2];
  double hx, hy, hz, dt, tau, l, c_w, c_n, beta_w, beta_n, P_atm, g_const, mu_w, mu_n, ro0_w, ro0_n, timeX;
  double S_n_gr;
  int Nx, Ny, Nz;
  int source, save_plots, print_screen, newton_iterations;
  double K[2];
  double Q, InjWell_Pw, InjWell_Sn, OutWell_Pw, OutWell_Sn, Background_Sn, Background_Pw;
#ifdef CAPAZ_REFABI_THREE_PHASE
  double S_w_init, S_n_init;
  double S_nr[2];
  double S_gr[2];
  double P_d_nw[2];
  double P_d_gn[2];
  double c_g, beta_g, mu_g, ro0_g, S_w_gr;
#else
  double P_d[2];
#endif
  int locNx, locNy, locNz;
  int size, rank;
  int sizex, sizey, sizez;
  int rankx, ranky, rankz;
  int blocksX, blocksY, blocksZ;
};
typedef struct consts_tag consts;

/* Stage functions (defines.h:186-194), replacing gpu.cu:243-258, 402-407,
 * 428-433, 629-650. */
void S_calculation(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, consts def);
void ro_P_Xi_calculation(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, consts def);
void u_calculation(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, consts def);
void roS_calculation(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, double t, consts def);
void P_S_calculation(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, consts def);
void boundary_conditions(ptr_Arrays HostArraysPtr, ptr_Arrays DevArraysPtr, consts def);

/* Memory (defines.h:121,124,134-136), replacing gpu.cu:653-758. */
void device_memory_allocation(ptr_Arrays* ArraysPtr, double** DevBuffer, consts def);
void device_memory_free(ptr_Arrays DevArraysPtr, double* DevBuffer);
void load_data_to_host(double* HostArrayPtr, double* DevArrayPtr, consts def);
void load_data_to_device(double* HostArrayPtr, double* DevArrayPtr, consts def);
void load_data_to_device_int(int* HostArrayPtr, int* DevArrayPtr, consts def);

/* Device set-up (defines.h:138-139), replacing gpu.cu:763-852. */
void device_initialization(consts* def);
void device_finalization(void);

/* Initial state on the host arrays (defines.h:126), replacing the GPU
 * build's copy in two-phase.cu:6-65 (three-phase: three-phase.cpp:438-500,
 * the CPU model's). */
void data_initialization(ptr_Arrays HostArraysPtr, long int* time_counter, consts def);

/* Halo pack/unpack for multi-rank backends (defines.h:196-207), replacing
 * gpu.cu:926-990, 1064-1128.  One rank only here: calling them is an error. */
void load_exchange_data_part_xl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void load_exchange_data_part_xr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void load_exchange_data_part_yl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void load_exchange_data_part_yr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void load_exchange_data_part_zl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void load_exchange_data_part_zr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_xl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_xr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_yl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_yr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_zl(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);
void save_exchange_data_part_zr(double* HostArrayPtr, double* DevArrayPtr, double* HostBuffer, double* DevBuffer, consts def);

/* CUDA error check helper of the GPU build (shared_test.cu:5-25). */
void checkErrors(char* label, char* file, int line);

#endif /* CAPAZ_REFABI_H */
