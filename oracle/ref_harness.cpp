// Test harness for the reference CPU implementation (oracle/_ref only).
//
// This file is test infrastructure: it is linked against the reference's own,
// unmodified sources (main.cpp with `main` renamed, cpu.cpp, the phase module,
// no_communication.cpp, shared_test.cpp, gauss.cpp) by oracle/Makefile, and it
// drives the reference's own `time_step_function` (main.cpp:93-108).  It is
// never part of the product.  The same harness can instead be linked against
// the product's drop-in library (libcapaz_dropin_2ph.so) in place of cpu.cpp,
// which is how the link-level drop-in is checked.
//
// Usage:
//   capaz_ref_<task> <workdir> <nsteps> [<state_in.bin>|-] [<state_out.bin>|-]
//                    [<derived_out.bin>]
//
// <workdir> must contain defines.ini.  The harness changes into <workdir>/run
// (created if needed) so the reference's read_defines (main.cpp:1280-1297),
// which first tries "..//defines.ini", reads <workdir>/defines.ini.
//
// State files are raw little-endian float64 arrays of locNx*locNy*locNz
// values each, x fastest (index i + j*Nx + k*Nx*Ny, main.cpp:695):
//   two-phase   in:  P_w, S_n, m               out: P_w, S_n
//   three-phase in:  P_w, S_w, S_n, P_n, P_g, m out: P_w, S_w, S_n, P_n, P_g
//   three-phase with ENERGY: T appended to both (in after m)
// With "-" as <state_in.bin> the reference's own data_initialization is used.
// <derived_out.bin> receives the reference's other per-cell arrays as they
// stand after the last step, in this order:
//   two-phase   S_w P_n ro_w ro_n ux_w uy_w uz_w ux_n uy_n uz_n Xi_w Xi_n
//               roS_w roS_w_old roS_n roS_n_old
//   three-phase the same, then S_g ro_g ux_g uy_g uz_g Xi_g roS_g roS_g_old
//   with ENERGY then H_w H_n H_g H_r E E_new
//
// On success one line "RESULT {json}" is printed with the cell count, the step
// count and the wall time of the step loop alone (CLOCK_MONOTONIC).
#include "defines.h"

#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

extern double* DevBuffer;  // defined in main.cpp

static double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int read_fields(const char* path, double** dst, int nf, long n) {
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  for (int a = 0; a < nf; a++) {
    if (fread(dst[a], sizeof(double), (size_t)n, f) != (size_t)n) {
      fclose(f);
      return 2;
    }
  }
  fclose(f);
  return 0;
}

static int write_fields(const char* path, double** src, int nf, long n) {
  FILE* f = fopen(path, "wb");
  if (!f) return 1;
  for (int a = 0; a < nf; a++) {
    if (fwrite(src[a], sizeof(double), (size_t)n, f) != (size_t)n) {
      fclose(f);
      return 2;
    }
  }
  fclose(f);
  return 0;
}

int main(int argc, char* argv[]) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <workdir> <nsteps> [state_in|-] [state_out|-]\n", argv[0]);
    return 2;
  }
  const char* workdir = argv[1];
  long nsteps = atol(argv[2]);
  const char* in_path = (argc > 3 && strcmp(argv[3], "-") != 0) ? argv[3] : NULL;
  const char* out_path = (argc > 4 && strcmp(argv[4], "-") != 0) ? argv[4] : NULL;
  const char* derived_path = (argc > 5) ? argv[5] : NULL;

  char rundir[4096];
  snprintf(rundir, sizeof rundir, "%s/run", workdir);
  mkdir(rundir, 0777);
  if (chdir(rundir) != 0) {
    fprintf(stderr, "cannot enter %s\n", rundir);
    return 2;
  }

  consts def;
  memset(&def, 0, sizeof def);
  ptr_Arrays H, D;
  memset(&H, 0, sizeof H);
  memset(&D, 0, sizeof D);
  long int time_counter = 0;

  // main.cpp:14-28, without the plot output.
  int fake_argc = 1;
  char* fake_argv[] = {argv[0], NULL};
  read_defines(fake_argc, fake_argv, &def);
  initialization(&H, &D, &time_counter, fake_argc, fake_argv, &def);

  long n = (long)def.locNx * def.locNy * def.locNz;
#if defined(THREE_PHASE) && defined(ENERGY)
  double* in_f[] = {H.P_w, H.S_w, H.S_n, H.P_n, H.P_g, H.m, H.T};
  double* dev_in[] = {D.P_w, D.S_w, D.S_n, D.P_n, D.P_g, D.m, D.T};
  double* out_f[] = {H.P_w, H.S_w, H.S_n, H.P_n, H.P_g, H.T};
  double* dev_out[] = {D.P_w, D.S_w, D.S_n, D.P_n, D.P_g, D.T};
  const int nin = 7, nout = 6;
#elif defined(THREE_PHASE)
  double* in_f[] = {H.P_w, H.S_w, H.S_n, H.P_n, H.P_g, H.m};
  double* dev_in[] = {D.P_w, D.S_w, D.S_n, D.P_n, D.P_g, D.m};
  double* out_f[] = {H.P_w, H.S_w, H.S_n, H.P_n, H.P_g};
  double* dev_out[] = {D.P_w, D.S_w, D.S_n, D.P_n, D.P_g};
  const int nin = 6, nout = 5;
#else
  double* in_f[] = {H.P_w, H.S_n, H.m};
  double* dev_in[] = {D.P_w, D.S_n, D.m};
  double* out_f[] = {H.P_w, H.S_n};
  double* dev_out[] = {D.P_w, D.S_n};
  const int nin = 3, nout = 2;
#endif
  if (in_path) {
    int rc = read_fields(in_path, in_f, nin, n);
    if (rc) {
      fprintf(stderr, "cannot read state %s (%d)\n", in_path, rc);
      return 3;
    }
    // Same uploads as main.cpp:329-339 (no-ops in the CPU build).
    for (int a = 0; a < nin; a++) load_data_to_device(in_f[a], dev_in[a], def);
  }

  double t0 = now_s();
  for (long s = 1; s <= nsteps; s++) {
    time_step_function(H, D, DevBuffer, def, s * def.dt);
  }
  for (int a = 0; a < nout; a++) load_data_to_host(out_f[a], dev_out[a], def);
  double t1 = now_s();

  if (out_path) {
    int rc = write_fields(out_path, out_f, nout, n);
    if (rc) {
      fprintf(stderr, "cannot write state %s (%d)\n", out_path, rc);
      return 4;
    }
  }
  if (derived_path) {
    double* der[] = {H.S_w, H.P_n, H.ro_w, H.ro_n, H.ux_w, H.uy_w, H.uz_w, H.ux_n, H.uy_n, H.uz_n,
                     H.Xi_w, H.Xi_n, H.roS_w, H.roS_w_old, H.roS_n, H.roS_n_old
#ifdef THREE_PHASE
                     , H.S_g, H.ro_g, H.ux_g, H.uy_g, H.uz_g, H.Xi_g, H.roS_g, H.roS_g_old
#endif
#ifdef ENERGY
                     , H.H_w, H.H_n, H.H_g, H.H_r, H.E, H.E_new
#endif
    };
    double* dder[] = {D.S_w, D.P_n, D.ro_w, D.ro_n, D.ux_w, D.uy_w, D.uz_w, D.ux_n, D.uy_n, D.uz_n,
                      D.Xi_w, D.Xi_n, D.roS_w, D.roS_w_old, D.roS_n, D.roS_n_old
#ifdef THREE_PHASE
                      , D.S_g, D.ro_g, D.ux_g, D.uy_g, D.uz_g, D.Xi_g, D.roS_g, D.roS_g_old
#endif
#ifdef ENERGY
                      , D.H_w, D.H_n, D.H_g, D.H_r, D.E, D.E_new
#endif
    };
    const int nd = (int)(sizeof der / sizeof der[0]);
    for (int a = 0; a < nd; a++) load_data_to_host(der[a], dder[a], def);
    int rc = write_fields(derived_path, der, nd, n);
    if (rc) {
      fprintf(stderr, "cannot write derived %s (%d)\n", derived_path, rc);
      return 4;
    }
  }
  printf("RESULT {\"nx\": %d, \"ny\": %d, \"nz\": %d, \"cells\": %ld, \"steps\": %ld, \"seconds\": %.9f}\n",
         def.locNx, def.locNy, def.locNz, n, nsteps, t1 - t0);
  fflush(stdout);
  finalization(H, D, DevBuffer);
  return 0;
}
