// Link-level drop-in for the reference's GPU backend: the reference's
// stage/memory/device call surface (include/capaz_refabi.h) on top of the C
// ABI (include/capaz_b200.h).  Built twice: libcapaz_dropin_2ph.so, and
// libcapaz_dropin_3ph.so with CAPAZ_REFABI_THREE_PHASE defined (the
// reference's THREE_PHASE struct layouts and the three-phase step).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "capaz_b200.h"
#include "capaz_refabi.h"

#ifdef CAPAZ_REFABI_THREE_PHASE
static_assert(sizeof(ptr_Arrays) == 232, "ptr_Arrays layout must match the reference (three-phase)");
static_assert(sizeof(consts) == 488, "consts layout must match the reference (three-phase)");
constexpr int kPhases = 3;
#define CAPAZ_DROPIN_LIB "libcapaz_dropin_3ph"
#else
static_assert(sizeof(ptr_Arrays) == 160, "ptr_Arrays layout must match the reference (two-phase)");
static_assert(sizeof(consts) == 384, "consts layout must match the reference (two-phase)");
constexpr int kPhases = 2;
#define CAPAZ_DROPIN_LIB "libcapaz_dropin_2ph"
#endif

namespace {

// Stages of time_step_function (main.cpp:95-107) in the order they run.
enum Stage { IDLE = 0, AFTER_S, AFTER_RO_P_XI, AFTER_U, AFTER_ROS, AFTER_P_S };

struct DropIn {
  capaz_ctx* ctx = nullptr;
  capaz_params p;
  long long n = 0;
  int device = 0;
  Stage stage = IDLE;
  long long steps = 0;     // fused steps run
  bool stepping = false;   // a step's stages have started since device set-up
  // Device arrays handed to the host program, by reference field.
  struct Handle {
    double* dev;
    int field;  // capaz field id, or -1 for arrays with no meaning here
  };
  std::vector<Handle> handles;
};

DropIn g;

[[noreturn]] void die(const char* msg, int line) {
  // Same shape and exit status as print_error (shared_test.cpp:23-33).
  printf("Error: %s\nFile: \"%s\"\nLine: %d\n\n", msg, __FILE__, line);
  fflush(stdout);
  exit(1);
}

void check(int st, const char* what, int line) {
  if (st != CAPAZ_OK) {
    char buf[600];
    snprintf(buf, sizeof buf, "%s failed (%d): %s", what, st, capaz_last_error(g.ctx));
    die(buf, line);
  }
}

void check_cuda(cudaError_t e, const char* what, int line) {
  if (e != cudaSuccess) {
    char buf[600];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    die(buf, line);
  }
}

capaz_params params_from(const consts& def) {
  capaz_params p;
  capaz_params_default(&p);
  p.nx = def.locNx;
  p.ny = def.locNy;
  p.nz = def.locNz;
  p.phases = kPhases;
  p.form = CAPAZ_FORM_FP64;
  p.newton_iterations = def.newton_iterations;
  p.source = def.source;
  p.flags = 0;
  p.hx = def.hx;
  p.hy = def.hy;
  p.hz = def.hz;
  p.dt = def.dt;
  p.beta_w = def.beta_w;
  p.beta_n = def.beta_n;
  p.ro0_w = def.ro0_w;
  p.ro0_n = def.ro0_n;
  p.mu_w = def.mu_w;
  p.mu_n = def.mu_n;
  p.g_const = def.g_const;
  p.P_atm = def.P_atm;
  p.lambda = def.lambda[0];
  p.S_wr = def.S_wr[0];
#ifdef CAPAZ_REFABI_THREE_PHASE
  // The CPU three-phase model has no capillary pressure (P_D_NW, P_D_GN unused).
  p.P_d = 0.;
  p.S_nr = def.S_nr[0];
  p.S_gr = def.S_gr[0];
  p.S_w_init = def.S_w_init;
  p.S_n_init = def.S_n_init;
  p.beta_g = def.beta_g;
  p.mu_g = def.mu_g;
  p.ro0_g = def.ro0_g;
  p.S_w_gr = def.S_w_gr;
#else
  p.P_d = def.P_d[0];
#endif
  p.S_n_gr = def.S_n_gr;
  p.porosity = def.porosity[0];
  p.K0 = def.K[0];
  p.timeX = def.timeX;
  p.P_top_offset = 0.;
  p.S_n_background = 0.;
  return p;
}

void require_one_rank(const consts& def, int line) {
  if (def.size > 1 || def.sizex > 1 || def.sizey > 1 || def.sizez > 1)
    die(CAPAZ_DROPIN_LIB " runs one rank (link no_communication.cpp)", line);
}

// Fields the context holds as state or media (set on upload).
bool is_state_or_media(int f) {
  if (f == CAPAZ_FIELD_P_W || f == CAPAZ_FIELD_S_N || f == CAPAZ_FIELD_M) return true;
  return kPhases == 3 && (f == CAPAZ_FIELD_S_W || f == CAPAZ_FIELD_P_N || f == CAPAZ_FIELD_P_G);
}

int field_of(const double* dev) {
  for (const auto& h : g.handles)
    if (h.dev == dev) return h.field;
  return -2;  // not one of ours
}

void advance(Stage from, Stage to, const char* name, int line) {
  // roS_calculation may follow ro_P_Xi_calculation directly (u is not used
  // by the NR scheme); every other stage must follow its predecessor.
  bool ok = (g.stage == from) || (to == AFTER_ROS && g.stage == AFTER_RO_P_XI);
  if (!ok) {
    char buf[300];
    snprintf(buf, sizeof buf,
             "%s called out of the order of time_step_function (main.cpp:93-108); "
             "this backend runs the step as one fused kernel",
             name);
    die(buf, line);
  }
  g.stage = to;
}

}  // namespace

// ---------------------------------------------------------------------------
void device_initialization(consts* def) {
  require_one_rank(*def, __LINE__);
  int ndev = 0;
  check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount", __LINE__);
  if (ndev <= 0) die("no CUDA device", __LINE__);
  g.device = def->rank % ndev;
  check_cuda(cudaSetDevice(g.device), "cudaSetDevice", __LINE__);
  // Thread-block counts as the reference computes them (gpu.cu:776-790);
  // the fused kernel chooses its own launch shape.
  def->blocksX = (def->locNx + 7) / 8;
  def->blocksY = (def->locNy + 7) / 8;
  def->blocksZ = (def->locNz + 7) / 8;
  g.p = params_from(*def);
  int st = 0;
  g.ctx = capaz_create(&g.p, g.device, &st);
  check(st, "capaz_create", __LINE__);
  g.n = (long long)def->locNx * def->locNy * def->locNz;
  g.stage = IDLE;
  if (def->rank == 0) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, g.device) == cudaSuccess) {
      printf("Name : %s\nCompute capability : %d.%d\nTotal Global Memory : %zu\n"
             "Number of multiprocessors: %d\n",
             prop.name, prop.major, prop.minor, prop.totalGlobalMem, prop.multiProcessorCount);
      fflush(stdout);
    }
  }
}

void device_finalization(void) {
  if (g.ctx) capaz_sync(g.ctx);
}

void device_memory_allocation(ptr_Arrays* A, double** DevBuffer, consts def) {
  require_one_rank(def, __LINE__);
  if (!g.ctx) die("device_initialization must run first", __LINE__);
  const size_t bytes = (size_t)g.n * sizeof(double);
  struct Slot {
    double** ptr;
    int field;
  } slots[] = {
      {&A->P_w, CAPAZ_FIELD_P_W},       {&A->P_n, CAPAZ_FIELD_P_N},       {&A->S_n, CAPAZ_FIELD_S_N},
      {&A->S_w, CAPAZ_FIELD_S_W},       {&A->ro_w, CAPAZ_FIELD_RO_W},     {&A->ro_n, CAPAZ_FIELD_RO_N},
      {&A->ux_w, CAPAZ_FIELD_UX_W},     {&A->uy_w, CAPAZ_FIELD_UY_W},     {&A->uz_w, CAPAZ_FIELD_UZ_W},
      {&A->ux_n, CAPAZ_FIELD_UX_N},     {&A->uy_n, CAPAZ_FIELD_UY_N},     {&A->uz_n, CAPAZ_FIELD_UZ_N},
      {&A->Xi_w, CAPAZ_FIELD_XI_W},     {&A->Xi_n, CAPAZ_FIELD_XI_N},     {&A->roS_w, CAPAZ_FIELD_ROS_W},
      {&A->roS_n, CAPAZ_FIELD_ROS_N},   {&A->roS_w_old, CAPAZ_FIELD_ROS_W_OLD},
      {&A->roS_n_old, CAPAZ_FIELD_ROS_N_OLD}, {&A->m, CAPAZ_FIELD_M},
      // K: the physics reads K_0 (two-phase.cpp:16-17, three-phase.cpp:220-222),
      // so the K array is kept but does not reach the step, as in the reference.
      {&A->K, -1},
#ifdef CAPAZ_REFABI_THREE_PHASE
      {&A->S_g, CAPAZ_FIELD_S_G},       {&A->P_g, CAPAZ_FIELD_P_G},       {&A->ro_g, CAPAZ_FIELD_RO_G},
      {&A->ux_g, CAPAZ_FIELD_UX_G},     {&A->uy_g, CAPAZ_FIELD_UY_G},     {&A->uz_g, CAPAZ_FIELD_UZ_G},
      {&A->Xi_g, CAPAZ_FIELD_XI_G},     {&A->roS_g, CAPAZ_FIELD_ROS_G},   {&A->roS_g_old, CAPAZ_FIELD_ROS_G_OLD},
#endif
  };
  g.handles.clear();
  for (auto& s : slots) {
    void* d = nullptr;
    check_cuda(cudaMalloc(&d, bytes), "cudaMalloc", __LINE__);
    check_cuda(cudaMemset(d, 0, bytes), "cudaMemset", __LINE__);
    *s.ptr = static_cast<double*>(d);
    g.handles.push_back({static_cast<double*>(d), s.field});
  }
  if (DevBuffer) *DevBuffer = nullptr;  // no halo buffer on one rank
}

void device_memory_free(ptr_Arrays DevArraysPtr, double* DevBuffer) {
  (void)DevArraysPtr;
  for (auto& h : g.handles) cudaFree(h.dev);
  g.handles.clear();
  if (DevBuffer) cudaFree(DevBuffer);
  if (g.ctx) capaz_destroy(g.ctx);
  g.ctx = nullptr;
}

void load_data_to_device(double* HostArrayPtr, double* DevArrayPtr, consts def) {
  (void)def;
  const size_t bytes = (size_t)g.n * sizeof(double);
  check_cuda(cudaMemcpy(DevArrayPtr, HostArrayPtr, bytes, cudaMemcpyHostToDevice), "copy double data to device",
             __LINE__);
  const int f = field_of(DevArrayPtr);
  if (is_state_or_media(f))
    check(capaz_set_field_device(g.ctx, f, DevArrayPtr, nullptr), "capaz_set_field_device", __LINE__);
}

void load_data_to_device_int(int* HostArrayPtr, int* DevArrayPtr, consts def) {
  (void)def;
  check_cuda(cudaMemcpy(DevArrayPtr, HostArrayPtr, (size_t)g.n * sizeof(int), cudaMemcpyHostToDevice),
             "copy int data to device", __LINE__);
}

void load_data_to_host(double* HostArrayPtr, double* DevArrayPtr, consts def) {
  (void)def;
  const size_t bytes = (size_t)g.n * sizeof(double);
  const int f = field_of(DevArrayPtr);
  const bool state_or_media = is_state_or_media(f);
  // Before the first stage call the reference's derived arrays hold what
  // the allocation left there (the handles are zeroed) or what the host
  // uploaded; they are computed only once a step has begun.
  if (f >= 0 && (state_or_media || g.stepping)) {
    // Before the Newton stage of a step has run, the reference's derived
    // arrays describe the current state; otherwise the start of the last step.
    const int sel = (g.stage == IDLE || g.stage == AFTER_P_S) ? CAPAZ_STATE_STEP_START : CAPAZ_STATE_CURRENT;
    check(capaz_get_derived(g.ctx, f, sel, DevArrayPtr, 1, nullptr), "capaz_get_derived", __LINE__);
  }
  check_cuda(cudaMemcpy(HostArrayPtr, DevArrayPtr, bytes, cudaMemcpyDeviceToHost), "copy data to host", __LINE__);
  if (g.ctx) check(capaz_sync(g.ctx), "capaz_sync", __LINE__);
}

void data_initialization(ptr_Arrays H, long int* time_counter, consts def) {
  require_one_rank(def, __LINE__);
  *time_counter = 0;
  capaz_params p = params_from(def);
  const long long n = (long long)def.locNx * def.locNy * def.locNz;
#ifdef CAPAZ_REFABI_THREE_PHASE
  check(capaz_reference_init(&p, H.m, 0, H.P_w, H.S_w, H.S_n, H.P_n, H.P_g), "capaz_reference_init", __LINE__);
  // S_g and the densities data_initialization also leaves in the host
  // arrays (three-phase.cpp:429-434, 479-481).
  for (long long l = 0; l < n; l++) {
    H.S_g[l] = 1. - def.S_w_init - def.S_n_init;
    H.ro_w[l] = def.ro0_w * (1. + (def.beta_w) * (H.P_w[l] - def.P_atm));
    H.ro_n[l] = def.ro0_n * (1. + (def.beta_n) * (H.P_n[l] - def.P_atm));
    H.ro_g[l] = def.ro0_g * H.P_g[l] / def.P_atm;
  }
#else
  check(capaz_reference_init(&p, H.m, 0, H.P_w, nullptr, H.S_n, nullptr, nullptr), "capaz_reference_init",
        __LINE__);
  // The densities data_initialization also leaves in the host arrays
  // (two-phase.cpp:147-150).
  for (long long l = 0; l < n; l++) {
    H.ro_w[l] = def.ro0_w * (1. + (def.beta_w) * (H.P_w[l] - def.P_atm));
    H.ro_n[l] = def.ro0_n * (1. + (def.beta_n) * (H.P_w[l] - def.P_atm));
  }
#endif
}

// ---- stages ----------------------------------------------------------------
void S_calculation(ptr_Arrays, ptr_Arrays, consts) {
  advance(IDLE, AFTER_S, "S_calculation", __LINE__);
  g.stepping = true;
}

void ro_P_Xi_calculation(ptr_Arrays, ptr_Arrays, consts) {
  advance(AFTER_S, AFTER_RO_P_XI, "ro_P_Xi_calculation", __LINE__);
}

void u_calculation(ptr_Arrays, ptr_Arrays, consts) { advance(AFTER_RO_P_XI, AFTER_U, "u_calculation", __LINE__); }

void roS_calculation(ptr_Arrays, ptr_Arrays, double t, consts) {
  (void)t;  // the NR scheme does not use t (cpu.cpp:619-731)
  advance(AFTER_U, AFTER_ROS, "roS_calculation", __LINE__);
}

void P_S_calculation(ptr_Arrays, ptr_Arrays, consts) {
  advance(AFTER_ROS, AFTER_P_S, "P_S_calculation", __LINE__);
  check(capaz_step(g.ctx, 1, nullptr), "capaz_step", __LINE__);
  g.steps++;
}

void boundary_conditions(ptr_Arrays, ptr_Arrays, consts) {
  // The boundary update ran inside the fused step.
  advance(AFTER_P_S, IDLE, "boundary_conditions", __LINE__);
}

// ---- one rank: no halo exchange ------------------------------------------------
#define CAPAZ_NO_HALO(name)                                                        \
  void name(double*, double*, double*, double*, consts) {                          \
    die(#name ": halo exchange needs a multi-rank backend (one rank here)", __LINE__); \
  }
CAPAZ_NO_HALO(load_exchange_data_part_xl)
CAPAZ_NO_HALO(load_exchange_data_part_xr)
CAPAZ_NO_HALO(load_exchange_data_part_yl)
CAPAZ_NO_HALO(load_exchange_data_part_yr)
CAPAZ_NO_HALO(load_exchange_data_part_zl)
CAPAZ_NO_HALO(load_exchange_data_part_zr)
CAPAZ_NO_HALO(save_exchange_data_part_xl)
CAPAZ_NO_HALO(save_exchange_data_part_xr)
CAPAZ_NO_HALO(save_exchange_data_part_yl)
CAPAZ_NO_HALO(save_exchange_data_part_yr)
CAPAZ_NO_HALO(save_exchange_data_part_zl)
CAPAZ_NO_HALO(save_exchange_data_part_zr)

void checkErrors(char* label, char* file, int line) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    printf("Error: %s (%s)\nFile: \"%s\"\nLine: %d\n\n", label, cudaGetErrorString(e), file, line);
    fflush(stdout);
    exit(1);
  }
}
