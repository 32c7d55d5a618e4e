// C ABI of the library (include/capaz_b200.h): contexts, parameters, field
// transfer, the reference's initial state and the step launcher.
//
// Host-side restatements of the reference's setup, with their origins:
//   capaz_params_from_ini  read_defines          main.cpp:1280-1639
//   capaz_init_state       data_initialization   two-phase.cpp:113-172,
//                                                three-phase.cpp:429-500
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <utility>
#include <string>
#include <vector>

#include "capaz_internal.h"
#include "capaz_ctx.h"

using namespace capaz;

namespace {

thread_local std::string g_create_error;

int fail(capaz_ctx* ctx, int code, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
int fail(capaz_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->last_error = buf;
  else g_create_error = buf;
  return code;
}

int cuda_fail(capaz_ctx* ctx, cudaError_t e, const char* what) {
  int code = (e == cudaErrorMemoryAllocation) ? CAPAZ_ERR_OUT_OF_MEMORY : CAPAZ_ERR_CUDA;
  return fail(ctx, code, "%s: %s", what, cudaGetErrorString(e));
}

#define CUDA_TRY(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

bool is_state_field(const capaz_params& p, int f) {
  if (f == CAPAZ_FIELD_P_W || f == CAPAZ_FIELD_S_N) return true;
  if (p.phases == 3 && (f == CAPAZ_FIELD_S_W || f == CAPAZ_FIELD_P_N || f == CAPAZ_FIELD_P_G)) return true;
  if (p.model == CAPAZ_MODEL_ENERGY && f == CAPAZ_FIELD_T) return true;
  return false;
}

// State arrays of a context: P_w, S_n[, S_w, P_n, P_g[, T]].
int state_count(const capaz_params& p) {
  if (p.phases == 2) return 2;
  return p.model == CAPAZ_MODEL_ENERGY ? 6 : 5;
}

}  // namespace

void capaz::set_create_error(const char* msg) { g_create_error = msg; }

// ---------------------------------------------------------------------------
// Step constants.
namespace capaz {

Step2Const make_step2_const(const capaz_params& p) {
  Step2Const c;
  memset(&c, 0, sizeof c);
  c.nx = p.nx;
  c.ny = p.ny;
  c.nz = p.nz;
  c.source = p.source;
  window_k(p, &c.win_k0, &c.win_k1);
  c.iters = p.newton_iterations;
  c.sy = p.nx;
  c.sz = (long long)p.nx * p.ny;
  c.ncell = c.sz * p.nz;
  c.tiles_x = (p.nx - 2 + TX - 1) / TX;
  c.tiles_y = (p.ny - 2 + TY - 1) / TY;
  if (p.nz == 1) {
    c.zchunk = 1;
    c.nzchunks = 1;
  } else {
    const int interior = p.nz - 2;
    const int tiles = c.tiles_x * c.tiles_y;
    // Enough CTAs to fill 148 SMs several times over; the z-chunk overlap
    // (two extra planes per chunk) stays small with chunks of >= 8 planes.
    int chunk = 32;
    while (chunk > 8 && (long long)tiles * ((interior + chunk - 1) / chunk) < 4 * 148) chunk /= 2;
    c.zchunk = std::min(chunk, interior);
    c.nzchunks = (interior + c.zchunk - 1) / c.zchunk;
  }
  c.hx = p.hx;
  c.hy = p.hy;
  c.hz = p.hz;
  c.dt = p.dt;
  c.g = p.g_const;
  c.P_atm = p.P_atm;
  c.P_top = p.P_top_offset;
  c.ro0_w = p.ro0_w;
  c.ro0_n = p.ro0_n;
  c.beta_w = p.beta_w;
  c.beta_n = p.beta_n;
  c.mu_w = p.mu_w;
  c.mu_n = p.mu_n;
  c.S_wr = p.S_wr;
  c.lambda = p.lambda;
  c.P_d = p.P_d;
  c.K0 = p.K0;
  c.S_n_gr = p.S_n_gr;
  const double lam = p.lambda;
  c.e_kw = (2. + 3. * lam) / lam;
  c.e_kn = (2. + lam) / lam;
  c.e_pk = -1. / lam;
  c.e_aaa = ((-1.) / lam) - 1.;
  // P_d == 0: P_d*pow(S_e, e) is +0 whenever pow is finite and positive,
  // i.e. for S_e >= 2^(1000/e) with e < 0, and PkS is +0 when
  // lambda*(1 - S_wr) > 0.  Otherwise the fast path is disabled (0).
  c.se_fast_min = 0.;
  if (p.P_d == 0. && lam > 0. && (1. - p.S_wr) > 0. && isfinite(c.e_aaa) && c.e_aaa < 0.)
    c.se_fast_min = ldexp(1.0, (int)floor(1000. / c.e_aaa) + 1);
  // num > 2 t (1 - S_wr) gives num / (1 - S_wr) > 2 t exactly, so the
  // rounded quotient is >= t: the Newton iterations skip the division.
  c.se_fast_num = 2. * c.se_fast_min * (1. - p.S_wr);
  c.vol = p.hx * p.hy * p.hz;
  c.lam2 = (p.flags & CAPAZ_FLAG_POW_PRODUCTS) && p.lambda == 2.0;
  return c;
}

BLConst make_bl_const(const capaz_params& p) {
  BLConst b;
  memset(&b, 0, sizeof b);
  b.c = make_step2_const(p);
  b.Q = p.Q;
  b.injwell_Pw = p.injwell_Pw;
  b.outwell_Pw = p.outwell_Pw;
  return b;
}

Step2FConst make_step2f_const(const capaz_params& p, double S_ref) {
  const Step2Const d = make_step2_const(p);
  Step2FConst c;
  memset(&c, 0, sizeof c);
  c.nx = d.nx;
  c.ny = d.ny;
  c.nz = d.nz;
  c.source = d.source;
  c.win_k0 = d.win_k0;
  c.win_k1 = d.win_k1;
  c.iters = 2;  // delta-form Newton: the system is bilinear and starts within one step's change
  c.tiles_x = d.tiles_x;
  c.tiles_y = d.tiles_y;
  c.zchunk = d.zchunk;
  c.nzchunks = d.nzchunks;
  c.sy = d.sy;
  c.sz = d.sz;
  const double ekw = d.e_kw, ekn = d.e_kn;
  c.intpow = (ekw == floor(ekw) && ekn == floor(ekn) && ekw >= 0 && ekn >= 0 && ekw <= 16 && ekn <= 16) ? 1 : 0;
  c.n_kw = (int)ekw;
  c.n_kn = (int)ekn;
  c.S_ref = S_ref;
  c.S_ref_f = (float)S_ref;
  c.one_m_swr_f = (float)(1. - p.S_wr);
  c.inv_one_m_swr_f = (float)(1. / (1. - p.S_wr));
  c.e_kw_f = (float)ekw;
  c.e_kn_f = (float)ekn;
  c.e_pk_f = (float)d.e_pk;
  c.P_d_f = (float)p.P_d;
  c.ro0_w_f = (float)p.ro0_w;
  c.ro0_n_f = (float)p.ro0_n;
  c.beta_w_f = (float)p.beta_w;
  c.beta_n_f = (float)p.beta_n;
  c.inv_mu_w_f = (float)(1. / p.mu_w);
  c.inv_mu_n_f = (float)(1. / p.mu_n);
  c.K0_f = (float)p.K0;
  c.g_f = (float)p.g_const;
  c.inv_hx_f = (float)(1. / p.hx);
  c.inv_hy_f = (float)(1. / p.hy);
  c.inv_hz_f = (float)(1. / p.hz);
  c.dt = p.dt;
  c.P_atm = p.P_atm;
  c.P_top = p.P_top_offset;
  c.P_d = p.P_d;
  c.S_wr = p.S_wr;
  c.e_pk = d.e_pk;
  c.ro0_w = p.ro0_w;
  c.ro0_n = p.ro0_n;
  c.beta_w = p.beta_w;
  c.beta_n = p.beta_n;
  c.g = p.g_const;
  c.hy = p.hy;
  c.S_n_gr = p.S_n_gr;
  c.vol = d.vol;
  return c;
}

Step3FConst make_step3f_const(const capaz_params& p, double S_ref_w, double S_ref_n) {
  const Step3Const d = make_step3_const(p);
  Step3FConst c;
  memset(&c, 0, sizeof c);
  c.nx = d.nx;
  c.ny = d.ny;
  c.nz = d.nz;
  c.source = d.source;
  c.source_window = d.source_window;
  c.win_k0 = d.win_k0;
  c.win_k1 = d.win_k1;
  c.tiles_x = d.tiles_x;
  c.tiles_y = d.tiles_y;
  c.zchunk = d.zchunk;
  c.nzchunks = d.nzchunks;
  c.i_lo = d.i_lo;
  c.i_hi = d.i_hi;
  c.a2 = p.lambda == 2.0 ? 1 : 0;
  c.sy = d.sy;
  c.sz = d.sz;
  c.S_ref_w = S_ref_w;
  c.S_ref_n = S_ref_n;
  c.S_ref_w_f = (float)S_ref_w;
  c.S_ref_n_f = (float)S_ref_n;
  c.S_wr_f = (float)p.S_wr;
  c.S_nr_f = (float)p.S_nr;
  c.inv_den = (float)(1. / (1. - p.S_wr - p.S_nr - p.S_gr));
  c.K0_f = (float)p.K0;
  c.aw = p.ro0_w * p.beta_w;
  c.an = p.ro0_n * p.beta_n;
  c.bg = p.ro0_g / p.P_atm;
  c.aw_f = (float)c.aw;
  c.an_f = (float)c.an;
  c.bg_f = (float)c.bg;
  c.inv_mu_w_f = (float)(1. / p.mu_w);
  c.inv_mu_n_f = (float)(1. / p.mu_n);
  c.inv_mu_g_f = (float)(1. / p.mu_g);
  c.inv_hx2_f = (float)(1. / (p.hx * p.hx));
  c.inv_hy2_f = (float)(1. / (p.hy * p.hy));
  c.inv_hz2_f = (float)(1. / (p.hz * p.hz));
  c.g_inv_hy_f = (float)(p.g_const / p.hy);
  c.dt_f = (float)p.dt;
  const double A = p.lambda;
  c.e1 = (float)(A / (A - 1.));
  c.e2 = (float)((A - 1.) / A);
  c.e3 = (float)(2. * (A - 1.) / A);
  c.P_atm = p.P_atm;
  c.ro0_w = p.ro0_w;
  c.ro0_n = p.ro0_n;
  c.ro0_g = p.ro0_g;
  c.beta_w = p.beta_w;
  c.beta_n = p.beta_n;
  c.g = p.g_const;
  c.hy = p.hy;
  c.S_w_gr = p.S_w_gr;
  c.S_n_gr = p.S_n_gr;
  c.vol = p.hx * p.hy * p.hz;
  return c;
}

PhysF make_physf(const capaz_params& p) {
  PhysF f;
  memset(&f, 0, sizeof f);
  f.inv_one_m_swr = (float)(1. / (1. - p.S_wr));
  f.ro0w_bw = (float)(p.ro0_w * p.beta_w);
  f.ro0n_bn = (float)(p.ro0_n * p.beta_n);
  f.inv_mu_w = (float)(1. / p.mu_w);
  f.inv_mu_n = (float)(1. / p.mu_n);
  f.K0 = (float)p.K0;
  f.inv_hx2 = (float)(1. / (p.hx * p.hx));
  f.inv_hy2 = (float)(1. / (p.hy * p.hy));
  f.inv_hz2 = (float)(1. / (p.hz * p.hz));
  f.g_inv_hy = (float)(p.g_const / p.hy);
  f.cw_mu = (float)(p.ro0_w * p.beta_w / p.mu_w);
  f.cn_mu = (float)(p.ro0_n * p.beta_n / p.mu_n);
  f.g_mu_w = (float)(p.g_const * p.mu_w / p.hy);
  f.g_mu_n = (float)(p.g_const * p.mu_n / p.hy);
  f.iters = 1;  // one Newton step: the delta-form solve of the TMA kernel
  f.ro0_w = p.ro0_w;
  f.ro0_n = p.ro0_n;
  f.aw = p.ro0_w * p.beta_w;
  f.bn = p.ro0_n * p.beta_n;
  f.P_atm = p.P_atm;
  f.P_top = p.P_top_offset;
  f.g = p.g_const;
  f.hy = p.hy;
  f.vol = p.hx * p.hy * p.hz;
  f.mu_w = p.mu_w;
  f.mu_n = p.mu_n;
  return f;
}

Step3Const make_step3_const(const capaz_params& p) {
  Step3Const c;
  memset(&c, 0, sizeof c);
  c.nx = p.nx;
  c.ny = p.ny;
  c.nz = p.nz;
  c.source = p.source;
  window_k(p, &c.win_k0, &c.win_k1);
  c.iters = p.newton_iterations;
  c.source_window = (p.flags & CAPAZ_FLAG_SOURCE_WINDOW) ? 1 : 0;
  // Interior x range: [1, nx-2], or the single column of an nx == 1 grid.
  c.i_lo = p.nx == 1 ? 0 : 1;
  c.i_hi = p.nx == 1 ? 0 : p.nx - 2;
  c.sy = p.nx;
  c.sz = (long long)p.nx * p.ny;
  c.ncell = c.sz * p.nz;
  c.tiles_x = (c.i_hi - c.i_lo + 1 + TX - 1) / TX;
  c.tiles_y = (p.ny - 2 + TY - 1) / TY;
  if (p.nz == 1) {
    c.zchunk = 1;
    c.nzchunks = 1;
  } else {
    const int interior = p.nz - 2;
    const int tiles = c.tiles_x * c.tiles_y;
    int chunk = 32;
    while (chunk > 4 && (long long)tiles * ((interior + chunk - 1) / chunk) < 4 * 148) chunk /= 2;
    c.zchunk = std::min(chunk, interior);
    c.nzchunks = (interior + c.zchunk - 1) / c.zchunk;
  }
  c.hx = p.hx;
  c.hy = p.hy;
  c.hz = p.hz;
  c.dt = p.dt;
  c.g = p.g_const;
  c.P_atm = p.P_atm;
  c.ro0_w = p.ro0_w;
  c.ro0_n = p.ro0_n;
  c.ro0_g = p.ro0_g;
  c.beta_w = p.beta_w;
  c.beta_n = p.beta_n;
  c.mu_w = p.mu_w;
  c.mu_n = p.mu_n;
  c.mu_g = p.mu_g;
  c.S_wr = p.S_wr;
  c.S_nr = p.S_nr;
  c.S_gr = p.S_gr;
  c.A = p.lambda;
  c.K0 = p.K0;
  c.S_w_gr = p.S_w_gr;
  c.S_n_gr = p.S_n_gr;
  c.vol = p.hx * p.hy * p.hz;
  c.a2 = (p.flags & CAPAZ_FLAG_POW_PRODUCTS) && p.lambda == 2.0;
  return c;
}

// data_initialization (two-phase.cpp:113-172; the GPU build's copy in
// two-phase.cu:6-65 is identical) and three-phase.cpp:438-500, on host
// arrays, m given.  Loop order i, j, k as the reference: the hydrostatic
// recurrence reads the cell above (j - 1), computed in the previous j pass.
void reference_init_host(const capaz_params& p, const double* m, double* Pw, double* Sw, double* Sn, double* Pn,
                         double* Pg) {
  const long long sy = p.nx, sz = (long long)p.nx * p.ny, n = sz * p.nz;
  if (p.model == CAPAZ_MODEL_BUCKLEY_LEVERETT) {
    // Buckley-Leverett data_initialization (b-l.cpp:173-219): uniform
    // BACKGROUND_Sn; BACKGROUND_Pw on the top row and down each column the
    // weight of the cell itself, taken with the reference densities.
    for (int i = 0; i < p.nx; i++)
      for (int j = 0; j < p.ny; j++)
        for (int k = 0; k < p.nz; k++) {
          long long l = i + j * sy + (long long)k * sz;
          Sn[l] = p.background_Sn;
          double ro_g_dy = (p.ro0_n * Sn[l] + p.ro0_w * (1 - Sn[l])) * (m[l]) * (p.g_const) * (p.hy);
          Pw[l] = (j == 0) ? p.background_Pw : Pw[l - sy] + ro_g_dy;
        }
    return;
  }
  if (p.phases == 2) {
    std::vector<double> ro_w(n), ro_n(n);
    for (int i = 0; i < p.nx; i++)
      for (int j = 0; j < p.ny; j++)
        for (int k = 0; k < p.nz; k++) {
          long long l = i + j * sy + (long long)k * sz;
          int wk0, wk1;
          window_k(p, &wk0, &wk1);
          bool win = (i >= p.nx / 2 - p.source) && (i <= p.nx / 2 + p.source) && (k >= wk0) && (k <= wk1);
          Sn[l] = ((j == 0) && win) ? p.S_n_gr : p.S_n_background;
          if (j == 0) {
            Pw[l] = p.P_atm;
          } else {
            long long u = l - sy;
            double ro_g_dy = (ro_n[u] * Sn[u] + ro_w[u] * (1 - Sn[u])) * (m[u]) * (p.g_const) * (p.hy);
            Pw[l] = Pw[u] + ro_g_dy;
          }
          ro_w[l] = p.ro0_w * (1. + (p.beta_w) * (Pw[l] - p.P_atm));
          ro_n[l] = p.ro0_n * (1. + (p.beta_n) * (Pw[l] - p.P_atm));
        }
    return;
  }
  for (long long l = 0; l < n; l++) {
    Sw[l] = p.S_w_init;
    Sn[l] = p.S_n_init;
    Pw[l] = p.P_atm;
    Pn[l] = p.P_atm;
    Pg[l] = p.P_atm;
  }
}

}  // namespace capaz

// ---------------------------------------------------------------------------
extern "C" {

int capaz_abi_version(void) { return CAPAZ_ABI_VERSION; }
size_t capaz_params_size(void) { return sizeof(capaz_params); }
size_t capaz_diag_size(void) { return sizeof(capaz_diag); }

int capaz_params_default(capaz_params* p) {
  if (!p) return CAPAZ_ERR_INVALID_ARGUMENT;
  memset(p, 0, sizeof *p);
  // Two-phase/defines.ini values.
  p->nx = 15;
  p->ny = 15;
  p->nz = 1;
  p->phases = 2;
  p->form = CAPAZ_FORM_FP64;
  p->newton_iterations = 10;
  p->source = 30;
  p->flags = 0;
  p->hx = p->hy = p->hz = 5e-2;
  p->dt = 1e-3;
  p->beta_w = 4.4e-7;
  p->beta_n = 1e-6;
  p->beta_g = 9.2e-6;
  p->ro0_w = 1000;
  p->ro0_n = 1460;
  p->ro0_g = 1.4;
  p->mu_w = 0.001;
  p->mu_n = 0.0009;
  p->mu_g = 1.84e-5;
  p->g_const = 9.807;
  p->P_atm = 100000;
  p->lambda = 2.7;
  p->S_wr = 0.09;
  p->S_nr = 0.;
  p->S_gr = 0.;
  p->P_d = 755;
  p->S_n_gr = 0.2;
  p->S_w_gr = 0.4;
  p->S_w_init = 0.4;
  p->S_n_init = 0.3;
  p->porosity = 0.4;
  p->K0 = 6.64e-11;
  p->timeX = 100;
  p->P_top_offset = 0.;
  p->S_n_background = 0.;
  return CAPAZ_OK;
}

int capaz_params_from_ini(const char* path, capaz_params* p) {
  if (!path || !p) return CAPAZ_ERR_INVALID_ARGUMENT;
  FILE* f = fopen(path, "rt");
  if (!f) return fail(nullptr, CAPAZ_ERR_INI, "cannot open %s", path);
  char str[250];
  while (fgets(str, sizeof str, f)) {
    if (str[0] == '#') continue;
    const char* eq = strchr(str, '=');
    if (!eq) continue;
    std::string name(str, eq - str);
    // The value runs to the first space (main.cpp:1319); atof/atoi stop at
    // the line end themselves.
    std::string value;
    for (const char* q = eq + 1; *q && *q != ' '; q++) value.push_back(*q);
    const char* v = value.c_str();
    double d = atof(v);
    int n = atoi(v);
    if (name == "HX") p->hx = d;
    else if (name == "HY") p->hy = d;
    else if (name == "HZ") p->hz = d;
    else if (name == "DT") p->dt = d;
    else if (name == "BETA_W") p->beta_w = d;
    else if (name == "BETA_N") p->beta_n = d;
    else if (name == "BETA_G") p->beta_g = d;
    else if (name == "RO_W") p->ro0_w = d;
    else if (name == "RO_N") p->ro0_n = d;
    else if (name == "RO_G") p->ro0_g = d;
    else if (name == "MU_W") p->mu_w = d;
    else if (name == "MU_N") p->mu_n = d;
    else if (name == "MU_G") p->mu_g = d;
    else if (name == "G_CONST") p->g_const = d;
    else if (name == "P_ATM") p->P_atm = d;
    else if (name == "LAMBDA_0") p->lambda = d;
    else if (name == "M_0") p->porosity = d;
    else if (name == "S_WR_0") p->S_wr = d;
    else if (name == "S_NR_0") p->S_nr = d;
    else if (name == "S_GR_0") p->S_gr = d;
    else if (name == "K_0") p->K0 = d;
    else if (name == "P_D_0") p->P_d = d;
    else if (name == "S_W_GR") p->S_w_gr = d;
    else if (name == "S_W_INIT") p->S_w_init = d;
    else if (name == "S_N_INIT") p->S_n_init = d;
    else if (name == "S_N_GR") p->S_n_gr = d;
    else if (name == "SOURCE") p->source = n;
    else if (name == "ITERATIONS") p->newton_iterations = n;
    else if (name == "TIMEX") p->timeX = d;
    else if (name == "NX") p->nx = n;
    else if (name == "NY") p->ny = n;
    else if (name == "NZ") p->nz = n;
    // Extensions (ignored by the reference, which skips unknown keys).
    else if (name == "P_TOP_OFFSET") p->P_top_offset = d;
    else if (name == "S_N_BACKGROUND") p->S_n_background = d;
    else if (name == "PERCELL_K") p->flags = n ? (p->flags | CAPAZ_FLAG_PERCELL_K) : (p->flags & ~CAPAZ_FLAG_PERCELL_K);
    else if (name == "PHASES") p->phases = n;
    // Buckley-Leverett task keys (main.cpp:1436-1480).
    else if (name == "Q") p->Q = d;
    else if (name == "BACKGROUND_Pw") p->background_Pw = d;
    else if (name == "BACKGROUND_Sn") p->background_Sn = d;
    else if (name == "INJECTION_WELL_Pw") p->injwell_Pw = d;
    else if (name == "OUTPUT_WELL_Pw") p->outwell_Pw = d;
    else if (name == "MODEL") p->model = n;
  }
  fclose(f);
  return CAPAZ_OK;
}

int capaz_params_validate(const capaz_params* p) {
  if (!p) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (p->phases != 2 && p->phases != 3) return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "phases must be 2 or 3");
  if (p->form != CAPAZ_FORM_FP64 && p->form != CAPAZ_FORM_FP32C)
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "unknown form %d", p->form);
  // Grids where every boundary cell's basic coordinate is an interior cell
  // (cpu.cpp:107-141); elsewhere the reference's result depends on its loop
  // order.  nx == 1 is the reference's own three-phase column case.
  const bool nx_ok = p->nx >= 3 || (p->phases == 3 && p->nx == 1);
  if (!nx_ok || p->ny < 3 || p->nz < 1 || p->nz == 2)
    return fail(nullptr, CAPAZ_ERR_UNSUPPORTED_GRID, "grid %dx%dx%d unsupported (need nx,ny>=3, nz==1 or >=3)",
                p->nx, p->ny, p->nz);
  if (p->z_offset < 0 || p->nz_global < 0 || (p->nz_global > 0 && p->z_offset + p->nz > p->nz_global))
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "z_offset/nz_global do not place the slab inside the grid");
  if ((long long)p->nx * p->ny * p->nz > (1LL << 34))
    return fail(nullptr, CAPAZ_ERR_UNSUPPORTED_GRID, "grid too large");
  if (!(p->hx > 0) || !(p->hy > 0) || !(p->hz > 0) || !(p->dt > 0))
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "hx, hy, hz and dt must be > 0");
  if (p->newton_iterations < 0 || p->newton_iterations > 1000)
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "newton_iterations out of range");
  if (!(p->mu_w > 0) || !(p->mu_n > 0) || !(p->P_atm > 0) || !(p->lambda != 0))
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "mu, P_atm must be > 0 and lambda != 0");
  if (!(p->K0 > 0)) return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "K_0 must be > 0");
  if (p->model != CAPAZ_MODEL_DEFAULT && p->model != CAPAZ_MODEL_BUCKLEY_LEVERETT && p->model != CAPAZ_MODEL_ENERGY)
    return fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "unknown model %d", p->model);
  if (p->model == CAPAZ_MODEL_ENERGY) {
    if (p->phases != 3 || p->form != CAPAZ_FORM_FP64)
      return fail(nullptr, CAPAZ_ERR_UNSUPPORTED, "the energy equation is three-phase, FP64 form");
    if (p->flags & CAPAZ_FLAG_DIAGNOSTICS)
      return fail(nullptr, CAPAZ_ERR_UNSUPPORTED, "diagnostics are not built for the energy equation");
    // Its advected enthalpy reaches two cells: one halo plane per slab is not enough.
    if (p->z_offset != 0 || (p->nz_global > 0 && p->nz_global != p->nz))
      return fail(nullptr, CAPAZ_ERR_UNSUPPORTED, "the energy equation does not run on z-slabs");
  }
  if (p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT && (p->phases != 2 || p->form != CAPAZ_FORM_FP64))
    return fail(nullptr, CAPAZ_ERR_UNSUPPORTED, "the Buckley-Leverett task is two-phase, FP64 form");
  // The injection and production well blocks (2x2 corners, b-l.cpp:221-237)
  // must neither overlap nor be the basic coordinate of a non-well boundary
  // cell; with nx, ny >= 4 the boundary rules need no particular cell order.
  if (p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT && (p->nx < 4 || p->ny < 4))
    return fail(nullptr, CAPAZ_ERR_UNSUPPORTED_GRID, "the Buckley-Leverett task needs nx, ny >= 4");
  if (p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT && (p->flags & CAPAZ_FLAG_DIAGNOSTICS))
    return fail(nullptr, CAPAZ_ERR_UNSUPPORTED, "diagnostics are not built for the Buckley-Leverett task");
  return CAPAZ_OK;
}

const char* capaz_last_error(const capaz_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

capaz_ctx* capaz_create(const capaz_params* p, int device, int* status) {
  int st = capaz_params_validate(p);
  if (st) {
    if (status) *status = st;
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    if (status) *status = fail(nullptr, CAPAZ_ERR_NO_DEVICE, "no CUDA device");
    return nullptr;
  }
  if (device < 0 || device >= ndev) {
    if (status) *status = fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    return nullptr;
  }
  capaz_ctx* ctx = new capaz_ctx();
  ctx->p = *p;
  ctx->device = device;
  st = ctx->allocate();
  if (st) {
    g_create_error = ctx->last_error;
    delete ctx;
    if (status) *status = st;
    return nullptr;
  }
  if (status) *status = CAPAZ_OK;
  return ctx;
}

int capaz_destroy(capaz_ctx* ctx) {
  if (!ctx) return CAPAZ_ERR_INVALID_ARGUMENT;
  ctx->release();
  delete ctx;
  return CAPAZ_OK;
}

int capaz_get_params(const capaz_ctx* ctx, capaz_params* out) {
  if (!ctx || !out) return CAPAZ_ERR_INVALID_ARGUMENT;
  *out = ctx->p;
  return CAPAZ_OK;
}

int64_t capaz_launch_count(const capaz_ctx* ctx) { return ctx ? ctx->launches : -1; }

int capaz_set_dt(capaz_ctx* ctx, double dt) {
  if (!ctx || !(dt > 0)) return CAPAZ_ERR_INVALID_ARGUMENT;
  ctx->p.dt = dt;
  return CAPAZ_OK;
}

int capaz_set_sweep_tile(capaz_ctx* ctx, int tile_y) {
  if (!ctx) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (!tma_tile_supported(tile_y)) return fail(ctx, CAPAZ_ERR_UNSUPPORTED, "tile_y must be 16 or 32");
  ctx->tma_tile_y = tile_y;  // the descriptor is rebuilt before the next step
  return CAPAZ_OK;
}

int capaz_set_field(capaz_ctx* ctx, int field, const double* host, void* stream) {
  if (!ctx || !host) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->set_field(field, host, false, (cudaStream_t)stream);
}
int capaz_set_field_device(capaz_ctx* ctx, int field, const void* dev, void* stream) {
  if (!ctx || !dev) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->set_field(field, dev, true, (cudaStream_t)stream);
}
int capaz_get_field(capaz_ctx* ctx, int field, double* host, void* stream) {
  if (!ctx || !host) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->get_field(field, host, false, (cudaStream_t)stream);
}
int capaz_get_field_device(capaz_ctx* ctx, int field, void* dev, void* stream) {
  if (!ctx || !dev) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->get_field(field, dev, true, (cudaStream_t)stream);
}
int capaz_get_derived(capaz_ctx* ctx, int field, int state_sel, void* dst, int dst_on_device, void* stream) {
  if (!ctx || !dst || (state_sel != CAPAZ_STATE_STEP_START && state_sel != CAPAZ_STATE_CURRENT))
    return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->get_derived(field, state_sel == CAPAZ_STATE_CURRENT, dst, dst_on_device != 0, (cudaStream_t)stream);
}

int capaz_reference_init(const capaz_params* p, double* m, int m_given, double* P_w, double* S_w, double* S_n,
                         double* P_n, double* P_g) {
  if (!p || !m || !P_w || !S_n) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (p->phases == 3 && (!S_w || !P_n || !P_g)) return CAPAZ_ERR_INVALID_ARGUMENT;
  int st = capaz_params_validate(p);
  if (st) return st;
  const long long n = (long long)p->nx * p->ny * p->nz;
  if (!m_given)
    for (long long l = 0; l < n; l++) m[l] = p->porosity;
  reference_init_host(*p, m, P_w, S_w, S_n, P_n, P_g);
  return CAPAZ_OK;
}

int capaz_init_state(capaz_ctx* ctx, void* stream) {
  if (!ctx) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->init_state((cudaStream_t)stream);
}
int capaz_step(capaz_ctx* ctx, int nsteps, void* stream) {
  if (!ctx || nsteps < 0) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->step(nsteps, (cudaStream_t)stream);
}
int capaz_step_split(capaz_ctx* ctx, void* edge_stream, void* interior_stream) {
  if (!ctx || edge_stream == interior_stream) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->step_split((cudaStream_t)edge_stream, (cudaStream_t)interior_stream);
}
int capaz_read_diag(capaz_ctx* ctx, capaz_diag* out, void* stream) {
  if (!ctx || !out) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->read_diag(out, (cudaStream_t)stream);
}
int capaz_post_diag(capaz_ctx* ctx, int slot, void* stream) {
  if (!ctx || slot < 0 || slot >= CAPAZ_DIAG_SLOTS) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->post_diag(slot, (cudaStream_t)stream);
}
int capaz_step_post_diag(capaz_ctx* ctx, int nsteps, int slot, void* stream) {
  if (!ctx || nsteps < 0 || slot < 0 || slot >= CAPAZ_DIAG_SLOTS) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->step_post_diag(nsteps, slot, (cudaStream_t)stream);
}
int capaz_wait_diag(capaz_ctx* ctx, int slot, capaz_diag* out) {
  if (!ctx || !out || slot < 0 || slot >= CAPAZ_DIAG_SLOTS) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->wait_diag(slot, out);
}
int capaz_sync(capaz_ctx* ctx) {
  if (!ctx) return CAPAZ_ERR_INVALID_ARGUMENT;
  return ctx->sync();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// capaz_ctx methods.
int capaz_ctx::fail_cuda(cudaError_t e, const char* what) { return cuda_fail(this, e, what); }
int capaz_ctx::fail_msg(int code, const char* msg) { return fail(this, code, "%s", msg); }

int capaz_ctx::allocate() {
  CUDA_TRY(this, cudaSetDevice(device));
  n = (long long)p.nx * p.ny * p.nz;
  const size_t es = (p.form == CAPAZ_FORM_FP64) ? sizeof(double) : sizeof(float);
  const int nstate = state_count(p);
  for (int b = 0; b < 2; b++)
    for (int s = 0; s < nstate; s++) CUDA_TRY(this, cudaMalloc(&state[b][s], n * es));
  CUDA_TRY(this, cudaMalloc(&m, n * es));
  if (p.flags & CAPAZ_FLAG_PERCELL_K) CUDA_TRY(this, cudaMalloc(&K, n * es));
  if (p.form == CAPAZ_FORM_FP32C) {
    CUDA_TRY(this, cudaMalloc(&Pref, sizeof(double) * p.ny));
    CUDA_TRY(this, cudaMalloc(&PrelF, sizeof(float) * p.ny));
    CUDA_TRY(this, cudaMalloc(&dPrefF, sizeof(float) * p.ny));
    CUDA_TRY(this, cudaMalloc(&rowF, sizeof(float4) * p.ny));
    std::vector<double> pref0(p.ny, p.P_atm);
    std::vector<float> z(p.ny, 0.f);
    CUDA_TRY(this, cudaMemcpy(Pref, pref0.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice));
    CUDA_TRY(this, cudaMemcpy(PrelF, z.data(), sizeof(float) * p.ny, cudaMemcpyHostToDevice));
    CUDA_TRY(this, cudaMemcpy(dPrefF, z.data(), sizeof(float) * p.ny, cudaMemcpyHostToDevice));
    if (p.phases == 3) CUDA_TRY(this, launch_row_tables3(Pref, p.ny, make_step3f_const(p, 0., 0.), rowF, nullptr));
    else CUDA_TRY(this, launch_row_tables(Pref, p.ny, make_physf(p), rowF, nullptr));
  }
  CUDA_TRY(this, cudaMalloc(&first_bad, sizeof(unsigned long long)));
  CUDA_TRY(this, cudaMalloc(&sum_parts, sizeof(double) * 1024));
  CUDA_TRY(this, cudaMalloc(&S_ref_dev, sizeof(double)));
  CUDA_TRY(this, cudaMalloc(&err_flag, sizeof(unsigned int)));
  CUDA_TRY(this, cudaMemset(err_flag, 0, sizeof(unsigned int)));
  CUDA_TRY(this, cudaMalloc(&diag_out, sizeof(double) * DIAG_STRIDE));
  CUDA_TRY(this, cudaMemset(diag_out, 0, sizeof(double) * DIAG_STRIDE));
  CUDA_TRY(this, cudaHostAlloc(&diag_host, sizeof(double) * DIAG_STRIDE * (CAPAZ_DIAG_SLOTS + 1), cudaHostAllocMapped));
  CUDA_TRY(this, cudaHostGetDevicePointer(&diag_host_dev, diag_host, 0));
  for (int q = 0; q <= CAPAZ_DIAG_SLOTS; q++)
    CUDA_TRY(this, cudaEventCreateWithFlags(&diag_ev[q], cudaEventDisableTiming));
  // Default porosity M_0 and a zero state until the caller sets one.
  for (int b = 0; b < 2; b++)
    for (int s = 0; s < nstate; s++) CUDA_TRY(this, cudaMemset(state[b][s], 0, n * es));
  if (p.model == CAPAZ_MODEL_ENERGY) {
    CUDA_TRY(this, cudaMalloc(&ework, sizeof(double) * EW_COUNT * n));
    CUDA_TRY(this, cudaMemset(ework, 0, sizeof(double) * EW_COUNT * n));
  }
  {
    // Defaults need no validation: the caller's own m and K are checked when
    // set.  A non-positive M_0 is kept as given until m is set.
    std::vector<double> mh(n, p.porosity);
    defaults_unchecked = true;
    int st = set_field(CAPAZ_FIELD_M, mh.data(), false, nullptr);
    if (!st && (p.flags & CAPAZ_FLAG_PERCELL_K)) {
      std::fill(mh.begin(), mh.end(), p.K0);
      st = set_field(CAPAZ_FIELD_K, mh.data(), false, nullptr);
    }
    defaults_unchecked = false;
    if (st) return st;
  }
  CUDA_TRY(this, cudaDeviceSynchronize());
  return CAPAZ_OK;
}

void capaz_ctx::release() {
  cudaSetDevice(device);
  for (int b = 0; b < 2; b++)
    for (int s = 0; s < 6; s++)
      if (state[b][s]) cudaFree(state[b][s]);
  if (ework) cudaFree(ework);
  if (m) cudaFree(m);
  if (K) cudaFree(K);
  if (err_flag) cudaFree(err_flag);
  if (t3_counter) cudaFree(t3_counter);
  if (split_items) cudaFree(split_items);
  if (split_counters) cudaFree(split_counters);
  for (auto& ev : split_ev)
    if (ev) cudaEventDestroy(ev);
  if (diag_out) cudaFree(diag_out);
  if (diag_host) cudaFreeHost(diag_host);
  for (int q = 0; q <= CAPAZ_DIAG_SLOTS; q++)
    if (diag_ev[q]) cudaEventDestroy(diag_ev[q]);
  if (diag_partials) cudaFree(diag_partials);
  if (scratch) cudaFree(scratch);
  if (Pref) cudaFree(Pref);
  if (rowF) cudaFree(rowF);
  if (stage) cudaFree(stage);
  if (tma_inst) cudaFree(tma_inst);
  if (tma_items) cudaFree(tma_items);
  if (tma_counter) cudaFree(tma_counter);
  if (tma_bitems) cudaFree(tma_bitems);
  if (first_bad) cudaFree(first_bad);
  if (sum_parts) cudaFree(sum_parts);
  if (S_ref_dev) cudaFree(S_ref_dev);
  if (PrelF) cudaFree(PrelF);
  if (dPrefF) cudaFree(dPrefF);
  for (int q = 0; q < 7; q++)
    if (wide[q]) cudaFree(wide[q]);
  if (host_stage) cudaFreeHost(host_stage);
}

int capaz_ctx::ensure_scratch() {
  if (!scratch) CUDA_TRY(this, cudaMalloc(&scratch, n * sizeof(double)));
  return CAPAZ_OK;
}

int capaz_ctx::set_field(int field, const void* src, bool on_device, cudaStream_t s) {
  CUDA_TRY(this, cudaSetDevice(device));
  void* dst = nullptr;
  if (field == CAPAZ_FIELD_M) {
    dst = m;
  } else if (field == CAPAZ_FIELD_K) {
    if (!K) return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "K per cell needs CAPAZ_FLAG_PERCELL_K");
    dst = K;
  } else if (is_state_field(p, field)) {
    dst = state[cur][state_slot(field)];
  } else {
    return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "field %d cannot be set", field);
  }
  // Stage the float64 values on the device (from pinned or pageable host
  // memory, or another device array), check them there, then store them in
  // the form's layout.
  const double* d = static_cast<const double*>(src);
  if (!on_device) {
    if (!stage) CUDA_TRY(this, cudaMalloc(&stage, n * sizeof(double)));
    CUDA_TRY(this, cudaMemcpyAsync(stage, src, n * sizeof(double), cudaMemcpyHostToDevice, s));
    d = stage;
  }
  if ((field == CAPAZ_FIELD_M || field == CAPAZ_FIELD_K || field == CAPAZ_FIELD_T) && !defaults_unchecked) {
    const unsigned long long none = (unsigned long long)n;
    CUDA_TRY(this, cudaMemcpyAsync(first_bad, &none, sizeof none, cudaMemcpyHostToDevice, s));
    CUDA_TRY(this, launch_first_invalid(d, n, first_bad, s));
    launches++;
    unsigned long long bad = 0;
    CUDA_TRY(this, cudaMemcpyAsync(&bad, first_bad, sizeof bad, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(this, cudaStreamSynchronize(s));
    if (bad < (unsigned long long)n) {
      double v = 0.;
      CUDA_TRY(this, cudaMemcpy(&v, d + bad, sizeof v, cudaMemcpyDeviceToHost));
      return fail(this, CAPAZ_ERR_BAD_STATE, "%s must be finite and > 0 (cell %llu: %g)",
                  field == CAPAZ_FIELD_M ? "m" : field == CAPAZ_FIELD_K ? "K" : "T", bad, v);
    }
  }
  if (p.form == CAPAZ_FORM_FP64) {
    if (d != dst) CUDA_TRY(this, cudaMemcpyAsync(dst, d, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else if (field == CAPAZ_FIELD_P_W) {
    if (p.phases == 3) {
      // P_n, P_g are deviations from the same per-row reference: decode them
      // with the old reference, re-encode with the new one.
      for (int q = 5; q < 7; q++)
        if (!wide[q]) CUDA_TRY(this, cudaMalloc(&wide[q], n * sizeof(double)));
      CUDA_TRY(this, launch_decode_pressure((const float*)state[cur][3], Pref, p.nx, p.ny, n, wide[5], s));
      CUDA_TRY(this, launch_decode_pressure((const float*)state[cur][4], Pref, p.nx, p.ny, n, wide[6], s));
      launches += 2;
    }
    if (ref_locked) {
      CUDA_TRY(this, launch_encode_pressure_rel(d, Pref, p.nx, p.ny, n, (float*)dst, s));
      launches++;
    } else {
      CUDA_TRY(this, launch_encode_pressure(d, p.nx, p.ny, p.nz, p.P_atm, Pref, PrelF, dPrefF, (float*)dst, s));
      launches += 3;
    }
    if (p.phases == 3) {
      CUDA_TRY(this, launch_encode_pressure_rel(wide[5], Pref, p.nx, p.ny, n, (float*)state[cur][3], s));
      CUDA_TRY(this, launch_encode_pressure_rel(wide[6], Pref, p.nx, p.ny, n, (float*)state[cur][4], s));
      CUDA_TRY(this, launch_row_tables3(Pref, p.ny, make_step3f_const(p, S_ref_w, S_ref), rowF, s));
      launches += 3;
    } else {
      CUDA_TRY(this, launch_row_tables(Pref, p.ny, make_physf(p), rowF, s));
      launches++;
    }
  } else if (p.phases == 3 && (field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G)) {
    CUDA_TRY(this, launch_encode_pressure_rel(d, Pref, p.nx, p.ny, n, (float*)dst, s));
    launches++;
  } else if (p.phases == 3 && field == CAPAZ_FIELD_S_W) {
    CUDA_TRY(this, launch_encode_saturation(d, n, sum_parts, S_ref_dev, (float*)dst, s));
    launches += 3;
    CUDA_TRY(this, cudaMemcpyAsync(&S_ref_w, S_ref_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  } else if (field == CAPAZ_FIELD_S_N && ref_locked) {
    CUDA_TRY(this, launch_encode_saturation_ref(d, n, S_ref_dev, (float*)dst, s));
    launches++;
  } else if (field == CAPAZ_FIELD_S_N) {
    CUDA_TRY(this, launch_encode_saturation(d, n, sum_parts, S_ref_dev, (float*)dst, s));
    launches += 3;
    CUDA_TRY(this, cudaMemcpyAsync(&S_ref, S_ref_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  } else if (field == CAPAZ_FIELD_M || field == CAPAZ_FIELD_K) {
    CUDA_TRY(this, launch_narrow(d, n, (float*)dst, s));
    launches++;
  } else {
    return fail(this, CAPAZ_ERR_UNSUPPORTED, "the precision form stores the state, m and K");
  }
  CUDA_TRY(this, cudaStreamSynchronize(s));
  return CAPAZ_OK;
}

int capaz_ctx::check_flag() {
  unsigned int f = 0;
  CUDA_TRY(this, cudaMemcpy(&f, err_flag, sizeof f, cudaMemcpyDeviceToHost));
  if (f & 2u)
    return fail(this, CAPAZ_ERR_CUDA,
                "a bounded wait for a shared-memory copy ran out (device error bit 1); the step is incomplete");
  if (f) return fail(this, CAPAZ_ERR_NONFINITE, "a step produced a non-finite P or S");
  return CAPAZ_OK;
}

int capaz_ctx::get_field(int field, void* dst, bool on_device, cudaStream_t s) {
  CUDA_TRY(this, cudaSetDevice(device));
  if (field < 0 || field >= CAPAZ_FIELD_COUNT) return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "bad field %d", field);
  const size_t es = (p.form == CAPAZ_FORM_FP64) ? sizeof(double) : sizeof(float);
  const void* src = nullptr;
  if (field == CAPAZ_FIELD_M) src = m;
  else if (field == CAPAZ_FIELD_K) {
    if (!K) return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "no per-cell K");
    src = K;
  } else if (p.phases == 3 && p.model != CAPAZ_MODEL_ENERGY && (field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G) &&
             steps_done > 0) {
    int st = derived(field, s);
    if (st) return st;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CUDA_TRY(this, cudaMemcpyAsync(dst, scratch, n * sizeof(double), kind, s));
    if (on_device) return CAPAZ_OK;
    CUDA_TRY(this, cudaStreamSynchronize(s));
    return check_flag();
  } else if (is_state_field(p, field) && p.form == CAPAZ_FORM_FP64) {
    src = state[cur][state_slot(field)];
  } else if (is_state_field(p, field)) {
    // Precision form: decode the FP32 deviations of the current state.
    int st = decode_all(cur, s);
    if (st) return st;
    src = wide[field == CAPAZ_FIELD_P_W ? 0 : field == CAPAZ_FIELD_S_N ? 1 : field == CAPAZ_FIELD_S_W ? 4
               : field == CAPAZ_FIELD_P_N ? 5 : 6];
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CUDA_TRY(this, cudaMemcpyAsync(dst, src, n * sizeof(double), kind, s));
    if (on_device) return CAPAZ_OK;
    CUDA_TRY(this, cudaStreamSynchronize(s));
    return check_flag();
  } else {
    int st = derived(field, s);
    if (st) return st;
    src = scratch;
    if (on_device) {
      CUDA_TRY(this, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      return CAPAZ_OK;
    }
    CUDA_TRY(this, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(this, cudaStreamSynchronize(s));
    return check_flag();
  }
  if (on_device) {
    CUDA_TRY(this, cudaMemcpyAsync(dst, src, n * es, cudaMemcpyDeviceToDevice, s));
    return CAPAZ_OK;
  }
  if (es == sizeof(double)) {
    CUDA_TRY(this, cudaMemcpyAsync(dst, src, n * es, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(this, cudaStreamSynchronize(s));
  } else {
    std::vector<float> tmp(n);
    CUDA_TRY(this, cudaMemcpyAsync(tmp.data(), src, n * es, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(this, cudaStreamSynchronize(s));
    double* d = static_cast<double*>(dst);
    for (long long l = 0; l < n; l++) d[l] = tmp[l];
  }
  return check_flag();
}

int capaz_ctx::init_state(cudaStream_t s) {
  CUDA_TRY(this, cudaSetDevice(device));
  std::vector<double> host_m(n);
  {
    int st = get_field(CAPAZ_FIELD_M, host_m.data(), false, s);
    if (st) return st;
  }
  std::vector<double> Pw(n), Sn(n), Sw, Pn, Pg;
  if (p.phases == 3) {
    Sw.resize(n);
    Pn.resize(n);
    Pg.resize(n);
  }
  reference_init_host(p, host_m.data(), Pw.data(), Sw.data(), Sn.data(), Pn.data(), Pg.data());
  const int fields[5] = {CAPAZ_FIELD_P_W, CAPAZ_FIELD_S_N, CAPAZ_FIELD_S_W, CAPAZ_FIELD_P_N, CAPAZ_FIELD_P_G};
  double* src[5] = {Pw.data(), Sn.data(), Sw.data(), Pn.data(), Pg.data()};
  const int nstate = p.phases == 2 ? 2 : 5;
  for (int q = 0; q < nstate; q++) {
    int st = set_field(fields[q], src[q], false, s);
    if (st) return st;
  }
  if (p.model == CAPAZ_MODEL_ENERGY) {
    std::vector<double> T(n, ENERGY_T_INIT);
    int st = set_field(CAPAZ_FIELD_T, T.data(), false, s);
    if (st) return st;
    // The other arrays data_initialization fills (S_local_initialization and
    // the densities, three-phase.cpp:429-434, 479-481), which the energy
    // model's derived fields show until the first step.
    std::vector<double> Sg(n), rw(n), rn(n), rg(n);
    for (long long l = 0; l < n; l++) {
      Sg[l] = 1. - p.S_w_init - p.S_n_init;
      rw[l] = p.ro0_w * (1. + (p.beta_w) * (Pw[l] - p.P_atm));
      rn[l] = p.ro0_n * (1. + (p.beta_n) * (Pn[l] - p.P_atm));
      rg[l] = p.ro0_g * Pg[l] / p.P_atm;
    }
    const std::pair<int, const std::vector<double>*> put[4] = {{EW_SG, &Sg}, {EW_RO_W, &rw}, {EW_RO_N, &rn},
                                                               {EW_RO_G, &rg}};
    for (const auto& q : put)
      CUDA_TRY(this, cudaMemcpyAsync(ework + (size_t)q.first * n, q.second->data(), n * sizeof(double),
                                     cudaMemcpyHostToDevice, s));
    CUDA_TRY(this, cudaStreamSynchronize(s));
  }
  return CAPAZ_OK;
}

int capaz_ctx::get_derived(int field, bool from_current, void* dst, bool on_device, cudaStream_t s) {
  CUDA_TRY(this, cudaSetDevice(device));
  if (field < 0 || field >= CAPAZ_FIELD_COUNT) return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "bad field %d", field);
  if (field == CAPAZ_FIELD_M || field == CAPAZ_FIELD_K || is_state_field(p, field))
    return get_field(field, dst, on_device, s);
  int st = derived(field, s, from_current);
  if (st) return st;
  if (on_device) {
    CUDA_TRY(this, cudaMemcpyAsync(dst, scratch, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return CAPAZ_OK;
  }
  CUDA_TRY(this, cudaMemcpyAsync(dst, scratch, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(this, cudaStreamSynchronize(s));
  return check_flag();
}

int capaz_ctx::decode_all(int b, cudaStream_t s) {
  const int nw = p.phases == 3 ? 7 : 4;
  for (int q = 0; q < nw; q++)
    if (!wide[q]) CUDA_TRY(this, cudaMalloc(&wide[q], n * sizeof(double)));
  CUDA_TRY(this, launch_decode2((const float*)state[b][0], (const float*)state[b][1], Pref, S_ref, p.nx, p.ny, n,
                                wide[0], wide[1], s));
  if (p.phases == 3) {
    // S_w, P_n, P_g (P_n, P_g hold the Border_P values on boundary cells).
    CUDA_TRY(this, launch_decode2((const float*)state[b][3], (const float*)state[b][2], Pref, S_ref_w, p.nx, p.ny, n,
                                  wide[5], wide[4], s));
    CUDA_TRY(this, launch_decode_pressure((const float*)state[b][4], Pref, p.nx, p.ny, n, wide[6], s));
    launches += 2;
  }
  CUDA_TRY(this, launch_widen((const float*)m, n, wide[2], s));
  launches += 2;
  if (K) {
    CUDA_TRY(this, launch_widen((const float*)K, n, wide[3], s));
    launches++;
  }
  return CAPAZ_OK;
}

int capaz_ctx::sync() {
  CUDA_TRY(this, cudaSetDevice(device));
  CUDA_TRY(this, cudaDeviceSynchronize());
  return check_flag();
}

int capaz_ctx::read_diag(capaz_diag* out, cudaStream_t s) {
  const int st = post_diag(CAPAZ_DIAG_SLOTS, s);  // the slot kept for this call
  return st ? st : wait_diag(CAPAZ_DIAG_SLOTS, out);
}

int capaz_ctx::post_diag(int slot, cudaStream_t s) {
  CUDA_TRY(this, cudaSetDevice(device));
  if (!(p.flags & CAPAZ_FLAG_DIAGNOSTICS))
    return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "diagnostics need CAPAZ_FLAG_DIAGNOSTICS");
  CUDA_TRY(this, launch_diag_publish(diag_out, diag_host_dev + DIAG_STRIDE * slot, s));
  launches++;
  CUDA_TRY(this, cudaEventRecord(diag_ev[slot], s));
  diag_posted[slot] = true;
  return CAPAZ_OK;
}

// A step whose last sweep writes the reduced diagnostics straight into the
// mapped ring slot (the precision form's TMA sweep), followed by the event
// the host waits for; other paths step and then publish with post_diag.
int capaz_ctx::step_post_diag(int nsteps, int slot, cudaStream_t s) {
  if (!(p.flags & CAPAZ_FLAG_DIAGNOSTICS))
    return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "diagnostics need CAPAZ_FLAG_DIAGNOSTICS");
  publish_to = diag_host_dev + DIAG_STRIDE * slot;
  published = false;
  const int r = step(nsteps, s);
  publish_to = nullptr;
  if (r != CAPAZ_OK) return r;
  if (!published) return post_diag(slot, s);
  CUDA_TRY(this, cudaEventRecord(diag_ev[slot], s));
  diag_posted[slot] = true;
  return CAPAZ_OK;
}

int capaz_ctx::wait_diag(int slot, capaz_diag* out) {
  if (!diag_posted[slot]) return fail(this, CAPAZ_ERR_INVALID_ARGUMENT, "no diagnostics posted to this slot");
  CUDA_TRY(this, cudaSetDevice(device));
  diag_posted[slot] = false;
  CUDA_TRY(this, cudaEventSynchronize(diag_ev[slot]));
  const double* h = diag_host + DIAG_STRIDE * slot;
  memset(out, 0, sizeof *out);
  out->mass[0] = h[0];
  out->mass[1] = h[1];
  out->mass[2] = h[2];
  out->max_residual = h[3];
  out->nonfinite_cells = h[4];
  return CAPAZ_OK;
}
