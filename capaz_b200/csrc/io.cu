// Output and checkpoint files in the reference's formats (host code).
//
//   capaz_write_plot   print_plots_top / print_plots / print_plot_row
//                      (main.cpp:549-781): the Tecplot point file
//                      <dir>/S=%012.4f.dat of one rank's whole grid;
//   capaz_save         save (main.cpp:1035-1094): save.dat;
//   capaz_restore      restore (main.cpp:1097-1145), reading the sizes save
//                      writes (the reference reads locNx*locNy*locNy values
//                      per array, which is wrong unless Ny == Nz).
//
// The fields are taken as the reference's host arrays hold them after
// time_step_function: the state as it is now, the derived arrays (velocities,
// S_g, roS_old) as the last step computed them from its start-of-step state.
// Rows are formatted by several host threads into memory and written in the
// reference's order (i outer, then j, then k).
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "capaz_ctx.h"
#include "capaz_internal.h"

namespace {

int io_fail(capaz_ctx* ctx, int code, const std::string& msg) {
  ctx->last_error = msg;
  return code;
}

// Field as the reference's array holds it after the last time step.
int fetch(capaz_ctx* ctx, int field, std::vector<double>& out) {
  out.resize(ctx->n);
  return capaz_get_derived(ctx, field, CAPAZ_STATE_STEP_START, out.data(), 0, nullptr);
}

struct PlotFields {
  std::vector<double> Pw, Sn, Sw, Sg, m, K, T, uxw, uyw, uzw, uxn, uyn, uzn, uxg, uyg, uzg;
};

// One row of print_plot_row for cell l = (i, j, k).
void plot_row(const capaz_params& p, const PlotFields& F, int i, int j, int k, std::string& out) {
  char buf[512];
  const long long l = i + (long long)j * p.nx + (long long)k * p.nx * p.ny;
  const int I = i, J = p.ny - 1 - j, K = k;
  int n;
  if (p.model == CAPAZ_MODEL_BUCKLEY_LEVERETT) {
    // The B_L branch of print_plot_row (main.cpp:769-779): S_w, u_y unflipped
    // in the planar row, the permeability instead of the porosity.
    if (p.nz < 2)
      n = snprintf(buf, sizeof buf, "%.2e %.2e %.3e %.3e %.3e %.3e %.3e\n", I * (p.hx), J * (p.hy), 1. - F.Sn[l],
                   F.Pw[l], F.uxn[l], F.uyn[l], F.K[l]);
    else
      n = snprintf(buf, sizeof buf, "%.2e %.2e %.2e %.3e %.3e %.3e %.3e %.3e %.3e\n", I * (p.hx), K * (p.hz),
                   J * (p.hy), 1 - F.Sn[l], F.Pw[l], F.uxn[l], F.uzn[l], (-1) * F.uyn[l], F.K[l]);
  } else if (p.phases == 2) {
    if (p.nz < 2)
      n = snprintf(buf, sizeof buf, "%.2e %.2e %.3e %.3e %.3e %.3e %.3e\n", I * (p.hx), J * (p.hy), F.Sn[l], F.Pw[l],
                   F.uxn[l], (-1) * F.uyn[l], F.m[l]);
    else
      n = snprintf(buf, sizeof buf, "%.2e %.2e %.2e %.3e %.3e %.3e %.3e %.3e %.3e\n", I * (p.hx), K * (p.hz),
                   J * (p.hy), F.Sn[l], F.Pw[l], F.uxn[l], F.uzn[l], (-1) * F.uyn[l], F.m[l]);
  } else if (p.model == CAPAZ_MODEL_ENERGY) {
    // The ENERGY branch of print_plot_row (main.cpp:707-747): T after P_w.
    if (p.nz < 2 && p.nx < 2)
      n = snprintf(buf, sizeof buf, "%.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n", J * (p.hy), F.Sw[l], F.Sn[l],
                   F.Sg[l], F.Pw[l], F.T[l], (-1) * F.uyw[l], (-1) * F.uyn[l], (-1) * F.uyg[l], F.m[l]);
    else if (p.nz < 2)
      n = snprintf(buf, sizeof buf, "%.2e %.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n",
                   I * (p.hx), J * (p.hy), F.Sw[l], F.Sn[l], F.Sg[l], F.Pw[l], F.T[l], F.uxw[l], (-1) * F.uyw[l],
                   F.uxn[l], (-1) * F.uyn[l], F.uxg[l], (-1) * F.uyg[l], F.m[l]);
    else
      n = snprintf(buf, sizeof buf,
                   "%.2e %.2e %.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n",
                   I * (p.hx), K * (p.hz), J * (p.hy), F.Sw[l], F.Sn[l], F.Sg[l], F.Pw[l], F.T[l], F.uxw[l],
                   F.uzw[l], (-1) * F.uyw[l], F.uxn[l], F.uzn[l], (-1) * F.uyn[l], F.uxg[l], F.uzg[l],
                   (-1) * F.uyg[l], F.m[l]);
  } else if (p.nz < 2 && p.nx < 2) {
    n = snprintf(buf, sizeof buf, "%.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n", J * (p.hy), F.Sw[l], F.Sn[l],
                 F.Sg[l], F.Pw[l], (-1) * F.uyw[l], (-1) * F.uyn[l], (-1) * F.uyg[l], F.m[l]);
  } else if (p.nz < 2) {
    n = snprintf(buf, sizeof buf, "%.2e %.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n", I * (p.hx),
                 J * (p.hy), F.Sw[l], F.Sn[l], F.Sg[l], F.Pw[l], F.uxw[l], (-1) * F.uyw[l], F.uxn[l],
                 (-1) * F.uyn[l], F.uxg[l], (-1) * F.uyg[l], F.m[l]);
  } else {
    n = snprintf(buf, sizeof buf,
                 "%.2e %.2e %.2e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e %.5e\n", I * (p.hx),
                 K * (p.hz), J * (p.hy), F.Sw[l], F.Sn[l], F.Sg[l], F.Pw[l], F.uxw[l], F.uzw[l], (-1) * F.uyw[l],
                 F.uxn[l], F.uzn[l], (-1) * F.uyn[l], F.uxg[l], F.uzg[l], (-1) * F.uyg[l], F.m[l]);
  }
  out.append(buf, (size_t)std::max(0, std::min(n, (int)sizeof buf - 1)));
}

void plot_header(const capaz_params& p, double t, std::string& out) {
  char buf[512];
  snprintf(buf, sizeof buf, "TITLE =  \"Filtration in time=%5.2f\" \n", t);
  out += buf;
  if (p.model == CAPAZ_MODEL_ENERGY) {
    if (p.nz < 2 && p.nx < 2) {
      out += "VARIABLES = \"Y\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"T\",\"uw_y\",\"un_y\",\"ug_y\",\"porosity\" \n";
      snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d, F = POINT\n", p.ny);
    } else if (p.nz < 2) {
      out += "VARIABLES = \"X\",\"Y\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"T\",\"uw_x\",\"uw_y\",\"un_x\",\"un_y\","
             "\"ug_x\",\"ug_y\",\"porosity\" \n";
      snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d,J=%d, F = POINT\n", p.nx, p.ny);
    } else {
      out += "VARIABLES = \"X\",\"Y\",\"Z\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"T\",\"uw_x\",\"uw_y\",\"uw_z\","
             "\"un_x\",\"un_y\",\"un_z\",\"ug_x\",\"ug_y\",\"ug_z\",\"porosity\" \n";
      snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d,J=%d,I=%d, F = POINT\n", p.nx, p.ny, p.nz);
    }
    out += buf;
    return;
  }
  if (p.nz < 2) {
    if (p.nx < 2) {
      out += p.phases == 3
                 ? "VARIABLES = \"Y\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"uw_y\",\"un_y\",\"ug_y\",\"porosity\" \n"
                 : "VARIABLES = \"Y\",\"S_w\",\"P_w\",\"u_y\",\"porosity\" \n";
      snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d, F = POINT\n", p.ny);
    } else {
      out += p.phases == 3 ? "VARIABLES = \"X\",\"Y\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"uw_x\",\"uw_y\",\"un_x\","
                             "\"un_y\",\"ug_x\",\"ug_y\",\"porosity\" \n"
                           : "VARIABLES = \"X\",\"Y\",\"S_w\",\"P_w\",\"u_x\", \"u_y\", \"porosity\" \n";
      snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d,J=%d, F = POINT\n", p.nx, p.ny);
    }
  } else {
    out += p.phases == 3 ? "VARIABLES = \"X\",\"Y\",\"Z\",\"S_w\",\"S_n\",\"S_g\",\"P_w\",\"uw_x\",\"uw_y\",\"uw_z\","
                           "\"un_x\",\"un_y\",\"un_z\",\"ug_x\",\"ug_y\",\"ug_z\",\"porosity\" \n"
                         : "VARIABLES = \"X\",\"Y\",\"Z\",\"S_n\",\"P_w\",\"u_x\", \"u_y\", \"u_z\", \"porosity\" \n";
    snprintf(buf, sizeof buf, "ZONE T = \"BIG ZONE\", K=%d,J=%d,I=%d, F = POINT\n", p.nx, p.ny, p.nz);
  }
  out += buf;
}

int make_dir(const char* dir) {
  if (mkdir(dir, 0777) == 0 || errno == EEXIST) return 0;
  return -1;
}

}  // namespace

extern "C" {

int capaz_write_plot(capaz_ctx* ctx, const char* dir, double t) {
  if (!ctx || !dir) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  PlotFields F;
  struct Want {
    int field;
    std::vector<double>* dst;
  };
  std::vector<Want> want = {{CAPAZ_FIELD_P_W, &F.Pw}, {CAPAZ_FIELD_S_N, &F.Sn}, {CAPAZ_FIELD_M, &F.m},
                            {CAPAZ_FIELD_UX_N, &F.uxn}, {CAPAZ_FIELD_UY_N, &F.uyn}, {CAPAZ_FIELD_UZ_N, &F.uzn}};
  if (p.phases == 3) {
    const Want more[] = {{CAPAZ_FIELD_S_W, &F.Sw},   {CAPAZ_FIELD_S_G, &F.Sg},   {CAPAZ_FIELD_UX_W, &F.uxw},
                         {CAPAZ_FIELD_UY_W, &F.uyw}, {CAPAZ_FIELD_UZ_W, &F.uzw}, {CAPAZ_FIELD_UX_G, &F.uxg},
                         {CAPAZ_FIELD_UY_G, &F.uyg}, {CAPAZ_FIELD_UZ_G, &F.uzg}};
    want.insert(want.end(), std::begin(more), std::end(more));
  }
  if (p.model == CAPAZ_MODEL_ENERGY) want.push_back({CAPAZ_FIELD_T, &F.T});
  if (p.model == CAPAZ_MODEL_BUCKLEY_LEVERETT) {
    if (p.flags & CAPAZ_FLAG_PERCELL_K) want.push_back({CAPAZ_FIELD_K, &F.K});
    else F.K.assign(ctx->n, p.K0);
  }
  for (const Want& w : want) {
    // Before the first step the reference's velocity arrays hold no values
    // yet (they are written by u_calculation); the plot shows zeros.
    const bool velocity = w.field >= CAPAZ_FIELD_UX_W && w.field <= CAPAZ_FIELD_UZ_G;
    if (velocity && ctx->steps_done == 0) {
      w.dst->assign(ctx->n, 0.);
      continue;
    }
    int st = fetch(ctx, w.field, *w.dst);
    if (st) return st;
  }
  if (make_dir(dir)) return io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, std::string("cannot create ") + dir);
  char name[64];
  snprintf(name, sizeof name, "/S=%012.4f.dat", t);
  const std::string path = std::string(dir) + name;
  FILE* fp = fopen(path.c_str(), "wt");
  if (!fp) return io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, "cannot open " + path);
  std::string head;
  plot_header(p, t, head);
  fwrite(head.data(), 1, head.size(), fp);
  // Rows in the reference's order (i outer), formatted in i-slices.
  const int nthreads = std::max(1, std::min(64, (int)std::thread::hardware_concurrency()));
  const int per = std::max(1, (p.nx + nthreads - 1) / nthreads);
  std::vector<std::string> parts((p.nx + per - 1) / per);
  std::vector<std::thread> pool;
  for (size_t q = 0; q < parts.size(); q++)
    pool.emplace_back([&, q] {
      std::string& out = parts[q];
      const int i0 = (int)q * per, i1 = std::min(p.nx, i0 + per);
      out.reserve((size_t)(i1 - i0) * p.ny * p.nz * 96);
      for (int i = i0; i < i1; i++)
        for (int j = 0; j < p.ny; j++)
          for (int k = 0; k < p.nz; k++) plot_row(p, F, i, j, k, out);
    });
  for (auto& th : pool) th.join();
  bool ok = true;
  for (const std::string& s : parts) ok = ok && fwrite(s.data(), 1, s.size(), fp) == s.size();
  ok = (fclose(fp) == 0) && ok;
  return ok ? CAPAZ_OK : io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, "write failed: " + path);
}

int capaz_save(capaz_ctx* ctx, const char* path, int time_counter) {
  if (!ctx || !path) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  std::vector<int> order;
  if (p.phases == 3) order.push_back(CAPAZ_FIELD_S_W);
  order.insert(order.end(), {CAPAZ_FIELD_P_W, CAPAZ_FIELD_S_N, CAPAZ_FIELD_ROS_W_OLD, CAPAZ_FIELD_ROS_N_OLD});
  if (p.phases == 3) order.push_back(CAPAZ_FIELD_ROS_G_OLD);
  order.push_back(CAPAZ_FIELD_M);
  std::vector<std::vector<double>> data(order.size());
  for (size_t q = 0; q < order.size(); q++) {
    int st = fetch(ctx, order[q], data[q]);
    if (st) return st;
  }
  FILE* f = fopen(path, "wb");
  if (!f) return io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  const int32_t tc = time_counter;
  bool ok = fwrite(&tc, sizeof tc, 1, f) == 1;
  for (const auto& d : data) ok = ok && fwrite(d.data(), sizeof(double), d.size(), f) == d.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? CAPAZ_OK : io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
}

int capaz_restore(capaz_ctx* ctx, const char* path, int* time_counter) {
  if (!ctx || !path) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  const size_t n = (size_t)ctx->n;
  const int nfields = p.phases == 3 ? 7 : 5;
  FILE* f = fopen(path, "rb");
  if (!f) return io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  int32_t tc = 0;
  std::vector<std::vector<double>> data(nfields, std::vector<double>(n));
  bool ok = fread(&tc, sizeof tc, 1, f) == 1;
  for (auto& d : data) ok = ok && fread(d.data(), sizeof(double), n, f) == n;
  const bool extra = ok && fgetc(f) != EOF;
  fclose(f);
  if (!ok || extra)
    return io_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT,
                   std::string(path) + ": size does not match this grid and phase count");
  // Layout: [S_w], P_w, S_n, roS_w_old, roS_n_old, [roS_g_old], m.
  const int off = p.phases == 3 ? 1 : 0;
  int st = capaz_set_field(ctx, CAPAZ_FIELD_M, data[nfields - 1].data(), nullptr);
  if (!st && p.phases == 3) st = capaz_set_field(ctx, CAPAZ_FIELD_S_W, data[0].data(), nullptr);
  if (!st) st = capaz_set_field(ctx, CAPAZ_FIELD_P_W, data[off].data(), nullptr);
  if (!st) st = capaz_set_field(ctx, CAPAZ_FIELD_S_N, data[off + 1].data(), nullptr);
  if (!st && p.phases == 3) {
    // The three-phase CPU model has no capillary pressure: P_n = P_g = P_w.
    st = capaz_set_field(ctx, CAPAZ_FIELD_P_N, data[off].data(), nullptr);
    if (!st) st = capaz_set_field(ctx, CAPAZ_FIELD_P_G, data[off].data(), nullptr);
  }
  if (st) return st;
  if (time_counter) *time_counter = tc;
  return CAPAZ_OK;
}

}  // extern "C"
