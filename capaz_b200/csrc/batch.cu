// Ensembles of uneven two-phase instances stepped by one persistent launch
// per step (capaz_batch_* in include/capaz_b200.h).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "capaz_ctx.h"
#include "capaz_internal.h"

using namespace capaz;

struct capaz_batch {
  std::vector<capaz_ctx*> ctx;
  int device = 0;
  bool fp32 = false;
  PhysF phys{};
  bool unik = true, pd0 = true, planar = false;
  InstT* d_instT = nullptr;
  Inst64* d_inst64 = nullptr;
  int4* d_items = nullptr;
  int nitems = 0;
  int2* d_bitems = nullptr;  // boundary-kernel blocks (precision form)
  int nbitems = 0;
  size_t items_cap = 0;
  unsigned int* counter = nullptr;
  int zchunk = 16;
  int ctas_per_sm = 0;  // 0: as many as fit
  int tile_y = TMA_TILE_Y;  // rows of a sweep tile (precision form)
  int grid = 0;
  std::vector<double> built_dt, built_Sref;
  bool built = false;
  cudaGraphExec_t pair = nullptr;  // two steps (parity 0 then 1), captured
  cudaGraph_t pair_graph = nullptr;
  long long launches = 0;
  std::string last_error;
};

namespace {

thread_local std::string g_batch_error;

int bfail(capaz_batch* b, int code, const std::string& msg) {
  if (b) b->last_error = msg;
  g_batch_error = msg;
  return code;
}

int bcuda(capaz_batch* b, cudaError_t e, const char* what) {
  return bfail(b, e == cudaErrorMemoryAllocation ? CAPAZ_ERR_OUT_OF_MEMORY : CAPAZ_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

#define BTRY(b, call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return bcuda(b, e_, #call); \
  } while (0)

int occupancy(const capaz_batch* b) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const int full = b->fp32 ? step2_fp32c_tma_grid(b->device, b->unik, b->tile_y) : step2_fp64_batch_grid(b->device);
  return std::max(1, full / std::max(1, sms));
}

// (Re)builds the per-instance descriptors and the work-item list for the
// current z-chunk depth.  Items are ordered z-chunk-major across instances.
int build(capaz_batch* b) {
  const int n = (int)b->ctx.size();
  BTRY(b, cudaSetDevice(b->device));
  std::vector<int> nz_chunks(n), ntiles(n);
  if (b->fp32) {
    std::vector<InstT> h(n);
    for (int q = 0; q < n; q++) {
      capaz_ctx* x = b->ctx[q];
      // The instance's own TMA descriptor carries its maps and arguments;
      // rebuild it for the batch's tile shape and z-chunk depth.
      x->tma_tile_y = b->tile_y;
      int st = x->tma_prepare();
      if (st) return bfail(b, st, x->last_error);
      BTRY(b, cudaMemcpy(&h[q], x->tma_inst, sizeof(InstT), cudaMemcpyDeviceToHost));
      if (x->p.nz > 1) {
        const int interior = x->p.nz - 2;
        h[q].zchunk = std::min(b->zchunk, interior);
        h[q].nzchunks = (interior + h[q].zchunk - 1) / h[q].zchunk;
      }
      nz_chunks[q] = h[q].nzchunks;
      ntiles[q] = h[q].tiles_x * h[q].tiles_y;
    }
    if (!b->d_instT) BTRY(b, cudaMalloc(&b->d_instT, sizeof(InstT) * n));
    BTRY(b, cudaMemcpy(b->d_instT, h.data(), sizeof(InstT) * n, cudaMemcpyHostToDevice));
  } else {
    std::vector<Inst64> h(n);
    for (int q = 0; q < n; q++) {
      capaz_ctx* x = b->ctx[q];
      Step2Const c = make_step2_const(x->p);
      if (x->p.nz > 1) {
        const int interior = x->p.nz - 2;
        c.zchunk = std::min(b->zchunk, interior);
        c.nzchunks = (interior + c.zchunk - 1) / c.zchunk;
      }
      h[q].c = c;
      for (int par = 0; par < 2; par++) {
        h[q].Pw[par] = (double*)x->state[par][0];
        h[q].Sn[par] = (double*)x->state[par][1];
      }
      h[q].m = (const double*)x->m;
      h[q].K = (const double*)x->K;
      h[q].err = x->err_flag;
      nz_chunks[q] = c.nzchunks;
      ntiles[q] = c.tiles_x * c.tiles_y;
    }
    if (!b->d_inst64) BTRY(b, cudaMalloc(&b->d_inst64, sizeof(Inst64) * n));
    BTRY(b, cudaMemcpy(b->d_inst64, h.data(), sizeof(Inst64) * n, cudaMemcpyHostToDevice));
  }
  std::vector<int4> items;
  const int maxc = *std::max_element(nz_chunks.begin(), nz_chunks.end());
  for (int zc = 0; zc < maxc; zc++)
    for (int q = 0; q < n; q++)
      if (zc < nz_chunks[q])
        for (int t = 0; t < ntiles[q]; t++) {
          if (b->fp32) {
            // The precision sweep takes explicit z ranges: centres kb .. ke-1.
            const capaz_params& pq = b->ctx[q]->p;
            const int zq = std::min(b->zchunk, std::max(pq.nz - 2, 1));
            const int kb = pq.nz == 1 ? 0 : 1 + zc * zq, ke = pq.nz == 1 ? 0 : std::min(kb + zq, pq.nz - 1);
            items.push_back(make_int4(q, t, kb, ke));
          } else {
            items.push_back(make_int4(q, t, zc, 0));
          }
        }
  b->nitems = (int)items.size();
  if (items.size() > b->items_cap) {
    if (b->d_items) cudaFree(b->d_items);
    BTRY(b, cudaMalloc(&b->d_items, sizeof(int4) * items.size()));
    b->items_cap = items.size();
  }
  BTRY(b, cudaMemcpy(b->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
  if (b->fp32 && !b->d_bitems) {
    std::vector<int2> bitems;
    for (int q = 0; q < n; q++) {
      const capaz_params& pq = b->ctx[q]->p;
      const int nb = boundary_cells(pq.nx, pq.ny, pq.nz);
      for (int f0 = 0; f0 < nb; f0 += BOUND_BLOCK) bitems.push_back(make_int2(q, f0));
    }
    b->nbitems = (int)bitems.size();
    BTRY(b, cudaMalloc(&b->d_bitems, sizeof(int2) * bitems.size()));
    BTRY(b, cudaMemcpy(b->d_bitems, bitems.data(), sizeof(int2) * bitems.size(), cudaMemcpyHostToDevice));
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const int per = b->ctas_per_sm > 0 ? std::min(b->ctas_per_sm, occupancy(b)) : occupancy(b);
  b->grid = std::max(1, std::min(b->nitems, sms * per));
  b->built_dt.resize(n);
  b->built_Sref.resize(n);
  for (int q = 0; q < n; q++) {
    b->built_dt[q] = b->ctx[q]->p.dt;
    b->built_Sref[q] = b->ctx[q]->S_ref;
  }
  if (b->pair) {
    cudaGraphExecDestroy(b->pair);
    cudaGraphDestroy(b->pair_graph);
    b->pair = nullptr;
    b->pair_graph = nullptr;
  }
  b->built = true;
  return CAPAZ_OK;
}

bool stale(const capaz_batch* b) {
  if (!b->built) return true;
  for (size_t q = 0; q < b->ctx.size(); q++)
    if (b->ctx[q]->p.dt != b->built_dt[q] || b->ctx[q]->S_ref != b->built_Sref[q]) return true;
  return false;
}

// Kernels one step launches: the precision form's sweep is followed by its
// boundary kernel.
int kernels_per_step(const capaz_batch* b) { return b->fp32 ? 2 : 1; }

cudaError_t launch_one(capaz_batch* b, int parity, cudaStream_t s) {
  if (b->fp32) {
    cudaError_t e = launch_step2_fp32c_tma(b->phys, b->d_instT, b->d_items, b->nitems, parity, b->unik, b->planar,
                                           b->counter, nullptr, b->grid, s, nullptr, b->tile_y);
    return e != cudaSuccess ? e : launch_boundary_fp32c(b->phys, b->d_instT, b->d_bitems, b->nbitems, parity, s);
  }
  return launch_step2_fp64_batch(b->d_inst64, b->d_items, b->nitems, parity, b->unik, b->pd0, b->counter, b->grid, s);
}

void advance(capaz_batch* b, int nsteps) {
  for (auto* x : b->ctx) {
    x->cur ^= (nsteps & 1);
    x->steps_done += nsteps;
  }
}

int capture_pair(capaz_batch* b) {
  cudaStream_t cs;
  BTRY(b, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = launch_one(b, 0, cs);
  if (e == cudaSuccess) e = launch_one(b, 1, cs);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->pair, g, 0);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    b->pair = nullptr;
    return bcuda(b, e, "graph capture");
  }
  b->pair_graph = g;
  return CAPAZ_OK;
}

int run_steps(capaz_batch* b, int nsteps, cudaStream_t s, bool use_graph) {
  if (stale(b)) {
    int st = build(b);
    if (st) return st;
  }
  int cur = b->ctx[0]->cur;
  for (auto* x : b->ctx)
    if (x->cur != cur) return bfail(b, CAPAZ_ERR_BAD_STATE, "instances were stepped separately; parities differ");
  int done = 0;
  if (use_graph && nsteps >= 2) {
    if (!b->pair) {
      int st = capture_pair(b);
      if (st) return st;
    }
    // The pair graph starts at parity 0: align with one plain launch first.
    if (cur == 1) {
      BTRY(b, launch_one(b, 1, s));
      b->launches += kernels_per_step(b);
      advance(b, 1);
      done = 1;
      cur = 0;
    }
    while (nsteps - done >= 2) {
      BTRY(b, cudaGraphLaunch(b->pair, s));
      b->launches += 2 * kernels_per_step(b);
      advance(b, 2);
      done += 2;
    }
  }
  while (done < nsteps) {
    BTRY(b, launch_one(b, b->ctx[0]->cur, s));
    b->launches += kernels_per_step(b);
    advance(b, 1);
    done++;
  }
  return CAPAZ_OK;
}

}  // namespace

extern "C" {

capaz_batch* capaz_batch_create(const capaz_params* params, int count, int device, int* status) {
  if (!params || count <= 0) {
    if (status) *status = CAPAZ_ERR_INVALID_ARGUMENT;
    return nullptr;
  }
  const capaz_params& p0 = params[0];
  for (int q = 0; q < count; q++) {
    const capaz_params& p = params[q];
    const bool same = p.phases == 2 && p.model == CAPAZ_MODEL_DEFAULT && p.form == p0.form && p.flags == p0.flags &&
                      (p.lambda == 2.0) == (p0.lambda == 2.0) && (p.P_d == 0.) == (p0.P_d == 0.);
    // Precision-form batches run the TMA-staged kernel: nx % 4 == 0, P_d = 0,
    // lambda = 2, and one set of physics constants for all instances.
    PhysF a = make_physf(p), z = make_physf(p0);
    const bool tma_ok = p.form != CAPAZ_FORM_FP32C ||
                        (p.nx % 4 == 0 && p.ny >= 4 && (p.nz == 1 || p.nz >= 4) && p.P_d == 0. && p.lambda == 2.0 &&
                         memcmp(&a, &z, sizeof a) == 0 && (p.nz == 1) == (p0.nz == 1));
    if (!same || !tma_ok) {
      g_batch_error = "batch instances must be two-phase with the same form, flags and model class; "
                      "precision-form batches need nx % 4 == 0, ny >= 4, nz == 1 or >= 4, P_d = 0, lambda = 2, "
                      "identical physics and "
                      "all instances planar (nz == 1) or all three-dimensional";
      if (status) *status = CAPAZ_ERR_INVALID_ARGUMENT;
      return nullptr;
    }
  }
  capaz_batch* b = new capaz_batch();
  b->device = device;
  b->fp32 = p0.form == CAPAZ_FORM_FP32C;
  b->unik = !(p0.flags & CAPAZ_FLAG_PERCELL_K);
  b->pd0 = p0.P_d == 0.;
  b->planar = p0.nz == 1;
  b->phys = make_physf(p0);
  for (int q = 0; q < count; q++) {
    int st = 0;
    capaz_ctx* x = capaz_create(&params[q], device, &st);
    if (!x) {
      g_batch_error = std::string("instance ") + std::to_string(q) + ": " + capaz_last_error(nullptr);
      capaz_batch_destroy(b);
      if (status) *status = st;
      return nullptr;
    }
    b->ctx.push_back(x);
  }
  // The work counter starts at zero; the precision form's boundary kernel
  // rearms it after every sweep.
  if (cudaMalloc(&b->counter, sizeof(unsigned int) * SWEEP_COUNTERS) != cudaSuccess ||
      cudaMemset(b->counter, 0, sizeof(unsigned int) * SWEEP_COUNTERS) != cudaSuccess) {
    capaz_batch_destroy(b);
    if (status) *status = CAPAZ_ERR_OUT_OF_MEMORY;
    return nullptr;
  }
  if (status) *status = CAPAZ_OK;
  return b;
}

int capaz_batch_destroy(capaz_batch* b) {
  if (!b) return CAPAZ_ERR_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  if (b->pair) cudaGraphExecDestroy(b->pair);
  if (b->pair_graph) cudaGraphDestroy(b->pair_graph);
  if (b->d_instT) cudaFree(b->d_instT);
  if (b->d_inst64) cudaFree(b->d_inst64);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_bitems) cudaFree(b->d_bitems);
  if (b->counter) cudaFree(b->counter);
  for (auto* x : b->ctx) capaz_destroy(x);
  delete b;
  return CAPAZ_OK;
}

capaz_ctx* capaz_batch_instance(capaz_batch* b, int index) {
  if (!b || index < 0 || index >= (int)b->ctx.size()) return nullptr;
  return b->ctx[index];
}

int capaz_batch_step(capaz_batch* b, int nsteps, void* stream) {
  if (!b || nsteps < 0) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (nsteps == 0) return CAPAZ_OK;
  BTRY(b, cudaSetDevice(b->device));
  return run_steps(b, nsteps, (cudaStream_t)stream, true);
}

int64_t capaz_batch_launch_count(const capaz_batch* b) { return b ? b->launches : -1; }

int capaz_batch_autotune(capaz_batch* b, void* stream, int* zchunk_out, int* per_sm_out) {
  if (!b) return CAPAZ_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  BTRY(b, cudaSetDevice(b->device));
  // Snapshot every instance's current state (P_w, S_n of buffer `cur`).
  const size_t es = b->fp32 ? sizeof(float) : sizeof(double);
  std::vector<void*> snap;
  for (auto* x : b->ctx) {
    for (int f = 0; f < 2; f++) {
      void* d = nullptr;
      BTRY(b, cudaMalloc(&d, x->n * es));
      BTRY(b, cudaMemcpyAsync(d, x->state[x->cur][f], x->n * es, cudaMemcpyDeviceToDevice, s));
      snap.push_back(d);
    }
  }
  std::vector<long long> done0;
  for (auto* x : b->ctx) done0.push_back(x->steps_done);
  const int zc_cands[4] = {8, 16, 32, 64};
  // Tile shapes: 32 x 16 and 32 x 32 for the precision form's sweep; the
  // FP64 batch kernel has one.
  const int tile_cands[2] = {16, 32};
  const int ntile = b->fp32 ? 2 : 1;
  float best = 1e30f;
  int best_zc = b->zchunk, best_per = 0, best_tile = b->tile_y;
  cudaEvent_t e0, e1;
  BTRY(b, cudaEventCreate(&e0));
  BTRY(b, cudaEventCreate(&e1));
  int rc = CAPAZ_OK;
  for (int ti = 0; ti < ntile && rc == CAPAZ_OK; ti++) {
    if (b->fp32) b->tile_y = tile_cands[ti];
    const int occ = occupancy(b);
    for (int zc : zc_cands) {
      for (int per = 1; per <= occ && rc == CAPAZ_OK; per++) {
        b->zchunk = zc;
        b->ctas_per_sm = per;
        if ((rc = build(b))) break;
        if ((rc = run_steps(b, 2, s, false))) break;  // warm-up (even: parity preserved)
        cudaEventRecord(e0, s);
        if ((rc = run_steps(b, 6, s, false))) break;
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          best_zc = zc;
          best_per = per;
          best_tile = b->tile_y;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // Restore the state and step counts.
  size_t k = 0;
  for (size_t q = 0; q < b->ctx.size(); q++) {
    capaz_ctx* x = b->ctx[q];
    for (int f = 0; f < 2; f++, k++) {
      cudaMemcpyAsync(x->state[x->cur][f], snap[k], x->n * es, cudaMemcpyDeviceToDevice, s);
    }
    x->steps_done = done0[q];
  }
  cudaStreamSynchronize(s);
  for (void* d : snap) cudaFree(d);
  if (rc) return rc;
  b->zchunk = best_zc;
  b->ctas_per_sm = best_per;
  b->tile_y = best_tile;
  int st = build(b);
  if (st) return st;
  if (zchunk_out) *zchunk_out = best_zc;
  if (per_sm_out) *per_sm_out = best_per;
  return CAPAZ_OK;
}

int capaz_batch_get_tuning(const capaz_batch* b, int* zchunk, int* ctas_per_sm, int* tile_y) {
  if (!b) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (zchunk) *zchunk = b->zchunk;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  if (tile_y) *tile_y = b->fp32 ? b->tile_y : 0;
  return CAPAZ_OK;
}

int capaz_batch_set_tuning(capaz_batch* b, int zchunk, int ctas_per_sm, int tile_y) {
  if (!b || zchunk < 1 || ctas_per_sm < 0) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (b->fp32 && !tma_tile_supported(tile_y)) return bfail(b, CAPAZ_ERR_UNSUPPORTED, "tile_y must be 16 or 32");
  BTRY(b, cudaSetDevice(b->device));
  BTRY(b, cudaDeviceSynchronize());  // earlier steps may still read the descriptors
  b->zchunk = zchunk;
  b->ctas_per_sm = ctas_per_sm;
  if (b->fp32) b->tile_y = tile_y;
  return build(b);
}

}  // extern "C"
