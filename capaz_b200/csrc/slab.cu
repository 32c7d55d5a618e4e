// Plane access for the z-slab decomposition of a grid over several GPUs:
// the halo exchange after each step moves one z-plane of each state field
// between neighbouring ranks (the reference's P_S_exchange, mpi.cpp:113-294,
// reduced to one exchange of the state per step: every derived quantity is
// recomputed from the state in the halo).
//
// capaz_get_plane / capaz_set_plane read and write plane k of the current
// state as float64 (nx*ny values, index i + j*nx) in device memory; the
// precision form decodes / encodes with the context's reference state.
#include "capaz_ctx.h"
#include "capaz_internal.h"

using namespace capaz;

namespace {

__global__ void plane_decode_kernel(const float* __restrict__ a, const double* __restrict__ Pref, double S_ref,
                                    int nx, int n, bool pressure, double* __restrict__ out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  out[l] = (pressure ? Pref[l / nx] : S_ref) + (double)a[l];
}

__global__ void plane_encode_kernel(const double* __restrict__ v, const double* __restrict__ Pref, double S_ref,
                                    int nx, int n, bool pressure, float* __restrict__ out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  out[l] = (float)(v[l] - (pressure ? Pref[l / nx] : S_ref));
}

int plane_args(capaz_ctx* ctx, int field, int k, int* slot) {
  if (!ctx) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  *slot = capaz_ctx::state_slot(field);
  const bool state = field == CAPAZ_FIELD_P_W || field == CAPAZ_FIELD_S_N ||
                     (p.phases == 3 && (field == CAPAZ_FIELD_S_W || field == CAPAZ_FIELD_P_N || field == CAPAZ_FIELD_P_G));
  if (!state || *slot < 0) return ctx->fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "planes are of the state fields only");
  if (k < 0 || k >= p.nz) return ctx->fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "plane index out of range");
  return CAPAZ_OK;
}

}  // namespace

extern "C" {

int capaz_get_plane(capaz_ctx* ctx, int field, int k, double* dst, void* stream) {
  int slot = 0;
  int st = plane_args(ctx, field, k, &slot);
  if (st || !dst) return st ? st : CAPAZ_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaSetDevice");
  const capaz_params& p = ctx->p;
  const int n = p.nx * p.ny;
  cudaStream_t s = (cudaStream_t)stream;
  if (p.form == CAPAZ_FORM_FP64) {
    const double* src = (const double*)ctx->state[ctx->cur][slot] + (size_t)k * n;
    e = cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  } else {
    const float* src = (const float*)ctx->state[ctx->cur][slot] + (size_t)k * n;
    plane_decode_kernel<<<(n + 255) / 256, 256, 0, s>>>(src, ctx->Pref, ctx->S_ref, p.nx, n,
                                                         field == CAPAZ_FIELD_P_W, dst);
    ctx->launches++;
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? CAPAZ_OK : ctx->fail_cuda(e, "capaz_get_plane");
}

int capaz_set_plane(capaz_ctx* ctx, int field, int k, const double* src, void* stream) {
  int slot = 0;
  int st = plane_args(ctx, field, k, &slot);
  if (st || !src) return st ? st : CAPAZ_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaSetDevice");
  const capaz_params& p = ctx->p;
  const int n = p.nx * p.ny;
  cudaStream_t s = (cudaStream_t)stream;
  if (p.form == CAPAZ_FORM_FP64) {
    double* dst = (double*)ctx->state[ctx->cur][slot] + (size_t)k * n;
    e = cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  } else {
    float* dst = (float*)ctx->state[ctx->cur][slot] + (size_t)k * n;
    plane_encode_kernel<<<(n + 255) / 256, 256, 0, s>>>(src, ctx->Pref, ctx->S_ref, p.nx, n,
                                                         field == CAPAZ_FIELD_P_W, dst);
    ctx->launches++;
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? CAPAZ_OK : ctx->fail_cuda(e, "capaz_set_plane");
}

// Plane k of a state field in its stored representation (float64 in the
// FP64 form, the float32 deviation in the precision form), device to device:
// the halo exchange of slabs that share one reference state moves these
// bytes unchanged.
int capaz_get_plane_raw(capaz_ctx* ctx, int field, int k, void* dst, void* stream) {
  int slot = 0;
  int st = plane_args(ctx, field, k, &slot);
  if (st || !dst) return st ? st : CAPAZ_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaSetDevice");
  const capaz_params& p = ctx->p;
  const size_t es = p.form == CAPAZ_FORM_FP64 ? sizeof(double) : sizeof(float), n = (size_t)p.nx * p.ny;
  const char* src = (const char*)ctx->state[ctx->cur][slot] + (size_t)k * n * es;
  e = cudaMemcpyAsync(dst, src, n * es, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? CAPAZ_OK : ctx->fail_cuda(e, "capaz_get_plane_raw");
}

int capaz_set_plane_raw(capaz_ctx* ctx, int field, int k, const void* src, void* stream) {
  int slot = 0;
  int st = plane_args(ctx, field, k, &slot);
  if (st || !src) return st ? st : CAPAZ_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaSetDevice");
  const capaz_params& p = ctx->p;
  const size_t es = p.form == CAPAZ_FORM_FP64 ? sizeof(double) : sizeof(float), n = (size_t)p.nx * p.ny;
  char* dst = (char*)ctx->state[ctx->cur][slot] + (size_t)k * n * es;
  e = cudaMemcpyAsync(dst, src, n * es, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? CAPAZ_OK : ctx->fail_cuda(e, "capaz_set_plane_raw");
}

// The precision form's reference state: per-row reference pressure (ny
// values) and reference saturation S_n.
int capaz_get_reference(capaz_ctx* ctx, double* Pref, double* S_ref) {
  if (!ctx || !Pref || !S_ref) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  if (p.form != CAPAZ_FORM_FP32C || p.phases != 2)
    return ctx->fail_msg(CAPAZ_ERR_UNSUPPORTED, "a reference state belongs to the two-phase precision form");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(Pref, ctx->Pref, sizeof(double) * p.ny, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "capaz_get_reference");
  *S_ref = ctx->S_ref;
  return CAPAZ_OK;
}

// Fixes the reference state: the current state is decoded with the old
// reference and encoded with the new one, and later P_w / S_n (set_field,
// init_state) are encoded against it instead of their own means.
int capaz_set_reference(capaz_ctx* ctx, const double* Pref, double S_ref) {
  if (!ctx || !Pref || !(S_ref == S_ref)) return CAPAZ_ERR_INVALID_ARGUMENT;
  const capaz_params& p = ctx->p;
  if (p.form != CAPAZ_FORM_FP32C || p.phases != 2)
    return ctx->fail_msg(CAPAZ_ERR_UNSUPPORTED, "a reference state belongs to the two-phase precision form");
  for (int j = 0; j < p.ny; j++)
    if (!(Pref[j] == Pref[j]) || Pref[j] - Pref[j] != 0.)
      return ctx->fail_msg(CAPAZ_ERR_INVALID_ARGUMENT, "reference pressures must be finite");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaSetDevice");
  e = cudaDeviceSynchronize();  // steps in flight read the old reference
  if (e != cudaSuccess) return ctx->fail_cuda(e, "cudaDeviceSynchronize");
  int st = ctx->decode_all(ctx->cur, nullptr);
  if (st) return st;
  const long long n = ctx->n;
  e = cudaMemcpy(ctx->Pref, Pref, sizeof(double) * p.ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->S_ref_dev, &S_ref, sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_pref_tables(ctx->Pref, p.ny, p.P_atm, ctx->PrelF, ctx->dPrefF, nullptr);
  if (e == cudaSuccess) e = launch_row_tables(ctx->Pref, p.ny, make_physf(p), ctx->rowF, nullptr);
  if (e == cudaSuccess)
    e = launch_encode_pressure_rel(ctx->wide[0], ctx->Pref, p.nx, p.ny, n, (float*)ctx->state[ctx->cur][0], nullptr);
  if (e == cudaSuccess) e = launch_encode_saturation_ref(ctx->wide[1], n, ctx->S_ref_dev, (float*)ctx->state[ctx->cur][1], nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return ctx->fail_cuda(e, "capaz_set_reference");
  ctx->launches += 4;
  ctx->S_ref = S_ref;
  ctx->ref_locked = true;
  ctx->tma_ready = false;  // S_ref is part of the sweep's descriptor
  return CAPAZ_OK;
}

}  // extern "C"
