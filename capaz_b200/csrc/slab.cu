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

}  // extern "C"
