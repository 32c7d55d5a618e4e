// Device-side field preparation for the C ABI (set-up path, not the step):
// validation of porosity/permeability and the precision form's encoding of
// a float64 state into FP32 deviations from a reference state.
#include <math.h>

#include "capaz_internal.h"

namespace capaz {
namespace {

// Smallest index of a cell that is not finite and > 0 (or n if none).
__global__ void first_invalid_kernel(const double* __restrict__ a, long long n, unsigned long long* __restrict__ first) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const double v = a[l];
    if (!(v > 0.) || !isfinite(v)) atomicMin(first, (unsigned long long)l);
  }
}

// Row sums of a (nz, ny, nx) field: one block per row j, fixed order.
__global__ void row_mean_kernel(const double* __restrict__ a, int nx, int ny, int nz, double* __restrict__ out) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  const long long sy = nx, sz = (long long)nx * ny;
  const long long cnt = (long long)nx * nz;
  double s = 0.;
  for (long long q = threadIdx.x; q < cnt; q += blockDim.x) {
    const int i = (int)(q % nx), k = (int)(q / nx);
    s += a[i + j * sy + k * sz];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0] / (double)cnt;
}

// Partial sums over fixed contiguous ranges (deterministic), then a final sum.
__global__ void partial_sum_kernel(const double* __restrict__ a, long long n, double* __restrict__ part) {
  __shared__ double red[256];
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  const long long b0 = blockIdx.x * per, b1 = min(n, b0 + per);
  double s = 0.;
  for (long long l = b0 + threadIdx.x; l < b1; l += blockDim.x) s += a[l];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void final_mean_kernel(const double* __restrict__ part, int nparts, long long n, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.;
    for (int q = 0; q < nparts; q++) s += part[q];
    out[0] = s / (double)n;
  }
}

__global__ void pref_tables_kernel(const double* __restrict__ Pref, int ny, double P_atm, float* __restrict__ rel,
                                   float* __restrict__ dref) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny) return;
  rel[j] = (float)(Pref[j] - P_atm);
  dref[j] = (j + 1 < ny) ? (float)(Pref[j + 1] - Pref[j]) : 0.f;
}

__global__ void encode_p_kernel(const double* __restrict__ P, const double* __restrict__ Pref, int nx, int ny,
                                long long n, float* __restrict__ out) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int j = (int)((l / nx) % ny);
  out[l] = (float)(P[l] - Pref[j]);
}

__global__ void encode_s_kernel(const double* __restrict__ S, const double* __restrict__ S_ref, long long n,
                                float* __restrict__ out) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= n) return;
  out[l] = (float)(S[l] - S_ref[0]);
}

__global__ void narrow_kernel(const double* __restrict__ a, long long n, float* __restrict__ out) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l < n) out[l] = (float)a[l];
}

__global__ void row_tables_kernel(const double* __restrict__ Pref, int ny, const PhysF f, float4* __restrict__ rowF) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny) return;
  const double prel = Pref[j] - f.P_atm;
  const double dnext = (j + 1 < ny) ? (Pref[j + 1] - Pref[j]) : 0.;
  rowF[j] = make_float4((float)((f.ro0_w + f.aw * prel) / f.mu_w), (float)((f.ro0_n + f.bn * prel) / f.mu_n),
                        (float)(dnext * (double)f.inv_hy2), 0.f);
}

unsigned grid_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

cudaError_t launch_first_invalid(const double* a, long long n, unsigned long long* first, cudaStream_t s) {
  first_invalid_kernel<<<4 * 148, 256, 0, s>>>(a, n, first);
  return cudaGetLastError();
}

cudaError_t launch_encode_pressure(const double* P, int nx, int ny, int nz, double P_atm, double* Pref, float* PrelF,
                                   float* dPrefF, float* out, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  row_mean_kernel<<<ny, 256, 0, s>>>(P, nx, ny, nz, Pref);
  pref_tables_kernel<<<(ny + 127) / 128, 128, 0, s>>>(Pref, ny, P_atm, PrelF, dPrefF);
  encode_p_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, Pref, nx, ny, n, out);
  return cudaGetLastError();
}

cudaError_t launch_encode_saturation(const double* S, long long n, double* part /* 1024 */, double* S_ref,
                                     float* out, cudaStream_t s) {
  partial_sum_kernel<<<1024, 256, 0, s>>>(S, n, part);
  final_mean_kernel<<<1, 32, 0, s>>>(part, 1024, n, S_ref);
  encode_s_kernel<<<grid_for(n, 256), 256, 0, s>>>(S, S_ref, n, out);
  return cudaGetLastError();
}

// Pressure deviations from an existing per-row reference (P_n, P_g of the
// three-phase precision form) and back.
__global__ void decode_p_kernel(const float* __restrict__ p, const double* __restrict__ Pref, int nx, int ny,
                                long long n, double* __restrict__ P) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= n) return;
  P[l] = Pref[(int)((l / nx) % ny)] + (double)p[l];
}

cudaError_t launch_encode_pressure_rel(const double* P, const double* Pref, int nx, int ny, long long n, float* out,
                                       cudaStream_t s) {
  encode_p_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, Pref, nx, ny, n, out);
  return cudaGetLastError();
}

cudaError_t launch_decode_pressure(const float* p, const double* Pref, int nx, int ny, long long n, double* out,
                                   cudaStream_t s) {
  decode_p_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, Pref, nx, ny, n, out);
  return cudaGetLastError();
}

cudaError_t launch_pref_tables(const double* Pref, int ny, double P_atm, float* PrelF, float* dPrefF, cudaStream_t s) {
  pref_tables_kernel<<<(ny + 127) / 128, 128, 0, s>>>(Pref, ny, P_atm, PrelF, dPrefF);
  return cudaGetLastError();
}

cudaError_t launch_encode_saturation_ref(const double* S, long long n, const double* S_ref, float* out,
                                         cudaStream_t s) {
  encode_s_kernel<<<grid_for(n, 256), 256, 0, s>>>(S, S_ref, n, out);
  return cudaGetLastError();
}

cudaError_t launch_row_tables(const double* Pref, int ny, const PhysF& f, float4* rowF, cudaStream_t s) {
  row_tables_kernel<<<(ny + 127) / 128, 128, 0, s>>>(Pref, ny, f, rowF);
  return cudaGetLastError();
}

cudaError_t launch_narrow(const double* a, long long n, float* out, cudaStream_t s) {
  narrow_kernel<<<grid_for(n, 256), 256, 0, s>>>(a, n, out);
  return cudaGetLastError();
}

}  // namespace capaz
