// capaz_mass_noalloc: the phase-mass reduction of the step diagnostics over a
// two-phase state in caller-owned device memory, with every byte of scratch
// in a fixed file-scope device array.  No call allocates device or host
// memory (no cudaMalloc/cudaFree, no library routine that allocates), so it
// can run between a caller's own steps while the caller's pool holds the rest
// of the device memory, and never triggers the implicit device-wide
// synchronisation of cudaFree.
//
// The per-cell quantity is the one the step kernels accumulate under
// CAPAZ_FLAG_DIAGNOSTICS (rho_p(P) S_p m vol over interior cells, plus the
// count of cells whose P or S is not finite); only the summation order
// differs (one warp per (j, k) row here, per tile there).
#include <math.h>
#include <stdio.h>

#include <mutex>

#include "capaz_internal.h"

namespace {

constexpr int kRowsPerBlock = 8;  // one warp per (j, k) row of interior cells
constexpr int kMaxPartials = CAPAZ_NOALLOC_MAX_ROWS / kRowsPerBlock;
constexpr int kStride = 4;  // mass_w, mass_n, nonfinite, unused
constexpr int kMaxDevices = 64;

// 16384 partials x 4 doubles = 512 KiB per device.  Every slot a call reads
// is written earlier in the same call, so nothing here has to start at zero.
__device__ __align__(256) double g_mass_scratch[kMaxPartials * kStride];

struct MassConst {
  int nx, ny, nz, rows, planar;
  double S_wr, P_d, e_pk, ro0_w, ro0_n, beta_w, beta_n, P_atm, vol;
};

__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(256) mass_rows_kernel(const MassConst c, const double* __restrict__ Pw,
                                                        const double* __restrict__ Sn, const double* __restrict__ m,
                                                        double* __restrict__ partials) {
  __shared__ double red[kRowsPerBlock][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = blockIdx.x * kRowsPerBlock + w;
  double aw = 0., an = 0., nf = 0.;
  if (r < c.rows) {
    const int j = 1 + r % (c.ny - 2);
    const int k = c.planar ? 0 : 1 + r / (c.ny - 2);
    const long long row = ((long long)k * c.ny + j) * c.nx;
    for (int i = 1 + lane; i <= c.nx - 2; i += 32) {
      const long long l = row + i;
      const double P = Pw[l], S = Sn[l], mc = m[l];
      const double S_e = (1 - S - c.S_wr) / (1 - c.S_wr);
      const double P_k = (c.P_d != 0.) ? c.P_d * pow(S_e, c.e_pk) : 0.;
      const double rw = c.ro0_w * (1. + c.beta_w * (P - c.P_atm));
      const double rn = c.ro0_n * (1. + c.beta_n * (P + P_k - c.P_atm));
      aw += mc * rw * (1. - S) * c.vol;
      an += mc * rn * S * c.vol;
      if (!(isfinite(P) && isfinite(S))) nf += 1.;
    }
  }
  aw = wsum(aw);
  an = wsum(an);
  nf = wsum(nf);
  if (lane == 0) {
    red[w][0] = aw;
    red[w][1] = an;
    red[w][2] = nf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0., t1 = 0., t2 = 0.;
    for (int q = 0; q < kRowsPerBlock; q++) {
      t0 += red[q][0];
      t1 += red[q][1];
      t2 += red[q][2];
    }
    double* o = partials + (size_t)kStride * blockIdx.x;
    o[0] = t0;
    o[1] = t1;
    o[2] = t2;
  }
}

// Block-ordered sum of the partials into the capaz_diag layout.
__global__ void __launch_bounds__(128) mass_finalize_kernel(const double* __restrict__ partials, int nblocks,
                                                            double* __restrict__ out) {
  __shared__ double red[4][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int per = (nblocks + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(nblocks, b0 + per);
  double s0 = 0., s1 = 0., s2 = 0.;
  for (int b = b0; b < b1; b++) {
    const double* q = partials + (size_t)kStride * b;
    s0 += q[0];
    s1 += q[1];
    s2 += q[2];
  }
  s0 = wsum(s0);
  s1 = wsum(s1);
  s2 = wsum(s2);
  if (lane == 0) {
    red[w][0] = s0;
    red[w][1] = s1;
    red[w][2] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0., t1 = 0., t2 = 0.;
    for (int q = 0; q < 4; q++) {
      t0 += red[q][0];
      t1 += red[q][1];
      t2 += red[q][2];
    }
    out[0] = t0;
    out[1] = t1;
    out[2] = 0.;
    out[3] = 0.;
    out[4] = t2;
  }
}

std::mutex g_setup_mu;
double* g_scratch_ptr[kMaxDevices] = {};

int fail(int code, const char* msg) {
  capaz::set_create_error(msg);
  return code;
}

// Device pointer on the current device (or managed memory) — anything else
// would be dereferenced by the kernel as a wild address.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int capaz_mass_noalloc(const capaz_params* p, const double* P_w, const double* S_n, const double* m,
                                  double* out, void* stream) {
  if (!p || !P_w || !S_n || !m || !out) return fail(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_mass_noalloc: null argument");
  if (p->phases != 2) return fail(CAPAZ_ERR_UNSUPPORTED, "capaz_mass_noalloc: two-phase states only");
  if (p->model != CAPAZ_MODEL_DEFAULT && p->model != CAPAZ_MODEL_BUCKLEY_LEVERETT)
    return fail(CAPAZ_ERR_UNSUPPORTED,
                "capaz_mass_noalloc: the isothermal two-phase and Buckley-Leverett models only");
  if (p->nx < 3 || p->ny < 3 || p->nz < 1 || p->nz == 2)
    return fail(CAPAZ_ERR_UNSUPPORTED_GRID, "capaz_mass_noalloc: grid needs nx,ny>=3 and nz==1 or >=3");
  const long long rows = (long long)(p->ny - 2) * (p->nz == 1 ? 1 : p->nz - 2);
  if (rows > CAPAZ_NOALLOC_MAX_ROWS) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "capaz_mass_noalloc: %lld interior rows (ny-2)*(nz-2) exceed the fixed scratch of %d rows", rows,
             (int)CAPAZ_NOALLOC_MAX_ROWS);
    return fail(CAPAZ_ERR_UNSUPPORTED_GRID, buf);
  }
  if (!(p->lambda != 0.) || !(1. - p->S_wr != 0.))
    return fail(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_mass_noalloc: lambda and 1-S_wr must be nonzero");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(CAPAZ_ERR_NO_DEVICE, "capaz_mass_noalloc: no current CUDA device");
  if (dev < 0 || dev >= kMaxDevices) return fail(CAPAZ_ERR_UNSUPPORTED, "capaz_mass_noalloc: device index too large");
  if (!on_device(P_w, dev) || !on_device(S_n, dev) || !on_device(m, dev) || !on_device(out, dev))
    return fail(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_mass_noalloc: pointers must be device memory of the current device");

  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &capture);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CAPAZ_ERR_INVALID_ARGUMENT, "capaz_mass_noalloc: stream does not belong to the current device");
  }
  double* scratch;
  {
    // The address of the fixed scratch in the current context's copy of the
    // module.  It is looked up again on every call made outside stream
    // capture (a lookup, no allocation), so a device reset or a caller's own
    // non-primary context gets the address of its own copy; a call on a
    // capturing stream uses the address the device's last uncaptured call
    // found, so the first call on a device must come before any capture.
    std::lock_guard<std::mutex> g(g_setup_mu);
    if (capture == cudaStreamCaptureStatusNone) {
      void* a = nullptr;
      e = cudaGetSymbolAddress(&a, g_mass_scratch);
      if (e != cudaSuccess || !a) {
        cudaGetLastError();
        return fail(CAPAZ_ERR_CUDA, "capaz_mass_noalloc: cudaGetSymbolAddress of the fixed scratch failed");
      }
      g_scratch_ptr[dev] = (double*)a;
    } else if (!g_scratch_ptr[dev]) {
      return fail(CAPAZ_ERR_BAD_STATE,
                  "capaz_mass_noalloc: the first call on a device must not be made on a capturing stream");
    }
    scratch = g_scratch_ptr[dev];
  }

  MassConst c;
  c.nx = p->nx;
  c.ny = p->ny;
  c.nz = p->nz;
  c.rows = (int)rows;
  c.planar = p->nz == 1;
  c.S_wr = p->S_wr;
  c.P_d = p->model == CAPAZ_MODEL_BUCKLEY_LEVERETT ? 0. : p->P_d;  // the B-L task has P_n = P_w
  c.e_pk = -1. / p->lambda;
  c.ro0_w = p->ro0_w;
  c.ro0_n = p->ro0_n;
  c.beta_w = p->beta_w;
  c.beta_n = p->beta_n;
  c.P_atm = p->P_atm;
  c.vol = p->hx * p->hy * p->hz;
  const int nblocks = (int)((rows + kRowsPerBlock - 1) / kRowsPerBlock);
  mass_rows_kernel<<<nblocks, 32 * kRowsPerBlock, 0, s>>>(c, P_w, S_n, m, scratch);
  mass_finalize_kernel<<<1, 128, 0, s>>>(scratch, nblocks, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CAPAZ_ERR_CUDA, cudaGetErrorString(e));
  return CAPAZ_OK;
}
