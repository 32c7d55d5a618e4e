// Heterogeneous media inputs: the reference's permeability file and an
// on-device seeded Gaussian random field for ln K and porosity.
//
//   capaz_read_permeability_file  load_permeability with LOAD_K_FROM_FILE
//                                 (main.cpp:918-1032): header "Nx Ny" (nz == 1)
//                                 or "Nx Ny Nz", then Ny lines of Nx values v,
//                                 K = 1e-10 exp(v) (upscale_l = 1), the same on
//                                 every z layer;
//   capaz_generate_media          no counterpart in the reference (its field
//                                 generator is a separate Delphi program): a
//                                 Gaussian field with covariance exp(-r/ell)
//                                 by the randomisation (spectral) method.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <random>
#include <string>
#include <vector>

#include "capaz_ctx.h"
#include "capaz_internal.h"

namespace {

int media_fail(capaz_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  else capaz::set_create_error(msg.c_str());
  return code;
}

// G(x) = sqrt(2/N) sum_n cos(k_n . x + phi_n): mean 0, variance 1, and for
// k_n drawn from the field's spectral density, covariance -> exp(-|r|/ell).
// Writes ln K = lnK_mean + sigma G and porosity = clip(phi0 + dphi G, lo, hi).
__global__ void media_kernel(int nx, int ny, int nz, const double4* __restrict__ modes, int nmodes, double lnk_mean,
                             double sigma, double phi0, double dphi, double lo, double hi, double* __restrict__ K,
                             double* __restrict__ m) {
  const long long n = (long long)nx * ny * nz;
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= n) return;
  const double x = (double)(l % nx), y = (double)((l / nx) % ny), z = (double)(l / ((long long)nx * ny));
  double g = 0.;
  for (int q = 0; q < nmodes; q++) {
    const double4 md = modes[q];  // (kx, ky, kz, phase)
    g += cos(fma(md.x, x, fma(md.y, y, fma(md.z, z, md.w))));
  }
  g *= sqrt(2. / (double)nmodes);
  K[l] = exp(lnk_mean + sigma * g);
  m[l] = fmin(hi, fmax(lo, phi0 + dphi * g));
}

}  // namespace

extern "C" {

int capaz_read_permeability_file(const char* path, int nx, int ny, int nz, double* K) {
  if (!path || !K || nx < 1 || ny < 1 || nz < 1)
    return media_fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, "capaz_read_permeability_file: bad arguments");
  FILE* f = fopen(path, "rt");
  if (!f) return media_fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  int fx = 0, fy = 0, fz = 1;
  const int got = nz < 2 ? fscanf(f, "%d %d", &fx, &fy) : fscanf(f, "%d %d %d", &fx, &fy, &fz);
  if (got != (nz < 2 ? 2 : 3) || fx != nx || fy != ny || fz != nz) {
    fclose(f);
    char buf[200];
    snprintf(buf, sizeof buf, "%s: header %dx%dx%d does not match the grid %dx%dx%d", path, fx, fy, fz, nx, ny, nz);
    return media_fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, buf);
  }
  // Values are separated by blanks; rows are j = 0..Ny-1, columns i.
  const long long plane = (long long)nx * ny;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      double v;
      if (fscanf(f, "%lf", &v) != 1) {
        fclose(f);
        char buf[160];
        snprintf(buf, sizeof buf, "%s: value (i=%d, j=%d) missing or not a number", path, i, j);
        return media_fail(nullptr, CAPAZ_ERR_INVALID_ARGUMENT, buf);
      }
      const double k = 1e-10 * exp(v);
      for (int kz = 0; kz < nz; kz++) K[i + (long long)j * nx + kz * plane] = k;
    }
  fclose(f);
  return CAPAZ_OK;
}

int capaz_load_permeability(capaz_ctx* ctx, const char* path) {
  if (!ctx || !path) return CAPAZ_ERR_INVALID_ARGUMENT;
  if (!(ctx->p.flags & CAPAZ_FLAG_PERCELL_K))
    return media_fail(ctx, CAPAZ_ERR_UNSUPPORTED, "capaz_load_permeability: needs CAPAZ_FLAG_PERCELL_K");
  std::vector<double> K((size_t)ctx->n);
  int st = capaz_read_permeability_file(path, ctx->p.nx, ctx->p.ny, ctx->p.nz, K.data());
  if (st) return media_fail(ctx, st, capaz_last_error(nullptr));
  return capaz_set_field(ctx, CAPAZ_FIELD_K, K.data(), nullptr);
}

int capaz_generate_media(capaz_ctx* ctx, unsigned long long seed, double sigma, double ell, double K_mean,
                         double phi0, double dphi, int nmodes) {
  if (!ctx || !(ell > 0.) || !(K_mean > 0.) || nmodes < 1 || nmodes > (1 << 20))
    return media_fail(ctx, CAPAZ_ERR_INVALID_ARGUMENT, "capaz_generate_media: bad arguments");
  if (!(ctx->p.flags & CAPAZ_FLAG_PERCELL_K))
    return media_fail(ctx, CAPAZ_ERR_UNSUPPORTED, "capaz_generate_media: needs CAPAZ_FLAG_PERCELL_K");
  const capaz_params& p = ctx->p;
  const bool planar = p.nz < 2;
  // Spectral density of exp(-|r|/ell) in d dimensions: a d-variate Cauchy
  // law, sampled as g / (ell |w|) with g ~ N(0, I_d), w ~ N(0, 1).
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> N01(0., 1.);
  std::uniform_real_distribution<double> U(0., 2. * M_PI);
  std::vector<double4> modes((size_t)nmodes);
  for (auto& md : modes) {
    const double gx = N01(rng), gy = N01(rng), gz = planar ? 0. : N01(rng);
    double w = fabs(N01(rng));
    if (w < 1e-300) w = 1e-300;
    md = make_double4(gx / (ell * w), gy / (ell * w), gz / (ell * w), U(rng));
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  double *dK = nullptr, *dm = nullptr;
  double4* dmodes = nullptr;
  const size_t fb = sizeof(double) * (size_t)ctx->n;
  if (e == cudaSuccess) e = cudaMalloc(&dK, fb);
  if (e == cudaSuccess) e = cudaMalloc(&dm, fb);
  if (e == cudaSuccess) e = cudaMalloc(&dmodes, sizeof(double4) * modes.size());
  if (e == cudaSuccess) e = cudaMemcpy(dmodes, modes.data(), sizeof(double4) * modes.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int bs = 256;
    media_kernel<<<(unsigned)((ctx->n + bs - 1) / bs), bs>>>(p.nx, p.ny, p.nz, dmodes, nmodes, log(K_mean), sigma,
                                                            phi0, dphi, 0.1, 0.4, dK, dm);
    e = cudaGetLastError();
    ctx->launches++;
  }
  int st = e == cudaSuccess ? CAPAZ_OK : media_fail(ctx, CAPAZ_ERR_CUDA, cudaGetErrorString(e));
  // The field setters validate (porosity and K positive and finite) and
  // encode them for the form.
  if (!st) st = capaz_set_field_device(ctx, CAPAZ_FIELD_K, dK, nullptr);
  if (!st) st = capaz_set_field_device(ctx, CAPAZ_FIELD_M, dm, nullptr);
  if (!st && cudaDeviceSynchronize() != cudaSuccess) st = media_fail(ctx, CAPAZ_ERR_CUDA, "capaz_generate_media");
  cudaFree(dK);
  cudaFree(dm);
  cudaFree(dmodes);
  return st;
}

}  // extern "C"
