// Deterministic block reduction of the per-CTA diagnostics partials
// (DIAG_STRIDE doubles each: mass_w, mass_n, mass_g, max residual,
// non-finite cells) into out[DIAG_STRIDE].  Every thread of the calling block
// must call it (it synchronises the block); the block has at most
// 32 * MAX_WARPS threads, the rows of `red`.  Each thread sums a contiguous
// range of partials, then an ordered tree over the lanes of each warp and a
// sequential sum over the warps: the order depends only on the block size and
// the partials' count, never on timing.
#pragma once

#include "capaz_internal.h"

namespace capaz {

template <int MAX_WARPS>
__device__ __forceinline__ void diag_reduce_block(const double* __restrict__ partials, int nparts,
                                                  double* __restrict__ out, double (*red)[DIAG_STRIDE]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double s[DIAG_STRIDE] = {0, 0, 0, 0, 0};
  const int per = (nparts + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(nparts, b0 + per);
  for (int b = b0; b < b1; b++) {
    const double* p = partials + (size_t)DIAG_STRIDE * b;
    s[0] += p[0];
    s[1] += p[1];
    s[2] += p[2];
    s[3] = fmax(s[3], p[3]);
    s[4] += p[4];
  }
  for (int o = 1; o < 32; o <<= 1) {
    const double t0 = __shfl_down_sync(0xffffffffu, s[0], o), t1 = __shfl_down_sync(0xffffffffu, s[1], o);
    const double t2 = __shfl_down_sync(0xffffffffu, s[2], o), t3 = __shfl_down_sync(0xffffffffu, s[3], o);
    const double t4 = __shfl_down_sync(0xffffffffu, s[4], o);
    if ((lane & (2 * o - 1)) == 0) {
      s[0] += t0;
      s[1] += t1;
      s[2] += t2;
      s[3] = fmax(s[3], t3);
      s[4] += t4;
    }
  }
  if (lane == 0 && wid < MAX_WARPS)
    for (int q = 0; q < DIAG_STRIDE; q++) red[wid][q] = s[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[DIAG_STRIDE] = {0, 0, 0, 0, 0};
    const int nw = min((int)(blockDim.x / 32), MAX_WARPS);
    for (int w = 0; w < nw; w++) {
      r[0] += red[w][0];
      r[1] += red[w][1];
      r[2] += red[w][2];
      r[3] = fmax(r[3], red[w][3]);
      r[4] += red[w][4];
    }
    for (int q = 0; q < DIAG_STRIDE; q++) out[q] = r[q];
  }
}

}  // namespace capaz
