// FP32 constitutive relations of the three-phase precision form, shared by
// its sweeps (step3_fp32c.cu, step3_fp32c_tma.cu).
#pragma once

#include <math.h>

#include "capaz_internal.h"

namespace capaz {

// Square root for the FP32 relative permeabilities: x * rsqrt(x) (a few
// ulp, no slow path), 0 for x <= 0.
__device__ __forceinline__ float sqrt_fast(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

// Relative permeabilities (three-phase.cpp:146-186) in FP32.  A2: A = 2, so
// the exponents A/(A-1), (A-1)/A and 2(A-1)/A are 2, 1/2 and 1.
template <bool A2>
__device__ __forceinline__ void relperm3f(const Step3FConst& f, float S_w_e, float S_n_e, float& k_w, float& k_n,
                                          float& k_g) {
  const float S_g_e = 1.f - S_w_e - S_n_e;
  if (A2) {
    // Branch-free: every relation is evaluated and then selected, which keeps
    // a warp converged; the same operations as the general form below with
    // the exponents 2, 1/2 and 1 (sqrt_fast is 0 for x <= 0, and a quotient
    // by zero is selected away).
    const float w2 = S_w_e * S_w_e;
    const float tw = 1.f - sqrt_fast(1.f - w2);
    const float kw = sqrt_fast(S_w_e) * tw * tw;
    const float g1 = 1.f - S_g_e;
    const float kg = sqrt_fast(S_g_e) * (1.f - g1 * g1);
    const float knw = sqrt_fast(1.f - S_w_e) * (1.f - w2);
    const float tn = 1.f - sqrt_fast(1.f - S_n_e * S_n_e);
    const float kng = sqrt_fast(S_n_e) * tn * tn;
    const float kn = __fdividef(__fdividef(S_n_e * knw * kng, 1.f - S_w_e), 1.f - S_g_e);
    k_w = S_w_e >= 1e-3f ? kw : 0.f;
    k_g = S_g_e >= 1e-3f ? kg : 0.f;
    k_n = S_n_e >= 1e-3f ? kn : 0.f;
    return;
  }
  auto p1 = [&](float x) { return A2 ? x * x : powf(x, f.e1); };         // x^(A/(A-1))
  auto p2 = [&](float x) { return A2 ? sqrt_fast(x) : powf(x, f.e2); };  // x^((A-1)/A)
  auto p3 = [&](float x) { return A2 ? x : powf(x, f.e3); };             // x^(2(A-1)/A)
  k_w = 0.f;
  if (S_w_e >= 1e-3f) {
    const float t = 1.f - p2(1.f - p1(S_w_e));
    k_w = sqrt_fast(S_w_e) * t * t;
  }
  k_g = 0.f;
  if (S_g_e >= 1e-3f) k_g = sqrt_fast(S_g_e) * p3(1.f - p1(1.f - S_g_e));
  k_n = 0.f;
  if (S_n_e >= 1e-3f) {
    const float k_n_w = sqrt_fast(1.f - S_w_e) * p3(1.f - p1(S_w_e));
    const float t = 1.f - p2(1.f - p1(S_n_e));
    const float k_n_g = sqrt_fast(S_n_e) * t * t;
    k_n = __fdividef(__fdividef(S_n_e * k_n_w * k_n_g, 1.f - S_w_e), 1.f - S_g_e);
  }
}

}  // namespace capaz
