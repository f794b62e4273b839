// Device math shared by the matvec kernels: the equispaced Lagrange basis
// and the plane-wave phases exp(i a) of both precisions.
#pragma once

#include <cuda_runtime.h>

#include "fp64_math.hpp"

namespace dfb {

// ----------------------------------------------------------------- basics --
// equispaced Lagrange basis of order L on [-rad, rad] at x
// (thetis_polynomials.hpp:81-94): b[l] = prod_{j != l} (x/rad - p_j)/(p_l - p_j),
// p_j = -1 + 2 j/(L-1)
template <int L, typename T>
__device__ __forceinline__ void lagrange_all(T x, T rad, T* b) {
  const T nx = x / rad;
#pragma unroll
  for (int l = 0; l < L; l++) {
    T r = 1;
    const T pl = T(-1) + T(2) * (T(l) / T(L - 1));
#pragma unroll
    for (int j = 0; j < L; j++) {
      if (j == l) continue;
      const T pj = T(-1) + T(2) * (T(j) / T(L - 1));
      r *= (nx - pj) / (pl - pj);
    }
    b[l] = r;
  }
}

// FP64 sin and cos of x (Cody-Waite reduction by pi/2, Taylor series; the
// same function the host plan uses, fp64_math.hpp)
__device__ __forceinline__ void sincos_cw(double x, double& s, double& c) { sincos_fp64(x, s, c); }

// exp(i a) with a in FP64
template <typename C>
__device__ __forceinline__ C expi64(double a) {
  double s, c;
  sincos_cw(a, s, c);
  C r;
  r.x = c;
  r.y = s;
  return r;
}

// exp(i a) for the FP32 path: a = n pi + x reduced in FP64 (n from the low
// mantissa bits of a / pi + 1.5 * 2^52, exact for |a / pi| < 2^51, any sign),
// sin/cos of x in FP32 by Taylor polynomials of degree 13/12 on
// [-pi/2, pi/2] (truncation < 7e-10), (-1)^n applied to both.
__device__ __forceinline__ float2 expi_reduced(double a) {
  const double t = fma(a, 0.31830988618379067154, 6755399441055744.0);
  const double n = t - 6755399441055744.0;
  const int odd = __double2loint(t) & 1;
  const float x = (float)fma(-n, 3.14159265358979323846, a);
  const float xx = x * x;
  float ps = fmaf(xx, 1.6059043836821613e-10f, -2.5052108385441720e-08f);
  ps = fmaf(xx, ps, 2.7557319223985893e-06f);
  ps = fmaf(xx, ps, -1.9841269841269841e-04f);
  ps = fmaf(xx, ps, 8.3333333333333333e-03f);
  ps = fmaf(xx, ps, -1.6666666666666667e-01f);
  ps = fmaf(xx, ps, 1.0f);
  float pc = fmaf(xx, 2.0876756987868099e-09f, -2.7557319223985891e-07f);
  pc = fmaf(xx, pc, 2.4801587301587302e-05f);
  pc = fmaf(xx, pc, -1.3888888888888889e-03f);
  pc = fmaf(xx, pc, 4.1666666666666667e-02f);
  pc = fmaf(xx, pc, -0.5f);
  pc = fmaf(xx, pc, 1.0f);
  const float sg = odd ? -1.0f : 1.0f;
  return make_float2(sg * pc, sg * x * ps);
}

// Plane-wave phase exp(i a) at the precision of the complex type.
template <typename C>
__device__ __forceinline__ C expi(double a);
template <>
__device__ __forceinline__ double2 expi<double2>(double a) {
  return expi64<double2>(a);
}
template <>
__device__ __forceinline__ float2 expi<float2>(double a) {
  return expi_reduced(a);
}

}  // namespace dfb
