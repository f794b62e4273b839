// FP64 sine and cosine shared by the host plan and the device kernels, so
// that tables built on either side (transfer spectra, plane-wave signatures)
// are bit-identical: every step is an IEEE operation (fma, rint, +, *) with
// no contraction left to the compiler.
//
// Method: Cody-Waite reduction by pi/2 (pi/2 split into its double and the
// remainder), then the Taylor series of sin to degree 15 and of cos to degree
// 16 on [-pi/4, pi/4] (truncation below 7e-17 relative), quadrant by n mod 4.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define DFB_HD __host__ __device__
#else
#define DFB_HD
#endif

namespace dfb {

DFB_HD inline void sincos_fp64(double x, double& s, double& c) {
  const double n = rint(x * 0.6366197723675814);
  double r = fma(-n, 1.5707963267948966, x);
  r = fma(-n, 6.123233995736766e-17, r);
  const double r2 = r * r;
  double ps = fma(r2, -7.647163731819816e-13, 1.6059043836821613e-10);
  ps = fma(r2, ps, -2.505210838544172e-08);
  ps = fma(r2, ps, 2.7557319223985893e-06);
  ps = fma(r2, ps, -1.984126984126984e-04);
  ps = fma(r2, ps, 8.333333333333333e-03);
  ps = fma(r2, ps, -1.6666666666666666e-01);
  const double r3 = r * r2;
  const double sr = fma(r3, ps, r);
  double pc = fma(r2, 4.779477332387385e-14, -1.1470745597729725e-11);
  pc = fma(r2, pc, 2.08767569878681e-09);
  pc = fma(r2, pc, -2.755731922398589e-07);
  pc = fma(r2, pc, 2.48015873015873e-05);
  pc = fma(r2, pc, -1.388888888888889e-03);
  pc = fma(r2, pc, 4.1666666666666664e-02);
  pc = fma(r2, pc, -0.5);
  const double cr = fma(r2, pc, 1.0);
  const int q = (int)((long long)n & 3);
  const double ss = (q & 1) ? cr : sr, cc = (q & 1) ? sr : cr;
  s = (q & 2) ? -ss : ss;
  c = ((q + 1) & 2) ? -cc : cc;
}

}  // namespace dfb
