// voigt.cuh -- the two Voigt functions of the hot path, device side.
//
//  * voigt_weideman: SYNTHE's voigt_profile (synthe_module.f90:463-537),
//    Weideman (1994) N=32 rational approximation for |v|+a <= 15 and the
//    Humlicek (1982) R_{1,2} asymptote beyond, in FP64 exactly as written.
//    The coefficients were generated from Weideman's published construction
//    (FFT of exp(-t^2)(L^2+t^2) on t = L tan(theta/2), L = sqrt(N/sqrt 2));
//    they coincide bit-for-bit with the reference table (checked by the
//    test suite).  FP64 is required: the same recurrence in FP32 loses up to
//    1e-2 relative accuracy to cancellation for a < 1e-3.
//  * voigt_kurucz: ATLAS12's VOIGT (atlas12_modules.f90:21033-21097), three
//    regimes on the H0/H1/H2 tables of TABVOIGT (200 steps per Doppler width).
#pragma once
#include "common.cuh"

namespace atlasgpu {

static __constant__ double kWeiA[32] = {
    -1.30317978630500875e-12, 3.74088129316536249e-12, 8.03036789996388945e-12,
    -2.15436320778387687e-11, -5.54423594816646238e-11, 1.16582510935237737e-10,
    4.15374309183345315e-10, -5.23102048119632885e-10, -3.20801509172336887e-09,
    8.12488945684665156e-10, 2.37975567798974168e-08, 2.29304390650999664e-08,
    -1.48130789151209774e-07, -4.18407637021697758e-07, 4.25583313757500854e-07,
    4.40153173157854990e-06, 6.82103194400198485e-06, -2.14096192017107501e-05,
    -1.30754492546153456e-04, -2.45329802700214317e-04, 3.92591360700703107e-04,
    4.51954110534921738e-03, 1.90061557848454077e-02, 5.73044035298372195e-02,
    1.40607162268937685e-01, 2.95444510715087316e-01, 5.46013972063934094e-01,
    9.01925489364799882e-01, 1.34554416923454490e+00, 1.82566962963248147e+00,
    2.26353729990026764e+00, 2.57225340812456960e+00};
constexpr double kWeiL = 4.75682846001088411;

__device__ __forceinline__ double voigt_weideman(double v, double a) {
  const double x = fabs(v), y = a;
  if (x + y > 15.0) {
    const double dr = x * x - y * y - 0.5;
    const double di = 2.0 * x * y;
    const double d2 = dr * dr + di * di;
    return (-y * dr + x * di) / (kSqrtPi * d2);
  }
  const double dr = kWeiL + y, di = -x;
  const double nr = kWeiL - y, ni = x;
  const double d2 = dr * dr + di * di;
  const double rd2 = 1.0 / d2;
  const double zr = (nr * dr + ni * di) * rd2;
  const double zi = (ni * dr - nr * di) * rd2;
  double pr = kWeiA[0], pim = 0.0;
#pragma unroll
  for (int k = 1; k < 32; ++k) {
    const double tmp = pr * zr - pim * zi + kWeiA[k];
    pim = pr * zi + pim * zr;
    pr = tmp;
  }
  const double sq_r = dr * dr - di * di;
  const double sq_i = 2.0 * dr * di;
  const double sq_d = sq_r * sq_r + sq_i * sq_i;
  const double term1 = 2.0 * (pr * sq_r + pim * sq_i) / sq_d;
  const double term2 = dr * rd2 * kInvSqrtPi;
  return term1 + term2;
}

// VOIGT(V, A) with 1-based table index IV = INT(V*200 + 1.5)
__device__ __forceinline__ double voigt_kurucz(double v, double a, const double* __restrict__ h0,
                                               const double* __restrict__ h1,
                                               const double* __restrict__ h2) {
  const int iv = (int)(v * 200.0 + 1.5);
  if (a < 0.2) {
    if (v <= 10.0) return (h2[iv - 1] * a + h1[iv - 1]) * a + h0[iv - 1];
    return 0.5642 * a / (v * v);
  } else if (a <= 1.4 && a + v <= 3.2) {
    const double vv = v * v;
    const double H0 = h0[iv - 1], H1 = h1[iv - 1], H2 = h2[iv - 1];
    const double hh1 = H1 + H0 * 1.12838;
    const double hh2 = H2 + hh1 * 1.12838 - H0;
    const double hh3 = (1.0 - H2) * 0.37613 - hh1 * 0.66667 * vv + hh2 * 1.12838;
    const double hh4 = (3.0 * hh3 - hh1) * 0.37613 + H0 * 0.66667 * vv * vv;
    return ((((hh4 * a + hh3) * a + hh2) * a + hh1) * a + H0) *
           (((-.122727278 * a + .532770573) * a - .96284325) * a + .979895032);
  } else {
    const double aa = a * a, vv = v * v;
    const double u = (aa + vv) * 1.4142;
    double r = a * 0.79788 / u;
    if (a <= 100.0) {
      const double aau = aa / u, vvu = vv / u, uu = u * u;
      r = ((((aau - 10.0 * vvu) * aau * 3.0 + 15.0 * vvu * vvu) + 3.0 * vv - aa) / uu + 1.0) * r;
    }
    return r;
  }
}

}  // namespace atlasgpu
