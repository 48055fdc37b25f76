// common.cuh -- shared constants, error plumbing and warp helpers for the
// sm_100a kernels of the ATLAS12 / SYNTHE hot path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/atlasgpu.h"

namespace atlasgpu {

// mod_constants (atlas12_modules.f90:315-355) and mod_parameters (:175)
constexpr double kPi = 3.141592653589793;
constexpr double kSqrtPi = 1.7724538509055159;
constexpr double kInvSqrtPi = 0.5641895835477563;
constexpr double kClightNms = 2.99792458e17;
constexpr double kHplanck = 6.62607015e-27;
constexpr double kClight = 2.99792458e10;
constexpr double kLineCutoff = 1.0e-3;
constexpr double kEulerM1 = 0.922784335098467;  // 1 - gamma_Euler + ln 2 (:2373)
constexpr double kBnuPrefac = 2.0 * kHplanck / (kClight * kClight) * 1.0e45;

constexpr int kNx = ATLASGPU_NXTAU;  // JOSH's 51-point tau grid
constexpr int kKwMax = 100;          // depth capacity (SYNTHE kw = 99, ATLAS kw = 80)
constexpr int kLd = 52;              // leading dimension of the 51x51 SMEM matrix

// JOSH operator set in device memory (atlas12_modules.f90:18409-18451, 18792-18860)
struct JoshOps {
  double xtau[kNx];
  double ch[kNx];
  double ck[kNx];
  double coefj[kNx * kNx];  // column-major
  double coefh[kNx * kNx];
};

// gfortran's REAL(8)**INTEGER (libgcc binary exponentiation), host and device
// one Stehle Stark-profile series on the device (n_dens 0: not loaded), as
// INIT_STARK_TABLES reads it (atlas12_modules.f90:17682-17746); SYNTHE's
// hydrogen lines and ATLAS's STARK_MMM read it
struct StehleDev {
  int n_lower, n_upper_min, n_upper_max, n_dens;
  double density_grid[20], temp_grid[10], log_dalpha_grid[60];
  const int32_t* max_dens_idx;
  const double* k_alpha;
  const double* profiles;  // [n_trans][n_dens][10][60]
};

__host__ __device__ inline double powi(double x, int m) {
  unsigned n = m < 0 ? (unsigned)(-m) : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// EXPI(1, x) (atlas12_modules.f90:21103-21225): the exponential integral E1
// by the rational approximations of Cody & Thacher (1968), 0 for x <= 0
__device__ __forceinline__ double expi1(double x) {
  const double ex = exp(-x);
  if (x > 4.0) {
    return (ex + ex * (-0.999999999998447 +
                       (-26.6271060431811 +
                        (-241.055827097015 +
                         (-895.927957772937 + (-1298.85688746484 + (-545.374158883133 + -5.66575206533869 / x) / x) / x) /
                             x) /
                            x) /
                           x) /
                     (x + 28.6271060422192 +
                      (292.310039388533 +
                       (1332.78537748257 + (2777.61949509163 + (2404.01713225909 + 631.657483280800 / x) / x) / x) / x) /
                          x)) /
           x;
  } else if (x > 1.0) {
    return ex *
           (0.430967839469389 +
            (6.90522522784444 +
             (23.0192559391333 + (24.3784088791317 + (9.04161556946329 + (0.999979577051595 + 4.65627107975096e-7 * x) * x) * x) * x) *
                 x) *
                x) /
           (0.103400130404874 +
            (3.31909213593302 + (20.4494785013794 + (41.2807841891424 + (32.4264210695138 + (10.0411643829054 + x) * x) * x) * x) * x) *
                x);
  } else if (x > 0.0) {
    return (-44178.5471728217 +
            (57721.7247139444 + (9938.31388962037 + (1842.11088668000 + (101.093806161906 + 5.03416184097568 * x) * x) * x) * x) * x) /
               (76537.3323337614 + (32597.1881290275 + (6106.10794245759 + (635.419418378382 + (37.2298352833327 + x) * x) * x) * x) * x) -
           log(x);
  }
  return 0.0;
}

// EXPI(3, x): E3 from E1 by the recurrence E(n+1) = (e^-x - x E(n)) / n, as
// the reference climbs from E1 (:21103-21225)
__device__ __forceinline__ double expi3(double x) {
  const double ex = exp(-x);
  double r = expi1(x);
  r = (ex - x * r) / 1.0;
  r = (ex - x * r) / 2.0;
  return r;
}

}  // namespace atlasgpu
