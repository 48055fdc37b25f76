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

}  // namespace atlasgpu
