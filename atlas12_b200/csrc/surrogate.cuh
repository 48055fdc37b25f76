// surrogate.cuh -- device side of the synthetic physics surrogate that stands
// in for the off-path EOS (populations, electron density) and continuum
// opacity (KAPP).  Same formulas as atlas12_b200/surrogate.py; the per-depth
// factors are folded into coefficient vectors once per iteration so that the
// per-(frequency, depth) continuum is a handful of FMAs.
#pragma once
#include "common.cuh"

namespace atlasgpu {

constexpr double kKbol = 1.380649e-16;
constexpr double kAmu = 1.66053906892e-24;
constexpr double kEvErg = 1.602176634e-12;
constexpr int kNMetal = 18;
constexpr int kNMol = 5;
constexpr int kSurrNspec = 270;  // covers nelion of every surrogate species

// (Z, mass, chi_I [eV], log eps, U_I, U_II) -- surrogate.METALS
static __constant__ double kMetal[kNMetal][6] = {
    {26, 55.845, 7.902, 7.50, 25.0, 40.0}, {22, 47.867, 6.828, 4.95, 30.0, 50.0},
    {24, 51.996, 6.767, 5.64, 10.0, 7.0},  {28, 58.693, 7.640, 6.22, 30.0, 10.0},
    {20, 40.078, 6.113, 6.34, 1.0, 2.0},   {23, 50.942, 6.746, 3.93, 35.0, 30.0},
    {27, 58.933, 7.881, 4.99, 30.0, 25.0}, {25, 54.938, 7.434, 5.43, 6.0, 7.0},
    {21, 44.956, 6.561, 3.15, 10.0, 20.0}, {12, 24.305, 7.646, 7.60, 1.0, 2.0},
    {14, 28.086, 8.152, 7.51, 9.0, 6.0},   {11, 22.990, 5.139, 6.24, 2.0, 1.0},
    {13, 26.982, 5.986, 6.45, 6.0, 1.0},   {6, 12.011, 11.260, 8.43, 9.0, 6.0},
    {8, 15.999, 13.618, 8.69, 9.0, 4.0},   {7, 14.007, 14.534, 7.83, 9.0, 9.0},
    {39, 88.906, 6.217, 2.21, 10.0, 15.0}, {40, 91.224, 6.634, 2.58, 30.0, 40.0}};
// (slot, mass, log abundance, T exponent) -- surrogate.MOLECULES
static __constant__ double kMol[kNMol][4] = {{41, 13.02, -7.0, 8.0},
                                      {42, 26.02, -8.0, 10.0},
                                      {43, 28.01, -4.5, 6.0},
                                      {44, 17.01, -7.5, 9.0},
                                      {45, 63.87, -9.0, 14.0}};


// per-depth continuum coefficients: kabs(w) = hm*abf(w) + ff*(w/1000)^2 +
// sum_n pop[n]*sig_n(w) + 1e-12 ;  sigma(w) = es + ray*5.8e-24*(121.6/max(w,125))^4
struct ContCoef {
  double hm, ff, pop[3], es, ray;
  double mbf[kNMetal];  // neutral-metal density * cross-section / rho
};
constexpr double kMbfSigma = 2.0e-17;  // surrogate.MBF_SIGMA
// Fraction of the metal / molecule populations seen by the ATLAS12 line list
// (surrogate.ATLAS_LINE_POP): the device surrogate serves only the ATLAS12
// model, whose purely radiative structure stays convergent at this strength.
constexpr double kAtlasLinePop = 0.01;

struct EosOut {
  double xne, rho, nh, xh;
};

// surrogate.eos + populations for one depth (mh = [M/H]).  xnfdop/dopple: [nspec][kw]
// column (depth j).  Returns EOS fields and fills the continuum coefficients.
__device__ inline EosOut surrogate_depth(double t, double p, double vturb_cms, double mh, int j, int kw,
                                         double* xnfdop, double* dopple, ContCoef* cc) {
  // the T-only factors of every Saha ratio, evaluated once (same operand
  // order as surrogate._saha, so the ratios are the same numbers)
  const double st = 2.4147e15 * pow(t, 1.5);
  const double kt = kKbol * t;
  const double bh = (2.0 * 1.0 / 2.0), eh = exp(-13.598 * kEvErg / kt);
  double bm[kNMetal], em[kNMetal], am[kNMetal];
#pragma unroll
  for (int m = 0; m < kNMetal; ++m) {
    bm[m] = 2.0 * kMetal[m][5] / kMetal[m][4];
    em[m] = exp(-kMetal[m][2] * kEvErg / kt);
    am[m] = exp10(kMetal[m][3] - 12.0 + mh);  // [M/H] scales every metal
  }
  const double ntot = p / kt;
  double ne = fmax(ntot * 1e-4, 1.0);
  double nh = 0, xh = 0;
  for (int it = 0; it < 30; ++it) {
    nh = ntot / (1.1 + ne / ntot);
    const double sn = st / fmax(ne, 1.0);
    const double rh = sn * bh * eh;
    xh = rh / (1.0 + rh);
    double sm = 0.0;
#pragma unroll
    for (int m = 0; m < kNMetal; ++m) {
      const double rm = sn * bm[m] * em[m];
      sm += am[m] * (rm / (1.0 + rm));
    }
    const double ne_new = nh * xh + nh * sm + 1.0;
    ne = sqrt(ne * ne_new);
  }
  nh = ntot / (1.1 + ne / ntot);
  const double rho = nh * 1.4 * kAmu;
  const double sn = st / fmax(ne, 1.0);
  auto dop = [&](double m) { return sqrt(2.0 * kKbol * t / (m * kAmu) + vturb_cms * vturb_cms) / kClight; };
  auto put = [&](int nel, double xnfp, double d) {
    xnfdop[(size_t)(nel - 1) * kw + j] = xnfp / d / rho;
    dopple[(size_t)(nel - 1) * kw + j] = d;
  };
  const double dh = dop(1.008);
  put(1, nh * (1 - xh) / 2.0, dh);
  put(2, nh * xh, dh);
#pragma unroll
  for (int m = 0; m < kNMetal; ++m) {
    const double r = sn * bm[m] * em[m];
    const double n = nh * am[m];
    const int z = (int)kMetal[m][0];
    const double d = dop(kMetal[m][1]);
    put((z - 1) * 6 + 1, n / (1.0 + r) / kMetal[m][4] * kAtlasLinePop, d);
    put((z - 1) * 6 + 2, n * r / (1.0 + r) / kMetal[m][5] * kAtlasLinePop, d);
    cc->mbf[m] = nh * am[m] / (1.0 + r) * kMbfSigma / rho;
  }
  for (int m = 0; m < kNMol; ++m) {
    const int slot = (int)kMol[m][0];
    const double v = nh * exp10(kMol[m][2]) * fmin(pow(5000.0 / t, kMol[m][3]), 1e6) / 1000.0 * kAtlasLinePop;
    put((slot - 1) * 6 + 1, v, dop(kMol[m][1]));
  }
  // continuum coefficients (surrogate.continuum_opacity)
  const double nh1 = nh * (1.0 - xh);
  const double theta = 5040.0 / t;
  const double pe = ne * kKbol * t;
  cc->hm = 4.158e-10 * pe * pow(theta, 2.5) * exp10(0.754 * theta) * nh1 / rho;
  cc->ff = 1.0e-26 * pe * nh1 * (0.5 + 1.5 * theta) / rho;
  for (int n = 1; n <= 3; ++n)
    cc->pop[n - 1] = nh1 * 2.0 * n * n * exp(-13.598 * (1.0 - 1.0 / (n * n)) * kEvErg / (kKbol * t)) / 2.0 / rho;
  cc->es = 6.6524587051e-25 * ne / rho;
  cc->ray = nh1 / rho;
  EosOut o{ne, rho, nh, xh};
  return o;
}

static __device__ __noinline__ void surrogate_kapp(const ContCoef& c, double w, double& kabs, double& sigma) {
  double x = w / 1642.0;
  x = x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x);
  const double abf = 4.0e-17 * 6.0 * (x * sqrt(x)) * ((1.0 - x) * sqrt(1.0 - x)) * 4.0;
  double k = c.hm * abf + c.ff * (w / 1000.0) * (w / 1000.0);
  const double edges[3] = {91.175, 364.70, 820.6};
#pragma unroll
  for (int n = 1; n <= 3; ++n) {
    if (w <= edges[n - 1]) {
      const double q = w / edges[n - 1];
      k += c.pop[n - 1] * (7.9e-18 / (double)(n * n * n * n * n) * (q * q * q) * (double)(n * n * n));
    }
  }
  for (int m = 0; m < kNMetal; ++m) {
    const double edge = 1239.84198 / kMetal[m][2];
    if (w <= edge) {
      const double q = w / edge;
      k += c.mbf[m] * (q * q * q);
    }
  }
  kabs = k + 1e-12;
  const double r = 121.6 / fmax(w, 125.0);
  sigma = c.es + c.ray * 5.8e-24 * (r * r) * (r * r);
}

}  // namespace atlasgpu
