/*
 * oracle.c -- CPU restatement of the ATLAS12 / SYNTHE hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path,
 * never the product.  Every function cites the reference routine it
 * restates (paths inside cconroy20/atlas12).  Statement order and operand
 * order follow the reference so that IEEE results agree to the last few
 * ulps; the file is compiled with -ffp-contract=off.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KW_MAX 128

/* mod_constants (atlas12_modules.f90:315-355) */
static const double PI_ = 3.141592653589793;
static const double SQRTPI = 1.7724538509055159;
static const double INVSQRTPI = 0.5641895835477563;
static const double CLIGHT_NMS = 2.99792458e17;
static const double HPLANCK = 6.62607015e-27;
static const double CLIGHT = 2.99792458e10;
static const double LINE_CUTOFF = 1.0e-3;      /* :175 */
static const double EULER_M1 = 0.922784335098467; /* :2373 */

static double bnu_prefac(void) { return 2.0 * HPLANCK / (CLIGHT * CLIGHT) * 1.0e45; }

/* gfortran lowers REAL(8)**INTEGER to libgcc's binary exponentiation. */
double orc_powi(double x, int m) {
  unsigned n = m < 0 ? (unsigned)(-m) : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

/* ======================================================================
 * Numerics
 * ==================================================================== */

/* PARCOE, atlas12_modules.f90:5358-5434 */
void orc_parcoe(const double *f, const double *x, double *a, double *b,
                double *c, int n) {
  int j;
  double d, wt;
  c[0] = 0.0;
  b[0] = (f[1] - f[0]) / (x[1] - x[0]);
  a[0] = f[0] - x[0] * b[0];
  c[n - 1] = 0.0;
  b[n - 1] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
  a[n - 1] = f[n - 1] - x[n - 1] * b[n - 1];
  if (n == 2) return;
  if (n == 3) {
    a[1] = a[2];
    b[1] = b[2];
    c[1] = c[2];
    return;
  }
  for (j = 1; j <= n - 2; ++j) {
    d = (f[j] - f[j - 1]) / (x[j] - x[j - 1]);
    c[j] = f[j + 1] / ((x[j + 1] - x[j]) * (x[j + 1] - x[j - 1])) -
           f[j] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j])) +
           f[j - 1] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j - 1]));
    b[j] = d - (x[j] + x[j - 1]) * c[j];
    a[j] = f[j - 1] - x[j - 1] * d + x[j] * x[j - 1] * c[j];
  }
  c[1] = 0.0;
  b[1] = (f[2] - f[1]) / (x[2] - x[1]);
  a[1] = f[1] - x[1] * b[1];
  c[2] = 0.0;
  b[2] = (f[3] - f[2]) / (x[3] - x[2]);
  a[2] = f[2] - x[2] * b[2];
  for (j = 1; j <= n - 2; ++j) {
    if (c[j] != 0.0) {
      wt = fabs(c[j + 1]) / (fabs(c[j + 1]) + fabs(c[j]));
      a[j] = a[j + 1] + wt * (a[j] - a[j + 1]);
      b[j] = b[j + 1] + wt * (b[j] - b[j + 1]);
      c[j] = c[j + 1] + wt * (c[j] - c[j + 1]);
    }
  }
  a[n - 2] = a[n - 1];
  b[n - 2] = b[n - 1];
  c[n - 2] = c[n - 1];
}

/* INTEG (IQUAD=0 branch), atlas12_modules.f90:5293-5324 */
void orc_integ(const double *x, const double *f, double *fint, int n,
               double start) {
  double a[KW_MAX], b[KW_MAX], c[KW_MAX];
  orc_parcoe(f, x, a, b, c, n);
  fint[0] = start;
  for (int i = 0; i < n - 1; ++i) {
    double xlo = x[i], xhi = x[i + 1];
    fint[i + 1] = fint[i] + (a[i] + b[i] * 0.5 * (xhi + xlo) +
                             c[i] / 3.0 * ((xhi + xlo) * xhi + xlo * xlo)) *
                                (xhi - xlo);
  }
}

/* DERIV, atlas12_modules.f90:5228-5266 */
void orc_deriv(const double *x, const double *f, double *dfdx, int n) {
  dfdx[0] = (f[1] - f[0]) / (x[1] - x[0]);
  dfdx[n - 1] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
  if (n == 2) return;
  double s = fabs(x[1] - x[0]) / (x[1] - x[0]);
  for (int j = 1; j <= n - 2; ++j) {
    double scale = fmax(fmax(fabs(f[j - 1]), fabs(f[j])), fabs(f[j + 1])) / fabs(x[j]);
    if (scale == 0.0) scale = 1.0;
    double dr = (f[j + 1] - f[j]) / (x[j + 1] - x[j]) / scale;
    double dl = (f[j] - f[j - 1]) / (x[j] - x[j - 1]) / scale;
    double tr = dr / (s * sqrt(1.0 + dr * dr) + 1.0);
    double tl = dl / (s * sqrt(1.0 + dl * dl) + 1.0);
    dfdx[j] = (tr + tl) / (1.0 - tr * tl) * scale;
  }
}

/* MAP1, atlas12_modules.f90:5570-5692.  L is kept 1-based as in the source. */
int orc_map1(const double *xold, const double *fold, int nold,
             const double *xnew, double *fnew, int nnew) {
#define XO(i) xold[(i)-1]
#define FO(i) fold[(i)-1]
  double a = 0, b = 0, c = 0, abac = 0, bbac = 0, cbac = 0, afor = 0, bfor = 0,
         cfor = 0, d, wt;
  int l = 2, ll = 0, l1, l2;
  for (int k = 0; k < nnew; ++k) {
    int past = 0;
    while (xnew[k] >= XO(l)) {
      l = l + 1;
      if (l > nold) {
        past = 1;
        break;
      }
    }
    if (!past && l == ll) {
      fnew[k] = a + (b + c * xnew[k]) * xnew[k];
      continue;
    }
    if (l <= 3 || past) {
      l = l < nold ? l : nold;
      if (!past && l == ll) {
        fnew[k] = a + (b + c * xnew[k]) * xnew[k];
        continue;
      }
      c = 0.0;
      b = (FO(l) - FO(l - 1)) / (XO(l) - XO(l - 1));
      a = FO(l) - XO(l) * b;
      ll = l;
      fnew[k] = a + b * xnew[k];
      continue;
    }
    l1 = l - 1;
    if (l == ll + 1 && l != 3 && l != 4) {
      cbac = cfor;
      bbac = bfor;
      abac = afor;
    } else {
      l2 = l - 2;
      d = (FO(l1) - FO(l2)) / (XO(l1) - XO(l2));
      cbac = FO(l) / ((XO(l) - XO(l1)) * (XO(l) - XO(l2))) +
             (FO(l2) / (XO(l) - XO(l2)) - FO(l1) / (XO(l) - XO(l1))) /
                 (XO(l1) - XO(l2));
      bbac = d - (XO(l1) + XO(l2)) * cbac;
      abac = FO(l2) - XO(l2) * d + XO(l1) * XO(l2) * cbac;
    }
    if (l >= nold) {
      a = abac;
      b = bbac;
      c = cbac;
      ll = l;
      fnew[k] = a + (b + c * xnew[k]) * xnew[k];
      continue;
    }
    d = (FO(l) - FO(l1)) / (XO(l) - XO(l1));
    cfor = FO(l + 1) / ((XO(l + 1) - XO(l)) * (XO(l + 1) - XO(l1))) +
           (FO(l1) / (XO(l + 1) - XO(l1)) - FO(l) / (XO(l + 1) - XO(l))) /
               (XO(l) - XO(l1));
    bfor = d - (XO(l) + XO(l1)) * cfor;
    afor = FO(l1) - XO(l1) * d + XO(l) * XO(l1) * cfor;
    wt = 0.0;
    if (fabs(cfor) != 0.0) wt = fabs(cfor) / (fabs(cfor) + fabs(cbac));
    a = afor + wt * (abac - afor);
    b = bfor + wt * (bbac - bfor);
    c = cfor + wt * (cbac - cfor);
    ll = l;
    fnew[k] = a + (b + c * xnew[k]) * xnew[k];
  }
  return ll - 1;
#undef XO
#undef FO
}

/* SOLVIT, atlas12_modules.f90:5739-5847.  A column-major n x n. */
void orc_solvit(double *A, int n, double *B, int *ipivot) {
#define AA(r, c) A[((c)-1) * n + (r)-1]
#define BB(r) B[(r)-1]
  const double PIVOT_TOL = 1.0e-30;
  int i, j, k, m;
  double pivot, t, c;
  for (i = 1; i <= n - 1; ++i) {
    m = i;
    for (k = i + 1; k <= n; ++k)
      if (fabs(AA(k, i)) > fabs(AA(m, i))) m = k;
    ipivot[i - 1] = m;
    if (m != i) {
      for (k = i + 1; k <= n; ++k) {
        t = AA(i, k);
        AA(i, k) = AA(m, k);
        AA(m, k) = t;
      }
    }
    if (fabs(AA(m, i)) < PIVOT_TOL) AA(m, i) = copysign(PIVOT_TOL, AA(m, i));
    pivot = 1.0 / AA(m, i);
    AA(m, i) = AA(i, i);
    AA(i, i) = pivot;
    for (k = i + 1; k <= n; ++k) AA(k, i) = AA(k, i) * pivot;
    for (j = i + 1; j <= n; ++j) {
      c = AA(i, j);
      if (c == 0.0) continue;
      for (k = i + 1; k <= n; ++k) AA(k, j) = AA(k, j) - AA(k, i) * c;
    }
  }
  if (fabs(AA(n, n)) < PIVOT_TOL) AA(n, n) = copysign(PIVOT_TOL, AA(n, n));
  AA(n, n) = 1.0 / AA(n, n);
  for (i = 1; i <= n - 1; ++i) {
    m = ipivot[i - 1];
    if (m != i) {
      t = BB(m);
      BB(m) = BB(i);
      BB(i) = t;
    }
    c = BB(i);
    for (k = i + 1; k <= n; ++k) BB(k) = BB(k) - AA(k, i) * c;
  }
  for (j = n; j >= 2; --j) {
    BB(j) = BB(j) * AA(j, j);
    c = BB(j);
    for (k = 1; k <= j - 1; ++k) BB(k) = BB(k) - AA(k, j) * c;
  }
  BB(1) = BB(1) * AA(1, 1);
#undef AA
#undef BB
}

/* EXPI, atlas12_modules.f90:21103-21225 (Cody & Thacher 1968 rational fits).
 * The reference caches E1 between calls; the cache does not change values. */
double orc_expi(int n, double x) {
  static const double A0 = -44178.5471728217, A1 = 57721.7247139444,
                      A2 = 9938.31388962037, A3 = 1842.11088668000,
                      A4 = 101.093806161906, A5 = 5.03416184097568;
  static const double B0 = 76537.3323337614, B1 = 32597.1881290275,
                      B2 = 6106.10794245759, B3 = 635.419418378382,
                      B4 = 37.2298352833327;
  static const double C0 = 4.65627107975096e-7, C1 = 0.999979577051595,
                      C2 = 9.04161556946329, C3 = 24.3784088791317,
                      C4 = 23.0192559391333, C5 = 6.90522522784444,
                      C6 = 0.430967839469389;
  static const double D1 = 10.0411643829054, D2 = 32.4264210695138,
                      D3 = 41.2807841891424, D4 = 20.4494785013794,
                      D5 = 3.31909213593302, D6 = 0.103400130404874;
  static const double E0 = -0.999999999998447, E1C = -26.6271060431811,
                      E2 = -241.055827097015, E3 = -895.927957772937,
                      E4 = -1298.85688746484, E5 = -545.374158883133,
                      E6 = -5.66575206533869;
  static const double F1 = 28.6271060422192, F2 = 292.310039388533,
                      F3 = 1332.78537748257, F4 = 2777.61949509163,
                      F5 = 2404.01713225909, F6 = 631.657483280800;
  double ex = exp(-x), e1;
  if (x > 4.0) {
    e1 = (ex + ex * (E0 + (E1C + (E2 + (E3 + (E4 + (E5 + E6 / x) / x) / x) / x) / x) / x) /
                   (x + F1 + (F2 + (F3 + (F4 + (F5 + F6 / x) / x) / x) / x) / x)) /
         x;
  } else if (x > 1.0) {
    e1 = ex * (C6 + (C5 + (C4 + (C3 + (C2 + (C1 + C0 * x) * x) * x) * x) * x) * x) /
         (D6 + (D5 + (D4 + (D3 + (D2 + (D1 + x) * x) * x) * x) * x) * x);
  } else if (x > 0.0) {
    e1 = (A0 + (A1 + (A2 + (A3 + (A4 + A5 * x) * x) * x) * x) * x) /
             (B0 + (B1 + (B2 + (B3 + (B4 + x) * x) * x) * x) * x) -
         log(x);
  } else {
    e1 = 0.0;
  }
  double r = e1;
  if (n == 1) return r;
  for (int i = 1; i <= n - 1; ++i) r = (ex - x * r) / (double)i;
  return r;
}

/* ======================================================================
 * Voigt functions
 * ==================================================================== */

/* Weideman (1994) N=32 coefficients: computed by tests/golden/make_golden.py
 * from the published construction (FFT of exp(-t^2)(L^2+t^2) on
 * t = L tan(theta/2)), Horner order.  They coincide bit-for-bit with the
 * reference's AWEI table (synthe_module.f90:91-126). */
static const double WEI_L = 4.75682846001088411;
static const double WEI_A[32] = {
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

/* voigt_profile, synthe_module.f90:463-537, without the final REAL(4). */
double orc_voigt_weideman(double v, double a) {
  double x = fabs(v), y = a, s = x + y;
  if (s > 15.0) {
    double dr = x * x - y * y - 0.5;
    double di = 2.0 * x * y;
    double d2 = dr * dr + di * di;
    return (-y * dr + x * di) / (SQRTPI * d2);
  }
  double dr = WEI_L + y, di = -x;
  double nr = WEI_L - y, ni = x;
  double d2 = dr * dr + di * di;
  double zr = (nr * dr + ni * di) / d2;
  double zi = (ni * dr - nr * di) / d2;
  double pr = WEI_A[0], pim = 0.0, tmp;
  for (int k = 1; k < 32; ++k) {
    tmp = pr * zr - pim * zi + WEI_A[k];
    pim = pr * zi + pim * zr;
    pr = tmp;
  }
  double sq_r = dr * dr - di * di;
  double sq_i = 2.0 * dr * di;
  double sq_d = sq_r * sq_r + sq_i * sq_i;
  double term1 = 2.0 * (pr * sq_r + pim * sq_i) / sq_d;
  double term2 = dr / (SQRTPI * d2);
  return term1 + term2;
}

float orc_voigt_profile(float v, float a) {
  return (float)orc_voigt_weideman((double)fabsf(v), (double)a);
}

/* TABVOIGT, atlas12_modules.f90:19796-19851 */
void orc_tabvoigt(double vsteps, int n, const double *tabvi,
                  const double *tabh1, int ntab, double *h0tab, double *h1tab,
                  double *h2tab) {
  for (int i = 1; i <= n; ++i) h0tab[i - 1] = (double)(i - 1) / vsteps;
  orc_map1(tabvi, tabh1, ntab, h0tab, h1tab, n);
  for (int i = 1; i <= n; ++i) {
    double vv = orc_powi((double)(i - 1) / vsteps, 2);
    h0tab[i - 1] = exp(-vv);
    h2tab[i - 1] = h0tab[i - 1] - (vv + vv) * h0tab[i - 1];
  }
}

/* VOIGT, atlas12_modules.f90:21033-21097 (tables 1-based via IV) */
double orc_voigt_kurucz(double v, double a, const double *h0, const double *h1,
                        const double *h2) {
  int iv = (int)(v * 200.0 + 1.5);
  if (a < 0.2) {
    if (v <= 10.0) return (h2[iv - 1] * a + h1[iv - 1]) * a + h0[iv - 1];
    return 0.5642 * a / orc_powi(v, 2);
  } else if (a <= 1.4 && a + v <= 3.2) {
    double vv = v * v;
    double hh1 = h1[iv - 1] + h0[iv - 1] * 1.12838;
    double hh2 = h2[iv - 1] + hh1 * 1.12838 - h0[iv - 1];
    double hh3 = (1.0 - h2[iv - 1]) * 0.37613 - hh1 * 0.66667 * vv + hh2 * 1.12838;
    double hh4 = (3.0 * hh3 - hh1) * 0.37613 + h0[iv - 1] * 0.66667 * vv * vv;
    return ((((hh4 * a + hh3) * a + hh2) * a + hh1) * a + h0[iv - 1]) *
           (((-.122727278 * a + .532770573) * a - .96284325) * a + .979895032);
  } else {
    double aa = a * a, vv = v * v;
    double u = (aa + vv) * 1.4142;
    double r = a * 0.79788 / u;
    if (a <= 100.0) {
      double aau = aa / u, vvu = vv / u, uu = u * u;
      r = ((((aau - 10.0 * vvu) * aau * 3.0 + 15.0 * vvu * vvu) + 3.0 * vv - aa) / uu + 1.0) * r;
    }
    return r;
  }
}

/* ======================================================================
 * SYNTHE grid, binning, continuum, line opacity
 * ==================================================================== */

/* synthe.f90:316-324 */
void orc_synthe_grid(double wlbeg, double wlend, double resolu, orc_grid_t *g) {
  g->ratio = 1.0 + 1.0 / resolu;
  g->ratiolg = log(g->ratio);
  g->length = (int32_t)(log(wlend / wlbeg) / g->ratiolg);
  g->ixwlbeg = (int32_t)(log(wlbeg) / g->ratiolg);
  g->wbegin = exp((double)g->ixwlbeg * g->ratiolg);
  if (g->wbegin < wlbeg) {
    g->ixwlbeg = g->ixwlbeg + 1;
    g->wbegin = exp((double)g->ixwlbeg * g->ratiolg);
  }
}

/* mod_mklinelist.f90:898-899 */
int32_t orc_synthe_nbuff(double wlvac, double ratiolg, int32_t ixwlbeg) {
  int32_t ixwl = (int32_t)(log(wlvac) / ratiolg + 0.5);
  return ixwl - ixwlbeg + 1;
}

/* synthe.f90:483-516: quadratic interpolation in log10 kappa across the
 * continuum edges, floor at -15, then 10**x (REAL(4) in REF32). */
void orc_synthe_continuum(int mode, const double *wledge, int nedge,
                          const double *continall, int ncont_stride, int nrhox,
                          double wbegin, double ratio, int length, void *out) {
  double *half = (double *)malloc(sizeof(double) * nedge);
  double *del = (double *)malloc(sizeof(double) * nedge);
  for (int ie = 2; ie <= nedge; ++ie) {
    half[ie - 2] = (wledge[ie - 2] + wledge[ie - 1]) * 0.5;
    del[ie - 2] = orc_powi(wledge[ie - 1] - wledge[ie - 2], 2) * 0.5;
  }
  for (int j = 0; j < nrhox; ++j) {
    const double *ab = continall + (size_t)j * ncont_stride;
    int iedge = 1;
    for (int i = 1; i <= length; ++i) {
      double w = wbegin * orc_powi(ratio, i - 1);
      while (w >= wledge[iedge] && iedge < nedge - 1) iedge = iedge + 1;
      const double *q = ab + 3 * (iedge - 1);
      double wl0 = wledge[iedge - 1], wl1 = wledge[iedge];
      double h = half[iedge - 1], dd = del[iedge - 1];
      double v = ((w - h) * (w - wl1) * q[0] + (wl0 - w) * (w - wl1) * 2.0 * q[1] +
                  (w - wl0) * (w - h) * q[2]) /
                 dd;
      if (mode == ORC_REF32) {
        float cf = (float)v;
        if (cf < -15.0f) cf = -15.0f;
        ((float *)out)[(size_t)j * length + i - 1] = powf(10.0f, cf);
      } else {
        if (v < -15.0) v = -15.0;
        ((double *)out)[(size_t)j * length + i - 1] = pow(10.0, v);
      }
    }
  }
  free(half);
  free(del);
}

/* Scatter one line's profile into buf (1-based bins).  synthe.f90:652-682 */
#define SCATTER(BUF, T)                                                        \
  do {                                                                         \
    if (nb + nstep < 1 || nb - nstep > length) break;                          \
    if (nb < length) {                                                         \
      int maxred = (length - nb) < nstep ? (length - nb) : nstep;              \
      int mb = 1 > (1 - nb) ? 1 : (1 - nb);                                    \
      for (int is = mb; is <= maxred; ++is) BUF[nb + is - 1] += (T)prof[is];    \
      if (nb <= 1) break;                                                      \
    }                                                                          \
    int maxblue = (nb - 1) < nstep ? (nb - 1) : nstep;                         \
    int mb2 = 1 > (nb - length) ? 1 : (nb - length);                           \
    for (int is = mb2; is <= maxblue; ++is) BUF[nb - is - 1] += (T)prof[is];    \
  } while (0)

/* SYNTHE LTE line loop, synthe.f90:559-683 (NLTE tags and the Ca I 4227
 * developer switch are off in production: NLTE_MODE=0, CA4227_MODE=0). */
void orc_synthe_line_opacity(int mode, const orc_lines_t *L, int length,
                             int nrhox, double resolu, const void *continuum,
                             const double *xnfdop, const double *dopple,
                             int nspec, const double *xne, const double *txnxn,
                             const double *hckt, int maxprof,
                             double *opacity_f64_out, float *opacity_out) {
  /* the core walk runs to n10dop even when MAXPROF is smaller */
  double dmax = 0.0;
  for (size_t k = 0; k < (size_t)nrhox * nspec; ++k) dmax = fmax(dmax, dopple[k]);
  size_t cap = (size_t)maxprof + (size_t)(10.0 * dmax * resolu) + 2;
  double *prof = (double *)malloc(sizeof(double) * cap);
  float *pf = (float *)malloc(sizeof(float) * cap);
  float *bufs = (float *)malloc(sizeof(float) * (size_t)length);
  double *bufd = (double *)malloc(sizeof(double) * (size_t)length);
  for (int j = 0; j < nrhox; ++j) {
    const double *xd = xnfdop + (size_t)j * nspec;
    const double *dp = dopple + (size_t)j * nspec;
    memset(bufs, 0, sizeof(float) * length);
    memset(bufd, 0, sizeof(double) * length);
    for (int64_t il = 0; il < L->n; ++il) {
      int nb = L->nbuff[il];
      int nel = L->nelion[il] - 1;
      int ic = nb < 1 ? 1 : (nb > length ? length : nb);
      int nstep, n10dop = (int)(10.0 * dp[nel] * resolu);
      if (mode == ORC_REF32) {
        const float *cont = (const float *)continuum + (size_t)j * length;
        float kappa0 = L->cgf[il] * (float)xd[nel];
        float kapmin = cont[ic - 1] * (float)LINE_CUTOFF;
        if (kappa0 < kapmin) continue;
        kappa0 = kappa0 * (float)exp(-(double)L->elo[il] * hckt[j]);
        if (kappa0 < kapmin) continue;
        float gw = L->gamwf[il] * (float)txnxn[j];
        float adamp = (float)(((double)L->gamrf[il] + (double)L->gamsf[il] * xne[j] + (double)gw) / dp[nel]);
        float dopple_nel = (float)dp[nel];
        if (nb >= 1 && nb <= length) bufs[nb - 1] += kappa0 * orc_voigt_profile(0.0f, adamp);
        float dvoigt = 1.0f / dopple_nel / (float)resolu;
        for (nstep = 1; nstep <= n10dop; ++nstep) {
          pf[nstep] = kappa0 * orc_voigt_profile((float)nstep * dvoigt, adamp);
          if (pf[nstep] < kapmin) break;
        }
        if (nstep > n10dop) {
          float xs = (float)n10dop;
          float x_wing = pf[n10dop] * (xs * xs);
          float qs = sqrtf(x_wing / kapmin);
          int maxstep = qs >= (float)maxprof ? maxprof : (int)qs + 1;
          if (maxstep > maxprof) maxstep = maxprof;
          for (nstep = n10dop + 1; nstep <= maxstep; ++nstep) {
            float s = (float)nstep;
            pf[nstep] = x_wing / (s * s);
          }
          nstep = maxstep;
        }
        /* accumulate the REAL(4) profile in REAL(4) */
        {
          float *BUF = bufs;
          do {
            if (nb + nstep < 1 || nb - nstep > length) break;
            if (nb < length) {
              int maxred = (length - nb) < nstep ? (length - nb) : nstep;
              int mb = 1 > (1 - nb) ? 1 : (1 - nb);
              for (int is = mb; is <= maxred; ++is) BUF[nb + is - 1] += pf[is];
              if (nb <= 1) break;
            }
            int maxblue = (nb - 1) < nstep ? (nb - 1) : nstep;
            int mb2 = 1 > (nb - length) ? 1 : (nb - length);
            for (int is = mb2; is <= maxblue; ++is) BUF[nb - is - 1] += pf[is];
          } while (0);
        }
      } else {
        const float *cont = (const float *)continuum + (size_t)j * length;
        double kappa0 = (double)L->cgf[il] * xd[nel];
        double kapmin = (double)cont[ic - 1] * LINE_CUTOFF;
        if (kappa0 < kapmin) continue;
        kappa0 = kappa0 * exp(-(double)L->elo[il] * hckt[j]);
        if (kappa0 < kapmin) continue;
        double adamp = ((double)L->gamrf[il] + (double)L->gamsf[il] * xne[j] +
                        (double)L->gamwf[il] * txnxn[j]) / dp[nel];
        if (nb >= 1 && nb <= length) bufd[nb - 1] += kappa0 * orc_voigt_weideman(0.0, adamp);
        double dvoigt = 1.0 / dp[nel] / resolu;
        for (nstep = 1; nstep <= n10dop; ++nstep) {
          prof[nstep] = kappa0 * orc_voigt_weideman((double)nstep * dvoigt, adamp);
          if (prof[nstep] < kapmin) break;
        }
        if (nstep > n10dop) {
          double x_wing = prof[n10dop] * ((double)n10dop * (double)n10dop);
          double qs = sqrt(x_wing / kapmin);
          int maxstep = qs >= (double)maxprof ? maxprof : (int)qs + 1;
          if (maxstep > maxprof) maxstep = maxprof;
          for (nstep = n10dop + 1; nstep <= maxstep; ++nstep)
            prof[nstep] = x_wing / ((double)nstep * (double)nstep);
          nstep = maxstep;
        }
        SCATTER(bufd, double);
      }
    }
    for (int i = 0; i < length; ++i) {
      double v = (mode == ORC_REF32) ? (double)bufs[i] : bufd[i];
      if (opacity_f64_out) opacity_f64_out[(size_t)j * length + i] = v;
      if (opacity_out) opacity_out[(size_t)j * length + i] = (float)v;
    }
  }
  free(prof);
  free(pf);
  free(bufs);
  free(bufd);
}

/* ======================================================================
 * JOSH, atlas12_modules.f90:18398-18776 (IFSURF 0 and 1 paths)
 * ==================================================================== */
void orc_josh(const orc_ops_t *ops, int ifscat, int ifsurf, orc_josh_t *s) {
  const int NX = ORC_NXTAU, NR = s->nrhox;
  const double *xtau8 = ops->xtau;
  double xs[ORC_NXTAU], xsbar[ORC_NXTAU], xalpha[ORC_NXTAU];
  double xsbar8[ORC_NXTAU], xalpha8[ORC_NXTAU], xs8[ORC_NXTAU];
  double xh[ORC_NXTAU], xjs[ORC_NXTAU], amat[ORC_NXTAU * ORC_NXTAU];
  double snubar[KW_MAX];
  int ipiv[ORC_NXTAU];
  int j, l, m, maxj = 0;
  s->edd_iters = 0;
  for (j = 0; j < NR; ++j) {
    s->abtot[j] = s->acont[j] + s->aline[j] + s->sigmac[j] + s->sigmal[j];
    s->alpha[j] = (s->sigmac[j] + s->sigmal[j]) / s->abtot[j];
    snubar[j] = (s->acont[j] * s->scont[j] + s->aline[j] * s->sline[j]) /
                (s->acont[j] + s->aline[j]);
  }
  orc_integ(s->rhox, s->abtot, s->taunu, NR, s->abtot[0] * s->rhox[0]);
  if (ifscat == 0) {
    /* IFSCAT=0 never occurs on the hot path (IFSCAT=1 default :1293);
     * restated for IFSURF=1 only. */
    for (j = 0; j < NR; ++j) s->snu[j] = snubar[j];
    maxj = orc_map1(s->taunu, s->snu, NR, xtau8, xs8, NX);
    for (l = 0; l < NX; ++l) xs[l] = xs8[l];
    double h = 0.0;
    for (m = 0; m < NX; ++m) h = h + ops->ch[m] * xs[m];
    s->hnu[0] = h;
    s->maxj = maxj;
    return;
  }
  if (s->taunu[0] > xtau8[NX - 1]) maxj = 1;
  if (maxj != 1) {
    maxj = orc_map1(s->taunu, snubar, NR, xtau8, xsbar8, NX);
    maxj = orc_map1(s->taunu, s->alpha, NR, xtau8, xalpha8, NX);
    for (l = 0; l < NX; ++l) {
      xalpha8[l] = fmax(xalpha8[l], 0.0);
      xsbar8[l] = fmax(xsbar8[l], 1.0e-38);
      xalpha[l] = xalpha8[l];
      xsbar[l] = xsbar8[l];
      if (xtau8[l] < s->taunu[0]) {
        xsbar8[l] = fmax(snubar[0], 1.0e-38);
        xalpha8[l] = fmax(s->alpha[0], 0.0);
        xsbar[l] = xsbar8[l];
        xalpha[l] = xalpha8[l];
      }
    }
    double amax = xalpha[0];
    for (l = 1; l < NX; ++l) amax = fmax(amax, xalpha[l]);
    if (amax <= 0.0) {
      for (l = 0; l < NX; ++l) xs[l] = fmax(xsbar[l], 1.0e-37);
    } else {
      for (l = 0; l < NX; ++l) {
        for (m = 0; m < NX; ++m) amat[m * NX + l] = -xalpha[l] * ops->coefj[m * NX + l];
        amat[l * NX + l] = amat[l * NX + l] + 1.0;
        xs[l] = (1.0 - xalpha[l]) * xsbar[l];
      }
      orc_solvit(amat, NX, xs, ipiv);
      for (l = 0; l < NX; ++l) xs[l] = fmax(xs[l], 1.0e-37);
    }
    if (ifsurf == 1) {
      double h = 0.0;
      for (m = 0; m < NX; ++m) h = h + ops->ch[m] * xs[m];
      s->hnu[0] = h;
      s->maxj = maxj;
      return;
    }
    for (m = 0; m < NX; ++m) xs8[m] = xs[m];
    orc_map1(xtau8, xs8, NX, s->taunu, s->snu, maxj);
  }
  if (maxj != NR) {
    int maxj1 = maxj + 1;
    if (maxj == 1) maxj1 = 1;
    for (j = maxj1; j <= NR; ++j) s->snu[j - 1] = snubar[j - 1];
    m = maxj - 1 > 1 ? maxj - 1 : 1;
    int nm1 = NR - m + 1, nmj = NR - maxj + 1;
    double error = 0.0;
    for (l = 1; l <= 50; ++l) {
      error = 0.0;
      int ifneg = 0;
      s->edd_iters = l;
      for (j = m; j <= NR; ++j) {
        if (s->snu[j - 1] <= 0.0) {
          ifneg = 1;
          for (int jj = m; jj <= NR; ++jj) {
            snubar[jj - 1] = s->bnu[jj - 1];
            s->snu[jj - 1] = s->bnu[jj - 1];
          }
          break;
        }
      }
      orc_deriv(s->taunu + m - 1, s->snu + m - 1, s->hnu + m - 1, nm1);
      for (j = m; j <= NR; ++j) {
        if (s->hnu[j - 1] <= 0.0) {
          ifneg = 1;
          for (int jj = m; jj <= NR; ++jj) {
            snubar[jj - 1] = s->bnu[jj - 1];
            s->snu[jj - 1] = s->bnu[jj - 1];
          }
          orc_deriv(s->taunu + m - 1, s->snu + m - 1, s->hnu + m - 1, nm1);
          break;
        }
      }
      for (j = m; j <= NR; ++j) s->hnu[j - 1] = s->hnu[j - 1] / 3.0;
      orc_deriv(s->taunu + maxj - 1, s->hnu + maxj - 1, s->jmins + maxj - 1, nmj);
      for (j = maxj1; j <= NR; ++j) {
        if (ifneg == 1) s->jmins[j - 1] = 0.0;
        s->jnu[j - 1] = s->jmins[j - 1] + s->snu[j - 1];
        double snew = (1.0 - s->alpha[j - 1]) * snubar[j - 1] + s->alpha[j - 1] * s->jnu[j - 1];
        error = fabs(snew - s->snu[j - 1]) / snew + error;
        s->snu[j - 1] = snew;
      }
      if (error < 0.00001) break;
    }
  }
  s->maxj = maxj;
  if (maxj == 1) {
    s->knu1 = s->jnu[0] / 3.0;
    return;
  }
  double xjs8[ORC_NXTAU], xh8[ORC_NXTAU];
  for (l = 0; l < NX; ++l) {
    xjs[l] = -xs[l];
    for (m = 0; m < NX; ++m) xjs[l] = xjs[l] + ops->coefj[m * NX + l] * xs[m];
    xjs8[l] = xjs[l];
    xh[l] = 0.0;
    for (m = 0; m < NX; ++m) xh[l] = xh[l] + ops->coefh[m * NX + l] * xs[m];
    xh8[l] = xh[l];
  }
  orc_map1(xtau8, xjs8, NX, s->taunu, s->jmins, maxj);
  orc_map1(xtau8, xh8, NX, s->taunu, s->hnu, maxj);
  double xk = 0.0;
  for (m = 0; m < NX; ++m) xk = xk + ops->ck[m] * xs[m];
  s->knu1 = xk;
  for (j = 0; j < maxj; ++j) {
    s->snu[j] = fmax(s->snu[j], 1.0e-38);
    s->jnu[j] = fmax(s->jmins[j] + s->snu[j], 1.0e-38);
  }
}

/* ======================================================================
 * SYNTHE spectrum: synthe.f90:698-718 + setup_opacity_sv :797-833 +
 * process_wavelength_point :848-902 (LTE, fscat=0, bfudge=1, IFSURF=1)
 * ==================================================================== */
void orc_synthe_spectrum(const orc_ops_t *ops, const double *wledge, int nedge,
                         const double *contabs, const double *contscat,
                         int ncont_stride, int nrhox, const double *rhox,
                         const double *hkt, double wbegin, double ratio,
                         int length, const float *opacity, int iw0, int iw1,
                         double *flux, double *cont) {
  double half[4096], del[4096];
  for (int ie = 2; ie <= nedge; ++ie) {
    half[ie - 2] = (wledge[ie - 2] + wledge[ie - 1]) * 0.5;
    del[ie - 2] = orc_powi(wledge[ie - 1] - wledge[ie - 2], 2) * 0.5;
  }
  double acont[KW_MAX], sigmac[KW_MAX], aline[KW_MAX], sigmal[KW_MAX],
      sline[KW_MAX], scont[KW_MAX], bnu[KW_MAX], ehvkt[KW_MAX], stim[KW_MAX];
  double abtot[KW_MAX], alpha[KW_MAX], taunu[KW_MAX], snu[KW_MAX], jnu[KW_MAX],
      hnu[KW_MAX], jmins[KW_MAX];
  float asyn[KW_MAX];
  const double BP = bnu_prefac();
  int iedge = 1;
  /* the reference walks iedge_sv from 1 over every lambda in order; for a
   * sub-range start the search from the beginning as well */
  for (int iw = 1; iw <= iw1; ++iw) {
    double wave8 = wbegin * orc_powi(ratio, iw - 1);
    while (wave8 >= wledge[iedge]) iedge = iedge + 1;
    if (iw < iw0) continue;
    double freq8 = CLIGHT_NMS / wave8;
    for (int j = 0; j < nrhox; ++j)
      asyn[j] = (float)((double)opacity[(size_t)j * length + iw - 1] * (1.0 - exp(-freq8 * hkt[j])));
    double wv = wave8;
    double c1 = (wv - half[iedge - 1]) * (wv - wledge[iedge]) / del[iedge - 1];
    double c2 = (wledge[iedge - 1] - wv) * (wv - wledge[iedge]) * 2.0 / del[iedge - 1];
    double c3 = (wv - wledge[iedge - 1]) * (wv - half[iedge - 1]) / del[iedge - 1];
    for (int j = 0; j < nrhox; ++j) {
      const double *ca = contabs + (size_t)j * ncont_stride + 3 * (iedge - 1);
      const double *cs = contscat + (size_t)j * ncont_stride + 3 * (iedge - 1);
      acont[j] = pow(10.0, c1 * ca[0] + c2 * ca[1] + c3 * ca[2]);
      sigmac[j] = pow(10.0, c1 * cs[0] + c2 * cs[1] + c3 * cs[2]);
    }
    double freq = CLIGHT_NMS / wv;
    double freq15 = freq / 1.0e15;
    for (int j = 0; j < nrhox; ++j) {
      ehvkt[j] = exp(-freq * hkt[j]);
      stim[j] = 1.0 - ehvkt[j];
      bnu[j] = BP * orc_powi(freq15, 3) * ehvkt[j] / stim[j];
      aline[j] = 0.0;
      sigmal[j] = 0.0;
      sline[j] = bnu[j];
      scont[j] = bnu[j];
    }
    orc_josh_t st = {rhox, acont, aline, sigmac, sigmal, scont, sline, bnu, nrhox,
                     abtot, alpha, taunu, snu, jnu, hnu, jmins, 0.0, 0, 0};
    orc_josh(ops, 1, 1, &st);
    double surf = hnu[0];
    for (int j = 0; j < nrhox; ++j) {
      aline[j] = (double)asyn[j] * (1.0 - 0.0);
      sline[j] = bnu[j] * stim[j] / (1.0 - ehvkt[j]);
      sigmal[j] = (double)asyn[j] * 0.0;
    }
    orc_josh(ops, 1, 1, &st);
    double resid = hnu[0] / surf;
    flux[iw - iw0] = resid * surf;
    cont[iw - iw0] = surf;
  }
}

/* ======================================================================
 * ATLAS12 LINOP1, atlas12_modules.f90:18132-18374
 * ==================================================================== */
/* TABLOG, atlas12_modules.f90:2083-2086: 10**((I-16384)*0.001) for every
 * INTEGER(2) I, stored at [I + 32768]. */
void orc_build_tablog(double *out) {
  for (int k = 0; k < 65536; ++k) out[k] = pow(10.0, (double)((k - 32768) - 16384) * 0.001);
}

static inline double tablog_(const orc_atlas_tables_t *tb, int16_t i) {
  return tb->tablog[(int)i + 32768];
}

static void linop_wings(const orc_atlas_tables_t *tb, double center, double adamp,
                        double dopwave, double wlvac, int nu, int numnu,
                        const double *waveset, double tc, double *xl, int kw) {
  /* xl points at XLINES(J,1); XLINES(J,IW) = xl[(IW-1)*kw] */
  const int MAX_WING = 100;
  const double *H0 = tb->h0tab, *H1 = tb->h1tab, *H2 = tb->h2tab;
  int iwmax = nu + MAX_WING < numnu ? nu + MAX_WING : numnu;
  for (int iw = nu; iw <= iwmax; ++iw) {
    double cv;
    if (adamp > 0.20) {
      cv = center * orc_voigt_kurucz((waveset[iw - 1] - wlvac) / dopwave, adamp, H0, H1, H2);
    } else {
      double vv = (waveset[iw - 1] - wlvac) / dopwave;
      if (vv > 10.0) {
        cv = center * INVSQRTPI * adamp / orc_powi(vv, 2);
      } else {
        int iv = (int)(vv * 200.0 + 1.5);
        cv = center * ((H2[iv - 1] * adamp + H1[iv - 1]) * adamp + H0[iv - 1]);
      }
    }
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
  for (int i = 1; i <= MAX_WING; ++i) {
    int iw = nu - i;
    if (iw <= 0) break;
    double cv;
    if (adamp > 0.20) {
      cv = center * orc_voigt_kurucz((wlvac - waveset[iw - 1]) / dopwave, adamp, H0, H1, H2);
    } else {
      double vv = (wlvac - waveset[iw - 1]) / dopwave;
      if (vv > 10.0) {
        cv = center * INVSQRTPI * adamp / orc_powi(vv, 2);
      } else {
        int iv = (int)(vv * 200.0 + 1.5);
        cv = center * ((H2[iv - 1] * adamp + H1[iv - 1]) * adamp + H0[iv - 1]);
      }
    }
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
}

int64_t orc_atlas_linop1(const orc_atlas_tables_t *tb, const int32_t *linedata,
                         int64_t nlines, int nrhox, int kw, const double *xnfdop,
                         const double *dopple, int nspec, const double *xne,
                         const double *txnxn, const double *hckt,
                         const double *tabcont, const int32_t *iwavetab,
                         int nwave, const double *waveset, int numnu,
                         double *xlines) {
  const double CEN_PREFAC4 = 0.026538 / SQRTPI / CLIGHT_NMS;
  const double FOURPI_C_INV = 1.0 / (4.0 * PI_ * CLIGHT_NMS);
  const double RATIOLG = log(1.0 + 1.0 / 2000000.0);
  int ifj[KW_MAX + 2];
  ifj[0] = 0;
  memset(xlines, 0, sizeof(double) * (size_t)numnu * kw);
  int nucont = 1, nu = 1, iwlold = 0;
  double start = waveset[0] - 1.0, stop = waveset[numnu - 1] + 1.0;
  int64_t lineused = 0;
  double gammar = 0, gammas = 0, gammaw = 0;
  for (int64_t line = 0; line < nlines; ++line) {
    const int32_t *rec = linedata + 4 * line;
    int32_t iwl = rec[0];
    int16_t ielion = (int16_t)(rec[1] & 0xffff), ielo = (int16_t)((uint32_t)rec[1] >> 16);
    int16_t igflog = (int16_t)(rec[2] & 0xffff), igr = (int16_t)((uint32_t)rec[2] >> 16);
    int16_t igs = (int16_t)(rec[3] & 0xffff), igw = (int16_t)((uint32_t)rec[3] >> 16);
    if (iwl < iwlold) {
      nucont = 1;
      nu = 1;
    }
    while (iwl >= iwavetab[nucont - 1]) {
      nucont = nucont + 1;
      if (nucont > nwave + 1) {
        nucont = nwave + 1;
        break;
      }
    }
    int nelion = abs(ielion / 10);
    if (nelion < 1 || nelion > nspec) {
      iwlold = iwl;
      continue;
    }
    double wlvac = exp(iwl * RATIOLG);
    double wlvac4 = wlvac;
    if (wlvac < start || wlvac > stop) {
      iwlold = iwl;
      continue;
    }
    /* The reference's CYCLE inside this DO WHILE walks past NUMNU for lines
     * redward of WAVESET(NUMNU-1) (reads beyond the grid); the restatement
     * clamps at NUMNU.  Synthetic inputs keep lines inside the grid. */
    while (nu <= numnu && wlvac >= waveset[nu - 1]) nu = nu + 1;
    if (nu > numnu) nu = numnu;
    double cgf = CEN_PREFAC4 * wlvac4 * tablog_(tb, igflog);
    double elo = tablog_(tb, ielo);
    double adamp = 0.0;
    int ifline = 0;
    const double *xdn = xnfdop + (size_t)(nelion - 1) * kw;
    const double *dpn = dopple + (size_t)(nelion - 1) * kw;
    const double *tcv = tabcont + (size_t)(nucont - 1) * kw;
    for (int J = 8; J <= nrhox; J += 8) {
      ifj[J] = 0;
      double center = cgf * xdn[J - 1];
      if (center < tcv[J - 1]) continue;
      center = center * exp(-elo * hckt[J - 1]);
      if (center < tcv[J - 1]) continue;
      ifj[J] = 1;
      ifline = 1;
      if (adamp == 0.0) {
        gammar = tablog_(tb, igr) * wlvac4 * FOURPI_C_INV;
        gammas = tablog_(tb, igs) * wlvac4 * FOURPI_C_INV;
        gammaw = tablog_(tb, igw) * wlvac4 * FOURPI_C_INV;
      }
      adamp = (gammar + gammas * xne[J - 1] + gammaw * txnxn[J - 1]) / dpn[J - 1];
      double dopwave = dpn[J - 1] * wlvac4;
      linop_wings(tb, center, adamp, dopwave, wlvac, nu, numnu, waveset, tcv[J - 1],
                  xlines + (J - 1), kw);
    }
    for (int K = 8; K <= nrhox; K += 8) {
      if (ifj[K - 8] + ifj[K] == 0) continue;
      for (int J = K - 7; J <= K - 1; ++J) {
        double center = cgf * xdn[J - 1];
        if (center < tcv[J - 1]) continue;
        center = center * exp(-elo * hckt[J - 1]);
        if (center < tcv[J - 1]) continue;
        adamp = (gammar + gammas * xne[J - 1] + gammaw * txnxn[J - 1]) / dpn[J - 1];
        double dopwave = dpn[J - 1] * wlvac4;
        linop_wings(tb, center, adamp, dopwave, wlvac, nu, numnu, waveset, tcv[J - 1],
                    xlines + (J - 1), kw);
      }
    }
    if (ifline == 1) lineused = lineused + 1;
    iwlold = iwl;
  }
  return lineused;
}

/* ======================================================================
 * XLINOP, normal-line branch (TYPE 0 and 3), atlas12_modules.f90:19873-20174.
 * The read loop advances NUCONT on IWL and NU on WLVAC (:20017-20031) and
 * stops at the first record with NU >= NUMNU or WLVAC > WAVESET(NUHI);
 * TYPE 2 is skipped (:20036-20038); the other types (hydrogen, autoionizing,
 * merged continuum) are outside this restatement and skipped.  The walk is
 * LINOP1's with MAX_WING = 2000, LORENTZ_PREFAC = 0.5642 (:19877-19879), and
 * the blue wing and the whole depth cut at the continuum edge WCON
 * (:20057-20060, 20074-20075).
 * ==================================================================== */
static void xlinop_wings(const orc_atlas_tables_t *tb, double center, double adamp, double dopwave,
                         double wlvac, int nu, int numnu, const double *waveset, double tc, double wcon,
                         double *xl, int kw) {
  const int MAX_WING = 2000;
  const double LORENTZ_PREFAC = 0.5642;
  const double *H0 = tb->h0tab, *H1 = tb->h1tab, *H2 = tb->h2tab;
  int iwmax = nu + MAX_WING < numnu ? nu + MAX_WING : numnu;
  for (int iw = nu; iw <= iwmax; ++iw) {
    double cv;
    if (adamp > 0.20) {
      cv = center * orc_voigt_kurucz((waveset[iw - 1] - wlvac) / dopwave, adamp, H0, H1, H2);
    } else {
      double vv = (waveset[iw - 1] - wlvac) / dopwave;
      if (vv > 10.0) {
        cv = center * LORENTZ_PREFAC * adamp / orc_powi(vv, 2);
      } else {
        int iv = (int)(vv * 200.0 + 1.5);
        cv = center * ((H2[iv - 1] * adamp + H1[iv - 1]) * adamp + H0[iv - 1]);
      }
    }
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
  for (int i = 1; i <= MAX_WING; ++i) {
    int iw = nu - i;
    if (iw <= 0) break;
    if (waveset[iw - 1] < wcon) break;
    double cv;
    if (adamp > 0.20) {
      cv = center * orc_voigt_kurucz((wlvac - waveset[iw - 1]) / dopwave, adamp, H0, H1, H2);
    } else {
      double vv = (wlvac - waveset[iw - 1]) / dopwave;
      if (vv > 10.0) {
        cv = center * LORENTZ_PREFAC * adamp / orc_powi(vv, 2);
      } else {
        int iv = (int)(vv * 200.0 + 1.5);
        cv = center * ((H2[iv - 1] * adamp + H1[iv - 1]) * adamp + H0[iv - 1]);
      }
    }
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
}

/* ---- hydrogen line profile (atlas12_modules.f90:20263-21002) ---------- */

/* HFNM: hydrogen oscillator strength f(n,m), :20263-20305 */
double orc_hfnm(int n, int m) {
  if (m <= n) return 0.0;
  const double xn = (double)n;
  const double ginf = 0.2027 / pow(xn, 0.71);
  const double gca = 0.124 / xn;
  const double fkn = xn * 1.9603;
  const double wtc = 0.45 - 2.4 / orc_powi(xn, 3) * (xn - 1.0);
  const double xm = (double)m, xmn = (double)(m - n);
  const double fk = fkn * orc_powi(xm / (xmn * (xm + (double)n)), 3);
  const double xmn12 = pow(xmn, 1.2);
  const double wt = (xmn12 - 1.0) / (xmn12 + wtc);
  return fk * (1.0 - wt * ginf - (0.222 + gca / xm) * (1.0 - wt));
}

/* STARK_PROFILE: the quasistatic Stark wing S(beta, P), :20376-20514 */
double orc_stark_profile(const orc_htab_t *h, double b, double p, int n, int m) {
  int indx = 7;
  const int mmn = m - n;
  if (n <= 3 && mmn <= 2) indx = 2 * (n - 1) + mmn;
  double corr = 1.0;
  const double b2 = b * b, sb = sqrt(b);
  if (b > 500.0) return (1.5 / sb + 27.0 / b2) / b2 * corr;
  int im = (int)(5.0 * p) + 1;
  if (im > 4) im = 4;
  const int ip = im + 1;
  const double wtpp = 5.0 * (p - h->pp[im - 1]);
  const double wtpm = 1.0 - wtpp;
  if (b > 25.12) {
    const double cc = h->c[indx - 1][ip - 1] * wtpp + h->c[indx - 1][im - 1] * wtpm;
    const double dd = h->d[indx - 1][ip - 1] * wtpp + h->d[indx - 1][im - 1] * wtpm;
    corr = 1.0 + dd / (cc + b * sb);
    return (1.5 / sb + 27.0 / b2) / b2 * corr;
  }
  int jm = 1;
  for (int j = 2; j <= 15; ++j)
    if (b <= h->betagrid[j - 1]) {
      jm = j - 1;
      break;
    }
  const int jp = jm + 1;
  const double wtbp = (b - h->betagrid[jm - 1]) / (h->betagrid[jp - 1] - h->betagrid[jm - 1]);
  const double wtbm = 1.0 - wtbp;
  const double cbp = h->propbm[indx - 1][jp - 1][ip - 1] * wtpp + h->propbm[indx - 1][jp - 1][im - 1] * wtpm;
  const double cbm = h->propbm[indx - 1][jm - 1][ip - 1] * wtpp + h->propbm[indx - 1][jm - 1][im - 1] * wtpm;
  corr = 1.0 + cbp * wtbp + cbm * wtbm;
  double pr1 = 0.0, pr2 = 0.0;
  double wt = 0.5 * (10.0 - b);
  wt = wt < 1.0 ? wt : 1.0;
  wt = wt > 0.0 ? wt : 0.0;
  if (b <= 10.0) pr1 = 8.0 / (83.0 + (2.0 + 0.95 * b2) * b);
  if (b >= 8.0) pr2 = (1.5 / sb + 27.0 / b2) / b2;
  return (pr1 * wt + pr2 * (1.0 - wt)) * corr;
}

/* HPROF4's depth vectors (Section 1, :20708-20728) at one depth */
typedef struct {
  double xne, pp, fo, y1b, y1s, t3nhe, t3nh2, c1d, c2d, gcon1, gcon2;
  double xnf1, xnf2, xnfp1, dop1; /* XNF(J,1), XNF(J,2), XNFP(J,1), DOPPLE(J,1) */
} orc_hdepth_t;

static void orc_hdepth(double xne, double t, double xnfp3, double xnh2, double xnf1, double xnf2, double xnfp1,
                       double dop1, orc_hdepth_t *d) {
  const double xne16 = pow(xne, 1.0 / 6.0);
  d->xne = xne;
  d->pp = xne16 * 0.08989 / sqrt(t);
  d->fo = orc_powi(xne16, 4) * 1.25e-9;
  d->y1b = 2.0 / (1.0 + 0.012 / t * sqrt(xne / t));
  const double t4 = t / 10000.0;
  const double t43 = pow(t4, 0.3);
  d->y1s = t43 / xne16;
  d->t3nhe = t43 * xnfp3;
  d->t3nh2 = t43 * xnh2;
  d->c1d = d->fo * 78940.0 / t;
  d->c2d = orc_powi(d->fo, 2) / 5.96e-23 / xne;
  d->gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + xne / 1.0e13);
  d->gcon2 = 0.2 / (1.0 + xne / 1.0e15);
  d->xnf1 = xnf1;
  d->xnf2 = xnf2;
  d->xnfp1 = xnfp1;
  d->dop1 = dop1;
}

/* HPROF4's line constants (Section 2, :20733-20817) */
typedef struct {
  int n, m, ifins;
  double xknm, freqnm, dbeta, wavenm, c1con, c2con, radamp, resont, vdw, starkc, y1num, y1wht;
  double finest[14], finswt[14];
} orc_hline_t;

static void orc_hline(const orc_htab_t *h, int n, int m, orc_hline_t *L) {
  const double FREQ_RYDH = 109677.583403 * 2.99792458e10, CLIGHT_ANGS = 2.99792458e18;
  const double FOURPI = 4.0 * 3.141592653589793;
  const int mmn = m - n;
  const double xn = (double)n, xn2 = xn * xn, xm = (double)m, xm2 = xm * xm;
  const double xmn2 = xm2 * xn2, xm2mn2 = xm2 - xn2, gnm = xm2mn2 / xmn2;
  L->n = n;
  L->m = m;
  if (mmn <= 3 && n <= 4)
    L->xknm = h->xknmtb[n - 1][mmn - 1];
  else
    L->xknm = 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / (double)mmn);
  L->y1num = m == 2 ? 550.0 : m == 3 ? 380.0 : 320.0;
  L->y1wht = 1.0e13;
  if (mmn <= 3) L->y1wht = 1.0e14;
  if (mmn <= 2 && n <= 2) L->y1wht = h->y1wtm[n - 1][mmn - 1];
  L->freqnm = FREQ_RYDH * gnm;
  L->dbeta = CLIGHT_ANGS / orc_powi(L->freqnm, 2) / L->xknm;
  L->wavenm = CLIGHT_ANGS / L->freqnm;
  L->c1con = L->xknm / L->wavenm * gnm * xm2mn2;
  L->c2con = orc_powi(L->xknm / L->wavenm, 2);
  double radamp = h->asum[n - 1] + h->asum[m - 1];
  if (n == 1) radamp = h->asumlyman[m - 1];
  radamp = radamp / FOURPI;
  L->radamp = radamp / L->freqnm;
  double resont = orc_hfnm(1, m) / xm / (1.0 - 1.0 / xm2);
  if (n != 1) resont = resont + orc_hfnm(1, n) / xn / (1.0 - 1.0 / xn2);
  L->resont = resont * 3.92e-24 / gnm;
  L->vdw = 4.45e-26 / gnm * pow(xm2 * (7.0 * xm2 + 5.0), 0.4);
  L->starkc = 1.6678e-18 * L->freqnm * L->xknm;
  if (n > 4 || m > 10) {
    L->ifins = 1;
    L->finest[0] = 0.0;
    L->finswt[0] = 1.0;
  } else if (mmn != 1) {
    L->ifins = h->lncomp[n - 1];
    for (int i = 1; i <= L->ifins; ++i) {
      L->finest[i - 1] = h->stcomp[i - 1][n - 1] * 1.0e7;
      L->finswt[i - 1] = h->stcpwt[i - 1][n - 1] / xn2;
    }
  } else {
    L->ifins = h->lnghal[n - 1];
    const int ipos = h->istal[n - 1];
    for (int i = 1; i <= L->ifins; ++i) {
      const int k = ipos - 1 + i;
      L->finest[i - 1] = h->stalph[k - 1] * 1.0e7;
      L->finswt[i - 1] = h->stwtal[k - 1] / xn2 / 3.0;
    }
  }
}

/* HPROF4(N, M, J, DELW), Section 3 (:20821-21000), in Voigt normalization */
static double orc_hprof4(const orc_htab_t *h, const orc_hline_t *L, const orc_hdepth_t *d, double delw) {
  const double CLIGHT = 2.99792458e10, CLIGHT_ANGS = 2.99792458e18, PI = 3.141592653589793;
  const double SQRTPI = 1.7724538509055159;
  const int n = L->n, m = L->m;
  const double freqnm = L->freqnm;
  const double delstark = -10.0 * delw / L->wavenm * freqnm;
  const double wl = L->wavenm + delw * 10.0;
  const double freq4 = CLIGHT_ANGS / wl;
  const double del = fabs(freq4 - freqnm);
  const double hwstk = L->starkc * d->fo;
  const double hwvdw = L->vdw * d->t3nhe + 2.0 * L->vdw * d->t3nh2;
  const double hwrad = L->radamp;
  double hwres = L->resont * d->xnf1;
  double hwlor = hwres + hwvdw + hwrad;
  int nwid;
  if (d->dop1 >= hwstk && d->dop1 >= hwlor)
    nwid = 1;
  else if (hwlor >= hwstk)
    nwid = 2;
  else
    nwid = 3;
  double mx = d->dop1 > hwlor ? d->dop1 : hwlor;
  mx = mx > hwstk ? mx : hwstk;
  const double hfwid = freqnm * mx;
  double hp = 0.0;
  const int ifcore = fabs(del) <= hfwid;
  const double dop = freqnm * d->dop1;
  if (!ifcore || nwid == 1) {
    for (int i = 0; i < L->ifins; ++i) {
      const double dd = fabs(freq4 - freqnm - L->finest[i]) / dop;
      if (dd <= 7.0) hp = hp + exp(-dd * dd) * L->finswt[i];
    }
    if (ifcore) return hp;
  }
  if (!ifcore || nwid == 2) {
    if (n == 1 && m == 2) {
      hwres = hwres * 4.0;
      hwlor = hwres + hwvdw + hwrad;
      const double hhw = freqnm * hwlor;
      double hprofres;
      if (freq4 > (82259.105 - 4000.0) * CLIGHT) {
        hprofres = hwres * freqnm / PI / (del * del + hhw * hhw) * SQRTPI * dop;
      } else {
        double cutoff = 0.0;
        if (freq4 >= 50000.0 * CLIGHT) {
          const double spacing = 200.0 * CLIGHT;
          const double f22000 = (82259.105 - 22000.0) * CLIGHT;
          if (freq4 < f22000) {
            cutoff = (h->cutoffh2[1] - h->cutoffh2[0]) / spacing * (freq4 - f22000) + h->cutoffh2[0];
          } else {
            int icut = (int)((freq4 - f22000) / spacing);
            if (icut > 89) icut = 89; /* at the 4000 cm^-1 boundary itself the reference reads past the table */
            const double cutfreq = (double)icut * spacing + f22000;
            cutoff = (h->cutoffh2[icut + 1] - h->cutoffh2[icut]) / spacing * (freq4 - cutfreq) + h->cutoffh2[icut];
          }
          cutoff = pow(10.0, cutoff - 14.0) * d->xnfp1 * 2.0 / CLIGHT;
        }
        hprofres = cutoff * SQRTPI * dop;
      }
      double hprofrad = hwrad * freqnm / PI / (del * del + hhw * hhw) * SQRTPI * dop;
      if (freq4 <= 2.463e15) hprofrad = 0.0;
      double hprofvdw = hwvdw * freqnm / PI / (del * del + hhw * hhw) * SQRTPI * dop;
      if (freq4 < 1.8e15) hprofvdw = 0.0;
      hp = hp + (hprofres + hprofrad + hprofvdw);
    } else {
      const double hhw = freqnm * hwlor;
      hp = hp + hhw / PI / (del * del + hhw * hhw) * SQRTPI * dop;
    }
    if (ifcore) return hp;
  }
  const double wty1 = 1.0 / (1.0 + d->xne / L->y1wht);
  const double y1scal = L->y1num * d->y1s * wty1 + d->y1b * (1.0 - wty1);
  const double c1 = d->c1d * L->c1con * y1scal;
  const double c2 = d->c2d * L->c2con;
  const double g1 = 6.77 * sqrt(c1);
  double lg = 0.2114 + log(sqrt(c2) / c1);
  lg = lg > 0.0 ? lg : 0.0;
  const double gnot = g1 * lg * (1.0 - d->gcon1 - d->gcon2);
  const double beta = fabs(delstark) / d->fo * L->dbeta;
  const double y1 = c1 * beta;
  const double y2 = c2 * beta * beta;
  double gam = gnot;
  if (!(y2 <= 1.0e-4 && y1 <= 1.0e-5)) {
    const double e = exp(-(y1 < 80.0 ? y1 : 80.0));
    gam = g1 * (0.5 * e + orc_expi(1, y1) - 0.5 * orc_expi(1, y2)) *
          (1.0 - d->gcon1 / (1.0 + orc_powi(90.0 * y1, 3)) - d->gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1.0e-20) gam = 0.0;
  }
  double prqs = orc_stark_profile(h, beta, d->pp, n, m);
  if (m <= 2) {
    prqs = prqs * 0.5;
    if (freq4 >= (82259.105 - 20000.0) * CLIGHT) {
      if (freq4 > (82259.105 - 4000.0) * CLIGHT) {
        const double beta4000 = 4000.0 * CLIGHT / d->fo * L->dbeta;
        const double prqsp4000 = orc_stark_profile(h, beta4000, d->pp, n, m) * 0.5 / d->fo * L->dbeta;
        const double cutoff4000 = pow(10.0, -11.07 - 14.0) / CLIGHT * d->xnf2;
        hp = hp + cutoff4000 / prqsp4000 * prqs / d->fo * L->dbeta * SQRTPI * dop;
      } else {
        const double f15000 = (82259.105 - 15000.0) * CLIGHT;
        const double spacing = 100.0 * CLIGHT;
        double cutoff;
        if (freq4 < f15000) {
          cutoff = (h->cutoffh2plus[1] - h->cutoffh2plus[0]) / spacing * (freq4 - f15000) + h->cutoffh2plus[0];
        } else {
          int icut = (int)((freq4 - f15000) / spacing);
          if (icut > 109) icut = 109; /* the same at the table's end */
          const double cutfreq = (double)icut * spacing + f15000;
          cutoff = (h->cutoffh2plus[icut + 1] - h->cutoffh2plus[icut]) / spacing * (freq4 - cutfreq) +
                   h->cutoffh2plus[icut];
        }
        cutoff = pow(10.0, cutoff - 14.0) / CLIGHT * d->xnf2;
        hp = hp + cutoff * SQRTPI * dop;
      }
    }
  }
  double f = 0.0;
  if (gam > 0.0) f = gam / PI / (gam * gam + beta * beta);
  const double p1 = orc_powi(0.9 * y1, 2);
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  hp = hp + (prqs * (1.0 + fns) + f) / d->fo * L->dbeta * SQRTPI * dop;
  return hp;
}

/* HPROF4 at one point, for the tests: n, m, the depth's inputs, DELW (nm) */
double orc_hprof4_point(const orc_htab_t *h, int n, int m, double xne, double t, double xnfp3, double xnh2,
                        double xnf1, double xnf2, double xnfp1, double dop1, double delw) {
  orc_hdepth_t d;
  orc_hline_t L;
  orc_hdepth(xne, t, xnfp3, xnh2, xnf1, xnf2, xnfp1, dop1, &d);
  orc_hline(h, n, m, &L);
  return orc_hprof4(h, &L, &d, delw);
}

/* XLINOP's autoionizing lines (TYPE 1, Fano profile, :20201-20226):
 * CENTER = BSHORE*G*XNFP(J,NELION)/RHO(J) with the two TABCONT gates around
 * the Boltzmann factor, then both wings up to MAX_WING = 2000 points of
 * CENTER*(ASHORE*EPSIL + BSHORE)/(EPSIL**2 + 1)/BSHORE, EPSIL =
 * 2*(FREQ - FRELIN)/GAMMAR, each stopping after the first point below
 * TABCONT(J, NUCONT). */
static void xlinop_fano(const orc_nlte_line_t *r, int nu, int numnu, const double *waveset, double xnfp,
                        double rho, double elo_hckt, double tc, double *xl, int kw) {
  const double CLIGHT_NMS = 2.99792458e17;
  const double g = (double)r->gf, ashore = (double)r->gammas, bshore = (double)r->gammaw;
  const double gammar = (double)r->gammar;
  const double frelin = CLIGHT_NMS / r->wlvac;
  double center = bshore * g * xnfp / rho;
  if (center < tc) return;
  center = center * exp(-elo_hckt);
  if (center < tc) return;
  const int hi = nu + 2000 < numnu ? nu + 2000 : numnu;
  for (int iw = nu; iw <= hi; ++iw) {
    const double epsil = 2.0 * (CLIGHT_NMS / waveset[iw - 1] - frelin) / gammar;
    const double cv = center * (ashore * epsil + bshore) / (epsil * epsil + 1.0) / bshore;
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
  for (int i = 1; i <= 2000; ++i) {
    const int iw = nu - i;
    if (iw <= 0) break;
    const double epsil = 2.0 * (CLIGHT_NMS / waveset[iw - 1] - frelin) / gammar;
    const double cv = center * (ashore * epsil + bshore) / (epsil * epsil + 1.0) / bshore;
    xl[(size_t)(iw - 1) * kw] += cv;
    if (cv < tc) break;
  }
}

int64_t orc_atlas_xlinop(const orc_atlas_tables_t *tb, const orc_nlte_line_t *recs, int64_t nrec,
                         int nrhox, int kw, const double *xnfdop, const double *dopple, int nspec,
                         const double *xne, const double *txnxn, const double *hckt,
                         const double *tabcont, const int32_t *iwavetab, int nwave,
                         const double *waveset, int numnu, const double *contx, const double *xnfp,
                         const double *rho, const orc_htab_t *htab, const orc_hatm_t *hatm,
                         double *xlines) {
  const double RYDBERG_INF = 109737.31568157;
  double emerge[KW_MAX];
  for (int j = 0; j < nrhox; ++j) {
    double nstark = 1600.0 / pow(xne[j], 2.0 / 15.0);
    double nmerge = nstark;
    emerge[j] = RYDBERG_INF / (nmerge * nmerge);
  }
  int ifj[KW_MAX + 2];
  ifj[0] = 0;
  int nucont = 1, nu = 1;
  int64_t line;
  for (line = 0; line < nrec; ++line) {
    const orc_nlte_line_t *r = recs + line;
    double wlvac = r->wlvac;
    if (wlvac > waveset[numnu - 1]) return line;
    double wlvac4 = wlvac;
    int32_t iwl = r->nbuff;
    while (iwl >= iwavetab[nucont - 1]) {
      nucont = nucont + 1;
      if (nucont > nwave + 1) {
        nucont = nwave + 1;
        break;
      }
    }
    int stop = 0;
    while (wlvac >= waveset[nu - 1]) {
      nu = nu + 1;
      if (nu >= numnu) {
        stop = 1;
        break;
      }
    }
    if (stop) return line;
    if (r->itype == 2) continue; /* coronal: skipped */
    if (r->itype == -1) {
      /* hydrogen (:20177-20199): CENTER = CGF * BOLTH(J, NBLO), BOLTH =
       * exp(-EH(NBLO)*HCKT)*XNFDOP(J,1); wings in HPROF4 up to MAX_WING, the
       * red one skipping and the blue one stopping blueward of WCON =
       * 1e7 / (CONTX(NCON,1) - EMERGE(J)) */
      const int n = r->nblo, m = r->nbup, ncon = r->ncon;
      if (!htab || !hatm || !xnfp || n < 1 || m <= n || m > 100 || ncon < 1 || ncon > 25 || nspec < 3) continue;
      const double RYDBERG_H = 109677.583403;
      const double eh = n <= 10 ? htab->eh[n - 1] : htab->elim - RYDBERG_H / orc_powi((double)n, 2);
      orc_hline_t L;
      orc_hline(htab, n, m, &L);
      const double cgf = (double)r->gf;
      for (int J = 1; J <= nrhox; ++J) {
        const double tc = tabcont[(size_t)(nucont - 1) * kw + J - 1];
        const double center = cgf * (exp(-eh * hckt[J - 1]) * xnfdop[J - 1]);
        if (center < tc) continue;
        const double wcon = 1.0e7 / (contx[ncon - 1] - emerge[J - 1]);
        orc_hdepth_t d;
        orc_hdepth(xne[J - 1], hatm->t[J - 1], xnfp[(size_t)2 * kw + J - 1], hatm->xnh2[J - 1],
                   hatm->xnf1[J - 1], hatm->xnf2[J - 1], xnfp[J - 1], dopple[J - 1], &d);
        const int hi = nu + 2000 < numnu ? nu + 2000 : numnu;
        for (int iw = nu; iw <= hi; ++iw) {
          if (waveset[iw - 1] < wcon) continue;
          const double cv = center * orc_hprof4(htab, &L, &d, waveset[iw - 1] - wlvac);
          xlines[(size_t)(iw - 1) * kw + J - 1] += cv;
          if (cv < tc) break;
        }
        for (int i = 1; i <= 2000; ++i) {
          const int iw = nu - i;
          if (iw <= 0) break;
          if (waveset[iw - 1] < wcon) break;
          const double cv = center * orc_hprof4(htab, &L, &d, waveset[iw - 1] - wlvac);
          xlines[(size_t)(iw - 1) * kw + J - 1] += cv;
          if (cv < tc) break;
        }
      }
      continue;
    }
    if (r->itype != 0 && r->itype != 3) {
      /* autoionizing (TYPE 1) and merged-continuum (any other TYPE, NLAST =
       * TYPE, :20228-20245) records read XNFP(J, NELION) and RHO(J) */
      const int nel = r->nelion;
      if (!xnfp || !rho || nel < 1 || nel > nspec) continue;
      const double *xp = xnfp + (size_t)(nel - 1) * kw;
      const double elo = (double)r->elo;
      if (r->itype == 1) {
        for (int J = 1; J <= nrhox; ++J)
          xlinop_fano(r, nu, numnu, waveset, xp[J - 1], rho[J - 1], elo * hckt[J - 1],
                      tabcont[(size_t)(nucont - 1) * kw + J - 1], xlines + (J - 1), kw);
      } else {
        const double z = nel == 4 ? 2.0 : 1.0;
        const double nlast = (double)r->itype;
        const double wshift = 1.0e7 / (1.0e7 / wlvac - RYDBERG_INF * (z * z) / (nlast * nlast));
        const double xsectg = (double)r->gf;
        for (int J = 1; J <= nrhox; ++J) {
          const double wmerge = 1.0e7 / (1.0e7 / wlvac - emerge[J - 1] * (z * z));
          const double wmax = wmerge > wshift ? wmerge : wshift;
          const double con = xsectg * xp[J - 1] * exp(-elo * hckt[J - 1]) / rho[J - 1];
          const int hi = nu + 1000 < numnu ? nu + 1000 : numnu;
          for (int iw = nu; iw <= hi; ++iw) {
            if (wmax < waveset[iw - 1]) break;
            xlines[(size_t)(iw - 1) * kw + J - 1] += con;
          }
        }
      }
      continue;
    }
    int nelion = r->nelion;
    if (nelion < 1 || nelion > nspec) continue;
    double cgf = (double)r->gf, elo = (double)r->elo;
    double gammar = (double)r->gammar, gammas = (double)r->gammas, gammaw = (double)r->gammaw;
    int ncon = r->ncon;
    const double *xdn = xnfdop + (size_t)(nelion - 1) * kw;
    const double *dpn = dopple + (size_t)(nelion - 1) * kw;
    const double *tcv = tabcont + (size_t)(nucont - 1) * kw;
    for (int pass = 0; pass < 2; ++pass) {
      /* pass 0: coarse depths 8, 16, ...; pass 1: the gated fine depths */
      for (int K = 8; K <= nrhox; K += 8) {
        int j0 = K, j1 = K;
        if (pass == 0) ifj[K] = 0;
        else {
          if (ifj[K - 8] + ifj[K] == 0) continue;
          j0 = K - 7;
          j1 = K - 1;
        }
        for (int J = j0; J <= j1; ++J) {
          double center = cgf * xdn[J - 1];
          if (center < tcv[J - 1]) continue;
          center = center * exp(-elo * hckt[J - 1]);
          if (center < tcv[J - 1]) continue;
          if (pass == 0) ifj[K] = 1;
          double adamp = (gammar + gammas * xne[J - 1] + gammaw * txnxn[J - 1]) / dpn[J - 1];
          double dopwave = dpn[J - 1] * wlvac4;
          double wcon = 0.0;
          if (ncon > 10) ncon = 0;
          if (ncon > 0) wcon = 1.0e7 / (contx[(size_t)(r->nelionx - 1) * 25 + (ncon - 1)] - emerge[J - 1]);
          if (wlvac < wcon) continue;
          xlinop_wings(tb, center, adamp, dopwave, wlvac, nu, numnu, waveset, tcv[J - 1], wcon,
                       xlines + (J - 1), kw);
        }
      }
    }
  }
  return line;
}

/* ======================================================================
 * SYNTHE compute_line_opacity, normal-metal branch (TYPE 0, 3 and the He I
 * fallthrough TYPE <= -3), synthe_module.f90:3167-3458, in FP64.
 * EMERGE keeps the reference's REAL(4) INGLIS/NMERGE (:3306-3311); the
 * wavelength walk keeps its sequential products (:3429-3452): red wing
 * test-before-add from MAX(1,NBUFF), blue wing add-then-test below NBUFF;
 * points blueward of WCON are skipped, the WCON..WTAIL ramp tapers.
 * ==================================================================== */
/* The grid indices of a merged-continuum edge at one depth
 * (synthe_module.f90:3664-3689, IFVAC = 1): NBUFF1 the first point redward
 * of the line, NBUFF2 at WMERGE, NBUFF3 at WTAIL.  EMERGE and EMERGEH from
 * the REAL(4) Inglis-Teller NMERGE = 1600/XNE**(2/15) - 1.5 (:3344-3347);
 * NELION 1 (H I) takes RYDBERG_H.  Returns 0 when the edge misses the grid. */
static int orc_synthe_merged_bins(double wl, int nlast, int nelion, double xne, double wbegin, double ratio,
                                  int *n1, int *n2, int *n3, int length) {
  const double RYDBERG_INF = 109737.31568157, RYDBERG_H = 109677.583403;
  const double ratiolg = log(ratio);
  const int ixwlbeg = (int)lrint(log(wbegin) / ratiolg);
  const float inglis = (float)(1600.0 / pow(xne, (double)(2.0f / 15.0f)));
  const float nmerge = inglis - 1.5f;
  const double ryd = nelion == 1 ? RYDBERG_H : RYDBERG_INF;
  const double em = ryd / ((double)nmerge * (double)nmerge);
  double wshift = 1.0e7 / (1.0e7 / wl - ryd / ((double)nlast * (double)nlast));
  double wmerge = 1.0e7 / (1.0e7 / wl - em);
  if (wmerge < 0.0) wmerge = wshift + wshift;
  wmerge = wmerge > wshift ? wmerge : wshift;
  wmerge = (wshift + wshift) < wmerge ? (wshift + wshift) : wmerge;
  double wtail = 1.0e7 / (1.0e7 / wmerge - 500.0);
  if (wtail < 0.0) wtail = wmerge + wmerge;
  wtail = (wmerge + wmerge) < wtail ? (wmerge + wmerge) : wtail;
  int ixwl = (int)(log(wl) / ratiolg);
  const float edgeblue = expf((float)ixwl * (float)ratiolg);
  if (edgeblue > (float)wl) ixwl = ixwl - 1;
  *n1 = ixwl + 1 - ixwlbeg + 1;
  *n2 = (int)(log(wmerge) / ratiolg + 0.5) - ixwlbeg + 1;
  *n3 = (int)(log(wtail) / ratiolg + 0.5) - ixwlbeg + 1;
  if (*n1 > length || *n3 < 1) return 0;
  if (*n1 < 1) *n1 = 1;
  return 1;
}

void orc_synthe_nlte_opacity(const orc_nlte_line_t *recs, int64_t n, int length, int nrhox,
                             double wbegin, double ratio, double wlend, double velshift_kms,
                             const float *continuum, const double *xnfdop, const double *dopple,
                             const double *xnfpel, int nspec, const double *xne, const double *txnxn,
                             const double *hckt, const double *contx, double *out) {
  const double RYDBERG_INF = 109737.31568157, CLIGHT_KMS = 299792.458, CUTOFF = LINE_CUTOFF;
  const double dopratio = 1.0 + velshift_kms / CLIGHT_KMS;
  for (int j = 0; j < nrhox; ++j) {
    float inglis = (float)(1600.0 / pow(xne[j], (double)(2.0f / 15.0f)));
    float nmerge = inglis - 1.5f;
    double emerge = RYDBERG_INF / ((double)nmerge * (double)nmerge);
    const float *cont = continuum + (size_t)j * length;
    const double *xd = xnfdop + (size_t)j * nspec, *dp = dopple + (size_t)j * nspec;
    double *buf = out + (size_t)j * length;
    for (int64_t il = 0; il < n; ++il) {
      const orc_nlte_line_t *r = recs + il;
      int t = r->itype;
      if (t == 1 && xnfpel) {
        /* autoionizing (Shore) line, synthe_module.f90:3609-3650: GAMMAS and
         * GAMMAW hold the Shore parameters; the red wing adds then tests */
        const int nel = r->nelion;
        if (nel < 1 || nel > nspec) continue;
        const double wl = r->wlvac * dopratio;
        const int nbuff = r->nbuff;
        const double gr = (double)r->gammar, gs = (double)r->gammas, gw = (double)r->gammaw;
        double kappa0 = gw * (double)r->gf * xnfpel[(size_t)j * nspec + nel - 1];
        const int ic = nbuff < 1 ? 1 : (nbuff > length ? length : nbuff);
        const double kapmin = (double)cont[ic - 1] * CUTOFF;
        if (kappa0 < kapmin) continue;
        kappa0 = kappa0 * exp(-(double)r->elo * hckt[j]);
        if (kappa0 < kapmin) continue;
        const double frelin = CLIGHT_NMS / wl;
        if (wl <= wlend) {
          const int minred = nbuff > 1 ? nbuff : 1;
          double freq = CLIGHT_NMS / (wbegin * orc_powi(ratio, minred - 1));
          for (int ib = minred; ib <= length; ++ib) {
            const double eps = 2.0 * (freq - frelin) / gr;
            const double kappa = kappa0 * (gs * eps + gw) / (eps * eps + 1.0) / gw;
            buf[ib - 1] += kappa;
            if (kappa < (double)cont[ib - 1] * CUTOFF) break;
            freq = freq / ratio;
          }
          if (nbuff == 1) continue;
          if (wl < wbegin) continue;
        }
        int ib = length + 1 < nbuff ? length + 1 : nbuff;
        const int maxblue = ib - 1;
        double freq = CLIGHT_NMS / (wbegin * orc_powi(ratio, ib - 1));
        for (int i = 1; i <= maxblue; ++i) {
          ib = ib - 1;
          freq = freq * ratio;
          const double eps = 2.0 * (freq - frelin) / gr;
          const double kappa = kappa0 * (gs * eps + gw) / (eps * eps + 1.0) / gw;
          buf[ib - 1] += kappa;
          if (kappa < (double)cont[ib - 1] * CUTOFF) break;
        }
        continue;
      }
      if (t >= 4 && xnfpel) {
        /* merged-continuum edge, synthe_module.f90:3652-3696 (vacuum
         * wavelengths, IFVAC = 1): flat opacity from the line to WMERGE,
         * tapering linearly to zero at WTAIL (500 cm^-1 redder) */
        const int nel = r->nelion;
        if (nel < 1 || nel > nspec) continue;
        int n1, n2, n3;
        if (!orc_synthe_merged_bins(r->wlvac * dopratio, t, nel, xne[j], wbegin, ratio, &n1, &n2, &n3, length))
          continue;
        const double kappa = (double)r->gf * xnfpel[(size_t)j * nspec + nel - 1] * exp(-(double)r->elo * hckt[j]);
        const double dn = (double)(n3 - n2);
        double tail = 1.0;
        for (int ib = n1; ib <= (n3 < length ? n3 : length); ++ib) {
          if (ib > n2) tail = (double)(n3 - ib) / dn;
          buf[ib - 1] += kappa * tail;
        }
        continue;
      }
      if (!(t == 0 || t == 3 || t <= -3)) continue;
      int nel = r->nelion;
      if (nel < 1 || nel > nspec) continue;
      double wl = r->wlvac * dopratio;
      int nbuff = r->nbuff;
      double kappa0 = (double)r->gf * xd[nel - 1];
      int ic = nbuff < 1 ? 1 : (nbuff > length ? length : nbuff);
      double kapmin = (double)cont[ic - 1] * CUTOFF;
      if (kappa0 < kapmin) continue;
      kappa0 = kappa0 * exp(-(double)r->elo * hckt[j]);
      if (kappa0 < kapmin) continue;
      double wcon = 0.0, wtail = 0.0;
      if (r->ncon > 0) {
        double cx = contx[(size_t)(r->nelionx - 1) * 26 + (r->ncon - 1)];
        wcon = 1.0e7 / (cx - emerge) * dopratio;
        wtail = 1.0e7 / (cx - emerge - 500.0) * dopratio;
      }
      double adamp = ((double)r->gammar + (double)r->gammas * xne[j] + (double)r->gammaw * txnxn[j]) / dp[nel - 1];
      double dopwl = dp[nel - 1] * wl;
      if (wl <= wlend) {
        int minred = nbuff > 1 ? nbuff : 1;
        double wave = wbegin * orc_powi(ratio, minred - 1);
        for (int ib = minred; ib <= length; ++ib) {
          if (wave >= wcon) {
            double v = fabs(wave - wl) / dopwl;
            double kappa = kappa0 * orc_voigt_weideman(v, adamp);
            if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
            if (kappa < (double)cont[ib - 1] * CUTOFF) break;
            buf[ib - 1] += kappa;
          }
          wave = wave * ratio;
        }
        if (minred == 1) continue;
        if (wl < wbegin) continue;
      }
      int ib = length + 1 < nbuff ? length + 1 : nbuff;
      int maxblue = ib - 1;
      double wave = wbegin * orc_powi(ratio, ib - 1);
      for (int i = 1; i <= maxblue; ++i) {
        ib = ib - 1;
        wave = wave / ratio;
        if (wave < wcon) continue;
        double v = fabs(wave - wl) / dopwl;
        double kappa = kappa0 * orc_voigt_weideman(v, adamp);
        if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
        buf[ib - 1] += kappa;
        if (kappa < (double)cont[ib - 1] * CUTOFF) break;
      }
    }
  }
}

/* ======================================================================
 * ATLAS12 RUN_RT_PASS frequency loop with TCORR/RADIAP/ROSS mode 2,
 * atlas12_modules.f90:3880-3951, :2457-2522, :5072-5097, :5178-5190.
 * KAPP is replaced by the caller's per-frequency ACONT/SIGMAC/SCONT
 * (scont NULL => SCONT = BNU); ALINE = XLINES*STIM, SIGMAL = 0, SLINE = BNU.
 * acc arrays are accumulated into (call with zeroed arrays for mode 1).
 * ==================================================================== */
static void rt_pass_range(const orc_ops_t *ops, int numnu, const double *waveset,
                          const double *rcoset, const double *acont,
                          const double *sigmac, const double *scont, int kw,
                          const double *xlines, int nrhox, const double *rhox,
                          const double *t, const double *hkt, double teff, int nu0,
                          int nu1, orc_accum_t *acc, double *hsurf) {
  const double BP = bnu_prefac();
  double ehvkt[KW_MAX], stim[KW_MAX], bnu[KW_MAX], aline[KW_MAX], sigmal[KW_MAX],
      sline[KW_MAX], sc[KW_MAX];
  double abtot[KW_MAX], alpha[KW_MAX], taunu[KW_MAX], snu[KW_MAX], jnu[KW_MAX],
      hnu[KW_MAX], jmins[KW_MAX], dabtot[KW_MAX];
  for (int nu = nu0; nu <= nu1; ++nu) {
    double wave = waveset[nu - 1];
    double freq = CLIGHT_NMS / wave;
    double rcowt = rcoset[nu - 1];
    double freq15 = freq / 1.0e15;
    const double *ac = acont + (size_t)(nu - 1) * kw;
    const double *sg = sigmac + (size_t)(nu - 1) * kw;
    for (int j = 0; j < nrhox; ++j) {
      ehvkt[j] = exp(-freq * hkt[j]);
      stim[j] = 1.0 - ehvkt[j];
      bnu[j] = BP * orc_powi(freq15, 3) * ehvkt[j] / stim[j];
      sc[j] = scont ? scont[(size_t)(nu - 1) * kw + j] : bnu[j];
      aline[j] = 0.0 + xlines[(size_t)(nu - 1) * kw + j] * stim[j];
      sigmal[j] = 0.0;
      sline[j] = bnu[j];
      jnu[j] = 0.0;
      hnu[j] = 0.0;
      jmins[j] = 0.0;
      snu[j] = 0.0;
    }
    orc_josh_t st = {rhox, ac, aline, sg, sigmal, sc, sline, bnu, nrhox,
                     abtot, alpha, taunu, snu, jnu, hnu, jmins, 0.0, 0, 0};
    orc_josh(ops, 1, 0, &st);
    int neg = 0;
    for (int j = 0; j < nrhox; ++j)
      if (snu[j] < 0.0 || jnu[j] < 0.0 || hnu[j] < 0.0) {
        neg = 1;
        break;
      }
    if (neg) {
      for (int j = 0; j < nrhox; ++j) {
        jnu[j] = fmax(jnu[j], 1.0e-99);
        snu[j] = fmax(snu[j], 1.0e-99);
        hnu[j] = fmax(hnu[j], 1.0e-99);
      }
    }
    if (hsurf) hsurf[nu - nu0] = hnu[0];
    /* TCORR mode 2 */
    orc_deriv(rhox, abtot, dabtot, nrhox);
    for (int j = 0; j < nrhox; ++j) {
      acc->rdabh[j] = acc->rdabh[j] + dabtot[j] / abtot[j] * hnu[j] * rcowt;
      acc->rjmins[j] = acc->rjmins[j] + abtot[j] * jmins[j] * rcowt;
      acc->flxrad[j] = acc->flxrad[j] + hnu[j] * rcowt;
    }
    double term2 = 0.0, d = 0.0;
    for (int j = 1; j <= nrhox; ++j) {
      double term1 = term2;
      if (j != nrhox) d = taunu[j] - taunu[j - 1];
      d = fmax(1.0e-10, d);
      if (d <= 0.01) {
        term2 = (EULER_M1 - log(d)) * d / 4.0 + orc_powi(d, 2) / 12.0 -
                orc_powi(d, 3) / 96.0 + orc_powi(d, 4) / 720.0;
      } else {
        double ex = 0.0;
        if (d < 10.0) ex = orc_expi(3, d);
        if (teff <= 4250.0 && d > 0.005 && d < 0.02) ex = 0.0;
        term2 = 0.5 * (d + ex - 0.5) / d;
      }
      double diagj = term1 + term2;
      double dbdt;
      if (numnu == 1)
        dbdt = 0.0; /* single-frequency branch is not on the hot path */
      else
        dbdt = bnu[j - 1] * freq * hkt[j - 1] / t[j - 1] / fmax(stim[j - 1], 1.0e-30);
      acc->rdiagj[j - 1] = acc->rdiagj[j - 1] +
                           abtot[j - 1] * (diagj - 1.0) / (1.0 - alpha[j - 1] * diagj) *
                               (1.0 - alpha[j - 1]) * dbdt * rcowt;
    }
    /* RADIAP mode 2 */
    for (int j = 0; j < nrhox; ++j) {
      acc->raden[j] = acc->raden[j] + jnu[j] * rcowt;
      acc->h_total[j] = acc->h_total[j] + hnu[j] * rcowt;
      acc->accrad[j] = acc->accrad[j] + abtot[j] * hnu[j] * rcowt;
    }
    acc->pradk0 = acc->pradk0 + st.knu1 * rcowt;
    /* ROSS mode 2 */
    for (int j = 0; j < nrhox; ++j) {
      double dbdt = bnu[j] * freq * hkt[j] / t[j] / stim[j];
      acc->abross[j] = acc->abross[j] + dbdt / abtot[j] * rcowt;
    }
  }
}

/* The frequency loop split into contiguous chunks over the host threads
 * (OMP_NUM_THREADS); each chunk sums in frequency order into private
 * accumulators, which are added in chunk order. */
void orc_atlas_rt_pass(const orc_ops_t *ops, int numnu, const double *waveset,
                       const double *rcoset, const double *acont,
                       const double *sigmac, const double *scont, int kw,
                       const double *xlines, int nrhox, const double *rhox,
                       const double *t, const double *hkt, double teff, int nu0,
                       int nu1, orc_accum_t *acc, double *hsurf) {
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  if (nth > nu1 - nu0 + 1) nth = nu1 - nu0 + 1;
  if (nth <= 1) {
    rt_pass_range(ops, numnu, waveset, rcoset, acont, sigmac, scont, kw, xlines, nrhox, rhox,
                  t, hkt, teff, nu0, nu1, acc, hsurf);
    return;
  }
  double *priv = (double *)calloc((size_t)nth * (8 * KW_MAX + 1), sizeof(double));
#pragma omp parallel num_threads(nth)
  {
    int id = 0;
#ifdef _OPENMP
    id = omp_get_thread_num();
#endif
    int len = nu1 - nu0 + 1;
    int a = nu0 + (int)((long)len * id / nth), b = nu0 + (int)((long)len * (id + 1) / nth) - 1;
    double *p = priv + (size_t)id * (8 * KW_MAX + 1);
    orc_accum_t loc = {p, p + KW_MAX, p + 2 * KW_MAX, p + 3 * KW_MAX, p + 4 * KW_MAX,
                       p + 5 * KW_MAX, p + 6 * KW_MAX, p + 7 * KW_MAX, 0.0};
    if (a <= b)
      rt_pass_range(ops, numnu, waveset, rcoset, acont, sigmac, scont, kw, xlines, nrhox, rhox,
                    t, hkt, teff, a, b, &loc, hsurf ? hsurf + (a - nu0) : NULL);
    p[8 * KW_MAX] = loc.pradk0;
  }
  double *dst[8] = {acc->rjmins, acc->rdabh, acc->rdiagj, acc->flxrad,
                    acc->raden, acc->h_total, acc->accrad, acc->abross};
  for (int id = 0; id < nth; ++id) {
    double *p = priv + (size_t)id * (8 * KW_MAX + 1);
    for (int q = 0; q < 8; ++q)
      for (int j = 0; j < nrhox; ++j) dst[q][j] = dst[q][j] + p[q * KW_MAX + j];
    acc->pradk0 = acc->pradk0 + p[8 * KW_MAX];
  }
  free(priv);
}

/* ======================================================================
 * ROSS(3) :5193-5198, RADIAP(3) :5108-5135, TCORR(3) :2528-2977 (radiative
 * branch), TTAUP :6303-6523, with ROSSTAB a caller table.
 * ==================================================================== */
static const double SIGMA_SB = 5.670374419e-5;

/* ROSSTAB(0,0,0): append the current (T, P, ABROSS) profile */
void orc_rosstab_store(orc_tcorr_t *s) {
  int n = s->nrhox;
  if (s->nross == 0) {
    s->zerot = log10(s->t[0]);
    s->zerop = log10(s->p[0]);
    s->slopet = log10(s->t[n - 1]) - s->zerot;
    s->slopep = log10(s->p[n - 1]) - s->zerop;
  }
  for (int j = 0; j < n; ++j) {
    s->nross = s->nross + 1;
    if (s->nross > s->maxtab) {
      s->nross = s->maxtab;
      break;
    }
    int k = s->nross - 1;
    s->tabt[k] = (log10(s->t[j]) - s->zerot) / s->slopet;
    s->tabp[k] = (log10(s->p[j]) - s->zerop) / s->slopep;
    s->tabk[k] = log10(s->abross[j]);
  }
}

/* ROSSTAB(T, P, V) lookup, IROSSTAB = 1: nearest stored point in each of the
 * four (T, P) quadrants, bilinear when all four exist, else inverse distance */
double orc_rosstab(const orc_tcorr_t *s, double temp, double pres) {
  double tl = (log10(temp) - s->zerot) / s->slopet;
  double pl = (log10(pres) - s->zerop) / s->slopep;
  double rpp = 1e30, rpm = 1e30, rmp = 1e30, rmm = 1e30;
  int ipp = 0, ipm = 0, imp = 0, imm = 0;
  for (int i = 1; i <= s->nross; ++i) {
    double dt = s->tabt[i - 1] - tl, dp = s->tabp[i - 1] - pl;
    double r2 = orc_powi(dt, 2) + orc_powi(dp, 2);
    if (dt >= 0.0) {
      if (dp >= 0.0) {
        if (r2 < rpp) { rpp = r2; ipp = i; }
      } else {
        if (r2 < rpm) { rpm = r2; ipm = i; }
      }
    } else {
      if (dp >= 0.0) {
        if (r2 < rmp) { rmp = r2; imp = i; }
      } else {
        if (r2 < rmm) { rmm = r2; imm = i; }
      }
    }
  }
  double R;
  if (ipp && ipm && imp && imm) {
    double Tpp = s->tabt[ipp - 1], Ppp = s->tabp[ipp - 1], Rpp = s->tabk[ipp - 1];
    double Tpm = s->tabt[ipm - 1], Ppm = s->tabp[ipm - 1], Rpm = s->tabk[ipm - 1];
    double Tmp = s->tabt[imp - 1], Pmp = s->tabp[imp - 1], Rmp = s->tabk[imp - 1];
    double Tmm = s->tabt[imm - 1], Pmm = s->tabp[imm - 1], Rmm = s->tabk[imm - 1];
    double rhi = ((tl - Tmp) * Rpp + (Tpp - tl) * Rmp) / (Tpp - Tmp);
    double phi = ((tl - Tmp) * Ppp + (Tpp - tl) * Pmp) / (Tpp - Tmp);
    double rlo = ((tl - Tmm) * Rpm + (Tpm - tl) * Rmm) / (Tpm - Tmm);
    double plo = ((tl - Tmm) * Ppm + (Tpm - tl) * Pmm) / (Tpm - Tmm);
    R = ((pl - plo) * rhi + (phi - pl) * rlo) / (phi - plo);
  } else {
    double dpp = sqrt(rpp) + 1.0e-5, dpm = sqrt(rpm) + 1.0e-5, dmp = sqrt(rmp) + 1.0e-5,
           dmm = sqrt(rmm) + 1.0e-5;
    double rwt = 1.0 / dpp + 1.0 / dpm + 1.0 / dmp + 1.0 / dmm;
    R = (s->tabk[(ipp > 1 ? ipp : 1) - 1] / dpp + s->tabk[(ipm > 1 ? ipm : 1) - 1] / dpm +
         s->tabk[(imp > 1 ? imp : 1) - 1] / dmp + s->tabk[(imm > 1 ? imm : 1) - 1] / dmm) / rwt;
  }
  return pow(10.0, R);
}

void orc_ttaup(const orc_tcorr_t *s, const double *tin, const double *tau, double *abstd,
               double *ptotal, double *pout, const double *prad, int n) {
  const int MAX_CORRECTOR = 50, STALL_DECREASE = 3, RELAX_TRIGGER = 4;
  const double CONV_TOL = 1.0e-4, DPLOG_MAX = 10.0, OPACITY_REBOOT = 2.0, STALL_RATIO = 0.9;
  const double RELAX_LADDER[4] = {0.5, 0.3, 0.1, 0.05};
  const double g = s->grav;
  double dlgtau = log(tau[1] / tau[0]);
  double plog1 = 0, plog2 = 0, plog3 = 0, plog4 = 0, dplog1 = 0, dplog2 = 0, dplog3 = 0;
  double plog = 0, pnew, dplog = 0, err, perr, best_err, best_plog;
  abstd[0] = 0.1;
  if (prad[0] > 0.0) abstd[0] = fmin(0.1, g * tau[0] / prad[0] / 2.0);
  double abstd1_init = abstd[0];
  for (int J = 1; J <= n; ++J) {
    int j = J - 1;
    if (J == 1) plog = log(g / abstd[0] * tau[0]);
    else if (J <= 4) plog = plog1 + dplog1;
    else plog = (3.0 * plog4 + 8.0 * dplog1 - 4.0 * dplog2 + 8.0 * dplog3) / 3.0;
    err = 1.0;
    perr = 1.0;
    best_err = HUGE_VAL;
    best_plog = plog;
    int N = 0, conv = 0, nstall = 0, rl = 1;
    double relax = 0.5;
    for (;;) {
      ptotal[j] = exp(plog);
      pout[j] = ptotal[j] + (prad[0] - prad[j]) + (0.0 - 0.0);
      if (pout[j] <= 0.0) {
        pout[j] = ptotal[j] * 1.0e-4;
        if (pout[j] <= 0.0) pout[j] = 1.0e-10;
      }
      abstd[j] = orc_rosstab(s, tin[j], pout[j]);
      dplog = g / abstd[j] * tau[j] / ptotal[j] * dlgtau;
      dplog = fmax(0.0, fmin(DPLOG_MAX, dplog));
      N = N + 1;
      if (N == 1) continue;
      if (J == 1) pnew = log(g / abstd[0] * tau[0]);
      else if (J <= 4) pnew = (plog + 2.0 * plog1 + dplog + dplog1) / 3.0;
      else
        pnew = (126.0 * plog1 - 14.0 * plog3 + 9.0 * plog4 + 42.0 * dplog + 108.0 * dplog1 -
                54.0 * dplog2 + 24.0 * dplog3) / 121.0;
      perr = err;
      err = fabs(pnew - plog);
      if (err < best_err) {
        best_err = err;
        best_plog = pnew;
      }
      if (N > STALL_DECREASE && err > STALL_RATIO * perr) {
        nstall = nstall + 1;
        if (nstall >= RELAX_TRIGGER && rl < 4) {
          rl = rl + 1;
          nstall = 0;
        }
      } else {
        nstall = nstall - 1 > 0 ? nstall - 1 : 0;
      }
      relax = RELAX_LADDER[rl - 1];
      plog = (1.0 - relax) * plog + relax * pnew;
      if (err <= CONV_TOL) {
        conv = 1;
        break;
      }
      if (N >= MAX_CORRECTOR) break;
    }
    if (!conv) {
      plog = best_plog;
      ptotal[j] = exp(plog);
      pout[j] = ptotal[j] + (prad[0] - prad[j]);
      if (pout[j] <= 0.0) pout[j] = fmax(ptotal[j] * 1.0e-4, 1.0e-10);
      abstd[j] = orc_rosstab(s, tin[j], pout[j]);
      dplog = g / abstd[j] * tau[j] / ptotal[j] * dlgtau;
      dplog = fmax(0.0, fmin(DPLOG_MAX, dplog));
    }
    if (J == 1 && (abstd[0] / abstd1_init > OPACITY_REBOOT || abstd1_init / abstd[0] > OPACITY_REBOOT)) {
      abstd1_init = abstd[0];
      plog = log(g / abstd[0] * tau[0]);
      ptotal[0] = exp(plog);
      pout[0] = ptotal[0];
      if (pout[0] > 0.0) {
        abstd[0] = orc_rosstab(s, tin[0], pout[0]);
        plog = log(g / abstd[0] * tau[0]);
        ptotal[0] = exp(plog);
        pout[0] = ptotal[0];
      }
      dplog = g / abstd[0] * tau[0] / ptotal[0] * dlgtau;
      dplog = fmax(0.0, fmin(DPLOG_MAX, dplog));
    }
    plog4 = plog3;
    plog3 = plog2;
    plog2 = plog1;
    plog1 = plog;
    dplog3 = dplog2;
    dplog2 = dplog1;
    dplog1 = dplog;
  }
}

double orc_atlas_finish(orc_tcorr_t *s) {
  const int n = s->nrhox;
  const double FOUR_SIGMA_OVER_PI = 4.0 * SIGMA_SB / PI_;
  const double FOURPI_OVER_C = 4.0 * PI_ / CLIGHT;
  const double FLUX = SIGMA_SB * orc_powi(s->teff, 4) / (4.0 * PI_);
  const double ABROSS_FLOOR = 1.0e-30, RDIAGJ_FLOOR = 1.0e-30, HRATIO_DTLAMB_OFF = 1.0e-3;
  double dtdrhx[KW_MAX], dabros[KW_MAX], codrhx[KW_MAX], G[KW_MAX], gflux[KW_MAX], dtau[KW_MAX];
  double flxdrv[KW_MAX], dum[KW_MAX], tinteg[KW_MAX], tplus[KW_MAX], taustd[KW_MAX];
  double tnew1[KW_MAX], tnew2[KW_MAX], prdnew[KW_MAX], ab1[KW_MAX], ab2[KW_MAX], pt1[KW_MAX],
      pt2[KW_MAX], p1[KW_MAX], p2[KW_MAX], ppp[KW_MAX], rrr[KW_MAX], drhox[KW_MAX];
  double remap[10][KW_MAX];
  int j;
  /* ROSS(3) */
  for (j = 0; j < n; ++j) s->abross[j] = FOUR_SIGMA_OVER_PI * orc_powi(s->t[j], 3) / s->abross[j];
  orc_integ(s->rhox, s->abross, s->tauros, n, s->abross[0] * s->rhox[0]);
  orc_rosstab_store(s); /* RX = ROSSTAB(0,0,0), atlas12c.f90:586 */
  /* RADIAP(3) */
  double errormax = 0.0;
  for (j = 0; j < n; ++j) {
    s->raden[j] = s->raden[j] * FOURPI_OVER_C;
    s->accrad[j] = s->accrad[j] * FOURPI_OVER_C;
    if (s->h_total[j] / FLUX > 1.0) s->accrad[j] = s->accrad[j] * FLUX / s->h_total[j];
    errormax = fmax(errormax, s->h_total[j] / FLUX);
  }
  s->pradk0 = s->pradk0 * FOURPI_OVER_C;
  if (errormax > 1.0) s->pradk0 = s->pradk0 / errormax;
  orc_integ(s->rhox, s->accrad, s->prad, n, s->accrad[0] * s->rhox[0]);
  /* TCORR(3) */
  orc_deriv(s->rhox, s->t, dtdrhx, n);
  orc_deriv(s->rhox, s->abross, dabros, n);
  for (j = 0; j < n; ++j) {
    double abs_ = fmax(s->abross[j], ABROSS_FLOOR);
    s->rdabh[j] = s->rdabh[j] - s->flxrad[j] * dabros[j] / abs_;
    codrhx[j] = (s->rdabh[j] + 0.0) / (s->flxrad[j] + 0.0);
  }
  codrhx[0] = 0.0;
  codrhx[1] = 0.0;
  orc_integ(s->rhox, codrhx, G, n, 0.0);
  for (j = 0; j < n; ++j) {
    G[j] = exp(G[j]);
    gflux[j] = G[j] * (s->flxrad[j] + 0.0 - FLUX) / (s->flxrad[j] + 0.0);
  }
  orc_integ(s->tauros, gflux, dtau, n, 0.0);
  for (j = 0; j < n; ++j) {
    dtau[j] = dtau[j] / G[j];
    dtau[j] = fmax(-s->tauros[j] / 3.0, fmin(s->tauros[j] / 3.0, dtau[j]));
    s->dtflux[j] = -dtau[j] * dtdrhx[j] / fmax(s->abross[j], ABROSS_FLOOR);
  }
  const double MAX_DT = 0.04 * s->teff;
  double maxerr = 0.0;
  for (j = 0; j < n; ++j) {
    s->flxerr[j] = (s->flxrad[j] + 0.0 - FLUX) / FLUX * 100.0;
    maxerr = fmax(maxerr, fabs(s->flxerr[j]));
  }
  orc_deriv(s->tauros, s->flxerr, flxdrv, n);
  for (j = 0; j < n; ++j) {
    double hratio = 0.0 / (0.0 + fmax(s->flxrad[j], 1.0e-30));
    if (hratio < HRATIO_DTLAMB_OFF) flxdrv[j] = s->rjmins[j] / fmax(s->abross[j], ABROSS_FLOOR) / FLUX * 100.0;
    s->dtlamb[j] = -flxdrv[j] * FLUX / 100.0 / fmax(fabs(s->rdiagj[j]), RDIAGJ_FLOOR) *
                   copysign(1.0, s->rdiagj[j]) * fmax(s->abross[j], ABROSS_FLOOR);
    s->dtlamb[j] = fmax(-MAX_DT, fmin(MAX_DT, s->dtlamb[j]));
  }
  double dtsur = (FLUX - s->flxrad[0]) / FLUX * 0.25 * s->t[0];
  dtsur = fmax(-MAX_DT, fmin(MAX_DT, dtsur));
  for (j = 0; j < n; ++j) dum[j] = s->dtflux[j] + s->dtlamb[j];
  orc_integ(s->tauros, dum, tinteg, n, 0.0);
  double xn = 0.1, tone, ttwo;
  orc_map1(s->tauros, tinteg, n, &xn, &tone, 1);
  xn = 2.0;
  orc_map1(s->tauros, tinteg, n, &xn, &ttwo, 1);
  double tav = (ttwo - tone) / 2.0;
  if (dtsur * tav <= 0.0) tav = 0.0;
  if (fabs(tav) > fabs(dtsur)) tav = dtsur;
  dtsur = dtsur - tav;
  for (j = 0; j < n; ++j) {
    s->dtsurf[j] = dtsur;
    s->t1[j] = s->dtflux[j] + s->dtlamb[j] + s->dtsurf[j];
  }
  for (j = 0; j < n; ++j) {
    if (s->iter == 1) {
    } else if (s->oldt1[j] * s->t1[j] > 0.0 && fabs(s->oldt1[j]) > fabs(s->t1[j])) {
      s->t1[j] = s->t1[j] * 1.25;
    } else if (s->oldt1[j] * s->t1[j] < 0.0) {
      s->t1[j] = s->t1[j] * 0.5;
    }
    s->oldt1[j] = s->t1[j];
  }
  for (j = 0; j < n; ++j) {
    tplus[j] = s->t[j] + s->t1[j];
    taustd[j] = pow(10.0, -6.875 + (double)j * 0.125);
  }
  orc_map1(s->tauros, s->t, n, taustd, tnew1, n);
  orc_map1(s->tauros, s->prad, n, taustd, prdnew, n);
  orc_ttaup(s, tnew1, taustd, ab1, pt1, p1, prdnew, n);
  orc_map1(s->tauros, tplus, n, taustd, tnew2, n);
  orc_ttaup(s, tnew2, taustd, ab2, pt2, p2, prdnew, n);
  for (j = 0; j < n; ++j) ppp[j] = (pt2[j] - pt1[j]) / pt1[j];
  orc_map1(taustd, ppp, n, s->tauros, rrr, n);
  for (j = 0; j < n; ++j) drhox[j] = rrr[j] * s->rhox[j];
  for (j = 0; j < n; ++j) s->t[j] = s->t[j] + s->t1[j];
  for (int i = 2; i <= n; ++i) {
    int jj = n + 1 - i;
    s->t[jj - 1] = fmin(s->t[jj - 1], s->t[jj] - 1.0);
  }
  for (j = 0; j < n; ++j) s->t[j] = fmax(s->t[j], 1200.0);
  for (j = 0; j < n; ++j) s->rhox[j] = s->rhox[j] + drhox[j];
  double *src[9] = {s->rhox, s->t, s->p, s->xne, s->abross, s->prad, s->vturb, s->pturb, s->accrad};
  for (int q = 0; q < 9; ++q) orc_map1(s->tauros, src[q], n, taustd, remap[q], n);
  for (j = 0; j < n; ++j)
    if (s->tauros[0] > taustd[j] && remap[4][j] < 0.0) remap[4][j] = s->abross[0];
  for (int q = 0; q < 8; ++q)
    for (j = 0; j < n; ++j) src[q][j] = remap[q][j];
  for (j = 0; j < n; ++j) s->tauros[j] = taustd[j];
  return maxerr;
}

/* ---- SELECTLINES (atlas12_modules.f90:19171-19781) -------------------- */

/* XNFDOPMAX(NELION, NU) = max over J of XNFDOP(J, NELION) / TABCONT(J, NU),
 * starting from 0 (:19248-19256).  xmax [nwave+1][nspec]. */
void orc_xnfdopmax(int nrhox, int kw, const double *xnfdop, int nspec, const double *tabcont,
                   int nwave, double *xmax) {
  for (int nu = 0; nu <= nwave; ++nu)
    for (int e = 0; e < nspec; ++e) {
      double m = 0.0;
      for (int j = 0; j < nrhox; ++j) {
        const double r = xnfdop[(size_t)e * kw + j] / tabcont[(size_t)nu * kw + j];
        if (r > m) m = r;
      }
      xmax[(size_t)nu * nspec + e] = m;
    }
}

/* INT() of a REAL(8) as x86-64 converts it (cvttsd2si): truncation toward
 * zero, and the integer-indefinite -2**31 for NaN or a value out of range */
static int32_t sel_fint(double x) {
  if (!(x > -2147483649.0 && x < 2147483648.0)) return INT32_MIN;
  return (int32_t)x;
}
/* INTEGER(2) = INTEGER(4): the low 16 bits */
static int16_t sel_i16(int32_t v) { return (int16_t)(uint16_t)(uint32_t)v; }
static double sel_tablog(int16_t i) { return pow(10.0, (double)((int32_t)i - 16384) * 0.001); } /* :2083 */
static void sel_unpack(const int32_t *r, int32_t *iwl, int16_t *f) { /* UNPACK_LINEDATA :1950-1963 */
  *iwl = r[0];
  for (int k = 0; k < 3; ++k) {
    f[2 * k] = (int16_t)(uint16_t)((uint32_t)r[1 + k] & 0xffffu);
    f[2 * k + 1] = (int16_t)(uint16_t)((uint32_t)r[1 + k] >> 16);
  }
}
static void sel_pack(int32_t *o, int32_t iwl, const int16_t *f) { /* PACK_LINEDATA :1967-1977 */
  o[0] = iwl;
  for (int k = 0; k < 3; ++k)
    o[1 + k] = (int32_t)((uint32_t)(uint16_t)f[2 * k] | ((uint32_t)(uint16_t)f[2 * k + 1] << 16));
}

/* One database loop of SELECTLINES.  The loop body follows the reference
 * case by case: the NU advance (DO WHILE IWL >= IWAVETAB(NU), setting FREQ
 * and, for H2O, IGR), the species index, the XNFDOPMAX / CENRATIO /
 * Boltzmann tests against HCKT(NRHOX), and the packed record.  Module
 * variables that outlive the loop (NU, FREQ, IGR) go through st. */
int64_t orc_atlas_selectlines(const orc_select_tables_t *tb, int kind, const void *recs, int64_t n,
                              orc_select_state_t *st, const double *xmax, int nspec, double hckt_last,
                              const int32_t *iwt, const double *wavetab, int nwave,
                              int32_t *out, int64_t cap, int64_t *bad) {
  const double CLIGHT_NMS = 2.99792458e17;          /* :325 */
  const double CEN_PREFAC = 0.026538 / 1.7724538509055159; /* :19178, SQRTPI :317 */
  const double RATIOLG = log(1.0 + 1.0 / 2000000.0);
  int nu = st->nu;
  double freq = st->freq;
  int16_t igr = (int16_t)st->igr;
  int64_t ns = 0;
  *bad = -1;
  for (int64_t i = 0; i < n; ++i) {
    int32_t iwl = 0;
    int16_t f[6] = {0, 0, 0, 0, 0, 0}; /* IELION, IELO, IGFLOG, IGR, IGS, IGW */
    double elo_exp = 0.0;                 /* the energy in the Boltzmann test */
    int nelion;
    if (kind == ORC_SEL_TIO) {
      const int32_t *w = (const int32_t *)recs + 8 * i;
      if (w[4] != 822) continue;           /* :19599 */
      const int iso = w[5] - 45;
      if (iso < 1 || iso > 5) continue;
      float wl4, e1, e2, gf4;
      memcpy(&wl4, &w[0], 4);
      memcpy(&gf4, &w[1], 4);
      memcpy(&e1, &w[2], 4);
      memcpy(&e2, &w[3], 4);
      const double W = (double)wl4;
      if (W <= 0.0) continue;
      iwl = sel_fint(log(W) / RATIOLG + 0.5);
      while (iwl >= iwt[nu - 1]) {
        if (nu == nwave + 1) { *bad = i; return ORC_SEL_ESENTINEL; }
        freq = CLIGHT_NMS / wavetab[nu - 1];
        ++nu;
      }
      const int32_t kgflog = sel_fint(round((double)gf4 * 1000.0)) + 16384;
      f[2] = sel_i16(kgflog + tb->tio_isocorr[iso - 1] > 1 ? kgflog + tb->tio_isocorr[iso - 1] : 1);
      nelion = 895;
      if (nelion > nspec) { *bad = i; return ORC_SEL_ENELION; }
      const double xm = xmax[(size_t)(nu - 1) * nspec + nelion - 1];
      if (xm == 0.0) continue;
      const double cen = CEN_PREFAC * sel_tablog(f[2]) * xm / freq;
      if (cen < 1.0) continue;
      const double a1 = fabs((double)e1), a2 = fabs((double)e2);
      const double elo = a2 < a1 ? a2 : a1;
      if (cen * exp(-elo * hckt_last) < 1.0) continue;
      f[0] = (int16_t)(8949 + iso);
      f[1] = sel_i16(sel_fint(log10(elo > 1.0e-10 ? elo : 1.0e-10) * 1000.0 + 16384.5));
      const double g = w[6] == 0 ? 2.223e13 / (W * W) : pow(10.0, (double)w[6] * 0.01);
      igr = sel_i16(sel_fint(log10(g) * 1000.0 + 16384.5));
      f[3] = igr;
      f[4] = 1;
      f[5] = 9384;
    } else if (kind == ORC_SEL_H2O) {
      const unsigned char *b = (const unsigned char *)recs + 8 * i;
      int16_t ielo_in, igf_in;
      memcpy(&iwl, b, 4);
      memcpy(&ielo_in, b + 4, 2);
      memcpy(&igf_in, b + 6, 2);
      while (iwl >= iwt[nu - 1]) {
        if (nu == nwave + 1) { *bad = i; return ORC_SEL_ESENTINEL; }
        freq = CLIGHT_NMS / wavetab[nu - 1];
        /* GAMMAR = 2.474D-22 * FREQ**2 * 0.001 (a default REAL literal) */
        const double gammar = 2.474e-22 * (freq * freq) * (double)0.001f;
        igr = sel_i16(sel_fint(log10(gammar) * 1000.0 + 16384.5));
        ++nu;
      }
      int iso;
      if (ielo_in > 0 && igf_in > 0) iso = 1;
      else if (ielo_in > 0) iso = 2;
      else if (igf_in > 0) iso = 3;
      else iso = 4;
      f[0] = (int16_t)(-(9399 + iso));
      const double elo = (double)abs((int32_t)ielo_in);
      const int32_t kgflog = abs((int32_t)igf_in);
      f[2] = sel_i16(kgflog + tb->h2o_isocorr[iso - 1] > 1 ? kgflog + tb->h2o_isocorr[iso - 1] : 1);
      nelion = 940;
      if (nelion > nspec) { *bad = i; return ORC_SEL_ENELION; }
      const double xm = xmax[(size_t)(nu - 1) * nspec + nelion - 1];
      if (xm == 0.0) continue;
      const double cen = CEN_PREFAC * sel_tablog(f[2]) * xm / freq;
      if (cen < 1.0) continue;
      if (cen * exp(-elo * hckt_last) < 1.0) continue;
      f[1] = sel_i16(sel_fint(log10(elo) * 1000.0 + 16384.5));
      f[3] = igr;
      f[4] = 1;
      f[5] = 9384;
    } else {
      /* LINEREC databases: UNPACK_LINEDATA sets every field, IGR included */
      const int32_t *r = (const int32_t *)recs + 4 * i;
      sel_unpack(r, &iwl, f);
      igr = f[3];
      while (iwl >= iwt[nu - 1]) {
        if (nu == nwave + 1) { *bad = i; return ORC_SEL_ESENTINEL; }
        freq = CLIGHT_NMS / wavetab[nu - 1];
        ++nu;
      }
      if (kind == ORC_SEL_DIATOMIC) {
        const int32_t molcode = f[0];
        int imol = -1;
        for (int k = 0; k < tb->nmol; ++k)
          if (tb->molcodes[k] == molcode) { imol = k; break; }
        if (imol < 0) { *bad = i; return ORC_SEL_EMOLCODE; }
        const int32_t kgflog = f[2];
        f[2] = sel_i16(kgflog + tb->isox[imol] > 1 ? kgflog + tb->isox[imol] : 1);
      } else if (kind == ORC_SEL_H3PLUS) {
        const int32_t kgflog = f[2];
        f[2] = sel_i16(kgflog - 1272 > 1 ? kgflog - 1272 : 1);
        f[4] = 1;
        f[5] = 9384;
      }
      nelion = kind == ORC_SEL_H3PLUS ? 895 : abs((int32_t)f[0] / 10);
      if (nelion < 1 || nelion > nspec) {
        if (kind == ORC_SEL_LOWPRED) continue; /* :19283-19287 */
        *bad = i;
        return ORC_SEL_ENELION;
      }
      const double xm = xmax[(size_t)(nu - 1) * nspec + nelion - 1];
      if (kind == ORC_SEL_LOWPRED || kind == ORC_SEL_LOWOBS) {
        if (xm <= 1.0e-37) continue;
      } else if (xm == 0.0) {
        continue;
      }
      const double cen = CEN_PREFAC * sel_tablog(f[2]) * xm / freq;
      if (cen < 1.0) continue;
      elo_exp = sel_tablog(f[1]);
      if (cen * exp(-elo_exp * hckt_last) < 1.0) continue;
    }
    if (ns >= cap) { *bad = i; return ORC_SEL_EOVERFLOW; }
    sel_pack(out + 4 * ns, iwl, f);
    ++ns;
  }
  st->nu = nu;
  st->freq = freq;
  st->igr = igr;
  return ns;
}

/* ======================================================================
 * SYNTHE's hydrogen and deuterium lines: compute_line_opacity's TYPE -1/-2
 * branch (synthe_module.f90:3460-3606) with hydrogen_line_profile
 * (:1032-1980).  FP64 restatement; the tables are SYNTHE's REAL(4) ones and
 * the frequency thresholds the reference forms in single precision
 * ((82259.10 - 4000.0) * REAL(CLIGHT,4) and the like) are formed in float.
 * ==================================================================== */
static const double S_CLIGHT = 2.99792458e10, S_CLIGHT_ANGS = 2.99792458e18;
static const double S_RYDBERG_H = 109677.583403, S_ELIM_HI = 109678.764;
static const double S_PI = 3.141592653589793;
/* H_SERIES_LIMITS (atlas12_modules.f90:392-395), CONTH in compute_line_opacity */
static const double S_CONTH[15] = {109678.764, 27419.659, 12186.462, 6854.871, 4387.113,
                                   3046.604,   2238.320,  1713.713,  1354.044, 1096.776,
                                   906.426,    761.650,   648.980,   559.579,  487.456};

/* Lyman alpha's frequency thresholds: (82259.10 - dw) * REAL(CLIGHT,4) in REAL(4) */
static double s_lya_freq(float dw) { return (double)((82259.10f - dw) * (float)2.99792458e10); }

/* lya_h2_blue_cutoff (:1916-1940): the H2 quasi-molecular satellite on a
 * 200 cm^-1 grid blueward of 22000 cm^-1 below Lyman alpha; zero below
 * 50000 cm^-1.  The table index stays inside CUTOFFH2 at the window's edge. */
static double s_lya_h2_blue(const orc_htab_t *h, double freq, double xnfph1) {
  const float c4 = (float)2.99792458e10;
  const float spc = 200.0f * c4, freq22 = (82259.10f - 22000.0f) * c4;
  if (freq < (double)(50000.0f * c4)) return 0.0;
  double cval;
  if (freq < (double)freq22) {
    cval = (h->cutoffh2[1] - h->cutoffh2[0]) / (double)spc * (freq - (double)freq22) + h->cutoffh2[0];
  } else {
    int ic = (int)((freq - (double)freq22) / (double)spc);
    if (ic > 89) ic = 89;
    const float cfreq = (float)ic * spc + freq22;
    cval = (h->cutoffh2[ic + 1] - h->cutoffh2[ic]) / (double)spc * (freq - (double)cfreq) + h->cutoffh2[ic];
  }
  return pow(10.0, cval - 14.0) * (double)(float)xnfph1 * 2.0 / (double)c4;
}

/* lya_h2plus_red_cutoff (:1956-1978): the H2+ satellite, 100 cm^-1 grid */
static double s_lya_h2plus_red(const orc_htab_t *h, double freq, double xnfph2) {
  const float c4 = (float)2.99792458e10;
  const float spc = 100.0f * c4, freq15 = (82259.10f - 15000.0f) * c4;
  double cval;
  if (freq < (double)freq15) {
    cval = (h->cutoffh2plus[1] - h->cutoffh2plus[0]) / (double)spc * (freq - (double)freq15) + h->cutoffh2plus[0];
  } else {
    int ic = (int)((freq - (double)freq15) / (double)spc);
    if (ic > 109) ic = 109;
    const float cfreq = (float)ic * spc + freq15;
    cval = (h->cutoffh2plus[ic + 1] - h->cutoffh2plus[ic]) / (double)spc * (freq - (double)cfreq) +
           h->cutoffh2plus[ic];
  }
  return pow(10.0, cval - 14.0) / (double)c4 * (double)(float)xnfph2;
}

/* expint1 (:731-753): A&S 5.1.56 below 1, a Pade form to 30, zero beyond */
static double s_expint1(double x) {
  if (x <= 0.0) return 0.0;
  if (x <= 1.0)
    return -log(x) - 0.57721566 +
           x * (0.99999193 + x * (-0.24991055 + x * (0.05519968 + x * (-0.00976004 + x * 0.00107857))));
  if (x <= 30.0) return (x * (x + 2.334733) + 0.25062) / (x * (x + 3.330657) + 1.681534) / x * exp(-x);
  return 0.0;
}

/* the depth arrays hydrogen_line_profile recomputes when the atmosphere
 * changes (:1203-1248) */
typedef struct {
  double xne, t, pp, fo, y1b, y1s, t3nhe, t3nh2, c1d, c2d, gcon1, gcon2, xnfph1, xnfph2;
} orc_shdepth_t;

static void orc_shdepth(double xne, double t, double xnfph1, double xnfph2, double xnfhe1, double xnfh2,
                        orc_shdepth_t *d) {
  const double xne16 = pow(xne, 1.0 / 6.0);
  d->xne = xne;
  d->t = t;
  d->pp = xne16 * 0.08989 / sqrt(t);
  d->fo = orc_powi(xne16, 4) * 1.25e-9;
  d->y1b = 2.0 / (1.0 + 0.012 / t * sqrt(xne / t));
  const double t4 = t / 10000.0, t43 = pow(t4, 0.3);
  d->y1s = t43 / xne16;
  d->t3nhe = t43 * xnfhe1;
  d->t3nh2 = t43 * xnfh2;
  d->c1d = d->fo * 78940.0 / t;
  d->c2d = d->fo * d->fo / 5.96e-23 / xne;
  d->gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + xne / 1.0e13);
  d->gcon2 = 0.2 / (1.0 + xne / 1.0e15);
  d->xnfph1 = xnfph1;
  d->xnfph2 = xnfph2;
}

/* the line constants recomputed when N or M changes (:1254-1358) */
typedef struct {
  int n, m, ifins;
  double xknm, freqnm, dbeta, wavenm, c1con, c2con, radamp, resont, vdw, stark, y1num, y1wht;
  double finest[14], finswt[14];
} orc_shline_t;

static void orc_shline(const orc_htab_t *h, int n, int m, orc_shline_t *L) {
  const int mmn = m - n;
  const double xn = (double)n, xm = (double)m, xn2 = xn * xn, xm2 = xm * xm;
  const double xmn2 = xm2 * xn2, xm2mn2 = xm2 - xn2, gnm = xm2mn2 / xmn2;
  L->n = n;
  L->m = m;
  L->xknm = (mmn <= 3 && n <= 4) ? h->xknmtb[n - 1][mmn - 1] : 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / (double)mmn);
  L->y1num = m == 2 ? 550.0 : (m == 3 ? 380.0 : 320.0);
  L->y1wht = mmn <= 3 ? 1.0e14 : 1.0e13;
  if (mmn <= 2 && n <= 2) L->y1wht = h->y1wtm[n - 1][mmn - 1];
  L->freqnm = S_RYDBERG_H * S_CLIGHT * gnm;
  L->dbeta = S_CLIGHT_ANGS / (L->freqnm * L->freqnm) / L->xknm;
  L->wavenm = S_CLIGHT_ANGS / L->freqnm;
  L->c1con = L->xknm / L->wavenm * gnm * xm2mn2;
  L->c2con = orc_powi(L->xknm / L->wavenm, 2);
  double radamp = n == 1 ? h->asumlyman[m - 1] : h->asum[n - 1] + h->asum[m - 1];
  L->radamp = radamp / (4.0 * S_PI) / L->freqnm;
  double resont = orc_hfnm(1, m) / xm / (1.0 - 1.0 / xm2);
  if (n != 1) resont = resont + orc_hfnm(1, n) / xn / (1.0 - 1.0 / xn2);
  L->resont = resont * 3.579e-24 / gnm;
  L->vdw = 4.45e-26 / gnm * pow(xm2 * (7.0 * xm2 + 5.0), 0.4);
  L->stark = 1.6678e-18 * L->freqnm * L->xknm;
  if (n > 4 || m > 10) {
    L->ifins = 1;
    L->finest[0] = 0.0;
    L->finswt[0] = 1.0;
  } else if (mmn == 1) {
    L->ifins = h->lnghal[n - 1];
    const int ipos = h->istal[n - 1];
    for (int i = 0; i < L->ifins; ++i) {
      L->finest[i] = h->stalph[ipos - 1 + i] * 1.0e7;
      L->finswt[i] = h->stwtal[ipos - 1 + i] / xn2 / 3.0;
    }
  } else {
    L->ifins = h->lncomp[n - 1];
    for (int i = 0; i < L->ifins; ++i) {
      L->finest[i] = h->stcomp[i][n - 1] * 1.0e7;
      L->finswt[i] = h->stcpwt[i][n - 1] / xn2;
    }
  }
}

/* the Peterson/Kurucz analytic profile (:1698-1892): Doppler, Lorentz and
 * Stark blocks, only the widest inside the core */
static double orc_shprof_kp(const orc_htab_t *h, const orc_shline_t *L, const orc_shdepth_t *d, double hwdop,
                            double delw) {
  const double FREQ_RYDH = S_RYDBERG_H * S_CLIGHT, c4 = (double)(float)2.99792458e10;
  const int n = L->n, m = L->m;
  const double freqnm = L->freqnm;
  const double freq = S_CLIGHT_ANGS / (L->wavenm + delw * 10.0);
  const double del = fabs(freq - freqnm);
  const double hwstk = L->stark * d->fo;
  const double hwvdw = L->vdw * d->t3nhe + 2.0 * L->vdw * d->t3nh2;
  const double hwrad = L->radamp;
  const double hwres = L->resont * d->xnfph1 * 2.0;
  double hwlor = hwres + hwvdw + hwrad;
  const double dop = freqnm * hwdop;
  int nwid = 1;
  if (hwdop < hwstk || hwdop < hwlor) {
    nwid = 2;
    if (hwlor < hwstk) nwid = 3;
  }
  double mx = hwdop > hwlor ? hwdop : hwlor;
  if (hwstk > mx) mx = hwstk;
  const int ifcore = del <= freqnm * mx;
  double result = 0.0;
  if (!ifcore || nwid == 1) {
    for (int i = 0; i < L->ifins; ++i) {
      const double dd = fabs(freq - freqnm - L->finest[i]) / dop;
      if (dd <= 7.0) result = result + exp(-dd * dd) * L->finswt[i];
    }
    if (ifcore) return result;
  }
  if (!ifcore || nwid == 2) {
    if (n == 1 && m == 2) {
      const double hwres4 = hwres * 4.0;
      hwlor = hwres4 + hwvdw + hwrad;
      const double hhw = freqnm * hwlor;
      double hprofres;
      if (freq > s_lya_freq(4000.0f))
        hprofres = hwres4 * freqnm / S_PI / (del * del + hhw * hhw) * SQRTPI * dop;
      else
        hprofres = s_lya_h2_blue(h, freq, d->xnfph1) * SQRTPI * dop;
      double hprofrad = 0.0;
      if (freq > (double)2.4190611e15f && freq < (double)0.77f * FREQ_RYDH)
        hprofrad = hwrad * freqnm / S_PI / (del * del + hhw * hhw) * SQRTPI * dop;
      double hprofvdw = hwvdw * freqnm / S_PI / (del * del + hhw * hhw) * SQRTPI * dop;
      if (freq < (double)1.8e15f) hprofvdw = 0.0;
      result = result + hprofres + hprofrad + hprofvdw;
    } else {
      const double hhw = freqnm * hwlor;
      double top = hhw;
      if (n == 1 && m <= 5) {
        if (m == 3 && freq > (double)0.885f * FREQ_RYDH && freq < (double)0.890f * FREQ_RYDH) top = hhw - freqnm * hwrad;
        if (m == 4 && freq > (double)0.936f * FREQ_RYDH && freq < (double)0.938f * FREQ_RYDH) top = hhw - freqnm * hwrad;
        if (m == 5 && freq > (double)0.959f * FREQ_RYDH && freq < (double)0.961f * FREQ_RYDH) top = hhw - freqnm * hwrad;
      }
      result = result + top / S_PI / (del * del + hhw * hhw) * SQRTPI * dop;
    }
    if (ifcore) return result;
  }
  const double wty1 = 1.0 / (1.0 + d->xne / L->y1wht);
  const double y1scal = L->y1num * d->y1s * wty1 + d->y1b * (1.0 - wty1);
  const double c1 = d->c1d * L->c1con * y1scal, c2 = d->c2d * L->c2con;
  const double g1 = 6.77 * sqrt(c1);
  double lg = 0.2114 + log(sqrt(c2) / c1);
  if (lg < 0.0) lg = 0.0;
  const double gnot = g1 * lg * (1.0 - d->gcon1 - d->gcon2);
  const double beta = fabs(del) / d->fo * L->dbeta;
  const double y1 = c1 * beta, y2 = c2 * (beta * beta);
  double gam = gnot;
  if (!(y2 <= 1.0e-4 && y1 <= 1.0e-5)) {
    gam = g1 * (0.5 * exp(-(y1 < 80.0 ? y1 : 80.0)) + s_expint1(y1) - 0.5 * s_expint1(y2)) *
          (1.0 - d->gcon1 / (1.0 + orc_powi(90.0 * y1, 3)) - d->gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1.0e-20) gam = 0.0;
  }
  double prqs = orc_stark_profile(h, beta, d->pp, n, m);
  if (m == 2) {
    prqs = prqs * 0.5;
    if (freq >= s_lya_freq(20000.0f) && freq <= s_lya_freq(4000.0f)) {
      result = result + s_lya_h2plus_red(h, freq, d->xnfph2) * SQRTPI * dop;
    } else if (freq > s_lya_freq(4000.0f)) {
      const double beta4000 = 4000.0 * c4 / d->fo * L->dbeta;
      const double prqsp4000 = orc_stark_profile(h, beta4000, d->pp, n, m) * 0.5 / d->fo * L->dbeta;
      const double cutoff4000 = pow(10.0, -11.07 - 14.0) / c4 * d->xnfph2;
      result = result + cutoff4000 / prqsp4000 * prqs / d->fo * L->dbeta * SQRTPI * dop;
    }
  }
  const double f = gam > 0.0 ? gam / S_PI / (gam * gam + beta * beta) : 0.0;
  const double p1 = orc_powi(0.9 * y1, 2);
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  return result + (prqs * (1.0 + fns) + f) / d->fo * L->dbeta * SQRTPI * dop;
}

double orc_synthe_hprof_kp(const orc_htab_t *h, int n, int m, double xne, double t, double xnfph1,
                           double xnfph2, double xnfhe1, double xnfh2, double dopph, double delw) {
  orc_shline_t L;
  orc_shdepth_t d;
  orc_shline(h, n, m, &L);
  orc_shdepth(xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, &d);
  return orc_shprof_kp(h, &L, &d, dopph, delw);
}

/* the Stehle-path convolution the reference keeps between calls (SAVE'd
 * CONV_* variables): rebuilt when N, M or J differ from the last build or
 * the line constants were recomputed since (another N, M called between) */
typedef struct {
  int valid, n, m, last_n, last_m;
  double F0, lambda0, dop_dalpha, voigt_a;
  double prof[60];
} orc_sconv_t;

/* interp_stark_at (:2007-2037): log-log interpolation of the Stark profile */
static double s_interp_stark(const orc_stehle_t *S, const double *sp, double da) {
  if (da >= pow(10.0, S->log_dalpha_grid[59])) return sp[59];
  const double lda = log10(da);
  int idx;
  for (idx = 1; idx <= 59; ++idx)
    if (lda <= S->log_dalpha_grid[idx]) break;
  if (idx > 59) idx = 59;
  const double frac = (lda - S->log_dalpha_grid[idx - 1]) / (S->log_dalpha_grid[idx] - S->log_dalpha_grid[idx - 1]);
  if (sp[idx - 1] > 0.0 && sp[idx] > 0.0) return exp(log(sp[idx - 1]) * (1.0 - frac) + log(sp[idx]) * frac);
  return sp[idx - 1] * (1.0 - frac) + sp[idx] * frac;
}

/* the Stark (x) Voigt convolution on the 60-point Delta-alpha grid
 * (:1427-1640): the table bilinear in (log Ne, T), Ne capped at the
 * transition's Inglis-Teller density; the kernel on a symmetric grid of the
 * log points below sigma/3 spacing plus up to 200 wing points at sigma/3 */
static void orc_sconv_build(const orc_stehle_t *S, const orc_shline_t *L, const orc_shdepth_t *d, double hwdop,
                            double hwlor_conv, orc_sconv_t *c) {
  enum { NA = 60, NT = 10, NCONV = 600, NWING = 200 };
  const int n = L->n, m = L->m;
  const double xn8 = (double)n, xm8 = (double)m;
  const double lambda0 = 1.0e8 / S_RYDBERG_H * orc_powi(xn8 * xm8, 2) / ((xm8 - xn8) * (xm8 + xn8));
  const int itrans = m - S->n_upper_min + 1, nd = S->n_dens;
  const double dcap = S->density_grid[S->max_dens_idx[itrans - 1] - 1];
  const double ne_cap = d->xne < dcap ? d->xne : dcap;
  const double F0 = 1.25e-9 * pow(ne_cap, 2.0 / 3.0);
  double dag[NA], sp[NA];
  for (int ia = 0; ia < NA; ++ia) dag[ia] = pow(10.0, S->log_dalpha_grid[ia]);
  int id1;
  for (id1 = 1; id1 <= nd - 1; ++id1)
    if (ne_cap <= S->density_grid[id1]) break;
  if (id1 > nd - 1) id1 = nd - 1;
  if (id1 < 1) id1 = 1;
  const int id2 = id1 + 1;
  double fd = (log10(ne_cap) - log10(S->density_grid[id1 - 1])) /
              (log10(S->density_grid[id2 - 1]) - log10(S->density_grid[id1 - 1]));
  fd = fd < 0.0 ? 0.0 : (fd > 1.0 ? 1.0 : fd);
  int it1;
  for (it1 = 1; it1 <= NT - 1; ++it1)
    if (d->t <= S->temp_grid[it1]) break;
  if (it1 > NT - 1) it1 = NT - 1;
  const int it2 = it1 + 1;
  double ft = (d->t - S->temp_grid[it1 - 1]) / (S->temp_grid[it2 - 1] - S->temp_grid[it1 - 1]);
  ft = ft < 0.0 ? 0.0 : (ft > 1.0 ? 1.0 : ft);
  const double *P = S->profiles + (size_t)(itrans - 1) * nd * NT * NA;
#define SP_AT(ia, it, id) P[((size_t)((id) - 1) * NT + (it) - 1) * NA + (ia)]
  for (int ia = 0; ia < NA; ++ia) {
    const double v00 = SP_AT(ia, it1, id1), v01 = SP_AT(ia, it2, id1);
    const double v10 = SP_AT(ia, it1, id2), v11 = SP_AT(ia, it2, id2);
    if (v00 > 0 && v01 > 0 && v10 > 0 && v11 > 0)
      sp[ia] = exp(log(v00) * (1 - fd) * (1 - ft) + log(v01) * (1 - fd) * ft + log(v10) * fd * (1 - ft) +
                   log(v11) * fd * ft);
    else
      sp[ia] = v00 * (1 - fd) * (1 - ft) + v01 * (1 - fd) * ft + v10 * fd * (1 - ft) + v11 * fd * ft;
  }
#undef SP_AT
  const double dop_dalpha = lambda0 * lambda0 / S_CLIGHT_ANGS * L->freqnm * hwdop / F0;
  const double lor_dalpha = lambda0 * lambda0 / S_CLIGHT_ANGS * L->freqnm * hwlor_conv / F0;
  const double voigt_a = (double)(float)(lor_dalpha / dop_dalpha);
  const double dx_wing = dop_dalpha / 3.0;
  const double d_log = (S->log_dalpha_grid[NA - 1] - S->log_dalpha_grid[0]) / (double)(NA - 1);
  int n_log = NA;
  for (int ia = 1; ia <= NA; ++ia)
    if (dag[ia - 1] * d_log * log(10.0) > dx_wing) {
      n_log = ia - 1;
      break;
    }
  if (n_log < 1) n_log = 1;
  const double da_trans = dag[n_log - 1];
  int n_wing = NWING;
  double da_wing_max = da_trans + (double)n_wing * dx_wing;
  if (da_wing_max > dag[NA - 1]) {
    da_wing_max = dag[NA - 1];
    n_wing = (int)((da_wing_max - da_trans) / dx_wing);
    if (n_wing < 0) n_wing = 0;
  }
  if (2 * n_wing + 2 * n_log + 1 > NCONV) {
    n_wing = (NCONV - 2 * n_log - 1) / 2;
    da_wing_max = da_trans + (double)n_wing * dx_wing;
  }
  double cda[NCONV], cpa[NCONV], cst[NCONV];
  int ic = 0;
  for (int iw = n_wing; iw >= 1; --iw) {
    const double da = da_trans + (double)iw * dx_wing;
    cda[ic] = -da;
    cpa[ic++] = s_interp_stark(S, sp, da);
  }
  for (int ia = n_log; ia >= 1; --ia) {
    cda[ic] = -dag[ia - 1];
    cpa[ic++] = sp[ia - 1];
  }
  cda[ic] = 0.0;
  cpa[ic++] = sp[0];
  for (int ia = 1; ia <= n_log; ++ia) {
    cda[ic] = dag[ia - 1];
    cpa[ic++] = sp[ia - 1];
  }
  for (int iw = 1; iw <= n_wing; ++iw) {
    const double da = da_trans + (double)iw * dx_wing;
    cda[ic] = da;
    cpa[ic++] = s_interp_stark(S, sp, da);
  }
  cst[0] = cda[1] - cda[0];
  cst[ic - 1] = cda[ic - 1] - cda[ic - 2];
  for (int iw = 1; iw < ic - 1; ++iw) cst[iw] = 0.5 * (cda[iw + 1] - cda[iw - 1]);
  for (int ia = 0; ia < NA; ++ia) {
    const double da_i = dag[ia];
    if (da_i > da_wing_max && da_wing_max > 0.0) {
      c->prof[ia] = sp[ia] + voigt_a * dop_dalpha / (S_PI * (da_i * da_i));
    } else {
      double gsum = 0.0;
      for (int iw = 0; iw < ic; ++iw) {
        const float vv = (float)((da_i - cda[iw]) / dop_dalpha);
        const double kern = (double)(float)orc_voigt_weideman((double)vv, voigt_a);
        gsum = gsum + cpa[iw] * kern * cst[iw];
      }
      c->prof[ia] = gsum / (dop_dalpha * SQRTPI);
    }
  }
  c->F0 = F0;
  c->lambda0 = lambda0;
  c->dop_dalpha = dop_dalpha;
  c->voigt_a = voigt_a;
  c->n = n;
  c->m = m;
  c->valid = 1;
}

static int s_use_stehle(const orc_stehle_t *st, int n, int m, double xne) {
  if (!st || n < 1 || n > 4) return 0;
  const orc_stehle_t *S = st + (n - 1);
  return S->n_dens > 0 && m >= S->n_upper_min && m <= S->n_upper_max && xne <= S->density_grid[S->n_dens - 1];
}

/* hydrogen_line_profile(N, M, J, DELW) with its call-to-call state */
static double orc_shprof(const orc_htab_t *h, const orc_stehle_t *st, orc_sconv_t *cv, const orc_shline_t *L,
                         const orc_shdepth_t *d, double hwdop, double delw) {
  const int n = L->n, m = L->m;
  if (n != cv->last_n || m != cv->last_m) {
    cv->last_n = n;
    cv->last_m = m;
    cv->valid = 0;
  }
  if (!s_use_stehle(st, n, m, d->xne)) return orc_shprof_kp(h, L, d, hwdop, delw);
  const orc_stehle_t *S = st + (n - 1);
  const double freq = S_CLIGHT_ANGS / (L->wavenm + delw * 10.0);
  const double del = fabs(freq - L->freqnm);
  const double hwvdw = L->vdw * d->t3nhe + 2.0 * L->vdw * d->t3nh2;
  const double hwres = L->resont * d->xnfph1 * 2.0;
  const double hwlor = hwres + hwvdw + L->radamp;
  const double dop = L->freqnm * hwdop;
  if (!cv->valid || cv->n != n || cv->m != m) {
    const double hwlor_conv = (n == 1 && m == 2) ? hwres * 4.0 + hwvdw + L->radamp : hwlor;
    orc_sconv_build(S, L, d, hwdop, hwlor_conv, cv);
  }
  const double dac = cv->lambda0 * cv->lambda0 / S_CLIGHT_ANGS * del / cv->F0;
  double I;
  if (dac <= pow(10.0, S->log_dalpha_grid[0])) {
    I = cv->prof[0];
  } else if (dac >= pow(10.0, S->log_dalpha_grid[59])) {
    I = S->k_alpha[m - S->n_upper_min] / pow(dac, 2.5) + cv->voigt_a * cv->dop_dalpha / (S_PI * (dac * dac));
  } else {
    const double lda = log10(dac);
    int ia1;
    for (ia1 = 1; ia1 <= 59; ++ia1)
      if (lda <= S->log_dalpha_grid[ia1]) break;
    if (ia1 > 59) ia1 = 59;
    const double fa = (lda - S->log_dalpha_grid[ia1 - 1]) / (S->log_dalpha_grid[ia1] - S->log_dalpha_grid[ia1 - 1]);
    const double p1 = cv->prof[ia1 - 1], p2 = cv->prof[ia1];
    I = (p1 > 0.0 && p2 > 0.0) ? exp(log(p1) * (1.0 - fa) + log(p2) * fa) : p1 * (1.0 - fa) + p2 * fa;
  }
  const double phi = I * (cv->lambda0 * cv->lambda0) / (S_CLIGHT_ANGS * cv->F0);
  double result = phi * SQRTPI * dop;
  if (n == 1 && m == 2) {
    if (freq <= s_lya_freq(4000.0f)) result = result + s_lya_h2_blue(h, freq, d->xnfph1) * SQRTPI * dop;
    if (freq >= s_lya_freq(20000.0f) && freq <= s_lya_freq(4000.0f))
      result = result + s_lya_h2plus_red(h, freq, d->xnfph2) * SQRTPI * dop;
    if (freq < (double)(50000.0f * (float)2.99792458e10)) result = 0.0;
  }
  return result;
}

double orc_synthe_hprof_stehle(const orc_htab_t *h, const orc_stehle_t *stehle, int n, int m, double xne,
                               double t, double xnfph1, double xnfph2, double xnfhe1, double xnfh2,
                               double dopph_conv, double dopph, double delw) {
  orc_shline_t L;
  orc_shdepth_t d;
  orc_sconv_t cv;
  orc_shline(h, n, m, &L);
  orc_shdepth(xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, &d);
  const orc_stehle_t *st = stehle;
  cv.valid = 0;
  cv.n = cv.m = cv.last_n = cv.last_m = 0;
  if (!s_use_stehle(st, n, m, xne)) return orc_shprof_kp(h, &L, &d, dopph, delw);
  orc_shprof(h, st, &cv, &L, &d, dopph_conv, delw); /* builds the convolution */
  return orc_shprof(h, st, &cv, &L, &d, dopph, delw);
}

int orc_synthe_hydrogen_opacity(const orc_nlte_line_t *recs, int64_t n, int length, int nrhox,
                                double wbegin, double ratio, double wlend, double velshift_kms,
                                const float *continuum, const double *xnfdop, const double *dopple,
                                int nspec, const double *xne, const double *hckt, const orc_htab_t *tab,
                                const orc_stehle_t *stehle, const orc_shatm_t *atm, double *out) {
  const double CUTOFF = LINE_CUTOFF, dopratio = 1.0 + velshift_kms / 299792.458;
  double ehyd[100], alphahyd[99];
  for (int k = 1; k <= 100; ++k)
    ehyd[k - 1] = k <= 10 ? tab->eh[k - 1] : tab->elim - S_RYDBERG_H / ((double)k * (double)k);
  for (int k = 1; k <= 99; ++k) alphahyd[k - 1] = 1.0e7 / (ehyd[k] - ehyd[k - 1]);
  for (int64_t i = 0; i < n; ++i) {
    const orc_nlte_line_t *r = recs + i;
    if (r->itype != -1 && r->itype != -2) continue;
    if (r->nblo < 1 || r->nblo > 99 || r->nbup <= r->nblo || r->nbup > 100 || r->ncon < 0 || r->ncon > 15)
      return -1;
  }
  for (int j = 0; j < nrhox; ++j) {
    const float inglis = (float)(1600.0 / pow(xne[j], (double)(2.0f / 15.0f)));
    const float nmerge = inglis - 1.5f;
    const double emergeh = S_RYDBERG_H / ((double)nmerge * (double)nmerge);
    const float *cont = continuum + (size_t)j * length;
    double *buf = out + (size_t)j * length;
    orc_shdepth_t d;
    orc_shdepth(xne[j], atm->t[j], atm->xnfph1[j], atm->xnfph2[j], atm->xnfhe1[j], atm->xnfh2[j], &d);
    orc_sconv_t cv;
    cv.valid = 0;
    cv.n = cv.m = cv.last_n = cv.last_m = 0;
    for (int64_t il = 0; il < n; ++il) {
      const orc_nlte_line_t *r = recs + il;
      if (r->itype != -1 && r->itype != -2) continue;
      const int nblo = r->nblo, nbup = r->nbup, ncon = r->ncon, nbuff = r->nbuff;
      const double wl = r->wlvac * dopratio;
      double kappa0 = (double)r->gf * xnfdop[(size_t)j * nspec];
      const int ick = nbuff < 1 ? 1 : (nbuff > length ? length : nbuff);
      double kapmin = (double)cont[ick - 1] * CUTOFF;
      if (nbup == 2) kapmin = (double)cont[length - 1] * CUTOFF;
      if (kappa0 < kapmin) continue;
      const double bolth = exp(-(double)r->elo * hckt[j]);
      float dopph = (float)dopple[(size_t)j * nspec];
      if (r->itype == -2) dopph = dopph / 1.4142f;
      kappa0 = kappa0 * bolth;
      if (kappa0 < kapmin) continue;
      orc_shline_t L;
      orc_shline(tab, nblo, nbup, &L);
#define HPROF(w) (kappa0 * orc_shprof(tab, stehle, &cv, &L, &d, (double)dopph, (w) - wl))
      const int minred = nbuff > 1 ? nbuff : 1;
      int blue = 1;
      double wcon = 0.0, wtail = 0.0;
      const int general = !(ncon == 0 || nbup == nblo + 1) && nbup != nblo + 2;
      if (!general && (ncon == 0 || nbup == nblo + 1)) {
        /* alpha / isolated line (:3483-3509) */
        if (wl <= wlend) {
          double wave = wbegin * orc_powi(ratio, minred - 1);
          for (int ib = minred; ib <= length; ++ib) {
            const double kappa = HPROF(wave);
            buf[ib - 1] += kappa;
            if (kappa < (double)cont[ib - 1] * CUTOFF) break;
            wave = wave * ratio;
          }
          if (minred == 1 || wl < wbegin) blue = 0;
        }
      } else if (!general) {
        /* beta line (:3511-3541): the red wing stops at the alpha line */
        if (wl <= wlend) {
          double wave = wbegin * orc_powi(ratio, minred - 1);
          int exited = 0;
          for (int ib = minred; ib <= length; ++ib) {
            if (wave > alphahyd[nblo - 1]) {
              exited = 1;
              break;
            }
            const double kappa = HPROF(wave);
            buf[ib - 1] += kappa;
            if (kappa < (double)cont[ib - 1] * CUTOFF) {
              exited = 1;
              break;
            }
            wave = wave * ratio;
          }
          if (!exited && (minred == 1 || wl < wbegin || nbuff < 1)) blue = 0;
        } else if (nbuff < 1) {
          blue = 0;
        }
      } else {
        /* higher series members with the merged-continuum taper
         * (:3543-3606, vacuum wavelengths) */
        const double wshift = 1.0e7 / (S_CONTH[ncon - 1] - S_RYDBERG_H / (81.0 * 81.0));
        double wmerge = 1.0e7 / (S_CONTH[ncon - 1] - emergeh);
        if (wmerge < 0.0) wmerge = wshift + wshift;
        wcon = wshift > wmerge ? wshift : wmerge;
        wtail = 1.0e7 / (1.0e7 / wcon - 500.0);
        if (wshift + wshift < wcon) wcon = wshift + wshift;
        if (wtail < 0.0) wtail = wcon + wcon;
        if (wcon + wcon < wtail) wtail = wcon + wcon;
        wcon = wcon * dopratio;
        if (wl <= wlend) {
          if (wcon > wlend) continue;
          if (wbegin <= alphahyd[nblo - 1]) {
            double wave = wbegin * orc_powi(ratio, minred - 1);
            if (wave >= wcon) {
              double kappa = HPROF(wave);
              if (kappa >= (double)cont[(minred < length ? minred : length) - 1] * CUTOFF) {
                if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
                if (minred <= length) buf[minred - 1] += kappa; /* the reference's BUFFER(MINRED) */
                wave = wave * ratio;
                for (int ib = minred + 1; ib <= length; ++ib) {
                  if (wave >= wcon) {
                    kappa = HPROF(wave);
                    if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
                    buf[ib - 1] += kappa;
                    if (kappa < (double)cont[ib - 1] * CUTOFF) break;
                  }
                  wave = wave * ratio;
                }
              }
            }
            if (minred == 1) continue;
          }
          if (wl < wbegin) continue;
        }
      }
      if (!blue) continue;
      int ib = nbuff < length + 1 ? nbuff : length + 1;
      const int maxblue = ib - 1;
      double wave = wbegin * orc_powi(ratio, ib - 1);
      for (int i = 1; i <= maxblue; ++i) {
        ib = ib - 1;
        wave = wave / ratio;
        if (general && wave < wcon) break;
        double kappa = HPROF(wave);
        if (general && wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
        buf[ib - 1] += kappa;
        if (kappa < (double)cont[ib - 1] * CUTOFF) break;
      }
#undef HPROF
    }
  }
  return 0;
}
