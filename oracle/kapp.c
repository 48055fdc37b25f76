/* kapp.c -- CPU oracle (test infrastructure) of KAPP's hydrogen continuum
 * sources: the checker of atlasgpu_atlas_kapp_hydrogen.  Never part of the
 * product; only tests/ load it.
 *
 * Restates, per frequency and depth, the reference's (src/atlas12_modules.f90):
 *   KAPP assembly        :11202-11324 (ACONT, SCONT, SIGMAC from the sources built here;
 *                                      helium, metals, H2 and the line sources are zero)
 *   HOP                  :11359-11608 (bound-free n = 1..15 with the cascade exit,
 *                                      n = 16..80, the dissolved-level pseudo-continuum,
 *                                      free-free)
 *   XKARZAS              :11635-11804 (REAL(4) Karzas-Latter interpolation)
 *   COULFF               :11995-12196 (van Hoof free-free Gaunt factor, bilinear in log)
 *   H2PLOP               :12224-12252
 *   HMINOP               :12360-12558 (with LINTER :5859-5880 and MAP1)
 *   HRAYOP               :12740-12906
 *   ELECOP               :17212-17222
 *   occupation_prob      :22549-22567, holtsmark_Q :22492-22519
 * Constants from mod_constants (:315-464).  The tables come from the
 * reference's data files and DATA statements (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stddef.h>

#include "oracle.h"

#define K_KBOL 1.380649e-16
#define K_HPLANCK 6.62607015e-27
#define K_CLIGHT 2.99792458e10
#define K_CLIGHT_NMS 2.99792458e17
#define K_EMASS 9.1093837139e-28
#define K_SIGMA_THOMSON 6.6524587051e-25
#define K_EV_ERG 1.602176634e-12
#define K_PI 3.141592653589793
#define K_LN10 2.30258509299405
#define K_COEFF_FF 3.69196e8
#define K_RYDBERG_H 109677.583403
#define K_ELIM_HI 109678.764
#define K_HMINUS_EA 0.75419
#define K_BETA_COEFF_HM88 8.798905203085208e+14
#define K_LOG_BETA_MIN (-2.0)
#define K_LOG_BETA_STEP 2.4825302042523617e-02

static const double H_SERIES_LIMITS[15] = {109678.764, 27419.659, 12186.462, 6854.871, 4387.113,
                                           3046.604,   2238.320,  1713.713,  1354.044, 1096.776,
                                           906.426,    761.650,   648.980,   559.579,  487.456};

/* derived PARAMETERs, evaluated in the source's order */
static double kbol_ev(void) { return K_KBOL / K_EV_ERG; }
static double hoverk(void) { return K_HPLANCK / K_KBOL; }
static double freq_rydh(void) { return K_RYDBERG_H * K_CLIGHT; }
static double theta_coeff(void) { return 0.4342944819032518 / kbol_ev(); }
static double bnu_prefac(void) { return 2.0 * K_HPLANCK / (K_CLIGHT * K_CLIGHT) * 1.0e45; }
static double saha_prefac(void) {
  return 2.0 * pow(2.0 * K_PI * K_EMASS * K_KBOL / (K_HPLANCK * K_HPLANCK), 1.5);
}

/* holtsmark_Q (:22492-22519) */
static double holtsmark_q(const orc_kapp_tables *tb, double beta) {
  if (beta <= 0.01) return 0.0;
  if (beta >= 50.0) return 1.0;
  const double lb = log10(beta);
  const double idx_f = (lb - K_LOG_BETA_MIN) / K_LOG_BETA_STEP;
  int idx = (int)idx_f;
  if (idx > 148) idx = 148;
  if (idx < 0) idx = 0;
  const double frac = idx_f - (double)idx;
  return tb->q_holtsmark[idx] + frac * (tb->q_holtsmark[idx + 1] - tb->q_holtsmark[idx]);
}

/* occupation_prob (:22549-22567); DBLE(n)**5 is exact for n <= 80 */
double orc_occupation_prob(const orc_kapp_tables *tb, int n, double xne) {
  if (n <= 1 || xne <= 0.0) return 1.0;
  const double dn = (double)n;
  const double n5 = dn * dn * dn * dn * dn;
  const double beta = K_BETA_COEFF_HM88 / (n5 * pow(xne, 2.0 / 3.0));
  return holtsmark_q(tb, beta);
}

/* XKARZAS (:11635-11804) in its REAL(4) arithmetic.  Tables column-major:
 * FREQN(29,15), XN(29,15), XL(29,6,6).  For n > 15 FREQN15(1) is never set
 * by the reference (it is read only above 1.5e19 Hz); it is formed here like
 * the other points. */
double orc_xkarzas(const orc_kapp_tables *tb, double freq, double zeff2, int n, int l) {
  enum { NPTS = 29, NMAX = 15, NLMAX = 6 };
  const float freqlg = (float)log10(freq / zeff2);
  float x;
  if (l >= n || n > NLMAX) {
    if (n > NMAX) {
      float fq[NPTS];
      const float rn = (float)n;
      const float rn2 = rn * rn;
      fq[NPTS - 1] = (float)log10(freq_rydh() / (double)rn2);
      if (freqlg < fq[NPTS - 1]) return 0.0;
      int i;
      for (i = 2; i <= NPTS - 1; ++i) {
        fq[i - 1] = (float)log10((double)(tb->ekarzas[i - 1] + 1.0f / rn2) * freq_rydh());
        if (freqlg > fq[i - 1]) break;
      }
      if (i > NPTS - 1) i = NPTS;
      if (i == 2) fq[0] = (float)log10((double)(tb->ekarzas[0] + 1.0f / rn2) * freq_rydh());
      const float *xn = tb->xn + (NMAX - 1) * NPTS;
      x = (freqlg - fq[i - 1]) / (fq[i - 2] - fq[i - 1]) * (xn[i - 2] - xn[i - 1]) + xn[i - 1];
    } else {
      const float *fn = tb->freqn + (n - 1) * NPTS, *xn = tb->xn + (n - 1) * NPTS;
      if (freqlg < fn[NPTS - 1]) return 0.0;
      int i;
      for (i = 2; i <= NPTS; ++i)
        if (freqlg > fn[i - 1]) break;
      if (i > NPTS) i = NPTS;
      x = (freqlg - fn[i - 1]) / (fn[i - 2] - fn[i - 1]) * (xn[i - 2] - xn[i - 1]) + xn[i - 1];
    }
  } else {
    const float *fn = tb->freqn + (n - 1) * NPTS;
    const float *xl = tb->xl + ((size_t)(n - 1) * NLMAX + l) * NPTS;
    if (freqlg < fn[NPTS - 1]) return 0.0;
    int i;
    for (i = 2; i <= NPTS; ++i)
      if (freqlg > fn[i - 1]) break;
    if (i > NPTS) i = NPTS;
    x = (freqlg - fn[i - 1]) / (fn[i - 2] - fn[i - 1]) * (xl[i - 2] - xl[i - 1]) + xl[i - 1];
  }
  return exp((double)x * K_LN10) / zeff2;
}

/* COULFF(J, 1) (:11995-12196): GFF_LOGTAB(81,146) column-major, log10 of the
 * tabulated g_ff as the reader stores it */
static double coulff_h(const orc_kapp_tables *tb, double freqlg, double tlog) {
  enum { NG = 81, NU = 146 };
  const double log10_ryh_over_k = log10(freq_rydh() * hoverk());
  const double log10_k_over_h = -log10(hoverk());
  const double lgam2 = 0.0 + log10_ryh_over_k - tlog / K_LN10;
  const double lu = (freqlg - tlog) / K_LN10 - log10_k_over_h;
  const double xi = (lgam2 - -6.0) / 0.2 + 1.0;
  const double xj = (lu - -16.0) / 0.2 + 1.0;
  int i0 = (int)xi, j0 = (int)xj;
  if (i0 > NG - 1) i0 = NG - 1;
  if (i0 < 1) i0 = 1;
  if (j0 > NU - 1) j0 = NU - 1;
  if (j0 < 1) j0 = 1;
  double fi = xi - (double)i0, fj = xj - (double)j0;
  fi = fmax(0.0, fmin(fi, 1.0));
  fj = fmax(0.0, fmin(fj, 1.0));
#define GT(I, J) tb->gff_logtab[(size_t)((J)-1) * NG + (I)-1]
  const double lg00 = GT(i0, j0), lg01 = GT(i0, j0 + 1), lg10 = GT(i0 + 1, j0), lg11 = GT(i0 + 1, j0 + 1);
#undef GT
  const double lg = (1.0 - fi) * ((1.0 - fj) * lg00 + fj * lg01) + fi * ((1.0 - fj) * lg10 + fj * lg11);
  return pow(10.0, lg);
}

/* LINTER (:5859-5880) */
static double linter(const double *xold, const double *yold, int nold, double xnew) {
  int i;
  for (i = 2; i <= nold; ++i)
    if (xnew < xold[i - 1]) break;
  if (i > nold) i = nold;
  return yold[i - 2] + (yold[i - 1] - yold[i - 2]) / (xold[i - 1] - xold[i - 2]) * (xnew - xold[i - 2]);
}

/* gfortran's REAL(8)**INTEGER (binary exponentiation, as libgcc's powi) */
static double ipow(double x, int m) {
  unsigned n = (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return y;
}

/* HRAYOP's cross-section (:12740-12906): Gavrila's Rayleigh factors */
static double hrayop_xsect(const orc_kapp_tables *tb, double freq) {
  const double fr = freq_rydh();
  const double d1 = 0.01 * fr, dab = 0.005 * fr, dbc = 0.002 * fr, dcd = 0.001 * fr;
  double g;
  int i;
  if (freq < d1) return K_SIGMA_THOMSON * ipow(tb->ray_m[0], 2) * ipow(freq / d1, 4);
  if (freq <= 0.74 * fr) {
    i = (int)(freq / d1);
    i = i + 1 < 74 ? i + 1 : 74;
    g = tb->ray_m[i - 2] + (tb->ray_m[i - 1] - tb->ray_m[i - 2]) / d1 * (freq - (double)(i - 1) * d1);
    return K_SIGMA_THOMSON * ipow(g, 2);
  }
  if (freq < 0.77 * fr) return 0.0;
  if (freq <= 0.885 * fr) {
    i = (int)((freq - 0.755 * fr) / dab) + 1;
    i = i + 1 < 27 ? i + 1 : 27;
    g = tb->ray_ab[i - 2] + (tb->ray_ab[i - 1] - tb->ray_ab[i - 2]) / dab *
                               (freq - (0.755 * fr + (double)(i - 1 - 1) * dab));
    return K_SIGMA_THOMSON * ipow(g, 2);
  }
  if (freq < 0.890 * fr) return 0.0;
  if (freq <= 0.936 * fr) {
    i = (int)((freq - 0.890 * fr) / dbc) + 1;
    i = i + 1 < 24 ? i + 1 : 24;
    g = tb->ray_bc[i - 2] + (tb->ray_bc[i - 1] - tb->ray_bc[i - 2]) / dbc *
                               (freq - (0.890 * fr + (double)(i - 1 - 1) * dbc));
    return K_SIGMA_THOMSON * ipow(g, 2);
  }
  if (freq < 0.938 * fr) return 0.0;
  if (freq <= 0.959 * fr) {
    i = (int)((freq - 0.938 * fr) / dcd) + 1;
    i = i + 1 < 22 ? i + 1 : 22;
    g = tb->ray_cd[i - 2] + (tb->ray_cd[i - 1] - tb->ray_cd[i - 2]) / dcd *
                               (freq - (0.938 * fr + (double)(i - 1 - 1) * dcd));
    return K_SIGMA_THOMSON * ipow(g, 2);
  }
  if (freq < 0.961 * fr) return 0.0;
  if (freq <= fr) return K_SIGMA_THOMSON * tb->ray_ly[0];
  const double xnew = freq / fr;
  double fnew;
  orc_map1(tb->ray_fly, tb->ray_ly, 64, &xnew, &fnew, 1);
  return K_SIGMA_THOMSON * fnew;
}

/* KAPP with its hydrogen, H-, H2+ and scattering sources at one frequency
 * (WAVE in nm), all depths.  out[q * nrhox + j] for q = ORC_KAPP_AHYD ..
 * ORC_KAPP_SIGMAC.  bhyd: BHYD(J, n) at [(n-1) * nrhox + j] (null: 1),
 * bmin: BMIN(J) (null: 1). */
void orc_kapp_hydrogen(const orc_kapp_tables *tb, double wave, int nrhox, const double *t, const double *xne,
                       const double *rho, const double *xnfp1, const double *xnfp2, const double *bhyd,
                       const double *bmin, double *out) {
  /* RUN_RT_PASS's per-frequency quantities (:3907-3917) */
  const double freq = K_CLIGHT_NMS / wave;
  const double waveno = 1.0e7 / wave;
  const double freqlg = log(freq);
  const double f3 = ipow(freq / 1.0e15, 3);
  const double fr = freq_rydh();
  /* XKARZAS of every level this frequency reaches (n = 1..80) */
  double xk[81];
  for (int n = 1; n <= 80; ++n) xk[n] = orc_xkarzas(tb, freq, 1.0, n, n);
  /* HMINOP's free-free table at this wavelength and its bound-free cross-section */
  double wfflog[22], fflog[11][22], fftt[11];
  for (int iw = 0; iw < 22; ++iw) {
    wfflog[iw] = log(91.134 / tb->hmin_wavek[iw]);
    for (int it = 0; it < 11; ++it) fflog[it][iw] = log(tb->hmin_ff[it + 11 * iw] * 1.0e-26);
  }
  const double wavelog = log(wave);
  for (int it = 0; it < 11; ++it)
    fftt[it] = exp(linter(wfflog, fflog[it], 22, wavelog)) / tb->hmin_thetaff[it] * theta_coeff() * K_KBOL;
  double hminbf = 0.0;
  if (freq > 1.82365e14) orc_map1(tb->hmin_wbf, tb->hmin_bf, 116, &wave, &hminbf, 1);
  /* H2PLOP's fit */
  const double *c = tb->h2p_fr, *e = tb->h2p_es;
  const double frh2 = c[0] + (c[1] + (c[2] + (c[3] + c[4] * freqlg) * freqlg) * freqlg) * freqlg;
  const double esh2 = e[0] + (e[1] + (e[2] + (e[3] + (e[4] + e[5] * freq) * freq) * freq) * freq) * freq;
  const double xray = hrayop_xsect(tb, freq);
  for (int j = 0; j < nrhox; ++j) {
    const double T = t[j];
    const double tk = K_KBOL * T;
    const double hkt = K_HPLANCK / tk, hckt = hkt * K_CLIGHT;
    const double tkev = kbol_ev() * T, tlog = log(T);
    const double ehvkt = exp(-freq * hkt);
    const double stim = 1.0 - ehvkt;
    const double bnu = bnu_prefac() * f3 * ehvkt / stim;
    double bh[6];
    for (int n = 0; n < 6; ++n) bh[n] = bhyd ? bhyd[(size_t)n * nrhox + j] : 1.0;
    const double bm = bmin ? bmin[j] : 1.0;
    /* HOP */
    double H = 0.0, S = 0.0, A;
    for (int n = 15; n >= 1; --n) {
      if (waveno < H_SERIES_LIMITS[n - 1]) break;
      if (n >= 7) {
        const double w = orc_occupation_prob(tb, n, xne[j]);
        A = w * xk[n] * (double)(2 * n * n) * exp(-tb->hop_elev[n - 1] * hckt) * stim;
        H = H + A;
        S = S + A * bnu;
      } else if (n >= 2) {
        A = xk[n] * (double)(2 * n * n) * exp(-tb->hop_elev[n - 1] * hckt) * (bh[n - 1] - ehvkt);
        H = H + A;
        S = S + A * bnu * stim / (bh[n - 1] - ehvkt);
      } else {
        A = xk[1] * 2.0 * 1.0 * (bh[0] - ehvkt);
        H = H + A;
        S = S + A * bnu * stim / (bh[0] - ehvkt);
      }
    }
    for (int n = 16; n <= 80; ++n) {
      const double dn2 = ipow((double)n, 2);
      if (waveno < K_ELIM_HI / dn2) continue;
      const double w = orc_occupation_prob(tb, n, xne[j]);
      if (w < 1.0e-6) continue;
      const double en = K_ELIM_HI - K_RYDBERG_H / dn2;
      A = w * xk[n] * 2.0 * dn2 * exp(-en * hckt) * stim;
      H = H + A;
      S = S + A * bnu;
    }
    const double freq3_inv = 1.0 / (freq * freq * freq);
    for (int n = 7; n <= 80; ++n) {
      const double w = orc_occupation_prob(tb, n, xne[j]);
      if (1.0 - w < 1.0e-6) continue;
      const double en = K_ELIM_HI - K_RYDBERG_H / ipow((double)n, 2);
      A = (1.0 - w) * 2.815e29 * freq3_inv * 2.0 / ipow((double)n, 3) * exp(-en * hckt) * stim;
      H = H + A;
      S = S + A * bnu;
    }
    H = H * xnfp1[j] / rho[j];
    S = S * xnfp1[j] / rho[j];
    A = K_COEFF_FF / sqrt(T) * coulff_h(tb, freqlg, tlog) / freq * xne[j] / freq * xnfp2[j] / freq * stim / rho[j];
    H = H + A;
    S = S + A * bnu;
    const double ahyd = H, shyd = H > 0.0 ? S / H : 0.0;
    /* H2PLOP */
    const double ah2p = freq > fr ? 0.0 : exp(-esh2 / tkev + frh2) * xnfp1[j] * 2.0 * bh[0] * xnfp2[j] / rho[j] * stim;
    /* HMINOP */
    const double theta = theta_coeff() / T;
    const double xhmin = exp(K_HMINUS_EA / tkev) / (saha_prefac() * T * sqrt(T)) * bm * bh[0] * xnfp1[j] * xne[j];
    const double ffth = linter(tb->hmin_thetaff, fftt, 11, theta);
    const double hminff = ffth * xnfp1[j] * 2.0 * bh[0] * xne[j] / rho[j];
    const double hbf = hminbf * 1.0e-18 * (1.0 - ehvkt / bm) * xhmin / rho[j];
    const double ahmin = hbf + hminff;
    const double shmin = (hbf * bnu * stim / (bm - ehvkt) + hminff * bnu) / ahmin;
    /* HRAYOP, ELECOP */
    const double sigh = xray * xnfp1[j] * 2.0 * bh[0] / rho[j];
    const double sigel = K_SIGMA_THOMSON * xne[j] / rho[j];
    /* KAPP's totals (:11300-11320); the sources not built here are zero */
    const double a = ah2p + 0.0 + 0.0 + 0.0 + 0.0 + 0.0 + 0.0;
    const double acont = a + ahyd + ahmin;
    double scont = bnu;
    if (acont > 0.0) scont = (a * bnu + ahyd * shyd + ahmin * shmin) / acont;
    const double sigmac = sigh + 0.0 + sigel + 0.0 + 0.0;
    const double q[ORC_KAPP_NOUT] = {ahyd, shyd, ah2p, ahmin, shmin, sigh, sigel, acont, scont, sigmac};
    for (int k = 0; k < ORC_KAPP_NOUT; ++k) out[(size_t)k * nrhox + j] = q[k];
  }
}

/* log10 by the C library, element by element (COULFF's reader stores
 * log10 of the tabulated g_ff) */
void orc_log10_array(const double *in, double *out, int n) {
  for (int i = 0; i < n; ++i) out[i] = log10(in[i]);
}
