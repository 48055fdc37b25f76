/* kapp.c -- CPU oracle (test infrastructure) of KAPP's hydrogen and helium
 * continuum sources: the checker of atlasgpu_atlas_kapp_hydrogen and
 * atlasgpu_atlas_kapp.  Never part of the product; only tests/ load it.
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
 *   HE1OP                :12939-13143 (with CROSSHE :13160-13236 and the 2s/2p fits
 *                                      HE12S1S, HE12S3S, HE12P1P, HE12P3P :13299-13545)
 *   HE2OP                :13569-13674
 *   HEMIOP               :13716-13833
 *   HERAOP               :13918-13941
 *   H2MINOP              :12611-12708
 *   H2COLLOP             :16371-16527
 *   H2RAOP               :17289-17338
 *   PARTFNH2             :22324-22418, EQUILH2 :22437-22469
 *   HLINOP               :17381-17503 (with STARK :17528-17659, STARK_MMM
 *                                      :17854-18106, hydrogen_f_value :17760-17829)
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
#define K_RYDBERG_HE 109722.277609
#define K_CLIGHT_ANGS 2.99792458e18
#define K_AMU 1.66053906892e-24

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

/* COULFF(J, NZ) (:11995-12196): GFF_LOGTAB(81,146) column-major, log10 of
 * the tabulated g_ff as the reader stores it; z2log = Z2LOG(NZ) */
static double coulff(const orc_kapp_tables *tb, double freqlg, double tlog, double z2log) {
  enum { NG = 81, NU = 146 };
  const double log10_ryh_over_k = log10(freq_rydh() * hoverk());
  const double log10_k_over_h = -log10(hoverk());
  const double lgam2 = z2log + log10_ryh_over_k - tlog / K_LN10;
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
    A = K_COEFF_FF / sqrt(T) * coulff(tb, freqlg, tlog, 0.0) / freq * xne[j] / freq * xnfp2[j] / freq * stim / rho[j];
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

/* ---- helium ---- */

/* CROSSHE (:13160-13236) */
double orc_crosshe(const orc_kapp_tables *tb, double freq) {
  if (freq < 5.945209e15) return 0.0;
  const double wave = K_CLIGHT_ANGS / freq;
  int i;
  if (wave > 50.0) {
    i = (int)(93.0 - (wave - 50.0) / 5.0);
    i = i < 2 ? 2 : (i > 92 ? 92 : i);
    return ((wave - (92 - i) * 5.0 - 50.0) / 5.0 * (tb->he_x505[i - 2] - tb->he_x505[i - 1]) + tb->he_x505[i - 1]) *
           1.e-18;
  } else if (wave > 20.0) {
    i = (int)(17.0 - (wave - 20.0) / 2.0);
    i = i < 2 ? 2 : (i > 16 ? 16 : i);
    return ((wave - (16 - i) * 2.0 - 20.0) / 2.0 * (tb->he_x50[i - 2] - tb->he_x50[i - 1]) + tb->he_x50[i - 1]) *
           1.e-18;
  } else if (wave > 10.0) {
    i = (int)(12.0 - (wave - 10.0) / 1.0);
    i = i < 2 ? 2 : (i > 11 ? 11 : i);
    return ((wave - (11 - i) * 1.0 - 10.0) / 1.0 * (tb->he_x20[i - 2] - tb->he_x20[i - 1]) + tb->he_x20[i - 1]) *
           1.e-18;
  }
  i = (int)(22.0 - wave / 0.5);
  i = i < 2 ? 2 : (i > 21 ? 21 : i);
  return ((wave - (21 - i) * 0.5) / 0.5 * (tb->he_x10[i - 2] - tb->he_x10[i - 1]) + tb->he_x10[i - 1]) * 1.e-18;
}

/* the log10-knot branch of HE12S1S, HE12S3S, HE12P1P, HE12P3P */
static double he_knots(const double *fk, const double *xk, double freq) {
  const double freqlg = log10(freq);
  int i;
  for (i = 2; i <= 16; ++i)
    if (freqlg > fk[i - 1]) break;
  if (i > 16) i = 16;
  const double x = (freqlg - fk[i - 1]) / (fk[i - 2] - fk[i - 1]) * (xk[i - 2] - xk[i - 1]) + xk[i - 1];
  return exp(x * K_LN10);
}

/* HE12S1S (:13299-13343) */
static double he12s1s(const orc_kapp_tables *tb, double freq) {
  if (freq < 32033.214 * K_CLIGHT) return 0.0;
  if (freq > 2.4 * K_RYDBERG_HE * K_CLIGHT) {
    const double wavno = freq / K_CLIGHT;
    const double ek = (wavno - 32033.214) / K_RYDBERG_HE;
    const double eps = 2.0 * (ek - 2.612316) / 0.00322;
    return 0.008175 * pow(484940.0 / wavno, 2.71) * 8.067e-18 * ipow(eps + 76.21, 2) / (1.0 + ipow(eps, 2));
  }
  return he_knots(tb->he2s1s_f, tb->he2s1s_x, freq);
}

/* HE12S3S (:13346-13390) */
static double he12s3s(const orc_kapp_tables *tb, double freq) {
  if (freq < 38454.691 * K_CLIGHT) return 0.0;
  if (freq > 2.4 * K_RYDBERG_HE * K_CLIGHT) {
    const double wavno = freq / K_CLIGHT;
    const double ek = (wavno - 38454.691) / K_RYDBERG_HE;
    const double eps = 2.0 * (ek - 2.47898) / 0.000780;
    return 0.01521 * pow(470310.0 / wavno, 3.12) * 8.067e-18 * ipow(eps - 122.4, 2) / (1.0 + ipow(eps, 2));
  }
  return he_knots(tb->he2s3s_f, tb->he2s3s_x, freq);
}

/* HE12P1P (:13393-13440) */
static double he12p1p(const orc_kapp_tables *tb, double freq) {
  if (freq < 27175.76 * K_CLIGHT) return 0.0;
  if (freq > 2.4 * K_RYDBERG_HE * K_CLIGHT) {
    const double wavno = freq / K_CLIGHT;
    const double ek = (wavno - 27175.76) / K_RYDBERG_HE;
    const double eps1s = 2.0 * (ek - 2.446534) / 0.01037;
    const double eps1d = 2.0 * (ek - 2.59427) / 0.00538;
    return 0.0009487 * pow(466750.0 / wavno, 3.69) * 8.067e-18 *
           (ipow(eps1s - 29.30, 2) / (1.0 + ipow(eps1s, 2)) + ipow(eps1d + 172.4, 2) / (1.0 + ipow(eps1d, 2)));
  }
  return he_knots(tb->he2p1p_f, tb->he2p1p_x, freq);
}

/* HE12P3P (:13443-13480) */
static double he12p3p(const orc_kapp_tables *tb, double freq) {
  if (freq < 29223.753 * K_CLIGHT) return 0.0;
  return he_knots(tb->he2p3p_f, tb->he2p3p_x, freq);
}

/* HE1OP (:12939-13143) at one frequency, all depths, into ahe1[] */
static void he1op(const orc_kapp_tables *tb, double freq, int nrhox, const double *t, const double *xne,
                  const double *rho, const double *xnfp3, const double *xnf4, double *ahe1) {
  const double ryd = K_RYDBERG_HE * K_CLIGHT;
  const double freq3 = ipow(freq, 3);
  const double cfree = K_COEFF_FF / freq3;
  const double c = 2.815e29 / freq3;
  int imin = 0;
  for (int n = 1; n <= 10; ++n)
    if (tb->he1_freq[n - 1] <= freq) {
      imin = n;
      break;
    }
  double trans[11] = {0};
  if (imin > 0 && imin <= 1) trans[1] = orc_crosshe(tb, freq);
  if (imin > 0 && imin <= 2) trans[2] = he12s3s(tb, freq);
  if (imin > 0 && imin <= 3) trans[3] = he12s1s(tb, freq);
  if (imin > 0 && imin <= 4) trans[4] = he12p3p(tb, freq);
  if (imin > 0 && imin <= 5) trans[5] = he12p1p(tb, freq);
  if (imin > 0 && imin <= 6) trans[6] = orc_xkarzas(tb, freq, 1.236439, 3, 0);
  if (imin > 0 && imin <= 7) trans[7] = orc_xkarzas(tb, freq, 1.102898, 3, 0);
  if (imin > 0 && imin <= 8) trans[8] = orc_xkarzas(tb, freq, 1.045499, 3, 1);
  if (imin > 0 && imin <= 9) trans[9] = orc_xkarzas(tb, freq, 1.001427, 3, 2);
  if (imin > 0 && imin <= 10) trans[10] = orc_xkarzas(tb, freq, 0.9926, 3, 1);
  if (imin >= 1) {
    /* inner shell to He II n = 2: 1s2p 1P, 1s2p 3P, 1s2s 1S, 1s2s 3S */
    double elim = 527490.06, fhe;
    fhe = (elim - 171135.000) * K_CLIGHT;
    if (freq >= fhe) {
      trans[5] = trans[5] + orc_xkarzas(tb, freq, fhe / ryd, 1, 0);
      fhe = (elim - 169087.0) * K_CLIGHT;
      if (freq >= fhe) {
        trans[4] = trans[4] + orc_xkarzas(tb, freq, fhe / ryd, 1, 0);
        fhe = (elim - 166277.546) * K_CLIGHT;
        if (freq >= fhe) {
          trans[3] = trans[3] + orc_xkarzas(tb, freq, fhe / ryd, 1, 0);
          fhe = (elim - 159856.069) * K_CLIGHT;
          if (freq >= fhe) trans[2] = trans[2] + orc_xkarzas(tb, freq, fhe / ryd, 1, 0);
        }
      }
    }
    /* inner shell to He II n = 3: levels 10, 9, 8, 7, 6 */
    elim = 588451.59;
    const double e3[5] = {186209.471, 186101.0, 185564.0, 184864.0, 183236.0};
    for (int k = 0; k < 5; ++k) {
      fhe = (elim - e3[k]) * K_CLIGHT;
      if (!(freq >= fhe)) break;
      trans[10 - k] = trans[10 - k] + orc_xkarzas(tb, freq, fhe / ryd, 1, 0);
    }
  }
  double transn[28] = {0};
  if (freq >= 1.25408e16)
    for (int n = 4; n <= 27; ++n) transn[n] = orc_xkarzas(tb, freq, 4.0 - 3.0 / ipow((double)n, 2), 1, 0);
  const double freqlg = log(freq);
  for (int j = 0; j < nrhox; ++j) {
    const double T = t[j], tkev = kbol_ev() * T, tlog = log(T);
    const double hkt = K_HPLANCK / (K_KBOL * T);
    const double ehvkt = exp(-freq * hkt), stim = 1.0 - ehvkt;
    const double xr = xnfp3[j] * (4.0 / 2.0 / 13.595) * tkev / rho[j];
    const double boltex = exp(-23.730 / tkev) * xr;
    const double exlim = exp(-24.587 / tkev) * xr;
    const double freet = xne[j] * xnf4[j] / rho[j] / sqrt(T);
    double ex = boltex;
    if (freq < 2.055e14) ex = exlim / ehvkt;
    double he1 = (ex - exlim) * c;
    if (imin > 0)
      for (int n = imin; n <= 10; ++n) {
        const double bolt = exp(-tb->he1_chi[n - 1] / tkev) * tb->he1_g[n - 1] * xnfp3[j] / rho[j];
        he1 = he1 + trans[n] * bolt;
      }
    if (freq >= 1.25408e16)
      for (int n = 4; n <= 27; ++n) {
        const double boltn =
            exp(-24.587 * (1.0 - 1.0 / ipow((double)n, 2)) / tkev) * 4.0 * ipow((double)n, 2) * xnfp3[j] / rho[j];
        he1 = he1 + transn[n] * boltn;
      }
    ahe1[j] = (he1 + coulff(tb, freqlg, tlog, 0.0) * freet * cfree) * stim;
  }
}

/* HE2OP (:13569-13674) at one frequency, all depths (AHE2 only: KAPP weights
 * it by BNU, so SHE2 is not formed) */
static void he2op(const orc_kapp_tables *tb, double freq, double waveno, int nrhox, const double *t,
                  const double *xne, const double *rho, const double *xnfp4, const double *xnfp5, double *ahe2) {
  /* levels n = 9..1: threshold (cm^-1), X's denominator n^5, g = 2n^2, E_n (cm^-1), Gaunt fit (none for n >= 7) */
  static const double thr[9] = {5418.390, 6857.660, 8956.950, 12191.437, 17555.715,
                                27430.925, 48766.491, 109726.529, 438908.850};
  static const double g[9] = {162.0, 128.0, 98.0, 72.0, 50.0, 32.0, 18.0, 8.0, 2.0};
  static const double en[9] = {433490.46, 432051.19, 429951.90, 426717.413, 421353.135,
                               411477.925, 390142.359, 329182.321, 0.0};
  static const double ga[9] = {0, 0, 0, 1.0986, 1.102, 1.101, 1.101, 1.105, 0.9916};
  static const double gb[9] = {0, 0, 0, -2.704e13, -3.909e13, -5.765e13, -9.863e13, -2.375e14, 2.719e13};
  static const double gc[9] = {0, 0, 0, 1.229e27, 2.371e27, 4.593e27, 1.035e28, 4.077e28, -2.268e30};
  static const double den[9] = {59049.0, 32768.0, 16807.0, 7776.0, 3125.0, 1024.0, 243.0, 32.0, 1.0};
  const double freq3 = 2.815e29 / freq / freq / freq;
  const double freqlg = log(freq);
  for (int j = 0; j < nrhox; ++j) {
    const double T = t[j], tlog = log(T);
    const double hkt = K_HPLANCK / (K_KBOL * T), hckt = hkt * K_CLIGHT;
    const double stim = 1.0 - exp(-freq * hkt);
    const double xnfprho = xnfp4[j] / rho[j];
    double h = freq3 * 16.0 * 2.0 / 2.0 / (438889.068 * hckt) *
               (exp(-fmax(434519.959, 438908.85 - waveno) * hckt) - exp(-438908.85 * hckt)) * stim * xnfprho;
    for (int k = 0; k < 9; ++k) {
      if (waveno < thr[k]) break;
      double x;
      if (k == 0) x = freq3 / den[k] * 16.0;
      else if (k < 3) x = freq3 * 16.0 / den[k];
      else x = freq3 * 16.0 / den[k] * (ga[k] + (gb[k] + gc[k] / freq) / freq);
      const double a = k < 8 ? x * g[k] * exp(-en[k] * hckt) * stim * xnfprho : x * g[k] * stim * xnfprho;
      h = h + a;
    }
    const double a = K_COEFF_FF * 4.0 / sqrt(T) * coulff(tb, freqlg, tlog, 0.60206) / freq * xne[j] / freq *
                     xnfp5[j] / freq * stim / rho[j];
    ahe2[j] = h + a;
  }
}

/* HEMIOP (:13716-13833); wave in nm */
static void hemiop(const orc_kapp_tables *tb, double wave, int nrhox, const double *t, const double *xne,
                   const double *rho, const double *xnfp3, double *ahemin) {
  double logw[17], logt[12], kt[12];
  for (int i = 0; i < 17; ++i) logw[i] = log(tb->hem_w[i]);
  for (int i = 0; i < 12; ++i) logt[i] = log(tb->hem_t[i]);
  double wl = wave;
  if (wl > tb->hem_w[16]) wl = tb->hem_w[16];
  int iw = 1;
  for (int i = 1; i <= 16; ++i)
    if (wl >= tb->hem_w[i - 1]) iw = i;
  const double xw = (log(wl) - logw[iw - 1]) / (logw[iw] - logw[iw - 1]);
  for (int jt = 0; jt < 12; ++jt)
    kt[jt] = log(tb->hem_k[jt * 17 + iw - 1]) * (1.0 - xw) + log(tb->hem_k[jt * 17 + iw]) * xw;
  for (int j = 0; j < nrhox; ++j) {
    int it = 1;
    for (int i = 1; i <= 11; ++i)
      if (t[j] >= tb->hem_t[i - 1]) it = i;
    double xt = (log(fmax(t[j], 1.0)) - logt[it - 1]) / (logt[it] - logt[it - 1]);
    xt = fmax(0.0, fmin(1.0, xt));
    const double lkv = kt[it - 1] * (1.0 - xt) + kt[it] * xt;
    ahemin[j] = exp(lkv) * xne[j] * K_KBOL * t[j] * xnfp3[j] / rho[j];
  }
}

/* HERAOP (:13918-13941) */
static double heraop_sig(double freq) {
  const double w = K_CLIGHT_ANGS / fmin(freq, 5.15e15);
  const double ww = ipow(w, 2);
  return 5.484e-14 / ww / ww * ipow(1.0 + (2.44e5 + 5.94e10 / (ww - 2.90e5)) / ww, 2);
}

void orc_kapp(const orc_kapp_tables *tb, double wave, int nrhox, const double *t, const double *xne,
              const double *rho, const double *xnfp1, const double *xnfp2, const double *xnfp3,
              const double *xnfp4, const double *xnfp5, const double *xnf4, const double *bhyd, const double *bmin,
              double *out) {
  const double freq = K_CLIGHT_NMS / wave;
  const double waveno = 1.0e7 / wave;
  const double f3 = ipow(freq / 1.0e15, 3);
  double *ahe1 = out + (size_t)ORC_KAPP_AHE1 * nrhox, *ahe2 = out + (size_t)ORC_KAPP_AHE2 * nrhox;
  double *ahemin = out + (size_t)ORC_KAPP_AHEMIN * nrhox, *sighe = out + (size_t)ORC_KAPP_SIGHE * nrhox;
  orc_kapp_hydrogen(tb, wave, nrhox, t, xne, rho, xnfp1, xnfp2, bhyd, bmin, out);
  he1op(tb, freq, nrhox, t, xne, rho, xnfp3, xnf4, ahe1);
  he2op(tb, freq, waveno, nrhox, t, xne, rho, xnfp4, xnfp5, ahe2);
  hemiop(tb, wave, nrhox, t, xne, rho, xnfp3, ahemin);
  const double sig = heraop_sig(freq);
  for (int j = 0; j < nrhox; ++j) sighe[j] = sig * xnfp3[j] / rho[j];
  /* KAPP's totals (:11300-11320) again, with the helium sources */
  for (int j = 0; j < nrhox; ++j) {
    const double hkt = K_HPLANCK / (K_KBOL * t[j]);
    const double ehvkt = exp(-freq * hkt), stim = 1.0 - ehvkt;
    const double bnu = bnu_prefac() * f3 * ehvkt / stim;
    const double ahyd = out[(size_t)ORC_KAPP_AHYD * nrhox + j], shyd = out[(size_t)ORC_KAPP_SHYD * nrhox + j];
    const double ahmin = out[(size_t)ORC_KAPP_AHMIN * nrhox + j], shmin = out[(size_t)ORC_KAPP_SHMIN * nrhox + j];
    const double ah2p = out[(size_t)ORC_KAPP_AH2P * nrhox + j];
    const double a = ah2p + ahe1[j] + ahe2[j] + ahemin[j] + 0.0 + 0.0 + 0.0;
    const double acont = a + ahyd + ahmin;
    double scont = bnu;
    if (acont > 0.0) scont = (a * bnu + ahyd * shyd + ahmin * shmin) / acont;
    out[(size_t)ORC_KAPP_ACONT * nrhox + j] = acont;
    out[(size_t)ORC_KAPP_SCONT * nrhox + j] = scont;
    out[(size_t)ORC_KAPP_SIGMAC * nrhox + j] =
        out[(size_t)ORC_KAPP_SIGH * nrhox + j] + sighe[j] + out[(size_t)ORC_KAPP_SIGEL * nrhox + j] + 0.0 + 0.0;
  }
}

/* ---- H2 ---- */

/* PARTFNH2 (:22324-22418): natural cubic spline through the tabulated Q(T),
 * its second derivatives formed as the reader forms them */
double orc_partfnh2(const orc_kapp_h2_tables *h2, double t) {
  const int npf = h2->pf_n;
  const double *pf = h2->pf, tstart = h2->pf_tstart, tstep = h2->pf_tstep;
  double pf2[512], cwk[512];
  pf2[0] = 0.0;
  pf2[npf - 1] = 0.0;
  cwk[0] = 0.0;
  for (int n = 2; n <= npf - 1; ++n) {
    pf2[n - 1] = (6.0 * (pf[n] - 2.0 * pf[n - 1] + pf[n - 2]) / ipow(tstep, 2) - pf2[n - 2]) / (4.0 - cwk[n - 2]);
    cwk[n - 1] = 1.0 / (4.0 - cwk[n - 2]);
  }
  for (int n = npf - 1; n >= 2; --n) pf2[n - 1] = pf2[n - 1] - cwk[n - 1] * pf2[n];
  const double tt = fmin(tstart + (npf - 1) * tstep, fmax(tstart, t));
  int n = (int)((tt - tstart) / tstep) + 1;
  if (n > npf - 1) n = npf - 1;
  if (n < 1) n = 1;
  const double frac = (tt - (tstart + (n - 1) * tstep)) / tstep;
  return (1.0 - frac) * pf[n - 1] + frac * pf[n] + (ipow(1.0 - frac, 3) - (1.0 - frac)) * pf2[n - 1] * ipow(tstep, 2) / 6.0 +
         (ipow(frac, 3) - frac) * pf2[n] * ipow(tstep, 2) / 6.0;
}

/* EQUILH2 (:22437-22469): n(H2) / n(H I)^2 */
double orc_equilh2(const orc_kapp_h2_tables *h2, double t) {
  const double m_h = 1.008 * K_AMU;
  const double d0 = 36118.11 * (K_HPLANCK * K_CLIGHT / K_KBOL);
  const double pref = pow(2.0, 1.5) / 4.0 / pow(2.0 * K_PI * m_h * K_KBOL / (K_HPLANCK * K_HPLANCK), 1.5);
  return orc_partfnh2(h2, t) * pref / pow(t, 1.5) * exp(d0 / t);
}

void orc_kapp_h2(const orc_kapp_tables *tb, const orc_kapp_h2_tables *h2, double wave, int nrhox, const double *t,
                 const double *xne, const double *rho, const double *xnfp1, const double *xnfp2, const double *xnfp3,
                 const double *xnfp4, const double *xnfp5, const double *xnf4, const double *xnf3, const double *bhyd,
                 const double *bmin, double *out) {
  const double freq = K_CLIGHT_NMS / wave;
  const double waveno = 1.0e7 / wave;
  const double f3 = ipow(freq / 1.0e15, 3);
  orc_kapp(tb, wave, nrhox, t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4, bhyd, bmin, out);
  double *ah2min = out + (size_t)ORC_KAPP_AH2MIN * nrhox, *ah2coll = out + (size_t)ORC_KAPP_AH2COLL * nrhox;
  double *sigh2 = out + (size_t)ORC_KAPP_SIGH2 * nrhox;
  /* H2MINOP: log k at this wavelength for each tabulated temperature */
  double logw[10], logt[7], kt[7];
  for (int i = 0; i < 10; ++i) logw[i] = log(h2->h2m_w[i]);
  for (int i = 0; i < 7; ++i) logt[i] = log(h2->h2m_t[i]);
  double wl = wave;
  if (wl > h2->h2m_w[9]) wl = h2->h2m_w[9];
  int iw = 1;
  for (int i = 1; i <= 9; ++i)
    if (wl >= h2->h2m_w[i - 1]) iw = i;
  const double xw = (log(wl) - logw[iw - 1]) / (logw[iw] - logw[iw - 1]);
  for (int jt = 0; jt < 7; ++jt)
    kt[jt] = log(h2->h2m_k[jt * 10 + iw - 1]) * (1.0 - xw) + log(h2->h2m_k[jt * 10 + iw]) * xw;
  /* H2RAOP's cross-section */
  const double w = K_CLIGHT_ANGS / fmin(freq, 2.922e15);
  const double ww = ipow(w, 2);
  const double sig = (8.14e-13 + 1.28e-6 / ww + 1.61 / (ww * ww)) / (ww * ww);
  /* H2COLLOP's wavenumber bracket */
  const double numax = h2->cia_nu0 + h2->cia_dnu * (double)(h2->cia_nnu - 1);
  int cia = 0, inu = 1;
  double delnu = 0.0, dlow = 0.0;
  if (!(waveno > numax)) {
    if (waveno <= h2->cia_nu0) {
      if (waveno > 0.0) {
        cia = 1;
        dlow = 2.0 * log10(waveno / h2->cia_nu0);
      }
    } else {
      cia = 1;
      inu = (int)((waveno - h2->cia_nu0) / h2->cia_dnu) + 1;
      if (inu > h2->cia_nnu - 1) inu = h2->cia_nnu - 1;
      delnu = (waveno - h2->cia_nu0 - h2->cia_dnu * (double)(inu - 1)) / h2->cia_dnu;
    }
  }
  for (int j = 0; j < nrhox; ++j) {
    const double T = t[j];
    const double bh1 = bhyd ? bhyd[j] : 1.0;
    const double eq = orc_equilh2(h2, T);
    const double xnh2m = ipow(xnfp1[j] * 2.0 * bh1, 2) * eq;
    const double xnhi = xnfp1[j] * 2.0 * bh1;
    const double xnh2 = T <= 20000.0 ? ipow(xnhi, 2) * eq : 0.0;
    /* H2MINOP */
    int it = 1;
    for (int i = 1; i <= 6; ++i)
      if (T >= h2->h2m_t[i - 1]) it = i;
    double xt = (log(fmax(T, 1.0)) - logt[it - 1]) / (logt[it] - logt[it - 1]);
    xt = fmax(0.0, fmin(1.0, xt));
    ah2min[j] = exp(kt[it - 1] * (1.0 - xt) + kt[it] * xt) * xne[j] * K_KBOL * T * xnh2m / rho[j];
    /* H2COLLOP */
    const double den[4] = {xnh2 * xnh2, xnh2 * xnf3[j], xnh2 * xnhi, xnhi * xnf3[j]};
    double a = 0.0;
    if (cia)
      for (int ip = 0; ip < 4; ++ip) {
        if (!h2->use_pair[ip]) continue;
        const double *tp = h2->cia_temp + (size_t)ip * h2->cia_ntmax;
        const int nt = h2->cia_nt[ip];
        const double tcl = fmax(tp[0], fmin(tp[nt - 1], T));
        int ic = 1;
        for (int i = 1; i <= nt - 1; ++i)
          if (tcl >= tp[i - 1]) ic = i;
        const double wt = (tcl - tp[ic - 1]) / (tp[ic] - tp[ic - 1]);
        if (den[ip] <= 0.0) continue;
        const double *tab = h2->cia_tab + (size_t)ip * h2->cia_ntmax * h2->cia_nnu;
        const double c0 = tab[(size_t)(ic - 1) * h2->cia_nnu + inu - 1] * (1.0 - delnu) +
                          tab[(size_t)(ic - 1) * h2->cia_nnu + inu] * delnu + dlow;
        const double c1 = tab[(size_t)ic * h2->cia_nnu + inu - 1] * (1.0 - delnu) +
                          tab[(size_t)ic * h2->cia_nnu + inu] * delnu + dlow;
        a = a + pow(10.0, c0 * (1.0 - wt) + c1 * wt) * den[ip] / rho[j];
      }
    ah2coll[j] = a;
    sigh2[j] = sig * xnh2 / rho[j];
    /* KAPP's totals with the H2 sources */
    const double hkt = K_HPLANCK / (K_KBOL * T);
    const double ehvkt = exp(-freq * hkt), stim = 1.0 - ehvkt;
    const double bnu = bnu_prefac() * f3 * ehvkt / stim;
    const double ahyd = out[(size_t)ORC_KAPP_AHYD * nrhox + j], shyd = out[(size_t)ORC_KAPP_SHYD * nrhox + j];
    const double ahmin = out[(size_t)ORC_KAPP_AHMIN * nrhox + j], shmin = out[(size_t)ORC_KAPP_SHMIN * nrhox + j];
    const double av = out[(size_t)ORC_KAPP_AH2P * nrhox + j] + out[(size_t)ORC_KAPP_AHE1 * nrhox + j] +
                      out[(size_t)ORC_KAPP_AHE2 * nrhox + j] + out[(size_t)ORC_KAPP_AHEMIN * nrhox + j] + ah2min[j] +
                      ah2coll[j] + 0.0;
    const double acont = av + ahyd + ahmin;
    double scont = bnu;
    if (acont > 0.0) scont = (av * bnu + ahyd * shyd + ahmin * shmin) / acont;
    out[(size_t)ORC_KAPP_ACONT * nrhox + j] = acont;
    out[(size_t)ORC_KAPP_SCONT * nrhox + j] = scont;
    out[(size_t)ORC_KAPP_SIGMAC * nrhox + j] = out[(size_t)ORC_KAPP_SIGH * nrhox + j] +
                                               out[(size_t)ORC_KAPP_SIGHE * nrhox + j] +
                                               out[(size_t)ORC_KAPP_SIGEL * nrhox + j] + sigh2[j] + 0.0;
  }
}

/* ---- HLINOP ---- */

/* hydrogen_f_value (:17760-17829) */
static double hf_value(const orc_kapp_tables *tb, int n, int m) {
  if (m <= n) return 0.0;
  const double xn = n, xm = m;
  const int idx = m - n;
  double gf;
  if (n == 1 && idx <= 29) gf = tb->gf_lyman[idx - 1];
  else if (n == 2 && idx <= 28) gf = tb->gf_balmer[idx - 1];
  else if (n == 3 && idx <= 27) gf = tb->gf_paschen[idx - 1];
  else if (n == 4 && idx <= 3) gf = tb->gf_brackett[idx - 1];
  else {
    gf = 1.9603 * ipow(xn, 2) / (ipow(xm, 3) * ipow(1.0 / ipow(xn, 2) - 1.0 / ipow(xm, 2), 3));
    gf = gf * 0.80;
  }
  return gf / (2.0 * ipow(xn, 2));
}

static double exint(double x) {
  return -log(x) - 0.57516 + (0.97996 + (-0.21654 + (0.033572 + (-0.0029222 + 1.05439e-4 * x) * x) * x) * x) * x;
}

/* STARK (:17528-17659) at one depth */
static double stark(const orc_kapp_tables *tb, int n, int m, double freq, double t, double xne) {
  const double f0 = 1.25e-9 * pow(xne, 2.0 / 3.0);
  const double hkt = K_HPLANCK / (K_KBOL * t);
  const double xn = n, xm = m, x = xn / xm, xx = ipow(x, 2), nn = xn * xn, mm = xm * xm;
  const int mminn = m - n;
  double knm, fnm;
  if (mminn <= 5) knm = tb->stark_knm[(n - 1) * 5 + mminn - 1];
  else knm = 5.5e-5 * ipow(nn * mm, 2) / (mm - nn);
  if (mminn <= 10) fnm = tb->stark_f[(n - 1) * 10 + mminn - 1];
  else fnm = tb->stark_f[(n - 1) * 10 + 9] * ipow((20.0 * xn + 100.0) / ((xn + 10.0) * xm * (1.0 - xx)), 3);
  const double ryd = freq_rydh();
  const double freqnm = ryd * (1.0 / nn - 1.0 / mm);
  const double del = fabs(freq - freqnm);
  const double dbeta = K_CLIGHT_ANGS / ipow(freqnm, 2) / f0 / knm;
  const double beta = dbeta * del;
  const double y1 = mm * del * hkt / 2.0;
  const double y2 = (K_PI * K_PI / 2.0 / 0.0265384 / K_CLIGHT) * ipow(del, 2) / xne;
  const double qstat = 1.5 + 0.5 * (ipow(y1, 2) - 1.384) / (ipow(y1, 2) + 1.384);
  double impact = 0.0;
  if (y1 < 8.0 && y1 < y2) {
    const double exy2 = y2 <= 8.0 ? exint(y2) : 0.0;
    impact = 1.438 * sqrt(y1 * (1.0 - xx)) * (0.4 * exp(-y1) + exint(y1) - 0.5 * exy2);
  }
  double prof, ratio;
  if (beta <= 20.0) {
    prof = 8.0 / (80.0 + ipow(beta, 3));
    ratio = qstat + impact;
  } else {
    prof = 1.5 / beta / beta / sqrt(beta);
    const double dioi = 6.28 * 1.48e-25 * (2.0 * mm * ryd / del) * xne *
                        (sqrt(2.0 * mm * ryd / del) * (1.3 * qstat + 0.30 * impact) - 3.9 * ryd * hkt);
    ratio = qstat * fmin(1.0 + dioi, 1.25) + impact;
  }
  return 0.0265384 * fnm * prof * dbeta * ratio;
}

/* STARK_MMM (:17854-18106) */
double orc_stark_mmm(const orc_kapp_tables *tb, const orc_stehle_t *stehle, int n, int m, double freq, double t,
                     double xne) {
  if (n < 1 || n > 4 || m <= n || !stehle) return stark(tb, n, m, freq, t, xne);
  const orc_stehle_t *S = &stehle[n - 1];
  if (S->n_dens == 0 || m < S->n_upper_min || m > S->n_upper_max) return stark(tb, n, m, freq, t, xne);
  const int itrans = m - S->n_upper_min + 1;
  if (xne > S->density_grid[S->n_dens - 1]) return stark(tb, n, m, freq, t, xne);
  const double ne_eff = fmin(xne, S->density_grid[S->max_dens_idx[itrans - 1] - 1]);
  const double xn = n, xm = m;
  const double lambda0 = (1.0e8 / K_RYDBERG_H) * ipow(xn * xm, 2) / ((xm - xn) * (xm + xn));
  const double del_freq = fabs(freq - K_CLIGHT_ANGS / lambda0);
  const double f0 = 1.25e-9 * pow(ne_eff, 2.0 / 3.0);
  if (f0 <= 0.0) return stark(tb, n, m, freq, t, xne);
  const double dalpha = ipow(lambda0, 2) / K_CLIGHT_ANGS * del_freq / f0;
  const int nd = S->n_dens, nt = 10, na = 60;
  const double log_ne = log10(ne_eff);
  if (t < S->temp_grid[0] * 0.5 || t > S->temp_grid[nt - 1] * 2.0) return stark(tb, n, m, freq, t, xne);
  int id1;
  for (id1 = 1; id1 <= nd - 1; ++id1)
    if (ne_eff <= S->density_grid[id1]) break;
  if (id1 > nd - 1) id1 = nd - 1;
  const int id2 = id1 + 1;
  double frac_d =
      (log_ne - log10(S->density_grid[id1 - 1])) / (log10(S->density_grid[id2 - 1]) - log10(S->density_grid[id1 - 1]));
  frac_d = fmax(0.0, fmin(1.0, frac_d));
  int it1;
  for (it1 = 1; it1 <= nt - 1; ++it1)
    if (t <= S->temp_grid[it1]) break;
  if (it1 > nt - 1) it1 = nt - 1;
  const int it2 = it1 + 1;
  double frac_t = (log(t) - log(S->temp_grid[it1 - 1])) / (log(S->temp_grid[it2 - 1]) - log(S->temp_grid[it1 - 1]));
  frac_t = fmax(0.0, fmin(1.0, frac_t));
  int ia1 = 1, ia2 = 1;
  double frac_a = 0.0;
  if (dalpha > 0.0) {
    const double lda = log10(dalpha);
    if (lda >= S->log_dalpha_grid[na - 1]) {
      const double i_da = S->k_alpha[itrans - 1] / pow(dalpha, 2.5);
      return 0.0265384 * hf_value(tb, n, m) * i_da * ipow(lambda0, 2) / (K_CLIGHT_ANGS * f0);
    }
    if (lda > S->log_dalpha_grid[0]) {
      for (ia1 = 1; ia1 <= na - 1; ++ia1)
        if (lda <= S->log_dalpha_grid[ia1]) break;
      if (ia1 > na - 1) ia1 = na - 1;
      ia2 = ia1 + 1;
      frac_a = (lda - S->log_dalpha_grid[ia1 - 1]) / (S->log_dalpha_grid[ia2 - 1] - S->log_dalpha_grid[ia1 - 1]);
      frac_a = fmax(0.0, fmin(1.0, frac_a));
    }
  }
#define PV(IA, IT, ID) S->profiles[(((size_t)(itrans - 1) * nd + (ID)-1) * nt + (IT)-1) * na + (IA)-1]
  double v[8] = {PV(ia1, it1, id1), PV(ia2, it1, id1), PV(ia1, it2, id1), PV(ia2, it2, id1),
                 PV(ia1, it1, id2), PV(ia2, it1, id2), PV(ia1, it2, id2), PV(ia2, it2, id2)};
#undef PV
  int pos = 1;
  for (int k = 0; k < 8; ++k)
    if (v[k] <= 0.0) pos = 0;
  if (pos)
    for (int k = 0; k < 8; ++k) v[k] = log(v[k]);
  const double v00 = v[0] + frac_a * (v[1] - v[0]), v01 = v[2] + frac_a * (v[3] - v[2]);
  const double v10 = v[4] + frac_a * (v[5] - v[4]), v11 = v[6] + frac_a * (v[7] - v[6]);
  const double v0 = v00 + frac_t * (v01 - v00), v1 = v10 + frac_t * (v11 - v10);
  double i_da = pos ? exp(v0 + frac_d * (v1 - v0)) : v0 + frac_d * (v1 - v0);
  i_da = fmax(i_da, 0.0);
  return 0.0265384 * hf_value(tb, n, m) * i_da * ipow(lambda0, 2) / (K_CLIGHT_ANGS * f0);
}

void orc_hlinop(const orc_kapp_tables *tb, const orc_stehle_t *stehle, double wave, int nrhox, const double *t,
                const double *xne, const double *rho, const double *xnfp1, const double *bhyd, double *ahline,
                double *shline) {
  const double nu_lyman = freq_rydh();
  const double freq = K_CLIGHT_NMS / wave;
  const double f3 = ipow(freq / 1.0e15, 3);
  for (int j = 0; j < nrhox; ++j) ahline[j] = shline[j] = 0.0;
  const int n = (int)sqrt(nu_lyman / freq);
  if (n == 0 || n > 4) return;
  if (n == 1 && freq < 2.0e15) return;
  if (n == 2 && freq < 4.44e14) return;
  const double q = sqrt(nu_lyman / (nu_lyman / ipow((double)n, 2) - freq));
  const int mfreq = q < 1.0e6 ? (int)round(q) : 1000000; /* the series limit itself: past every level */
  for (int j = 0; j < nrhox; ++j) {
    const double T = t[j], tkev = kbol_ev() * T;
    const double ehvkt = exp(-freq * (K_HPLANCK / (K_KBOL * T))), stim = 1.0 - ehvkt;
    const double bnu = bnu_prefac() * f3 * ehvkt / stim;
#define BH(K) (bhyd ? bhyd[(size_t)((K)-1) * nrhox + j] : 1.0)
    double bolt[5];
    for (int k = 1; k <= 4; ++k)
      bolt[k] = exp(-(13.595 - 13.595 / ipow((double)k, 2)) / tkev) * 2.0 * ipow((double)k, 2) * BH(k) * xnfp1[j] / rho[j];
    int m1 = mfreq, m2 = m1 + 1;
    if (m1 < n + 1) m1 = n + 1;
    double h = 0.0, s = 0.0;
    if (m1 > 6) {
      if (m1 > 80 || orc_occupation_prob(tb, m1, xne[j]) < 1.0e-3) {
        ahline[j] = 0.0;
        shline[j] = bnu;
        continue;
      }
      m1 = m1 - 1;
      m2 = m2 + 3;
      if (n >= 4 && m1 <= 8) {
        h = orc_stark_mmm(tb, stehle, 3, 4, freq, T, xne[j]) * (1.0 - ehvkt * BH(4) / BH(3)) * bolt[3];
        s = h * bnu * stim / (BH(3) / BH(4) - ehvkt);
      }
    }
    for (int m = m1; m <= m2; ++m) {
      const double bm = m <= 6 ? BH(m) : 1.0;
      double w = 1.0;
      if (m >= 2 && m <= 80) w = orc_occupation_prob(tb, m, xne[j]);
      if (m > 80) w = 0.0;
      const double a = w * orc_stark_mmm(tb, stehle, n, m, freq, T, xne[j]) * (1.0 - ehvkt * bm / BH(n)) * bolt[n];
      h = h + a;
      s = s + a * bnu * stim / (BH(n) / bm - ehvkt);
    }
#undef BH
    ahline[j] = h;
    shline[j] = h > 0.0 ? s / h : bnu;
  }
}

/* log10 by the C library, element by element (COULFF's reader stores
 * log10 of the tabulated g_ff) */
void orc_log10_array(const double *in, double *out, int n) {
  for (int i = 0; i < n; ++i) out[i] = log10(in[i]);
}
