// kapp.cuh -- KAPP's hydrogen, helium and H2 continuum sources on the device (sm_100a).
//
// KAPP (atlas12_modules.f90:11202-11324) is called once per frequency inside
// RUN_RT_PASS's loop and evaluates every source at every depth.  Here the
// work is split by what it depends on:
//   k_kapp_depth  once per call, per depth: the temperature and density
//                 factors, the Hummer-Mihalas occupation probabilities w_n of
//                 n = 1..80 (occupation_prob :22549-22567, holtsmark_Q
//                 :22492-22519) and the level populations' Boltzmann factors
//                 exp(-E_n HCKT) -- none depends on the frequency
//   k_kapp_nu     warp per frequency: the per-frequency parts first (XKARZAS
//                 :11635-11804 for n = 1..80 in its REAL(4) arithmetic,
//                 HMINOP's free-free table at this wavelength and its
//                 bound-free cross-section, HRAYOP's and H2PLOP's factors),
//                 then lanes over depths: HOP (:11359-11608), H2PLOP
//                 (:12224-12252), HMINOP (:12360-12558), HRAYOP (:12740-12906),
//                 ELECOP (:17212-17222) and KAPP's totals; with helium
//                 populations also HE1OP (:12939-13143, its cross-sections
//                 per frequency on lanes), HE2OP (:13569-13674), HEMIOP
//                 (:13716-13833) and HERAOP (:13918-13941); with the H2
//                 tables also H2MINOP (:12611-12708), H2COLLOP (:16371-16527)
//                 and H2RAOP (:17289-17338), their H2 densities from
//                 EQUILH2 (:22437-22469) and PARTFNH2 (:22324-22418) per depth.
// Every output is the reference's expression in its order; where the
// reference evaluates a depth-only factor inside the frequency loop, the
// factor is the same function of the same inputs.
#pragma once
#include "common.cuh"
#include "tcorr.cuh"

namespace atlasgpu {

// mod_constants (atlas12_modules.f90:315-464)
constexpr double kKbol = 1.380649e-16;
constexpr double kEvErg = 1.602176634e-12;
constexpr double kEmass = 9.1093837139e-28;
constexpr double kSigmaThomson = 6.6524587051e-25;
constexpr double kLn10 = 2.30258509299405;
constexpr double kCoeffFF = 3.69196e8;
constexpr double kRydbergH = 109677.583403;
constexpr double kElimHI = 109678.764;
constexpr double kHminusEA = 0.75419;
constexpr double kBetaHM88 = 8.798905203085208e+14;
constexpr double kRydbergHe = 109722.277609;
constexpr double kClightAngs = 2.99792458e18;
constexpr double kAmu = 1.66053906892e-24;
constexpr double kRydAng = 1.0e8 / kRydbergH;  // RYD_ANG
constexpr double kA0Stark = 0.0265384;         // STARK's A0 = pi e^2 / (m_e c)
constexpr double kLogBetaMin = -2.0, kLogBetaStep = 2.4825302042523617e-02;
constexpr int kHLev = 80;  // HOP's NMAX_HLEVELS

// the tables on the device (set by atlasgpu_atlas_set_kapp_tables)
struct KappDev {
  float freqn[15 * 29], xn[15 * 29], xl[36 * 29], ekarzas[29];
  double gff_log[146 * 81];  // log10 g_ff, GFF_LOGTAB(I, J) at (J-1)*81 + I-1
  double q[150];
  double hop_elev[15];
  double wbf[116], bf[116], thetaff[11], wfflog[22], fflog[11 * 22];  // FFLOG(IWAVE, ITHETA) at it*22 + iw
  double h2p_fr[5], h2p_es[6];
  double ray_m[74], ray_ab[27], ray_bc[24], ray_cd[22], ray_ly[64], ray_fly[64];
  double series_limits[15];  // H_SERIES_LIMITS
  // helium: HE1OP's levels, CROSSHE, the 2s/2p fits (log10 knots), HEMIOP's
  // table and its logs (LOGK(IW, IT) at it*17 + iw)
  double he1_chi[10], he1_freq[10], he1_g[10];
  double he_x505[92], he_x50[16], he_x20[11], he_x10[21];
  double he2s1s_f[16], he2s1s_x[16], he2s3s_f[16], he2s3s_x[16];
  double he2p1p_f[16], he2p1p_x[16], he2p3p_f[16], he2p3p_x[16];
  double hem_w[17], hem_t[12], hem_logw[17], hem_logt[12], hem_logk[12 * 17];
  // HLINOP: hydrogen_f_value's gf tables, STARK's KNMTAB(MMINN, N) at
  // (N-1)*5 + MMINN-1 and FSTARK(MMINN, N) at (N-1)*10 + MMINN-1
  double gf_lyman[29], gf_balmer[28], gf_paschen[27], gf_brackett[3];
  double stark_knm[20], stark_f[40];
};

// the H2 tables on the device (set by atlasgpu_atlas_set_kapp_h2_tables):
// H2MINOP's table and logs (LOGK(IW, IT) at it*10 + iw), PARTFNH2's values
// and spline second derivatives, H2COLLOP's CIA grid (pf, pf2, cia_temp,
// cia_tab point into the same allocation), EQUILH2's two constants
struct KappH2Dev {
  double h2m_w[10], h2m_t[7], h2m_logw[10], h2m_logt[7], h2m_logk[7 * 10];
  int pf_n, cia_nnu, cia_ntmax, cia_nt[4], use_pair[4];
  double pf_tstart, pf_tstep, cia_nu0, cia_dnu, cia_numax;
  double equil_pref, equil_d0;  // EQUILH2's trans_prefactor and D0_over_kT_coeff
  const double *pf, *pf2, *cia_temp, *cia_tab;
};

// per-depth factors (k_kapp_depth), each [kw]; w, bz: [kHLev][kw] (level n at
// (n-1)*kw), bp: [9][kw] for the pseudo-continuum's n = 7..15; HE1OP's BOLT
// [10][kw], BOLTN of n = 4..27 [24][kw], FREET, BOLTEX, EXLIM (helium only);
// H2MINOP's XNH2M, XNH2, H2COLLOP's CIADEN, CIAIT (as doubles), CIAWT [4][kw]
// each (H2 only)
struct KappDepth {
  double *hkt, *hckt, *tkev, *tlog, *theta, *xhmin;
  double *w, *bz, *bp;
  double *he_bolt, *he_boltn, *he_freet, *he_boltex, *he_exlim;
  double *xnh2m, *xnh2, *ciaden, *ciait, *ciawt;
};

struct KappArgs {
  const KappDev* tb;
  int numnu, nrhox, kw;
  const double* waveset;
  const double *t, *xne, *rho, *xnfp1, *xnfp2, *bhyd, *bmin;  // bhyd [6][kw], bmin [kw]; may be null
  const double *xnfp3, *xnfp4, *xnfp5, *xnf4;  // helium populations; xnfp3 null: no helium sources
  const double* xnf3;                           // XNF(J,3); null: no H2 sources
  const KappH2Dev* h2;
  KappDepth d;
  double *acont, *sigmac, *scont;  // [numnu][kw]
  double* parts;                   // [numnu][nparts][kw] or null
  int nparts;                      // 7 (hydrogen), 11 (with helium) or 14 (with H2)
  double *ahline, *shline;         // HLINOP's outputs [numnu][kw] (k_hlinop)
  const StehleDev* stehle;         // [4] or null: STARK throughout
};

__host__ __device__ inline double kapp_kbol_ev() { return kKbol / kEvErg; }
__host__ __device__ inline double kapp_freq_rydh() { return kRydbergH * kClight; }
__host__ __device__ inline double kapp_hoverk() { return kHplanck / kKbol; }

// holtsmark_Q and occupation_prob; DBLE(n)**5 is exact for n <= 80
__device__ inline double kapp_occupation(const KappDev& tb, int n, double xne, double xne23) {
  if (n <= 1 || xne <= 0.0) return 1.0;
  const double dn = (double)n;
  const double beta = kBetaHM88 / (dn * dn * dn * dn * dn * xne23);
  if (beta <= 0.01) return 0.0;
  if (beta >= 50.0) return 1.0;
  const double idx_f = (log10(beta) - kLogBetaMin) / kLogBetaStep;
  int idx = (int)idx_f;
  idx = idx > 148 ? 148 : (idx < 0 ? 0 : idx);
  const double frac = idx_f - (double)idx;
  return tb.q[idx] + frac * (tb.q[idx + 1] - tb.q[idx]);
}

// XKARZAS(FREQ, ZEFF2, N, L): the Karzas-Latter cross-section, level-averaged
// (L >= N or N > 6) or l-resolved, the interpolation in REAL(4) with every
// operation rounded as written (no contraction)
__device__ inline double kapp_xkarzas(const KappDev& tb, double freq, double zeff2, int n, int l) {
  constexpr int NPTS = 29, NMAX = 15, NLMAX = 6;
  const float fl = __double2float_rn(log10(freq / zeff2));
  float x;
  if (l >= n || n > NLMAX) {
    if (n > NMAX) {
      const float rn = (float)n;
      const float rn2 = __fmul_rn(rn, rn);
      const float flast = __double2float_rn(log10(kapp_freq_rydh() / (double)rn2));
      if (fl < flast) return 0.0;
      const float r = __fdiv_rn(1.0f, rn2);
      float fprev = 0.0f, fcur = flast;
      int i;
      for (i = 2; i <= NPTS - 1; ++i) {
        fcur = __double2float_rn(log10((double)__fadd_rn(tb.ekarzas[i - 1], r) * kapp_freq_rydh()));
        if (fl > fcur) break;
      }
      if (i > NPTS - 1) {
        i = NPTS;
        fprev = fcur;  // FREQN15(NPTS-1), set by the loop's last pass
        fcur = flast;
      } else {
        // FREQN15(I-1): the previous pass's value, or (I = 2, only above
        // 1.5e19 Hz) formed like the others
        fprev = __double2float_rn(log10((double)__fadd_rn(tb.ekarzas[i - 2], r) * kapp_freq_rydh()));
      }
      const float* xn = tb.xn + (NMAX - 1) * NPTS;
      x = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(fl, fcur), __fsub_rn(fprev, fcur)), __fsub_rn(xn[i - 2], xn[i - 1])),
                    xn[i - 1]);
    } else {
      const float* fn = tb.freqn + (n - 1) * NPTS;
      const float* xn = tb.xn + (n - 1) * NPTS;
      if (fl < fn[NPTS - 1]) return 0.0;
      int i;
      for (i = 2; i <= NPTS; ++i)
        if (fl > fn[i - 1]) break;
      if (i > NPTS) i = NPTS;
      x = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(fl, fn[i - 1]), __fsub_rn(fn[i - 2], fn[i - 1])),
                              __fsub_rn(xn[i - 2], xn[i - 1])),
                    xn[i - 1]);
    }
  } else {
    const float* fn = tb.freqn + (n - 1) * NPTS;
    const float* xl = tb.xl + ((n - 1) * NLMAX + l) * NPTS;  // XL(I, L+1, N)
    if (fl < fn[NPTS - 1]) return 0.0;
    int i;
    for (i = 2; i <= NPTS; ++i)
      if (fl > fn[i - 1]) break;
    if (i > NPTS) i = NPTS;
    x = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(fl, fn[i - 1]), __fsub_rn(fn[i - 2], fn[i - 1])),
                            __fsub_rn(xl[i - 2], xl[i - 1])),
                  xl[i - 1]);
  }
  return exp((double)x * kLn10) / zeff2;
}

// COULFF(J, NZ) (:11995-12196): bilinear interpolation in log g_ff; z2log is
// Z2LOG(NZ) (0 for H, 0.60206 for He II)
__device__ inline double kapp_coulff(const KappDev& tb, double freqlg, double tlog, double z2log = 0.0) {
  constexpr int NG = 81, NU = 146;
  const double l10ryk = log10(kapp_freq_rydh() * kapp_hoverk());
  const double l10kh = -log10(kapp_hoverk());
  const double lgam2 = z2log + l10ryk - tlog / kLn10;
  const double lu = (freqlg - tlog) / kLn10 - l10kh;
  const double xi = (lgam2 - -6.0) / 0.2 + 1.0;
  const double xj = (lu - -16.0) / 0.2 + 1.0;
  int i0 = (int)xi, j0 = (int)xj;
  i0 = i0 > NG - 1 ? NG - 1 : (i0 < 1 ? 1 : i0);
  j0 = j0 > NU - 1 ? NU - 1 : (j0 < 1 ? 1 : j0);
  const double fi = fmax(0.0, fmin(xi - (double)i0, 1.0));
  const double fj = fmax(0.0, fmin(xj - (double)j0, 1.0));
  const double* g = tb.gff_log;
  const double lg00 = g[(j0 - 1) * NG + i0 - 1], lg01 = g[j0 * NG + i0 - 1];
  const double lg10 = g[(j0 - 1) * NG + i0], lg11 = g[j0 * NG + i0];
  const double lg = (1.0 - fi) * ((1.0 - fj) * lg00 + fj * lg01) + fi * ((1.0 - fj) * lg10 + fj * lg11);
  return pow(10.0, lg);
}

// LINTER (:5859-5880)
__device__ inline double kapp_linter(const double* xo, const double* yo, int n, double x) {
  int i;
  for (i = 2; i <= n; ++i)
    if (x < xo[i - 1]) break;
  if (i > n) i = n;
  return yo[i - 2] + (yo[i - 1] - yo[i - 2]) / (xo[i - 1] - xo[i - 2]) * (x - xo[i - 2]);
}

// HRAYOP's cross-section at FREQ (:12793-12900)
__device__ inline double kapp_rayleigh(const KappDev& tb, double freq) {
  const double fr = kapp_freq_rydh();
  const double d1 = 0.01 * fr, dab = 0.005 * fr, dbc = 0.002 * fr, dcd = 0.001 * fr;
  int i;
  double g;
  if (freq < d1) return kSigmaThomson * powi(tb.ray_m[0], 2) * powi(freq / d1, 4);
  if (freq <= 0.74 * fr) {
    i = min((int)(freq / d1) + 1, 74);
    g = tb.ray_m[i - 2] + (tb.ray_m[i - 1] - tb.ray_m[i - 2]) / d1 * (freq - (double)(i - 1) * d1);
    return kSigmaThomson * powi(g, 2);
  }
  if (freq < 0.77 * fr) return 0.0;
  if (freq <= 0.885 * fr) {
    i = min((int)((freq - 0.755 * fr) / dab) + 1 + 1, 27);
    g = tb.ray_ab[i - 2] + (tb.ray_ab[i - 1] - tb.ray_ab[i - 2]) / dab * (freq - (0.755 * fr + (double)(i - 2) * dab));
    return kSigmaThomson * powi(g, 2);
  }
  if (freq < 0.890 * fr) return 0.0;
  if (freq <= 0.936 * fr) {
    i = min((int)((freq - 0.890 * fr) / dbc) + 1 + 1, 24);
    g = tb.ray_bc[i - 2] + (tb.ray_bc[i - 1] - tb.ray_bc[i - 2]) / dbc * (freq - (0.890 * fr + (double)(i - 2) * dbc));
    return kSigmaThomson * powi(g, 2);
  }
  if (freq < 0.938 * fr) return 0.0;
  if (freq <= 0.959 * fr) {
    i = min((int)((freq - 0.938 * fr) / dcd) + 1 + 1, 22);
    g = tb.ray_cd[i - 2] + (tb.ray_cd[i - 1] - tb.ray_cd[i - 2]) / dcd * (freq - (0.938 * fr + (double)(i - 2) * dcd));
    return kSigmaThomson * powi(g, 2);
  }
  if (freq < 0.961 * fr) return 0.0;
  if (freq <= fr) return kSigmaThomson * tb.ray_ly[0];
  const double xnew = freq / fr;
  double fnew;
  s_map1(tb.ray_fly, tb.ray_ly, 64, &xnew, &fnew, 1);
  return kSigmaThomson * fnew;
}

// CROSSHE (:13160-13236): Marr & West's He I ground-state cross-section on
// four uniform wavelength grids
__device__ inline double kapp_crosshe(const KappDev& tb, double freq) {
  if (freq < 5.945209e15) return 0.0;
  const double wave = kClightAngs / freq;
  int i;
  if (wave > 50.0) {
    i = min(92, max(2, (int)(93.0 - (wave - 50.0) / 5.0)));
    return ((wave - (double)(92 - i) * 5.0 - 50.0) / 5.0 * (tb.he_x505[i - 2] - tb.he_x505[i - 1]) +
            tb.he_x505[i - 1]) *
           1.0e-18;
  }
  if (wave > 20.0) {
    i = min(16, max(2, (int)(17.0 - (wave - 20.0) / 2.0)));
    return ((wave - (double)(16 - i) * 2.0 - 20.0) / 2.0 * (tb.he_x50[i - 2] - tb.he_x50[i - 1]) +
            tb.he_x50[i - 1]) *
           1.0e-18;
  }
  if (wave > 10.0) {
    i = min(11, max(2, (int)(12.0 - (wave - 10.0) / 1.0)));
    return ((wave - (double)(11 - i) * 1.0 - 10.0) / 1.0 * (tb.he_x20[i - 2] - tb.he_x20[i - 1]) +
            tb.he_x20[i - 1]) *
           1.0e-18;
  }
  i = min(21, max(2, (int)(22.0 - wave / 0.5)));
  return ((wave - (double)(21 - i) * 0.5) / 0.5 * (tb.he_x10[i - 2] - tb.he_x10[i - 1]) + tb.he_x10[i - 1]) * 1.0e-18;
}

// the knot interpolation in log10 frequency shared by HE12S1S, HE12S3S,
// HE12P1P and HE12P3P (:13299-13545)
__device__ inline double kapp_he_knots(const double* f, const double* x, double freq) {
  const double freqlg = log10(freq);
  int i;
  for (i = 2; i <= 16; ++i)
    if (freqlg > f[i - 1]) break;
  if (i > 16) i = 16;
  const double v = (freqlg - f[i - 1]) / (f[i - 2] - f[i - 1]) * (x[i - 2] - x[i - 1]) + x[i - 1];
  return exp(v * kLn10);
}

// HE1OP's TRANS(N) (:13006-13097): the level's own cross-section when
// IMIN <= N, plus its inner-shell term to He II n = 2 (N = 2..5) or n = 3
// (N = 6..10) when IMIN >= 1 and every threshold of the nested tests is
// reached
__device__ __noinline__ double kapp_he1_trans(const KappDev& tb, double freq, int n, int imin) {
  double tr = 0.0;
  if (imin > 0 && imin <= n) {
    switch (n) {
      case 1: tr = kapp_crosshe(tb, freq); break;
      case 2:  // HE12S3S
        if (freq >= 38454.691 * kClight) {
          if (freq > 2.4 * kRydbergHe * kClight) {
            const double wavno = freq / kClight;
            const double ek = (wavno - 38454.691) / kRydbergHe;
            const double eps = 2.0 * (ek - 2.47898) / 0.000780;
            tr = 0.01521 * pow(470310.0 / wavno, 3.12) * 8.067e-18 * powi(eps - 122.4, 2) / (1.0 + powi(eps, 2));
          } else {
            tr = kapp_he_knots(tb.he2s3s_f, tb.he2s3s_x, freq);
          }
        }
        break;
      case 3:  // HE12S1S
        if (freq >= 32033.214 * kClight) {
          if (freq > 2.4 * kRydbergHe * kClight) {
            const double wavno = freq / kClight;
            const double ek = (wavno - 32033.214) / kRydbergHe;
            const double eps = 2.0 * (ek - 2.612316) / 0.00322;
            tr = 0.008175 * pow(484940.0 / wavno, 2.71) * 8.067e-18 * powi(eps + 76.21, 2) / (1.0 + powi(eps, 2));
          } else {
            tr = kapp_he_knots(tb.he2s1s_f, tb.he2s1s_x, freq);
          }
        }
        break;
      case 4:  // HE12P3P
        if (freq >= 29223.753 * kClight) tr = kapp_he_knots(tb.he2p3p_f, tb.he2p3p_x, freq);
        break;
      case 5:  // HE12P1P
        if (freq >= 27175.76 * kClight) {
          if (freq > 2.4 * kRydbergHe * kClight) {
            const double wavno = freq / kClight;
            const double ek = (wavno - 27175.76) / kRydbergHe;
            const double eps1s = 2.0 * (ek - 2.446534) / 0.01037;
            const double eps1d = 2.0 * (ek - 2.59427) / 0.00538;
            tr = 0.0009487 * pow(466750.0 / wavno, 3.69) * 8.067e-18 *
                 (powi(eps1s - 29.30, 2) / (1.0 + powi(eps1s, 2)) + powi(eps1d + 172.4, 2) / (1.0 + powi(eps1d, 2)));
          } else {
            tr = kapp_he_knots(tb.he2p1p_f, tb.he2p1p_x, freq);
          }
        }
        break;
      case 6: tr = kapp_xkarzas(tb, freq, 1.236439, 3, 0); break;
      case 7: tr = kapp_xkarzas(tb, freq, 1.102898, 3, 0); break;
      case 8: tr = kapp_xkarzas(tb, freq, 1.045499, 3, 1); break;
      case 9: tr = kapp_xkarzas(tb, freq, 1.001427, 3, 2); break;
      default: tr = kapp_xkarzas(tb, freq, 0.9926, 3, 1); break;
    }
  }
  if (imin >= 1 && n >= 2) {
    const double ryd = kRydbergHe * kClight;
    // excited-level energies (cm^-1) of the nested tests: N = 5, 4, 3, 2 below
    // ELIM 527490.06 (He II n = 2), N = 10 .. 6 below ELIM 588451.59 (n = 3)
    const double elim = n <= 5 ? 527490.06 : 588451.59;
    const int top = n <= 5 ? 5 : 10;
    for (int k = top; k >= n; --k) {
      double e;
      switch (k) {
        case 5: e = 171135.000; break;
        case 4: e = 169087.0; break;
        case 3: e = 166277.546; break;
        case 2: e = 159856.069; break;
        case 10: e = 186209.471; break;
        case 9: e = 186101.0; break;
        case 8: e = 185564.0; break;
        case 7: e = 184864.0; break;
        default: e = 183236.0; break;
      }
      const double freqhe = (elim - e) * kClight;
      if (!(freq >= freqhe)) break;
      if (k == n) tr = tr + kapp_xkarzas(tb, freq, freqhe / ryd, 1, 0);
    }
  }
  return tr;
}

// HE2OP (:13569-13674) at one depth: He II bound-free (dissolved levels
// n >= 10, n = 9..1 down to the frequency's threshold) and free-free
__device__ __noinline__ double kapp_he2op(const KappDev& tb, double freq, double freqlg, double waveno, double T,
                                    double tlog, double hckt, double stim, double xne, double rho, double x4,
                                    double x5) {
  const double freq3 = 2.815e29 / freq / freq / freq;
  const double xnfprho = x4 / rho;
  double H = freq3 * 16.0 * 2.0 / 2.0 / (438889.068 * hckt) *
             (exp(-fmax(434519.959, 438908.85 - waveno) * hckt) - exp(-438908.85 * hckt)) * stim * xnfprho;
  double X, A;
  do {
    if (waveno < 5418.390) break;
    X = freq3 / 59049.0 * 16.0;
    A = X * 162.0 * exp(-433490.46 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 6857.660) break;
    X = freq3 * 16.0 / 32768.0;
    A = X * 128.0 * exp(-432051.19 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 8956.950) break;
    X = freq3 * 16.0 / 16807.0;
    A = X * 98.0 * exp(-429951.90 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 12191.437) break;
    X = freq3 * 16.0 / 7776.0 * (1.0986 + (-2.704e13 + 1.229e27 / freq) / freq);
    A = X * 72.0 * exp(-426717.413 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 17555.715) break;
    X = freq3 * 16.0 / 3125.0 * (1.102 + (-3.909e13 + 2.371e27 / freq) / freq);
    A = X * 50.0 * exp(-421353.135 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 27430.925) break;
    X = freq3 * 16.0 / 1024.0 * (1.101 + (-5.765e13 + 4.593e27 / freq) / freq);
    A = X * 32.0 * exp(-411477.925 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 48766.491) break;
    X = freq3 * 16.0 / 243.0 * (1.101 + (-9.863e13 + 1.035e28 / freq) / freq);
    A = X * 18.0 * exp(-390142.359 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 109726.529) break;
    X = freq3 * 16.0 / 32.0 * (1.105 + (-2.375e14 + 4.077e28 / freq) / freq);
    A = X * 8.0 * exp(-329182.321 * hckt) * stim * xnfprho;
    H = H + A;
    if (waveno < 438908.850) break;
    X = freq3 * 16.0 / 1.0 * (0.9916 + (2.719e13 - 2.268e30 / freq) / freq);
    A = X * 2.0 * stim * xnfprho;
    H = H + A;
  } while (false);
  A = kCoeffFF * 4.0 / sqrt(T) * kapp_coulff(tb, freqlg, tlog, 0.60206) / freq * xne / freq * x5 / freq * stim / rho;
  return H + A;
}

// H2COLLOP's sum over the pairs at one depth (:16510-16522): the wavenumber
// interpolation of the two temperature rows that bracket the depth, then the
// temperature interpolation, in log10
__device__ __noinline__ double kapp_h2coll(const KappH2Dev* __restrict__ h, const double* __restrict__ ciaden,
                                           const double* __restrict__ ciait, const double* __restrict__ ciawt, int kw,
                                           int j, double rho, int inu, double delnu, double dlow) {
  double s = 0.0;
  for (int ip = 0; ip < 4; ++ip) {
    if (!h->use_pair[ip]) continue;
    const double den = ciaden[(size_t)ip * kw + j];
    if (den <= 0.0) continue;
    const int ic = (int)ciait[(size_t)ip * kw + j];
    const double wt = ciawt[(size_t)ip * kw + j];
    const double* r0 = h->cia_tab + ((size_t)ip * h->cia_ntmax + ic - 1) * h->cia_nnu + inu - 1;
    const double* r1 = r0 + h->cia_nnu;
    const double c0 = r0[0] * (1.0 - delnu) + r0[1] * delnu + dlow;
    const double c1 = r1[0] * (1.0 - delnu) + r1[1] * delnu + dlow;
    const double xlog = c0 * (1.0 - wt) + c1 * wt;
    s = s + pow(10.0, xlog) * den / rho;
  }
  return s;
}

// per-depth factors; threads over depths
static __global__ void k_kapp_depth(KappArgs a) {
  const KappDev& tb = *a.tb;
  const int kw = a.kw;
  const double saha = 2.0 * pow(2.0 * kPi * kEmass * kKbol / (kHplanck * kHplanck), 1.5);
  const double theta_c = 0.4342944819032518 / kapp_kbol_ev();
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.nrhox; j += gridDim.x * blockDim.x) {
    const double T = a.t[j];
    const double tk = kKbol * T;
    const double hkt = kHplanck / tk, hckt = hkt * kClight;
    const double tkev = kapp_kbol_ev() * T;
    a.d.hkt[j] = hkt;
    a.d.hckt[j] = hckt;
    a.d.tkev[j] = tkev;
    a.d.tlog[j] = log(T);
    a.d.theta[j] = theta_c / T;
    const double bm = a.bmin ? a.bmin[j] : 1.0, bh1 = a.bhyd ? a.bhyd[j] : 1.0;
    // XHMIN (HMINOP :12505-12509)
    a.d.xhmin[j] = exp(kHminusEA / tkev) / (saha * T * sqrt(T)) * bm * bh1 * a.xnfp1[j] * a.xne[j];
    const double xne = a.xne[j];
    const double xne23 = pow(xne, 2.0 / 3.0);
    for (int n = 1; n <= kHLev; ++n) {
      a.d.w[(size_t)(n - 1) * kw + j] = kapp_occupation(tb, n, xne, xne23);
      const double dn2 = powi((double)n, 2);
      const double en = n <= 15 ? tb.hop_elev[n - 1] : kElimHI - kRydbergH / dn2;
      a.d.bz[(size_t)(n - 1) * kw + j] = exp(-en * hckt);
      if (n >= 7 && n <= 15) a.d.bp[(size_t)(n - 7) * kw + j] = exp(-(kElimHI - kRydbergH / dn2) * hckt);
    }
    if (a.xnfp3) {
      // HE1OP's temperature block (:12978-12995)
      const double x3 = a.xnfp3[j], rho = a.rho[j];
      for (int n = 1; n <= 10; ++n)
        a.d.he_bolt[(size_t)(n - 1) * kw + j] = exp(-tb.he1_chi[n - 1] / tkev) * tb.he1_g[n - 1] * x3 / rho;
      for (int n = 4; n <= 27; ++n) {
        const double dn2 = powi((double)n, 2);
        a.d.he_boltn[(size_t)(n - 4) * kw + j] = exp(-24.587 * (1.0 - 1.0 / dn2) / tkev) * 4.0 * dn2 * x3 / rho;
      }
      a.d.he_freet[j] = xne * a.xnf4[j] / rho / sqrt(T);
      const double xr = x3 * (4.0 / 2.0 / 13.595) * tkev / rho;
      a.d.he_boltex[j] = exp(-23.730 / tkev) * xr;
      a.d.he_exlim[j] = exp(-24.587 / tkev) * xr;
    }
    if (a.xnf3) {
      // PARTFNH2 (:22398-22416), EQUILH2, then H2MINOP's XNH2M (:12668-12673)
      // and H2COLLOP's densities and temperature brackets (:16457-16481)
      const KappH2Dev& h = *a.h2;
      const double tt = fmin(h.pf_tstart + (double)(h.pf_n - 1) * h.pf_tstep, fmax(h.pf_tstart, T));
      int n = (int)((tt - h.pf_tstart) / h.pf_tstep) + 1;
      n = min(h.pf_n - 1, max(1, n));
      const double frac = (tt - (h.pf_tstart + (double)(n - 1) * h.pf_tstep)) / h.pf_tstep;
      const double q = (1.0 - frac) * h.pf[n - 1] + frac * h.pf[n] +
                       (powi(1.0 - frac, 3) - (1.0 - frac)) * h.pf2[n - 1] * powi(h.pf_tstep, 2) / 6.0 +
                       (powi(frac, 3) - frac) * h.pf2[n] * powi(h.pf_tstep, 2) / 6.0;
      const double equil = q * h.equil_pref / pow(T, 1.5) * exp(h.equil_d0 / T);
      const double bh1 = a.bhyd ? a.bhyd[j] : 1.0;
      const double xnhi = a.xnfp1[j] * 2.0 * bh1;
      a.d.xnh2m[j] = powi(a.xnfp1[j] * 2.0 * bh1, 2) * equil;
      const double xnh2 = T <= 20000.0 ? powi(xnhi, 2) * equil : 0.0;
      a.d.xnh2[j] = xnh2;
      const double x3 = a.xnf3[j];
      const double den[4] = {xnh2 * xnh2, xnh2 * x3, xnh2 * xnhi, xnhi * x3};
#pragma unroll
      for (int ip = 0; ip < 4; ++ip) {
        const double* tp = h.cia_temp + ip * h.cia_ntmax;
        const int nt = h.cia_nt[ip];
        const double tcl = fmax(tp[0], fmin(tp[nt - 1], T));
        int it = 1;
        for (int i = 1; i <= nt - 1; ++i)
          if (tcl >= tp[i - 1]) it = i;
        a.d.ciaden[(size_t)ip * kw + j] = den[ip];
        a.d.ciait[(size_t)ip * kw + j] = (double)it;
        a.d.ciawt[(size_t)ip * kw + j] = (tcl - tp[it - 1]) / (tp[it] - tp[it - 1]);
      }
    }
  }
}

constexpr int kKappWarps = 8;  // warps per CTA of k_kapp_nu

// warp per frequency (grid-stride), lanes over depths; kHelium adds the
// helium sources and kH2 (with kHelium) the H2 ones (separate instantiations
// keep the hydrogen one lean)
template <bool kHelium, bool kH2>
static __global__ void __launch_bounds__(kKappWarps * 32) k_kapp_nu(KappArgs a) {
  __shared__ double s_xk[kKappWarps][kHLev + 1];
  __shared__ double s_fftt[kKappWarps][11];
  __shared__ double s_he[kKappWarps][10 + 24 + 12 + 7];  // HE1OP's TRANS, TRANSN of n = 4..27; HEMIOP's and H2MINOP's KT
  const KappDev& tb = *a.tb;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kw = a.kw;
  const double fr = kapp_freq_rydh();
  const double theta_c = 0.4342944819032518 / kapp_kbol_ev();
  double* xk = s_xk[wid];
  double* fftt = s_fftt[wid];
  double* trans = s_he[wid];
  double* transn = trans + 10;
  double* hem_kt = transn + 24;
  double* h2m_kt = hem_kt + 12;
  constexpr bool helium = kHelium;
  for (int nu = blockIdx.x * kKappWarps + wid; nu < a.numnu; nu += gridDim.x * kKappWarps) {
    // RUN_RT_PASS's frequency quantities (:3907-3917)
    const double wave = a.waveset[nu];
    const double freq = kClightNms / wave;
    const double waveno = 1.0e7 / wave;
    const double freqlg = log(freq);
    const double f3 = powi(freq / 1.0e15, 3);
    // XKARZAS(FREQ, 1, n, n) of n = 1..80, HMINOP's free-free table at this wavelength
    for (int n = lane + 1; n <= kHLev; n += 32) xk[n] = kapp_xkarzas(tb, freq, 1.0, n, n);
    if (lane < 11)
      fftt[lane] = exp(kapp_linter(tb.wfflog, tb.fflog + lane * 22, 22, log(wave))) / tb.thetaff[lane] * theta_c *
                   kKbol;
    double hminbf = 0.0;
    if (freq > 1.82365e14) s_map1(tb.wbf, tb.bf, 116, &wave, &hminbf, 1);
    const double xray = kapp_rayleigh(tb, freq);
    const double* c = tb.h2p_fr;
    const double* e = tb.h2p_es;
    const double frh2 = c[0] + (c[1] + (c[2] + (c[3] + c[4] * freqlg) * freqlg) * freqlg) * freqlg;
    const double esh2 = e[0] + (e[1] + (e[2] + (e[3] + (e[4] + e[5] * freq) * freq) * freq) * freq) * freq;
    const double freq3_inv = 1.0 / (freq * freq * freq);
    // helium per frequency: HE1OP's IMIN and cross-sections (lanes over the
    // levels), HEMIOP's log k at this wavelength for the twelve temperatures,
    // HERAOP's cross-section
    int imin = 0;
    double sighe_x = 0.0;
    const double freq3he = powi(freq, 3);
    if (helium) {
      for (int n = 1; n <= 10; ++n)
        if (tb.he1_freq[n - 1] <= freq) {
          imin = n;
          break;
        }
      if (lane < 10) trans[lane] = kapp_he1_trans(tb, freq, lane + 1, imin);
      if (lane < 24) {
        const double zeff2 = 4.0 - 3.0 / powi((double)(lane + 4), 2);
        transn[lane] = freq >= 1.25408e16 ? kapp_xkarzas(tb, freq, zeff2, 1, 0) : 0.0;
      }
      double wl = wave;
      if (wl > tb.hem_w[16]) wl = tb.hem_w[16];
      int iw = 1;
      for (int i = 1; i <= 16; ++i)
        if (wl >= tb.hem_w[i - 1]) iw = i;
      const double xw = (log(wl) - tb.hem_logw[iw - 1]) / (tb.hem_logw[iw] - tb.hem_logw[iw - 1]);
      if (lane < 12)
        hem_kt[lane] = tb.hem_logk[lane * 17 + iw - 1] * (1.0 - xw) + tb.hem_logk[lane * 17 + iw] * xw;
      const double w = kClightAngs / fmin(freq, 5.15e15);
      const double ww = powi(w, 2);
      sighe_x = 5.484e-14 / ww / ww * powi(1.0 + (2.44e5 + 5.94e10 / (ww - 2.90e5)) / ww, 2);
    }
    // H2 per frequency: H2MINOP's log k at this wavelength for its seven
    // temperatures, H2RAOP's cross-section, H2COLLOP's wavenumber bracket
    double sigh2_x = 0.0, cia_delnu = 0.0, cia_dlow = 0.0;
    int cia_inu = 0;
    bool cia_on = false;
    if (kH2) {
      const KappH2Dev& h = *a.h2;
      double wl = wave;
      if (wl > h.h2m_w[9]) wl = h.h2m_w[9];
      int iw = 1;
      for (int i = 1; i <= 9; ++i)
        if (wl >= h.h2m_w[i - 1]) iw = i;
      const double xw = (log(wl) - h.h2m_logw[iw - 1]) / (h.h2m_logw[iw] - h.h2m_logw[iw - 1]);
      if (lane < 7) h2m_kt[lane] = h.h2m_logk[lane * 10 + iw - 1] * (1.0 - xw) + h.h2m_logk[lane * 10 + iw] * xw;
      const double w = kClightAngs / fmin(freq, 2.922e15);
      const double ww = powi(w, 2);
      sigh2_x = (8.14e-13 + 1.28e-6 / ww + 1.61 / (ww * ww)) / (ww * ww);
      if (!(waveno > h.cia_numax)) {
        if (waveno <= h.cia_nu0) {
          if (waveno > 0.0) {
            cia_on = true;
            cia_inu = 1;
            cia_dlow = 2.0 * log10(waveno / h.cia_nu0);
          }
        } else {
          cia_on = true;
          cia_inu = min((int)((waveno - h.cia_nu0) / h.cia_dnu) + 1, h.cia_nnu - 1);
          cia_delnu = (waveno - h.cia_nu0 - h.cia_dnu * (double)(cia_inu - 1)) / h.cia_dnu;
        }
      }
    }
    __syncwarp();
    for (int j = lane; j < a.nrhox; j += 32) {
      const double T = a.t[j];
      const double ehvkt = exp(-freq * a.d.hkt[j]);
      const double stim = 1.0 - ehvkt;
      const double bnu = kBnuPrefac * f3 * ehvkt / stim;
      const double xne = a.xne[j], rho = a.rho[j], x1 = a.xnfp1[j], x2 = a.xnfp2[j];
      const double bm = a.bmin ? a.bmin[j] : 1.0;
      const double* W = a.d.w + j;
      const double* BZ = a.d.bz + j;
      const double* BP = a.d.bp + j;
      // HOP: explicit levels n = 15 .. 1, each exit below its series limit
      double H = 0.0, S = 0.0, A;
      for (int n = 15; n >= 1; --n) {
        if (waveno < tb.series_limits[n - 1]) break;
        if (n >= 7) {
          A = W[(n - 1) * kw] * xk[n] * (double)(2 * n * n) * BZ[(n - 1) * kw] * stim;
          H = H + A;
          S = S + A * bnu;
        } else {
          const double bh = a.bhyd ? a.bhyd[(size_t)(n - 1) * kw + j] : 1.0;
          if (n >= 2) A = xk[n] * (double)(2 * n * n) * BZ[(n - 1) * kw] * (bh - ehvkt);
          else A = xk[1] * 2.0 * 1.0 * (bh - ehvkt);
          H = H + A;
          S = S + A * bnu * stim / (bh - ehvkt);
        }
      }
      // n = 16..80 from XKARZAS's n = 15 rescaling
      for (int n = 16; n <= kHLev; ++n) {
        const double dn2 = powi((double)n, 2);
        if (waveno < kElimHI / dn2) continue;
        const double w = W[(n - 1) * kw];
        if (w < 1.0e-6) continue;
        A = w * xk[n] * 2.0 * dn2 * BZ[(n - 1) * kw] * stim;
        H = H + A;
        S = S + A * bnu;
      }
      // the dissolved fraction 1 - w_n of n = 7..80 as a Kramers pseudo-continuum
      for (int n = 7; n <= kHLev; ++n) {
        const double w = W[(n - 1) * kw];
        if (1.0 - w < 1.0e-6) continue;
        const double bz = n <= 15 ? BP[(n - 7) * kw] : BZ[(n - 1) * kw];
        A = (1.0 - w) * 2.815e29 * freq3_inv * 2.0 / powi((double)n, 3) * bz * stim;
        H = H + A;
        S = S + A * bnu;
      }
      H = H * x1 / rho;
      S = S * x1 / rho;
      const double gff1 = kapp_coulff(tb, freqlg, a.d.tlog[j]);  // COULFF(J, 1), also HE1OP's
      A = kCoeffFF / sqrt(T) * gff1 / freq * xne / freq * x2 / freq * stim / rho;
      H = H + A;
      S = S + A * bnu;
      const double ahyd = H, shyd = H > 0.0 ? S / H : 0.0;
      const double bh1 = a.bhyd ? a.bhyd[j] : 1.0;
      // H2PLOP
      const double ah2p = freq > fr ? 0.0 : exp(-esh2 / a.d.tkev[j] + frh2) * x1 * 2.0 * bh1 * x2 / rho * stim;
      // HMINOP
      const double ffth = kapp_linter(tb.thetaff, fftt, 11, a.d.theta[j]);
      const double hminff = ffth * x1 * 2.0 * bh1 * xne / rho;
      const double hbf = hminbf * 1.0e-18 * (1.0 - ehvkt / bm) * a.d.xhmin[j] / rho;
      const double ahmin = hbf + hminff;
      const double shmin = (hbf * bnu * stim / (bm - ehvkt) + hminff * bnu) / ahmin;
      // HRAYOP, ELECOP
      const double sigh = xray * x1 * 2.0 * bh1 / rho;
      const double sigel = kSigmaThomson * xne / rho;
      // helium: HE1OP (:13108-13140), HE2OP, HEMIOP, HERAOP
      double ahe1 = 0.0, ahe2 = 0.0, ahemin = 0.0, sighe = 0.0;
      if (helium) {
        const double exlim = a.d.he_exlim[j];
        double ex = a.d.he_boltex[j];
        if (freq < 2.055e14) ex = exlim / ehvkt;
        double he1 = (ex - exlim) * (2.815e29 / freq3he);
        if (imin > 0)
          for (int n = imin; n <= 10; ++n) he1 = he1 + trans[n - 1] * a.d.he_bolt[(size_t)(n - 1) * kw + j];
        if (freq >= 1.25408e16)
          for (int n = 4; n <= 27; ++n) he1 = he1 + transn[n - 4] * a.d.he_boltn[(size_t)(n - 4) * kw + j];
        ahe1 = (he1 + gff1 * a.d.he_freet[j] * (kCoeffFF / freq3he)) * stim;
        ahe2 = kapp_he2op(tb, freq, freqlg, waveno, T, a.d.tlog[j], a.d.hckt[j], stim, xne, rho, a.xnfp4[j],
                          a.xnfp5[j]);
        int it = 1;
        for (int i = 1; i <= 11; ++i)
          if (T >= tb.hem_t[i - 1]) it = i;
        double xt = (log(fmax(T, 1.0)) - tb.hem_logt[it - 1]) / (tb.hem_logt[it] - tb.hem_logt[it - 1]);
        xt = fmax(0.0, fmin(1.0, xt));
        const double lkv = hem_kt[it - 1] * (1.0 - xt) + hem_kt[it] * xt;
        const double x3 = a.xnfp3[j];
        ahemin = exp(lkv) * xne * kKbol * T * x3 / rho;
        sighe = sighe_x * x3 / rho;
      }
      // H2: H2MINOP (:12686-12704), H2COLLOP (:16483-16522), H2RAOP
      double ah2min = 0.0, ah2coll = 0.0, sigh2 = 0.0;
      if (kH2) {
        const KappH2Dev& h = *a.h2;
        int it = 1;
        for (int i = 1; i <= 6; ++i)
          if (T >= h.h2m_t[i - 1]) it = i;
        double xt = (log(fmax(T, 1.0)) - h.h2m_logt[it - 1]) / (h.h2m_logt[it] - h.h2m_logt[it - 1]);
        xt = fmax(0.0, fmin(1.0, xt));
        const double lkv = h2m_kt[it - 1] * (1.0 - xt) + h2m_kt[it] * xt;
        ah2min = exp(lkv) * xne * kKbol * T * a.d.xnh2m[j] / rho;
        if (cia_on)
          ah2coll = kapp_h2coll(a.h2, a.d.ciaden, a.d.ciait, a.d.ciawt, kw, j, rho, cia_inu, cia_delnu, cia_dlow);
        sigh2 = sigh2_x * a.d.xnh2[j] / rho;
      }
      // KAPP's totals (:11300-11320); the metal and line sources are zero
      const double av = ah2p + ahe1 + ahe2 + ahemin + ah2min + ah2coll + 0.0;
      const double acont = av + ahyd + ahmin;
      double scont = bnu;
      if (acont > 0.0) scont = (av * bnu + ahyd * shyd + ahmin * shmin) / acont;
      const size_t o = (size_t)nu * kw + j;
      a.acont[o] = acont;
      a.scont[o] = scont;
      a.sigmac[o] = sigh + sighe + sigel + sigh2 + 0.0;
      if (a.parts) {
        double* p = a.parts + (size_t)nu * a.nparts * kw + j;
        p[0] = ahyd;
        p[kw] = shyd;
        p[2 * kw] = ah2p;
        p[3 * kw] = ahmin;
        p[4 * kw] = shmin;
        p[5 * kw] = sigh;
        p[6 * kw] = sigel;
        if (a.nparts > 7) {
          p[7 * kw] = ahe1;
          p[8 * kw] = ahe2;
          p[9 * kw] = ahemin;
          p[10 * kw] = sighe;
        }
        if (a.nparts > 11) {
          p[11 * kw] = ah2min;
          p[12 * kw] = ah2coll;
          p[13 * kw] = sigh2;
        }
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ HLINOP
// hydrogen_f_value (:17760-17829): tabulated gf of the first members, a
// Kramers estimate with an average Gaunt factor beyond
__device__ inline double kapp_hf_value(const KappDev& tb, int n, int m) {
  if (m <= n) return 0.0;
  const double xn = (double)n, xm = (double)m;
  const int idx = m - n;
  double gf;
  if (n == 1 && idx <= 29) gf = tb.gf_lyman[idx - 1];
  else if (n == 2 && idx <= 28) gf = tb.gf_balmer[idx - 1];
  else if (n == 3 && idx <= 27) gf = tb.gf_paschen[idx - 1];
  else if (n == 4 && idx <= 3) gf = tb.gf_brackett[idx - 1];
  else {
    gf = 1.9603 * powi(xn, 2) / (powi(xm, 3) * powi(1.0 / powi(xn, 2) - 1.0 / powi(xm, 2), 3));
    gf = gf * 0.80;
  }
  return gf / (2.0 * powi(xn, 2));
}

// STARK's EXINT (:17650-17655)
__device__ inline double kapp_exint(double x) {
  return -log(x) - 0.57516 + (0.97996 + (-0.21654 + (0.033572 + (-0.0029222 + 1.05439e-4 * x) * x) * x) * x) * x;
}

// STARK(N, M, J) (:17528-17659): Griem's quasi-static profile with the
// impact correction; f0 = 1.25e-9 XNE^(2/3) of the depth
__device__ __noinline__ double kapp_stark(const KappDev& tb, int n, int m, double freq, double xne, double hkt,
                                          double f0) {
  const double xn = (double)n, xm = (double)m;
  const double x = xn / xm;
  const double xx = powi(x, 2);
  const double nn = xn * xn, mm = xm * xm;
  const int mminn = m - n;
  const double knm = mminn <= 5 ? tb.stark_knm[(n - 1) * 5 + mminn - 1] : 5.5e-5 * powi(nn * mm, 2) / (mm - nn);
  const double fnm = mminn <= 10 ? tb.stark_f[(n - 1) * 10 + mminn - 1]
                                 : tb.stark_f[(n - 1) * 10 + 9] *
                                       powi((20.0 * xn + 100.0) / ((xn + 10.0) * xm * (1.0 - xx)), 3);
  const double ryd = kapp_freq_rydh();
  const double freqnm = ryd * (1.0 / nn - 1.0 / mm);
  const double del = fabs(freq - freqnm);
  const double dbeta = kClightAngs / powi(freqnm, 2) / f0 / knm;
  const double beta = dbeta * del;
  const double y1 = mm * del * hkt / 2.0;
  const double y2 = (kPi * kPi / 2.0 / kA0Stark / kClight) * powi(del, 2) / xne;
  const double qstat = 1.5 + 0.5 * (powi(y1, 2) - 1.384) / (powi(y1, 2) + 1.384);
  double impact = 0.0;
  if (y1 < 8.0 && y1 < y2) {
    double exy2 = 0.0;
    if (y2 <= 8.0) exy2 = kapp_exint(y2);
    impact = 1.438 * sqrt(y1 * (1.0 - xx)) * (0.4 * exp(-y1) + kapp_exint(y1) - 0.5 * exy2);
  }
  double prof, ratio;
  if (beta <= 20.0) {
    prof = 8.0 / (80.0 + powi(beta, 3));
    ratio = qstat + impact;
  } else {
    prof = 1.5 / beta / beta / sqrt(beta);
    const double dioi = 6.28 * 1.48e-25 * (2.0 * mm * ryd / del) * xne *
                        (sqrt(2.0 * mm * ryd / del) * (1.3 * qstat + 0.30 * impact) - 3.9 * ryd * hkt);
    ratio = qstat * fmin(1.0 + dioi, 1.25) + impact;
  }
  return kA0Stark * fnm * prof * dbeta * ratio;
}

// STARK_MMM(N, M, J) (:17854-18106): the Stehle table of the series, trilinear
// in (log Delta-alpha, log T, log Ne) on log profile values (linear where one
// of the eight corners is not positive), the Delta-alpha^-2.5 wing past the
// table; STARK where the series, the transition, the density or the
// temperature is off the table
__device__ __noinline__ double kapp_stark_mmm(const KappDev& tb, const StehleDev* st, int n, int m, double freq,
                                              double T, double xne, double hkt, double f0) {
  if (n < 1 || n > 4 || m <= n || !st) return kapp_stark(tb, n, m, freq, xne, hkt, f0);
  const StehleDev& S = st[n - 1];
  if (S.n_dens == 0 || m < S.n_upper_min || m > S.n_upper_max) return kapp_stark(tb, n, m, freq, xne, hkt, f0);
  const int itrans = m - S.n_upper_min + 1;
  if (xne > S.density_grid[S.n_dens - 1]) return kapp_stark(tb, n, m, freq, xne, hkt, f0);
  const double ne_eff = fmin(xne, S.density_grid[S.max_dens_idx[itrans - 1] - 1]);
  const double xn = (double)n, xm = (double)m;
  const double lambda0 = kRydAng * powi(xn * xm, 2) / ((xm - xn) * (xm + xn));
  const double freq_nm = kClightAngs / lambda0;
  const double del_freq = fabs(freq - freq_nm);
  const double F0 = 1.25e-9 * pow(ne_eff, 2.0 / 3.0);
  if (F0 <= 0.0) return kapp_stark(tb, n, m, freq, xne, hkt, f0);
  const double dalpha = powi(lambda0, 2) / kClightAngs * del_freq / F0;
  const int nd = S.n_dens, nt = 10, na = 60;
  const double log_ne = log10(ne_eff);
  if (T < S.temp_grid[0] * 0.5 || T > S.temp_grid[nt - 1] * 2.0) return kapp_stark(tb, n, m, freq, xne, hkt, f0);
  int id1;
  for (id1 = 1; id1 <= nd - 1; ++id1)
    if (ne_eff <= S.density_grid[id1]) break;
  id1 = max(1, min(nd - 1, id1));
  const int id2 = id1 + 1;
  double frac_d = (log_ne - log10(S.density_grid[id1 - 1])) /
                  (log10(S.density_grid[id2 - 1]) - log10(S.density_grid[id1 - 1]));
  frac_d = fmax(0.0, fmin(1.0, frac_d));
  int it1;
  for (it1 = 1; it1 <= nt - 1; ++it1)
    if (T <= S.temp_grid[it1]) break;
  it1 = max(1, min(nt - 1, it1));
  const int it2 = it1 + 1;
  double frac_t = (log(T) - log(S.temp_grid[it1 - 1])) / (log(S.temp_grid[it2 - 1]) - log(S.temp_grid[it1 - 1]));
  frac_t = fmax(0.0, fmin(1.0, frac_t));
  int ia1 = 1, ia2 = 1;
  double frac_a = 0.0;
  if (dalpha > 0.0) {
    const double log_dalpha = log10(dalpha);
    if (log_dalpha <= S.log_dalpha_grid[0]) {
    } else if (log_dalpha >= S.log_dalpha_grid[na - 1]) {
      const double f_nm = kapp_hf_value(tb, n, m);
      const double I = S.k_alpha[itrans - 1] / pow(dalpha, 2.5);
      return kA0Stark * f_nm * I * powi(lambda0, 2) / (kClightAngs * F0);
    } else {
      for (ia1 = 1; ia1 <= na - 1; ++ia1)
        if (log_dalpha <= S.log_dalpha_grid[ia1]) break;
      ia1 = max(1, min(na - 1, ia1));
      ia2 = ia1 + 1;
      frac_a = (log_dalpha - S.log_dalpha_grid[ia1 - 1]) / (S.log_dalpha_grid[ia2 - 1] - S.log_dalpha_grid[ia1 - 1]);
      frac_a = fmax(0.0, fmin(1.0, frac_a));
    }
  }
  const double* P = S.profiles + (size_t)(itrans - 1) * nd * nt * na;
  auto pv = [&](int ia, int it, int id) { return P[((size_t)(id - 1) * nt + (it - 1)) * na + ia - 1]; };
  double v000 = pv(ia1, it1, id1), v001 = pv(ia2, it1, id1), v010 = pv(ia1, it2, id1), v011 = pv(ia2, it2, id1);
  double v100 = pv(ia1, it1, id2), v101 = pv(ia2, it1, id2), v110 = pv(ia1, it2, id2), v111 = pv(ia2, it2, id2);
  double I;
  if (v000 <= 0.0 || v001 <= 0.0 || v010 <= 0.0 || v011 <= 0.0 || v100 <= 0.0 || v101 <= 0.0 || v110 <= 0.0 ||
      v111 <= 0.0) {
    const double v00 = v000 + frac_a * (v001 - v000), v01 = v010 + frac_a * (v011 - v010);
    const double v10 = v100 + frac_a * (v101 - v100), v11 = v110 + frac_a * (v111 - v110);
    const double v0 = v00 + frac_t * (v01 - v00), v1 = v10 + frac_t * (v11 - v10);
    I = v0 + frac_d * (v1 - v0);
  } else {
    v000 = log(v000);
    v001 = log(v001);
    v010 = log(v010);
    v011 = log(v011);
    v100 = log(v100);
    v101 = log(v101);
    v110 = log(v110);
    v111 = log(v111);
    const double v00 = v000 + frac_a * (v001 - v000), v01 = v010 + frac_a * (v011 - v010);
    const double v10 = v100 + frac_a * (v101 - v100), v11 = v110 + frac_a * (v111 - v110);
    const double v0 = v00 + frac_t * (v01 - v00), v1 = v10 + frac_t * (v11 - v10);
    I = exp(v0 + frac_d * (v1 - v0));
  }
  I = fmax(I, 0.0);
  const double f_nm = kapp_hf_value(tb, n, m);
  return kA0Stark * f_nm * I * powi(lambda0, 2) / (kClightAngs * F0);
}

// HLINOP (:17381-17503): warp per frequency (grid-stride), lanes over depths;
// reads the occupation probabilities k_kapp_depth left in d.w
static __global__ void __launch_bounds__(kKappWarps * 32) k_hlinop(KappArgs a) {
  const KappDev& tb = *a.tb;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kw = a.kw;
  const double nu_lyman = kapp_freq_rydh();
  for (int nu = blockIdx.x * kKappWarps + wid; nu < a.numnu; nu += gridDim.x * kKappWarps) {
    const double wave = a.waveset[nu];
    const double freq = kClightNms / wave;
    const double f3 = powi(freq / 1.0e15, 3);
    const int n = (int)sqrt(nu_lyman / freq);
    bool none = n == 0 || n > 4 || (n == 1 && freq < 2.0e15) || (n == 2 && freq < 4.44e14);
    // MFREQ = NINT(SQRT(NU_LYMAN / (NU_LYMAN / N^2 - FREQ))); at the series
    // limit itself the argument is infinite and every upper level is past
    // the dissolved-level cut, as any MFREQ above 80 gives
    int mfreq = 1000000;
    if (!none) {
      const double q = sqrt(nu_lyman / (nu_lyman / powi((double)n, 2) - freq));
      if (q < 1.0e6) mfreq = (int)round(q);
    }
    for (int j = lane; j < a.nrhox; j += 32) {
      const size_t o = (size_t)nu * kw + j;
      if (none) {
        a.ahline[o] = 0.0;
        a.shline[o] = 0.0;
        continue;
      }
      const double T = a.t[j], xne = a.xne[j];
      const double hkt = a.d.hkt[j];
      const double ehvkt = exp(-freq * hkt);
      const double stim = 1.0 - ehvkt;
      const double bnu = kBnuPrefac * f3 * ehvkt / stim;
      const double f0 = 1.25e-9 * pow(xne, 2.0 / 3.0);
      const double* W = a.d.w + j;  // w_n at (n-1)*kw
      auto bh = [&](int k) { return a.bhyd ? a.bhyd[(size_t)(k - 1) * kw + j] : 1.0; };
      auto bolt = [&](int k) {
        const double dk2 = powi((double)k, 2);
        return exp(-(13.595 - 13.595 / dk2) / a.d.tkev[j]) * 2.0 * dk2 * bh(k) * a.xnfp1[j] / a.rho[j];
      };
      int m1 = mfreq, m2 = m1 + 1;
      m1 = max(m1, n + 1);
      double H = 0.0, S = 0.0;
      if (m1 > 6) {
        if (m1 > kHLev || W[(size_t)(m1 - 1) * kw] < 1.0e-3) {
          a.ahline[o] = 0.0;
          a.shline[o] = bnu;
          continue;
        }
        m1 = m1 - 1;
        m2 = m2 + 3;
        if (n >= 4 && m1 <= 8) {
          H = kapp_stark_mmm(tb, a.stehle, 3, 4, freq, T, xne, hkt, f0) * (1.0 - ehvkt * bh(4) / bh(3)) * bolt(3);
          S = H * bnu * stim / (bh(3) / bh(4) - ehvkt);
        }
      }
      const double bn = bh(n), boltn = bolt(n);
      for (int m = m1; m <= m2; ++m) {
        const double bm = m <= 6 ? bh(m) : 1.0;
        double w = 1.0;
        if (m >= 2 && m <= kHLev) w = W[(size_t)(m - 1) * kw];
        if (m > kHLev) w = 0.0;
        const double A = w * kapp_stark_mmm(tb, a.stehle, n, m, freq, T, xne, hkt, f0) * (1.0 - ehvkt * bm / bn) * boltn;
        H = H + A;
        S = S + A * bnu * stim / (bn / bm - ehvkt);
      }
      a.ahline[o] = H;
      a.shline[o] = H > 0.0 ? S / H : bnu;
    }
  }
}

}  // namespace atlasgpu
