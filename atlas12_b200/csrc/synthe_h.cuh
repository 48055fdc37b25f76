// synthe_h.cuh -- SYNTHE's hydrogen and deuterium lines: compute_line_opacity's
// TYPE -1/-2 branch (synthe_module.f90:3460-3606) with hydrogen_line_profile
// (:1032-1980), in FP64.  A warp per (record, depth): the Stehle Stark (x)
// Voigt convolution, when the line is on a loaded Stehle table, is built by
// the warp into its shared-memory slot (60 outputs, each a warp-reduced sum
// over up to 600 grid points), then the wings are walked 32 grid points a
// step with FP64 atomics into the depth's accumulator row.  The reference's
// SAVE'd convolution is reused across consecutive records of the same
// (N, M), so a deuterium line can be convolved with the Doppler width of the
// hydrogen line before it: the host works out, per (record, depth), whose
// Doppler width the convolution was built with and passes it in the flags.
#pragma once
#include "common.cuh"
#include "hydrogen.cuh"
#include "voigt.cuh"

namespace atlasgpu {

constexpr int kShWarps = 2;  // warps per block; each owns one ShConv slot


// a hydrogen record as the walk needs it (prepared on the host)
struct ShRec {
  double wl;     // WLVAC * DOPRATIO
  double alpha;  // ALPHAHYD(NBLO): the red-wing limit of beta lines
  float gf, elo;
  int n, m, nbuff;
  int variant;  // 0: alpha or isolated (NCON 0), 1: beta, 2: higher member with the merged-continuum taper
  int deut;     // TYPE -2
};

// per (record, depth), from the host: WCON, WTAIL of the taper (variant 2) and
// flags: bit 0 the record passes the KAPPA0 gates at this depth, bit 1 the
// convolution it uses was built with a deuterium line's Doppler width
struct ShPair {
  double wcon, wtail;
  int flags, pad;
};

struct ShArgs {
  const ShRec* rec;
  const ShPair* pair;  // [nrec][nrhox]
  int64_t nrec;
  int nrhox, length, nspec;
  double wbegin, ratio, wlend;
  const float* cont;               // [nrhox][length]
  const double *xnfdop, *dopple;   // [nrhox][nspec]: species 1
  const double *xne, *hckt, *t, *xnfph1, *xnfph2, *xnfhe1, *xnfh2;  // [nrhox]
  const atlasgpu_hydrogen_tables* tab;  // SYNTHE's tables
  const StehleDev* stehle;              // [4], or null: the K-P profile throughout
  double* acc;                          // [nrhox][length]
};

struct ShConv {
  double sp[60], prof[60], cda[600], cpa[600], cst[600];
  double F0, lambda0, dop_dalpha, voigt_a;
};

// (82259.10 - dw) * REAL(CLIGHT,4), formed in REAL(4) as the reference does
__device__ __forceinline__ double sh_lya_freq(float dw) {
  return (double)__fmul_rn(__fsub_rn(82259.10f, dw), 2.99792458e10f);
}

// lya_h2_blue_cutoff (:1916-1940)
__device__ inline double sh_lya_h2_blue(const atlasgpu_hydrogen_tables& h, double freq, double xnfph1) {
  const float c4 = 2.99792458e10f;
  const float spc = __fmul_rn(200.0f, c4), freq22 = __fmul_rn(__fsub_rn(82259.10f, 22000.0f), c4);
  if (freq < (double)__fmul_rn(50000.0f, c4)) return 0.0;
  double cval;
  if (freq < (double)freq22) {
    cval = (h.cutoffh2[1] - h.cutoffh2[0]) / (double)spc * (freq - (double)freq22) + h.cutoffh2[0];
  } else {
    const int ic = min((int)((freq - (double)freq22) / (double)spc), 89);  // in the table at the window's edge
    const float cfreq = __fadd_rn(__fmul_rn((float)ic, spc), freq22);
    cval = (h.cutoffh2[ic + 1] - h.cutoffh2[ic]) / (double)spc * (freq - (double)cfreq) + h.cutoffh2[ic];
  }
  return pow(10.0, cval - 14.0) * (double)(float)xnfph1 * 2.0 / (double)c4;
}

// lya_h2plus_red_cutoff (:1956-1978)
__device__ inline double sh_lya_h2plus_red(const atlasgpu_hydrogen_tables& h, double freq, double xnfph2) {
  const float c4 = 2.99792458e10f;
  const float spc = __fmul_rn(100.0f, c4), freq15 = __fmul_rn(__fsub_rn(82259.10f, 15000.0f), c4);
  double cval;
  if (freq < (double)freq15) {
    cval = (h.cutoffh2plus[1] - h.cutoffh2plus[0]) / (double)spc * (freq - (double)freq15) + h.cutoffh2plus[0];
  } else {
    const int ic = min((int)((freq - (double)freq15) / (double)spc), 109);
    const float cfreq = __fadd_rn(__fmul_rn((float)ic, spc), freq15);
    cval = (h.cutoffh2plus[ic + 1] - h.cutoffh2plus[ic]) / (double)spc * (freq - (double)cfreq) + h.cutoffh2plus[ic];
  }
  return pow(10.0, cval - 14.0) / (double)c4 * (double)(float)xnfph2;
}

// expint1 (:731-753)
__device__ __forceinline__ double sh_expint1(double x) {
  if (x <= 0.0) return 0.0;
  if (x <= 1.0)
    return -log(x) - 0.57721566 +
           x * (0.99999193 + x * (-0.24991055 + x * (0.05519968 + x * (-0.00976004 + x * 0.00107857))));
  if (x <= 30.0) return (x * (x + 2.334733) + 0.25062) / (x * (x + 3.330657) + 1.681534) / x * exp(-x);
  return 0.0;
}

// the depth arrays (:1203-1248)
struct ShDepth {
  double xne, t, pp, fo, y1b, y1s, t3nhe, t3nh2, c1d, c2d, gcon1, gcon2, xnfph1, xnfph2;
};

__device__ inline void sh_depth(double xne, double t, double xnfph1, double xnfph2, double xnfhe1, double xnfh2,
                                ShDepth& d) {
  const double xne16 = pow(xne, 1.0 / 6.0);
  d.xne = xne;
  d.t = t;
  d.pp = xne16 * 0.08989 / sqrt(t);
  d.fo = powi(xne16, 4) * 1.25e-9;
  d.y1b = 2.0 / (1.0 + 0.012 / t * sqrt(xne / t));
  const double t4 = t / 10000.0, t43 = pow(t4, 0.3);
  d.y1s = t43 / xne16;
  d.t3nhe = t43 * xnfhe1;
  d.t3nh2 = t43 * xnfh2;
  d.c1d = d.fo * 78940.0 / t;
  d.c2d = d.fo * d.fo / 5.96e-23 / xne;
  d.gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + xne / 1.0e13);
  d.gcon2 = 0.2 / (1.0 + xne / 1.0e15);
  d.xnfph1 = xnfph1;
  d.xnfph2 = xnfph2;
}

// the line constants (:1254-1358)
struct ShLine {
  int n, m, ifins;
  double xknm, freqnm, dbeta, wavenm, c1con, c2con, radamp, resont, vdw, stark, y1num, y1wht;
  double finest[14], finswt[14];
};

__device__ inline void sh_line(const atlasgpu_hydrogen_tables& h, int n, int m, ShLine& L) {
  const double clight_angs = 2.99792458e18;
  const int mmn = m - n;
  const double xn = (double)n, xm = (double)m, xn2 = xn * xn, xm2 = xm * xm;
  const double xmn2 = xm2 * xn2, xm2mn2 = xm2 - xn2, gnm = xm2mn2 / xmn2;
  L.n = n;
  L.m = m;
  L.xknm = (mmn <= 3 && n <= 4) ? h.xknmtb[n - 1][mmn - 1] : 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / (double)mmn);
  L.y1num = m == 2 ? 550.0 : (m == 3 ? 380.0 : 320.0);
  L.y1wht = mmn <= 3 ? 1.0e14 : 1.0e13;
  if (mmn <= 2 && n <= 2) L.y1wht = h.y1wtm[n - 1][mmn - 1];
  L.freqnm = 109677.583403 * 2.99792458e10 * gnm;
  L.dbeta = clight_angs / (L.freqnm * L.freqnm) / L.xknm;
  L.wavenm = clight_angs / L.freqnm;
  L.c1con = L.xknm / L.wavenm * gnm * xm2mn2;
  L.c2con = powi(L.xknm / L.wavenm, 2);
  const double radamp = n == 1 ? h.asumlyman[m - 1] : h.asum[n - 1] + h.asum[m - 1];
  L.radamp = radamp / (4.0 * kPi) / L.freqnm;
  double resont = hfnm(1, m) / xm / (1.0 - 1.0 / xm2);
  if (n != 1) resont = resont + hfnm(1, n) / xn / (1.0 - 1.0 / xn2);
  L.resont = resont * 3.579e-24 / gnm;
  L.vdw = 4.45e-26 / gnm * pow(xm2 * (7.0 * xm2 + 5.0), 0.4);
  L.stark = 1.6678e-18 * L.freqnm * L.xknm;
  if (n > 4 || m > 10) {
    L.ifins = 1;
    L.finest[0] = 0.0;
    L.finswt[0] = 1.0;
  } else if (mmn == 1) {
    L.ifins = h.lnghal[n - 1];
    const int ipos = h.istal[n - 1];
    for (int i = 0; i < L.ifins; ++i) {
      L.finest[i] = h.stalph[ipos - 1 + i] * 1.0e7;
      L.finswt[i] = h.stwtal[ipos - 1 + i] / xn2 / 3.0;
    }
  } else {
    L.ifins = h.lncomp[n - 1];
    for (int i = 0; i < L.ifins; ++i) {
      L.finest[i] = h.stcomp[i][n - 1] * 1.0e7;
      L.finswt[i] = h.stcpwt[i][n - 1] / xn2;
    }
  }
}

// the Peterson/Kurucz analytic path (:1698-1892)
__device__ inline double sh_prof_kp(const atlasgpu_hydrogen_tables& h, const ShLine& L, const ShDepth& d,
                                    double hwdop, double delw) {
  const double freq_rydh = 109677.583403 * 2.99792458e10, c4 = (double)2.99792458e10f;
  const int n = L.n, m = L.m;
  const double freqnm = L.freqnm;
  const double freq = 2.99792458e18 / (L.wavenm + delw * 10.0);
  const double del = fabs(freq - freqnm);
  const double hwstk = L.stark * d.fo;
  const double hwvdw = L.vdw * d.t3nhe + 2.0 * L.vdw * d.t3nh2;
  const double hwrad = L.radamp;
  const double hwres = L.resont * d.xnfph1 * 2.0;
  double hwlor = hwres + hwvdw + hwrad;
  const double dop = freqnm * hwdop;
  int nwid = 1;
  if (hwdop < hwstk || hwdop < hwlor) nwid = hwlor < hwstk ? 3 : 2;
  double mx = hwdop > hwlor ? hwdop : hwlor;
  mx = hwstk > mx ? hwstk : mx;
  const bool core = del <= freqnm * mx;
  double result = 0.0;
  if (!core || nwid == 1) {
    for (int i = 0; i < L.ifins; ++i) {
      const double dd = fabs(freq - freqnm - L.finest[i]) / dop;
      if (dd <= 7.0) result = result + exp(-dd * dd) * L.finswt[i];
    }
    if (core) return result;
  }
  if (!core || nwid == 2) {
    if (n == 1 && m == 2) {
      const double hwres4 = hwres * 4.0;
      hwlor = hwres4 + hwvdw + hwrad;
      const double hhw = freqnm * hwlor;
      const double hprofres = freq > sh_lya_freq(4000.0f)
                                  ? hwres4 * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop
                                  : sh_lya_h2_blue(h, freq, d.xnfph1) * kSqrtPi * dop;
      double hprofrad = 0.0;
      if (freq > (double)2.4190611e15f && freq < (double)0.77f * freq_rydh)
        hprofrad = hwrad * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
      double hprofvdw = hwvdw * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
      if (freq < (double)1.8e15f) hprofvdw = 0.0;
      result = result + hprofres + hprofrad + hprofvdw;
    } else {
      const double hhw = freqnm * hwlor;
      double top = hhw;
      if (n == 1 && m <= 5) {
        if (m == 3 && freq > (double)0.885f * freq_rydh && freq < (double)0.890f * freq_rydh) top = hhw - freqnm * hwrad;
        if (m == 4 && freq > (double)0.936f * freq_rydh && freq < (double)0.938f * freq_rydh) top = hhw - freqnm * hwrad;
        if (m == 5 && freq > (double)0.959f * freq_rydh && freq < (double)0.961f * freq_rydh) top = hhw - freqnm * hwrad;
      }
      result = result + top / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
    }
    if (core) return result;
  }
  const double wty1 = 1.0 / (1.0 + d.xne / L.y1wht);
  const double y1scal = L.y1num * d.y1s * wty1 + d.y1b * (1.0 - wty1);
  const double c1 = d.c1d * L.c1con * y1scal, c2 = d.c2d * L.c2con;
  const double g1 = 6.77 * sqrt(c1);
  double lg = 0.2114 + log(sqrt(c2) / c1);
  lg = lg > 0.0 ? lg : 0.0;
  const double gnot = g1 * lg * (1.0 - d.gcon1 - d.gcon2);
  const double beta = fabs(del) / d.fo * L.dbeta;
  const double y1 = c1 * beta, y2 = c2 * (beta * beta);
  double gam = gnot;
  if (!(y2 <= 1.0e-4 && y1 <= 1.0e-5)) {
    gam = g1 * (0.5 * exp(-(y1 < 80.0 ? y1 : 80.0)) + sh_expint1(y1) - 0.5 * sh_expint1(y2)) *
          (1.0 - d.gcon1 / (1.0 + powi(90.0 * y1, 3)) - d.gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1.0e-20) gam = 0.0;
  }
  double prqs = stark_profile(h, beta, d.pp, n, m);
  if (m == 2) {
    prqs = prqs * 0.5;
    if (freq >= sh_lya_freq(20000.0f) && freq <= sh_lya_freq(4000.0f)) {
      result = result + sh_lya_h2plus_red(h, freq, d.xnfph2) * kSqrtPi * dop;
    } else if (freq > sh_lya_freq(4000.0f)) {
      const double beta4000 = 4000.0 * c4 / d.fo * L.dbeta;
      const double prqsp4000 = stark_profile(h, beta4000, d.pp, n, m) * 0.5 / d.fo * L.dbeta;
      const double cutoff4000 = pow(10.0, -11.07 - 14.0) / c4 * d.xnfph2;
      result = result + cutoff4000 / prqsp4000 * prqs / d.fo * L.dbeta * kSqrtPi * dop;
    }
  }
  const double f = gam > 0.0 ? gam / kPi / (gam * gam + beta * beta) : 0.0;
  const double p1 = powi(0.9 * y1, 2);
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  return result + (prqs * (1.0 + fns) + f) / d.fo * L.dbeta * kSqrtPi * dop;
}

__device__ __forceinline__ bool sh_use_stehle(const StehleDev* st, int n, int m, double xne) {
  if (!st || n < 1 || n > 4) return false;
  const StehleDev& S = st[n - 1];
  return S.n_dens > 0 && m >= S.n_upper_min && m <= S.n_upper_max && xne <= S.density_grid[S.n_dens - 1];
}

// interp_stark_at (:2007-2037)
__device__ inline double sh_interp_stark(const StehleDev& S, const double* sp, double da) {
  if (da >= pow(10.0, S.log_dalpha_grid[59])) return sp[59];
  const double lda = log10(da);
  int idx = 1;
  while (idx <= 59 && !(lda <= S.log_dalpha_grid[idx])) ++idx;
  idx = min(idx, 59);
  const double frac = (lda - S.log_dalpha_grid[idx - 1]) / (S.log_dalpha_grid[idx] - S.log_dalpha_grid[idx - 1]);
  if (sp[idx - 1] > 0.0 && sp[idx] > 0.0) return exp(log(sp[idx - 1]) * (1.0 - frac) + log(sp[idx]) * frac);
  return sp[idx - 1] * (1.0 - frac) + sp[idx] * frac;
}

// the Stark (x) Voigt convolution (:1427-1640), built by the whole warp into c
__device__ void sh_conv_build(const StehleDev& S, const ShLine& L, const ShDepth& d, double hwdop, double hwlor_conv,
                              ShConv& c, int lane) {
  const int n = L.n, m = L.m;
  const double xn8 = (double)n, xm8 = (double)m;
  const double lambda0 = 1.0e8 / 109677.583403 * powi(xn8 * xm8, 2) / ((xm8 - xn8) * (xm8 + xn8));
  const int itrans = m - S.n_upper_min + 1, nd = S.n_dens;
  const double dcap = S.density_grid[S.max_dens_idx[itrans - 1] - 1];
  const double ne_cap = d.xne < dcap ? d.xne : dcap;
  const double F0 = 1.25e-9 * pow(ne_cap, 2.0 / 3.0);
  int id1 = 1;
  while (id1 <= nd - 1 && !(ne_cap <= S.density_grid[id1])) ++id1;
  id1 = max(1, min(nd - 1, id1));
  const int id2 = id1 + 1;
  double fd = (log10(ne_cap) - log10(S.density_grid[id1 - 1])) /
              (log10(S.density_grid[id2 - 1]) - log10(S.density_grid[id1 - 1]));
  fd = fd < 0.0 ? 0.0 : (fd > 1.0 ? 1.0 : fd);
  int it1 = 1;
  while (it1 <= 9 && !(d.t <= S.temp_grid[it1])) ++it1;
  it1 = min(9, it1);
  const int it2 = it1 + 1;
  double ft = (d.t - S.temp_grid[it1 - 1]) / (S.temp_grid[it2 - 1] - S.temp_grid[it1 - 1]);
  ft = ft < 0.0 ? 0.0 : (ft > 1.0 ? 1.0 : ft);
  const double* P = S.profiles + (size_t)(itrans - 1) * nd * 600;
  for (int ia = lane; ia < 60; ia += 32) {
    const double v00 = P[((size_t)(id1 - 1) * 10 + it1 - 1) * 60 + ia], v01 = P[((size_t)(id1 - 1) * 10 + it2 - 1) * 60 + ia];
    const double v10 = P[((size_t)(id2 - 1) * 10 + it1 - 1) * 60 + ia], v11 = P[((size_t)(id2 - 1) * 10 + it2 - 1) * 60 + ia];
    c.sp[ia] = (v00 > 0 && v01 > 0 && v10 > 0 && v11 > 0)
                   ? exp(log(v00) * (1 - fd) * (1 - ft) + log(v01) * (1 - fd) * ft + log(v10) * fd * (1 - ft) +
                         log(v11) * fd * ft)
                   : v00 * (1 - fd) * (1 - ft) + v01 * (1 - fd) * ft + v10 * fd * (1 - ft) + v11 * fd * ft;
  }
  __syncwarp();
  const double dop_dalpha = lambda0 * lambda0 / 2.99792458e18 * L.freqnm * hwdop / F0;
  const double lor_dalpha = lambda0 * lambda0 / 2.99792458e18 * L.freqnm * hwlor_conv / F0;
  const double voigt_a = (double)(float)(lor_dalpha / dop_dalpha);
  const double dx_wing = dop_dalpha / 3.0;
  const double d_log = (S.log_dalpha_grid[59] - S.log_dalpha_grid[0]) / 59.0;
  int n_log = 60;
  for (int ia = 1; ia <= 60; ++ia)
    if (pow(10.0, S.log_dalpha_grid[ia - 1]) * d_log * log(10.0) > dx_wing) {
      n_log = ia - 1;
      break;
    }
  n_log = max(n_log, 1);
  const double da_trans = pow(10.0, S.log_dalpha_grid[n_log - 1]);
  const double da_last = pow(10.0, S.log_dalpha_grid[59]);
  int n_wing = 200;
  double da_wing_max = da_trans + 200.0 * dx_wing;
  if (da_wing_max > da_last) {
    da_wing_max = da_last;
    n_wing = max((int)((da_wing_max - da_trans) / dx_wing), 0);
  }
  if (2 * n_wing + 2 * n_log + 1 > 600) {
    n_wing = (600 - 2 * n_log - 1) / 2;
    da_wing_max = da_trans + (double)n_wing * dx_wing;
  }
  const int ic = 2 * n_wing + 2 * n_log + 1;
  for (int k = lane; k < ic; k += 32) {
    double da, pv;
    if (k < n_wing) {  // negative wing, largest |Delta-alpha| first
      const double x = da_trans + (double)(n_wing - k) * dx_wing;
      da = -x;
      pv = sh_interp_stark(S, c.sp, x);
    } else if (k < n_wing + n_log) {
      const int ia = n_log - (k - n_wing);
      da = -pow(10.0, S.log_dalpha_grid[ia - 1]);
      pv = c.sp[ia - 1];
    } else if (k == n_wing + n_log) {
      da = 0.0;
      pv = c.sp[0];
    } else if (k <= n_wing + 2 * n_log) {
      const int ia = k - n_wing - n_log;
      da = pow(10.0, S.log_dalpha_grid[ia - 1]);
      pv = c.sp[ia - 1];
    } else {
      const double x = da_trans + (double)(k - n_wing - 2 * n_log) * dx_wing;
      da = x;
      pv = sh_interp_stark(S, c.sp, x);
    }
    c.cda[k] = da;
    c.cpa[k] = pv;
  }
  __syncwarp();
  for (int k = lane; k < ic; k += 32)
    c.cst[k] = k == 0 ? c.cda[1] - c.cda[0]
                      : (k == ic - 1 ? c.cda[ic - 1] - c.cda[ic - 2] : 0.5 * (c.cda[k + 1] - c.cda[k - 1]));
  __syncwarp();
  for (int ia = 0; ia < 60; ++ia) {
    const double da_i = pow(10.0, S.log_dalpha_grid[ia]);
    if (da_i > da_wing_max && da_wing_max > 0.0) {
      if (lane == 0) c.prof[ia] = c.sp[ia] + voigt_a * dop_dalpha / (kPi * (da_i * da_i));
    } else {
      double g = 0.0;
      for (int k = lane; k < ic; k += 32) {
        const float vv = (float)((da_i - c.cda[k]) / dop_dalpha);
        g += c.cpa[k] * (double)(float)voigt_weideman((double)vv, voigt_a) * c.cst[k];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
      if (lane == 0) c.prof[ia] = g / (dop_dalpha * kSqrtPi);
    }
  }
  if (lane == 0) {
    c.F0 = F0;
    c.lambda0 = lambda0;
    c.dop_dalpha = dop_dalpha;
    c.voigt_a = voigt_a;
  }
  __syncwarp();
}

// hydrogen_line_profile on the Stehle path (:1642-1696), from the convolution
__device__ inline double sh_prof_stehle(const atlasgpu_hydrogen_tables& h, const StehleDev& S, const ShConv& c,
                                        const ShLine& L, const ShDepth& d, double hwdop, double delw) {
  const double freq = 2.99792458e18 / (L.wavenm + delw * 10.0);
  const double del = fabs(freq - L.freqnm);
  const double dop = L.freqnm * hwdop;
  const double dac = c.lambda0 * c.lambda0 / 2.99792458e18 * del / c.F0;
  double I;
  if (dac <= pow(10.0, S.log_dalpha_grid[0])) {
    I = c.prof[0];
  } else if (dac >= pow(10.0, S.log_dalpha_grid[59])) {
    I = S.k_alpha[L.m - S.n_upper_min] / pow(dac, 2.5) + c.voigt_a * c.dop_dalpha / (kPi * (dac * dac));
  } else {
    const double lda = log10(dac);
    int ia1 = 1;
    while (ia1 <= 59 && !(lda <= S.log_dalpha_grid[ia1])) ++ia1;
    ia1 = min(ia1, 59);
    const double fa = (lda - S.log_dalpha_grid[ia1 - 1]) / (S.log_dalpha_grid[ia1] - S.log_dalpha_grid[ia1 - 1]);
    const double p1 = c.prof[ia1 - 1], p2 = c.prof[ia1];
    I = (p1 > 0.0 && p2 > 0.0) ? exp(log(p1) * (1.0 - fa) + log(p2) * fa) : p1 * (1.0 - fa) + p2 * fa;
  }
  const double phi = I * (c.lambda0 * c.lambda0) / (2.99792458e18 * c.F0);
  double result = phi * kSqrtPi * dop;
  if (L.n == 1 && L.m == 2) {
    if (freq <= sh_lya_freq(4000.0f)) result = result + sh_lya_h2_blue(h, freq, d.xnfph1) * kSqrtPi * dop;
    if (freq >= sh_lya_freq(20000.0f) && freq <= sh_lya_freq(4000.0f))
      result = result + sh_lya_h2plus_red(h, freq, d.xnfph2) * kSqrtPi * dop;
    if (freq < (double)__fmul_rn(50000.0f, 2.99792458e10f)) result = 0.0;
  }
  return result;
}

static __global__ void __launch_bounds__(32 * kShWarps) k_synthe_hydrogen(ShArgs a) {
  __shared__ ShConv conv[kShWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  ShConv& cv = conv[wib];
  const atlasgpu_hydrogen_tables& h = *a.tab;
  const double CUTOFF = 1.0e-3;
  const int64_t npairs = a.nrec * a.nrhox;
  const int64_t nw = (int64_t)gridDim.x * kShWarps;
  for (int64_t p = (int64_t)blockIdx.x * kShWarps + wib; p < npairs; p += nw) {
    const ShPair pr = a.pair[p];
    if (!(pr.flags & 1)) continue;
    const int64_t i = p / a.nrhox;
    const int j = (int)(p - i * a.nrhox);
    const ShRec r = a.rec[i];
    const float* cont = a.cont + (size_t)j * a.length;
    double* acc = a.acc + (size_t)j * a.length;
    const double kappa0 = (double)r.gf * a.xnfdop[(size_t)j * a.nspec] * exp(-(double)r.elo * a.hckt[j]);
    float dopph = (float)a.dopple[(size_t)j * a.nspec];
    const float dopph_h = dopph;
    if (r.deut) dopph = __fdiv_rn(dopph, 1.4142f);
    ShLine L;
    sh_line(h, r.n, r.m, L);
    ShDepth d;
    sh_depth(a.xne[j], a.t[j], a.xnfph1[j], a.xnfph2[j], a.xnfhe1[j], a.xnfh2[j], d);
    const bool st = sh_use_stehle(a.stehle, r.n, r.m, d.xne);
    if (st) {
      const float dconv = (pr.flags & 2) ? __fdiv_rn(dopph_h, 1.4142f) : dopph_h;
      const double hwvdw = L.vdw * d.t3nhe + 2.0 * L.vdw * d.t3nh2;
      const double hwres = L.resont * d.xnfph1 * 2.0;
      const double hwlor_conv = (r.n == 1 && r.m == 2) ? hwres * 4.0 + hwvdw + L.radamp : hwres + hwvdw + L.radamp;
      sh_conv_build(a.stehle[r.n - 1], L, d, (double)dconv, hwlor_conv, cv, lane);
    }
    const double hwdop = (double)dopph;
    auto prof = [&](double wave) -> double {
      return kappa0 * (st ? sh_prof_stehle(h, a.stehle[r.n - 1], cv, L, d, hwdop, wave - r.wl)
                          : sh_prof_kp(h, L, d, hwdop, wave - r.wl));
    };
    const int length = a.length, minred = max(1, r.nbuff);
    const double wcon = pr.wcon, wtail = pr.wtail;
    auto taper = [&](double wave, double kappa) -> double {
      return (r.variant == 2 && wave < wtail) ? kappa * ((wave - wcon) / (wtail - wcon)) : kappa;
    };
    bool blue = true;
    if (r.variant == 0) {  // alpha / isolated line (:3483-3509)
      if (r.wl <= a.wlend) {
        for (int b0 = minred; b0 <= length; b0 += 32) {
          const int ib = b0 + lane;
          const bool in = ib <= length;
          const double kappa = in ? prof(a.wbegin * powi(a.ratio, ib - 1)) : 0.0;
          const unsigned below = __ballot_sync(0xffffffffu, in && kappa < (double)cont[ib - 1] * CUTOFF);
          const int stop = below ? __ffs(below) - 1 : 32;
          if (in && lane <= stop) atomicAdd(acc + ib - 1, kappa);
          if (below) break;
        }
        if (minred == 1 || r.wl < a.wbegin) blue = false;
      }
    } else if (r.variant == 1) {  // beta line: the red wing stops at the alpha line (:3511-3541)
      if (r.wl <= a.wlend) {
        bool exited = false;
        for (int b0 = minred; b0 <= length; b0 += 32) {
          const int ib = b0 + lane;
          const bool in = ib <= length;
          const double wave = a.wbegin * powi(a.ratio, ib - 1);
          const bool over = in && wave > r.alpha;
          const double kappa = (in && !over) ? prof(wave) : 0.0;
          const unsigned ov = __ballot_sync(0xffffffffu, over);
          const unsigned below = __ballot_sync(0xffffffffu, in && !over && kappa < (double)cont[ib - 1] * CUTOFF);
          const int first_ov = ov ? __ffs(ov) - 1 : 32, first_below = below ? __ffs(below) - 1 : 32;
          if (in && !over && lane < first_ov && lane <= first_below) atomicAdd(acc + ib - 1, kappa);
          if (ov || below) {
            exited = true;
            break;
          }
        }
        if (!exited && (minred == 1 || r.wl < a.wbegin || r.nbuff < 1)) blue = false;
      } else if (r.nbuff < 1) {
        blue = false;
      }
    } else {  // higher members with the merged-continuum taper (:3543-3606)
      if (r.wl <= a.wlend) {
        if (wcon > a.wlend) continue;
        if (a.wbegin <= r.alpha) {
          const double wave0 = a.wbegin * powi(a.ratio, minred - 1);
          if (wave0 >= wcon) {
            double k0 = prof(wave0);
            if (k0 >= (double)cont[min(minred, length) - 1] * CUTOFF) {
              k0 = taper(wave0, k0);
              if (lane == 0 && minred <= length) atomicAdd(acc + minred - 1, k0);
              for (int b0 = minred + 1; b0 <= length; b0 += 32) {
                const int ib = b0 + lane;
                const double wave = a.wbegin * powi(a.ratio, ib - 1);
                const bool ok = ib <= length && wave >= wcon;
                const double kappa = ok ? taper(wave, prof(wave)) : 0.0;
                const unsigned below = __ballot_sync(0xffffffffu, ok && kappa < (double)cont[ib - 1] * CUTOFF);
                const int stop = below ? __ffs(below) - 1 : 32;
                if (ok && lane <= stop) atomicAdd(acc + ib - 1, kappa);
                if (below) break;
              }
            }
          }
          if (minred == 1) continue;
        }
        if (r.wl < a.wbegin) continue;
      }
    }
    if (!blue) continue;
    // blue wing (:3499-3508, :3531-3541, :3592-3605): add, then stop below the
    // continuum cutoff; higher members also stop (not added) blueward of WCON
    const int ib0 = min(length + 1, r.nbuff), maxblue = ib0 - 1;
    for (int s0 = 1; s0 <= maxblue; s0 += 32) {
      const int s = s0 + lane, ib = ib0 - s;
      const bool valid = s <= maxblue;
      const double wave = a.wbegin * powi(a.ratio, ib - 1);
      const bool edge = valid && r.variant == 2 && wave < wcon;
      const double kappa = (valid && !edge) ? taper(wave, prof(wave)) : 0.0;
      const unsigned eb = __ballot_sync(0xffffffffu, edge);
      const unsigned below = __ballot_sync(0xffffffffu, valid && !edge && kappa < (double)cont[ib - 1] * CUTOFF);
      const int first_edge = eb ? __ffs(eb) - 1 : 32, first_below = below ? __ffs(below) - 1 : 32;
      if (valid && !edge && lane < first_edge && lane <= first_below) atomicAdd(acc + ib - 1, kappa);
      if (eb || below) break;
    }
  }
}

}  // namespace atlasgpu
