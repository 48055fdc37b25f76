// hydrogen.cuh -- the hydrogen line profile HPROF4 (atlas12_modules.f90:
// 20553-21002) with STARK_PROFILE (:20376-20514) and HFNM (:20263-20305) as
// device functions, and XLINOP's hydrogen lines (TYPE -1, :20177-20199): a
// warp per (record, depth), 32 wing points per step, FP64 atomics into
// XLINES.  The tables are the caller's (atlasgpu_hydrogen_tables).
#pragma once
#include "atlas.cuh"
#include "common.cuh"

namespace atlasgpu {

__device__ inline double hfnm(int n, int m) {
  if (m <= n) return 0.0;
  const double xn = (double)n;
  const double ginf = 0.2027 / pow(xn, 0.71);
  const double gca = 0.124 / xn;
  const double fkn = xn * 1.9603;
  const double wtc = 0.45 - 2.4 / powi(xn, 3) * (xn - 1.0);
  const double xm = (double)m, xmn = (double)(m - n);
  const double fk = fkn * powi(xm / (xmn * (xm + (double)n)), 3);
  const double xmn12 = pow(xmn, 1.2);
  const double wt = (xmn12 - 1.0) / (xmn12 + wtc);
  return fk * (1.0 - wt * ginf - (0.222 + gca / xm) * (1.0 - wt));
}

__device__ inline double stark_profile(const atlasgpu_hydrogen_tables& h, double b, double p, int n, int m) {
  int indx = 7;
  const int mmn = m - n;
  if (n <= 3 && mmn <= 2) indx = 2 * (n - 1) + mmn;
  const double b2 = b * b, sb = sqrt(b);
  if (b > 500.0) return (1.5 / sb + 27.0 / b2) / b2;
  int im = (int)(5.0 * p) + 1;
  if (im > 4) im = 4;
  if (im < 1) im = 1;  // P >= 0 for any atmosphere; keeps a NaN P inside PP
  const int ip = im + 1;
  const double wtpp = 5.0 * (p - h.pp[im - 1]);
  const double wtpm = 1.0 - wtpp;
  if (b > 25.12) {
    const double cc = h.c[indx - 1][ip - 1] * wtpp + h.c[indx - 1][im - 1] * wtpm;
    const double dd = h.d[indx - 1][ip - 1] * wtpp + h.d[indx - 1][im - 1] * wtpm;
    return (1.5 / sb + 27.0 / b2) / b2 * (1.0 + dd / (cc + b * sb));
  }
  int jm = 1;
  for (int j = 2; j <= 15; ++j)
    if (b <= h.betagrid[j - 1]) {
      jm = j - 1;
      break;
    }
  const int jp = jm + 1;
  const double wtbp = (b - h.betagrid[jm - 1]) / (h.betagrid[jp - 1] - h.betagrid[jm - 1]);
  const double wtbm = 1.0 - wtbp;
  const double cbp = h.propbm[indx - 1][jp - 1][ip - 1] * wtpp + h.propbm[indx - 1][jp - 1][im - 1] * wtpm;
  const double cbm = h.propbm[indx - 1][jm - 1][ip - 1] * wtpp + h.propbm[indx - 1][jm - 1][im - 1] * wtpm;
  const double corr = 1.0 + cbp * wtbp + cbm * wtbm;
  double wt = 0.5 * (10.0 - b);
  wt = wt < 1.0 ? wt : 1.0;
  wt = wt > 0.0 ? wt : 0.0;
  const double pr1 = b <= 10.0 ? 8.0 / (83.0 + (2.0 + 0.95 * b2) * b) : 0.0;
  const double pr2 = b >= 8.0 ? (1.5 / sb + 27.0 / b2) / b2 : 0.0;
  return (pr1 * wt + pr2 * (1.0 - wt)) * corr;
}

// HPROF4's depth vectors (Section 1) at one depth
struct HDepth {
  double xne, pp, fo, y1b, y1s, t3nhe, t3nh2, c1d, c2d, gcon1, gcon2;
  double xnf1, xnf2, xnfp1, dop1;
};

__device__ inline void hdepth(double xne, double t, double xnfp3, double xnh2, double xnf1, double xnf2,
                              double xnfp1, double dop1, HDepth& d) {
  const double xne16 = pow(xne, 1.0 / 6.0);
  d.xne = xne;
  d.pp = xne16 * 0.08989 / sqrt(t);
  d.fo = powi(xne16, 4) * 1.25e-9;
  d.y1b = 2.0 / (1.0 + 0.012 / t * sqrt(xne / t));
  const double t4 = t / 10000.0;
  const double t43 = pow(t4, 0.3);
  d.y1s = t43 / xne16;
  d.t3nhe = t43 * xnfp3;
  d.t3nh2 = t43 * xnh2;
  d.c1d = d.fo * 78940.0 / t;
  d.c2d = powi(d.fo, 2) / 5.96e-23 / xne;
  d.gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + xne / 1.0e13);
  d.gcon2 = 0.2 / (1.0 + xne / 1.0e15);
  d.xnf1 = xnf1;
  d.xnf2 = xnf2;
  d.xnfp1 = xnfp1;
  d.dop1 = dop1;
}

// HPROF4's line constants (Section 2)
struct HLine {
  int n, m, ifins;
  double xknm, freqnm, dbeta, wavenm, c1con, c2con, radamp, resont, vdw, starkc, y1num, y1wht;
  double finest[14], finswt[14];
};

__device__ inline void hline(const atlasgpu_hydrogen_tables& h, int n, int m, HLine& L) {
  const double freq_rydh = 109677.583403 * 2.99792458e10, clight_angs = 2.99792458e18;
  const int mmn = m - n;
  const double xn = (double)n, xn2 = xn * xn, xm = (double)m, xm2 = xm * xm;
  const double xmn2 = xm2 * xn2, xm2mn2 = xm2 - xn2, gnm = xm2mn2 / xmn2;
  L.n = n;
  L.m = m;
  L.xknm = (mmn <= 3 && n <= 4) ? h.xknmtb[n - 1][mmn - 1] : 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / (double)mmn);
  L.y1num = m == 2 ? 550.0 : m == 3 ? 380.0 : 320.0;
  L.y1wht = 1.0e13;
  if (mmn <= 3) L.y1wht = 1.0e14;
  if (mmn <= 2 && n <= 2) L.y1wht = h.y1wtm[n - 1][mmn - 1];
  L.freqnm = freq_rydh * gnm;
  L.dbeta = clight_angs / powi(L.freqnm, 2) / L.xknm;
  L.wavenm = clight_angs / L.freqnm;
  L.c1con = L.xknm / L.wavenm * gnm * xm2mn2;
  L.c2con = powi(L.xknm / L.wavenm, 2);
  double radamp = n == 1 ? h.asumlyman[m - 1] : h.asum[n - 1] + h.asum[m - 1];
  radamp = radamp / (4.0 * kPi);
  L.radamp = radamp / L.freqnm;
  double resont = hfnm(1, m) / xm / (1.0 - 1.0 / xm2);
  if (n != 1) resont = resont + hfnm(1, n) / xn / (1.0 - 1.0 / xn2);
  L.resont = resont * 3.92e-24 / gnm;
  L.vdw = 4.45e-26 / gnm * pow(xm2 * (7.0 * xm2 + 5.0), 0.4);
  L.starkc = 1.6678e-18 * L.freqnm * L.xknm;
  if (n > 4 || m > 10) {
    L.ifins = 1;
    L.finest[0] = 0.0;
    L.finswt[0] = 1.0;
  } else if (mmn != 1) {
    L.ifins = h.lncomp[n - 1];
    for (int i = 0; i < L.ifins; ++i) {
      L.finest[i] = h.stcomp[i][n - 1] * 1.0e7;
      L.finswt[i] = h.stcpwt[i][n - 1] / xn2;
    }
  } else {
    L.ifins = h.lnghal[n - 1];
    const int ipos = h.istal[n - 1];
    for (int i = 0; i < L.ifins; ++i) {
      L.finest[i] = h.stalph[ipos - 1 + i] * 1.0e7;
      L.finswt[i] = h.stwtal[ipos - 1 + i] / xn2 / 3.0;
    }
  }
}

// HPROF4(N, M, J, DELW), Section 3, in Voigt normalization
__device__ inline double hprof4(const atlasgpu_hydrogen_tables& h, const HLine& L, const HDepth& d, double delw) {
  const double c = 2.99792458e10, clight_angs = 2.99792458e18;
  const int n = L.n, m = L.m;
  const double freqnm = L.freqnm;
  const double delstark = -10.0 * delw / L.wavenm * freqnm;
  const double freq4 = clight_angs / (L.wavenm + delw * 10.0);
  const double del = fabs(freq4 - freqnm);
  const double hwstk = L.starkc * d.fo;
  const double hwvdw = L.vdw * d.t3nhe + 2.0 * L.vdw * d.t3nh2;
  const double hwrad = L.radamp;
  double hwres = L.resont * d.xnf1;
  double hwlor = hwres + hwvdw + hwrad;
  const int nwid = (d.dop1 >= hwstk && d.dop1 >= hwlor) ? 1 : (hwlor >= hwstk ? 2 : 3);
  double mx = d.dop1 > hwlor ? d.dop1 : hwlor;
  mx = mx > hwstk ? mx : hwstk;
  const bool core = fabs(del) <= freqnm * mx;
  const double dop = freqnm * d.dop1;
  double hp = 0.0;
  if (!core || nwid == 1) {
    for (int i = 0; i < L.ifins; ++i) {
      const double dd = fabs(freq4 - freqnm - L.finest[i]) / dop;
      if (dd <= 7.0) hp = hp + exp(-dd * dd) * L.finswt[i];
    }
    if (core) return hp;
  }
  if (!core || nwid == 2) {
    if (n == 1 && m == 2) {
      hwres = hwres * 4.0;
      hwlor = hwres + hwvdw + hwrad;
      const double hhw = freqnm * hwlor;
      double hprofres;
      if (freq4 > (82259.105 - 4000.0) * c) {
        hprofres = hwres * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
      } else {
        double cutoff = 0.0;
        if (freq4 >= 50000.0 * c) {
          const double spacing = 200.0 * c, f22000 = (82259.105 - 22000.0) * c;
          if (freq4 < f22000) {
            cutoff = (h.cutoffh2[1] - h.cutoffh2[0]) / spacing * (freq4 - f22000) + h.cutoffh2[0];
          } else {
            const int icut = min((int)((freq4 - f22000) / spacing), 89);  // in the table (the reference's exact-boundary case)
            const double cutfreq = (double)icut * spacing + f22000;
            cutoff = (h.cutoffh2[icut + 1] - h.cutoffh2[icut]) / spacing * (freq4 - cutfreq) + h.cutoffh2[icut];
          }
          cutoff = pow(10.0, cutoff - 14.0) * d.xnfp1 * 2.0 / c;
        }
        hprofres = cutoff * kSqrtPi * dop;
      }
      double hprofrad = hwrad * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
      if (freq4 <= 2.463e15) hprofrad = 0.0;
      double hprofvdw = hwvdw * freqnm / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
      if (freq4 < 1.8e15) hprofvdw = 0.0;
      hp = hp + (hprofres + hprofrad + hprofvdw);
    } else {
      const double hhw = freqnm * hwlor;
      hp = hp + hhw / kPi / (del * del + hhw * hhw) * kSqrtPi * dop;
    }
    if (core) return hp;
  }
  const double wty1 = 1.0 / (1.0 + d.xne / L.y1wht);
  const double y1scal = L.y1num * d.y1s * wty1 + d.y1b * (1.0 - wty1);
  const double c1 = d.c1d * L.c1con * y1scal;
  const double c2 = d.c2d * L.c2con;
  const double g1 = 6.77 * sqrt(c1);
  double lg = 0.2114 + log(sqrt(c2) / c1);
  lg = lg > 0.0 ? lg : 0.0;
  const double gnot = g1 * lg * (1.0 - d.gcon1 - d.gcon2);
  const double beta = fabs(delstark) / d.fo * L.dbeta;
  const double y1 = c1 * beta;
  const double y2 = c2 * beta * beta;
  double gam = gnot;
  if (!(y2 <= 1.0e-4 && y1 <= 1.0e-5)) {
    gam = g1 * (0.5 * exp(-(y1 < 80.0 ? y1 : 80.0)) + expi1(y1) - 0.5 * expi1(y2)) *
          (1.0 - d.gcon1 / (1.0 + powi(90.0 * y1, 3)) - d.gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1.0e-20) gam = 0.0;
  }
  double prqs = stark_profile(h, beta, d.pp, n, m);
  if (m <= 2) {
    prqs = prqs * 0.5;
    if (freq4 >= (82259.105 - 20000.0) * c) {
      if (freq4 > (82259.105 - 4000.0) * c) {
        const double beta4000 = 4000.0 * c / d.fo * L.dbeta;
        const double prqsp4000 = stark_profile(h, beta4000, d.pp, n, m) * 0.5 / d.fo * L.dbeta;
        const double cutoff4000 = pow(10.0, -11.07 - 14.0) / c * d.xnf2;
        hp = hp + cutoff4000 / prqsp4000 * prqs / d.fo * L.dbeta * kSqrtPi * dop;
      } else {
        const double f15000 = (82259.105 - 15000.0) * c, spacing = 100.0 * c;
        double cutoff;
        if (freq4 < f15000) {
          cutoff = (h.cutoffh2plus[1] - h.cutoffh2plus[0]) / spacing * (freq4 - f15000) + h.cutoffh2plus[0];
        } else {
          const int icut = min((int)((freq4 - f15000) / spacing), 109);  // in the table (exact-boundary case)
          const double cutfreq = (double)icut * spacing + f15000;
          cutoff = (h.cutoffh2plus[icut + 1] - h.cutoffh2plus[icut]) / spacing * (freq4 - cutfreq) + h.cutoffh2plus[icut];
        }
        cutoff = pow(10.0, cutoff - 14.0) / c * d.xnf2;
        hp = hp + cutoff * kSqrtPi * dop;
      }
    }
  }
  const double f = gam > 0.0 ? gam / kPi / (gam * gam + beta * beta) : 0.0;
  const double p1 = powi(0.9 * y1, 2);
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  return hp + (prqs * (1.0 + fns) + f) / d.fo * L.dbeta * kSqrtPi * dop;
}

struct XHydArgs {
  const atlasgpu_nlte_line* rec;
  const AtlasLine* lines;  // NU and NUCONT of every record (k_xlinop_prep)
  int64_t n;
  int nrhox, kw, numnu;
  const atlasgpu_hydrogen_tables* tab;
  const double* waveset;
  const double* tabcont;            // [nwave+1][kw]
  const double *xnfdop, *dopple;    // [nspec][kw]: species 1 (H I) rows
  const double* xnfp;               // [nspec][kw]: XNFP(J,1), XNFP(J,3)
  const double *xne, *hckt, *emerge;
  const double *t, *xnf1, *xnf2, *xnh2;
  const double* contx;              // CONTX(25,16) column-major
  double* xl;                       // XLINES(J, NU): [numnu][kw]
};

// XLINOP's hydrogen lines: CENTER = CGF * exp(-EH(NBLO)*HCKT(J)) * XNFDOP(J,1),
// red wing NU..NU+2000 skipping points blueward of WCON, blue wing down to
// NU-2000 stopping there; each point added, then the wing stops below TABCONT
static __global__ void __launch_bounds__(256) k_xlinop_hydrogen(XHydArgs a) {
  const int lane = threadIdx.x & 31;
  const atlasgpu_hydrogen_tables& h = *a.tab;
  const int64_t npairs = a.n * a.nrhox;
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = w0; p < npairs; p += nw) {
    const int64_t i = p / a.nrhox;
    const int j = (int)(p - i * a.nrhox);
    const atlasgpu_nlte_line r = a.rec[i];
    if (r.itype != -1) continue;
    const int n = r.nblo, m = r.nbup, ncon = r.ncon;
    const int nu = a.lines[i].nu, nucont = a.lines[i].nucont;
    if (nu >= a.numnu || n < 1 || m <= n || m > 100 || ncon < 1 || ncon > 25) continue;
    const double eh = n <= 10 ? h.eh[n - 1] : h.elim - 109677.583403 / powi((double)n, 2);
    const double tc = a.tabcont[(size_t)(nucont - 1) * a.kw + j];
    const double center = (double)r.gf * (exp(-eh * a.hckt[j]) * a.xnfdop[j]);
    if (center < tc) continue;
    const double wcon = 1.0e7 / (a.contx[ncon - 1] - a.emerge[j]);
    HLine L;
    hline(h, n, m, L);
    HDepth d;
    hdepth(a.xne[j], a.t[j], a.xnfp[(size_t)2 * a.kw + j], a.xnh2[j], a.xnf1[j], a.xnf2[j], a.xnfp[j], a.dopple[j],
           d);
    double* xl = a.xl + j;
    // red wing: points blueward of WCON are skipped, the walk goes on
    const int hi = min(nu + 2000, a.numnu);
    for (int iw0 = nu; iw0 <= hi; iw0 += 32) {
      const int iw = iw0 + lane;
      const bool in = iw <= hi && !(a.waveset[iw - 1] < wcon);
      double cv = 0.0;
      if (in) cv = center * hprof4(h, L, d, a.waveset[iw - 1] - r.wlvac);
      const unsigned below = __ballot_sync(0xffffffffu, in && cv < tc);
      const int stop = below ? __ffs(below) - 1 : 32;
      if (in && lane <= stop) atomicAdd(xl + (size_t)(iw - 1) * a.kw, cv);
      if (below) break;
    }
    // blue wing: the walk ends at the first point blueward of WCON (not added)
    // or after the first point below TABCONT (added)
    const int nb = min(2000, nu - 1);
    for (int s0 = 1; s0 <= nb; s0 += 32) {
      const int s = s0 + lane;
      const int iw = nu - s;
      const bool valid = s <= nb;
      const bool blue_of_edge = valid && a.waveset[iw - 1] < wcon;
      double cv = 0.0;
      if (valid && !blue_of_edge) cv = center * hprof4(h, L, d, a.waveset[iw - 1] - r.wlvac);
      const unsigned edge = __ballot_sync(0xffffffffu, blue_of_edge);
      const unsigned below = __ballot_sync(0xffffffffu, valid && !blue_of_edge && cv < tc);
      const int first_edge = edge ? __ffs(edge) - 1 : 32;
      const int first_below = below ? __ffs(below) - 1 : 32;
      const bool add = valid && !blue_of_edge && lane < first_edge && lane <= first_below;
      if (add) atomicAdd(xl + (size_t)(iw - 1) * a.kw, cv);
      if (edge || below) break;
    }
  }
}

}  // namespace atlasgpu
