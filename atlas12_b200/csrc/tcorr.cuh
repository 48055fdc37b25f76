// tcorr.cuh -- end of an ATLAS12 iteration on the device: ROSS(3), RADIAP(3)
// and the radiative branch of TCORR(3) with TTAUP's RHOX correction and the
// remap onto the standard Rosseland grid.  One CTA per model: a 72-depth
// serial recurrence (atlas12_modules.f90 :5193-5198, :5108-5135, :2528-2977,
// :6303-6523) run by one thread on shared-memory copies of the model, and the
// two TTAUP integrations run side by side with their ROSSTAB searches split
// over a thread group.  Keeping it on the device lets a whole iteration run
// as one captured CUDA graph.
//
// Radiative branch: IFCONV = 0 (no CONVEC, CNVFLX = 0, CZ_CONSTRUCT returns
// at once), no smoothing (J1SMOOTH = 0), USE_DTGRAD = .FALSE.  TTAUP's
// opacities come from ROSSTAB, the model's own kappa_R history.
#pragma once
#include "common.cuh"
#include "josh.cuh"

namespace atlasgpu {

constexpr double kSigmaSB = 5.670374419e-5;
constexpr int kAcc8 = 8;  // mode-2 sums per depth (RJMINS ... ABROSS), then PRADK0

// ---- serial numerics (one thread) -------------------------------------
__device__ inline void s_parcoe(const double* f, const double* x, double* a, double* b, double* c,
                                int n) {
  c[0] = 0.0;
  b[0] = (f[1] - f[0]) / (x[1] - x[0]);
  a[0] = f[0] - x[0] * b[0];
  c[n - 1] = 0.0;
  b[n - 1] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
  a[n - 1] = f[n - 1] - x[n - 1] * b[n - 1];
  for (int j = 1; j <= n - 2; ++j) {
    if (j <= 2) {
      c[j] = 0.0;
      b[j] = (f[j + 1] - f[j]) / (x[j + 1] - x[j]);
      a[j] = f[j] - x[j] * b[j];
    } else {
      const double d = (f[j] - f[j - 1]) / (x[j] - x[j - 1]);
      c[j] = f[j + 1] / ((x[j + 1] - x[j]) * (x[j + 1] - x[j - 1])) -
             f[j] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j])) +
             f[j - 1] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j - 1]));
      b[j] = d - (x[j] + x[j - 1]) * c[j];
      a[j] = f[j - 1] - x[j - 1] * d + x[j] * x[j - 1] * c[j];
    }
  }
  for (int j = 1; j <= n - 2; ++j) {
    if (c[j] != 0.0) {
      const double wt = fabs(c[j + 1]) / (fabs(c[j + 1]) + fabs(c[j]));
      a[j] = a[j + 1] + wt * (a[j] - a[j + 1]);
      b[j] = b[j + 1] + wt * (b[j] - b[j + 1]);
      c[j] = c[j + 1] + wt * (c[j] - c[j + 1]);
    }
  }
  a[n - 2] = a[n - 1];
  b[n - 2] = b[n - 1];
  c[n - 2] = c[n - 1];
}

__device__ inline void s_integ(const double* x, const double* f, double* fint, int n, double start,
                               double* wa, double* wb, double* wc) {
  s_parcoe(f, x, wa, wb, wc, n);
  fint[0] = start;
  for (int i = 0; i < n - 1; ++i) {
    const double xlo = x[i], xhi = x[i + 1];
    fint[i + 1] = fint[i] + (wa[i] + wb[i] * 0.5 * (xhi + xlo) +
                             wc[i] / 3.0 * ((xhi + xlo) * xhi + xlo * xlo)) * (xhi - xlo);
  }
}

__device__ inline void s_deriv(const double* x, const double* f, double* d, int n) {
  d[0] = (f[1] - f[0]) / (x[1] - x[0]);
  d[n - 1] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
  if (n == 2) return;
  const double s = fabs(x[1] - x[0]) / (x[1] - x[0]);
  for (int j = 1; j <= n - 2; ++j) {
    double scale = fmax(fmax(fabs(f[j - 1]), fabs(f[j])), fabs(f[j + 1])) / fabs(x[j]);
    if (scale == 0.0) scale = 1.0;
    const double dr = (f[j + 1] - f[j]) / (x[j + 1] - x[j]) / scale;
    const double dl = (f[j] - f[j - 1]) / (x[j] - x[j - 1]) / scale;
    const double tr = dr / (s * sqrt(1.0 + dr * dr) + 1.0);
    const double tl = dl / (s * sqrt(1.0 + dl * dl) + 1.0);
    d[j] = (tr + tl) / (1.0 - tr * tl) * scale;
  }
}

// MAP1 as a sequential walk (1-based L as in the reference)
__host__ __device__ inline int s_map1(const double* xo, const double* fo, int nold, const double* xn,
                             double* fn, int nnew) {
#define XO(i) xo[(i)-1]
#define FO(i) fo[(i)-1]
  double A = 0, B = 0, C = 0, ab = 0, bb = 0, cb = 0, af = 0, bf = 0, cf = 0;
  int L = 2, LL = 0;
  for (int k = 0; k < nnew; ++k) {
    bool past = false;
    while (xn[k] >= XO(L)) {
      L = L + 1;
      if (L > nold) {
        past = true;
        break;
      }
    }
    if (!past && L == LL) {
      fn[k] = A + (B + C * xn[k]) * xn[k];
      continue;
    }
    if (L <= 3 || past) {
      L = L < nold ? L : nold;
      if (!past && L == LL) {
        fn[k] = A + (B + C * xn[k]) * xn[k];
        continue;
      }
      C = 0.0;
      B = (FO(L) - FO(L - 1)) / (XO(L) - XO(L - 1));
      A = FO(L) - XO(L) * B;
      LL = L;
      fn[k] = A + B * xn[k];
      continue;
    }
    const int l1 = L - 1;
    if (L == LL + 1 && L != 3 && L != 4) {
      cb = cf;
      bb = bf;
      ab = af;
    } else {
      const int l2 = L - 2;
      const double d = (FO(l1) - FO(l2)) / (XO(l1) - XO(l2));
      cb = FO(L) / ((XO(L) - XO(l1)) * (XO(L) - XO(l2))) +
           (FO(l2) / (XO(L) - XO(l2)) - FO(l1) / (XO(L) - XO(l1))) / (XO(l1) - XO(l2));
      bb = d - (XO(l1) + XO(l2)) * cb;
      ab = FO(l2) - XO(l2) * d + XO(l1) * XO(l2) * cb;
    }
    if (L >= nold) {
      A = ab;
      B = bb;
      C = cb;
      LL = L;
      fn[k] = A + (B + C * xn[k]) * xn[k];
      continue;
    }
    const double d = (FO(L) - FO(l1)) / (XO(L) - XO(l1));
    cf = FO(L + 1) / ((XO(L + 1) - XO(L)) * (XO(L + 1) - XO(l1))) +
         (FO(l1) / (XO(L + 1) - XO(l1)) - FO(L) / (XO(L + 1) - XO(L))) / (XO(L) - XO(l1));
    bf = d - (XO(L) + XO(l1)) * cf;
    af = FO(l1) - XO(l1) * d + XO(L) * XO(l1) * cf;
    double wt = 0.0;
    if (fabs(cf) != 0.0) wt = fabs(cf) / (fabs(cf) + fabs(cb));
    A = af + wt * (ab - af);
    B = bf + wt * (bb - bf);
    C = cf + wt * (cb - cf);
    LL = L;
    fn[k] = A + (B + C * xn[k]) * xn[k];
  }
  return LL - 1;
#undef XO
#undef FO
}

// ROSSTAB (atlas12_modules.f90:5937-6228, IROSSTAB = 1): the model's own
// (normalised log T, log P, log10 kappa_R) history, appended after every ROSS(3)
struct RossStore {
  int n, maxtab;
  double zerot, slopet, zerop, slopep;
  double *t, *p, *k;  // [maxtab]
};

// ROSSTAB(0,0,0): one thread
__device__ inline void s_rosstab_store(RossStore& R, const double* t, const double* p,
                                       const double* abross, int n) {
  if (R.n == 0) {
    R.zerot = log10(t[0]);
    R.zerop = log10(p[0]);
    R.slopet = log10(t[n - 1]) - R.zerot;
    R.slopep = log10(p[n - 1]) - R.zerop;
  }
  for (int j = 0; j < n; ++j) {
    if (R.n + 1 > R.maxtab) break;
    R.t[R.n] = (log10(t[j]) - R.zerot) / R.slopet;
    R.p[R.n] = (log10(p[j]) - R.zerop) / R.slopep;
    R.k[R.n] = log10(abross[j]);
    R.n = R.n + 1;
  }
}
// ---- the finish as one CTA ---------------------------------------------
// kFinThreads threads: thread 0 runs the serial recurrences on shared-memory
// copies of the model; the two TTAUP integrations (current and corrected
// T) run at the same time, one per group of kFinGroup threads, each ROSSTAB
// lookup split across its group.  Every thread of a group runs TTAUP's
// control flow on identical values (a lookup's result is folded in the same
// order by every thread), so the groups need no broadcast of scalars.
constexpr int kFinThreads = 512;
constexpr int kFinGroup = 256;
constexpr int kFinGroupWarps = kFinGroup / 32;
constexpr int kFinVec = 17;   // model vectors kept on chip
constexpr int kFinWork = 26;  // scratch vectors

// per-group fold buffer of the per-warp quadrant minima (double-buffered so
// that one barrier per lookup suffices)
struct FinFold {
  double r[2][kFinGroupWarps][4];
  int i[2][kFinGroupWarps][4];
};

// shared-memory bytes of b_atlas_finish for kw depths and cap ROSSTAB points
__host__ __device__ inline size_t fin_smem_bytes(int kw, int cap) {
  return sizeof(double) * ((size_t)(kFinVec + kFinWork + kAcc8) * kw + 1 + 3 * (size_t)cap) +
         2 * sizeof(FinFold) + sizeof(JoshWS) + 64;
}

__device__ __forceinline__ void group_bar(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kFinGroup) : "memory");
}

// lexicographic (r2, index) minimum: the sequential scan keeps the first minimum
__device__ __forceinline__ void wmin2(double& r, int& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double orr = __shfl_xor_sync(0xffffffffu, r, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (orr < r || (orr == r && oi < i)) {
      r = orr;
      i = oi;
    }
  }
}

// ROSSTAB(T, P, V) lookup (atlas12_modules.f90:5937-6228): nearest stored point
// in each (log T, log P) quadrant, bilinear blend of the four (inverse-
// distance weights when a quadrant is empty).  R's arrays are in shared
// memory; every thread of the group returns the value.
struct RossView {
  int n;
  double zerot, slopet, zerop, slopep;
  const double *t, *p, *k;
};

// tl = (log10 T - zerot) / slopet, hoisted by the caller (T is fixed per depth)
__device__ inline double b_rosstab(const RossView& R, double tl, double pres, int gtid, FinFold& fold,
                                   int& parity, int bar) {
  const double pl = (log10(pres) - R.zerop) / R.slopep;
  double r[4] = {1e30, 1e30, 1e30, 1e30};  // PP, PM, MP, MM
  int id[4] = {1 << 30, 1 << 30, 1 << 30, 1 << 30};
  for (int i = gtid; i < R.n; i += kFinGroup) {
    const double dt = R.t[i] - tl, dp = R.p[i] - pl;
    const double r2 = dt * dt + dp * dp;
    const int q = (dt >= 0.0) ? (dp >= 0.0 ? 0 : 1) : (dp >= 0.0 ? 2 : 3);
    if (r2 < r[q]) {
      r[q] = r2;
      id[q] = i + 1;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) wmin2(r[q], id[q]);
  const int w = gtid >> 5;
  if ((gtid & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      fold.r[parity][w][q] = r[q];
      fold.i[parity][w][q] = id[q];
    }
  }
  group_bar(bar);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double rr = fold.r[parity][0][q];
    int ii = fold.i[parity][0][q];
    for (int v = 1; v < kFinGroupWarps; ++v) {
      const double orr = fold.r[parity][v][q];
      const int oi = fold.i[parity][v][q];
      if (orr < rr || (orr == rr && oi < ii)) {
        rr = orr;
        ii = oi;
      }
    }
    r[q] = rr;
    id[q] = ii == (1 << 30) ? 0 : ii;
  }
  parity ^= 1;
  double res;
  if (id[0] && id[1] && id[2] && id[3]) {
    const double Tpp = R.t[id[0] - 1], Ppp = R.p[id[0] - 1], Rpp = R.k[id[0] - 1];
    const double Tpm = R.t[id[1] - 1], Ppm = R.p[id[1] - 1], Rpm = R.k[id[1] - 1];
    const double Tmp = R.t[id[2] - 1], Pmp = R.p[id[2] - 1], Rmp = R.k[id[2] - 1];
    const double Tmm = R.t[id[3] - 1], Pmm = R.p[id[3] - 1], Rmm = R.k[id[3] - 1];
    const double rhi = ((tl - Tmp) * Rpp + (Tpp - tl) * Rmp) / (Tpp - Tmp);
    const double phi = ((tl - Tmp) * Ppp + (Tpp - tl) * Pmp) / (Tpp - Tmp);
    const double rlo = ((tl - Tmm) * Rpm + (Tpm - tl) * Rmm) / (Tpm - Tmm);
    const double plo = ((tl - Tmm) * Ppm + (Tpm - tl) * Pmm) / (Tpm - Tmm);
    res = ((pl - plo) * rhi + (phi - pl) * rlo) / (phi - plo);
  } else {
    double d[4], rwt = 0.0, num = 0.0;
    for (int q = 0; q < 4; ++q) d[q] = sqrt(r[q]) + 1.0e-5;
    for (int q = 0; q < 4; ++q) rwt += 1.0 / d[q];
    for (int q = 0; q < 4; ++q) num += R.k[(id[q] > 1 ? id[q] : 1) - 1] / d[q];
    res = num / rwt;
  }
  return exp10(res);
}

// TTAUP (atlas12_modules.f90:6303-6523; radiative: P_turb = 0) by one group.
// Values are carried in registers; thread 0 of the group stores the outputs.
__device__ inline void b_ttaup(const RossView& R, double g, const double* tin, const double* tau,
                               double* abstd, double* ptotal, double* pout, const double* prad, int n,
                               int gtid, FinFold& fold, int bar) {
  const double RELAX[4] = {0.5, 0.3, 0.1, 0.05};
  int parity = 0;
  const double dlgtau = log(tau[1] / tau[0]);
  const double prad0 = prad[0];
  double plog1 = 0, plog2 = 0, plog3 = 0, plog4 = 0, dplog1 = 0, dplog2 = 0, dplog3 = 0;
  double plog = 0, dplog = 0;
  double ab0 = 0.1;  // ABSTD(1)
  if (prad0 > 0.0) ab0 = fmin(0.1, g * tau[0] / prad0 / 2.0);
  double ab1init = ab0;
  for (int J = 1; J <= n; ++J) {
    const int j = J - 1;
    const double tj = tin[j], tauj = tau[j], pradj = prad[j];
    const double tlj = (log10(tj) - R.zerot) / R.slopet;
    double ptj = 0.0, poj = 0.0, abj = 0.0;
    if (J == 1) plog = log(g / ab0 * tau[0]);
    else if (J <= 4) plog = plog1 + dplog1;
    else plog = (3.0 * plog4 + 8.0 * dplog1 - 4.0 * dplog2 + 8.0 * dplog3) / 3.0;
    double err = 1.0, perr = 1.0, best_err = 1.0e308, best_plog = plog;
    int N = 0, nstall = 0, rl = 1;
    bool conv = false;
    for (;;) {  // bounded: exits at N = 50
      ptj = exp(plog);
      poj = ptj + (prad0 - pradj);
      if (poj <= 0.0) {
        poj = ptj * 1.0e-4;
        if (poj <= 0.0) poj = 1.0e-10;
      }
      abj = b_rosstab(R, tlj, poj, gtid, fold, parity, bar);
      if (J == 1) ab0 = abj;
      dplog = g / abj * tauj / ptj * dlgtau;
      dplog = fmax(0.0, fmin(10.0, dplog));
      N = N + 1;
      if (N == 1) continue;
      double pnew;
      if (J == 1) pnew = log(g / ab0 * tau[0]);
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
      if (N > 3 && err > 0.9 * perr) {
        nstall = nstall + 1;
        if (nstall >= 4 && rl < 4) {
          rl = rl + 1;
          nstall = 0;
        }
      } else {
        nstall = nstall - 1 > 0 ? nstall - 1 : 0;
      }
      const double relax = RELAX[rl - 1];
      plog = (1.0 - relax) * plog + relax * pnew;
      if (err <= 1.0e-4) {
        conv = true;
        break;
      }
      if (N >= 50) break;
    }
    if (!conv) {
      plog = best_plog;
      ptj = exp(plog);
      poj = ptj + (prad0 - pradj);
      if (poj <= 0.0) poj = fmax(ptj * 1.0e-4, 1.0e-10);
      abj = b_rosstab(R, tlj, poj, gtid, fold, parity, bar);
      if (J == 1) ab0 = abj;
      dplog = g / abj * tauj / ptj * dlgtau;
      dplog = fmax(0.0, fmin(10.0, dplog));
    }
    if (J == 1 && (ab0 / ab1init > 2.0 || ab1init / ab0 > 2.0)) {
      ab1init = ab0;
      plog = log(g / ab0 * tau[0]);
      ptj = exp(plog);
      poj = ptj;
      if (poj > 0.0) {
        ab0 = b_rosstab(R, (log10(tin[0]) - R.zerot) / R.slopet, poj, gtid, fold, parity, bar);
        abj = ab0;
        plog = log(g / ab0 * tau[0]);
        ptj = exp(plog);
        poj = ptj;
      }
      dplog = g / ab0 * tau[0] / ptj * dlgtau;
      dplog = fmax(0.0, fmin(10.0, dplog));
    }
    if (gtid == 0) {
      abstd[j] = abj;
      ptotal[j] = ptj;
      pout[j] = poj;
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

// Model state of one atmosphere, device pointers to [kw] vectors
struct ModelState {
  double *t, *rhox, *p, *xne, *abross, *prad, *vturb, *pturb, *tauros, *accrad, *raden, *oldt1;
  double *flxerr, *dtflux, *dtlamb, *dtsurf, *t1;
  double pradk0;
  double maxerr;
};

// finish one iteration.  gacc = the reduced mode-2 sums [kAcc*kw + 1] (order
// rjmins, rdabh, rdiagj, flxrad, raden, h_total, accrad, abross, pradk0;
// rdabh is updated in place as TCORR(3) does); gms / gR in device memory,
// updated in place.  Launched with kFinThreads threads and
// fin_smem_bytes(kw, gR->maxtab) bytes of dynamic shared memory (smem).
// Returns max |FLXERR| (percent) to every thread.
__device__ inline double b_atlas_finish(ModelState* gms, double* gacc, int kw, int n, int iter, double teff,
                                        double grav, RossStore* gR, double* smem) {
  const int tid = threadIdx.x;
  const double FOUR_SIGMA_OVER_PI = 4.0 * kSigmaSB / kPi;
  const double FOURPI_OVER_C = 4.0 * kPi / kClight;
  const double FLUX = kSigmaSB * powi(teff, 4) / (4.0 * kPi);
  const int cap = gR->maxtab;
  // shared-memory layout
  double* V = smem;                           // [kFinVec][kw]
  double* acc = V + kFinVec * kw;             // [kAcc8*kw + 1]
  double* work = acc + kAcc8 * kw + 1;        // [kFinWork][kw]
  double* rt = work + kFinWork * kw;          // ROSSTAB [3][cap]
  double* rp = rt + cap;
  double* rk = rp + cap;
  FinFold* fold = reinterpret_cast<FinFold*>(rk + cap);  // [2]
  __shared__ double s_scal[8];  // zerot, slopet, zerop, slopep, maxerr, pradk0
  __shared__ int s_n[2];        // ROSSTAB points before / after the store
  double* gv[kFinVec] = {gms->t, gms->rhox, gms->p, gms->xne, gms->abross, gms->prad, gms->vturb, gms->pturb,
                         gms->tauros, gms->accrad, gms->raden, gms->oldt1, gms->flxerr, gms->dtflux,
                         gms->dtlamb, gms->dtsurf, gms->t1};
  const int n0 = gR->n;
  for (int e = tid; e < kFinVec * n; e += blockDim.x) V[(e / n) * kw + e % n] = gv[e / n][e % n];
  for (int e = tid; e < kAcc8 * kw + 1; e += blockDim.x) acc[e] = gacc[e];
  for (int e = tid; e < n0; e += blockDim.x) {
    rt[e] = gR->t[e];
    rp[e] = gR->p[e];
    rk[e] = gR->k[e];
  }
  __syncthreads();
  ModelState s;
  double** f[kFinVec] = {&s.t, &s.rhox, &s.p, &s.xne, &s.abross, &s.prad, &s.vturb, &s.pturb, &s.tauros,
                         &s.accrad, &s.raden, &s.oldt1, &s.flxerr, &s.dtflux, &s.dtlamb, &s.dtsurf, &s.t1};
  for (int q = 0; q < kFinVec; ++q) *f[q] = V + q * kw;
  double* rjmins = acc + 0 * kw;
  double* rdabh = acc + 1 * kw;
  double* rdiagj = acc + 2 * kw;
  double* flxrad = acc + 3 * kw;
  double* raden = acc + 4 * kw;
  double* h_total = acc + 5 * kw;
  double* accrad = acc + 6 * kw;
  double* abross = acc + 7 * kw;
  double* W[kFinWork];
  for (int q = 0; q < kFinWork; ++q) W[q] = work + q * kw;
  double *wa = W[0], *wb = W[1], *wc = W[2], *dtdrhx = W[3], *dabros = W[4], *codrhx = W[5],
         *G = W[6], *gflux = W[7], *dtau = W[8], *flxdrv = W[9], *dum = W[10], *tinteg = W[11],
         *tplus = W[12], *taustd = W[13], *tnew1 = W[14], *tnew2 = W[15], *prdnew = W[16],
         *ab1 = W[17], *pt1 = W[18], *p1 = W[19], *pt2 = W[20], *ppp = W[21], *rrr = W[22],
         *rmp = W[23], *ab2 = W[24], *p2 = W[25];
  JoshWS& jw = *reinterpret_cast<JoshWS*>(fold + 2);  // MAP1 / PARCOE scratch of warp 0
  if (tid < 32) {
    // warp 0: the recurrences of ROSS(3), RADIAP(3) and TCORR(3), depths over lanes
    WarpG w(tid);
    const int L = tid;
    double maxerr = 0.0;
    bool nonfinite = false;
    // ROSS(3)
    for (int j = L; j < n; j += 32) s.abross[j] = FOUR_SIGMA_OVER_PI * powi(s.t[j], 3) / abross[j];
    w.sync();
    g_integ(w, s.rhox, s.abross, s.tauros, n, s.abross[0] * s.rhox[0], jw);
    RossStore R{n0, cap, gR->zerot, gR->slopet, gR->zerop, gR->slopep, rt, rp, rk};
    if (L == 0) s_rosstab_store(R, s.t, s.p, s.abross, n);  // RX = ROSSTAB(0,0,0), atlas12c.f90:586
    // RADIAP(3)
    double errormax = 0.0;
    for (int j = L; j < n; j += 32) {
      s.raden[j] = raden[j] * FOURPI_OVER_C;
      s.accrad[j] = accrad[j] * FOURPI_OVER_C;
      if (h_total[j] / FLUX > 1.0) s.accrad[j] = s.accrad[j] * FLUX / h_total[j];
      errormax = fmax(errormax, h_total[j] / FLUX);
    }
    errormax = w.max(errormax);
    double pradk0 = acc[kAcc8 * kw] * FOURPI_OVER_C;
    if (errormax > 1.0) pradk0 = pradk0 / errormax;
    w.sync();
    g_integ(w, s.rhox, s.accrad, s.prad, n, s.accrad[0] * s.rhox[0], jw);
    // TCORR(3)
    g_deriv(w, s.rhox, s.t, dtdrhx, n);
    g_deriv(w, s.rhox, s.abross, dabros, n);
    for (int j = L; j < n; j += 32) {
      rdabh[j] = rdabh[j] - flxrad[j] * dabros[j] / fmax(s.abross[j], 1.0e-30);
      codrhx[j] = (rdabh[j] + 0.0) / (flxrad[j] + 0.0);
    }
    w.sync();
    if (L == 0) {
      codrhx[0] = 0.0;
      codrhx[1] = 0.0;
    }
    w.sync();
    g_integ(w, s.rhox, codrhx, G, n, 0.0, jw);
    for (int j = L; j < n; j += 32) {
      G[j] = exp(G[j]);
      gflux[j] = G[j] * (flxrad[j] + 0.0 - FLUX) / (flxrad[j] + 0.0);
    }
    w.sync();
    g_integ(w, s.tauros, gflux, dtau, n, 0.0, jw);
    const double MAX_DT = 0.04 * teff;
    for (int j = L; j < n; j += 32) {
      dtau[j] = dtau[j] / G[j];
      dtau[j] = fmax(-s.tauros[j] / 3.0, fmin(s.tauros[j] / 3.0, dtau[j]));
      s.dtflux[j] = -dtau[j] * dtdrhx[j] / fmax(s.abross[j], 1.0e-30);
      s.flxerr[j] = (flxrad[j] + 0.0 - FLUX) / FLUX * 100.0;
      maxerr = fmax(maxerr, fabs(s.flxerr[j]));
      nonfinite |= !(fabs(s.flxerr[j]) <= 1.0e308);
    }
    maxerr = w.max(maxerr);
    // fmax drops NaN: a non-finite FLXERR anywhere makes the metric NaN
    if (__any_sync(0xffffffffu, nonfinite)) maxerr = __longlong_as_double(0x7ff8000000000000ll);
    w.sync();
    g_deriv(w, s.tauros, s.flxerr, flxdrv, n);
    for (int j = L; j < n; j += 32) {
      // HRATIO = 0 in radiative layers: FLXDRV from the thermal imbalance
      flxdrv[j] = rjmins[j] / fmax(s.abross[j], 1.0e-30) / FLUX * 100.0;
      double d = -flxdrv[j] * FLUX / 100.0 / fmax(fabs(rdiagj[j]), 1.0e-30) * copysign(1.0, rdiagj[j]) *
                 fmax(s.abross[j], 1.0e-30);
      s.dtlamb[j] = fmax(-MAX_DT, fmin(MAX_DT, d));
      dum[j] = s.dtflux[j] + s.dtlamb[j];
    }
    w.sync();
    double dtsur = (FLUX - flxrad[0]) / FLUX * 0.25 * s.t[0];
    dtsur = fmax(-MAX_DT, fmin(MAX_DT, dtsur));
    g_integ(w, s.tauros, dum, tinteg, n, 0.0, jw);
    if (L == 0) {
      double xq = 0.1, tone, ttwo;
      s_map1(s.tauros, tinteg, n, &xq, &tone, 1);
      xq = 2.0;
      s_map1(s.tauros, tinteg, n, &xq, &ttwo, 1);
      double tav = (ttwo - tone) / 2.0;
      if (dtsur * tav <= 0.0) tav = 0.0;
      if (fabs(tav) > fabs(dtsur)) tav = dtsur;
      jw.red[0] = dtsur - tav;
    }
    w.sync();
    dtsur = jw.red[0];
    for (int j = L; j < n; j += 32) {
      s.dtsurf[j] = dtsur;
      double t1 = s.dtflux[j] + s.dtlamb[j] + dtsur;
      if (iter == 1) {
      } else if (s.oldt1[j] * t1 > 0.0 && fabs(s.oldt1[j]) > fabs(t1)) {
        t1 = t1 * 1.25;
      } else if (s.oldt1[j] * t1 < 0.0) {
        t1 = t1 * 0.5;
      }
      s.oldt1[j] = t1;
      s.t1[j] = t1;
      tplus[j] = s.t[j] + t1;
      taustd[j] = exp10(-6.875 + (double)j * 0.125);
    }
    w.sync();
    g_map1(w, s.tauros, s.t, n, taustd, tnew1, n, jw.lidx);
    g_map1(w, s.tauros, s.prad, n, taustd, prdnew, n, jw.lidx);
    g_map1(w, s.tauros, tplus, n, taustd, tnew2, n, jw.lidx);
    if (L == 0) {
      s_scal[0] = R.zerot;
      s_scal[1] = R.slopet;
      s_scal[2] = R.zerop;
      s_scal[3] = R.slopep;
      s_scal[4] = maxerr;
      s_scal[5] = pradk0;
      s_n[0] = n0;
      s_n[1] = R.n;
    }
  }
  __syncthreads();
  {
    const RossView RV{s_n[1], s_scal[0], s_scal[1], s_scal[2], s_scal[3], rt, rp, rk};
    const int grp = tid / kFinGroup, gtid = tid % kFinGroup;
    if (grp == 0) b_ttaup(RV, grav, tnew1, taustd, ab1, pt1, p1, prdnew, n, gtid, fold[0], 1);
    else if (grp == 1) b_ttaup(RV, grav, tnew2, taustd, ab2, pt2, p2, prdnew, n, gtid, fold[1], 2);
  }
  __syncthreads();
  if (tid < 32) {
    WarpG w(tid);
    const int L = tid;
    for (int j = L; j < n; j += 32) ppp[j] = (pt2[j] - pt1[j]) / pt1[j];
    w.sync();
    g_map1(w, taustd, ppp, n, s.tauros, rrr, n, jw.lidx);
    for (int j = L; j < n; j += 32) s.t[j] = s.t[j] + s.t1[j];
    w.sync();
    if (L == 0) {
      // monotone T from the bottom up, then the 1200 K floor
      for (int i = 2; i <= n; ++i) {
        const int jj = n + 1 - i;
        s.t[jj - 1] = fmin(s.t[jj - 1], s.t[jj] - 1.0);
      }
    }
    w.sync();
    for (int j = L; j < n; j += 32) {
      s.t[j] = fmax(s.t[j], 1200.0);
      s.rhox[j] = s.rhox[j] + rrr[j] * s.rhox[j];
    }
    w.sync();
    double* src[8] = {s.rhox, s.t, s.p, s.xne, s.abross, s.prad, s.vturb, s.pturb};
    const double ab_surf = s.abross[0];
    for (int q = 0; q < 8; ++q) {
      g_map1(w, s.tauros, src[q], n, taustd, rmp, n, jw.lidx);
      for (int j = L; j < n; j += 32) {
        double v = rmp[j];
        if (q == 4 && s.tauros[0] > taustd[j] && v < 0.0) v = ab_surf;
        src[q][j] = v;
      }
      w.sync();
    }
    for (int j = L; j < n; j += 32) s.tauros[j] = taustd[j];
    if (L == 0) {
      gms->pradk0 = s_scal[5];
      gms->maxerr = s_scal[4];
      gR->n = s_n[1];
      gR->zerot = s_scal[0];
      gR->slopet = s_scal[1];
      gR->zerop = s_scal[2];
      gR->slopep = s_scal[3];
    }
  }
  __syncthreads();
  // write back the model, TCORR's RDABH and the new ROSSTAB points
  for (int e = tid; e < kFinVec * n; e += blockDim.x) gv[e / n][e % n] = V[(e / n) * kw + e % n];
  for (int e = tid; e < n; e += blockDim.x) gacc[kw + e] = rdabh[e];
  for (int e = s_n[0] + tid; e < s_n[1]; e += blockDim.x) {
    gR->t[e] = rt[e];
    gR->p[e] = rp[e];
    gR->k[e] = rk[e];
  }
  return s_scal[4];
}

}  // namespace atlasgpu
