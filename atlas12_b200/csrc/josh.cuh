// josh.cuh -- warp-cooperative JOSH radiative transfer (FP64) for sm_100a.
//
// One warp solves one frequency.  Depth vectors (<= kKwMax) and the 51x51
// scattering system live in the warp's shared-memory workspace; lanes split
// depths, grid points, matrix rows or columns.  Every routine restates the
// reference formula for each output element (atlas12_modules.f90):
//   PARCOE :5358-5434, INTEG :5293-5324, DERIV :5228-5266, MAP1 :5570-5692,
//   SOLVIT :5739-5847, JOSH :18398-18776.
// MAP1 is evaluated in parallel over output points: the sequential routine's
// only cross-point state is the bracketing interval and the reuse of the
// previous forward parabola as the next backward one, and both are recovered
// per point from the bracket indices of the neighbouring outputs, so each
// output gets the formula the sequential walk would have used.
// Running sums whose order decides later branches (the INTEG cumulative sum)
// are summed in the reference order by one lane.
#pragma once
#include "common.cuh"

namespace atlasgpu {

struct JoshWS {
  double A[kNx * kLd];  // scattering system, column-major, ld = kLd
  double xs[kNx], xsbar[kNx], xalpha[kNx], xw[kNx];
  double abtot[kKwMax], alpha[kKwMax], snubar[kKwMax], taunu[kKwMax];
  double t1[kKwMax], t2[kKwMax], t3[kKwMax];  // scratch (PARCOE a,b,c / terms)
  int lidx[kKwMax + 4];                       // MAP1 bracket indices
};

// Full-solution extras for IFSURF = 0 (ATLAS)
struct JoshWSFull {
  double snu[kKwMax], hnu[kKwMax], jmins[kKwMax], jnu[kKwMax], bnu[kKwMax];
  double knu1;
  int maxj;
};

__device__ __forceinline__ void wsync() { __syncwarp(0xffffffffu); }

// ---------------------------------------------------------------- PARCOE/INTEG
// Coefficients into (a, b, c); n >= 4 assumed (n = NRHOX >= 4 on the hot path).
__device__ inline void w_parcoe(const double* f, const double* x, double* a, double* b, double* c,
                                int n, int lane) {
  // steps 1-3: endpoints linear, j = 1, 2 linear, interior parabolic
  for (int j = lane; j < n; j += 32) {
    double aj, bj, cj;
    if (j == 0 || j == 1 || j == 2 || j == n - 1) {
      const int i0 = (j == n - 1) ? n - 2 : j;
      cj = 0.0;
      bj = (f[i0 + 1] - f[i0]) / (x[i0 + 1] - x[i0]);
      aj = f[j] - x[j] * bj;
    } else {
      const double d = (f[j] - f[j - 1]) / (x[j] - x[j - 1]);
      cj = f[j + 1] / ((x[j + 1] - x[j]) * (x[j + 1] - x[j - 1])) -
           f[j] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j])) +
           f[j - 1] / ((x[j] - x[j - 1]) * (x[j + 1] - x[j - 1]));
      bj = d - (x[j] + x[j - 1]) * cj;
      aj = f[j - 1] - x[j - 1] * d + x[j] * x[j - 1] * cj;
    }
    a[j] = aj;
    b[j] = bj;
    c[j] = cj;
  }
  wsync();
  // step 4: blend each interval with its right neighbour's unsmoothed fit
  double na[4], nb[4], nc[4];
  int cnt = 0;
  for (int j = lane; j < n; j += 32, ++cnt) {
    na[cnt] = a[j];
    nb[cnt] = b[j];
    nc[cnt] = c[j];
    if (j >= 1 && j <= n - 2 && c[j] != 0.0) {
      const double wt = fabs(c[j + 1]) / (fabs(c[j + 1]) + fabs(c[j]));
      na[cnt] = a[j + 1] + wt * (a[j] - a[j + 1]);
      nb[cnt] = b[j + 1] + wt * (b[j] - b[j + 1]);
      nc[cnt] = c[j + 1] + wt * (c[j] - c[j + 1]);
    }
  }
  wsync();
  cnt = 0;
  for (int j = lane; j < n; j += 32, ++cnt) {
    a[j] = na[cnt];
    b[j] = nb[cnt];
    c[j] = nc[cnt];
  }
  wsync();
  // step 5: penultimate interval takes the endpoint linear fit
  if (lane == 0) {
    a[n - 2] = a[n - 1];
    b[n - 2] = b[n - 1];
    c[n - 2] = c[n - 1];
  }
  wsync();
}

// fint = running parabolic integral of f over x, fint[0] = start
__device__ inline void w_integ(const double* x, const double* f, double* fint, int n, double start,
                               JoshWS& ws, int lane) {
  double *a = ws.t1, *b = ws.t2, *c = ws.t3;
  w_parcoe(f, x, a, b, c, n, lane);
  for (int i = lane; i < n - 1; i += 32) {
    const double xlo = x[i], xhi = x[i + 1];
    // reuse a[] for the interval terms after reading this interval's a,b,c
    const double term = (a[i] + b[i] * 0.5 * (xhi + xlo) +
                         c[i] / 3.0 * ((xhi + xlo) * xhi + xlo * xlo)) *
                        (xhi - xlo);
    b[i] = term;
  }
  wsync();
  if (lane == 0) {
    double s = start;
    fint[0] = s;
    for (int i = 0; i < n - 1; ++i) {
      s = s + b[i];
      fint[i + 1] = s;
    }
  }
  wsync();
}

// ---------------------------------------------------------------- DERIV
__device__ inline void w_deriv(const double* x, const double* f, double* dfdx, int n, int lane) {
  const double s = fabs(x[1] - x[0]) / (x[1] - x[0]);
  double v[4];
  int cnt = 0;
  for (int j = lane; j < n; j += 32, ++cnt) {
    if (j == 0) {
      v[cnt] = (f[1] - f[0]) / (x[1] - x[0]);
    } else if (j == n - 1) {
      v[cnt] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
    } else {
      double scale = fmax(fmax(fabs(f[j - 1]), fabs(f[j])), fabs(f[j + 1])) / fabs(x[j]);
      if (scale == 0.0) scale = 1.0;
      const double dr = (f[j + 1] - f[j]) / (x[j + 1] - x[j]) / scale;
      const double dl = (f[j] - f[j - 1]) / (x[j] - x[j - 1]) / scale;
      const double tr = dr / (s * sqrt(1.0 + dr * dr) + 1.0);
      const double tl = dl / (s * sqrt(1.0 + dl * dl) + 1.0);
      v[cnt] = (tr + tl) / (1.0 - tr * tl) * scale;
    }
  }
  wsync();  // dfdx may alias f in callers
  cnt = 0;
  for (int j = lane; j < n; j += 32, ++cnt) dfdx[j] = v[cnt];
  wsync();
}

// ---------------------------------------------------------------- MAP1
// backward parabola through (L-2, L-1, L) as MAP1 writes it (1-based L)
__device__ __forceinline__ void map1_bac(const double* xo, const double* fo, int L, double& A,
                                         double& B, double& C) {
  const int l1 = L - 1, l2 = L - 2;
#define XO(i) xo[(i)-1]
#define FO(i) fo[(i)-1]
  const double d = (FO(l1) - FO(l2)) / (XO(l1) - XO(l2));
  C = FO(L) / ((XO(L) - XO(l1)) * (XO(L) - XO(l2))) +
      (FO(l2) / (XO(L) - XO(l2)) - FO(l1) / (XO(L) - XO(l1))) / (XO(l1) - XO(l2));
  B = d - (XO(l1) + XO(l2)) * C;
  A = FO(l2) - XO(l2) * d + XO(l1) * XO(l2) * C;
}
// forward parabola through (L-1, L, L+1)
__device__ __forceinline__ void map1_for(const double* xo, const double* fo, int L, double& A,
                                         double& B, double& C) {
  const int l1 = L - 1;
  const double d = (FO(L) - FO(l1)) / (XO(L) - XO(l1));
  C = FO(L + 1) / ((XO(L + 1) - XO(L)) * (XO(L + 1) - XO(l1))) +
      (FO(l1) / (XO(L + 1) - XO(l1)) - FO(L) / (XO(L + 1) - XO(L))) / (XO(L) - XO(l1));
  B = d - (XO(L) + XO(l1)) * C;
  A = FO(l1) - XO(l1) * d + XO(L) * XO(l1) * C;
#undef XO
#undef FO
}

// Returns MAP1 (index of the last old interval used).  xnew ascending.
__device__ inline int w_map1(const double* xo, const double* fo, int nold, const double* xn,
                             double* fn, int nnew, int* lidx, int lane) {
  // bracket: L_k = min{L >= 2 : XOLD(L) > XNEW(k)}, nold+1 when past the end
  for (int k = lane; k < nnew; k += 32) {
    const double v = xn[k];
    int lo = 2, hi = nold + 1;  // search in [2, nold+1)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (xo[mid - 1] > v) hi = mid;
      else lo = mid + 1;
    }
    lidx[k] = lo;
  }
  wsync();
  for (int k = lane; k < nnew; k += 32) {
    const int Lraw = lidx[k];
    const bool past = Lraw > nold;
    const double v = xn[k];
    double A, B, C;
    if (Lraw <= 3 || past) {
      const int L = past ? nold : Lraw;
      B = (fo[L - 1] - fo[L - 2]) / (xo[L - 1] - xo[L - 2]);
      A = fo[L - 1] - xo[L - 1] * B;
      fn[k] = A + B * v;  // a reused linear fit (C = 0) gives the same value
      continue;
    }
    const int L = Lraw;
    // first output point of this interval and the interval used before it
    int k0 = k;
    while (k0 > 0 && lidx[k0 - 1] == L) --k0;
    int prevL = 0;
    if (k0 > 0) prevL = lidx[k0 - 1] > nold ? nold : lidx[k0 - 1];
    double ab, bb, cb;
    if (L == prevL + 1 && L != 3 && L != 4) map1_for(xo, fo, L - 1, ab, bb, cb);
    else map1_bac(xo, fo, L, ab, bb, cb);
    if (L >= nold) {
      A = ab;
      B = bb;
      C = cb;
    } else {
      double af, bf, cf;
      map1_for(xo, fo, L, af, bf, cf);
      double wt = 0.0;
      if (fabs(cf) != 0.0) wt = fabs(cf) / (fabs(cf) + fabs(cb));
      A = af + wt * (ab - af);
      B = bf + wt * (bb - bf);
      C = cf + wt * (cb - cf);
    }
    fn[k] = A + (B + C * v) * v;
  }
  wsync();
  const int Llast = lidx[nnew - 1];
  const int ll = Llast > nold ? nold : Llast;
  wsync();
  return ll - 1;
}

// ---------------------------------------------------------------- SOLVIT
// Gaussian elimination with partial pivoting on ws.A (kNx x kNx, ld kLd),
// right-hand side / solution in b.  Reference pivot rule: first maximum.
__device__ inline void w_solvit(double* __restrict__ A, double* __restrict__ b, int lane) {
  constexpr double PIVOT_TOL = 1.0e-30;
  constexpr int n = kNx;
  int mypiv0 = 0, mypiv1 = 0;  // pivot of column i for i = lane, lane+32
  for (int i = 0; i < n - 1; ++i) {
    // (a) pivot search over rows i..n-1 of column i
    double best = -1.0;
    int bidx = n;
    for (int k = i + lane; k < n; k += 32) {
      const double v = fabs(A[i * kLd + k]);
      if (v > best) {
        best = v;
        bidx = k;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (ob > best || (ob == best && oi < bidx)) {
        best = ob;
        bidx = oi;
      }
    }
    const int m = bidx;
    if (lane == (i & 31)) {
      if (i < 32) mypiv0 = m;
      else mypiv1 = m;
    }
    // (b) swap rows i and m, columns i+1..n-1
    if (m != i) {
      for (int c = i + 1 + lane; c < n; c += 32) {
        const double t = A[c * kLd + i];
        A[c * kLd + i] = A[c * kLd + m];
        A[c * kLd + m] = t;
      }
    }
    wsync();
    // (c) reciprocal pivot on the diagonal
    double pv = A[i * kLd + m];
    if (fabs(pv) < PIVOT_TOL) pv = copysign(PIVOT_TOL, pv);
    const double pivot = 1.0 / pv;
    const double aii = A[i * kLd + i];
    wsync();
    if (lane == 0) {
      A[i * kLd + m] = aii;
      A[i * kLd + i] = pivot;
    }
    wsync();
    // (d) multipliers, (e) trailing update: lanes own rows i+1+lane, i+33+lane
    const int r0 = i + 1 + lane, r1 = i + 33 + lane;
    double l0 = 0.0, l1 = 0.0;
    if (r0 < n) {
      l0 = A[i * kLd + r0] * pivot;
      A[i * kLd + r0] = l0;
    }
    if (r1 < n) {
      l1 = A[i * kLd + r1] * pivot;
      A[i * kLd + r1] = l1;
    }
    for (int j = i + 1; j < n; ++j) {
      const double cj = A[j * kLd + i];
      if (r0 < n) A[j * kLd + r0] = A[j * kLd + r0] - l0 * cj;
      if (r1 < n) A[j * kLd + r1] = A[j * kLd + r1] - l1 * cj;
    }
    wsync();
  }
  if (lane == 0) {
    double v = A[(n - 1) * kLd + n - 1];
    if (fabs(v) < PIVOT_TOL) v = copysign(PIVOT_TOL, v);
    A[(n - 1) * kLd + n - 1] = 1.0 / v;
  }
  wsync();
  // forward substitution with the row interchanges
  for (int i = 0; i < n - 1; ++i) {
    const int m = __shfl_sync(0xffffffffu, i < 32 ? mypiv0 : mypiv1, i & 31);
    if (m != i && lane == 0) {
      const double t = b[m];
      b[m] = b[i];
      b[i] = t;
    }
    wsync();
    const double c = b[i];
    for (int k = i + 1 + lane; k < n; k += 32) b[k] = b[k] - A[i * kLd + k] * c;
    wsync();
  }
  // back substitution
  for (int j = n - 1; j >= 1; --j) {
    double bj = 0.0;
    if (lane == 0) {
      bj = b[j] * A[j * kLd + j];
      b[j] = bj;
    }
    bj = __shfl_sync(0xffffffffu, bj, 0);
    for (int k = lane; k < j; k += 32) b[k] = b[k] - A[j * kLd + k] * bj;
    wsync();
  }
  if (lane == 0) b[0] = b[0] * A[0];
  wsync();
}

// ---------------------------------------------------------------- JOSH
// Inputs in ws.*: abtot/alpha/snubar are formed here from the opacity
// vectors.  rhox is shared by the CTA.  ifsurf = 1 returns H(1); ifsurf = 0
// fills full (SNU, JNU, HNU, JMINS, KNU(1), MAXJ) as the reference does.
// Returns the number of Eddington sweeps run (0 if none).
__device__ inline int w_josh(const JoshOps& ops, const double* rhox, int nr, const double* acont,
                             const double* aline, const double* sigmac, const double* sigmal,
                             const double* scont, const double* sline, const double* bnu,
                             JoshWS& ws,
                             JoshWSFull* full, double* hsurf, int lane) {
  for (int j = lane; j < nr; j += 32) {
    const double ab = acont[j] + aline[j] + sigmac[j] + sigmal[j];
    ws.abtot[j] = ab;
    ws.alpha[j] = (sigmac[j] + sigmal[j]) / ab;
    ws.snubar[j] = (acont[j] * scont[j] + aline[j] * sline[j]) / (acont[j] + aline[j]);
  }
  wsync();
  w_integ(rhox, ws.abtot, ws.taunu, nr, ws.abtot[0] * rhox[0], ws, lane);
  int maxj = 0;
  if (ws.taunu[0] > ops.xtau[kNx - 1]) maxj = 1;
  if (maxj != 1) {
    maxj = w_map1(ws.taunu, ws.snubar, nr, ops.xtau, ws.xsbar, kNx, ws.lidx, lane);
    maxj = w_map1(ws.taunu, ws.alpha, nr, ops.xtau, ws.xalpha, kNx, ws.lidx, lane);
    const double tau1 = ws.taunu[0];
    double amax = 0.0;
    bool any = false;
    for (int l = lane; l < kNx; l += 32) {
      double xa = fmax(ws.xalpha[l], 0.0);
      double xb = fmax(ws.xsbar[l], 1.0e-38);
      if (ops.xtau[l] < tau1) {
        xb = fmax(ws.snubar[0], 1.0e-38);
        xa = fmax(ws.alpha[0], 0.0);
      }
      ws.xalpha[l] = xa;
      ws.xsbar[l] = xb;
      if (!any || xa > amax) amax = xa;
      any = true;
    }
    amax = warp_max(any ? amax : -1.0);
    wsync();
    if (amax <= 0.0) {
      for (int l = lane; l < kNx; l += 32) ws.xs[l] = fmax(ws.xsbar[l], 1.0e-37);
      wsync();
    } else {
      // AMAT(L,M) = -XALPHA(L)*COEFJ(L,M), +1 on the diagonal; lanes own rows
      for (int m = 0; m < kNx; ++m) {
        for (int l = lane; l < kNx; l += 32) {
          double v = -ws.xalpha[l] * ops.coefj[m * kNx + l];
          if (l == m) v = v + 1.0;
          ws.A[m * kLd + l] = v;
        }
      }
      for (int l = lane; l < kNx; l += 32) ws.xs[l] = (1.0 - ws.xalpha[l]) * ws.xsbar[l];
      wsync();
      w_solvit(ws.A, ws.xs, lane);
      for (int l = lane; l < kNx; l += 32) ws.xs[l] = fmax(ws.xs[l], 1.0e-37);
      wsync();
    }
    if (full == nullptr) {
      // IFSURF = 1: H(1) = sum CH_J * XS in the reference order
      if (lane == 0) {
        double h = 0.0;
        for (int m = 0; m < kNx; ++m) h = h + ops.ch[m] * ws.xs[m];
        *hsurf = h;
      }
      wsync();
      return 0;
    }
    w_map1(ops.xtau, ws.xs, kNx, ws.taunu, full->snu, maxj, ws.lidx, lane);
  }
  // JOSH with IFSURF = 1 and MAXJ = 1 falls through to the Eddington sweep
  // IFSURF = 1 with an optically thick surface borrows the scratch vectors
  // t1..t3 for SNU/HNU/JMINS (JNU is not needed beyond HNU(1)).
  JoshWSFull* F = full;
  int sweeps = 0;
  double* snu = F ? F->snu : ws.t1;
  double* hnu = F ? F->hnu : ws.t2;
  double* jmins = F ? F->jmins : ws.t3;
  double* jnu = F ? F->jnu : nullptr;
  if (maxj != nr) {
    const int maxj1 = (maxj == 1) ? 1 : maxj + 1;
    for (int j = maxj1 - 1 + lane; j < nr; j += 32) snu[j] = ws.snubar[j];
    wsync();
    const int m = maxj - 1 > 1 ? maxj - 1 : 1;
    const int nm1 = nr - m + 1, nmj = nr - maxj + 1;
    for (int l = 1; l <= 50; ++l) {
      sweeps = l;
      // negative SNU -> reset to BNU
      bool neg = false;
      for (int j = m - 1 + lane; j < nr; j += 32) neg |= (snu[j] <= 0.0);
      int ifneg = __any_sync(0xffffffffu, neg) ? 1 : 0;
      if (ifneg) {
        for (int j = m - 1 + lane; j < nr; j += 32) {
          ws.snubar[j] = bnu[j];
          snu[j] = bnu[j];
        }
        wsync();
      }
      w_deriv(ws.taunu + m - 1, snu + m - 1, hnu + m - 1, nm1, lane);
      bool hneg = false;
      for (int j = m - 1 + lane; j < nr; j += 32) hneg |= (hnu[j] <= 0.0);
      if (__any_sync(0xffffffffu, hneg)) {
        ifneg = 1;
        for (int j = m - 1 + lane; j < nr; j += 32) {
          ws.snubar[j] = bnu[j];
          snu[j] = bnu[j];
        }
        wsync();
        w_deriv(ws.taunu + m - 1, snu + m - 1, hnu + m - 1, nm1, lane);
      }
      for (int j = m - 1 + lane; j < nr; j += 32) hnu[j] = hnu[j] / 3.0;
      wsync();
      w_deriv(ws.taunu + maxj - 1, hnu + maxj - 1, jmins + maxj - 1, nmj, lane);
      double err = 0.0;
      for (int j = maxj1 - 1 + lane; j < nr; j += 32) {
        if (ifneg) jmins[j] = 0.0;
        const double jv = jmins[j] + snu[j];
        if (jnu) jnu[j] = jv;
        const double snew = (1.0 - ws.alpha[j]) * ws.snubar[j] + ws.alpha[j] * jv;
        err += fabs(snew - snu[j]) / snew;
        snu[j] = snew;
      }
      err = warp_sum(err);
      wsync();
      if (err < 0.00001) break;
    }
  }
  if (maxj == 1) {
    if (F) {
      F->knu1 = jnu[0] / 3.0;
      F->maxj = maxj;
    } else if (lane == 0) {
      *hsurf = hnu[0];
    }
    wsync();
    return sweeps;
  }
  // (IFSURF = 1 never reaches here with MAXJ != 1: it returned above.)
  // J - S and H on the 51-point grid, mapped back onto the first MAXJ depths
  for (int l = lane; l < kNx; l += 32) {
    double xj = -ws.xs[l];
    double xh = 0.0;
    for (int mm = 0; mm < kNx; ++mm) {
      xj = xj + ops.coefj[mm * kNx + l] * ws.xs[mm];
      xh = xh + ops.coefh[mm * kNx + l] * ws.xs[mm];
    }
    ws.xw[l] = xj;
    ws.xsbar[l] = xh;  // XSBAR no longer needed: holds XH
  }
  wsync();
  w_map1(ops.xtau, ws.xw, kNx, ws.taunu, F->jmins, maxj, ws.lidx, lane);
  w_map1(ops.xtau, ws.xsbar, kNx, ws.taunu, F->hnu, maxj, ws.lidx, lane);
  if (lane == 0) {
    double xk = 0.0;
    for (int mm = 0; mm < kNx; ++mm) xk = xk + ops.ck[mm] * ws.xs[mm];
    F->knu1 = xk;
    F->maxj = maxj;
  }
  for (int j = lane; j < maxj; j += 32) {
    F->snu[j] = fmax(F->snu[j], 1.0e-38);
    F->jnu[j] = fmax(F->jmins[j] + F->snu[j], 1.0e-38);
  }
  wsync();
  return sweeps;
}

}  // namespace atlasgpu
