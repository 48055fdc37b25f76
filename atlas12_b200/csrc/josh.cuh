// josh.cuh -- cooperative JOSH radiative transfer (FP64) for sm_100a.
//
// A thread group solves one frequency: either one warp (WarpG) or a pair of
// warps (PairG, 64 threads synchronised by a named barrier).  Depth vectors
// (<= kKwMax) live in the group's shared-memory workspace; threads split
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
// are summed in the reference order by one thread.
//
// The 51x51 scattering system: a warp group factors it in shared memory
// (w_solvit); a pair group keeps one matrix row per thread in registers and
// writes only the pivot rows to shared memory, which takes the row updates
// off the shared-memory pipe.
#pragma once
#include "common.cuh"

namespace atlasgpu {

// ---------------------------------------------------------------- groups
struct WarpG {
  static constexpr int N = 32;
  int r;  // lane
  __device__ explicit WarpG(int lane) : r(lane) {}
  __device__ __forceinline__ void sync() const { __syncwarp(0xffffffffu); }
  __device__ __forceinline__ double max(double v) { return warp_max(v); }
  __device__ __forceinline__ double sum(double v) { return warp_sum(v); }
  __device__ __forceinline__ bool any(bool p) { return __any_sync(0xffffffffu, p); }
};

// NW warps on named barrier `bar`; red = 2*NW doubles of the group's shared
// scratch (one slot per warp and parity, alternated so one barrier per
// reduction suffices: a slot is rewritten only after every thread has passed
// the barrier of the reduction in between).  Warp partials are combined in
// warp order, so the result does not depend on scheduling.
template <int NW>
struct MultiG {
  static constexpr int N = 32 * NW;
  int r;  // 0..N-1
  int bar;
  double* red;
  int par;
  __device__ MultiG(int rank, int barrier, double* scratch) : r(rank), bar(barrier), red(scratch), par(0) {}
  __device__ __forceinline__ void sync() const {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(N) : "memory");
  }
  __device__ __forceinline__ double sum(double v) {
    v = warp_sum(v);
    if ((r & 31) == 0) red[par * NW + (r >> 5)] = v;
    sync();
    double s = red[par * NW];
#pragma unroll
    for (int w = 1; w < NW; ++w) s += red[par * NW + w];
    par ^= 1;
    return s;
  }
  __device__ __forceinline__ double max(double v) {
    v = warp_max(v);
    if ((r & 31) == 0) red[par * NW + (r >> 5)] = v;
    sync();
    double s = red[par * NW];
#pragma unroll
    for (int w = 1; w < NW; ++w) s = fmax(s, red[par * NW + w]);
    par ^= 1;
    return s;
  }
  __device__ __forceinline__ bool any(bool p) { return max(__any_sync(0xffffffffu, p) ? 1.0 : 0.0) > 0.0; }
};
using PairG = MultiG<2>;

struct JoshWS {
  double xs[kNx], xsbar[kNx], xalpha[kNx], xw[kNx];
  double abtot[kKwMax], alpha[kKwMax], snubar[kKwMax], taunu[kKwMax];
  double t1[kKwMax], t2[kKwMax], t3[kKwMax];  // scratch (PARCOE a,b,c / terms)
  double red[8];                              // group reductions (multi-warp groups)
  double piv[kNx];                            // pivots of the elimination without interchanges
  int lidx[kKwMax + 4];                       // MAP1 bracket indices
  unsigned pk[4][3];                          // pivot key exchange between a group's warps
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
template <class G>
__device__ inline void g_parcoe(G& g, const double* f, const double* x, double* a, double* b, double* c,
                                int n) {
  constexpr int C = (kKwMax + G::N - 1) / G::N;
  // steps 1-3: endpoints linear, j = 1, 2 linear, interior parabolic
  for (int j = g.r; j < n; j += G::N) {
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
  g.sync();
  // step 4: blend each interval with its right neighbour's unsmoothed fit
  double na[C], nb[C], nc[C];
  int cnt = 0;
  for (int j = g.r; j < n; j += G::N, ++cnt) {
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
  g.sync();
  cnt = 0;
  for (int j = g.r; j < n; j += G::N, ++cnt) {
    a[j] = na[cnt];
    b[j] = nb[cnt];
    c[j] = nc[cnt];
  }
  g.sync();
  // step 5: penultimate interval takes the endpoint linear fit
  if (g.r == 0) {
    a[n - 2] = a[n - 1];
    b[n - 2] = b[n - 1];
    c[n - 2] = c[n - 1];
  }
  g.sync();
}

// fint = running parabolic integral of f over x, fint[0] = start
template <class G, class WS>
__device__ inline void g_integ(G& g, const double* x, const double* f, double* fint, int n, double start,
                               WS& ws) {
  double *a = ws.t1, *b = ws.t2, *c = ws.t3;
  g_parcoe(g, f, x, a, b, c, n);
  for (int i = g.r; i < n - 1; i += G::N) {
    const double xlo = x[i], xhi = x[i + 1];
    const double term = (a[i] + b[i] * 0.5 * (xhi + xlo) +
                         c[i] / 3.0 * ((xhi + xlo) * xhi + xlo * xlo)) *
                        (xhi - xlo);
    b[i] = term;
  }
  g.sync();
  if (g.r == 0) {
    double s = start;
    fint[0] = s;
    for (int i = 0; i < n - 1; ++i) {
      s = s + b[i];
      fint[i + 1] = s;
    }
  }
  g.sync();
}

// ---------------------------------------------------------------- DERIV
template <class G>
__device__ __noinline__ void g_deriv(G& g, const double* x, const double* f, double* dfdx, int n) {
  constexpr int C = (kKwMax + G::N - 1) / G::N;
  const double s = fabs(x[1] - x[0]) / (x[1] - x[0]);
  double v[C];
  int cnt = 0;
  for (int j = g.r; j < n; j += G::N, ++cnt) {
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
  g.sync();  // dfdx may alias f in callers
  cnt = 0;
  for (int j = g.r; j < n; j += G::N, ++cnt) dfdx[j] = v[cnt];
  g.sync();
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
template <class G>
__device__ __noinline__ int g_map1(G& g, const double* xo, const double* fo, int nold, const double* xn,
                             double* fn, int nnew, int* lidx) {
  // bracket: L_k = min{L >= 2 : XOLD(L) > XNEW(k)}, nold+1 when past the end
  for (int k = g.r; k < nnew; k += G::N) {
    const double v = xn[k];
    int lo = 2, hi = nold + 1;  // search in [2, nold+1)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (xo[mid - 1] > v) hi = mid;
      else lo = mid + 1;
    }
    lidx[k] = lo;
  }
  g.sync();
  for (int k = g.r; k < nnew; k += G::N) {
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
  g.sync();
  const int Llast = lidx[nnew - 1];
  const int ll = Llast > nold ? nold : Llast;
  g.sync();
  return ll - 1;
}

// ---------------------------------------------------------------- SOLVIT
constexpr double kPivotTol = 1.0e-30;

// Gaussian elimination with partial pivoting on A (kNx x kNx, column-major,
// ld kLd, shared memory), right-hand side / solution in b.  Reference pivot
// rule: first maximum.  One warp.
__device__ inline void w_solvit(double* __restrict__ A, double* __restrict__ b, int lane) {
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
    if (fabs(pv) < kPivotTol) pv = copysign(kPivotTol, pv);
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
    if (fabs(v) < kPivotTol) v = copysign(kPivotTol, v);
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

// (I - diag(XALPHA) COEFJ) XS = (1 - XALPHA) XSBAR by one warp: the matrix
// AMAT(L,M) = -XALPHA(L)*COEFJ(L,M) (+1 on the diagonal) in shared memory A.
__device__ inline void scatter_solve(WarpG& g, const JoshOps& ops, JoshWS& ws, double* A) {
  for (int m = 0; m < kNx; ++m) {
    for (int l = g.r; l < kNx; l += 32) {
      double v = -ws.xalpha[l] * ops.coefj[m * kNx + l];
      if (l == m) v = v + 1.0;
      A[m * kLd + l] = v;
    }
  }
  for (int l = g.r; l < kNx; l += 32) ws.xs[l] = (1.0 - ws.xalpha[l]) * ws.xsbar[l];
  g.sync();
  w_solvit(A, ws.xs, g.r);
}

// Pivot-row traffic in 16-byte words: the row owner stores [1/pivot, a[1..]]
// and every pending row reads it back as double2 words (U rows are 16-byte
// aligned: 52 doubles per row on a 16-byte aligned base).  From step 26 on,
// only the first 26 entries of a shifted row can be nonzero (columns i..50
// and the rhs), so those steps move and update NW = 13 words instead of 26.
template <int NW = (kNx + 1) / 2>
__device__ __forceinline__ void store_pivot_row(double* ur, double rpiv, const double (&a)[kNx + 1]) {
  double2* u2 = reinterpret_cast<double2*>(ur);
  u2[0] = make_double2(rpiv, a[1]);
#pragma unroll
  for (int q = 1; q < NW; ++q) u2[q] = make_double2(a[2 * q], a[2 * q + 1]);
}

// a[t-1] = a[t] - l * ur[t] (t = 1..2NW-1), l = a[0] * ur[0]; the entry
// shifted in from beyond the stored words is zero (a[2NW-1] = 0)
template <int NW = (kNx + 1) / 2>
__device__ __forceinline__ void eliminate_shift(double (&a)[kNx + 1], const double* ur) {
  const double2* u2 = reinterpret_cast<const double2*>(ur);
  const double2 u0 = u2[0];
  const double l = a[0] * u0.x;
  a[0] = a[1] - l * u0.y;
#pragma unroll
  for (int q = 1; q < NW; ++q) {
    const double2 u = u2[q];
    a[2 * q - 1] = a[2 * q] - l * u.x;
    a[2 * q] = a[2 * q + 1] - l * u.y;
  }
  a[2 * NW - 1] = 0.0;
}

constexpr int kHalfStep = (kNx + 1) / 2;  // first step whose pending rows fit in half a row

// Back substitution from the stored pivot rows U (row k: U[k][0] = 1/pivot,
// U[k][t] = column k+t, the rhs at t = 51-k) by the group's first warp: lane
// q holds positions q and q+32, X(j) = B(j) * (1/pivot) is passed by shuffle
// and B(k) -= A(k,j) X(j) for k < j, in SOLVIT's order.  XS receives X.
__device__ __forceinline__ void u_back_substitute(int r, const double* U, double* xs) {
  constexpr int n = kNx, W = kNx + 1;
  if (r >= 32) return;
  const int k0 = r, k1 = r + 32;
  double b0 = U[k0 * W + (W - 1 - k0)];
  double b1 = k1 < n ? U[k1 * W + (W - 1 - k1)] : 0.0;
  for (int j = n - 1; j >= 0; --j) {
    const int src = j & 31;
    double x = (j < 32 ? b0 : b1) * U[j * W];
    x = __shfl_sync(0xffffffffu, x, src);
    if (r == src) xs[j] = x;
    if (k0 < j) b0 = b0 - U[k0 * W + (j - k0)] * x;
    if (k1 < j) b1 = b1 - U[k1 * W + (j - k1)] * x;
  }
}

// The same system by a pair group, thread r < 51 holding row r of
// [AMAT | rhs] in registers.  The elimination follows SOLVIT's arithmetic:
// the pivot of step i is the first maximum |A(k,i)| over the rows at
// positions i..50 (rows are swapped logically: each thread tracks the
// position of its row), the pivot is replaced by its reciprocal (clamped at
// 1e-30), multipliers are A(k,i) * (1/pivot), the right-hand side is
// eliminated with the same multipliers in step order, and back substitution
// runs column by column from the last.
// Each step shifts the pending rows one column left, so column i is always
// register a[0] and the loop over steps stays rolled (one short loop body
// instead of 51 unrolled steps).  The pivot row of step i is stored in
// U[i][0..51] (U[i][0] = 1/pivot, U[i][t] = column i+t, the rhs at t = 51-i)
// for the other rows' update and for the back substitution.
// The pivot search reduces a 64-bit key (|a| bits, then position) with
// redux.sync per warp and one exchange between the two warps.
template <class WS>
static __device__ __forceinline__ void scatter_solve(PairG& g, const JoshOps& ops, WS& ws, double* U) {
  constexpr int n = kNx, W = kNx + 1;
  constexpr unsigned FULL = 0xffffffffu;
  const bool own = g.r < n;
  double a[W];
  {
    const int l = own ? g.r : 0;
    const double xa = ws.xalpha[l];
#pragma unroll
    for (int m = 0; m < n; ++m) {
      double v = -xa * ops.coefj[m * kNx + l];
      if (l == m) v = v + 1.0;
      a[m] = v;
    }
    a[n] = (1.0 - xa) * ws.xsbar[l];
  }
  int pos = own ? g.r : n + 1;  // current row position
  bool done = !own;
  for (int i = 0; i < n - 1; ++i) {
    // (a) pivot: max |A(pos, i)| over pending rows, ties to the lowest position
    unsigned hi = 0u, lo = 0u;
    if (!done) {
      const unsigned long long bits = (unsigned long long)__double_as_longlong(fabs(a[0]));
      hi = (unsigned)(bits >> 32) + 1u;  // 0 marks rows already eliminated
      lo = (unsigned)bits;
    }
    const unsigned mhi = __reduce_max_sync(FULL, hi);
    const unsigned mlo = __reduce_max_sync(FULL, hi == mhi ? lo : 0u);
    const unsigned mpos =
        __reduce_min_sync(FULL, (hi != 0u && hi == mhi && lo == mlo) ? (unsigned)pos : 0xffffffffu);
    if ((g.r & 31) == 0) {
      ws.pk[g.r >> 5][0] = mhi;
      ws.pk[g.r >> 5][1] = mlo;
      ws.pk[g.r >> 5][2] = mpos;
    }
    g.sync();
    unsigned bpos;
    {
      const unsigned h0 = ws.pk[0][0], l0 = ws.pk[0][1], p0 = ws.pk[0][2];
      const unsigned h1 = ws.pk[1][0], l1 = ws.pk[1][1], p1 = ws.pk[1][2];
      const bool second = h1 > h0 || (h1 == h0 && (l1 > l0 || (l1 == l0 && p1 < p0)));
      bpos = second ? p1 : p0;
    }
    const bool me = !done && (unsigned)pos == bpos;
    // (b) the row at position i moves to the pivot's position
    if (!done && !me && pos == i) pos = (int)bpos;
    // (c) the pivot row, with its reciprocal pivot, to every thread
    double* ur = U + i * W;
    if (me) {
      double pv = a[0];
      if (fabs(pv) < kPivotTol) pv = copysign(kPivotTol, pv);
      if (i < kHalfStep) store_pivot_row(ur, 1.0 / pv, a);
      else store_pivot_row<kHalfStep / 2>(ur, 1.0 / pv, a);
      pos = i;
      done = true;
    }
    g.sync();
    // (d, e) multiplier and trailing update of the pending rows, shifted left
    if (!done) {
      if (i < kHalfStep) eliminate_shift(a, ur);
      else eliminate_shift<kHalfStep / 2>(a, ur);
    }
  }
  // the last pending row takes position n-1: column n-1 in a[0], rhs in a[1]
  if (!done) {
    pos = n - 1;
    double v = a[0];
    if (fabs(v) < kPivotTol) v = copysign(kPivotTol, v);
    U[(n - 1) * W] = 1.0 / v;
    U[(n - 1) * W + 1] = a[1];
  }
  g.sync();
  u_back_substitute(g.r, U, ws.xs);
  g.sync();
}

// Elimination without interchanges, checked: thread r < 51 holds row r,
// which becomes the pivot row at step r.  At step i every pending row
// compares its |A(k,i)| with the pivot |A(i,i)|; SOLVIT's first-maximum rule
// would pick another row only if some |A(k,i)| is strictly larger.  Returns
// false (the caller then redoes the system with interchanges) if that ever
// happened; otherwise the operations were exactly SOLVIT's, in its order.
// (For these systems it does not happen: AMAT is column diagonally dominant
// because the columns of COEFJ sum to at most 1 and XALPHA < 1.)
template <class WS>
static __device__ __forceinline__ bool scatter_solve_nopivot(PairG& g, const JoshOps& ops, WS& ws, double* U) {
  constexpr int n = kNx, W = kNx + 1;
  const bool own = g.r < n;
  double a[W];
  {
    const int l = own ? g.r : 0;
    const double xa = ws.xalpha[l];
#pragma unroll
    for (int m = 0; m < n; ++m) {
      double v = -xa * ops.coefj[m * kNx + l];
      if (l == m) v = v + 1.0;
      a[m] = v;
    }
    a[n] = (1.0 - xa) * ws.xsbar[l];
  }
  bool swap = false;
  for (int i = 0; i < n - 1; ++i) {
    double* ur = U + i * W;
    if (g.r == i) {
      ws.piv[i] = a[0];
      double pv = a[0];
      if (fabs(pv) < kPivotTol) pv = copysign(kPivotTol, pv);
      if (i < kHalfStep) store_pivot_row(ur, 1.0 / pv, a);
      else store_pivot_row<kHalfStep / 2>(ur, 1.0 / pv, a);
    }
    g.sync();
    if (own && g.r > i) {
      swap |= fabs(a[0]) > fabs(ws.piv[i]);
      if (i < kHalfStep) eliminate_shift(a, ur);
      else eliminate_shift<kHalfStep / 2>(a, ur);
    }
  }
  if (g.r == n - 1) {
    double v = a[0];
    if (fabs(v) < kPivotTol) v = copysign(kPivotTol, v);
    U[(n - 1) * W] = 1.0 / v;
    U[(n - 1) * W + 1] = a[1];
  }
  if (g.any(swap)) return false;
  u_back_substitute(g.r, U, ws.xs);
  g.sync();
  return true;
}


template <class WS>
__device__ __forceinline__ void solve_scatter(PairG& g, const JoshOps& ops, WS& ws, double* U) {
  if (!scatter_solve_nopivot(g, ops, ws, U)) scatter_solve(g, ops, ws, U);
}
__device__ __forceinline__ void solve_scatter(WarpG& g, const JoshOps& ops, JoshWS& ws, double* A) {
  scatter_solve(g, ops, ws, A);
}

// ---------------------------------------------------------------- JOSH
// JOSH in three parts, so that a caller may run them in separate launches
// (the ATLAS12 RT pass runs the 51x51 solve in its own kernel):
//   g_josh_prepare  TAUNU = INTEG(ABTOT dRHOX), MAXJ, and for MAXJ != 1 XSBAR
//                   and XALPHA on the 51-point grid with their floors
//                   (atlas12_modules.f90:18491-18570); solve = max XALPHA > 0,
//                   otherwise XS = XSBAR
//   solve_scatter   (I - diag(XALPHA) COEFJ) XS = (1 - XALPHA) XSBAR
//   g_josh_finish   XS floor, IFSURF = 1 surface flux or SNU = MAP1(XS),
//                   the Eddington sweeps below MAXJ, J/H/K from the operators
//                   mapped back onto the depths (:18571-18776)
// ws.abtot, ws.alpha and ws.snubar are formed by the caller (g_josh_fill).
template <class G, class WS>
__device__ inline void g_josh_fill(G& g, int nr, const double* acont, const double* aline, const double* sigmac,
                                   const double* sigmal, const double* scont, const double* sline, WS& ws) {
  for (int j = g.r; j < nr; j += G::N) {
    const double ab = acont[j] + aline[j] + sigmac[j] + sigmal[j];
    ws.abtot[j] = ab;
    ws.alpha[j] = (sigmac[j] + sigmal[j]) / ab;
    ws.snubar[j] = (acont[j] * scont[j] + aline[j] * sline[j]) / (acont[j] + aline[j]);
  }
  g.sync();
}

// mapped: the surface is optically thin enough for the 51-point grid (MAP1
// may still return MAXJ = 1 there, and IFSURF = 1 then takes H(1) from XS).
template <class G, class WS>
__device__ inline int g_josh_prepare(G& g, const JoshOps& ops, const double* rhox, int nr, WS& ws, bool& mapped,
                                     bool& solve) {
  g_integ(g, rhox, ws.abtot, ws.taunu, nr, ws.abtot[0] * rhox[0], ws);
  int maxj = 0;
  solve = false;
  if (ws.taunu[0] > ops.xtau[kNx - 1]) maxj = 1;
  mapped = maxj != 1;
  if (mapped) {
    maxj = g_map1(g, ws.taunu, ws.snubar, nr, ops.xtau, ws.xsbar, kNx, ws.lidx);
    maxj = g_map1(g, ws.taunu, ws.alpha, nr, ops.xtau, ws.xalpha, kNx, ws.lidx);
    const double tau1 = ws.taunu[0];
    double amax = -1.0;
    for (int l = g.r; l < kNx; l += G::N) {
      double xa = fmax(ws.xalpha[l], 0.0);
      double xb = fmax(ws.xsbar[l], 1.0e-38);
      if (ops.xtau[l] < tau1) {
        xb = fmax(ws.snubar[0], 1.0e-38);
        xa = fmax(ws.alpha[0], 0.0);
      }
      ws.xalpha[l] = xa;
      ws.xsbar[l] = xb;
      amax = fmax(amax, xa);
    }
    amax = g.max(amax);
    g.sync();
    solve = amax > 0.0;
    if (!solve) {
      for (int l = g.r; l < kNx; l += G::N) ws.xs[l] = ws.xsbar[l];
      g.sync();
    }
  }
  return maxj;
}

// J - S and H on the 51-point grid from XS (COEFJ.XS - XS into xw, COEFH.XS
// into xh), four interleaved partial sums per product (instruction-level
// parallelism instead of one 51-long dependent chain; the grouping differs
// from the reference's sequential sum only at rounding level), and
// KNU(1) = CK.XS in the reference order (:18700-18735)
template <class G>
__device__ __forceinline__ void josh_operators(G& g, const JoshOps& ops, const double* xs, double* xw, double* xh,
                                               double* knu1) {
  for (int l = g.r; l < kNx; l += G::N) {
    double sj[4] = {0.0, 0.0, 0.0, 0.0}, sh[4] = {0.0, 0.0, 0.0, 0.0};
    // sum k takes the terms mm = k, k+4, k+8, ... in that order
#pragma unroll 2
    for (int m0 = 0; m0 < kNx - kNx % 4; m0 += 4) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double x = xs[m0 + k];
        sj[k] = sj[k] + ops.coefj[(m0 + k) * kNx + l] * x;
        sh[k] = sh[k] + ops.coefh[(m0 + k) * kNx + l] * x;
      }
    }
#pragma unroll
    for (int k = 0; k < kNx % 4; ++k) {
      const int mm = kNx - kNx % 4 + k;
      const double x = xs[mm];
      sj[k] = sj[k] + ops.coefj[mm * kNx + l] * x;
      sh[k] = sh[k] + ops.coefh[mm * kNx + l] * x;
    }
    xw[l] = -xs[l] + ((sj[0] + sj[1]) + (sj[2] + sj[3]));
    xh[l] = (sh[0] + sh[1]) + (sh[2] + sh[3]);
  }
  if (g.r == 0) {
    double xk = 0.0;
    for (int mm = 0; mm < kNx; ++mm) xk = xk + ops.ck[mm] * xs[mm];
    *knu1 = xk;
  }
}

// ws.xs holds the solution (or XSBAR); ws.taunu, ws.alpha, ws.snubar as
// g_josh_prepare left them.  full (JoshWSFull or a view with the same
// members in shared memory) receives SNU, HNU, JMINS, JNU, KNU(1), MAXJ, or
// is null for IFSURF = 1.  Returns the number of Eddington sweeps run.
// kOpsGiven: the caller has floored XS and formed XW (J - S), XH (in
// ws.xsbar) and KNU(1) with josh_operators already.
template <bool kOpsGiven = false, class G, class WS, class FullT>
__device__ inline int g_josh_finish(G& g, const JoshOps& ops, int nr, int maxj, bool mapped, WS& ws, FullT* full,
                                    const double* bnu, double* hsurf) {
  if (mapped) {
    if (!kOpsGiven) {
      for (int l = g.r; l < kNx; l += G::N) ws.xs[l] = fmax(ws.xs[l], 1.0e-37);
      g.sync();
    }
    if (full == nullptr) {
      // IFSURF = 1: H(1) = sum CH_J * XS in the reference order
      if (g.r == 0) {
        double h = 0.0;
        for (int m = 0; m < kNx; ++m) h = h + ops.ch[m] * ws.xs[m];
        *hsurf = h;
      }
      g.sync();
      return 0;
    }
    g_map1(g, ops.xtau, ws.xs, kNx, ws.taunu, full->snu, maxj, ws.lidx);
  }
  // JOSH with IFSURF = 1 and MAXJ = 1 falls through to the Eddington sweep
  // IFSURF = 1 with an optically thick surface borrows the scratch vectors
  // t1..t3 for SNU/HNU/JMINS (JNU is not needed beyond HNU(1)).
  FullT* F = full;
  int sweeps = 0;
  double* snu = F ? F->snu : ws.t1;
  double* hnu = F ? F->hnu : ws.t2;
  double* jmins = F ? F->jmins : ws.t3;
  double* jnu = F ? F->jnu : nullptr;
  if (maxj != nr) {
    const int maxj1 = (maxj == 1) ? 1 : maxj + 1;
    for (int j = maxj1 - 1 + g.r; j < nr; j += G::N) snu[j] = ws.snubar[j];
    g.sync();
    const int m = maxj - 1 > 1 ? maxj - 1 : 1;
    const int nm1 = nr - m + 1, nmj = nr - maxj + 1;
    for (int l = 1; l <= 50; ++l) {
      sweeps = l;
      // negative SNU -> reset to BNU
      bool neg = false;
      for (int j = m - 1 + g.r; j < nr; j += G::N) neg |= (snu[j] <= 0.0);
      int ifneg = g.any(neg) ? 1 : 0;
      if (ifneg) {
        for (int j = m - 1 + g.r; j < nr; j += G::N) {
          ws.snubar[j] = bnu[j];
          snu[j] = bnu[j];
        }
        g.sync();
      }
      g_deriv(g, ws.taunu + m - 1, snu + m - 1, hnu + m - 1, nm1);
      bool hneg = false;
      for (int j = m - 1 + g.r; j < nr; j += G::N) hneg |= (hnu[j] <= 0.0);
      if (g.any(hneg)) {
        ifneg = 1;
        for (int j = m - 1 + g.r; j < nr; j += G::N) {
          ws.snubar[j] = bnu[j];
          snu[j] = bnu[j];
        }
        g.sync();
        g_deriv(g, ws.taunu + m - 1, snu + m - 1, hnu + m - 1, nm1);
      }
      for (int j = m - 1 + g.r; j < nr; j += G::N) hnu[j] = hnu[j] / 3.0;
      g.sync();
      g_deriv(g, ws.taunu + maxj - 1, hnu + maxj - 1, jmins + maxj - 1, nmj);
      double err = 0.0;
      for (int j = maxj1 - 1 + g.r; j < nr; j += G::N) {
        if (ifneg) jmins[j] = 0.0;
        const double jv = jmins[j] + snu[j];
        if (jnu) jnu[j] = jv;
        const double snew = (1.0 - ws.alpha[j]) * ws.snubar[j] + ws.alpha[j] * jv;
        err += fabs(snew - snu[j]) / snew;
        snu[j] = snew;
      }
      err = g.sum(err);
      g.sync();
      if (err < 0.00001) break;
    }
  }
  if (maxj == 1) {
    if (F) {
      F->knu1 = jnu[0] / 3.0;
      F->maxj = maxj;
    } else if (g.r == 0) {
      *hsurf = hnu[0];
    }
    g.sync();
    return sweeps;
  }
  // (IFSURF = 1 never reaches here with MAXJ != 1: it returned above.)
  if (!kOpsGiven) {
    josh_operators(g, ops, ws.xs, ws.xw, ws.xsbar, &F->knu1);  // XSBAR no longer needed: holds XH
    g.sync();
  }
  g_map1(g, ops.xtau, ws.xw, kNx, ws.taunu, F->jmins, maxj, ws.lidx);
  g_map1(g, ops.xtau, ws.xsbar, kNx, ws.taunu, F->hnu, maxj, ws.lidx);
  if (g.r == 0) F->maxj = maxj;
  for (int j = g.r; j < maxj; j += G::N) {
    F->snu[j] = fmax(F->snu[j], 1.0e-38);
    F->jnu[j] = fmax(F->jmins[j] + F->snu[j], 1.0e-38);
  }
  g.sync();
  return sweeps;
}

// The whole of JOSH by one group.  Inputs in ws.*: abtot/alpha/snubar are
// formed here from the opacity vectors.  rhox is shared by the CTA.
// ifsurf = 1 returns H(1); ifsurf = 0 fills full (SNU, JNU, HNU, JMINS,
// KNU(1), MAXJ) as the reference does.  A: shared-memory matrix for a warp
// group, the U rows for a pair group.  Returns the number of Eddington
// sweeps run (0 if none).
template <class G>
__device__ inline int g_josh(G& g, const JoshOps& ops, const double* rhox, int nr, const double* acont,
                             const double* aline, const double* sigmac, const double* sigmal,
                             const double* scont, const double* sline, const double* bnu, JoshWS& ws,
                             double* A, JoshWSFull* full, double* hsurf) {
  g_josh_fill(g, nr, acont, aline, sigmac, sigmal, scont, sline, ws);
  bool mapped, solve;
  const int maxj = g_josh_prepare(g, ops, rhox, nr, ws, mapped, solve);
  if (solve) solve_scatter(g, ops, ws, A);
  return g_josh_finish(g, ops, nr, maxj, mapped, ws, full, bnu, hsurf);
}

}  // namespace atlasgpu
