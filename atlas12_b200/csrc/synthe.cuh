// synthe.cuh -- SYNTHE hot-path kernels (sm_100a).
//
//  k_bin        line -> grid index (mod_mklinelist.f90:898-899)
//  k_continuum  continuum per depth on the grid (synthe.f90:483-516)
//  k_core       gates, line centre and Voigt core walk of every (line, depth)
//               pair (synthe.f90:559-640), one pair per lane at a time,
//               core values scattered with FP64 atomics; far-wing lines
//               recorded for k_farwing
//  k_far_*      per-(depth, tile) inverted index of the far-wing lines
//  k_farwing    the x_wing/n^2 far wings (synthe.f90:641-650) per 128-bin
//               sub-tile: distant lines as Taylor expansions about the
//               sub-tile centre, near ones bin by bin; plus the core
//               accumulator, written as the REAL(4) opacity matrix
//  k_spectrum   the wavelength loop (synthe.f90:698-718, 797-902): two
//               warp-cooperative JOSH(1,1) solves per wavelength
#pragma once
#include "common.cuh"
#include "josh.cuh"
#include "voigt.cuh"

namespace atlasgpu {

constexpr int kTile = 1024;      // bins per far-wing tile

struct FarLine {
  int c;    // line centre nbuff (1-based)
  int n10;  // n10dop: core extent
  int m;    // maxstep: far-wing extent
  int pad;
  double x; // x_wing = profile(n10dop) * n10dop**2
};

// ---------------------------------------------------------------- binning
static __global__ void k_bin(const double* __restrict__ wl, int64_t n, double ratiolg, int ixwlbeg,
                      int32_t* __restrict__ nbuff, int64_t* __restrict__ flagged,
                      unsigned long long* __restrict__ nflag, int64_t flag_cap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double q = log(wl[i]) / ratiolg + 0.5;
    const int ixwl = (int)q;
    nbuff[i] = ixwl - ixwlbeg + 1;
    // a 1-ulp difference in log moves q by < 1e-9: re-evaluate near-integers on the host
    if (fabs(q - rint(q)) < 1.0e-8) {
      const unsigned long long k = atomicAdd(nflag, 1ull);
      if ((int64_t)k < flag_cap) flagged[k] = i;
    }
  }
}

// ---------------------------------------------------------------- continuum
static __global__ void k_continuum(const double* __restrict__ wledge, int nedge,
                            const double* __restrict__ continall, int stride, int nrhox,
                            double wbegin, double ratio, int length, float* __restrict__ out) {
  const int j = blockIdx.y;
  const double* ab = continall + (size_t)j * stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < length; i += gridDim.x * blockDim.x) {
    const double w = wbegin * powi(ratio, i);
    // iedge = 1 + #{e in [2, nedge-1] : wledge(e) <= w}
    int lo = 1, hi = nedge - 1;  // answer in [1, nedge-1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;  // candidate iedge
      if (wledge[mid - 1] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int ie = lo;
    const double wl0 = wledge[ie - 1], wl1 = wledge[ie];
    const double h = (wl0 + wl1) * 0.5;
    const double dd = powi(wl1 - wl0, 2) * 0.5;
    const double* q = ab + 3 * (ie - 1);
    const double v = ((w - h) * (w - wl1) * q[0] + (wl0 - w) * (w - wl1) * 2.0 * q[1] +
                      (w - wl0) * (w - h) * q[2]) / dd;
    float cf = (float)v;
    if (cf < -15.0f) cf = -15.0f;
    out[(size_t)j * length + i] = (float)exp10((double)cf);
  }
}

// ---------------------------------------------------------------- core pass
struct CoreArgs {
  const atlasgpu_lte_line* lines;
  int64_t n;
  int length, nrhox, nspec, maxprof, j0, nj;  // depths [j0, j0+nj)
  double resolu;
  const float* cont;     // [nrhox][length]
  const double *xnfdop, *dopple;  // [nrhox][nspec]
  const double *xne, *txnxn, *hckt;
  double* acc;           // [nrhox][length] core accumulator
  FarLine* far;          // [nj][n]
  unsigned int* nfar;    // [nj]
  int* tdiff;            // [nj][ntiles+1]
  int ntiles;
  // work counters (timed launches only, else null): [0] Voigt evaluations,
  // [1] far-wing bin updates the gather will make
  unsigned long long* work = nullptr;
};

// Every lane walks (line, depth) pairs on its own, one Voigt evaluation per
// trip of the loop: the centre point first, then the core points
// s = 1, 2, ... until the first value below kapmin (scattered too, as the
// reference's loop does) or s = n10dop.  The evaluation is the only
// expensive step, and all lanes with a pair run it together whatever the
// lengths of their walks, so the warp keeps every lane supplied: it gates
// the pairs 32 at a time (a chunk of its grid-stride sequence, one pair per
// lane), a pair that passes both kapmin gates stays with its lane as a
// pending candidate, and a lane whose walk has ended takes the next pending
// candidate of the warp (k-th idle lane, k-th candidate, by shuffles).
// With MAXPROF < n10dop the reference scatters only min(n10dop, maxstep)
// core points when no point falls below kapmin; that limit is known only
// after the walk, so such pairs walk once to decide (phase 1) and once to
// scatter (phase 2).
// A walk that reaches n10dop without a point below kapmin records its far
// wing x_wing/n^2 (n10dop < n <= maxstep) for k_farwing.
static __global__ void __launch_bounds__(256, 4) k_core(CoreArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  const int64_t npairs = a.n * a.nj;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t chunk = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;  // next chunk of 32 pairs
  unsigned long long nev = 0, nfw = 0;  // counted only when a.work is set
  // the lane's walk
  bool act = false;
  int phase = 0, s = 0, lim = 0, nb = 0, n10 = 0, jj = 0;
  double kappa0 = 0.0, adamp = 0.0, dv = 0.0, kapmin = 0.0;
  double* accj = nullptr;
  // the lane's pending candidate
  bool pend = false;
  int c_nb = 0, c_n10 = 0, c_jj = 0;
  double c_k0 = 0.0, c_km = 0.0, c_ad = 0.0, c_dv = 0.0;
  while (true) {
    // refill the idle lanes: pending candidates first, new chunks when none is left
    while (true) {
      const unsigned idle = __ballot_sync(FULL, !act);
      if (!idle) break;
      const unsigned pm = __ballot_sync(FULL, pend);
      if (!pm) {
        if (chunk * 32 >= npairs) break;
        const int64_t pp = chunk * 32 + lane;
        chunk += nw;
        if (pp < npairs) {
          const int jp = (int)(pp / a.n);
          const int64_t il = pp - (int64_t)jp * a.n;
          const int j = a.j0 + jp;
          const atlasgpu_lte_line L = a.lines[il];
          const int nel = L.nelion - 1;
          if (nel >= 0 && nel < a.nspec) {  // invalid species: no opacity
            const int ic = L.nbuff < 1 ? 1 : (L.nbuff > a.length ? a.length : L.nbuff);
            const double xd = a.xnfdop[(size_t)j * a.nspec + nel];
            const double dp = a.dopple[(size_t)j * a.nspec + nel];
            double k0 = (double)L.cgf * xd;
            const double km = (double)a.cont[(size_t)j * a.length + ic - 1] * kLineCutoff;
            if (k0 >= km) {
              k0 = k0 * exp(-(double)L.elo * a.hckt[j]);
              if (k0 >= km) {
                pend = true;
                c_k0 = k0;
                c_km = km;
                c_ad = ((double)L.gamrf + (double)L.gamsf * a.xne[j] + (double)L.gamwf * a.txnxn[j]) / dp;
                c_n10 = (int)(10.0 * dp * a.resolu);
                c_dv = 1.0 / dp / a.resolu;
                c_nb = L.nbuff;
                c_jj = jp;
              }
            }
          }
        }
        continue;
      }
      // the k-th idle lane takes the k-th pending candidate
      const int npend = __popc(pm), nidle = __popc(idle);
      const int rank = __popc(idle & lt);
      const bool take = !act && rank < npend;
      int src = lane;
      if (take) {
        unsigned m = pm;
        for (int q = 0; q < rank; ++q) m &= m - 1u;
        src = __ffs(m) - 1;
      }
      const double t_k0 = __shfl_sync(FULL, c_k0, src), t_km = __shfl_sync(FULL, c_km, src);
      const double t_ad = __shfl_sync(FULL, c_ad, src), t_dv = __shfl_sync(FULL, c_dv, src);
      const int t_n10 = __shfl_sync(FULL, c_n10, src), t_nb = __shfl_sync(FULL, c_nb, src);
      const int t_jj = __shfl_sync(FULL, c_jj, src);
      if (pend && __popc(pm & lt) < nidle) pend = false;  // this candidate was taken
      if (take) {
        act = true;
        kappa0 = t_k0;
        kapmin = t_km;
        adamp = t_ad;
        dv = t_dv;
        n10 = t_n10;
        nb = t_nb;
        jj = t_jj;
        accj = a.acc + (size_t)(a.j0 + jj) * a.length;
        s = 0;
        phase = a.maxprof < n10 ? 1 : 0;
      }
    }
    if (!__any_sync(FULL, act)) break;
    if (!act) continue;
    const double pv = kappa0 * voigt_weideman((double)s * dv, adamp);
    ++nev;
    bool far = false;
    if (s == 0) {
      // the line centre, then the core walk (none when n10dop < 1)
      if (nb >= 1 && nb <= a.length) atomicAdd(accj + nb - 1, pv);
      s = 1;
      act = n10 >= 1;
    } else if (phase == 1) {
      // deciding walk: the scatter limit, then the walk again from s = 1
      const bool below = pv < kapmin;
      if (below || s == n10) {
        lim = below ? s : a.maxprof;
        phase = 2;
        s = 1;
      } else {
        ++s;
      }
    } else {
      const int r = nb + s, b = nb - s;
      if (r >= 1 && r <= a.length) atomicAdd(accj + r - 1, pv);
      if (b >= 1 && b <= a.length) atomicAdd(accj + b - 1, pv);
      if (phase == 2) {
        act = s < lim;
        ++s;
      } else if (pv < kapmin) {
        act = false;
      } else if (s == n10) {
        act = false;
        far = true;
      } else {
        ++s;
      }
    }
    if (far) {
      // far wing: x_wing/n**2 for n10dop < n <= maxstep
      const double xw = pv * ((double)n10 * (double)n10);
      // INT(SQRT(x_wing/kapmin))+1 capped at MAXPROF; saturate before the
      // integer conversion (the reference's INT overflows for huge ratios)
      const double q = sqrt(xw / kapmin);
      const int maxstep = q >= (double)a.maxprof ? a.maxprof : min((int)q + 1, a.maxprof);
      const int lo = max(nb - maxstep, 1), hi = min(nb + maxstep, a.length);
      if (maxstep > n10 && lo <= hi) {
        const unsigned slot = atomicAdd(a.nfar + jj, 1u);
        FarLine f;
        f.c = nb;
        f.n10 = n10;
        f.m = maxstep;
        f.pad = 0;
        f.x = xw;
        a.far[(size_t)jj * a.n + slot] = f;
        int* td = a.tdiff + (size_t)jj * (a.ntiles + 1);
        atomicAdd(td + (lo - 1) / kTile, 1);
        atomicAdd(td + (hi - 1) / kTile + 1, -1);
        // bins n10 < |i - nb| <= maxstep inside the grid
        const int r0 = max(nb + n10 + 1, 1), r1 = min(nb + maxstep, a.length);
        const int b0 = max(nb - maxstep, 1), b1 = min(nb - n10 - 1, a.length);
        nfw += (unsigned long long)(r1 >= r0 ? r1 - r0 + 1 : 0) + (unsigned long long)(b1 >= b0 ? b1 - b0 + 1 : 0);
      }
    }
  }
  if (a.work) {
    for (int o = 16; o > 0; o >>= 1) {
      nev += __shfl_xor_sync(0xffffffffu, nev, o);
      nfw += __shfl_xor_sync(0xffffffffu, nfw, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(a.work, nev);
      atomicAdd(a.work + 1, nfw);
    }
  }
}

// per depth: tile counts from the difference array, exclusive offsets
static __global__ void k_far_scan(int* __restrict__ tdiff, int ntiles, int64_t* __restrict__ off,
                           int64_t* __restrict__ fillptr, int64_t* __restrict__ total) {
  // one block per depth; sequential over tiles in chunks (ntiles is small)
  const int jj = blockIdx.x;
  if (threadIdx.x != 0) return;
  int* td = tdiff + (size_t)jj * (ntiles + 1);
  int64_t* o = off + (size_t)jj * (ntiles + 1);
  int64_t* fp = fillptr + (size_t)jj * ntiles;
  int cnt = 0;
  int64_t run = 0;
  for (int t = 0; t < ntiles; ++t) {
    cnt += td[t];
    o[t] = run;
    fp[t] = run;
    run += cnt;
  }
  o[ntiles] = run;
  total[jj] = run;
}

static __global__ void k_far_fill(const FarLine* __restrict__ far, const unsigned* __restrict__ nfar,
                           int64_t nlines, int length, const int64_t* __restrict__ base,
                           int64_t* __restrict__ fillptr, int ntiles, int* __restrict__ csr) {
  const int jj = blockIdx.y;
  const unsigned nf = nfar[jj];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (unsigned s = warp; s < nf; s += nwarps) {
    const FarLine f = far[(size_t)jj * nlines + s];
    const int lo = max(f.c - f.m, 1), hi = min(f.c + f.m, length);
    const int t0 = (lo - 1) / kTile, t1 = (hi - 1) / kTile;
    for (int t = t0 + lane; t <= t1; t += 32) {
      const int64_t pos = atomicAdd((unsigned long long*)(fillptr + (size_t)jj * ntiles + t), 1ull);
      csr[base[jj] + pos] = (int)s;
    }
  }
}

// far-wing gather + core accumulator -> REAL(4) opacity; zeroes acc for reuse.
//
// One warp (one CTA) takes one sub-tile of kSub bins at one depth, lane l
// the bins lane + 32k; it walks the CSR list of the kTile-bin tile the
// sub-tile belongs to, 32 lines at a time (one line record per lane, the
// next group's records already in flight), and classifies each line
// against the sub-tile:
//   * distant: the whole sub-tile lies inside one far wing of the line
//     (n10 < |i - c| <= m for every bin i) and the sub-tile centre is at
//     least kFarSep bins from c.  The line's terms x/(i - c)^2 are then the
//     Taylor series in v = (i - centre)/h (h = kSub/2) about the centre,
//       x/(D + h v)^2 = sum_k (x/D^2) (k+1) (-h/D)^k v^k,  D = centre - c,
//     |h v / D| < 1/4, and the lane adds the first kFarTerms coefficients
//     (relative truncation below 1e-8);
//   * otherwise, if any of its bins is in the line's far wing, the line is
//     broadcast to the warp (shuffles) and every bin takes x/n^2 itself,
//     the lines in list order.
// At the end the warp adds its lanes' coefficients and each bin evaluates
// the polynomial.  Most of the C3 far-wing terms come from strong lines
// thousands of bins away, so the direct work drops to a few per cent of
// the terms.  Warps share nothing, so a sub-tile next to strong line
// centres (long direct list) holds up no other sub-tile.
constexpr int kSub = 128;       // bins per sub-tile (one warp)
constexpr int kSubs = kTile / kSub;
constexpr int kFarSep = 256;    // minimum |centre - c| for an expansion
constexpr int kFarTerms = 16;   // Taylor terms

template <bool kMixed>
static __global__ void __launch_bounds__(32) k_farwing(const FarLine* __restrict__ far, int64_t nlines,
                                                 const int64_t* __restrict__ off,
                                                 const int64_t* __restrict__ base,
                                                 const int* __restrict__ csr, int ntiles, int length,
                                                 int j0, double* __restrict__ acc,
                                                 float* __restrict__ opac,
                                                 unsigned long long* __restrict__ work) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int kPer = kSub / 32;
  const int jj = blockIdx.y, t = blockIdx.x / kSubs, j = j0 + jj;
  const int lane = threadIdx.x;
  const int lo = t * kTile + (blockIdx.x % kSubs) * kSub + 1;  // first bin of the sub-tile (1-based)
  if (lo > length) return;
  const int hi = min(lo + kSub - 1, length);                   // last bin inside the grid
  const double centre = lo + 0.5 * (kSub - 1);                 // expansion centre
  const int i0 = lo + lane;                                    // bins i0 + 32k
  double sum[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) sum[k] = 0.0;
  double b[kFarTerms];
#pragma unroll
  for (int k = 0; k < kFarTerms; ++k) b[k] = 0.0;
  unsigned nexp = 0, ndir = 0;
  const int64_t* o = off + (size_t)jj * (ntiles + 1);
  const int64_t e0 = base[jj] + o[t], e1 = base[jj] + o[t + 1];
  const FarLine* fj = far + (size_t)jj * nlines;
  const FarLine none{0, 0, 0, 0, 0.0};
  // two-stage prefetch: the record of the next group, the index of the one after
  int idx = e0 + lane < e1 ? csr[e0 + lane] : -1;
  FarLine f = idx >= 0 ? fj[idx] : none;
  idx = e0 + 32 + lane < e1 ? csr[e0 + 32 + lane] : -1;
  for (int64_t c0 = e0; c0 < e1; c0 += 32) {
    const FarLine fn = idx >= 0 ? fj[idx] : none;
    idx = c0 + 64 + lane < e1 ? csr[c0 + 64 + lane] : -1;
    bool direct = false;
    if (c0 + lane < e1) {
      int dmin, dmax;
      bool outside = true;
      if (f.c < lo) {
        dmin = lo - f.c;
        dmax = hi - f.c;
      } else if (f.c > hi) {
        dmin = f.c - hi;
        dmax = f.c - lo;
      } else {
        outside = false;
        dmin = 0;
        dmax = max(f.c - lo, hi - f.c);
      }
      const double D = centre - (double)f.c;
      if (outside && dmin > f.n10 && dmax <= f.m && fabs(D) >= (double)kFarSep) {
        // 1/D from the single-precision reciprocal and one Newton-Raphson
        // step (relative error ~1e-14, far below the truncation)
        const double r0 = (double)__frcp_rn((float)D);
        const double r = fma(r0, fma(-D, r0, 1.0), r0);
        const double g = -0.5 * kSub * r, g2 = g * g, g4 = g2 * g2;
        // powers p*g^k in four independent chains (k mod 4)
        double p0 = f.x * r * r, p1 = p0 * g, p2 = p0 * g2, p3 = p1 * g2;
#pragma unroll
        for (int k = 0; k < kFarTerms; k += 4) {
          b[k] = fma((double)(k + 1), p0, b[k]);
          b[k + 1] = fma((double)(k + 2), p1, b[k + 1]);
          b[k + 2] = fma((double)(k + 3), p2, b[k + 2]);
          b[k + 3] = fma((double)(k + 4), p3, b[k + 3]);
          p0 *= g4;
          p1 *= g4;
          p2 *= g4;
          p3 *= g4;
        }
        ++nexp;
      } else {
        direct = dmax > f.n10 && dmin <= f.m;
      }
    }
    // the direct lines of this group, in list order, broadcast to every bin
    unsigned bal = __ballot_sync(FULL, direct);
    ndir += __popc(bal);
    while (bal) {
      const int src = __ffs(bal) - 1;
      bal &= bal - 1u;
      const int c = __shfl_sync(FULL, f.c, src);
      const int n10 = __shfl_sync(FULL, f.n10, src);
      const int m = __shfl_sync(FULL, f.m, src);
      const double x = __shfl_sync(FULL, f.x, src);
      if (kMixed) {
        const float xf = (float)x;
        const float fb = (float)(i0 - c);  // exact: |i - c| < 2^24
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          const int d = abs(i0 + 32 * k - c);
          if (d > n10 && d <= m) {
            const float df = fb + (float)(32 * k);
            sum[k] += (double)(xf * __frcp_rn(df * df));
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          const int d = abs(i0 + 32 * k - c);
          if (d > n10 && d <= m) {
            const double dd = (double)d;
            sum[k] += x / (dd * dd);
          }
        }
      }
    }
    f = fn;
  }
  // the warp's expansion: lane sums, then the polynomial at each bin
#pragma unroll
  for (int k = 0; k < kFarTerms; ++k)
    for (int sh = 16; sh > 0; sh >>= 1) b[k] += __shfl_xor_sync(FULL, b[k], sh);
  double* accj = acc + (size_t)j * length;
  float* oj = opac + (size_t)j * length;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int i = i0 + 32 * k;
    if (i <= length) {
      const double v = ((double)i - centre) * (2.0 / kSub);
      double pv = b[kFarTerms - 1];
#pragma unroll
      for (int q = kFarTerms - 2; q >= 0; --q) pv = fma(pv, v, b[q]);
      oj[i - 1] = (float)(accj[i - 1] + (sum[k] + pv));
      accj[i - 1] = 0.0;
    }
  }
  if (work) {
    for (int sh = 16; sh > 0; sh >>= 1) nexp += __shfl_xor_sync(FULL, nexp, sh);
    if (lane == 0) {
      atomicAdd(work + 2, (unsigned long long)nexp);
      atomicAdd(work + 3, (unsigned long long)ndir);
    }
  }
}

// ---------------------------------------------------------------- spectrum
struct SpecArgs {
  const JoshOps* ops;
  const double *wledge, *contabs, *contscat, *rhox, *hkt;
  int nedge, stride, nrhox, length;
  double wbegin, ratio;
  const float* opac;  // [nrhox][length]
  double *flux, *cont;
};

struct SpecWS {
  JoshWS w;
  double A[kNx * kLd];  // the warp's scattering matrix
  double acont[kKwMax], sigmac[kKwMax], aline[kKwMax], sigmal[kKwMax], sline[kKwMax],
      bnu[kKwMax];
};

static __global__ void __launch_bounds__(128) k_spectrum(SpecArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpG g(lane);
  const int nwarp = blockDim.x >> 5;
  double* rhox_s = reinterpret_cast<double*>(smem_raw);
  SpecWS* wsa = reinterpret_cast<SpecWS*>(smem_raw + sizeof(double) * kKwMax);
  SpecWS& S = wsa[wid];
  for (int j = threadIdx.x; j < a.nrhox; j += blockDim.x) rhox_s[j] = a.rhox[j];
  __syncthreads();
  const JoshOps& ops = *a.ops;
  const int nr = a.nrhox;
  for (int iw = blockIdx.x * nwarp + wid; iw < a.length; iw += gridDim.x * nwarp) {
    const double wave8 = a.wbegin * powi(a.ratio, iw);
    // iedge_sv = 1 + #{e >= 2 : wledge(e) <= wave}  (setup_opacity_sv walk)
    int lo = 1, hi = a.nedge - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.wledge[mid - 1] <= wave8) lo = mid;
      else hi = mid - 1;
    }
    const int ie = lo;
    const double wl0 = a.wledge[ie - 1], wl1 = a.wledge[ie];
    const double half = (wl0 + wl1) * 0.5, del = powi(wl1 - wl0, 2) * 0.5;
    const double c1 = (wave8 - half) * (wave8 - wl1) / del;
    const double c2 = (wl0 - wave8) * (wave8 - wl1) * 2.0 / del;
    const double c3 = (wave8 - wl0) * (wave8 - half) / del;
    const double freq = kClightNms / wave8;
    const double freq15 = freq / 1.0e15;
    const double f3 = powi(freq15, 3);
    for (int j = lane; j < nr; j += 32) {
      const double* ca = a.contabs + (size_t)j * a.stride + 3 * (ie - 1);
      const double* cs = a.contscat + (size_t)j * a.stride + 3 * (ie - 1);
      S.acont[j] = exp10(c1 * ca[0] + c2 * ca[1] + c3 * ca[2]);
      S.sigmac[j] = exp10(c1 * cs[0] + c2 * cs[1] + c3 * cs[2]);
      const double ehvkt = exp(-freq * a.hkt[j]);
      const double stim = 1.0 - ehvkt;
      const double bnu = kBnuPrefac * f3 * ehvkt / stim;
      S.bnu[j] = bnu;
      S.aline[j] = 0.0;
      S.sigmal[j] = 0.0;
      S.sline[j] = bnu;
    }
    wsync();
    double surf = 0.0, hnu = 0.0;
    g_josh(g, ops, rhox_s, nr, S.acont, S.aline, S.sigmac, S.sigmal, S.bnu, S.sline, S.bnu, S.w, S.A,
           nullptr, &surf);
    surf = __shfl_sync(0xffffffffu, surf, 0);
    for (int j = lane; j < nr; j += 32) {
      const double ehvkt = exp(-freq * a.hkt[j]);
      const double stim = 1.0 - ehvkt;
      const float asyn =
          (float)((double)a.opac[(size_t)j * a.length + iw] * (1.0 - exp(-freq * a.hkt[j])));
      S.aline[j] = (double)asyn * (1.0 - 0.0);
      S.sline[j] = S.bnu[j] * stim / (1.0 - ehvkt);
      S.sigmal[j] = 0.0;
    }
    wsync();
    g_josh(g, ops, rhox_s, nr, S.acont, S.aline, S.sigmac, S.sigmal, S.bnu, S.sline, S.bnu, S.w, S.A,
           nullptr, &hnu);
    if (lane == 0) {
      const double resid = hnu / surf;
      a.flux[iw] = resid * surf;
      a.cont[iw] = surf;
    }
    wsync();
  }
}

// ---------------------------------------------------------------- NLTE list
// compute_line_opacity's normal-metal branch (TYPE 0, 3 and the He I
// fallthrough TYPE <= -3; synthe_module.f90:3400-3458), FP64.  One warp per
// (record, depth); lanes take 32 consecutive grid points of a wing, the
// first lane below the cutoff ends the wing (red: tested before the add,
// blue: after it).  Points blueward of WCON are skipped, WCON..WTAIL tapers.
// Grid wavelengths are wbegin * ratio**(i-1) per point (the reference walks
// them by repeated multiplication; the two agree to ~1e-11 relative).
struct NlteArgs {
  const atlasgpu_nlte_line* rec;
  int64_t n;
  int length, nrhox, nspec;
  double wbegin, ratio, wlend, dopratio;
  const float* cont;                // [nrhox][length]
  const double *xnfdop, *dopple;    // [nrhox][nspec]
  const double *xne, *txnxn, *hckt, *emerge;  // [nrhox]
  const double* contx;              // CONTX(26,17) column-major
  double* acc;                      // [nrhox][length]
  const double* xnfpel = nullptr;   // [nrhox][nspec] XNFPEL = populations / RHO; null: Shore lines skipped
  // merged-continuum edges (TYPE >= 4): per record its ordinal m (-1: none)
  // and per (m, depth) the grid indices NBUFF1, NBUFF2, NBUFF3 and a flag
  // (0: the edge misses the grid), computed on the host with the C library
  const int* mord = nullptr;
  const int4* mbins = nullptr;
};

// compute_line_opacity's autoionizing (Shore) lines, synthe_module.f90:3609-3650:
// KAPPA0 = GAMMAW*GF*XNFPEL with the two continuum gates around the Boltzmann
// factor, then the Fano profile KAPPA0*(GAMMAS*EPSIL + GAMMAW)/(EPSIL**2+1)/GAMMAW,
// EPSIL = 2*(FREQ - FRELIN)/GAMMAR, red wing from nbuff to the grid end and blue
// wing to its start, each point added and then tested against
// continuum(i)*LINE_CUTOFF.  One warp per (record, depth), 32 points per step.
static __device__ __forceinline__ void synthe_shore_pair(const NlteArgs& a, const atlasgpu_nlte_line& r, int j,
                                                         int lane) {
  const int nel = r.nelion - 1;
  const float* cont = a.cont + (size_t)j * a.length;
  double* acc = a.acc + (size_t)j * a.length;
  const double wl = r.wlvac * a.dopratio;
  const int nbuff = r.nbuff;
  const double gr = (double)r.gammar, gs = (double)r.gammas, gw = (double)r.gammaw;
  double kappa0 = gw * (double)r.gf * a.xnfpel[(size_t)j * a.nspec + nel];
  const int ic = nbuff < 1 ? 1 : (nbuff > a.length ? a.length : nbuff);
  const double kapmin = (double)cont[ic - 1] * kLineCutoff;
  if (kappa0 < kapmin) return;
  kappa0 = kappa0 * exp(-(double)r.elo * a.hckt[j]);
  if (kappa0 < kapmin) return;
  const double frelin = kClightNms / wl;
  auto kappa_at = [&](int ib) {
    const double freq = kClightNms / (a.wbegin * powi(a.ratio, ib - 1));
    const double eps = 2.0 * (freq - frelin) / gr;
    return kappa0 * (gs * eps + gw) / (eps * eps + 1.0) / gw;
  };
  if (wl <= a.wlend) {
    const int minred = nbuff > 1 ? nbuff : 1;
    for (int base = minred; base <= a.length; base += 32) {
      const int ib = base + lane;
      const bool in = ib <= a.length;
      const double k = in ? kappa_at(ib) : 0.0;
      const unsigned sb = __ballot_sync(0xffffffffu, in && k < (double)cont[ib - 1] * kLineCutoff);
      const int first = sb ? __ffs(sb) - 1 : 32;
      if (in && lane <= first) atomicAdd(acc + ib - 1, k);
      if (sb) break;
    }
    if (nbuff == 1 || wl < a.wbegin) return;
  }
  const int ib0 = a.length + 1 < nbuff ? a.length + 1 : nbuff;
  const int maxblue = ib0 - 1;
  for (int i0 = 1; i0 <= maxblue; i0 += 32) {
    const int i = i0 + lane;
    const int ib = ib0 - i;
    const bool in = i <= maxblue;
    const double k = in ? kappa_at(ib) : 0.0;
    const unsigned sb = __ballot_sync(0xffffffffu, in && k < (double)cont[ib - 1] * kLineCutoff);
    const int first = sb ? __ffs(sb) - 1 : 32;
    if (in && lane <= first) atomicAdd(acc + ib - 1, k);
    if (sb) break;
  }
}

static __global__ void __launch_bounds__(256) k_synthe_nlte(NlteArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t npair = a.n * a.nrhox;
  for (int64_t p = w0; p < npair; p += nw) {
    const int64_t il = p / a.nrhox;
    const int j = (int)(p % a.nrhox);
    const atlasgpu_nlte_line r = a.rec[il];
    const int t = r.itype;
    if (t == 1 && a.xnfpel && r.nelion >= 1 && r.nelion <= a.nspec) {
      synthe_shore_pair(a, r, j, lane);
      continue;
    }
    if (t >= 4) {
      // merged-continuum edge (synthe_module.f90:3652-3696): flat to NBUFF2,
      // then tapering to zero at NBUFF3
      if (!a.mbins) continue;
      const int m = a.mord[il];
      if (m < 0) continue;
      const int4 b = a.mbins[(size_t)m * a.nrhox + j];
      if (!b.w) continue;
      const double kappa = (double)r.gf * a.xnfpel[(size_t)j * a.nspec + r.nelion - 1] *
                           exp(-(double)r.elo * a.hckt[j]);
      const double dn = (double)(b.z - b.y);
      const int hi = b.z < a.length ? b.z : a.length;
      double* acc = a.acc + (size_t)j * a.length;
      for (int ib = b.x + lane; ib <= hi; ib += 32) {
        const double tail = ib > b.y ? (double)(b.z - ib) / dn : 1.0;
        atomicAdd(acc + ib - 1, kappa * tail);
      }
      continue;
    }
    if (!(t == 0 || t == 3 || t <= -3) || r.nelion < 1 || r.nelion > a.nspec) continue;
    const float* cont = a.cont + (size_t)j * a.length;
    double* acc = a.acc + (size_t)j * a.length;
    const double wl = r.wlvac * a.dopratio;
    const int nbuff = r.nbuff;
    const int nel = r.nelion - 1;
    const double xd = a.xnfdop[(size_t)j * a.nspec + nel], dp = a.dopple[(size_t)j * a.nspec + nel];
    double kappa0 = (double)r.gf * xd;
    const int ic = nbuff < 1 ? 1 : (nbuff > a.length ? a.length : nbuff);
    const double kapmin = (double)cont[ic - 1] * kLineCutoff;
    if (kappa0 < kapmin) continue;
    kappa0 = kappa0 * exp(-(double)r.elo * a.hckt[j]);
    if (kappa0 < kapmin) continue;
    double wcon = 0.0, wtail = 0.0;
    if (r.ncon > 0) {
      const double cx = a.contx[(size_t)(r.nelionx - 1) * 26 + (r.ncon - 1)];
      wcon = 1.0e7 / (cx - a.emerge[j]) * a.dopratio;
      wtail = 1.0e7 / (cx - a.emerge[j] - 500.0) * a.dopratio;
    }
    const double adamp = ((double)r.gammar + (double)r.gammas * a.xne[j] + (double)r.gammaw * a.txnxn[j]) / dp;
    const double dopwl = dp * wl;
    if (wl <= a.wlend) {
      const int minred = nbuff > 1 ? nbuff : 1;
      for (int base = minred; base <= a.length; base += 32) {
        const int ib = base + lane;
        bool use = false, stop = false;
        double kappa = 0.0;
        if (ib <= a.length) {
          const double wave = a.wbegin * powi(a.ratio, ib - 1);
          if (wave >= wcon) {
            use = true;
            kappa = kappa0 * voigt_weideman(fabs(wave - wl) / dopwl, adamp);
            if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
            stop = kappa < (double)cont[ib - 1] * kLineCutoff;
          }
        }
        const unsigned sb = __ballot_sync(0xffffffffu, stop);
        const int first = sb ? __ffs(sb) - 1 : 32;
        if (use && lane < first) atomicAdd(acc + ib - 1, kappa);
        if (sb) break;
      }
      if (minred == 1 || wl < a.wbegin) continue;
    }
    const int ib0 = a.length + 1 < nbuff ? a.length + 1 : nbuff;
    const int maxblue = ib0 - 1;
    for (int i0 = 1; i0 <= maxblue; i0 += 32) {
      const int i = i0 + lane;
      const int ib = ib0 - i;
      bool use = false, stop = false;
      double kappa = 0.0;
      if (i <= maxblue) {
        const double wave = a.wbegin * powi(a.ratio, ib - 1);
        if (wave >= wcon) {
          use = true;
          kappa = kappa0 * voigt_weideman(fabs(wave - wl) / dopwl, adamp);
          if (wave < wtail) kappa = kappa * ((wave - wcon) / (wtail - wcon));
          stop = kappa < (double)cont[ib - 1] * kLineCutoff;
        }
      }
      const unsigned sb = __ballot_sync(0xffffffffu, stop);
      const int first = sb ? __ffs(sb) - 1 : 32;
      if (use && lane <= first) atomicAdd(acc + ib - 1, kappa);
      if (sb) break;
    }
  }
}

// opacity [nrhox][length] (REAL(4)) += the FP64 contribution
static __global__ void k_add_f64_to_f32(const double* __restrict__ acc, float* __restrict__ out, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = (float)((double)out[e] + acc[e]);
}

}  // namespace atlasgpu
