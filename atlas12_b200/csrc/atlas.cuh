// atlas.cuh -- ATLAS12 opacity-sampling hot path (sm_100a).
//
//  k_atlas_prep   per stored line: unpack LINEREC, wavelength, frequency and
//                 continuum-table brackets, TABLOG conversions (the
//                 iteration-invariant half of LINOP1, atlas12_modules.f90:18176-18235)
//  k_atlas_linop  per line: coarse/fine depth gating and the <= 100-point red
//                 and blue wing walks of LINOP1 (:18236-18370) with the
//                 tabulated / full Kurucz Voigt, into XLINES (FP64 atomics)
//  k_atlas_rt     per frequency (one warp): Planck terms, opacities, JOSH,
//                 negative floor and the TCORR/RADIAP/ROSS mode-2 sums of
//                 RUN_RT_PASS (:3905-3949), accumulated per warp in frequency
//                 order (deterministic)
//  k_atlas_reduce per depth: fixed-order sum of the per-warp partials
#pragma once
#include "common.cuh"
#include "josh.cuh"
#include "surrogate.cuh"
#include "voigt.cuh"

namespace atlasgpu {

struct AtlasLine {
  double wlvac;          // WLVAC (nm)
  double cgf, elo;       // CGF, ELO (TABLOG-decoded)
  double gr, gs, gw;     // GAMMAR, GAMMAS, GAMMAW
  int nu, nucont;        // 1-based brackets
  int nelion;            // 1-based species, 0 = line skipped
  int pad;
};

struct AtlasPrepArgs {
  const int32_t* linedata;  // [n][4]
  int64_t n;
  const double* tablog;     // [65536]
  const double* waveset;    // [numnu]
  int numnu;
  const int32_t* iwavetab;  // [nwave+1]
  int nwave;
  int nspec;
  AtlasLine* out;
  int64_t* flagged;
  unsigned long long* nflag;
  int64_t flag_cap;
};

static __global__ void k_atlas_prep(AtlasPrepArgs a) {
  const double RATIOLG = log(1.0 + 1.0 / 2000000.0);
  const double CEN_PREFAC4 = 0.026538 / kSqrtPi / kClightNms;
  const double FOURPI_C_INV = 1.0 / (4.0 * kPi * kClightNms);
  const double start = a.waveset[0] - 1.0, stop = a.waveset[a.numnu - 1] + 1.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t* r = a.linedata + 4 * i;
    const int32_t iwl = r[0];
    const int16_t ielion = (int16_t)(r[1] & 0xffff), ielo = (int16_t)((uint32_t)r[1] >> 16);
    const int16_t igf = (int16_t)(r[2] & 0xffff), igr = (int16_t)((uint32_t)r[2] >> 16);
    const int16_t igs = (int16_t)(r[3] & 0xffff), igw = (int16_t)((uint32_t)r[3] >> 16);
    AtlasLine L;
    L.pad = 0;
    // NUCONT = first k with IWL < IWAVETAB(k), clamped to NWAVE+1
    int lo = 1, hi = a.nwave + 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (iwl < a.iwavetab[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    L.nucont = lo;
    int nel = ielion / 10;
    nel = nel < 0 ? -nel : nel;
    const double wl = exp(iwl * RATIOLG);
    L.wlvac = wl;
    L.nelion = (nel < 1 || nel > a.nspec || wl < start || wl > stop) ? 0 : nel;
    // NU = first grid point with WLVAC < WAVESET(NU) (clamped at NUMNU)
    lo = 1;
    hi = a.numnu;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (wl < a.waveset[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    L.nu = lo;
    // a one-ulp difference of the device exp could move a line across a grid
    // point only within a few ulps of it: flag those for the host
    const double g0 = a.waveset[lo - 1];
    const double gm = lo > 1 ? a.waveset[lo - 2] : -1.0;
    if (fabs(g0 - wl) <= 8.0 * 2.2e-16 * wl || fabs(wl - gm) <= 8.0 * 2.2e-16 * wl) {
      const unsigned long long k = atomicAdd(a.nflag, 1ull);
      if ((int64_t)k < a.flag_cap) a.flagged[k] = i;
    }
    const double wl4 = wl;
    L.cgf = CEN_PREFAC4 * wl4 * a.tablog[(int)igf + 32768];
    L.elo = a.tablog[(int)ielo + 32768];
    L.gr = a.tablog[(int)igr + 32768] * wl4 * FOURPI_C_INV;
    L.gs = a.tablog[(int)igs + 32768] * wl4 * FOURPI_C_INV;
    L.gw = a.tablog[(int)igw + 32768] * wl4 * FOURPI_C_INV;
    a.out[i] = L;
  }
}

// XLINOP record preparation: the per-record part of XLINOP's read loop
// (atlas12_modules.f90:19992-20036) -- NUCONT from IWL, NU from WLVAC (both
// advanced monotonically in the reference; binary searches here, the same on
// wavelength-sorted records), the TYPE dispatch, and CONTX(NCON,NELIONX) for
// the continuum-edge cutoff.  Records the normal branch does not walk get
// NELION = 0.
struct XlinopPrepArgs {
  const atlasgpu_nlte_line* rec;
  int64_t n;
  const double* waveset;
  int numnu;
  const int32_t* iwavetab;  // [nwave+1]
  int nwave, nspec;
  const double* contx;      // CONTX(25,16) column-major
  AtlasLine* out;
  double* lcontx;           // [n] CONTX(NCON,NELIONX) or 0
};

static __global__ void k_xlinop_prep(XlinopPrepArgs a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const atlasgpu_nlte_line r = a.rec[i];
    AtlasLine L;
    L.pad = 0;
    L.wlvac = r.wlvac;
    L.cgf = (double)r.gf;
    L.elo = (double)r.elo;
    L.gr = (double)r.gammar;
    L.gs = (double)r.gammas;
    L.gw = (double)r.gammaw;
    int lo = 1, hi = a.nwave + 1;  // NUCONT = first k with IWL < IWAVETAB(k), clamped to NWAVE+1
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (r.nbuff < a.iwavetab[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    L.nucont = lo;
    lo = 1;  // NU = first grid point with WLVAC < WAVESET(NU); NUMNU+1 when none
    hi = a.numnu + 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (r.wlvac < a.waveset[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    L.nu = lo;
    const bool normal = r.itype == 0 || r.itype == 3;
    L.nelion = (normal && r.nelion >= 1 && r.nelion <= a.nspec && L.nu < a.numnu) ? r.nelion : 0;
    const int ncon = r.ncon > 10 ? 0 : r.ncon;
    a.lcontx[i] = (ncon > 0) ? a.contx[(size_t)(r.nelionx - 1) * 25 + (ncon - 1)] : 0.0;
    a.out[i] = L;
  }
}

// XLINOP's autoionizing (TYPE 1, Fano profile, atlas12_modules.f90:20201-20226)
// and merged-continuum (any other TYPE but 0, 2, 3 and -1, :20228-20245)
// records: one warp per (record, depth), 32 grid points per step; the same
// operations as the reference per point, FP64 atomics into XLINES.
struct XShoreArgs {
  const atlasgpu_nlte_line* rec;
  const AtlasLine* lines;  // NU and NUCONT of every record (k_xlinop_prep)
  int64_t n;
  int nrhox, kw, nspec, numnu;
  const double* waveset;
  const double* tabcont;    // [nwave+1][kw]
  const double *xnfp, *rho;  // XNFP(J,NELION) [nspec][kw], RHO(J) [kw]
  const double *hckt, *emerge;
  double* xl;               // XLINES(J, NU): [numnu][kw]
};

static __global__ void __launch_bounds__(256) k_xlinop_shore(XShoreArgs a) {
  constexpr double kRydbergInf = 109737.31568157;
  const int lane = threadIdx.x & 31;
  const int64_t npairs = a.n * a.nrhox;
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = w0; p < npairs; p += nw) {
    const int64_t i = p / a.nrhox;
    const int j = (int)(p - i * a.nrhox);
    const atlasgpu_nlte_line r = a.rec[i];
    const int t = r.itype;
    if (t == 0 || t == 2 || t == 3 || t == -1) continue;
    const int nu = a.lines[i].nu, nucont = a.lines[i].nucont;
    if (nu >= a.numnu || r.nelion < 1 || r.nelion > a.nspec) continue;
    const double xnfp = a.xnfp[(size_t)(r.nelion - 1) * a.kw + j], rho = a.rho[j];
    const double bz = exp(-((double)r.elo * a.hckt[j]));
    double* xl = a.xl + j;
    if (t == 1) {
      const double tc = a.tabcont[(size_t)(nucont - 1) * a.kw + j];
      const double g = (double)r.gf, ashore = (double)r.gammas, bshore = (double)r.gammaw;
      const double gammar = (double)r.gammar;
      const double frelin = __ddiv_rn(kClightNms, r.wlvac);
      double center = __ddiv_rn(__dmul_rn(__dmul_rn(bshore, g), xnfp), rho);
      if (center < tc) continue;
      center = __dmul_rn(center, bz);
      if (center < tc) continue;
      // red wing NU .. min(NU + 2000, NUMNU), blue wing NU-1 .. max(NU-2000, 1)
      for (int side = 0; side < 2; ++side) {
        const int first = side == 0 ? nu : nu - 1;
        const int count = side == 0 ? min(nu + 2000, a.numnu) - nu + 1 : min(2000, nu - 1);
        for (int s0 = 0; s0 < count; s0 += 32) {
          const int s = s0 + lane;
          const bool valid = s < count;
          const int iw = side == 0 ? first + s : first - s;
          double cv = 0.0;
          if (valid) {
            const double ep = __ddiv_rn(
                __dmul_rn(2.0, __dsub_rn(__ddiv_rn(kClightNms, a.waveset[iw - 1]), frelin)), gammar);
            cv = __ddiv_rn(__ddiv_rn(__dmul_rn(center, __dadd_rn(__dmul_rn(ashore, ep), bshore)),
                                     __dadd_rn(__dmul_rn(ep, ep), 1.0)),
                           bshore);
          }
          const unsigned below = __ballot_sync(0xffffffffu, valid && cv < tc);
          const int stop = below ? __ffs(below) - 1 : 32;  // the first point below TABCONT is added, then the wing ends
          if (valid && lane <= stop) atomicAdd(xl + (size_t)(iw - 1) * a.kw, cv);
          if (below) break;
        }
      }
    } else {
      const double z = r.nelion == 4 ? 2.0 : 1.0;
      const double nlast = (double)t;
      const double rw = __ddiv_rn(1.0e7, r.wlvac);
      const double wshift =
          __ddiv_rn(1.0e7, __dsub_rn(rw, __ddiv_rn(__dmul_rn(kRydbergInf, __dmul_rn(z, z)), __dmul_rn(nlast, nlast))));
      const double wmerge = __ddiv_rn(1.0e7, __dsub_rn(rw, __dmul_rn(a.emerge[j], __dmul_rn(z, z))));
      const double wmax = wmerge > wshift ? wmerge : wshift;
      const double con = __ddiv_rn(__dmul_rn(__dmul_rn((double)r.gf, xnfp), bz), rho);
      const int hi = min(nu + 1000, a.numnu);
      for (int iw0 = nu; iw0 <= hi; iw0 += 32) {
        const int iw = iw0 + lane;
        const bool in = iw <= hi && !(wmax < a.waveset[iw - 1]);
        const unsigned out = __ballot_sync(0xffffffffu, iw <= hi && !in);
        const int stop = out ? __ffs(out) - 1 : 32;  // the walk ends at the first point past WMAX
        if (in && lane < stop) atomicAdd(xl + (size_t)(iw - 1) * a.kw, con);
        if (out) break;
      }
    }
  }
}

// ------------------------------------------------------ exact XLINES sums
// LINOP1 adds each wing value into XLINES(J, NU).  In the reference the adds
// come one at a time in line order; here thousands of warps add at once, and
// FP64 atomics would make the sum depend on their order.  So each value is
// added as a fixed-point integer instead: y = value * 2^k_J (k_J per depth,
// from a bound on the largest value there) split into three 48-bit chunks,
// each added to its own unsigned 64-bit word (16 bits of headroom: 65,536
// adds of the largest value per bin).  Integer sums do not depend on the
// order, and the words hold the exact sum (values below 2^-k_J, i.e. about
// 2^-137 of the depth's bound, round to that unit), so XLINES is the exact
// sum rounded once to FP64: bit-identical from run to run and within an
// ulp of any order of FP64 additions.  Layout [numnu][3][kw] (word w of
// (J, NU) at ((NU-1)*3 + w)*kw + J-1): a warp's lanes at consecutive
// depths add to consecutive words.
constexpr int kFixWords = 3;
constexpr double kFixTop = 0x1p-96, kFixMid = 0x1p-48;

__device__ __forceinline__ void fix_add(unsigned long long* w, int wstride, double y) {
  const double t2 = floor(y * kFixTop);
  const double r2 = y - t2 * 0x1p96;  // exact: the bits of y below 2^96
  const double t1 = floor(r2 * kFixMid);
  const double r1 = r2 - t1 * 0x1p48;  // exact: the bits below 2^48
  const double t0 = rint(r1);          // the one rounding, to the unit 2^-k
  if (t2 > 0.0) atomicAdd(w + 2 * wstride, (unsigned long long)t2);
  if (t1 > 0.0) atomicAdd(w + wstride, (unsigned long long)t1);
  if (t0 > 0.0) atomicAdd(w, (unsigned long long)t0);
}

// The exact integer x2 2^96 + x1 2^48 + x0, rounded to nearest FP64, times unscale (a power of 2)
__host__ __device__ inline double fix_to_double(unsigned long long x0, unsigned long long x1, unsigned long long x2,
                                                double unscale) {
  constexpr unsigned long long m48 = (1ull << 48) - 1;
  x1 += x0 >> 48;
  x0 &= m48;
  x2 += x1 >> 48;
  x1 &= m48;
  // 64-bit limbs of the value (at most 160 bits)
  const unsigned long long lo = x0 | (x1 << 48);
  const unsigned long long mid = (x1 >> 16) | (x2 << 32);
  const unsigned long long hi = x2 >> 32;
  unsigned long long top;
  bool sticky;
  int e;  // value = (top with sticky) * 2^e
  if (hi) {
#ifdef __CUDA_ARCH__
    const int z = __clzll((long long)hi);
#else
    const int z = __builtin_clzll(hi);
#endif
    top = (hi << z) | (mid >> (64 - z));  // z >= 32 (hi < 2^32)
    sticky = (mid << z) != 0 || lo != 0;
    e = 128 - z;
  } else if (mid) {
#ifdef __CUDA_ARCH__
    const int z = __clzll((long long)mid);
#else
    const int z = __builtin_clzll(mid);
#endif
    top = z ? (mid << z) | (lo >> (64 - z)) : mid;
    sticky = z ? (lo << z) != 0 : lo != 0;
    e = 64 - z;
  } else {
    top = lo;
    sticky = false;
    e = 0;
  }
  // the sticky bit in bit 0 keeps the round-to-nearest of the 64-bit top exact
#ifdef __CUDA_ARCH__
  const double d = __ull2double_rn(top | (sticky ? 1ull : 0ull));
#else
  const double d = (double)(top | (sticky ? 1ull : 0ull));
#endif
  return ldexp(d, e) * unscale;
}

// The scale 2^k of depth j: every value added there is at most
// CGF(line) * XNFDOP(J, NELION) (the Boltzmann factor and the profile are at
// most 1; 8x margin), so the largest value maps below 2^140 and a bin's
// words stay below 2^64.  cgfmax: the largest CGF of each species' lines.
__device__ inline void fix_scale_depth(const double* xnfdop, int nspec, int kw, int j, const double* cgfmax,
                                       double* scale, double* unscale) {
  double bound = 0.0;
  for (int s = 0; s < nspec; ++s) bound = fmax(bound, cgfmax[s] * xnfdop[(size_t)s * kw + j]);
  if (!(bound > 0.0) || !(bound < 1e300)) {
    scale[j] = 1.0;
    unscale[j] = 1.0;
    return;
  }
  int e;
  frexp(bound, &e);  // bound < 2^e
  scale[j] = ldexp(1.0, 137 - e);
  unscale[j] = ldexp(1.0, e - 137);
}

struct LinopArgs {
  const AtlasLine* lines;
  int64_t n;
  int nrhox, kw, nspec, numnu;
  const double *xnfdop, *dopple;  // [nspec][kw]  (XNFDOP(J,NELION))
  const double *xne, *txnxn, *hckt;
  const double* tabcont;          // [nwave+1][kw]
  const double* waveset;
  const double *h0, *h1, *h2;     // 2001
  const float4* hf;               // (H0, H1, H2, 0) in FP32 [2001], for the mixed-precision walk
  double* xl;                     // XLINES(J, NU): [numnu][kw]
  unsigned long long* npairs;     // diagnostics: walked (line, depth) pairs
  unsigned long long* used;       // LINEUSED: lines above TABCONT at a coarse depth
  // frequency shard NU_LO..NU_HI (1-based; 0 => NUMNU) that receives XLINES: a
  // line is walked only if its +-100-point window meets the shard, and only
  // points inside the shard are added (the walk itself is unchanged)
  int nu_lo = 1, nu_hi = 0;
  // XLINOP's normal-line branch (atlas12_modules.f90:20040-20174) walks the
  // same way with MAX_WING = 2000, LORENTZ_PREFAC = 0.5642 and a blue-wing
  // cutoff at the continuum edge WCON = 1e7 / (CONTX(NCON,NELIONX) - EMERGE(J))
  // per (line, depth): lcontx [n] holds CONTX(NCON,NELIONX) (0: no cutoff),
  // emerge [kw] EMERGE(J).  LINOP1: 100, 1/sqrt(pi), no cutoff (null).
  int max_wing = 100;
  double lorentz = kInvSqrtPi;
  const double* lcontx = nullptr;
  const double* emerge = nullptr;
  // work counter (timed launches only, else null): wing points added into XLINES
  unsigned long long* work = nullptr;
  // exact fixed-point XLINES (see fix_add): words [numnu][3][kw] and the
  // per-depth scale; null: FP64 atomics into xl (XLINOP adds to a caller's XLINES)
  unsigned long long* xfix = nullptr;
  const double* fscale = nullptr;
};

// Adds one wing value into XLINES(J, IW).  kDry: adds nothing and returns
// the number of atomics the add would issue (the counting pass of a timed
// measurement; the walk is the same), else returns 0.
template <bool kDry>
__device__ __forceinline__ int linop_add(const LinopArgs& a, int J, int iw, double cv) {
  if (kDry) {
    if (!a.xfix) return 1;
    const double y = cv * a.fscale[J - 1];
    const double t2 = floor(y * kFixTop);
    const double r2 = y - t2 * 0x1p96;
    const double t1 = floor(r2 * kFixMid);
    const double t0 = rint(r2 - t1 * 0x1p48);
    return (t2 > 0.0) + (t1 > 0.0) + (t0 > 0.0);
  }
  if (a.xfix) fix_add(a.xfix + ((size_t)(iw - 1) * kFixWords) * a.kw + (J - 1), a.kw, cv * a.fscale[J - 1]);
  else atomicAdd(a.xl + (size_t)(iw - 1) * a.kw + (J - 1), cv);
  return 0;
}

// LINOP1's profile value at one wing point, V = (distance in nm) * RDOP with
// RDOP = 1 / (DOPPLE * WLVAC) taken once per (line, depth): tabulated H(v, a)
// for ADAMP <= 0.2 and v <= 10, the Lorentz wing 1/sqrt(pi) a / v^2 beyond,
// the full VOIGT for ADAMP > 0.2 (atlas12_modules.f90:18290-18345).
// F32 (mixed precision) evaluates the tabulated and Lorentz values in FP32
// from FP32 copies of the tables (hf = H0, H1, H2); V, the table index and
// the regime tests stay FP64, so every point uses the table entry the FP64
// walk uses.
static __device__ __noinline__ double linop_full_voigt(const LinopArgs& a, double vv, double adamp) {
  return voigt_kurucz(vv, adamp, a.h0, a.h1, a.h2);
}

template <bool F32>
__device__ __forceinline__ double linop_cv(const LinopArgs& a, double center, double adamp, double dl, double rdop) {
  const double vv = dl * rdop;
  if (adamp > 0.20) return center * linop_full_voigt(a, vv, adamp);
  // written as !(vv <= 10): a V that is not a number (a non-finite model
  // structure) takes the Lorentz branch and never reaches the table index
  if (!(vv <= 10.0)) {
    if (F32) return (double)((float)center * ((float)(a.lorentz * adamp) * __frcp_rn((float)(vv * vv))));
    return center * a.lorentz * adamp / (vv * vv);
  }
  const int iv = (int)(vv * 200.0 + 1.5);
  if (F32) {
    const float4 h = a.hf[iv - 1];
    const float af = (float)adamp;
    return (double)((float)center * fmaf(fmaf(h.z, af, h.y), af, h.x));
  }
  return center * ((a.h2[iv - 1] * adamp + a.h1[iv - 1]) * adamp + a.h0[iv - 1]);
}

// The wing walk stops at the first point whose value is below TABCONT.  In
// FP32 a value within 1e-5 of the threshold is re-evaluated in FP64 for the
// decision, so both precisions stop at the same point.
template <bool F32>
__device__ __forceinline__ bool linop_below(const LinopArgs& a, double cv, double tc, double center, double adamp,
                                            double dl, double rdop) {
  if (F32 && fabs(cv - tc) <= 1.0e-5 * tc) return linop_cv<false>(a, center, adamp, dl, rdop) < tc;
  return cv < tc;
}

// The rest of one (line, depth) walk after a lane gave up on it, by the
// whole warp (lanes over wing points), add-then-test as in the reference:
// red points rnext..iwmax unless rdone, blue offsets bnext..100 unless bdone.
template <bool F32, bool kDry>
static __device__ __noinline__ unsigned linop_finish_warp(const LinopArgs& a, int J, double center, double adamp,
                                                          double rdop, double wlvac, int nu, double tc, int rnext,
                                                          bool rdone, int bnext, bool bdone, double wcon, int lane,
                                                          unsigned long long& atoms) {
  unsigned added = 0;  // points this lane added
  const int iwmax = min(nu + a.max_wing, a.numnu);
  const int nuh = a.nu_hi > 0 ? a.nu_hi : a.numnu;
  if (!rdone) {
    for (int base = rnext; base <= iwmax; base += 32) {
      const int iw = base + lane;
      const bool valid = iw <= iwmax;
      double cv = 0.0;
      bool below = false;
      if (valid) {
        const double dl = a.waveset[iw - 1] - wlvac;
        cv = linop_cv<F32>(a, center, adamp, dl, rdop);
        below = linop_below<F32>(a, cv, tc, center, adamp, dl, rdop);
      }
      const unsigned stop = __ballot_sync(0xffffffffu, valid && below);
      const int last = stop ? base + __ffs(stop) - 1 : iwmax;
      if (valid && iw <= last && iw >= a.nu_lo && iw <= nuh) {
        atoms += linop_add<kDry>(a, J, iw, cv);
        ++added;
      }
      if (stop) break;
    }
  }
  if (!bdone) {
    for (int i0 = bnext; i0 <= a.max_wing; i0 += 32) {
      const int i = i0 + lane;
      const int iw = nu - i;
      // the walk ends before the grid start and (XLINOP) before the continuum edge
      const bool valid = i <= a.max_wing && iw >= 1 && !(a.waveset[iw - 1] < wcon);
      double cv = 0.0;
      bool below = false;
      if (valid) {
        const double dl = wlvac - a.waveset[iw - 1];
        cv = linop_cv<F32>(a, center, adamp, dl, rdop);
        below = linop_below<F32>(a, cv, tc, center, adamp, dl, rdop);
      }
      const unsigned stop = __ballot_sync(0xffffffffu, valid && below);
      const unsigned inval = __ballot_sync(0xffffffffu, !valid);
      const int ilast = stop ? i0 + __ffs(stop) - 1 : a.max_wing;
      if (valid && i <= ilast && iw >= a.nu_lo && iw <= nuh) {
        atoms += linop_add<kDry>(a, J, iw, cv);
        ++added;
      }
      if (stop || inval) break;
    }
  }
  return added;
}

// Warp per line, lane per depth.  Most (line, depth) wing walks stop after a
// few points (the C2 grid is ~50 Doppler widths per step), so each lane
// walks its own depth's red and blue wings for up to kLinopLanePts points,
// and the walks still going are finished by the whole warp.  Lanes of a
// warp touch XLINES(J, IW) at consecutive J: one coalesced atomic per step.
// A warp takes kLinopChunk consecutive lines at a time, so the warps of a
// CTA work on neighbouring lines (the lines are in wavelength order) and
// share the WAVESET window and the XLINES lines they touch in cache.
// Measured on the 500,000-line, 30,000-frequency pass (solar / cool model):
// 4 points per lane and one line per warp 4.45 / 5.49 ms; 16 points, chunks
// of 8 lines and four CTAs per SM (64 registers) 3.74 / 4.80 ms.  In the
// 32-slot batch of one model (per model-iteration, solar / cool giant): 16
// points 2.42 / 3.39 ms, 32 points 2.36 / 3.39, 64 points 2.31 / 3.39; but on
// the bench's mixed 32-model batch 64 points took 2.37 ms against 2.27 for 16.
constexpr int kLinopLanePts = 16;
constexpr int kLinopChunk = 8;
constexpr int kLinopMinBlocks = 4;

// One stored line by one warp (lanes over depths): the coarse and fine
// depth gates and the red and blue wing walks of LINOP1 (:18236-18370).
// walked / points count the walked (line, depth) pairs and the wing points
// this lane added.
template <bool F32, bool kDry = false>
static __device__ __forceinline__ void linop_line(const LinopArgs& a, int64_t il, int lane, unsigned long long& walked,
                                                  unsigned long long& points, unsigned long long& atoms) {
  const int nuh = a.nu_hi > 0 ? a.nu_hi : a.numnu;
  const AtlasLine L = a.lines[il];
  if (L.nelion == 0 || L.nu + a.max_wing < a.nu_lo || L.nu - a.max_wing > nuh) return;
  const double cx = a.lcontx ? a.lcontx[il] : 0.0;
  const double* xdn = a.xnfdop + (size_t)(L.nelion - 1) * a.kw;
  const double* dpn = a.dopple + (size_t)(L.nelion - 1) * a.kw;
  const double* tcv = a.tabcont + (size_t)(L.nucont - 1) * a.kw;
  // coarse gates: depths 8, 16, ... (lane k -> depth 8(k+1)); bit k = IFJ at depth 8(k+1)
  int pass = 0;
  {
    const int J = 8 * (lane + 1);
    if (J <= a.nrhox) {
      double c = L.cgf * xdn[J - 1];
      if (c >= tcv[J - 1]) {
        c = c * exp(-L.elo * a.hckt[J - 1]);
        pass = c >= tcv[J - 1];
      }
    }
  }
  const unsigned ifj = __ballot_sync(0xffffffffu, pass);
  if (ifj == 0) return;
  if (lane == 0 && a.used) atomicAdd(a.used, 1ull);
  const int iwmax = min(L.nu + a.max_wing, a.numnu);
  for (int J0 = 1; J0 <= a.nrhox; J0 += 32) {
    // a round of 32 depths can walk only where its coarse blocks, or the
    // block just above its first, passed: skip it before any load if none did
    {
      const int kl = (J0 + 7) / 8 - 1, kh = (min(J0 + 31, a.nrhox) + 7) / 8 - 1;
      const unsigned rmask = ((2u << kh) - 1u) & ~((1u << (kl > 0 ? kl - 1 : 0)) - 1u);
      if (!(ifj & rmask)) continue;
    }
    const int J = J0 + lane;
    bool walk = false;
    double center = 0.0, tc = 0.0;
    const int K = 8 * ((J + 7) / 8);  // the coarse depth closing J's block
    if (J <= a.nrhox && K <= a.nrhox) {
      const int k = K / 8 - 1;
      const bool cur = (ifj >> k) & 1u;
      tc = tcv[J - 1];
      if (J == K) {
        walk = cur;
        if (walk) center = L.cgf * xdn[J - 1] * exp(-L.elo * a.hckt[J - 1]);
      } else if (cur || (k > 0 && ((ifj >> (k - 1)) & 1u))) {
        // fine depth K-7..K-1 of a block next to a passing coarse depth
        center = L.cgf * xdn[J - 1];
        if (center >= tc) {
          center = center * exp(-L.elo * a.hckt[J - 1]);
          walk = center >= tc;
        }
      }
    }
    if (!__any_sync(0xffffffffu, walk)) continue;
    // XLINOP: no walk at a depth whose continuum edge lies redward of the line
    double wcon = 0.0;
    if (walk && cx > 0.0) {
      wcon = 1.0e7 / (cx - a.emerge[J - 1]);
      if (L.wlvac < wcon) walk = false;
    }
    double adamp = 0.0, rdop = 1.0;
    if (walk) {
      adamp = (L.gr + L.gs * a.xne[J - 1] + L.gw * a.txnxn[J - 1]) / dpn[J - 1];
      rdop = 1.0 / (dpn[J - 1] * L.wlvac);
      ++walked;
    }
    bool rdone = !walk, bdone = !walk;
    int rnext = L.nu, bnext = 1;
    // each walk's next grid wavelength is loaded one point ahead, so the load
    // is in flight while the current point is evaluated (the last load of a
    // walk goes unused; every index stays inside WAVESET)
    double wr = walk ? a.waveset[rnext - 1] : 0.0;
    double wb = (walk && L.nu >= 2) ? a.waveset[L.nu - 2] : 0.0;
#pragma unroll 1
    for (int s = 0; s < kLinopLanePts && __any_sync(0xffffffffu, !rdone || !bdone); ++s) {
      if (!rdone) {
        const int iw = rnext;
        const double wr_next = iw < a.numnu ? a.waveset[iw] : 0.0;
        const double dl = wr - L.wlvac;
        const double cv = linop_cv<F32>(a, center, adamp, dl, rdop);
        if (iw >= a.nu_lo && iw <= nuh) {
          atoms += linop_add<kDry>(a, J, iw, cv);
          ++points;
        }
        if (linop_below<F32>(a, cv, tc, center, adamp, dl, rdop) || iw >= iwmax) {
          rdone = true;
        } else {
          rnext = iw + 1;
          wr = wr_next;
        }
      }
      if (!bdone) {
        const int iw = L.nu - bnext;
        if (iw < 1 || wb < wcon) {
          bdone = true;
        } else {
          const double wb_next = iw >= 2 ? a.waveset[iw - 2] : 0.0;
          const double dl = L.wlvac - wb;
          const double cv = linop_cv<F32>(a, center, adamp, dl, rdop);
          if (iw >= a.nu_lo && iw <= nuh) {
            atoms += linop_add<kDry>(a, J, iw, cv);
            ++points;
          }
          if (linop_below<F32>(a, cv, tc, center, adamp, dl, rdop) || bnext >= a.max_wing) {
            bdone = true;
          } else {
            bnext = bnext + 1;
            wb = wb_next;
          }
        }
      }
    }
    // walks still going: the warp finishes them one at a time
    unsigned ov = __ballot_sync(0xffffffffu, !rdone || !bdone);
    while (ov) {
      const int src = __ffs(ov) - 1;
      ov &= ov - 1;
      const int Js = __shfl_sync(0xffffffffu, J, src);
      const double cs = __shfl_sync(0xffffffffu, center, src);
      const double as = __shfl_sync(0xffffffffu, adamp, src);
      const double ds = __shfl_sync(0xffffffffu, rdop, src);
      const double ts = __shfl_sync(0xffffffffu, tc, src);
      const int rn = __shfl_sync(0xffffffffu, rnext, src);
      const int bn = __shfl_sync(0xffffffffu, bnext, src);
      const bool rd = __shfl_sync(0xffffffffu, (int)rdone, src) != 0;
      const bool bd = __shfl_sync(0xffffffffu, (int)bdone, src) != 0;
      const double wc = __shfl_sync(0xffffffffu, wcon, src);
      points += linop_finish_warp<F32, kDry>(a, Js, cs, as, ds, L.wlvac, L.nu, ts, rn, rd, bn, bd, wc, lane, atoms);
    }
  }
}

// walked (line, depth) pairs, wing points and XLINES atomics, summed over
// the warp's lanes (work[0] points, work[1] atomics)
__device__ __forceinline__ void linop_counts(const LinopArgs& a, int lane, unsigned long long walked,
                                             unsigned long long points, unsigned long long atoms) {
  for (int o = 16; o > 0; o >>= 1) walked += __shfl_xor_sync(0xffffffffu, walked, o);
  if (lane == 0 && walked && a.npairs) atomicAdd(a.npairs, walked);
  if (a.work) {
    for (int o = 16; o > 0; o >>= 1) points += __shfl_xor_sync(0xffffffffu, points, o);
    for (int o = 16; o > 0; o >>= 1) atoms += __shfl_xor_sync(0xffffffffu, atoms, o);
    if (lane == 0) {
      atomicAdd(a.work, points);
      if (atoms) atomicAdd(a.work + 1, atoms);
    }
  }
}

// kDry: the counting pass (walks, counts the wing points and the atomics the
// adds would issue, adds nothing)
template <bool F32, bool kDry = false>
static __device__ __forceinline__ void linop_body(const LinopArgs& a) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long walked = 0, points = 0, atoms = 0;
  for (int64_t il0 = w0 * kLinopChunk; il0 < a.n; il0 += nw * kLinopChunk)
    for (int64_t il = il0; il < il0 + kLinopChunk && il < a.n; ++il)
      linop_line<F32, kDry>(a, il, lane, walked, points, atoms);
  linop_counts(a, lane, walked, points, atoms);
}

template <bool F32>
static __global__ void __launch_bounds__(256, kLinopMinBlocks) k_atlas_linop(LinopArgs a) { linop_body<F32>(a); }

// XLINES(J, NU) from the fixed-point words, which are cleared for the next
// accumulation (grid-stride over NU, threads over depths J < nrhox)
__device__ inline void fix_finalize_range(unsigned long long* __restrict__ xfix, const double* __restrict__ unscale,
                                          int numnu, int nrhox, int kw, double* __restrict__ xl) {
  const int64_t n = (int64_t)numnu * nrhox;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t nu = e / nrhox;
    const int j = (int)(e - nu * nrhox);
    unsigned long long* w = xfix + (size_t)nu * kFixWords * kw + j;
    const unsigned long long x0 = w[0], x1 = w[kw], x2 = w[2 * kw];
    xl[(size_t)nu * kw + j] = (x0 | x1 | x2) ? fix_to_double(x0, x1, x2, unscale[j]) : 0.0;
    if (x0) w[0] = 0ull;
    if (x1) w[kw] = 0ull;
    if (x2) w[2 * kw] = 0ull;
  }
}

static __global__ void k_fix_finalize(unsigned long long* xfix, const double* unscale, int numnu, int nrhox, int kw,
                                      double* xl) {
  fix_finalize_range(xfix, unscale, numnu, nrhox, kw, xl);
}

// the largest CGF of each species' lines (CGF > 0: the bit patterns order as the values)
static __global__ void k_cgf_max(const AtlasLine* __restrict__ lines, int64_t n, int nspec,
                                 unsigned long long* __restrict__ cgfmax) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const AtlasLine L = lines[i];
    if (L.nelion >= 1 && L.nelion <= nspec && L.cgf > 0.0)
      atomicMax(cgfmax + L.nelion - 1, (unsigned long long)__double_as_longlong(L.cgf));
  }
}

// the per-depth scales of a model (threads over depths)
static __global__ void k_fix_scale(const double* xnfdop, int nspec, int kw, int nrhox, const double* cgfmax,
                                   double* scale, double* unscale) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nrhox) fix_scale_depth(xnfdop, nspec, kw, j, cgfmax, scale, unscale);
}

// ---------------------------------------------------------------- RT pass
constexpr int kAcc = 8;  // rjmins, rdabh, rdiagj, flxrad, raden, h_total, accrad, abross

struct RtArgs {
  const JoshOps* ops;
  int numnu, nrhox, kw;
  const double *waveset, *rcoset;
  const double *acont, *sigmac, *scont;  // [numnu][kw]; scont may be null (=> BNU)
  const double* xl;                      // XLINES: element (J, NU) at xl[(J-1)*xl_sj + (NU-1)*xl_snu]
  const double *rhox, *t, *hkt;
  double teff;
  int nu_per_warp;    // contiguous frequencies per group
  int xl_sj, xl_snu;  // XLINES strides (depth, frequency)
  double* partial;   // [groups][kAcc*kw + 1]
  double* hsurf;     // [numnu] HNU(1) per frequency (the .flux record)
  int* sweeps;       // [numnu] Eddington sweeps (diagnostic; may be null)
  // frequency shard NU_FIRST..NU_LAST (1-based; 0 => NUMNU): groups start at NU_FIRST
  int nu_first = 1, nu_last = 0;
  // split pass (k_rt_pre / k_rt_solve / k_rt_post): per-frequency records
  // handed from stage to stage, rec_stride doubles per frequency at
  // (NU - NU_FIRST) * rec_stride; frequencies per pre warp and per solve
  // group (nu_per_warp is the post warps', one partial row per post warp)
  double* rec = nullptr;
  int rec_stride = 0;
  int nu_per_pre = 1, nu_per_solve = 1;
  // work counters of the solve stage (timed launches only, else null):
  // [0] systems eliminated, [1] systems summed as a series, [2] series steps
  unsigned long long* work = nullptr;
};

struct RtWS {
  JoshWS w;
  JoshWSFull f;
  double acont[kKwMax], sigmac[kKwMax], aline[kKwMax], stim[kKwMax];
  double dab[kKwMax];           // SCONT while JOSH runs (when given), then d(abtot)/d(rhox)
  alignas(16) double U[kNx * (kNx + 1)];  // pivot rows of the 51x51 factorisation (rows 16-byte aligned)
};

// One pair group (64 threads) per frequency, kRtGroups groups per CTA.  The
// group's 51 matrix rows live in registers (pair elimination), so the
// shared-memory footprint is the depth vectors and the pivot rows.  (A
// 128-thread group holding the system block-cyclically, 28 entries per
// thread and one barrier per step, measured slower: 3.62 ms against 3.34 ms
// for the 30,000-frequency pass unrolled, 5.79 ms with the step loop
// rolled; four groups fit per SM against six.)
using RtG = PairG;
constexpr int kRtMinBlocks = 3;
constexpr int kRtGroups = 2;
constexpr int kRtThreads = kRtGroups * RtG::N;

// shared memory: RHOX and a zero vector (SIGMAL) for the CTA, then the groups' workspaces
__host__ __device__ inline size_t rt_smem_bytes() { return 2 * sizeof(double) * kKwMax + kRtGroups * sizeof(RtWS); }

// After JOSH: the negative floor (RUN_RT_PASS :3926-3937), HNU(1) for the
// .flux record, and the TCORR / RADIAP / ROSS mode-2 terms of this frequency
// added into the group's accumulators (threads over depths, C per thread).
// add(q, c, j, v) adds term q of depth j (the thread's c-th depth) to its sum.
template <class G, class WS, int C, class Add>
static __device__ __forceinline__ void rt_accumulate(G& g, const RtArgs& a, WS& S, const double* rhox_s, int nu,
                                                     double freq, double rcowt, Add&& add, double& pradk0) {
  const int nr = a.nrhox;
  // negative floor (RUN_RT_PASS :3926-3937)
  bool neg = false;
  for (int j = g.r; j < nr; j += G::N) neg |= (S.f.snu[j] < 0.0 || S.f.jnu[j] < 0.0 || S.f.hnu[j] < 0.0);
  if (g.any(neg)) {
    for (int j = g.r; j < nr; j += G::N) {
      S.f.jnu[j] = fmax(S.f.jnu[j], 1.0e-99);
      S.f.snu[j] = fmax(S.f.snu[j], 1.0e-99);
      S.f.hnu[j] = fmax(S.f.hnu[j], 1.0e-99);
    }
    g.sync();
  }
  if (g.r == 0) a.hsurf[nu - 1] = S.f.hnu[0];
  // TCORR mode 2: d(abtot)/d(rhox)
  g_deriv(g, rhox_s, S.w.abtot, S.dab, nr);
  // TERM2 per depth (E3 diagonal of Lambda); D(NRHOX) repeats D(NRHOX-1)
  for (int j = g.r; j < nr; j += G::N) {
    const int jd = j < nr - 1 ? j : nr - 2;
    double d = S.w.taunu[jd + 1] - S.w.taunu[jd];
    d = fmax(1.0e-10, d);
    double term2;
    if (d <= 0.01) {
      term2 = (kEulerM1 - log(d)) * d / 4.0 + (d * d) / 12.0 - (d * d * d) / 96.0 +
              ((d * d) * (d * d)) / 720.0;
    } else {
      double ex = 0.0;
      if (d < 10.0) ex = expi3(d);
      if (a.teff <= 4250.0 && d > 0.005 && d < 0.02) ex = 0.0;
      term2 = 0.5 * (d + ex - 0.5) / d;
    }
    S.w.t1[j] = term2;
  }
  g.sync();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = g.r + c * G::N;
    if (j >= nr) break;
    const double ab = S.w.abtot[j], al = S.w.alpha[j], h = S.f.hnu[j];
    const double rab = 1.0 / ab;
    add(1, c, j, S.dab[j] * rab * h * rcowt);                // RDABH
    add(0, c, j, ab * S.f.jmins[j] * rcowt);                 // RJMINS
    add(3, c, j, h * rcowt);                                 // FLXRAD
    const double diagj = (j > 0 ? S.w.t1[j - 1] : 0.0) + S.w.t1[j];
    const double hk = a.hkt[j], tt = a.t[j];
    // dB/dT = BNU * freq * HKT / T / STIM (floored at 1e-30 for RDIAGJ, as the reference)
    const double bft = S.f.bnu[j] * freq * hk / tt;
    const double dbdt = bft / fmax(S.stim[j], 1.0e-30);
    add(2, c, j, ab * (diagj - 1.0) / (1.0 - al * diagj) * (1.0 - al) * dbdt * rcowt);  // RDIAGJ
    add(4, c, j, S.f.jnu[j] * rcowt);                        // RADEN
    add(5, c, j, h * rcowt);                                 // H_TOTAL
    add(6, c, j, ab * h * rcowt);                            // ACCRAD
    const double dbdt2 = (S.stim[j] >= 1.0e-30) ? dbdt : bft / S.stim[j];
    add(7, c, j, dbdt2 * rab * rcowt);                       // ABROSS
  }
  pradk0 += S.f.knu1 * rcowt;
}

// A group's partial-sum row.  The whole row is written: depths nrhox..kw-1
// (padding when kw > nrhox) get zeros, so the fixed-order reduction never
// sums stale entries.
template <class G, int C>
static __device__ __forceinline__ void rt_write_partial(G& g, const RtArgs& a, int row, const double (&acc)[kAcc][C],
                                                        double pradk0) {
  double* out = a.partial + (size_t)row * (kAcc * a.kw + 1);
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = g.r + c * G::N;
    if (j < a.kw) {
#pragma unroll
      for (int q = 0; q < kAcc; ++q) out[q * a.kw + j] = j < a.nrhox ? acc[q][c] : 0.0;
    }
  }
  if (g.r == 0) out[kAcc * a.kw] = pradk0;
}

static __device__ __forceinline__ void rt_body(const RtArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / RtG::N;
  double* rhox_s = reinterpret_cast<double*>(smem_raw);
  double* zero_s = rhox_s + kKwMax;
  RtWS& S = reinterpret_cast<RtWS*>(smem_raw + 2 * sizeof(double) * kKwMax)[gid];
  for (int j = threadIdx.x; j < a.nrhox; j += blockDim.x) {
    rhox_s[j] = a.rhox[j];
    zero_s[j] = 0.0;
  }
  __syncthreads();
  RtG g(threadIdx.x % RtG::N, 1 + gid, S.w.red);
  constexpr int C = (kKwMax + RtG::N - 1) / RtG::N;
  const JoshOps& ops = *a.ops;
  const int nr = a.nrhox;
  const int gw = blockIdx.x * kRtGroups + gid;  // partial-sum row of this group
  const int nu0 = a.nu_first + gw * a.nu_per_warp;
  const int nu1 = min(nu0 + a.nu_per_warp - 1, a.nu_last > 0 ? a.nu_last : a.numnu);
  double acc[kAcc][C];
#pragma unroll
  for (int q = 0; q < kAcc; ++q)
#pragma unroll
    for (int c = 0; c < C; ++c) acc[q][c] = 0.0;
  double pradk0 = 0.0;
  for (int nu = nu0; nu <= nu1; ++nu) {
    const double wave = a.waveset[nu - 1];
    const double freq = kClightNms / wave;
    const double rcowt = a.rcoset[nu - 1];
    const double f3 = powi(freq / 1.0e15, 3);
    for (int j = g.r; j < nr; j += RtG::N) {
      const double ehvkt = exp(-freq * a.hkt[j]);
      const double stim = 1.0 - ehvkt;
      const double bnu = kBnuPrefac * f3 * ehvkt / stim;
      S.stim[j] = stim;
      S.f.bnu[j] = bnu;
      S.acont[j] = a.acont[(size_t)(nu - 1) * a.kw + j];
      S.sigmac[j] = a.sigmac[(size_t)(nu - 1) * a.kw + j];
      if (a.scont) S.dab[j] = a.scont[(size_t)(nu - 1) * a.kw + j];
      S.aline[j] = 0.0 + a.xl[(size_t)j * a.xl_sj + (size_t)(nu - 1) * a.xl_snu] * stim;
    }
    g.sync();
    const int sw = g_josh(g, ops, rhox_s, nr, S.acont, S.aline, S.sigmac, zero_s, a.scont ? S.dab : S.f.bnu,
                          S.f.bnu, S.f.bnu, S.w, S.U, &S.f, nullptr);
    if (a.sweeps && g.r == 0) a.sweeps[nu - 1] = sw;
    rt_accumulate<RtG, RtWS, C>(
        g, a, S, rhox_s, nu, freq, rcowt, [&](int q, int c, int, double v) { acc[q][c] += v; }, pradk0);
    g.sync();
  }
  rt_write_partial(g, a, gw, acc, pradk0);
}

static __global__ void __launch_bounds__(kRtThreads, kRtMinBlocks) k_atlas_rt(RtArgs a) { rt_body(a); }

// ---------------------------------------------------------------- split RT pass
// The same pass in three launches.  JOSH's 51x51 solve needs ~100 registers
// of matrix row per thread, which caps the fused kernel at six frequencies
// per SM; its vector work (INTEG, the MAP1s, the Eddington sweeps, the
// operator products, DERIV and the mode-2 sums) is a chain of short
// barrier-separated steps that wants many frequencies in flight instead.
//   k_rt_pre    warp per frequency: STIM, BNU, ABTOT, ALPHA, SNUBAR, TAUNU,
//               MAXJ, XSBAR and XALPHA on the 51-point grid
//   k_rt_solve  pair group per frequency that needs it: the scattering system
//   k_rt_post   warp per frequency: the rest of JOSH and the mode-2 sums,
//               one partial-sum row per warp (reduced in fixed order)
// Each frequency's record goes from stage to stage through device memory,
// rec_stride doubles: TAUNU [kw], then on the 51-point grid XALPHA, XSBAR
// and XS, then MAXJ and the solve flag.  Every value is computed by the same
// expressions as in the fused kernel.  (Forming J - S and H in the solve
// stage as well, where COEFJ and COEFH stay in L1, measured slower: 2.00
// against 1.85 ms per model-iteration.)
struct RtRec {
  int kw;
  __host__ __device__ int xalpha() const { return kw; }
  __host__ __device__ int xsbar() const { return kw + kNx; }
  __host__ __device__ int xs() const { return kw + 2 * kNx; }
  __host__ __device__ int maxj() const { return kw + 3 * kNx; }
  __host__ __device__ int solve() const { return kw + 3 * kNx + 1; }
};
__host__ __device__ inline int rt_rec_stride(int kw) { return (kw + 3 * kNx + 2 + 1) & ~1; }

// STIM, BNU and JOSH's ABTOT, ALPHA, SNUBAR (SIGMAL = 0, SLINE = BNU) of one
// depth at frequency NU, as the fused kernel forms them (RUN_RT_PASS
// :3905-3922, JOSH :18491-18500)
struct RtDepth {
  double stim, bnu, abtot, alpha, snubar;
};
__device__ __forceinline__ RtDepth rt_depth(const RtArgs& a, int nu, double freq, double f3, int j) {
  const double ehvkt = exp(-freq * a.hkt[j]);
  const double stim = 1.0 - ehvkt;
  const double bnu = kBnuPrefac * f3 * ehvkt / stim;
  const double ac = a.acont[(size_t)(nu - 1) * a.kw + j];
  const double sg = a.sigmac[(size_t)(nu - 1) * a.kw + j];
  const double sc = a.scont ? a.scont[(size_t)(nu - 1) * a.kw + j] : bnu;
  const double al = 0.0 + a.xl[(size_t)j * a.xl_sj + (size_t)(nu - 1) * a.xl_snu] * stim;
  const double sl = 0.0;
  RtDepth d;
  d.stim = stim;
  d.bnu = bnu;
  d.abtot = ac + al + sg + sl;
  d.alpha = (sg + sl) / d.abtot;
  d.snubar = (ac * sc + al * bnu) / (ac + al);
  return d;
}

constexpr int kRtSplitWarps = 4;      // warps per CTA of the pre and post stages
constexpr int kRtSolveGroups = 2;     // pair groups per CTA of the solve stage
constexpr int kRtSolveThreads = kRtSolveGroups * PairG::N;
constexpr int kRtSolveMinBlocks = 4;  // 8 systems per SM (128 registers per thread)

struct RtPreWS {
  double abtot[kKwMax], alpha[kKwMax], snubar[kKwMax], taunu[kKwMax];
  double t1[kKwMax], t2[kKwMax], t3[kKwMax];
  double xsbar[kNx], xalpha[kNx], xs[kNx];
  int lidx[kKwMax + 4];
};
struct RtSolveWS {
  double xs[kNx], xsbar[kNx], xalpha[kNx], piv[kNx];
  double rowabs[kNx];  // row sums of |COEFJ| (the contraction bound's factors)
  double red[8];
  unsigned pk[4][3];
  alignas(16) double U[kNx * (kNx + 1)];
};
// The post stage's workspace: one warp's vectors carved from shared memory
// at a stride of kv >= NRHOX doubles (rt_post_kv), its 51-point vectors, the
// mode-2 sums of the warp's depths (kAcc x kv) and two scalars.
struct RtPostFull {
  double *snu, *hnu, *jmins, *jnu, *bnu;
  double& knu1;
  int& maxj;
};
struct RtPostVec {
  double *abtot, *alpha, *snubar, *taunu, *t1, *t2, *t3, *xs, *xsbar, *xw;
  int* lidx;
};
struct RtPostView {
  RtPostVec w;
  RtPostFull f;
  double *stim, *dab, *acc;
};
__host__ __device__ inline int rt_post_kv(int nrhox) { return (nrhox + 1) & ~1; }
__host__ __device__ inline size_t rt_post_warp_doubles(int kv) {
  return (size_t)(12 + kAcc) * kv + 3 * kNx + 2 + (kv + 4 + 1) / 2 + 1;
}
__host__ __device__ inline size_t rt_pre_smem_bytes() { return sizeof(double) * kKwMax + kRtSplitWarps * sizeof(RtPreWS); }
__host__ __device__ inline size_t rt_solve_smem_bytes() { return kRtSolveGroups * sizeof(RtSolveWS); }
__host__ __device__ inline size_t rt_post_smem_bytes(int nrhox) {
  return sizeof(double) * (kKwMax + kRtSplitWarps * rt_post_warp_doubles(rt_post_kv(nrhox)));
}

__device__ __forceinline__ double* rt_rec(const RtArgs& a, int nu) {
  return a.rec + (size_t)(nu - a.nu_first) * a.rec_stride;
}

static __device__ __forceinline__ void rt_pre_body(const RtArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* rhox_s = reinterpret_cast<double*>(smem_raw);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RtPreWS& S = reinterpret_cast<RtPreWS*>(smem_raw + sizeof(double) * kKwMax)[wid];
  for (int j = threadIdx.x; j < a.nrhox; j += blockDim.x) rhox_s[j] = a.rhox[j];
  __syncthreads();
  WarpG g(lane);
  const JoshOps& ops = *a.ops;
  const int nr = a.nrhox, kw = a.kw;
  const int w = blockIdx.x * kRtSplitWarps + wid;
  const int nu0 = a.nu_first + w * a.nu_per_pre;
  const int nu1 = min(nu0 + a.nu_per_pre - 1, a.nu_last > 0 ? a.nu_last : a.numnu);
  for (int nu = nu0; nu <= nu1; ++nu) {
    const double freq = kClightNms / a.waveset[nu - 1];
    const double f3 = powi(freq / 1.0e15, 3);
    for (int j = lane; j < nr; j += 32) {
      const RtDepth d = rt_depth(a, nu, freq, f3, j);
      S.abtot[j] = d.abtot;
      S.alpha[j] = d.alpha;
      S.snubar[j] = d.snubar;
    }
    g.sync();
    bool mapped, solve;
    // (with IFSURF = 0 a mapped surface with MAXJ = 1 ends as an unmapped
    // one: the sweeps overwrite SNU at every depth, so XS is not needed)
    const int maxj = g_josh_prepare(g, ops, rhox_s, nr, S, mapped, solve);
    (void)mapped;
    double* rec = rt_rec(a, nu);
    const RtRec R{kw};
    for (int j = lane; j < nr; j += 32) rec[j] = S.taunu[j];
    if (maxj != 1) {
      for (int l = lane; l < kNx; l += 32) {
        rec[R.xalpha() + l] = S.xalpha[l];
        rec[R.xsbar() + l] = S.xsbar[l];
        if (!solve) rec[R.xs() + l] = S.xs[l];
      }
    }
    if (lane == 0) {
      rec[R.maxj()] = (double)maxj;
      rec[R.solve()] = (solve && maxj != 1) ? 1.0 : 0.0;
    }
    g.sync();
  }
}

// The scattering system X = (1 - XALPHA) XSBAR + XALPHA (COEFJ X) is a
// contraction with factor q = max_l XALPHA(l) sum_m |COEFJ(l,m)| (the
// infinity norm of diag(XALPHA) COEFJ).  Where q <= kRtSeriesQ the solve
// stage sums its Neumann series instead of eliminating: K steps of
// X <- (1 - XALPHA) XSBAR + XALPHA (COEFJ X) from X = (1 - XALPHA) XSBAR
// leave an error of at most q^(K+1) |X|, and K is taken so that
// q^(K+1) <= 2^-60, far below the rounding of the elimination itself (the
// two solutions agree to rounding).  A step is one matrix-vector product
// with no sequential dependence between rows and one barrier, against the
// elimination's 50 dependent pivot steps, so the series is cheaper up to
// q ~ 0.5.  Systems with larger q (strongly scattering layers) are
// eliminated as SOLVIT does.
constexpr double kRtSeriesQ = 0.5;
constexpr int kRtSeriesMaxSteps = 64;

__device__ __forceinline__ int rt_series_steps(double q) {
  if (!(q > 0.0)) return 1;
  const int k = (int)ceil(-60.0 * 0.6931471805599453 / log(q)) - 1;
  return k < 1 ? 1 : (k > kRtSeriesMaxSteps ? kRtSeriesMaxSteps : k);
}

static __device__ __forceinline__ void rt_solve_body(const RtArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / PairG::N;
  RtSolveWS& S = reinterpret_cast<RtSolveWS*>(smem_raw)[gid];
  PairG g(threadIdx.x % PairG::N, 1 + gid, S.red);
  const JoshOps& ops = *a.ops;
  const int kw = a.kw;
  const int grp = blockIdx.x * kRtSolveGroups + gid;
  const int nu0 = a.nu_first + grp * a.nu_per_solve;
  const int nu1 = min(nu0 + a.nu_per_solve - 1, a.nu_last > 0 ? a.nu_last : a.numnu);
  for (int l = g.r; l < kNx; l += PairG::N) {
    double r = 0.0;
    for (int m = 0; m < kNx; ++m) r += fabs(ops.coefj[m * kNx + l]);
    S.rowabs[l] = r;
  }
  g.sync();
  unsigned long long nelim = 0, nseries = 0, nsteps = 0;
  const RtRec R{kw};
  for (int nu = nu0; nu <= nu1; ++nu) {
    double* rec = rt_rec(a, nu);
    if (rec[R.solve()] == 0.0) continue;  // the same word for the whole group
    {
      double qv = 0.0;
      for (int l = g.r; l < kNx; l += PairG::N) {
        const double xa = rec[R.xalpha() + l];
        S.xalpha[l] = xa;
        S.xsbar[l] = rec[R.xsbar() + l];
        qv = fmax(qv, xa * S.rowabs[l]);
      }
      const double q = g.max(qv);  // (its barrier also publishes XALPHA, XSBAR)
      if (q <= kRtSeriesQ) continue;  // summed by k_rt_series
      solve_scatter(g, ops, S, S.U);
      ++nelim;
    }
    for (int l = g.r; l < kNx; l += PairG::N) rec[R.xs() + l] = S.xs[l];
    g.sync();
  }
  if (a.work && g.r == 0 && (nelim | nseries)) {
    atomicAdd(a.work, nelim);
    atomicAdd(a.work + 1, nseries);
    atomicAdd(a.work + 2, nsteps);
  }
}

// The Neumann series of the systems with q <= kRtSeriesQ, by their own
// kernel (k_rt_series; k_rt_solve eliminates the rest): thread l of a pair
// group keeps row l of COEFJ in registers for the whole launch (it is the
// same for every frequency), so a step is 51 FMAs on registers and the
// broadcast reads of X from shared memory, with no loads of COEFJ.  Sum k of
// the four partial sums takes the terms m = k, k+4, ... in that order; q is
// formed as in rt_solve_body, so the two kernels split the systems the same
// way.  (The series inside k_rt_solve, reading COEFJ from L1 every step,
// took 2.6k cycles per step at eight groups per SM.)
constexpr int kRtSeriesMinBlocks = 3;
struct RtSeriesWS {
  alignas(16) double xa[kNx + 1];
  alignas(16) double xb[kNx + 1];
  double red[8];
};

static __device__ __forceinline__ void rt_series_body(const RtArgs& a) {
  __shared__ RtSeriesWS s_ws[kRtSolveGroups];
  const int gid = threadIdx.x / PairG::N;
  RtSeriesWS& S = s_ws[gid];
  PairG g(threadIdx.x % PairG::N, 1 + gid, S.red);
  const JoshOps& ops = *a.ops;
  const int kw = a.kw, l = g.r;
  const bool own = l < kNx;
  double c[kNx];
  double rowabs = 0.0;
#pragma unroll
  for (int m = 0; m < kNx; ++m) c[m] = own ? ops.coefj[m * kNx + l] : 0.0;
  for (int m = 0; m < kNx; ++m) rowabs += fabs(own ? ops.coefj[m * kNx + l] : 0.0);
  const int grp = blockIdx.x * kRtSolveGroups + gid;
  const int nu0 = a.nu_first + grp * a.nu_per_solve;
  const int nu1 = min(nu0 + a.nu_per_solve - 1, a.nu_last > 0 ? a.nu_last : a.numnu);
  unsigned long long nseries = 0, nsteps = 0;
  const RtRec R{kw};
  for (int nu = nu0; nu <= nu1; ++nu) {
    double* rec = rt_rec(a, nu);
    if (rec[R.solve()] == 0.0) continue;  // the same word for the whole group
    const double al = own ? rec[R.xalpha() + l] : 0.0;
    const double xb = own ? rec[R.xsbar() + l] : 0.0;
    double qv = 0.0;
    if (own) qv = fmax(qv, al * rowabs);
    const double q = g.max(qv);
    if (q > kRtSeriesQ) continue;  // eliminated by k_rt_solve
    const int K = rt_series_steps(q);
    const double b = own ? (1.0 - al) * xb : 0.0;
    double* cur = S.xa;
    double* nxt = S.xb;
    if (own) cur[l] = b;
    for (int k = 0; k < K; ++k) {
      g.sync();
      if (own) {
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < kNx; ++m) s4[m & 3] = s4[m & 3] + c[m] * cur[m];
        nxt[l] = b + al * ((s4[0] + s4[1]) + (s4[2] + s4[3]));
      }
      double* t = cur;
      cur = nxt;
      nxt = t;
    }
    g.sync();
    if (own) rec[R.xs() + l] = cur[l];
    ++nseries;
    nsteps += K;
  }
  if (a.work && g.r == 0 && nseries) {
    atomicAdd(a.work + 1, nseries);
    atomicAdd(a.work + 2, nsteps);
  }
}

static __device__ __forceinline__ void rt_post_body(const RtArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* rhox_s = reinterpret_cast<double*>(smem_raw);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nr = a.nrhox, kw = a.kw, kv = rt_post_kv(nr);
  double* p = rhox_s + kKwMax + (size_t)wid * rt_post_warp_doubles(kv);
  auto take = [&](size_t n) {
    double* q = p;
    p += n;
    return q;
  };
  double *abtot = take(kv), *alpha = take(kv), *snubar = take(kv), *taunu = take(kv), *t1 = take(kv);
  double *snu = take(kv), *hnu = take(kv), *jmins = take(kv), *jnu = take(kv), *bnu = take(kv);
  double *stim = take(kv), *dab = take(kv), *acc = take((size_t)kAcc * kv);
  double *xs = take(kNx), *xsbar = take(kNx), *xw = take(kNx);
  double* knu1 = take(1);
  int* maxj_s = reinterpret_cast<int*>(take(1));
  int* lidx = reinterpret_cast<int*>(take((kv + 4 + 1) / 2));
  // t2 and t3 serve JOSH only with IFSURF = 1, which this stage never runs
  RtPostView S{RtPostVec{abtot, alpha, snubar, taunu, t1, t1, t1, xs, xsbar, xw, lidx},
               RtPostFull{snu, hnu, jmins, jnu, bnu, *knu1, *maxj_s}, stim, dab, acc};
  for (int j = threadIdx.x; j < nr; j += blockDim.x) rhox_s[j] = a.rhox[j];
  for (int e = lane; e < kAcc * kv; e += 32) acc[e] = 0.0;
  __syncthreads();
  WarpG g(lane);
  constexpr int C = (kKwMax + 31) / 32;
  const JoshOps& ops = *a.ops;
  const int w = blockIdx.x * kRtSplitWarps + wid;  // partial-sum row of this warp
  const int nu0 = a.nu_first + w * a.nu_per_warp;
  const int nu1 = min(nu0 + a.nu_per_warp - 1, a.nu_last > 0 ? a.nu_last : a.numnu);
  double pradk0 = 0.0;
  for (int nu = nu0; nu <= nu1; ++nu) {
    const double freq = kClightNms / a.waveset[nu - 1];
    const double rcowt = a.rcoset[nu - 1];
    const double f3 = powi(freq / 1.0e15, 3);
    const double* rec = rt_rec(a, nu);
    const RtRec R{kw};
    const int maxj = (int)rec[R.maxj()];
    for (int j = lane; j < nr; j += 32) {
      const RtDepth d = rt_depth(a, nu, freq, f3, j);
      abtot[j] = d.abtot;
      alpha[j] = d.alpha;
      snubar[j] = d.snubar;
      stim[j] = d.stim;
      bnu[j] = d.bnu;
      taunu[j] = rec[j];
    }
    if (maxj != 1)
      for (int l = lane; l < kNx; l += 32) xs[l] = rec[R.xs() + l];
    g.sync();
    const int sw = g_josh_finish(g, ops, nr, maxj, maxj != 1, S.w, &S.f, bnu, (double*)nullptr);
    if (a.sweeps && lane == 0) a.sweeps[nu - 1] = sw;
    rt_accumulate<WarpG, RtPostView, C>(
        g, a, S, rhox_s, nu, freq, rcowt, [&](int q, int, int j, double v) { acc[q * kv + j] += v; }, pradk0);
    g.sync();
  }
  double* out = a.partial + (size_t)w * (kAcc * kw + 1);
  for (int j = lane; j < kw; j += 32) {
#pragma unroll
    for (int q = 0; q < kAcc; ++q) out[q * kw + j] = j < nr ? acc[q * kv + j] : 0.0;
  }
  if (lane == 0) out[kAcc * kw] = pradk0;
}

static __global__ void __launch_bounds__(kRtSplitWarps * 32, 6) k_rt_pre(RtArgs a) { rt_pre_body(a); }
static __global__ void __launch_bounds__(kRtSolveThreads, kRtSolveMinBlocks) k_rt_solve(RtArgs a) { rt_solve_body(a); }
static __global__ void __launch_bounds__(kRtSolveThreads, kRtSeriesMinBlocks) k_rt_series(RtArgs a) { rt_series_body(a); }
static __global__ void __launch_bounds__(kRtSplitWarps * 32, 4) k_rt_post(RtArgs a) { rt_post_body(a); }

// Launch shape of the split pass over LEN frequencies with 1/NB of the GPU
// (NB slots of a batch share it): every stage gets about WAVES resident waves
// of its units (warps or pair groups), frequencies contiguous per unit.
struct RtSplitShape {
  int pre_per = 1, pre_blocks = 1, solve_per = 1, solve_blocks = 1, post_per = 1, post_blocks = 1;
  int rows() const { return post_blocks * kRtSplitWarps; }
};
inline void rt_split_fit(int len, int units, int per_block, int& per, int& blocks) {
  per = (len + units - 1) / units;
  if (per < 1) per = 1;
  const int n = (len + per - 1) / per;
  blocks = (n + per_block - 1) / per_block;
}
inline RtSplitShape rt_split_shape(int len, int nsm, int nb, int waves) {
  RtSplitShape sh;
  auto units = [&](int per_sm) {
    const long long u = (long long)nsm * per_sm * waves / (nb > 0 ? nb : 1);
    return (int)(u < 1 ? 1 : u);
  };
  rt_split_fit(len, units(16), kRtSplitWarps, sh.pre_per, sh.pre_blocks);
  rt_split_fit(len, units(8), kRtSolveGroups, sh.solve_per, sh.solve_blocks);
  rt_split_fit(len, units(16), kRtSplitWarps, sh.post_per, sh.post_blocks);
  return sh;
}
// the most partial-sum rows any frequency range of a model can need
// (rt_split_shape never makes more post warps than frequencies or units)
inline int rt_split_rows_max(int numnu, int nsm, int waves) {
  const long long units = (long long)nsm * 16 * waves;
  const long long n = numnu < units ? numnu : units;
  return (int)((n + kRtSplitWarps - 1) / kRtSplitWarps * kRtSplitWarps);
}
// shared-memory opt-in of the three stages (nrhox <= kKwMax)
inline cudaError_t rt_split_attributes(int nrhox) {
  cudaError_t e = cudaFuncSetAttribute(k_rt_pre, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rt_pre_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rt_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rt_solve_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rt_post, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rt_post_smem_bytes(nrhox));
  return e;
}
inline void rt_split_args(RtArgs& a, const RtSplitShape& sh) {
  a.nu_per_pre = sh.pre_per;
  a.nu_per_solve = sh.solve_per;
  a.nu_per_warp = sh.post_per;
  a.rec_stride = rt_rec_stride(a.kw);
}

// fixed-order sum of the per-warp partials: out[kAcc*kw + 1].  A block owns
// 32 consecutive sums (threadIdx.x) and splits the rows over 32 row groups
// (threadIdx.y: rows y, y+32, ...); the 32 group sums are then added in group
// order.  The order is fixed by the launch shape, so the result does not
// depend on scheduling.
constexpr int kRedCols = 32, kRedRows = 32;
static __device__ __forceinline__ void reduce_body(const double* __restrict__ partial, int nwarps, int kw,
                                                   double* __restrict__ out) {
  __shared__ double s[kRedRows][kRedCols + 1];
  const int stride = kAcc * kw + 1;
  const int e = blockIdx.x * kRedCols + threadIdx.x;
  double v = 0.0;
  if (e < stride) {
    int w = threadIdx.y;
    // four independent loads in flight per step, added in row order
    for (; w + 3 * kRedRows < nwarps; w += 4 * kRedRows) {
      const double a0 = partial[(size_t)w * stride + e];
      const double a1 = partial[(size_t)(w + kRedRows) * stride + e];
      const double a2 = partial[(size_t)(w + 2 * kRedRows) * stride + e];
      const double a3 = partial[(size_t)(w + 3 * kRedRows) * stride + e];
      v = (((v + a0) + a1) + a2) + a3;
    }
    for (; w < nwarps; w += kRedRows) v += partial[(size_t)w * stride + e];
  }
  s[threadIdx.y][threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.y == 0 && e < stride) {
    double t = 0.0;
    for (int y = 0; y < kRedRows; ++y) t += s[y][threadIdx.x];
    out[e] = t;
  }
}

static __global__ void __launch_bounds__(kRedCols* kRedRows)
    k_atlas_reduce(const double* __restrict__ partial, int nwarps, int kw, double* __restrict__ out) {
  reduce_body(partial, nwarps, kw, out);
}

inline void launch_reduce(const double* partial, int nwarps, int kw, double* out, cudaStream_t st) {
  const int stride = kAcc * kw + 1;
  k_atlas_reduce<<<(stride + kRedCols - 1) / kRedCols, dim3(kRedCols, kRedRows), 0, st>>>(partial, nwarps, kw, out);
}

}  // namespace atlasgpu
