// select.cuh -- SELECTLINES (atlas12_modules.f90:19171-19781) on the device:
// the filter that turns the line databases into the LINEDATA records LINOP1
// walks.  HBM-bound streaming passes over tiles of 2048 records, with no
// CTA waiting on another:
//
//  * the NU advance (DO WHILE (IWL >= IWAVETAB(NU)) ...) is a running
//    maximum: after a record, NU = max(NU at entry, UB(max IWL so far)) with
//    UB(x) = the first bin whose IWAVETAB exceeds x.  k_sel_tile_ub takes
//    each tile's maximum UB and k_sel_scan the exclusive maximum over tiles,
//    so a tile knows NU at its entry;
//  * k_selectlines filters each tile at its records' NU and writes the
//    selected LINEDATA compacted at the tile's own place in a scratch array,
//    with the tile's count; k_sel_scan sums the counts and k_sel_move puts
//    every tile's records at its offset, in file order.
//
// The tests follow the reference's arithmetic in FP64 with explicit
// round-to-nearest operations.  Three quantities pass through a
// transcendental the C library evaluates on the host (exp in the Boltzmann
// test, log / log10 in the TiO and H2O fields).  Where the device result is
// within a guard band of a decision boundary the record is listed for the
// host, which decides with the C library: the TiO IWL before the passes (an
// override table), the Boltzmann test and the IELO / IGR fields after them
// (a fix list with output positions).
#pragma once
#include <type_traits>

#include "common.cuh"

namespace atlasgpu {

constexpr int kSelThreads = 256;
constexpr int kSelItems = 8;
constexpr int kSelTile = kSelThreads * kSelItems;  // records per tile
constexpr int kSelGroup = 2;                       // records whose table loads are issued together
constexpr int kSelMaxWave = 1024;                  // IWAVETAB entries held in shared memory
constexpr double kSelKeepBand = 1.0e-12;  // |CENRATIO*exp(...) - 1| left to the host
constexpr double kSelIntBand = 1.0e-6;    // distance of an INT() argument from an integer left to the host

enum SelKind { kSelLowPred = 1, kSelLowObs = 2, kSelHi = 3, kSelDiatomic = 4, kSelTio = 5, kSelH2o = 6, kSelH3plus = 7 };
enum SelFixWhat { kFixKeep = 0, kFixIelo = 1, kFixIgr = 2 };
enum SelErr { kSelErrNelion = 1, kSelErrMolcode = 2, kSelErrSentinel = 3, kSelErrOverride = 4 };

// a record the host finishes: kFixKeep decides a*exp(b) >= 1 (drop the output
// record otherwise); kFixIelo / kFixIgr recompute the INTEGER(2) field from
// a (and arg) with the C library
struct SelFix {
  long long pos;
  int what, arg;
  double a, b;
};

// one MOL2 record (mod_mklinelist read_molec_bin layout, 32 bytes)
struct alignas(16) SelMol2 {
  float wl, gflog, e1, e2;
  int code, iso, gr, label;
};
// one H2O record: READ(51) IWL, IELO, IGFLOG with INTEGER(2) IELO, IGFLOG (8 bytes)
struct alignas(8) SelH2o {
  int iwl;
  short ielo, igflog;
};

struct SelArgs {
  const void* recs;
  long long n;
  int nu0, igr0;  // NU (1-based) and IGR at entry
  double freq0;   // FREQ at entry
  const int* iwt; // IWAVETAB [nwave+1], sentinel last
  int nwave;
  const double* freqtab;  // [nwave]: CLIGHT_NMS / WAVETAB(k) at k-1 (FREQ after advancing past bin k)
  const short* igrtab;    // [nwave]: H2O's IGR after advancing past bin k
  const double* xmax;     // XNFDOPMAX [nwave+1][nspec]
  int nspec;
  const double* tablog;   // TABLOG for every INTEGER(2), index I + 32768
  double hckt_last, cen_prefac, ratiolg;
  const int* molcor;      // ISOX by MOLCODE - 8410 [551], kSelMolUnknown for codes not in MOLCODES
  const int* tio_isocorr;  // TIO_ISOCORR [5]; H2O_ISOCORR [4]
  const int* h2o_isocorr;
  const long long* ovr_idx;  // TiO records whose IWL the host decided, sorted
  const int* ovr_iwl;
  int novr;
  const long long* tile_nu;  // [ntiles] NU at entry to each tile (exclusive maximum of UB, NU at entry first)
  int* tile_count;      // [ntiles] selected records per tile
  int4* scratch;        // [ntiles * kSelTile] each tile's LINEDATA, compacted at the tile's start
  SelFix* fix;
  unsigned int* nfix;
  unsigned int fixcap;
  unsigned long long* err;  // min over (record << 8 | code)
};

__device__ __forceinline__ int sel_fint(double x) {
  // INT() of a REAL(8) as x86-64 converts it: truncation, -2**31 for NaN or out of range
  return (x > -2147483649.0 && x < 2147483648.0) ? (int)x : (int)0x80000000;
}
__device__ __forceinline__ short sel_i16(int v) { return (short)(unsigned short)(unsigned)v; }
__device__ __forceinline__ bool sel_near_int(double x) { return fabs(x - rint(x)) <= kSelIntBand; }

// TiO's IWL = INT(LOG(WLVAC)/RATIOLG + 0.5) and whether the record takes
// part in the NU advance (molecule 822, Ti isotope 46-50, WLVAC > 0)
__device__ __forceinline__ bool sel_tio_iwl(const SelMol2& r, double ratiolg, int* iwl, bool* border) {
  *border = false;
  if (r.code != 822) return false;
  const int iso = r.iso - 45;
  if (iso < 1 || iso > 5) return false;
  const double w = (double)r.wl;
  if (w <= 0.0) return false;
  const double x = __dadd_rn(__ddiv_rn(log(w), ratiolg), 0.5);
  *iwl = sel_fint(x);
  *border = sel_near_int(x);
  return true;
}

// the TiO records whose IWL the host decides (before the selection pass)
__global__ void __launch_bounds__(256) k_sel_tio_border(const SelMol2* __restrict__ recs, long long n, double ratiolg,
                                                        long long* list, unsigned int* count, unsigned int cap) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int iwl;
    bool border;
    if (sel_tio_iwl(recs[i], ratiolg, &iwl, &border) && border) {
      const unsigned k = atomicAdd(count, 1u);
      if (k < cap) list[k] = i;
    }
  }
}

// XNFDOPMAX(NELION, NU) = max_J XNFDOP(J, NELION) / TABCONT(J, NU) (:19248-19256)
__global__ void __launch_bounds__(256) k_sel_xnfdopmax(int nrhox, int kw, const double* __restrict__ xnfdop, int nspec,
                                                       const double* __restrict__ tabcont, int nwave, double* xmax) {
  const long long total = (long long)(nwave + 1) * nspec;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int nu = (int)(k / nspec), e = (int)(k % nspec);
    double m = 0.0;
    for (int j = 0; j < nrhox; ++j) {
      const double r = __ddiv_rn(xnfdop[(size_t)e * kw + j], tabcont[(size_t)nu * kw + j]);
      if (r > m) m = r;
    }
    xmax[k] = m;
  }
}

template <int KIND>
struct SelRecType {
  using T = int4;  // LINEREC [4] int32
};
template <>
struct SelRecType<kSelTio> {
  using T = SelMol2;
};
template <>
struct SelRecType<kSelH2o> {
  using T = SelH2o;
};

// padded slot of the k-th record of a tile: each thread's kSelItems
// consecutive records are followed by one spare, so the blocked reads of a
// warp fall in different banks
__device__ __forceinline__ int sel_slot(int k) { return k + k / kSelItems; }

// UB(x): the first 1-based bin k with IWAVETAB(k) > x, over the shared copy
__device__ __forceinline__ int sel_ub(const int* s_iwt, int nwave, int x, int hint) {
  if (hint >= 1 && hint <= nwave + 1 && s_iwt[hint - 1] > x && (hint == 1 || s_iwt[hint - 2] <= x)) return hint;
  int lo = 0, hi = nwave + 1;  // answer index in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s_iwt[mid] > x)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo + 1;  // nwave + 2 when x is at or past the sentinel
}

__device__ __forceinline__ int4 sel_pack(int iwl, short ielion, short ielo, short igflog, short igr, short igs,
                                         short igw) {
  auto w = [](short lo, short hi) { return (int)((unsigned)(unsigned short)lo | ((unsigned)(unsigned short)hi << 16)); };
  return make_int4(iwl, w(ielion, ielo), w(igflog, igr), w(igs, igw));
}

__device__ __forceinline__ void sel_error(unsigned long long* err, long long rec, int code) {
  atomicMin(err, ((unsigned long long)rec << 8) | (unsigned)code);
}

// Per-record pass 1: the IWL taking part in the NU advance (or none).
template <int KIND>
__device__ __forceinline__ bool sel_advance_iwl(const typename SelRecType<KIND>::T& r, const SelArgs& a, long long gi,
                                                int* iwl) {
  if constexpr (KIND == kSelTio) {
    bool border;
    if (!sel_tio_iwl(r, a.ratiolg, iwl, &border)) return false;
    if (border) {
      int lo = 0, hi = a.novr;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.ovr_idx[mid] < gi)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo < a.novr && a.ovr_idx[lo] == gi)
        *iwl = a.ovr_iwl[lo];
      else
        sel_error(a.err, gi, kSelErrOverride);
    }
    return true;
  } else if constexpr (KIND == kSelH2o) {
    *iwl = r.iwl;
    return true;
  } else {
    *iwl = r.x;
    return true;
  }
}

// Codes of the diatomic species, MOLCODES(1) .. MOLCODES(NMOL), as offsets
// into a direct lookup table of their ISOX corrections
constexpr int kSelMolLo = 8410, kSelMolN = 551;
constexpr int kSelMolUnknown = -2147483647 - 1;

// The operands of a record's tests, gathered before any test runs so that a
// thread's table loads (XNFDOPMAX, TABLOG, FREQ) are in flight together.
struct SelOps {
  double freq, xm, tgf, tel;
  int nelion;  // the XNFDOPMAX row; out of 1..nspec when the record has none
  int bad;     // kSelErrMolcode for an unknown diatomic MOLCODE
  short igflog;  // IGFLOG after the database's correction
};

template <int KIND>
__device__ __forceinline__ void sel_gather(const typename SelRecType<KIND>::T& r, const SelArgs& a, int nu,
                                           const int* s_molcor, SelOps& o) {
  o.freq = nu > a.nu0 ? a.freqtab[nu - 2] : a.freq0;
  o.tel = 0.0;
  o.bad = 0;
  if constexpr (KIND == kSelTio) {
    const int iso = min(max(r.iso - 45, 1), 5);  // records outside 46-50 are dropped before any test
    const int kgflog = sel_fint(round(__dmul_rn((double)r.gflog, 1000.0))) + 16384;
    const int g = kgflog + a.tio_isocorr[iso - 1];
    o.igflog = sel_i16(g > 1 ? g : 1);
    o.nelion = 895;
  } else if constexpr (KIND == kSelH2o) {
    const int iso = (r.ielo > 0 && r.igflog > 0) ? 1 : r.ielo > 0 ? 2 : r.igflog > 0 ? 3 : 4;
    const int g = abs((int)r.igflog) + a.h2o_isocorr[iso - 1];
    o.igflog = sel_i16(g > 1 ? g : 1);
    o.nelion = 940;
  } else {
    const short ielion = (short)(r.y & 0xffff), ielo = (short)((unsigned)r.y >> 16);
    short igflog = (short)(r.z & 0xffff);
    if constexpr (KIND == kSelDiatomic) {
      const int c = (int)ielion - kSelMolLo;
      const int cor = (c >= 0 && c < kSelMolN) ? s_molcor[c] : kSelMolUnknown;
      if (cor == kSelMolUnknown) {
        o.bad = kSelErrMolcode;
      } else {
        const int g = (int)igflog + cor;
        igflog = sel_i16(g > 1 ? g : 1);
      }
    } else if constexpr (KIND == kSelH3plus) {
      const int g = (int)igflog - 1272;
      igflog = sel_i16(g > 1 ? g : 1);
    }
    o.igflog = igflog;
    o.nelion = KIND == kSelH3plus ? 895 : abs((int)ielion / 10);
    o.tel = a.tablog[ielo + 32768];
  }
  const bool row = nu >= 1 && o.nelion >= 1 && o.nelion <= a.nspec;
  o.xm = row ? a.xmax[(size_t)(nu - 1) * a.nspec + (o.nelion - 1)] : 0.0;
  o.tgf = a.tablog[o.igflog + 32768];
}

// Per-record pass 2: the filter at bin nu with the gathered operands.
// Returns 0 (rejected), 1 (selected) or 2 (selected, the Boltzmann test left
// to the host); *fixes gets kFixIelo / kFixIgr bits for fields the host
// recomputes.
template <int KIND>
__device__ __forceinline__ int sel_decide(const typename SelRecType<KIND>::T& r, const SelArgs& a, long long gi, int nu,
                                          const SelOps& o, int4* outrec, unsigned* fixes, double* kb_cen,
                                          double* kb_y) {
  *fixes = 0;
  short ielion, ielo = 0, igr = 0, igs = 1, igw = 9384;
  double e;  // the lower-level energy in the Boltzmann test
  int iwl;
  if constexpr (KIND == kSelTio) {
    // skipped before the NU advance (a NaN wavelength is not: WLVAC .LE. 0 is false)
    if (r.code != 822 || r.iso - 45 < 1 || r.iso - 45 > 5 || (double)r.wl <= 0.0) return 0;
    const int iso = r.iso - 45;
    const double w = (double)r.wl;
    sel_advance_iwl<KIND>(r, a, gi, &iwl);
    if (o.nelion > a.nspec) {
      sel_error(a.err, gi, kSelErrNelion);
      return 0;
    }
    if (o.xm == 0.0) return 0;
    const double cen = __ddiv_rn(__dmul_rn(__dmul_rn(a.cen_prefac, o.tgf), o.xm), o.freq);
    if (cen < 1.0) return 0;
    const double a1 = fabs((double)r.e1), a2 = fabs((double)r.e2);
    e = a2 < a1 ? a2 : a1;
    const double y = __dmul_rn(-e, a.hckt_last);
    const double p = __dmul_rn(cen, exp(y));
    const bool band = fabs(p - 1.0) <= kSelKeepBand;
    if (!band && p < 1.0) return 0;
    ielion = (short)(8949 + iso);
    const double el = e > 1.0e-10 ? e : 1.0e-10;
    const double xe = __dadd_rn(__dmul_rn(log10(el), 1000.0), 16384.5);
    ielo = sel_i16(sel_fint(xe));
    if (sel_near_int(xe)) *fixes |= 1u << kFixIelo;
    const double gam = r.gr == 0 ? __ddiv_rn(2.223e13, __dmul_rn(w, w)) : pow(10.0, __dmul_rn((double)r.gr, 0.01));
    const double xg = __dadd_rn(__dmul_rn(log10(gam), 1000.0), 16384.5);
    igr = sel_i16(sel_fint(xg));
    if (sel_near_int(xg)) *fixes |= 1u << kFixIgr;
    *outrec = sel_pack(iwl, ielion, ielo, o.igflog, igr, igs, igw);
    if (band) {
      *kb_cen = cen;
      *kb_y = y;
      return 2;
    }
    return 1;
  } else if constexpr (KIND == kSelH2o) {
    iwl = r.iwl;
    const int iso = (r.ielo > 0 && r.igflog > 0) ? 1 : r.ielo > 0 ? 2 : r.igflog > 0 ? 3 : 4;
    ielion = (short)(-(9399 + iso));
    e = (double)abs((int)r.ielo);
    igr = nu > a.nu0 ? a.igrtab[nu - 2] : (short)a.igr0;
    if (o.nelion > a.nspec) {
      sel_error(a.err, gi, kSelErrNelion);
      return 0;
    }
    if (o.xm == 0.0) return 0;
    const double cen = __ddiv_rn(__dmul_rn(__dmul_rn(a.cen_prefac, o.tgf), o.xm), o.freq);
    if (cen < 1.0) return 0;
    const double y = __dmul_rn(-e, a.hckt_last);
    const double p = __dmul_rn(cen, exp(y));
    const bool band = fabs(p - 1.0) <= kSelKeepBand;
    if (!band && p < 1.0) return 0;
    const double xe = __dadd_rn(__dmul_rn(log10(e), 1000.0), 16384.5);
    ielo = sel_i16(sel_fint(xe));
    if (sel_near_int(xe)) *fixes |= 1u << kFixIelo;
    *outrec = sel_pack(iwl, ielion, ielo, o.igflog, igr, igs, igw);
    if (band) {
      *kb_cen = cen;
      *kb_y = y;
      return 2;
    }
    return 1;
  } else {
    iwl = r.x;
    ielion = (short)(r.y & 0xffff);
    ielo = (short)((unsigned)r.y >> 16);
    igr = (short)((unsigned)r.z >> 16);
    igs = (short)(r.w & 0xffff);
    igw = (short)((unsigned)r.w >> 16);
    if (KIND == kSelH3plus) {
      igs = 1;
      igw = 9384;
    }
    if (o.bad) {
      sel_error(a.err, gi, o.bad);
      return 0;
    }
    if (o.nelion < 1 || o.nelion > a.nspec) {
      if (KIND != kSelLowPred) sel_error(a.err, gi, kSelErrNelion);
      return 0;
    }
    if (KIND == kSelLowPred || KIND == kSelLowObs) {
      if (o.xm <= 1.0e-37) return 0;
    } else if (o.xm == 0.0) {
      return 0;
    }
    const double cen = __ddiv_rn(__dmul_rn(__dmul_rn(a.cen_prefac, o.tgf), o.xm), o.freq);
    if (cen < 1.0) return 0;
    const double y = __dmul_rn(-o.tel, a.hckt_last);
    const double p = __dmul_rn(cen, exp(y));
    *outrec = sel_pack(iwl, ielion, ielo, o.igflog, igr, igs, igw);
    if (fabs(p - 1.0) <= kSelKeepBand) {
      *kb_cen = cen;
      *kb_y = y;
      return 2;
    }
    return p < 1.0 ? 0 : 1;
  }
}

template <int T>
__device__ __forceinline__ int block_scan_excl(int v, int* s_warp, int* total, bool use_max) {
  // exclusive scan over the block (sum, or max with identity 0); T threads
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x = use_max ? (y > x ? y : x) : x + y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < T / 32 ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w = use_max ? (y > w ? y : w) : w + y;
    }
    if (lane < T / 32) s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const int before = wid > 0 ? s_warp[wid - 1] : 0;
  const int xin = __shfl_up_sync(0xffffffffu, x, 1);
  int excl = lane > 0 ? (use_max ? (before > xin ? before : xin) : before + xin) : before;
  *total = s_warp[T / 32 - 1];
  __syncthreads();
  return excl;
}

// shared-memory slot of one record: at least 16 bytes, so a selected
// record's LINEDATA can be staged where the record was
template <class R>
using SelSlotT = typename std::conditional<(sizeof(R) < sizeof(int4)), int4, R>::type;

template <int KIND>
__device__ __forceinline__ void sel_push_fixes(const SelArgs& a, const typename SelRecType<KIND>::T& r, long long gi,
                                               long long pos, int nu, unsigned keep, unsigned fx,
                                               const int* s_molcor) {
  SelFix f;
  f.pos = pos;
  if (keep) {
    unsigned fx2;
    int4 o2;
    double c = 0.0, y = 0.0;
    SelOps op;
    sel_gather<KIND>(r, a, nu, s_molcor, op);
    sel_decide<KIND>(r, a, gi, nu, op, &o2, &fx2, &c, &y);  // the test's operands again
    f.what = kFixKeep;
    f.arg = 0;
    f.a = c;
    f.b = y;
    const unsigned s = atomicAdd(a.nfix, 1u);
    if (s < a.fixcap) a.fix[s] = f;
  }
  if constexpr (KIND == kSelTio || KIND == kSelH2o) {
    if (fx & (1u << kFixIelo)) {
      f.what = kFixIelo;
      f.arg = 0;
      if constexpr (KIND == kSelTio) {
        const double a1 = fabs((double)r.e1), a2 = fabs((double)r.e2);
        const double e = a2 < a1 ? a2 : a1;
        f.a = e > 1.0e-10 ? e : 1.0e-10;
      } else {
        f.a = (double)abs((int)r.ielo);
      }
      f.b = 0.0;
      const unsigned s = atomicAdd(a.nfix, 1u);
      if (s < a.fixcap) a.fix[s] = f;
    }
    if constexpr (KIND == kSelTio) {
      if (fx & (1u << kFixIgr)) {
        f.what = kFixIgr;
        f.arg = r.gr;
        f.a = (double)r.wl;
        f.b = 0.0;
        const unsigned s = atomicAdd(a.nfix, 1u);
        if (s < a.fixcap) a.fix[s] = f;
      }
    }
  }
}

// Pass A: the largest UB of each tile's records (the NU a tile leaves
// behind, before the carry from earlier tiles).  Record k of the tile is
// read by thread k % 256: the maximum does not depend on the order.
template <int KIND>
__global__ void __launch_bounds__(kSelThreads) k_sel_tile_ub(SelArgs a, int* __restrict__ tile_ub) {
  using R = typename SelRecType<KIND>::T;
  __shared__ int s_iwt[kSelMaxWave];
  __shared__ int s_warp[kSelThreads / 32];
  const int t = threadIdx.x, tile = blockIdx.x;
  for (int k = t; k <= a.nwave; k += kSelThreads) s_iwt[k] = a.iwt[k];
  __syncthreads();
  const long long base = (long long)tile * kSelTile;
  const int cnt = (int)min((long long)kSelTile, a.n - base);
  const R* g = reinterpret_cast<const R*>(a.recs) + base;
  int m = 0;
#pragma unroll 4
  for (int k = t; k < cnt; k += kSelThreads) {
    int iwl;
    if (sel_advance_iwl<KIND>(g[k], a, base + k, &iwl)) {
      const int u = min(sel_ub(s_iwt, a.nwave, iwl, 0), a.nwave + 1);
      m = u > m ? u : m;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) s_warp[t >> 5] = m;
  __syncthreads();
  if (t == 0) {
    int r = 0;
    for (int w = 0; w < kSelThreads / 32; ++w) r = max(r, s_warp[w]);
    tile_ub[tile] = r;
  }
}

// Exclusive scan over n tile values by one CTA of 1024 threads, in chunks:
// the maximum with `init` folded in first (MAX), or the sum from 0.  out[n]
// receives the total.
template <bool MAX>
__global__ void __launch_bounds__(1024) k_sel_scan(const int* __restrict__ in, int n, long long init,
                                                   long long* __restrict__ out) {
  __shared__ long long s_warp[32];
  __shared__ long long s_carry;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  if (t == 0) s_carry = MAX ? init : 0;
  __syncthreads();
  for (int c0 = 0; c0 < n; c0 += 1024) {
    const int i = c0 + t;
    long long v = i < n ? (long long)in[i] : 0;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x = MAX ? (y > x ? y : x) : x + y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
      long long w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w = MAX ? (y > w ? y : w) : w + y;
      }
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const long long carry = s_carry;
    const long long before = wid > 0 ? s_warp[wid - 1] : (MAX ? 0 : 0);
    const long long xin = __shfl_up_sync(0xffffffffu, x, 1);
    long long ex = lane > 0 ? (MAX ? (before > xin ? before : xin) : before + xin) : before;
    ex = MAX ? (ex > carry ? ex : carry) : ex + carry;
    if (i < n) out[i] = ex;
    __syncthreads();
    if (t == 1023) {
      const long long inc = MAX ? (ex > v ? ex : v) : ex + v;
      s_carry = inc;
    }
    __syncthreads();
  }
  if (t == 0) out[n] = s_carry;
}

// Pass B: the filter.  One tile of kSelTile records per CTA, staged
// coalesced in shared memory; thread t takes records 8t..8t+7.  NU at the
// tile's entry comes from the scan of pass A.  The selected records'
// LINEDATA goes to the tile's place in the scratch array, compacted in file
// order, with the host's cases listed at their scratch positions.
template <int KIND>
__global__ void __launch_bounds__(kSelThreads, 4) k_selectlines(SelArgs a) {
  using R = typename SelRecType<KIND>::T;
  using Slot = SelSlotT<R>;
  extern __shared__ __align__(16) unsigned char sel_smem[];
  Slot* s_slot = reinterpret_cast<Slot*>(sel_smem);  // padded tile
  __shared__ int s_iwt[kSelMaxWave];
  __shared__ int s_molcor[KIND == kSelDiatomic ? kSelMolN : 1];
  __shared__ int s_warp[kSelThreads / 32];
  auto rec = [&](int k) -> const R& { return *reinterpret_cast<const R*>(&s_slot[sel_slot(k)]); };

  const int t = threadIdx.x, tile = blockIdx.x;
  for (int k = t; k <= a.nwave; k += kSelThreads) s_iwt[k] = a.iwt[k];
  if constexpr (KIND == kSelDiatomic)
    for (int k = t; k < kSelMolN; k += kSelThreads) s_molcor[k] = a.molcor[k];
  const long long base = (long long)tile * kSelTile;
  const int cnt = (int)min((long long)kSelTile, a.n - base);
  const R* g = reinterpret_cast<const R*>(a.recs) + base;
  for (int k = t; k < cnt; k += kSelThreads) *reinterpret_cast<R*>(&s_slot[sel_slot(k)]) = g[k];
  const int tile_nu = (int)a.tile_nu[tile];
  __syncthreads();

  // UB of each record's IWL, running maximum in file order
  int run = 0, hint = 0;
  int ubs[kSelItems];
#pragma unroll
  for (int i = 0; i < kSelItems; ++i) {
    const int k = t * kSelItems + i;
    ubs[i] = 0;
    if (k < cnt) {
      int iwl;
      if (sel_advance_iwl<KIND>(rec(k), a, base + k, &iwl)) {
        int u = sel_ub(s_iwt, a.nwave, iwl, hint);
        hint = u;
        if (u > a.nwave + 1) {
          sel_error(a.err, base + k, kSelErrSentinel);
          u = a.nwave + 1;
        }
        ubs[i] = u;
        run = u > run ? u : run;
      }
    }
  }
  int agg;
  const int pre = block_scan_excl<kSelThreads>(run, s_warp, &agg, true);
  const int nu_in = tile_nu > pre ? tile_nu : pre;  // NU before this thread's records

  // the filter at each record's NU, operands gathered a group at a time; a
  // selected record's LINEDATA replaces it in its slot
  int nu = nu_in;
  unsigned sel = 0, keep = 0, fixbits = 0;
  int mycount = 0;
#pragma unroll
  for (int g0 = 0; g0 < kSelItems; g0 += kSelGroup) {
    SelOps ops[kSelGroup];
    int nug[kSelGroup];
#pragma unroll
    for (int j = 0; j < kSelGroup; ++j) {
      const int i = g0 + j, k = t * kSelItems + i;
      nu = ubs[i] > nu ? ubs[i] : nu;
      nug[j] = nu;
      if (k < cnt) sel_gather<KIND>(rec(k), a, nu, s_molcor, ops[j]);
    }
#pragma unroll
    for (int j = 0; j < kSelGroup; ++j) {
      const int i = g0 + j, k = t * kSelItems + i;
      if (k < cnt) {
        unsigned fx;
        double c, y;
        int4 o;
        const int d = sel_decide<KIND>(rec(k), a, base + k, nug[j], ops[j], &o, &fx, &c, &y);
        if (d) {
          *reinterpret_cast<int4*>(&s_slot[sel_slot(k)]) = o;
          sel |= 1u << i;
          if (d == 2) keep |= 1u << i;
          fixbits |= fx << (2 * i);
          ++mycount;
        }
      }
    }
  }
  int total;
  const int opre = block_scan_excl<kSelThreads>(mycount, s_warp, &total, false);
  if (t == 0) a.tile_count[tile] = total;

  // the tile's LINEDATA to its scratch place in file order; the host's cases
  // (the original record comes from global memory: its slot holds LINEDATA)
  int4* sc = a.scratch + base;
  int q = opre;
  nu = nu_in;
#pragma unroll
  for (int i = 0; i < kSelItems; ++i) {
    nu = ubs[i] > nu ? ubs[i] : nu;
    if (sel >> i & 1u) {
      const int k = t * kSelItems + i;
      sc[q] = *reinterpret_cast<const int4*>(&s_slot[sel_slot(k)]);
      const unsigned fx = (fixbits >> (2 * i)) & 3u;
      if ((keep >> i & 1u) || fx) sel_push_fixes<KIND>(a, g[k], base + k, base + q, nu, keep >> i & 1u, fx, s_molcor);
      ++q;
    }
  }
}

// Pass C: every tile's LINEDATA from its scratch place to its offset (the
// exclusive sum of the counts); positions at or past cap are not written
__global__ void __launch_bounds__(256) k_sel_move(const int4* __restrict__ scratch, const int* __restrict__ count,
                                                  const long long* __restrict__ off, int ntiles, int4* out,
                                                  long long cap) {
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int c = count[tile];
    const long long o = off[tile];
    const int4* src = scratch + (long long)tile * kSelTile;
    for (int k = threadIdx.x; k < c; k += blockDim.x)
      if (o + k < cap) out[o + k] = src[k];
  }
}

// the fix list's scratch positions -> output positions
__global__ void k_sel_fixpos(SelFix* fix, const unsigned* nfix, unsigned fixcap, const long long* __restrict__ off) {
  const unsigned e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= min(*nfix, fixcap)) return;
  const long long p = fix[e].pos;
  fix[e].pos = off[p / kSelTile] + p % kSelTile;
}

// drop the records at sorted positions rm [nrm] from in [n] into out
__global__ void __launch_bounds__(256) k_sel_remove(const int4* __restrict__ in, long long n, const long long* rm,
                                                    int nrm, int4* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nrm;  // removed positions below i
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (rm[mid] < i)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < nrm && rm[lo] == i) continue;
    out[i - lo] = in[i];
  }
}

}  // namespace atlasgpu
