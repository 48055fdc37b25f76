// api_select.cu -- C ABI: SELECTLINES (atlas12_modules.f90:19171-19781),
// the line databases filtered into LINEDATA on the device.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "api_common.cuh"
#include "select.cuh"

using namespace atlasgpu;

namespace {

// SELECTLINES's constant tables (atlas12_modules.f90:19182-19207): the
// diatomic species codes with their isotopologue log gf corrections, and the
// TiO / H2O isotope corrections, all in millidex
constexpr int kNmol = 46;
const int kMolcodes[kNmol] = {8410, 8411, 8460, 8461, 8470, 8471, 8480, 8481, 8482, 8510, 8511, 8512,
                              8530, 8531, 8532, 8580, 8581, 8582, 8583, 8584, 8620, 8621, 8622, 8623,
                              8640, 8641, 8642, 8643, 8680, 8681, 8682, 8690, 8691, 8692, 8693, 8700,
                              8701, 8702, 8703, 8704, 8705, 8890, 8891, 8892, 8896, 8960};
const int kIsox[kNmol] = {0,     -4469, -5,    -1955, -2,    -2444, -1,    -3398, -2690, -105,  -996,  -947,
                          -35,   -1331, -1516, -13,   -2189, -2870, -1681, -4398, -1362, -77,   -1022, -1626,
                          -1237, -38,   -1658, -2553, -10,   -1960, -3910, -7,    -1957, -2449, -4399, -6,
                          -1956, -3403, -5353, -2695, -4645, -36,   -1332, -1517, -2725, -2};
const int kTioIsocorr[5] = {-1101, -1138, -131, -1259, -1272};
const int kH2oIsocorr[4] = {-1, -3398, -2690, -5000};

constexpr unsigned kFixCap = 1u << 16;
constexpr double kCenPrefac = 0.026538 / kSqrtPi;  // CEN_PREFAC (:19178)

// INT() of a REAL(8) as x86-64 converts it, and INTEGER(2) assignment
int32_t h_fint(double x) { return (x > -2147483649.0 && x < 2147483648.0) ? (int32_t)x : INT32_MIN; }
int16_t h_i16(int32_t v) { return (int16_t)(uint16_t)(uint32_t)v; }
// INT(LOG10(x)*1000 + 16384.5) with each operation rounded separately
int16_t h_log_field(double x) {
  volatile double m = log10(x) * 1000.0;
  return h_i16(h_fint(m + 16384.5));
}

double ratiolg_lines() { return log(1.0 + 1.0 / 2000000.0); }

size_t rec_bytes(int kind) { return kind == kSelTio ? 32 : kind == kSelH2o ? 8 : 16; }

size_t sel_smem(int kind) { return std::max<size_t>(rec_bytes(kind), 16) * (kSelTile + kSelThreads); }

// pass A (tile maxima of UB), the scan of NU at each tile's entry, pass B
template <int K>
int launch_select(atlasgpu_ctx* ctx, const SelArgs& a, int ntiles) {
  int* d_tub;
  int r;
  if ((r = bufT(ctx, "sel_tub", ntiles, &d_tub))) return r;
  k_sel_tile_ub<K><<<ntiles, kSelThreads, 0, ctx->stream>>>(a, d_tub);
  CKL(ctx);
  k_sel_scan<true><<<1, 1024, 0, ctx->stream>>>(d_tub, ntiles, a.nu0, const_cast<long long*>(a.tile_nu));
  CKL(ctx);
  const size_t smem = sel_smem(K);
  CK(cudaFuncSetAttribute(k_selectlines<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_selectlines<K><<<ntiles, kSelThreads, smem, ctx->stream>>>(a);
  CKL(ctx);
  return 0;
}

int dispatch(atlasgpu_ctx* ctx, int kind, const SelArgs& a, int ntiles) {
  switch (kind) {
    case kSelLowPred: return launch_select<kSelLowPred>(ctx, a, ntiles);
    case kSelLowObs: return launch_select<kSelLowObs>(ctx, a, ntiles);
    case kSelHi: return launch_select<kSelHi>(ctx, a, ntiles);
    case kSelDiatomic: return launch_select<kSelDiatomic>(ctx, a, ntiles);
    case kSelTio: return launch_select<kSelTio>(ctx, a, ntiles);
    case kSelH2o: return launch_select<kSelH2o>(ctx, a, ntiles);
    case kSelH3plus: return launch_select<kSelH3plus>(ctx, a, ntiles);
  }
  return fail(ctx, ATLASGPU_EINVAL, "selectlines: unknown database kind %d", kind);
}

const char* err_text(int code) {
  switch (code) {
    case kSelErrNelion: return "NELION outside 1..nspec";
    case kSelErrMolcode: return "diatomic MOLCODE not in MOLCODES";
    case kSelErrSentinel: return "IWL at or past the IWAVETAB sentinel";
    default: return "TiO IWL missing from the host decisions";
  }
}

// The TiO records near an IWL rounding boundary, decided with the C library
// log; uploaded sorted by record index for the selection pass.
int tio_overrides(atlasgpu_ctx* ctx, const void* d_recs, int64_t n, const long long** d_idx, const int** d_iwl,
                  int* novr) {
  long long* d_list;
  unsigned* d_cnt;
  int r;
  if ((r = bufT(ctx, "sel_ovr_list", kFixCap, &d_list)) || (r = bufT(ctx, "sel_ovr_cnt", 1, &d_cnt))) return r;
  CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned), ctx->stream));
  const double ratiolg = ratiolg_lines();
  k_sel_tio_border<<<grid_for(ctx, n, 256, 8), 256, 0, ctx->stream>>>((const SelMol2*)d_recs, n, ratiolg, d_list,
                                                                       d_cnt, kFixCap);
  CKL(ctx);
  unsigned cnt = 0;
  CK(cudaMemcpyAsync(&cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (cnt > kFixCap) return fail(ctx, ATLASGPU_EINVAL, "selectlines: %u TiO wavelengths near a bin boundary", cnt);
  std::vector<long long> idx(cnt);
  if (cnt) CK(cudaMemcpy(idx.data(), d_list, cnt * sizeof(long long), cudaMemcpyDeviceToHost));
  std::sort(idx.begin(), idx.end());
  std::vector<int> iwl(cnt);
  for (unsigned k = 0; k < cnt; ++k) {
    SelMol2 rec;
    CK(cudaMemcpy(&rec, (const SelMol2*)d_recs + idx[k], sizeof rec, cudaMemcpyDeviceToHost));
    iwl[k] = h_fint(log((double)rec.wl) / ratiolg + 0.5);
  }
  long long* di;
  int* dw;
  if ((r = bufT(ctx, "sel_ovr_idx", cnt + 1, &di)) || (r = bufT(ctx, "sel_ovr_iwl", cnt + 1, &dw))) return r;
  if (cnt) {
    CK(cudaMemcpyAsync(di, idx.data(), cnt * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dw, iwl.data(), cnt * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  }
  *d_idx = di;
  *d_iwl = dw;
  *novr = (int)cnt;
  return 0;
}

// Records per pass of the kernels (scratch: 16 bytes per record)
constexpr int64_t kSelChunk = int64_t(1) << 27;

// One chunk through passes A-C and the host's decisions.  Output at d_out
// (at most cap records); *n_out the count; error records offset by rec0.
int select_chunk(atlasgpu_ctx* ctx, int kind, const void* d_recs, int64_t n, atlasgpu_select_state* st, int4* d_out,
                 int64_t cap, int64_t* n_out, int64_t rec0) {
  const int nwave = ctx->sel_nwave;
  const long long* d_ovr_idx = nullptr;
  const int* d_ovr_iwl = nullptr;
  int novr = 0, r;
  if (kind == kSelTio && (r = tio_overrides(ctx, d_recs, n, &d_ovr_idx, &d_ovr_iwl, &novr))) return r;

  const int ntiles = (int)((n + kSelTile - 1) / kSelTile);
  int *d_tub, *d_cnt;
  long long *d_nu, *d_off;
  int4* d_scr;
  unsigned long long* d_err;
  unsigned* d_nfix;
  SelFix* d_fix;
  if ((r = bufT(ctx, "sel_tub", ntiles, &d_tub)) || (r = bufT(ctx, "sel_tcnt", ntiles, &d_cnt)) ||
      (r = bufT(ctx, "sel_tnu", ntiles + 1, &d_nu)) || (r = bufT(ctx, "sel_toff", ntiles + 1, &d_off)) ||
      (r = bufT(ctx, "sel_scratch", (size_t)ntiles * kSelTile, &d_scr)) || (r = bufT(ctx, "sel_err", 1, &d_err)) ||
      (r = bufT(ctx, "sel_nfix", 1, &d_nfix)) || (r = bufT(ctx, "sel_fix", kFixCap, &d_fix)))
    return r;
  CK(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), ctx->stream));
  CK(cudaMemsetAsync(d_nfix, 0, sizeof(unsigned), ctx->stream));

  SelArgs a{};
  a.recs = d_recs;
  a.n = n;
  a.nu0 = st->nu;
  a.igr0 = (int16_t)st->igr;
  a.freq0 = st->freq;
  int *d_iwt, *d_mol;
  double *d_freq, *d_xmax, *d_tablog;
  short* d_igr;
  if ((r = bufT(ctx, "sel_iwt", nwave + 1, &d_iwt)) || (r = bufT(ctx, "sel_freq", nwave, &d_freq)) ||
      (r = bufT(ctx, "sel_igr", nwave, &d_igr)) || (r = bufT(ctx, "sel_mol", kSelMolN + 9, &d_mol)) ||
      (r = bufT(ctx, "sel_xmax", (size_t)(nwave + 1) * ctx->sel_nspec, &d_xmax)) || (r = ensure_tablog(ctx, &d_tablog)))
    return r;
  a.iwt = d_iwt;
  a.nwave = nwave;
  a.freqtab = d_freq;
  a.igrtab = d_igr;
  a.xmax = d_xmax;
  a.nspec = ctx->sel_nspec;
  a.tablog = d_tablog;
  a.hckt_last = ctx->sel_hckt_last;
  a.cen_prefac = kCenPrefac;
  a.ratiolg = ratiolg_lines();
  a.molcor = d_mol;
  a.tio_isocorr = d_mol + kSelMolN;
  a.h2o_isocorr = d_mol + kSelMolN + 5;
  a.ovr_idx = d_ovr_idx;
  a.ovr_iwl = d_ovr_iwl;
  a.novr = novr;
  a.tile_nu = d_nu;
  a.tile_count = d_cnt;
  a.scratch = d_scr;
  a.fix = d_fix;
  a.nfix = d_nfix;
  a.fixcap = kFixCap;
  a.err = d_err;
  {
    Timer tk(ctx, "k_selectlines");
    if ((r = dispatch(ctx, kind, a, ntiles))) return r;
    k_sel_scan<false><<<1, 1024, 0, ctx->stream>>>(d_cnt, ntiles, 0, d_off);
    CKL(ctx);
    k_sel_move<<<std::min(ntiles, ctx->nsm * 8), 256, 0, ctx->stream>>>(d_scr, d_cnt, d_off, ntiles, d_out, cap);
    CKL(ctx);
  }
  k_sel_fixpos<<<(kFixCap + 255) / 256, 256, 0, ctx->stream>>>(d_fix, d_nfix, kFixCap, d_off);
  CKL(ctx);

  long long last[2];
  unsigned long long err;
  unsigned nfix;
  CK(cudaMemcpyAsync(&last[0], d_nu + ntiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&last[1], d_off + ntiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&err, d_err, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&nfix, d_nfix, sizeof nfix, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (err != ~0ull)
    return fail(ctx, ATLASGPU_EINVAL, "selectlines: record %lld: %s", (long long)(err >> 8) + (long long)rec0,
                err_text((int)(err & 0xff)));
  const int nu = (int)last[0];
  int64_t total = (int64_t)last[1];
  if (total > cap)
    return fail(ctx, ATLASGPU_EINVAL, "selectlines: LINEDATA overflow (record set beyond cap %lld)", (long long)cap);
  if (nfix > kFixCap) return fail(ctx, ATLASGPU_EINVAL, "selectlines: %u records near a rounding boundary", nfix);

  // the host's decisions: fields first (positions before any removal), then the Boltzmann tests
  std::vector<SelFix> fx(nfix);
  if (!fx.empty()) CK(cudaMemcpy(fx.data(), d_fix, fx.size() * sizeof(SelFix), cudaMemcpyDeviceToHost));
  std::vector<long long> drop;
  for (const SelFix& f : fx) {
    if (f.what == kFixKeep) {
      if (f.a * exp(f.b) < 1.0) drop.push_back(f.pos);
      continue;
    }
    int4 rec;
    CK(cudaMemcpy(&rec, d_out + f.pos, sizeof rec, cudaMemcpyDeviceToHost));
    if (f.what == kFixIelo) {
      const int16_t v = h_log_field(f.a);
      rec.y = (int)(((unsigned)rec.y & 0xffffu) | ((unsigned)(uint16_t)v << 16));
    } else {
      const double w = f.a;
      const double g = f.arg == 0 ? 2.223e13 / (w * w) : pow(10.0, (double)f.arg * 0.01);
      const int16_t v = h_log_field(g);
      rec.z = (int)(((unsigned)rec.z & 0xffffu) | ((unsigned)(uint16_t)v << 16));
    }
    CK(cudaMemcpy(d_out + f.pos, &rec, sizeof rec, cudaMemcpyHostToDevice));
  }
  if (!drop.empty()) {
    std::sort(drop.begin(), drop.end());
    long long* d_rm;
    int4* d_tmp;
    if ((r = bufT(ctx, "sel_rm", drop.size(), &d_rm)) || (r = bufT(ctx, "sel_tmp", (size_t)total, &d_tmp))) return r;
    CK(cudaMemcpyAsync(d_rm, drop.data(), drop.size() * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    k_sel_remove<<<grid_for(ctx, total, 256, 8), 256, 0, ctx->stream>>>(d_out, total, d_rm, (int)drop.size(), d_tmp);
    CKL(ctx);
    total -= (int64_t)drop.size();
    if (total) CK(cudaMemcpyAsync(d_out, d_tmp, total * sizeof(int4), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }

  // the module variables the loop leaves behind (IGR of the LINEREC kinds: by the caller)
  const bool adv = nu > st->nu;
  if (adv) st->freq = ctx->sel_freqtab[nu - 2];
  if (kind == kSelH2o) {
    if (adv) st->igr = ctx->sel_igrtab[nu - 2];
  } else if (kind == kSelTio && total > 0) {
    int4 rec;
    CK(cudaMemcpy(&rec, d_out + total - 1, sizeof rec, cudaMemcpyDeviceToHost));
    st->igr = (int16_t)((unsigned)rec.z >> 16);
  }
  st->nu = nu;
  *n_out = total;
  return 0;
}

// All records, a chunk at a time with the loop state carried over.
// last_rec_igr: the IGR field of the last input record (LINEREC kinds),
// which UNPACK_LINEDATA leaves in the module variable.
int select_core(atlasgpu_ctx* ctx, int kind, const void* d_recs, int64_t n, atlasgpu_select_state* st, int4* d_out,
                int64_t cap, int64_t* n_out, int16_t last_rec_igr) {
  const size_t rb = rec_bytes(kind);
  int64_t written = 0;
  for (int64_t c0 = 0; c0 < n; c0 += kSelChunk) {
    const int64_t cn = std::min(kSelChunk, n - c0);
    int64_t m = 0;
    int r = select_chunk(ctx, kind, (const char*)d_recs + c0 * rb, cn, st, d_out + written, cap - written, &m, c0);
    if (r) return r;
    written += m;
  }
  if (kind != kSelTio && kind != kSelH2o) st->igr = last_rec_igr;
  *n_out = written;
  return 0;
}

int check_call(atlasgpu_ctx* ctx, int kind, int64_t n, const atlasgpu_select_state* st, int64_t cap, int64_t* n_out) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (!ctx->sel_ready) return fail(ctx, ATLASGPU_ESTATE, "selectlines: call atlasgpu_atlas_select_tables first");
  if (kind < kSelLowPred || kind > kSelH3plus) return fail(ctx, ATLASGPU_EINVAL, "selectlines: unknown kind %d", kind);
  if (n < 0 || cap < 0 || !st || !n_out) return fail(ctx, ATLASGPU_EINVAL, "selectlines: bad argument");
  if (st->nu < 1 || st->nu > ctx->sel_nwave + 1)
    return fail(ctx, ATLASGPU_EINVAL, "selectlines: NU %d outside 1..%d", st->nu, ctx->sel_nwave + 1);
  if ((n + kSelTile - 1) / kSelTile > 0x7fffffffLL) return fail(ctx, ATLASGPU_EINVAL, "selectlines: too many records");
  return 0;
}

}  // namespace

extern "C" {

int atlasgpu_atlas_select_tables(atlasgpu_ctx* ctx, int nrhox, int kw, const double* xnfdop, int nspec,
                                 const double* hckt, const double* tabcont, const int32_t* iwavetab,
                                 const double* wavetab, int nwave) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (nrhox < 1 || kw < nrhox || nspec < 1 || nwave < 1 || nwave + 1 > kSelMaxWave || !xnfdop || !hckt || !tabcont ||
      !iwavetab || !wavetab)
    return fail(ctx, ATLASGPU_EINVAL, "select_tables: bad argument");
  for (int k = 0; k < nwave; ++k)
    if (iwavetab[k + 1] < iwavetab[k]) return fail(ctx, ATLASGPU_EINVAL, "select_tables: IWAVETAB decreases at %d", k + 1);
  if (!finite_all(xnfdop, (size_t)nspec * kw) || !finite_all(tabcont, (size_t)(nwave + 1) * kw) ||
      !finite_all(hckt, nrhox) || !finite_all(wavetab, nwave))
    return fail(ctx, ATLASGPU_ENONFINITE, "select_tables: non-finite table value");
  cudaSetDevice(ctx->device);
  ctx->sel_ready = false;
  double *d_xn, *d_tc, *d_xmax, *d_freq, *d_tl;
  int *d_iwt, *d_mol;
  short* d_igr;
  int r;
  if ((r = bufT(ctx, "sel_xnfdop", (size_t)nspec * kw, &d_xn)) ||
      (r = bufT(ctx, "sel_tabcont", (size_t)(nwave + 1) * kw, &d_tc)) ||
      (r = bufT(ctx, "sel_xmax", (size_t)(nwave + 1) * nspec, &d_xmax)) || (r = bufT(ctx, "sel_iwt", nwave + 1, &d_iwt)) ||
      (r = bufT(ctx, "sel_freq", nwave, &d_freq)) || (r = bufT(ctx, "sel_igr", nwave, &d_igr)) ||
      (r = bufT(ctx, "sel_mol", kSelMolN + 9, &d_mol)) || (r = ensure_tablog(ctx, &d_tl)))
    return r;
  CK(cudaMemcpyAsync(d_xn, xnfdop, (size_t)nspec * kw * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_tc, tabcont, (size_t)(nwave + 1) * kw * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_sel_xnfdopmax<<<grid_for(ctx, (int64_t)(nwave + 1) * nspec, 256, 8), 256, 0, ctx->stream>>>(nrhox, kw, d_xn, nspec,
                                                                                                 d_tc, nwave, d_xmax);
  CKL(ctx);
  // FREQ and H2O's IGR after the advance past bin k (:19614, :19668-19673)
  std::vector<double> freq(nwave);
  std::vector<int16_t> igr(nwave);
  for (int k = 0; k < nwave; ++k) {
    freq[k] = kClightNms / wavetab[k];
    volatile double f2 = freq[k] * freq[k];
    volatile double g = 2.474e-22 * f2;
    volatile double gammar = g * (double)0.001f;  // 0.001 is a default REAL literal there
    igr[k] = h_log_field(gammar);
  }
  // ISOX by MOLCODE (the reference searches MOLCODES, :19467-19481), then TIO_ISOCORR, H2O_ISOCORR
  std::vector<int> mol(kSelMolN + 9, kSelMolUnknown);
  for (int k = 0; k < kNmol; ++k) mol[kMolcodes[k] - kSelMolLo] = kIsox[k];
  std::copy(kTioIsocorr, kTioIsocorr + 5, mol.begin() + kSelMolN);
  std::copy(kH2oIsocorr, kH2oIsocorr + 4, mol.begin() + kSelMolN + 5);
  CK(cudaMemcpyAsync(d_iwt, iwavetab, (nwave + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_freq, freq.data(), nwave * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_igr, igr.data(), nwave * sizeof(short), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_mol, mol.data(), mol.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->sel_nwave = nwave;
  ctx->sel_nspec = nspec;
  ctx->sel_hckt_last = hckt[nrhox - 1];
  ctx->sel_freqtab = std::move(freq);
  ctx->sel_igrtab = std::move(igr);
  ctx->sel_ready = true;
  return 0;
}

int atlasgpu_atlas_selectlines_dev(atlasgpu_ctx* ctx, int kind, const void* d_recs, int64_t n,
                                   atlasgpu_select_state* state, int32_t* d_linedata_out, int64_t cap,
                                   int64_t* n_out) {
  int r = check_call(ctx, kind, n, state, cap, n_out);
  if (r) return r;
  const size_t align = kind == kSelH2o ? 8 : 16;
  if (n > 0 && (!d_recs || (uintptr_t)d_recs % align))
    return fail(ctx, ATLASGPU_EINVAL, "selectlines_dev: records must be %zu-byte aligned", align);
  if (cap > 0 && (!d_linedata_out || (uintptr_t)d_linedata_out % 16))
    return fail(ctx, ATLASGPU_EINVAL, "selectlines_dev: output must be 16-byte aligned");
  if (n == 0) {
    *n_out = 0;
    return 0;
  }
  cudaSetDevice(ctx->device);
  int16_t igr = 0;
  if (kind != kSelTio && kind != kSelH2o) {
    int32_t w;
    CK(cudaMemcpy(&w, (const int32_t*)d_recs + 4 * (n - 1) + 2, sizeof w, cudaMemcpyDeviceToHost));
    igr = (int16_t)((uint32_t)w >> 16);
  }
  return select_core(ctx, kind, d_recs, n, state, (int4*)d_linedata_out, cap, n_out, igr);
}

int atlasgpu_atlas_selectlines(atlasgpu_ctx* ctx, int kind, const void* recs, int64_t n,
                               atlasgpu_select_state* state, int32_t* linedata_out, int64_t cap,
                               int64_t* n_out) {
  int r = check_call(ctx, kind, n, state, cap, n_out);
  if (r) return r;
  if (n > 0 && !recs) return fail(ctx, ATLASGPU_EINVAL, "selectlines: records missing");
  if (cap > 0 && !linedata_out) return fail(ctx, ATLASGPU_EINVAL, "selectlines: output missing");
  if (n == 0) {
    *n_out = 0;
    return 0;
  }
  cudaSetDevice(ctx->device);
  const size_t rb = rec_bytes(kind);
  void* d_in;
  int4* d_out;
  const int64_t ocap = std::min<int64_t>(cap, n);
  if ((r = buf(ctx, "sel_in", (size_t)n * rb, &d_in)) || (r = bufT(ctx, "sel_out", (size_t)ocap + 1, &d_out))) return r;
  CK(cudaMemcpyAsync(d_in, recs, (size_t)n * rb, cudaMemcpyHostToDevice, ctx->stream));
  int16_t igr = 0;
  if (kind != kSelTio && kind != kSelH2o) igr = (int16_t)((uint32_t)((const int32_t*)recs)[4 * (n - 1) + 2] >> 16);
  if ((r = select_core(ctx, kind, d_in, n, state, d_out, cap, n_out, igr))) return r;
  if (*n_out) CK(cudaMemcpy(linedata_out, d_out, (size_t)*n_out * sizeof(int4), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
