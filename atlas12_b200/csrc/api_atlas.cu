// api_atlas.cu -- C ABI: the ATLAS12 entry points (LINOP1, RT pass, finish)
// and the device-resident model iteration.
#include <cmath>
#include <vector>

#include "api_common.cuh"
#include "atlas.cuh"
#include "hydrogen.cuh"
#include "tcorr.cuh"

using namespace atlasgpu;

namespace atlasgpu {

int ensure_tablog(atlasgpu_ctx* ctx, double** out) {
  double* d;
  const bool fresh = ctx->bufs.find("tablog") == ctx->bufs.end();
  int r = bufT(ctx, "tablog", 65536, &d);
  if (r) return r;
  if (fresh) {
    // TABLOG(I) = 10**((I-16384)*0.001) for every INTEGER(2) I, with the C
    // library pow that the reference's ** calls
    std::vector<double> h(65536);
    for (int k = 0; k < 65536; ++k) h[k] = pow(10.0, (double)((k - 32768) - 16384) * 0.001);
    CK(cudaMemcpy(d, h.data(), 65536 * sizeof(double), cudaMemcpyHostToDevice));
  }
  *out = d;
  return 0;
}

}  // namespace atlasgpu

namespace {

constexpr int kTabN = 2001;

}  // namespace

namespace {

// the flagged LINEDATA records and their device-prepared lines, gathered
// into compact arrays
__global__ void k_prep_gather(const int4* __restrict__ ld, const AtlasLine* __restrict__ lines,
                              const int64_t* __restrict__ idx, int64_t n, int4* __restrict__ rec,
                              AtlasLine* __restrict__ fix) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    rec[k] = ld[idx[k]];
    fix[k] = lines[idx[k]];
  }
}

// the host-recomputed lines back to their places
__global__ void k_prep_scatter(const AtlasLine* __restrict__ fix, const int64_t* __restrict__ idx, int64_t n,
                               AtlasLine* __restrict__ lines) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    lines[idx[k]] = fix[k];
}

}  // namespace

namespace atlasgpu {
// Line preparation (k_atlas_prep) with the host fix of near-tie frequency
// brackets: a line whose device wavelength lies within a few ulps of a grid
// point is recomputed with the C library's exp and pow, the functions the
// reference's EXP and ** call.  The flagged records are gathered on the
// device and crossed in one copy each way; when more lines are flagged than
// the flag buffer holds, the buffer grows to the count and the pass runs
// again.
int atlas_prep_lines(atlasgpu_ctx* ctx, const int32_t* d_ld, const int32_t* h_ld, int64_t n,
                     const double* d_tablog, const double* d_ws, const double* h_ws, int numnu,
                     const int32_t* d_iwt, int nwave, int nspec, AtlasLine* d_lines) {
  (void)h_ld;
  unsigned long long* d_nf;
  int r;
  if ((r = bufT(ctx, "ap_nflag", 1, &d_nf))) return r;
  int64_t cap = 1 << 12;
  unsigned long long nf = 0;
  int64_t* d_fl = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    if ((r = bufT(ctx, "ap_flag", cap, &d_fl))) return r;
    CK(cudaMemsetAsync(d_nf, 0, sizeof(unsigned long long), ctx->stream));
    AtlasPrepArgs a{d_ld, n, d_tablog, d_ws, numnu, d_iwt, nwave, nspec, d_lines, d_fl, d_nf, cap};
    {
      Timer tm(ctx, "atlas_prep");
      k_atlas_prep<<<grid_for(ctx, n, 256, 16), 256, 0, ctx->stream>>>(a);
      CKL(ctx);
    }
    CK(cudaMemcpyAsync(&nf, d_nf, sizeof nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((int64_t)nf <= cap) break;
    cap = (int64_t)nf;  // every flag fits on the second pass
  }
  if (nf == 0) return 0;
  int4* d_rec;
  AtlasLine* d_fix;
  if ((r = bufT(ctx, "ap_rec", nf, &d_rec)) || (r = bufT(ctx, "ap_fix", nf, &d_fix))) return r;
  const int g = grid_for(ctx, (int64_t)nf, 256, 4);
  k_prep_gather<<<g, 256, 0, ctx->stream>>>(reinterpret_cast<const int4*>(d_ld), d_lines, d_fl, (int64_t)nf,
                                            d_rec, d_fix);
  CKL(ctx);
  std::vector<int4> rec(nf);
  std::vector<AtlasLine> fix(nf);
  CK(cudaMemcpyAsync(rec.data(), d_rec, nf * sizeof(int4), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(fix.data(), d_fix, nf * sizeof(AtlasLine), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double RATIOLG = log(1.0 + 1.0 / 2000000.0);
  const double CEN_PREFAC4 = 0.026538 / kSqrtPi / kClightNms;
  const double FOURPI_C_INV = 1.0 / (4.0 * kPi * kClightNms);
  auto tablog = [](int32_t word, int hi) {
    const int16_t v = (int16_t)(hi ? ((uint32_t)word >> 16) : (word & 0xffff));
    return pow(10.0, (double)((int)v - 16384) * 0.001);
  };
  for (unsigned long long k = 0; k < nf; ++k) {
    const int32_t r0 = rec[k].x, r2 = rec[k].z, r3 = rec[k].w;
    const double wl = exp(r0 * RATIOLG);  // the reference's EXP
    // NU = first grid point with WLVAC < WAVESET(NU), clamped at NUMNU
    int lo = 1, hi = numnu;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (wl < h_ws[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    AtlasLine& L = fix[k];
    L.cgf = CEN_PREFAC4 * wl * tablog(r2, 0);
    L.gr = tablog(r2, 1) * wl * FOURPI_C_INV;
    L.gs = tablog(r3, 0) * wl * FOURPI_C_INV;
    L.gw = tablog(r3, 1) * wl * FOURPI_C_INV;
    L.wlvac = wl;
    L.nu = lo;
  }
  CK(cudaMemcpyAsync(d_fix, fix.data(), nf * sizeof(AtlasLine), cudaMemcpyHostToDevice, ctx->stream));
  k_prep_scatter<<<g, 256, 0, ctx->stream>>>(d_fix, d_fl, (int64_t)nf, d_lines);
  CKL(ctx);
  // the host vectors are pageable: the copy has consumed them when it returns,
  // but wait so that the caller's next step sees the fixed lines
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}
}  // namespace atlasgpu

namespace {

int rt_launch(atlasgpu_ctx* ctx, RtArgs& a, double* d_sum, int* nwarps_out) {
  // the split pass (k_rt_pre, k_rt_solve, k_rt_post): enough warps and pair
  // groups to fill every SM several times, frequencies contiguous per unit
  const RtSplitShape sh = rt_split_shape(a.numnu, ctx->nsm, 1, 4);
  rt_split_args(a, sh);
  const int nwl = sh.rows();
  double *part, *rec;
  int r;
  if ((r = bufT(ctx, "rt_part", (size_t)nwl * (kAcc * a.kw + 1), &part))) return r;
  if ((r = bufT(ctx, "rt_rec", (size_t)a.numnu * a.rec_stride, &rec))) return r;
  a.partial = part;
  a.rec = rec;
  CK(rt_split_attributes(a.nrhox));
  {
    Timer tm(ctx, "atlas_rt");
    k_rt_pre<<<sh.pre_blocks, kRtSplitWarps * 32, rt_pre_smem_bytes(), ctx->stream>>>(a);
    CKL(ctx);
    k_rt_series<<<sh.solve_blocks, kRtSolveThreads, 0, ctx->stream>>>(a);
    CKL(ctx);
    k_rt_solve<<<sh.solve_blocks, kRtSolveThreads, rt_solve_smem_bytes(), ctx->stream>>>(a);
    CKL(ctx);
    k_rt_post<<<sh.post_blocks, kRtSplitWarps * 32, rt_post_smem_bytes(a.nrhox), ctx->stream>>>(a);
    CKL(ctx);
  }
  {
    Timer tm(ctx, "atlas_reduce");
    launch_reduce(part, nwl, a.kw, d_sum, ctx->stream);
    CKL(ctx);
  }
  if (nwarps_out) *nwarps_out = nwl;
  return 0;
}

__global__ void __launch_bounds__(kFinThreads) k_finish_one(ModelState* s, double* acc, int kw, int n, int iter,
                                                             double teff, double grav, RossStore* R) {
  extern __shared__ __align__(16) double fin_smem[];
  if (blockIdx.x == 0) b_atlas_finish(s, acc, kw, n, iter, teff, grav, R, fin_smem);
}

}  // namespace

extern "C" {

int atlasgpu_atlas_tabvoigt(double vsteps, int n, const double* tabvi, const double* tabh1, int ntab,
                            double* h0, double* h1, double* h2) {
  if (!tabvi || !tabh1 || !h0 || !h1 || !h2 || n < 2 || ntab < 4 || !(vsteps > 0.0)) return ATLASGPU_EINVAL;
  for (int i = 1; i < ntab; ++i)
    if (!(tabvi[i] > tabvi[i - 1])) return ATLASGPU_EINVAL;
  // H1 = MAP1 of the tabulated H1(v) onto v = (i-1)/vsteps, H0 = exp(-v^2),
  // H2 = H0 - 2 v^2 H0 (atlas12_modules.f90:19796-19851)
  for (int i = 1; i <= n; ++i) h0[i - 1] = (double)(i - 1) / vsteps;
  s_map1(tabvi, tabh1, ntab, h0, h1, n);
  for (int i = 1; i <= n; ++i) {
    const double vv = powi((double)(i - 1) / vsteps, 2);
    h0[i - 1] = exp(-vv);
    h2[i - 1] = h0[i - 1] - (vv + vv) * h0[i - 1];
  }
  return ATLASGPU_OK;
}

int atlasgpu_atlas_set_voigt_tables(atlasgpu_ctx* ctx, const double* h0, const double* h1,
                                    const double* h2, int n) {
  if (!ctx || !h0 || !h1 || !h2 || n != kTabN) return fail(ctx, ATLASGPU_EINVAL, "voigt tables: n must be 2001");
  if (!finite_all(h0, n) || !finite_all(h1, n) || !finite_all(h2, n))
    return fail(ctx, ATLASGPU_ENONFINITE, "voigt tables: non-finite entry");
  cudaSetDevice(ctx->device);
  double *d0, *d1, *d2, *tl;
  int r;
  if ((r = bufT(ctx, "tab_h0", n, &d0)) || (r = bufT(ctx, "tab_h1", n, &d1)) || (r = bufT(ctx, "tab_h2", n, &d2)) ||
      (r = ensure_tablog(ctx, &tl)))
    return r;
  CK(cudaMemcpy(d0, h0, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d1, h1, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d2, h2, n * sizeof(double), cudaMemcpyHostToDevice));
  float4* df;
  if ((r = bufT(ctx, "tab_hf", n, &df))) return r;
  const std::vector<float4> hf = pack_voigt_f32(h0, h1, h2, n);
  CK(cudaMemcpy(df, hf.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
  return 0;
}

int atlasgpu_atlas_linop(atlasgpu_ctx* ctx, const int32_t* linedata, int64_t n, int nrhox, int kw,
                         const double* xnfdop, const double* dopple, int nspec, const double* xne,
                         const double* txnxn, const double* hckt, const double* tabcont,
                         const int32_t* iwavetab, int nwave, const double* waveset, int numnu,
                         double* xlines_out, int64_t* lines_used) {
  if (!ctx || n < 0 || (n > 0 && !linedata) || nrhox < 8 || kw < nrhox || kw > kKwMax || nspec < 1 ||
      !xnfdop || !dopple || !xne || !txnxn || !hckt || !tabcont || !iwavetab || nwave < 1 || !waveset ||
      numnu < 2 || !xlines_out)
    return fail(ctx, ATLASGPU_EINVAL, "atlas_linop: bad argument");
  if (ctx->bufs.find("tab_h0") == ctx->bufs.end())
    return fail(ctx, ATLASGPU_ESTATE, "atlas_linop: Voigt tables not set");
  for (int i = 1; i < numnu; ++i)
    if (!(waveset[i] > waveset[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "WAVESET not increasing");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  int32_t *d_ld, *d_iw;
  double *d_xd, *d_dp, *d_xne, *d_tx, *d_hc, *d_tc, *d_ws, *d_xl, *tl;
  AtlasLine* d_lines;
  unsigned long long* d_cnt;
  int r;
  const size_t nd = (size_t)nspec * kw;
  const int64_t nn = std::max<int64_t>(n, 1);
  if ((r = bufT(ctx, "al_ld", (size_t)nn * 4, &d_ld)) || (r = bufT(ctx, "al_iw", nwave + 1, &d_iw)) ||
      (r = bufT(ctx, "al_xd", nd, &d_xd)) || (r = bufT(ctx, "al_dp", nd, &d_dp)) ||
      (r = bufT(ctx, "al_xne", kw, &d_xne)) || (r = bufT(ctx, "al_tx", kw, &d_tx)) ||
      (r = bufT(ctx, "al_hc", kw, &d_hc)) || (r = bufT(ctx, "al_tc", (size_t)(nwave + 1) * kw, &d_tc)) ||
      (r = bufT(ctx, "al_ws", numnu, &d_ws)) || (r = bufT(ctx, "al_xl", (size_t)kw * numnu, &d_xl)) ||
      (r = bufT(ctx, "al_lines", nn, &d_lines)) ||
      (r = bufT(ctx, "al_cnt", 2, &d_cnt)) || (r = ensure_tablog(ctx, &tl)))
    return r;
  if (n > 0) CK(cudaMemcpyAsync(d_ld, linedata, n * 4 * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_iw, iwavetab, (nwave + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xd, xnfdop, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_dp, dopple, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xne, xne, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tx, txnxn, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hc, hckt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tc, tabcont, (size_t)(nwave + 1) * kw * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ws, waveset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(d_xl, 0, (size_t)kw * numnu * sizeof(double), s));
  CK(cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), s));
  if (n > 0) {
    if ((r = atlas_prep_lines(ctx, d_ld, linedata, n, tl, d_ws, waveset, numnu, d_iw, nwave, nspec, d_lines))) return r;
    LinopArgs a{d_lines, n, nrhox, kw, nspec, numnu, d_xd, d_dp, d_xne, d_tx, d_hc, d_tc, d_ws,
                (const double*)ctx->bufs["tab_h0"].first, (const double*)ctx->bufs["tab_h1"].first,
                (const double*)ctx->bufs["tab_h2"].first, (const float4*)ctx->bufs["tab_hf"].first, d_xl, d_cnt,
                d_cnt + 1};
    // exact fixed-point sums (fix_add): per-species CGF maxima, per-depth scales
    unsigned long long *d_fix, *d_cgf;
    double *d_fs, *d_fu;
    if ((r = bufT(ctx, "al_fix", (size_t)kFixWords * kw * numnu, &d_fix)) || (r = bufT(ctx, "al_cgf", nspec, &d_cgf)) ||
        (r = bufT(ctx, "al_fs", kw, &d_fs)) || (r = bufT(ctx, "al_fu", kw, &d_fu)))
      return r;
    CK(cudaMemsetAsync(d_fix, 0, (size_t)kFixWords * kw * numnu * sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(d_cgf, 0, (size_t)nspec * sizeof(unsigned long long), s));
    k_cgf_max<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(d_lines, n, nspec, d_cgf);
    CKL(ctx);
    k_fix_scale<<<1, 128, 0, s>>>(d_xd, nspec, kw, nrhox, (const double*)d_cgf, d_fs, d_fu);
    CKL(ctx);
    a.xfix = d_fix;
    a.fscale = d_fs;
    a.work = work_counters(ctx, 1);
    {
      Timer tm(ctx, "atlas_linop");
      if (ctx->precision == ATLASGPU_PREC_MIXED) k_atlas_linop<true><<<grid_for(ctx, n * 32, 256, 16), 256, 0, s>>>(a);
      else k_atlas_linop<false><<<grid_for(ctx, n * 32, 256, 16), 256, 0, s>>>(a);
      CKL(ctx);
      k_fix_finalize<<<grid_for(ctx, (int64_t)numnu * nrhox, 256, 8), 256, 0, s>>>(d_fix, d_fu, numnu, nrhox, kw,
                                                                                     d_xl);
      CKL(ctx);
    }
    work_collect(ctx, a.work, {"atlas_linop_points"});
  }
  CK(cudaMemcpyAsync(xlines_out, d_xl, (size_t)kw * numnu * sizeof(double), cudaMemcpyDeviceToHost, s));
  unsigned long long cnt[2];
  CK(cudaMemcpyAsync(cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (lines_used) *lines_used = (int64_t)cnt[1];
  return 0;
}

int atlasgpu_atlas_xlinop(atlasgpu_ctx* ctx, const atlasgpu_nlte_line* recs, int64_t n, int nrhox, int kw,
                          const double* xnfdop, const double* dopple, int nspec, const double* xne,
                          const double* txnxn, const double* hckt, const double* tabcont,
                          const int32_t* iwavetab, int nwave, const double* waveset, int numnu,
                          const double* contx, const double* xnfp, const double* rho,
                          const atlasgpu_xlinop_hydrogen* hyd, double* xlines_inout, int64_t* n_other) {
  if (!ctx || n < 0 || (n > 0 && !recs) || nrhox < 8 || kw < nrhox || kw > kKwMax || nspec < 1 || !xnfdop ||
      !dopple || !xne || !txnxn || !hckt || !tabcont || !iwavetab || nwave < 1 || !waveset || numnu < 2 ||
      !contx || !xlines_inout || (!xnfp) != (!rho))
    return fail(ctx, ATLASGPU_EINVAL, "atlas_xlinop: bad argument");
  const bool pops = xnfp != nullptr;
  const bool hlines = hyd != nullptr;
  if (hlines) {
    if (!pops || nspec < 3 || !hyd->t || !hyd->xnf1 || !hyd->xnf2 || !hyd->xnh2)
      return fail(ctx, ATLASGPU_EINVAL, "atlas_xlinop: hydrogen lines need XNFP (species 1-3) and T, XNF, XNH2");
    if (ctx->bufs.find("h_tab") == ctx->bufs.end())
      return fail(ctx, ATLASGPU_ESTATE, "atlas_xlinop: hydrogen tables not set");
  }
  if (ctx->bufs.find("tab_h0") == ctx->bufs.end())
    return fail(ctx, ATLASGPU_ESTATE, "atlas_xlinop: Voigt tables not set");
  for (int i = 1; i < numnu; ++i)
    if (!(waveset[i] > waveset[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "WAVESET not increasing");
  int64_t other = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (i > 0 && recs[i].wlvac < recs[i - 1].wlvac)
      return fail(ctx, ATLASGPU_EINVAL, "atlas_xlinop: records not sorted by wavelength at %lld", (long long)i);
    const int t = recs[i].itype, nc = recs[i].ncon > 10 ? 0 : recs[i].ncon;
    if ((t == 0 || t == 3) && nc > 0 && (recs[i].nelionx < 1 || recs[i].nelionx > 16))
      return fail(ctx, ATLASGPU_EINVAL, "atlas_xlinop: NELIONX %d outside CONTX at record %lld", recs[i].nelionx,
                  (long long)i);
    other += (t == -1 && !hlines) || (!pops && t != 0 && t != 2 && t != 3 && t != -1);
  }
  if (n_other) *n_other = other;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  atlasgpu_nlte_line* d_rec;
  int32_t* d_iw;
  double *d_xd, *d_dp, *d_xne, *d_tx, *d_hc, *d_tc, *d_ws, *d_xl, *d_cx, *d_lc, *d_em;
  AtlasLine* d_lines;
  int r;
  const size_t nd = (size_t)nspec * kw;
  const int64_t nn = std::max<int64_t>(n, 1);
  if ((r = bufT(ctx, "xl_rec", (size_t)nn, &d_rec)) || (r = bufT(ctx, "al_iw", nwave + 1, &d_iw)) ||
      (r = bufT(ctx, "al_xd", nd, &d_xd)) || (r = bufT(ctx, "al_dp", nd, &d_dp)) ||
      (r = bufT(ctx, "al_xne", kw, &d_xne)) || (r = bufT(ctx, "al_tx", kw, &d_tx)) ||
      (r = bufT(ctx, "al_hc", kw, &d_hc)) || (r = bufT(ctx, "al_tc", (size_t)(nwave + 1) * kw, &d_tc)) ||
      (r = bufT(ctx, "al_ws", numnu, &d_ws)) || (r = bufT(ctx, "al_xl", (size_t)kw * numnu, &d_xl)) ||
      (r = bufT(ctx, "xl_lines", (size_t)nn, &d_lines)) || (r = bufT(ctx, "xl_contx", 25 * 16, &d_cx)) ||
      (r = bufT(ctx, "xl_lcontx", (size_t)nn, &d_lc)) || (r = bufT(ctx, "xl_emerge", kw, &d_em)))
    return r;
  // EMERGE(J) = RYDBERG_INF / NMERGE**2, NMERGE = NSTARK = 1600 / XNE(J)**(2/15) (:19964-19977)
  std::vector<double> em(kw, 0.0);
  for (int j = 0; j < nrhox; ++j) {
    const double nmerge = 1600.0 / pow(xne[j], 2.0 / 15.0);
    em[j] = 109737.31568157 / (nmerge * nmerge);
  }
  if (n > 0) CK(cudaMemcpyAsync(d_rec, recs, n * sizeof(atlasgpu_nlte_line), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_iw, iwavetab, (nwave + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xd, xnfdop, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_dp, dopple, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xne, xne, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tx, txnxn, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hc, hckt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tc, tabcont, (size_t)(nwave + 1) * kw * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ws, waveset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xl, xlines_inout, (size_t)kw * numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_cx, contx, 25 * 16 * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_em, em.data(), kw * sizeof(double), cudaMemcpyHostToDevice, s));
  if (n > 0) {
    XlinopPrepArgs pa{d_rec, n, d_ws, numnu, d_iw, nwave, nspec, d_cx, d_lines, d_lc};
    k_xlinop_prep<<<grid_for(ctx, n, 256, 16), 256, 0, s>>>(pa);
    CKL(ctx);
    LinopArgs a{d_lines, n, nrhox, kw, nspec, numnu, d_xd, d_dp, d_xne, d_tx, d_hc, d_tc, d_ws,
                (const double*)ctx->bufs["tab_h0"].first, (const double*)ctx->bufs["tab_h1"].first,
                (const double*)ctx->bufs["tab_h2"].first, (const float4*)ctx->bufs["tab_hf"].first, d_xl, nullptr,
                nullptr, 1, 0, 2000, 0.5642, d_lc, d_em};
    Timer tm(ctx, "atlas_xlinop");
    if (ctx->precision == ATLASGPU_PREC_MIXED) k_atlas_linop<true><<<grid_for(ctx, n * 32, 256, 16), 256, 0, s>>>(a);
    else k_atlas_linop<false><<<grid_for(ctx, n * 32, 256, 16), 256, 0, s>>>(a);
    CKL(ctx);
    if (pops) {
      double *d_xp, *d_rho;
      if ((r = bufT(ctx, "xl_xnfp", nd, &d_xp)) || (r = bufT(ctx, "xl_rho", kw, &d_rho))) return r;
      CK(cudaMemcpyAsync(d_xp, xnfp, nd * sizeof(double), cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(d_rho, rho, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
      XShoreArgs xa{d_rec, d_lines, n, nrhox, kw, nspec, numnu, d_ws, d_tc, d_xp, d_rho, d_hc, d_em, d_xl};
      k_xlinop_shore<<<grid_for(ctx, n * nrhox * 32, 256, 16), 256, 0, s>>>(xa);
      CKL(ctx);
      if (hlines) {
        double* d_hv;
        if ((r = bufT(ctx, "xl_hv", 4 * (size_t)kw, &d_hv))) return r;
        const double* hv[4] = {hyd->t, hyd->xnf1, hyd->xnf2, hyd->xnh2};
        for (int q = 0; q < 4; ++q)
          CK(cudaMemcpyAsync(d_hv + (size_t)q * kw, hv[q], nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
        XHydArgs ha{d_rec, d_lines, n, nrhox, kw, numnu, (const atlasgpu_hydrogen_tables*)ctx->bufs["h_tab"].first,
                    d_ws, d_tc, d_xd, d_dp, d_xp, d_xne, d_hc, d_em, d_hv, d_hv + kw, d_hv + 2 * kw, d_hv + 3 * kw,
                    d_cx, d_xl};
        k_xlinop_hydrogen<<<grid_for(ctx, n * nrhox * 32, 256, 16), 256, 0, s>>>(ha);
        CKL(ctx);
      }
    }
  }
  CK(cudaMemcpyAsync(xlines_inout, d_xl, (size_t)kw * numnu * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int atlasgpu_atlas_set_hydrogen_tables(atlasgpu_ctx* ctx, const atlasgpu_hydrogen_tables* tables) {
  if (!ctx || !tables) return fail(ctx, ATLASGPU_EINVAL, "set_hydrogen_tables: null argument");
  for (int n = 0; n < 4; ++n)
    if (tables->lnghal[n] < 1 || tables->lnghal[n] > 14 || tables->istal[n] < 1 ||
        tables->istal[n] + tables->lnghal[n] - 1 > 34 || tables->lncomp[n] < 1 || tables->lncomp[n] > 5)
      return fail(ctx, ATLASGPU_EINVAL, "set_hydrogen_tables: fine-structure index out of range");
  cudaSetDevice(ctx->device);
  atlasgpu_hydrogen_tables* d;
  int r;
  if ((r = bufT(ctx, "h_tab", 1, &d))) return r;
  CK(cudaMemcpyAsync(d, tables, sizeof *tables, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int atlasgpu_atlas_rt_pass(atlasgpu_ctx* ctx, int numnu, const double* waveset, const double* rcoset,
                           const double* acont, const double* sigmac, const double* scont, int kw,
                           const double* xlines, int nrhox, const double* rhox, const double* t,
                           const double* hkt, double teff, atlasgpu_accum* out, double* hsurf_out) {
  if (!ctx || !ctx->ops_set) return fail(ctx, ATLASGPU_ESTATE, "atlas_rt_pass: operators not set");
  if (numnu < 1 || !waveset || !rcoset || !acont || !sigmac || kw < nrhox || kw > kKwMax || nrhox < 4 ||
      !xlines || !rhox || !t || !hkt || !out)
    return fail(ctx, ATLASGPU_EINVAL, "atlas_rt_pass: bad argument");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t nt = (size_t)numnu * kw;
  double *d_ws, *d_rc, *d_ac, *d_sg, *d_sc = nullptr, *d_xl0, *d_rx, *d_t, *d_hk, *d_hs, *d_sum;
  int r;
  if ((r = bufT(ctx, "rt_ws", numnu, &d_ws)) || (r = bufT(ctx, "rt_rc", numnu, &d_rc)) ||
      (r = bufT(ctx, "rt_ac", nt, &d_ac)) || (r = bufT(ctx, "rt_sg", nt, &d_sg)) ||
      (r = bufT(ctx, "rt_xl0", nt, &d_xl0)) ||
      (r = bufT(ctx, "rt_rx", kw, &d_rx)) || (r = bufT(ctx, "rt_t", kw, &d_t)) || (r = bufT(ctx, "rt_hk", kw, &d_hk)) ||
      (r = bufT(ctx, "rt_hs", numnu, &d_hs)) || (r = bufT(ctx, "rt_sum", kAcc * kw + 1, &d_sum)))
    return r;
  if (scont && (r = bufT(ctx, "rt_sc", nt, &d_sc))) return r;
  CK(cudaMemcpyAsync(d_ws, waveset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_rc, rcoset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ac, acont, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_sg, sigmac, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  if (scont) CK(cudaMemcpyAsync(d_sc, scont, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xl0, xlines, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_rx, rhox, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_t, t, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hk, hkt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  RtArgs a{ctx->ops, numnu, nrhox, kw, d_ws, d_rc, d_ac, d_sg, d_sc, d_xl0, d_rx, d_t, d_hk, teff,
           1, 1, kw, nullptr, d_hs, nullptr};
  if ((r = rt_launch(ctx, a, d_sum, nullptr))) return r;
  std::vector<double> hsum(kAcc * kw + 1);
  CK(cudaMemcpyAsync(hsum.data(), d_sum, hsum.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (hsurf_out) CK(cudaMemcpyAsync(hsurf_out, d_hs, numnu * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double* dst[kAcc] = {out->rjmins, out->rdabh, out->rdiagj, out->flxrad, out->raden, out->h_total, out->accrad, out->abross};
  for (int q = 0; q < kAcc; ++q)
    if (dst[q]) memcpy(dst[q], hsum.data() + q * kw, nrhox * sizeof(double));
  out->pradk0 = hsum[kAcc * kw];
  return 0;
}

int atlasgpu_atlas_finish(atlasgpu_ctx* ctx, atlasgpu_finish_state* st, const atlasgpu_accum* acc,
                          double* max_flxerr) {
  if (!ctx || !st || !acc || st->nrhox < 8 || st->nrhox > kKwMax || !st->ross_t || !st->ross_p || !st->ross_k ||
      st->ross_max < 1 || st->ross_n < 0 || st->ross_n > st->ross_max)
    return fail(ctx, ATLASGPU_EINVAL, "atlas_finish: bad argument");
  const int n = st->nrhox, kw = n;
  const size_t fsm = fin_smem_bytes(kw, st->ross_max);
  if (fsm > (size_t)ctx->smem_optin)
    return fail(ctx, ATLASGPU_EINVAL, "atlas_finish: ross_max %d exceeds the on-chip ROSSTAB capacity",
                st->ross_max);
  double* hv[17] = {st->t, st->rhox, st->p, st->xne, st->abross, st->prad, st->vturb, st->pturb,
                    st->tauros, st->accrad, st->raden, st->oldt1, st->flxerr, st->dtflux, st->dtlamb,
                    st->dtsurf, st->t1};
  for (int q = 0; q < 17; ++q)
    if (!hv[q]) return fail(ctx, ATLASGPU_EINVAL, "atlas_finish: null array %d", q);
  const double* ha[kAcc] = {acc->rjmins, acc->rdabh, acc->rdiagj, acc->flxrad, acc->raden, acc->h_total, acc->accrad, acc->abross};
  for (int q = 0; q < kAcc; ++q)
    if (!ha[q]) return fail(ctx, ATLASGPU_EINVAL, "atlas_finish: null accumulator %d", q);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  double *d_arr, *d_acc, *d_ross;
  ModelState* d_ms;
  RossStore* d_rs;
  int r;
  const size_t nr = (size_t)st->ross_max;
  if ((r = bufT(ctx, "fin_arr", 17 * kw, &d_arr)) || (r = bufT(ctx, "fin_acc", kAcc * kw + 1, &d_acc)) ||
      (r = bufT(ctx, "fin_ross", 3 * nr, &d_ross)) ||
      (r = bufT(ctx, "fin_ms", 1, &d_ms)) || (r = bufT(ctx, "fin_rs", 1, &d_rs)))
    return r;
  std::vector<double> h(17 * kw), ha2(kAcc * kw + 1);
  for (int q = 0; q < 17; ++q) memcpy(h.data() + q * kw, hv[q], n * sizeof(double));
  for (int q = 0; q < kAcc; ++q) memcpy(ha2.data() + q * kw, ha[q], n * sizeof(double));
  ha2[kAcc * kw] = acc->pradk0;
  ModelState ms;
  double** f[17] = {&ms.t, &ms.rhox, &ms.p, &ms.xne, &ms.abross, &ms.prad, &ms.vturb, &ms.pturb, &ms.tauros,
                    &ms.accrad, &ms.raden, &ms.oldt1, &ms.flxerr, &ms.dtflux, &ms.dtlamb, &ms.dtsurf, &ms.t1};
  for (int q = 0; q < 17; ++q) *f[q] = d_arr + q * kw;
  ms.pradk0 = st->pradk0;
  ms.maxerr = 0;
  CK(cudaMemcpyAsync(d_arr, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_acc, ha2.data(), ha2.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ross, st->ross_t, nr * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ross + nr, st->ross_p, nr * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ross + 2 * nr, st->ross_k, nr * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ms, &ms, sizeof ms, cudaMemcpyHostToDevice, s));
  RossStore R{st->ross_n, st->ross_max, st->ross_zerot, st->ross_slopet, st->ross_zerop, st->ross_slopep,
              d_ross, d_ross + nr, d_ross + 2 * nr};
  CK(cudaMemcpyAsync(d_rs, &R, sizeof R, cudaMemcpyHostToDevice, s));
  {
    Timer tm(ctx, "atlas_finish");
    CK(cudaFuncSetAttribute(k_finish_one, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
    k_finish_one<<<1, kFinThreads, fsm, s>>>(d_ms, d_acc, kw, n, st->iter, st->teff, st->grav, d_rs);
    CKL(ctx);
  }
  CK(cudaMemcpyAsync(h.data(), d_arr, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&ms, d_ms, sizeof ms, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&R, d_rs, sizeof R, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(st->ross_t, d_ross, nr * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(st->ross_p, d_ross + nr, nr * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(st->ross_k, d_ross + 2 * nr, nr * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  st->ross_n = R.n;
  st->ross_zerot = R.zerot;
  st->ross_slopet = R.slopet;
  st->ross_zerop = R.zerop;
  st->ross_slopep = R.slopep;
  for (int q = 0; q < 17; ++q) memcpy(hv[q], h.data() + q * kw, n * sizeof(double));
  st->pradk0 = ms.pradk0;
  if (max_flxerr) *max_flxerr = ms.maxerr;
  return 0;
}

}  // extern "C"
